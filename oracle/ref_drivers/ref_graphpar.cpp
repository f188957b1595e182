// ORACLE — test infrastructure only.  Runs the reference's offline single-process edge
// partitioner (Graph/GraphIngress.hpp EdgePartition::divideEdges = loadMetaFromFile +
// redistributeEdgeFiles), as usr/debug/test_graphPar.cpp does: it reads <prefix>.meta and
// <prefix>.edges.<i> and writes <prefix>.part.<n>.<r>, <prefix>.outdegree.<n>.<p> and
// <prefix>.scatterMap.<n>.<p>.
//
// The partitioner's per-vertex part sets (FixedBitmap, Util/Bitmap.hpp:137-140) are never
// cleared: std::vector::resize copies one default-constructed temporary, whose bits are whatever
// the stack held, into every vertex.  The partitioner means them to start empty (the
// constructor's comment asks callers to clear them).  So that the harness runs that intended
// form, the stack region the partitioner's frame will use is zeroed just before the call; the
// two steps of divideEdges are called one after the other for that.
//
//   ref_graphpar <prefix> <nparts>
#include "ref_harness.hpp"

static void __attribute__((noinline)) zero_stack() {
  volatile char buf[1 << 20];
  for (size_t i = 0; i < sizeof buf; ++i) buf[i] = 0;
}

#define private public
#include "Graph/GraphIngress.hpp"
#undef private

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s prefix nparts\n", argv[0]);
    return 2;
  }
  GRE::Graph::EdgePartition par;
  const std::string prefix(argv[1]);
  par.loadMetaFromFile(prefix);
  zero_stack();
  par.redistributeEdgeFiles(prefix, atoi(argv[2]));
  return 0;
}

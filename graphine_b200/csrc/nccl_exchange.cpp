// The library's own exchange for the partitioned paths (gre_part_*): NCCL collectives enqueued on
// the part's CUDA stream, so a superstep's exchange costs no host round trip.  This takes the
// role of the reference's buffered MPI scatter/combiner syncs (Engine.hpp:273-315, 333-374).
//
// NCCL is loaded when the first communicator is made (dlopen of libnccl.so.2: the copy the
// process already holds, e.g. PyTorch's, else the system's), so loading libgre_gpu.so does not
// need NCCL.  Only the core API is used: unique id, init by rank, all-gather, grouped
// send/receive (the all-to-all), destroy.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>
#include <string.h>

#include <mutex>

#include "gre_internal.cuh"

struct gre_nccl_s {
  ncclComm_t comm = nullptr;
  int nranks = 1, rank = 0, device = 0;
};

namespace gre {
namespace {

struct NcclApi {
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  ncclResult_t (*all_gather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*group_start)() = nullptr;
  ncclResult_t (*group_end)() = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
  bool ok = false;
  std::string why;
};

const NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      const char* e = dlerror();
      api.why = e ? e : "dlopen(libnccl.so.2) failed";
      return;
    }
    auto sym = [&](const char* name, auto** fn) {
      *fn = reinterpret_cast<std::remove_pointer_t<decltype(fn)>>(dlsym(h, name));
      if (!*fn && api.why.empty()) api.why = std::string("missing NCCL symbol ") + name;
    };
    sym("ncclGetUniqueId", &api.get_unique_id);
    sym("ncclCommInitRank", &api.comm_init_rank);
    sym("ncclCommDestroy", &api.comm_destroy);
    sym("ncclAllGather", &api.all_gather);
    sym("ncclSend", &api.send);
    sym("ncclRecv", &api.recv);
    sym("ncclGroupStart", &api.group_start);
    sym("ncclGroupEnd", &api.group_end);
    sym("ncclGetErrorString", &api.error_string);
    api.ok = api.why.empty();
  });
  return api;
}

int nccl_status(ncclResult_t r, const char* what) {
  if (r == ncclSuccess) return GRE_SUCCESS;
  set_error("%s: %s", what, nccl().error_string ? nccl().error_string(r) : "NCCL error");
  return GRE_FAILURE;
}

int need_nccl() {
  if (nccl().ok) return GRE_SUCCESS;
  set_error("NCCL unavailable: %s", nccl().why.c_str());
  return GRE_NOT_IMPLEMENTED;
}

}  // namespace
}  // namespace gre

using namespace gre;

extern "C" {

int gre_nccl_unique_id(uint8_t* id) {
  if (!id) return GRE_NULL;
  GRE_CHECK(need_nccl());
  ncclUniqueId u;
  GRE_CHECK(nccl_status(nccl().get_unique_id(&u), "ncclGetUniqueId"));
  memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
  return GRE_SUCCESS;
}

int gre_nccl_create(const uint8_t* id, uint32_t nranks, uint32_t rank, int device, gre_nccl* out) {
  if (!id || !out) return GRE_NULL;
  *out = nullptr;
  if (nranks == 0 || rank >= nranks) {
    set_error("gre_nccl_create: rank %u of %u", rank, nranks);
    return GRE_INVALID_ARG;
  }
  GRE_CHECK(need_nccl());
  GRE_CUDA(cudaSetDevice(device));
  ncclUniqueId u;
  memcpy(u.internal, id, NCCL_UNIQUE_ID_BYTES);
  gre_nccl c = new gre_nccl_s;
  c->nranks = (int)nranks;
  c->rank = (int)rank;
  c->device = device;
  const int st = nccl_status(nccl().comm_init_rank(&c->comm, (int)nranks, u, (int)rank), "ncclCommInitRank");
  if (st) {
    delete c;
    return st;
  }
  *out = c;
  return GRE_SUCCESS;
}

int gre_nccl_free(gre_nccl c) {
  if (!c) return GRE_SUCCESS;
  int st = GRE_SUCCESS;
  if (c->comm) {
    cudaSetDevice(c->device);
    st = nccl_status(nccl().comm_destroy(c->comm), "ncclCommDestroy");
  }
  delete c;
  return st;
}

int gre_nccl_exchange(void* ctx, int kind, const void* send, void* recv, uint64_t bytes, void* stream) {
  gre_nccl c = (gre_nccl)ctx;
  if (!c || !c->comm || (bytes && (!send || !recv))) return 1;
  const cudaStream_t s = (cudaStream_t)stream;
  if (kind == GRE_XCHG_ALLGATHER)
    return nccl_status(nccl().all_gather(send, recv, bytes, ncclUint8, c->comm, s), "ncclAllGather") ? 1 : 0;
  if (kind != GRE_XCHG_ALLTOALL) {
    set_error("gre_nccl_exchange: unknown kind %d", kind);
    return 1;
  }
  // all-to-all as grouped point-to-point: block q of `send` to rank q, block q of `recv` from it
  const uint8_t* sb = (const uint8_t*)send;
  uint8_t* rb = (uint8_t*)recv;
  if (nccl_status(nccl().group_start(), "ncclGroupStart")) return 1;
  int st = GRE_SUCCESS;
  for (int q = 0; q < c->nranks && !st; ++q) {
    st = nccl_status(nccl().send(sb + (uint64_t)q * bytes, bytes, ncclUint8, q, c->comm, s), "ncclSend");
    if (!st) st = nccl_status(nccl().recv(rb + (uint64_t)q * bytes, bytes, ncclUint8, q, c->comm, s), "ncclRecv");
  }
  const int end = nccl_status(nccl().group_end(), "ncclGroupEnd");
  return (st || end) ? 1 : 0;
}

}  // extern "C"

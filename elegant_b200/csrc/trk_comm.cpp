/*
 * trk_comm.cpp -- NCCL communicator for sharded tracking (see trk_comm.h).
 * The NCCL entry points are resolved with dlopen/dlsym from libnccl.so.2 (the
 * copy PyTorch loaded, if any, is the one found) when a communicator is first
 * requested.
 */
#include "trk_comm.h"

#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <nccl.h>
#include <vector>

#include "trk_lattice.h"

namespace {

struct NcclApi {
  void *lib = nullptr;
  ncclResult_t (*getUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*commInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*allReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*allGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  const char *(*errorString)(ncclResult_t) = nullptr;
};

NcclApi g_nccl;
std::mutex g_nccl_mu;

int load_nccl() {
  std::lock_guard<std::mutex> lk(g_nccl_mu);
  if (g_nccl.lib)
    return TRK_OK;
  void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h)
    h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h)
    return trk_set_error(TRK_ERR_NCCL, "cannot load libnccl.so.2: %s", dlerror());
  NcclApi a;
  a.lib = h;
  a.getUniqueId = (decltype(a.getUniqueId))dlsym(h, "ncclGetUniqueId");
  a.commInitRank = (decltype(a.commInitRank))dlsym(h, "ncclCommInitRank");
  a.commDestroy = (decltype(a.commDestroy))dlsym(h, "ncclCommDestroy");
  a.allReduce = (decltype(a.allReduce))dlsym(h, "ncclAllReduce");
  a.allGather = (decltype(a.allGather))dlsym(h, "ncclAllGather");
  a.errorString = (decltype(a.errorString))dlsym(h, "ncclGetErrorString");
  if (!a.getUniqueId || !a.commInitRank || !a.commDestroy || !a.allReduce || !a.allGather || !a.errorString)
    return trk_set_error(TRK_ERR_NCCL, "libnccl.so.2 lacks an expected entry point");
  g_nccl = a;
  return TRK_OK;
}

int nccl_err(ncclResult_t r, const char *what) {
  if (r == ncclSuccess)
    return TRK_OK;
  return trk_set_error(TRK_ERR_NCCL, "%s: %s", what, g_nccl.errorString ? g_nccl.errorString(r) : "NCCL error");
}

} // namespace

struct trk_comm {
  ncclComm_t comm = nullptr;
  int rank = 0, size = 1;
  /* host-exchange communicators: the caller's collectives and a staging
   * buffer (8-byte words) */
  const trk_exchange *ex = nullptr;
  std::vector<unsigned long long> host;
};

namespace {

/* device buffer -> host, the caller's collective, host -> device */
int stage_out(trk_comm *c, const void *dev, size_t bytes, size_t words, cudaStream_t st) {
  if (c->host.size() < words)
    c->host.resize(words);
  if (cudaMemcpyAsync(c->host.data(), dev, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "host exchange: device-to-host copy failed");
  return TRK_OK;
}

int stage_in(trk_comm *c, void *dev, size_t bytes, cudaStream_t st) {
  /* synchronous so the host buffer can be reused by the next exchange */
  if (cudaMemcpyAsync(dev, c->host.data(), bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "host exchange: host-to-device copy failed");
  return TRK_OK;
}

int ex_rc(int r, const char *what) {
  return r == 0 ? TRK_OK : trk_set_error(TRK_ERR_NCCL, "host exchange %s returned %d", what, r);
}

} // namespace

int trk_comm_create_exchange(trk_comm **out, const trk_exchange *ex, int nranks, int rank) {
  if (!out || !ex || !ex->sum_f64 || !ex->sum_u64 || !ex->sum_i64 || !ex->gather_f64 || nranks < 1 || rank < 0 ||
      rank >= nranks)
    return trk_set_error(TRK_ERR_ARG, "bad host-exchange arguments (nranks=%d, rank=%d)", nranks, rank);
  trk_comm *c = new trk_comm();
  c->rank = rank;
  c->size = nranks;
  c->ex = ex;
  *out = c;
  return TRK_OK;
}

int trk_comm_unique_id(void *out128) {
  if (!out128)
    return trk_set_error(TRK_ERR_ARG, "null id buffer");
  int rc = load_nccl();
  if (rc)
    return rc;
  ncclUniqueId id;
  if ((rc = nccl_err(g_nccl.getUniqueId(&id), "ncclGetUniqueId")))
    return rc;
  static_assert(sizeof(id) == NCCL_UNIQUE_ID_BYTES, "NCCL id size");
  memcpy(out128, &id, sizeof(id));
  return TRK_OK;
}

int trk_comm_create(trk_comm **out, const void *unique_id, int nranks, int rank, int device) {
  if (!out || !unique_id || nranks < 1 || rank < 0 || rank >= nranks)
    return trk_set_error(TRK_ERR_ARG, "bad communicator arguments (nranks=%d, rank=%d)", nranks, rank);
  int rc = load_nccl();
  if (rc)
    return rc;
  if (cudaSetDevice(device) != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  trk_comm *c = new trk_comm();
  c->rank = rank;
  c->size = nranks;
  ncclUniqueId id;
  memcpy(&id, unique_id, sizeof(id));
  if ((rc = nccl_err(g_nccl.commInitRank(&c->comm, nranks, id, rank), "ncclCommInitRank"))) {
    delete c;
    return rc;
  }
  *out = c;
  return TRK_OK;
}

void trk_comm_destroy(trk_comm *c) {
  if (!c)
    return;
  if (c->comm && g_nccl.commDestroy)
    g_nccl.commDestroy(c->comm);
  delete c;
}

int trk_comm_rank(const trk_comm *c) { return c ? c->rank : 0; }
int trk_comm_size(const trk_comm *c) { return c ? c->size : 1; }

int trk_comm_sum_f64(trk_comm *c, double *buf, size_t n, cudaStream_t st) {
  if (c->ex) {
    int rc = stage_out(c, buf, sizeof(double) * n, n, st);
    if (rc || (rc = ex_rc(c->ex->sum_f64(c->ex->user, (double *)c->host.data(), n), "sum_f64")))
      return rc;
    return stage_in(c, buf, sizeof(double) * n, st);
  }
  return nccl_err(g_nccl.allReduce(buf, buf, n, ncclFloat64, ncclSum, c->comm, st), "ncclAllReduce(f64)");
}

int trk_comm_sum_u64(trk_comm *c, unsigned long long *buf, size_t n, cudaStream_t st) {
  if (c->ex) {
    int rc = stage_out(c, buf, sizeof(uint64_t) * n, n, st);
    if (rc || (rc = ex_rc(c->ex->sum_u64(c->ex->user, (uint64_t *)c->host.data(), n), "sum_u64")))
      return rc;
    return stage_in(c, buf, sizeof(uint64_t) * n, st);
  }
  return nccl_err(g_nccl.allReduce(buf, buf, n, ncclUint64, ncclSum, c->comm, st), "ncclAllReduce(u64)");
}

int trk_comm_sum_i64(trk_comm *c, long long *buf, size_t n, cudaStream_t st) {
  if (c->ex) {
    int rc = stage_out(c, buf, sizeof(int64_t) * n, n, st);
    if (rc || (rc = ex_rc(c->ex->sum_i64(c->ex->user, (int64_t *)c->host.data(), n), "sum_i64")))
      return rc;
    return stage_in(c, buf, sizeof(int64_t) * n, st);
  }
  return nccl_err(g_nccl.allReduce(buf, buf, n, ncclInt64, ncclSum, c->comm, st), "ncclAllReduce(i64)");
}

int trk_comm_gather_f64(trk_comm *c, const double *send, double *recv, size_t n, cudaStream_t st) {
  if (c->ex) {
    /* host layout: [send (n)] [recv (size * n)] */
    const size_t words = n * (1 + (size_t)c->size);
    int rc = stage_out(c, send, sizeof(double) * n, words, st);
    if (rc)
      return rc;
    double *h = (double *)c->host.data();
    if ((rc = ex_rc(c->ex->gather_f64(c->ex->user, h, h + n, n), "gather_f64")))
      return rc;
    if (cudaMemcpyAsync(recv, h + n, sizeof(double) * n * c->size, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return trk_set_error(TRK_ERR_CUDA, "host exchange: host-to-device copy failed");
    return TRK_OK;
  }
  return nccl_err(g_nccl.allGather(send, recv, n, ncclFloat64, c->comm, st), "ncclAllGather(f64)");
}

/*
 * trk_api.cu -- contexts, device beam, run orchestration and the C ABI of
 * libtrkgpu.so (declared in include/trk.h).
 *
 * A run is scheduled as a list of steps per pass:
 *   SEG(ob, oe)   one launch of the fused tracking kernel over ops [ob, oe)
 *   FID(op)       RFCA "tmean" fiducial before the first pass through op
 *   TAVE(op)      mean arrival time at a LOCK_PHASE / LINEARIZE RFCA, every
 *                 later pass (the first pass takes it from the fiducial's sum)
 *   WAKE(op)      time statistics, binning, convolution and kick of a wake
 * Passes whose step list is one SEG over the whole lattice are merged into a
 * single multi-pass launch, so a lattice without collective elements runs
 * all its passes in one kernel with the coordinates held in registers.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "trk.h"
#include "trk_compile.h"
#include "trk_constants.h"
#include "trk_comm.h"
#include "trk_kernels.h"
#include "trk_lattice.h"

#include <cub/device/device_partition.cuh>
#include <cub/device/device_select.cuh>

#define CUDA_TRY(call)                                                                                       \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess)                                                                                   \
      return trk_set_error(TRK_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                           __LINE__);                                                                        \
  } while (0)

struct WakeBuffers {
  unsigned long long *counts = nullptr;
  double *hist_x = nullptr, *hist_y = nullptr, *V = nullptr, *Vy = nullptr;
  double *W = nullptr, *Wy = nullptr;
  WakeState *state = nullptr;
  long max_bins = 0, points = 0;
  double macro = 0;
  int macro_set = 0;
};

struct trk_context {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> kev; /* start/stop pairs for trk_run.time_kernels */
  long np = 0, cap = 0;
  double *d_cols = nullptr; /* 7 columns x cap */
  int32_t *d_lost_pass = nullptr, *d_lost_elem = nullptr;
  /* compiled lattice */
  CompiledLattice comp;
  const trk_lattice *comp_src = nullptr;
  trk_op *d_ops = nullptr;
  size_t ops_cap = 0;
  trk_aperture *d_aps = nullptr;
  size_t aps_cap = 0;
  double *d_field = nullptr;
  size_t field_cap = 0;
  double *d_rf_phase = nullptr; /* fiducial phase per RF slot, then (at + rf_cap) the pass's mean time */
  double *d_rf_tave = nullptr;
  int rf_cap = 0;
  std::vector<int> rf_fid_done;
  int *d_status = nullptr;
  /* reductions */
  double *d_part = nullptr; /* hi, lo, min, max per block */
  long long *d_part_n = nullptr;
  int part_cap = 0;
  double *d_stats = nullptr; /* 6 doubles: sum, n, min, max, sum_hi, sum_lo */
  trk_comm *comm = nullptr;  /* set for sharded runs (trk_context_set_comm) */
  long long *d_i64 = nullptr; /* one int64 for count exchanges */
  double *d_matrix = nullptr; /* trk_track_matrix: C, R, T (168 doubles) */
  bool element_mode = false;  /* inside trk_track_element: element bodies only, no after-element filters */
  long *d_ens_offsets = nullptr; /* ensemble variant offsets (n_variants + 1) */
  size_t ens_offsets_cap = 0;
  char *d_tune = nullptr;        /* autotuner's scratch copy of the beam */
  size_t tune_cap = 0;
  struct Tuned {
    int nops;
    long np;
    bool lean, fast;
    int variant;
  };
  std::vector<Tuned> ens_tuned;  /* autotuner choices */
  int ens_last_variant = -1;
  /* gradient runs: pass checkpoints, element entry states, adjoints */
  double *d_adj_ck = nullptr, *d_adj_entry = nullptr, *d_adj_lam = nullptr, *d_adj_grad = nullptr;
  double *d_adj_dk = nullptr, *d_adj_mom = nullptr;
  int *d_adj_param = nullptr;
  int *d_adj_dfo = nullptr;        /* per op: offset of a CSBEND's field derivative tables */
  double *d_adj_dfield = nullptr;  /* the tables */
  size_t adj_dfo_cap = 0, adj_dfield_cap = 0;
  size_t adj_ck_cap = 0, adj_entry_cap = 0, adj_lam_cap = 0, adj_grad_cap = 0, adj_dk_cap = 0, adj_mom_cap = 0,
         adj_param_cap = 0;
  size_t matrix_cap = 0;
  double *d_gather = nullptr; /* 6 doubles per rank */
  long long *d_effort = nullptr;
  /* wakes, keyed by op index */
  std::vector<std::pair<int, WakeBuffers>> wake_bufs;
  /* staging */
  double *d_aos = nullptr;
  size_t aos_cap = 0;
  void *d_cub = nullptr;
  size_t cub_cap = 0;
  long *d_perm = nullptr;
  long *d_nsel = nullptr;
  char *d_flags = nullptr;
  long perm_cap = 0;
  /* survivor compaction (trk_run.compact_every): index list, its length,
   * flags and identity indices for the selection, and the selection's
   * scratch */
  long *d_live = nullptr, *d_live_n = nullptr, *d_live_idx = nullptr;
  char *d_live_flags = nullptr;
  long live_cap = 0;
  void *d_live_cub = nullptr;
  size_t live_cub_cap = 0;
  long passes_done = 0; /* passes tracked since the beam was loaded */
  long n_original = 0;  /* particles at the start of the run (do_tracking's nOriginal) */
  long n_global = 0;    /* the same summed over the ranks of a sharded run */
  int tuned_variant = -1; /* tracking-kernel variant used when trk_run.variant < 0 (-1: by lattice class) */
  int last_launches = 0;
  /* device scratch of the beam observers (trk_observe.cu), keyed by call
   * site and slot, grown on demand, freed with the context */
  struct ScratchSlot {
    int site, slot;
    void *p;
    size_t bytes;
  };
  std::vector<ScratchSlot> obs_scratch;
  /* pinned host buffer the observers copy their results into */
  void *h_obs = nullptr;
  size_t h_obs_bytes = 0;
};

/* Passes per launch when compacting: 1, 2, 4, ... up to compact_every,
 * so particles lost in the first turns (most of a dynamic-aperture grid's
 * outer points) free their lanes early, then every compact_every passes. */
static long compact_chunk(long k, long every) { return k >= 30 ? every : std::min<long>(every, 1L << k); }

/* survivor compaction (defined with the ensemble launches) */
extern "C" {
static int prepare_live(trk_context *ctx);
static int compact_live(trk_context *ctx);
}

/* Observer scratch of a context: `bytes` of device memory for (site, slot),
 * reused between calls and grown when a call needs more.  The observers
 * synchronize their stream before returning, so a buffer is idle whenever
 * a new call asks for it. */
int trk_context_scratch(trk_context *ctx, int site, int slot, size_t bytes, void **out) {
  for (trk_context::ScratchSlot &e : ctx->obs_scratch)
    if (e.site == site && e.slot == slot) {
      if (e.bytes < bytes) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(e.p);
        e.p = nullptr;
        e.bytes = 0;
        cudaError_t er = cudaMalloc(&e.p, bytes);
        if (er != cudaSuccess)
          return trk_set_error(TRK_ERR_CUDA, "cudaMalloc: %s", cudaGetErrorString(er));
        e.bytes = bytes;
      }
      *out = e.p;
      return TRK_OK;
    }
  void *q = nullptr;
  cudaError_t er = cudaMalloc(&q, bytes);
  if (er != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "cudaMalloc: %s", cudaGetErrorString(er));
  ctx->obs_scratch.push_back({site, slot, q, bytes});
  *out = q;
  return TRK_OK;
}

/* The observers' pinned host buffer of at least `bytes` (one buffer per
 * context, grown on demand, freed with the context): results copied into
 * pinned memory need no staging copy and no extra synchronization. */
int trk_context_host_scratch(trk_context *ctx, size_t bytes, void **out) {
  if (ctx->h_obs_bytes < bytes) {
    cudaStreamSynchronize(ctx->stream);
    cudaFreeHost(ctx->h_obs);
    ctx->h_obs = nullptr;
    ctx->h_obs_bytes = 0;
    cudaError_t er = cudaHostAlloc(&ctx->h_obs, bytes, cudaHostAllocDefault);
    if (er != cudaSuccess)
      return trk_set_error(TRK_ERR_CUDA, "cudaHostAlloc: %s", cudaGetErrorString(er));
    ctx->h_obs_bytes = bytes;
  }
  *out = ctx->h_obs;
  return TRK_OK;
}

namespace {

int grid_for(const trk_context *ctx, long n, int block) {
  long g = (n + block - 1) / block;
  if (g < 1)
    g = 1;
  long cap = (long)ctx->sm_count * 64;
  return (int)std::min(g, cap);
}

/* Test hook (trk_test_fail_allocation): the number of growing allocations
 * still to succeed before one is refused; negative = never refuse. */
static std::atomic<int> g_fail_alloc_after{-1};

/* true when the hook refuses this allocation (it then disarms itself) */
static bool alloc_refused() {
  int v = g_fail_alloc_after.load();
  while (v >= 0) {
    if (g_fail_alloc_after.compare_exchange_weak(v, v - 1))
      return v == 0;
  }
  return false;
}

template <typename T> int ensure(T **p, size_t &cap, size_t need) {
  if (need <= cap && *p)
    return TRK_OK;
  if (*p)
    cudaFree(*p);
  *p = nullptr;
  size_t n = std::max(need, (size_t)1);
  if (alloc_refused()) {
    cap = 0;
    return trk_set_error(TRK_ERR_NOMEM, "cudaMalloc of %zu bytes refused (test hook)", n * sizeof(T));
  }
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    cap = 0;
    return trk_set_error(TRK_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
  }
  cap = n;
  return TRK_OK;
}

__global__ void aos_to_soa_kernel(const double *aos, long np, long stride, double *cols, long cap,
                                  int32_t *lost_pass, int32_t *lost_elem) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np)
    return;
  for (int c = 0; c < 7; c++)
    cols[c * cap + i] = aos[i * stride + c];
  lost_pass[i] = -1;
  lost_elem[i] = -1;
}

__global__ void soa_copy_kernel(const double *src, long ld, long np, double *cols, long cap, int32_t *lost_pass,
                                int32_t *lost_elem) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np)
    return;
  for (int c = 0; c < 7; c++)
    cols[c * cap + i] = src[c * ld + i];
  lost_pass[i] = -1;
  lost_elem[i] = -1;
}

/* reverse perm[nsel..np) in place (the partition writes rejected items in
 * reverse order); nsel is read on the device */
__global__ void reverse_tail_kernel(long *perm, const long *nsel_p, long np) {
  const long nsel = *nsel_p;
  const long m = np - nsel;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < m / 2; i += (long)gridDim.x * blockDim.x) {
    const long a = nsel + i, b = np - 1 - i;
    const long t = perm[a];
    perm[a] = perm[b];
    perm[b] = t;
  }
}

__global__ void alive_flags_kernel(const int32_t *lost_pass, long np, char *flags, long *idx) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np)
    return;
  flags[i] = lost_pass[i] < 0;
  idx[i] = i;
}

/* survivors' indices for compaction: flags[i] = alive, idx[i] = i */
__global__ void live_flags_kernel(const int32_t *lost_pass, long np, char *flags, long *idx) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (long)gridDim.x * blockDim.x) {
    flags[i] = lost_pass[i] < 0;
    idx[i] = i;
  }
}

__global__ void gather_aos_kernel(const double *cols, long cap, const long *perm, long np, long stride, double *aos,
                                  const int32_t *lost_pass, const int32_t *lost_elem, int32_t *out_pass,
                                  int32_t *out_elem) {
  long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= np)
    return;
  long i = perm[r];
  for (int c = 0; c < 7; c++)
    aos[r * stride + c] = cols[c * cap + i];
  if (out_pass) {
    out_pass[r] = lost_pass[i];
    out_elem[r] = lost_elem[i];
  }
}

/* sum over particles of the passes each one entered alive within
 * [pass_begin, pass_end): elegant's `effort` (src/do_tracking.c:2812-2819) */
__global__ void effort_kernel(const int32_t *lost_pass, long np, long pass_begin, long pass_end,
                              unsigned long long *out) {
  __shared__ unsigned long long sh[256];
  unsigned long long acc = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (long)gridDim.x * blockDim.x) {
    long lp = lost_pass[i];
    long c;
    if (lp < 0)
      c = pass_end - pass_begin;
    else
      c = (lp < pass_end ? lp : pass_end) - pass_begin;
    if (c < 0)
      c = 0;
    acc += (unsigned long long)c;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    atomicAdd(out, sh[0]);
}

/* initial NaN/inf screen of do_tracking (src/do_tracking.c:478-484):
 * limit_amplitudes(DBL_MAX, DBL_MAX) at z = 0 before the first pass */
__global__ void screen_kernel(double *cols, long cap, int32_t *lost_pass, int32_t *lost_elem, long np, long pass,
                              double Po) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np || lost_pass[i] >= 0)
    return;
  double x = cols[i], y = cols[2 * cap + i];
  if (isinf(x) || isinf(y) || isnan(x) || isnan(y)) {
    cols[4 * cap + i] = 0.0;
    cols[5 * cap + i] = Po * (1 + cols[5 * cap + i]);
    lost_pass[i] = (int32_t)pass;
    lost_elem[i] = -1;
  }
}

__global__ void count_alive_kernel(const int32_t *lost_pass, long np, unsigned long long *out) {
  __shared__ unsigned long long sh[256];
  unsigned long long acc = 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (long)gridDim.x * blockDim.x)
    acc += lost_pass[i] < 0;
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    atomicAdd(out, sh[0]);
}

int ensure_beam(trk_context *ctx, long np) {
  if (np <= ctx->cap && ctx->d_cols)
    return TRK_OK;
  cudaFree(ctx->d_cols);
  cudaFree(ctx->d_lost_pass);
  cudaFree(ctx->d_lost_elem);
  ctx->d_cols = nullptr;
  ctx->d_lost_pass = ctx->d_lost_elem = nullptr;
  ctx->cap = 0;
  /* a multiple of 32 entries: every column starts 256-byte aligned and the
   * beam-sum tiles may round their bulk copies up to 16 bytes inside it */
  const long cap = (std::max(np, 1L) + 31) / 32 * 32;
  if (alloc_refused())
    return trk_set_error(TRK_ERR_NOMEM, "device beam allocation for %ld particles refused (test hook)", np);
  if (cudaMalloc(&ctx->d_cols, sizeof(double) * 7 * cap) != cudaSuccess ||
      cudaMalloc(&ctx->d_lost_pass, sizeof(int32_t) * cap) != cudaSuccess ||
      cudaMalloc(&ctx->d_lost_elem, sizeof(int32_t) * cap) != cudaSuccess)
    return trk_set_error(TRK_ERR_NOMEM, "device beam allocation for %ld particles failed", np);
  ctx->cap = cap;
  return TRK_OK;
}

void reset_run_state(trk_context *ctx) {
  ctx->passes_done = 0;
  ctx->rf_fid_done.clear();
  for (auto &wb : ctx->wake_bufs) {
    wb.second.macro_set = 0;
    wb.second.macro = 0;
  }
}

TrackArgs track_args(trk_context *ctx) {
  TrackArgs a;
  std::memset(&a, 0, sizeof(a));
  double *c = ctx->d_cols;
  long cap = ctx->cap;
  a.x = c;
  a.xp = c + cap;
  a.y = c + 2 * cap;
  a.yp = c + 3 * cap;
  a.s = c + 4 * cap;
  a.dp = c + 5 * cap;
  a.lost_pass = ctx->d_lost_pass;
  a.lost_elem = ctx->d_lost_elem;
  a.ops = ctx->d_ops;
  a.aps = ctx->d_aps;
  a.field = ctx->d_field;
  a.rf_phase = ctx->d_rf_phase;
  a.rf_tave = ctx->d_rf_tave;
  a.n = ctx->np;
  a.id = c + 6 * cap;
  a.isr_limit = 3.0; /* srGaussianLimit's default (src/track_data.c:65) */
  return a;
}

int upload_compiled(trk_context *ctx);

int upload_lattice(trk_context *ctx, const trk_lattice *lat, double Po) {
  int rc = trk_compile(lat, Po, ctx->comp);
  if (rc)
    return rc;
  ctx->comp_src = lat;
  return upload_compiled(ctx);
}

/* copy ctx->comp (ops, apertures, field tables) to the device and size the
 * RF and wake buffers it needs */
int upload_compiled(trk_context *ctx) {
  int rc;
  CompiledLattice &c = ctx->comp;
  if ((rc = ensure(&ctx->d_ops, ctx->ops_cap, c.ops.size())))
    return rc;
  if ((rc = ensure(&ctx->d_aps, ctx->aps_cap, std::max<size_t>(c.aps.size(), 1))))
    return rc;
  if ((rc = ensure(&ctx->d_field, ctx->field_cap, std::max<size_t>(c.field.size(), 1))))
    return rc;
  if (!c.ops.empty())
    CUDA_TRY(cudaMemcpyAsync(ctx->d_ops, c.ops.data(), sizeof(trk_op) * c.ops.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
  if (!c.aps.empty())
    CUDA_TRY(cudaMemcpyAsync(ctx->d_aps, c.aps.data(), sizeof(trk_aperture) * c.aps.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
  if (!c.field.empty())
    CUDA_TRY(cudaMemcpyAsync(ctx->d_field, c.field.data(), sizeof(double) * c.field.size(), cudaMemcpyHostToDevice,
                             ctx->stream));
  if (c.n_rf_slots > ctx->rf_cap) {
    cudaFree(ctx->d_rf_phase);
    ctx->d_rf_phase = nullptr;
    ctx->d_rf_tave = nullptr;
    CUDA_TRY(cudaMalloc(&ctx->d_rf_phase, sizeof(double) * 2 * c.n_rf_slots));
    CUDA_TRY(cudaMemsetAsync(ctx->d_rf_phase, 0, sizeof(double) * 2 * c.n_rf_slots, ctx->stream));
    ctx->rf_cap = c.n_rf_slots;
    ctx->d_rf_tave = ctx->d_rf_phase + c.n_rf_slots;
  }
  if ((int)ctx->rf_fid_done.size() < c.n_rf_slots)
    ctx->rf_fid_done.resize(c.n_rf_slots, 0);
  /* wake buffers */
  for (const CompiledWake &w : c.wakes) {
    WakeBuffers *wb = nullptr;
    for (auto &p : ctx->wake_bufs)
      if (p.first == w.op)
        wb = &p.second;
    if (!wb) {
      ctx->wake_bufs.push_back({w.op, WakeBuffers()});
      wb = &ctx->wake_bufs.back().second;
    }
    if (wb->max_bins < w.max_bins || wb->points < w.points) {
      cudaFree(wb->counts);
      cudaFree(wb->hist_x);
      cudaFree(wb->hist_y);
      cudaFree(wb->V);
      cudaFree(wb->Vy);
      cudaFree(wb->W);
      cudaFree(wb->Wy);
      cudaFree(wb->state);
      long nb = w.max_bins + 2;
      CUDA_TRY(cudaMalloc(&wb->counts, sizeof(unsigned long long) * nb));
      CUDA_TRY(cudaMalloc(&wb->hist_x, sizeof(double) * nb));
      CUDA_TRY(cudaMalloc(&wb->hist_y, sizeof(double) * nb));
      CUDA_TRY(cudaMalloc(&wb->V, sizeof(double) * nb));
      CUDA_TRY(cudaMalloc(&wb->Vy, sizeof(double) * nb));
      CUDA_TRY(cudaMalloc(&wb->W, sizeof(double) * w.points));
      CUDA_TRY(cudaMalloc(&wb->Wy, sizeof(double) * w.points));
      CUDA_TRY(cudaMalloc(&wb->state, sizeof(WakeState)));
      CUDA_TRY(cudaMemsetAsync(wb->state, 0, sizeof(WakeState), ctx->stream));
      wb->max_bins = w.max_bins;
      wb->points = w.points;
    }
    CUDA_TRY(cudaMemcpyAsync(wb->W, w.W, sizeof(double) * w.points, cudaMemcpyHostToDevice, ctx->stream));
    if (w.transverse)
      CUDA_TRY(cudaMemcpyAsync(wb->Wy, w.Wy, sizeof(double) * w.points, cudaMemcpyHostToDevice, ctx->stream));
  }
  return TRK_OK;
}

WakeBuffers *wake_buffers(trk_context *ctx, int op) {
  for (auto &p : ctx->wake_bufs)
    if (p.first == op)
      return &p.second;
  return nullptr;
}

int ensure_partials(trk_context *ctx, int blocks) {
  if (blocks <= ctx->part_cap)
    return TRK_OK;
  cudaFree(ctx->d_part);
  cudaFree(ctx->d_part_n);
  CUDA_TRY(cudaMalloc(&ctx->d_part, sizeof(double) * 4 * blocks));
  CUDA_TRY(cudaMalloc(&ctx->d_part_n, sizeof(long long) * blocks));
  ctx->part_cap = blocks;
  return TRK_OK;
}

/* launch per-particle time statistics (mode 0 wake, 1 RF fiducial) */
int time_stats(trk_context *ctx, bool fast, int mode, double sOffset, double Po) {
  const long chunk = 4096;
  int blocks = (int)std::min<long>((ctx->np + chunk - 1) / chunk, (long)ctx->sm_count * 8);
  blocks = std::max(blocks, 1);
  int rc = ensure_partials(ctx, blocks);
  if (rc)
    return rc;
  TimeStatsArgs t;
  std::memset(&t, 0, sizeof(t));
  t.s = ctx->d_cols + 4 * ctx->cap;
  t.dp = ctx->d_cols + 5 * ctx->cap;
  t.lost_pass = ctx->d_lost_pass;
  t.n = ctx->np;
  t.chunk = chunk;
  t.mode = mode;
  t.Po = Po;
  t.sOffset = sOffset;
  t.part_hi = ctx->d_part;
  t.part_lo = ctx->d_part + blocks;
  t.part_min = ctx->d_part + 2 * blocks;
  t.part_max = ctx->d_part + 3 * blocks;
  t.part_n = ctx->d_part_n;
  t.out = ctx->d_stats;
  if (fast)
    trk_fast::launch_time_stats(t, blocks, ctx->stream);
  else
    trk_exact::launch_time_stats(t, blocks, ctx->stream);
  ctx->last_launches += 2;
  if (ctx->comm) {
    /* every rank's {sum, n, min, max}, combined in rank order on each rank */
    const int R = trk_comm_size(ctx->comm);
    if ((rc = trk_comm_gather_f64(ctx->comm, ctx->d_stats, ctx->d_gather, 6, ctx->stream)))
      return rc;
    if (fast)
      trk_fast::launch_stats_combine(ctx->d_gather, R, ctx->d_stats, ctx->stream);
    else
      trk_exact::launch_stats_combine(ctx->d_gather, R, ctx->d_stats, ctx->stream);
    ctx->last_launches++;
  }
  return TRK_OK;
}

int run_wake(trk_context *ctx, bool fast, int opi, long pass, long fresh_pass, double Po) {
  const CompiledLattice &c = ctx->comp;
  const trk_op &op = c.ops[opi];
  const CompiledWake &w = c.wakes[op.i[0]];
  WakeBuffers *wb = wake_buffers(ctx, opi);
  if (!wb)
    return trk_set_error(TRK_ERR_STATE, "wake buffers missing");
  TrackArgs ta = track_args(ctx);
  int grid = grid_for(ctx, ctx->np, TRK_BLOCK);
  if (w.transverse && w.tilt) {
    double ca = std::cos(w.tilt), sa = std::sin(w.tilt);
    if (std::fabs(std::fabs(w.tilt) - TRK_PI) < 1e-12) {
      ca = -1;
      sa = 0;
    }
    if (fast)
      trk_fast::launch_rotate(ta, ca, sa, grid, ctx->stream);
    else
      trk_exact::launch_rotate(ta, ca, sa, grid, ctx->stream);
    ctx->last_launches++;
  }
  int rc = time_stats(ctx, fast, 0, 0.0, Po);
  if (rc)
    return rc;
  WakeArgs a;
  std::memset(&a, 0, sizeof(a));
  a.x = ta.x;
  a.xp = ta.xp;
  a.y = ta.y;
  a.yp = ta.yp;
  a.s = ta.s;
  a.dp = ta.dp;
  a.lost_pass = ta.lost_pass;
  a.lost_elem = ta.lost_elem;
  a.n = ctx->np;
  a.Po = Po;
  a.stats = ctx->d_stats;
  a.state = wb->state;
  a.status = ctx->d_status;
  a.dt = w.dt;
  a.wake_span = w.span;
  a.wake_points = w.points;
  a.i0 = w.i0;
  a.n_bins = w.n_bins;
  a.max_bins = w.max_bins;
  a.smem_bins = 12288;
  a.allow_long_beam = w.allow_long_beam;
  a.pass = pass;
  a.ramp_passes = w.ramp_passes;
  /* macroparticle charge: CHARGE element, else CHARGE/np on pass 0 (src/wake.c:346-372) */
  int charge_elem = -1;
  const trk_lattice *lat = ctx->comp_src;
  for (int i = 0; i < lat->n; i++)
    if (lat->e[i].type == TRK_CHARGE)
      charge_elem = i;
  if (charge_elem >= 0) {
    /* CHARGE element (src/do_tracking.c:797-812) */
    const trk_elem *ce = &lat->e[charge_elem];
    double macro = 0;
    if (ctx->n_global)
      macro = TRK_P(ce, CHARGE_TOTAL) / ctx->n_global;
    if (TRK_P(ce, CHARGE_PER_PARTICLE))
      macro = TRK_P(ce, CHARGE_PER_PARTICLE);
    a.macro_mode = 0;
    a.macro_charge = macro;
  } else if (pass == 0) {
    a.macro_mode = 1;
    a.charge = w.charge;
  } else
    a.macro_mode = 2;
  a.factor = w.factor;
  a.xfactor = w.xfactor;
  a.yfactor = w.yfactor;
  a.interpolate = w.interpolate;
  a.transverse = w.transverse;
  double ramp = (pass >= w.ramp_passes - 1) ? 1.0 : (pass + 1.0) / w.ramp_passes;
  a.active_planes = 0;
  if (w.transverse) {
    /* `if (!factor) continue` per plane (src/trwake.c:192-199); a zero macro
     * charge makes both planes idle */
    double fx = w.factor * w.xfactor * ramp, fy = w.factor * w.yfactor * ramp;
    if (fx)
      a.active_planes |= 1;
    if (fy)
      a.active_planes |= 2;
  }
  a.x_power = w.x_power;
  a.y_power = w.y_power;
  a.x_probe = w.x_probe;
  a.y_probe = w.y_probe;
  a.tdx = w.tdx;
  a.tdy = w.tdy;
  if (w.transverse && w.tilt) {
    a.untilt = 1;
    a.tilt_c = std::cos(-w.tilt);
    a.tilt_s = std::sin(-w.tilt);
    if (std::fabs(std::fabs(w.tilt) - TRK_PI) < 1e-12) {
      a.tilt_c = -1;
      a.tilt_s = 0;
    }
  }
  a.W = wb->W;
  a.W_y = wb->Wy;
  a.counts = wb->counts;
  a.hist_x = wb->hist_x;
  a.hist_y = wb->hist_y;
  a.V = wb->V;
  a.V_y = wb->Vy;
  a.aps = ctx->d_aps;
  int var = (pass == fresh_pass) ? 0 : 1;
  a.ap_post = op.ap_post[var];
  a.z_end = op.z_end;
  a.elem = op.elem;
  a.element_only = ctx->element_mode ? 1 : 0;
  long nb = w.max_bins + 2;
  if (w.transverse) {
    CUDA_TRY(cudaMemsetAsync(wb->hist_x, 0, sizeof(double) * nb, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(wb->hist_y, 0, sizeof(double) * nb, ctx->stream));
  } else
    CUDA_TRY(cudaMemsetAsync(wb->counts, 0, sizeof(unsigned long long) * nb, ctx->stream));
  if (fast)
    trk_fast::launch_wake_bin(a, grid, ctx->stream);
  else
    trk_exact::launch_wake_bin(a, grid, ctx->stream);
  if (ctx->comm) {
    /* histogram sum over ranks (src/wake.c:226-233, src/trwake.c:195-204) */
    if (w.transverse) {
      if ((rc = trk_comm_sum_f64(ctx->comm, wb->hist_x, nb, ctx->stream)) ||
          (rc = trk_comm_sum_f64(ctx->comm, wb->hist_y, nb, ctx->stream)))
        return rc;
    } else if ((rc = trk_comm_sum_u64(ctx->comm, wb->counts, nb, ctx->stream)))
      return rc;
  }
  if (fast)
    trk_fast::launch_wake_apply(a, grid, ctx->stream);
  else
    trk_exact::launch_wake_apply(a, grid, ctx->stream);
  ctx->last_launches += w.transverse ? 5 : 4;
  return TRK_OK;
}

struct Step {
  int kind; /* 0 SEG, 1 FID (and TAVE where the cavity needs it), 2 WAKE, 3 TAVE, 4 MATCH (CHANGE_P0) */
  int ob, oe;
};

bool rf_needs_tave(const trk_op &op) { return op.kind == OPK_RF && (op.i[3] & (RF_LOCK | RF_LINEAR)); }

void pass_steps(const CompiledLattice &c, std::vector<int> &fid_done, std::vector<Step> &steps) {
  steps.clear();
  int seg = 0;
  const int n = (int)c.ops.size();
  for (int k = 0; k < n; k++) {
    const trk_op &op = c.ops[k];
    if (op.kind == OPK_RF && (!fid_done[op.i[1]] || rf_needs_tave(op))) {
      if (k > seg)
        steps.push_back({0, seg, k});
      steps.push_back({fid_done[op.i[1]] ? 3 : 1, k, k + 1});
      fid_done[op.i[1]] = 1;
      seg = k;
    } else if (op.kind == OPK_WAKE || op.kind == OPK_TRWAKE) {
      if (k > seg)
        steps.push_back({0, seg, k});
      steps.push_back({2, k, k + 1});
      seg = k + 1;
      if (c.wakes[op.i[0]].change_p0)
        steps.push_back({4, k, k + 1});
    }
    if (op.kind == OPK_RF && (op.i[3] & RF_CHANGE_P0)) {
      /* the cavity ends its segment; the central momentum follows the beam's */
      steps.push_back({0, seg, k + 1});
      steps.push_back({4, k, k + 1});
      seg = k + 1;
    }
  }
  if (n > seg)
    steps.push_back({0, seg, n});
}

int check_status(trk_context *ctx) {
  int st = 0;
  CUDA_TRY(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (st) {
    CUDA_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    if (st & TRK_STATUS_LONG_BEAM)
      return trk_set_error(TRK_ERR_PHYSICS, "The beam is longer than the longitudinal wake function.");
    if (st & TRK_STATUS_TOO_MANY_BINS)
      return trk_set_error(TRK_ERR_PHYSICS, "autoscaled wake bins exceed the allocated histogram");
    if (st & TRK_STATUS_NO_PARTICLES)
      return trk_set_error(TRK_ERR_PHYSICS, "No available particle for RF cavity fiducialization");
    return trk_set_error(TRK_ERR_DEVICE, "device status 0x%x", st);
  }
  return TRK_OK;
}

} // namespace

/* ======================================================================= C ABI */
extern "C" {

int trk_test_fail_allocation(int after) {
  g_fail_alloc_after.store(after < 0 ? -1 : after);
  return TRK_OK;
}

void trk_run_defaults(trk_run *run) {
  if (!run)
    return;
  std::memset(run, 0, sizeof(*run));
  run->p_central = 1.0;
  run->n_passes = 1;
  run->fast_math = 1;
  run->variant = -1;
  run->compact_every = 64;
}

int trk_context_create(trk_context **out, int device) {
  if (!out)
    return trk_set_error(TRK_ERR_ARG, "null context pointer");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return trk_set_error(TRK_ERR_CUDA, "no CUDA device available");
  if (device < 0)
    CUDA_TRY(cudaGetDevice(&device));
  if (device >= ndev)
    return trk_set_error(TRK_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
  CUDA_TRY(cudaSetDevice(device));
  trk_context *ctx = new trk_context();
  ctx->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess)
    ctx->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
      cudaMalloc(&ctx->d_status, sizeof(int)) != cudaSuccess || cudaMalloc(&ctx->d_stats, 6 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&ctx->d_effort, sizeof(long long)) != cudaSuccess) {
    trk_context_destroy(ctx);
    return trk_set_error(TRK_ERR_CUDA, "context set-up failed");
  }
  cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
  double coef[10];
  trk_expansion_coefficients(coef);
  if (trk_exact::set_coefficients(coef) != cudaSuccess || trk_fast::set_coefficients(coef) != cudaSuccess) {
    trk_context_destroy(ctx);
    return trk_set_error(TRK_ERR_CUDA, "coefficient upload failed");
  }
  *out = ctx;
  return TRK_OK;
}

void trk_context_destroy(trk_context *ctx) {
  if (!ctx)
    return;
  cudaSetDevice(ctx->device);
  if (ctx->stream)
    cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->d_cols);
  cudaFree(ctx->d_lost_pass);
  cudaFree(ctx->d_lost_elem);
  cudaFree(ctx->d_ops);
  cudaFree(ctx->d_aps);
  cudaFree(ctx->d_field);
  cudaFree(ctx->d_rf_phase);
  cudaFree(ctx->d_status);
  cudaFree(ctx->d_part);
  cudaFree(ctx->d_part_n);
  cudaFree(ctx->d_stats);
  cudaFree(ctx->d_gather);
  cudaFree(ctx->d_i64);
  cudaFree(ctx->d_matrix);
  cudaFree(ctx->d_ens_offsets);
  cudaFree(ctx->d_tune);
  cudaFree(ctx->d_adj_ck);
  cudaFree(ctx->d_adj_entry);
  cudaFree(ctx->d_adj_lam);
  cudaFree(ctx->d_adj_grad);
  cudaFree(ctx->d_adj_dk);
  cudaFree(ctx->d_adj_mom);
  cudaFree(ctx->d_adj_param);
  cudaFree(ctx->d_adj_dfo);
  cudaFree(ctx->d_adj_dfield);
  cudaFree(ctx->d_live);
  cudaFree(ctx->d_live_n);
  cudaFree(ctx->d_live_idx);
  cudaFree(ctx->d_live_flags);
  cudaFree(ctx->d_live_cub);
  for (trk_context::ScratchSlot &e : ctx->obs_scratch)
    cudaFree(e.p);
  ctx->obs_scratch.clear();
  cudaFreeHost(ctx->h_obs);
  ctx->h_obs = nullptr;
  ctx->h_obs_bytes = 0;
  trk_comm_destroy(ctx->comm);
  cudaFree(ctx->d_effort);
  cudaFree(ctx->d_aos);
  cudaFree(ctx->d_cub);
  cudaFree(ctx->d_perm);
  cudaFree(ctx->d_nsel);
  cudaFree(ctx->d_flags);
  for (auto &p : ctx->wake_bufs) {
    WakeBuffers &w = p.second;
    cudaFree(w.counts);
    cudaFree(w.hist_x);
    cudaFree(w.hist_y);
    cudaFree(w.V);
    cudaFree(w.Vy);
    cudaFree(w.W);
    cudaFree(w.Wy);
    cudaFree(w.state);
  }
  for (cudaEvent_t e : ctx->kev)
    cudaEventDestroy(e);
  if (ctx->ev0)
    cudaEventDestroy(ctx->ev0);
  if (ctx->ev1)
    cudaEventDestroy(ctx->ev1);
  if (ctx->stream)
    cudaStreamDestroy(ctx->stream);
  delete ctx;
}

void *trk_context_stream(trk_context *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int trk_beam_load(trk_context *ctx, const double *coord, long np, long stride) {
  if (!ctx || (np > 0 && !coord) || np < 0 || stride < 7)
    return trk_set_error(TRK_ERR_ARG, "bad beam (np=%ld, stride=%ld)", np, stride);
  CUDA_TRY(cudaSetDevice(ctx->device));
  /* the previous beam is gone from here on: a failed load leaves no beam */
  ctx->np = ctx->n_original = ctx->n_global = 0;
  int rc = ensure_beam(ctx, np);
  if (rc)
    return rc;
  if ((rc = ensure(&ctx->d_aos, ctx->aos_cap, (size_t)std::max(np, 1L) * stride)))
    return rc;
  ctx->np = np;
  reset_run_state(ctx);
  ctx->n_original = np;
  ctx->n_global = np;
  if (np == 0)
    return TRK_OK;
  CUDA_TRY(cudaMemcpyAsync(ctx->d_aos, coord, sizeof(double) * np * stride, cudaMemcpyHostToDevice, ctx->stream));
  aos_to_soa_kernel<<<(int)((np + 255) / 256), 256, 0, ctx->stream>>>(ctx->d_aos, np, stride, ctx->d_cols, ctx->cap,
                                                                      ctx->d_lost_pass, ctx->d_lost_elem);
  CUDA_TRY(cudaGetLastError());
  return TRK_OK;
}

int trk_beam_load_device(trk_context *ctx, const double *d_soa, long np, long ld) {
  if (!ctx || (np > 0 && !d_soa) || np < 0 || ld < np)
    return trk_set_error(TRK_ERR_ARG, "bad device beam (np=%ld, ld=%ld)", np, ld);
  CUDA_TRY(cudaSetDevice(ctx->device));
  ctx->np = ctx->n_original = ctx->n_global = 0;
  int rc = ensure_beam(ctx, np);
  if (rc)
    return rc;
  ctx->np = np;
  reset_run_state(ctx);
  ctx->n_original = np;
  ctx->n_global = np;
  if (np == 0)
    return TRK_OK;
  soa_copy_kernel<<<(int)((np + 255) / 256), 256, 0, ctx->stream>>>(d_soa, ld, np, ctx->d_cols, ctx->cap,
                                                                    ctx->d_lost_pass, ctx->d_lost_elem);
  CUDA_TRY(cudaGetLastError());
  return TRK_OK;
}

int trk_beam_device_columns(trk_context *ctx, double **columns, long *np, int32_t **loss) {
  if (!ctx)
    return trk_set_error(TRK_ERR_ARG, "null context");
  if (columns)
    for (int c = 0; c < 7; c++)
      columns[c] = ctx->d_cols ? ctx->d_cols + (size_t)c * ctx->cap : nullptr;
  if (np)
    *np = ctx->np;
  if (loss) {
    loss[0] = ctx->d_lost_pass;
    loss[1] = ctx->d_lost_elem;
  }
  return TRK_OK;
}

int trk_beam_count(trk_context *ctx, long *n_left) {
  if (!ctx || !n_left)
    return trk_set_error(TRK_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(ctx->device));
  if (ctx->np == 0) {
    *n_left = 0;
    return TRK_OK;
  }
  CUDA_TRY(cudaMemsetAsync(ctx->d_effort, 0, sizeof(long long), ctx->stream));
  count_alive_kernel<<<std::min(grid_for(ctx, ctx->np, 256), 1024), 256, 0, ctx->stream>>>(
    ctx->d_lost_pass, ctx->np, (unsigned long long *)ctx->d_effort);
  long long v = 0;
  CUDA_TRY(cudaMemcpyAsync(&v, ctx->d_effort, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *n_left = (long)v;
  return TRK_OK;
}

int trk_beam_store(trk_context *ctx, double *coord, long stride, long *n_left, long *lost_pass,
                   int32_t *lost_element) {
  if (!ctx || stride < 7 || (ctx->np > 0 && !coord))
    return trk_set_error(TRK_ERR_ARG, "bad store arguments");
  CUDA_TRY(cudaSetDevice(ctx->device));
  const long np = ctx->np;
  if (np == 0) {
    if (n_left)
      *n_left = 0;
    return TRK_OK;
  }
  int rc;
  if (np > ctx->perm_cap) {
    cudaFree(ctx->d_perm);
    cudaFree(ctx->d_flags);
    cudaFree(ctx->d_nsel);
    CUDA_TRY(cudaMalloc(&ctx->d_perm, sizeof(long) * 2 * np));
    CUDA_TRY(cudaMalloc(&ctx->d_flags, np));
    CUDA_TRY(cudaMalloc(&ctx->d_nsel, sizeof(long)));
    ctx->perm_cap = np;
  }
  long *d_idx = ctx->d_perm + np;
  alive_flags_kernel<<<(int)((np + 255) / 256), 256, 0, ctx->stream>>>(ctx->d_lost_pass, np, ctx->d_flags, d_idx);
  size_t tmp = 0;
  /* stable partition: survivors first in original order, then the lost ones
   * (DevicePartition::Flagged writes the rejected items in reverse order) */
  cub::DevicePartition::Flagged(nullptr, tmp, d_idx, ctx->d_flags, ctx->d_perm, ctx->d_nsel, np, ctx->stream);
  if ((rc = ensure((char **)&ctx->d_cub, ctx->cub_cap, tmp)))
    return rc;
  CUDA_TRY(cub::DevicePartition::Flagged(ctx->d_cub, tmp, d_idx, ctx->d_flags, ctx->d_perm, ctx->d_nsel, np,
                                         ctx->stream));
  /* reverse the rejected tail so lost particles keep their original order */
  reverse_tail_kernel<<<(int)((np / 2 + 255) / 256 + 1), 256, 0, ctx->stream>>>(ctx->d_perm, ctx->d_nsel, np);
  CUDA_TRY(cudaGetLastError());
  if ((rc = ensure(&ctx->d_aos, ctx->aos_cap, (size_t)np * stride)))
    return rc;
  int32_t *d_out = nullptr;
  if (lost_pass || lost_element) {
    CUDA_TRY(cudaMalloc(&d_out, sizeof(int32_t) * 2 * np));
  }
  gather_aos_kernel<<<(int)((np + 255) / 256), 256, 0, ctx->stream>>>(
    ctx->d_cols, ctx->cap, ctx->d_perm, np, stride, ctx->d_aos, ctx->d_lost_pass, ctx->d_lost_elem, d_out,
    d_out ? d_out + np : nullptr);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(coord, ctx->d_aos, sizeof(double) * np * stride, cudaMemcpyDeviceToHost, ctx->stream));
  if (d_out) {
    std::vector<int32_t> h(2 * np);
    CUDA_TRY(cudaMemcpyAsync(h.data(), d_out, sizeof(int32_t) * 2 * np, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (long r = 0; r < np; r++) {
      if (lost_pass)
        lost_pass[r] = h[r];
      if (lost_element)
        lost_element[r] = h[np + r];
    }
    cudaFree(d_out);
  }
  long nsel = 0;
  CUDA_TRY(cudaMemcpyAsync(&nsel, ctx->d_nsel, sizeof(long), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (n_left)
    *n_left = nsel;
  return TRK_OK;
}

static int ensure_i64(trk_context *ctx) {
  if (!ctx->d_i64)
    CUDA_TRY(cudaMalloc(&ctx->d_i64, sizeof(long long)));
  return TRK_OK;
}

int trk_comm_get_unique_id(void *id128) { return trk_comm_unique_id(id128); }

int trk_context_set_exchange(trk_context *ctx, const trk_exchange *ex, int nranks, int rank) {
  if (!ctx)
    return trk_set_error(TRK_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(ctx->device));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  trk_comm_destroy(ctx->comm);
  ctx->comm = nullptr;
  cudaFree(ctx->d_gather);
  ctx->d_gather = nullptr;
  if (nranks <= 0)
    return TRK_OK;
  int rc = trk_comm_create_exchange(&ctx->comm, ex, nranks, rank);
  if (rc)
    return rc;
  CUDA_TRY(cudaMalloc(&ctx->d_gather, sizeof(double) * 6 * nranks));
  return TRK_OK;
}

int trk_context_set_comm(trk_context *ctx, const void *id128, int nranks, int rank) {
  if (!ctx)
    return trk_set_error(TRK_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(ctx->device));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  trk_comm_destroy(ctx->comm);
  ctx->comm = nullptr;
  cudaFree(ctx->d_gather);
  ctx->d_gather = nullptr;
  if (nranks <= 0)
    return TRK_OK;
  int rc = trk_comm_create(&ctx->comm, id128, nranks, rank, ctx->device);
  if (rc)
    return rc;
  CUDA_TRY(cudaMalloc(&ctx->d_gather, sizeof(double) * 6 * nranks));
  return TRK_OK;
}

int trk_context_comm(const trk_context *ctx, int *rank, int *nranks) {
  if (!ctx)
    return trk_set_error(TRK_ERR_ARG, "null context");
  if (rank)
    *rank = trk_comm_rank(ctx->comm);
  if (nranks)
    *nranks = trk_comm_size(ctx->comm);
  return TRK_OK;
}

/* per-launch timing events for trk_run.time_kernels (created on demand,
 * reused across calls) */
#define TRK_MAX_TIMED 4096
static int timing_events(trk_context *ctx, int pairs) {
  while ((int)ctx->kev.size() < 2 * pairs) {
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreate(&e));
    ctx->kev.push_back(e);
  }
  return TRK_OK;
}

int trk_track(trk_context *ctx, const trk_lattice *lattice, const trk_run *run, trk_stats *stats) {
  if (!ctx || !lattice || !run)
    return trk_set_error(TRK_ERR_ARG, "null argument to trk_track");
  if (run->n_passes < 0)
    return trk_set_error(TRK_ERR_ARG, "negative pass count");
  CUDA_TRY(cudaSetDevice(ctx->device));
  double Po = run->p_central; /* follows the beam at CHANGE_P0 elements */
  if (!(Po > 0))
    return trk_set_error(TRK_ERR_ARG, "p_central must be positive");
  int rc = upload_lattice(ctx, lattice, Po);
  if (rc)
    return rc;
  const bool fast = run->fast_math != 0;
  const CompiledLattice &c = ctx->comp;
  ctx->last_launches = 0;
  const long p0 = run->pass_offset;
  const long fresh = ctx->passes_done == 0 ? p0 : -1;
  int variant = run->variant;
  int n_timed = 0;
  if (variant < 0 || variant >= TRK_N_VARIANTS)
    variant = ctx->tuned_variant;
  if (variant < 0)
    variant = trk_default_variant(fast, c);
  CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
  if (ctx->np > 0 && run->n_passes > 0 && fresh >= 0) {
    screen_kernel<<<(int)((ctx->np + 255) / 256), 256, 0, ctx->stream>>>(
      ctx->d_cols, ctx->cap, ctx->d_lost_pass, ctx->d_lost_elem, ctx->np, p0, Po);
    ctx->last_launches++;
  }
  if (ctx->comm && fresh >= 0) {
    /* total_nOriginal of a sharded run (src/do_tracking.c:1378-1381) */
    long long n = ctx->n_original;
    if ((rc = ensure_i64(ctx)))
      return rc;
    CUDA_TRY(cudaMemcpyAsync(ctx->d_i64, &n, sizeof(n), cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = trk_comm_sum_i64(ctx->comm, ctx->d_i64, 1, ctx->stream)))
      return rc;
    CUDA_TRY(cudaMemcpyAsync(&n, ctx->d_i64, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->n_global = (long)n;
  }
  /* every rank of a sharded run takes the same collective steps, so a rank
   * whose shard is empty still runs the schedule (its kernels see n = 0) */
  if ((ctx->np > 0 || ctx->comm) && run->n_passes > 0 && !c.ops.empty()) {
    TrackArgs ta = track_args(ctx);
    ta.fresh_pass = fresh;
    ta.Po = Po;
    ta.isr_seed = run->isr_seed;
    const int max_blocks = ctx->sm_count * 256;
    std::vector<Step> steps;
    long pass = p0;
    const long pend = p0 + run->n_passes;
    long n_compact = 0;
    while (pass < pend) {
      std::vector<int> fid = ctx->rf_fid_done;
      pass_steps(c, fid, steps);
      bool simple = steps.size() == 1 && steps[0].kind == 0;
      long npass = 1;
      bool compact = false;
      if (simple) {
        /* merge passes while the schedule stays one full segment (the
         * first pass's fresh MAXAMP state is selected inside the kernel);
         * with compaction, compact_every passes per launch */
        npass = pend - pass;
        if (run->compact_every > 0 && ctx->np > 0 && !ctx->comm && npass > 1) {
          compact = true;
          npass = std::min<long>(npass, compact_chunk(n_compact++, run->compact_every));
          if ((rc = prepare_live(ctx)) || (rc = compact_live(ctx)))
            return rc;
        }
      }
      ta.live = compact ? ctx->d_live : nullptr;
      ta.live_n = compact ? ctx->d_live_n : nullptr;
      for (const Step &st : steps) {
        if (st.kind == 0) {
          ta.op_begin = st.ob;
          ta.op_end = st.oe;
          ta.pass_begin = pass;
          ta.pass_end = pass + npass;
          const bool timed = run->time_kernels && n_timed < TRK_MAX_TIMED;
          if (timed) {
            if ((rc = timing_events(ctx, n_timed + 1)))
              return rc;
            CUDA_TRY(cudaEventRecord(ctx->kev[2 * n_timed], ctx->stream));
          }
          if (fast)
            trk_fast::launch_track(ta, variant, trk_lean_flavor(c), ctx->np, max_blocks, ctx->stream);
          else
            trk_exact::launch_track(ta, variant, trk_lean_flavor(c), ctx->np, max_blocks, ctx->stream);
          if (timed)
            CUDA_TRY(cudaEventRecord(ctx->kev[2 * n_timed++ + 1], ctx->stream));
          ctx->last_launches++;
        } else if (st.kind == 1) {
          const trk_op &op = c.ops[st.ob];
          int slot = op.i[1];
          if ((rc = time_stats(ctx, fast, 1, op.d[RD_SOFF], Po)))
            return rc;
          if (fast)
            trk_fast::launch_rf_fiducial(ctx->d_stats, op.d[RD_OMEGA], op.d[RD_TREF], ctx->d_rf_phase, slot,
                                         ctx->d_status, ctx->stream);
          else
            trk_exact::launch_rf_fiducial(ctx->d_stats, op.d[RD_OMEGA], op.d[RD_TREF], ctx->d_rf_phase, slot,
                                          ctx->d_status, ctx->stream);
          ctx->last_launches++;
          ctx->rf_fid_done[slot] = 1;
          if (rf_needs_tave(op)) {
            trk_exact::launch_rf_tave(ctx->d_stats, ctx->d_rf_tave, slot, ctx->stream);
            ctx->last_launches++;
          }
        } else if (st.kind == 4) {
          /* do_match_energy(part, np, P_central, 0) (src/simple_rfca.c:977, src/wake.c:289) */
          if (ctx->comm)
            return trk_set_error(TRK_ERR_UNSUPPORTED, "CHANGE_P0 in a sharded run is not on this path");
          double pc = Po;
          if ((rc = trk_match_energy(ctx, &pc, 0)))
            return rc;
          Po = pc;
          ta.Po = Po;
          ctx->last_launches += 3;
        } else if (st.kind == 3) {
          const trk_op &op = c.ops[st.ob];
          if ((rc = time_stats(ctx, fast, 1, op.d[RD_SOFF], Po)))
            return rc;
          trk_exact::launch_rf_tave(ctx->d_stats, ctx->d_rf_tave, op.i[1], ctx->stream);
          ctx->last_launches++;
        } else {
          if ((rc = run_wake(ctx, fast, st.ob, pass, fresh, Po)))
            return rc;
        }
      }
      pass += npass;
    }
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
  if ((rc = check_status(ctx)))
    return rc;
  ctx->passes_done += run->n_passes;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    stats->device_ms = ms;
    stats->n_total = ctx->np;
    stats->kernel_launches = ctx->last_launches;
    stats->p_central = Po;
    for (int k = 0; k < n_timed; k++) {
      float kms = 0;
      CUDA_TRY(cudaEventElapsedTime(&kms, ctx->kev[2 * k], ctx->kev[2 * k + 1]));
      stats->track_ms += kms;
    }
    stats->track_launches = n_timed;
    if (ctx->np > 0) {
      CUDA_TRY(cudaMemsetAsync(ctx->d_effort, 0, sizeof(long long), ctx->stream));
      effort_kernel<<<std::min(grid_for(ctx, ctx->np, 256), 1024), 256, 0, ctx->stream>>>(
        ctx->d_lost_pass, ctx->np, p0, p0 + run->n_passes, (unsigned long long *)ctx->d_effort);
      long long eff = 0;
      CUDA_TRY(cudaMemcpyAsync(&eff, ctx->d_effort, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      stats->particle_passes = eff;
      long nl = 0;
      if ((rc = trk_beam_count(ctx, &nl)))
        return rc;
      stats->n_left = nl;
    }
  }
  return TRK_OK;
}

static void default_elem(trk_elem &t, int type) {
  std::memset(&t, 0, sizeof(t));
  t.type = type;
  for (int i = 0; i < trk_param_count(type); i++)
    t.p[i] = trk_param_default(type, i);
}

int trk_track_element(trk_context *ctx, const trk_lattice *lattice, int element, long pass, int loss_element,
                      double z_start, const trk_maxamp *maxamp, trk_element_state *state, const trk_run *run,
                      long *n_left) {
  if (!ctx || !lattice || !run)
    return trk_set_error(TRK_ERR_ARG, "null argument");
  if (element < 0 || element >= lattice->n)
    return trk_set_error(TRK_ERR_ARG, "element index out of range");
  CUDA_TRY(cudaSetDevice(ctx->device));
  const trk_elem *e = &lattice->e[element];
  const bool wake = e->type == TRK_WAKE || e->type == TRK_TRWAKE;
  const bool rf = e->type == TRK_RFCA;
  if ((wake || rf) && !state)
    return trk_set_error(TRK_ERR_ARG, "RFCA/WAKE/TRWAKE need an element state");
  /* a private lattice: [MAXAMP of the caller's state] [CHARGE with the
   * caller's macroparticle charge] element */
  trk_elem tmp[3];
  int n = 0;
  if (maxamp) {
    default_elem(tmp[n], TRK_MAXAMP);
    TRK_P(&tmp[n], MAXAMP_X_MAX) = maxamp->x_max;
    TRK_P(&tmp[n], MAXAMP_Y_MAX) = maxamp->y_max;
    TRK_P(&tmp[n], MAXAMP_ELLIPTICAL) = maxamp->elliptical;
    TRK_P(&tmp[n], MAXAMP_EXPONENT) = maxamp->exponent;
    TRK_P(&tmp[n], MAXAMP_YEXPONENT) = maxamp->y_exponent;
    n++;
  }
  if (wake) {
    default_elem(tmp[n], TRK_CHARGE);
    TRK_P(&tmp[n], CHARGE_PER_PARTICLE) = state->macro_charge;
    n++;
  }
  tmp[n++] = *e;
  trk_lattice L;
  L.n = L.cap = n;
  L.e = tmp;
  const double Po = run->p_central;
  if (!(Po > 0))
    return trk_set_error(TRK_ERR_ARG, "p_central must be positive");
  int rc = trk_compile(&L, Po, ctx->comp);
  if (rc)
    return rc;
  CompiledLattice &c = ctx->comp;
  int k = -1;
  for (size_t i = 0; i < c.ops.size(); i++) {
    trk_op &op = c.ops[i];
    op.z_start += z_start;
    op.z_end += z_start;
    op.ap_post[0] = op.ap_post[1] = -1;
    if (op.elem == n - 1) {
      k = (int)i;
      op.elem = loss_element;
    }
  }
  ctx->comp_src = &L;
  if ((rc = upload_compiled(ctx))) {
    ctx->comp_src = nullptr;
    return rc;
  }
  const bool fast = run->fast_math != 0;
  int variant = run->variant;
  if (variant < 0 || variant >= TRK_N_VARIANTS)
    variant = trk_default_variant(fast, c);
  ctx->last_launches = 0;
  if (k >= 0 && (ctx->np > 0 || ctx->comm)) {
    const trk_op &op = c.ops[k];
    if (wake) {
      ctx->element_mode = true;
      rc = run_wake(ctx, fast, k, pass, -1, Po);
      ctx->element_mode = false;
      if (rc) {
        ctx->comp_src = nullptr;
        return rc;
      }
    } else {
      if (rf && op.kind == OPK_RF) {
        const int slot = op.i[1];
        if (state->rf_fiducial_seen) {
          CUDA_TRY(cudaMemcpyAsync(ctx->d_rf_phase + slot, &state->rf_phase_fiducial, sizeof(double),
                                   cudaMemcpyHostToDevice, ctx->stream));
        } else {
          /* findFiducialTime on the first call (src/simple_rfca.c:412-445) */
          if ((rc = time_stats(ctx, fast, 1, op.d[RD_SOFF], Po))) {
            ctx->comp_src = nullptr;
            return rc;
          }
          if (fast)
            trk_fast::launch_rf_fiducial(ctx->d_stats, op.d[RD_OMEGA], op.d[RD_TREF], ctx->d_rf_phase, slot,
                                         ctx->d_status, ctx->stream);
          else
            trk_exact::launch_rf_fiducial(ctx->d_stats, op.d[RD_OMEGA], op.d[RD_TREF], ctx->d_rf_phase, slot,
                                          ctx->d_status, ctx->stream);
          CUDA_TRY(cudaMemcpyAsync(&state->rf_phase_fiducial, ctx->d_rf_phase + slot, sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx->stream));
          CUDA_TRY(cudaStreamSynchronize(ctx->stream));
          state->rf_fiducial_seen = 1;
        }
        if (rf_needs_tave(op)) {
          /* the mean arrival time of this call's beam (src/simple_rfca.c:503-556) */
          if ((rc = time_stats(ctx, fast, 1, op.d[RD_SOFF], Po))) {
            ctx->comp_src = nullptr;
            return rc;
          }
          trk_exact::launch_rf_tave(ctx->d_stats, ctx->d_rf_tave, slot, ctx->stream);
        }
      }
      TrackArgs ta = track_args(ctx);
      ta.fresh_pass = pass;
      ta.Po = Po;
      ta.isr_seed = run->isr_seed;
      ta.element_only = 1;
      ta.op_begin = k;
      ta.op_end = k + 1;
      ta.pass_begin = pass;
      ta.pass_end = pass + 1;
      if (fast)
        trk_fast::launch_track(ta, variant, trk_lean_flavor(c), ctx->np, ctx->sm_count * 256, ctx->stream);
      else
        trk_exact::launch_track(ta, variant, trk_lean_flavor(c), ctx->np, ctx->sm_count * 256, ctx->stream);
      ctx->last_launches++;
    }
    CUDA_TRY(cudaGetLastError());
  }
  ctx->comp_src = nullptr;
  if ((rc = check_status(ctx)))
    return rc;
  return n_left ? trk_beam_count(ctx, n_left) : TRK_OK;
}

int trk_limit_amplitudes(trk_context *ctx, double x_max, double y_max, int elliptical, int exponent, int y_exponent,
                         int extrapolate_z, double z, double p_central, long pass, int element, long *n_left) {
  if (!ctx)
    return trk_set_error(TRK_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(ctx->device));
  trk_aperture ap;
  std::memset(&ap, 0, sizeof(ap));
  ap.x_max = x_max;
  ap.y_max = y_max;
  ap.elliptical = elliptical;
  ap.xexp = exponent;
  ap.yexp = y_exponent ? y_exponent : exponent;
  if (elliptical && (x_max || y_max)) {
    /* elimit_amplitudes exits on a bad exponent (src/limit_amplitudes.c:523-538) */
    if (exponent < 2 || exponent % 2 || (y_exponent && (y_exponent < 2 || y_exponent % 2)))
      return trk_set_error(TRK_ERR_PHYSICS, "aperture exponent is not valid: give an even integer >= 2");
  }
  ap.valid = 1;
  ap.a2 = ipow_h(x_max, ap.xexp);
  ap.b2 = ipow_h(y_max, ap.yexp);
  if (ctx->np > 0) {
    TrackArgs ta = track_args(ctx);
    ta.Po = p_central;
    const int grid = grid_for(ctx, ctx->np, TRK_BLOCK);
    /* the reference's arithmetic (no FMA contraction in the extrapolation) */
    trk_exact::launch_limit(ta, ap, 0, extrapolate_z, z, pass, element, grid, ctx->stream);
    CUDA_TRY(cudaGetLastError());
  }
  return n_left ? trk_beam_count(ctx, n_left) : TRK_OK;
}

int trk_remove_invalid(trk_context *ctx, double z, double p_central, long pass, int element, long *n_left) {
  if (!ctx)
    return trk_set_error(TRK_ERR_ARG, "null context");
  CUDA_TRY(cudaSetDevice(ctx->device));
  if (ctx->np > 0) {
    TrackArgs ta = track_args(ctx);
    ta.Po = p_central;
    trk_aperture ap;
    std::memset(&ap, 0, sizeof(ap));
    trk_exact::launch_limit(ta, ap, 1, 0, z, pass, element, grid_for(ctx, ctx->np, TRK_BLOCK), ctx->stream);
    CUDA_TRY(cudaGetLastError());
  }
  return n_left ? trk_beam_count(ctx, n_left) : TRK_OK;
}

int trk_track_matrix(trk_context *ctx, int order, const double *C, const double *R, const double *T, int fast_math,
                     long *n_left) {
  if (!ctx || !C || !R || (order == 2 && !T))
    return trk_set_error(TRK_ERR_ARG, "null argument");
  if (order != 1 && order != 2)
    return trk_set_error(TRK_ERR_UNSUPPORTED, "matrix order %d (1 or 2 supported)", order);
  CUDA_TRY(cudaSetDevice(ctx->device));
  double h[6 + 36 + 126];
  std::memcpy(h, C, sizeof(double) * 6);
  std::memcpy(h + 6, R, sizeof(double) * 36);
  if (order == 2)
    std::memcpy(h + 42, T, sizeof(double) * 126);
  else
    std::memset(h + 42, 0, sizeof(double) * 126);
  int rc;
  if ((rc = ensure(&ctx->d_matrix, ctx->matrix_cap, 168)))
    return rc;
  CUDA_TRY(cudaMemcpyAsync(ctx->d_matrix, h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream));
  if (ctx->np > 0) {
    TrackArgs ta = track_args(ctx);
    const int grid = grid_for(ctx, ctx->np, TRK_BLOCK);
    if (fast_math)
      trk_fast::launch_matrix(ta, ctx->d_matrix, order, grid, ctx->stream);
    else
      trk_exact::launch_matrix(ta, ctx->d_matrix, order, grid, ctx->stream);
    CUDA_TRY(cudaGetLastError());
  }
  return n_left ? trk_beam_count(ctx, n_left) : TRK_OK;
}

/* ------------------------------------------------------------ ensembles */
/* Launch shapes the autotuner tries (block size x resident blocks, see
 * TRK_N_VARIANTS), timed on a scratch copy of the beam. */
/* Survivor compaction: buffers and selection scratch sized for the loaded
 * beam (outside any stream capture), then compact_live() writes the
 * ascending indices of the particles still alive into d_live and their
 * number into *d_live_n, on the stream (capturable: no host sync, fixed
 * sizes).  The tracking kernels then walk d_live instead of the whole beam,
 * so lost particles no longer hold lanes of the warps. */
static int prepare_live(trk_context *ctx) {
  const long np = ctx->np;
  if (np > ctx->live_cap) {
    cudaFree(ctx->d_live);
    cudaFree(ctx->d_live_idx);
    cudaFree(ctx->d_live_flags);
    ctx->d_live = ctx->d_live_idx = nullptr;
    ctx->d_live_flags = nullptr;
    ctx->live_cap = 0;
    CUDA_TRY(cudaMalloc(&ctx->d_live, sizeof(long) * np));
    CUDA_TRY(cudaMalloc(&ctx->d_live_idx, sizeof(long) * np));
    CUDA_TRY(cudaMalloc(&ctx->d_live_flags, np));
    ctx->live_cap = np;
  }
  if (!ctx->d_live_n)
    CUDA_TRY(cudaMalloc(&ctx->d_live_n, sizeof(long)));
  size_t tmp = 0;
  CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, tmp, ctx->d_live_idx, ctx->d_live_flags, ctx->d_live, ctx->d_live_n,
                                      np, ctx->stream));
  if (tmp > ctx->live_cub_cap) {
    cudaFree(ctx->d_live_cub);
    ctx->d_live_cub = nullptr;
    ctx->live_cub_cap = 0;
    CUDA_TRY(cudaMalloc(&ctx->d_live_cub, tmp));
    ctx->live_cub_cap = tmp;
  }
  return TRK_OK;
}

static int compact_live(trk_context *ctx) {
  const long np = ctx->np;
  live_flags_kernel<<<grid_for(ctx, np, 256), 256, 0, ctx->stream>>>(ctx->d_lost_pass, np, ctx->d_live_flags,
                                                                      ctx->d_live_idx);
  size_t tmp = ctx->live_cub_cap;
  CUDA_TRY(cub::DeviceSelect::Flagged(ctx->d_live_cub, tmp, ctx->d_live_idx, ctx->d_live_flags, ctx->d_live,
                                      ctx->d_live_n, np, ctx->stream));
  ctx->last_launches += 2;
  return TRK_OK;
}

static const int k_tune_candidates[] = {1, 4, 7, 8};

static int ensemble_launches(trk_context *ctx, const TrackArgs &base, int nv, int nops, int variant, int lean,
                             bool fast, long p0, long n_passes, long every, bool compact) {
  long k = 0, chunk;
  for (long pass = p0; pass < p0 + n_passes; pass += chunk) {
    chunk = compact ? compact_chunk(k++, every) : every;
    TrackArgs ta = base;
    if (compact) {
      int rc = compact_live(ctx);
      if (rc)
        return rc;
      ta.live = ctx->d_live;
      ta.live_n = ctx->d_live_n;
    }
    ta.op_begin = 0;
    ta.op_end = nops;
    ta.pass_begin = pass;
    ta.pass_end = std::min(pass + chunk, p0 + n_passes);
    if (fast)
      trk_fast::launch_track_ensemble(ta, ctx->d_ens_offsets, nv, nops, variant, lean, ctx->np, ctx->sm_count * 256,
                                      ctx->stream);
    else
      trk_exact::launch_track_ensemble(ta, ctx->d_ens_offsets, nv, nops, variant, lean, ctx->np,
                                       ctx->sm_count * 256, ctx->stream);
    ctx->last_launches++;
  }
  CUDA_TRY(cudaGetLastError());
  return TRK_OK;
}

/* beam columns and loss arrays to / from the tuning scratch copy */
static int beam_snapshot(trk_context *ctx, bool save) {
  const size_t cols = sizeof(double) * 7 * ctx->cap, loss = sizeof(int32_t) * ctx->cap;
  if (save) {
    int rc;
    if ((rc = ensure(&ctx->d_tune, ctx->tune_cap, cols + 2 * loss)))
      return rc;
  }
  char *t = ctx->d_tune;
  if (save) {
    CUDA_TRY(cudaMemcpyAsync(t, ctx->d_cols, cols, cudaMemcpyDeviceToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(t + cols, ctx->d_lost_pass, loss, cudaMemcpyDeviceToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(t + cols + loss, ctx->d_lost_elem, loss, cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    CUDA_TRY(cudaMemcpyAsync(ctx->d_cols, t, cols, cudaMemcpyDeviceToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(ctx->d_lost_pass, t + cols, loss, cudaMemcpyDeviceToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(ctx->d_lost_elem, t + cols + loss, loss, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  return TRK_OK;
}

/* Checks an ensemble (same element types in every variant, no collective
 * elements, offsets from 0 to the loaded particle count), compiles every
 * variant and uploads the concatenated records and the variant offsets.
 * Sets *nops_out to the records per variant and *lean_out. */
static int prepare_ensemble(trk_context *ctx, const trk_lattice *const *lattices, int n_variants, const long *offsets,
                            double Po, int *nops_out, bool *lean_out) {
  if (!ctx || !lattices || !offsets || n_variants < 1)
    return trk_set_error(TRK_ERR_ARG, "bad ensemble arguments");
  if (offsets[0] != 0 || offsets[n_variants] != ctx->np)
    return trk_set_error(TRK_ERR_ARG, "offsets must run from 0 to the loaded particle count (%ld)", ctx->np);
  for (int v = 0; v < n_variants; v++)
    if (!lattices[v] || offsets[v + 1] < offsets[v])
      return trk_set_error(TRK_ERR_ARG, "variant %d: null lattice or decreasing offsets", v);
  const trk_lattice *L0 = lattices[0];
  for (int v = 0; v < n_variants; v++) {
    if (lattices[v]->n != L0->n)
      return trk_set_error(TRK_ERR_ARG, "variant %d has %d elements, variant 0 has %d", v, lattices[v]->n, L0->n);
    for (int i = 0; i < L0->n; i++) {
      const int t = lattices[v]->e[i].type;
      if (t != L0->e[i].type)
        return trk_set_error(TRK_ERR_ARG, "variant %d differs in the type of element %d", v, i);
      if (t == TRK_WAKE || t == TRK_TRWAKE || t == TRK_RFCA)
        return trk_set_error(TRK_ERR_UNSUPPORTED, "collective elements (RFCA, WAKE, TRWAKE) in an ensemble");
    }
  }
  CUDA_TRY(cudaSetDevice(ctx->device));
  if (!(Po > 0))
    return trk_set_error(TRK_ERR_ARG, "p_central must be positive");
  /* one compiled record set per variant, concatenated; aperture and field
   * indices shifted to the concatenated pools */
  CompiledLattice all, c;
  int rc = 0, nops = -1;
  bool lean = true;
  for (int v = 0; v < n_variants; v++) {
    if ((rc = trk_compile(lattices[v], Po, c)))
      return rc;
    if (nops < 0)
      nops = (int)c.ops.size();
    else if ((int)c.ops.size() != nops)
      return trk_set_error(TRK_ERR_ARG, "variant %d compiles to a different element sequence", v);
    lean = lean && c.lean;
    all.has_cfbend = all.has_cfbend || c.has_cfbend;
    const int apo = (int)all.aps.size(), fo = (int)all.field.size();
    for (trk_op op : c.ops) {
      for (int k = 0; k < 2; k++) {
        if (op.ap_post[k] >= 0)
          op.ap_post[k] += apo;
        if (op.ap_in[k] >= 0)
          op.ap_in[k] += apo;
      }
      if (op.kind == OPK_BEND || op.kind == OPK_DIPOLE || op.kind == OPK_CFBEND)
        op.i[4] += fo;
      all.ops.push_back(op);
    }
    all.aps.insert(all.aps.end(), c.aps.begin(), c.aps.end());
    all.field.insert(all.field.end(), c.field.begin(), c.field.end());
  }
  all.lean = lean;
  ctx->comp = all;
  ctx->comp_src = nullptr;
  if ((rc = upload_compiled(ctx)))
    return rc;
  if ((rc = ensure(&ctx->d_ens_offsets, ctx->ens_offsets_cap, (size_t)n_variants + 1)))
    return rc;
  CUDA_TRY(cudaMemcpyAsync(ctx->d_ens_offsets, offsets, sizeof(long) * (n_variants + 1), cudaMemcpyHostToDevice,
                           ctx->stream));
  *nops_out = nops;
  *lean_out = lean;
  return TRK_OK;
}

int trk_track_ensemble(trk_context *ctx, const trk_lattice *const *lattices, int n_variants, const long *offsets,
                       const trk_run *run, trk_stats *stats) {
  if (!run)
    return trk_set_error(TRK_ERR_ARG, "bad ensemble arguments");
  if (run->n_passes < 0)
    return trk_set_error(TRK_ERR_ARG, "negative pass count");
  const double Po = run->p_central;
  int rc = 0, nops = 0;
  bool lean = true;
  if ((rc = prepare_ensemble(ctx, lattices, n_variants, offsets, Po, &nops, &lean)))
    return rc;
  const bool fast = run->fast_math != 0;
  const long p0 = run->pass_offset;
  const long fresh = ctx->passes_done == 0 ? p0 : -1;
  /* passes per launch: compact_every when compacting, else 64 */
  const bool compact = run->compact_every > 0 && ctx->np > 0;
  const long chunk = compact ? run->compact_every : 64;
  if (compact && (rc = prepare_live(ctx)))
    return rc;
  ctx->last_launches = 0;
  TrackArgs base = track_args(ctx);
  base.fresh_pass = fresh;
  base.Po = Po;
  base.isr_seed = run->isr_seed;

  /* launch shape: the caller's, else the autotuner's choice for this
   * (element count, particle count, build) */
  int variant = run->variant;
  if (!trk_fast::ensemble_variant_ok(variant)) {
    variant = -1;
    for (const auto &t : ctx->ens_tuned)
      if (t.nops == nops && t.np == ctx->np && t.lean == lean && t.fast == fast)
        variant = t.variant;
  }
  if (variant < 0 && ctx->np > 0 && nops > 0 && run->n_passes > 0) {
    const long tune_passes = std::min<long>(run->n_passes, 2);
    if ((rc = beam_snapshot(ctx, true)))
      return rc;
    float best = 0;
    for (int cand : k_tune_candidates) {
      if ((rc = beam_snapshot(ctx, false)))
        return rc;
      CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
      if ((rc = ensemble_launches(ctx, base, n_variants, nops, cand, trk_lean_flavor(ctx->comp), fast, p0, tune_passes,
                                  chunk, compact)))
        return rc;
      CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
      CUDA_TRY(cudaEventSynchronize(ctx->ev1));
      float ms = 0;
      CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
      if (variant < 0 || ms < best) {
        best = ms;
        variant = cand;
      }
    }
    if ((rc = beam_snapshot(ctx, false)))
      return rc;
    ctx->ens_tuned.push_back({nops, ctx->np, lean, fast, variant});
    ctx->last_launches = 0;
  }
  if (variant < 0)
    variant = 1;
  ctx->ens_last_variant = variant;

  CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
  if (ctx->np > 0 && run->n_passes > 0 && fresh >= 0) {
    screen_kernel<<<(int)((ctx->np + 255) / 256), 256, 0, ctx->stream>>>(
      ctx->d_cols, ctx->cap, ctx->d_lost_pass, ctx->d_lost_elem, ctx->np, p0, Po);
    ctx->last_launches++;
  }
  if (ctx->np > 0 && run->n_passes > 0 && nops > 0) {
    /* the chunked pass loop is captured once into a CUDA graph and replayed */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    rc = ensemble_launches(ctx, base, n_variants, nops, variant, trk_lean_flavor(ctx->comp), fast, p0, run->n_passes,
                           chunk, compact);
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc)
      return rc;
    if (ce != cudaSuccess)
      return trk_set_error(TRK_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce == cudaSuccess)
      ce = cudaGraphLaunch(exec, ctx->stream);
    if (exec)
      cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess)
      return trk_set_error(TRK_ERR_CUDA, "graph launch: %s", cudaGetErrorString(ce));
  }
  CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
  if ((rc = check_status(ctx)))
    return rc;
  ctx->passes_done += run->n_passes;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    stats->device_ms = ms;
    stats->track_ms = ms;
    stats->track_launches = ctx->last_launches;
    stats->n_total = ctx->np;
    stats->kernel_launches = ctx->last_launches;
    stats->p_central = Po;
    if (ctx->np > 0) {
      CUDA_TRY(cudaMemsetAsync(ctx->d_effort, 0, sizeof(long long), ctx->stream));
      effort_kernel<<<std::min(grid_for(ctx, ctx->np, 256), 1024), 256, 0, ctx->stream>>>(
        ctx->d_lost_pass, ctx->np, p0, p0 + run->n_passes, (unsigned long long *)ctx->d_effort);
      long long eff = 0;
      CUDA_TRY(cudaMemcpyAsync(&eff, ctx->d_effort, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      stats->particle_passes = eff;
      long nl = 0;
      if ((rc = trk_beam_count(ctx, &nl)))
        return rc;
      stats->n_left = nl;
    }
  }
  return TRK_OK;
}

int trk_ensemble_variant(const trk_context *ctx) { return ctx ? ctx->ens_last_variant : -1; }

/* ------------------------------------------------------------- gradients */
/* variant of particle i: offsets[v] <= i < offsets[v+1]; 0 without offsets */
__device__ __forceinline__ int adj_variant(const long *offsets, int nv, long i) {
  if (!offsets)
    return 0;
  int lo = 0, hi = nv;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (offsets[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

/* sums over surviving particles per variant: x^2 + y^2, x, y, count
 * (out[4 v .. 4 v + 3]) */
__global__ void adj_moments_kernel(const double *x, const double *y, const int32_t *lost, long n,
                                   const long *offsets, int nv, double *out) {
  const long stride = (long)gridDim.x * blockDim.x;
  /* every lane runs the same number of rounds so the warp shuffles see all
   * 32 lanes */
  const long rounds = (n + stride - 1) / stride;
  for (long r = 0; r < rounds; r++) {
    const long i = r * stride + (long)blockIdx.x * blockDim.x + threadIdx.x;
    double s2 = 0, sx = 0, sy = 0, c = 0;
    int v = 0;
    if (i < n) {
      v = adj_variant(offsets, nv, i);
      if (lost[i] < 0) {
        s2 = x[i] * x[i] + y[i] * y[i];
        sx = x[i];
        sy = y[i];
        c = 1;
      }
    } else if (n > 0) {
      v = adj_variant(offsets, nv, n - 1);
    }
    const bool uniform = __all_sync(0xffffffffu, v == __shfl_sync(0xffffffffu, v, 0));
    if (uniform) {
      for (int off = 16; off > 0; off >>= 1) {
        s2 += __shfl_xor_sync(0xffffffffu, s2, off);
        sx += __shfl_xor_sync(0xffffffffu, sx, off);
        sy += __shfl_xor_sync(0xffffffffu, sy, off);
        c += __shfl_xor_sync(0xffffffffu, c, off);
      }
    }
    if ((uniform ? (threadIdx.x & 31) == 0 : true) && c != 0) {
      atomicAdd(out + 4 * v, s2);
      atomicAdd(out + 4 * v + 1, sx);
      atomicAdd(out + 4 * v + 2, sy);
      atomicAdd(out + 4 * v + 3, c);
    }
  }
}

/* lambda at the end of the run: dL/dx = (2 x + 2 w mean(x)) / N, same in y,
 * with coef[3 v .. 3 v + 2] = (2 w mean(x) / N, 2 w mean(y) / N, 1 / N) of
 * the particle's variant */
__global__ void adj_seed_kernel(const double *x, const double *y, const int32_t *lost, long n, double *lam,
                                const long *offsets, int nv, const double *coef) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const bool act = lost[i] < 0;
    const double *c = coef + 3 * adj_variant(offsets, nv, i);
    lam[i] = act ? 2 * x[i] * c[2] + c[0] : 0;
    lam[n + i] = 0;
    lam[2 * n + i] = act ? 2 * y[i] * c[2] + c[1] : 0;
    lam[3 * n + i] = 0;
    lam[4 * n + i] = 0;
  }
}

/* L_v = mean(x^2 + y^2) + w (mean(x)^2 + mean(y)^2) over the survivors of
 * each variant (nv = 1 and offsets = null: the whole beam); mom receives
 * (L, mean x, mean y, count) per variant */
static int objective_variants(trk_context *ctx, double w, const long *d_offsets, int nv, std::vector<double> &mom) {
  int rc;
  if ((rc = ensure(&ctx->d_adj_mom, ctx->adj_mom_cap, (size_t)4 * nv)))
    return rc;
  CUDA_TRY(cudaMemsetAsync(ctx->d_adj_mom, 0, 4 * sizeof(double) * nv, ctx->stream));
  if (ctx->np > 0)
    adj_moments_kernel<<<std::min(grid_for(ctx, ctx->np, 256), 1184), 256, 0, ctx->stream>>>(
      ctx->d_cols, ctx->d_cols + 2 * ctx->cap, ctx->d_lost_pass, ctx->np, d_offsets, nv, ctx->d_adj_mom);
  std::vector<double> h(4 * (size_t)nv);
  CUDA_TRY(cudaMemcpyAsync(h.data(), ctx->d_adj_mom, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                           ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  mom.assign(4 * (size_t)nv, 0.0);
  for (int v = 0; v < nv; v++) {
    const double *q = &h[4 * (size_t)v];
    if (q[3] <= 0)
      return nv == 1 ? trk_set_error(TRK_ERR_PHYSICS, "no surviving particles for the loss function")
                     : trk_set_error(TRK_ERR_PHYSICS, "variant %d: no surviving particles for the loss function", v);
    const double mx = q[1] / q[3], my = q[2] / q[3];
    mom[4 * v] = q[0] / q[3] + w * (mx * mx + my * my);
    mom[4 * v + 1] = mx;
    mom[4 * v + 2] = my;
    mom[4 * v + 3] = q[3];
  }
  return TRK_OK;
}

int trk_objective(trk_context *ctx, double centroid_weight, double *loss) {
  if (!ctx || !loss)
    return trk_set_error(TRK_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(ctx->device));
  std::vector<double> mom;
  int rc = objective_variants(ctx, centroid_weight, nullptr, 1, mom);
  if (rc == TRK_OK)
    *loss = mom[0];
  return rc;
}

/* the parameter of an element and the derivative of its per-step kick
 * strengths with respect to it (the element compiled with the parameter
 * set to 1; kick strengths are linear in it) */
static int param_derivative(const trk_elem *e, double Po, double *dk3) {
  trk_elem t = *e;
  const char *name = e->type == TRK_KQUAD ? "K1" : "K2";
  const int pi = trk_param_index(e->type, name);
  if (pi < 0)
    return pi;
  t.p[pi] = 1.0;
  trk_lattice L;
  L.n = L.cap = 1;
  L.e = &t;
  CompiledLattice c;
  int rc = trk_compile(&L, Po, c);
  if (rc)
    return rc;
  if (c.ops.size() != 1 || c.ops[0].kind != OPK_MULT1)
    return trk_set_error(TRK_ERR_UNSUPPORTED, "%s: gradients need a single-order multipole without tilt, "
                         "misalignment or steering", e->name);
  for (int s = 0; s < 3; s++)
    dk3[s] = c.ops[0].d[MD_KQ + s * 3];
  return TRK_OK;
}

/* d(Fx, Fy)/dK1 and d(Fx, Fy)/dK2 of a CSBEND's field expansion, as 4 x 121
 * doubles (Fx, Fy per unit K1, then per unit K2).  The expansion is linear
 * in b[] (trk_csbend_field_table), and b1 = K1 (L/ANGLE) (1+FSE+FSE_Q)/
 * (1+FSE+FSE_D), b2 = K2 (L/ANGLE) (1+FSE)/(1+FSE+FSE_D), odd b's flipped
 * for ANGLE < 0 (compile_bend): the tables are the expansion of those unit
 * b's without the constant dipole and steering terms, to the order the
 * element's own expansion takes. */
static int csbend_field_derivatives(const trk_elem *e, double *out) {
  const double L = TRK_P(e, CSBEND_L), ANGLE = TRK_P(e, CSBEND_ANGLE);
  const double fse = TRK_P(e, CSBEND_FSE), fseD = TRK_P(e, CSBEND_FSE_DIPOLE), fseQ = TRK_P(e, CSBEND_FSE_QUADRUPOLE);
  const double rho = std::fabs(L / ANGLE);
  for (int q = 0; q < 2; q++) {
    double b[9] = {0}, c[9] = {0};
    if (q == 0)
      b[1] = (L / ANGLE) * ((1 + fse + fseQ) / (1 + fse + fseD)) * (ANGLE < 0 ? -1 : 1);
    else
      b[2] = (L / ANGLE) * ((1 + fse) / (1 + fse + fseD));
    long order = (long)TRK_P(e, CSBEND_EXPANSION_ORDER);
    if (order == 0)
      order = 4; /* the automatic order with K1 and/or K2 (i + 2 < 4 for i <= 2) */
    if (order != 4)
      return trk_set_error(TRK_ERR_UNSUPPORTED, "CSBEND gradients need EXPANSION_ORDER 0 or 4");
    int eo1, hn, hs;
    double *Fx = out + 242 * q, *Fy = Fx + 121;
    if (trk_csbend_field_table(b, c, 1 / rho, (int)TRK_P(e, CSBEND_NONLINEAR), order, Fx, Fy, &eo1, &hn, &hs))
      return trk_set_error(TRK_ERR_UNSUPPORTED, "CSBEND expansion order too high");
    Fx[0] = 0;
    Fy[0] = 0;
  }
  return TRK_OK;
}

/* The adjoint run of one lattice (offsets = null: lattices[0]) or of an
 * ensemble of nv lattices over the variant offsets. */
static int adjoint_run(trk_context *ctx, const trk_lattice *const *lattices, int nv, const long *offsets,
                       const trk_run *run, double centroid_weight, double *loss, double *grad, int n_grad) {
  if (!ctx || !lattices || !lattices[0] || !run || nv < 1)
    return trk_set_error(TRK_ERR_ARG, "null argument");
  const trk_lattice *lattice = lattices[0];
  const int n_params = trk_adjoint_param_count(lattice);
  if (grad && n_grad != n_params * nv)
    return trk_set_error(TRK_ERR_ARG, "grad has %d entries, the run has %d parameters", n_grad, n_params * nv);
  if (run->n_passes < 1)
    return trk_set_error(TRK_ERR_ARG, "at least one pass");
  if (ctx->np <= 0)
    return trk_set_error(TRK_ERR_STATE, "no beam loaded");
  CUDA_TRY(cudaSetDevice(ctx->device));
  const double Po = run->p_central;
  const bool ensemble = offsets != nullptr;
  int rc = 0, nops = 0;
  bool lean = true;
  if (ensemble) {
    if ((rc = prepare_ensemble(ctx, lattices, nv, offsets, Po, &nops, &lean)))
      return rc;
  } else {
    if ((rc = upload_lattice(ctx, lattice, Po)))
      return rc;
    nops = (int)ctx->comp.ops.size();
    lean = ctx->comp.lean;
  }
  const CompiledLattice &c = ctx->comp;
  std::vector<int> op_param(std::max(nops, 1), -1);
  std::vector<double> op_dk(3 * (size_t)nv * std::max(nops, 1), 0.0);
  std::vector<int> param_of_elem(lattice->n, -1);
  for (int i = 0, k = 0; i < lattice->n; i++) {
    const int t = lattice->e[i].type;
    if (t == TRK_KQUAD || t == TRK_KSEXT)
      param_of_elem[i] = k++;
    else if (t == TRK_CSBEND) { /* K1 at k, K2 at k + 1 */
      param_of_elem[i] = k;
      k += 2;
    }
  }
  std::vector<int> op_dfield(std::max(nops, 1), -1);
  std::vector<double> dfield;
  for (int k = 0; k < nops; k++) {
    const trk_op &op = c.ops[k];
    switch (op.kind) {
    case OPK_NOP:
    case OPK_DRIFT:
    case OPK_EDRIFT:
    case OPK_RFDRIFT:
      break;
    case OPK_MULT1:
      if (op.i[0] * 3 > 48)
        return trk_set_error(TRK_ERR_UNSUPPORTED, "multipole with more than 16 slices in a gradient run");
      break;
    case OPK_DIPOLE:
    case OPK_CFBEND:
      if (op.i[0] > 32)
        return trk_set_error(TRK_ERR_UNSUPPORTED, "CSBEND with more than 32 slices in a gradient run");
      break;
    default:
      return trk_set_error(TRK_ERR_UNSUPPORTED, "element %d: gradients cover DRIF, EDRIFT, KQUAD/KSEXT/KOCT "
                           "(single order, no tilt or misalignment) and CSBEND (pure dipole or K1/K2 "
                           "expansion, no misalignment or edge kick)", op.elem);
    }
    const int pe = (op.elem >= 0 && op.elem < lattice->n) ? param_of_elem[op.elem] : -1;
    if (pe >= 0 && lattice->e[op.elem].type == TRK_CSBEND) {
      /* K1 and K2 of a bend: the kicks' field derivatives (a zero-angle
       * CSBEND is a drift, and USE_BN ignores K: zero gradient) */
      if (op.kind != OPK_DIPOLE && op.kind != OPK_CFBEND)
        continue;
      const trk_elem *e0 = &lattices[0]->e[op.elem];
      if (TRK_P(e0, CSBEND_USE_BN))
        continue;
      static const int same[] = {P_CSBEND_L, P_CSBEND_ANGLE, P_CSBEND_FSE, P_CSBEND_FSE_DIPOLE,
                                 P_CSBEND_FSE_QUADRUPOLE, P_CSBEND_NONLINEAR, P_CSBEND_EXPANSION_ORDER};
      for (int v = 1; v < nv; v++)
        for (int q : same)
          if (lattices[v]->e[op.elem].p[q] != e0->p[q])
            return trk_set_error(TRK_ERR_UNSUPPORTED, "element %d: CSBEND gradients need the variants to share "
                                 "L, ANGLE, FSE* and the expansion settings", op.elem);
      op_param[k] = pe;
      op_dfield[k] = (int)dfield.size();
      dfield.resize(dfield.size() + 4 * 121);
      if ((rc = csbend_field_derivatives(e0, dfield.data() + op_dfield[k])))
        return rc;
    } else if (pe >= 0) {
      if (op.kind != OPK_MULT1)
        return trk_set_error(TRK_ERR_UNSUPPORTED, "element %d: gradients need a single-order multipole", op.elem);
      op_param[k] = pe;
      for (int v = 0; v < nv; v++)
        if ((rc = param_derivative(&lattices[v]->e[op.elem], Po, &op_dk[3 * ((size_t)v * nops + k)])))
          return rc;
    }
  }
  const long np = ctx->np, T = run->n_passes;
  const size_t n_grad_all = (size_t)n_params * nv;
  if ((rc = ensure(&ctx->d_adj_ck, ctx->adj_ck_cap, (size_t)T * 4 * np)) ||
      (rc = ensure(&ctx->d_adj_entry, ctx->adj_entry_cap, (size_t)std::max(nops, 1) * 4 * np)) ||
      (rc = ensure(&ctx->d_adj_lam, ctx->adj_lam_cap, (size_t)5 * np)) ||
      (rc = ensure(&ctx->d_adj_grad, ctx->adj_grad_cap, std::max<size_t>(n_grad_all, 1))) ||
      (rc = ensure(&ctx->d_adj_param, ctx->adj_param_cap, op_param.size())) ||
      (rc = ensure(&ctx->d_adj_dk, ctx->adj_dk_cap, op_dk.size())) ||
      (rc = ensure(&ctx->d_adj_dfo, ctx->adj_dfo_cap, op_dfield.size())) ||
      (rc = ensure(&ctx->d_adj_dfield, ctx->adj_dfield_cap, std::max<size_t>(dfield.size(), 1))))
    return rc;
  CUDA_TRY(cudaMemcpyAsync(ctx->d_adj_dfo, op_dfield.data(), sizeof(int) * op_dfield.size(), cudaMemcpyHostToDevice,
                           ctx->stream));
  if (!dfield.empty())
    CUDA_TRY(cudaMemcpyAsync(ctx->d_adj_dfield, dfield.data(), sizeof(double) * dfield.size(),
                             cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(ctx->d_adj_param, op_param.data(), sizeof(int) * op_param.size(), cudaMemcpyHostToDevice,
                           ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(ctx->d_adj_dk, op_dk.data(), sizeof(double) * op_dk.size(), cudaMemcpyHostToDevice,
                           ctx->stream));

  /* forward, one pass per launch, the beam at the start of every pass kept */
  const long p0 = run->pass_offset;
  const long fresh = ctx->passes_done == 0 ? p0 : -1;
  if (fresh >= 0)
    screen_kernel<<<(int)((np + 255) / 256), 256, 0, ctx->stream>>>(ctx->d_cols, ctx->cap, ctx->d_lost_pass,
                                                                    ctx->d_lost_elem, np, p0, Po);
  TrackArgs ta = track_args(ctx);
  ta.fresh_pass = fresh;
  ta.Po = Po;
  ta.op_begin = 0;
  ta.op_end = nops;
  const long *d_off = ensemble ? ctx->d_ens_offsets : nullptr;
  const int shape = trk_default_variant(true, c);
  for (long t = 0; t < T; t++) {
    for (int q = 0; q < 4; q++)
      CUDA_TRY(cudaMemcpyAsync(ctx->d_adj_ck + ((size_t)t * 4 + q) * np, ctx->d_cols + (size_t)q * ctx->cap,
                               sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    ta.pass_begin = p0 + t;
    ta.pass_end = p0 + t + 1;
    if (nops > 0) {
      if (ensemble)
        trk_fast::launch_track_ensemble(ta, d_off, nv, nops, shape, trk_lean_flavor(c), np, ctx->sm_count * 256,
                                        ctx->stream);
      else
        trk_fast::launch_track(ta, shape, trk_lean_flavor(c), np, ctx->sm_count * 256, ctx->stream);
    }
  }
  CUDA_TRY(cudaGetLastError());
  ctx->passes_done += T;
  std::vector<double> mom;
  if ((rc = objective_variants(ctx, centroid_weight, d_off, nv, mom)))
    return rc;
  if (loss)
    for (int v = 0; v < nv; v++)
      loss[v] = mom[4 * v];
  if (!grad)
    return TRK_OK;

  /* reverse: seed, then per pass (last first) record the element entry
   * states from the pass checkpoint and sweep the elements backwards */
  std::vector<double> coef(3 * (size_t)nv);
  for (int v = 0; v < nv; v++) {
    const double cnt = mom[4 * v + 3];
    coef[3 * v] = 2 * centroid_weight * mom[4 * v + 1] / cnt;
    coef[3 * v + 1] = 2 * centroid_weight * mom[4 * v + 2] / cnt;
    coef[3 * v + 2] = 1.0 / cnt;
  }
  /* the seed coefficients go to the moments buffer (4 per variant), whose
   * contents are no longer needed */
  CUDA_TRY(cudaMemcpyAsync(ctx->d_adj_mom, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice,
                           ctx->stream));
  adj_seed_kernel<<<std::min(grid_for(ctx, np, 256), 1184), 256, 0, ctx->stream>>>(
    ctx->d_cols, ctx->d_cols + 2 * ctx->cap, ctx->d_lost_pass, np, ctx->d_adj_lam, d_off, nv, ctx->d_adj_mom);
  CUDA_TRY(cudaMemsetAsync(ctx->d_adj_grad, 0, sizeof(double) * std::max<size_t>(n_grad_all, 1), ctx->stream));
  AdjArgs g;
  g.entry = ctx->d_adj_entry;
  g.lam = ctx->d_adj_lam;
  g.grad = ctx->d_adj_grad;
  g.op_param = ctx->d_adj_param;
  g.op_dk = ctx->d_adj_dk;
  g.op_dfield = ctx->d_adj_dfo;
  g.dfield = ctx->d_adj_dfield;
  g.n_ops = nops;
  g.n_params = n_params;
  if (ensemble) {
    ta.ens_offsets = d_off;
    ta.ens_variants = nv;
    ta.ens_ops = nops;
  }
  for (long t = T - 1; t >= 0; t--) {
    g.ck = ctx->d_adj_ck + (size_t)t * 4 * np;
    trk_fast::launch_adjoint_record(ta, g, ctx->stream);
    trk_fast::launch_adjoint_reverse(ta, g, ctx->stream);
  }
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(grad, ctx->d_adj_grad, sizeof(double) * n_grad_all, cudaMemcpyDeviceToHost,
                           ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return check_status(ctx);
}

int trk_adjoint(trk_context *ctx, const trk_lattice *lattice, const trk_run *run, double centroid_weight,
                double *loss, double *grad, int n_grad) {
  const trk_lattice *one[1] = {lattice};
  return adjoint_run(ctx, one, 1, nullptr, run, centroid_weight, loss, grad, n_grad);
}

int trk_adjoint_ensemble(trk_context *ctx, const trk_lattice *const *lattices, int n_variants, const long *offsets,
                         const trk_run *run, double centroid_weight, double *loss, double *grad, int n_grad) {
  if (!offsets)
    return trk_set_error(TRK_ERR_ARG, "null offsets");
  return adjoint_run(ctx, lattices, n_variants, offsets, run, centroid_weight, loss, grad, n_grad);
}

int trk_adjoint_param_count(const trk_lattice *lattice) {
  if (!lattice)
    return trk_set_error(TRK_ERR_ARG, "null lattice");
  int n = 0;
  for (int i = 0; i < lattice->n; i++) {
    if (lattice->e[i].type == TRK_KQUAD || lattice->e[i].type == TRK_KSEXT)
      n++;
    else if (lattice->e[i].type == TRK_CSBEND)
      n += 2;
  }
  return n;
}

} /* extern "C" */

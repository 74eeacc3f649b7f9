/*
 * trk_observe.cu -- beam observers and beam-wide operations on the device
 * beam, for the do_tracking steps between elements that read or rearrange
 * the whole beam:
 *   trk_beam_centroids        compute_centroids (src/compute_centroids.c:53-160)
 *                             and the trajectory centroids (src/do_tracking.c:2585-2610)
 *   trk_accumulate_beam_sums  accumulate_beam_sums (src/compute_centroids.c:286-461)
 *   trk_match_energy          do_match_energy (src/do_tracking.c:3376-3546)
 *   trk_sort_by_id            the particle-ID sort (src/do_tracking.c:935-950)
 * Sums the reference forms with Kahan's compensated summation are formed in
 * double-double and rounded once, as the library's other beam statistics;
 * every other operation rounds as the reference's does.  This file is built
 * without FMA contraction.  Lost particles (loss word >= 0) are left out, as
 * the reference leaves out the rows past nLeft.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "trk.h"
#include "trk_constants.h"
#include "trk_lattice.h"

#include "trk_crmath.h"

#define OBS_CUDA(call)                                                                                              \
  do {                                                                                                              \
    cudaError_t e_ = (call);                                                                                        \
    if (e_ != cudaSuccess)                                                                                          \
      return trk_set_error(TRK_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));                                  \
  } while (0)

/* observer scratch held by the context (defined in trk_api.cu) */
int trk_context_scratch(trk_context *ctx, int site, int slot, size_t bytes, void **out);

namespace {

constexpr int OBS_THREADS = 128;
constexpr long OBS_CHUNK = 2048; /* particles per block: block partials independent of the grid */
constexpr double OBS_BIG = 1.7976931348623157e308;

struct Beam {
  const double *c[7]; /* x, xp, y, yp, s, delta, id */
  const int32_t *lost;
  long n;
};

/* the time coordinate of computeTimeCoordinates (src/trwake.c:533-548) */
__device__ __forceinline__ double time_of(double Po, double dp, double s) {
  const double P = __dmul_rn(Po, __dadd_rn(dp, 1.0));
  return __ddiv_rn(__dmul_rn(s, __dsqrt_rn(__dadd_rn(__dmul_rn(P, P), 1.0))), __dmul_rn(TRK_C_MKS, P));
}

/* double-double sum over the block, in a fixed order (warp shuffles, then
 * the warps in index order); the total is valid in thread 0 */
__device__ trkcr_dd block_dd_sum(trkcr_dd v, double *sh) {
  for (int off = 16; off > 0; off >>= 1) {
    const double h = __shfl_down_sync(0xffffffffu, v.hi, off);
    const double l = __shfl_down_sync(0xffffffffu, v.lo, off);
    v = trkcr_add(v, trkcr_make(h, l));
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) {
    sh[2 * warp] = v.hi;
    sh[2 * warp + 1] = v.lo;
  }
  __syncthreads();
  trkcr_dd t = trkcr_make(0.0, 0.0);
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      t = trkcr_add(t, trkcr_make(sh[2 * w], sh[2 * w + 1]));
  return t;
}

__device__ double block_min(double v, double *sh) {
  for (int off = 16; off > 0; off >>= 1)
    v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
  __syncthreads();
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = OBS_BIG;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      t = fmin(t, sh[w]);
  return t;
}

__device__ double block_max(double v, double *sh) {
  for (int off = 16; off > 0; off >>= 1)
    v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  __syncthreads();
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = -OBS_BIG;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
      t = fmax(t, sh[w]);
  return t;
}

/* selection of accumulate_beam_sums (src/compute_centroids.c:346-354) */
struct Select {
  double Po, tmin, tmax;
  long start_pid, end_pid;
  const double *time; /* caller's time coordinates, or null */
};

__device__ __forceinline__ bool chosen(const Beam &b, const Select &s, long i, double &t) {
  if (b.lost[i] >= 0)
    return false;
  t = s.time ? s.time[i] : time_of(s.Po, b.c[5][i], b.c[4][i]);
  const double id = b.c[6][i];
  return ((s.start_pid < 0 && s.end_pid < 0) || (id >= s.start_pid && id <= s.end_pid)) &&
         (s.tmin >= s.tmax || (t >= s.tmin && t <= s.tmax));
}

/* Pass 1 of the beam sums, one chunk per block.  Per chunk: double-double
 * sums of x, x', y, y', s, delta, t (and of x' pz, y' pz when `pz_mode`),
 * the count, and min / max / max |.| of x, x', y, y', delta.  Layout of a
 * block's partial (P1 doubles): [0..17] 9 sums as (hi, lo), [18] count,
 * [19..33] (min, max, maxabs) for coordinates 0, 1, 2, 3, 5. */
constexpr int P1 = 34;
__global__ void __launch_bounds__(OBS_THREADS) sums_pass1(Beam b, Select s, int pz_mode, double *part) {
  __shared__ double sh[2 * (OBS_THREADS / 32)];
  const long lo = (long)blockIdx.x * OBS_CHUNK, hi = min(b.n, lo + OBS_CHUNK);
  trkcr_dd acc[9];
  for (int k = 0; k < 9; k++)
    acc[k] = trkcr_make(0.0, 0.0);
  double cnt = 0, mn[5], mx[5], ma[5];
  for (int k = 0; k < 5; k++) {
    mn[k] = OBS_BIG;
    mx[k] = -OBS_BIG;
    ma[k] = 0;
  }
  for (long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double t;
    if (!chosen(b, s, i, t))
      continue;
    for (int k = 0; k < 6; k++)
      acc[k] = trkcr_add(acc[k], trkcr_make(b.c[k][i], 0.0));
    acc[6] = trkcr_add(acc[6], trkcr_make(t, 0.0));
    if (pz_mode) {
      /* pz = p_central (1 + delta) / sqrt(1 + x'^2 + y'^2) (src/compute_centroids.c:338-342) */
      const double xp = b.c[1][i], yp = b.c[3][i];
      const double pz = __ddiv_rn(__dmul_rn(s.Po, __dadd_rn(1.0, b.c[5][i])),
                                  __dsqrt_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(xp, xp)), __dmul_rn(yp, yp))));
      acc[7] = trkcr_add(acc[7], trkcr_make(__dmul_rn(xp, pz), 0.0));
      acc[8] = trkcr_add(acc[8], trkcr_make(__dmul_rn(yp, pz), 0.0));
    }
    cnt += 1;
    const int cols[5] = {0, 1, 2, 3, 5};
    for (int k = 0; k < 5; k++) {
      const double v = b.c[cols[k]][i];
      mn[k] = fmin(mn[k], v);
      mx[k] = fmax(mx[k], v);
      ma[k] = fmax(ma[k], fabs(v));
    }
  }
  double *out = part + (size_t)blockIdx.x * P1;
  for (int k = 0; k < 9; k++) {
    const trkcr_dd t = block_dd_sum(acc[k], sh);
    if (threadIdx.x == 0) {
      out[2 * k] = t.hi;
      out[2 * k + 1] = t.lo;
    }
  }
  {
    const trkcr_dd t = block_dd_sum(trkcr_make(cnt, 0.0), sh);
    if (threadIdx.x == 0)
      out[18] = t.hi;
  }
  for (int k = 0; k < 5; k++) {
    const double a = block_min(mn[k], sh), c = block_max(mx[k], sh), d = block_max(ma[k], sh);
    if (threadIdx.x == 0) {
      out[19 + 3 * k] = a;
      out[20 + 3 * k] = c;
      out[21 + 3 * k] = d;
    }
  }
}

/* Pass 2: second moments about the centroids.  Per chunk: double-double
 * sums of (c_i - m_i)(c_j - m_j), i <= j over x, x', y, y', s, delta, t
 * (28 pairs, in row order), of the normalized products when `pz_mode`
 * (src/compute_centroids.c:418-420, as written there: the second factor is
 * not centered and index 6 reads the particle ID column), and min / max /
 * max |.| of s - m_s and t - m_t.  Block partial: [0..55] sigma (hi, lo),
 * [56..111] sigman, [112..117] (min, max, maxabs) of s and t. */
constexpr int P2 = 118;
struct Moments {
  double m[7];  /* centroids (t: time centroid) */
  double mn[7]; /* centroids of the normalized coordinates */
  int sparse;
};

/* the pairs BEAM_SUMS_SPARSE keeps: diagonal blocks and dispersive
 * correlations (src/compute_centroids.c:301-308) */
#define OBS_SPARSE                                                                                                \
  {                                                                                                               \
    {1, 1, 0, 0, 0, 1, 0}, {0, 1, 0, 0, 0, 1, 0}, {0, 0, 1, 1, 0, 1, 0}, {0, 0, 0, 1, 0, 1, 0},                   \
      {0, 0, 0, 0, 1, 1, 1}, {0, 0, 0, 0, 0, 1, 0}, {0, 0, 0, 0, 0, 0, 1}                                         \
  }
__constant__ signed char k_sparse[7][7] = OBS_SPARSE;
static const signed char k_sparse_host[7][7] = OBS_SPARSE;

__global__ void __launch_bounds__(OBS_THREADS) sums_pass2(Beam b, Select s, Moments M, int pz_mode, double *part) {
  __shared__ double sh[2 * (OBS_THREADS / 32)];
  const long lo = (long)blockIdx.x * OBS_CHUNK, hi = min(b.n, lo + OBS_CHUNK);
  double *out = part + (size_t)blockIdx.x * P2;
  double smn = OBS_BIG, smx = -OBS_BIG, sma = 0, tmn = OBS_BIG, tmx = -OBS_BIG, tma = 0;
  /* one pair at a time keeps the per-thread state small; the chunk is read
   * from L1/L2 again for each pair */
  int pair = 0;
  for (int i = 0; i < 7; i++)
    for (int j = i; j < 7; j++, pair++) {
      trkcr_dd acc = trkcr_make(0.0, 0.0), accn = trkcr_make(0.0, 0.0);
      const bool skip = M.sparse && !k_sparse[i][j];
      if (!skip)
        for (long p = lo + threadIdx.x; p < hi; p += blockDim.x) {
          double t;
          if (!chosen(b, s, p, t))
            continue;
          const double tc = __dsub_rn(t, M.m[6]);
          const double di = i < 6 ? __dsub_rn(b.c[i][p], M.m[i]) : tc;
          const double dj = j < 6 ? __dsub_rn(b.c[j][p], M.m[j]) : tc;
          acc = trkcr_add(acc, trkcr_make(__dmul_rn(di, dj), 0.0));
          if (pz_mode) {
            const double xp = b.c[1][p], yp = b.c[3][p];
            const double pz = __ddiv_rn(__dmul_rn(s.Po, __dadd_rn(1.0, b.c[5][p])),
                                        __dsqrt_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(xp, xp)), __dmul_rn(yp, yp))));
            const double ui = (i == 1 || i == 3) ? __dmul_rn(b.c[i][p], pz) : b.c[i][p];
            const double uj = (j == 1 || j == 3) ? __dmul_rn(b.c[j][p], pz) : b.c[j][p];
            accn = trkcr_add(accn, trkcr_make(__dmul_rn(__dsub_rn(ui, M.mn[i]), uj), 0.0));
          }
          if (pair == 0) {
            const double ds = __dsub_rn(b.c[4][p], M.m[4]);
            smn = fmin(smn, ds);
            smx = fmax(smx, ds);
            sma = fmax(sma, fabs(ds));
            tmn = fmin(tmn, tc);
            tmx = fmax(tmx, tc);
            tma = fmax(tma, fabs(tc));
          }
        }
      else if (pair == 0)
        for (long p = lo + threadIdx.x; p < hi; p += blockDim.x) {
          double t;
          if (!chosen(b, s, p, t))
            continue;
          const double tc = __dsub_rn(t, M.m[6]);
          const double ds = __dsub_rn(b.c[4][p], M.m[4]);
          smn = fmin(smn, ds);
          smx = fmax(smx, ds);
          sma = fmax(sma, fabs(ds));
          tmn = fmin(tmn, tc);
          tmx = fmax(tmx, tc);
          tma = fmax(tma, fabs(tc));
        }
      const trkcr_dd r = block_dd_sum(acc, sh);
      const trkcr_dd rn = block_dd_sum(accn, sh);
      if (threadIdx.x == 0) {
        out[2 * pair] = r.hi;
        out[2 * pair + 1] = r.lo;
        out[56 + 2 * pair] = rn.hi;
        out[57 + 2 * pair] = rn.lo;
      }
    }
  const double v[6] = {block_min(smn, sh), block_max(smx, sh), block_max(sma, sh),
                       block_min(tmn, sh), block_max(tmx, sh), block_max(tma, sh)};
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; k++)
      out[112 + k] = v[k];
}

/* Combine the block partials in block order: `n_dd` double-double pairs at
 * the front, then `n_plain` values combined with `ops` (0 sum, 1 min, 2 max)
 * per value; one block, thread k owns value k. */
__global__ void combine_partials(const double *part, int nblocks, int stride, int n_dd, int n_plain,
                                 const signed char *ops, double *out) {
  const int k = threadIdx.x;
  if (k < n_dd) {
    trkcr_dd acc = trkcr_make(0.0, 0.0);
    for (int b = 0; b < nblocks; b++)
      acc = trkcr_add(acc, trkcr_make(part[(size_t)b * stride + 2 * k], part[(size_t)b * stride + 2 * k + 1]));
    out[2 * k] = acc.hi;
    out[2 * k + 1] = acc.lo;
  } else if (k < n_dd + n_plain) {
    const int q = 2 * n_dd + (k - n_dd);
    const int op = ops[k - n_dd];
    double acc = op == 0 ? 0.0 : (op == 1 ? OBS_BIG : -OBS_BIG);
    for (int b = 0; b < nblocks; b++) {
      const double v = part[(size_t)b * stride + q];
      acc = op == 0 ? __dadd_rn(acc, v) : (op == 1 ? fmin(acc, v) : fmax(acc, v));
    }
    out[q] = acc;
  }
}

/* Sum over survivors of Po (1 + delta) (src/do_tracking.c:3448-3455); one
 * chunk per block, partial = (hi, lo, count). */
__global__ void __launch_bounds__(OBS_THREADS) momentum_sum(Beam b, double Po, double *part) {
  __shared__ double sh[2 * (OBS_THREADS / 32)];
  const long lo = (long)blockIdx.x * OBS_CHUNK, hi = min(b.n, lo + OBS_CHUNK);
  trkcr_dd acc = trkcr_make(0.0, 0.0);
  double cnt = 0;
  for (long i = lo + threadIdx.x; i < hi; i += blockDim.x)
    if (b.lost[i] < 0) {
      acc = trkcr_add(acc, trkcr_make(__dmul_rn(Po, __dadd_rn(1.0, b.c[5][i])), 0.0));
      cnt += 1;
    }
  const trkcr_dd t = block_dd_sum(acc, sh);
  const trkcr_dd c = block_dd_sum(trkcr_make(cnt, 0.0), sh);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = t.hi;
    part[3 * blockIdx.x + 1] = t.lo;
    part[3 * blockIdx.x + 2] = c.hi;
  }
}

/* do_match_energy's updates (src/do_tracking.c:3479-3486 and 3518-3524) */
__global__ void match_energy_update(double *dp, double *s, const int32_t *lost, long n, int change_beam, double a,
                                    double b2, double Po) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    if (lost[i] >= 0)
      continue;
    if (!change_beam) {
      /* coord[5] = dp + coord[5] * dr */
      dp[i] = __dadd_rn(a, __dmul_rn(dp[i], b2));
    } else {
      /* a = dP_centroid */
      double P = __dmul_rn(__dadd_rn(1.0, dp[i]), Po);
      const double t = __ddiv_rn(s[i], __ddiv_rn(P, __dsqrt_rn(__dadd_rn(__dmul_rn(P, P), 1.0))));
      P = __dadd_rn(P, a);
      dp[i] = __ddiv_rn(__dsub_rn(P, Po), Po);
      s[i] = __dmul_rn(t, __ddiv_rn(P, __dsqrt_rn(__dadd_rn(__dmul_rn(P, P), 1.0))));
    }
  }
}

/* sort keys: survivors by particle ID, lost particles after them in their
 * current order */
__global__ void sort_keys(const double *id, const int32_t *lost, long n, long long *key, long *idx) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    key[i] = lost[i] < 0 ? (long long)id[i] : (1LL << 62) + i;
    idx[i] = i;
  }
}

template <typename T>
__global__ void gather(const T *src, const long *idx, long n, T *dst) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

/* the beam of a context: columns, loss words, device, stream */
struct Ctx {
  double *col[7];
  int32_t *loss[2];
  long n;
  int device;
  cudaStream_t st;
  trk_context *ctx;
};

int context_beam(trk_context *ctx, Ctx &c) {
  if (!ctx)
    return trk_set_error(TRK_ERR_ARG, "null context");
  int rc = trk_beam_device_columns(ctx, c.col, &c.n, c.loss);
  if (rc)
    return rc;
  c.st = (cudaStream_t)trk_context_stream(ctx);
  c.ctx = ctx;
  c.device = -1;
  if (c.n > 0) {
    cudaPointerAttributes at;
    OBS_CUDA(cudaPointerGetAttributes(&at, c.col[0]));
    c.device = at.device;
    OBS_CUDA(cudaSetDevice(c.device));
  }
  return TRK_OK;
}

Beam beam_of(const Ctx &c) {
  Beam b;
  for (int k = 0; k < 7; k++)
    b.c[k] = c.col[k];
  b.lost = c.loss[0];
  b.n = c.n;
  return b;
}

/* Device scratch of the observers, kept between calls in the context that
 * owns the beam (trk_context_scratch, trk_api.cu; freed by
 * trk_context_destroy): a cudaMalloc/cudaFree pair per call would cost more
 * than the reductions themselves, and cudaFree synchronizes the device.
 * Every call ends with a stream synchronization before it returns, so the
 * next call on the same context may reuse the buffers. */
struct Scratch {
  trk_context *ctx;
  int site, slot = 0;
  Scratch(trk_context *c, int site_) : ctx(c), site(site_) {}
  template <typename T>
  int get(T **out, size_t count) {
    void *p = nullptr;
    int rc = trk_context_scratch(ctx, site, slot, sizeof(T) * std::max<size_t>(count, 1), &p);
    if (rc)
      return rc;
    *out = (T *)p;
    slot++;
    return TRK_OK;
  }
};

/* pass-1 totals on the host: 9 rounded sums, count, 5 x (min, max, maxabs) */
int pass1(const Ctx &c, const Select &s, int pz_mode, double sums[9], double &count, double mm[15]) {
  const int nb = (int)((c.n + OBS_CHUNK - 1) / OBS_CHUNK);
  Scratch sc(c.ctx, 1);
  double *part, *out;
  signed char *ops;
  int rc;
  if ((rc = sc.get(&part, (size_t)nb * P1)) || (rc = sc.get(&out, P1)) || (rc = sc.get(&ops, 16)))
    return rc;
  signed char h_ops[16] = {0};
  for (int k = 0; k < 5; k++) {
    h_ops[1 + 3 * k] = 1;
    h_ops[2 + 3 * k] = 2;
    h_ops[3 + 3 * k] = 2;
  }
  OBS_CUDA(cudaMemcpyAsync(ops, h_ops, sizeof(h_ops), cudaMemcpyHostToDevice, c.st));
  sums_pass1<<<nb, OBS_THREADS, 0, c.st>>>(beam_of(c), s, pz_mode, part);
  combine_partials<<<1, 64, 0, c.st>>>(part, nb, P1, 9, 16, ops, out);
  double h[P1];
  OBS_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c.st));
  OBS_CUDA(cudaStreamSynchronize(c.st));
  for (int k = 0; k < 9; k++)
    sums[k] = h[2 * k] + h[2 * k + 1];
  count = h[18];
  for (int k = 0; k < 15; k++)
    mm[k] = h[19 + k];
  return TRK_OK;
}

} // namespace

extern "C" {

int trk_beam_centroids(trk_context *ctx, double *centroid, long *n) {
  if (!centroid)
    return trk_set_error(TRK_ERR_ARG, "null centroid array");
  Ctx c;
  int rc = context_beam(ctx, c);
  if (rc)
    return rc;
  for (int k = 0; k < 6; k++)
    centroid[k] = 0;
  if (n)
    *n = 0;
  if (c.n <= 0)
    return TRK_OK;
  Select s;
  s.Po = 1.0;
  s.tmin = s.tmax = 0;
  s.start_pid = s.end_pid = -1;
  s.time = nullptr;
  double sums[9], count, mm[15];
  if ((rc = pass1(c, s, 0, sums, count, mm)))
    return rc;
  if (count > 0)
    for (int k = 0; k < 6; k++)
      centroid[k] = sums[k] / count;
  if (n)
    *n = (long)count;
  return TRK_OK;
}

int trk_accumulate_beam_sums(trk_context *ctx, trk_beam_sums *sums, double p_central, double mp_charge,
                             const double *time_value, double t_min, double t_max, long start_pid, long end_pid,
                             unsigned int flags) {
  if (!sums)
    return trk_set_error(TRK_ERR_ARG, "null sums");
  Ctx c;
  int rc = context_beam(ctx, c);
  if (rc)
    return rc;
  const bool second = (flags & TRK_SUMS_SECOND_ORDER) != 0;
  const int pz_mode = (flags & TRK_SUMS_EXACT_NORMEMIT) ? 1 : 0;
  if (!sums->n_part)
    sums->p0 = p_central;
  long alive = 0;
  if ((rc = trk_beam_count(ctx, &alive)))
    return rc;
  double np_count = 0;
  if (alive > 0) {
    Scratch sc(c.ctx, 2);
    Select s;
    s.Po = p_central;
    s.tmin = t_min;
    s.tmax = t_max;
    s.start_pid = start_pid;
    s.end_pid = end_pid;
    s.time = nullptr;
    if (time_value) {
      /* the caller's time coordinates, one per loaded particle */
      double *d_time;
      if ((rc = sc.get(&d_time, (size_t)c.n)))
        return rc;
      OBS_CUDA(cudaMemcpyAsync(d_time, time_value, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.st));
      s.time = d_time;
    }
    double sum[9], mm[15];
    if ((rc = pass1(c, s, pz_mode, sum, np_count, mm)))
      return rc;
    if (!(flags & TRK_SUMS_NOMINMAX) && second) {
      const int cols[5] = {0, 1, 2, 3, 5};
      for (int k = 0; k < 5; k++) {
        const int i = cols[k];
        if (np_count > 0) {
          if (mm[3 * k + 2] > sums->maxabs[i])
            sums->maxabs[i] = mm[3 * k + 2];
          if (mm[3 * k + 1] > sums->max[i])
            sums->max[i] = mm[3 * k + 1];
          if (mm[3 * k] < sums->min[i])
            sums->min[i] = mm[3 * k];
        }
      }
    }
    /* centroids of this beam, folded into the running ones
     * (src/compute_centroids.c:357-385) */
    double cen[7], cenn[7];
    for (int i = 0; i < 7; i++) {
      cen[i] = sum[i];
      cenn[i] = 0;
    }
    cenn[1] = sum[7];
    cenn[3] = sum[8];
    if (np_count > 0)
      for (int i = 0; i < 7; i++) {
        sums->centroid[i] = (sums->centroid[i] * sums->n_part + cen[i]) / (sums->n_part + np_count);
        cen[i] /= np_count;
        cenn[i] /= np_count;
      }
    for (int i = 0; i < 7; i++)
      if (i != 1 && i != 3)
        cenn[i] = cen[i];
    if (second) {
      const int nb = (int)((c.n + OBS_CHUNK - 1) / OBS_CHUNK);
      double *part, *out;
      signed char *ops;
      if ((rc = sc.get(&part, (size_t)nb * P2)) || (rc = sc.get(&out, P2)) || (rc = sc.get(&ops, 8)))
        return rc;
      const signed char h_ops[6] = {1, 2, 2, 1, 2, 2};
      OBS_CUDA(cudaMemcpyAsync(ops, h_ops, sizeof(h_ops), cudaMemcpyHostToDevice, c.st));
      Moments M;
      for (int i = 0; i < 7; i++) {
        M.m[i] = cen[i];
        M.mn[i] = cenn[i];
      }
      M.sparse = (flags & TRK_SUMS_SPARSE) ? 1 : 0;
      sums_pass2<<<nb, OBS_THREADS, 0, c.st>>>(beam_of(c), s, M, pz_mode, part);
      combine_partials<<<1, 64, 0, c.st>>>(part, nb, P2, 56, 6, ops, out);
      double h[P2];
      OBS_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c.st));
      OBS_CUDA(cudaStreamSynchronize(c.st));
      if (!(flags & TRK_SUMS_NOMINMAX) && second && np_count > 0) {
        const int idx[2] = {4, 6};
        for (int k = 0; k < 2; k++) {
          const int i = idx[k];
          if (h[112 + 3 * k + 2] > sums->maxabs[i])
            sums->maxabs[i] = h[112 + 3 * k + 2];
          if (h[112 + 3 * k + 1] > sums->max[i])
            sums->max[i] = h[112 + 3 * k + 1];
          if (h[112 + 3 * k] < sums->min[i])
            sums->min[i] = h[112 + 3 * k];
        }
      }
      if (second) {
        /* (src/compute_centroids.c:398-450) */
        int pair = 0;
        for (int i = 0; i < 7; i++)
          for (int j = i; j < 7; j++, pair++) {
            if ((flags & TRK_SUMS_SPARSE) && !k_sparse_host[i][j]) {
              sums->sigma[j][i] = sums->sigma[i][j] = 0;
              sums->sigman[j][i] = sums->sigman[i][j] = 0;
              continue;
            }
            const double Sij = h[2 * pair] + h[2 * pair + 1];
            sums->sigma[j][i] = sums->sigma[i][j] = (sums->sigma[i][j] * sums->n_part + Sij) / (sums->n_part + np_count);
            if (pz_mode) {
              const double Sn = h[56 + 2 * pair] + h[57 + 2 * pair];
              sums->sigman[j][i] = sums->sigman[i][j] =
                (sums->sigman[i][j] * sums->n_part + Sn) / (sums->n_part + np_count);
            }
          }
      }
    }
  }
  sums->charge = mp_charge * np_count;
  sums->n_part += (long)np_count;
  return TRK_OK;
}

int trk_match_energy(trk_context *ctx, double *p_central, int change_beam) {
  if (!p_central)
    return trk_set_error(TRK_ERR_ARG, "null p_central");
  Ctx c;
  int rc = context_beam(ctx, c);
  if (rc)
    return rc;
  if (c.n <= 0)
    return TRK_OK;
  const double Po = *p_central;
  const int nb = (int)((c.n + OBS_CHUNK - 1) / OBS_CHUNK);
  Scratch sc(c.ctx, 4);
  double *part, *out;
  signed char *ops;
  if ((rc = sc.get(&part, (size_t)nb * 3)) || (rc = sc.get(&out, 3)) || (rc = sc.get(&ops, 1)))
    return rc;
  const signed char op = 0;
  OBS_CUDA(cudaMemcpyAsync(ops, &op, 1, cudaMemcpyHostToDevice, c.st));
  momentum_sum<<<nb, OBS_THREADS, 0, c.st>>>(beam_of(c), Po, part);
  combine_partials<<<1, 32, 0, c.st>>>(part, nb, 3, 1, 1, ops, out);
  double h[3];
  OBS_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, c.st));
  OBS_CUDA(cudaStreamSynchronize(c.st));
  const double np_alive = h[2];
  if (np_alive <= 0)
    return TRK_OK;
  const double P_average = (h[0] + h[1]) / np_alive;
  const int grid = (int)std::min<long>((c.n + 255) / 256, 4096);
  if (!change_beam) {
    /* change the central momentum to the beam's (src/do_tracking.c:3474-3487) */
    if (fabs(P_average - Po) / Po > 1e-14) {
      const double dp = (Po - P_average) / P_average;
      const double dr = Po / P_average;
      match_energy_update<<<grid, 256, 0, c.st>>>(c.col[5], c.col[4], c.loss[0], c.n, 0, dp, dr, Po);
      *p_central = P_average;
    }
  } else {
    /* change the momenta so the centroid is the central momentum, keeping
     * each particle's time of flight (src/do_tracking.c:3516-3524) */
    match_energy_update<<<grid, 256, 0, c.st>>>(c.col[5], c.col[4], c.loss[0], c.n, 1, Po - P_average, 0.0, Po);
  }
  OBS_CUDA(cudaGetLastError());
  OBS_CUDA(cudaStreamSynchronize(c.st));
  return TRK_OK;
}

int trk_sort_by_id(trk_context *ctx) {
  Ctx c;
  int rc = context_beam(ctx, c);
  if (rc)
    return rc;
  if (c.n <= 1)
    return TRK_OK;
  const long n = c.n;
  Scratch sc(c.ctx, 5);
  long long *k0, *k1;
  long *i0, *i1;
  if ((rc = sc.get(&k0, n)) || (rc = sc.get(&k1, n)) || (rc = sc.get(&i0, n)) || (rc = sc.get(&i1, n)))
    return rc;
  const int grid = (int)std::min<long>((n + 255) / 256, 4096);
  sort_keys<<<grid, 256, 0, c.st>>>(c.col[6], c.loss[0], n, k0, i0);
  /* CUB's radix sort is stable: equal IDs keep their order */
  size_t tmp_bytes = 0;
  OBS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, k0, k1, i0, i1, (int)n, 0, 64, c.st));
  unsigned char *tmp_sort;
  if ((rc = sc.get(&tmp_sort, tmp_bytes)))
    return rc;
  OBS_CUDA(cub::DeviceRadixSort::SortPairs(tmp_sort, tmp_bytes, k0, k1, i0, i1, (int)n, 0, 64, c.st));
  std::swap(k0, k1);
  std::swap(i0, i1);
  /* permute every column and both loss words by i0 */
  double *tmp;
  int32_t *tmpi;
  if ((rc = sc.get(&tmp, n)) || (rc = sc.get(&tmpi, n)))
    return rc;
  for (int k = 0; k < 7; k++) {
    gather<double><<<grid, 256, 0, c.st>>>(c.col[k], i0, n, tmp);
    OBS_CUDA(cudaMemcpyAsync(c.col[k], tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.st));
  }
  for (int k = 0; k < 2; k++) {
    gather<int32_t><<<grid, 256, 0, c.st>>>(c.loss[k], i0, n, tmpi);
    OBS_CUDA(cudaMemcpyAsync(c.loss[k], tmpi, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, c.st));
  }
  OBS_CUDA(cudaGetLastError());
  OBS_CUDA(cudaStreamSynchronize(c.st));
  return TRK_OK;
}

} /* extern "C" */

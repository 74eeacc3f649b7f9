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
int trk_context_host_scratch(trk_context *ctx, size_t bytes, void **out);

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

/* selection of accumulate_beam_sums (src/compute_centroids.c:346-354) */
struct Select {
  double Po, tmin, tmax;
  long start_pid, end_pid;
  int pid_window;     /* start_pid or end_pid given */
  const double *time; /* time coordinates to read (the caller's, or pass 1's), or null */
  double *time_out;   /* pass 1 writes the time coordinates it computes here, when set */
};

/* Beam sums.  The beam is cut into chunks whose size depends on the number
 * of particles only (sum_chunk), and every chunk gets its own partial, so the
 * partials do not depend on the device, the grid or on which block summed
 * which chunk.  Within a block a thread keeps, per sum, a running double and
 * the plain sum of the exact errors of its additions (Knuth's TwoSum): a
 * compensated sum whose error is of order u^2 per term.  The lanes then
 * combine their pairs as double-double values in a fixed order (a butterfly,
 * warp_dd_scatter), the warps in index order, and the chunks in chunk order,
 * so every total is the double-double of the exact sum of the rounded terms to
 * about 2^-100 relative, rounded once at the end.  Particles that are lost or
 * outside the windows are skipped.
 *
 * Data movement: persistent block b takes chunks b, b + G, b + 2G, ... (G
 * blocks; about ten chunks a block), and a ring of SUM_STAGES tiles of
 * sum_tile particles in shared memory is filled by 1-D bulk copies
 * (cp.async.bulk, from this device's own beam columns) that complete on a
 * "full" mbarrier per stage; each warp arrives on the stage's "empty"
 * mbarrier when it has read the tile, and the issuing thread refills the
 * stage once every warp has, so the warps synchronize only at chunk ends.
 * Every warp steps through the same tile sequence itself, so all agree on
 * the chunk boundaries without reading shared state.  Bulk copies need 16-byte aligned sources
 * and sizes: the beam columns are tile-aligned slices of arrays whose
 * stride (the beam capacity) is a multiple of 32 entries, and a tile's copy
 * is rounded up to whole 16-byte units inside that capacity.
 *
 * Pass 1 runs 128 threads a block, one particle a thread.  Pass 2 runs 256:
 * the even warps take the first 14 of the 28 second moments of a particle and
 * the odd warps the other 14, which halves the running sums a thread holds,
 * and so its registers, and doubles the warps an SM keeps in flight. */
constexpr int SUM_STAGES = 2;
constexpr long SUM_CHUNK_MIN = 1024, SUM_CHUNK_MAX = 8192;
/* particles per tile: pass 1 512, pass 2 896 (7 particles a thread between
 * barriers, and two blocks of two stages fit an SM with the time column) */
template <int PASS> __host__ __device__ constexpr int sum_tile() { return PASS == 1 ? 512 : 896; }
/* the most shared memory a pass's stages take (every column staged) */
template <int PASS> __host__ __device__ constexpr int sum_smem_max() { return SUM_STAGES * sum_tile<PASS>() * (8 * 8 + 4); }
constexpr int COMBINE_THREADS = 512, COMBINE_BATCH = 8;
/* a bulk copy that has not completed after this long is reported as an error */
constexpr unsigned long long SUM_WAIT_NS = 2000000000ull;

template <int PASS> __host__ __device__ constexpr int sum_threads() { return PASS == 1 ? 128 : 256; }
template <int PASS> __host__ __device__ constexpr int sum_blocks_per_sm() { return PASS == 1 ? 4 : 2; }

/* Particles per chunk of a pass: about 4096 chunks (enough for every block
 * of a persistent grid to take several, so the last ones balance), between
 * SUM_CHUNK_MIN and SUM_CHUNK_MAX so the per-chunk combination stays a small
 * part of the work, a multiple of the pass's tile.  A function of n alone. */
template <int PASS>
__host__ __device__ inline long sum_chunk(long n) {
  constexpr long T = sum_tile<PASS>();
  long c = (n + 4095) / 4096;
  c = c < SUM_CHUNK_MIN ? SUM_CHUNK_MIN : (c > SUM_CHUNK_MAX ? SUM_CHUNK_MAX : c);
  return (c + T - 1) / T * T;
}

/* kernel variants: the time coordinate is needed; the ID column is read;
 * the pz-normalized sums (pass 1: x' pz, y' pz; pass 2: sigman) */
enum { SF_TIME = 1, SF_ID = 2, SF_PZ = 4 };

/* status word of the sums kernels */
enum { SUM_STATUS_OK = 0, SUM_STATUS_COPY_TIMEOUT = 1 };

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

/* wait for the phase of `parity` to complete, for SUM_WAIT_NS at most, and
 * give up at once when `fail` (when given) is set */
__device__ bool mbar_wait(uint64_t *bar, unsigned parity, const volatile int *fail = nullptr) {
  if (mbar_test(bar, parity))
    return true;
  const unsigned long long t0 = global_ns();
  for (long k = 0; k < (1L << 28); k++) {
    if (mbar_test(bar, parity))
      return true;
    if ((fail && *fail) || global_ns() - t0 > SUM_WAIT_NS)
      return false;
    __nanosleep(32);
  }
  return false;
}

/* one 1-D bulk copy global -> shared, completing on `bar` */
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                 smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

/* s + x with the exact error of the addition added into e (Knuth's TwoSum) */
__device__ __forceinline__ void csum_add(double &s, double &e, double x) {
  const double t = __dadd_rn(s, x);
  const double bb = __dsub_rn(t, s);
  e = __dadd_rn(e, __dadd_rn(__dsub_rn(s, __dsub_rn(t, bb)), __dsub_rn(x, bb)));
  s = t;
}

/* double-double addition with the low parts added in plain double (Dekker):
 * the combinations of already compensated sums, whose low parts are a few
 * units of 2^-53 of their high parts */
__device__ __forceinline__ trkcr_dd dd_add(trkcr_dd a, trkcr_dd b) {
  const trkcr_dd s = trkcr_two_sum(a.hi, b.hi);
  return trkcr_quick_two_sum(s.hi, __dadd_rn(s.lo, __dadd_rn(a.lo, b.lo)));
}

/* log2 of a power of two up to 32 */
template <int NP> __host__ __device__ constexpr int log2_of() { return NP <= 1 ? 0 : 1 + log2_of<NP / 2>(); }

/* Lane butterfly over NP (a power of two <= 32) double-double values: steps
 * at distances 16, 8, ... keep half of the values (the upper half in the lane
 * whose distance bit is set) and add the partner's copy of that half, until
 * one value is left; the remaining steps add it across the lane pair.
 * Afterwards lane L holds value L >> (5 - log2 NP) in h[0], l[0]: NP - 1 + 5 -
 * log2 NP additions a lane.  Both lanes of a pair add the lower lane's value
 * first, so the result does not depend on the lane. */
template <int NP>
__device__ __forceinline__ void warp_dd_scatter(double (&h)[NP], double (&l)[NP]) {
  const int lane = threadIdx.x & 31;
  constexpr int K = log2_of<NP>();
#pragma unroll
  for (int j = 0; j < K; j++) {
    const int m = 16 >> j, half = NP >> (j + 1);
    const bool up = (lane & m) != 0;
#pragma unroll
    for (int i = 0; i < half; i++) {
      const double sh = up ? h[i] : h[i + half], sl = up ? l[i] : l[i + half];
      const double kh = up ? h[i + half] : h[i], kl = up ? l[i + half] : l[i];
      const double rh = __shfl_xor_sync(0xffffffffu, sh, m), rl = __shfl_xor_sync(0xffffffffu, sl, m);
      const trkcr_dd s = dd_add(trkcr_make(up ? rh : kh, up ? rl : kl), trkcr_make(up ? kh : rh, up ? kl : rl));
      h[i] = s.hi;
      l[i] = s.lo;
    }
  }
#pragma unroll
  for (int j = K; j < 5; j++) {
    const int m = 16 >> j;
    const bool up = (lane & m) != 0;
    const double rh = __shfl_xor_sync(0xffffffffu, h[0], m), rl = __shfl_xor_sync(0xffffffffu, l[0], m);
    const trkcr_dd s = dd_add(trkcr_make(up ? rh : h[0], up ? rl : l[0]), trkcr_make(up ? h[0] : rh, up ? l[0] : rl));
    h[0] = s.hi;
    l[0] = s.lo;
  }
}

/* The block's NG x NV double-double totals from the threads' compensated
 * sums (s, e).  The warps form NG groups (group of warp w: w % NG), each with
 * its own NV values; after the butterfly in each warp, thread g NV + u adds
 * value u over the warps of group g in index order and writes it to
 * out[2 (g NV + u) os], out[(2 (g NV + u) + 1) os].  `sh` holds 2 NV WARPS
 * doubles; every thread of the block calls it. */
template <int NV, int NP, int WARPS, int NG>
__device__ __forceinline__ void block_dd_totals(double (&s)[NP], double (&e)[NP], double *sh, double *out,
                                                long os) {
  constexpr int SHIFT = 5 - log2_of<NP>();
#pragma unroll
  for (int v = 0; v < NP; v++) {
    const trkcr_dd t = trkcr_two_sum(s[v], e[v]);
    s[v] = t.hi;
    e[v] = t.lo;
  }
  warp_dd_scatter<NP>(s, e);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int v = lane >> SHIFT;
  if ((lane & ((1 << SHIFT) - 1)) == 0 && v < NV) {
    sh[2 * (warp * NV + v)] = s[0];
    sh[2 * (warp * NV + v) + 1] = e[0];
  }
  __syncthreads();
  if (threadIdx.x < NG * NV) {
    const int g = threadIdx.x / NV, u = threadIdx.x % NV;
    trkcr_dd t = trkcr_make(sh[2 * (g * NV + u)], sh[2 * (g * NV + u) + 1]);
    for (int w = g + NG; w < WARPS; w += NG)
      t = dd_add(t, trkcr_make(sh[2 * (w * NV + u)], sh[2 * (w * NV + u) + 1]));
    out[2 * threadIdx.x * os] = t.hi;
    out[(2 * threadIdx.x + 1) * os] = t.lo;
  }
  __syncthreads();
}

/* the block's extremes -> out[v os]: value v is a minimum when bit v of
 * `min_mask` is set, else a maximum; `sh` holds NV WARPS doubles */
template <int NV, int WARPS>
__device__ __forceinline__ void block_extremes(double (&x)[NV], unsigned min_mask, double *sh, double *out,
                                               long os) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; v++) {
    const bool is_min = (min_mask >> v) & 1u;
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, x[v], off);
      x[v] = is_min ? fmin(x[v], o) : fmax(x[v], o);
    }
    if (lane == 0)
      sh[warp * NV + v] = x[v];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int v = threadIdx.x;
    const bool is_min = (min_mask >> v) & 1u;
    double t = sh[v];
    for (int w = 1; w < WARPS; w++)
      t = is_min ? fmin(t, sh[w * NV + v]) : fmax(t, sh[w * NV + v]);
    out[v * os] = t;
  }
  __syncthreads();
}

/* the block's count of a per-thread integer -> out[0] */
template <int WARPS>
__device__ __forceinline__ void block_count(int n, int *sh, double *out) {
  n = __reduce_add_sync(0xffffffffu, n);
  if ((threadIdx.x & 31) == 0)
    sh[threadIdx.x >> 5] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    long t = 0;
    for (int w = 0; w < WARPS; w++)
      t += sh[w];
    out[0] = (double)t;
  }
  __syncthreads();
}

/* one particle's columns, read from a staged tile */
struct Row {
  double v[6], id, t;
  int32_t lost;
};

/* the time coordinate and the selection of one loaded particle */
template <int F>
__device__ __forceinline__ bool select_row(const Select &s, Row &r) {
  bool ok = r.lost < 0;
  if (F & SF_TIME) {
    if (!s.time)
      r.t = time_of(s.Po, r.v[5], r.v[4]);
    ok = ok && (s.tmin >= s.tmax || (r.t >= s.tmin && r.t <= s.tmax));
  }
  if ((F & SF_ID) && s.pid_window)
    ok = ok && r.id >= s.start_pid && r.id <= s.end_pid;
  return ok;
}

/* pz = p_central (1 + delta) / sqrt(1 + x'^2 + y'^2) (src/compute_centroids.c:338-342) */
__device__ __forceinline__ double pz_of(double Po, const Row &r) {
  const double xp = r.v[1], yp = r.v[3];
  return __ddiv_rn(__dmul_rn(Po, __dadd_rn(1.0, r.v[5])),
                   __dsqrt_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(xp, xp)), __dmul_rn(yp, yp))));
}

/* P1 / P2: the chunk partial layouts of the two passes (doubles per chunk,
 * stored value-major: value i of chunk c at part[i nchunks + c]) */
constexpr int P1 = 39;
constexpr int P1_COUNT = 18;
/* plain values (from P1_COUNT): count, 5 x (min, max, maxabs), survivors,
 * min s, max s, min t, max t */
constexpr unsigned P1_MIN_MASK = 0x2492u | (1u << 17) | (1u << 19);
constexpr unsigned P1_MAX_MASK = 0xDB6Cu | (1u << 18) | (1u << 20);
constexpr int P2 = 118;
constexpr unsigned P2_MIN_MASK = 0x9u; /* plain values 0 and 3 */
constexpr unsigned P2_MAX_MASK = 0x36u;

/* (min, max) pairs -> (min, max, max |.|) triples; max |.| = max(|min|,
 * |max|), which is the largest |value| of the values seen, 0 when none */
template <int N>
__device__ __forceinline__ void with_maxabs(const double *mm, double (&x)[3 * N]) {
#pragma unroll
  for (int k = 0; k < N; k++) {
    x[3 * k] = mm[2 * k];
    x[3 * k + 1] = mm[2 * k + 1];
    x[3 * k + 2] = mm[2 * k] <= mm[2 * k + 1] ? fmax(fabs(mm[2 * k]), fabs(mm[2 * k + 1])) : 0.0;
  }
}

/* the pairs BEAM_SUMS_SPARSE keeps: diagonal blocks and dispersive
 * correlations (src/compute_centroids.c:301-308) */
#define OBS_SPARSE                                                                                                \
  {                                                                                                               \
    {1, 1, 0, 0, 0, 1, 0}, {0, 1, 0, 0, 0, 1, 0}, {0, 0, 1, 1, 0, 1, 0}, {0, 0, 0, 1, 0, 1, 0},                   \
      {0, 0, 0, 0, 1, 1, 1}, {0, 0, 0, 0, 0, 1, 0}, {0, 0, 0, 0, 0, 0, 1}                                         \
  }
__constant__ signed char k_sparse[7][7] = OBS_SPARSE;
static const signed char k_sparse_host[7][7] = OBS_SPARSE;

/* centroids of pass 1 (m) and of the normalized coordinates (mn) */
__device__ __forceinline__ void moments_of(const double *tot1, double m[7], double mn[7]) {
  const double count = tot1[P1_COUNT];
#pragma unroll
  for (int k = 0; k < 7; k++) {
    m[k] = __dadd_rn(tot1[2 * k], tot1[2 * k + 1]);
    mn[k] = 0.0;
  }
  mn[1] = __dadd_rn(tot1[14], tot1[15]);
  mn[3] = __dadd_rn(tot1[16], tot1[17]);
  if (count > 0)
#pragma unroll
    for (int k = 0; k < 7; k++) {
      m[k] = __ddiv_rn(m[k], count);
      mn[k] = __ddiv_rn(mn[k], count);
    }
#pragma unroll
  for (int k = 0; k < 7; k++)
    if (k != 1 && k != 3)
      mn[k] = m[k];
}

/* a power of two above x > 0 (2^-1022 for x = 0 or subnormal; infinity
 * past the range) */
__device__ __forceinline__ double pow2_above(double x) {
  const long long e = __double_as_longlong(x) & 0x7ff0000000000000LL;
  return __longlong_as_double(e + (1LL << 52));
}

/* Biases of the 28 second-moment sums (pairs in row order).  A thread's sum
 * of pair (a, c) starts at B = a power of two above 4 K max|d_a| max|d_c|,
 * K the particles a thread sums per chunk and max|d| the largest centered
 * value of pass 1's extremes (rounded subtraction and product are monotonic,
 * so these bound every term).  The running sum then stays within [B/2, 2B]
 * and above every term, Dekker's condition for Fast2Sum: each addition's
 * rounding error is x - ((s + x) - s) exactly, 3 operations instead of
 * TwoSum's 6, and the sum less B is exact at the end.  A bound that
 * overflows gives B = 0: that pair is then a plain compensated sum. */
__device__ __forceinline__ void sum_biases(const double *tot1, const double m[7], long K, double bias[28]) {
  /* extremes of pass 1 by coordinate: x, x', y, y', s, delta, t */
  const int lo[7] = {19, 22, 25, 28, 35, 31, 37};
  double D[7];
  for (int k = 0; k < 7; k++)
    D[k] = fmax(fabs(__dsub_rn(tot1[lo[k]], m[k])), fabs(__dsub_rn(tot1[lo[k] + 1], m[k])));
  int pair = 0;
  for (int a = 0; a < 7; a++)
    for (int c = a; c < 7; c++, pair++) {
      const double b = pow2_above(__dmul_rn(4.0 * (double)K, __dmul_rn(D[a], D[c])));
      bias[pair] = isfinite(b) ? b : 0.0;
    }
}

/* the ring of staged tiles: per stage a "full" mbarrier (the tile's copies
 * landed) and an "empty" one (every warp has read the tile) */
struct Ring {
  uint64_t full[SUM_STAGES], empty[SUM_STAGES];
  volatile int fail;
};

/* tiles of chunk c */
template <int TILE>
__device__ __forceinline__ int tiles_of(long c, long n, long chunk_n) {
  const long lo = c * chunk_n, hi = min(n, lo + chunk_n);
  return (int)((hi - lo + TILE - 1) / TILE);
}

/* where a stage keeps its columns: doubles 0..5 the coordinates, then the ID
 * and the caller's time when the variant reads them (column -1 when not),
 * the loss words after the last column */
struct Layout {
  int id_col, t_col, ncols;
  unsigned stage_bytes;
};

template <int F, int TILE>
__host__ __device__ inline Layout layout_of(const Select &s) {
  Layout l;
  l.ncols = 6;
  l.id_col = (F & SF_ID) ? l.ncols++ : -1;
  l.t_col = ((F & SF_TIME) && s.time) ? l.ncols++ : -1;
  l.stage_bytes = (unsigned)TILE * (8u * (unsigned)l.ncols + 4u);
  return l;
}

/* A position in a block's stream of tiles: chunks b, b + G, b + 2G, ... (G
 * blocks), each cut into tiles.  Every thread can step through it, so all
 * warps agree on the chunk boundaries without reading shared state. */
struct TilePos {
  long chunk;
  int tile, ntiles;
};

struct TileStream {
  long nchunks, stride, n, chunk_n;
  template <int TILE>
  __device__ TilePos first(long c) const {
    TilePos p;
    p.chunk = c;
    p.tile = 0;
    p.ntiles = c < nchunks ? tiles_of<TILE>(c, n, chunk_n) : 0;
    return p;
  }
  template <int TILE>
  __device__ void next(TilePos &p) const {
    if (++p.tile >= p.ntiles) {
      p.chunk += stride;
      p.tile = 0;
      p.ntiles = p.chunk < nchunks ? tiles_of<TILE>(p.chunk, n, chunk_n) : 0;
    }
  }
  __device__ bool done(const TilePos &p) const { return p.chunk >= nchunks; }
};

/* Issue the copies of tile `tile` of chunk `chunk` into `stage` (thread 0). */
template <int TILE>
__device__ void issue_tile(Ring &r, unsigned char *smem, const Layout &L, int stage, long chunk, int tile,
                           const Beam &b, const Select &s, long chunk_n) {
  unsigned char *st = smem + (size_t)stage * L.stage_bytes;
  const long start = chunk * chunk_n + (long)tile * TILE;
  const int cnt = (int)min((long)TILE, b.n - start);
  /* whole 16-byte units: 2 doubles, 4 loss words (inside the capacity) */
  const unsigned bd = (unsigned)((cnt + 1) & ~1) * 8u, bl = (unsigned)((cnt + 3) & ~3) * 4u;
  mbar_arrive_expect_tx(&r.full[stage], bd * (unsigned)L.ncols + bl);
  for (int k = 0; k < 6; k++)
    bulk_load(st + (size_t)k * TILE * 8, b.c[k] + start, bd, &r.full[stage]);
  if (L.id_col >= 0)
    bulk_load(st + (size_t)L.id_col * TILE * 8, b.c[6] + start, bd, &r.full[stage]);
  if (L.t_col >= 0)
    bulk_load(st + (size_t)L.t_col * TILE * 8, s.time + start, bd, &r.full[stage]);
  bulk_load(st + (size_t)L.ncols * TILE * 8, b.lost + start, bl, &r.full[stage]);
}

/* The 14 second moments of pair group G (pairs 14 G .. 14 G + 13 in row
 * order) of one particle: S[k], E[k] += (x_a - c_a) y_c for pair 14 G + k =
 * (a, c), with c_a = 0 when `center` is null (the factors are then already
 * centered); pairs BEAM_SUMS_SPARSE drops are left out when SPARSE.
 * BIASED: the sums run from the biases of sum_biases (Fast2Sum). */
template <int G, bool BIASED, bool SPARSE>
__device__ __forceinline__ void pair_sums(double (&S)[16], double (&E)[16], const double (&x)[7],
                                          const double (&y)[7], const double *center) {
  int pair = 0;
#pragma unroll
  for (int a = 0; a < 7; a++)
#pragma unroll
    for (int c = a; c < 7; c++, pair++)
      if (pair >= 14 * G && pair < 14 * G + 14 && (!SPARSE || k_sparse[a][c])) {
        const double xa = center ? __dsub_rn(x[a], center[a]) : x[a];
        const double t = __dmul_rn(xa, y[c]);
        if (BIASED) {
          /* Fast2Sum: the running sum is above every term (sum_biases) */
          double &sk = S[pair - 14 * G];
          const double u = __dadd_rn(sk, t);
          E[pair - 14 * G] = __dadd_rn(E[pair - 14 * G], __dsub_rn(t, __dsub_rn(u, sk)));
          sk = u;
        } else {
          csum_add(S[pair - 14 * G], E[pair - 14 * G], t);
        }
      }
}

/* The beam-sum passes, one partial per chunk.
 *
 * Pass 1 (PASS = 1): sums of x, x', y, y', s, delta, t (SF_TIME) and of
 * x' pz, y' pz (SF_PZ) per chunk: [0..17] 9 sums as (hi, lo).  Per block:
 * [0] the count of selected particles, [1..15] (min, max, max |.|) of x, x',
 * y, y', delta, [16] the count of surviving particles, [17..20] min / max of
 * s and t.
 *
 * Pass 2 (PASS = 2): second moments about the centroids, which each block
 * forms from the combined pass-1 totals `tot1` as the host forms them
 * (src/compute_centroids.c:357-385).  Sums of (c_i - m_i)(c_j - m_j), i <= j
 * over x, x', y, y', s, delta, t (28 pairs, in row order), and min / max /
 * max |.| of s - m_s and t - m_t; or, with SF_PZ, the sums of the normalized
 * products (src/compute_centroids.c:418-420, as written there: the second
 * factor is not centered and index 6 reads the particle ID column).  Per
 * chunk: [0..55] sigma (hi, lo), [56..111] sigman.  Per block (without
 * SF_PZ): (min, max, max |.|) of s - m_s and t - m_t.
 *
 * `status` gets SUM_STATUS_COPY_TIMEOUT when a staged copy did not complete
 * in time; the block then waits (bounded) for its copies in flight and
 * returns. */
template <int PASS, int F>
__global__ void __launch_bounds__(sum_threads<PASS>(), sum_blocks_per_sm<PASS>())
  beam_sums(Beam b, Select s, const double *tot1, int sparse, int *status, double *part, double *blk) {
  constexpr int THREADS = sum_threads<PASS>(), WARPS = THREADS / 32, TILE = sum_tile<PASS>();
  constexpr int NV = PASS == 1 ? 9 : 14;  /* sums a thread keeps */
  constexpr int NP = 16;                  /* butterfly width */
  constexpr int NM = PASS == 1 ? 14 : 4; /* running (min, max) values */
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ Ring r;
  __shared__ double red[2 * 14 * 8];
  __shared__ int redc[WARPS];
  __shared__ double sm_m[7], sm_mn[7], sm_bias[28];
  const long n = b.n, chunk_n = sum_chunk<PASS>(n), nchunks = (n + chunk_n - 1) / chunk_n;
  const Layout L = layout_of<F, TILE>(s);
  constexpr bool BIASED = PASS == 2 && !(F & SF_PZ);
  if (PASS == 2 && threadIdx.x == 0) {
    moments_of(tot1, sm_m, sm_mn);
    if (BIASED)
      sum_biases(tot1, sm_m, (chunk_n + 127) / 128, sm_bias);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  /* pass 2: the pair group of the warp and the particle slot of the thread */
  const int grp = PASS == 2 ? (warp & 1) : 0;
  const int slot = PASS == 2 ? (warp >> 1) * 32 + lane : (int)threadIdx.x;
  double S[NP], E[NP], M[NM];
  int cnt = 0, alive = 0;
  /* the sums restart at every chunk; extremes and counts, which do not
   * depend on the order they are formed in, run over the block's chunks */
  auto reset = [&]() {
#pragma unroll
    for (int k = 0; k < NP; k++)
      S[k] = E[k] = 0.0;
    if (BIASED)
#pragma unroll
      for (int k = 0; k < 14; k++)
        S[k] = sm_bias[14 * grp + k];
  };
#pragma unroll
  for (int k = 0; k < NM; k++)
    M[k] = (k % 2 == 0) ? OBS_BIG : -OBS_BIG;
  __syncthreads();
  reset();
  if (threadIdx.x == 0) {
    for (int k = 0; k < SUM_STAGES; k++) {
      mbar_init(&r.full[k], 1);
      mbar_init(&r.empty[k], WARPS);
    }
    r.fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const double *m = sm_m, *mn = sm_mn;
  /* the consumers' position in the block's tiles; the issuing thread keeps
   * SUM_STAGES tiles ahead */
  TileStream ts;
  ts.nchunks = nchunks;
  ts.stride = gridDim.x;
  ts.n = n;
  ts.chunk_n = chunk_n;
  TilePos cs = ts.first<TILE>(blockIdx.x);
  long issued = 0;
  if (threadIdx.x == 0) {
    TilePos ps = cs;
    for (int k = 0; k < SUM_STAGES && !ts.done(ps); k++, issued++, ts.next<TILE>(ps))
      issue_tile<TILE>(r, smem, L, k, ps.chunk, ps.tile, b, s, chunk_n);
  }
  long it = 0;
  for (; !ts.done(cs); it++, ts.next<TILE>(cs)) {
    const int stage = (int)(it % SUM_STAGES);
    const unsigned parity = (unsigned)((it / SUM_STAGES) & 1);
    const bool ok = mbar_wait(&r.full[stage], parity, &r.fail);
    if (!ok)
      r.fail = 1;
    const long chunk = cs.chunk;
    const int tile = cs.tile;
    if (ok) {
      const double *col = (const double *)(smem + (size_t)stage * L.stage_bytes);
      const int32_t *lost = (const int32_t *)(col + L.ncols * TILE);
      const long start = chunk * chunk_n + (long)tile * TILE;
      const int n_tile = (int)min((long)TILE, n - start);
      for (int q = slot; q < n_tile; q += 128) {
        Row w;
        w.lost = lost[q];
#pragma unroll
        for (int k = 0; k < 6; k++)
          w.v[k] = col[k * TILE + q];
        w.id = (F & SF_ID) ? col[L.id_col * TILE + q] : 0.0;
        w.t = ((F & SF_TIME) && s.time) ? col[L.t_col * TILE + q] : 0.0;
        const bool sel = select_row<F>(s, w);
        if (PASS == 1) {
          alive += w.lost < 0;
          if ((F & SF_TIME) && s.time_out)
            s.time_out[start + q] = w.t;
        }
        if (!sel)
          continue;
        if constexpr (PASS == 1) {
          cnt++;
#pragma unroll
          for (int k = 0; k < 6; k++)
            csum_add(S[k], E[k], w.v[k]);
          if (F & SF_TIME)
            csum_add(S[6], E[6], w.t);
          if (F & SF_PZ) {
            const double pz = pz_of(s.Po, w);
            csum_add(S[7], E[7], __dmul_rn(w.v[1], pz));
            csum_add(S[8], E[8], __dmul_rn(w.v[3], pz));
          }
          const int cols[6] = {0, 1, 2, 3, 5, 4};
#pragma unroll
          for (int k = 0; k < 6; k++) {
            M[2 * k] = fmin(M[2 * k], w.v[cols[k]]);
            M[2 * k + 1] = fmax(M[2 * k + 1], w.v[cols[k]]);
          }
          if (F & SF_TIME) {
            M[12] = fmin(M[12], w.t);
            M[13] = fmax(M[13], w.t);
          }
        } else if constexpr (!(F & SF_PZ)) {
          double d[7];
#pragma unroll
          for (int k = 0; k < 6; k++)
            d[k] = __dsub_rn(w.v[k], m[k]);
          d[6] = __dsub_rn(w.t, m[6]);
          if (grp == 0) {
            if (sparse)
              pair_sums<0, BIASED, true>(S, E, d, d, nullptr);
            else
              pair_sums<0, BIASED, false>(S, E, d, d, nullptr);
            M[0] = fmin(M[0], d[4]);
            M[1] = fmax(M[1], d[4]);
            M[2] = fmin(M[2], d[6]);
            M[3] = fmax(M[3], d[6]);
          } else if (sparse) {
            pair_sums<1, BIASED, true>(S, E, d, d, nullptr);
          } else {
            pair_sums<1, BIASED, false>(S, E, d, d, nullptr);
          }
        } else {
          const double pz = pz_of(s.Po, w);
          double u[7];
#pragma unroll
          for (int k = 0; k < 6; k++)
            u[k] = (k == 1 || k == 3) ? __dmul_rn(w.v[k], pz) : w.v[k];
          u[6] = w.id;
          if (grp == 0)
            pair_sums<0, false, false>(S, E, u, u, mn);
          else
            pair_sums<1, false, false>(S, E, u, u, mn);
        }
      }
    }
    /* this warp is done with the stage; the issuing thread refills it once
     * every warp is */
    __syncwarp();
    if (lane == 0)
      mbar_arrive(&r.empty[stage]);
    if (threadIdx.x == 0 && !r.fail) {
      /* the tile SUM_STAGES ahead of this one goes into this stage */
      TilePos ps = cs;
      for (int k = 0; k < SUM_STAGES; k++)
        ts.next<TILE>(ps);
      if (!ts.done(ps)) {
        if (mbar_wait(&r.empty[stage], parity, &r.fail)) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          issue_tile<TILE>(r, smem, L, stage, ps.chunk, ps.tile, b, s, chunk_n);
          issued++;
        } else {
          r.fail = 1;
        }
      }
    }
    if (cs.tile == cs.ntiles - 1) {
      /* the chunk is complete: its sums (value i at out[i nchunks]) */
      double *out = part + chunk;
      if constexpr (PASS == 1) {
        block_dd_totals<NV, NP, WARPS, 1>(S, E, red, out, nchunks);
      } else if constexpr (!(F & SF_PZ)) {
#pragma unroll
        for (int k = 0; k < 14; k++)
          S[k] = __dsub_rn(S[k], sm_bias[14 * grp + k]);
        block_dd_totals<NV, NP, WARPS, 2>(S, E, red, out, nchunks);
      } else {
        block_dd_totals<NV, NP, WARPS, 2>(S, E, red, out + 56 * nchunks, nchunks);
      }
      reset();
    }
  }
  __syncthreads();
  const bool failed = r.fail != 0;
  if (failed && threadIdx.x == 0) {
    /* copies still in flight land before the block's shared memory is
     * released: wait for the last ones issued, again for a bounded time */
    for (long t = issued > SUM_STAGES ? issued - SUM_STAGES : 0; t < issued; t++)
      mbar_wait(&r.full[t % SUM_STAGES], (unsigned)((t / SUM_STAGES) & 1));
    atomicExch(status, SUM_STATUS_COPY_TIMEOUT);
  }
  /* the block's extremes and counts (value i at blk[i gridDim.x + block]) */
  if (!failed) {
    double *bo = blk + blockIdx.x;
    const long bs = gridDim.x;
    if constexpr (PASS == 1) {
      double X[15], Y[4] = {M[10], M[11], M[12], M[13]};
      with_maxabs<5>(M, X);
      block_count<WARPS>(cnt, redc, bo);
      block_extremes<15, WARPS>(X, 0x1249u, red, bo + bs, bs);
      block_count<WARPS>(alive, redc, bo + 16 * bs);
      block_extremes<4, WARPS>(Y, 0x5u, red, bo + 17 * bs, bs);
    } else if constexpr (!(F & SF_PZ)) {
      double X[6];
      with_maxabs<2>(M, X);
      block_extremes<6, WARPS>(X, 0x9u, red, bo, bs);
    }
  }
}

/* Combine partials: `n_dd` double-double values from the chunk partials
 * `part` (value-major, `nchunks` per value, combined in chunk order) to
 * out[2 v], out[2 v + 1]; then `n_plain` values from `plain` (value-major,
 * `nplain_rows` per value) to out[plain_base + k], value k a minimum when bit
 * k of `min_mask` is set, a maximum when bit k of `max_mask` is set, else a
 * sum.  One block per value: thread t takes rows t, t + COMBINE_THREADS, ...
 * in order (COMBINE_BATCH loads in flight at a time), then the lanes combine
 * in a fixed tree and the warps in index order. */
__global__ void __launch_bounds__(COMBINE_THREADS)
  combine_partials(const double *part, int nchunks, int n_dd, const double *plain, int nplain_rows, int n_plain,
                   int plain_base, unsigned min_mask, unsigned max_mask, double *out) {
  __shared__ double sh[2 * (COMBINE_THREADS / 32)];
  const int v = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (v < n_dd) {
    const double *ph = part + (size_t)(2 * v) * nchunks, *pl = ph + nchunks;
    trkcr_dd acc = trkcr_make(0.0, 0.0);
    for (int c0 = threadIdx.x; c0 < nchunks; c0 += COMBINE_THREADS * COMBINE_BATCH) {
      /* the batch's loads first, all in flight together, then the sums in order */
      double h[COMBINE_BATCH], l[COMBINE_BATCH];
#pragma unroll
      for (int j = 0; j < COMBINE_BATCH; j++) {
        const int c = c0 + j * COMBINE_THREADS;
        h[j] = c < nchunks ? ph[c] : 0.0;
        l[j] = c < nchunks ? pl[c] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < COMBINE_BATCH; j++)
        acc = dd_add(acc, trkcr_make(h[j], l[j]));
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double h = __shfl_down_sync(0xffffffffu, acc.hi, off), l = __shfl_down_sync(0xffffffffu, acc.lo, off);
      acc = dd_add(acc, trkcr_make(h, l));
    }
    if (lane == 0) {
      sh[2 * warp] = acc.hi;
      sh[2 * warp + 1] = acc.lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      trkcr_dd t = trkcr_make(sh[0], sh[1]);
      for (int w = 1; w < COMBINE_THREADS / 32; w++)
        t = dd_add(t, trkcr_make(sh[2 * w], sh[2 * w + 1]));
      out[2 * v] = t.hi;
      out[2 * v + 1] = t.lo;
    }
  } else if (v < n_dd + n_plain) {
    const int k = v - n_dd, q = plain_base + k;
    const int op = ((min_mask >> k) & 1u) ? 1 : (((max_mask >> k) & 1u) ? 2 : 0);
    const double *px = plain + (size_t)k * nplain_rows;
    const double init = op == 0 ? 0.0 : (op == 1 ? OBS_BIG : -OBS_BIG);
    double acc = init;
    for (int c0 = threadIdx.x; c0 < nplain_rows; c0 += COMBINE_THREADS * COMBINE_BATCH) {
      double x[COMBINE_BATCH];
#pragma unroll
      for (int j = 0; j < COMBINE_BATCH; j++) {
        const int c = c0 + j * COMBINE_THREADS;
        x[j] = c < nplain_rows ? px[c] : init;
      }
#pragma unroll
      for (int j = 0; j < COMBINE_BATCH; j++)
        acc = op == 0 ? __dadd_rn(acc, x[j]) : (op == 1 ? fmin(acc, x[j]) : fmax(acc, x[j]));
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double x = __shfl_down_sync(0xffffffffu, acc, off);
      acc = op == 0 ? __dadd_rn(acc, x) : (op == 1 ? fmin(acc, x) : fmax(acc, x));
    }
    if (lane == 0)
      sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = sh[0];
      for (int w = 1; w < COMBINE_THREADS / 32; w++)
        t = op == 0 ? __dadd_rn(t, sh[w]) : (op == 1 ? fmin(t, sh[w]) : fmax(t, sh[w]));
      out[q] = t;
    }
  }
}

/* Sum over survivors of Po (1 + delta) (src/do_tracking.c:3448-3455); one
 * chunk per block, partial = (hi, lo, count), value-major. */
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
    part[blockIdx.x] = t.hi;
    part[gridDim.x + blockIdx.x] = t.lo;
    part[2 * gridDim.x + blockIdx.x] = c.hi;
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

/* blocks of a pass's persistent grid on the context's device */
template <int PASS>
int sums_grid(const Ctx &c, int *grid) {
  int sms = 0;
  OBS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
  const long chunk_n = sum_chunk<PASS>(c.n), nchunks = (c.n + chunk_n - 1) / chunk_n;
  *grid = (int)std::max(1L, std::min<long>(nchunks, (long)sms * sum_blocks_per_sm<PASS>()));
  return TRK_OK;
}

/* one pass of the beam sums into the chunk partials `part` and the block
 * values `blk` over `grid` blocks; `status` is a device int the caller has
 * zeroed */
template <int PASS, int F>
int launch_sums(const Ctx &c, const Select &s, const double *tot1, int sparse, int grid, int *status, double *part,
                double *blk) {
  auto kernel = beam_sums<PASS, F>;
  static int configured[64] = {0}; /* per device: the shared-memory attribute is set */
  if (c.device < 0 || c.device >= 64 || !configured[c.device]) {
    OBS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sum_smem_max<PASS>()));
    if (c.device >= 0 && c.device < 64)
      configured[c.device] = 1;
  }
  const unsigned smem = SUM_STAGES * layout_of<F, sum_tile<PASS>()>(s).stage_bytes;
  kernel<<<grid, sum_threads<PASS>(), smem, c.st>>>(beam_of(c), s, tot1, sparse, status, part, blk);
  OBS_CUDA(cudaGetLastError());
  return TRK_OK;
}

/* chunk partials of a pass over a beam of c.n particles */
template <int PASS>
int blocks_of(const Ctx &c) {
  const long chunk_n = sum_chunk<PASS>(c.n);
  return (int)((c.n + chunk_n - 1) / chunk_n);
}

/* pass 1 on the device: chunk partials and block values, then their
 * combination into tot1; `ctl` (4 ints, the status word last) is zeroed
 * here */
int enqueue_pass1(const Ctx &c, Scratch &sc, const Select &s, int F, double *tot1, int *ctl) {
  const int nb = blocks_of<1>(c);
  int grid, rc;
  if ((rc = sums_grid<1>(c, &grid)))
    return rc;
  double *part, *blk;
  if ((rc = sc.get(&part, (size_t)nb * 18)) || (rc = sc.get(&blk, (size_t)grid * 21)))
    return rc;
  OBS_CUDA(cudaMemsetAsync(ctl, 0, 4 * sizeof(int), c.st));
  switch (F) {
  case 0:
    rc = launch_sums<1, 0>(c, s, nullptr, 0, grid, ctl + 3, part, blk);
    break;
  case SF_TIME:
    rc = launch_sums<1, SF_TIME>(c, s, nullptr, 0, grid, ctl + 3, part, blk);
    break;
  case SF_TIME | SF_ID:
    rc = launch_sums<1, SF_TIME | SF_ID>(c, s, nullptr, 0, grid, ctl + 3, part, blk);
    break;
  case SF_TIME | SF_PZ:
    rc = launch_sums<1, SF_TIME | SF_PZ>(c, s, nullptr, 0, grid, ctl + 3, part, blk);
    break;
  case SF_TIME | SF_ID | SF_PZ:
    rc = launch_sums<1, SF_TIME | SF_ID | SF_PZ>(c, s, nullptr, 0, grid, ctl + 3, part, blk);
    break;
  default:
    return trk_set_error(TRK_ERR_ARG, "beam sums: no pass-1 variant %d", F);
  }
  if (rc)
    return rc;
  combine_partials<<<9 + 21, COMBINE_THREADS, 0, c.st>>>(part, nb, 9, blk, grid, 21, P1_COUNT, P1_MIN_MASK,
                                                          P1_MAX_MASK, tot1);
  OBS_CUDA(cudaGetLastError());
  return TRK_OK;
}

/* the status word of the passes, after the stream has been synchronized */
int sums_status(int status) {
  if (status == SUM_STATUS_COPY_TIMEOUT)
    return trk_set_error(TRK_ERR_CUDA, "beam sums: a staged copy of the beam did not complete");
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
  s.pid_window = 0;
  s.time = nullptr;
  s.time_out = nullptr;
  /* results: pass 1's totals, then the control words, copied back at once */
  Scratch sc(c.ctx, 1);
  double *res, *h;
  if ((rc = sc.get(&res, P1 + 2)) || (rc = trk_context_host_scratch(c.ctx, sizeof(double) * (P1 + 2), (void **)&h)))
    return rc;
  if ((rc = enqueue_pass1(c, sc, s, 0, res, (int *)(res + P1))))
    return rc;
  OBS_CUDA(cudaMemcpyAsync(h, res, sizeof(double) * (P1 + 2), cudaMemcpyDeviceToHost, c.st));
  OBS_CUDA(cudaStreamSynchronize(c.st));
  if ((rc = sums_status(((const int *)(h + P1))[3])))
    return rc;
  const double count = h[18];
  if (count > 0)
    for (int k = 0; k < 6; k++)
      centroid[k] = (h[2 * k] + h[2 * k + 1]) / count;
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
  double np_count = 0;
  if (c.n > 0) {
    Scratch sc(c.ctx, 2);
    Select s;
    s.Po = p_central;
    s.tmin = t_min;
    s.tmax = t_max;
    s.start_pid = start_pid;
    s.end_pid = end_pid;
    s.pid_window = start_pid >= 0 || end_pid >= 0;
    s.time = nullptr;
    s.time_out = nullptr;
    if (time_value) {
      /* the caller's time coordinates, one per loaded particle */
      double *d_time;
      if ((rc = sc.get(&d_time, (size_t)(c.n + 31) / 32 * 32)))
        return rc;
      OBS_CUDA(cudaMemcpyAsync(d_time, time_value, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.st));
      s.time = d_time;
    }
    /* pass 1 keeps the time coordinates it computes for pass 2 */
    Select s2 = s;
    if (second && !s.time) {
      double *d_t;
      if ((rc = sc.get(&d_t, (size_t)(c.n + 31) / 32 * 32)))
        return rc;
      s.time_out = d_t;
      s2.time = d_t;
    }
    /* the whole computation is queued on the device: pass 2 forms the
     * centroids from pass 1's totals itself, and the host waits once */
    const int id = s.pid_window ? SF_ID : 0;
    /* results: pass 1's totals, pass 2's, the control words; one copy back */
    double *res, *hres;
    if ((rc = sc.get(&res, P1 + P2 + 2)) ||
        (rc = trk_context_host_scratch(c.ctx, sizeof(double) * (P1 + P2 + 2), (void **)&hres)))
      return rc;
    double *tot1 = res, *tot2 = res + P1;
    int *ctl = (int *)(res + P1 + P2);
    if ((rc = enqueue_pass1(c, sc, s, SF_TIME | id | (pz_mode ? SF_PZ : 0), tot1, ctl)))
      return rc;
    const double *h1 = hres, *h = hres + P1;
    if (second) {
      const int nb = blocks_of<2>(c);
      int grid;
      if ((rc = sums_grid<2>(c, &grid)))
        return rc;
      double *part, *blk;
      if ((rc = sc.get(&part, (size_t)nb * 112)) || (rc = sc.get(&blk, (size_t)grid * 6)))
        return rc;
      const int sparse = (flags & TRK_SUMS_SPARSE) ? 1 : 0;
      if (id)
        rc = launch_sums<2, SF_TIME | SF_ID>(c, s2, tot1, sparse, grid, ctl + 3, part, blk);
      else
        rc = launch_sums<2, SF_TIME>(c, s2, tot1, sparse, grid, ctl + 3, part, blk);
      if (!rc && pz_mode)
        rc = launch_sums<2, SF_TIME | SF_ID | SF_PZ>(c, s2, tot1, sparse, grid, ctl + 3, part, blk);
      if (rc)
        return rc;
      /* sigma, and sigman when asked for; the s and t extremes */
      const int n_dd = pz_mode ? 56 : 28;
      combine_partials<<<n_dd + 6, COMBINE_THREADS, 0, c.st>>>(part, nb, n_dd, blk, grid, 6, 112, P2_MIN_MASK,
                                                                P2_MAX_MASK, tot2);
      OBS_CUDA(cudaGetLastError());
    }
    OBS_CUDA(cudaMemcpyAsync(hres, res, sizeof(double) * (P1 + P2 + 2), cudaMemcpyDeviceToHost, c.st));
    OBS_CUDA(cudaStreamSynchronize(c.st));
    if ((rc = sums_status(((const int *)(hres + P1 + P2))[3])))
      return rc;
    /* nothing is accumulated without survivors (src/compute_centroids.c:313) */
    if (h1[34] > 0) {
      double sum[9], mm[15];
      for (int k = 0; k < 9; k++)
        sum[k] = h1[2 * k] + h1[2 * k + 1];
      np_count = h1[18];
      for (int k = 0; k < 15; k++)
        mm[k] = h1[19 + k];
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
      if (np_count > 0)
        for (int i = 0; i < 7; i++)
          sums->centroid[i] = (sums->centroid[i] * sums->n_part + sum[i]) / (sums->n_part + np_count);
      if (second) {
        if (!(flags & TRK_SUMS_NOMINMAX) && np_count > 0) {
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
  if ((rc = sc.get(&part, (size_t)nb * 3)) || (rc = sc.get(&out, 3)))
    return rc;
  momentum_sum<<<nb, OBS_THREADS, 0, c.st>>>(beam_of(c), Po, part);
  combine_partials<<<2, COMBINE_THREADS, 0, c.st>>>(part, nb, 1, part + 2 * nb, nb, 1, 2, 0u, 0u, out);
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

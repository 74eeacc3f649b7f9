/*
 * trk_noalloc.cu -- the WAKE kick on a caller-owned device beam without any
 * device allocation (trk_wake_noalloc, declared in include/trk.h).
 *
 * Some callers cannot allocate device memory at the point where they track:
 * an application whose device memory is handed out entirely by its own pool
 * allocator (a framework's caching allocator, an MPI code with a fixed
 * budget), or a latency-sensitive pipeline that cannot afford cudaMalloc /
 * cudaFree, which may synchronize the whole device.  For them this entry
 * point keeps all of its scratch (histogram, convolved voltage, block
 * partials, wake state, status word) in one file-scope static __device__
 * array of TRK_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library
 * holds until the process exits.  The caller still passes the beam and the
 * wake table.
 *
 * In host code the array's name only stands for the symbol; its device
 * address is looked up with cudaGetSymbolAddress once per device (the first
 * call on each device does this, with that device current), and the kernels
 * get that address.  All calls share the one array and it keeps the last
 * call's contents: each call clears the parts that must start at zero, and
 * calls that overlap on the GPU (different streams, or different host
 * threads on the same device) race on it.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>

#include "trk.h"
#include "trk_kernels.h"
#include "trk_lattice.h"

namespace {

constexpr long kMaxBins = TRK_NOALLOC_MAX_BINS;
constexpr int kMaxBlocks = TRK_NOALLOC_MAX_BLOCKS;
constexpr long kChunk = 4096;

/* byte offsets inside the scratch array (256-byte aligned sections) */
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kOffCounts = 0;
constexpr size_t kOffV = align256(kOffCounts + sizeof(unsigned long long) * (kMaxBins + 2));
constexpr size_t kOffState = align256(kOffV + sizeof(double) * (kMaxBins + 2));
constexpr size_t kOffStats = align256(kOffState + sizeof(WakeState));
/* time statistics: sum, count, min, max, sum_hi, sum_lo (time_stats_finish_kernel) */
constexpr size_t kOffPart = align256(kOffStats + sizeof(double) * 6);
constexpr size_t kOffPartN = align256(kOffPart + sizeof(double) * 4 * kMaxBlocks);
constexpr size_t kOffStatus = align256(kOffPartN + sizeof(long long) * kMaxBlocks);
constexpr size_t kBytes = align256(kOffStatus + sizeof(int));
static_assert(kBytes <= TRK_NOALLOC_SCRATCH_BYTES, "scratch sections exceed the declared size");

} // namespace

static __device__ __align__(256) unsigned char trk_noalloc_scratch[TRK_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch[kMaxDevices];
int g_sm_count[kMaxDevices];
std::atomic<bool> g_ready[kMaxDevices];

/* Once per device, with that device current: the device address of the
 * scratch array and the SM count. */
int device_setup(int dev, unsigned char **scratch, int *sms) {
  if (dev < 0 || dev >= kMaxDevices)
    return trk_set_error(TRK_ERR_ARG, "device %d outside the supported range for trk_wake_noalloc", dev);
  if (!g_ready[dev].load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_ready[dev].load(std::memory_order_relaxed)) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, trk_noalloc_scratch);
      if (e != cudaSuccess)
        return trk_set_error(TRK_ERR_CUDA, "cudaGetSymbolAddress of the wake scratch failed on device %d: %s", dev,
                             cudaGetErrorString(e));
      int sm = 0;
      e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess)
        return trk_set_error(TRK_ERR_CUDA, "SM count query failed: %s", cudaGetErrorString(e));
      g_scratch[dev] = (unsigned char *)p;
      g_sm_count[dev] = sm;
      g_ready[dev].store(true, std::memory_order_release);
    }
  }
  *scratch = g_scratch[dev];
  *sms = g_sm_count[dev];
  return TRK_OK;
}

} // namespace

extern "C" int trk_wake_noalloc(double *const *columns, int32_t *lost_pass, int32_t *lost_element, long np,
                                double p_central, const double *wake_W, long wake_points, double wake_dt,
                                long n_bins, double macro_charge, double factor, int interpolate,
                                int allow_long_beam, long pass, int fast_math, void *stream) {
  if (!columns || np < 0 || (np > 0 && (!lost_pass || !lost_element)) || !wake_W)
    return trk_set_error(TRK_ERR_ARG, "trk_wake_noalloc: null beam, loss or wake pointer");
  for (int c = 0; c < 6; c++)
    if (np > 0 && !columns[c])
      return trk_set_error(TRK_ERR_ARG, "trk_wake_noalloc: column %d is null", c);
  if (!(p_central > 0))
    return trk_set_error(TRK_ERR_ARG, "trk_wake_noalloc: p_central must be positive");
  if (wake_points < 2 || !(wake_dt > 0))
    return trk_set_error(TRK_ERR_PHYSICS, "trk_wake_noalloc: wake table needs >= 2 points and a positive spacing");
  if (n_bins < 2 || n_bins > kMaxBins)
    return trk_set_error(TRK_ERR_ARG,
                         "trk_wake_noalloc: n_bins=%ld outside [2, %ld], the size of its static histogram; use "
                         "trk_track for larger histograms",
                         n_bins, kMaxBins);
  if (np == 0)
    return TRK_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  unsigned char *base = nullptr;
  int sms = 0;
  int rc = device_setup(dev, &base, &sms);
  if (rc)
    return rc;
  cudaStream_t st = (cudaStream_t)stream;
  /* the time-statistics reduction takes the block count trk_track takes
   * (one block per 4096 particles, at most 8 per SM), capped at the static
   * partials' size: on a GPU with more than 148 SMs a large beam then uses
   * fewer blocks than trk_track, and its mean time may differ in the last
   * bit */
  const int blocks =
    (int)std::max(1L, std::min(std::min((np + kChunk - 1) / kChunk, (long)sms * 8), (long)kMaxBlocks));
  unsigned long long *counts = (unsigned long long *)(base + kOffCounts);
  double *V = (double *)(base + kOffV);
  WakeState *state = (WakeState *)(base + kOffState);
  double *stats = (double *)(base + kOffStats);
  double *part = (double *)(base + kOffPart);
  long long *part_n = (long long *)(base + kOffPartN);
  int *status = (int *)(base + kOffStatus);

  /* the array keeps the previous call's contents: clear what starts at zero */
  if ((e = cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * (n_bins + 2), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(status, 0, sizeof(int), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(state, 0, sizeof(WakeState), st)) != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "trk_wake_noalloc: clearing scratch failed: %s", cudaGetErrorString(e));

  TimeStatsArgs t;
  std::memset(&t, 0, sizeof(t));
  t.s = columns[4];
  t.dp = columns[5];
  t.lost_pass = lost_pass;
  t.n = np;
  t.chunk = kChunk;
  t.mode = 0;
  t.Po = p_central;
  t.part_hi = part;
  t.part_lo = part + blocks;
  t.part_min = part + 2 * blocks;
  t.part_max = part + 3 * blocks;
  t.part_n = part_n;
  t.out = stats;

  WakeArgs a;
  std::memset(&a, 0, sizeof(a));
  a.x = columns[0];
  a.xp = columns[1];
  a.y = columns[2];
  a.yp = columns[3];
  a.s = columns[4];
  a.dp = columns[5];
  a.lost_pass = lost_pass;
  a.lost_elem = lost_element;
  a.n = np;
  a.Po = p_central;
  a.stats = stats;
  a.state = state;
  a.status = status;
  a.dt = wake_dt;
  a.wake_span = wake_dt * (wake_points - 1);
  a.wake_points = wake_points;
  a.i0 = 0;
  a.n_bins = n_bins;
  a.max_bins = n_bins;
  a.smem_bins = 12288;
  a.allow_long_beam = allow_long_beam;
  a.pass = pass;
  a.ramp_passes = 0;
  a.macro_mode = 0;
  a.macro_charge = macro_charge;
  a.factor = factor;
  a.xfactor = a.yfactor = 1;
  a.interpolate = interpolate;
  a.transverse = 0;
  a.W = wake_W;
  a.W_y = wake_W;
  a.counts = counts;
  a.hist_x = a.hist_y = V;
  a.V = V;
  a.V_y = V;
  a.aps = nullptr;
  a.ap_post = -1;
  a.z_end = 0;
  a.elem = -1;
  long g = (np + TRK_BLOCK - 1) / TRK_BLOCK;
  const int grid = (int)std::min(g, (long)sms * 64);
  if (fast_math) {
    trk_fast::launch_time_stats(t, blocks, st);
    trk_fast::launch_wake(a, grid, st);
  } else {
    trk_exact::launch_time_stats(t, blocks, st);
    trk_exact::launch_wake(a, grid, st);
  }
  if ((e = cudaGetLastError()) != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "trk_wake_noalloc launch failed: %s", cudaGetErrorString(e));
  int h_status = 0;
  if ((e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return trk_set_error(TRK_ERR_CUDA, "trk_wake_noalloc: status read failed: %s", cudaGetErrorString(e));
  if (h_status & TRK_STATUS_LONG_BEAM)
    return trk_set_error(TRK_ERR_PHYSICS, "The beam is longer than the longitudinal wake function.");
  if (h_status)
    return trk_set_error(TRK_ERR_DEVICE, "trk_wake_noalloc: device status 0x%x", h_status);
  return TRK_OK;
}

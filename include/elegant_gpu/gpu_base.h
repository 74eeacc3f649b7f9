/*
 * gpu_base.h -- the GPU hooks elegant's sources call when built with
 * -DHAVE_GPU (src/do_tracking.c:23, src/csbend.c:19-22, src/trwake.c:18-21),
 * implemented over libtrkgpu.so by elegant_b200/hooks/trk_elegant_hooks.c.
 * Include after elegant's track.h.  The reference does not ship these
 * headers; the signatures are those its call sites use.
 */
#ifndef TRK_ELEGANT_GPU_BASE_H
#define TRK_ELEGANT_GPU_BASE_H

#ifdef __cplusplus
extern "C" {
#endif

/* what do_tracking reads back (src/do_tracking.c:928-931, :3177) */
typedef struct {
  long elementOnGpu; /* the current element runs on the GPU */
  double **coord;    /* host rows, valid after forceParticlesToCpu */
  long nOriginal;    /* particles handed to gpuBaseInit */
  long nLeft;        /* survivors after the last hook */
} GPUBASE;

/* device beam from host rows (src/do_tracking.c:413) */
void gpuBaseInit(double **coord, long nOriginal, double **accepted, double **lostParticles, long isMaster);
/* release the device beam (src/do_tracking.c:3178) */
void gpuBaseDealloc(void);
/* decide whether eptr runs on the GPU (src/do_tracking.c:925) */
void setElementGpuData(void *eptr);
long getElementOnGpu(void);
GPUBASE *getGpuBase(void);
/* device -> host rows, survivors first; column lossPassIndex holds the
 * pass of loss (-1 survivors) (src/do_tracking.c:525 and 12 more sites) */
double **forceParticlesToCpu(const char *reason);
void startGpuTimer(void);
void startCpuTimer(void);
void compareGpuCpu(long n_part, const char *name);

/* Not in the reference: the pass the hooks record losses with.  The hooks
 * count passes themselves (setElementGpuData starts the next pass when the
 * line's first element comes round again), starting at the pass given here
 * before a run (0 when never called); a caller that drives its own pass
 * loop may call it at the start of every pass instead. */
void trk_hooks_begin_pass(long i_pass);
/* loss element index (position in the pass, from setElementGpuData) of each
 * row returned by the last forceParticlesToCpu; -1 for survivors */
const long *trk_hooks_loss_elements(void);

#ifdef __cplusplus
}
#endif
#endif

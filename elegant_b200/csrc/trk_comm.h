/*
 * trk_comm.h -- the cross-GPU exchanges of the tracking path over NCCL.
 *
 * Particles are sharded across ranks (one process per GPU); the only
 * collective steps of a pass are those of Pelegant's MPI build, restated on
 * device buffers and ordered on the context's stream:
 *  - beam time statistics for WAKE/TRWAKE and the first-pass RF fiducial
 *    (src/wake.c:118-130 find_global_min_max, src/simple_rfca.c:222-230
 *    KahanParallel): every rank's {sum (double-double), count, min, max} is
 *    all-gathered and combined in rank order, so all ranks hold the same,
 *    partition-independent values;
 *  - the wake histograms (src/wake.c:226-233, src/trwake.c:195-204
 *    MPI_Allreduce SUM): integer counts for WAKE, FP64 sums for TRWAKE;
 *  - the particle count behind the CHARGE element's macroparticle charge
 *    (src/do_tracking.c:1378-1381 total_nOriginal).
 * NCCL is loaded at run time (dlopen), so single-GPU use never needs it.
 */
#ifndef TRK_COMM_H
#define TRK_COMM_H

#include <cuda_runtime.h>
#include <stddef.h>

#include "trk.h"

struct trk_comm;

/* 0 on success; message in trk_last_error() otherwise */
int trk_comm_create(trk_comm **out, const void *unique_id, int nranks, int rank, int device);
/* a communicator over the caller's host-side collectives (trk_exchange in
 * trk.h): device buffers are staged through host memory around each call */
int trk_comm_create_exchange(trk_comm **out, const trk_exchange *ex, int nranks, int rank);
void trk_comm_destroy(trk_comm *c);
int trk_comm_rank(const trk_comm *c);
int trk_comm_size(const trk_comm *c);
/* in-place sums on the stream: doubles / unsigned 64-bit integers / signed 64-bit */
int trk_comm_sum_f64(trk_comm *c, double *buf, size_t n, cudaStream_t st);
int trk_comm_sum_u64(trk_comm *c, unsigned long long *buf, size_t n, cudaStream_t st);
int trk_comm_sum_i64(trk_comm *c, long long *buf, size_t n, cudaStream_t st);
/* all-gather n doubles from every rank into recv[rank * n ...] */
int trk_comm_gather_f64(trk_comm *c, const double *send, double *recv, size_t n, cudaStream_t st);
/* NCCL unique id (128 bytes) for trk_context_set_comm */
int trk_comm_unique_id(void *out128);

#endif

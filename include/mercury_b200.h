/* Extensions of the B200 test-particle library beside the drop-in ABI of
 * mercury_cuda.h. They have no counterpart in the reference's C ABI; the
 * reference host reaches the same work one step at a time through
 * mercury_cuda_step + mercury_cuda_events. */
#ifndef MERCURY_B200_H
#define MERCURY_B200_H
#include "mercury_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Advance the uploaded MVS system (algorithm 1 or 9) by nsteps steps of h
 * from `time`, with the close-encounter screen (mce_stat) and the central-body
 * screen (mce_cent, radius rcen) of every step, as mal_hcon would call
 * mercury_cuda_step + mercury_cuda_events nsteps times. Steps are fused
 * steps_per_launch at a time (0 = automatic). *nevents receives the number of
 * event records, fetched with mercury_b200_events. */
int mercury_b200_mvs_advance(double time, double h, int nsteps, double rcen, int steps_per_launch, int* nevents);
/* Copy up to cap records of the last advance, sorted by (step, min(i,j),
 * max(i,j)), with the 0-based step of each; returns the total count. */
int mercury_b200_events(MercuryEvent* events, int* steps, int cap);
/* Device time of the last advance (CUDA events on the library's stream),
 * and the summed duration and count of its particle-kernel launches. */
int mercury_b200_timing(double* advance_ms, double* particle_kernel_ms, int* particle_launches);
/* Launch shape of the particle kernel: threads per CTA (multiple of 32) and
 * steps fused per launch (0 = automatic); a negative value keeps the setting. */
int mercury_b200_set_launch(int particle_threads, int steps_per_launch);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (2 FLOP per
 * FMA), best of five launches of independent fma() chains on every SM. */
int mercury_b200_fp64_peak(double* tflops, double* ms);

#ifdef __cplusplus
}
#endif
#endif

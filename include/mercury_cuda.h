/* Drop-in C ABI of the B200 test-particle library.
 *
 * These are exactly the entry points that MERCURY6's Fortran host binds with
 * ISO_C_BINDING (mercury_gpu.f90:14-86) and that the reference declares in
 * mercury_cuda.h:12-34; libmercury_cuda.so exports them with the same names,
 * argument meanings, 0/nonzero status convention and one "MERCURY CUDA: ..."
 * line on stderr per failure. Host arrays keep the Fortran layout: x(3,n)
 * interleaved per body, ngf(5,n) = A1, A2, A3, beta, yar; index 1 (C index 0)
 * is the central body; masses are in K2 units.
 *
 * The library is single-threaded and owns one global device context, as the
 * reference does (mercury_cuda.cu:16-33). */
#ifndef MERCURY_CUDA_H
#define MERCURY_CUDA_H
#include <stdint.h>

/* One encounter or impact record (reference mercury_cuda.h:7-11). Ids are
 * 1-based. kind bits: 1 close-encounter minimum, 2 near miss, 4 collision,
 * 8 impact on the central body. For bit 1 the states xi/xj are linearly
 * interpolated to the time of minimum separation. 128 bytes. */
typedef struct MercuryEvent {
    int i, j, kind, now;
    double distance, time;
    double xi[6], xj[6];
} MercuryEvent;

#ifdef __cplusplus
extern "C" {
#endif

/* 1 if a CUDA device is usable (reference mercury_cuda.cu:360-362). */
int mercury_cuda_available(void);
/* Select the integrator: 1 MVS, 2 BS, 3 BS2, 4 RADAU, 9 TEST (MVS map), 10 HYBRID
 * (reference mercury_cuda.cu:371-378). Changing algorithm frees device state. */
int mercury_cuda_configure(int algorithm);
/* dtflag handshake of mal_hcon/mal_hvar: any value but 2 discards the cached
 * force/predictor history before the next step (reference mercury_cuda.cu:379). */
void mercury_cuda_reset(int flag);
/* Replace the close-encounter radii rce(n) without touching history
 * (reference mercury_cuda.cu:607-612, mercury_gpu.f90:88-92). */
int mercury_cuda_limits(const double* rce);
/* Copy the current state out; physical=1 applies the MVS output corrector
 * (mco_mvs2h) or the HYBRID physical-velocity map (reference mercury_cuda.cu:503-517). */
int mercury_cuda_export(double h, int physical, double* x, double* v);
/* Upload n bodies, nbig of them Big (central body included); pn enables solar
 * 1PN, ngflag as derived by mio_in (reference mercury_cuda.cu:380-409). */
int mercury_cuda_upload(int n, int nbig, int pn, int ngflag, const double* m, const double* x,
                        const double* v, const double* ngf, const double* jcen, const double* rce,
                        const double* rphys);
/* Advance one step from `time`. Fixed-step methods set *hdid = *h; adaptive
 * ones return the step done and the next trial step (reference mercury_cuda.cu:410-469). */
int mercury_cuda_step(double time, double* h, double* hdid, double tol, int64_t* forces,
                      int64_t* rejected);
/* Copy the state after (previous=0) or before (previous=1) the last step
 * (reference mercury_cuda.cu:466-469, mercury_gpu.f90:180-185,202-205). */
int mercury_cuda_download(double* x, double* v, int previous);
/* Encounter, collision and central-impact records of the last step, sorted by
 * (min(i,j), max(i,j)); *events stays valid until the next events or
 * hybrid_begin call (reference mercury_cuda.cu:470-493). */
int mercury_cuda_events(double time, double h, double rcen, const MercuryEvent** events, int* count);
/* Heliocentric accelerations of mfo_all on the current state, Fortran layout
 * (reference mercury_cuda.cu:494-501). */
int mercury_cuda_force(double* a);
/* HYBRID first half (reference mercury_cuda.cu:519-559): kick, solar drift,
 * Kepler drift, mce_snif pair list; encounter members get their pre-drift state. */
int mercury_cuda_hybrid_begin(double h, const double* crit, int flag, int cap, int* ce, int* nce,
                              int* pi, int* pj, double* x, double* v, int64_t* forces);
/* HYBRID second half (reference mercury_cuda.cu:560-576). */
int mercury_cuda_hybrid_finish(double h, const double* m, const double* x, const double* v,
                               int64_t* forces);
/* Compact BS2 sub-context for an encounter subsystem (reference mercury_cuda.cu:577-597). */
int mercury_cuda_encounter_enter(int n, int nb, const double* m, const double* x, const double* v,
                                 const double* crit, const double* rce, const double* rphys, int np,
                                 const int* pi, const int* pj);
int mercury_cuda_encounter_update(const double* m, const double* x, const double* v);
void mercury_cuda_encounter_exit(void);
/* Release every device allocation (reference mercury_cuda.cu:363-370). */
void mercury_cuda_free(void);

#ifdef __cplusplus
}
#endif
#endif

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
/* Upload, advance and download in one call: the same results as
 * mercury_cuda_upload(n, nbig, pn, ngflag, m, xx, vv, ng, jcen, limits, radii),
 * mercury_b200_mvs_advance(time, h, nsteps, rcen, steps_per_launch, nevents)
 * and mercury_cuda_download(xout, vout, 0). When the run is one launch and
 * every host array is page-locked, the particles are copied in and out in
 * chunks while other chunks are stepped; the system stays uploaded in its end
 * state and the records are fetched with mercury_b200_events. */
int mercury_b200_mvs_run(int n, int nbig, int pn, int ngflag, const double* m, const double* xx, const double* vv,
                         const double* ng, const double* jcen, const double* limits, const double* radii,
                         double time, double h, int nsteps, double rcen, int steps_per_launch, double* xout,
                         double* vout, int* nevents);
/* Copy up to cap records of the last advance, sorted by (step, min(i,j),
 * max(i,j)), with the 0-based step of each; returns the total count. */
int mercury_b200_events(MercuryEvent* events, int* steps, int cap);
/* Device time of the last advance (CUDA events on the library's stream), the
 * summed duration and count of its particle-kernel launches, and the number
 * of kernels it launched on all streams. */
int mercury_b200_timing(double* advance_ms, double* particle_kernel_ms, int* particle_launches,
                        int* kernel_launches);
/* The launches of the last mercury_b200_mvs_advance: up to cap of their step
 * counts and particle-kernel times (ms, CUDA events); returns their number. */
int mercury_b200_advance_launches(int* steps, double* kernel_ms, int cap);
/* Device time (CUDA events on the library's streams) spent in the drop-in
 * mercury_cuda_step, mercury_cuda_events and mercury_cuda_hybrid_begin/_finish
 * calls of the resident system and the encounter subsystem, and the number of
 * kernels they launched, since the last call with reset != 0 (which zeroes
 * both). No counterpart in the reference. */
int mercury_b200_dropin_time(double* ms, int64_t* launches, int reset);
/* Energy and angular momentum of the resident system: mxx_en
 * (mercury6_2.for:7226-7315, barycentric through mco_h2b, 2348-2405) applied
 * to the heliocentric state that mercury_cuda_export(h, physical, ...) would
 * return, computed on the device with the same statement order as the
 * Fortran, so that e and l2 equal a CPU mxx_en on the exported arrays bit for
 * bit. spin is the (3, n) array of spin angular momenta (Fortran s(3,nbod)),
 * or NULL for none; *e receives the energy, *l2 the angular momentum's
 * magnitude. The reference host calls mxx_en itself after downloading every
 * body (mercury6_2.for:919-920); this reads back two numbers instead. */
int mercury_b200_energy(double h, int physical, const double* spin, double* e, double* l2);
/* mxx_ejec's test (mercury6_2.for:7050-7085) on the device state: *count
 * receives the number of bodies j >= i0 (1-based; i0 <= 0 means 2, as in
 * mxx_ejec) whose heliocentric distance exceeds rmax, and ids[0 .. cap) the
 * first cap of their 1-based ids in ascending order. Positions are those
 * mercury_cuda_export(h, physical, ...) would return (mal_hcon tests MVS on
 * its map variables, mco_iden, i.e. physical = 0). The state is not changed:
 * the host flags and removes the bodies (mxx_elim) and uploads again. The
 * reference host downloads every body at the nfun cadence for this test
 * (mercury6_2.for:929-948); this reads back the ids only. */
int mercury_b200_ejections(double h, int physical, double rmax, int i0, int* ids, int cap, int* count);
/* mio_ce's close-encounter records (mercury6_2.for:5456-5510) encoded on the
 * device: for each record of events[0 .. n) with kind bit 1 (a close
 * encounter, as gpu_find_events selects them), in order, the 70-character
 * record body c(1:70) that mio_ce writes after char(12)//'6b' (base-224
 * fields from mio_fl2c, mio_re2c and mco_x2ov: time, ids, distance, then each
 * body's log-distance, angles, velocity ratio and velocity angles), into
 * lines + 70 k. mcen is the central mass m(1) in K2 units, rcen and rmax the
 * run's radii. *count receives the number of lines. The reference host
 * encodes every record itself; a 4,100-record burst (tests/test_events.py)
 * is one launch here. */
int mercury_b200_encode_ce(const MercuryEvent* events, int n, double mcen, double rcen, double rmax, char* lines,
                           int* count);
/* Between mercury_cuda_hybrid_begin and _finish: replace the set of bodies
 * (0-based indices 1 .. n-1 of the resident system) whose rows
 * mercury_cuda_hybrid_finish takes from its x, v arrays, which otherwise are
 * the members that hybrid_begin's pairs named. A process holding a share of
 * the particles lists the Big bodies that any process found in an encounter
 * (their subsystem end states) besides its own members. */
int mercury_b200_hybrid_members(const int* ids, int count);
/* Between mercury_cuda_hybrid_begin and _finish: the bodies whose rows
 * hybrid_finish takes (ascending 0-based indices, the central body left out:
 * the members that hybrid_begin's pairs named, or the set given to
 * mercury_b200_hybrid_members). Copies up to cap of them into ids and returns
 * their number, or -1 outside a HYBRID step. */
int mercury_b200_hybrid_member_list(int* ids, int cap);
/* mdt_hkce's substep loop (mercury6_2.for:3884-3937) over the active
 * encounter subsystem, inside the library: from local time 0 to h, BS2
 * substeps (mercury_cuda_reset + mercury_cuda_step, dtflag 1 then 2) of
 * length *hrec (clipped to the remainder), each followed by the pair screen
 * of mercury_cuda_events at time + tlocal, with the arithmetic of a host
 * driving these drop-in calls (the same states, records and force calls) but
 * one host round trip per BS2 attempt (its level decision) and no download
 * per substep; the records stay on the device until the run ends, and after
 * a record-buffer overflow the run is redone from its start with larger
 * buffers. With member tangents kept (the HYBRID adjoint) the drop-in calls
 * are made one by one. *hrec receives the last
 * substep length tried (mdt_hkce's hrec), *forces the force calls, *nrecords
 * the number of close-encounter and collision records (central-body records
 * left out; subsystem ids, 1-based), fetched with mercury_b200_events(dst,
 * NULL, cap). Call between mercury_cuda_encounter_enter and
 * mercury_cuda_download / _exit. */
int mercury_b200_encounter_run(double time, double h, double tol, double rcen, double* hrec, int64_t* forces,
                               int* nrecords);
/* mxx_sync's epoch synchronisation (mercury6_2.for:7442-7574) before a run,
 * in two parts. mercury_b200_epoch_order (host only) gives its order of the
 * nsml Small bodies: sorted by epoch with mxx_sort's Shell sort, reversed when
 * the last is further from tstart than the first; order[k] is the 0-based
 * Small body at position k. The host uploads the system in that order
 * (configure(2), mdt_bs1), the Big bodies at their common epoch *time, Small
 * body j at epoch[j] (epoch[n], Big entries ignored), and calls
 * mercury_b200_sync_epochs: for each Small body j in order, the bodies before
 * it are advanced by mdt_bs1 steps (clipped to dtout and to j's epoch,
 * mercury_support.f90:202-212) until they reach j's epoch, then j joins. On
 * return every body is at *time, the last epoch; *steps counts the BS steps.
 * Massless Small bodies only. The reference runs this on the host before its
 * GPU backend is selected (mercury6_2.for:158-185). */
int mercury_b200_epoch_order(int nsml, const double* epochs, double tstart, int* order);
int mercury_b200_sync_epochs(const double* epoch, double* time, double h0, double tol, double dtout, int* steps);
/* Adaptive steps (RADAU, BS, BS2) of one system whose massless particles are
 * split across processes, each holding the whole massive set and its own
 * particles: before every step-control decision the library passes its
 * maxima to fn, which must replace each by the maximum over all processes
 * (an all-reduce MAX). RADAU passes one value (max |b7|, +inf after a
 * non-finite force or predictor); BS/BS2 pass 26 (the error maximum of levels
 * 0..12, +inf where non-finite, then 1 or 0 for a failed force at each
 * level). With every process taking the same decisions, each one's particles
 * follow the steps the whole system would take in one process, bit for bit.
 * Applies to the resident system only, never to HYBRID's encounter subsystem.
 * fn = NULL (the default) reduces nothing. No counterpart in the reference,
 * which runs one process. */
typedef void (*mercury_b200_reduce_fn)(double* values, int count, void* user);
int mercury_b200_set_step_reduce(mercury_b200_reduce_fn fn, void* user);
/* Starting capacity of the close-encounter record and candidate buffers of
 * every later upload (cap > 0; 0 restores the default of max(4096, particles
 * / 64) records and max(16384, particles / 2) candidates). The buffers grow
 * after an overflow and the affected step or run is redone, so the results
 * do not depend on it; a small capacity exercises those paths in tests. */
int mercury_b200_set_event_capacity(int cap);
/* Launch shape of the particle kernel: threads per CTA (multiple of 32) and
 * steps fused per launch (0 = automatic); a negative value keeps the setting. */
int mercury_b200_set_launch(int particle_threads, int steps_per_launch);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (2 FLOP per
 * FMA), best of five launches of independent fma() chains on every SM. */
int mercury_b200_fp64_peak(double* tflops, double* ms);

/* ---- Batched systems (no counterpart in the reference, which integrates one
 * system per process). Thousands of independent MVS systems advance together:
 * system s owns bodies [body_offset[s], body_offset[s+1]) of the concatenated
 * host arrays (Fortran layout as in mercury_cuda_upload: m in K2 units, x/v
 * (n,3) rows, rce/rphys per body), its central body first, then nbig[s]-1 Big
 * bodies, then massless Small bodies; h[s] is its step. No non-gravitational
 * forces, no oblateness; nbig[s] <= 32. The upload replaces any previous
 * batch and resets every system's cached acceleration. */
int mercury_b200_batch_upload(int nsys, const int* body_offset, const int* nbig, const double* h,
                              const double* m, const double* x, const double* v, const double* rce,
                              const double* rphys);
/* nsteps MVS steps of every system (mdt_mvs with mce_stat and mce_cent at
 * radius rcen every step; system s's clock runs time, time + h[s], ...).
 * *nevents receives the number of event records, fetched with
 * mercury_b200_batch_events. */
int mercury_b200_batch_advance(double time, int nsteps, double rcen, int* nevents);
/* Copy up to cap records of the last advance, sorted by (system, step,
 * min(i,j), max(i,j)); ids are 1-based within the system; sys/steps (may be
 * null) receive each record's system and 0-based step. Returns the total. */
int mercury_b200_batch_events(MercuryEvent* events, int* sys, int* steps, int cap);
/* Current state of every body into the concatenated host arrays x, v. */
int mercury_b200_batch_download(double* x, double* v);
/* Launch shape: particle CTA size (64, 128 or 256; 0 = tuned), steps per
 * launch (1..64; 0 = tuned), CUDA-graph replay of the chunk loop (1/0); a
 * negative value keeps the setting. Before the first advance after an upload
 * or a change here, the library times short trial runs of every free choice
 * (steps per launch 8, 16, 31, 64 x CTA size 64, 128, 256), rolls the state
 * back, and keeps the fastest per step. */
int mercury_b200_batch_set(int threads, int steps_per_launch, int use_graph);
/* Device time and kernel count of the last advance, and the launch shape it used. */
int mercury_b200_batch_timing(double* ms, int* launches, int* threads, int* steps_per_launch);
void mercury_b200_batch_free(void);

/* ---- Gradients through the MVS test-particle integration (no counterpart in
 * the reference). Massless particles never act on the Big bodies, so each
 * particle's final state depends only on its own initial state and Yarkovsky
 * coefficient; the backward call returns those gradients for a given
 * gradient of the final states.
 *
 * Forward: the Big bodies (host rows: mbig[nbig] in K2 units, xbig/vbig
 * (nbig,3), body 0 the central body) and np massless particles (DEVICE
 * arrays: x0/v0 (np,3) rows, yar[np] or NULL for none) advance nsteps MVS
 * steps of h, exactly as the MVS path steps them; the final states go to the
 * device arrays x_final/v_final (np,3). The state every checkpoint_every
 * steps is kept for the backward call (9 doubles per particle per
 * checkpoint, plus 12 per particle per step of one segment). The device
 * inputs must stay unchanged until the backward call. No oblateness and no
 * non-gravitational term other than yar. */
int mercury_b200_adjoint_forward(int nbig, const double* mbig, const double* xbig, const double* vbig, int np,
                                 const double* x0, const double* v0, const double* yar, double h, int nsteps,
                                 int checkpoint_every, double* x_final, double* v_final);
/* Backward for the last forward run: gx/gv (device (np,3); gv may be NULL)
 * hold dL/dx_final and dL/dv_final; dx0/dv0 (device (np,3)) and dyar
 * (device [np], may be NULL) receive dL/dx0, dL/dv0, dL/dyar. */
int mercury_b200_adjoint_backward(const double* gx, const double* gv, double* dx0, double* dv0, double* dyar);
/* Device time of the last forward and backward calls. */
int mercury_b200_adjoint_timing(double* forward_ms, double* backward_ms);
void mercury_b200_adjoint_free(void);

/* ---- Gradients through the HYBRID test-particle integration (no counterpart
 * in the reference). Massless particles never act on the Big bodies; each
 * particle's final state depends on its own initial state and Yarkovsky
 * coefficient, through mdt_hy's changeover kicks, solar drifts and Kepler
 * drift, and, in the steps where mce_snif makes it an encounter member,
 * through mdt_hkce's BS2 integration of the encounter subsystem.
 *
 * Forward: the Big bodies (host rows: mbig[nbig] in K2 units, xbig/vbig
 * (nbig,3) democratic-heliocentric, i.e. heliocentric positions and
 * barycentric velocities as mercury_cuda_upload receives them for HYBRID,
 * rcrit_big[nbig] changeover radii) and np massless particles (DEVICE arrays
 * x0/v0 (np,3) in the same coordinates, yar[np] or NULL; HOST array
 * rcrit[np]) advance nsteps mdt_hy steps of h with encounter tolerance tol,
 * through the library's own HYBRID path (mercury_cuda_hybrid_begin,
 * encounter_enter/step/download/exit, hybrid_finish: it replaces the resident
 * system, as mercury_cuda_upload does). The final states go to the device
 * arrays x_final/v_final. Kept for the backward call: the particle state every
 * checkpoint_every steps, the Big-body rows of every step and, per encounter
 * member step, the member's end state and the 6x6 Jacobian of its BS2
 * segment (accumulated in forward mode over the accepted substeps; the step
 * control's choices are held fixed). No oblateness and no non-gravitational
 * term other than yar. The device inputs must stay unchanged until the
 * backward call. For massless particles the democratic-heliocentric velocity
 * differs from the heliocentric one by a Big-body term only, so the gradients
 * are the same in either. */
int mercury_b200_hybrid_adjoint_forward(int nbig, const double* mbig, const double* xbig, const double* vbig,
                                        const double* rcrit_big, int np, const double* x0, const double* v0,
                                        const double* yar, const double* rcrit, double h, double tol, int nsteps,
                                        int checkpoint_every, double* x_final, double* v_final);
/* Backward for the last HYBRID forward run: gx/gv (device (np,3); gv may be
 * NULL) hold dL/dx_final and dL/dv_final; dx0/dv0 (device (np,3)) and dyar
 * (device [np], may be NULL) receive dL/dx0, dL/dv0, dL/dyar. */
int mercury_b200_hybrid_adjoint_backward(const double* gx, const double* gv, double* dx0, double* dv0, double* dyar);
/* Wall time of the last forward call (host-driven: encounter subsystems step
 * through the drop-in calls), device time of the last backward call, and the
 * number of (particle, step) encounter-member pairs the forward run recorded. */
int mercury_b200_hybrid_adjoint_timing(double* forward_ms, double* backward_ms, int64_t* member_steps);
void mercury_b200_hybrid_adjoint_free(void);

/* One MVS step (kick, drift, mce_stat pair screen, kick) of a system whose
 * arrays the caller already holds on the current device, with no device
 * allocation: for hosts that cannot call cudaMalloc (device memory owned by
 * another allocator or budget, or no implicit device-wide synchronization
 * allowed). This entry point has no counterpart in the reference's C ABI.
 *
 * Device pointers, SoA with npcap = max(2, np rounded up to even), 16-byte
 * aligned: mbig/rcebig/rphysbig[nbig], ngfbig[nbig][5]; big_in/big_out
 * [9][nbig] and part_in/part_out [9][npcap] holding x,y,z, vx,vy,vz and the
 * cached acceleration ax,ay,az of the last force call; part_const[8][npcap]
 * holding m, rce, rphys, A1, A2, A3, beta, yar. reset != 0 recomputes the
 * cached accelerations first (mdt_mvs with dtflag != 2). events[event_cap]
 * receives the pair records of the step (1-based ids, times absolute), and
 * *event_count (host) their total. No oblateness and no central-impact screen.
 * Limits: nbig <= 64, np <= 262144, event_cap <= 8192, 8192 encounter
 * candidates per step; beyond them the call fails with a message.
 *
 * Scratch lives in one static device array (about 2.2 MB per device, held
 * until exit) that every call shares: calls that overlap on the GPU (other
 * streams, other host threads) race on it. The first call on a device looks
 * up the array's address and fills its slot map with one kernel on `stream`,
 * waiting for that stream; with CUDA's lazy module loading that first call is
 * also when the driver loads this library's device code, and with it the
 * array, so it may allocate: make the first call during set-up, before any
 * stream capture. Each call reads the central mass back from mbig[0] and then
 * waits for `stream` at its end (a cudaStream_t; 0 = legacy default stream);
 * an error already pending from the caller's earlier work makes it fail
 * without clearing that error. */
int mercury_b200_mvs_step_noalloc(int nbig, int np, const double* mbig, const double* rcebig,
                                  const double* rphysbig, const double* ngfbig, const double* big_in,
                                  double* big_out, const double* part_in, double* part_out,
                                  const double* part_const, int ngflag, double time, double h, int reset,
                                  MercuryEvent* events, int event_cap, int* event_count, void* stream);

#ifdef __cplusplus
}
#endif
#endif

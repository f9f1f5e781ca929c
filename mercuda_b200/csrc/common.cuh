// Shared definitions of the B200 test-particle library.
//
// Every translation unit is compiled with --fmad=false and IEEE division and
// square root, so each FP64 statement rounds exactly as the Fortran reference
// (built with -ffp-contract=off) rounds it; the statement order of each routine
// follows the Fortran routine it restates (cited at each function).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mercury_cuda.h"

namespace mb200 {

constexpr double K2 = 2.959122082855911e-4;
constexpr double HUGE_VAL_F = 9.9e29;          // mercury.inc HUGE
constexpr double PI_D = 3.141592653589793;
constexpr double TWOPI_SWIFT = 2.0 * PI_D;     // swift.inc TWOPI
constexpr double DANBYB = 1.0e-13;             // swift.inc DANBYB
// Speed of light in AU/day from the exact SI value and the IAU 2012 au.
constexpr double C_LIGHT = 299792458.0 * 86400.0 / 1.495978707e11;

// Event kinds of the reference ABI (mercury_cuda.h:7-11, mercury_gpu.f90:215-246).
constexpr int EV_CLOSE = 1, EV_NEAR = 2, EV_HIT = 4, EV_CENTRAL = 8;

// Fault bits of the device status word (kernels never trap): a non-finite
// acceleration, an undefined non-gravitational direction (mfo_ngf's fail()),
// coincident bodies (mfo_grav's fail() on a zero separation).
constexpr int FAULT_NONFINITE = 1, FAULT_NGF = 2, FAULT_COINCIDENT = 4;

// Rows of the per-slot particle constants: m, rce, rphys, ngf(5), rcrit.
constexpr int PCONST_ROWS = 9;
constexpr int PC_M = 0, PC_RCE = 1, PC_RPHYS = 2, PC_NGF = 3, PC_RCRIT = 8;

// Device-side status word written by kernels.
struct DeviceStatus {
    int fault;
    int events;        // pair/central events claimed (may exceed capacity)
    int overflow;      // bit 0: an event slot was beyond capacity; bit 1: a candidate slot
    int cands;         // encounter candidates claimed in the current launch
    int next_tile;     // dynamic work counter of the current particle launch
    int pad[3];
};

// A Small body whose padded x-y box overlapped a Big body's box during one
// step (mce_stat's first test): enough to finish mce_stat's test and write the
// record without the particle kernel holding the record path's registers.
struct EncounterCandidate {
    int slot, body, step, id;   // particle slot, Big body index - 1, global step, Fortran id
    double rce, rphys;
    double x0[3], v0[3], x1[3], v1[3];
};

__device__ __forceinline__ void raise_fault(DeviceStatus* st, int bit) { atomicOr(&st->fault, bit); }

// Step control of the HYBRID encounter subsystem held on the device
// (mdt_hkce's substep loop, mercury6_2.for:3884-3937, with mdt_bs2's level
// choice, 3568-3596): the BS2 attempt kernels read the trial step h0 here;
// the post-attempt kernel takes each attempt's decision, advances the local
// clock into the next attempt's copy (two copies alternate), and commits and
// screens only after an acceptance. The host reads it back every few dozen
// attempts.
struct EncCtl {
    double h0;          // trial step of the next attempt
    double hdid;        // step of the last accepted substep
    double tlocal;      // the subsystem's local clock
    double hrec;        // the step before it was clipped to the subsystem's end
    double h;           // the HYBRID step the subsystem runs to
    double tol;
    double time;        // start of the HYBRID step (records' times are time + tlocal)
    long long forces;   // force calls, counted as mdt_bs2 counts them
    int accepted;       // level accepted by the last decision (0: rejected or none)
    int stop;           // 1 once the local clock reached h, or after an error
    int error;          // 0 or an ENC_ERR_* code
    int substeps;       // accepted substeps
    int attempts;
    int step_cap;       // entries of tstep
    double* tstep;      // [step_cap] end time (time + tlocal) of each accepted substep
};
constexpr int ENC_ERR_FORCE = 1, ENC_ERR_NONFINITE = 2, ENC_ERR_ADVANCE = 3, ENC_ERR_STEPS = 4;

}  // namespace mb200

// Adaptive integrators on the device: the heliocentric force mfo_all and the
// RA15 Gauss-Radau step (mdt_ra15), plus the generic encounter screen the
// adaptive integrators use (mce_stat/mce_cent on the states before and after
// a step).
#pragma once
#include "allforce.cuh"
#include "common.cuh"
#include "mvs.cuh"

namespace mb200 {

struct Ra15Args {
    ForceCfg f;
    int np, npcap;
    int niter;        // 6 on a reset sequence, else 2
    int reset;        // dtflag == 1: B and E start from zero
    double t;         // trial sequence length
    // massive set (the "big" arrays), [.][nsplit]
    const double* bx;  // [9][nsplit] x(3) v(3) a(3) of the current buffer; a1 goes to a(3)
    double* bx_a1;     // = bx + 6*nsplit (written: force at the sequence start)
    const double* mbig;
    const double* ngfbig;  // [nsplit][5]
    double* bb;            // [21][nsplit] B (component-major m*3+c)
    double* bg;            // [21][nsplit] G scratch
    double* bpx;           // [6][nsplit] predicted x, v scratch
    // particles
    double* px;            // [9][npcap] current buffer; a(3) receives a1
    const double* pconst;  // [PCONST_ROWS][npcap]
    double* pb;            // [21][npcap] B
    double* table;         // [1 + 7*niter][force_row(nb)]
    unsigned long long* maxb7;  // max |b7| over every coordinate (bit pattern of a non-negative double)
    DeviceStatus* status;
};

struct Ra15CommitArgs {
    int nsplit, np, npcap;
    int reset;
    double tdid, q;
    const double* bx;      // [9][nsplit] current buffer (x1, v1, a1)
    double* bx_out;        // [9][nsplit] other buffer
    double* bb;
    double* be;
    const double* px;      // [9][npcap] current buffer (x1, v1, a1)
    double* px_out;
    double* pb;
    double* pe;
};

void launch_ra15_sequence(const Ra15Args& a, cudaStream_t s);
void launch_ra15_commit(const Ra15CommitArgs& a, cudaStream_t s);

// mfo_all of every body into a[3][n] rows of the caller's layout.
struct ForceAllArgs {
    ForceCfg f;
    int np, npcap;
    const double* bx;      // [9][nsplit]
    const double* mbig;
    const double* ngfbig;
    const double* px;      // [9][npcap]
    const double* pconst;
    double* abig;          // [3][nsplit]
    double* apart;         // [3][npcap]
    double* table;         // [1][force_row(nb)]
    DeviceStatus* status;
};
void launch_force_all(const ForceAllArgs& a, cudaStream_t s);

// Generic encounter screen between the states before (x0,v0) and after
// (x1,v1) a step, for every pair (Big i, j > i): Big/massive pairs by one CTA,
// particle pairs as candidates finished by the classify pass.
struct ScreenArgs {
    int nbig, nsplit, np, npcap;
    double h;
    const double* b0;      // [9][nsplit] previous buffer
    const double* b1;      // [9][nsplit] current buffer
    const double* mbig, *rcebig, *rphysbig;
    const double* p0;      // [9][npcap]
    const double* p1;
    const double* pconst;  // m, rce, rphys, ...
    const int* perm;
    double* boxes;         // [nbig-1][4]
    double* detail;        // [nbig-1][TAB_DETAIL]
    MercuryEvent* events;
    int* event_step;
    int event_cap;
    EncounterCandidate* cands;
    int cand_cap;
    DeviceStatus* status;
    int step;              // event_step of this screen's records
};
void launch_screen(const ScreenArgs& a, cudaStream_t s);

}  // namespace mb200

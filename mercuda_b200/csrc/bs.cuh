// Bulirsch-Stoer steps on the device: mdt_bs1 (modified midpoint, 8 levels,
// mercury6_2.for:3227-3404) and mdt_bs2 (Stoermer form with the start
// velocities, 12 levels, mercury6_2.for:3428-3596), with force = mfo_all.
//
// The Fortran stops at the first level n > 3 whose global error passes; that
// decision needs the maximum over every body. One sequence of launches
// computes every level instead, the levels side by side (they are independent
// given the start-of-step state and force): one massive-set CTA per level
// writes that level's force table rows and raw state, an extrapolation pass
// runs the massive set's Neville updates in level order, and the particle
// kernel gives each warp a balanced pair of levels for 32 particles, then
// extrapolates in level order. Each reduces a per-level error maximum and
// stores the level's extrapolated state. The host then takes the first
// passing level (or halves the step) and a commit pass copies that level's
// state.
#pragma once
#include "allforce.cuh"
#include "common.cuh"

namespace mb200 {

__host__ __device__ constexpr int bs_levels(int variant) { return variant == 1 ? 8 : 12; }
// Force calls of level n (1-based): 2n for mdt_bs1, n for mdt_bs2.
__host__ __device__ constexpr int bs_level_forces(int variant, int n) { return variant == 1 ? 2 * n : n; }
// Table rows: the start-of-step force, then every force call of every level.
__host__ __device__ constexpr int bs_rows(int variant) { return variant == 1 ? 1 + 72 : 1 + 78; }
// Candidate states kept per body: levels 4 .. bs_levels.
__host__ __device__ constexpr int bs_candidates(int variant) { return bs_levels(variant) - 3; }
// Shared-memory rows ([rows][nsplit] doubles) of one level CTA of the massive
// set: eight 3-vectors (states, accelerations, B, C); then 12 more for the
// starting state, masses and non-gravitational constants.
constexpr int BS_LEVEL_ROWS = 24;
// Global scratch of the massive set: the raw level states D(n) [levels][6][nsplit],
// then the private start-of-step table rows of levels 2.. [levels - 1][force_row(nb)].
__host__ __device__ constexpr size_t bs_massive_scratch(int variant, int nsplit, int nb) {
    return (size_t)bs_levels(variant) * 6 * nsplit + (size_t)(bs_levels(variant) - 1) * force_row(nb);
}

struct BsArgs {
    ForceCfg f;
    int variant;                 // 1: mdt_bs1, 2: mdt_bs2
    int np, npcap;
    double h0;                   // trial step
    const double* bx;            // [9][nsplit] start-of-step state of the massive set
    const double* mbig;
    const double* ngfbig;        // [nsplit][5]
    double* draw;                // [levels][6][nsplit] raw level states of the massive set
    double* tscr;                // [levels - 1][force_row(nb)] private start-of-step rows
    const double* px;            // [9][npcap] start-of-step particle state
    const double* pconst;        // [PCONST_ROWS][npcap]
    double* table;               // [bs_rows][force_row(nb)]
    double* bcand;               // [bs_candidates * 6][nsplit]
    double* pcand;               // [bs_candidates * 6][npcap]
    unsigned long long* errs;    // [13] max error of level n (bit pattern of a non-negative double; +inf
                                 // when an extrapolated value is not finite)
    DeviceStatus* lvst;          // [13] force faults of level n (0: the start-of-step force)
    // mfo_hkce instead of mfo_all (the compact encounter subsystem): pairs of
    // body g (0-based subsystem index) are adj[adj_off[g] .. adj_off[g+1]) =
    // {partner, 0 if g is the pair's first body else 1}, in pair-list order.
    // A massless member's pairs all have a Big first body, and massless
    // members add exactly zero to a massive body's sum, so the massive set and
    // the particle slots split as for mfo_all.
    int hkce;
    const double* rcrit;         // [nsplit] massive set; particles use pconst row PC_RCRIT
    const int* adj_off;
    const int2* adj;
    const int* perm;             // slot -> particle index
    int active_np;               // particles with index >= active_np sit the step out (epoch synchronisation)
    const EncCtl* ctl = nullptr; // non-null: the trial step is ctl->h0, nothing runs once ctl->stop
    double* bx_pre = nullptr;    // non-null: [6][nsplit] copy of the massive set's start state (level kernel)
    int fuse_extrap = 0;         // 1: the massive set's extrapolation runs as the particle launch's last CTA
    int stage_bodies = 0;        // set at launch: the particle kernel keeps the table's Big bodies in shared memory
    double* ptab = nullptr;      // mdt_bs2 with mfo_all: [8][6][npcap] the particles' Neville tableau after
                                 // level 8; non-null makes launch_bs_sequence run the particles' levels 1..8
                                 // only (launch_bs_particles_late runs 9..12)
};

struct BsCommitArgs {
    int nsplit, np, npcap;
    int cand;                    // candidate index (accepted level - 4)
    const double* bcand;
    const double* pcand;
    const double* bx;            // start-of-step state (central body row copied)
    double* bx_out;              // [9][nsplit]
    double* px_out;              // [9][npcap]
    const double* px;            // start-of-step particle state (kept by inactive particles)
    const int* perm;             // slot -> particle index
    int active_np;               // as in BsArgs
};

// Everything after one attempt of the encounter subsystem (enc_post_kernel):
// the step decision from this attempt's level maxima and faults, the control
// block of the next attempt with its level maxima cleared, and after an
// acceptance the commit in place and the pair screen of the substep.
struct EncPostArgs {
    const EncCtl* ctl_in;              // the control block this attempt ran with
    EncCtl* ctl_out;                   // the next attempt's
    const unsigned long long* errs;    // [13] this attempt's level maxima
    const DeviceStatus* lvst;          // [13] and force faults
    unsigned long long* errs_next;     // [13] cleared for the next attempt
    DeviceStatus* lvst_next;           // [13]
    int nbig, nsplit, np, npcap, active_np;
    const double* bx_pre;              // [6][nsplit] massive set at the attempt's start
    double* bx;                        // [9][nsplit] massive set, committed in place
    const double* bcand;               // BsArgs::bcand
    const double* pcand;               // BsArgs::pcand
    double* px;                        // [9][npcap] particles, committed in place
    const double* mbig;
    const double* rcebig;
    const double* rphysbig;
    const double* pconst;              // rows 1, 2: rce, rphys of the particle slots
    const int* perm;
    MercuryEvent* events;
    int* event_step;
    int event_cap;
    DeviceStatus* status;
};
void launch_enc_post(const EncPostArgs& a, cudaStream_t s);

void launch_bs_sequence(const BsArgs& a, cudaStream_t s);
// Levels 9..12 of the particles after a launch_bs_sequence with a.ptab set,
// adding to the same level maxima and candidates.
void launch_bs_particles_late(const BsArgs& a, cudaStream_t s);
void launch_bs_commit(const BsCommitArgs& a, cudaStream_t s);
// Tangent of the accepted mdt_bs2 step (levels = accepted level) of the
// encounter subsystem's massless members: tg [36][npcap], entry
// (d * 6 + r) * npcap + slot = d state_r / d (step start)_d, is advanced in
// place from the start-of-step state a.px and the sequence's table a.table.
void launch_bs2_tangent(const BsArgs& a, int levels, double* tg, cudaStream_t s);

}  // namespace mb200

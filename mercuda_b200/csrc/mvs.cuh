// MVS map on the device (mdt_mvs, mercury6_2.for:3987-4101).
//
// The Big bodies never feel the test particles in this map (mfo_mvs,
// mercury6_2.for:5034-5045 is one-way), so their trajectory is integrated by
// one CTA (mvs_big_kernel), which writes for every step a table of what the
// particles need: post-drift Big positions and masses for the kick, each Big
// body's padded x-y box and end states for the encounter screen, and the
// indirect term a0tp. The particle kernel stages those tables in shared memory
// and advances every test particle through K steps in registers.
#pragma once
#include "common.cuh"

namespace mb200 {

// Per-step table, in doubles. The head and per-body force/box rows are staged
// in shared memory by the particle kernel; the per-body detail rows (end
// states, radii) are read from global memory only when a box overlaps.
constexpr int TAB_HEAD = 8;        // a0tp[3], acen[3], pad[2]
constexpr int TAB_BODY = 8;        // x1, y1, z1, m, xmin, xmax, ymin, ymax
constexpr int TAB_DETAIL = 16;     // x0[3], v0[3], x1[3], v1[3], rce, rphys, pad[2]

__host__ __device__ constexpr int tab_stride(int nb) { return TAB_HEAD + TAB_BODY * nb; }

// Device-resident Big-body state, Fortran-style C indices 0..nbig-1 (0 is the
// central body). SoA with stride nbig.
struct BigState {
    double* x;   // [3][nbig]
    double* v;   // [3][nbig]
    double* a;   // [3][nbig] cached total acceleration (angf + a) of the last force call
};

struct MvsBigArgs {
    int nbig;
    // Bodies held by the CTA: 0..nbig-1 Big, nbig..nmass-1 massive Small
    // bodies (MVS with central-body oblateness: they enter the oblateness
    // reaction acen that every body feels, mfo_mvs mercury6_2.for:5061-5068,
    // but move as test particles). nmass <= nbig: Big bodies only.
    int nmass;
    int ngflag;
    int obl;
    int reset;          // recompute the cached acceleration before the first kick
    int nsteps;
    int central;        // screen Big bodies against the central body (fused runs)
    int step0;          // global index of the first step (for event step tags)
    double jcen[3];
    double h;
    double rcen;
    const double* m;    // [nbig]
    const double* rce;  // [nbig]
    const double* rphys;
    const double* ngf;  // [nbig][5]
    BigState in, out;
    double* tab;        // [(nsteps + 1)][tab_stride(nb)], row 0 = start-of-run force table
    double* detail;     // [nsteps][nb][TAB_DETAIL]
    MercuryEvent* events;
    int* event_step;
    int event_cap;
    DeviceStatus* status;
    int* event_sys;     // batched systems: system index of each event record (null otherwise)
    int sys;
};

struct MvsParticleArgs {
    int np;             // number of test particles
    int npcap;          // allocated length of every particle array (even)
    int nb;             // Big bodies (nbig - 1)
    int nbig;           // bodies before the particle slots (event ids: nbig + particle + 1)
    int nsteps;
    int reset;
    int central;
    int step0;
    int ngf_on;         // mfo_ngf terms present
    double mu;          // central mass
    double h;
    double rcen;
    double jcen[3];
    const double* xin;  // [9][npcap]: x y z vx vy vz ax ay az
    double* xout;
    const double* m;    // [npcap]
    const double* rce;
    const double* rphys;
    const double* ngf;  // [5][npcap]
    const int* perm;    // slot -> particle index (ids of event records)
    const double* tab;
    const double* detail;
    MercuryEvent* events;
    int* event_step;
    int event_cap;
    EncounterCandidate* cands;
    int cand_cap;
    DeviceStatus* status;
    int* tiles;         // the launch's work counter, zeroed before it (null: status->next_tile)
    double* rows_x;     // also the end states as host rows (3 per particle, by particle index), or null
    double* rows_v;
};

// Output corrector mco_mvs2h / mco_h2mvs (mercury6_2.for:2107-2227,
// 2420-2535) of the whole state into scratch arrays: two stages of
// drift(ha) kick(-+hb) drift(-2 ha) kick(+-hb) drift(ha), with the Big bodies'
// four force tables written by the Big-body CTA for the particle kernel.
struct CorrectorArgs {
    int np, npcap, nb;
    int ngf_on, obl;
    int forward;          // mco_mvs2h (1) or mco_h2mvs (0)
    double mu;
    double ha[2], hb[2];
    double jcen[3];
    const double* xin;    // [9][npcap] particle state (x, v used)
    double* xout;         // [6][npcap]
    const double* ngf;    // [5][npcap]
    const double* tab;    // [4][tab_stride(nb)] written by the Big-body CTA
    DeviceStatus* status;
};
// big.in: current Big state, big.out: scratch, big.tab: 4 table rows.
void launch_mvs_corrector(const MvsBigArgs& big, const CorrectorArgs& a, cudaStream_t s);

// ------------------------------------------------------------ batched systems
// Many independent planetary systems advanced together by the MVS map (no
// counterpart in the reference, which integrates one system per process):
// one 32-thread CTA per system runs the Big-body integrator above, and one
// launch advances every test particle of every system, each warp on a tile of
// 32 slots of a single system. Systems have no non-gravitational forces and
// no central-body oblateness.
struct BatchSys {
    double mu, h;
    int nbig, nb;
    int first_slot, np;   // the system's particle slots
    int tab_off;          // doubles into a table set: [K + 1][tab_stride(nb)]
    int det_off;          // doubles into a detail set: [K][nb][TAB_DETAIL]
};
struct BatchTile {
    int sys, first, count, pad;
};

struct BatchBigArgs {
    const MvsBigArgs* proto;  // per system: constants, state buffers (in = set 0, out = set 1)
    const BatchSys* sys;
    int flip;                 // read set 1, write set 0
    int nsteps, reset, central, step0;
    double rcen;
    double* tab;              // table set of this chunk
    double* detail;           // detail set of this chunk
    MercuryEvent* events;
    int* event_step;
    int* event_sys;
    int event_cap;
    DeviceStatus* status;
};

struct BatchParticleArgs {
    int ntiles, npcap;
    int nsteps, reset, central, step0;
    double rcen;
    const BatchSys* sys;
    const BatchTile* tiles;
    const double* xin;        // [9][npcap]
    double* xout;
    const double* rce;        // [npcap]
    const double* rphys;
    const int* local;         // slot -> particle index within its system
    const double* tab;
    const double* detail;
    MercuryEvent* events;
    int* event_step;
    int* event_sys;
    int event_cap;
    EncounterCandidate* cands;  // slot field holds the system index
    int cand_cap;
    DeviceStatus* status;
};

void launch_mvs_big_batch(const BatchBigArgs& a, int nsys, int max_nbig, cudaStream_t s);
void launch_mvs_particles_batch(const BatchParticleArgs& a, cudaStream_t s, int threads);
void launch_classify_batch(const BatchParticleArgs& a, cudaStream_t s);

// Finishes mce_stat's test for the candidates of the last particle launch and
// writes the event records; detail is the base of the run's detail rows.
struct ClassifyArgs {
    int nb, nbig;
    double h;
    const double* detail;
    const EncounterCandidate* cands;
    int cand_cap;
    MercuryEvent* events;
    int* event_step;
    int event_cap;
    DeviceStatus* status;
    int step_base;         // added to a candidate's step in event_step
};
void launch_classify(const ClassifyArgs& a, cudaStream_t s);

void launch_mvs_big(const MvsBigArgs& a, cudaStream_t s);
void launch_mvs_particles(const MvsParticleArgs& a, cudaStream_t s, int threads);
size_t mvs_particle_smem(int nb, int nsteps, int reset, int threads, bool ngf);
int mvs_max_steps_per_launch(int nb);

}  // namespace mb200

// HYBRID on the device: the democratic-heliocentric step of mdt_hy
// (mercury6_2.for:3618-3782) split at the close-encounter hand-off as the
// reference's C ABI splits it (mercury_cuda_hybrid_begin / _finish):
//
//   begin:  [interaction force if stale] kick h/2, solar drift h/2, Kepler
//           drift h of every body, mce_snif -> encounter pairs
//   (host:  the members' subsystem integrated by BS2 with mfo_hkce)
//   finish: solar drift h/2, interaction force (mfo_hy + mfo_ngf), kick h/2
//
// The massive set (Big bodies and massive Small bodies, bodies [0, nsplit))
// is advanced by one CTA, which writes for the particles the solar-drift
// shift and a table row per force evaluation; massless particles run one
// thread per slot.
#pragma once
#include "common.cuh"

namespace mb200 {

constexpr int HY_HEAD = 8;        // shift or acen (3), acen (3), pad (2)
constexpr int HY_BEGIN_BODY = 20; // x0 v0 x1 v1 (12), padded box (4), rcrit, m, pad (2)
constexpr int HY_FORCE_BODY = 8;  // x (3), m, rcrit, pad (3)
__host__ __device__ constexpr int hy_begin_row(int nb) { return HY_HEAD + HY_BEGIN_BODY * nb; }
__host__ __device__ constexpr int hy_force_row(int nb) { return HY_HEAD + HY_FORCE_BODY * nb; }

struct HyArgs {
    int nbig, nsplit, np, npcap;
    int ngflag, obl, recompute;
    double jcen[3];
    double m0, h;
    const double* mbig;      // [nsplit]
    const double* rcritbig;  // [nsplit]
    const double* ngfbig;    // [nsplit][5]
    double* bx_in;           // [9][nsplit] start of step (its a(3) receives a recomputed acceleration)
    double* bx_out;          // [9][nsplit]
    double* bscr;            // [6][nsplit] massive set after the first solar drift (x0, v0 of mce_snif)
    double* px_in;           // [9][npcap]
    double* px_out;          // [9][npcap]
    const double* pconst;    // [PCONST_ROWS][npcap]
    const int* perm;         // slot -> particle index
    double* tab;             // 3 rows: force at the start, begin row, force at the end
    int2* pairs;             // encounter pairs (0-based global i < j)
    int pair_cap;
    DeviceStatus* status;    // events counts pairs; overflow bit 0
};

// Row offsets inside HyArgs::tab.
__host__ __device__ constexpr size_t hy_tab_force0(int) { return 0; }
__host__ __device__ constexpr size_t hy_tab_begin(int nb) { return (size_t)hy_force_row(nb); }
__host__ __device__ constexpr size_t hy_tab_force1(int nb) { return (size_t)hy_force_row(nb) + hy_begin_row(nb); }
__host__ __device__ constexpr size_t hy_tab_size(int nb) { return 2 * (size_t)hy_force_row(nb) + hy_begin_row(nb); }

void launch_hybrid_begin(const HyArgs& a, cudaStream_t s);
void launch_hybrid_finish(const HyArgs& a, cudaStream_t s);

// Members' pre-drift states (after the first solar drift) written into the
// out buffers and packed as rows {x(3), v(3)} for the host; ids are 0-based
// global body indices, inv maps a particle index to its slot.
void launch_hybrid_restore(const HyArgs& a, const int* ids, int count, const int* inv, double* packed,
                           cudaStream_t s);

// (1/m0) sum_j m_j v_j over the massive set in index order (mco_dh2h's
// velocity shift) of the state bx into out[3]; one thread.
void launch_dh_shift(const double* bx, const double* m, int nsplit, double m0, double* out, cudaStream_t s);

}  // namespace mb200

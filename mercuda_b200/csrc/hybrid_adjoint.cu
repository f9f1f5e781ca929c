// Gradients through the HYBRID test-particle integration (no counterpart in the
// reference): a forward run of the library's own HYBRID path that keeps
// checkpoints and the encounter members' step Jacobians, then a reverse sweep.
//
// Massless particles never act on the Big bodies, so each particle's final
// state is a function of its own initial state and Yarkovsky coefficient. Per
// step mdt_hy (mercury6_2.for:3618-3782) maps a particle by
//
//   kick h/2 (mfo_hy's changeover-weighted direct terms + yar) -> solar drift
//   h/2 (a shift set by the Big bodies alone) -> Kepler drift h, or, when
//   mce_snif makes it an encounter member, mdt_hkce's BS2 integration over h
//   -> solar drift h/2 -> kick h/2,
//
// so the reverse sweep is one thread per particle slot: transposed kicks
// (gravity with the changeover factor and its derivative, yar), the Kepler
// drift's state-transition matrix transposed, and for member steps the 6x6
// Jacobian of its BS2 segment, which the forward run accumulates in forward
// mode (bs2_tangent_kernel after every accepted BS2 substep) and stores.
//
//   forward:  mercury_cuda_hybrid_begin / encounter_enter / step / download /
//             encounter_exit / hybrid_finish per step, as mdt_hkce drives them
//             (the same calls and kernels as the drop-in HYBRID path); per step
//             the Big-body rows the particles need (solar-drift shifts, the
//             force row) and each massless member's end state and Jacobian;
//             the particle state every K steps
//   backward: per segment, last first: recompute the segment from its
//             checkpoint (members take their recorded end states), keeping each
//             step's drift input and output, then walk it backwards.
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/mercury_b200.h"
#include "context.cuh"
#include "force_adjoint.cuh"
#include "hybrid_device.cuh"
#include "kepler.cuh"
#include "kepler_adjoint.cuh"

namespace mb200 {
namespace {

constexpr int HREC = 12;  // per step of a segment: drift (or BS2) input x, v and output x, v
constexpr int MREC = 42;  // per member step: end state x, v (6), then the 6x6 Jacobian (row-major, d out / d in)

// Table row per step: [0..2] the first solar-drift shift, then the force row
// of the step's end (head: the second shift; per Big body x, m, rcrit). Row 0
// holds the force row of the initial state at offset 8.
__host__ __device__ constexpr int ha_row(int nb) { return 8 + hy_force_row(nb); }

struct HaArgs {
    HyArgs hy;               // nbig, m0, ngflag, status: the kick force's configuration
    int np, npcap, nsteps, K;
    double h;
    const double* tab;       // [nsteps + 1][ha_row(nb)]
    const double* ckpt;      // [nseg][9][npcap] particle state (x, v, cached a) in slot order
    const double* pcon;      // [2][npcap]: rcrit, yar per slot
    const int* perm;         // slot -> particle index
    const double* mrec;      // [members][MREC]
    const int* midx;         // [K][npcap]: member record of (step of the segment, slot), or -1
    double* rec;             // [K][HREC][npcap]
    double* lam;             // [10][npcap] adjoint state between segments
    const double* gx;        // (np, 3) adjoint of the final positions (particle order)
    const double* gv;        // (np, 3) or null
    double* dx0;             // (np, 3)
    double* dv0;
    double* dyar;            // [np] or null
};

__device__ __forceinline__ double3 ld_col(const double* a, int S, int p) {
    return make_double3(a[p], a[S + p], a[2 * (size_t)S + p]);
}

// The recomputation of one segment, keeping each step's drift input/output.
__global__ void __launch_bounds__(128) ha_recompute_kernel(HaArgs A, int seg) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const int S = A.npcap, W = ha_row(A.hy.nbig - 1);
    const double h = A.h, hby2 = 0.5 * h;
    const double rcrit_p = A.pcon[p];
    const double g[5] = {0.0, 0.0, 0.0, 0.0, A.pcon[S + p]};
    const double* c = A.ckpt + (size_t)seg * 9 * S;
    double3 x = ld_col(c, S, p), v = ld_col(c + 3 * (size_t)S, S, p), acc = ld_col(c + 6 * (size_t)S, S, p);
    if (seg == 0) acc = particle_hy_accel(A.hy, x, v, rcrit_p, g, A.tab + 8);
    auto R = [&](int sl, int k) -> double& { return A.rec[((size_t)sl * HREC + k) * S + p]; };
    const int s0 = seg * A.K, s1 = min(A.nsteps, s0 + A.K);
#pragma unroll 1
    for (int s = s0; s < s1; ++s) {
        const int sl = s - s0;
        const double* row = A.tab + (size_t)(s + 1) * W;
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
        x.x = x.x + row[0];
        x.y = x.y + row[1];
        x.z = x.z + row[2];
        R(sl, 0) = x.x; R(sl, 1) = x.y; R(sl, 2) = x.z;
        R(sl, 3) = v.x; R(sl, 4) = v.y; R(sl, 5) = v.z;
        const int m = A.midx[(size_t)sl * S + p];
        if (m >= 0) {
            const double* r = A.mrec + (size_t)m * MREC;
            x = make_double3(r[0], r[1], r[2]);
            v = make_double3(r[3], r[4], r[5]);
        } else {
            drift_one(A.hy.m0, x, v, h);
        }
        R(sl, 6) = x.x; R(sl, 7) = x.y; R(sl, 8) = x.z;
        R(sl, 9) = v.x; R(sl, 10) = v.y; R(sl, 11) = v.z;
        const double* T1 = row + 8;
        x.x = x.x + T1[0];
        x.y = x.y + T1[1];
        x.z = x.z + T1[2];
        acc = particle_hy_accel(A.hy, x, v, rcrit_p, g, T1);
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
    }
}

// J^T la of the kick force at (x, v) against force row T.
template <bool YAR>
__device__ __forceinline__ void hy_accel_vjp(int nb, const double3 x, const double3 v, double yar, double rcrit_p,
                                             const double* T, const double3 la, double3& gx, double3& gv,
                                             double& gyar) {
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* row = T + HY_HEAD + b * HY_FORCE_BODY;
        drct_term_vjp(x, row, row[3], fmax(row[4], rcrit_p), la, gx);
    }
    if (YAR) yar_vjp(x, v, yar, la, gx, gv, gyar);
}

// The segment backwards: second kick, force, Kepler drift (or the member's
// BS2 Jacobian), first kick; solar drifts shift by Big-body sums only and
// pass the adjoint through unchanged.
template <bool YAR> __global__ void __launch_bounds__(128) ha_vjp_kernel(HaArgs A, int seg, int last) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const int S = A.npcap, nb = A.hy.nbig - 1, W = ha_row(nb);
    const double h = A.h, hby2 = 0.5 * h;
    const double rcrit_p = A.pcon[p], yar = A.pcon[S + p];
    const int part = A.perm[p];
    auto R = [&](int sl, int k) -> double { return A.rec[((size_t)sl * HREC + k) * S + p]; };
    auto L = [&](int k) -> double& { return A.lam[(size_t)k * S + p]; };
    double3 lx, lv, la;
    double lyar;
    if (last) {
        lx = make_double3(A.gx[3 * (size_t)part], A.gx[3 * (size_t)part + 1], A.gx[3 * (size_t)part + 2]);
        lv = A.gv ? make_double3(A.gv[3 * (size_t)part], A.gv[3 * (size_t)part + 1], A.gv[3 * (size_t)part + 2])
                  : make_double3(0.0, 0.0, 0.0);
        la = make_double3(0.0, 0.0, 0.0);
        lyar = 0.0;
    } else {
        lx = make_double3(L(0), L(1), L(2));
        lv = make_double3(L(3), L(4), L(5));
        la = make_double3(L(6), L(7), L(8));
        lyar = L(9);
    }
    bool ok = true;
    const int s0 = seg * A.K, s1 = min(A.nsteps, s0 + A.K);
#pragma unroll 1
    for (int s = s1 - 1; s >= s0; --s) {
        const int sl = s - s0;
        const double* T1 = A.tab + (size_t)(s + 1) * W + 8;
        const double3 xd = make_double3(R(sl, 6), R(sl, 7), R(sl, 8));
        const double3 vd = make_double3(R(sl, 9), R(sl, 10), R(sl, 11));
        const double3 x2 = make_double3(xd.x + T1[0], xd.y + T1[1], xd.z + T1[2]);
        // second kick v3 = vd + hby2 a(x2, vd)
        const double3 lacc = make_double3(la.x + hby2 * lv.x, la.y + hby2 * lv.y, la.z + hby2 * lv.z);
        double3 gx = make_double3(0.0, 0.0, 0.0), gv = make_double3(0.0, 0.0, 0.0);
        hy_accel_vjp<YAR>(nb, x2, vd, yar, rcrit_p, T1, lacc, gx, gv, lyar);
        const double l1[6] = {lx.x + gx.x, lx.y + gx.y, lx.z + gx.z, lv.x + gv.x, lv.y + gv.y, lv.z + gv.z};
        double lo[6];
        const int m = A.midx[(size_t)sl * S + p];
        if (m >= 0) {
            const double* J = A.mrec + (size_t)m * MREC + 6;
            for (int c = 0; c < 6; ++c) {
                double acc = 0.0;
                for (int r = 0; r < 6; ++r) acc += J[6 * r + c] * l1[r];
                lo[c] = acc;
            }
        } else {
            const double xin[3] = {R(sl, 0), R(sl, 1), R(sl, 2)};
            const double vin[3] = {R(sl, 3), R(sl, 4), R(sl, 5)};
            const double xend[3] = {xd.x, xd.y, xd.z};
            ok = drift_vjp(A.hy.m0, xin, vin, h, xend, l1, l1 + 3, lo, lo + 3) && ok;
        }
        // first kick v1 = v + hby2 acc (acc: the cached acceleration)
        lx = make_double3(lo[0], lo[1], lo[2]);
        lv = make_double3(lo[3], lo[4], lo[5]);
        la = make_double3(hby2 * lo[3], hby2 * lo[4], hby2 * lo[5]);
    }
    if (!ok) raise_fault(A.hy.status, FAULT_NONFINITE);
    if (seg > 0) {
        L(0) = lx.x; L(1) = lx.y; L(2) = lx.z;
        L(3) = lv.x; L(4) = lv.y; L(5) = lv.z;
        L(6) = la.x; L(7) = la.y; L(8) = la.z;
        L(9) = lyar;
        return;
    }
    // the acceleration of the initial state (computed before the first kick)
    const double3 x0 = ld_col(A.ckpt, S, p), v0 = ld_col(A.ckpt + 3 * (size_t)S, S, p);
    double3 gx = make_double3(0.0, 0.0, 0.0), gv = make_double3(0.0, 0.0, 0.0);
    hy_accel_vjp<YAR>(nb, x0, v0, yar, rcrit_p, A.tab + 8, la, gx, gv, lyar);
    const double out[6] = {lx.x + gx.x, lx.y + gx.y, lx.z + gx.z, lv.x + gv.x, lv.y + gv.y, lv.z + gv.z};
    for (int c = 0; c < 3; ++c) {
        A.dx0[3 * (size_t)part + c] = out[c];
        A.dv0[3 * (size_t)part + c] = out[3 + c];
    }
    if (A.dyar) A.dyar[part] = lyar;
    for (int c = 0; c < 6; ++c)
        if (!isfinite(out[c])) raise_fault(A.hy.status, FAULT_NONFINITE);
}

// midx of one segment: record r of step s and slot k -> midx[(s - s0)][k].
__global__ void ha_member_index_kernel(const int2* key, int first, int count, int s0, int S, int* midx) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const int2 k = key[first + q];
    midx[(size_t)(k.x - s0) * S + k.y] = first + q;
}

// Slot-ordered particle state [9][S] -> particle-ordered (np, 3) rows.
__global__ void ha_gather_kernel(const double* px, int S, int np, const int* perm, double* xf, double* vf) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int part = perm[p];
    for (int c = 0; c < 3; ++c) {
        xf[3 * (size_t)part + c] = px[(size_t)c * S + p];
        vf[3 * (size_t)part + c] = px[(size_t)(3 + c) * S + p];
    }
}

struct HyAdjoint {
    int nbig = 0, np = 0, npcap = 0, nsteps = 0, K = 0, has_yar = 0;
    double h = 0.0, m0 = 0.0;
    DBuf<double> tab, ckpt, pcon, mrec, rec, lam;
    DBuf<int> perm, midx;
    DBuf<int2> mkey;
    DBuf<DeviceStatus> status;
    std::vector<int> rec_off;   // first member record of each step, [nsteps + 1]
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double fwd_ms = 0.0;
    float bwd_ms = 0.0f;
    bool ready = false;
    void ensure() {
        if (stream) return;
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
    }
    void release() {
        DBuf<double>* b[] = {&tab, &ckpt, &pcon, &mrec, &rec, &lam};
        for (auto* d : b) d->release();
        perm.release();
        midx.release();
        mkey.release();
        status.release();
        rec_off.clear();
        ready = false;
    }
};

HyAdjoint& hadj() {
    static HyAdjoint a;
    return a;
}

void d2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes) check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s), "copy");
}

// One encounter step of the resident system's members (mdt_hkce, as the
// drop-in host drives it): the subsystem of the central body and every member
// integrated by BS2 on a local clock, the members' end states written into
// xx, vv, and for each massless member its slot in the resident system, end
// state and 6x6 Jacobian appended to keys / records.
void encounter_step(int step, double h, double tol, double& hrec, int n, int nbig, const std::vector<double>& m,
                    const std::vector<double>& crit, const std::vector<int>& ce, const std::vector<int>& pi,
                    const std::vector<int>& pj, int count, const std::vector<int>& inv_main, std::vector<double>& xx,
                    std::vector<double>& vv, std::vector<int2>& keys, std::vector<double>& records) {
    std::vector<int> sub(1, 0), back(n, -1);
    for (int j = 1; j < n; ++j)
        if (ce[j]) sub.push_back(j);
    const int nbs = (int)sub.size();
    int nbsbig = 1;
    for (int k = 1; k < nbs; ++k) {
        back[sub[k]] = k;
        if (sub[k] < nbig) ++nbsbig;
    }
    std::vector<double> mbs(nbs), xbs(3 * (size_t)nbs, 0.0), vbs(3 * (size_t)nbs, 0.0), rcritbs(nbs, 0.0),
        zeros(nbs, 0.0);
    for (int k = 0; k < nbs; ++k) {
        const int j = sub[k];
        mbs[k] = m[j];
        if (k == 0) continue;
        rcritbs[k] = crit[j];
        for (int c = 0; c < 3; ++c) {
            xbs[3 * k + c] = xx[3 * (size_t)j + c];
            vbs[3 * k + c] = vv[3 * (size_t)j + c];
        }
    }
    std::vector<int> ibs(count), jbs(count);
    for (int k = 0; k < count; ++k) {
        ibs[k] = back[pi[k] - 1] + 1;
        jbs[k] = back[pj[k] - 1] + 1;
    }
    if (mercury_cuda_encounter_enter(nbs, nbsbig, mbs.data(), xbs.data(), vbs.data(), rcritbs.data(), zeros.data(),
                                     zeros.data(), count, ibs.data(), jbs.data()))
        throw std::runtime_error("hybrid adjoint: encounter initialization failed");
    struct Exit {
        ~Exit() {
            ctx().tangent = false;
            mercury_cuda_encounter_exit();
        }
    } exit_guard;
    Context& e = ctx();
    const int nps = e.np, S = e.npcap;
    if (nps > 0) {
        std::vector<double> eye((size_t)36 * S, 0.0);
        for (int d = 0; d < 6; ++d)
            for (int q = 0; q < nps; ++q) eye[(size_t)(6 * d + d) * S + q] = 1.0;
        e.tg.reserve((size_t)36 * S);
        h2d(e.tg.p, eye.data(), sizeof(double) * eye.size(), e.stream, "tangent");
        e.tangent = true;
    }
    int dtflag = 1;
    double tlocal = 0.0, hlocal = std::copysign(hrec, h);
    for (;;) {
        const double tmp0 = std::fabs(h) - std::fabs(tlocal);
        hrec = hlocal;
        if (std::fabs(hlocal) > tmp0) hlocal = std::copysign(tmp0, h);
        mercury_cuda_reset(dtflag);
        double hdid = 0.0;
        int64_t nf = 0, nr = 0;
        if (mercury_cuda_step(tlocal, &hlocal, &hdid, tol, &nf, &nr))
            throw std::runtime_error("hybrid adjoint: encounter step failed");
        dtflag = 2;
        tlocal = tlocal + hdid;
        if (!((tlocal - h) * h < 0.0)) break;
    }
    if (mercury_cuda_download(xbs.data(), vbs.data(), 0)) throw std::runtime_error("hybrid adjoint: download failed");
    std::vector<double> tg;
    std::vector<int> inv_sub(std::max(1, nps));
    if (nps > 0) {
        tg.resize((size_t)36 * S);
        check(cudaMemcpyAsync(tg.data(), e.tg.p, sizeof(double) * tg.size(), cudaMemcpyDeviceToHost, e.stream),
              "tangent");
        check(cudaMemcpyAsync(inv_sub.data(), e.inv.p, sizeof(int) * nps, cudaMemcpyDeviceToHost, e.stream), "slots");
        check(cudaStreamSynchronize(e.stream), "tangent");
    }
    const int nsplit_sub = e.nsplit;
    for (int k = 1; k < nbs; ++k) {
        const int j = sub[k];
        for (int c = 0; c < 3; ++c) {
            xx[3 * (size_t)j + c] = xbs[3 * k + c];
            vv[3 * (size_t)j + c] = vbs[3 * k + c];
        }
        if (j < nbig) continue;
        if (k < nsplit_sub) throw std::runtime_error("hybrid adjoint: massless member outside the particle slots");
        const int q = inv_sub[k - nsplit_sub];
        keys.push_back(make_int2(step, inv_main[j - nbig]));
        for (int c = 0; c < 3; ++c) records.push_back(xbs[3 * k + c]);
        for (int c = 0; c < 3; ++c) records.push_back(vbs[3 * k + c]);
        for (int r = 0; r < 6; ++r)
            for (int d = 0; d < 6; ++d) records.push_back(tg[(size_t)(6 * d + r) * S + q]);
    }
}

HaArgs ha_args(HyAdjoint& J) {
    HaArgs a{};
    a.hy.nbig = J.nbig;
    a.hy.nsplit = J.nbig;
    a.hy.np = J.np;
    a.hy.npcap = J.npcap;
    a.hy.ngflag = J.has_yar ? 1 : 0;
    a.hy.obl = 0;
    a.hy.m0 = J.m0;
    a.hy.h = J.h;
    a.hy.status = J.status.p;
    a.np = J.np;
    a.npcap = J.npcap;
    a.nsteps = J.nsteps;
    a.K = J.K;
    a.h = J.h;
    a.tab = J.tab.p;
    a.ckpt = J.ckpt.p;
    a.pcon = J.pcon.p;
    a.perm = J.perm.p;
    a.mrec = J.mrec.p;
    a.midx = J.midx.p;
    a.rec = J.rec.p;
    a.lam = J.lam.p;
    return a;
}

}  // namespace
}  // namespace mb200

using namespace mb200;

extern "C" {

int mercury_b200_hybrid_adjoint_forward(int nbig, const double* mbig, const double* xbig, const double* vbig,
                                        const double* rcrit_big, int np, const double* x0, const double* v0,
                                        const double* yar, const double* rcrit, double h, double tol, int nsteps,
                                        int checkpoint_every, double* x_final, double* v_final) {
    HyAdjoint& J = hadj();
    J.ready = false;
    try {
        if (active_context() != 0) throw std::runtime_error("hybrid adjoint: an encounter subsystem is active");
        if (nbig < 1 || nbig > 512) throw std::runtime_error("hybrid adjoint: nbig must be 1..512");
        if (np < 1 || nsteps < 1 || checkpoint_every < 1) throw std::runtime_error("hybrid adjoint: invalid sizes");
        if (!(h != 0.0) || !std::isfinite(h) || !(tol > 0.0))
            throw std::runtime_error("hybrid adjoint: invalid step or tolerance");
        const auto wall0 = std::chrono::steady_clock::now();
        J.ensure();
        const int n = nbig + np, nb = nbig - 1, W = ha_row(nb);
        // the whole system in the drop-in's host layout (democratic heliocentric)
        std::vector<double> m(n, 0.0), xx(3 * (size_t)n), vv(3 * (size_t)n), ngf(5 * (size_t)n, 0.0),
            zeros(n, 0.0), crit(n, 0.0), yh(np, 0.0);
        std::memcpy(m.data(), mbig, sizeof(double) * nbig);
        std::memcpy(xx.data(), xbig, sizeof(double) * 3 * nbig);
        std::memcpy(vv.data(), vbig, sizeof(double) * 3 * nbig);
        std::memcpy(crit.data(), rcrit_big, sizeof(double) * nbig);
        std::memcpy(crit.data() + nbig, rcrit, sizeof(double) * np);
        check(cudaMemcpy(xx.data() + 3 * (size_t)nbig, x0, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost), "x0");
        check(cudaMemcpy(vv.data() + 3 * (size_t)nbig, v0, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost), "v0");
        if (yar) check(cudaMemcpy(yh.data(), yar, sizeof(double) * np, cudaMemcpyDeviceToHost), "yar");
        for (int q = 0; q < np; ++q) ngf[5 * (size_t)(nbig + q) + 4] = yh[q];
        const double jc[3] = {0.0, 0.0, 0.0};
        if (mercury_cuda_configure(10)) throw std::runtime_error("hybrid adjoint: configure failed");
        if (mercury_cuda_upload(n, nbig, 0, yar ? 1 : 0, m.data(), xx.data(), vv.data(), ngf.data(), jc, zeros.data(),
                                zeros.data()))
            throw std::runtime_error("hybrid adjoint: upload failed");
        Context& c = ctx();
        if (c.nsplit != nbig || c.np != np) throw std::runtime_error("hybrid adjoint: unexpected body split");
        J.nbig = nbig;
        J.np = np;
        J.npcap = c.npcap;
        J.nsteps = nsteps;
        J.K = std::min(checkpoint_every, nsteps);
        J.h = h;
        J.m0 = mbig[0];
        J.has_yar = yar != nullptr;
        const int S = J.npcap, nseg = (nsteps + J.K - 1) / J.K;
        J.tab.reserve((size_t)(nsteps + 1) * W);
        J.ckpt.reserve((size_t)nseg * 9 * S);
        J.pcon.reserve((size_t)2 * S);
        J.perm.reserve(S);
        J.lam.reserve((size_t)10 * S);
        J.rec.reserve((size_t)J.K * HREC * S);
        J.midx.reserve((size_t)J.K * S);
        J.status.reserve(1);
        check(cudaMemsetAsync(J.tab.p, 0, sizeof(double) * (size_t)(nsteps + 1) * W, c.stream), "memset");
        check(cudaMemsetAsync(J.pcon.p, 0, sizeof(double) * 2 * S, c.stream), "memset");
        d2d(J.pcon.p, c.pconst[c.kc].p + (size_t)PC_RCRIT * S, sizeof(double) * S, c.stream);
        d2d(J.pcon.p + S, c.pconst[c.kc].p + (size_t)(PC_NGF + 4) * S, sizeof(double) * S, c.stream);
        d2d(J.perm.p, c.permp(), sizeof(int) * S, c.stream);
        std::vector<int> inv_main(np);
        check(cudaMemcpyAsync(inv_main.data(), c.inv.p, sizeof(int) * np, cudaMemcpyDeviceToHost, c.stream), "slots");
        check(cudaStreamSynchronize(c.stream), "slots");
        const int cap = std::max(1 << 16, 4 * n);
        std::vector<int> ce(n), pi(cap), pj(cap);
        std::vector<int2> keys;
        std::vector<double> records;
        J.rec_off.assign(nsteps + 1, 0);
        double hrec = h;
        for (int s = 0; s < nsteps; ++s) {
            Context& r = ctx();
            if (s % J.K == 0)
                d2d(J.ckpt.p + (size_t)(s / J.K) * 9 * S, r.pstate[r.cur].p, sizeof(double) * 9 * S, r.stream);
            int count = 0;
            int64_t f = 0;
            if (mercury_cuda_hybrid_begin(h, crit.data(), s == 0 ? 0 : 2, cap, ce.data(), &count, pi.data(), pj.data(),
                                          xx.data(), vv.data(), &f))
                throw std::runtime_error("hybrid adjoint: hybrid_begin failed");
            double* row = J.tab.p + (size_t)(s + 1) * W;
            d2d(row, r.hy_tab.p + hy_tab_begin(nb), sizeof(double) * 3, r.stream);
            if (s == 0) d2d(J.tab.p + 8, r.hy_tab.p + hy_tab_force0(nb), sizeof(double) * hy_force_row(nb), r.stream);
            if (count > 0)
                encounter_step(s, h, tol, hrec, n, nbig, m, crit, ce, pi, pj, count, inv_main, xx, vv, keys, records);
            J.rec_off[s + 1] = (int)keys.size();
            if (mercury_cuda_hybrid_finish(h, m.data(), xx.data(), vv.data(), &f))
                throw std::runtime_error("hybrid adjoint: hybrid_finish failed");
            d2d(row + 8, r.hy_tab.p + hy_tab_force1(nb), sizeof(double) * hy_force_row(nb), r.stream);
        }
        const size_t nrec = keys.size();
        J.mkey.reserve(std::max<size_t>(1, nrec));
        J.mrec.reserve(std::max<size_t>(1, nrec) * MREC);
        h2d(J.mkey.p, keys.data(), sizeof(int2) * nrec, c.stream, "members");
        h2d(J.mrec.p, records.data(), sizeof(double) * records.size(), c.stream, "members");
        ha_gather_kernel<<<(np + 127) / 128, 128, 0, c.stream>>>(c.pstate[c.cur].p, S, np, J.perm.p, x_final,
                                                                 v_final);
        check(cudaGetLastError(), "launch");
        check(cudaStreamSynchronize(c.stream), "hybrid adjoint forward");
        J.fwd_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
        J.ready = true;
        return 0;
    } catch (const std::exception& e) {
        if (active_context() != 0) mercury_cuda_encounter_exit();
        return report(e);
    }
}

int mercury_b200_hybrid_adjoint_backward(const double* gx, const double* gv, double* dx0, double* dv0, double* dyar) {
    HyAdjoint& J = hadj();
    try {
        if (!J.ready) throw std::runtime_error("hybrid adjoint backward without a forward run");
        const int S = J.npcap, nseg = (J.nsteps + J.K - 1) / J.K, grid = (J.np + 127) / 128;
        check(cudaMemsetAsync(J.status.p, 0, sizeof(DeviceStatus), J.stream), "memset");
        HaArgs a = ha_args(J);
        a.gx = gx;
        a.gv = gv;
        a.dx0 = dx0;
        a.dv0 = dv0;
        a.dyar = dyar;
        check(cudaEventRecord(J.e0, J.stream), "event");
        for (int seg = nseg - 1; seg >= 0; --seg) {
            const int s0 = seg * J.K, s1 = std::min(J.nsteps, s0 + J.K);
            check(cudaMemsetAsync(J.midx.p, 0xff, sizeof(int) * (size_t)J.K * S, J.stream), "memset");
            const int first = J.rec_off[s0], count = J.rec_off[s1] - first;
            if (count > 0)
                ha_member_index_kernel<<<(count + 127) / 128, 128, 0, J.stream>>>(J.mkey.p, first, count, s0, S,
                                                                                 J.midx.p);
            ha_recompute_kernel<<<grid, 128, 0, J.stream>>>(a, seg);
            const int last = seg == nseg - 1 ? 1 : 0;
            if (J.has_yar) ha_vjp_kernel<true><<<grid, 128, 0, J.stream>>>(a, seg, last);
            else ha_vjp_kernel<false><<<grid, 128, 0, J.stream>>>(a, seg, last);
        }
        check(cudaEventRecord(J.e1, J.stream), "event");
        check(cudaGetLastError(), "launch");
        DeviceStatus st;
        check(cudaMemcpyAsync(&st, J.status.p, sizeof(st), cudaMemcpyDeviceToHost, J.stream), "status");
        check(cudaStreamSynchronize(J.stream), "hybrid adjoint backward");
        check(cudaEventElapsedTime(&J.bwd_ms, J.e0, J.e1), "timer");
        if (st.fault) throw std::runtime_error("hybrid adjoint backward: non-finite gradient");
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_hybrid_adjoint_timing(double* forward_ms, double* backward_ms, int64_t* member_steps) {
    HyAdjoint& J = hadj();
    if (forward_ms) *forward_ms = J.fwd_ms;
    if (backward_ms) *backward_ms = J.bwd_ms;
    if (member_steps) *member_steps = J.rec_off.empty() ? 0 : J.rec_off.back();
    return 0;
}

void mercury_b200_hybrid_adjoint_free(void) { hadj().release(); }

}  // extern "C"

// Gradients through the MVS test-particle integration (no counterpart in the
// reference): a forward run that keeps checkpoints, then a reverse sweep.
//
// The Big bodies never feel massless particles, so their trajectory (and
// each step's force table) is fixed: one Big-body CTA integrates it, K steps
// per launch on a second stream, ahead of the particles. Each particle's
// final state is then a function of its own initial position, velocity and
// Yarkovsky coefficient only, and the reverse sweep is one thread per
// particle:
//
//   forward:  per K-step segment, the mdt_mvs step of every particle (the
//             same statements as the MVS kernels); (x, v, a) at each
//             segment's start is the checkpoint
//   backward: per segment, from the last: recompute the segment from its
//             checkpoint keeping each step's drift input and output, then
//             walk it backwards: kick, force (gravity from the table, yar) and
//             the Kepler drift's state-transition matrix, transposed. The
//             recomputation of segment k-1 (second stream, second record
//             buffer) overlaps the walk through segment k.
#include <cmath>
#include <cstdio>

#include "../../include/mercury_b200.h"
#include "context.cuh"
#include "force_adjoint.cuh"
#include "kepler.cuh"
#include "kepler_adjoint.cuh"
#include "mvs.cuh"
#include "mvs_device.cuh"

namespace mb200 {
namespace {

constexpr int REC = 12;  // per step of a segment: x, v after the kick (drift input), x, v after the drift

struct AdjArgs {
    int np, nb, nsteps, K, has_yar;
    double h, mu;
    const double* tab;       // [nsteps + 1][tab_stride(nb)]
    const double* x0;        // (np, 3) rows
    const double* v0;
    const double* yar;       // [np] or null
    double* xf;              // (np, 3)
    double* vf;
    double* ckpt;            // [nseg][9][np]
    double* rec;             // [K][REC][np] records of one segment
    double* lam;             // [10][np] adjoint state between segments
    const double* gx;        // (np, 3) adjoint of the final positions
    const double* gv;        // (np, 3) or null
    double* dx0;             // (np, 3)
    double* dv0;
    double* dyar;            // [np] or null
    DeviceStatus* status;
};

__device__ __forceinline__ double3 ld_row(const double* a, int p) {
    return make_double3(a[3 * (size_t)p], a[3 * (size_t)p + 1], a[3 * (size_t)p + 2]);
}
__device__ __forceinline__ void st_row(double* a, int p, double3 v) {
    a[3 * (size_t)p] = v.x;
    a[3 * (size_t)p + 1] = v.y;
    a[3 * (size_t)p + 2] = v.z;
}

// The kick acceleration (angf + 0) + a of mdt_mvs for a massless particle
// with Yarkovsky coefficient yar (no other non-gravitational terms).
template <bool YAR>
__device__ __forceinline__ double3 accel(const double3 x, const double3 v, double yar, const double* T, int nb,
                                         double mu, DeviceStatus* st) {
    return small_body_force<YAR, false>(x, v, [&](int c) -> double { return c == 4 ? yar : 0.0; }, T, nb, nullptr,
                                        mu, st);
}

// Transposed Jacobian of that acceleration applied to la: adds to gx, gv and
// gyar. Gravity: -sum_b m_b d/|d|^3 with d = x - x_b; Yarkovsky: yar_vjp.
template <bool YAR>
__device__ __forceinline__ void accel_vjp(const double3 x, const double3 v, double yar, const double* T, int nb,
                                          const double3 la, double3& gx, double3& gv, double& gyar) {
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* row = T + TAB_HEAD + b * TAB_BODY;
        const double dx = x.x - row[0], dy = x.y - row[1], dz = x.z - row[2];
        const double s2 = dx * dx + dy * dy + dz * dz;
        const double s_1 = 1.0 / sqrt(s2);
        const double s_3 = s_1 * s_1 * s_1;
        const double s_5 = s_3 * s_1 * s_1;
        const double dl = dx * la.x + dy * la.y + dz * la.z;
        const double m = row[3];
        gx.x -= m * (s_3 * la.x - 3.0 * s_5 * dl * dx);
        gx.y -= m * (s_3 * la.y - 3.0 * s_5 * dl * dy);
        gx.z -= m * (s_3 * la.z - 3.0 * s_5 * dl * dz);
    }
    if (YAR) yar_vjp(x, v, yar, la, gx, gv, gyar);
}

__device__ __forceinline__ void st_ckpt(double* c, int np, int p, double3 x, double3 v, double3 a) {
    const double q[9] = {x.x, x.y, x.z, v.x, v.y, v.z, a.x, a.y, a.z};
    for (int k = 0; k < 9; ++k) c[(size_t)k * np + p] = q[k];
}

// One K-step segment of the forward run: from the initial state (segment 0)
// or the segment's checkpoint, to the next checkpoint or the final state.
template <bool YAR> __global__ void __launch_bounds__(128) adj_forward_kernel(AdjArgs A, int seg) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const int stride = tab_stride(A.nb), np = A.np;
    const double hby2 = 0.5 * A.h;
    const double yar = YAR ? A.yar[p] : 0.0;
    const int s0 = seg * A.K, s1 = min(A.nsteps, s0 + A.K);
    double3 x, v, acc;
    if (seg == 0) {
        x = ld_row(A.x0, p);
        v = ld_row(A.v0, p);
        acc = accel<YAR>(x, v, yar, A.tab, A.nb, A.mu, A.status);
        st_ckpt(A.ckpt, np, p, x, v, acc);
    } else {
        const double* c = A.ckpt + (size_t)seg * 9 * np;
        x = make_double3(c[p], c[np + p], c[2 * (size_t)np + p]);
        v = make_double3(c[3 * (size_t)np + p], c[4 * (size_t)np + p], c[5 * (size_t)np + p]);
        acc = make_double3(c[6 * (size_t)np + p], c[7 * (size_t)np + p], c[8 * (size_t)np + p]);
    }
#pragma unroll 1
    for (int s = s0; s < s1; ++s) {
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
        drift_one(A.mu, x, v, A.h);
        acc = accel<YAR>(x, v, yar, A.tab + (size_t)(s + 1) * stride, A.nb, A.mu, A.status);
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
    }
    if (s1 < A.nsteps) {
        st_ckpt(A.ckpt + (size_t)(seg + 1) * 9 * np, np, p, x, v, acc);
    } else {
        st_row(A.xf, p, x);
        st_row(A.vf, p, v);
    }
}

// Reverse sweep, per segment (last first): recompute the segment from its
// checkpoint keeping each step's drift input and output ...
template <bool YAR> __global__ void __launch_bounds__(128) adj_recompute_kernel(AdjArgs A, int seg) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const int stride = tab_stride(A.nb), np = A.np;
    const double hby2 = 0.5 * A.h;
    const double yar = YAR ? A.yar[p] : 0.0;
    auto R = [&](int sl, int c) -> double& { return A.rec[((size_t)sl * REC + c) * np + p]; };
    const int s0 = seg * A.K, s1 = min(A.nsteps, s0 + A.K);
    const double* c = A.ckpt + (size_t)seg * 9 * np;
    double3 x = make_double3(c[p], c[np + p], c[2 * (size_t)np + p]);
    double3 v = make_double3(c[3 * (size_t)np + p], c[4 * (size_t)np + p], c[5 * (size_t)np + p]);
    double3 acc = make_double3(c[6 * (size_t)np + p], c[7 * (size_t)np + p], c[8 * (size_t)np + p]);
#pragma unroll 1
    for (int s = s0; s < s1; ++s) {
        const int sl = s - s0;
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
        R(sl, 0) = x.x; R(sl, 1) = x.y; R(sl, 2) = x.z;
        R(sl, 3) = v.x; R(sl, 4) = v.y; R(sl, 5) = v.z;
        drift_one(A.mu, x, v, A.h);
        R(sl, 6) = x.x; R(sl, 7) = x.y; R(sl, 8) = x.z;
        R(sl, 9) = v.x; R(sl, 10) = v.y; R(sl, 11) = v.z;
        acc = accel<YAR>(x, v, yar, A.tab + (size_t)(s + 1) * stride, A.nb, A.mu, A.status);
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
    }
}

// ... then walk it backwards: second kick, force, Kepler drift, first kick.
// The adjoint state (lx, lv, la, lyar) lives in A.lam [10][np] between
// segments; the first segment also differentiates the initial acceleration
// and writes the gradients.
template <bool YAR> __global__ void __launch_bounds__(128) adj_vjp_kernel(AdjArgs A, int seg, int last) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const int stride = tab_stride(A.nb), np = A.np;
    const double hby2 = 0.5 * A.h;
    const double yar = YAR ? A.yar[p] : 0.0;
    auto R = [&](int sl, int c) -> double { return A.rec[((size_t)sl * REC + c) * np + p]; };
    auto L = [&](int c) -> double& { return A.lam[(size_t)c * np + p]; };
    double3 lx, lv, la;
    double lyar;
    if (last) {
        lx = ld_row(A.gx, p);
        lv = A.gv ? ld_row(A.gv, p) : make_double3(0.0, 0.0, 0.0);
        la = make_double3(0.0, 0.0, 0.0);
        lyar = 0.0;
    } else {
        lx = make_double3(L(0), L(1), L(2));
        lv = make_double3(L(3), L(4), L(5));
        la = make_double3(L(6), L(7), L(8));
        lyar = L(9);
    }
    const int s0 = seg * A.K, s1 = min(A.nsteps, s0 + A.K);
#pragma unroll 1
    for (int s = s1 - 1; s >= s0; --s) {
        const int sl = s - s0;
        const double xin[3] = {R(sl, 0), R(sl, 1), R(sl, 2)};
        const double vin[3] = {R(sl, 3), R(sl, 4), R(sl, 5)};
        const double xend[3] = {R(sl, 6), R(sl, 7), R(sl, 8)};
        const double3 x2 = make_double3(xend[0], xend[1], xend[2]);
        const double3 v2 = make_double3(R(sl, 9), R(sl, 10), R(sl, 11));
        // second kick v3 = v2 + hby2 a(x2, v2)
        const double3 lacc = make_double3(la.x + hby2 * lv.x, la.y + hby2 * lv.y, la.z + hby2 * lv.z);
        double3 gx = make_double3(0.0, 0.0, 0.0), gv = make_double3(0.0, 0.0, 0.0);
        accel_vjp<YAR>(x2, v2, yar, A.tab + (size_t)(s + 1) * stride, A.nb, lacc, gx, gv, lyar);
        const double lx1[3] = {lx.x + gx.x, lx.y + gx.y, lx.z + gx.z};
        const double lv1[3] = {lv.x + gv.x, lv.y + gv.y, lv.z + gv.z};
        double lxo[3], lvo[3];
        if (!drift_vjp(A.mu, xin, vin, A.h, xend, lx1, lv1, lxo, lvo)) raise_fault(A.status, FAULT_NONFINITE);
        // first kick v1 = v + hby2 acc
        lx = make_double3(lxo[0], lxo[1], lxo[2]);
        lv = make_double3(lvo[0], lvo[1], lvo[2]);
        la = make_double3(hby2 * lvo[0], hby2 * lvo[1], hby2 * lvo[2]);
    }
    if (seg > 0) {
        L(0) = lx.x; L(1) = lx.y; L(2) = lx.z;
        L(3) = lv.x; L(4) = lv.y; L(5) = lv.z;
        L(6) = la.x; L(7) = la.y; L(8) = la.z;
        L(9) = lyar;
        return;
    }
    // the acceleration of the initial state (computed before the first kick)
    const double3 x0 = ld_row(A.x0, p), v0 = ld_row(A.v0, p);
    double3 gx = make_double3(0.0, 0.0, 0.0), gv = make_double3(0.0, 0.0, 0.0);
    accel_vjp<YAR>(x0, v0, yar, A.tab, A.nb, la, gx, gv, lyar);
    st_row(A.dx0, p, make_double3(lx.x + gx.x, lx.y + gx.y, lx.z + gx.z));
    st_row(A.dv0, p, make_double3(lv.x + gv.x, lv.y + gv.y, lv.z + gv.z));
    if (A.dyar) A.dyar[p] = lyar;
    if (!isfinite(lx.x) || !isfinite(lv.x) || !isfinite(lyar)) raise_fault(A.status, FAULT_NONFINITE);
}

struct Adjoint {
    int nbig = 0, np = 0, nsteps = 0, K = 0, has_yar = 0;
    double h = 0.0, mu = 0.0;
    const double *x0 = nullptr, *v0 = nullptr, *yar = nullptr;
    DBuf<double> bigstate[2], mbig, zeros, tab, detail, ckpt, rec[2], lam;
    DBuf<MercuryEvent> events;
    DBuf<int> event_step;
    DBuf<DeviceStatus> status;
    cudaStream_t stream = nullptr, stream2 = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<cudaEvent_t> done2, done1;   // per segment: second-stream and main-stream work finished
    float fwd_ms = 0.0f, bwd_ms = 0.0f;
    bool ready = false;
    void ensure() {
        if (stream) return;
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking), "stream");
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
    }
    void ensure_events(int n) {
        while ((int)done2.size() < n) {
            cudaEvent_t a, b;
            check(cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "event");
            check(cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "event");
            done2.push_back(a);
            done1.push_back(b);
        }
    }
    void release() {
        DBuf<double>* b[] = {&bigstate[0], &bigstate[1], &mbig, &zeros, &tab, &detail, &ckpt, &rec[0], &rec[1], &lam};
        for (auto* d : b) d->release();
        events.release();
        event_step.release();
        status.release();
        ready = false;
    }
};

Adjoint& adj() {
    static Adjoint a;
    return a;
}

AdjArgs adj_args(Adjoint& J) {
    AdjArgs a{};
    a.np = J.np;
    a.nb = J.nbig - 1;
    a.nsteps = J.nsteps;
    a.K = J.K;
    a.has_yar = J.has_yar;
    a.h = J.h;
    a.mu = J.mu;
    a.tab = J.tab.p;
    a.x0 = J.x0;
    a.v0 = J.v0;
    a.yar = J.yar;
    a.ckpt = J.ckpt.p;
    a.rec = J.rec[0].p;
    a.lam = J.lam.p;
    a.status = J.status.p;
    return a;
}

}  // namespace
}  // namespace mb200

using namespace mb200;

extern "C" {

int mercury_b200_adjoint_forward(int nbig, const double* mbig, const double* xbig, const double* vbig, int np,
                                 const double* x0, const double* v0, const double* yar, double h, int nsteps,
                                 int checkpoint_every, double* x_final, double* v_final) {
    Adjoint& J = adj();
    try {
        if (nbig < 1 || nbig > 512) throw std::runtime_error("adjoint: nbig must be 1..512");
        if (np < 1 || nsteps < 1 || checkpoint_every < 1) throw std::runtime_error("adjoint: invalid sizes");
        if (!(h != 0.0) || !std::isfinite(h)) throw std::runtime_error("adjoint: invalid step");
        J.ensure();
        J.nbig = nbig;
        J.np = np;
        J.nsteps = nsteps;
        J.K = std::min(checkpoint_every, nsteps);
        J.h = h;
        J.mu = mbig[0];
        J.x0 = x0;
        J.v0 = v0;
        J.yar = yar;
        J.has_yar = yar != nullptr;
        const int nb = nbig - 1, nseg = (nsteps + J.K - 1) / J.K;
        for (int k = 0; k < 2; ++k) J.bigstate[k].reserve((size_t)9 * nbig);
        J.mbig.reserve(nbig);
        J.zeros.reserve(nbig);
        J.tab.reserve((size_t)(nsteps + 1) * tab_stride(nb));
        J.detail.reserve((size_t)nsteps * std::max(1, nb) * TAB_DETAIL);
        J.ckpt.reserve((size_t)nseg * 9 * np);
        J.rec[0].reserve((size_t)J.K * REC * np);
        J.rec[1].reserve(nseg > 1 ? (size_t)J.K * REC * np : 1);
        J.ensure_events(nseg);
        J.lam.reserve((size_t)10 * np);
        J.events.reserve(4096);
        J.event_step.reserve(4096);
        J.status.reserve(1);
        // Big bodies: SoA [9][nbig] from the host rows, a(3) zero (reset)
        std::vector<double> b(9 * (size_t)nbig, 0.0);
        for (int k = 0; k < nbig; ++k)
            for (int c = 0; c < 3; ++c) {
                b[c * nbig + k] = xbig[3 * k + c];
                b[(3 + c) * nbig + k] = vbig[3 * k + c];
            }
        h2d(J.bigstate[0].p, b.data(), sizeof(double) * b.size(), J.stream);
        h2d(J.mbig.p, mbig, sizeof(double) * nbig, J.stream);
        check(cudaMemsetAsync(J.zeros.p, 0, sizeof(double) * nbig, J.stream), "memset");
        check(cudaMemsetAsync(J.status.p, 0, sizeof(DeviceStatus), J.stream), "memset");
        check(cudaEventRecord(J.e0, J.stream), "event");
        check(cudaStreamWaitEvent(J.stream2, J.e0, 0), "wait");
        AdjArgs f = adj_args(J);
        f.xf = x_final;
        f.vf = v_final;
        const int grid = (np + 127) / 128, stride = tab_stride(nb);
        for (int seg = 0; seg < nseg; ++seg) {
            const int s0 = seg * J.K, ks = std::min(J.K, nsteps - s0);
            // the Big bodies' steps of this segment and their force tables
            // (rows s0 + 1 .. s0 + ks; row 0 too on the first)
            MvsBigArgs a{};
            a.nbig = nbig;
            a.reset = seg == 0 ? 1 : 0;
            a.nsteps = ks;
            a.step0 = s0;
            a.h = h;
            a.m = J.mbig.p;
            a.rce = J.zeros.p;
            a.rphys = J.zeros.p;
            double* bin = J.bigstate[seg & 1].p;
            double* bout = J.bigstate[(seg + 1) & 1].p;
            a.in.x = bin;
            a.in.v = bin + 3 * nbig;
            a.in.a = bin + 6 * nbig;
            a.out.x = bout;
            a.out.v = bout + 3 * nbig;
            a.out.a = bout + 6 * nbig;
            a.tab = J.tab.p + (size_t)s0 * stride;
            a.detail = J.detail.p + (size_t)s0 * std::max(1, nb) * TAB_DETAIL;
            a.events = J.events.p;
            a.event_step = J.event_step.p;
            a.event_cap = (int)J.events.n;
            a.status = J.status.p;
            launch_mvs_big(a, J.stream2);
            check(cudaEventRecord(J.done2[seg], J.stream2), "event");
            check(cudaStreamWaitEvent(J.stream, J.done2[seg], 0), "wait");
            if (J.has_yar) adj_forward_kernel<true><<<grid, 128, 0, J.stream>>>(f, seg);
            else adj_forward_kernel<false><<<grid, 128, 0, J.stream>>>(f, seg);
        }
        check(cudaEventRecord(J.e1, J.stream), "event");
        check(cudaGetLastError(), "launch");
        DeviceStatus st;
        check(cudaMemcpyAsync(&st, J.status.p, sizeof(st), cudaMemcpyDeviceToHost, J.stream), "status");
        check(cudaStreamSynchronize(J.stream), "adjoint forward");
        check(cudaEventElapsedTime(&J.fwd_ms, J.e0, J.e1), "timer");
        if (st.fault) throw std::runtime_error("adjoint forward: force failed");
        J.ready = true;
        return 0;
    } catch (const std::exception& e) {
        J.ready = false;
        return report(e);
    }
}

int mercury_b200_adjoint_backward(const double* gx, const double* gv, double* dx0, double* dv0, double* dyar) {
    Adjoint& J = adj();
    try {
        if (!J.ready) throw std::runtime_error("adjoint backward without a forward run");
        check(cudaMemsetAsync(J.status.p, 0, sizeof(DeviceStatus), J.stream), "memset");
        AdjArgs a = adj_args(J);
        a.gx = gx;
        a.gv = gv;
        a.dx0 = dx0;
        a.dv0 = dv0;
        a.dyar = dyar;
        check(cudaEventRecord(J.e0, J.stream), "event");
        check(cudaStreamWaitEvent(J.stream2, J.e0, 0), "wait");
        const int grid = (J.np + 127) / 128;
        const int nseg = (J.nsteps + J.K - 1) / J.K;
        // segment seg's records live in rec[seg & 1]: recomputing seg - 1 on
        // the second stream waits only for the walk through seg + 1, the last
        // reader of that buffer
        auto recompute = [&](int seg) {
            AdjArgs r = a;
            r.rec = J.rec[seg & 1].p;
            if (seg + 2 < nseg) check(cudaStreamWaitEvent(J.stream2, J.done1[seg + 2], 0), "wait");
            if (J.has_yar) adj_recompute_kernel<true><<<grid, 128, 0, J.stream2>>>(r, seg);
            else adj_recompute_kernel<false><<<grid, 128, 0, J.stream2>>>(r, seg);
            check(cudaEventRecord(J.done2[seg], J.stream2), "event");
        };
        recompute(nseg - 1);
        for (int seg = nseg - 1; seg >= 0; --seg) {
            const int last = seg == nseg - 1 ? 1 : 0;
            if (seg > 0) recompute(seg - 1);
            check(cudaStreamWaitEvent(J.stream, J.done2[seg], 0), "wait");
            AdjArgs w = a;
            w.rec = J.rec[seg & 1].p;
            if (J.has_yar) adj_vjp_kernel<true><<<grid, 128, 0, J.stream>>>(w, seg, last);
            else adj_vjp_kernel<false><<<grid, 128, 0, J.stream>>>(w, seg, last);
            check(cudaEventRecord(J.done1[seg], J.stream), "event");
        }
        check(cudaEventRecord(J.e1, J.stream), "event");
        check(cudaGetLastError(), "launch");
        DeviceStatus st;
        check(cudaMemcpyAsync(&st, J.status.p, sizeof(st), cudaMemcpyDeviceToHost, J.stream), "status");
        check(cudaStreamSynchronize(J.stream), "adjoint backward");
        check(cudaEventElapsedTime(&J.bwd_ms, J.e0, J.e1), "timer");
        if (st.fault) throw std::runtime_error("adjoint backward: non-finite gradient");
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_adjoint_timing(double* forward_ms, double* backward_ms) {
    Adjoint& J = adj();
    if (forward_ms) *forward_ms = J.fwd_ms;
    if (backward_ms) *backward_ms = J.bwd_ms;
    return 0;
}

void mercury_b200_adjoint_free(void) { adj().release(); }

}  // extern "C"

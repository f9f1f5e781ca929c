// MVS kernels: the Big-body integrator (one CTA) and the fused test-particle
// step (kick, Kepler drift, encounter screen, interaction kick) for K steps
// per launch with the particle state in registers.
#include <stdexcept>

#include "kepler.cuh"
#include "mvs.cuh"
#include "mvs_device.cuh"

// Minimum resident CTAs per SM requested from ptxas for the particle kernel
// (bounds its registers per thread at 65536 / (128 * this)).
#ifndef MB200_PARTICLE_MIN_BLOCKS
#define MB200_PARTICLE_MIN_BLOCKS 5
#endif

namespace mb200 {
static_assert(sizeof(MercuryEvent) == 8 * sizeof(double2), "event records are eight double2 words");

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ double3 ld3(const double* p, int stride, int k) {
    return make_double3(p[k], p[stride + k], p[2 * stride + k]);
}
__device__ __forceinline__ void st3(double* p, int stride, int k, double3 v) {
    p[k] = v.x;
    p[stride + k] = v.y;
    p[2 * stride + k] = v.z;
}

// ------------------------------------------------------------ Big bodies
// Shared-memory workspace of the Big-body CTA, all [3][nbig] unless noted.
struct BigSmem {
    double *X, *V, *XJ, *VJ, *ACC, *X0, *V0, *XS, *VS, *A1, *A2, *AOBL, *GM, *misc;
    __device__ void carve(double* base, int nbig) {
        double* p = base;
        double** arrays[] = {&X, &V, &XJ, &VJ, &ACC, &X0, &V0, &XS, &VS, &A1, &A2, &AOBL};
        for (double** a : arrays) { *a = p; p += 3 * nbig; }
        GM = p; p += nbig;
        misc = p;  // a0[3], a0tp[3], acen[3]
    }
};

// Bodies held by the Big-body CTA (Big, then massive Small bodies).
__device__ __forceinline__ int big_count(const MvsBigArgs& A) { return A.nmass > A.nbig ? A.nmass : A.nbig; }

// mco_h2j for the Big bodies (mercury6_2.for:2613-2682), one thread; arrays
// [3][S].
__device__ void big_h2j(int nbig, const double* m, const double* X, const double* V, double* XJ, double* VJ, int S) {
    if (nbig < 2) return;
    double mtot = m[1];
    double mx[3], mv[3];
    for (int c = 0; c < 3; ++c) {
        XJ[c * S + 1] = X[c * S + 1];
        VJ[c * S + 1] = V[c * S + 1];
        mx[c] = m[1] * X[c * S + 1];
        mv[c] = m[1] * V[c * S + 1];
    }
    for (int j = 2; j <= nbig - 2; ++j) {
        const double temp = 1.0 / (mtot + m[0]);
        mtot = mtot + m[j];
        for (int c = 0; c < 3; ++c) {
            XJ[c * S + j] = X[c * S + j] - temp * mx[c];
            VJ[c * S + j] = V[c * S + j] - temp * mv[c];
        }
        for (int c = 0; c < 3; ++c) {
            mx[c] = mx[c] + m[j] * X[c * S + j];
            mv[c] = mv[c] + m[j] * V[c * S + j];
        }
    }
    if (nbig > 2) {
        const double temp = 1.0 / (mtot + m[0]);
        const int j = nbig - 1;
        for (int c = 0; c < 3; ++c) {
            XJ[c * S + j] = X[c * S + j] - temp * mx[c];
            VJ[c * S + j] = V[c * S + j] - temp * mv[c];
        }
    }
}

// mco_j2h for the Big bodies (mercury6_2.for:2700-2770), one thread; arrays
// [3][S].
__device__ void big_j2h(int nbig, const double* m, const double* XJ, const double* VJ, double* X, double* V, int S) {
    if (nbig < 2) return;
    double mtot = m[1];
    double temp = m[1] / (mtot + m[0]);
    double mx[3], mv[3];
    for (int c = 0; c < 3; ++c) {
        X[c * S + 1] = XJ[c * S + 1];
        V[c * S + 1] = VJ[c * S + 1];
        mx[c] = temp * XJ[c * S + 1];
        mv[c] = temp * VJ[c * S + 1];
    }
    for (int j = 2; j <= nbig - 2; ++j) {
        for (int c = 0; c < 3; ++c) {
            X[c * S + j] = XJ[c * S + j] + mx[c];
            V[c * S + j] = VJ[c * S + j] + mv[c];
        }
        mtot = mtot + m[j];
        temp = m[j] / (mtot + m[0]);
        for (int c = 0; c < 3; ++c) {
            mx[c] = mx[c] + temp * XJ[c * S + j];
            mv[c] = mv[c] + temp * VJ[c * S + j];
        }
    }
    if (nbig > 2) {
        const int j = nbig - 1;
        for (int c = 0; c < 3; ++c) {
            X[c * S + j] = XJ[c * S + j] + mx[c];
            V[c * S + j] = VJ[c * S + j] + mv[c];
        }
    }
}

// mfo_mvs for the Big bodies plus the indirect term a0tp that every Small
// body receives (mercury6_2.for:4946-5070), with mfo_ngf for Big bodies.
// Writes S.ACC = (angf + 0) + a and S.misc = {a0, a0tp, acen}. All threads.
// With massive Small bodies held (A.nmass > nbig) their oblateness terms
// enter acen in body order, as mfo_obl sums over every body
// (mercury6_2.for:5176-5230); their own accelerations follow from the force
// row (small_type_force).
__device__ void big_force(const MvsBigArgs& A, BigSmem& S, const double* V_ngf) {
    const int nbig = A.nbig, N = big_count(A), tid = threadIdx.x, nt = blockDim.x;
    const double* m = A.m;
    double* a0 = S.misc;
    double* a0tp = S.misc + 3;
    double* acen = S.misc + 6;
    if (tid == 0) {
        a0[0] = a0[1] = a0[2] = 0.0;
        if (nbig >= 2)
            for (int c = 0; c < 3; ++c) { S.A1[c * N + 1] = 0.0; S.A2[c * N + 1] = 0.0; }
        double minside = 0.0;
        for (int k = 2; k < nbig; ++k) {
            const int k1 = k - 1;
            minside = minside + m[k1];
            const double3 p = ld3(S.X, N, k), pj = ld3(S.XJ, N, k);
            const double r2 = p.x * p.x + p.y * p.y + p.z * p.z;
            const double rj2 = pj.x * pj.x + pj.y * pj.y + pj.z * pj.z;
            const double r = 1.0 / sqrt(r2);
            const double rj = 1.0 / sqrt(rj2);
            const double r3 = r * r * r;
            const double rj3 = rj * rj * rj;
            const double fac0 = m[k] * r3;
            const double fac12 = m[0] * rj3;
            const double fac2 = m[k] * fac12 / (minside + m[0]);
            const double q = (r2 - rj2) * 0.5 / rj2;
            const double q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3, q6 = q3 * q3, q7 = q3 * q4;
            const double fac1 = 402.1875 * q7 - 187.6875 * q6 + 86.625 * q5 - 39.375 * q4 + 17.5 * q3 -
                                7.5 * q2 + 3.0 * q - 1.0;
            const double pc[3] = {p.x, p.y, p.z}, pjc[3] = {pj.x, pj.y, pj.z};
            for (int c = 0; c < 3; ++c) {
                a0[c] = a0[c] - fac0 * pc[c];
                S.A1[c * N + k] = fac12 * (pjc[c] + fac1 * pc[c]);
                S.A2[c * N + k] = S.A2[c * N + k1] + fac2 * pjc[c];
            }
        }
        a0tp[0] = a0tp[1] = a0tp[2] = 0.0;
        if (nbig >= 2) {
            const double3 p = ld3(S.X, N, 1);
            const double r2 = p.x * p.x + p.y * p.y + p.z * p.z;
            const double r = 1.0 / sqrt(r2);
            const double r3 = r * r * r;
            const double fac0 = m[1] * r3;
            a0tp[0] = a0[0] - fac0 * p.x;
            a0tp[1] = a0[1] - fac0 * p.y;
            a0tp[2] = a0[2] - fac0 * p.z;
        }
    }
    if (A.obl)
        for (int k = 1 + tid; k < N; k += nt) st3(S.AOBL, N, k, oblate_accel(ld3(S.X, N, k), A.jcen, m[0]));
    __syncthreads();
    if (tid == 0) {
        acen[0] = acen[1] = acen[2] = 0.0;
        if (A.obl)
            for (int k = 1; k < N; ++k) {
                const double tmp4 = m[k] / m[0];
                const double3 ao = ld3(S.AOBL, N, k);
                acen[0] = acen[0] - tmp4 * ao.x;
                acen[1] = acen[1] - tmp4 * ao.y;
                acen[2] = acen[2] - tmp4 * ao.z;
            }
    }
    __syncthreads();
    for (int k = 1 + tid; k < nbig; k += nt) {
        const double3 pk = ld3(S.X, N, k);
        double3 a3 = make_double3(0.0, 0.0, 0.0);
        for (int i = 1; i < nbig; ++i) {
            if (i == k) continue;
            const double3 pi = ld3(S.X, N, i);
            // The pair (lower, higher) is differenced higher - lower in mfo_mvs.
            const bool lower = i < k;
            const double dx = lower ? pk.x - pi.x : pi.x - pk.x;
            const double dy = lower ? pk.y - pi.y : pi.y - pk.y;
            const double dz = lower ? pk.z - pi.z : pi.z - pk.z;
            const double s2 = dx * dx + dy * dy + dz * dz;
            const double s_1 = 1.0 / sqrt(s2);
            const double s_3 = s_1 * s_1 * s_1;
            const double fac = m[i] * s_3;
            if (lower) { a3.x = a3.x - fac * dx; a3.y = a3.y - fac * dy; a3.z = a3.z - fac * dz; }
            else { a3.x = a3.x + fac * dx; a3.y = a3.y + fac * dy; a3.z = a3.z + fac * dz; }
        }
        double3 a;
        a.x = a0[0] + S.A1[k] + S.A2[k] + a3.x;
        a.y = a0[1] + S.A1[N + k] + S.A2[N + k] + a3.y;
        a.z = a0[2] + S.A1[2 * N + k] + S.A2[2 * N + k] + a3.z;
        if (A.obl) {
            const double3 ao = ld3(S.AOBL, N, k);
            a.x = a.x + (ao.x - acen[0]);
            a.y = a.y + (ao.y - acen[1]);
            a.z = a.z + (ao.z - acen[2]);
        }
        if (A.ngflag == 1 || A.ngflag == 3) {
            double3 g;
            if (!nongrav_accel(pk, ld3(V_ngf, N, k), A.ngf + 5 * k, g)) raise_fault(A.status, 2);
            a.x = g.x + 0.0 + a.x;
            a.y = g.y + 0.0 + a.y;
            a.z = g.z + 0.0 + a.z;
        }
        if (!isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z)) raise_fault(A.status, 1);
        st3(S.ACC, N, k, a);
    }
    __syncthreads();
}

// Force row of a table: head {a0tp, acen} and per-Big-body {x, m}.
__device__ void write_force_table(const MvsBigArgs& A, const BigSmem& S, double* row) {
    const int nbig = A.nbig, N = big_count(A);
    if (threadIdx.x == 0)
        for (int c = 0; c < 6; ++c) row[c] = S.misc[3 + c];
    for (int k = 1 + threadIdx.x; k < nbig; k += blockDim.x) {
        double* b = row + TAB_HEAD + (k - 1) * TAB_BODY;
        b[0] = S.X[k];
        b[1] = S.X[N + k];
        b[2] = S.X[2 * N + k];
        b[3] = A.m[k];
    }
}

// Accelerations of the massive Small bodies held by the CTA: the particles'
// mfo_mvs + mfo_ngf statements (small_body_force) against the force row just
// written. All threads; the row must be visible (after __syncthreads).
__device__ void small_type_force(const MvsBigArgs& A, BigSmem& S, const double* row, const double* V_ngf) {
    const int nbig = A.nbig, N = big_count(A), nb = nbig - 1;
    const bool ngf = A.ngflag == 1 || A.ngflag == 3;
    for (int k = nbig + threadIdx.x; k < N; k += blockDim.x) {
        const double3 x = ld3(S.X, N, k), v = ld3(V_ngf, N, k);
        auto g = [&](int c) -> double { return A.ngf[5 * k + c]; };
        double3 a;
        if (ngf) a = A.obl ? small_body_force<true, true>(x, v, g, row, nb, A.jcen, A.m[0], A.status)
                           : small_body_force<true, false>(x, v, g, row, nb, A.jcen, A.m[0], A.status);
        else a = A.obl ? small_body_force<false, true>(x, v, g, row, nb, A.jcen, A.m[0], A.status)
                       : small_body_force<false, false>(x, v, g, row, nb, A.jcen, A.m[0], A.status);
        st3(S.ACC, N, k, a);
    }
    __syncthreads();
}

// The drift of mdt_mvs: h2j, Kepler drift of each Jacobi Big body with gm_j,
// j2h; each massive Small body drifts heliocentrically about the central
// mass (mercury6_2.for:4031-4052). All threads.
__device__ void big_drift(const MvsBigArgs& A, BigSmem& S, double h) {
    const int nbig = A.nbig, N = big_count(A), tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) big_h2j(nbig, A.m, S.X, S.V, S.XJ, S.VJ, N);
    __syncthreads();
    for (int k = 1 + tid; k < N; k += nt) {
        if (k < nbig) {
            double3 p = ld3(S.XJ, N, k), w = ld3(S.VJ, N, k);
            drift_one(S.GM[k], p, w, h);
            st3(S.XJ, N, k, p);
            st3(S.VJ, N, k, w);
        } else {
            double3 p = ld3(S.X, N, k), w = ld3(S.V, N, k);
            drift_one(A.m[0], p, w, h);
            st3(S.X, N, k, p);
            st3(S.V, N, k, w);
        }
    }
    __syncthreads();
    if (tid == 0) big_j2h(nbig, A.m, S.XJ, S.VJ, S.X, S.V, N);
    __syncthreads();
}

__device__ void big_load(const MvsBigArgs& A, BigSmem& S, double* smem) {
    const int nbig = A.nbig, N = big_count(A), tid = threadIdx.x, nt = blockDim.x;
    S.carve(smem, N);
    for (int k = tid; k < N; k += nt)
        for (int c = 0; c < 3; ++c) {
            S.X[c * N + k] = A.in.x[c * N + k];
            S.V[c * N + k] = A.in.v[c * N + k];
            S.ACC[c * N + k] = A.in.a[c * N + k];
        }
    if (tid == 0) {
        double minside = A.m[0];
        for (int j = 1; j < nbig; ++j) {
            const double msofar = minside + A.m[j];
            S.GM[j] = A.m[0] * msofar / minside;
            minside = msofar;
        }
    }
    __syncthreads();
}

// The Big-body integrator of one system (all threads of the CTA), with the
// massive Small bodies it holds (A.nmass > nbig).
__device__ void big_run(const MvsBigArgs& A, double* smem) {
    const int nbig = A.nbig, N = big_count(A), nb = nbig - 1, tid = threadIdx.x, nt = blockDim.x;
    const int stride = tab_stride(nb);
    BigSmem S;
    big_load(A, S, smem);
    if (A.reset) {
        if (tid == 0) big_h2j(nbig, A.m, S.X, S.V, S.XJ, S.VJ, N);
        __syncthreads();
        big_force(A, S, S.V);
        write_force_table(A, S, A.tab);
        __syncthreads();
        if (N > nbig) small_type_force(A, S, A.tab, S.V);
    }
    const double h = A.h, hby2 = 0.5 * h, hm1 = 1.0 / h;
    for (int s = 0; s < A.nsteps; ++s) {
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                S.XS[z] = S.X[z];
                S.VS[z] = S.V[z];
                S.V[z] = S.V[z] + hby2 * S.ACC[z];
                S.X0[z] = S.X[z];
                S.V0[z] = S.V[z];
            }
        __syncthreads();
        big_drift(A, S, h);
        double* row = A.tab + (size_t)(s + 1) * stride;
        double* det = A.detail + (size_t)s * nb * TAB_DETAIL;
        for (int k = 1 + tid; k < nbig; k += nt) {
            double* b = row + TAB_HEAD + (k - 1) * TAB_BODY;
            const double pad = A.rce[k] * 1.2;
            double lo, hi;
            box_extent(S.X0[k], S.X[k], S.V0[k], S.V[k], h, lo, hi);
            b[4] = lo - pad;
            b[5] = hi + pad;
            box_extent(S.X0[N + k], S.X[N + k], S.V0[N + k], S.V[N + k], h, lo, hi);
            b[6] = lo - pad;
            b[7] = hi + pad;
            double* d = det + (k - 1) * TAB_DETAIL;
            for (int c = 0; c < 3; ++c) {
                d[c] = S.X0[c * N + k];
                d[3 + c] = S.V0[c * N + k];
                d[6 + c] = S.X[c * N + k];
                d[9 + c] = S.V[c * N + k];
            }
            d[12] = A.rce[k];
            d[13] = A.rphys[k];
        }
        // mce_stat between Big bodies (pairs 1 <= i < j < nbig), then between
        // Big bodies and the massive Small bodies held (i < nbig <= j < N).
        const int npair_big = nb * (nb - 1) / 2;
        const int npair = npair_big + nb * (N - nbig);
        for (int q = tid; q < npair; q += nt) {
            int i = 1, j;
            if (q < npair_big) {
                int rem = q;
                while (rem >= nbig - 1 - i) { rem -= nbig - 1 - i; ++i; }
                j = i + 1 + rem;
            } else {
                const int r = q - npair_big;
                i = 1 + r / (N - nbig);
                j = nbig + r % (N - nbig);
            }
            double lo_i, hi_i, lo_j, hi_j, ylo_i, yhi_i, ylo_j, yhi_j;
            const double pi_ = A.rce[i] * 1.2, pj_ = A.rce[j] * 1.2;
            box_extent(S.X0[i], S.X[i], S.V0[i], S.V[i], h, lo_i, hi_i);
            box_extent(S.X0[N + i], S.X[N + i], S.V0[N + i], S.V[N + i], h, ylo_i, yhi_i);
            box_extent(S.X0[j], S.X[j], S.V0[j], S.V[j], h, lo_j, hi_j);
            box_extent(S.X0[N + j], S.X[N + j], S.V0[N + j], S.V[N + j], h, ylo_j, yhi_j);
            lo_i = lo_i - pi_; hi_i = hi_i + pi_; ylo_i = ylo_i - pi_; yhi_i = yhi_i + pi_;
            lo_j = lo_j - pj_; hi_j = hi_j + pj_; ylo_j = ylo_j - pj_; yhi_j = yhi_j + pj_;
            if (!(hi_i >= lo_j && hi_j >= lo_i && yhi_i >= ylo_j && yhi_j >= ylo_i)) continue;
            PairEnds I{ld3(S.X0, N, i), ld3(S.V0, N, i), ld3(S.X, N, i), ld3(S.V, N, i)};
            PairEnds J{ld3(S.X0, N, j), ld3(S.V0, N, j), ld3(S.X, N, j), ld3(S.V, N, j)};
            PairClass pc;
            if (pair_classify(I, J, A.rce[i], A.rce[j], A.rphys[i], A.rphys[j], h, pc)) {
                const int slot = atomicAdd(&A.status->events, 1);
                if (slot < A.event_cap) {
                    pair_record(A.events + slot, I, J, pc, hm1, i + 1, j + 1, A.m[j] > A.m[i] && j < nbig);
                    A.event_step[slot] = A.step0 + s;
                    if (A.event_sys) A.event_sys[slot] = A.sys;
                } else {
                    atomicExch(&A.status->overflow, 1);
                }
            }
        }
        __syncthreads();
        big_force(A, S, S.V);
        write_force_table(A, S, row);
        if (N > nbig) {
            __syncthreads();
            small_type_force(A, S, row, S.V);
        }
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                S.V[z] = S.V[z] + hby2 * S.ACC[z];
            }
        __syncthreads();
        if (A.central)
            for (int k = 1 + tid; k < N; k += nt) {
                double temp;
                if (central_impact(ld3(S.XS, N, k), ld3(S.VS, N, k), ld3(S.X, N, k), ld3(S.V, N, k), A.m[0],
                                   A.m[k], h, A.rcen, temp)) {
                    const int slot = atomicAdd(&A.status->events, 1);
                    if (slot < A.event_cap) {
                        MercuryEvent rec = {};
                        rec.i = 1;
                        rec.j = k + 1;
                        rec.kind = EV_CENTRAL;
                        rec.time = temp;
                        rec.distance = A.rcen;
                        store_event(A.events + slot, rec);
                        A.event_step[slot] = A.step0 + s;
                        if (A.event_sys) A.event_sys[slot] = A.sys;
                    } else {
                        atomicExch(&A.status->overflow, 1);
                    }
                }
            }
    }
    __syncthreads();
    for (int k = tid; k < N; k += nt)
        for (int c = 0; c < 3; ++c) {
            A.out.x[c * N + k] = S.X[c * N + k];
            A.out.v[c * N + k] = S.V[c * N + k];
            A.out.a[c * N + k] = S.ACC[c * N + k];
        }
}

__global__ void __launch_bounds__(128) mvs_big_kernel(MvsBigArgs A) {
    extern __shared__ double smem[];
    big_run(A, smem);
}

// ------------------------------------------------------------ test particles
// Warp-aggregated slot claim: one atomic per warp, slots in lane order by a
// ballot prefix count; -1 for lanes without a record or beyond capacity.
// Must be reached by all 32 lanes.
__device__ __forceinline__ int claim_slot(bool has, int cap, DeviceStatus* st, int* counter, int overflow_bit) {
    const unsigned mask = __ballot_sync(FULL, has);
    if (mask == 0) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(FULL, base, leader);
    if (!has) return -1;
    const int slot = base + __popc(mask & ((1u << lane) - 1u));
    if (slot >= cap) {
        atomicOr(&st->overflow, overflow_bit);
        return -1;
    }
    return slot;
}

// Thread-private shared-memory columns of the particle kernel, one double per
// thread per column (column-major, so the lanes of a warp hit distinct banks).
// Only x, v and the cached acceleration of the particle being advanced live in
// registers; its constants, its pre-drift state and the second particle of the
// thread's pair wait here, which keeps the drift's register footprint small.
struct Cols {
    static constexpr int PARK = 0;     // 9: x, v, acc of the waiting particle
    static constexpr int RCE = 9;      // 2: per particle of the pair
    static constexpr int RPHYS = 11;   // 2
    static constexpr int MASS = 13;    // 2
    static constexpr int X0 = 15;      // 3: state after the first kick
    static constexpr int V0 = 18;      // 3
    static constexpr int CEN = 21;     // 4: mce_cent start quantities
    static constexpr int NGF = 25;     // 10: five coefficients per particle
    static constexpr int count(bool ngf) { return ngf ? 35 : 25; }
    // column stride: the kernel's largest CTA, so that a column offset is a
    // constant (base already points at the thread's own entry)
    static constexpr int STRIDE = 128;
    volatile double* base;
    __device__ volatile double& at(int c) const { return base[c * STRIDE]; }
    __device__ double3 ld3(int c) const { return make_double3(at(c), at(c + 1), at(c + 2)); }
    __device__ void st3(int c, double3 v) const { at(c) = v.x; at(c + 1) = v.y; at(c + 2) = v.z; }
};

// small_body_force with the coefficients of pair member u in the columns.
template <bool NGF, bool OBL>
__device__ __forceinline__ double3 particle_force(const double3 x, const double3 v_ngf, const Cols& cols, int u,
                                                  const double* T, int nb, const double* jcen, double mu,
                                                  DeviceStatus* st) {
    return small_body_force<NGF, OBL>(x, v_ngf, [&](int c) -> double { return cols.at(Cols::NGF + 5 * u + c); }, T,
                                      nb, jcen, mu, st);
}

// One mdt_mvs step of one Small body (slot p, pair member u) against the staged
// table T of step s.
template <bool NGF, bool OBL, bool CENTRAL>
__device__ __forceinline__ void particle_step(double3& x, double3& v, double3& acc, bool ok, int p, int u,
                                              const Cols& cols, const double* T, int s, const MvsParticleArgs& A,
                                              double hby2, double hm1) {
    const int nb = A.nb;
    const double h = A.h;
    double bxlo = 0.0, bxhi = 0.0, bylo = 0.0, byhi = 0.0;
    if (ok) {
        if (CENTRAL) {
            const CentralStart c = central_start(x, v);
            cols.at(Cols::CEN) = c.rr0;
            cols.at(Cols::CEN + 1) = c.rv0;
            cols.at(Cols::CEN + 2) = c.h2;
            cols.at(Cols::CEN + 3) = c.v2;
        }
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
        cols.st3(Cols::X0, x);
        cols.st3(Cols::V0, v);
        drift_one(A.mu, x, v, h);
        box_extent(cols.at(Cols::X0), x.x, cols.at(Cols::V0), v.x, h, bxlo, bxhi);
        box_extent(cols.at(Cols::X0 + 1), x.y, cols.at(Cols::V0 + 1), v.y, h, bylo, byhi);
        const double pad = cols.at(Cols::RCE + u) * 1.2;
        bxlo = bxlo - pad;
        bxhi = bxhi + pad;
        bylo = bylo - pad;
        byhi = byhi + pad;
    }
    // mce_stat against each Big body; the loop is uniform across the warp.
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* row = T + TAB_HEAD + b * TAB_BODY;
        const bool cand = ok && row[5] >= bxlo && bxhi >= row[4] && row[7] >= bylo && byhi >= row[6];
        if (__any_sync(FULL, cand)) {
            const int slot = claim_slot(cand, A.cand_cap, A.status, &A.status->cands, 2);
            if (slot >= 0) {
                EncounterCandidate* c = A.cands + slot;
                *reinterpret_cast<int4*>(c) = make_int4(p, b, A.step0 + s, A.nbig + A.perm[p] + 1);
                double2* w = reinterpret_cast<double2*>(c);
                w[1] = make_double2(cols.at(Cols::RCE + u), cols.at(Cols::RPHYS + u));
                w[2] = make_double2(cols.at(Cols::X0), cols.at(Cols::X0 + 1));
                w[3] = make_double2(cols.at(Cols::X0 + 2), cols.at(Cols::V0));
                w[4] = make_double2(cols.at(Cols::V0 + 1), cols.at(Cols::V0 + 2));
                w[5] = make_double2(x.x, x.y);
                w[6] = make_double2(x.z, v.x);
                w[7] = make_double2(v.y, v.z);
            }
        }
    }
    if (ok) {
        acc = particle_force<NGF, OBL>(x, v, cols, u, T, nb, A.jcen, A.mu, A.status);
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
    }
    if (CENTRAL) {
        double temp = 0.0;
        bool hit = false;
        if (ok) {
            const CentralStart c{cols.at(Cols::CEN), cols.at(Cols::CEN + 1), cols.at(Cols::CEN + 2),
                                 cols.at(Cols::CEN + 3)};
            hit = central_finish(c, x, v, A.mu, cols.at(Cols::MASS + u), h, A.rcen, temp);
        }
        const int slot = claim_slot(hit, A.event_cap, A.status, &A.status->events, 1);
        if (slot >= 0) {
            MercuryEvent* e = A.events + slot;
            *reinterpret_cast<int4*>(e) = make_int4(1, A.nbig + A.perm[p] + 1, EV_CENTRAL, 0);
            reinterpret_cast<double2*>(e)[1] = make_double2(A.rcen, temp);
            // a central-body record carries no states (xi = xj = 0)
            for (int k = 2; k < 8; ++k) reinterpret_cast<double2*>(e)[k] = make_double2(0.0, 0.0);
            A.event_step[slot] = A.step0 + s;
        }
    }
}

// Test-particle kernel: each thread owns a pair of adjacent particle slots (one
// double2 per state component), advances the first through all K steps while
// the second waits in shared memory, then the second; the Big-body tables of
// the K steps are staged in shared memory once per CTA.
template <bool NGF, bool OBL, bool CENTRAL>
__global__ void __launch_bounds__(128, MB200_PARTICLE_MIN_BLOCKS) mvs_particle_kernel(MvsParticleArgs A) {
    extern __shared__ double smem[];
    const int nb = A.nb, stride = tab_stride(nb);
    const int rows = A.nsteps + (A.reset ? 1 : 0);
    double* stab = smem;
    const Cols cols{smem + (size_t)rows * stride + threadIdx.x};
    const double* gtab = A.tab + (A.reset ? 0 : stride);
    for (int k = threadIdx.x; k < rows * stride; k += blockDim.x) stab[k] = gtab[k];
    __syncthreads();
    const double* steps_tab = stab + (A.reset ? stride : 0);
    const double hby2 = 0.5 * A.h, hm1 = 1.0 / A.h;
    const int lane = threadIdx.x & 31;
    const int npairs = (A.np + 1) >> 1;
    // Warps claim 32-pair tiles from a launch-wide counter: slots are ordered
    // slowest-first (Newton-path particles lead), so claiming dynamically
    // balances the SMs (longest-processing-time-first).
    const int ntiles = (npairs + 31) >> 5;
    const int S = A.npcap, H = S / 2;
    const double2* in = reinterpret_cast<const double2*>(A.xin);
    double2* out = reinterpret_cast<double2*>(A.xout);
    int* const tiles = A.tiles ? A.tiles : &A.status->next_tile;
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = atomicAdd(tiles, 1);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= ntiles) break;
        const int pair = tile * 32 + lane;
        const bool live = pair < npairs;
        const int j0 = 2 * pair;
        double3 x, v, acc;
        if (live) {
            double2 t[9];
#pragma unroll
            for (int c = 0; c < 9; ++c) t[c] = in[c * H + pair];
            x = make_double3(t[0].x, t[1].x, t[2].x);
            v = make_double3(t[3].x, t[4].x, t[5].x);
            acc = make_double3(t[6].x, t[7].x, t[8].x);
#pragma unroll
            for (int c = 0; c < 9; ++c) cols.at(Cols::PARK + c) = t[c].y;
            const double2 rc = reinterpret_cast<const double2*>(A.rce)[pair];
            const double2 rp = reinterpret_cast<const double2*>(A.rphys)[pair];
            const double2 ms = reinterpret_cast<const double2*>(A.m)[pair];
            cols.at(Cols::RCE) = rc.x; cols.at(Cols::RCE + 1) = rc.y;
            cols.at(Cols::RPHYS) = rp.x; cols.at(Cols::RPHYS + 1) = rp.y;
            cols.at(Cols::MASS) = ms.x; cols.at(Cols::MASS + 1) = ms.y;
            if (NGF)
                for (int c = 0; c < 5; ++c) {
                    const double2 g = reinterpret_cast<const double2*>(A.ngf + (size_t)c * S)[pair];
                    cols.at(Cols::NGF + c) = g.x;
                    cols.at(Cols::NGF + 5 + c) = g.y;
                }
        }
#pragma unroll 1
        for (int u = 0; u < 2; ++u) {
            const bool ok = live && j0 + u < A.np;
            if (u == 1 && live) {
                // the first particle's result waits; the second comes in
                const double3 px = cols.ld3(Cols::PARK), pv = cols.ld3(Cols::PARK + 3),
                              pa = cols.ld3(Cols::PARK + 6);
                cols.st3(Cols::PARK, x);
                cols.st3(Cols::PARK + 3, v);
                cols.st3(Cols::PARK + 6, acc);
                x = px;
                v = pv;
                acc = pa;
            }
            if (A.reset && ok) acc = particle_force<NGF, OBL>(x, v, cols, u, stab, nb, A.jcen, A.mu, A.status);
            for (int s = 0; s < A.nsteps; ++s)
                particle_step<NGF, OBL, CENTRAL>(x, v, acc, ok, j0 + u, u, cols, steps_tab + s * stride, s, A, hby2,
                                                 hm1);
        }
        if (live) {
            const double3 fx = cols.ld3(Cols::PARK), fv = cols.ld3(Cols::PARK + 3), fa = cols.ld3(Cols::PARK + 6);
            out[0 * H + pair] = make_double2(fx.x, x.x);
            out[1 * H + pair] = make_double2(fx.y, x.y);
            out[2 * H + pair] = make_double2(fx.z, x.z);
            out[3 * H + pair] = make_double2(fv.x, v.x);
            out[4 * H + pair] = make_double2(fv.y, v.y);
            out[5 * H + pair] = make_double2(fv.z, v.z);
            out[6 * H + pair] = make_double2(fa.x, acc.x);
            out[7 * H + pair] = make_double2(fa.y, acc.y);
            out[8 * H + pair] = make_double2(fa.z, acc.z);
            if (A.rows_x) {
                // rows in particle order for the copy back to the host
                const int i0 = A.perm[j0];
                A.rows_x[3 * (size_t)i0] = fx.x;
                A.rows_x[3 * (size_t)i0 + 1] = fx.y;
                A.rows_x[3 * (size_t)i0 + 2] = fx.z;
                A.rows_v[3 * (size_t)i0] = fv.x;
                A.rows_v[3 * (size_t)i0 + 1] = fv.y;
                A.rows_v[3 * (size_t)i0 + 2] = fv.z;
                if (j0 + 1 < A.np) {
                    const int i1 = A.perm[j0 + 1];
                    A.rows_x[3 * (size_t)i1] = x.x;
                    A.rows_x[3 * (size_t)i1 + 1] = x.y;
                    A.rows_x[3 * (size_t)i1 + 2] = x.z;
                    A.rows_v[3 * (size_t)i1] = v.x;
                    A.rows_v[3 * (size_t)i1 + 1] = v.y;
                    A.rows_v[3 * (size_t)i1 + 2] = v.z;
                }
            }
        }
    }
}

// ------------------------------------------------------------ output corrector
// The Big bodies' part of the corrector (mercury6_2.for:2200-2222 in
// mco_mvs2h, 2510-2532 in mco_h2mvs) from big.in into big.out, writing the
// force table of each of the four kicks.
__global__ void __launch_bounds__(128) mvs_corrector_big_kernel(MvsBigArgs A, CorrectorArgs K) {
    extern __shared__ double smem[];
    const int nbig = A.nbig, N = big_count(A), nb = nbig - 1, tid = threadIdx.x, nt = blockDim.x;
    const int stride = tab_stride(nb);
    BigSmem S;
    big_load(A, S, smem);
    auto force = [&](double* row) {
        big_force(A, S, S.V);
        write_force_table(A, S, row);
        if (N > nbig) {
            __syncthreads();
            small_type_force(A, S, row, S.V);
        }
    };
    auto kick = [&](double hk, bool subtract) {
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                const double term = hk * S.ACC[z];
                S.V[z] = subtract ? S.V[z] - term : S.V[z] + term;
            }
        __syncthreads();
    };
    for (int k = 0; k < 2; ++k) {
        big_drift(A, S, K.ha[k]);
        force(A.tab + (size_t)(2 * k) * stride);
        kick(K.hb[k], K.forward != 0);
        big_drift(A, S, -2.0 * K.ha[k]);
        force(A.tab + (size_t)(2 * k + 1) * stride);
        kick(K.hb[k], K.forward == 0);
        big_drift(A, S, K.ha[k]);
    }
    for (int k = tid; k < N; k += nt)
        for (int c = 0; c < 3; ++c) {
            A.out.x[c * N + k] = S.X[c * N + k];
            A.out.v[c * N + k] = S.V[c * N + k];
        }
}

// The Small bodies' part: heliocentric drifts with the central mass and the
// mfo_mvs + mfo_ngf kicks against the Big-body tables; one thread per slot.
template <bool NGF, bool OBL>
__global__ void __launch_bounds__(128) mvs_corrector_particle_kernel(CorrectorArgs K) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x, S = K.npcap;
    if (p >= K.np) return;
    const int stride = tab_stride(K.nb);
    double3 x = make_double3(K.xin[p], K.xin[S + p], K.xin[2 * S + p]);
    double3 v = make_double3(K.xin[3 * S + p], K.xin[4 * S + p], K.xin[5 * S + p]);
    auto g = [&](int c) -> double { return K.ngf[(size_t)c * S + p]; };
    auto kick = [&](const double* T, double hk, bool subtract) {
        const double3 a = small_body_force<NGF, OBL>(x, v, g, T, K.nb, K.jcen, K.mu, K.status);
        v.x = subtract ? v.x - hk * a.x : v.x + hk * a.x;
        v.y = subtract ? v.y - hk * a.y : v.y + hk * a.y;
        v.z = subtract ? v.z - hk * a.z : v.z + hk * a.z;
    };
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        drift_one(K.mu, x, v, K.ha[k]);
        kick(K.tab + (size_t)(2 * k) * stride, K.hb[k], K.forward != 0);
        drift_one(K.mu, x, v, -2.0 * K.ha[k]);
        kick(K.tab + (size_t)(2 * k + 1) * stride, K.hb[k], K.forward == 0);
        drift_one(K.mu, x, v, K.ha[k]);
    }
    K.xout[p] = x.x;
    K.xout[S + p] = x.y;
    K.xout[2 * S + p] = x.z;
    K.xout[3 * S + p] = v.x;
    K.xout[4 * S + p] = v.y;
    K.xout[5 * S + p] = v.z;
}

// mce_stat's test for each encounter candidate of the last launch
// (mercury6_2.for:1815-1908) and the record it produces.
__global__ void __launch_bounds__(256) classify_kernel(ClassifyArgs A) {
    const int count = min(A.status->cands, A.cand_cap);
    const double hm1 = 1.0 / A.h;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const EncounterCandidate& c = A.cands[k];
        const double* d = A.detail + ((size_t)c.step * A.nb + c.body) * TAB_DETAIL;
        const PairEnds I{make_double3(d[0], d[1], d[2]), make_double3(d[3], d[4], d[5]),
                         make_double3(d[6], d[7], d[8]), make_double3(d[9], d[10], d[11])};
        const PairEnds J{make_double3(c.x0[0], c.x0[1], c.x0[2]), make_double3(c.v0[0], c.v0[1], c.v0[2]),
                         make_double3(c.x1[0], c.x1[1], c.x1[2]), make_double3(c.v1[0], c.v1[1], c.v1[2])};
        PairClass pc;
        if (!pair_classify(I, J, d[12], c.rce, d[13], c.rphys, A.h, pc)) continue;
        const int slot = atomicAdd(&A.status->events, 1);
        if (slot < A.event_cap) {
            pair_record(A.events + slot, I, J, pc, hm1, c.body + 2, c.id, false);
            A.event_step[slot] = c.step + A.step_base;
        } else {
            atomicOr(&A.status->overflow, 1);
        }
    }
}

// ------------------------------------------------------------ batched systems
__global__ void __launch_bounds__(32) mvs_big_batch_kernel(BatchBigArgs B) {
    extern __shared__ double smem[];
    const int q = blockIdx.x;
    MvsBigArgs A = B.proto[q];
    if (B.flip) {
        const BigState t = A.in;
        A.in = A.out;
        A.out = t;
    }
    A.nsteps = B.nsteps;
    A.reset = B.reset;
    A.central = B.central;
    A.step0 = B.step0;
    A.rcen = B.rcen;
    A.tab = B.tab + B.sys[q].tab_off;
    A.detail = B.detail + B.sys[q].det_off;
    A.events = B.events;
    A.event_step = B.event_step;
    A.event_sys = B.event_sys;
    A.event_cap = B.event_cap;
    A.status = B.status;
    A.sys = q;
    big_run(A, smem);
}

// One mdt_mvs step of one test particle of a batched system against its
// step table T (the same statements as particle_step).
template <bool CENTRAL>
__device__ __forceinline__ void batch_particle_step(double3& x, double3& v, double3& acc, bool ok, int p, int sysid,
                                                    const BatchSys& S, const double* T, int s,
                                                    const BatchParticleArgs& A, double rce, double rphys, int id) {
    const int nb = S.nb;
    const double h = S.h, hby2 = 0.5 * h;
    double bxlo = 0.0, bxhi = 0.0, bylo = 0.0, byhi = 0.0;
    double3 x0 = x, v0 = v;
    CentralStart c0{0.0, 0.0, 0.0, 0.0};
    if (ok) {
        if (CENTRAL) c0 = central_start(x, v);
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
        x0 = x;
        v0 = v;
        drift_one(S.mu, x, v, h);
        box_extent(x0.x, x.x, v0.x, v.x, h, bxlo, bxhi);
        box_extent(x0.y, x.y, v0.y, v.y, h, bylo, byhi);
        const double pad = rce * 1.2;
        bxlo = bxlo - pad;
        bxhi = bxhi + pad;
        bylo = bylo - pad;
        byhi = byhi + pad;
    }
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* row = T + TAB_HEAD + b * TAB_BODY;
        const bool cand = ok && row[5] >= bxlo && bxhi >= row[4] && row[7] >= bylo && byhi >= row[6];
        if (__any_sync(FULL, cand)) {
            const int slot = claim_slot(cand, A.cand_cap, A.status, &A.status->cands, 2);
            if (slot >= 0) {
                EncounterCandidate* c = A.cands + slot;
                *reinterpret_cast<int4*>(c) = make_int4(sysid, b, A.step0 + s, id);
                double2* w = reinterpret_cast<double2*>(c);
                w[1] = make_double2(rce, rphys);
                w[2] = make_double2(x0.x, x0.y);
                w[3] = make_double2(x0.z, v0.x);
                w[4] = make_double2(v0.y, v0.z);
                w[5] = make_double2(x.x, x.y);
                w[6] = make_double2(x.z, v.x);
                w[7] = make_double2(v.y, v.z);
            }
        }
    }
    if (ok) {
        acc = small_body_force<false, false>(x, v, [](int) -> double { return 0.0; }, T, nb, nullptr, S.mu,
                                             A.status);
        v.x = v.x + hby2 * acc.x;
        v.y = v.y + hby2 * acc.y;
        v.z = v.z + hby2 * acc.z;
    }
    if (CENTRAL) {
        double temp = 0.0;
        bool hit = false;
        if (ok) hit = central_finish(c0, x, v, S.mu, 0.0, h, A.rcen, temp);
        const int slot = claim_slot(hit, A.event_cap, A.status, &A.status->events, 1);
        if (slot >= 0) {
            MercuryEvent* e = A.events + slot;
            *reinterpret_cast<int4*>(e) = make_int4(1, id, EV_CENTRAL, 0);
            reinterpret_cast<double2*>(e)[1] = make_double2(A.rcen, temp);
            for (int k = 2; k < 8; ++k) reinterpret_cast<double2*>(e)[k] = make_double2(0.0, 0.0);
            A.event_step[slot] = A.step0 + s;
            A.event_sys[slot] = sysid;
        }
    }
    (void)p;
}

// Every test particle of every system: warps claim 32-slot tiles (each of a
// single system) from a launch-wide counter and run K steps per particle in
// registers; the step tables are read through the cache.
template <bool CENTRAL> __global__ void __launch_bounds__(256) mvs_particle_batch_kernel(BatchParticleArgs A) {
    const int lane = threadIdx.x & 31, S2 = A.npcap;
    for (;;) {
        int tile = 0;
        if (lane == 0) tile = atomicAdd(&A.status->next_tile, 1);
        tile = __shfl_sync(FULL, tile, 0);
        if (tile >= A.ntiles) break;
        const BatchTile t = A.tiles[tile];
        const BatchSys S = A.sys[t.sys];
        const bool ok = lane < t.count;
        const int p = t.first + (ok ? lane : 0);
        const int stride = tab_stride(S.nb);
        const double* tab = A.tab + S.tab_off;
        double3 x = ld3(A.xin, S2, p), v = ld3(A.xin + 3 * (size_t)S2, S2, p);
        double3 acc = ld3(A.xin + 6 * (size_t)S2, S2, p);
        const double rce = A.rce[p], rphys = A.rphys[p];
        const int id = S.nbig + A.local[p] + 1;
        if (A.reset && ok)
            acc = small_body_force<false, false>(x, v, [](int) -> double { return 0.0; }, tab, S.nb, nullptr, S.mu,
                                                 A.status);
#pragma unroll 1
        for (int s = 0; s < A.nsteps; ++s)
            batch_particle_step<CENTRAL>(x, v, acc, ok, p, t.sys, S, tab + (size_t)(s + 1) * stride, s, A, rce,
                                         rphys, id);
        if (ok) {
            st3(A.xout, S2, p, x);
            st3(A.xout + 3 * (size_t)S2, S2, p, v);
            st3(A.xout + 6 * (size_t)S2, S2, p, acc);
        }
    }
}

// mce_stat's test for the candidates of the last batched launch.
__global__ void __launch_bounds__(256) classify_batch_kernel(BatchParticleArgs A) {
    const int count = min(A.status->cands, A.cand_cap);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const EncounterCandidate& c = A.cands[k];
        const BatchSys S = A.sys[c.slot];
        const double* d = A.detail + S.det_off + ((size_t)(c.step - A.step0) * S.nb + c.body) * TAB_DETAIL;
        const PairEnds I{make_double3(d[0], d[1], d[2]), make_double3(d[3], d[4], d[5]),
                         make_double3(d[6], d[7], d[8]), make_double3(d[9], d[10], d[11])};
        const PairEnds J{make_double3(c.x0[0], c.x0[1], c.x0[2]), make_double3(c.v0[0], c.v0[1], c.v0[2]),
                         make_double3(c.x1[0], c.x1[1], c.x1[2]), make_double3(c.v1[0], c.v1[1], c.v1[2])};
        PairClass pc;
        if (!pair_classify(I, J, d[12], c.rce, d[13], c.rphys, S.h, pc)) continue;
        const int slot = atomicAdd(&A.status->events, 1);
        if (slot < A.event_cap) {
            pair_record(A.events + slot, I, J, pc, 1.0 / S.h, c.body + 2, c.id, false);
            A.event_step[slot] = c.step;
            A.event_sys[slot] = c.slot;
        } else {
            atomicOr(&A.status->overflow, 1);
        }
    }
}

template <bool NGF, bool OBL, bool CENTRAL>
void launch_variant(const MvsParticleArgs& a, cudaStream_t s, int threads) {
    auto kern = mvs_particle_kernel<NGF, OBL, CENTRAL>;
    const size_t smem = mvs_particle_smem(a.nb, a.nsteps, a.reset, threads, NGF);
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int npairs = (a.np + 1) / 2;
    int tiles = (npairs + threads - 1) / threads;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (per_sm < 1) per_sm = 1;
    // One CTA slot fewer than the device holds, so that the Big-body CTA of
    // the next chunk (another stream) can start beside this persistent grid.
    int slots = sms * per_sm - 1;
    if (slots < 1) slots = 1;
    const int grid = tiles < slots ? tiles : slots;
    if (grid > 0) kern<<<grid, threads, smem, s>>>(a);
}

}  // namespace

size_t mvs_particle_smem(int nb, int nsteps, int reset, int threads, bool ngf) {
    return sizeof(double) * ((size_t)tab_stride(nb) * (size_t)(nsteps + (reset ? 1 : 0)) +
                             (size_t)Cols::STRIDE * Cols::count(ngf));
}

// Steps fused per launch: the staged tables are kept to ~18 KB so that, with
// the 25.6 KB of per-thread columns, five 128-thread CTAs fit on an SM.
int mvs_max_steps_per_launch(int nb) {
    const size_t budget = 18 * 1024;
    const size_t row = sizeof(double) * (size_t)tab_stride(nb);
    long k = (long)(budget / row) - 1;
    if (k < 1) k = 1;
    if (k > 64) k = 64;
    return (int)k;
}

void launch_mvs_corrector(const MvsBigArgs& big, const CorrectorArgs& a, cudaStream_t s) {
    const int N = big.nmass > big.nbig ? big.nmass : big.nbig;
    const size_t smem = sizeof(double) * ((size_t)12 * 3 * N + N + 16);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(mvs_corrector_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    mvs_corrector_big_kernel<<<1, 128, smem, s>>>(big, a);
    if (a.np <= 0) return;
    const int grid = (a.np + 127) / 128;
    if (a.ngf_on) {
        if (a.obl) mvs_corrector_particle_kernel<true, true><<<grid, 128, 0, s>>>(a);
        else mvs_corrector_particle_kernel<true, false><<<grid, 128, 0, s>>>(a);
    } else {
        if (a.obl) mvs_corrector_particle_kernel<false, true><<<grid, 128, 0, s>>>(a);
        else mvs_corrector_particle_kernel<false, false><<<grid, 128, 0, s>>>(a);
    }
}

void launch_mvs_big_batch(const BatchBigArgs& a, int nsys, int max_nbig, cudaStream_t s) {
    const size_t smem = sizeof(double) * ((size_t)12 * 3 * max_nbig + max_nbig + 16);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(mvs_big_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (nsys > 0) mvs_big_batch_kernel<<<nsys, 32, smem, s>>>(a);
}

void launch_mvs_particles_batch(const BatchParticleArgs& a, cudaStream_t s, int threads) {
    if (a.ntiles <= 0) return;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (a.central) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mvs_particle_batch_kernel<true>, threads, 0);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mvs_particle_batch_kernel<false>, threads, 0);
    }
    if (per_sm < 1) per_sm = 1;
    const int warps = threads / 32;
    const int want = (a.ntiles + warps - 1) / warps;
    const int slots = sms * per_sm;
    const int grid = want < slots ? want : slots;
    if (a.central) mvs_particle_batch_kernel<true><<<grid, threads, 0, s>>>(a);
    else mvs_particle_batch_kernel<false><<<grid, threads, 0, s>>>(a);
}

void launch_classify_batch(const BatchParticleArgs& a, cudaStream_t s) {
    classify_batch_kernel<<<296, 256, 0, s>>>(a);
}

void launch_classify(const ClassifyArgs& a, cudaStream_t s) {
    classify_kernel<<<296, 256, 0, s>>>(a);
}

void launch_mvs_big(const MvsBigArgs& a, cudaStream_t s) {
    const int N = a.nmass > a.nbig ? a.nmass : a.nbig;
    const size_t smem = sizeof(double) * ((size_t)12 * 3 * N + N + 16);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(mvs_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    mvs_big_kernel<<<1, 128, smem, s>>>(a);
}

void launch_mvs_particles(const MvsParticleArgs& a, cudaStream_t s, int threads) {
    const bool ngf = a.ngf_on != 0;
    const bool obl = a.jcen[0] != 0.0 || a.jcen[1] != 0.0 || a.jcen[2] != 0.0;
    const bool cen = a.central != 0;
    if (ngf) {
        if (obl) cen ? launch_variant<true, true, true>(a, s, threads) : launch_variant<true, true, false>(a, s, threads);
        else cen ? launch_variant<true, false, true>(a, s, threads) : launch_variant<true, false, false>(a, s, threads);
    } else {
        if (obl) cen ? launch_variant<false, true, true>(a, s, threads) : launch_variant<false, true, false>(a, s, threads);
        else cen ? launch_variant<false, false, true>(a, s, threads) : launch_variant<false, false, false>(a, s, threads);
    }
}

}  // namespace mb200

// Bulirsch-Stoer kernels (mdt_bs1, mdt_bs2): every statement keeps the
// Fortran's evaluation order so that each level's extrapolated state rounds
// as the CPU's does.
#include <algorithm>
#include "allforce.cuh"
#include "bs.cuh"
#include "mvs.cuh"

namespace mb200 {
namespace {

constexpr unsigned FULLMASK = 0xffffffffu;
constexpr unsigned long long ERR_NONFINITE = 0x7ff0000000000000ull;  // +inf

// The step length of level n and its h2 entry (mercury6_2.for:3285-3287,
// 3476-3479).
template <int VARIANT> __device__ __forceinline__ double level_h(double h0, int n) {
    return VARIANT == 1 ? h0 / (2.0 * double(n)) : h0 / double(n);
}
template <int VARIANT> __device__ __forceinline__ double level_h2(double h0, int n) {
    if (VARIANT == 1) return 0.25 / double(n * n);
    const double h = h0 / double(n);
    return h * h;
}

// The Neville update of mdt_bs1/mdt_bs2 (mercury6_2.for:3352-3366,
// 3545-3560) for level n and j < n: D(j) = tmp1 * D(j + 1) - tmp2 * D(j) with
// tmp0 = 1 / (h2(j) - h2(n)), tmp1 = tmp0 * h2(j + 1), tmp2 = tmp0 * h2(n).
// The coefficients depend on the trial step only, so each CTA evaluates the
// L(L-1)/2 pairs once (the same statements) into co[coef_index(n, j)].
__host__ __device__ constexpr int coef_index(int n, int j) { return (n - 1) * (n - 2) / 2 + j - 1; }
template <int VARIANT> __device__ __forceinline__ void neville_coefficients(double h0, double (*co)[2]) {
    constexpr int L = bs_levels(VARIANT);
    for (int q = threadIdx.x; q < L * (L - 1) / 2; q += blockDim.x) {
        int n = 2;
        while (q >= n * (n - 1) / 2) ++n;
        const int j = q - (n - 1) * (n - 2) / 2 + 1;
        const double h2n = level_h2<VARIANT>(h0, n);
        const double tmp0 = 1.0 / (level_h2<VARIANT>(h0, j) - h2n);
        co[q][0] = tmp0 * level_h2<VARIANT>(h0, j + 1);
        co[q][1] = tmp0 * h2n;
    }
}

__device__ __forceinline__ void level_error(double err, bool finite, unsigned long long* dst) {
    atomicMax(dst, finite ? (unsigned long long)__double_as_longlong(err) : ERR_NONFINITE);
}

// Error term of one body (mercury6_2.for:3372-3378): false if not finite.
__device__ __forceinline__ bool body_error(const double* q, double xscal, double vscal, double& e) {
    for (int c = 0; c < 6; ++c)
        if (!isfinite(q[c])) return false;
    const double tmp1 = fmax(fmax(q[0] * q[0], q[1] * q[1]), q[2] * q[2]);
    const double tmp2 = fmax(fmax(q[3] * q[3], q[4] * q[4]), q[5] * q[5]);
    e = fmax(tmp1 * xscal, tmp2 * vscal);
    return true;
}

// The pair term of mfo_hkce (mercury6_2.for:4875-4894): 1 - K(r) inside rc,
// nothing outside; false when the pair is outside rc.
__device__ __forceinline__ bool hkce_pair(double s2, double rc, double& tmp2) {
    const double rc2 = rc * rc;
    if (!(s2 < rc2)) return false;
    const double s_1 = 1.0 / sqrt(s2);
    const double s_3 = s_1 * s_1 * s_1;
    if (s2 <= 0.01 * rc2) {
        tmp2 = s_3;
    } else {
        const double s = 1.0 / s_1;
        const double q = (s - 0.1 * rc) / (0.9 * rc);
        const double q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3;
        tmp2 = (1.0 - 10.0 * q3 + 15.0 * q4 - 6.0 * q5) * s_3;
    }
    return true;
}

// mfo_hkce's central term (mercury6_2.for:4898-4905).
__device__ __forceinline__ double3 hkce_central(double3 a, const double3 x, double m0) {
    const double s2 = x.x * x.x + x.y * x.y + x.z * x.z;
    const double s_1 = 1.0 / sqrt(s2);
    const double tmp2 = m0 * s_1 * s_1 * s_1;
    a.x = a.x - tmp2 * x.x;
    a.y = a.y - tmp2 * x.y;
    a.z = a.z - tmp2 * x.z;
    return a;
}

// mfo_hkce for body k of the massive set: its pairs with massive partners in
// pair-list order (massless partners, which add exactly zero, are not in its
// list), then the central attraction.
__device__ double3 hkce_force(const BsArgs& A, int k, const double* X) {
    const int N = A.f.nsplit;
    const double* m = A.mbig;
    double3 a = make_double3(0.0, 0.0, 0.0);
    for (int e = A.adj_off[k]; e < A.adj_off[k + 1]; ++e) {
        const int q = A.adj[e].x;
        if (q >= N) continue;
        const bool first = A.adj[e].y == 0;
        const int i = first ? k : q, j = first ? q : k;
        const double dx = X[j] - X[i], dy = X[N + j] - X[N + i], dz = X[2 * N + j] - X[2 * N + i];
        double tmp2;
        if (!hkce_pair(dx * dx + dy * dy + dz * dz, fmax(A.rcrit[i], A.rcrit[j]), tmp2)) continue;
        if (first) {
            const double facj = tmp2 * m[j];
            a.x = a.x + facj * dx;
            a.y = a.y + facj * dy;
            a.z = a.z + facj * dz;
        } else {
            const double faci = tmp2 * m[i];
            a.x = a.x - faci * dx;
            a.y = a.y - faci * dy;
            a.z = a.z - faci * dz;
        }
    }
    return hkce_central(a, make_double3(X[k], X[N + k], X[2 * N + k]), A.f.m0);
}

// Pairs of a massless member kept in its CTA's shared memory for the
// sequence (partner, rc = max(rcrit_i, rcrit_member)); further pairs are read
// from the pair list where they are used.
constexpr int PAIR_CACHE = 4;

// hkce_particle_force with the member's first PAIR_CACHE pairs from the
// lane-strided shared copies ci / crc (npair pairs in all) and the Big bodies
// (x, y, z, m) from the body block B of a table row. The same terms in the
// same order.
__device__ __forceinline__ double3 hkce_member_force(const BsArgs& A, int g, int npair, const int* ci,
                                                     const double* crc, const double3 x, double rcrit_p,
                                                     const double* B) {
    double3 a = make_double3(0.0, 0.0, 0.0);
    auto term = [&](int i, double rc) {
        const double* row = B + 4 * (i - 1);
        const double dx = x.x - row[0], dy = x.y - row[1], dz = x.z - row[2];
        double tmp2;
        if (!hkce_pair(dx * dx + dy * dy + dz * dz, rc, tmp2)) return;
        const double faci = tmp2 * row[3];
        a.x = a.x - faci * dx;
        a.y = a.y - faci * dy;
        a.z = a.z - faci * dz;
    };
    const int nc = npair < PAIR_CACHE ? npair : PAIR_CACHE;
    for (int q = 0; q < nc; ++q) term(ci[32 * q], crc[32 * q]);
    if (npair > PAIR_CACHE)
        for (int e = A.adj_off[g] + PAIR_CACHE; e < A.adj_off[g + 1]; ++e) {
            const int i = A.adj[e].x;
            term(i, fmax(A.rcrit[i], rcrit_p));
        }
    return hkce_central(a, x, A.f.m0);
}

// hkce_particle_force and its derivative along dx (J dx with J = da/dx; the
// partners' positions are fixed: massless members never act on the Big
// bodies). Pair terms: a -= t(s) m_i d with t = s^-3 inside 0.1 rc and
// (1 - K(q)) s^-3 up to rc, so J dx -= m_i [t dx + t'(s)/s (d.dx) d];
// K'(q) = 30 q^2 (1 - q)^2.
__device__ double3 hkce_particle_force_jvp(const BsArgs& A, int g, const double3 x, const double3 dx,
                                           double rcrit_p, const double* T, double3& da) {
    double3 a = make_double3(0.0, 0.0, 0.0);
    da = a;
    for (int e = A.adj_off[g]; e < A.adj_off[g + 1]; ++e) {
        const int i = A.adj[e].x;
        const double* row = T + FT_HEAD + 4 * (i - 1);
        const double ex = x.x - row[0], ey = x.y - row[1], ez = x.z - row[2];
        const double s2 = ex * ex + ey * ey + ez * ez;
        const double rc = fmax(A.rcrit[i], rcrit_p);
        double tmp2;
        if (!hkce_pair(s2, rc, tmp2)) continue;
        const double s_1 = 1.0 / sqrt(s2);
        const double s_3 = s_1 * s_1 * s_1;
        double t1;  // t'(s) / s
        if (s2 <= 0.01 * rc * rc) {
            t1 = -3.0 * s_3 * s_1 * s_1;
        } else {
            const double s = 1.0 / s_1;
            const double q = (s - 0.1 * rc) / (0.9 * rc);
            const double q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3;
            const double K = 10.0 * q3 - 15.0 * q4 + 6.0 * q5;
            const double Kq = 30.0 * q2 * (1.0 - q) * (1.0 - q);
            t1 = (-Kq / (0.9 * rc) * s_3 - 3.0 * (1.0 - K) * s_3 * s_1) * s_1;
        }
        const double mi = row[3];
        const double faci = tmp2 * mi;
        a.x = a.x - faci * ex;
        a.y = a.y - faci * ey;
        a.z = a.z - faci * ez;
        const double ed = (ex * dx.x + ey * dx.y + ez * dx.z) * t1;
        da.x -= mi * (tmp2 * dx.x + ed * ex);
        da.y -= mi * (tmp2 * dx.y + ed * ey);
        da.z -= mi * (tmp2 * dx.z + ed * ez);
    }
    const double s2 = x.x * x.x + x.y * x.y + x.z * x.z;
    const double s_1 = 1.0 / sqrt(s2);
    const double s_3 = s_1 * s_1 * s_1;
    const double m0 = A.f.m0;
    const double xd = (x.x * dx.x + x.y * dx.y + x.z * dx.z) * 3.0 * s_3 * s_1 * s_1;
    da.x -= m0 * (s_3 * dx.x - xd * x.x);
    da.y -= m0 * (s_3 * dx.y - xd * x.y);
    da.z -= m0 * (s_3 * dx.z - xd * x.z);
    return hkce_central(a, x, m0);
}

// ------------------------------------------------------------ massive set
// One force call of the massive set into `out` and table row T; mb and ngf
// are the set's masses and non-gravitational constants, head a shared copy of
// the row's head for the set's own forces, PT shared scratch for the terms
// computed in parallel (null: the sequential loops).
template <bool HKCE>
__device__ void massive_call(const BsArgs& A, const double* X, const double* V, double* out, double* T,
                             DeviceStatus* st, const double* mb, const double* ngf, double* head, double* PT) {
    const ForceCfg& f = A.f;
    const int N = f.nsplit;
    __syncthreads();
    if (HKCE) {
        for (int k = 1 + threadIdx.x; k < N; k += blockDim.x) {
            if (k < f.nbig) {
                double* row = T + FT_HEAD + 4 * (k - 1);
                row[0] = X[k]; row[1] = X[N + k]; row[2] = X[2 * N + k]; row[3] = mb[k];
            }
            const double3 a = hkce_force(A, k, X);
            out[k] = a.x; out[N + k] = a.y; out[2 * N + k] = a.z;
        }
        __syncthreads();
        return;
    }
    if (PT) {
        massive_terms(X, mb, f, PT, st);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (PT) row_head_terms(PT, f, T);
        else row_head(X, mb, f, T);
        for (int q = 0; q < FT_HEAD; ++q) head[q] = T[q];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        if (k >= 1 && k < f.nbig) {
            double* row = T + FT_HEAD + 4 * (k - 1);
            row[0] = X[k]; row[1] = X[N + k]; row[2] = X[2 * N + k]; row[3] = mb[k];
        }
        if (k < 1) continue;
        const double3 a = PT ? massive_allforce_terms(k, X, V, mb, ngf, head, f, PT, st)
                             : massive_allforce(k, X, V, mb, ngf, head, f, st);
        out[k] = a.x; out[N + k] = a.y; out[2 * N + k] = a.z;
    }
    __syncthreads();
}

// The massive set through one level per CTA (level n = blockIdx.x + 1): the
// levels of a BS step are independent given the start-of-step state and force,
// so the CTAs run side by side and the step's critical path is its longest
// level instead of the sum of all levels. Each CTA keeps its states,
// accelerations, the starting state, masses and non-gravitational constants
// in shared memory, writes the table rows of its level's force calls and its
// raw level state D(n) to A.draw; bs_massive_extrap_kernel then runs the
// Neville updates in level order. The start-of-step force is computed by
// every CTA (the same statements), level 1's writing table row 0 and the
// others a private row.
template <int VARIANT, bool HKCE> __global__ void __launch_bounds__(256) bs_massive_level_kernel(BsArgs A) {
    extern __shared__ double sm[];
    double h0 = A.h0;
    if (A.ctl) {
        if (A.ctl->stop) return;
        h0 = A.ctl->h0;
    }
    const int N = A.f.nsplit, tid = threadIdx.x, nt = blockDim.x, n = blockIdx.x + 1;
    const int stride = force_row(A.f.nbig - 1);
    if (A.bx_pre && n == 1)
        for (int q = tid; q < 6 * N; q += nt) A.bx_pre[q] = A.bx[q];
    double* X = sm;
    double* V = sm + 3 * N;
    double* XE = sm + 6 * N;
    double* VE = sm + 9 * N;
    double* Acc = sm + 12 * N;
    double* A0 = sm + 15 * N;
    double* B = sm + 18 * N;
    double* C = sm + 21 * N;
    double* p = sm + (size_t)BS_LEVEL_ROWS * N;
    for (int q = tid; q < 6 * N; q += nt) p[q] = A.bx[q];
    for (int q = tid; q < N; q += nt) p[6 * N + q] = A.mbig[q];
    for (int q = tid; q < 5 * N; q += nt) p[7 * N + q] = A.ngfbig[q];
    const double* X0 = p;
    const double* V0 = p + 3 * N;
    const double* mb = p + 6 * N;
    const double* ngf = p + 7 * N;
    double* PT = massive_par_scratch(N) ? p + 12 * N : nullptr;
    __syncthreads();
    __shared__ double head[FT_HEAD];
    auto call = [&](const double* Xc, const double* Vc, double* out, double* T, DeviceStatus* st) {
        massive_call<HKCE>(A, Xc, Vc, out, T, st, mb, ngf, head, PT);
    };
    for (int k = tid; k < N; k += nt)
        for (int c = 0; c < 3; ++c) {
            const int z = c * N + k;
            X[z] = X0[z]; V[z] = V0[z]; XE[z] = X0[z]; VE[z] = V0[z];
        }
    call(X0, V0, A0, n == 1 ? A.table : A.tscr + (size_t)(n - 2) * stride, &A.lvst[0]);
    int row = 1;
    for (int m = 1; m < n; ++m) row += bs_level_forces(VARIANT, m);
    DeviceStatus* st = &A.lvst[n];
    const double h = level_h<VARIANT>(h0, n);
    const double h2n = level_h2<VARIANT>(h0, n);
    double* Dn = A.draw + (size_t)(n - 1) * 6 * N;
    if (VARIANT == 1) {
        const double hx2 = h * 2.0;
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                X[z] = X0[z] + h * V0[z];
                V[z] = V0[z] + h * A0[z];
            }
        call(X, V, Acc, A.table + (size_t)(row++) * stride, st);
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                XE[z] = X0[z] + hx2 * V[z];
                VE[z] = V0[z] + hx2 * Acc[z];
            }
        for (int j = 2; j <= n; ++j) {
            call(XE, VE, Acc, A.table + (size_t)(row++) * stride, st);
            for (int k = 1 + tid; k < N; k += nt)
                for (int c = 0; c < 3; ++c) {
                    const int z = c * N + k;
                    X[z] = X[z] + hx2 * VE[z];
                    V[z] = V[z] + hx2 * Acc[z];
                }
            call(X, V, Acc, A.table + (size_t)(row++) * stride, st);
            for (int k = 1 + tid; k < N; k += nt)
                for (int c = 0; c < 3; ++c) {
                    const int z = c * N + k;
                    XE[z] = XE[z] + hx2 * V[z];
                    VE[z] = VE[z] + hx2 * Acc[z];
                }
        }
        call(XE, VE, Acc, A.table + (size_t)(row++) * stride, st);
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                Dn[z] = 0.5 * (XE[z] + X[z] + h * VE[z]);
                Dn[3 * N + z] = 0.5 * (VE[z] + V[z] + h * Acc[z]);
            }
    } else {
        const double hby2 = 0.5 * h, h2by2 = 0.5 * h2n;
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                B[z] = 0.5 * A0[z];
                C[z] = 0.0;
                XE[z] = h2by2 * A0[z] + h * V0[z] + X0[z];
            }
        for (int j = 2; j <= n; ++j) {
            call(XE, V0, Acc, A.table + (size_t)(row++) * stride, st);
            const double tmp0 = h * double(j);
            for (int k = 1 + tid; k < N; k += nt)
                for (int c = 0; c < 3; ++c) {
                    const int z = c * N + k;
                    B[z] = B[z] + Acc[z];
                    C[z] = C[z] + B[z];
                    XE[z] = h2n * C[z] + h2by2 * A0[z] + tmp0 * V0[z] + X0[z];
                }
        }
        call(XE, V0, Acc, A.table + (size_t)(row++) * stride, st);
        for (int k = 1 + tid; k < N; k += nt)
            for (int c = 0; c < 3; ++c) {
                const int z = c * N + k;
                Dn[z] = XE[z];
                Dn[3 * N + z] = h * B[z] + hby2 * Acc[z] + V0[z];
            }
    }
}

// The massive set's extrapolation in level order (mercury6_2.for:3352-3378)
// by the calling block: one thread per (body, component) takes its raw level
// states D(1..L) through the Neville updates in registers, writes each
// level's candidate sum from level 4 on, and parks D(1) after level n in
// level n's raw slot; then one thread per (body, level) adds the body's error
// term to the level's maximum. Per (body, component) the same statements in
// the same order as a level loop; a maximum does not depend on the order.
template <int VARIANT> __device__ void massive_extrap_block(const BsArgs& A, const double (*co)[2]) {
    constexpr int L = bs_levels(VARIANT);
    const int N = A.f.nsplit, nb1 = N - 1, M = 6 * nb1, tid = threadIdx.x, nt = blockDim.x;
    double* raw = A.draw;
    for (int q = tid; q < M; q += nt) {
        const int c = q / nb1, k = 1 + q % nb1;
        double D[L];
#pragma unroll
        for (int n = 0; n < L; ++n) D[n] = raw[(size_t)n * 6 * N + c * N + k];
#pragma unroll
        for (int n = 1; n <= L; ++n) {
#pragma unroll
            for (int j = n - 1; j >= 1; --j) {
                // read where used: hoisted out of the (body, component) loop
                // the 66 coefficient pairs would not fit in registers
                const volatile double* cj = co[coef_index(n, j)];
                D[j - 1] = cj[0] * D[j] - cj[1] * D[j - 1];
            }
            if (n > 3) {
                double sum = D[0];
#pragma unroll
                for (int j = 2; j <= n; ++j) sum = sum + D[j - 1];
                A.bcand[(size_t)(n - 4) * 6 * N + c * N + k] = sum;
            }
            raw[(size_t)(n - 1) * 6 * N + c * N + k] = D[0];
        }
    }
    __syncthreads();
    const double* X0 = A.bx;
    const double* V0 = A.bx + 3 * N;
    for (int q = tid; q < nb1 * (L - 3); q += nt) {
        const int k = 1 + q % nb1, n = 4 + q / nb1;
        const double tmp1 = X0[k] * X0[k] + X0[N + k] * X0[N + k] + X0[2 * N + k] * X0[2 * N + k];
        const double tmp2 = V0[k] * V0[k] + V0[N + k] * V0[N + k] + V0[2 * N + k] * V0[2 * N + k];
        const double xscal = 1.0 / fmax(tmp1, 1e-300);
        const double vscal = 1.0 / fmax(tmp2, 1e-300);
        double q6[6];
        for (int c = 0; c < 6; ++c) q6[c] = raw[(size_t)(n - 1) * 6 * N + c * N + k];
        double e = 0.0;
        const bool finite = body_error(q6, xscal, vscal, e);
        level_error(e, finite, &A.errs[n]);
    }
}

// The massive set's extrapolation as a launch of its own (one CTA).
template <int VARIANT> __global__ void __launch_bounds__(256) bs_massive_extrap_kernel(BsArgs A) {
    constexpr int L = bs_levels(VARIANT);
    __shared__ double co[L * (L - 1) / 2][2];
    double h0 = A.h0;
    if (A.ctl) {
        if (A.ctl->stop) return;
        h0 = A.ctl->h0;
    }
    neville_coefficients<VARIANT>(h0, co);
    __syncthreads();
    massive_extrap_block<VARIANT>(A, co);
}

// ------------------------------------------------------------ particles
// Thirty-two particle slots per CTA, one lane each; warp w computes the raw
// states D(n) of levels w + 1 and L - w (n + (L + 1 - n) force calls per warp,
// balanced) into shared memory, from the start-of-step force that warp 0
// computes. Then warp w takes components w, w + (warps), ... of every
// particle through the Neville updates in level order, in registers, with the
// coefficients computed once per CTA, writing each level's candidate
// component and the error inputs; last, the warps share the levels' error
// maxima. Per particle and component the same statements, in the same order,
// as a level loop would run them.
// With mfo_hkce (encounter members: a few pairs each) three CTAs share an SM,
// so that a subsystem of up to 444 x 32 members runs in one wave.
//
// Levels LO..HI only (LO > 1 or HI < L): the plain mdt_bs2 step runs levels
// 1..8 first and 9..12 only when none of 4..8 passed (its step control aims
// at level 7), so that most steps make 36 of the 78 force calls. The first
// stage keeps each particle's Neville tableau after level HI in A.ptab and
// the second resumes from it; the statements and their order per particle
// and component are those of one pass over all levels.
// Registers are held to ~170 (the full sequence's 192 threads twice per SM).
template <int VARIANT, bool HKCE, int LO = 1, int HI = bs_levels(VARIANT)>
__global__ void __launch_bounds__((HI - LO + 1) * 16, HKCE ? 3 : 384 / ((HI - LO + 1) * 16))
    bs_particle_kernel(BsArgs A) {
    constexpr int L = bs_levels(VARIANT);
    constexpr int NW = (HI - LO + 1) / 2;   // warps of the CTA: levels LO + w and HI - w
    static_assert((HI - LO + 1) % 2 == 0, "levels come in pairs");
    __shared__ double dsm[HI][6][32];
    __shared__ double a0sm[3][32];
    __shared__ double co[L * (L - 1) / 2][2];
    // encounter members: their first pairs, and (A.stage_bodies) the Big
    // bodies' (x, y, z, m) of every table row, [rows][4 nb]
    __shared__ int pair_n[32];
    __shared__ int pair_i[PAIR_CACHE * 32];
    __shared__ double pair_rc[PAIR_CACHE * 32];
    extern __shared__ double staged[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double h0 = A.h0;
    if (A.ctl) {
        if (A.ctl->stop) return;
        h0 = A.ctl->h0;
    }
    neville_coefficients<VARIANT>(h0, co);
    if (A.fuse_extrap && blockIdx.x == gridDim.x - 1) {
        // the launch's last CTA: the massive set's extrapolation
        __syncthreads();
        massive_extrap_block<VARIANT>(A, co);
        return;
    }
    const int p = blockIdx.x * 32 + lane;
    const bool ok = p < A.np && A.perm[p] < A.active_np;
    const int nb = A.f.nbig - 1, stride = force_row(nb), S = A.npcap;
    double3 x0 = make_double3(0.0, 0.0, 0.0), v0 = x0;
    double mj = 0.0, g5[5] = {0, 0, 0, 0, 0};
    // the encounter subsystem (BS2 only): mfo_hkce from the member's pairs
    constexpr bool hkce = VARIANT == 2 && HKCE;
    const bool stage = hkce && A.stage_bodies;
    const int bw = 4 * nb;   // body block of a table row
    int g = 0;
    double rcrit_p = 0.0;
    if (hkce) {
        if (ok) {
            g = A.f.nsplit + A.perm[p];
            rcrit_p = A.pconst[(size_t)PC_RCRIT * S + p];
        }
        if (w == 0) {
            const int e0 = ok ? A.adj_off[g] : 0, e1 = ok ? A.adj_off[g + 1] : 0;
            pair_n[lane] = e1 - e0;
            for (int q = 0; q < PAIR_CACHE && e0 + q < e1; ++q) {
                const int i = A.adj[e0 + q].x;
                pair_i[32 * q + lane] = i;
                pair_rc[32 * q + lane] = fmax(A.rcrit[i], rcrit_p);
            }
        }
        if (stage)
            for (int q = threadIdx.x; q < bs_rows(VARIANT) * bw; q += blockDim.x) {
                const int r = q / bw;
                staged[q] = A.table[(size_t)r * stride + FT_HEAD + (q - r * bw)];
            }
        __syncthreads();
    }
    const int npair = hkce ? pair_n[lane] : 0;
    auto force = [&](const double3 x, const double3 v, int r, DeviceStatus* st) {
        if (hkce)
            return hkce_member_force(A, g, npair, pair_i + lane, pair_rc + lane, x, rcrit_p,
                                     stage ? staged + (size_t)r * bw : A.table + (size_t)r * stride + FT_HEAD);
        return particle_allforce(x, v, A.table + (size_t)r * stride, nb, A.f, mj, g5, st);
    };
    if (ok) {
        x0 = make_double3(A.px[p], A.px[S + p], A.px[2 * S + p]);
        v0 = make_double3(A.px[3 * S + p], A.px[4 * S + p], A.px[5 * S + p]);
        if (!hkce) {
            mj = A.pconst[p];
            for (int c = 0; c < 5; ++c) g5[c] = A.pconst[(3 + c) * (size_t)S + p];
        }
        if (w == 0) {
            const double3 a = force(x0, v0, 0, &A.lvst[0]);
            a0sm[0][lane] = a.x;
            a0sm[1][lane] = a.y;
            a0sm[2][lane] = a.z;
        }
    }
    __syncthreads();
    const double3 a0 = ok ? make_double3(a0sm[0][lane], a0sm[1][lane], a0sm[2][lane]) : make_double3(0.0, 0.0, 0.0);
#pragma unroll 1
    for (int half = 0; half < 2 && ok; ++half) {
        const int n = half == 0 ? LO + w : HI - w;
        int row = 1;
        for (int m = 1; m < n; ++m) row += bs_level_forces(VARIANT, m);
        DeviceStatus* st = &A.lvst[n];
        const double h = level_h<VARIANT>(h0, n);
        const double h2n = level_h2<VARIANT>(h0, n);
        auto call = [&](const double3 x, const double3 v) { return force(x, v, row++, st); };
        auto D = [&](int c) -> double& { return dsm[n - 1][c][lane]; };
        if (VARIANT == 1) {
            const double hx2 = h * 2.0;
            double3 x = make_double3(x0.x + h * v0.x, x0.y + h * v0.y, x0.z + h * v0.z);
            double3 v = make_double3(v0.x + h * a0.x, v0.y + h * a0.y, v0.z + h * a0.z);
            double3 a = call(x, v);
            double3 xe = make_double3(x0.x + hx2 * v.x, x0.y + hx2 * v.y, x0.z + hx2 * v.z);
            double3 ve = make_double3(v0.x + hx2 * a.x, v0.y + hx2 * a.y, v0.z + hx2 * a.z);
#pragma unroll 1
            for (int j = 2; j <= n; ++j) {
                a = call(xe, ve);
                x = make_double3(x.x + hx2 * ve.x, x.y + hx2 * ve.y, x.z + hx2 * ve.z);
                v = make_double3(v.x + hx2 * a.x, v.y + hx2 * a.y, v.z + hx2 * a.z);
                a = call(x, v);
                xe = make_double3(xe.x + hx2 * v.x, xe.y + hx2 * v.y, xe.z + hx2 * v.z);
                ve = make_double3(ve.x + hx2 * a.x, ve.y + hx2 * a.y, ve.z + hx2 * a.z);
            }
            a = call(xe, ve);
            D(0) = 0.5 * (xe.x + x.x + h * ve.x);
            D(1) = 0.5 * (xe.y + x.y + h * ve.y);
            D(2) = 0.5 * (xe.z + x.z + h * ve.z);
            D(3) = 0.5 * (ve.x + v.x + h * a.x);
            D(4) = 0.5 * (ve.y + v.y + h * a.y);
            D(5) = 0.5 * (ve.z + v.z + h * a.z);
        } else {
            const double hby2 = 0.5 * h, h2by2 = 0.5 * h2n;
            double3 b = make_double3(0.5 * a0.x, 0.5 * a0.y, 0.5 * a0.z);
            double3 c = make_double3(0.0, 0.0, 0.0);
            double3 xe = make_double3(h2by2 * a0.x + h * v0.x + x0.x, h2by2 * a0.y + h * v0.y + x0.y,
                                      h2by2 * a0.z + h * v0.z + x0.z);
#pragma unroll 1
            for (int j = 2; j <= n; ++j) {
                const double3 a = call(xe, v0);
                const double tmp0 = h * double(j);
                b = make_double3(b.x + a.x, b.y + a.y, b.z + a.z);
                c = make_double3(c.x + b.x, c.y + b.y, c.z + b.z);
                xe = make_double3(h2n * c.x + h2by2 * a0.x + tmp0 * v0.x + x0.x,
                                  h2n * c.y + h2by2 * a0.y + tmp0 * v0.y + x0.y,
                                  h2n * c.z + h2by2 * a0.z + tmp0 * v0.z + x0.z);
            }
            const double3 a = call(xe, v0);
            D(0) = xe.x;
            D(1) = xe.y;
            D(2) = xe.z;
            D(3) = h * b.x + hby2 * a.x + v0.x;
            D(4) = h * b.y + hby2 * a.y + v0.y;
            D(5) = h * b.z + hby2 * a.z + v0.z;
        }
    }
    __syncthreads();
    // Neville updates in level order, one component per warp pass: D(j) of the
    // lane's particle in registers; after level n (n > 3) the candidate
    // component D(1) + ... + D(n) goes out and D(1) stays in dsm for the error
    if (ok) {
        for (int c = w; c < 6; c += NW) {
            double D[HI];
            // levels before LO: their tableau as the first stage left it
#pragma unroll
            for (int n = 0; n < LO - 1; ++n) D[n] = A.ptab[((size_t)n * 6 + c) * S + p];
#pragma unroll
            for (int n = LO - 1; n < HI; ++n) D[n] = dsm[n][c][lane];
#pragma unroll
            for (int n = LO; n <= HI; ++n) {
#pragma unroll
                for (int j = n - 1; j >= 1; --j) {
                    const double* cj = co[coef_index(n, j)];
                    D[j - 1] = cj[0] * D[j] - cj[1] * D[j - 1];
                }
                if (n > 3) {
                    double sum = D[0];
#pragma unroll
                    for (int j = 2; j <= n; ++j) sum = sum + D[j - 1];
                    A.pcand[(size_t)(n - 4) * 6 * S + (size_t)c * S + p] = sum;
                    dsm[n - 1][c][lane] = D[0];
                }
            }
            if (HI < L) {
#pragma unroll
                for (int n = 0; n < HI; ++n) A.ptab[((size_t)n * 6 + c) * S + p] = D[n];
            }
        }
    }
    __syncthreads();
    double xscal = 0.0, vscal = 0.0;
    if (ok) {
        const double tmp1 = x0.x * x0.x + x0.y * x0.y + x0.z * x0.z;
        const double tmp2 = v0.x * v0.x + v0.y * v0.y + v0.z * v0.z;
        xscal = 1.0 / fmax(tmp1, 1e-300);
        vscal = 1.0 / fmax(tmp2, 1e-300);
    }
    // each level's error maximum (mercury6_2.for:3372-3378), levels shared by the warps
    for (int n = (LO > 4 ? LO : 4) + w; n <= HI; n += NW) {
        double emax = 0.0;
        int bad = 0;
        if (ok) {
            double q[6];
            for (int c = 0; c < 6; ++c) q[c] = dsm[n - 1][c][lane];
            double e;
            if (body_error(q, xscal, vscal, e)) emax = e;
            else bad = 1;
        }
        for (int o = 16; o; o >>= 1) {
            emax = fmax(emax, __shfl_xor_sync(FULLMASK, emax, o));
            bad |= __shfl_xor_sync(FULLMASK, bad, o);
        }
        if (lane == 0 && (emax > 0.0 || bad)) level_error(emax, !bad, &A.errs[n]);
    }
}

// Tangent of one accepted BS2 step of the encounter subsystem for its
// massless members: thread (slot p, direction d) pushes column d of the
// slot's accumulated 6x6 Jacobian tg (entry (d * 6 + r) * npcap + p holds
// d state_r / d start_d) through levels 1..levels and the Neville
// extrapolation that produced the accepted state: the particle kernel's
// statements differentiated, with the step control's choices fixed. The
// primal midpoint states are recomputed alongside from the same table rows.
__global__ void __launch_bounds__(64) bs2_tangent_kernel(BsArgs A, int levels, double* tg) {
    extern __shared__ double dcol[];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = q / 6, d = q - 6 * p;
    if (p >= A.np) return;
    const int nb = A.f.nbig - 1, stride = force_row(nb), S = A.npcap, T = blockDim.x;
    auto D = [&](int j, int c) -> double& { return dcol[((j - 1) * 6 + c) * T + threadIdx.x]; };
    const double3 x0 = make_double3(A.px[p], A.px[S + p], A.px[2 * S + p]);
    const double3 v0 = make_double3(A.px[3 * S + p], A.px[4 * S + p], A.px[5 * S + p]);
    const int g = A.f.nsplit + A.perm[p];
    const double rcrit_p = A.pconst[(size_t)PC_RCRIT * S + p];
    double* col = tg + (size_t)(6 * d) * S + p;
    const double3 dx0 = make_double3(col[0], col[S], col[2 * (size_t)S]);
    const double3 dv0 = make_double3(col[3 * (size_t)S], col[4 * (size_t)S], col[5 * (size_t)S]);
    double3 da0;
    const double3 a0 = hkce_particle_force_jvp(A, g, x0, dx0, rcrit_p, A.table, da0);
    int row = 1;
#pragma unroll 1
    for (int n = 1; n <= levels; ++n) {
        const double h = level_h<2>(A.h0, n);
        const double h2n = level_h2<2>(A.h0, n);
        const double hby2 = 0.5 * h, h2by2 = 0.5 * h2n;
        double3 b = make_double3(0.5 * a0.x, 0.5 * a0.y, 0.5 * a0.z);
        double3 c = make_double3(0.0, 0.0, 0.0);
        double3 xe = make_double3(h2by2 * a0.x + h * v0.x + x0.x, h2by2 * a0.y + h * v0.y + x0.y,
                                  h2by2 * a0.z + h * v0.z + x0.z);
        double3 db = make_double3(0.5 * da0.x, 0.5 * da0.y, 0.5 * da0.z);
        double3 dc = make_double3(0.0, 0.0, 0.0);
        double3 dxe = make_double3(h2by2 * da0.x + h * dv0.x + dx0.x, h2by2 * da0.y + h * dv0.y + dx0.y,
                                   h2by2 * da0.z + h * dv0.z + dx0.z);
#pragma unroll 1
        for (int j = 2; j <= n; ++j) {
            double3 da;
            const double3 a = hkce_particle_force_jvp(A, g, xe, dxe, rcrit_p, A.table + (size_t)(row++) * stride, da);
            const double tmp0 = h * double(j);
            b = make_double3(b.x + a.x, b.y + a.y, b.z + a.z);
            c = make_double3(c.x + b.x, c.y + b.y, c.z + b.z);
            xe = make_double3(h2n * c.x + h2by2 * a0.x + tmp0 * v0.x + x0.x,
                              h2n * c.y + h2by2 * a0.y + tmp0 * v0.y + x0.y,
                              h2n * c.z + h2by2 * a0.z + tmp0 * v0.z + x0.z);
            db = make_double3(db.x + da.x, db.y + da.y, db.z + da.z);
            dc = make_double3(dc.x + db.x, dc.y + db.y, dc.z + db.z);
            dxe = make_double3(h2n * dc.x + h2by2 * da0.x + tmp0 * dv0.x + dx0.x,
                               h2n * dc.y + h2by2 * da0.y + tmp0 * dv0.y + dx0.y,
                               h2n * dc.z + h2by2 * da0.z + tmp0 * dv0.z + dx0.z);
        }
        double3 da;
        hkce_particle_force_jvp(A, g, xe, dxe, rcrit_p, A.table + (size_t)(row++) * stride, da);
        D(n, 0) = dxe.x;
        D(n, 1) = dxe.y;
        D(n, 2) = dxe.z;
        D(n, 3) = h * db.x + hby2 * da.x + dv0.x;
        D(n, 4) = h * db.y + hby2 * da.y + dv0.y;
        D(n, 5) = h * db.z + hby2 * da.z + dv0.z;
#pragma unroll 1
        for (int j = n - 1; j >= 1; --j) {
            const double tmp0 = 1.0 / (level_h2<2>(A.h0, j) - h2n);
            const double tmp1 = tmp0 * level_h2<2>(A.h0, j + 1);
            const double tmp2 = tmp0 * h2n;
            for (int c6 = 0; c6 < 6; ++c6) D(j, c6) = tmp1 * D(j + 1, c6) - tmp2 * D(j, c6);
        }
    }
    for (int c6 = 0; c6 < 6; ++c6) {
        double s = D(1, c6);
        for (int j = 2; j <= levels; ++j) s = s + D(j, c6);
        col[(size_t)c6 * S] = s;
    }
}

__global__ void __launch_bounds__(128) bs_commit_kernel(BsCommitArgs A) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = A.nsplit, S = A.npcap;
    const int level_cand = A.cand;
    if (q < N) {
        if (q == 0) {
            for (int c = 0; c < 9; ++c) A.bx_out[c * N] = A.bx[c * N];
            return;
        }
        const double* cand = A.bcand + (size_t)level_cand * 6 * N;
        for (int c = 0; c < 6; ++c) A.bx_out[c * N + q] = cand[c * N + q];
        for (int c = 6; c < 9; ++c) A.bx_out[c * N + q] = 0.0;
        return;
    }
    const int p = q - N;
    if (p >= A.np) return;
    if (A.perm[p] >= A.active_np) {
        for (int c = 0; c < 9; ++c) A.px_out[(size_t)c * S + p] = A.px[(size_t)c * S + p];
        return;
    }
    const double* cand = A.pcand + (size_t)level_cand * 6 * S;
    for (int c = 0; c < 6; ++c) A.px_out[(size_t)c * S + p] = cand[(size_t)c * S + p];
    for (int c = 6; c < 9; ++c) A.px_out[(size_t)c * S + p] = 0.0;
}

// mdt_bs2's decision after one attempt of the encounter subsystem
// (mercury6_2.for:3568-3596; the host loop of mdt_hkce, 3884-3937) applied
// to the control block c: the first level n > 3 whose error maximum is <=
// tol^2 is accepted, else the step is halved; after an acceptance the next
// trial step (x0.55 for a level >= 8, x1.3 below 7), the local clock, the
// substep count and the clipping of the next substep to the subsystem's end.
// Returns the accepted level (0: rejected, stopped or failed). A pure
// function of its inputs, so every thread of a launch reaches the same
// decision.
__device__ __forceinline__ int enc_decide(EncCtl& c, const unsigned long long* errs, const DeviceStatus* lv) {
    if (c.stop) {
        c.accepted = 0;
        return 0;
    }
    constexpr int L = 12;
    const int fails = FAULT_NGF | FAULT_COINCIDENT;
    // every level's maximum and fault word first: independent loads in flight together
    unsigned long long em[L + 1];
    int fw[L + 1];
#pragma unroll
    for (int n = 0; n <= L; ++n) {
        em[n] = errs[n];
        fw[n] = lv[n].fault;
    }
    c.attempts += 1;
    int accepted = 0, error = 0;
    long long forces = 0;
    if (fw[0] & fails) error = ENC_ERR_FORCE;
#pragma unroll
    for (int n = 1; n <= L; ++n) {
        if (error || accepted) break;
        forces += n;
        if (fw[n] & fails) {
            error = ENC_ERR_FORCE;
            break;
        }
        if (n <= 3) continue;
        const double e = __longlong_as_double((long long)em[n]);
        if (!isfinite(e)) {
            error = ENC_ERR_NONFINITE;
            break;
        }
        if (e <= c.tol * c.tol) accepted = n;
    }
    c.forces += forces;
    if (error) {
        c.error = error;
        c.stop = 1;
        c.accepted = 0;
        return 0;
    }
    if (!accepted) {
        c.accepted = 0;
        c.h0 = c.h0 * 0.5;
        if (c.tlocal + c.h0 == c.tlocal) {
            c.error = ENC_ERR_ADVANCE;
            c.stop = 1;
        }
        return 0;
    }
    c.accepted = accepted;
    const double hdid = c.h0;
    double hnext = c.h0;
    if (accepted >= 8) hnext = hnext * 0.55;
    if (accepted < 7) hnext = hnext * 1.3;
    c.hdid = hdid;
    c.tlocal = c.tlocal + hdid;
    if (c.substeps >= c.step_cap) {
        c.error = ENC_ERR_STEPS;
        c.stop = 1;
        c.accepted = 0;
        return 0;
    }
    c.substeps += 1;
    if (!((c.tlocal - c.h) * c.h < 0.0)) {
        c.stop = 1;
        return accepted;
    }
    // the next substep: hrec before the clip to the subsystem's end
    const double tmp0 = fabs(c.h) - fabs(c.tlocal);
    c.hrec = hnext;
    if (fabs(hnext) > tmp0) hnext = copysign(tmp0, c.h);
    c.h0 = hnext;
    c.forces += 1;   // the next substep's start-of-step force
    if (c.tlocal + c.h0 == c.tlocal) {
        c.error = ENC_ERR_ADVANCE;
        c.stop = 1;
    }
    return accepted;
}

// Everything after one attempt of the encounter subsystem, in one launch:
// the decision (every thread), the new control block and the cleared level
// maxima of the next attempt (thread 0 of block 0), and after an acceptance
// the commit of the accepted level in place with mce_stat between the
// attempt's start and the committed state (mercury6_2.for:1765-1918): the
// Big bodies' boxes and end states in each block's shared memory, the
// massive pairs and the massive set's commit in block 0 (from the start
// state the level kernel kept), one particle slot per thread with its box
// test and classification inline. Records carry the substep index.
__global__ void __launch_bounds__(128) enc_post_kernel(EncPostArgs A) {
    extern __shared__ double sh[];
    EncCtl c = *A.ctl_in;
    const int acc = enc_decide(c, A.errs, A.lvst);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (acc) c.tstep[c.substeps - 1] = c.time + c.tlocal;
        *A.ctl_out = c;
        for (int n = 0; n < 13; ++n) {
            A.errs_next[n] = 0ull;
            A.lvst_next[n] = DeviceStatus{};
        }
    }
    if (!acc) return;
    const int N = A.nsplit, nb = A.nbig - 1, S = A.npcap;
    const double h = c.hdid, hm1 = 1.0 / h;
    const int step = c.substeps - 1;
    const double* bpost = A.bcand + (size_t)(acc - 4) * 6 * N;
    const double* ppost = A.pcand + (size_t)(acc - 4) * 6 * S;
    auto ends = [&](int k) {
        return PairEnds{make_double3(A.bx_pre[k], A.bx_pre[N + k], A.bx_pre[2 * N + k]),
                        make_double3(A.bx_pre[3 * N + k], A.bx_pre[4 * N + k], A.bx_pre[5 * N + k]),
                        make_double3(bpost[k], bpost[N + k], bpost[2 * N + k]),
                        make_double3(bpost[3 * N + k], bpost[4 * N + k], bpost[5 * N + k])};
    };
    auto box = [&](int k, double* bx) {
        const PairEnds E = ends(k);
        const double pad = A.rcebig[k] * 1.2;
        double lo, hi;
        box_extent(E.x0.x, E.x1.x, E.v0.x, E.v1.x, h, lo, hi);
        bx[0] = lo - pad;
        bx[1] = hi + pad;
        box_extent(E.x0.y, E.x1.y, E.v0.y, E.v1.y, h, lo, hi);
        bx[2] = lo - pad;
        bx[3] = hi + pad;
    };
    double* sbox = sh;                                  // [nb][4]
    double* sdet = sh + 4 * (size_t)(nb > 0 ? nb : 1);  // [nb][TAB_DETAIL]
    for (int k = 1 + threadIdx.x; k < A.nbig; k += blockDim.x) {
        box(k, sbox + 4 * (k - 1));
        const PairEnds E = ends(k);
        double* d = sdet + (size_t)(k - 1) * TAB_DETAIL;
        const double3 q[4] = {E.x0, E.v0, E.x1, E.v1};
        for (int w = 0; w < 4; ++w) {
            d[3 * w] = q[w].x;
            d[3 * w + 1] = q[w].y;
            d[3 * w + 2] = q[w].z;
        }
        d[12] = A.rcebig[k];
        d[13] = A.rphysbig[k];
    }
    __syncthreads();
    auto record = [&](const PairEnds& I, const PairEnds& J, const PairClass& pc, int id_i, int id_j, bool swap) {
        const int slot = atomicAdd(&A.status->events, 1);
        if (slot < A.event_cap) {
            pair_record(A.events + slot, I, J, pc, hm1, id_i, id_j, swap);
            A.event_step[slot] = step;
        } else {
            atomicOr(&A.status->overflow, 1);
        }
    };
    if (blockIdx.x == 0) {
        // pairs within the massive set: i Big, i < j < nsplit
        const int npair_max = nb * (N - 1);
        for (int q = threadIdx.x; q < npair_max; q += blockDim.x) {
            const int i = 1 + q / (N - 1), j = 1 + q % (N - 1);
            if (j <= i) continue;
            double bi[4], bj[4];
            box(i, bi);
            box(j, bj);
            if (!(bi[1] >= bj[0] && bj[1] >= bi[0] && bi[3] >= bj[2] && bj[3] >= bi[2])) continue;
            PairClass pc;
            const PairEnds I = ends(i), J = ends(j);
            if (pair_classify(I, J, A.rcebig[i], A.rcebig[j], A.rphysbig[i], A.rphysbig[j], h, pc))
                record(I, J, pc, i + 1, j + 1, A.mbig[j] > A.mbig[i] && j < A.nbig);
        }
        // the massive set's commit (the central body's row stays)
        for (int k = 1 + threadIdx.x; k < N; k += blockDim.x) {
            for (int q = 0; q < 6; ++q) A.bx[q * N + k] = bpost[q * N + k];
            for (int q = 6; q < 9; ++q) A.bx[q * N + k] = 0.0;
        }
    }
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const bool moves = A.perm[p] < A.active_np;
    const PairEnds J{make_double3(A.px[p], A.px[S + p], A.px[2 * S + p]),
                     make_double3(A.px[3 * S + p], A.px[4 * S + p], A.px[5 * S + p]),
                     moves ? make_double3(ppost[p], ppost[S + p], ppost[2 * S + p])
                           : make_double3(A.px[p], A.px[S + p], A.px[2 * S + p]),
                     moves ? make_double3(ppost[3 * S + p], ppost[4 * S + p], ppost[5 * S + p])
                           : make_double3(A.px[3 * S + p], A.px[4 * S + p], A.px[5 * S + p])};
    const double rce = A.pconst[S + p], rphys = A.pconst[2 * (size_t)S + p];
    double lo_x, hi_x, lo_y, hi_y;
    box_extent(J.x0.x, J.x1.x, J.v0.x, J.v1.x, h, lo_x, hi_x);
    box_extent(J.x0.y, J.x1.y, J.v0.y, J.v1.y, h, lo_y, hi_y);
    const double pad = rce * 1.2;
    lo_x -= pad;
    hi_x += pad;
    lo_y -= pad;
    hi_y += pad;
    for (int b = 0; b < nb; ++b) {
        const double* bb = sbox + 4 * b;
        if (!(bb[1] >= lo_x && hi_x >= bb[0] && bb[3] >= lo_y && hi_y >= bb[2])) continue;
        const double* d = sdet + (size_t)b * TAB_DETAIL;
        const PairEnds I{make_double3(d[0], d[1], d[2]), make_double3(d[3], d[4], d[5]),
                         make_double3(d[6], d[7], d[8]), make_double3(d[9], d[10], d[11])};
        PairClass pc;
        if (pair_classify(I, J, d[12], rce, d[13], rphys, h, pc)) record(I, J, pc, b + 2, N + A.perm[p] + 1, false);
    }
    if (moves) {
        A.px[p] = J.x1.x;
        A.px[S + p] = J.x1.y;
        A.px[2 * S + p] = J.x1.z;
        A.px[3 * S + p] = J.v1.x;
        A.px[4 * S + p] = J.v1.y;
        A.px[5 * S + p] = J.v1.z;
        for (int q = 6; q < 9; ++q) A.px[(size_t)q * S + p] = 0.0;
    }
}

// mfo_all (HKCE false) or, for mdt_bs2 in the encounter subsystem, mfo_hkce:
// separate instantiations, so that the encounter kernels carry neither the
// registers nor the code of the general force law.
template <int VARIANT, bool HKCE> void launch_variant(const BsArgs& a, cudaStream_t s) {
    const int N = a.f.nsplit;
    const size_t msmem = sizeof(double) * (((size_t)BS_LEVEL_ROWS + 12) * N + massive_par_scratch(N));
    if (msmem > 48 * 1024)
        cudaFuncSetAttribute(bs_massive_level_kernel<VARIANT, HKCE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)msmem);
    // one warp per 32 bodies, and with the parallel force terms (mfo_all)
    // enough for one term each
    int mthreads = std::min(256, std::max(32, (N + 31) / 32 * 32));
    if (massive_par_scratch(N) && !a.hkce) mthreads = std::max(mthreads, std::min(256, (N * N + 31) / 32 * 32));
    bs_massive_level_kernel<VARIANT, HKCE><<<bs_levels(VARIANT), mthreads, msmem, s>>>(a);
    if (!a.fuse_extrap) bs_massive_extrap_kernel<VARIANT><<<1, mthreads, 0, s>>>(a);
    const int pblocks = (a.np > 0 ? (a.np + 31) / 32 : 0) + (a.fuse_extrap ? 1 : 0);
    if (pblocks <= 0) return;
    size_t psmem = 0;
    BsArgs b = a;
    b.stage_bodies = 0;
    if (VARIANT == 2 && HKCE) {
        // the Big bodies of every table row, while that stays modest
        const size_t bytes = sizeof(double) * (size_t)bs_rows(VARIANT) * 4 * (size_t)(a.f.nbig - 1);
        if (bytes <= 96 * 1024) {
            psmem = bytes;
            b.stage_bodies = 1;
            if (bytes > 16 * 1024)
                cudaFuncSetAttribute(bs_particle_kernel<VARIANT, HKCE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bytes);
        }
    }
    if (VARIANT == 2 && !HKCE && a.ptab) {
        // the plain mdt_bs2 step: levels 1..8 now, 9..12 on demand (launch_bs_particles_late)
        bs_particle_kernel<2, false, 1, 8><<<pblocks, 8 * 16, 0, s>>>(b);
        return;
    }
    bs_particle_kernel<VARIANT, HKCE><<<pblocks, bs_levels(VARIANT) * 16, psmem, s>>>(b);
}

}  // namespace

void launch_bs_particles_late(const BsArgs& a, cudaStream_t s) {
    if (a.variant != 2 || a.hkce || !a.ptab || a.np <= 0) return;
    bs_particle_kernel<2, false, 9, 12><<<(a.np + 31) / 32, 4 * 16, 0, s>>>(a);
}

void launch_bs_sequence(const BsArgs& a, cudaStream_t s) {
    if (a.variant == 1) launch_variant<1, false>(a, s);
    else if (a.hkce) launch_variant<2, true>(a, s);
    else launch_variant<2, false>(a, s);
}

void launch_bs2_tangent(const BsArgs& a, int levels, double* tg, cudaStream_t s) {
    if (a.np <= 0 || levels < 1 || levels > bs_levels(2)) return;
    const int threads = 64;
    const size_t smem = sizeof(double) * 6 * bs_levels(2) * threads;
    const long long total = 6LL * a.np;
    bs2_tangent_kernel<<<(unsigned)((total + threads - 1) / threads), threads, smem, s>>>(a, levels, tg);
}

void launch_enc_post(const EncPostArgs& a, cudaStream_t s) {
    const int nb = a.nbig - 1;
    const size_t smem = sizeof(double) * (size_t)(nb > 0 ? nb : 1) * (4 + TAB_DETAIL);
    if (smem > 48 * 1024) cudaFuncSetAttribute(enc_post_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int blocks = std::max(1, (a.np + 127) / 128);
    enc_post_kernel<<<blocks, 128, smem, s>>>(a);
}

void launch_bs_commit(const BsCommitArgs& a, cudaStream_t s) {
    const int total = a.nsplit + a.np;
    bs_commit_kernel<<<(total + 127) / 128, 128, 0, s>>>(a);
}

}  // namespace mb200

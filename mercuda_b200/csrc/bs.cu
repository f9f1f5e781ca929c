// Bulirsch-Stoer kernels (mdt_bs1, mdt_bs2): every statement keeps the
// Fortran's evaluation order so that each level's extrapolated state rounds
// as the CPU's does.
#include <algorithm>
#include "allforce.cuh"
#include "bs.cuh"

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

// mfo_hkce for a massless member (subsystem index g) against table row T:
// every pair has a Big first body i, whose position is in the row.
__device__ double3 hkce_particle_force(const BsArgs& A, int g, const double3 x, double rcrit_p, const double* T) {
    double3 a = make_double3(0.0, 0.0, 0.0);
    for (int e = A.adj_off[g]; e < A.adj_off[g + 1]; ++e) {
        const int i = A.adj[e].x;
        const double* row = T + FT_HEAD + 4 * (i - 1);
        const double dx = x.x - row[0], dy = x.y - row[1], dz = x.z - row[2];
        double tmp2;
        if (!hkce_pair(dx * dx + dy * dy + dz * dz, fmax(A.rcrit[i], rcrit_p), tmp2)) continue;
        const double faci = tmp2 * row[3];
        a.x = a.x - faci * dx;
        a.y = a.y - faci * dy;
        a.z = a.z - faci * dz;
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
__device__ void massive_call(const BsArgs& A, const double* X, const double* V, double* out, double* T,
                             DeviceStatus* st, const double* mb, const double* ngf, double* head, double* PT) {
    const ForceCfg& f = A.f;
    const int N = f.nsplit;
    __syncthreads();
    if (A.hkce) {
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
template <int VARIANT> __global__ void __launch_bounds__(256) bs_massive_level_kernel(BsArgs A) {
    extern __shared__ double sm[];
    double h0 = A.h0;
    if (A.ctl) {
        if (A.ctl->stop) return;
        h0 = A.ctl->h0;
    }
    const int N = A.f.nsplit, tid = threadIdx.x, nt = blockDim.x, n = blockIdx.x + 1;
    const int stride = force_row(A.f.nbig - 1);
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
        massive_call(A, Xc, Vc, out, T, st, mb, ngf, head, PT);
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

// The massive set's extrapolation in level order (one CTA): per level the
// Neville updates (mercury6_2.for:3352-3366) with one thread per (body,
// component) and the coefficients computed once, then from level 4 on each
// (body, component)'s candidate sum and each body's error term for the
// level's maximum.
template <int VARIANT> __global__ void __launch_bounds__(256) bs_massive_extrap_kernel(BsArgs A) {
    const int N = A.f.nsplit, tid = threadIdx.x, nt = blockDim.x;
    constexpr int L = bs_levels(VARIANT);
    double* D = A.draw;
    __shared__ double co[L * (L - 1) / 2][2];
    __shared__ double wmax[8];
    __shared__ int wbad[8];
    double h0 = A.h0;
    if (A.ctl) {
        if (A.ctl->stop) return;
        h0 = A.ctl->h0;
    }
    neville_coefficients<VARIANT>(h0, co);
    __syncthreads();
    const int nb1 = N - 1, M = 6 * nb1;
    for (int n = 1; n <= L; ++n) {
        for (int q = tid; q < M; q += nt) {
            const int c = q / nb1, k = 1 + q % nb1;
            for (int j = n - 1; j >= 1; --j) {
                const double* cj = co[coef_index(n, j)];
                double* Dj = D + (size_t)(j - 1) * 6 * N;
                const double* Dj1 = D + (size_t)j * 6 * N;
                Dj[c * N + k] = cj[0] * Dj1[c * N + k] - cj[1] * Dj[c * N + k];
            }
        }
        if (n > 3) {
            __syncthreads();
            double* cand = A.bcand + (size_t)(n - 4) * 6 * N;
            for (int q = tid; q < M; q += nt) {
                const int c = q / nb1, k = 1 + q % nb1;
                double s = D[c * N + k];
                for (int j = 2; j <= n; ++j) s = s + D[(size_t)(j - 1) * 6 * N + c * N + k];
                cand[c * N + k] = s;
            }
            double emax = 0.0;
            int bad = 0;
            for (int k = 1 + tid; k < N; k += nt) {
                const double* X0 = A.bx;
                const double* V0 = A.bx + 3 * N;
                const double tmp1 = X0[k] * X0[k] + X0[N + k] * X0[N + k] + X0[2 * N + k] * X0[2 * N + k];
                const double tmp2 = V0[k] * V0[k] + V0[N + k] * V0[N + k] + V0[2 * N + k] * V0[2 * N + k];
                const double xscal = 1.0 / fmax(tmp1, 1e-300);
                const double vscal = 1.0 / fmax(tmp2, 1e-300);
                double q6[6];
                for (int c = 0; c < 6; ++c) q6[c] = D[c * N + k];
                double e;
                if (body_error(q6, xscal, vscal, e)) emax = fmax(emax, e);
                else bad = 1;
            }
            for (int o = 16; o; o >>= 1) {
                emax = fmax(emax, __shfl_xor_sync(FULLMASK, emax, o));
                bad |= __shfl_xor_sync(FULLMASK, bad, o);
            }
            if ((tid & 31) == 0) { wmax[tid >> 5] = emax; wbad[tid >> 5] = bad; }
            __syncthreads();
            if (tid == 0) {
                double m = 0.0;
                int b = 0;
                for (int w = 0; w < (nt + 31) / 32; ++w) { m = fmax(m, wmax[w]); b |= wbad[w]; }
                level_error(m, !b, &A.errs[n]);
            }
        }
        __syncthreads();
    }
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
template <int VARIANT> __global__ void __launch_bounds__(bs_levels(VARIANT) * 16) bs_particle_kernel(BsArgs A) {
    constexpr int L = bs_levels(VARIANT);
    constexpr int NW = L * 16 / 32;   // warps of the CTA
    __shared__ double dsm[L][6][32];
    __shared__ double a0sm[3][32];
    __shared__ double co[L * (L - 1) / 2][2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double h0 = A.h0;
    if (A.ctl) {
        if (A.ctl->stop) return;
        h0 = A.ctl->h0;
    }
    neville_coefficients<VARIANT>(h0, co);
    const int p = blockIdx.x * 32 + lane;
    const bool ok = p < A.np && A.perm[p] < A.active_np;
    const int nb = A.f.nbig - 1, stride = force_row(nb), S = A.npcap;
    double3 x0 = make_double3(0.0, 0.0, 0.0), v0 = x0;
    double mj = 0.0, g5[5] = {0, 0, 0, 0, 0};
    // the encounter subsystem (BS2 only): mfo_hkce from the member's pairs
    const bool hkce = VARIANT == 2 && A.hkce;
    int g = 0;
    double rcrit_p = 0.0;
    auto force = [&](const double3 x, const double3 v, const double* Tr, DeviceStatus* st) {
        return hkce ? hkce_particle_force(A, g, x, rcrit_p, Tr) : particle_allforce(x, v, Tr, nb, A.f, mj, g5, st);
    };
    if (ok) {
        x0 = make_double3(A.px[p], A.px[S + p], A.px[2 * S + p]);
        v0 = make_double3(A.px[3 * S + p], A.px[4 * S + p], A.px[5 * S + p]);
        mj = A.pconst[p];
        for (int c = 0; c < 5; ++c) g5[c] = A.pconst[(3 + c) * (size_t)S + p];
        if (hkce) {
            g = A.f.nsplit + A.perm[p];
            rcrit_p = A.pconst[(size_t)PC_RCRIT * S + p];
        }
        if (w == 0) {
            const double3 a = force(x0, v0, A.table, &A.lvst[0]);
            a0sm[0][lane] = a.x;
            a0sm[1][lane] = a.y;
            a0sm[2][lane] = a.z;
        }
    }
    __syncthreads();
    const double3 a0 = ok ? make_double3(a0sm[0][lane], a0sm[1][lane], a0sm[2][lane]) : make_double3(0.0, 0.0, 0.0);
#pragma unroll 1
    for (int half = 0; half < 2 && ok; ++half) {
        const int n = half == 0 ? w + 1 : L - w;
        int row = 1;
        for (int m = 1; m < n; ++m) row += bs_level_forces(VARIANT, m);
        DeviceStatus* st = &A.lvst[n];
        const double h = level_h<VARIANT>(h0, n);
        const double h2n = level_h2<VARIANT>(h0, n);
        auto call = [&](const double3 x, const double3 v) {
            const double* Tr = A.table + (size_t)(row++) * stride;
            return force(x, v, Tr, st);
        };
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
            double D[L];
#pragma unroll
            for (int n = 0; n < L; ++n) D[n] = dsm[n][c][lane];
#pragma unroll
            for (int n = 1; n <= L; ++n) {
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
    for (int n = 4 + w; n <= L; n += NW) {
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
    int level_cand = A.cand;
    if (A.ctl) {
        if (!A.ctl->accepted) return;
        level_cand = A.ctl->accepted - 4;
    }
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
// (mercury6_2.for:3568-3596; the same as bs_accept_level and the host loop
// of mdt_hkce, 3884-3937): the first level n > 3 whose error maximum is <=
// tol^2 is accepted, else the step is halved; after an acceptance the next
// trial step (x0.55 for a level >= 8, x1.3 below 7), the local clock, and the
// clipping of the next substep to the subsystem's end. One thread.
__global__ void bs_decide_kernel(EncCtl* c, unsigned long long* errs, DeviceStatus* lv, DeviceStatus* status) {
    if (c->stop) {
        c->accepted = 0;
        return;
    }
    constexpr int L = 12;
    const int fails = FAULT_NGF | FAULT_COINCIDENT;
    c->attempts += 1;
    int accepted = 0, error = 0;
    long long forces = 0;
    if (lv[0].fault & fails) error = ENC_ERR_FORCE;
    for (int n = 1; n <= L && !error && !accepted; ++n) {
        forces += n;
        if (lv[n].fault & fails) {
            error = ENC_ERR_FORCE;
            break;
        }
        if (n <= 3) continue;
        const double e = __longlong_as_double((long long)errs[n]);
        if (!isfinite(e)) {
            error = ENC_ERR_NONFINITE;
            break;
        }
        if (e <= c->tol * c->tol) accepted = n;
    }
    for (int n = 0; n < 13; ++n) {
        errs[n] = 0ull;
        lv[n].fault = 0;
    }
    c->forces += forces;
    if (error) {
        c->error = error;
        c->stop = 1;
        c->accepted = 0;
        return;
    }
    if (!accepted) {
        c->accepted = 0;
        c->h0 = c->h0 * 0.5;
        if (c->tlocal + c->h0 == c->tlocal) {
            c->error = ENC_ERR_ADVANCE;
            c->stop = 1;
        }
        return;
    }
    c->accepted = accepted;
    const double hdid = c->h0;
    double hnext = c->h0;
    if (accepted >= 8) hnext = hnext * 0.55;
    if (accepted < 7) hnext = hnext * 1.3;
    c->hdid = hdid;
    c->tlocal = c->tlocal + hdid;
    if (c->substeps >= c->step_cap) {
        c->error = ENC_ERR_STEPS;
        c->stop = 1;
        c->accepted = 0;
        return;
    }
    c->tstep[c->substeps] = c->time + c->tlocal;
    c->substeps += 1;
    // the previous substep's screen candidates, cleared for this one's
    c->max_cands = max(c->max_cands, status->cands);
    status->cands = 0;
    if (!((c->tlocal - c->h) * c->h < 0.0)) {
        c->stop = 1;
        return;
    }
    // the next substep: hrec before the clip to the subsystem's end
    const double tmp0 = fabs(c->h) - fabs(c->tlocal);
    c->hrec = hnext;
    if (fabs(hnext) > tmp0) hnext = copysign(tmp0, c->h);
    c->h0 = hnext;
    c->forces += 1;   // the next substep's start-of-step force
    if (c->tlocal + c->h0 == c->tlocal) {
        c->error = ENC_ERR_ADVANCE;
        c->stop = 1;
    }
}

__global__ void __launch_bounds__(256) bs_copyback_kernel(const EncCtl* c, const double* bsrc, double* bdst,
                                                          int nsplit, const double* psrc, double* pdst, int npcap) {
    if (!c->accepted) return;
    const size_t nb = (size_t)9 * nsplit, np = (size_t)9 * npcap;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nb + np; q += (size_t)gridDim.x * blockDim.x) {
        if (q < nb) bdst[q] = bsrc[q];
        else pdst[q - nb] = psrc[q - nb];
    }
}

template <int VARIANT> void launch_variant(const BsArgs& a, cudaStream_t s) {
    const int N = a.f.nsplit;
    const size_t msmem = sizeof(double) * (((size_t)BS_LEVEL_ROWS + 12) * N + massive_par_scratch(N));
    if (msmem > 48 * 1024)
        cudaFuncSetAttribute(bs_massive_level_kernel<VARIANT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem);
    // one warp per 32 bodies, and with the parallel force terms enough for one term each
    int mthreads = std::min(256, std::max(32, (N + 31) / 32 * 32));
    if (massive_par_scratch(N)) mthreads = std::max(mthreads, std::min(256, (N * N + 31) / 32 * 32));
    bs_massive_level_kernel<VARIANT><<<bs_levels(VARIANT), mthreads, msmem, s>>>(a);
    bs_massive_extrap_kernel<VARIANT><<<1, mthreads, 0, s>>>(a);
    if (a.np <= 0) return;
    bs_particle_kernel<VARIANT><<<(a.np + 31) / 32, bs_levels(VARIANT) * 16, 0, s>>>(a);
}

}  // namespace

void launch_bs_sequence(const BsArgs& a, cudaStream_t s) {
    if (a.variant == 1) launch_variant<1>(a, s);
    else launch_variant<2>(a, s);
}

void launch_bs2_tangent(const BsArgs& a, int levels, double* tg, cudaStream_t s) {
    if (a.np <= 0 || levels < 1 || levels > bs_levels(2)) return;
    const int threads = 64;
    const size_t smem = sizeof(double) * 6 * bs_levels(2) * threads;
    const long long total = 6LL * a.np;
    bs2_tangent_kernel<<<(unsigned)((total + threads - 1) / threads), threads, smem, s>>>(a, levels, tg);
}

void launch_bs_decide(EncCtl* ctl, unsigned long long* errs, DeviceStatus* lv, DeviceStatus* status,
                      cudaStream_t s) {
    bs_decide_kernel<<<1, 1, 0, s>>>(ctl, errs, lv, status);
}

void launch_bs_copyback(const EncCtl* ctl, const double* bsrc, double* bdst, int nsplit, const double* psrc,
                        double* pdst, int npcap, cudaStream_t s) {
    const size_t total = (size_t)9 * (nsplit + npcap);
    const int blocks = (int)std::min<size_t>(148 * 4, (total + 255) / 256);
    bs_copyback_kernel<<<blocks, 256, 0, s>>>(ctl, bsrc, bdst, nsplit, psrc, pdst, npcap);
}

void launch_bs_commit(const BsCommitArgs& a, cudaStream_t s) {
    const int total = a.nsplit + a.np;
    bs_commit_kernel<<<(total + 127) / 128, 128, 0, s>>>(a);
}

}  // namespace mb200

// HYBRID kernels (mdt_hy's two halves, mfo_hy, mce_snif). Every sum keeps
// the Fortran's order: the solar-drift momentum over bodies in index order,
// mfo_drct's direct terms with Big i outer and j > i inner, mfo_obl's
// (a + aobl) - acen.
#include "hybrid_device.cuh"
#include "kepler.cuh"

namespace mb200 {
namespace {

__device__ __forceinline__ double3 ld3(const double* p, int stride, int k) {
    return make_double3(p[k], p[stride + k], p[2 * stride + k]);
}
__device__ __forceinline__ void st3(double* p, int stride, int k, double3 v) {
    p[k] = v.x;
    p[stride + k] = v.y;
    p[2 * stride + k] = v.z;
}

// mfo_obl's reaction acen over the massive set in index order (one thread).
__device__ double3 obl_reaction(const HyArgs& A, const double* X) {
    double3 acen = make_double3(0.0, 0.0, 0.0);
    if (!A.obl) return acen;
    const int N = A.nsplit;
    for (int i = 1; i < N; ++i) {
        const double3 ao = oblate_accel(ld3(X, N, i), A.jcen, A.m0);
        const double tmp4 = A.mbig[i] / A.m0;
        acen.x = acen.x - tmp4 * ao.x;
        acen.y = acen.y - tmp4 * ao.y;
        acen.z = acen.z - tmp4 * ao.z;
    }
    return acen;
}

// (angf + 0) + a of mdt_hy's kick for body k of the massive set: mfo_hy
// (mercury6_2.for:4781-4819) at positions X, mfo_ngf with velocities V.
__device__ double3 massive_hy_accel(const HyArgs& A, int k, const double* X, const double* V, double3 acen) {
    const int N = A.nsplit, nbig = A.nbig;
    const double* m = A.mbig;
    const double* rcrit = A.rcritbig;
    const double3 xk = ld3(X, N, k);
    double3 a = make_double3(0.0, 0.0, 0.0);
    const int last_i = k < nbig ? k : nbig;
    for (int i = 1; i < last_i; ++i) {
        const double dx = xk.x - X[i], dy = xk.y - X[N + i], dz = xk.z - X[2 * N + i];
        const double tmp2 = drct_factor(dx * dx + dy * dy + dz * dz, fmax(rcrit[i], rcrit[k]));
        const double faci = tmp2 * m[i];
        a.x = a.x - faci * dx;
        a.y = a.y - faci * dy;
        a.z = a.z - faci * dz;
    }
    if (k < nbig)
        for (int j = k + 1; j < N; ++j) {
            const double dx = X[j] - xk.x, dy = X[N + j] - xk.y, dz = X[2 * N + j] - xk.z;
            const double tmp2 = drct_factor(dx * dx + dy * dy + dz * dz, fmax(rcrit[k], rcrit[j]));
            const double facj = tmp2 * m[j];
            a.x = a.x + facj * dx;
            a.y = a.y + facj * dy;
            a.z = a.z + facj * dz;
        }
    if (A.obl) {
        const double3 ao = oblate_accel(xk, A.jcen, A.m0);
        a.x = a.x + ao.x - acen.x;
        a.y = a.y + ao.y - acen.y;
        a.z = a.z + ao.z - acen.z;
    }
    if (A.ngflag == 1 || A.ngflag == 3) {
        double3 g;
        if (!nongrav_accel(xk, ld3(V, N, k), A.ngfbig + 5 * k, g)) raise_fault(A.status, FAULT_NGF);
        a.x = g.x + 0.0 + a.x;
        a.y = g.y + 0.0 + a.y;
        a.z = g.z + 0.0 + a.z;
    }
    if (!isfinite(a.x) || !isfinite(a.y) || !isfinite(a.z)) raise_fault(A.status, FAULT_NONFINITE);
    return a;
}

// Force row: head {shift(3), acen(3)}, per Big body {x, m, rcrit}. All threads.
__device__ void write_force_row(const HyArgs& A, const double* X, double3 shift, double3 acen, double* T) {
    const int N = A.nsplit;
    if (threadIdx.x == 0) {
        T[0] = shift.x; T[1] = shift.y; T[2] = shift.z;
        T[3] = acen.x; T[4] = acen.y; T[5] = acen.z;
        T[6] = 0.0; T[7] = 0.0;
    }
    for (int k = 1 + threadIdx.x; k < A.nbig; k += blockDim.x) {
        double* b = T + HY_HEAD + (k - 1) * HY_FORCE_BODY;
        b[0] = X[k]; b[1] = X[N + k]; b[2] = X[2 * N + k];
        b[3] = A.mbig[k];
        b[4] = A.rcritbig[k];
        b[5] = 0.0; b[6] = 0.0; b[7] = 0.0;
    }
}

// The solar-drift shift (hby2 / m0) sum_j m_j v_j over the massive set in
// index order (mercury6_2.for:3693-3707); one thread.
__device__ double3 solar_shift(const HyArgs& A, const double* V, double hby2) {
    const int N = A.nsplit;
    double3 s = make_double3(0.0, 0.0, 0.0);
    for (int j = 1; j < N; ++j) {
        const double mj = A.mbig[j];
        s.x = s.x + mj * V[j];
        s.y = s.y + mj * V[N + j];
        s.z = s.z + mj * V[2 * N + j];
    }
    const double temp = hby2 / A.m0;
    return make_double3(temp * s.x, temp * s.y, temp * s.z);
}

// mce_snif's test for one pair (mercury6_2.for:1691-1722).
__device__ __forceinline__ bool snif_pair(const PairEnds& I, const PairEnds& J, double rc, double h) {
    const double rc2 = rc * rc;
    const double dx0 = I.x0.x - J.x0.x, dy0 = I.x0.y - J.x0.y, dz0 = I.x0.z - J.x0.z;
    const double dx1 = I.x1.x - J.x1.x, dy1 = I.x1.y - J.x1.y, dz1 = I.x1.z - J.x1.z;
    const double d0 = dx0 * dx0 + dy0 * dy0 + dz0 * dz0;
    const double d1 = dx1 * dx1 + dy1 * dy1 + dz1 * dz1;
    const double du0 = I.v0.x - J.v0.x, dv0 = I.v0.y - J.v0.y, dw0 = I.v0.z - J.v0.z;
    const double du1 = I.v1.x - J.v1.x, dv1 = I.v1.y - J.v1.y, dw1 = I.v1.z - J.v1.z;
    const double d0t = (dx0 * du0 + dy0 * dv0 + dz0 * dw0) * 2.0;
    const double d1t = (dx1 * du1 + dy1 * dv1 + dz1 * dw1) * 2.0;
    double d2min = HUGE_VAL_F, tmin;
    if (d0t * h <= 0.0 && d1t * h >= 0.0) encounter_minimum(d0, d1, d0t, d1t, h, d2min, tmin);
    return fmin(fmin(d0, d1), d2min) <= rc2;
}

__device__ __forceinline__ void append_pair(const HyArgs& A, int i, int j) {
    const int slot = atomicAdd(&A.status->events, 1);
    if (slot < A.pair_cap) A.pairs[slot] = make_int2(i, j);
    else atomicOr(&A.status->overflow, 1);
}

__global__ void __launch_bounds__(256) hy_begin_massive(HyArgs A) {
    const int N = A.nsplit, nb = A.nbig - 1, tid = threadIdx.x, nt = blockDim.x;
    const double h = A.h, hby2 = 0.5 * h;
    double* Xin = A.bx_in;
    double* Vin = A.bx_in + 3 * N;
    double* Ain = A.bx_in + 6 * N;
    double* X = A.bx_out;
    double* V = A.bx_out + 3 * N;
    double* Acc = A.bx_out + 6 * N;
    double* X0 = A.bscr;
    double* V0 = A.bscr + 3 * N;
    double* T0 = A.tab + hy_tab_force0(nb);
    double* TB = A.tab + hy_tab_begin(nb);
    __shared__ double sh[6];
    if (A.recompute) {
        if (tid == 0) {
            const double3 acen = obl_reaction(A, Xin);
            sh[0] = acen.x; sh[1] = acen.y; sh[2] = acen.z;
        }
        __syncthreads();
        const double3 acen = make_double3(sh[0], sh[1], sh[2]);
        write_force_row(A, Xin, make_double3(0.0, 0.0, 0.0), acen, T0);
        for (int k = 1 + tid; k < N; k += nt) st3(Ain, N, k, massive_hy_accel(A, k, Xin, Vin, acen));
        __syncthreads();
    }
    for (int k = tid; k < N; k += nt)
        for (int c = 0; c < 3; ++c) {
            const int z = c * N + k;
            Acc[z] = Ain[z];
            X[z] = Xin[z];
            V[z] = k == 0 ? Vin[z] : Vin[z] + hby2 * Ain[z];
        }
    __syncthreads();
    if (tid == 0) {
        const double3 s = solar_shift(A, V, hby2);
        sh[3] = s.x; sh[4] = s.y; sh[5] = s.z;
        TB[0] = s.x; TB[1] = s.y; TB[2] = s.z;
        for (int c = 3; c < HY_HEAD; ++c) TB[c] = 0.0;
    }
    __syncthreads();
    const double shift[3] = {sh[3], sh[4], sh[5]};
    for (int k = 1 + tid; k < N; k += nt) {
        for (int c = 0; c < 3; ++c) {
            const int z = c * N + k;
            X[z] = X[z] + shift[c];
            X0[z] = X[z];
            V0[z] = V[z];
        }
        double3 p = ld3(X, N, k), w = ld3(V, N, k);
        drift_one(A.m0, p, w, h);
        st3(X, N, k, p);
        st3(V, N, k, w);
    }
    __syncthreads();
    // begin row for the particles' sniff: end states and the rcrit-padded box
    for (int k = 1 + tid; k < A.nbig; k += nt) {
        double* b = TB + HY_HEAD + (k - 1) * HY_BEGIN_BODY;
        for (int c = 0; c < 3; ++c) {
            b[c] = X0[c * N + k];
            b[3 + c] = V0[c * N + k];
            b[6 + c] = X[c * N + k];
            b[9 + c] = V[c * N + k];
        }
        const double rc = A.rcritbig[k];
        double lo, hi;
        box_extent(X0[k], X[k], V0[k], V[k], h, lo, hi);
        b[12] = lo - rc;
        b[13] = hi + rc;
        box_extent(X0[N + k], X[N + k], V0[N + k], V[N + k], h, lo, hi);
        b[14] = lo - rc;
        b[15] = hi + rc;
        b[16] = rc;
        b[17] = A.mbig[k];
        b[18] = 0.0;
        b[19] = 0.0;
    }
    // mce_snif within the massive set: Big i, any j > i (boxes padded by
    // rcrit for Big bodies only)
    const int span = N - 1;
    for (int q = tid; q < nb * span; q += nt) {
        const int i = 1 + q / span, j = 1 + q % span;
        if (j <= i) continue;
        double bi[4], bj[4];
        box_extent(X0[i], X[i], V0[i], V[i], h, bi[0], bi[1]);
        box_extent(X0[N + i], X[N + i], V0[N + i], V[N + i], h, bi[2], bi[3]);
        box_extent(X0[j], X[j], V0[j], V[j], h, bj[0], bj[1]);
        box_extent(X0[N + j], X[N + j], V0[N + j], V[N + j], h, bj[2], bj[3]);
        const double pi = A.rcritbig[i], pj = j < A.nbig ? A.rcritbig[j] : 0.0;
        bi[0] = bi[0] - pi; bi[1] = bi[1] + pi; bi[2] = bi[2] - pi; bi[3] = bi[3] + pi;
        if (j < A.nbig) { bj[0] = bj[0] - pj; bj[1] = bj[1] + pj; bj[2] = bj[2] - pj; bj[3] = bj[3] + pj; }
        if (!(bi[1] >= bj[0] && bj[1] >= bi[0] && bi[3] >= bj[2] && bj[3] >= bi[2])) continue;
        const PairEnds I{ld3(X0, N, i), ld3(V0, N, i), ld3(X, N, i), ld3(V, N, i)};
        const PairEnds J{ld3(X0, N, j), ld3(V0, N, j), ld3(X, N, j), ld3(V, N, j)};
        if (snif_pair(I, J, fmax(A.rcritbig[i], A.rcritbig[j]), h)) append_pair(A, i, j);
    }
}

__global__ void __launch_bounds__(128) hy_begin_particles(HyArgs A) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x, S = A.npcap, nb = A.nbig - 1;
    if (p >= A.np) return;
    const double h = A.h, hby2 = 0.5 * h;
    const double* T0 = A.tab + hy_tab_force0(nb);
    const double* TB = A.tab + hy_tab_begin(nb);
    double3 x = ld3(A.px_in, S, p), v = ld3(A.px_in + 3 * (size_t)S, S, p);
    double3 acc = ld3(A.px_in + 6 * (size_t)S, S, p);
    const double rcrit_p = A.pconst[(size_t)PC_RCRIT * S + p];
    if (A.recompute) {
        double g[5];
        for (int c = 0; c < 5; ++c) g[c] = A.pconst[(size_t)(PC_NGF + c) * S + p];
        acc = particle_hy_accel(A, x, v, rcrit_p, g, T0);
    }
    v.x = v.x + hby2 * acc.x;
    v.y = v.y + hby2 * acc.y;
    v.z = v.z + hby2 * acc.z;
    x.x = x.x + TB[0];
    x.y = x.y + TB[1];
    x.z = x.z + TB[2];
    const double3 x0 = x, v0 = v;
    drift_one(A.m0, x, v, h);
    double lo_x, hi_x, lo_y, hi_y;
    box_extent(x0.x, x.x, v0.x, v.x, h, lo_x, hi_x);
    box_extent(x0.y, x.y, v0.y, v.y, h, lo_y, hi_y);
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
        const double* r = TB + HY_HEAD + b * HY_BEGIN_BODY;
        if (!(r[13] >= lo_x && hi_x >= r[12] && r[15] >= lo_y && hi_y >= r[14])) continue;
        const PairEnds I{make_double3(r[0], r[1], r[2]), make_double3(r[3], r[4], r[5]),
                         make_double3(r[6], r[7], r[8]), make_double3(r[9], r[10], r[11])};
        const PairEnds J{x0, v0, x, v};
        if (snif_pair(I, J, fmax(r[16], rcrit_p), h)) append_pair(A, b + 1, A.nsplit + A.perm[p]);
    }
    st3(A.px_out, S, p, x);
    st3(A.px_out + 3 * (size_t)S, S, p, v);
    st3(A.px_out + 6 * (size_t)S, S, p, acc);
}

__global__ void __launch_bounds__(256) hy_finish_massive(HyArgs A) {
    const int N = A.nsplit, nb = A.nbig - 1, tid = threadIdx.x, nt = blockDim.x;
    const double hby2 = 0.5 * A.h;
    double* X = A.bx_out;
    double* V = A.bx_out + 3 * N;
    double* Acc = A.bx_out + 6 * N;
    double* T1 = A.tab + hy_tab_force1(nb);
    __shared__ double sh[6];
    if (tid == 0) {
        const double3 s = solar_shift(A, V, hby2);
        sh[0] = s.x; sh[1] = s.y; sh[2] = s.z;
    }
    __syncthreads();
    const double3 shift = make_double3(sh[0], sh[1], sh[2]);
    for (int k = 1 + tid; k < N; k += nt) {
        X[k] = X[k] + shift.x;
        X[N + k] = X[N + k] + shift.y;
        X[2 * N + k] = X[2 * N + k] + shift.z;
    }
    __syncthreads();
    if (tid == 0) {
        const double3 acen = obl_reaction(A, X);
        sh[3] = acen.x; sh[4] = acen.y; sh[5] = acen.z;
    }
    __syncthreads();
    const double3 acen = make_double3(sh[3], sh[4], sh[5]);
    write_force_row(A, X, shift, acen, T1);
    for (int k = 1 + tid; k < N; k += nt) {
        const double3 a = massive_hy_accel(A, k, X, V, acen);
        st3(Acc, N, k, a);
    }
    __syncthreads();
    for (int k = 1 + tid; k < N; k += nt)
        for (int c = 0; c < 3; ++c) {
            const int z = c * N + k;
            V[z] = V[z] + hby2 * Acc[z];
        }
}

__global__ void __launch_bounds__(128) hy_finish_particles(HyArgs A) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x, S = A.npcap, nb = A.nbig - 1;
    if (p >= A.np) return;
    const double hby2 = 0.5 * A.h;
    const double* T1 = A.tab + hy_tab_force1(nb);
    double3 x = ld3(A.px_out, S, p), v = ld3(A.px_out + 3 * (size_t)S, S, p);
    x.x = x.x + T1[0];
    x.y = x.y + T1[1];
    x.z = x.z + T1[2];
    double g[5];
    for (int c = 0; c < 5; ++c) g[c] = A.pconst[(size_t)(PC_NGF + c) * S + p];
    const double3 acc = particle_hy_accel(A, x, v, A.pconst[(size_t)PC_RCRIT * S + p], g, T1);
    v.x = v.x + hby2 * acc.x;
    v.y = v.y + hby2 * acc.y;
    v.z = v.z + hby2 * acc.z;
    st3(A.px_out, S, p, x);
    st3(A.px_out + 3 * (size_t)S, S, p, v);
    st3(A.px_out + 6 * (size_t)S, S, p, acc);
}

__global__ void hy_restore(HyArgs A, const int* ids, int count, const int* inv, double* packed) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const int g = ids[q], N = A.nsplit, S = A.npcap, nb = A.nbig - 1;
    double3 x0, v0;
    if (g < N) {
        x0 = ld3(A.bscr, N, g);
        v0 = ld3(A.bscr + 3 * N, N, g);
        st3(A.bx_out, N, g, x0);
        st3(A.bx_out + 3 * N, N, g, v0);
    } else {
        // the begin kernel's kick and first solar drift, recomputed
        const int s = inv[g - N];
        const double hby2 = 0.5 * A.h;
        const double* TB = A.tab + hy_tab_begin(nb);
        const double3 xi = ld3(A.px_in, S, s), vi = ld3(A.px_in + 3 * (size_t)S, S, s);
        const double3 acc = ld3(A.px_out + 6 * (size_t)S, S, s);
        v0 = make_double3(vi.x + hby2 * acc.x, vi.y + hby2 * acc.y, vi.z + hby2 * acc.z);
        x0 = make_double3(xi.x + TB[0], xi.y + TB[1], xi.z + TB[2]);
        st3(A.px_out, S, s, x0);
        st3(A.px_out + 3 * (size_t)S, S, s, v0);
    }
    double* o = packed + 6 * (size_t)q;
    o[0] = x0.x; o[1] = x0.y; o[2] = x0.z;
    o[3] = v0.x; o[4] = v0.y; o[5] = v0.z;
}

__global__ void dh_shift_kernel(const double* bx, const double* m, int N, double m0, double* out) {
    if (threadIdx.x || blockIdx.x) return;
    double s[3] = {0.0, 0.0, 0.0};
    for (int j = 1; j < N; ++j)
        for (int c = 0; c < 3; ++c) s[c] = s[c] + m[j] * bx[(3 + c) * N + j];
    const double temp = 1.0 / m0;
    for (int c = 0; c < 3; ++c) out[c] = temp * s[c];
}

}  // namespace

void launch_hybrid_begin(const HyArgs& a, cudaStream_t s) {
    hy_begin_massive<<<1, 256, 0, s>>>(a);
    if (a.np > 0) hy_begin_particles<<<(a.np + 127) / 128, 128, 0, s>>>(a);
}

void launch_hybrid_finish(const HyArgs& a, cudaStream_t s) {
    hy_finish_massive<<<1, 256, 0, s>>>(a);
    if (a.np > 0) hy_finish_particles<<<(a.np + 127) / 128, 128, 0, s>>>(a);
}

void launch_hybrid_restore(const HyArgs& a, const int* ids, int count, const int* inv, double* packed,
                           cudaStream_t s) {
    if (count > 0) hy_restore<<<(count + 127) / 128, 128, 0, s>>>(a, ids, count, inv, packed);
}

void launch_dh_shift(const double* bx, const double* m, int nsplit, double m0, double* out, cudaStream_t s) {
    dh_shift_kernel<<<1, 1, 0, s>>>(bx, m, nsplit, m0, out);
}

}  // namespace mb200

// RA15 Gauss-Radau integrator (mdt_ra15, mercury6_2.for:4133-4485) with the
// heliocentric force mfo_all (mercury6_2.for:4506-4689, 5106-5343), and the
// generic encounter screen of the adaptive integrators.
//
// The massive set (Big bodies and any Small body with mass, which acts on the
// Big bodies) is integrated by one CTA; it writes, for every force call of the
// sequence, a table row with the Big bodies' predicted positions and the
// indirect/oblateness terms that every massless particle needs. The particle
// kernel then runs the whole sequence (7 Gauss-Radau nodes x 2 or 6
// iterations) per particle in registers and reduces max |b7| for the global
// step controller; a commit pass applies the accepted sequence.
#include <algorithm>
#include <cstring>

#include "allforce.cuh"
#include "mvs_device.cuh"
#include "radau.cuh"

namespace mb200 {
namespace {

constexpr unsigned FULLMASK = 0xffffffffu;

struct RaConst {
    double h[8], xc[8], vc[7], r[28], c[21], d[21];
};
__constant__ RaConst RK;

// The constants of mdt_ra15 (mercury6_2.for:4164-4209), computed on the host
// with the same statements as the Fortran initialisation.
RaConst make_constants() {
    RaConst K;
    const double hh[8] = {0.0, .0562625605369221, .1802406917368924, .3526247171131696,
                          .5471536263305554, .7342101772154105, .8853209468390958, .9775206135612875};
    const double xx[8] = {.5, .1666666666666667, .08333333333333333, .05, .03333333333333333,
                          .02380952380952381, .01785714285714286, .01388888888888889};
    const double vv[7] = {.5, .3333333333333333, .25, .2, .1666666666666667, .1428571428571429, .125};
    for (int k = 0; k < 8; ++k) {
        K.h[k] = hh[k];
        K.xc[k] = xx[k];
    }
    for (int k = 0; k < 7; ++k) K.vc[k] = vv[k];
    int n = 0;
    for (int j = 1; j < 8; ++j)
        for (int k = 0; k < j; ++k) K.r[n++] = 1.0 / (K.h[j] - K.h[k]);
    double C[22], D[22];
    C[1] = -K.h[1];
    D[1] = K.h[1];
    n = 1;
    for (int j = 3; j <= 7; ++j) {
        ++n;
        C[n] = -K.h[j - 1] * C[n - j + 2];
        D[n] = K.h[1] * D[n - j + 2];
        for (int k = 3; k <= j - 1; ++k) {
            ++n;
            C[n] = C[n - j + 1] - K.h[j - 1] * C[n - j + 2];
            D[n] = D[n - j + 1] + K.h[k - 1] * D[n - j + 2];
        }
        ++n;
        C[n] = C[n - j + 1] - K.h[j - 1];
        D[n] = D[n - j + 1] + K.h[j - 1];
    }
    for (int k = 0; k < 21; ++k) {
        K.c[k] = C[k + 1];
        K.d[k] = D[k + 1];
    }
    return K;
}

void ensure_constants() {
    static int done_on[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done_on[dev]) {
        // once per device; waits for the copy, which the library's streams
        // would not otherwise be ordered after
        const RaConst K = make_constants();
        if (cudaMemcpyToSymbol(RK, &K, sizeof(K)) == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess)
            done_on[dev] = 1;
    }
}

// ------------------------------------------------------------------- RA15
// Eqs. 7 of Everhart: G from B (one coordinate, 7 coefficients).
__device__ __forceinline__ void g_from_b(const double* b, double* g) {
    const double* d = RK.d;
    g[0] = b[6] * d[15] + b[5] * d[10] + b[4] * d[6] + b[3] * d[3] + b[2] * d[1] + b[1] * d[0] + b[0];
    g[1] = b[6] * d[16] + b[5] * d[11] + b[4] * d[7] + b[3] * d[4] + b[2] * d[2] + b[1];
    g[2] = b[6] * d[17] + b[5] * d[12] + b[4] * d[8] + b[3] * d[5] + b[2];
    g[3] = b[6] * d[18] + b[5] * d[13] + b[4] * d[9] + b[3];
    g[4] = b[6] * d[19] + b[5] * d[14] + b[4];
    g[5] = b[6] * d[20] + b[5];
    g[6] = b[6];
}

// Position and velocity predictor coefficients of node j (Eqs. 9, 10).
struct Pred {
    double sx[9], sv[8];
};
__device__ __forceinline__ Pred predictor(double t, int j) {
    Pred P;
    const double hj = RK.h[j - 1];
    P.sx[0] = t * hj;
    P.sx[1] = P.sx[0] * P.sx[0] * .5;
    P.sx[2] = P.sx[1] * hj * .3333333333333333;
    P.sx[3] = P.sx[2] * hj * .5;
    P.sx[4] = P.sx[3] * hj * .6;
    P.sx[5] = P.sx[4] * hj * .6666666666666667;
    P.sx[6] = P.sx[5] * hj * .7142857142857143;
    P.sx[7] = P.sx[6] * hj * .75;
    P.sx[8] = P.sx[7] * hj * .7777777777777778;
    P.sv[0] = t * hj;
    P.sv[1] = P.sv[0] * hj * .5;
    P.sv[2] = P.sv[1] * hj * .6666666666666667;
    P.sv[3] = P.sv[2] * hj * .75;
    P.sv[4] = P.sv[3] * hj * .8;
    P.sv[5] = P.sv[4] * hj * .8333333333333333;
    P.sv[6] = P.sv[5] * hj * .8571428571428571;
    P.sv[7] = P.sv[6] * hj * .875;
    return P;
}
__device__ __forceinline__ double pred_x(const Pred& P, const double* b, double a1, double v1, double x1) {
    const double* s = P.sx;
    return s[8] * b[6] + s[7] * b[5] + s[6] * b[4] + s[5] * b[3] + s[4] * b[2] + s[3] * b[1] + s[2] * b[0] +
           s[1] * a1 + s[0] * v1 + x1;
}
__device__ __forceinline__ double pred_v(const Pred& P, const double* b, double a1, double v1) {
    const double* s = P.sv;
    return s[7] * b[6] + s[6] * b[5] + s[5] * b[4] + s[4] * b[3] + s[3] * b[2] + s[2] * b[1] + s[1] * b[0] +
           s[0] * a1 + v1;
}

// Eqs. 4 and 5 of Everhart after the force at node j (one coordinate).
__device__ __forceinline__ void update_gb(int j, double ak, double a1k, double* g, double* b) {
    const double* r = RK.r;
    const double* c = RK.c;
    const double gk = ak - a1k;
    double temp;
    switch (j) {
    case 2:
        temp = g[0];
        g[0] = (ak - a1k) * r[0];
        b[0] = b[0] + g[0] - temp;
        break;
    case 3:
        temp = g[1];
        g[1] = (gk * r[1] - g[0]) * r[2];
        temp = g[1] - temp;
        b[0] = b[0] + temp * c[0];
        b[1] = b[1] + temp;
        break;
    case 4:
        temp = g[2];
        g[2] = ((gk * r[3] - g[0]) * r[4] - g[1]) * r[5];
        temp = g[2] - temp;
        b[0] = b[0] + temp * c[1];
        b[1] = b[1] + temp * c[2];
        b[2] = b[2] + temp;
        break;
    case 5:
        temp = g[3];
        g[3] = (((gk * r[6] - g[0]) * r[7] - g[1]) * r[8] - g[2]) * r[9];
        temp = g[3] - temp;
        b[0] = b[0] + temp * c[3];
        b[1] = b[1] + temp * c[4];
        b[2] = b[2] + temp * c[5];
        b[3] = b[3] + temp;
        break;
    case 6:
        temp = g[4];
        g[4] = ((((gk * r[10] - g[0]) * r[11] - g[1]) * r[12] - g[2]) * r[13] - g[3]) * r[14];
        temp = g[4] - temp;
        b[0] = b[0] + temp * c[6];
        b[1] = b[1] + temp * c[7];
        b[2] = b[2] + temp * c[8];
        b[3] = b[3] + temp * c[9];
        b[4] = b[4] + temp;
        break;
    case 7:
        temp = g[5];
        g[5] = (((((gk * r[15] - g[0]) * r[16] - g[1]) * r[17] - g[2]) * r[18] - g[3]) * r[19] - g[4]) * r[20];
        temp = g[5] - temp;
        b[0] = b[0] + temp * c[10];
        b[1] = b[1] + temp * c[11];
        b[2] = b[2] + temp * c[12];
        b[3] = b[3] + temp * c[13];
        b[4] = b[4] + temp * c[14];
        b[5] = b[5] + temp;
        break;
    default:
        temp = g[6];
        g[6] = ((((((gk * r[21] - g[0]) * r[22] - g[1]) * r[23] - g[2]) * r[24] - g[3]) * r[25] - g[4]) * r[26] -
                g[5]) *
               r[27];
        temp = g[6] - temp;
        b[0] = b[0] + temp * c[15];
        b[1] = b[1] + temp * c[16];
        b[2] = b[2] + temp * c[17];
        b[3] = b[3] + temp * c[18];
        b[4] = b[4] + temp * c[19];
        b[5] = b[5] + temp * c[20];
        b[6] = b[6] + temp;
        break;
    }
}

__device__ __forceinline__ void atomic_max_abs(unsigned long long* dst, double v) {
    // |v| of a finite double: its bit pattern orders like the value
    atomicMax(dst, (unsigned long long)__double_as_longlong(fabs(v)));
}

// The massive set's sequence: one CTA. Writes table rows 0 (sequence start)
// and 1 + (n-1)*7 + (j-2) (iteration n, node j) for the particles. With
// STAGED the set's positions, velocities, B, G, accelerations, masses and
// non-gravitational constants live in shared memory for the whole sequence
// (the set is small and every node reads all of it after a barrier); B, G
// and a1 go back to global memory at the end. The arithmetic is the same.
template <bool STAGED> __global__ void __launch_bounds__(256) ra15_massive_kernel(Ra15Args A) {
    extern __shared__ double sm[];
    const ForceCfg& f = A.f;
    const int N = f.nsplit, nb = f.nbig - 1, tid = threadIdx.x, nt = blockDim.x;
    const int stride = force_row(nb);
    const bool vpred = (f.ngflag != 0 || f.pn == 1);
    __shared__ double blockmax[8];
    __shared__ double head[FT_HEAD];
    double *X, *V, *B, *G, *a1, *PT = nullptr;
    const double *x1, *v1, *mb, *ngf;
    if (STAGED) {
        X = sm;
        V = X + 3 * N;
        B = V + 3 * N;
        G = B + 21 * N;
        a1 = G + 21 * N;
        double* sx1 = a1 + 3 * N;
        double* sv1 = sx1 + 3 * N;
        double* smb = sv1 + 3 * N;
        double* sngf = smb + N;
        PT = massive_par_scratch(N) ? sngf + 5 * N : nullptr;
        for (int q = tid; q < 3 * N; q += nt) {
            sx1[q] = A.bx[q];
            sv1[q] = A.bx[3 * N + q];
        }
        for (int q = tid; q < 21 * N; q += nt) B[q] = A.reset ? 0.0 : A.bb[q];
        for (int q = tid; q < N; q += nt) smb[q] = A.mbig[q];
        for (int q = tid; q < 5 * N; q += nt) sngf[q] = A.ngfbig[q];
        x1 = sx1;
        v1 = sv1;
        mb = smb;
        ngf = sngf;
        __syncthreads();
    } else {
        X = A.bpx;
        V = A.bpx + 3 * N;
        B = A.bb;
        G = A.bg;
        a1 = A.bx_a1;
        x1 = A.bx;
        v1 = A.bx + 3 * N;
        mb = A.mbig;
        ngf = A.ngfbig;
    }
    // the head of a table row: written to the table for the particles and
    // kept in shared memory for the massive set's forces
    // (with PT the force terms are computed by every thread first; the
    // caller synchronizes before and after)
    auto write_head = [&](double* T) {
        if (PT) {
            massive_terms(X, mb, f, PT, A.status);
            __syncthreads();
        }
        if (tid == 0) {
            if (PT) row_head_terms(PT, f, T);
            else row_head(X, mb, f, T);
            for (int q = 0; q < FT_HEAD; ++q) head[q] = T[q];
        }
    };
    auto force = [&](int k, const double* Vc) {
        return PT ? massive_allforce_terms(k, X, Vc, mb, ngf, head, f, PT, A.status)
                  : massive_allforce(k, X, Vc, mb, ngf, head, f, A.status);
    };
    double localmax = 0.0;
    // sequence start: force at (x1, v1), G from B
    for (int k = tid; k < N; k += nt)
        for (int c = 0; c < 3; ++c) {
            X[c * N + k] = x1[c * N + k];
            V[c * N + k] = v1[c * N + k];
        }
    __syncthreads();
    write_head(A.table);
    __syncthreads();
    for (int k = tid; k < N; k += nt) {
        if (k >= 1 && k < f.nbig) {
            double* row = A.table + FT_HEAD + 4 * (k - 1);
            row[0] = X[k]; row[1] = X[N + k]; row[2] = X[2 * N + k]; row[3] = mb[k];
        }
        if (k < 1) continue;
        const double3 a = force(k, V);
        a1[k] = a.x; a1[N + k] = a.y; a1[2 * N + k] = a.z;
        for (int c = 0; c < 3; ++c) {
            double b[7], g[7];
            for (int m = 0; m < 7; ++m) b[m] = (A.reset && !STAGED) ? 0.0 : B[(c * 7 + m) * N + k];
            g_from_b(b, g);
            for (int m = 0; m < 7; ++m) {
                B[(c * 7 + m) * N + k] = b[m];
                G[(c * 7 + m) * N + k] = g[m];
            }
        }
    }
    __syncthreads();
    for (int n = 1; n <= A.niter; ++n) {
        for (int j = 2; j <= 8; ++j) {
            const Pred P = predictor(A.t, j);
            double* T = A.table + (size_t)(1 + (n - 1) * 7 + (j - 2)) * stride;
            for (int k = tid; k < N; k += nt) {
                if (k < 1) continue;
                for (int c = 0; c < 3; ++c) {
                    double b[7];
                    for (int m = 0; m < 7; ++m) b[m] = B[(c * 7 + m) * N + k];
                    X[c * N + k] = pred_x(P, b, a1[c * N + k], v1[c * N + k], x1[c * N + k]);
                    if (vpred) V[c * N + k] = pred_v(P, b, a1[c * N + k], v1[c * N + k]);
                }
            }
            __syncthreads();
            write_head(T);
            __syncthreads();
            for (int k = tid; k < N; k += nt) {
                if (k >= 1 && k < f.nbig) {
                    double* row = T + FT_HEAD + 4 * (k - 1);
                    row[0] = X[k]; row[1] = X[N + k]; row[2] = X[2 * N + k]; row[3] = mb[k];
                }
                if (k < 1) continue;
                const double3 a = force(k, vpred ? V : v1);
                const double ac[3] = {a.x, a.y, a.z};
                for (int c = 0; c < 3; ++c) {
                    double b[7], g[7];
                    for (int m = 0; m < 7; ++m) {
                        b[m] = B[(c * 7 + m) * N + k];
                        g[m] = G[(c * 7 + m) * N + k];
                    }
                    update_gb(j, ac[c], a1[c * N + k], g, b);
                    for (int m = 0; m < 7; ++m) {
                        B[(c * 7 + m) * N + k] = b[m];
                        G[(c * 7 + m) * N + k] = g[m];
                    }
                }
            }
            __syncthreads();
        }
    }
    if (STAGED) {
        // every body but the central one (whose entries the sequence leaves alone)
        for (int q = tid; q < 21 * N; q += nt)
            if (q % N != 0) {
                A.bb[q] = B[q];
                A.bg[q] = G[q];
            }
        for (int q = tid; q < 3 * N; q += nt)
            if (q % N != 0) A.bx_a1[q] = a1[q];
    }
    for (int k = tid; k < N; k += nt) {
        if (k < 1) continue;
        for (int c = 0; c < 3; ++c) {
            const double b7 = B[(c * 7 + 6) * N + k];
            if (!isfinite(b7)) raise_fault(A.status, FAULT_NONFINITE);
            else localmax = fmax(localmax, fabs(b7));
        }
    }
    for (int o = 16; o; o >>= 1) localmax = fmax(localmax, __shfl_xor_sync(FULLMASK, localmax, o));
    if ((tid & 31) == 0) blockmax[tid >> 5] = localmax;
    __syncthreads();
    if (tid == 0) {
        double mx = 0.0;
        for (int w = 0; w < (nt + 31) / 32; ++w) mx = fmax(mx, blockmax[w]);
        atomic_max_abs(A.maxb7, mx);
    }
}

// The particles' sequence: one thread per particle slot, state in registers.
// Three CTAs of 128 per SM (at most 168 registers, a few spilled words): 12
// warps per SM hide the FP64 dependency chains better than the 8 the
// unbounded 194-register build fits (0.361 -> 0.322 ms per step at 100k).
constexpr int RA15_PARTICLE_THREADS = 128;
__global__ void __launch_bounds__(RA15_PARTICLE_THREADS, 3) ra15_particle_kernel(Ra15Args A) {
    const ForceCfg& f = A.f;
    const int nb = f.nbig - 1, stride = force_row(nb), S = A.npcap;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = p < A.np;
    double localmax = 0.0;
    if (ok) {
        const bool vpred = (f.ngflag != 0 || f.pn == 1);
        const double3 x1 = make_double3(A.px[p], A.px[S + p], A.px[2 * S + p]);
        const double3 v1 = make_double3(A.px[3 * S + p], A.px[4 * S + p], A.px[5 * S + p]);
        const double mj = A.pconst[p];
        double g5[5];
        for (int c = 0; c < 5; ++c) g5[c] = A.pconst[(3 + c) * (size_t)S + p];
        double b[21], g[21];
#pragma unroll
        for (int q = 0; q < 21; ++q) b[q] = A.reset ? 0.0 : A.pb[(size_t)q * S + p];
        const double3 a1 = particle_allforce(x1, v1, A.table, nb, f, mj, g5, A.status);
        A.px[6 * S + p] = a1.x;
        A.px[7 * S + p] = a1.y;
        A.px[8 * S + p] = a1.z;
#pragma unroll
        for (int c = 0; c < 3; ++c) g_from_b(b + 7 * c, g + 7 * c);
        const double a1c[3] = {a1.x, a1.y, a1.z};
        const double x1c[3] = {x1.x, x1.y, x1.z};
        const double v1c[3] = {v1.x, v1.y, v1.z};
#pragma unroll 1
        for (int n = 1; n <= A.niter; ++n) {
#pragma unroll 1
            for (int j = 2; j <= 8; ++j) {
                const Pred P = predictor(A.t, j);
                double xp[3], vp[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    xp[c] = pred_x(P, b + 7 * c, a1c[c], v1c[c], x1c[c]);
                    vp[c] = vpred ? pred_v(P, b + 7 * c, a1c[c], v1c[c]) : v1c[c];
                }
                const double* T = A.table + (size_t)(1 + (n - 1) * 7 + (j - 2)) * stride;
                const double3 a = particle_allforce(make_double3(xp[0], xp[1], xp[2]),
                                                    make_double3(vp[0], vp[1], vp[2]), T, nb, f, mj, g5, A.status);
                const double ac[3] = {a.x, a.y, a.z};
#pragma unroll
                for (int c = 0; c < 3; ++c) update_gb(j, ac[c], a1c[c], g + 7 * c, b + 7 * c);
            }
        }
#pragma unroll
        for (int q = 0; q < 21; ++q) A.pb[(size_t)q * S + p] = b[q];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double b7 = b[7 * c + 6];
            if (!isfinite(b7)) raise_fault(A.status, FAULT_NONFINITE);
            else localmax = fmax(localmax, fabs(b7));
        }
    }
    for (int o = 16; o; o >>= 1) localmax = fmax(localmax, __shfl_xor_sync(FULLMASK, localmax, o));
    if ((threadIdx.x & 31) == 0 && localmax > 0.0) atomic_max_abs(A.maxb7, localmax);
}

// Eqs. 11-13 of Everhart for one body: the accepted sequence (x1, v1 at
// tdid) and the B values predicted for the next one (q = t_next / tdid).
__device__ __forceinline__ void commit_body(const double* x1, const double* v1, const double* a1, double* b,
                                            double* e, double* xo, double* vo, double tdid, double q, bool reset) {
    const double* xc = RK.xc;
    const double* vc = RK.vc;
    const double temp = tdid * tdid;
    const double q2 = q * q, q3 = q * q2, q4 = q2 * q2, q5 = q2 * q3, q6 = q3 * q3, q7 = q3 * q4;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double* B = b + 7 * c;
        xo[c] = (xc[7] * B[6] + xc[6] * B[5] + xc[5] * B[4] + xc[4] * B[3] + xc[3] * B[2] + xc[2] * B[1] +
                 xc[1] * B[0] + xc[0] * a1[c]) *
                    temp +
                v1[c] * tdid + x1[c];
        vo[c] = (vc[6] * B[6] + vc[5] * B[5] + vc[4] * B[4] + vc[3] * B[3] + vc[2] * B[2] + vc[1] * B[1] +
                 vc[0] * B[0] + a1[c]) *
                    tdid +
                v1[c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double* Bc = b + 7 * c;
        double* Ec = e + 7 * c;
        double s[7];
        for (int m = 0; m < 7; ++m) s[m] = reset ? 0.0 : Bc[m] - Ec[m];
        Ec[0] = q * (Bc[6] * 7.0 + Bc[5] * 6.0 + Bc[4] * 5.0 + Bc[3] * 4.0 + Bc[2] * 3.0 + Bc[1] * 2.0 + Bc[0]);
        Ec[1] = q2 * (Bc[6] * 21.0 + Bc[5] * 15.0 + Bc[4] * 10.0 + Bc[3] * 6.0 + Bc[2] * 3.0 + Bc[1]);
        Ec[2] = q3 * (Bc[6] * 35.0 + Bc[5] * 20.0 + Bc[4] * 10.0 + Bc[3] * 4.0 + Bc[2]);
        Ec[3] = q4 * (Bc[6] * 35.0 + Bc[5] * 15.0 + Bc[4] * 5.0 + Bc[3]);
        Ec[4] = q5 * (Bc[6] * 21.0 + Bc[5] * 6.0 + Bc[4]);
        Ec[5] = q6 * (Bc[6] * 7.0 + Bc[5]);
        Ec[6] = q7 * Bc[6];
        for (int m = 0; m < 7; ++m) Bc[m] = Ec[m] + s[m];
    }
}

// Commit of every body: blocks [0, nbmassive) take the massive set, the rest
// the particle slots.
__global__ void __launch_bounds__(128) ra15_commit_kernel(Ra15CommitArgs A) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = A.nsplit, S = A.npcap;
    const bool massive = q < N;
    const int k = massive ? q : q - N;
    if (massive ? (k < 1) : (k >= A.np)) {
        // the central body keeps its (zero) state; copy it through
        if (massive && k == 0)
            for (int c = 0; c < 9; ++c) A.bx_out[c * N] = A.bx[c * N];
        return;
    }
    const double* X = massive ? A.bx : A.px;
    double* XO = massive ? A.bx_out : A.px_out;
    double* Bp = massive ? A.bb : A.pb;
    double* Ep = massive ? A.be : A.pe;
    const int L = massive ? N : S;
    double x1[3], v1[3], a1[3], b[21], e[21], xo[3], vo[3];
    for (int c = 0; c < 3; ++c) {
        x1[c] = X[c * (size_t)L + k];
        v1[c] = X[(3 + c) * (size_t)L + k];
        a1[c] = X[(6 + c) * (size_t)L + k];
    }
    for (int m = 0; m < 21; ++m) {
        b[m] = Bp[(size_t)m * L + k];
        e[m] = Ep[(size_t)m * L + k];
    }
    commit_body(x1, v1, a1, b, e, xo, vo, A.tdid, A.q, A.reset != 0);
    for (int c = 0; c < 3; ++c) {
        XO[c * (size_t)L + k] = xo[c];
        XO[(3 + c) * (size_t)L + k] = vo[c];
        XO[(6 + c) * (size_t)L + k] = a1[c];
    }
    for (int m = 0; m < 21; ++m) {
        Bp[(size_t)m * L + k] = b[m];
        Ep[(size_t)m * L + k] = e[m];
    }
}

// mfo_all of every body: the massive set by one CTA (which also writes the
// table row), then the particles.
__global__ void __launch_bounds__(256) force_massive_kernel(ForceAllArgs A) {
    const int N = A.f.nsplit;
    if (threadIdx.x == 0) row_head(A.bx, A.mbig, A.f, A.table);
    __syncthreads();
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        if (k >= 1 && k < A.f.nbig) {
            double* row = A.table + FT_HEAD + 4 * (k - 1);
            row[0] = A.bx[k]; row[1] = A.bx[N + k]; row[2] = A.bx[2 * N + k]; row[3] = A.mbig[k];
        }
        if (k < 1) {
            A.abig[k] = 0.0; A.abig[N + k] = 0.0; A.abig[2 * N + k] = 0.0;
            continue;
        }
        const double3 a = massive_allforce(k, A.bx, A.bx + 3 * N, A.mbig, A.ngfbig, A.table, A.f, A.status);
        A.abig[k] = a.x; A.abig[N + k] = a.y; A.abig[2 * N + k] = a.z;
    }
}

__global__ void __launch_bounds__(128) force_particle_kernel(ForceAllArgs A) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x, S = A.npcap;
    if (p >= A.np) return;
    const double3 x = make_double3(A.px[p], A.px[S + p], A.px[2 * S + p]);
    const double3 v = make_double3(A.px[3 * S + p], A.px[4 * S + p], A.px[5 * S + p]);
    double g5[5];
    for (int c = 0; c < 5; ++c) g5[c] = A.pconst[(3 + c) * (size_t)S + p];
    const double3 a = particle_allforce(x, v, A.table, A.f.nbig - 1, A.f, A.pconst[p], g5, A.status);
    A.apart[p] = a.x;
    A.apart[S + p] = a.y;
    A.apart[2 * S + p] = a.z;
}

// ---------------------------------------------------------------- screen
__global__ void __launch_bounds__(256) screen_massive_kernel(ScreenArgs A) {
    const int N = A.nsplit, nb = A.nbig - 1;
    const double h = A.h, hm1 = 1.0 / h;
    auto ends = [&](int k) {
        return PairEnds{make_double3(A.b0[k], A.b0[N + k], A.b0[2 * N + k]),
                        make_double3(A.b0[3 * N + k], A.b0[4 * N + k], A.b0[5 * N + k]),
                        make_double3(A.b1[k], A.b1[N + k], A.b1[2 * N + k]),
                        make_double3(A.b1[3 * N + k], A.b1[4 * N + k], A.b1[5 * N + k])};
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
    for (int k = 1 + threadIdx.x; k < A.nbig; k += blockDim.x) {
        box(k, A.boxes + 4 * (k - 1));
        const PairEnds E = ends(k);
        double* d = A.detail + (size_t)(k - 1) * TAB_DETAIL;
        const double3 q[4] = {E.x0, E.v0, E.x1, E.v1};
        for (int w = 0; w < 4; ++w) {
            d[3 * w] = q[w].x;
            d[3 * w + 1] = q[w].y;
            d[3 * w + 2] = q[w].z;
        }
        d[12] = A.rcebig[k];
        d[13] = A.rphysbig[k];
    }
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
        if (pair_classify(I, J, A.rcebig[i], A.rcebig[j], A.rphysbig[i], A.rphysbig[j], h, pc)) {
            const int slot = atomicAdd(&A.status->events, 1);
            if (slot < A.event_cap) {
                pair_record(A.events + slot, I, J, pc, hm1, i + 1, j + 1, A.mbig[j] > A.mbig[i] && j < A.nbig);
                A.event_step[slot] = A.step;
            } else {
                atomicOr(&A.status->overflow, 1);
            }
        }
    }
}

__global__ void __launch_bounds__(128) screen_particle_kernel(ScreenArgs A) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x, S = A.npcap, nb = A.nbig - 1;
    const bool ok = p < A.np;
    double3 x0, v0, x1, v1;
    double lo_x = 0, hi_x = 0, lo_y = 0, hi_y = 0, rce = 0, rphys = 0;
    if (ok) {
        x0 = make_double3(A.p0[p], A.p0[S + p], A.p0[2 * S + p]);
        v0 = make_double3(A.p0[3 * S + p], A.p0[4 * S + p], A.p0[5 * S + p]);
        x1 = make_double3(A.p1[p], A.p1[S + p], A.p1[2 * S + p]);
        v1 = make_double3(A.p1[3 * S + p], A.p1[4 * S + p], A.p1[5 * S + p]);
        rce = A.pconst[S + p];
        rphys = A.pconst[2 * (size_t)S + p];
        const double pad = rce * 1.2;
        box_extent(x0.x, x1.x, v0.x, v1.x, A.h, lo_x, hi_x);
        box_extent(x0.y, x1.y, v0.y, v1.y, A.h, lo_y, hi_y);
        lo_x -= pad; hi_x += pad; lo_y -= pad; hi_y += pad;
    }
    for (int b = 0; b < nb; ++b) {
        const double* bx = A.boxes + 4 * b;
        const bool cand = ok && bx[1] >= lo_x && hi_x >= bx[0] && bx[3] >= lo_y && hi_y >= bx[2];
        const unsigned mask = __ballot_sync(FULLMASK, cand);
        if (!mask) continue;
        const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&A.status->cands, __popc(mask));
        base = __shfl_sync(FULLMASK, base, leader);
        if (!cand) continue;
        const int slot = base + __popc(mask & ((1u << lane) - 1u));
        if (slot >= A.cand_cap) {
            atomicOr(&A.status->overflow, 2);
            continue;
        }
        EncounterCandidate* c = A.cands + slot;
        c->slot = p; c->body = b; c->step = 0; c->id = A.nsplit + A.perm[p] + 1;
        c->rce = rce; c->rphys = rphys;
        c->x0[0] = x0.x; c->x0[1] = x0.y; c->x0[2] = x0.z;
        c->v0[0] = v0.x; c->v0[1] = v0.y; c->v0[2] = v0.z;
        c->x1[0] = x1.x; c->x1[1] = x1.y; c->x1[2] = x1.z;
        c->v1[0] = v1.x; c->v1[1] = v1.y; c->v1[2] = v1.z;
    }
}

int nblocks(int n, int t) { return (n + t - 1) / t; }

}  // namespace

void launch_ra15_sequence(const Ra15Args& a, cudaStream_t s) {
    ensure_constants();
    const int N = a.f.nsplit;
    // x, v, B, G, a1, x1, v1 (57 N), m, ngf, then the force terms
    const size_t smem = sizeof(double) * ((size_t)63 * N + massive_par_scratch(N));
    if (smem <= 200 * 1024) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(ra15_massive_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        // one warp per 32 bodies, at most 8, and with the parallel force terms
        // enough for one term each
        int threads = std::min(256, std::max(32, (N + 31) / 32 * 32));
        if (massive_par_scratch(N)) threads = std::max(threads, std::min(256, (N * N + 31) / 32 * 32));
        ra15_massive_kernel<true><<<1, threads, smem, s>>>(a);
    } else {
        ra15_massive_kernel<false><<<1, 256, 0, s>>>(a);
    }
    if (a.np > 0) ra15_particle_kernel<<<nblocks(a.np, RA15_PARTICLE_THREADS), RA15_PARTICLE_THREADS, 0, s>>>(a);
}

void launch_ra15_commit(const Ra15CommitArgs& a, cudaStream_t s) {
    ensure_constants();
    ra15_commit_kernel<<<nblocks(a.nsplit + a.np, 128), 128, 0, s>>>(a);
}

void launch_force_all(const ForceAllArgs& a, cudaStream_t s) {
    force_massive_kernel<<<1, 256, 0, s>>>(a);
    if (a.np > 0) force_particle_kernel<<<nblocks(a.np, 128), 128, 0, s>>>(a);
}

void launch_screen(const ScreenArgs& a, cudaStream_t s) {
    screen_massive_kernel<<<1, 256, 0, s>>>(a);
    if (a.np > 0 && a.nbig > 1) screen_particle_kernel<<<nblocks(a.np, 128), 128, 0, s>>>(a);
}

}  // namespace mb200

// Energy and angular momentum (mxx_en, mercury6_2.for:7226-7315) of the
// resident system, from heliocentric states through mco_h2b's barycentric
// conversion (mercury6_2.for:2348-2405). Every sum runs in the Fortran's body
// order and statement order, so the result matches a CPU mxx_en on the
// exported arrays bit for bit (the library is built with --fmad=false). The
// pair sums of the potential are independent per body and run one body per
// thread; the running sums over bodies are serial. The massive set holds
// every body up to the last massive one; the massless bodies after it are
// left out, since with finite states each of their terms is an exact zero.
#include "energy.cuh"

namespace mb200 {
namespace {

struct Body {
    double x[3], v[3], m;
};

__device__ __forceinline__ Body body(const EnergyArgs& A, int j) {
    Body b;
    for (int c = 0; c < 3; ++c) {
        b.x[c] = A.big[(size_t)c * A.bs + j];
        b.v[c] = A.big[(size_t)(3 + c) * A.bs + j];
    }
    b.m = A.mbig[j];
    if (A.voff && j >= 1)
        for (int c = 0; c < 3; ++c) b.v[c] = b.v[c] + A.voff[c];
    return b;
}

__global__ void __launch_bounds__(256) energy_kernel(EnergyArgs A) {
    __shared__ double cen[6];  // barycentric x, v of the central body
    const int tid = threadIdx.x, nm = A.nm;
    if (tid == 0) {
        // mco_h2b: the central body's barycentric coordinates
        double mtot = 0.0, x1[3] = {0.0, 0.0, 0.0}, v1[3] = {0.0, 0.0, 0.0};
        for (int j = 1; j < nm; ++j) {
            const Body b = body(A, j);
            mtot = mtot + b.m;
            for (int c = 0; c < 3; ++c) {
                x1[c] = x1[c] + b.m * b.x[c];
                v1[c] = v1[c] + b.m * b.v[c];
            }
        }
        const double temp = -1.0 / (mtot + A.mbig[0]);
        for (int c = 0; c < 3; ++c) {
            cen[c] = temp * x1[c];
            cen[3 + c] = temp * v1[c];
        }
    }
    __syncthreads();
    // pair potential of body j with the bodies after it (barycentric x)
    for (int j = 1 + tid; j < nm; j += blockDim.x) {
        const Body bj = body(A, j);
        double tmp = 0.0;
        if (bj.m != 0.0) {
            const double xj[3] = {bj.x[0] + cen[0], bj.x[1] + cen[1], bj.x[2] + cen[2]};
            for (int k = j + 1; k < nm; ++k) {
                const Body bk = body(A, k);
                if (bk.m == 0.0) continue;
                const double dx = (bk.x[0] + cen[0]) - xj[0];
                const double dy = (bk.x[1] + cen[1]) - xj[1];
                const double dz = (bk.x[2] + cen[2]) - xj[2];
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 != 0.0) tmp = tmp + bk.m / sqrt(r2);
            }
        }
        A.tmp[j] = tmp;
    }
    __syncthreads();
    if (tid != 0) return;
    double l[3] = {A.spin[0], A.spin[1], A.spin[2]}, ke = 0.0, pe = 0.0;
    const double m0 = A.mbig[0];
    for (int j = 0; j < nm; ++j) {
        const Body b = body(A, j);
        double x[3], v[3];
        for (int c = 0; c < 3; ++c) {
            x[c] = j == 0 ? cen[c] : b.x[c] + cen[c];
            v[c] = j == 0 ? cen[3 + c] : b.v[c] + cen[3 + c];
        }
        l[0] = l[0] + b.m * (x[1] * v[2] - x[2] * v[1]);
        l[1] = l[1] + b.m * (x[2] * v[0] - x[0] * v[2]);
        l[2] = l[2] + b.m * (x[0] * v[1] - x[1] * v[0]);
        ke = ke + b.m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    for (int j = 1; j < nm; ++j) {
        const double mj = body(A, j).m;
        if (mj == 0.0) continue;
        pe = pe - A.tmp[j] * mj;
    }
    for (int j = 1; j < nm; ++j) {
        const Body b = body(A, j);
        const double dx = (b.x[0] + cen[0]) - cen[0];
        const double dy = (b.x[1] + cen[1]) - cen[1];
        const double dz = (b.x[2] + cen[2]) - cen[2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 != 0.0) pe = pe - m0 * b.m / sqrt(r2);
    }
    if (A.jcen[0] != 0.0 || A.jcen[1] != 0.0 || A.jcen[2] != 0.0) {
        for (int j = 1; j < nm; ++j) {
            const Body b = body(A, j);
            const double r2 = b.x[0] * b.x[0] + b.x[1] * b.x[1] + b.x[2] * b.x[2];
            const double r_1 = 1.0 / sqrt(r2);
            const double r_2 = r_1 * r_1;
            const double r_4 = r_2 * r_2;
            const double r_6 = r_4 * r_2;
            const double u2 = b.x[2] * b.x[2] * r_2;
            const double u4 = u2 * u2;
            const double u6 = u4 * u2;
            pe = pe + m0 * b.m * r_1 *
                          (A.jcen[0] * r_2 * (1.5 * u2 - 0.5) + A.jcen[1] * r_4 * (4.375 * u4 - 3.75 * u2 + 0.375) +
                           A.jcen[2] * r_6 * (14.4375 * u6 - 19.6875 * u4 + 6.5625 * u2 - 0.3125));
        }
    }
    A.out[0] = 0.5 * ke + pe;
    A.out[1] = sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
}

}  // namespace

void launch_energy(const EnergyArgs& a, cudaStream_t s) { energy_kernel<<<1, 256, 0, s>>>(a); }

}  // namespace mb200

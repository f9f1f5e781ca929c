// mio_ce's close-encounter record encoding on the device (no counterpart in
// the reference's C ABI, whose host encodes every record itself): the record
// body c(1:70) of mercury6_2.for:5456-5510 with mio_fl2c (5885-5918),
// mio_re2c (6926-6957) and mco_x2ov (3057-3086), one thread per record.
// Fortran semantics kept: INT truncates toward zero, real MOD is fmod,
// 10.d0**(-ex) is an integer power by right-to-left binary powering (the
// form gfortran's integer power takes), SIGN(y, x) takes x's sign, and
// mio_ce's overlapping substring assignments leave each field the characters
// the next field does not overwrite.
#include <cmath>
#include <vector>

#include "../../include/mercury_b200.h"
#include "context.cuh"

namespace mb200 {
namespace {

constexpr double IO_PI = 3.141592653589793;
constexpr double IO_TWOPI = IO_PI * 2.0;

// x^m for integer m: square-and-multiply over the bits of |m| from the lowest,
// then the reciprocal for negative m.
__device__ double int_power(double x, int m) {
    unsigned n = m < 0 ? 0u - (unsigned)m : (unsigned)m;
    double y = (n & 1u) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n & 1u) y = y * x;
    }
    return m < 0 ? 1.0 / y : y;
}

__device__ void re2c(double x, double xmin, double xmax, unsigned char out[8]) {
    for (int j = 0; j < 8; ++j) out[j] = ' ';
    const double y = (x - xmin) / (xmax - xmin);
    if (y >= 1.0) {
        for (int j = 0; j < 8; ++j) out[j] = 255;
    } else if (y > 0.0) {
        double z = y;
        for (int j = 0; j < 8; ++j) {
            z = fmod(z, 1.0) * 224.0;
            out[j] = (unsigned char)((int)z + 32);
        }
    }
}

// log10 for mio_fl2c's exponent: an exact power of ten gets its exact
// logarithm (the host library's correctly rounded value there).
__device__ double log10_exponent(double ax) {
    const double l = log10(ax);
    const double k = rint(l);
    if (fabs(l - k) < 1e-9 && fabs(k) < 300.0 && int_power(10.0, (int)k) == ax) return k;
    return l;
}

// mio_fl2c; the Fortran leaves the exponent undefined for x = 0, 0 here.
__device__ void fl2c(double x, unsigned char out[8]) {
    int ex = 0;
    double y;
    if (x == 0.0) {
        y = 0.5;
    } else {
        const double ax = fabs(x);
        ex = (int)log10_exponent(ax);
        if (ax >= 1.0) ex = ex + 1;
        y = ax * int_power(10.0, -ex);
        if (y == 1.0) {
            y = y * 0.1;
            ex = ex + 1;
        }
        y = copysign(y, x) * 0.5 + 0.5;
    }
    re2c(y, 0.0, 1.0, out);
    ex = ex + 112;
    if (ex > 223) ex = 223;
    if (ex < 0) ex = 0;
    out[7] = (unsigned char)(ex + 32);
}

struct CeArgs {
    const MercuryEvent* ev;
    const int* which;     // record index of line k
    int n;
    double mcen, rcen, rmax, rfac;
    unsigned char* lines; // [n][70]
};

__global__ void __launch_bounds__(128) mio_ce_kernel(CeArgs A) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.n) return;
    const MercuryEvent& e = A.ev[A.which[k]];
    unsigned char c[80];
    for (int q = 0; q < 80; ++q) c[q] = ' ';
    unsigned char f[8];
    auto put = [&](int first, int last) {  // c(first:last) = f, 1-based, blank-padded
        for (int q = first; q <= last; ++q) c[q - 1] = q - first < 8 ? f[q - first] : ' ';
    };
    fl2c(e.time, f);
    put(1, 8);
    re2c(double(e.i - 1), 0.0, 11239423.99, f);
    put(9, 16);
    re2c(double(e.j - 1), 0.0, 11239423.99, f);
    put(12, 19);
    fl2c(e.distance, f);
    put(15, 22);
#pragma unroll 1
    for (int b = 0; b < 2; ++b) {
        const double* xv = b == 0 ? e.xi : e.xj;
        const int o = b == 0 ? 23 : 47;
        // mco_x2ov with m = 0
        const double x = xv[0], y = xv[1], z = xv[2], u = xv[3], v = xv[4], w = xv[5];
        const double r = sqrt(x * x + y * y + z * z);
        const double v2 = u * u + v * v + w * w;
        const double v1 = sqrt(v2);
        const double be = (A.mcen + 0.0) / r;
        const double ke = 0.5 * v2;
        const double fr = log10(fmin(fmax(r, A.rcen), A.rmax) / A.rcen);
        const double temp = ke / be;
        const double fv = 1.0 / (1.0 + 2.0 * temp * temp);
        const double theta = fmod(acos(z / r) + IO_TWOPI, IO_TWOPI);
        const double vtheta = fmod(acos(w / v1) + IO_TWOPI, IO_TWOPI);
        const double phi = fmod(atan2(y, x) + IO_TWOPI, IO_TWOPI);
        const double vphi = fmod(atan2(v, u) + IO_TWOPI, IO_TWOPI);
        re2c(fr, 0.0, A.rfac, f);
        put(o, o + 7);
        re2c(theta, 0.0, IO_PI, f);
        put(o + 4, o + 11);
        re2c(phi, 0.0, IO_TWOPI, f);
        put(o + 8, o + 15);
        re2c(fv, 0.0, 1.0, f);
        put(o + 12, o + 19);
        re2c(vtheta, 0.0, IO_PI, f);
        put(o + 16, b == 0 ? o + 23 : o + 27);
        re2c(vphi, 0.0, IO_TWOPI, f);
        put(o + 20, b == 0 ? o + 27 : o + 31);
    }
    unsigned char* out = A.lines + 70 * (size_t)k;
    for (int q = 0; q < 70; ++q) out[q] = c[q];
}

struct Encoder {
    DBuf<MercuryEvent> ev;
    DBuf<int> which;
    DBuf<unsigned char> lines;
    cudaStream_t stream = nullptr;
};

Encoder& encoder() {
    static Encoder e;
    return e;
}

}  // namespace
}  // namespace mb200

using namespace mb200;

extern "C" int mercury_b200_encode_ce(const MercuryEvent* events, int n, double mcen, double rcen, double rmax,
                                      char* lines, int* count) {
    Encoder& E = encoder();
    try {
        if (n < 0 || !count || (n > 0 && (!events || !lines))) throw std::runtime_error("invalid encoder arguments");
        if (!(rcen > 0.0) || !(rmax > rcen) || !(mcen > 0.0)) throw std::runtime_error("invalid encoder radii or mass");
        std::vector<int> which;
        for (int q = 0; q < n; ++q)
            if (events[q].kind & 1) which.push_back(q);
        const int m = (int)which.size();
        *count = m;
        if (m == 0) return 0;
        if (!E.stream) check(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking), "stream");
        E.ev.reserve(n);
        E.which.reserve(m);
        E.lines.reserve((size_t)70 * m);
        check(cudaMemcpyAsync(E.ev.p, events, sizeof(MercuryEvent) * n, cudaMemcpyHostToDevice, E.stream), "events");
        check(cudaMemcpyAsync(E.which.p, which.data(), sizeof(int) * m, cudaMemcpyHostToDevice, E.stream), "events");
        CeArgs a{};
        a.ev = E.ev.p;
        a.which = E.which.p;
        a.n = m;
        a.mcen = mcen;
        a.rcen = rcen;
        a.rmax = rmax;
        a.rfac = std::log10(rmax / rcen);
        a.lines = E.lines.p;
        mio_ce_kernel<<<(m + 127) / 128, 128, 0, E.stream>>>(a);
        check(cudaGetLastError(), "launch");
        check(cudaMemcpyAsync(lines, E.lines.p, (size_t)70 * m, cudaMemcpyDeviceToHost, E.stream), "lines");
        check(cudaStreamSynchronize(E.stream), "encode");
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

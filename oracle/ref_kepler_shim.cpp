// Test infrastructure only: compiles the reference's own Kepler drift
// (mercury_cuda_kepler.cuh, an f2c translation of SWIFT drift_*) for the host,
// so the oracle's restatement of mercury6_2.for:7602-8330 can be checked
// against the reference's code on identical inputs. The reference header is
// read from the reference tree at build time; nothing of it is copied here.
#include <cmath>
using std::cos;
using std::fabs;
using std::fmod;
using std::pow;
using std::sqrt;
#define __device__
#include "mercury_cuda_kepler.cuh"

extern "C" int ref_drift_one(double mu, double* xv, double dt) {
    int flag = 0;
    drift_one__(&mu, xv, xv + 1, xv + 2, xv + 3, xv + 4, xv + 5, &dt, &flag);
    return flag;
}

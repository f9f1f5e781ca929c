// Energy and angular momentum of the resident system (mxx_en with mco_h2b,
// mercury6_2.for:7226-7315 and 2348-2405) computed on the device from the
// state the export call would return, in the Fortran's statement order.
#pragma once
#include <cuda_runtime.h>

namespace mb200 {

struct EnergyArgs {
    int nm;              // bodies 0..nm-1: the massive set, which ends at the last massive body
    const double* big;   // SoA x(3), v(3) rows, stride bs
    int bs;
    const double* mbig;  // masses of the massive set
    const double* voff;  // velocity shift added to bodies j >= 1 (democratic heliocentric), or null
    double jcen[3];
    double spin[3];      // the spin angular momenta, summed in body order
    double* tmp;         // [nm] scratch: each body's pair potential sum
    double* out;         // e, l2
};

void launch_energy(const EnergyArgs& a, cudaStream_t s);

}  // namespace mb200

// One MVS step that allocates no device memory.
//
// Who needs it: hosts that cannot call cudaMalloc. Examples are a host whose
// device memory is owned by another allocator or budget (a framework's pool),
// and a host that must not stall the whole device, which cudaMalloc/cudaFree
// can do because they synchronize implicitly. Such a caller keeps every
// input and output array in memory it already owns and passes device pointers
// to them. The scratch this step needs (the Big-body step table and its detail
// rows, the encounter candidates, the status word and an identity slot map)
// lives in one fixed static device array below, so nothing is allocated per
// call. Every GPU that loads this library holds that array until the process
// exits.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>

#include "../../include/mercury_b200.h"
#include "mvs.cuh"

namespace mb200 {
namespace {

// Limits of the allocation-free step (the scratch below is sized for them).
constexpr int NOALLOC_MAX_BIG = 64;          // nbig, central body included
constexpr int NOALLOC_MAX_PARTICLES = 1 << 18;
constexpr int NOALLOC_MAX_CANDIDATES = 8192;
constexpr int NOALLOC_MAX_EVENTS = 8192;

// Scratch layout in doubles.
constexpr size_t SCR_STATUS = 0;                                        // DeviceStatus (32 bytes)
constexpr size_t SCR_TAB = 8;                                           // 2 table rows
constexpr size_t SCR_DETAIL = SCR_TAB + 2 * (TAB_HEAD + TAB_BODY * NOALLOC_MAX_BIG);
constexpr size_t SCR_PERM = SCR_DETAIL + (size_t)TAB_DETAIL * NOALLOC_MAX_BIG;   // int slot map
constexpr size_t SCR_STEP = SCR_PERM + NOALLOC_MAX_PARTICLES / 2;               // int event step tags
constexpr size_t SCR_CANDS = SCR_STEP + NOALLOC_MAX_EVENTS / 2;                 // EncounterCandidate
constexpr size_t SCR_TOTAL = SCR_CANDS + (size_t)NOALLOC_MAX_CANDIDATES * (sizeof(EncounterCandidate) / 8);

// About 2.2 MB per device.
static __device__ __align__(256) double noalloc_scratch[SCR_TOTAL];

__global__ void identity_slots(int* perm, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) perm[k] = k;
}

// Pair records hold tmin; add the step's end time (tmin + (time + h), as
// mce_stat computes tclo = tmin + time).
__global__ void finish_pair_times(MercuryEvent* ev, const DeviceStatus* st, int cap, double tend) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = min(st->events, cap);
    if (k < n) ev[k].time = ev[k].time + tend;
}

// The device address of the scratch array, looked up once per device (with
// that device current): host code may not use the symbol itself as an
// address. The first call on a device also fills the identity slot map, on
// the caller's stream, and waits for that stream; host threads making their
// first calls at the same time take turns (the mutex), and later calls read
// the published address without locking.
constexpr int MAX_DEVICES = 64;
std::atomic<double*> scratch_address[MAX_DEVICES] = {};
std::mutex scratch_setup;

double* scratch_for_current_device(cudaStream_t s) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return nullptr;
    double* ptr = scratch_address[dev].load(std::memory_order_acquire);
    if (ptr) return ptr;
    std::lock_guard<std::mutex> lock(scratch_setup);
    ptr = scratch_address[dev].load(std::memory_order_acquire);
    if (ptr) return ptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), noalloc_scratch) != cudaSuccess) return nullptr;
    int* perm = reinterpret_cast<int*>(ptr + SCR_PERM);
    identity_slots<<<(NOALLOC_MAX_PARTICLES + 255) / 256, 256, 0, s>>>(perm, NOALLOC_MAX_PARTICLES);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return nullptr;
    scratch_address[dev].store(ptr, std::memory_order_release);
    return ptr;
}

int fail(const char* what) {
    std::fprintf(stderr, "MERCURY CUDA: %s\n", what);
    return 1;
}

}  // namespace
}  // namespace mb200

using namespace mb200;

extern "C" int mercury_b200_mvs_step_noalloc(int nbig, int np, const double* mbig, const double* rcebig,
                                             const double* rphysbig, const double* ngfbig, const double* big_in,
                                             double* big_out, const double* part_in, double* part_out,
                                             const double* part_const, int ngflag, double time, double h,
                                             int reset, MercuryEvent* events, int event_cap, int* event_count,
                                             void* stream) {
    if (nbig < 1 || nbig > NOALLOC_MAX_BIG) return fail("noalloc step: nbig must be 1..64");
    if (np < 0 || np > NOALLOC_MAX_PARTICLES) return fail("noalloc step: at most 262144 particles");
    if (event_cap < 0 || event_cap > NOALLOC_MAX_EVENTS) return fail("noalloc step: event_cap must be 0..8192");
    if (!(h != 0.0)) return fail("noalloc step: zero step");
    // An error left by earlier work of the caller is reported as such (and
    // left in place), not blamed on this step.
    if (cudaPeekAtLastError() != cudaSuccess) return fail("noalloc step: a CUDA error was pending before the call");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* scr = scratch_for_current_device(s);
    if (!scr) return fail("noalloc step: scratch address lookup failed");
    DeviceStatus* status = reinterpret_cast<DeviceStatus*>(scr + SCR_STATUS);
    double* tab = scr + SCR_TAB;
    double* detail = scr + SCR_DETAIL;
    int* perm = reinterpret_cast<int*>(scr + SCR_PERM);
    int* steps = reinterpret_cast<int*>(scr + SCR_STEP);
    EncounterCandidate* cands = reinterpret_cast<EncounterCandidate*>(scr + SCR_CANDS);
    // The array keeps the previous call's contents: clear the counters.
    if (cudaMemsetAsync(status, 0, sizeof(DeviceStatus), s) != cudaSuccess) return fail("noalloc step: memset");
    int npcap = np + (np & 1);  // particle columns are padded to an even length
    if (npcap < 2) npcap = 2;

    MvsBigArgs b{};
    b.nbig = nbig;
    b.ngflag = ngflag;
    b.obl = 0;
    b.reset = reset ? 1 : 0;
    b.nsteps = 1;
    b.central = 0;
    b.step0 = 0;
    b.h = h;
    b.m = mbig;
    b.rce = rcebig;
    b.rphys = rphysbig;
    b.ngf = ngfbig;
    b.in = BigState{const_cast<double*>(big_in), const_cast<double*>(big_in) + 3 * nbig,
                    const_cast<double*>(big_in) + 6 * nbig};
    b.out = BigState{big_out, big_out + 3 * nbig, big_out + 6 * nbig};
    b.tab = tab;
    b.detail = detail;
    b.events = events;
    b.event_step = steps;
    b.event_cap = event_cap;
    b.status = status;
    launch_mvs_big(b, s);
    if (cudaGetLastError() != cudaSuccess) return fail("noalloc step: Big-body launch failed");

    if (np > 0) {
        MvsParticleArgs p{};
        p.np = np;
        p.npcap = npcap;
        p.nb = nbig - 1;
        p.nbig = nbig;
        p.nsteps = 1;
        p.reset = b.reset;
        p.central = 0;
        p.step0 = 0;
        p.ngf_on = (ngflag == 1 || ngflag == 3);
        p.h = h;
        p.xin = part_in;
        p.xout = part_out;
        p.m = part_const;
        p.rce = part_const + npcap;
        p.rphys = part_const + 2 * (size_t)npcap;
        p.ngf = part_const + 3 * (size_t)npcap;
        p.perm = perm;
        p.tab = tab;
        p.detail = detail;
        p.events = events;
        p.event_step = steps;
        p.event_cap = event_cap;
        p.cands = cands;
        p.cand_cap = NOALLOC_MAX_CANDIDATES;
        p.status = status;
        // the central mass: read back from the caller's device array
        double mu = 0.0;
        if (cudaMemcpyAsync(&mu, mbig, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return fail("noalloc step: reading the central mass failed");
        p.mu = mu;
        launch_mvs_particles(p, s, 128);
        if (cudaGetLastError() != cudaSuccess) return fail("noalloc step: particle launch failed");
        if (nbig > 1) {
            ClassifyArgs c{};
            c.nb = nbig - 1;
            c.nbig = nbig;
            c.h = h;
            c.detail = detail;
            c.cands = cands;
            c.cand_cap = NOALLOC_MAX_CANDIDATES;
            c.events = events;
            c.event_step = steps;
            c.event_cap = event_cap;
            c.status = status;
            launch_classify(c, s);
            if (cudaGetLastError() != cudaSuccess) return fail("noalloc step: classify launch failed");
        }
    }
    if (event_cap > 0) {
        finish_pair_times<<<(event_cap + 255) / 256, 256, 0, s>>>(events, status, event_cap, time + h);
        if (cudaGetLastError() != cudaSuccess) return fail("noalloc step: record-time launch failed");
    }
    DeviceStatus host_status{};
    if (cudaMemcpyAsync(&host_status, status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail("noalloc step: the step's kernels failed");
    if (event_count) *event_count = host_status.events;
    if (host_status.fault) return fail("MVS force failed");
    if (host_status.overflow) return fail("noalloc step: event or candidate capacity exceeded");
    return 0;
}

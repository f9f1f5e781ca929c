// The drop-in C ABI (include/mercury_cuda.h) and the MVS extension entry
// points (include/mercury_b200.h): host orchestration of the device context.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>

#include <cub/device/device_radix_sort.cuh>

#include "../../include/mercury_b200.h"
#include "context.cuh"
#include "mvs_device.cuh"
#include "bs.cuh"
#include "hybrid.cuh"
#include "radau.cuh"
#include "energy.cuh"

namespace mb200 {

// The resident system and the compact close-encounter subsystem of HYBRID
// (mercury_cuda_encounter_enter switches to the second until _exit), as the
// reference swaps its whole context (mercury_cuda_hybrid.cuh:101-126); both
// keep their allocations for the next use.
Context g_contexts[2];
int g_active = 0;

Context& ctx() { return g_contexts[g_active]; }
int active_context() { return g_active; }

// Cross-process reduction of the adaptive step control's maxima (particles of
// one system split across processes); null: one process.
mercury_b200_reduce_fn g_step_reduce = nullptr;
void* g_step_reduce_user = nullptr;

// Replace each value by its maximum over the processes sharing the resident
// system (the encounter subsystem of HYBRID is never shared).
void reduce_step_maxima(double* values, int count) {
    if (g_step_reduce && g_active == 0) g_step_reduce(values, count, g_step_reduce_user);
}

int report(const std::exception& e) {
    std::fprintf(stderr, "MERCURY CUDA: %s\n", e.what());
    return 1;
}

// Failure injection for testing a host's error handling without a GPU fault
// (the reference tests rewrite and relink its CPU stub for this,
// tests/test_edges.py:18-32): MERCURY_B200_FAIL lists, comma-separated, the
// points that fail on purpose: an entry point's name without its prefix
// (configure, upload, step, events, download, export, force, limits,
// hybrid_begin, hybrid_finish, encounter_enter, encounter_update, advance),
// "memory" (the upload's workspace guard sees no free device memory) or
// "growth" (an event-buffer growth fails). Read on every call.
bool injected(const char* point) {
    const char* env = std::getenv("MERCURY_B200_FAIL");
    if (!env || !*env) return false;
    const size_t len = std::strlen(point);
    for (const char* p = env; *p;) {
        const char* end = std::strchr(p, ',');
        const size_t n = end ? (size_t)(end - p) : std::strlen(p);
        if (n == len && std::strncmp(p, point, n) == 0) return true;
        if (!end) break;
        p = end + 1;
    }
    return false;
}

void inject(const char* point) {
    if (injected(point)) throw std::runtime_error(std::string("injected failure: ") + point);
}

namespace {

// Host rows (Fortran layout, row j = body j) to the device SoA: Big bodies by
// index, Small body j to its slot inv[j - nbig] of the particle arrays.
__global__ void scatter_kernel(const double* rows, int n, int comps, int nbig, double* big, int bs, double* part,
                               int ps, const int* inv) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int c = 0; c < comps; ++c) {
        const double v = rows[(size_t)j * comps + c];
        if (j < nbig) {
            if (big) big[(size_t)c * bs + j] = v;
        } else {
            part[(size_t)c * ps + inv[j - nbig]] = v;
        }
    }
}

__global__ void gather_kernel(double* rows, int n, int comps, int nbig, const double* big, int bs,
                              const double* part, int ps, const int* inv) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int c = 0; c < comps; ++c)
        rows[(size_t)j * comps + c] = j < nbig ? big[(size_t)c * bs + j] : part[(size_t)c * ps + inv[j - nbig]];
}

// mce_cent over every body for the drop-in events call (mercury6_2.for:1059-1167):
// start-of-step states from the previous buffers, end states from the current.
struct CentralArgs {
    int nbig, np, npcap;
    double mu, h, rcen;
    const double *big0, *big1, *part0, *part1, *pm, *mbig;
    const double *voff0, *voff1;   // velocity shifts to heliocentric (HYBRID), or null
    const int* perm;
    MercuryEvent* events;
    int* event_step;
    int cap;
    DeviceStatus* status;
};

// Drops the central-body records from the first status->events records (one
// thread: a step's few hundred records, on the rare call whose radius or step
// differs from the one the step screened with).
__global__ void drop_central_kernel(MercuryEvent* ev, int* ev_step, int cap, DeviceStatus* st) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int n = min(st->events, cap);
    int m = 0;
    for (int k = 0; k < n; ++k) {
        if (ev[k].kind == EV_CENTRAL) continue;
        if (m != k) {
            ev[m] = ev[k];
            ev_step[m] = ev_step[k];
        }
        ++m;
    }
    st->events = m;
}

__global__ void central_kernel(CentralArgs A) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = A.nbig - 1, total = nb + A.np;
    bool hit = false;
    double temp = 0.0;
    int id = 0;
    if (q < total) {
        double3 p0, u0, p1, u1;
        double mj;
        if (q < nb) {
            const int k = q + 1, N = A.nbig;
            p0 = make_double3(A.big0[k], A.big0[N + k], A.big0[2 * N + k]);
            u0 = make_double3(A.big0[3 * N + k], A.big0[4 * N + k], A.big0[5 * N + k]);
            p1 = make_double3(A.big1[k], A.big1[N + k], A.big1[2 * N + k]);
            u1 = make_double3(A.big1[3 * N + k], A.big1[4 * N + k], A.big1[5 * N + k]);
            mj = A.mbig[k];
            id = k + 1;
        } else {
            const int p = q - nb, S = A.npcap;
            p0 = make_double3(A.part0[p], A.part0[S + p], A.part0[2 * S + p]);
            u0 = make_double3(A.part0[3 * S + p], A.part0[4 * S + p], A.part0[5 * S + p]);
            p1 = make_double3(A.part1[p], A.part1[S + p], A.part1[2 * S + p]);
            u1 = make_double3(A.part1[3 * S + p], A.part1[4 * S + p], A.part1[5 * S + p]);
            mj = A.pm[p];
            id = A.nbig + A.perm[p] + 1;
        }
        if (A.voff0) {
            u0 = make_double3(u0.x + A.voff0[0], u0.y + A.voff0[1], u0.z + A.voff0[2]);
            u1 = make_double3(u1.x + A.voff1[0], u1.y + A.voff1[1], u1.z + A.voff1[2]);
        }
        hit = central_impact(p0, u0, p1, u1, A.mu, mj, A.h, A.rcen, temp);
    }
    if (hit) {
        const int slot = atomicAdd(&A.status->events, 1);
        if (slot < A.cap) {
            MercuryEvent rec = {};
            rec.i = 1;
            rec.j = id;
            rec.kind = EV_CENTRAL;
            rec.time = temp;
            rec.distance = A.rcen;
            store_event(A.events + slot, rec);
            A.event_step[slot] = 0;
        } else {
            atomicExch(&A.status->overflow, 1);
        }
    }
}

int blocks(int n, int t = 256) { return (n + t - 1) / t; }
int reorder_slots(int src, double h, cudaStream_t st);

// Steps after which a fused run re-sorts the particle slots by drift path.
constexpr int ORDER_EVERY = 16;

bool is_mvs(int alg) { return alg == 1 || alg == 9; }

// Device time of the drop-in calls (both contexts) and the kernels they
// launched, since the last reset.
double g_dropin_ms = 0.0;

// > 0: the starting capacity of the record and candidate buffers of each
// upload (mercury_b200_set_event_capacity).
int g_event_cap = 0;

// Adds the device time of one drop-in call (CUDA events on the library
// stream around it) to the total.
struct DropinTimer {
    Context& c;
    DropinTimer() : c(ctx()) { check(cudaEventRecord(c.d0, c.stream), "event"); }
    ~DropinTimer() {
        float ms = 0.0f;
        if (cudaEventRecord(c.d1, c.stream) == cudaSuccess && cudaEventSynchronize(c.d1) == cudaSuccess &&
            cudaEventElapsedTime(&ms, c.d0, c.d1) == cudaSuccess)
            g_dropin_ms += ms;
    }
};

// Device bytes an upload of n bodies holds: the double-buffered particle
// state and constants, the slot maps, the upload stage, the transfer rows,
// the fused run's snapshot and the record buffers (~0.8 KB a body), plus the
// per-body B and E series of RA15 (algorithm 4).
size_t workspace_bytes(int n, int algorithm) {
    const size_t per_body = 800 + (algorithm == 4 ? 336 : 0);
    return (size_t)n * per_body;
}

void require_system() {
    if (ctx().n <= 0) throw std::runtime_error("no system uploaded");
}

void ensure_events(int cap) {
    Context& c = ctx();
    if ((int)c.events.n < cap) {
        if (injected("growth") && c.events.n > 0) throw std::runtime_error("event buffer growth failed");
        c.events.reserve(cap);
        c.event_step.reserve(cap);
    }
}

void read_status() {
    Context& c = ctx();
    check(cudaMemcpyAsync(c.status_host, c.status.p, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, c.stream), "status");
    check(cudaStreamSynchronize(c.stream), "step");
}

// Fixed-size table space for a run of `rows` table rows and `steps` detail rows.
void ensure_tables(int rows, int steps) {
    Context& c = ctx();
    const int nb = c.nbig - 1;
    c.tab.reserve((size_t)rows * tab_stride(nb));
    c.detail.reserve((size_t)std::max(1, steps) * std::max(1, nb) * TAB_DETAIL);
}

MvsBigArgs big_args(int in, int out, int nsteps, int reset, int central, int step0, double h, double rcen,
                    double* tab, double* detail) {
    Context& c = ctx();
    MvsBigArgs a{};
    a.nbig = c.nbig;
    a.nmass = c.nsplit;
    a.ngflag = c.ngflag;
    a.obl = (c.jcen[0] != 0.0 || c.jcen[1] != 0.0 || c.jcen[2] != 0.0);
    a.reset = reset;
    a.nsteps = nsteps;
    a.central = central;
    a.step0 = step0;
    for (int k = 0; k < 3; ++k) a.jcen[k] = c.jcen[k];
    a.h = h;
    a.rcen = rcen;
    a.m = c.mbig.p;
    a.rce = c.rcebig.p;
    a.rphys = c.rphysbig.p;
    a.ngf = c.ngfbig.p;
    a.in = c.big(in);
    a.out = c.big(out);
    a.tab = tab;
    a.detail = detail;
    a.events = c.events.p;
    a.event_step = c.event_step.p;
    a.event_cap = (int)c.events.n;
    a.status = c.status.p;
    return a;
}

MvsParticleArgs particle_args(int in, int out, int nsteps, int reset, int central, int step0, double h,
                              double rcen, const double* tab, const double* detail) {
    Context& c = ctx();
    MvsParticleArgs a{};
    a.np = c.np;
    a.npcap = c.npcap;
    a.nb = c.nbig - 1;
    a.nbig = c.nsplit;   // particle ids follow the bodies held by the Big-body CTA
    a.nsteps = nsteps;
    a.reset = reset;
    a.central = central;
    a.step0 = step0;
    a.ngf_on = (c.ngflag == 1 || c.ngflag == 3);
    a.mu = c.m_host[0];
    a.h = h;
    a.rcen = rcen;
    for (int k = 0; k < 3; ++k) a.jcen[k] = c.jcen[k];
    a.xin = c.pstate[in].p;
    a.xout = c.pstate[out].p;
    a.m = c.pm();
    a.rce = c.prce();
    a.rphys = c.prphys();
    a.ngf = c.pngf();
    a.perm = c.permp();
    a.tab = tab;
    a.detail = detail;
    a.events = c.events.p;
    a.event_step = c.event_step.p;
    a.event_cap = (int)c.events.n;
    a.cands = c.cands.p;
    a.cand_cap = (int)c.cands.n;
    a.status = c.status.p;
    return a;
}

// Particle kernel of one launch followed by the classification of its
// encounter candidates into event records (same stream, the records, status
// and candidates pa names). detail is the base of the run's pair details: a
// candidate carries its step within the run.
void particles_and_events(const MvsParticleArgs& pa, const double* detail, cudaStream_t s) {
    Context& c = ctx();
    check(cudaMemsetAsync(pa.tiles ? pa.tiles : &pa.status->next_tile, 0, sizeof(int), s), "memset");
    launch_mvs_particles(pa, s, c.particle_threads);
    ClassifyArgs ca{};
    ca.nb = c.nbig - 1;
    ca.nbig = c.nbig;
    ca.h = pa.h;
    ca.detail = detail;
    ca.cands = pa.cands;
    ca.cand_cap = pa.cand_cap;
    ca.events = pa.events;
    ca.event_step = pa.event_step;
    ca.event_cap = pa.event_cap;
    ca.status = pa.status;
    ca.step_base = 0;
    if (ca.nb > 0) launch_classify(ca, s);
    check(cudaMemsetAsync(&pa.status->cands, 0, sizeof(int), s), "memset");
}

// Candidate room for a launch of `steps` steps: box overlaps run at 2-4 % of
// the particles per step on a system with 1 % of its particles near planets,
// so steps x np / 25, kept from one run to the next (not with a fixed
// starting capacity set for tests, which exercise the overflow path).
void ensure_candidates(int steps) {
    Context& c = ctx();
    if (g_event_cap > 0) return;
    const size_t want = (size_t)std::max(1, steps) * (size_t)c.np / 25 + 16384;
    if (c.cands.n < want) c.cands.reserve(want);
}

// Grows the event or candidate buffer after an overflow flagged in the status.
void grow_after_overflow() {
    Context& c = ctx();
    // a quarter of headroom: the next run of a similar system rarely needs more
    if (c.status_host->overflow & 1) {
        const long long need = c.status_host->events;
        ensure_events((int)std::min<long long>(INT32_MAX / 2, std::max<long long>(2LL * c.events.n,
                                                                                   need + need / 4 + 1024)));
    }
    if (c.status_host->overflow & 2) {
        c.cands.reserve(2 * c.cands.n + 4096);
    }
}

// The per-step MVS path (one mercury_cuda_step per step, as mal_hcon calls
// it) runs the next step ahead: as soon as a step is committed, the next step
// with the same h (Big bodies, particles, their pair records and status) runs
// on the second stream into spare buffers while the host handles this step's
// events, and its status and first records are read back into pinned memory
// on that stream. The next mercury_cuda_step with the same h, the same
// central radius and no reset takes it: the spare states become the step's
// output (the pre-step state stays in place for download(previous)) and the
// records and status are already on the host. A speculative step that
// faulted or overflowed a buffer is dropped and the step is made again on the
// library stream, which reports or grows as usual.
//
// The Big bodies never feel the particles, so the Big-body step after the
// speculative one runs on a third stream beside the speculative particles
// (in the CTA slot the particle grid leaves free), and the next speculative
// step starts from its output: the particles' step is then the only kernel
// on the critical path of a step.
//
// Every call that may change the system or the buffers the speculative steps
// read first drops them (and waits for them); the calls that run beside them
// (events, download, export, energy) touch none of their outputs. The
// candidate buffer is shared: only steps and runs use it, and they drop the
// speculation first.
constexpr int AHEAD_RECORDS = 1024;   // records a Big-body step run ahead may hold

// Copies the records of a Big-body step run ahead to the head of a step's
// record buffer and starts that step's status from its count and faults.
__global__ void spec_merge_kernel(const DeviceStatus* ss, const MercuryEvent* sev, const int* sstep, int scap,
                                  DeviceStatus* st, MercuryEvent* ev, int* ev_step, int cap) {
    const int n = ss->events;
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        st->events = n;
        st->fault |= ss->fault;
        if (n > scap || n > cap || ss->overflow) st->overflow |= 1;
    }
    const int m = min(n, min(scap, cap));
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        store_event(ev + k, sev[k]);
        ev_step[k] = sstep[k];
    }
}

// Waits for the speculative step (host-side: later calls may copy into its
// inputs synchronously); the Big-body step ahead keeps running.
void spec_wait() {
    Context& c = ctx();
    if (!c.spec_live) return;
    c.spec_live = false;
    check(cudaEventSynchronize(c.spec_done), "step");
}

void spec_drop() {
    Context& c = ctx();
    spec_wait();
    if (!c.ah_live) return;
    c.ah_live = false;
    check(cudaEventSynchronize(c.ah_done), "step");
}

// An entry point that may change the system or read it in a way a step
// ahead does not expect: no step ahead, no records waiting on the host.
void drop_speculation() {
    spec_drop();
    ctx().head_ready = false;
}

// Resizes b to exactly n elements (a swapped-in record buffer keeps the
// library's event capacity).
template <class T> void reserve_exact(DBuf<T>& b, size_t n) {
    if (b.n != n) b.release();
    b.reserve(n);
}

BigState big_state_at(double* p, int nsplit) {
    BigState b;
    b.x = p;
    b.v = p + 3 * (size_t)nsplit;
    b.a = p + 6 * (size_t)nsplit;
    return b;
}

void spec_launch(double h, double rcen) {
    Context& c = ctx();
    const int nb = c.nbig - 1;
    const int cen = rcen > 0.0 ? 1 : 0;
    const size_t big_el = (size_t)9 * c.nsplit, tab_el = (size_t)2 * tab_stride(nb);
    const size_t det_el = (size_t)std::max(1, nb) * TAB_DETAIL;
    c.spec_big.reserve(big_el);
    c.spec_part.reserve((size_t)9 * c.npcap);
    c.spec_tab.reserve(tab_el);
    c.spec_detail.reserve(det_el);
    reserve_exact(c.spec_events, c.events.n);
    reserve_exact(c.spec_event_step, c.events.n);
    c.spec_status.reserve(1);
    c.ah_state.reserve(big_el);
    c.ah_tab.reserve(tab_el);
    c.ah_detail.reserve(det_el);
    c.ah_events.reserve(AHEAD_RECORDS);
    c.ah_event_step.reserve(AHEAD_RECORDS);
    c.ah_status.reserve(1);
    if (!c.spec_done) {
        for (cudaEvent_t* e : {&c.spec_done, &c.spec_ready, &c.ah_done, &c.spec_merged})
            check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "event");
    }
    cudaStream_t s = c.stream_big, sa = c.stream_ahead;
    check(cudaEventRecord(c.spec_ready, c.stream), "event");
    check(cudaStreamWaitEvent(s, c.spec_ready, 0), "wait");
    const int cap = (int)c.spec_events.n;
    check(cudaMemsetAsync(c.spec_status.p, 0, sizeof(DeviceStatus), s), "memset");
    if (c.ah_live && c.ah_h == h && c.ah_rcen == rcen) {
        // this step's Big bodies ran ahead: their state, table rows and
        // details become the step's, their records its first records
        check(cudaStreamWaitEvent(s, c.ah_done, 0), "wait");
        std::swap(c.spec_big, c.ah_state);
        std::swap(c.spec_tab, c.ah_tab);
        std::swap(c.spec_detail, c.ah_detail);
        spec_merge_kernel<<<4, 256, 0, s>>>(c.ah_status.p, c.ah_events.p, c.ah_event_step.p, AHEAD_RECORDS,
                                            c.spec_status.p, c.spec_events.p, c.spec_event_step.p, cap);
    } else {
        spec_drop();
        MvsBigArgs a = big_args(c.cur, 1 - c.cur, 1, 0, cen, 0, h, rcen, c.spec_tab.p, c.spec_detail.p);
        a.out = big_state_at(c.spec_big.p, c.nsplit);
        a.events = c.spec_events.p;
        a.event_step = c.spec_event_step.p;
        a.event_cap = cap;
        a.status = c.spec_status.p;
        launch_mvs_big(a, s);
    }
    c.ah_live = false;
    c.dropin_launches += 1;
    // the next Big-body step, from this one's state, once the buffers it
    // writes are read
    check(cudaEventRecord(c.spec_merged, s), "event");
    check(cudaStreamWaitEvent(sa, c.spec_merged, 0), "wait");
    check(cudaMemsetAsync(c.ah_status.p, 0, sizeof(DeviceStatus), sa), "memset");
    MvsBigArgs b = big_args(c.cur, 1 - c.cur, 1, 0, cen, 0, h, rcen, c.ah_tab.p, c.ah_detail.p);
    b.in = big_state_at(c.spec_big.p, c.nsplit);
    b.out = big_state_at(c.ah_state.p, c.nsplit);
    b.events = c.ah_events.p;
    b.event_step = c.ah_event_step.p;
    b.event_cap = AHEAD_RECORDS;
    b.status = c.ah_status.p;
    launch_mvs_big(b, sa);
    check(cudaEventRecord(c.ah_done, sa), "event");
    c.dropin_launches += 1;
    c.ah_live = true;
    c.ah_h = h;
    c.ah_rcen = rcen;
    if (c.np > 0) {
        MvsParticleArgs pa = particle_args(c.cur, 1 - c.cur, 1, 0, cen, 0, h, rcen, c.spec_tab.p, c.spec_detail.p);
        pa.xout = c.spec_part.p;
        pa.events = c.spec_events.p;
        pa.event_step = c.spec_event_step.p;
        pa.event_cap = cap;
        pa.status = c.spec_status.p;
        particles_and_events(pa, c.spec_detail.p, s);
        c.dropin_launches += 1 + (nb > 0 ? 1 : 0);
    }
    check(cudaMemcpyAsync(c.spec_status_host, c.spec_status.p, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, s),
          "status");
    const int head = std::min(Context::EVENT_HEAD, cap);
    if (head > 0)
        check(cudaMemcpyAsync(c.spec_head, c.spec_events.p, sizeof(MercuryEvent) * head, cudaMemcpyDeviceToHost, s),
              "events");
    check(cudaGetLastError(), "launch");
    check(cudaEventRecord(c.spec_done, s), "event");
    c.spec_live = true;
    c.spec_h = h;
    c.spec_rcen = rcen;
    c.spec_from = c.cur;
}

// The speculative step as this step, when it was made for it and ended
// without a fault or an overflow. The Big-body step run ahead of it stays.
bool spec_take(double h, double rcen) {
    Context& c = ctx();
    if (!c.spec_live) return false;
    const bool match = c.spec_h == h && c.spec_rcen == rcen && c.spec_from == c.cur && !c.reset;
    spec_wait();
    const DeviceStatus st = *c.spec_status_host;
    if (!match || st.fault || st.overflow) {
        spec_drop();
        return false;
    }
    const int out = 1 - c.cur;
    std::swap(c.bigstate[out], c.spec_big);
    std::swap(c.pstate[out], c.spec_part);
    std::swap(c.events, c.spec_events);
    std::swap(c.event_step, c.spec_event_step);
    std::swap(c.ev_head, c.spec_head);
    *c.status_host = st;
    check(cudaMemcpyAsync(c.status.p, c.spec_status.p, sizeof(DeviceStatus), cudaMemcpyDeviceToDevice, c.stream),
          "status");
    c.head_ready = true;
    c.head_count = std::min(Context::EVENT_HEAD, (int)c.events.n);
    return true;
}

// One MVS step (mdt_mvs) of the whole system: Big-body CTA then the particle
// kernel, double-buffered so the pre-step state stays available. Pair events
// are left in the event buffer with tmin in their time field. Once an events
// call has named the central body's radius, the step screens for central
// impacts in the same kernels (mce_cent with that radius, as the fused run
// does) and the next events call with the same radius and h only reads the
// records back.
void mvs_step_once(double h) {
    Context& c = ctx();
    if (c.steps_since_order >= 32) {
        const int src = c.cur;
        spec_drop();
        c.cur = reorder_slots(src, h, c.stream);
        // the Big bodies share the buffer index: carry their state across
        if (c.cur != src)
            check(cudaMemcpyAsync(c.bigstate[c.cur].p, c.bigstate[src].p, sizeof(double) * 9 * c.nsplit,
                                  cudaMemcpyDeviceToDevice, c.stream),
                  "copy");
    }
    c.steps_since_order += 1;
    const double rc = c.dropin_rcen;
    const int cen = rc > 0.0 ? 1 : 0;
    const bool ahead = spec_take(h, rc);
    for (int attempt = 0; !ahead; ++attempt) {
        c.head_ready = false;
        ensure_tables(2, 1);
        check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
        const int in = c.cur, out = 1 - c.cur;
        const int reset = c.reset ? 1 : 0;
        launch_mvs_big(big_args(in, out, 1, reset, cen, 0, h, rc, c.tab.p, c.detail.p), c.stream);
        c.dropin_launches += 1 + (c.np > 0 ? 1 + (c.nbig > 1 ? 1 : 0) : 0);
        if (c.np > 0)
            particles_and_events(particle_args(in, out, 1, reset, cen, 0, h, rc, c.tab.p, c.detail.p), c.detail.p,
                                 c.stream);
        check(cudaGetLastError(), "launch");
        read_status();
        if (c.status_host->fault) throw std::runtime_error("MVS force failed");
        if (!c.status_host->overflow) break;
        if (attempt > 8) throw std::runtime_error("event buffer growth failed");
        grow_after_overflow();   // the input buffers are untouched: redo the step
    }
    c.nforces += 1 + (c.reset ? 1 : 0);
    c.pair_events = c.status_host->events;
    c.step_central = cen != 0;
    c.step_rcen = rc;
    c.step_h = h;
    c.cur = 1 - c.cur;
    c.reset = false;
    c.stepped = true;
    if (c.steps_since_order < 32) spec_launch(h, rc);
}

ForceCfg force_cfg() {
    Context& c = ctx();
    ForceCfg f{};
    f.nbig = c.nbig;
    f.nsplit = c.nsplit;
    f.ngflag = c.ngflag;
    f.pn = c.pn;
    f.obl = (c.jcen[0] != 0.0 || c.jcen[1] != 0.0 || c.jcen[2] != 0.0);
    for (int k = 0; k < 3; ++k) f.jcen[k] = c.jcen[k];
    f.m0 = c.m_host[0];
    return f;
}

// One RA15 sequence with mdt_ra15's step control (mercury6_2.for:4401-4425):
// the sequence runs on the device, the controller here reads max |b7| and
// either retries a first sequence with 0.8 of the suggested length or
// commits it. h is the trial length in, the next one out.
void ra15_step_once(double time, double* h, double* hdid, double tol, int64_t* rejected) {
    Context& c = ctx();
    const int nb = c.nbig - 1;
    c.ftab.reserve((size_t)(1 + 7 * 6) * force_row(nb));
    for (;;) {
        const double t = *h;
        if (time + t == time) throw std::runtime_error("RADAU step cannot advance time");
        const int reset = c.reset ? 1 : 0;
        const int niter = reset ? 6 : 2;
        const int in = c.cur, out = 1 - c.cur;
        check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
        check(cudaMemsetAsync(c.ra_max.p, 0, sizeof(unsigned long long), c.stream), "memset");
        Ra15Args a{};
        a.f = force_cfg();
        a.np = c.np;
        a.npcap = c.npcap;
        a.niter = niter;
        a.reset = reset;
        a.t = t;
        a.bx = c.bigstate[in].p;
        a.bx_a1 = c.bigstate[in].p + 6 * c.nsplit;
        a.mbig = c.mbig.p;
        a.ngfbig = c.ngfbig.p;
        a.bb = c.ra_bb.p;
        a.bg = c.ra_bg.p;
        a.bpx = c.ra_bpx.p;
        a.px = c.pstate[in].p;
        a.pconst = c.pconst[c.kc].p;
        a.pb = c.ra_pb.p;
        a.table = c.ftab.p;
        a.maxb7 = c.ra_max.p;
        a.status = c.status.p;
        launch_ra15_sequence(a, c.stream);
        c.dropin_launches += 1 + (c.np > 0 ? 1 : 0);
        check(cudaGetLastError(), "launch");
        unsigned long long bits = 0;
        check(cudaMemcpyAsync(&bits, c.ra_max.p, sizeof(bits), cudaMemcpyDeviceToHost, c.stream), "status");
        read_status();
        c.nforces += 1 + 7 * niter;
        double err;
        std::memcpy(&err, &bits, sizeof(err));
        if (c.status_host->fault || !std::isfinite(err)) err = INFINITY;
        reduce_step_maxima(&err, 1);
        if (!std::isfinite(err)) throw std::runtime_error("Nonfinite RADAU force or predictor");
        err = err / (72.0 * std::pow(std::fabs(t), 7.0));
        double next = err == 0.0 ? t * 1.4 : std::copysign(std::pow(tol / err, 1.0 / 9.0), t);
        if (reset && std::fabs(next / t) < 1.0) {
            *h = next * 0.8;
            ++*rejected;
            continue;
        }
        if (std::fabs(next / t) > 1.4) next = t * 1.4;
        Ra15CommitArgs k{};
        k.nsplit = c.nsplit;
        k.np = c.np;
        k.npcap = c.npcap;
        k.reset = reset;
        k.tdid = t;
        k.q = next / t;
        k.bx = c.bigstate[in].p;
        k.bx_out = c.bigstate[out].p;
        k.bb = c.ra_bb.p;
        k.be = c.ra_be.p;
        k.px = c.pstate[in].p;
        k.px_out = c.pstate[out].p;
        k.pb = c.ra_pb.p;
        k.pe = c.ra_pe.p;
        launch_ra15_commit(k, c.stream);
        c.dropin_launches += 1;
        check(cudaGetLastError(), "launch");
        check(cudaStreamSynchronize(c.stream), "step");
        *hdid = t;
        *h = next;
        c.reset = false;
        c.cur = out;
        c.stepped = true;
        c.pair_events = 0;
        return;
    }
}

// Every level of one mdt_bs1 (algorithm 2) or mdt_bs2 (algorithm 3) attempt
// at trial step h from the current state buffer: per-level error maxima in
// bs_errs, per-level force faults in bs_lvst, candidates for the commit.
// The arguments of one BS/BS2 attempt from the current buffer with trial
// step h (the workspace reserved).
BsArgs bs_attempt_args(double h) {
    Context& c = ctx();
    const int V = c.algorithm == 2 ? 1 : 2;
    const int L = bs_levels(V), nb = c.nbig - 1, N = c.nsplit;
    c.ftab.reserve((size_t)bs_rows(V) * force_row(nb));
    c.bs_scr.reserve(bs_massive_scratch(V, N, nb));
    c.bs_bcand.reserve((size_t)bs_candidates(V) * 6 * N);
    c.bs_pcand.reserve((size_t)bs_candidates(V) * 6 * c.npcap);
    c.bs_errs.reserve(13);
    c.bs_lvst.reserve(13);
    const int in = c.cur;
    BsArgs a{};
    a.f = force_cfg();
    a.variant = V;
    a.np = c.np;
    a.npcap = c.npcap;
    a.h0 = h;
    a.bx = c.bigstate[in].p;
    a.mbig = c.mbig.p;
    a.ngfbig = c.ngfbig.p;
    a.draw = c.bs_scr.p;
    a.tscr = c.bs_scr.p + (size_t)L * 6 * N;
    a.px = c.pstate[in].p;
    a.pconst = c.pconst[c.kc].p;
    a.table = c.ftab.p;
    a.bcand = c.bs_bcand.p;
    a.pcand = c.bs_pcand.p;
    a.errs = c.bs_errs.p;
    a.lvst = c.bs_lvst.p;
    a.hkce = c.encounter ? 1 : 0;
    a.rcrit = c.rcritbig.p;
    a.adj_off = c.adj_off.p;
    a.adj = c.adj.p;
    a.perm = c.permp();
    a.active_np = c.bs_active_np >= 0 ? std::min(c.bs_active_np, c.np) : c.np;
    if (V == 2 && !a.hkce && c.np > 0) {
        // mdt_bs2 with mfo_all: the particles' levels 9..12 only when needed
        c.bs_ptab.reserve((size_t)8 * 6 * c.npcap);
        a.ptab = c.bs_ptab.p;
    }
    return a;
}

BsArgs launch_bs_attempt(double h) {
    Context& c = ctx();
    const BsArgs a = bs_attempt_args(h);
    check(cudaMemsetAsync(c.bs_errs.p, 0, sizeof(unsigned long long) * 13, c.stream), "memset");
    check(cudaMemsetAsync(c.bs_lvst.p, 0, sizeof(DeviceStatus) * 13, c.stream), "memset");
    launch_bs_sequence(a, c.stream);
    c.dropin_launches += 2 + (c.np > 0 ? 1 : 0);  // level CTAs, extrapolation, particles
    check(cudaGetLastError(), "launch");
    return a;
}

// The Fortran's choice (mercury6_2.for:3380-3404, 3568-3596) from the level
// maxima errs and faults lv of an attempt: the first level n > 3 whose global
// error is <= tol^2, or 0 when the step is to be halved and redone. Adds the
// force calls of the levels it looked at to *forces.
int bs_accept_level(const unsigned long long* errs, const DeviceStatus* lv, int V, double tol, int64_t* forces,
                    int first = 1, int last = 0) {
    const int L = last > 0 ? last : bs_levels(V);
    const double tol2 = tol * tol;
    const char* nonfinite = V == 1 ? "Nonfinite BS extrapolation; inspect input or close encounters"
                                   : "Nonfinite BS2 force or extrapolation";
    // per level: the error maximum, then whether a force failed
    const int fails = FAULT_NGF | FAULT_COINCIDENT;
    double red[26];
    for (int n = 0; n < 13; ++n) {
        std::memcpy(&red[n], &errs[n], sizeof(double));
        red[13 + n] = (lv[n].fault & fails) ? 1.0 : 0.0;
    }
    reduce_step_maxima(red, 26);
    if (red[13] > 0.0) throw std::runtime_error("BS force failed");
    for (int n = first; n <= L; ++n) {
        *forces += bs_level_forces(V, n);
        if (red[13 + n] > 0.0) throw std::runtime_error("BS force failed");
        if (n <= 3) continue;
        const double e = red[n];
        if (!std::isfinite(e)) throw std::runtime_error(nonfinite);
        if (e <= tol2) return n;
    }
    return 0;
}

// Copies level `accepted` of attempt a into the other state buffer (and
// pushes the encounter members' tangents through it when they are kept).
void launch_bs_commit_of(const BsArgs& a, int accepted) {
    Context& c = ctx();
    const int in = c.cur, out = 1 - c.cur;
    BsCommitArgs k{};
    k.nsplit = c.nsplit;
    k.np = c.np;
    k.npcap = c.npcap;
    k.cand = accepted - 4;
    k.bcand = c.bs_bcand.p;
    k.pcand = c.bs_pcand.p;
    k.bx = c.bigstate[in].p;
    k.bx_out = c.bigstate[out].p;
    k.px_out = c.pstate[out].p;
    k.px = c.pstate[in].p;
    k.perm = c.permp();
    k.active_np = a.active_np;
    launch_bs_commit(k, c.stream);
    c.dropin_launches += 1;
    if (c.tangent && c.encounter && a.variant == 2 && c.np > 0) {
        launch_bs2_tangent(a, accepted, c.tg.p, c.stream);
        c.dropin_launches += 1;
    }
    check(cudaGetLastError(), "launch");
}

// The next trial step after an accepted level (mercury6_2.for:3389-3390, 3581-3582).
void bs_next_trial(int V, int accepted, double* h) {
    if (V == 1) {
        if (accepted == 8) *h = *h * 0.55;
    } else {
        if (accepted >= 8) *h = *h * 0.55;
    }
    if (accepted < 7) *h = *h * 1.3;
}

// One mdt_bs1 (algorithm 2) or mdt_bs2 (algorithm 3) step with the Fortran's
// control: attempts at halved steps until a level passes, then the commit.
void bs_step_once(double time, double* h, double* hdid, double tol, int64_t* rejected) {
    Context& c = ctx();
    int64_t forces = 1;  // the start-of-step force
    for (;;) {
        if (time + *h == time) throw std::runtime_error("BS cannot advance time at the requested tolerance");
        const BsArgs a = launch_bs_attempt(*h);
        unsigned long long errs[13];
        DeviceStatus lv[13];
        auto read_levels = [&] {
            check(cudaMemcpyAsync(errs, c.bs_errs.p, sizeof(errs), cudaMemcpyDeviceToHost, c.stream), "status");
            check(cudaMemcpyAsync(lv, c.bs_lvst.p, sizeof(lv), cudaMemcpyDeviceToHost, c.stream), "status");
            check(cudaStreamSynchronize(c.stream), "step");
        };
        read_levels();
        int accepted = 0;
        if (a.ptab) {
            // levels 1..8 first; 9..12 of the particles only when none passed
            accepted = bs_accept_level(errs, lv, a.variant, tol, &forces, 1, 8);
            if (!accepted) {
                launch_bs_particles_late(a, c.stream);
                c.dropin_launches += 1;
                check(cudaGetLastError(), "launch");
                read_levels();
                accepted = bs_accept_level(errs, lv, a.variant, tol, &forces, 9, bs_levels(a.variant));
            }
        } else {
            accepted = bs_accept_level(errs, lv, a.variant, tol, &forces);
        }
        if (!accepted) {
            ++*rejected;
            *h = *h * 0.5;
            continue;
        }
        launch_bs_commit_of(a, accepted);
        check(cudaStreamSynchronize(c.stream), "step");
        *hdid = *h;
        bs_next_trial(a.variant, accepted, h);
        c.nforces += forces;
        c.cur = 1 - c.cur;
        c.stepped = true;
        c.pair_events = 0;
        return;
    }
}

// mce_stat between the buffers before and after the last step of an adaptive
// integrator (mercury6_2.for:1765-1918): Big/massive pairs by one CTA, the
// particles' box overlaps as candidates, classified like the MVS path's.
// Records are appended at the status counter and tagged `step`; the caller
// clears the candidate counter first.
void launch_pair_screen(double h, int step) {
    Context& c = ctx();
    const int nb = c.nbig - 1;
    c.boxes.reserve((size_t)4 * std::max(1, nb));
    c.detail.reserve((size_t)std::max(1, nb) * TAB_DETAIL);
    const int cur = c.cur, prev = 1 - cur;
    ScreenArgs a{};
    a.nbig = c.nbig;
    a.nsplit = c.nsplit;
    a.np = c.np;
    a.npcap = c.npcap;
    a.h = h;
    a.b0 = c.bigstate[prev].p;
    a.b1 = c.bigstate[cur].p;
    a.mbig = c.mbig.p;
    a.rcebig = c.rcebig.p;
    a.rphysbig = c.rphysbig.p;
    a.p0 = c.pstate[prev].p;
    a.p1 = c.pstate[cur].p;
    a.pconst = c.pconst[c.kc].p;
    a.perm = c.permp();
    a.boxes = c.boxes.p;
    a.detail = c.detail.p;
    a.events = c.events.p;
    a.event_step = c.event_step.p;
    a.event_cap = (int)c.events.n;
    a.cands = c.cands.p;
    a.cand_cap = (int)c.cands.n;
    a.status = c.status.p;
    a.step = step;
    launch_screen(a, c.stream);
    c.dropin_launches += 1 + (c.np > 0 && nb > 0 ? 2 : 0);
    if (nb > 0 && c.np > 0) {
        ClassifyArgs ca{};
        ca.nb = nb;
        ca.nbig = c.nbig;
        ca.h = h;
        ca.detail = c.detail.p;
        ca.cands = c.cands.p;
        ca.cand_cap = (int)c.cands.n;
        ca.events = c.events.p;
        ca.event_step = c.event_step.p;
        ca.event_cap = (int)c.events.n;
        ca.status = c.status.p;
        ca.step_base = step;
        launch_classify(ca, c.stream);
    }
    check(cudaGetLastError(), "screen");
}

// The pair screen of the last step, its records from slot 0 (grown and redone
// after an overflow).
void screen_pairs(double h) {
    Context& c = ctx();
    for (int attempt = 0;; ++attempt) {
        check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
        launch_pair_screen(h, 0);
        read_status();
        if (c.status_host->overflow) {
            if (attempt > 8) throw std::runtime_error("event buffer growth failed");
            grow_after_overflow();
            continue;
        }
        c.pair_events = c.status_host->events;
        return;
    }
}

// mco_mvs2h of the current MVS state into host rows (the reference exports
// with its corrector on scratch copies, mercury_cuda.cu:508-513); the state
// itself is not changed.
// The output corrector of MVS (mco_mvs2h) on scratch copies: corr_big and
// (unless big_only) corr_part receive the corrected heliocentric states.
void run_corrector(double h, bool big_only = false) {
    Context& c = ctx();
    const int nbig = c.nbig, ns = c.nsplit;
    ensure_tables(4, 1);
    c.corr_big.reserve((size_t)9 * ns);
    c.corr_part.reserve((size_t)6 * c.npcap);
    check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
    MvsBigArgs b = big_args(c.cur, c.cur, 0, 0, 0, 0, h, 0.0, c.tab.p, c.detail.p);
    b.out.x = c.corr_big.p;
    b.out.v = c.corr_big.p + 3 * ns;
    b.out.a = c.corr_big.p + 6 * ns;
    CorrectorArgs k{};
    k.np = big_only ? 0 : c.np;
    k.npcap = c.npcap;
    k.nb = nbig - 1;
    k.ngf_on = (c.ngflag == 1 || c.ngflag == 3);
    k.obl = (c.jcen[0] != 0.0 || c.jcen[1] != 0.0 || c.jcen[2] != 0.0);
    k.forward = 1;
    k.mu = c.m_host[0];
    const double rt10 = std::sqrt(10.0);
    k.ha[0] = h * rt10 * 3.0 / 10.0;
    k.hb[0] = -(h * rt10 / 72.0);
    k.ha[1] = h * rt10 / 5.0;
    k.hb[1] = h * rt10 / 24.0;
    for (int q = 0; q < 3; ++q) k.jcen[q] = c.jcen[q];
    k.xin = c.pstate[c.cur].p;
    k.xout = c.corr_part.p;
    k.ngf = c.pngf();
    k.tab = c.tab.p;
    k.status = c.status.p;
    launch_mvs_corrector(b, k, c.stream);
    check(cudaGetLastError(), "corrector");
    read_status();
    if (c.status_host->fault) throw std::runtime_error("Output corrector failed");
}

void export_corrected(double h, double* xx, double* vv) {
    Context& c = ctx();
    const int ns = c.nsplit;
    run_corrector(h);
    c.transfer.reserve((size_t)6 * c.n);
    for (int part = 0; part < 2; ++part)
        gather_kernel<<<blocks(c.n), 256, 0, c.stream>>>(c.transfer.p + (size_t)3 * part * c.n, c.n, 3, ns,
                                                          c.corr_big.p + 3 * part * ns, ns,
                                                          c.corr_part.p + (size_t)3 * part * c.npcap, c.npcap,
                                                          c.inv.p);
    check(cudaGetLastError(), "export");
    const size_t bytes = sizeof(double) * 3 * (size_t)c.n;
    copy_out({{c.transfer.p, xx, bytes}, {c.transfer.p + (size_t)3 * c.n, vv, bytes}}, c.stream);
}

// mxx_ejec's test (mercury6_2.for:7078-7080): bodies from index `first` on
// whose r^2 = x*x + y*y + z*z (the Fortran's order) exceeds rmax2, as 1-based
// ids; one atomic per warp (ballot, then each hit's rank among the warp's).
// ids[0] counts, ids[1 ..] receive up to cap ids in no particular order.
__global__ void ejection_kernel(const double* bx, int N, const double* px, int S, int np, const int* perm, int first,
                                double rmax2, int* ids, int cap) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    bool hit = false;
    int id = 0;
    if (q < N + np) {
        double x, y, z;
        int body;
        if (q < N) {
            body = q;
            x = bx[q]; y = bx[N + q]; z = bx[2 * N + q];
        } else {
            const int s = q - N;
            body = N + perm[s];
            x = px[s]; y = px[S + s]; z = px[2 * (size_t)S + s];
        }
        const double r2 = x * x + y * y + z * z;
        hit = body >= first && r2 > rmax2;
        id = body + 1;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    if (!mask) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(ids, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (hit) {
        const int k = base + __popc(mask & ((1u << lane) - 1u));
        if (k < cap) ids[1 + k] = id;
    }
}

// mco_dh2h's velocity shift (mercury6_2.for:2007-2051) of state buffer
// `which`, added on the host to downloaded rows (the same additions).
void add_dh_shift(int which, double* vv) {
    Context& c = ctx();
    c.hy_off.reserve(6);
    launch_dh_shift(c.bigstate[which].p, c.mbig.p, c.nsplit, c.m_host[0], c.hy_off.p, c.stream);
    double off[3];
    check(cudaMemcpyAsync(off, c.hy_off.p, sizeof(off), cudaMemcpyDeviceToHost, c.stream), "download");
    check(cudaStreamSynchronize(c.stream), "download");
    for (int j = 1; j < c.n; ++j)
        for (int q = 0; q < 3; ++q) vv[3 * j + q] = vv[3 * j + q] + off[q];
}

__global__ void scatter_members_kernel(const int* ids, int count, const double* packed, double* bx, int N, double* px,
                                       int S, const int* inv) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const int g = ids[q];
    for (int c = 0; c < 6; ++c) {
        const double val = packed[6 * (size_t)q + c];
        if (g < N) bx[c * N + g] = val;
        else px[(size_t)c * S + inv[g - N]] = val;
    }
}

// Members' rows {x, v} into the state buffers (massive set or particle slot).
void scatter_members(const int* ids, int count, const double* packed, double* bx, double* px) {
    Context& c = ctx();
    scatter_members_kernel<<<blocks(count), 256, 0, c.stream>>>(ids, count, packed, bx, c.nsplit, px, c.npcap, c.inv.p);
}

HyArgs hybrid_args(double h, int recompute) {
    Context& c = ctx();
    HyArgs a{};
    a.nbig = c.nbig;
    a.nsplit = c.nsplit;
    a.np = c.np;
    a.npcap = c.npcap;
    a.ngflag = c.ngflag;
    a.obl = (c.jcen[0] != 0.0 || c.jcen[1] != 0.0 || c.jcen[2] != 0.0);
    a.recompute = recompute;
    for (int q = 0; q < 3; ++q) a.jcen[q] = c.jcen[q];
    a.m0 = c.m_host[0];
    a.h = h;
    a.mbig = c.mbig.p;
    a.rcritbig = c.rcritbig.p;
    a.ngfbig = c.ngfbig.p;
    a.bx_in = c.bigstate[c.cur].p;
    a.bx_out = c.bigstate[1 - c.cur].p;
    a.bscr = c.hy_scr.p;
    a.px_in = c.pstate[c.cur].p;
    a.px_out = c.pstate[1 - c.cur].p;
    a.pconst = c.pconst[c.kc].p;
    a.perm = c.permp();
    a.tab = c.hy_tab.p;
    a.pairs = c.hy_pairs.p;
    a.pair_cap = (int)c.hy_pairs.n;
    a.status = c.status.p;
    return a;
}

// Warp-coherent ordering of the Small bodies. drift_dan leaves its elliptic
// fast path (drift_kepmd) for the Newton solver when dm^2 > 0.16 or
// e^2 dm^2 >= 0.0016 with dm = n h, or when the orbit is unbound or e^2 > 0.36,
// i.e. when max(e n / 0.04, n / 0.4) * |h| >= 1 for bound orbits with e <= 0.6.
// Sorting the particle slots by that key (largest first, 256 logarithmic
// buckets) puts the bodies that take the long path into the same warps for
// any step size. Slot order changes no result: each particle's arithmetic is
// independent of its slot, and event ids are mapped back through perm.
__host__ __device__ inline int path_bucket(double x0, double x1, double x2, double v0, double v1, double v2,
                                           double mu) {
    const double r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
    const double vv = v0 * v0 + v1 * v1 + v2 * v2;
    const double u = x0 * v0 + x1 * v1 + x2 * v2;
    const double alpha = 2.0 * mu / r - vv;
    if (!(alpha > 0.0) || !isfinite(alpha)) return 0;
    const double a = mu / alpha;
    const double en = sqrt(mu / (a * a * a));
    const double ec = 1.0 - r / a, es = u / (en * a * a);
    const double e = sqrt(ec * ec + es * es);
    const double key = fmax(e * en / 0.04, en / 0.4);
    if (!(e <= 0.6) || !(key > 0.0) || !isfinite(key)) return 0;
    const double l = log2(key) * 8.0 + 128.0;  // keys 2^-16 .. 2^16
    const int b = 255 - (int)fmin(255.0, fmax(0.0, l));
    return b < 1 ? 1 : b;
}

__global__ void path_key_kernel(const double* x, const double* v, int nbig, int np, double mu, unsigned char* key,
                                int* idx) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const double* xp = x + 3 * (size_t)(nbig + p);
    const double* vp = v + 3 * (size_t)(nbig + p);
    key[p] = (unsigned char)path_bucket(xp[0], xp[1], xp[2], vp[0], vp[1], vp[2], mu);
    idx[p] = p;
}

// perm (slot -> particle) from the sorted particle indices; padding slots map
// to themselves; inv (particle -> slot).
__global__ void slot_maps_kernel(const int* sorted, int np, int npcap, int* perm, int* inv) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= npcap) return;
    const int p = s < np ? sorted[s] : s;
    perm[s] = p;
    inv[p] = s;
}

// The upload's slot order on the device: particles in ascending path_bucket
// key (a stable radix sort of the 8-bit keys, so ties keep particle order),
// from the staged host rows x, v of the n bodies (the first nbig are not
// particles).
void order_particles(int n, int nbig, double mu, const double* x, const double* v) {
    Context& c = ctx();
    const int np = n - nbig;
    c.steps_since_order = 0;
    if (np <= 0) {
        slot_maps_kernel<<<blocks(c.npcap), 256, 0, c.stream>>>(nullptr, 0, c.npcap, c.perm[c.kc].p, c.inv.p);
        check(cudaGetLastError(), "order");
        return;
    }
    // scratch: keys in/out (bytes), indices in/out (ints), then the sort's own
    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t temp = 0;
    check(cub::DeviceRadixSort::SortPairs(nullptr, temp, (const unsigned char*)nullptr, (unsigned char*)nullptr,
                                          (const int*)nullptr, (int*)nullptr, np, 0, 8, c.stream),
          "order");
    const size_t kb = align(np), ib = align(sizeof(int) * (size_t)np);
    c.order_scratch.reserve(2 * kb + 2 * ib + align(temp));
    char* base = c.order_scratch.p;
    unsigned char* kin = reinterpret_cast<unsigned char*>(base);
    unsigned char* kout = kin + kb;
    int* iin = reinterpret_cast<int*>(base + 2 * kb);
    int* iout = reinterpret_cast<int*>(base + 2 * kb + ib);
    void* tmp = base + 2 * kb + 2 * ib;
    path_key_kernel<<<blocks(np), 256, 0, c.stream>>>(x, v, nbig, np, mu, kin, iin);
    check(cub::DeviceRadixSort::SortPairs(tmp, temp, kin, kout, iin, iout, np, 0, 8, c.stream), "order");
    slot_maps_kernel<<<blocks(c.npcap), 256, 0, c.stream>>>(iout, np, c.npcap, c.perm[c.kc].p, c.inv.p);
    check(cudaGetLastError(), "order");
}

// Slot maps of one chunk of particles [base, base + cnt) ordered within its
// own slots: perm[base + r] = base + sorted[r] and its inverse; with pad, the
// padding slot after the chunk maps to itself.
__global__ void chunk_slot_maps_kernel(const int* sorted, int cnt, int base, int pad, int* perm, int* inv) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cnt + pad) return;
    const int p = base + (r < cnt ? sorted[r] : r);
    perm[base + r] = p;
    inv[p] = base + r;
}

// The upload's slot order for the particles [plo, phi) alone (the same keys
// and stable sort as order_particles, within the chunk's slots), from the
// staged rows x, v of the bodies; pad: the chunk ends at the padding slot;
// cap: the largest chunk of the run.
void order_chunk(int plo, int phi, int pad, int cap, double mu, const double* x, const double* v, cudaStream_t s) {
    Context& c = ctx();
    const int cnt = phi - plo;
    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    // scratch laid out for the largest chunk (cap), so that it is not
    // reallocated between chunks (an empty chunk only sizes it)
    size_t temp = 0;
    check(cub::DeviceRadixSort::SortPairs(nullptr, temp, (const unsigned char*)nullptr, (unsigned char*)nullptr,
                                          (const int*)nullptr, (int*)nullptr, cap, 0, 8, s),
          "order");
    const size_t kb = align(cap), ib = align(sizeof(int) * (size_t)cap);
    c.order_scratch.reserve(2 * kb + 2 * ib + align(temp));
    if (cnt <= 0) return;
    char* base = c.order_scratch.p;
    unsigned char* kin = reinterpret_cast<unsigned char*>(base);
    unsigned char* kout = kin + kb;
    int* iin = reinterpret_cast<int*>(base + 2 * kb);
    int* iout = reinterpret_cast<int*>(base + 2 * kb + ib);
    void* tmp = base + 2 * kb + 2 * ib;
    path_key_kernel<<<blocks(cnt), 256, 0, s>>>(x, v, c.nsplit + plo, cnt, mu, kin, iin);
    check(cub::DeviceRadixSort::SortPairs(tmp, temp, kin, kout, iin, iout, cnt, 0, 8, s), "order");
    chunk_slot_maps_kernel<<<blocks(cnt + pad), 256, 0, s>>>(iout, cnt, plo, pad, c.perm[c.kc].p, c.inv.p);
    check(cudaGetLastError(), "order");
}

// The records of a fused run in (step, min(i,j), max(i,j)) order on the
// device: a 64-bit key per record (the step above the two 1-based ids, each
// in `idbits` bits; one record per pair per step makes the keys distinct),
// a radix sort of (key, record index), then a gather that also turns each
// record's time into an absolute one as the host would: tend[s] is the
// driver's clock after step s (time + h added step by step), central-body
// records hold their entry time from the step's start, pair records their
// minimum time from its end.
__global__ void event_key_kernel(const MercuryEvent* ev, const int* step, int n, int idbits,
                                 unsigned long long* key, int* idx) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const unsigned long long i = (unsigned)ev[k].i, j = (unsigned)ev[k].j;
    const unsigned long long lo = i < j ? i : j, hi = i < j ? j : i;
    key[k] = ((unsigned long long)(unsigned)step[k] << (2 * idbits)) | (lo << idbits) | hi;
    idx[k] = k;
}

__global__ void event_gather_kernel(const MercuryEvent* ev, const int* step, const int* order, int n,
                                   const double* tend, double h, MercuryEvent* out, int* out_step) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int k = order[r];
    MercuryEvent e = ev[k];
    const int s = step[k];
    const double te = tend[s];
    if (e.kind == EV_CENTRAL) e.time = te - h + e.time;
    else e.time = e.time + te;
    store_event(out + r, e);
    out_step[r] = s;
}

// Bits for one 1-based id of n bodies, or 0 when (step, id, id) keys of a
// run of nsteps steps do not fit in 64 bits.
int event_id_bits(int n, int nsteps) {
    int idbits = 1, stepbits = 1;
    while ((1ll << idbits) <= (long long)n) ++idbits;
    while ((1ll << stepbits) < (long long)nsteps) ++stepbits;
    return 2 * idbits + stepbits <= 64 ? idbits : 0;
}

// Orders the nev records of the last fused run into c.ev_sorted /
// c.ev_sorted_step (see event_key_kernel). False when the keys do not fit.
bool order_events_device(int nev, int nsteps, const std::vector<double>& tend, double h) {
    Context& c = ctx();
    const int idbits = event_id_bits(c.n, nsteps);
    if (!idbits) return false;
    int stepbits = 1;
    while ((1ll << stepbits) < (long long)nsteps) ++stepbits;
    const int end_bit = 2 * idbits + stepbits;
    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    // scratch for a quarter more records than this run's, so that the next
    // run of a similar system does not reallocate
    const int room = nev + nev / 4 + 1024;
    size_t temp = 0;
    check(cub::DeviceRadixSort::SortPairs(nullptr, temp, (const unsigned long long*)nullptr,
                                          (unsigned long long*)nullptr, (const int*)nullptr, (int*)nullptr, room, 0,
                                          64, c.stream),
          "events");
    const size_t kb = align(sizeof(unsigned long long) * (size_t)room), ib = align(sizeof(int) * (size_t)room);
    const size_t tb = align(sizeof(double) * (size_t)nsteps);
    c.order_scratch.reserve(2 * kb + 2 * ib + tb + align(temp));
    char* base = c.order_scratch.p;
    auto* kin = reinterpret_cast<unsigned long long*>(base);
    auto* kout = reinterpret_cast<unsigned long long*>(base + kb);
    int* iin = reinterpret_cast<int*>(base + 2 * kb);
    int* iout = reinterpret_cast<int*>(base + 2 * kb + ib);
    double* dtend = reinterpret_cast<double*>(base + 2 * kb + 2 * ib);
    void* tmp = base + 2 * kb + 2 * ib + tb;
    if ((int)c.ev_sorted.n < nev) {
        c.ev_sorted.reserve(room);
        c.ev_sorted_step.reserve(room);
    }
    check(cudaMemcpyAsync(dtend, tend.data(), sizeof(double) * (size_t)nsteps, cudaMemcpyHostToDevice, c.stream),
          "events");
    event_key_kernel<<<blocks(nev), 256, 0, c.stream>>>(c.events.p, c.event_step.p, nev, idbits, kin, iin);
    check(cub::DeviceRadixSort::SortPairs(tmp, temp, kin, kout, iin, iout, nev, 0, end_bit, c.stream), "events");
    event_gather_kernel<<<blocks(nev), 256, 0, c.stream>>>(c.events.p, c.event_step.p, iout, nev, dtend, h,
                                                           c.ev_sorted.p, c.ev_sorted_step.p);
    check(cudaGetLastError(), "events");
    // the host array of tend is read by the copy above: wait for it
    check(cudaStreamSynchronize(c.stream), "events");
    return true;
}

// Device re-ordering of the slots as the state evolves (scattered or eccentric
// particles move to the universal-variable solver): a stable partition, for
// the step size h of the coming launch, by the drift path of drift_dan
// (mercury6_2.for:7637-7685) so that a warp's 32 particles take one path:
//   0  unbound (drift_kepu_p3solve guess, hyperbolic Stumpff series)
//   1  bound, e > 0.6 (drift_kepu with the sine guess, most iterations)
//   2  bound, e <= 0.6, max(e n/0.04, n/0.4)·|h| >= 1 (drift_kepu)
//   3  the rest (drift_kepmd, no iteration)
// Buckets 0-2 lead so that the particle kernel's dynamic tiles take the slow
// slots first. Warp ballots give in-block ranks and one scan per bucket gives
// block offsets, so the pass is deterministic, atomic-free and writes
// contiguous runs.
constexpr int PATH_BUCKETS = 4;
__device__ __forceinline__ int drift_bucket(const double* x, int S, int s, double mu, double absh) {
    const double x0 = x[s], x1 = x[S + s], x2 = x[2 * S + s];
    const double v0 = x[3 * S + s], v1 = x[4 * S + s], v2 = x[5 * S + s];
    const double r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
    const double vv = v0 * v0 + v1 * v1 + v2 * v2;
    const double u = x0 * v0 + x1 * v1 + x2 * v2;
    const double alpha = 2.0 * mu / r - vv;
    if (!(alpha > 0.0)) return 0;
    const double a = mu / alpha;
    const double en = sqrt(mu / (a * a * a));
    const double ec = 1.0 - r / a, es = u / (en * a * a);
    const double e = sqrt(ec * ec + es * es);
    if (!(e <= 0.6)) return 1;
    return fmax(e * en / 0.04, en / 0.4) * absh >= 1.0 ? 2 : 3;
}

struct PartitionArgs {
    int np, npcap, nblk;
    double mu, absh;
    const double* xin;
    double* xout;
    const double* cin;
    double* cout;
    const int* pin;
    int* pout;
    int* inv;
    int* hist;   // [PATH_BUCKETS][nblk] per-block counts, then exclusive offsets within the bucket
    int* base;   // [PATH_BUCKETS] first slot of each bucket
};

constexpr int PART_THREADS = 256;

// Rank of this thread among the threads of its block with the same flag;
// returns the block's count of set flags in *nset. All threads must call.
__device__ __forceinline__ int block_rank(bool flag, int* nset) {
    __shared__ int warp_set[PART_THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) warp_set[w] = __popc(m);
    __syncthreads();
    int before_set = 0, all_set = 0;
    for (int k = 0; k < PART_THREADS / 32; ++k) {
        if (k < w) before_set += warp_set[k];
        all_set += warp_set[k];
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int set_rank = before_set + __popc(m & lt);
    const int clear_rank = (w * 32 + lane) - set_rank;
    *nset = all_set;
    return flag ? set_rank : clear_rank;
}

__global__ void __launch_bounds__(PART_THREADS) partition_count_kernel(PartitionArgs A) {
    const int s = blockIdx.x * PART_THREADS + threadIdx.x;
    const bool valid = s < A.np;
    const int key = valid ? drift_bucket(A.xin, A.npcap, s, A.mu, A.absh) : -1;
    for (int b = 0; b < PATH_BUCKETS; ++b) {
        int n;
        block_rank(key == b, &n);
        if (threadIdx.x == 0) A.hist[b * A.nblk + blockIdx.x] = n;
    }
}

// Exclusive scans of the per-block counts of every bucket and the buckets'
// first slots (one CTA of 1024 threads: per-thread runs, warp shuffles, one
// warp over the warp totals).
__global__ void __launch_bounds__(1024) partition_scan_kernel(PartitionArgs A) {
    __shared__ int warp_sum[32];
    __shared__ int bucket_total[PATH_BUCKETS];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int per = (A.nblk + 1023) / 1024;
    const int lo = min(A.nblk, t * per), hi = min(A.nblk, lo + per);
    for (int b = 0; b < PATH_BUCKETS; ++b) {
        int* h = A.hist + (size_t)b * A.nblk;
        int run = 0;
        for (int k = lo; k < hi; ++k) run += h[k];
        int incl = run;
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        if (lane == 31) warp_sum[w] = incl;
        __syncthreads();
        if (w == 0) {
            const int mine = warp_sum[lane];
            int wincl = mine;
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, wincl, d);
                if (lane >= d) wincl += y;
            }
            warp_sum[lane] = wincl - mine;
            if (lane == 31) bucket_total[b] = wincl;
        }
        __syncthreads();
        int off = warp_sum[w] + incl - run;
        for (int k = lo; k < hi; ++k) {
            const int x = h[k];
            h[k] = off;
            off += x;
        }
        __syncthreads();
    }
    if (t == 0) {
        int acc = 0;
        for (int b = 0; b < PATH_BUCKETS; ++b) {
            A.base[b] = acc;
            acc += bucket_total[b];
        }
    }
}

__global__ void __launch_bounds__(PART_THREADS) partition_scatter_kernel(PartitionArgs A) {
    const int s = blockIdx.x * PART_THREADS + threadIdx.x;
    const bool valid = s < A.np;
    const int key = valid ? drift_bucket(A.xin, A.npcap, s, A.mu, A.absh) : -1;
    int rank = 0;
    for (int b = 0; b < PATH_BUCKETS; ++b) {
        int n;
        const int r = block_rank(key == b, &n);
        if (key == b) rank = r;
    }
    if (!valid) return;
    const int ns = A.base[key] + A.hist[key * A.nblk + blockIdx.x] + rank;
    const size_t S = A.npcap;
    for (int c = 0; c < 9; ++c) A.xout[c * S + ns] = A.xin[c * S + s];
    for (int c = 0; c < PCONST_ROWS; ++c) A.cout[c * S + ns] = A.cin[c * S + s];
    const int p = A.pin[s];
    A.pout[ns] = p;
    A.inv[p] = ns;
}

// Re-orders the particle slots for a launch with step h: state from
// pstate[src] into pstate[1 - src], constants and perm into the other buffer
// pair. Returns the new state index.
int reorder_slots(int src, double h, cudaStream_t st) {
    Context& c = ctx();
    c.steps_since_order = 0;
    if (c.np < 64) return src;
    const int nblk = (c.np + PART_THREADS - 1) / PART_THREADS;
    c.order_hist.reserve((size_t)PATH_BUCKETS * nblk + PATH_BUCKETS);
    PartitionArgs a{};
    a.np = c.np;
    a.npcap = c.npcap;
    a.nblk = nblk;
    a.mu = c.m_host[0];
    a.absh = std::fabs(h);
    a.xin = c.pstate[src].p;
    a.xout = c.pstate[1 - src].p;
    a.cin = c.pconst[c.kc].p;
    a.cout = c.pconst[1 - c.kc].p;
    a.pin = c.perm[c.kc].p;
    a.pout = c.perm[1 - c.kc].p;
    a.inv = c.inv.p;
    a.hist = c.order_hist.p;
    a.base = c.order_hist.p + (size_t)PATH_BUCKETS * nblk;
    c.dropin_launches += 3;
    partition_count_kernel<<<nblk, PART_THREADS, 0, st>>>(a);
    partition_scan_kernel<<<1, 1024, 0, st>>>(a);
    partition_scatter_kernel<<<nblk, PART_THREADS, 0, st>>>(a);
    check(cudaGetLastError(), "reorder");
    c.kc = 1 - c.kc;
    return 1 - src;
}

// Resizes a host record array to n entries. Beyond its capacity it is
// re-allocated with a quarter of headroom and without copying the old entries
// (the caller overwrites them), so that the next run of a similar system,
// which may bring a few more records, does not grow it again: growing a few
// hundred MB by copy costs more than the run's other host work.
template <class T> void size_records(std::vector<T>& v, size_t n) {
    if (n > v.capacity()) {
        std::vector<T>().swap(v);
        v.reserve(n + n / 4);
    }
    v.resize(n);
}

// The order of records ev by (step, min(i,j), max(i,j)), ties in record
// order: a counting sort of (pair key, record) by step, then each step's
// short run by (key, record). steps == null: all in one step.
void order_events(const std::vector<MercuryEvent>& ev, const std::vector<int>* steps, std::vector<uint32_t>& order) {
    const size_t n = ev.size();
    size_records(order, n);
    if (n == 0) return;
    struct Item {
        uint64_t key;
        uint32_t k;
    };
    std::vector<size_t> first(2, 0);
    if (steps) {
        int smax = 0;
        for (size_t k = 0; k < n; ++k) smax = std::max(smax, (*steps)[k]);
        first.assign((size_t)smax + 2, 0);
        for (size_t k = 0; k < n; ++k) ++first[(size_t)(*steps)[k] + 1];
        for (size_t s = 1; s < first.size(); ++s) first[s] += first[s - 1];
    } else {
        first[1] = n;
    }
    // kept between calls (the library's calls come from one host thread)
    static std::vector<Item> items;
    size_records(items, n);
    {
        // stable scatter by step; with several threads each takes a contiguous
        // chunk of records and its own slice of every step's run (chunk order)
        const size_t nb = first.size() - 1;
        const size_t nthreads =
            (!steps || n < 262144) ? 1 : std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency()));
        const size_t chunk = (n + nthreads - 1) / nthreads;
        std::vector<std::vector<size_t>> fill(nthreads, std::vector<size_t>(nb, 0));
        if (nthreads == 1) {
            for (size_t s = 0; s < nb; ++s) fill[0][s] = first[s];
        } else {
            auto count = [&](size_t t) {
                for (size_t k = t * chunk; k < std::min(n, (t + 1) * chunk); ++k) ++fill[t][(size_t)(*steps)[k]];
            };
            std::vector<std::thread> pool;
            for (size_t w = 0; w < nthreads; ++w) pool.emplace_back(count, w);
            for (auto& th : pool) th.join();
            for (size_t s = 0; s < nb; ++s) {
                size_t at = first[s];
                for (size_t w = 0; w < nthreads; ++w) {
                    const size_t c = fill[w][s];
                    fill[w][s] = at;
                    at += c;
                }
            }
        }
        auto scatter = [&](size_t t) {
            std::vector<size_t>& f = fill[t];
            for (size_t k = t * chunk; k < std::min(n, (t + 1) * chunk); ++k) {
                const MercuryEvent& e = ev[k];
                const uint64_t key = ((uint64_t)(uint32_t)std::min(e.i, e.j) << 32) | (uint32_t)std::max(e.i, e.j);
                items[f[steps ? (size_t)(*steps)[k] : 0]++] = Item{key, (uint32_t)k};
            }
        };
        if (nthreads == 1) {
            scatter(0);
        } else {
            std::vector<std::thread> pool;
            for (size_t w = 0; w < nthreads; ++w) pool.emplace_back(scatter, w);
            for (auto& th : pool) th.join();
        }
    }
    // the steps' runs are independent: sort them on the host's cores
    const size_t nruns = first.size() - 1;
    auto sort_runs = [&](size_t lo, size_t hi) {
        for (size_t s = lo; s < hi; ++s)
            std::sort(items.begin() + first[s], items.begin() + first[s + 1],
                      [](const Item& a, const Item& b) { return a.key < b.key || (a.key == b.key && a.k < b.k); });
    };
    const size_t nthreads =
        n < 262144 ? 1 : std::max<size_t>(1, std::min<size_t>({16, std::thread::hardware_concurrency(), nruns}));
    if (nthreads == 1) {
        sort_runs(0, nruns);
    } else {
        std::vector<std::thread> pool;
        const size_t chunk = (nruns + nthreads - 1) / nthreads;
        for (size_t k = 0; k < nthreads; ++k)
            pool.emplace_back(sort_runs, std::min(nruns, k * chunk), std::min(nruns, (k + 1) * chunk));
        for (auto& th : pool) th.join();
    }
    for (size_t q = 0; q < n; ++q) order[q] = items[q].k;
}

void sort_events(std::vector<MercuryEvent>& ev, std::vector<int>* steps) {
    std::vector<uint32_t> order;
    order_events(ev, steps, order);
    std::vector<MercuryEvent> out(ev.size());
    std::vector<int> so(steps ? ev.size() : 0);
    for (size_t q = 0; q < order.size(); ++q) {
        out[q] = ev[order[q]];
        if (steps) so[q] = (*steps)[order[q]];
    }
    ev.swap(out);
    if (steps) steps->swap(so);
}

void download_buffer(int which, double* xx, double* vv) {
    Context& c = ctx();
    c.transfer.reserve((size_t)6 * c.n);
    // x rows then v rows, read back together
    for (int part = 0; part < 2; ++part) {
        const double* big = c.bigstate[which].p + 3 * part * c.nsplit;
        const double* prt = c.pstate[which].p + (size_t)3 * part * c.npcap;
        gather_kernel<<<blocks(c.n), 256, 0, c.stream>>>(c.transfer.p + (size_t)3 * part * c.n, c.n, 3, c.nsplit,
                                                          big, c.nsplit, prt, c.npcap, c.inv.p);
    }
    check(cudaGetLastError(), "download");
    const size_t bytes = sizeof(double) * 3 * (size_t)c.n;
    copy_out({{c.transfer.p, xx, bytes}, {c.transfer.p + (size_t)3 * c.n, vv, bytes}}, c.stream);
}

// Runs fn(lo, hi) over [0, total) on up to 16 of the host's cores (one
// thread below 4 MB).
template <class F> void host_parallel(size_t total, F fn) {
    const size_t nthreads = total < ((size_t)4 << 20)
                                ? 1
                                : std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency()));
    if (nthreads == 1) {
        fn((size_t)0, total);
        return;
    }
    const size_t chunk = (total + nthreads - 1) / nthreads;
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nthreads; ++t) {
        const size_t lo = std::min(total, t * chunk), hi = std::min(total, lo + chunk);
        if (lo < hi) pool.emplace_back(fn, lo, hi);
    }
    for (auto& th : pool) th.join();
}

// Copies the byte range [lo, hi) of the concatenated spans between their
// host arrays and the page-locked area (to_stage: host -> area).
void stage_bytes(const std::vector<HostSpan>& spans, const std::vector<size_t>& at, char* area, size_t lo, size_t hi,
                 bool to_stage) {
    size_t base = 0;
    for (size_t k = 0; k < spans.size(); ++k) {
        if (at[k] == SIZE_MAX) continue;
        const size_t b0 = base, b1 = base + spans[k].bytes;
        base = b1;
        const size_t s = std::max(lo, b0), e = std::min(hi, b1);
        if (s >= e) continue;
        char* host = static_cast<char*>(spans[k].host) + (s - b0);
        char* st = area + at[k] + (s - b0);
        if (to_stage) std::memcpy(st, host, e - s);
        else std::memcpy(host, st, e - s);
    }
}

}  // namespace

bool host_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();   // plain pageable memory on older drivers
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// The pageable spans' offsets in the page-locked area (SIZE_MAX: the span is
// page-locked and copied directly); returns their total size.
static size_t stage_plan(const std::vector<HostSpan>& spans, std::vector<size_t>& at) {
    size_t total = 0;
    at.assign(spans.size(), SIZE_MAX);
    for (size_t k = 0; k < spans.size(); ++k) {
        if (spans[k].bytes == 0 || host_pinned(spans[k].host)) continue;
        at[k] = total;
        total += spans[k].bytes;
    }
    return total;
}

void copy_in(const std::vector<HostSpan>& spans, cudaStream_t stream, bool sync) {
    Context& c = ctx();
    std::vector<size_t> at;
    const size_t staged = stage_plan(spans, at);
    if (staged) {
        c.reserve_pinned(staged);
        host_parallel(staged, [&](size_t lo, size_t hi) { stage_bytes(spans, at, c.pinned, lo, hi, true); });
    }
    for (size_t k = 0; k < spans.size(); ++k) {
        if (spans[k].bytes == 0) continue;
        const void* src = at[k] == SIZE_MAX ? spans[k].host : c.pinned + at[k];
        check(cudaMemcpyAsync(spans[k].dev, src, spans[k].bytes, cudaMemcpyHostToDevice, stream), "upload");
    }
    if (sync) check(cudaStreamSynchronize(stream), "upload");
}

void copy_out(const std::vector<HostSpan>& spans, cudaStream_t stream) {
    Context& c = ctx();
    std::vector<size_t> at;
    const size_t staged = stage_plan(spans, at);
    if (staged) c.reserve_pinned(staged);
    for (size_t k = 0; k < spans.size(); ++k) {
        if (spans[k].bytes == 0) continue;
        void* dst = at[k] == SIZE_MAX ? spans[k].host : c.pinned + at[k];
        check(cudaMemcpyAsync(dst, spans[k].dev, spans[k].bytes, cudaMemcpyDeviceToHost, stream), "download");
    }
    check(cudaStreamSynchronize(stream), "download");
    if (staged)
        host_parallel(staged, [&](size_t lo, size_t hi) { stage_bytes(spans, at, c.pinned, lo, hi, false); });
}


void scatter_rows(const double* rows, int n, int comps, int nbig, double* big, int big_stride, double* part,
                  int part_stride, const int* inv, cudaStream_t s) {
    scatter_kernel<<<blocks(n), 256, 0, s>>>(rows, n, comps, nbig, big, big_stride, part, part_stride, inv);
}
void gather_rows(double* rows, int n, int comps, int nbig, const double* big, int big_stride, const double* part,
                 int part_stride, const int* inv, cudaStream_t s) {
    gather_kernel<<<blocks(n), 256, 0, s>>>(rows, n, comps, nbig, big, big_stride, part, part_stride, inv);
}

// The upload's checks: body counts and the workspace guard, as the
// reference's (mercury_cuda.cu:384-388): a system that needs more device
// memory than 80% of what is free fails here with a message instead of
// part-way through allocating (checked whenever the particle buffers may have
// to grow).
void upload_checks(int n, int nbig) {
    Context& c = ctx();
    if (n < 1 || nbig < 1 || nbig > n) throw std::runtime_error("invalid body counts");
    if (is_mvs(c.algorithm) && nbig > 512) throw std::runtime_error("more than 512 Big bodies");
    const size_t need = workspace_bytes(n, c.algorithm);
    if ((size_t)9 * (size_t)std::max(2, (n - nbig + 1) & ~1) > c.pstate[0].n || injected("memory")) {
        size_t free_b = 0, total_b = 0;
        if (!injected("memory")) check(cudaMemGetInfo(&free_b, &total_b), "memory");
        if ((double)need > 0.8 * (double)free_b) throw std::runtime_error("Insufficient device workspace memory");
    }
}

// The upload's layout of a system on the device: the massive set, every
// buffer's size, zeroed states and constants (on the library stream). The
// host rows are not read here except for the masses.
// Whether a[0..n) and b[0..n) hold the same bytes (compared on up to 16 host
// threads for large n).
bool same_doubles(const double* a, const double* b, size_t n) {
    const size_t nthreads =
        n < ((size_t)1 << 18) ? 1 : std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency()));
    if (nthreads == 1) return std::memcmp(a, b, sizeof(double) * n) == 0;
    std::vector<char> diff(nthreads, 0);
    std::vector<std::thread> pool;
    const size_t chunk = (n + nthreads - 1) / nthreads;
    for (size_t t = 0; t < nthreads; ++t) {
        const size_t lo = std::min(n, t * chunk), hi = std::min(n, lo + chunk);
        pool.emplace_back([&, t, lo, hi] { diff[t] = std::memcmp(a + lo, b + lo, sizeof(double) * (hi - lo)) != 0; });
    }
    for (auto& th : pool) th.join();
    for (char d : diff)
        if (d) return false;
    return true;
}

// One past the last body at or after nbig whose mass is not zero (nbig if
// none). m[j] != 0.0 is the bits without the sign bit being non-zero (a NaN
// counts as massive, -0.0 as massless); blocks of 512 are tested by OR-ing
// those bits (a loop the compiler vectorizes), on up to 16 host threads for
// large n, each taking a range and reporting its last massive body.
int last_massive(const double* m, int n, int nbig) {
    auto last_in = [m](int lo, int hi) -> int {
        constexpr int B = 512;
        for (int top = hi; top > lo;) {
            const int bot = std::max(lo, top - B);
            uint64_t acc = 0;
            for (int j = bot; j < top; ++j) {
                uint64_t b;
                std::memcpy(&b, m + j, sizeof(b));
                acc |= b << 1;
            }
            if (acc != 0)
                for (int j = top - 1; j >= bot; --j)
                    if (m[j] != 0.0) return j;
            top = bot;
        }
        return -1;
    };
    const int count = n - nbig;
    const int nthreads = count < (1 << 18) ? 1 : (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    int last = -1;
    if (nthreads == 1) {
        last = last_in(nbig, n);
    } else {
        std::vector<int> found(nthreads, -1);
        std::vector<std::thread> pool;
        const int chunk = (count + nthreads - 1) / nthreads;
        for (int t = 0; t < nthreads; ++t) {
            const int lo = nbig + std::min(count, t * chunk), hi = nbig + std::min(count, (t + 1) * chunk);
            pool.emplace_back([&, t, lo, hi] { found[t] = last_in(lo, hi); });
        }
        for (auto& th : pool) th.join();
        for (int f : found) last = std::max(last, f);
    }
    return last >= 0 ? last + 1 : nbig;
}

void upload_layout_for(int n, int nbig, int nmass, int pn, int ngflag, const double* m, const double* jcen);

void upload_layout(int n, int nbig, int pn, int ngflag, const double* m, const double* jcen) {
    upload_layout_for(n, nbig, last_massive(m, n, nbig), pn, ngflag, m, jcen);
}

// The layout for a massive set that ends at nmass (last_massive).
void upload_layout_for(int n, int nbig, int nmass, int pn, int ngflag, const double* m, const double* jcen) {
    Context& c = ctx();
    cudaStream_t s = c.stream;
    // MVS: massive Small bodies move as test particles and act on nothing
    // but the central body's oblateness reaction (mfo_mvs,
    // mercury6_2.for:5061-5068); the Big-body CTA holds them (up to 512
    // bodies in all). Without oblateness more of them are exactly massless
    // for the map and stay in the particle slots.
    const bool obl = jcen[0] != 0.0 || jcen[1] != 0.0 || jcen[2] != 0.0;
    int ns = nmass;
    if (is_mvs(c.algorithm) && nmass > 512) {
        if (obl) throw std::runtime_error("MVS with oblateness and more than 512 Big and massive Small bodies");
        ns = nbig;
    }
    if (ns > 512) throw std::runtime_error("more than 512 Big and massive Small bodies");
    c.n = n;
    c.nbig = nbig;
    c.nmass = nmass;
    c.nsplit = ns;
    c.np = n - ns;
    c.npcap = std::max(2, (c.np + 1) & ~1);
    c.pn = pn != 0 ? 1 : 0;
    c.ngflag = ngflag;
    for (int k = 0; k < 3; ++k) c.jcen[k] = jcen[k];
    // HYBRID compares the masses of every body between calls; the others
    // read the central mass only
    c.m_host.assign(m, m + (c.algorithm == 10 ? n : 1));
    c.event_rate = 0.0;
    c.ev_device = 0;
    c.step_central = false;
    c.mbig.reserve(ns);
    c.rcebig.reserve(ns);
    c.rphysbig.reserve(ns);
    c.ngfbig.reserve((size_t)5 * ns);
    for (int k = 0; k < 2; ++k) {
        c.bigstate[k].reserve((size_t)9 * ns);
        c.pstate[k].reserve((size_t)9 * c.npcap);
    }
    for (int k = 0; k < 2; ++k) {
        c.pconst[k].reserve((size_t)PCONST_ROWS * c.npcap);
        c.perm[k].reserve(c.npcap);
    }
    c.inv.reserve(c.npcap);
    c.kc = 0;
    c.status.reserve(1);
    if (g_event_cap > 0) {
        c.events.release();
        c.event_step.release();
        c.cands.release();
        ensure_events(g_event_cap);
        c.cands.reserve(g_event_cap);
    } else {
        ensure_events(std::max(4096, c.np / 64));
        c.cands.reserve(std::max(16384, c.np));
    }
    c.transfer.reserve((size_t)6 * n);
    if (c.algorithm == 4) {
        c.ra_bb.reserve((size_t)21 * ns);
        c.ra_be.reserve((size_t)21 * ns);
        c.ra_bg.reserve((size_t)21 * ns);
        c.ra_bpx.reserve((size_t)6 * ns);
        c.ra_pb.reserve((size_t)21 * c.npcap);
        c.ra_pe.reserve((size_t)21 * c.npcap);
        c.ra_max.reserve(1);
    }
    // zero padding and cached accelerations
    check(cudaMemsetAsync(c.pstate[0].p, 0, sizeof(double) * 9 * c.npcap, s), "memset");
    check(cudaMemsetAsync(c.pstate[1].p, 0, sizeof(double) * 9 * c.npcap, s), "memset");
    check(cudaMemsetAsync(c.bigstate[0].p, 0, sizeof(double) * 9 * ns, s), "memset");
    check(cudaMemsetAsync(c.bigstate[1].p, 0, sizeof(double) * 9 * ns, s), "memset");
    check(cudaMemsetAsync(c.pconst[0].p, 0, sizeof(double) * PCONST_ROWS * c.npcap, s), "memset");
    check(cudaMemsetAsync(c.pconst[1].p, 0, sizeof(double) * PCONST_ROWS * c.npcap, s), "memset");
    c.cur = 0;
}

// The staged host rows of the Big bodies and of the particles [plo, phi)
// (particle indices, slots in the same range) into the device layout
// through the slot map: x and v rows (3 per body) into the state, the
// masses and radii, the ngf rows (5 per body) when a force law reads them.
// sm null: the particles' masses are zero (their rows stay as zeroed).
void scatter_staged(const double* sx, const double* sv, const double* sm, const double* sr, const double* sp,
                    const double* sg, bool big, int plo, int phi, cudaStream_t s) {
    Context& c = ctx();
    const int ns = c.nsplit;
    if (big) {
        for (int part = 0; part < 2; ++part)
            scatter_rows(part ? sv : sx, ns, 3, ns, c.bigstate[0].p + 3 * part * ns, ns, nullptr, 0, nullptr, s);
        const double* scalars[3] = {sm, sr, sp};
        double* bigdst[3] = {c.mbig.p, c.rcebig.p, c.rphysbig.p};
        for (int q = 0; q < 3; ++q) scatter_rows(scalars[q], ns, 1, ns, bigdst[q], ns, nullptr, 0, nullptr, s);
        if (sg) {
            check(cudaMemcpyAsync(c.ngfbig.p, sg, sizeof(double) * 5 * ns, cudaMemcpyDeviceToDevice, s), "upload");
        } else {
            check(cudaMemsetAsync(c.ngfbig.p, 0, sizeof(double) * 5 * ns, s), "upload");
        }
    }
    const int cnt = phi - plo;
    if (cnt <= 0) return;
    const size_t r0 = (size_t)ns + plo;
    const int* inv = c.inv.p + plo;
    for (int part = 0; part < 2; ++part)
        scatter_rows((part ? sv : sx) + 3 * r0, cnt, 3, 0, nullptr, 0, c.pstate[0].p + (size_t)3 * part * c.npcap,
                     c.npcap, inv, s);
    const double* scalars[3] = {sm, sr, sp};
    double* pdst[3] = {c.pm(), c.prce(), c.prphys()};
    for (int q = 0; q < 3; ++q)
        if (scalars[q]) scatter_rows(scalars[q] + r0, cnt, 1, 0, nullptr, 0, pdst[q], c.npcap, inv, s);
    if (sg) scatter_rows(sg + 5 * r0, cnt, 5, 0, nullptr, 0, c.pngf(), c.npcap, inv, s);
}

}  // namespace mb200

using namespace mb200;

extern "C" {

int mercury_cuda_available(void) {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

void mercury_cuda_free(void) {
    Context& c = ctx();
    try {
        drop_speculation();
    } catch (const std::exception& e) {
        report(e);
    }
    c.release_all();
}

int mercury_cuda_configure(int method) {
    if (method != 1 && method != 2 && method != 3 && method != 4 && method != 9 && method != 10) return 1;
    Context& c = ctx();
    try {
        drop_speculation();
        inject("configure");
        if (method != c.algorithm) mercury_cuda_free();
        c.algorithm = method;
        c.reset = true;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

void mercury_cuda_reset(int flag) {
    if (flag != 2) ctx().reset = true;   // a speculative Big-body step is not taken after this
}

int mercury_cuda_upload(int n, int nbig, int pn, int ngflag, const double* m, const double* xx, const double* vv,
                        const double* ng, const double* jcen, const double* limits, const double* radii) {
    Context& c = ctx();
    try {
        drop_speculation();
        inject("upload");
        upload_checks(n, nbig);
        c.ensure_streams();
        cudaStream_t s = c.stream;
        // Every host array in one round of copies into the upload stage (ngf
        // only when a force law reads it: with ngflag 0 no kernel does, and
        // its rows stay zero). The host's own work below runs while they fly;
        // then the slot order and the layout on the device.
        const size_t N = (size_t)n;
        const bool ngf_read = ngflag != 0;
        c.stage.reserve(9 * N + (ngf_read ? 5 * N : 0));
        double* sx = c.stage.p;
        double* sv = sx + 3 * N;
        double* sm = sv + 3 * N;
        double* sr = sm + N;
        double* sp = sr + N;
        double* sg = sp + N;
        std::vector<HostSpan> spans = {{sx, const_cast<double*>(xx), 24 * N}, {sv, const_cast<double*>(vv), 24 * N},
                                       {sm, const_cast<double*>(m), 8 * N}, {sr, const_cast<double*>(limits), 8 * N},
                                       {sp, const_cast<double*>(radii), 8 * N}};
        if (ngf_read) spans.push_back({sg, const_cast<double*>(ng), 40 * N});
        copy_in(spans, s, false);
        // the stage must not be reused while the copies may still read it
        struct Drain {
            cudaStream_t s;
            bool armed = true;
            ~Drain() {
                if (armed) cudaStreamSynchronize(s);
            }
        } drain{s};
        upload_layout(n, nbig, pn, ngflag, m, jcen);
        order_particles(n, c.nsplit, m[0], sx, sv);
        scatter_staged(sx, sv, sm, sr, sp, ngf_read ? sg : nullptr, true, 0, c.np, s);
        check(cudaGetLastError(), "upload");
        drain.armed = false;
        check(cudaStreamSynchronize(s), "upload");
        c.reset = true;
        c.stepped = false;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_step(double time, double* h, double* hdid, double tol, int64_t* forces, int64_t* rejected) {
    Context& c = ctx();
    try {
        inject("step");
        require_system();
        DropinTimer timer;
        *rejected = 0;
        const int64_t before = c.nforces;
        if (is_mvs(c.algorithm)) {
            mvs_step_once(*h);
            *hdid = *h;
        } else if (c.algorithm == 4) {
            ra15_step_once(time, h, hdid, tol, rejected);
        } else if (c.algorithm == 2 || c.algorithm == 3) {
            bs_step_once(time, h, hdid, tol, rejected);
        } else if (c.algorithm == 10) {
            throw std::runtime_error("HYBRID steps go through mercury_cuda_hybrid_begin/_finish");
        } else {
            throw std::runtime_error("algorithm not available in this build");
        }
        *forces = c.nforces - before;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_download(double* xx, double* vv, int previous) {
    Context& c = ctx();
    try {
        inject("download");
        require_system();
        const int which = previous ? 1 - c.cur : c.cur;
        download_buffer(which, xx, vv);
        // HYBRID's previous state comes back with heliocentric velocities, as
        // the reference keeps it (mercury_cuda.cu:538)
        if (previous && c.algorithm == 10) add_dh_shift(which, vv);
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_events(double time, double h, double rcen, const MercuryEvent** result, int* count) {
    Context& c = ctx();
    try {
        inject("events");
        require_system();
        DropinTimer timer;
        const int prev = 1 - c.cur;
        if (!is_mvs(c.algorithm) && c.algorithm != 10 && c.stepped) screen_pairs(h);
        const bool dh = c.algorithm == 10 && c.stepped;
        // an MVS step that screened for central impacts itself (mvs_step_once)
        bool central_done = false;
        if (c.stepped && c.step_central) {
            if (rcen == c.step_rcen && h == c.step_h) {
                central_done = true;
            } else {
                *c.status_host = DeviceStatus{0, c.pair_events, 0, 0};
                check(cudaMemcpyAsync(c.status.p, c.status_host, sizeof(DeviceStatus), cudaMemcpyHostToDevice,
                                      c.stream),
                      "status");
                drop_central_kernel<<<1, 1, 0, c.stream>>>(c.events.p, c.event_step.p, (int)c.events.n, c.status.p);
                c.dropin_launches += 1;
                read_status();
                c.pair_events = c.status_host->events;
                c.step_central = false;
            }
        }
        c.dropin_rcen = rcen;
        if (dh) {
            // heliocentric velocities of both states (mco_dh2h)
            c.hy_off.reserve(6);
            launch_dh_shift(c.bigstate[prev].p, c.mbig.p, c.nsplit, c.m_host[0], c.hy_off.p, c.stream);
            launch_dh_shift(c.bigstate[c.cur].p, c.mbig.p, c.nsplit, c.m_host[0], c.hy_off.p + 3, c.stream);
            c.dropin_launches += 2;
        }
        int head = 0;   // records read back with the status
        // a step taken from the step ahead brought its status and first
        // records to the host already
        const bool fast = central_done && c.head_ready && !dh;
        c.head_ready = false;
        if (fast) {
            c.status_host->events = c.pair_events;
            head = c.head_count;
        }
        for (int attempt = 0; !fast; ++attempt) {
            // restart the counter after the step's pair events (from pinned
            // memory: the copy does not block), then screen for central impacts
            *c.status_host = DeviceStatus{0, c.pair_events, 0, 0};
            check(cudaMemcpyAsync(c.status.p, c.status_host, sizeof(DeviceStatus), cudaMemcpyHostToDevice, c.stream),
                  "status");
            const int total = c.nsplit - 1 + c.np;
            if (c.stepped && total > 0 && !central_done) {
                CentralArgs a{};
                a.nbig = c.nsplit;
                a.np = c.np;
                a.npcap = c.npcap;
                a.mu = c.m_host[0];
                a.h = h;
                a.rcen = rcen;
                a.big0 = c.bigstate[prev].p;
                a.big1 = c.bigstate[c.cur].p;
                a.part0 = c.pstate[prev].p;
                a.part1 = c.pstate[c.cur].p;
                a.pm = c.pm();
                a.mbig = c.mbig.p;
                a.voff0 = dh ? c.hy_off.p : nullptr;
                a.voff1 = dh ? c.hy_off.p + 3 : nullptr;
                a.perm = c.permp();
                a.events = c.events.p;
                a.event_step = c.event_step.p;
                a.cap = (int)c.events.n;
                a.status = c.status.p;
                central_kernel<<<blocks(total), 256, 0, c.stream>>>(a);
                c.dropin_launches += 1;
                check(cudaGetLastError(), "central");
            }
            // the status and the first records in one round trip
            head = c.stepped ? std::min(Context::EVENT_HEAD, (int)c.events.n) : 0;
            check(cudaMemcpyAsync(c.status_host, c.status.p, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, c.stream),
                  "status");
            if (head > 0)
                check(cudaMemcpyAsync(c.ev_head, c.events.p, sizeof(MercuryEvent) * head, cudaMemcpyDeviceToHost,
                                      c.stream),
                      "events");
            check(cudaStreamSynchronize(c.stream), "step");
            if (!c.status_host->overflow) break;
            if (attempt > 8) throw std::runtime_error("event buffer growth failed");
            // keep the pair events: copy them out, grow, copy back
            std::vector<MercuryEvent> keep(c.pair_events);
            if (c.pair_events)
                check(cudaMemcpy(keep.data(), c.events.p, sizeof(MercuryEvent) * c.pair_events, cudaMemcpyDeviceToHost),
                      "events");
            DBuf<MercuryEvent> grown;
            grown.reserve(std::max(2 * (int)c.events.n, c.status_host->events + 1024));
            c.events.release();
            c.events = grown;
            c.event_step.release();
            c.event_step.reserve(c.events.n);
            if (c.pair_events)
                h2d(c.events.p, keep.data(), sizeof(MercuryEvent) * c.pair_events, c.stream, "events");
        }
        const int nev = c.stepped ? c.status_host->events : 0;
        c.ev_device = 0;
        size_records(c.host_events, nev);
        if (nev) {
            const int got = std::min(nev, head);
            std::memcpy(c.host_events.data(), c.ev_head, sizeof(MercuryEvent) * got);
            if (nev > got)
                check(cudaMemcpy(c.host_events.data() + got, c.events.p + got, sizeof(MercuryEvent) * (nev - got),
                                 cudaMemcpyDeviceToHost),
                      "events");
        }
        for (auto& e : c.host_events) {
            if (e.kind == EV_CENTRAL) e.time = time - h + e.time;
            else e.time = e.time + time;
        }
        sort_events(c.host_events, nullptr);
        c.event_order.clear();
        *count = nev;
        *result = c.host_events.data();
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_force(double* a) {
    Context& c = ctx();
    try {
        drop_speculation();
        inject("force");
        require_system();
        const int nb = c.nbig - 1, ns = c.nsplit;
        c.ftab.reserve((size_t)force_row(nb));
        c.force_out.reserve((size_t)3 * ns + (size_t)3 * c.npcap);
        check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
        ForceAllArgs f{};
        f.f = force_cfg();
        f.np = c.np;
        f.npcap = c.npcap;
        f.bx = c.bigstate[c.cur].p;
        f.mbig = c.mbig.p;
        f.ngfbig = c.ngfbig.p;
        f.px = c.pstate[c.cur].p;
        f.pconst = c.pconst[c.kc].p;
        f.abig = c.force_out.p;
        f.apart = c.force_out.p + 3 * (size_t)ns;
        f.table = c.ftab.p;
        f.status = c.status.p;
        launch_force_all(f, c.stream);
        check(cudaGetLastError(), "force");
        read_status();
        c.nforces += 1;
        if (c.status_host->fault) throw std::runtime_error("Nonfinite force or undefined orbit direction");
        c.transfer.reserve((size_t)6 * c.n);
        gather_rows(c.transfer.p, c.n, 3, ns, f.abig, ns, f.apart, c.npcap, c.inv.p, c.stream);
        check(cudaMemcpyAsync(a, c.transfer.p, sizeof(double) * 3 * c.n, cudaMemcpyDeviceToHost, c.stream), "force");
        check(cudaStreamSynchronize(c.stream), "force");
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_export(double h, int physical, double* xx, double* vv) {
    Context& c = ctx();
    try {
        inject("export");
        require_system();
        if (physical && c.algorithm == 1) {
            export_corrected(h, xx, vv);
        } else {
            download_buffer(c.cur, xx, vv);
            if (physical && c.algorithm == 10) add_dh_shift(c.cur, vv);
        }
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_limits(const double* limits) {
    Context& c = ctx();
    try {
        drop_speculation();
        inject("limits");
        require_system();
        check(cudaMemcpyAsync(c.transfer.p, limits, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream), "limits");
        scatter_rows(c.transfer.p, c.n, 1, c.nsplit, c.rcebig.p, c.nsplit, c.prce(), c.npcap, c.inv.p, c.stream);
        check(cudaStreamSynchronize(c.stream), "limits");
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_hybrid_begin(double h, const double* crit, int flag, int cap, int* ce, int* count, int* pi, int* pj,
                              double* xx, double* vv, int64_t* forces) {
    Context& c = ctx();
    try {
        drop_speculation();
        inject("hybrid_begin");
        require_system();
        if (c.algorithm != 10) throw std::runtime_error("hybrid_begin needs algorithm 10");
        DropinTimer timer;
        const int nb = c.nbig - 1, ns = c.nsplit;
        c.rcritbig.reserve(ns);
        c.hy_scr.reserve((size_t)6 * ns);
        c.hy_tab.reserve(hy_tab_size(nb));
        c.hy_pairs.reserve(4096);
        const int recompute = (flag != 2 || c.reset) ? 1 : 0;
        if (recompute) {
            // rcrit of every body: massive set and the particles' constant row
            c.transfer.reserve((size_t)6 * c.n);
            check(cudaMemcpyAsync(c.transfer.p, crit, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream),
                  "upload");
            scatter_rows(c.transfer.p, c.n, 1, ns, c.rcritbig.p, ns, c.pconst[c.kc].p + (size_t)PC_RCRIT * c.npcap,
                         c.npcap, c.inv.p, c.stream);
            c.dropin_launches += 1;
        }
        for (int attempt = 0;; ++attempt) {
            check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
            launch_hybrid_begin(hybrid_args(h, recompute), c.stream);
            c.dropin_launches += 1 + (c.np > 0 ? 1 : 0);
            check(cudaGetLastError(), "launch");
            read_status();
            if (!(c.status_host->overflow & 1)) break;
            if (attempt > 8) throw std::runtime_error("pair buffer growth failed");
            c.hy_pairs.reserve((size_t)c.status_host->events + 4096);
        }
        if (c.status_host->fault) throw std::runtime_error("Hybrid force failed");
        const int64_t nf = recompute;
        c.nforces += nf;
        const int npairs = c.status_host->events;
        std::vector<int2> pairs(npairs);
        if (npairs)
            check(cudaMemcpy(pairs.data(), c.hy_pairs.p, sizeof(int2) * npairs, cudaMemcpyDeviceToHost), "pairs");
        std::sort(pairs.begin(), pairs.end(),
                  [](const int2& a, const int2& b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
        if (npairs > cap) throw std::runtime_error("Hybrid encounter capacity exceeded");
        c.hy_members.clear();
        if (npairs) {
            std::fill(ce, ce + c.n, 0);
            for (int k = 0; k < npairs; ++k) {
                pi[k] = pairs[k].x + 1;
                pj[k] = pairs[k].y + 1;
                ce[pairs[k].x] = 2;
                ce[pairs[k].y] = 2;
            }
            // the members in ascending order: the pairs' bodies (not a scan of ce)
            c.hy_members.reserve((size_t)2 * npairs);
            for (int k = 0; k < npairs; ++k) {
                c.hy_members.push_back(pairs[k].x);
                c.hy_members.push_back(pairs[k].y);
            }
            std::sort(c.hy_members.begin(), c.hy_members.end());
            c.hy_members.erase(std::unique(c.hy_members.begin(), c.hy_members.end()), c.hy_members.end());
            if (!c.hy_members.empty() && c.hy_members.front() == 0) c.hy_members.erase(c.hy_members.begin());
            const int nm = (int)c.hy_members.size();
            c.hy_ids.reserve(nm);
            c.hy_packed.reserve((size_t)6 * nm);
            check(cudaMemcpyAsync(c.hy_ids.p, c.hy_members.data(), sizeof(int) * nm, cudaMemcpyHostToDevice,
                                  c.stream),
                  "members");
            launch_hybrid_restore(hybrid_args(h, recompute), c.hy_ids.p, nm, c.inv.p, c.hy_packed.p, c.stream);
            c.dropin_launches += 1;
            std::vector<double> packed((size_t)6 * nm);
            check(cudaMemcpyAsync(packed.data(), c.hy_packed.p, sizeof(double) * packed.size(),
                                  cudaMemcpyDeviceToHost, c.stream),
                  "members");
            check(cudaStreamSynchronize(c.stream), "members");
            for (int a = 0; a < nm; ++a)
                for (int q = 0; q < 3; ++q) {
                    xx[3 * c.hy_members[a] + q] = packed[6 * a + q];
                    vv[3 * c.hy_members[a] + q] = packed[6 * a + 3 + q];
                }
        }
        *count = npairs;
        *forces = nf;
        c.hy_begun = true;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_hybrid_finish(double h, const double* m, const double* xx, const double* vv, int64_t* forces) {
    Context& c = ctx();
    try {
        drop_speculation();
        inject("hybrid_finish");
        require_system();
        if (!c.hy_begun) throw std::runtime_error("hybrid_finish without hybrid_begin");
        DropinTimer timer;
        const int nm = (int)c.hy_members.size();
        const int out = 1 - c.cur;
        if (nm) {
            // the members' states after the encounter integration, and the masses
            std::vector<double> packed((size_t)6 * nm);
            for (int a = 0; a < nm; ++a)
                for (int q = 0; q < 3; ++q) {
                    packed[6 * a + q] = xx[3 * c.hy_members[a] + q];
                    packed[6 * a + 3 + q] = vv[3 * c.hy_members[a] + q];
                }
            check(cudaMemcpyAsync(c.hy_packed.p, packed.data(), sizeof(double) * packed.size(),
                                  cudaMemcpyHostToDevice, c.stream),
                  "members");
            scatter_members(c.hy_ids.p, nm, c.hy_packed.p, c.bigstate[out].p, c.pstate[out].p);
            c.dropin_launches += 1;
            // the masses (changed only where the host merged bodies)
            if (c.m_host.size() != (size_t)c.n || !same_doubles(m, c.m_host.data(), (size_t)c.n)) {
                c.transfer.reserve((size_t)6 * c.n);
                check(cudaMemcpyAsync(c.transfer.p, m, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream),
                      "upload");
                scatter_rows(c.transfer.p, c.n, 1, c.nsplit, c.mbig.p, c.nsplit, c.pm(), c.npcap, c.inv.p, c.stream);
                c.m_host.assign(m, m + c.n);
                c.dropin_launches += 1;
            }
            check(cudaStreamSynchronize(c.stream), "upload");
        }
        check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
        launch_hybrid_finish(hybrid_args(h, 0), c.stream);
        c.dropin_launches += 1 + (c.np > 0 ? 1 : 0);
        check(cudaGetLastError(), "launch");
        read_status();
        if (c.status_host->fault) throw std::runtime_error("Hybrid final force failed");
        c.nforces += 1;
        *forces = 1;
        c.cur = out;
        c.reset = false;
        c.stepped = true;
        c.pair_events = 0;
        c.hy_begun = false;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_cuda_encounter_enter(int n, int nb, const double* m, const double* xx, const double* vv,
                                 const double* crit, const double* limits, const double* radii, int np,
                                 const int* pi, const int* pj) {
    try {
        drop_speculation();
        inject("encounter_enter");
        if (g_active != 0) throw std::runtime_error("encounter subsystem already active");
        g_active = 1;
        Context& c = ctx();
        if (c.algorithm != 3) c.release_all();
        c.algorithm = 3;
        c.encounter = true;
        std::vector<double> zero((size_t)5 * n, 0.0);
        const double jc[3] = {0.0, 0.0, 0.0};
        if (mercury_cuda_upload(n, nb, 0, 0, m, xx, vv, zero.data(), jc, limits, radii))
            throw std::runtime_error("Encounter upload failed");
        // rcrit of the massive set and the particle slots' constant row
        c.rcritbig.reserve(c.nsplit);
        check(cudaMemcpyAsync(c.transfer.p, crit, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream), "upload");
        scatter_rows(c.transfer.p, n, 1, c.nsplit, c.rcritbig.p, c.nsplit,
                     c.pconst[c.kc].p + (size_t)PC_RCRIT * c.npcap, c.npcap, c.inv.p, c.stream);
        check(cudaStreamSynchronize(c.stream), "upload");
        // per-body pair lists in pair order (mfo_hkce's accumulation order); a
        // massive body's list leaves out massless partners, which add exactly
        // zero to its sum
        const int ns = c.nsplit;
        auto keep = [&](int body, int partner) { return !(body < ns && partner >= ns); };
        std::vector<int> off(n + 1, 0);
        for (int k = 0; k < np; ++k) {
            const int i = pi[k] - 1, j = pj[k] - 1;
            if (i < 0 || j < 0 || i >= n || j >= n) throw std::runtime_error("encounter pair out of range");
            if (keep(i, j)) ++off[i + 1];
            if (keep(j, i)) ++off[j + 1];
        }
        for (int k = 0; k < n; ++k) off[k + 1] += off[k];
        std::vector<int> fill(off.begin(), off.end() - 1);
        std::vector<int2> adj(std::max(1, off[n]));
        for (int k = 0; k < np; ++k) {
            const int i = pi[k] - 1, j = pj[k] - 1;
            if (keep(i, j)) adj[fill[i]++] = make_int2(j, 0);
            if (keep(j, i)) adj[fill[j]++] = make_int2(i, 1);
        }
        c.adj_off.reserve(n + 1);
        c.adj.reserve(adj.size());
        h2d(c.adj_off.p, off.data(), sizeof(int) * (n + 1), c.stream, "pairs");
        h2d(c.adj.p, adj.data(), sizeof(int2) * adj.size(), c.stream, "pairs");
        return 0;
    } catch (const std::exception& e) {
        g_active = 0;
        return report(e);
    }
}

int mercury_cuda_encounter_update(const double* m, const double* xx, const double* vv) {
    Context& c = ctx();
    try {
        inject("encounter_update");
        require_system();
        if (g_active != 1) throw std::runtime_error("no encounter subsystem active");
        c.transfer.reserve((size_t)6 * c.n);
        check(cudaMemcpyAsync(c.transfer.p, m, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream), "upload");
        scatter_rows(c.transfer.p, c.n, 1, c.nsplit, c.mbig.p, c.nsplit, c.pm(), c.npcap, c.inv.p, c.stream);
        check(cudaStreamSynchronize(c.stream), "upload");
        c.m_host.assign(m, m + c.n);
        for (int part = 0; part < 2; ++part) {
            check(cudaMemcpyAsync(c.transfer.p, part ? vv : xx, sizeof(double) * 3 * c.n, cudaMemcpyHostToDevice,
                                  c.stream),
                  "upload");
            scatter_rows(c.transfer.p, c.n, 3, c.nsplit, c.bigstate[c.cur].p + 3 * part * c.nsplit, c.nsplit,
                         c.pstate[c.cur].p + (size_t)3 * part * c.npcap, c.npcap, c.inv.p, c.stream);
            check(cudaStreamSynchronize(c.stream), "upload");
        }
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

void mercury_cuda_encounter_exit(void) { g_active = 0; }

// ---------------------------------------------------------------- extensions

int mercury_b200_mvs_advance(double time, double h, int nsteps, double rcen, int steps_per_launch,
                             int* nevents) {
    (void)time;
    Context& c = ctx();
    try {
        drop_speculation();
        inject("advance");
        require_system();
        if (!is_mvs(c.algorithm)) throw std::runtime_error("MVS advance needs algorithm 1 or 9");
        if (nsteps < 1) throw std::runtime_error("nsteps must be positive");
        const int nb = c.nbig - 1;
        int K = steps_per_launch > 0 ? steps_per_launch : (c.steps_per_launch > 0 ? c.steps_per_launch : 0);
        const bool auto_K = K <= 0;
        if (K <= 0) K = mvs_max_steps_per_launch(nb);
        K = std::min(K, mvs_max_steps_per_launch(nb));
        K = std::max(1, std::min(K, nsteps));
        // launch sizes: K steps each; with the automatic choice the first launch
        // is short, so that its Big-body steps (one CTA, serial, ~20 us a step)
        // hold up the particles briefly and the next launch's Big-body steps run
        // beside its particles
        std::vector<int>& ksz = c.launch_steps;
        ksz.clear();
        {
            int left = nsteps;
            if (auto_K && nsteps >= 10) {
                ksz.push_back(std::max(1, (K + 4) / 5));
                left -= ksz.back();
            }
            while (left > 0) {
                ksz.push_back(std::min(K, left));
                left -= ksz.back();
            }
        }
        const int nchunks = (int)ksz.size();
        const int stride = tab_stride(nb);
        ensure_candidates(*std::max_element(ksz.begin(), ksz.end()));
        ensure_tables(nsteps + nchunks, nsteps);
        // room for this run's records at the rate the earlier runs showed, so
        // that a long run is not redone after an event-buffer overflow
        {
            // without history, room for encounters of 0.1 % of the particles per step
            // (at most 2^24 records on a guess)
            const double rate = c.event_rate > 0.0 ? c.event_rate * 1.25 : c.np * 1e-3;
            double want = rate * nsteps + 1024.0;
            if (c.event_rate <= 0.0) want = std::min(want, 16777216.0);
            size_t free_b = 0, total_b = 0;
            if (want > (double)c.events.n && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
                want * (sizeof(MercuryEvent) + sizeof(int)) < 0.25 * (double)free_b)
                ensure_events((int)want);
        }
        if ((int)c.chunk_done.size() < nchunks) {
            size_t old = c.chunk_done.size();
            c.chunk_done.resize(nchunks);
            c.kt0.resize(nchunks);
            c.kt1.resize(nchunks);
            for (size_t k = old; k < (size_t)nchunks; ++k) {
                check(cudaEventCreateWithFlags(&c.chunk_done[k], cudaEventDisableTiming), "event");
                check(cudaEventCreate(&c.kt0[k]), "event");
                check(cudaEventCreate(&c.kt1[k]), "event");
            }
        }
        // keep the starting state (and slot order) so that an event-buffer
        // overflow can be redone from it
        c.snapshot.reserve((size_t)9 * c.npcap + 9 * c.nsplit);
        c.snap_const.reserve((size_t)PCONST_ROWS * c.npcap);
        c.snap_perm.reserve((size_t)2 * c.npcap);
        const int kc0 = c.kc;
        auto copy = [&](void* dst, const void* src, size_t bytes) {
            check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c.stream), "snapshot");
        };
        copy(c.snapshot.p, c.pstate[c.cur].p, sizeof(double) * 9 * c.npcap);
        copy(c.snapshot.p + 9 * c.npcap, c.bigstate[c.cur].p, sizeof(double) * 9 * c.nsplit);
        copy(c.snap_const.p, c.pconst[kc0].p, sizeof(double) * PCONST_ROWS * c.npcap);
        copy(c.snap_perm.p, c.perm[kc0].p, sizeof(int) * c.npcap);
        copy(c.snap_perm.p + c.npcap, c.inv.p, sizeof(int) * c.npcap);
        const bool reset0 = c.reset;
        const int order0 = c.steps_since_order;
        for (int attempt = 0;; ++attempt) {
            int launches = 0;
            check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
            check(cudaEventRecord(c.t0, c.stream), "event");
            check(cudaStreamWaitEvent(c.stream_big, c.t0, 0), "wait");
            int bcur = c.cur, pcur = c.cur;
            size_t row = 0;
            c.steps_since_order = order0;
            for (int ch = 0, s0 = 0; ch < nchunks; s0 += ksz[ch], ++ch) {
                const int ks = ksz[ch];
                const int reset = (ch == 0 && reset0) ? 1 : 0;
                double* tab = c.tab.p + row * stride;
                double* det = c.detail.p + (size_t)s0 * std::max(1, nb) * TAB_DETAIL;
                launch_mvs_big(big_args(bcur, 1 - bcur, ks, reset, 1, s0, h, rcen, tab, det), c.stream_big);
                launches += 1;
                check(cudaEventRecord(c.chunk_done[ch], c.stream_big), "event");
                bcur = 1 - bcur;
                if (c.np > 0) {
                    // re-sort the slots by drift path before a launch once 16
                    // steps have gone by since the last order (particles change
                    // path as they evolve, slowly)
                    if (c.steps_since_order >= ORDER_EVERY) {
                        if (c.np >= 64) launches += 3;
                        pcur = reorder_slots(pcur, h, c.stream);
                    }
                    check(cudaStreamWaitEvent(c.stream, c.chunk_done[ch], 0), "wait");
                    check(cudaEventRecord(c.kt0[ch], c.stream), "event");
                    particles_and_events(particle_args(pcur, 1 - pcur, ks, reset, 1, s0, h, rcen, tab, det), c.detail.p,
                                         c.stream);
                    launches += (nb > 0) ? 2 : 1;
                    check(cudaEventRecord(c.kt1[ch], c.stream), "event");
                }
                pcur = 1 - pcur;
                row += ks + 1;
                c.steps_since_order += ks;
            }
            check(cudaStreamWaitEvent(c.stream, c.chunk_done[nchunks - 1], 0), "wait");
            check(cudaEventRecord(c.t1, c.stream), "event");
            check(cudaGetLastError(), "launch");
            read_status();
            if (c.status_host->fault) throw std::runtime_error("MVS force failed");
            if (!c.status_host->overflow) {
                check(cudaEventElapsedTime(&c.last_advance_ms, c.t0, c.t1), "timer");
                double ksum = 0.0;
                c.launch_ms.assign(nchunks, 0.0);
                if (c.np > 0)
                    for (int ch = 0; ch < nchunks; ++ch) {
                        float ms = 0.0f;
                        check(cudaEventElapsedTime(&ms, c.kt0[ch], c.kt1[ch]), "timer");
                        c.launch_ms[ch] = ms;
                        ksum += ms;
                    }
                c.last_particle_kernel_ms = ksum;
                c.last_particle_launches = c.np > 0 ? nchunks : 0;
                c.last_kernel_launches = launches;
                // the Big and particle states must end in the same buffer index
                if (bcur != pcur)
                    copy(c.bigstate[pcur].p, c.bigstate[bcur].p, sizeof(double) * 9 * c.nsplit);
                c.cur = pcur;
                break;
            }
            if (attempt > 8) throw std::runtime_error("event buffer growth failed");
            grow_after_overflow();
            c.kc = kc0;
            copy(c.pstate[c.cur].p, c.snapshot.p, sizeof(double) * 9 * c.npcap);
            copy(c.bigstate[c.cur].p, c.snapshot.p + 9 * c.npcap, sizeof(double) * 9 * c.nsplit);
            copy(c.pconst[kc0].p, c.snap_const.p, sizeof(double) * PCONST_ROWS * c.npcap);
            copy(c.perm[kc0].p, c.snap_perm.p, sizeof(int) * c.npcap);
            copy(c.inv.p, c.snap_perm.p + c.npcap, sizeof(int) * c.npcap);
        }
        c.nforces += nsteps + (reset0 ? 1 : 0);
        c.reset = false;
        c.stepped = false;  // per-step event/previous semantics do not apply after a multi-step run
        c.pair_events = 0;
        const int nev = c.status_host->events;
        c.event_rate = std::max(c.event_rate, (double)nev / nsteps);
        // absolute times: the driver's clock advances by time = time + h per step
        std::vector<double> tend(nsteps);
        double t = time;
        for (int s = 0; s < nsteps; ++s) {
            t = t + h;
            tend[s] = t;
        }
        // ordered on the device; mercury_b200_events copies them straight
        // into the caller's arrays
        c.host_events.clear();
        c.host_steps.clear();
        c.event_order.clear();
        c.ev_device = 0;
        if (nev && order_events_device(nev, nsteps, tend, h)) {
            c.ev_device = nev;
            *nevents = nev;
            return 0;
        }
        size_records(c.host_events, nev);
        size_records(c.host_steps, nev);
        if (nev)
            copy_out({{c.events.p, c.host_events.data(), sizeof(MercuryEvent) * (size_t)nev},
                      {c.event_step.p, c.host_steps.data(), sizeof(int) * (size_t)nev}},
                     c.stream);
        for (int k = 0; k < nev; ++k) {
            MercuryEvent& e = c.host_events[k];
            const double te = tend[c.host_steps[k]];
            if (e.kind == EV_CENTRAL) e.time = te - h + e.time;
            else e.time = e.time + te;
        }
        // records stay in arrival order; mercury_b200_events gathers them in
        // (step, min(i,j), max(i,j)) order straight into the caller's arrays
        order_events(c.host_events, &c.host_steps, c.event_order);
        *nevents = nev;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

// mercury_b200_mvs_run splits the particles into RUN_PARTS parts of at least
// RUN_PART_MIN particles each (else the calls are made in turn).
#ifndef MB200_RUN_PARTS
#define MB200_RUN_PARTS 2
#endif
constexpr int RUN_PARTS = MB200_RUN_PARTS;
constexpr int RUN_PART_MIN = 1 << 17;

// Upload, nsteps fused MVS steps and download in one call: the same as
// mercury_cuda_upload, mercury_b200_mvs_advance and mercury_cuda_download
// (previous = 0), with the particles' copies overlapped with their steps
// when the run is one launch, the host arrays are page-locked and the Small
// bodies massless. The Big bodies go first and take their steps while the
// particles are copied in a few parts; each part is put in slot order within
// its own slots and stepped as soon as it is in (the next part is copied
// meanwhile), and its end states (written as host rows by the particle
// kernel) go back while the next part is stepped. Otherwise the three calls
// are made one after the other.
int mercury_b200_mvs_run(int n, int nbig, int pn, int ngflag, const double* m, const double* xx, const double* vv,
                         const double* ng, const double* jcen, const double* limits, const double* radii,
                         double time, double h, int nsteps, double rcen, int steps_per_launch, double* xout,
                         double* vout, int* nevents) {
    Context& c = ctx();
    auto in_turn = [&]() -> int {
        int rc = mercury_cuda_upload(n, nbig, pn, ngflag, m, xx, vv, ng, jcen, limits, radii);
        if (rc == 0) rc = mercury_b200_mvs_advance(time, h, nsteps, rcen, steps_per_launch, nevents);
        if (rc == 0) rc = mercury_cuda_download(xout, vout, 0);
        return rc;
    };
    try {
        if (!is_mvs(c.algorithm)) throw std::runtime_error("MVS run needs algorithm 1 or 9");
        if (nsteps < 1) throw std::runtime_error("nsteps must be positive");
        if (n < 1 || nbig < 1 || nbig > n) throw std::runtime_error("invalid body counts");
        const int nb = nbig - 1;
        int K = steps_per_launch > 0 ? steps_per_launch : (c.steps_per_launch > 0 ? c.steps_per_launch : 0);
        if (K <= 0) K = mvs_max_steps_per_launch(nb);
        K = std::min(K, mvs_max_steps_per_launch(nb));
        const int np0 = n - nbig;
        const int nparts = np0 >= RUN_PARTS * RUN_PART_MIN ? RUN_PARTS : 1;
        bool pinned = nparts > 1 && K >= nsteps;
        for (const void* p : {(const void*)xx, (const void*)vv, (const void*)m, (const void*)limits,
                              (const void*)radii, (const void*)xout, (const void*)vout})
            pinned = pinned && host_pinned(p);
        if (pinned && ngflag != 0) pinned = host_pinned(ng);
        if (!pinned) return in_turn();

        drop_speculation();
        inject("upload");
        upload_checks(n, nbig);
        c.ensure_streams();
        cudaStream_t s = c.stream, sin = c.stream_ahead, sout = c.stream_out, sbig = c.stream_big;
        const size_t N = (size_t)n;
        const bool ngf_read = ngflag != 0;
        c.stage.reserve(9 * N + (ngf_read ? 5 * N : 0));
        double* sx = c.stage.p;
        double* sv = sx + 3 * N;
        double* sm = sv + 3 * N;
        double* sr = sm + N;
        double* sp = sr + N;
        double* sg = ngf_read ? sp + N : nullptr;
        // nothing below may return before the streams are drained: the stage
        // and the caller's arrays are in use
        struct Drain {
            std::array<cudaStream_t, 4> ss;
            bool armed = true;
            ~Drain() {
                if (armed)
                    for (cudaStream_t q : ss) cudaStreamSynchronize(q);
            }
        } drain{{s, sin, sout, sbig}};
        // part boundaries in particle indices (slots in the same ranges),
        // multiples of 64 slots, for the particles after the Big bodies
        std::vector<int> lo(nparts + 1);
        for (int q = 0; q <= nparts; ++q) lo[q] = q == nparts ? np0 : (int)(((long long)q * np0 / nparts) & ~63LL);
        int cap = 0;
        for (int q = 0; q < nparts; ++q) cap = std::max(cap, lo[q + 1] - lo[q]);
        // events: run_in[q + 1] part q copied in, run_in[0] the Big bodies'
        // rows; run_done[q] part q stepped, run_done[nparts] the Big bodies
        if ((int)c.run_in.size() < nparts + 1) {
            const size_t old = c.run_in.size();
            c.run_in.resize(nparts + 1);
            c.run_done.resize(nparts + 1);
            for (size_t k = old; k < (size_t)nparts + 1; ++k) {
                check(cudaEventCreateWithFlags(&c.run_in[k], cudaEventDisableTiming), "event");
                check(cudaEventCreateWithFlags(&c.run_done[k], cudaEventDisableTiming), "event");
            }
        }
        // copies in first (the earlier calls have drained every stream, so
        // the stage is free): the Big bodies' rows, then every part's; the
        // host's scan and the layout below run while they fly (the masses of
        // the Big bodies only: a massless particle needs none)
        auto rows_in = [&](size_t r0, size_t r1, bool mass) {
            auto h2d_rows = [&](double* dst, const double* src, size_t width) {
                check(cudaMemcpyAsync(dst + r0 * width, src + r0 * width, sizeof(double) * width * (r1 - r0),
                                      cudaMemcpyHostToDevice, sin),
                      "upload");
            };
            h2d_rows(sx, xx, 3);
            h2d_rows(sv, vv, 3);
            if (mass) h2d_rows(sm, m, 1);
            h2d_rows(sr, limits, 1);
            h2d_rows(sp, radii, 1);
            if (ngf_read) h2d_rows(sg, ng, 5);
        };
        rows_in(0, nbig, true);
        check(cudaEventRecord(c.run_in[0], sin), "event");
        for (int q = 0; q < nparts; ++q) {
            rows_in(nbig + (size_t)lo[q], nbig + (size_t)lo[q + 1], false);
            check(cudaEventRecord(c.run_in[q + 1], sin), "event");
        }
        // the layout for massless particles; the host's scan of the masses
        // runs beside the queueing below and is checked at the end
        struct Scan {
            int nmass = -1;
            std::thread th;
            ~Scan() {
                if (th.joinable()) th.join();
            }
        } scan;
        scan.th = std::thread([&scan, m, n, nbig] { scan.nmass = last_massive(m, n, nbig); });
        upload_layout_for(n, nbig, nbig, pn, ngflag, m, jcen);
        const int ns = c.nsplit, np = c.np;
        // every buffer that may be reallocated (cudaFree waits for the device)
        {
            const double want = std::min(np * 1e-3 * nsteps + 1024.0, 16777216.0);
            size_t free_b = 0, total_b = 0;
            if (want > (double)c.events.n && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
                want * (sizeof(MercuryEvent) + sizeof(int)) < 0.25 * (double)free_b)
                ensure_events((int)want);
        }
        ensure_tables(nsteps + 1, nsteps);
        ensure_candidates(nsteps);   // every part's candidates before the one classification
        order_chunk(0, 0, 0, cap, m[0], sx, sv, s);   // sizes the ordering scratch
        c.run_tiles.reserve(nparts);
        check(cudaMemsetAsync(c.run_tiles.p, 0, sizeof(int) * nparts, s), "memset");
        // the Big bodies' steps, while the particles come in
        check(cudaStreamWaitEvent(s, c.run_in[0], 0), "wait");
        scatter_staged(sx, sv, sm, sr, sp, sg, true, 0, 0, s);
        check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), s), "memset");
        check(cudaEventRecord(c.t0, s), "event");
        check(cudaStreamWaitEvent(sbig, c.t0, 0), "wait");
        launch_mvs_big(big_args(0, 1, nsteps, 1, 1, 0, h, rcen, c.tab.p, c.detail.p), sbig);
        check(cudaEventRecord(c.run_done[nparts], sbig), "event");
        // each part, once in: put in slot order, laid out, stepped; its end
        // states (written as host rows by the kernel) go back while the next
        // part is laid out and stepped
        double* rx = c.transfer.p;
        double* rv = c.transfer.p + 3 * N;
        for (int q = 0; q < nparts; ++q) {
            const int plo = lo[q], phi = lo[q + 1], cnt = phi - plo;
            const int pad = (q == nparts - 1 && c.npcap > np) ? 1 : 0;
            check(cudaStreamWaitEvent(s, c.run_in[q + 1], 0), "wait");
            order_chunk(plo, phi, pad, cap, m[0], sx, sv, s);
            scatter_staged(sx, sv, nullptr, sr, sp, sg, false, plo, phi, s);
            if (q == 0) check(cudaStreamWaitEvent(s, c.run_done[nparts], 0), "wait");
            MvsParticleArgs pa = particle_args(0, 1, nsteps, 1, 1, 0, h, rcen, c.tab.p, c.detail.p);
            pa.np = cnt;
            pa.xin += plo;
            pa.xout += plo;
            pa.m += plo;
            pa.rce += plo;
            pa.rphys += plo;
            pa.ngf += plo;
            pa.perm += plo;
            pa.tiles = c.run_tiles.p + q;
            pa.rows_x = rx + 3 * (size_t)ns;
            pa.rows_v = rv + 3 * (size_t)ns;
            launch_mvs_particles(pa, s, c.particle_threads);
            check(cudaEventRecord(c.run_done[q], s), "event");
            check(cudaStreamWaitEvent(sout, c.run_done[q], 0), "wait");
            const size_t r0 = ns + (size_t)plo;
            check(cudaMemcpyAsync(xout + 3 * r0, rx + 3 * r0, sizeof(double) * 3 * cnt, cudaMemcpyDeviceToHost, sout),
                  "download");
            check(cudaMemcpyAsync(vout + 3 * r0, rv + 3 * r0, sizeof(double) * 3 * cnt, cudaMemcpyDeviceToHost, sout),
                  "download");
        }
        // the pair records of every part, the Big bodies' rows out
        ClassifyArgs ca{};
        ca.nb = nb;
        ca.nbig = nbig;
        ca.h = h;
        ca.detail = c.detail.p;
        ca.cands = c.cands.p;
        ca.cand_cap = (int)c.cands.n;
        ca.events = c.events.p;
        ca.event_step = c.event_step.p;
        ca.event_cap = (int)c.events.n;
        ca.status = c.status.p;
        ca.step_base = 0;
        if (nb > 0 && np > 0) launch_classify(ca, s);
        check(cudaMemsetAsync(&c.status.p->cands, 0, sizeof(int), s), "memset");
        gather_rows(rx, ns, 3, ns, c.bigstate[1].p, ns, nullptr, 0, nullptr, s);
        gather_rows(rv, ns, 3, ns, c.bigstate[1].p + 3 * ns, ns, nullptr, 0, nullptr, s);
        check(cudaMemcpyAsync(xout, rx, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost, s), "download");
        check(cudaMemcpyAsync(vout, rv, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost, s), "download");
        check(cudaGetLastError(), "launch");
        check(cudaEventRecord(c.t1, s), "event");
        scan.th.join();
        drain.armed = false;
        for (cudaStream_t q : {sin, sout, sbig}) check(cudaStreamSynchronize(q), "step");
        read_status();
        if (scan.nmass != nbig) return in_turn();   // a massive Small body
        c.steps_since_order = 0;
        c.cur = 1;
        c.stepped = false;
        c.pair_events = 0;
        if (c.status_host->fault) throw std::runtime_error("MVS force failed");
        if (c.status_host->overflow) {
            // more records than the buffers held: the whole run again from the
            // uploaded states (still in buffer 0), with room
            grow_after_overflow();
            c.cur = 0;
            c.reset = true;
            const int rc = mercury_b200_mvs_advance(time, h, nsteps, rcen, steps_per_launch, nevents);
            return rc ? rc : mercury_cuda_download(xout, vout, 0);
        }
        check(cudaEventElapsedTime(&c.last_advance_ms, c.t0, c.t1), "timer");
        c.last_particle_launches = nparts;
        c.last_kernel_launches = 1 + 11 * nparts + 3;
        c.nforces += nsteps + 1;
        c.reset = false;
        const int nev = c.status_host->events;
        c.event_rate = std::max(c.event_rate, (double)nev / nsteps);
        std::vector<double> tend(nsteps);
        double t = time;
        for (int q = 0; q < nsteps; ++q) {
            t = t + h;
            tend[q] = t;
        }
        c.host_events.clear();
        c.host_steps.clear();
        c.event_order.clear();
        c.ev_device = 0;
        if (nev && order_events_device(nev, nsteps, tend, h)) {
            c.ev_device = nev;
        } else if (nev) {
            size_records(c.host_events, nev);
            size_records(c.host_steps, nev);
            copy_out({{c.events.p, c.host_events.data(), sizeof(MercuryEvent) * (size_t)nev},
                      {c.event_step.p, c.host_steps.data(), sizeof(int) * (size_t)nev}},
                     c.stream);
            for (int k = 0; k < nev; ++k) {
                MercuryEvent& e = c.host_events[k];
                const double te = tend[c.host_steps[k]];
                if (e.kind == EV_CENTRAL) e.time = te - h + e.time;
                else e.time = e.time + te;
            }
            order_events(c.host_events, &c.host_steps, c.event_order);
        }
        *nevents = nev;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_events(MercuryEvent* dst, int* steps, int cap) {
    Context& c = ctx();
    if (c.ev_device > 0) {
        // the last fused run's records, ordered on the device
        const int nev = c.ev_device;
        const size_t k = (size_t)std::max(0, std::min(cap, nev));
        if (k == 0) return nev;
        try {
            std::vector<HostSpan> spans = {{c.ev_sorted.p, dst, sizeof(MercuryEvent) * k}};
            if (steps) spans.push_back({c.ev_sorted_step.p, steps, sizeof(int) * k});
            copy_out(spans, c.stream);
        } catch (const std::exception& e) {
            report(e);
            return -1;
        }
        return nev;
    }
    const int nev = (int)c.host_events.size();
    const int k = std::max(0, std::min(cap, nev));
    const bool ordered = c.event_order.size() == c.host_events.size();
    auto copy = [&](int lo, int hi) {
        for (int q = lo; q < hi; ++q) {
            const size_t r = ordered ? c.event_order[q] : (size_t)q;
            dst[q] = c.host_events[r];
            if (steps && r < c.host_steps.size()) steps[q] = c.host_steps[r];
        }
    };
    // a few hundred MB for a long run: gather on the host's cores
    const int nthreads = k < (1 << 18) ? 1 : (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (nthreads == 1) {
        copy(0, k);
    } else {
        std::vector<std::thread> pool;
        const int chunk = (k + nthreads - 1) / nthreads;
        for (int w = 0; w < nthreads; ++w) pool.emplace_back(copy, std::min(k, w * chunk), std::min(k, (w + 1) * chunk));
        for (auto& th : pool) th.join();
    }
    return nev;
}

int mercury_b200_timing(double* advance_ms, double* particle_kernel_ms, int* particle_launches,
                        int* kernel_launches) {
    Context& c = ctx();
    if (advance_ms) *advance_ms = c.last_advance_ms;
    if (particle_kernel_ms) *particle_kernel_ms = c.last_particle_kernel_ms;
    if (particle_launches) *particle_launches = c.last_particle_launches;
    if (kernel_launches) *kernel_launches = c.last_kernel_launches;
    return 0;
}

int mercury_b200_advance_launches(int* steps, double* kernel_ms, int cap) {
    Context& c = ctx();
    const int n = (int)c.launch_steps.size();
    for (int k = 0; k < std::min(n, cap); ++k) {
        if (steps) steps[k] = c.launch_steps[k];
        if (kernel_ms) kernel_ms[k] = k < (int)c.launch_ms.size() ? c.launch_ms[k] : 0.0;
    }
    return n;
}

int mercury_b200_dropin_time(double* ms, int64_t* launches, int reset) {
    if (ms) *ms = g_dropin_ms;
    if (launches) *launches = g_contexts[0].dropin_launches + g_contexts[1].dropin_launches;
    if (reset) {
        g_dropin_ms = 0.0;
        g_contexts[0].dropin_launches = 0;
        g_contexts[1].dropin_launches = 0;
    }
    return 0;
}

int mercury_b200_energy(double h, int physical, const double* spin, double* e, double* l2) {
    Context& c = ctx();
    try {
        require_system();
        // the massive set ends at the last massive body (MVS takes massless
        // Small bodies only; the other integrators keep bodies up to nmass)
        if (c.nmass != c.nsplit) throw std::runtime_error("massive bodies outside the massive set");
        EnergyArgs a{};
        a.nm = c.nmass;
        a.mbig = c.mbig.p;
        if (physical && c.algorithm == 1) {
            run_corrector(h, true);
            a.big = c.corr_big.p;
            a.bs = c.nsplit;
        } else {
            a.big = c.bigstate[c.cur].p;
            a.bs = c.nsplit;
            if (physical && c.algorithm == 10) {
                c.hy_off.reserve(6);
                launch_dh_shift(c.bigstate[c.cur].p, c.mbig.p, c.nsplit, c.m_host[0], c.hy_off.p, c.stream);
                a.voff = c.hy_off.p;
            }
        }
        for (int q = 0; q < 3; ++q) a.jcen[q] = c.jcen[q];
        // spin angular momenta first, in body order (mxx_en's first loop)
        for (int q = 0; q < 3; ++q) a.spin[q] = 0.0;
        if (spin)
            for (int j = 0; j < c.n; ++j)
                for (int q = 0; q < 3; ++q) a.spin[q] = a.spin[q] + spin[3 * (size_t)j + q];
        c.energy_scr.reserve((size_t)c.nmass + 2);
        a.tmp = c.energy_scr.p;
        a.out = c.energy_scr.p + c.nmass;
        launch_energy(a, c.stream);
        check(cudaGetLastError(), "energy");
        double out[2];
        check(cudaMemcpyAsync(out, a.out, sizeof(out), cudaMemcpyDeviceToHost, c.stream), "energy");
        check(cudaStreamSynchronize(c.stream), "energy");
        if (e) *e = out[0];
        if (l2) *l2 = out[1];
        return 0;
    } catch (const std::exception& ex) {
        return report(ex);
    }
}

int mercury_b200_ejections(double h, int physical, double rmax, int i0, int* ids, int cap, int* count) {
    Context& c = ctx();
    try {
        require_system();
        if (!(rmax > 0.0) || !std::isfinite(rmax)) throw std::runtime_error("ejection radius must be positive");
        if (cap < 0 || (cap > 0 && !ids) || !count) throw std::runtime_error("invalid ejection output");
        const double* bx = c.bigstate[c.cur].p;
        const double* px = c.pstate[c.cur].p;
        if (physical && c.algorithm == 1) {
            run_corrector(h);
            bx = c.corr_big.p;
            px = c.corr_part.p;
        }
        const int first = i0 <= 0 ? 1 : i0 - 1;   // mxx_ejec: i0 <= 0 means 2
        const int total = c.nsplit + c.np;
        c.ej_ids.reserve((size_t)c.n + 1);
        check(cudaMemsetAsync(c.ej_ids.p, 0, sizeof(int), c.stream), "memset");
        ejection_kernel<<<blocks(total), 256, 0, c.stream>>>(bx, c.nsplit, px, c.npcap, c.np, c.permp(), first,
                                                            rmax * rmax, c.ej_ids.p, c.n);
        check(cudaGetLastError(), "launch");
        int found = 0;
        check(cudaMemcpyAsync(&found, c.ej_ids.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream), "ejections");
        check(cudaStreamSynchronize(c.stream), "ejections");
        std::vector<int> got(found);
        if (found) {
            check(cudaMemcpyAsync(got.data(), c.ej_ids.p + 1, sizeof(int) * found, cudaMemcpyDeviceToHost, c.stream),
                  "ejections");
            check(cudaStreamSynchronize(c.stream), "ejections");
        }
        std::sort(got.begin(), got.end());
        for (int k = 0; k < found && k < cap; ++k) ids[k] = got[k];
        *count = found;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_hybrid_member_list(int* ids, int cap) {
    Context& c = ctx();
    if (!c.hy_begun) return -1;
    const int nm = (int)c.hy_members.size();
    if (ids && cap > 0) std::memcpy(ids, c.hy_members.data(), sizeof(int) * (size_t)std::min(cap, nm));
    return nm;
}

int mercury_b200_hybrid_members(const int* ids, int count) {
    Context& c = ctx();
    try {
        drop_speculation();
        require_system();
        if (!c.hy_begun) throw std::runtime_error("hybrid_members outside a HYBRID step");
        if (count < 0 || (count > 0 && !ids)) throw std::runtime_error("invalid member list");
        std::vector<int> m(ids, ids + count);
        std::sort(m.begin(), m.end());
        m.erase(std::unique(m.begin(), m.end()), m.end());
        for (int j : m)
            if (j < 1 || j >= c.n) throw std::runtime_error("member id out of range");
        c.hy_members = m;
        const int nm = (int)m.size();
        if (nm) {
            c.hy_ids.reserve(nm);
            c.hy_packed.reserve((size_t)6 * nm);
            h2d(c.hy_ids.p, m.data(), sizeof(int) * nm, c.stream, "members");
        }
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

namespace {

// Adds the device time between two completed events on the library stream
// to the drop-in total.
void add_dropin_span(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess) g_dropin_ms += ms;
}

// mdt_hkce's substep loop (mercury6_2.for:3884-3937) with mdt_bs2's step
// control (3568-3596) held on the device. One attempt is three launches: the
// massive set's levels (keeping its start state), the particles' levels with
// the massive set's extrapolation as the last CTA, and enc_post_kernel (the
// decision in every thread, the next attempt's control block, and after an
// acceptance the in-place commit and the substep's pair screen). Attempts
// alternate between two control blocks and two sets of level maxima
// (attempt parity p reads set p and prepares set 1 - p), so that no launch
// reads what it writes. After the subsystem reached h every launch returns at
// once. The host enqueues attempts in blocks, as replays of a CUDA graph of
// GRAPH_ATTEMPTS attempts, and reads the control block back once per block;
// the block size follows the attempts still needed, estimated from the
// progress. Records stay on the device, tagged with their substep, until the
// subsystem reaches h. The states do not depend on the records, so after an
// event-buffer or substep-table overflow the buffers grow and the run is
// redone from its starting state.
void encounter_run_device(double time, double h, double tol, double* hrec, int64_t* nforces_out,
                          std::vector<MercuryEvent>& keep) {
    Context& c = ctx();
    if (c.algorithm != 3) throw std::runtime_error("the encounter subsystem steps by algorithm 3 (mdt_bs2)");
    constexpr int GRAPH_ATTEMPTS = 8;   // even: a replay leaves the parity where it found it
    mercury_cuda_reset(1);
    const int in = c.cur;
    const double hrec0 = *hrec;
    const size_t np_el = c.pstate[in].n, nb_el = c.bigstate[in].n;
    c.snapshot.reserve(np_el + nb_el);
    check(cudaMemcpyAsync(c.snapshot.p, c.pstate[in].p, sizeof(double) * np_el, cudaMemcpyDeviceToDevice, c.stream),
          "snapshot");
    check(cudaMemcpyAsync(c.snapshot.p + np_el, c.bigstate[in].p, sizeof(double) * nb_el, cudaMemcpyDeviceToDevice,
                          c.stream),
          "snapshot");
    c.enc_ctl.reserve(2);
    c.enc_tstep.reserve(1024);
    c.enc_bpre.reserve((size_t)6 * c.nsplit);
    c.bs_errs.reserve(26);
    c.bs_lvst.reserve(26);
    struct Graph {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t e = nullptr;
        ~Graph() {
            if (e) cudaGraphExecDestroy(e);
            if (g) cudaGraphDestroy(g);
        }
    };
    for (int redo = 0;; ++redo) {
        // the first substep's trial step: hrec, clipped to the subsystem's end
        EncCtl k{};
        double hlocal = std::copysign(*hrec, h);
        k.hrec = hlocal;
        if (std::fabs(hlocal) > std::fabs(h)) hlocal = std::copysign(std::fabs(h), h);
        if (0.0 + hlocal == 0.0) throw std::runtime_error("BS cannot advance time at the requested tolerance");
        k.h0 = hlocal;
        k.h = h;
        k.tol = tol;
        k.time = time;
        k.forces = 1;   // the first substep's start-of-step force
        k.step_cap = (int)c.enc_tstep.n;
        k.tstep = c.enc_tstep.p;
        *c.enc_host = k;
        BsArgs base = bs_attempt_args(0.0);
        base.bx_pre = c.enc_bpre.p;
        base.fuse_extrap = 1;
        auto attempt = [&](int p) {
            BsArgs a = base;
            a.ctl = c.enc_ctl.p + p;
            a.errs = c.bs_errs.p + 13 * p;
            a.lvst = c.bs_lvst.p + 13 * p;
            launch_bs_sequence(a, c.stream);
            EncPostArgs e{};
            e.ctl_in = c.enc_ctl.p + p;
            e.ctl_out = c.enc_ctl.p + (1 - p);
            e.errs = a.errs;
            e.lvst = a.lvst;
            e.errs_next = c.bs_errs.p + 13 * (1 - p);
            e.lvst_next = c.bs_lvst.p + 13 * (1 - p);
            e.nbig = c.nbig;
            e.nsplit = c.nsplit;
            e.np = c.np;
            e.npcap = c.npcap;
            e.active_np = a.active_np;
            e.bx_pre = c.enc_bpre.p;
            e.bx = c.bigstate[in].p;
            e.bcand = a.bcand;
            e.pcand = a.pcand;
            e.px = c.pstate[in].p;
            e.mbig = c.mbig.p;
            e.rcebig = c.rcebig.p;
            e.rphysbig = c.rphysbig.p;
            e.pconst = c.pconst[c.kc].p;
            e.perm = c.permp();
            e.events = c.events.p;
            e.event_step = c.event_step.p;
            e.event_cap = (int)c.events.n;
            e.status = c.status.p;
            launch_enc_post(e, c.stream);
            check(cudaGetLastError(), "launch");
        };
        check(cudaMemcpyAsync(c.enc_ctl.p, c.enc_host, sizeof(EncCtl), cudaMemcpyHostToDevice, c.stream), "upload");
        check(cudaMemsetAsync(c.status.p, 0, sizeof(DeviceStatus), c.stream), "memset");
        check(cudaMemsetAsync(c.bs_errs.p, 0, sizeof(unsigned long long) * 26, c.stream), "memset");
        check(cudaMemsetAsync(c.bs_lvst.p, 0, sizeof(DeviceStatus) * 26, c.stream), "memset");
        // attempt 0 eagerly (kernel attributes set), then the graph of attempts
        // 1.. GRAPH_ATTEMPTS (parities 1, 0, 1, ...); after every block the
        // newest control block is copy 1
        check(cudaEventRecord(c.d0, c.stream), "event");
        attempt(0);
        Graph graph;
        check(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed), "graph");
        for (int q = 0; q < GRAPH_ATTEMPTS; ++q) attempt((1 + q) % 2);
        check(cudaStreamEndCapture(c.stream, &graph.g), "graph");
        check(cudaGraphInstantiate(&graph.e, graph.g, 0), "graph");
        c.dropin_launches += 3;
        int blocks = 2;   // graph replays in the first block
        for (;;) {
            for (int b = 0; b < blocks; ++b) check(cudaGraphLaunch(graph.e, c.stream), "graph");
            c.dropin_launches += (int64_t)blocks * GRAPH_ATTEMPTS * 3;
            check(cudaMemcpyAsync(c.enc_host, c.enc_ctl.p + 1, sizeof(EncCtl), cudaMemcpyDeviceToHost, c.stream),
                  "status");
            check(cudaEventRecord(c.d1, c.stream), "event");
            check(cudaEventSynchronize(c.d1), "step");
            add_dropin_span(c.d0, c.d1);
            const EncCtl& now = *c.enc_host;
            if (now.stop) break;
            // the attempts still needed at the rate so far, and a little more
            const double done = std::fabs(now.tlocal) / std::fabs(h);
            const double rate = now.attempts / std::max(done, 1e-3);
            const double need = rate * (1.0 - done) * 1.1 + 1.0;
            blocks = (int)std::min(64.0, std::max(1.0, std::ceil(need / GRAPH_ATTEMPTS)));
            check(cudaEventRecord(c.d0, c.stream), "event");
        }
        const EncCtl done = *c.enc_host;
        if (done.error == ENC_ERR_FORCE) throw std::runtime_error("BS force failed");
        if (done.error == ENC_ERR_NONFINITE) throw std::runtime_error("Nonfinite BS2 force or extrapolation");
        if (done.error == ENC_ERR_ADVANCE)
            throw std::runtime_error("BS cannot advance time at the requested tolerance");
        read_status();
        const bool steps_full = done.error == ENC_ERR_STEPS;
        if (!steps_full && !c.status_host->overflow) {
            const int nev = c.status_host->events;
            std::vector<MercuryEvent> ev(nev);
            std::vector<int> steps(nev);
            std::vector<double> tstep(done.substeps);
            if (done.substeps)
                check(cudaMemcpyAsync(tstep.data(), c.enc_tstep.p, sizeof(double) * done.substeps,
                                      cudaMemcpyDeviceToHost, c.stream),
                      "events");
            if (nev) {
                check(cudaMemcpyAsync(ev.data(), c.events.p, sizeof(MercuryEvent) * nev, cudaMemcpyDeviceToHost,
                                      c.stream),
                      "events");
                check(cudaMemcpyAsync(steps.data(), c.event_step.p, sizeof(int) * nev, cudaMemcpyDeviceToHost,
                                      c.stream),
                      "events");
            }
            check(cudaStreamSynchronize(c.stream), "events");
            // the drop-in events call adds the substep's end time to each record
            for (int r = 0; r < nev; ++r) ev[r].time = ev[r].time + tstep[steps[r]];
            std::vector<uint32_t> order;
            order_events(ev, &steps, order);
            keep.resize(nev);
            for (int r = 0; r < nev; ++r) keep[r] = ev[order[r]];
            *hrec = done.hrec;
            c.nforces += done.forces;
            *nforces_out = done.forces;
            c.stepped = true;
            c.pair_events = 0;
            return;
        }
        if (redo > 8) throw std::runtime_error("event buffer growth failed");
        if (steps_full) c.enc_tstep.reserve(2 * c.enc_tstep.n);
        if (c.status_host->overflow) grow_after_overflow();
        check(cudaMemcpyAsync(c.pstate[in].p, c.snapshot.p, sizeof(double) * np_el, cudaMemcpyDeviceToDevice,
                              c.stream),
              "restore");
        check(cudaMemcpyAsync(c.bigstate[in].p, c.snapshot.p + np_el, sizeof(double) * nb_el,
                              cudaMemcpyDeviceToDevice, c.stream),
              "restore");
        *hrec = hrec0;
    }
}

}  // namespace

int mercury_b200_encounter_run(double time, double h, double tol, double rcen, double* hrec, int64_t* forces,
                               int* nrecords) {
    try {
        if (g_active != 1) throw std::runtime_error("no encounter subsystem active");
        std::vector<MercuryEvent> keep;
        int64_t nforces = 0;
        if (!ctx().tangent) {
            encounter_run_device(time, h, tol, hrec, &nforces, keep);
        } else {
            // the members' tangents are kept: the drop-in calls one by one
            int dtflag = 1;
            double tlocal = 0.0, hlocal = std::copysign(*hrec, h);
            for (;;) {
                const double tmp0 = std::fabs(h) - std::fabs(tlocal);
                *hrec = hlocal;
                if (std::fabs(hlocal) > tmp0) hlocal = std::copysign(tmp0, h);
                mercury_cuda_reset(dtflag);
                double hdid = 0.0;
                int64_t nf = 0, nr = 0;
                if (mercury_cuda_step(tlocal, &hlocal, &hdid, tol, &nf, &nr))
                    throw std::runtime_error("encounter step failed");
                nforces += nf;
                dtflag = 2;
                tlocal = tlocal + hdid;
                const MercuryEvent* ev = nullptr;
                int count = 0;
                if (mercury_cuda_events(time + tlocal, hdid, rcen, &ev, &count))
                    throw std::runtime_error("encounter events failed");
                for (int k = 0; k < count; ++k)
                    if (!(ev[k].kind & EV_CENTRAL)) keep.push_back(ev[k]);
                if (!((tlocal - h) * h < 0.0)) break;
            }
        }
        Context& c = ctx();
        c.host_events.swap(keep);
        c.ev_device = 0;
        c.host_steps.clear();
        c.event_order.clear();
        *forces = nforces;
        *nrecords = (int)c.host_events.size();
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

// Fortran SPACING(x) for double x: 2^(EXPONENT(x) - 53), TINY for 0.
static double fortran_spacing(double x) {
    x = std::fabs(x);
    if (x == 0.0) return 2.2250738585072014e-308;
    int e = 0;
    std::frexp(x, &e);
    return std::ldexp(1.0, e - 53);
}

// mercury_support.f90:202-212: the tolerance of an epoch and a step towards it.
static double epoch_epsilon(double t, double target) {
    return std::max(1e-13, 2.0 * fortran_spacing(std::max(std::fabs(t), std::fabs(target))));
}
static double clipped_step(double t, double target, double proposed, double cap) {
    const double step =
        std::copysign(std::min(std::min(std::fabs(target - t), std::fabs(proposed)), std::fabs(cap)), target - t);
    if (!std::isfinite(step) || t + step == t)
        throw std::runtime_error("Timestep cannot advance the epoch; loosen tolerance or inspect the orbit");
    return step;
}

int mercury_b200_epoch_order(int nsml, const double* epochs, double tstart, int* order) {
    try {
        if (nsml < 0 || (nsml > 0 && (!epochs || !order))) throw std::runtime_error("invalid epoch arrays");
        // mxx_sort (mercury6_2.for:7392-7421): Shell sort with gaps 1, 4, 13, ...
        std::vector<double> x(epochs, epochs + nsml);
        std::vector<int> index(nsml);
        for (int i = 0; i < nsml; ++i) index[i] = i;
        int inc = 1;
        while (inc < nsml / 3) inc = 3 * inc + 1;
        while (inc >= 1) {
            for (int i = inc; i < nsml; ++i) {
                const double y = x[i];
                const int iy = index[i];
                int j = i;
                while (j >= inc) {
                    if (x[j - inc] <= y) break;
                    x[j] = x[j - inc];
                    index[j] = index[j - inc];
                    j = j - inc;
                }
                x[j] = y;
                index[j] = iy;
            }
            inc = inc / 3;
        }
        // mxx_sync (mercury6_2.for:7473-7486): the epoch furthest from tstart first
        if (nsml > 0 && std::fabs(x[0] - tstart) < std::fabs(x[nsml - 1] - tstart))
            for (int j = 0; j < nsml / 2; ++j) {
                std::swap(x[j], x[nsml - 1 - j]);
                std::swap(index[j], index[nsml - 1 - j]);
            }
        for (int i = 0; i < nsml; ++i) order[i] = index[i];
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_sync_epochs(const double* epoch, double* time, double h0, double tol, double dtout, int* steps) {
    Context& c = ctx();
    try {
        drop_speculation();
        require_system();
        if (c.algorithm != 2) throw std::runtime_error("epoch synchronisation needs algorithm 2 (mdt_bs1)");
        if (c.nsplit != c.nbig) throw std::runtime_error("epoch synchronisation needs massless Small bodies");
        struct Restore {
            Context& c;
            ~Restore() { c.bs_active_np = -1; }
        } restore{c};
        double t = *time, h = h0;
        int count = 0;
        // mxx_sync (mercury6_2.for:7556-7570): the bodies before Small body j
        // are integrated by mdt_bs1 to j's epoch, then j joins
        for (int j = c.nbig; j < c.n; ++j) {
            c.bs_active_np = j - c.nbig;
            while (std::fabs(t - epoch[j]) > epoch_epsilon(t, epoch[j])) {
                h = clipped_step(t, epoch[j], h, dtout);
                double hdid = 0.0;
                int64_t rejected = 0;
                bs_step_once(t, &h, &hdid, tol, &rejected);
                t = t + hdid;
                ++count;
            }
        }
        *time = t;
        if (steps) *steps = count;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_set_event_capacity(int cap) {
    if (cap < 0) return 1;
    g_event_cap = cap;
    return 0;
}

int mercury_b200_set_step_reduce(mercury_b200_reduce_fn fn, void* user) {
    g_step_reduce = fn;
    g_step_reduce_user = user;
    return 0;
}

int mercury_b200_set_launch(int particle_threads, int steps_per_launch) {
    Context& c = ctx();
    if (particle_threads > 0) {
        if (particle_threads % 32 != 0 || particle_threads > 1024) return 1;
        c.particle_threads = particle_threads;
    }
    if (steps_per_launch >= 0) c.steps_per_launch = steps_per_launch;
    return 0;
}

}  // extern "C"

// Host-side state of the library: one device context, as the reference's
// single global context (mercury_cuda.cu:16-33), plus the helpers every entry
// point uses (allocation, error reporting, layout kernels).
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "mvs.cuh"

namespace mb200 {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check(cudaError_t code, const char* what = nullptr) {
    if (code != cudaSuccess) {
        std::string msg = cudaGetErrorString(code);
        if (what) msg = std::string(what) + ": " + msg;
        throw CudaError(msg);
    }
}

// Host-to-device copy ordered on `stream` (the library's streams do not
// synchronize with the legacy default stream, and a plain cudaMemcpy from
// pageable memory may return before its data lands); returns once it is done.
inline void h2d(void* dst, const void* src, size_t bytes, cudaStream_t stream, const char* what = "upload") {
    if (bytes == 0) return;
    check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream), what);
    check(cudaStreamSynchronize(stream), what);
}

// Growable device array.
template <class T> struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void reserve(size_t count) {
        if (count <= n) return;
        release();
        check(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * (count ? count : 1)), "cudaMalloc");
        n = count;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct Context {
    int algorithm = 2;
    // system
    int n = 0, nbig = 0, np = 0, npcap = 0;
    // Bodies [0, nsplit) live in the "big" arrays, [nsplit, n) in the particle
    // slots. MVS splits at nbig; RADAU/BS also keep every massive Small body
    // (semi-active, it acts on the Big bodies) in the big arrays.
    int nsplit = 0, nmass = 0;
    int pn = 0, ngflag = 0;
    double jcen[3] = {0, 0, 0};
    std::vector<double> m_host;
    // Big bodies: masses, radii, ngf rows, double-buffered state
    DBuf<double> mbig, rcebig, rphysbig, ngfbig;
    DBuf<double> bigstate[2];   // [9][nbig]: x(3) v(3) a(3)
    // particles
    DBuf<double> pstate[2];     // [9][npcap]
    // per-slot constants [PCONST_ROWS][npcap]: m, rce, rphys, ngf(5), rcrit; double-buffered with
    // perm (slot -> particle index) so that the slots can be re-ordered
    DBuf<double> pconst[2];
    DBuf<int> perm[2];
    DBuf<int> inv;              // particle index -> slot
    int kc = 0;                 // constants/perm buffer in use
    DBuf<int> order_bucket, order_hist;
    DBuf<double> snap_const;
    DBuf<int> snap_perm;
    int cur = 0;
    bool reset = true;
    bool stepped = false;
    // MVS tables
    DBuf<double> tab, detail;
    // RA15: B, E, G and predictor scratch of the massive set ([21][nsplit],
    // [6][nsplit]), B and E of the particle slots ([21][npcap]), the per-node
    // force table, max |b7| and the force entry's output ([3][nsplit] then
    // [3][npcap]); screen boxes of the adaptive integrators ([nbig-1][4])
    DBuf<double> ra_bb, ra_be, ra_bg, ra_bpx, ra_pb, ra_pe, ftab, force_out, boxes;
    DBuf<unsigned long long> ra_max;
    // output corrector scratch: Big [9][nbig], particles [6][npcap]
    DBuf<double> corr_big, corr_part;
    DBuf<double> energy_scr;         // mxx_en: per-body pair sums, then e and l2
    DBuf<int> ej_ids;                // mxx_ejec screen: count, then the ids found
    // Bulirsch-Stoer: massive-set scratch, per-level candidate states, per-level
    // error maxima and force-fault words
    DBuf<double> bs_scr, bs_bcand, bs_pcand, bs_ptab;
    DBuf<unsigned long long> bs_errs;
    DBuf<DeviceStatus> bs_lvst;
    // HYBRID: rcrit of the massive set, the massive set after the first solar
    // drift, the three force/begin rows, dh2h velocity shifts of the previous
    // and current states, members' packed rows, encounter pairs and member ids
    DBuf<double> rcritbig, hy_scr, hy_tab, hy_off, hy_packed;
    DBuf<int2> hy_pairs;
    DBuf<int> hy_ids;
    std::vector<int> hy_members;
    bool hy_begun = false;
    // compact encounter subsystem: BS2 with mfo_hkce; massive members in the big
    // arrays, massless members in particle slots; per-body pair lists in pair
    // order (subsystem indices)
    bool encounter = false;
    DBuf<int> adj_off;
    DBuf<int2> adj;
    // BS steps integrate only the particles with index < bs_active_np (-1: all)
    int bs_active_np = -1;
    // with tangent set (HYBRID adjoint), every accepted BS2 step also advances
    // the massless members' 6x6 Jacobians tg [36][npcap]
    bool tangent = false;
    DBuf<double> tg;
    // events
    DBuf<MercuryEvent> events;
    DBuf<int> event_step;
    DBuf<EncounterCandidate> cands;
    DBuf<DeviceStatus> status;
    DeviceStatus* status_host = nullptr;
    std::vector<MercuryEvent> host_events;
    std::vector<int> host_steps;
    std::vector<uint32_t> event_order;   // last advance: host_events in (step, min, max) order
    // the last fused run's records in (step, min, max) order on the device
    // (ev_device of them; 0: the records are in host_events)
    DBuf<MercuryEvent> ev_sorted;
    DBuf<int> ev_sorted_step;
    int ev_device = 0;
    double event_rate = 0.0;             // most event records per step seen by an advance of this system
    int pair_events = 0;
    // staging
    DBuf<double> transfer;
    DBuf<double> snapshot;
    // upload: the host arrays as they arrive ([3n] x, [3n] v, [n] m, rce,
    // rphys, [5n] ngf), the slot-order sort's keys, indices and scratch, and
    // a page-locked host area for copies from and to pageable host arrays
    DBuf<double> stage;
    DBuf<char> order_scratch;
    char* pinned = nullptr;
    size_t pinned_n = 0;
    void reserve_pinned(size_t bytes) {
        if (bytes <= pinned_n) return;
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        pinned_n = 0;
        check(cudaMallocHost(reinterpret_cast<void**>(&pinned), bytes), "pinned staging");
        pinned_n = bytes;
    }
    // streams and timers
    cudaStream_t stream = nullptr, stream_big = nullptr, stream_ahead = nullptr, stream_out = nullptr;
    std::vector<cudaEvent_t> chunk_done;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> kt0, kt1;
    std::vector<int> launch_steps;   // steps of each launch of the last fused run
    std::vector<double> launch_ms;   // and each launch's particle-kernel time
    // mercury_b200_mvs_run's chunks: copied in, stepped; their work counters
    std::vector<cudaEvent_t> run_in, run_done;
    DBuf<int> run_tiles;
    float last_advance_ms = 0.0f;
    double last_particle_kernel_ms = 0.0;
    int last_particle_launches = 0;
    int last_kernel_launches = 0;   // every kernel of the last advance (all streams)
    int64_t nforces = 0;
    // timing events of the drop-in calls, and the kernels they launched
    cudaEvent_t d0 = nullptr, d1 = nullptr;
    int64_t dropin_launches = 0;
    // the central body's radius of the last drop-in events call (0: none yet),
    // and whether the last step screened for central impacts with it (for h)
    double dropin_rcen = 0.0, step_rcen = 0.0, step_h = 0.0, spec_rcen = 0.0;
    bool step_central = false;
    // the per-step MVS path's speculative next step: its Big-body and particle
    // states, force table, pair details, records and status (on the device and
    // read back into pinned memory with the first records), and whether one is
    // in flight for (spec_h, from buffer spec_from)
    DBuf<double> spec_big, spec_part, spec_tab, spec_detail;
    DBuf<MercuryEvent> spec_events;
    DBuf<int> spec_event_step;
    DBuf<DeviceStatus> spec_status;
    DeviceStatus* spec_status_host = nullptr;
    MercuryEvent* spec_head = nullptr;
    cudaEvent_t spec_done = nullptr, spec_ready = nullptr;
    bool spec_live = false;
    double spec_h = 0.0;
    int spec_from = -1;
    // the Big-body step after the speculative one (same h and radius), run
    // on a third stream beside the speculative step's particles: its state,
    // table rows, details, records and status
    DBuf<double> ah_state, ah_tab, ah_detail;
    DBuf<MercuryEvent> ah_events;
    DBuf<int> ah_event_step;
    DBuf<DeviceStatus> ah_status;
    cudaEvent_t ah_done = nullptr, spec_merged = nullptr;
    bool ah_live = false;
    double ah_h = 0.0, ah_rcen = 0.0;
    // the last step's status and first records are in status_host / ev_head
    // already (head_count records)
    bool head_ready = false;
    int head_count = 0;
    // the encounter subsystem's step control, read back once per block of
    // attempts
    EncCtl* enc_host = nullptr;
    // the encounter subsystem's step control on the device (two copies that
    // alternate between attempts), the end time of each accepted substep, and
    // the massive set's state at the start of the current attempt
    DBuf<EncCtl> enc_ctl;
    DBuf<double> enc_tstep;
    DBuf<double> enc_bpre;
    // the first records of a drop-in events call, read back with its status
    static constexpr int EVENT_HEAD = 1024;
    MercuryEvent* ev_head = nullptr;
    int particle_threads = 128;
    int steps_per_launch = 0;   // 0 = automatic

    double* pm() { return pconst[kc].p; }
    double* prce() { return pconst[kc].p + npcap; }
    double* prphys() { return pconst[kc].p + 2 * (size_t)npcap; }
    double* pngf() { return pconst[kc].p + 3 * (size_t)npcap; }
    int* permp() { return perm[kc].p; }
    int steps_since_order = 0;

    // The massive set's state buffer k as the MVS Big-body CTA reads it
    // (stride nsplit: Big bodies, then the massive Small bodies it holds).
    BigState big(int k) {
        BigState b;
        b.x = bigstate[k].p;
        b.v = bigstate[k].p + 3 * nsplit;
        b.a = bigstate[k].p + 6 * nsplit;
        return b;
    }
    void ensure_streams() {
        if (!stream) {
            check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
            check(cudaStreamCreateWithFlags(&stream_big, cudaStreamNonBlocking), "stream");
            check(cudaStreamCreateWithFlags(&stream_ahead, cudaStreamNonBlocking), "stream");
            check(cudaStreamCreateWithFlags(&stream_out, cudaStreamNonBlocking), "stream");
            check(cudaEventCreate(&t0), "event");
            check(cudaEventCreate(&t1), "event");
            check(cudaEventCreate(&d0), "event");
            check(cudaEventCreate(&d1), "event");
            check(cudaMallocHost(reinterpret_cast<void**>(&status_host), sizeof(DeviceStatus)), "pinned");
            check(cudaMallocHost(reinterpret_cast<void**>(&enc_host), sizeof(EncCtl)), "pinned");
            check(cudaMallocHost(reinterpret_cast<void**>(&ev_head), sizeof(MercuryEvent) * EVENT_HEAD), "pinned");
            check(cudaMallocHost(reinterpret_cast<void**>(&spec_head), sizeof(MercuryEvent) * EVENT_HEAD), "pinned");
            check(cudaMallocHost(reinterpret_cast<void**>(&spec_status_host), sizeof(DeviceStatus)), "pinned");
        }
    }
    void release_all() {
        DBuf<double>* bufs[] = {&mbig, &rcebig, &rphysbig, &ngfbig, &bigstate[0], &bigstate[1], &pstate[0],
                                &pstate[1], &pconst[0], &pconst[1], &tab, &detail, &transfer, &snapshot, &snap_const,
                                &ra_bb, &ra_be, &ra_bg, &ra_bpx, &ra_pb, &ra_pe, &ftab, &force_out, &boxes, &corr_big, &corr_part, &energy_scr,
                                &bs_scr, &bs_bcand, &bs_pcand, &bs_ptab, &rcritbig, &hy_scr, &hy_tab, &hy_off,
                                &hy_packed, &tg, &stage};
        for (auto* b : bufs) b->release();
        order_scratch.release();
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        pinned_n = 0;
        DBuf<int>* ibufs[] = {&perm[0], &perm[1], &inv, &order_bucket, &order_hist, &snap_perm, &ej_ids, &run_tiles};
        for (auto* b : ibufs) b->release();
        ra_max.release();
        bs_errs.release();
        bs_lvst.release();
        enc_ctl.release();
        enc_tstep.release();
        enc_bpre.release();
        spec_big.release();
        spec_part.release();
        spec_tab.release();
        spec_detail.release();
        spec_events.release();
        spec_event_step.release();
        spec_status.release();
        ah_state.release();
        ah_tab.release();
        ah_detail.release();
        ah_events.release();
        ah_event_step.release();
        ah_status.release();
        ah_live = false;
        spec_live = false;
        head_ready = false;
        dropin_rcen = 0.0;
        step_central = false;
        hy_pairs.release();
        hy_ids.release();
        adj_off.release();
        adj.release();
        hy_members.clear();
        hy_begun = false;
        tangent = false;
        kc = 0;
        events.release();
        event_step.release();
        cands.release();
        status.release();
        ev_sorted.release();
        ev_sorted_step.release();
        ev_device = 0;
        host_events.clear();
        host_steps.clear();
        event_order.clear();
        event_rate = 0.0;
        n = nbig = np = npcap = 0;
        stepped = false;
        reset = true;
    }
};

Context& ctx();
int active_context();   // 0: the resident system, 1: the encounter subsystem

// Layout kernels between the host's interleaved rows and the device SoA.
void scatter_rows(const double* rows, int n, int comps, int nbig, double* big, int big_stride, double* part,
                  int part_stride, const int* inv, cudaStream_t s);
void gather_rows(double* rows, int n, int comps, int nbig, const double* big, int big_stride, const double* part,
                 int part_stride, const int* inv, cudaStream_t s);

int report(const std::exception& e);

// One array of a host <-> device transfer: a host array (pageable or
// page-locked) and its device range.
struct HostSpan {
    void* dev;
    void* host;
    size_t bytes;
};
// True for page-locked host memory (cudaMallocHost, cudaHostAlloc, cudaHostRegister).
bool host_pinned(const void* p);
// Copy every span host -> device (copy_in) or device -> host (copy_out) on
// `stream`, returning when the data has landed (copy_in with sync false
// returns once the copies are queued; the host arrays and the stage must
// then stay untouched until the stream passes them). Page-locked host arrays are
// copied directly by DMA; pageable ones go through the context's page-locked
// area, which the host's cores fill or empty in parallel.
void copy_in(const std::vector<HostSpan>& spans, cudaStream_t stream, bool sync = true);
void copy_out(const std::vector<HostSpan>& spans, cudaStream_t stream);

}  // namespace mb200

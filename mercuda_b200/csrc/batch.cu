// Batched MVS systems: host orchestration of the extension entry points in
// include/mercury_b200.h (mercury_b200_batch_*). The reference integrates one
// system per process; these calls advance thousands of independent systems,
// each with its own Big bodies, particle count and step, in one pipelined run:
//
//   stream_big: Big-body CTAs of chunk c (every system) -> tables set c % 2
//   stream:     particles of chunk c (one launch over every system's tiles),
//               classification of its encounter candidates
//
// The chunk loop of a run is captured once into a CUDA graph and replayed for
// later runs of the same shape. The launch shape (steps per launch and the
// particle kernel's CTA size) is chosen by timing short trial runs before the
// first run (tune).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "../../include/mercury_b200.h"
#include "context.cuh"
#include "mvs.cuh"

namespace mb200 {
namespace {

constexpr int BATCH_MAX_NBIG = 32;

struct Batch {
    int nsys = 0, nbody = 0, npcap = 0, ntiles = 0, max_nbig = 1, K = 31;
    std::vector<int> body_off, nbig, np, first_slot, big_off;
    std::vector<double> h, mu;
    std::vector<BatchSys> sys;
    DBuf<BatchSys> d_sys;
    DBuf<BatchTile> d_tiles;
    DBuf<MvsBigArgs> d_proto;
    DBuf<double> bigbuf[2];          // per system [9][nbig] at 9 * big_off
    DBuf<double> bm, brce, brphys;   // per system [nbig] at big_off
    DBuf<double> pstate[2];          // [9][npcap]
    DBuf<double> prce, prphys;
    DBuf<int> plocal;
    DBuf<double> tab[2], det[2];
    size_t tab_size = 0, det_size = 0;
    DBuf<MercuryEvent> events;
    DBuf<int> event_step, event_sys;
    DBuf<EncounterCandidate> cands;
    DBuf<DeviceStatus> status;
    DeviceStatus* status_host = nullptr;
    DBuf<double> snap;
    int cur = 0;
    bool reset = true;
    int threads = 0;                 // 0: tune on the first run
    int tuned_K = 31, tuned_threads = 128;
    int forced_threads = 0, forced_K = 0, use_graph = 1;
    cudaStream_t stream = nullptr, stream_big = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> big_done, part_done;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::tuple<int, int, int, int, int, double, long> graph_key{};
    long epoch = 0;                  // bumped whenever a buffer is reallocated
    float last_ms = 0.0f;
    int last_launches = 0;
    std::vector<MercuryEvent> host_events;
    std::vector<int> host_sys, host_step;

    void release() {
        DBuf<double>* d[] = {&bigbuf[0], &bigbuf[1], &bm, &brce, &brphys, &pstate[0], &pstate[1],
                             &prce, &prphys, &tab[0], &tab[1], &det[0], &det[1], &snap};
        for (auto* b : d) b->release();
        d_sys.release();
        d_tiles.release();
        d_proto.release();
        plocal.release();
        events.release();
        event_step.release();
        event_sys.release();
        cands.release();
        status.release();
        drop_graph();
        nsys = nbody = npcap = ntiles = 0;
        host_events.clear();
        host_sys.clear();
        host_step.clear();
        ++epoch;
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void ensure_streams() {
        if (stream) return;
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&stream_big, cudaStreamNonBlocking), "stream");
        check(cudaEventCreate(&t0), "event");
        check(cudaEventCreate(&t1), "event");
        check(cudaMallocHost(reinterpret_cast<void**>(&status_host), sizeof(DeviceStatus)), "pinned");
    }
    void ensure_chunk_events(int n) {
        while ((int)big_done.size() < n) {
            cudaEvent_t a, b;
            check(cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "event");
            check(cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "event");
            big_done.push_back(a);
            part_done.push_back(b);
        }
    }
};

Batch& batch() {
    static Batch b;
    return b;
}

__global__ void batch_layout_kernel(const double* rows, int n, int comps, const int* dst_index, double* dst,
                                    int stride) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int d = dst_index[j];
    if (d < 0) return;
    for (int c = 0; c < comps; ++c) dst[(size_t)c * stride + d] = rows[(size_t)j * comps + c];
}

// Table and detail offsets of every system for K steps per chunk, and the
// sizes of one set.
void layout_tables(Batch& B, int K) {
    size_t t = 0, d = 0;
    for (int s = 0; s < B.nsys; ++s) {
        const int nb = B.nbig[s] - 1;
        B.sys[s].tab_off = (int)t;
        B.sys[s].det_off = (int)d;
        t += (size_t)(K + 1) * tab_stride(nb);
        d += (size_t)K * std::max(1, nb) * TAB_DETAIL;
    }
    if (t > (size_t)INT32_MAX || d > (size_t)INT32_MAX) throw std::runtime_error("batched tables too large");
    B.tab_size = t;
    B.det_size = d;
    for (int k = 0; k < 2; ++k) {
        const size_t n0 = B.tab[k].n, n1 = B.det[k].n;
        B.tab[k].reserve(t);
        B.det[k].reserve(d);
        if (B.tab[k].n != n0 || B.det[k].n != n1) ++B.epoch;
    }
    B.K = K;
    h2d(B.d_sys.p, B.sys.data(), sizeof(BatchSys) * B.nsys, B.stream);
}

BatchBigArgs big_chunk(Batch& B, int ch, int ks, int reset, int central, int s0, double rcen) {
    BatchBigArgs a{};
    a.proto = B.d_proto.p;
    a.sys = B.d_sys.p;
    a.flip = ((B.cur + ch) & 1) ? 1 : 0;
    a.nsteps = ks;
    a.reset = reset;
    a.central = central;
    a.step0 = s0;
    a.rcen = rcen;
    a.tab = B.tab[ch & 1].p;
    a.detail = B.det[ch & 1].p;
    a.events = B.events.p;
    a.event_step = B.event_step.p;
    a.event_sys = B.event_sys.p;
    a.event_cap = (int)B.events.n;
    a.status = B.status.p;
    return a;
}

BatchParticleArgs particle_chunk(Batch& B, int ch, int ks, int reset, int central, int s0, double rcen) {
    BatchParticleArgs a{};
    a.ntiles = B.ntiles;
    a.npcap = B.npcap;
    a.nsteps = ks;
    a.reset = reset;
    a.central = central;
    a.step0 = s0;
    a.rcen = rcen;
    a.sys = B.d_sys.p;
    a.tiles = B.d_tiles.p;
    const int in = (B.cur + ch) & 1;
    a.xin = B.pstate[in].p;
    a.xout = B.pstate[1 - in].p;
    a.rce = B.prce.p;
    a.rphys = B.prphys.p;
    a.local = B.plocal.p;
    a.tab = B.tab[ch & 1].p;
    a.detail = B.det[ch & 1].p;
    a.events = B.events.p;
    a.event_step = B.event_step.p;
    a.event_sys = B.event_sys.p;
    a.event_cap = (int)B.events.n;
    a.cands = B.cands.p;
    a.cand_cap = (int)B.cands.n;
    a.status = B.status.p;
    return a;
}

// The chunk loop of one run, enqueued on the two streams (also what a graph
// captures). Returns the number of kernels launched.
int enqueue_run(Batch& B, int nsteps, double rcen, int reset0, int central) {
    const int K = B.K, nchunks = (nsteps + K - 1) / K;
    int launches = 0;
    check(cudaMemsetAsync(B.status.p, 0, sizeof(DeviceStatus), B.stream), "memset");
    check(cudaEventRecord(B.big_done[0], B.stream), "event");  // fork point
    check(cudaStreamWaitEvent(B.stream_big, B.big_done[0], 0), "wait");
    for (int ch = 0; ch < nchunks; ++ch) {
        const int s0 = ch * K, ks = std::min(K, nsteps - s0);
        const int reset = (ch == 0 && reset0) ? 1 : 0;
        // the table set of this chunk is free once chunk ch - 2 was classified
        if (ch >= 2) check(cudaStreamWaitEvent(B.stream_big, B.part_done[ch - 2], 0), "wait");
        launch_mvs_big_batch(big_chunk(B, ch, ks, reset, central, s0, rcen), B.nsys, B.max_nbig, B.stream_big);
        ++launches;
        check(cudaEventRecord(B.big_done[ch], B.stream_big), "event");
        check(cudaStreamWaitEvent(B.stream, B.big_done[ch], 0), "wait");
        if (B.ntiles > 0) {
            check(cudaMemsetAsync(&B.status.p->next_tile, 0, sizeof(int), B.stream), "memset");
            const BatchParticleArgs pa = particle_chunk(B, ch, ks, reset, central, s0, rcen);
            launch_mvs_particles_batch(pa, B.stream, B.threads);
            launch_classify_batch(pa, B.stream);
            check(cudaMemsetAsync(&B.status.p->cands, 0, sizeof(int), B.stream), "memset");
            launches += 2;
        }
        check(cudaEventRecord(B.part_done[ch], B.stream), "event");
    }
    // join the Big-body stream
    check(cudaStreamWaitEvent(B.stream, B.big_done[nchunks - 1], 0), "wait");
    return launches;
}

// The launch shape of a batch: for every steps-per-launch K (8, 16, 31, 64)
// and particle CTA size (64, 128, 256) a short pipelined trial run of two
// chunks (Big-body CTAs on their stream ahead of the particle launches, as
// the real runs make them), timed with CUDA events; the fastest time per step
// wins. The trials start from the batch's state and it is restored after
// them (the snapshot), so tuning advances nothing. A forced CTA size or K
// (mercury_b200_batch_set) limits the search to it; the choice is kept and
// reported by mercury_b200_batch_timing.
void tune(Batch& B, double rcen, int nsteps) {
    std::vector<int> Ks = {8, 16, 31, 64};
    std::vector<int> Ts = {64, 128, 256};
    if (B.forced_K > 0) Ks = {B.forced_K};
    if (B.forced_threads > 0) Ts = {B.forced_threads};
    for (int& k : Ks) k = std::max(1, std::min(k, nsteps));
    std::sort(Ks.begin(), Ks.end());
    Ks.erase(std::unique(Ks.begin(), Ks.end()), Ks.end());
    B.threads = Ts[0];
    B.tuned_K = Ks[0];
    if (B.ntiles == 0 || (Ks.size() == 1 && Ts.size() == 1)) return;
    const size_t bigs = B.bm.n;
    auto copy = [&](void* d, const void* src, size_t bytes) {
        check(cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, B.stream), "tune");
    };
    copy(B.snap.p, B.pstate[B.cur].p, sizeof(double) * 9 * B.npcap);
    copy(B.snap.p + 9 * (size_t)B.npcap, B.bigbuf[B.cur].p, sizeof(double) * 9 * bigs);
    B.ensure_chunk_events(2);
    double best = 1e300;
    for (int K : Ks) {
        layout_tables(B, K);
        const int steps = std::min(nsteps, 2 * K);
        for (int threads : Ts) {
            B.threads = threads;
            check(cudaEventRecord(B.t0, B.stream), "event");
            enqueue_run(B, steps, rcen, B.reset ? 1 : 0, 1);
            check(cudaEventRecord(B.t1, B.stream), "event");
            check(cudaEventSynchronize(B.t1), "tune");
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, B.t0, B.t1), "tune");
            const double per_step = ms / steps;
            if (per_step < best) {
                best = per_step;
                B.tuned_K = K;
                B.tuned_threads = threads;
            }
            copy(B.pstate[B.cur].p, B.snap.p, sizeof(double) * 9 * B.npcap);
            copy(B.bigbuf[B.cur].p, B.snap.p + 9 * (size_t)B.npcap, sizeof(double) * 9 * bigs);
        }
    }
    B.threads = B.tuned_threads;
    check(cudaGetLastError(), "tune");
}

void sort_batch_events(Batch& B) {
    const size_t n = B.host_events.size();
    std::vector<size_t> idx(n);
    for (size_t k = 0; k < n; ++k) idx[k] = k;
    auto key = [&](size_t k) {
        const MercuryEvent& e = B.host_events[k];
        return std::make_tuple(B.host_sys[k], B.host_step[k], std::min(e.i, e.j), std::max(e.i, e.j));
    };
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return key(a) < key(b); });
    std::vector<MercuryEvent> e(n);
    std::vector<int> sy(n), st(n);
    for (size_t k = 0; k < n; ++k) {
        e[k] = B.host_events[idx[k]];
        sy[k] = B.host_sys[idx[k]];
        st[k] = B.host_step[idx[k]];
    }
    B.host_events.swap(e);
    B.host_sys.swap(sy);
    B.host_step.swap(st);
}

}  // namespace
}  // namespace mb200

using namespace mb200;

extern "C" {

int mercury_b200_batch_upload(int nsys, const int* body_offset, const int* nbig, const double* h, const double* m,
                              const double* xx, const double* vv, const double* rce, const double* rphys) {
    Batch& B = batch();
    try {
        if (nsys < 1) throw std::runtime_error("batch needs at least one system");
        B.ensure_streams();
        B.release();
        B.nsys = nsys;
        B.body_off.assign(body_offset, body_offset + nsys + 1);
        B.nbody = B.body_off[nsys];
        B.nbig.assign(nbig, nbig + nsys);
        B.h.assign(h, h + nsys);
        B.np.resize(nsys);
        B.first_slot.resize(nsys);
        B.big_off.resize(nsys);
        B.mu.resize(nsys);
        B.sys.resize(nsys);
        B.max_nbig = 1;
        int slots = 0, bigs = 0;
        std::vector<BatchTile> tiles;
        for (int s = 0; s < nsys; ++s) {
            const int n = B.body_off[s + 1] - B.body_off[s];
            if (n < 1 || B.nbig[s] < 1 || B.nbig[s] > n) throw std::runtime_error("invalid body counts of a system");
            if (B.nbig[s] > BATCH_MAX_NBIG) throw std::runtime_error("more than 32 Big bodies in a batched system");
            if (!(B.h[s] != 0.0) || !std::isfinite(B.h[s])) throw std::runtime_error("invalid step of a system");
            for (int j = B.body_off[s] + B.nbig[s]; j < B.body_off[s + 1]; ++j)
                if (m[j] != 0.0) throw std::runtime_error("batched systems take massless Small bodies only");
            B.np[s] = n - B.nbig[s];
            B.first_slot[s] = slots;
            B.big_off[s] = bigs;
            B.mu[s] = m[B.body_off[s]];
            B.max_nbig = std::max(B.max_nbig, B.nbig[s]);
            for (int t = 0; t < B.np[s]; t += 32) tiles.push_back(BatchTile{s, slots + t, std::min(32, B.np[s] - t), 0});
            slots += B.np[s];
            bigs += B.nbig[s];
            BatchSys& S = B.sys[s];
            S.mu = B.mu[s];
            S.h = B.h[s];
            S.nbig = B.nbig[s];
            S.nb = B.nbig[s] - 1;
            S.first_slot = B.first_slot[s];
            S.np = B.np[s];
        }
        B.npcap = std::max(1, slots);
        B.ntiles = (int)tiles.size();
        B.d_sys.reserve(nsys);
        B.d_tiles.reserve(std::max(1, B.ntiles));
        B.d_proto.reserve(nsys);
        for (int k = 0; k < 2; ++k) {
            B.bigbuf[k].reserve((size_t)9 * bigs);
            B.pstate[k].reserve((size_t)9 * B.npcap);
        }
        B.bm.reserve(bigs);
        B.brce.reserve(bigs);
        B.brphys.reserve(bigs);
        B.prce.reserve(B.npcap);
        B.prphys.reserve(B.npcap);
        B.plocal.reserve(B.npcap);
        B.events.reserve(std::max(4096, slots / 64));
        B.event_step.reserve(B.events.n);
        B.event_sys.reserve(B.events.n);
        B.cands.reserve(std::max(16384, slots / 2));
        B.status.reserve(1);
        B.snap.reserve((size_t)9 * B.npcap + (size_t)9 * bigs);
        if (B.ntiles)
            h2d(B.d_tiles.p, tiles.data(), sizeof(BatchTile) * B.ntiles, B.stream);
        // destination index of every body: Big rows at 9 * big_off + k (stride
        // nbig within the system) are written per component below; particles
        // go to their slot
        std::vector<int> slot_of(B.nbody, -1), local(B.npcap, 0);
        std::vector<double> hb(9 * (size_t)bigs, 0.0), hm(bigs), hrce(bigs), hrph(bigs);
        for (int s = 0; s < nsys; ++s) {
            const int o = B.body_off[s], nb = B.nbig[s];
            double* base = hb.data() + 9 * (size_t)B.big_off[s];
            for (int k = 0; k < nb; ++k) {
                for (int c = 0; c < 3; ++c) {
                    base[c * nb + k] = xx[3 * (size_t)(o + k) + c];
                    base[(3 + c) * nb + k] = vv[3 * (size_t)(o + k) + c];
                }
                hm[B.big_off[s] + k] = m[o + k];
                hrce[B.big_off[s] + k] = rce[o + k];
                hrph[B.big_off[s] + k] = rphys[o + k];
            }
            for (int q = 0; q < B.np[s]; ++q) {
                slot_of[o + nb + q] = B.first_slot[s] + q;
                local[B.first_slot[s] + q] = q;
            }
        }
        h2d(B.bigbuf[0].p, hb.data(), sizeof(double) * hb.size(), B.stream);
        check(cudaMemsetAsync(B.bigbuf[1].p, 0, sizeof(double) * hb.size(), B.stream), "upload");
        h2d(B.bm.p, hm.data(), sizeof(double) * bigs, B.stream);
        h2d(B.brce.p, hrce.data(), sizeof(double) * bigs, B.stream);
        h2d(B.brphys.p, hrph.data(), sizeof(double) * bigs, B.stream);
        h2d(B.plocal.p, local.data(), sizeof(int) * B.npcap, B.stream);
        // (on the stream of the layout kernels below, so that they run after)
        check(cudaMemsetAsync(B.pstate[0].p, 0, sizeof(double) * 9 * B.npcap, B.stream), "upload");
        check(cudaMemsetAsync(B.pstate[1].p, 0, sizeof(double) * 9 * B.npcap, B.stream), "upload");
        // particle rows through a device staging copy of the host arrays
        DBuf<double> stage;
        DBuf<int> dst;
        stage.reserve((size_t)3 * B.nbody);
        dst.reserve(B.nbody);
        h2d(dst.p, slot_of.data(), sizeof(int) * B.nbody, B.stream);
        const int blocks = (B.nbody + 255) / 256;
        for (int part = 0; part < 2; ++part) {
            h2d(stage.p, part ? vv : xx, sizeof(double) * 3 * B.nbody, B.stream);
            batch_layout_kernel<<<blocks, 256, 0, B.stream>>>(stage.p, B.nbody, 3, dst.p,
                                                               B.pstate[0].p + (size_t)3 * part * B.npcap, B.npcap);
            check(cudaStreamSynchronize(B.stream), "upload");
        }
        const double* scal[2] = {rce, rphys};
        double* sdst[2] = {B.prce.p, B.prphys.p};
        for (int q = 0; q < 2; ++q) {
            h2d(stage.p, scal[q], sizeof(double) * B.nbody, B.stream);
            batch_layout_kernel<<<blocks, 256, 0, B.stream>>>(stage.p, B.nbody, 1, dst.p, sdst[q], B.npcap);
            check(cudaStreamSynchronize(B.stream), "upload");
        }
        check(cudaGetLastError(), "upload");
        stage.release();
        dst.release();
        // per-system Big-body argument templates (in = set 0, out = set 1)
        std::vector<MvsBigArgs> proto(nsys);
        for (int s = 0; s < nsys; ++s) {
            MvsBigArgs& a = proto[s];
            a = MvsBigArgs{};
            a.nbig = B.nbig[s];
            a.h = B.h[s];
            a.m = B.bm.p + B.big_off[s];
            a.rce = B.brce.p + B.big_off[s];
            a.rphys = B.brphys.p + B.big_off[s];
            for (int k = 0; k < 2; ++k) {
                BigState& st = k ? a.out : a.in;
                double* base = B.bigbuf[k].p + 9 * (size_t)B.big_off[s];
                st.x = base;
                st.v = base + 3 * B.nbig[s];
                st.a = base + 6 * B.nbig[s];
            }
        }
        h2d(B.d_proto.p, proto.data(), sizeof(MvsBigArgs) * nsys, B.stream);
        layout_tables(B, B.forced_K > 0 ? B.forced_K : 31);
        B.cur = 0;
        B.reset = true;
        B.threads = 0;
        B.tuned_K = 31;
        B.tuned_threads = 128;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_batch_advance(double time, int nsteps, double rcen, int* nevents) {
    Batch& B = batch();
    try {
        if (B.nsys < 1) throw std::runtime_error("no batch uploaded");
        if (nsteps < 1) throw std::runtime_error("nsteps must be positive");
        if (B.threads == 0) tune(B, rcen, nsteps);
        int K = B.forced_K > 0 ? B.forced_K : B.tuned_K;
        K = std::max(1, std::min(K, nsteps));
        if (K != B.K) layout_tables(B, K);
        const int nchunks = (nsteps + K - 1) / K;
        B.ensure_chunk_events(std::max(2, nchunks));
        const int reset0 = B.reset ? 1 : 0;
        // starting state, for a redo after an event-buffer overflow
        const size_t bigs = B.bm.n;
        auto copy = [&](void* d, const void* s, size_t bytes) {
            check(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, B.stream), "snapshot");
        };
        copy(B.snap.p, B.pstate[B.cur].p, sizeof(double) * 9 * B.npcap);
        copy(B.snap.p + 9 * (size_t)B.npcap, B.bigbuf[B.cur].p, sizeof(double) * 9 * bigs);
        int launches = 0;
        for (int attempt = 0;; ++attempt) {
            const auto key = std::make_tuple(nsteps, K, B.threads, reset0, B.cur, rcen, B.epoch);
            check(cudaEventRecord(B.t0, B.stream), "event");
            if (B.use_graph) {
                if (!B.exec || B.graph_key != key) {
                    B.drop_graph();
                    check(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal), "capture");
                    launches = enqueue_run(B, nsteps, rcen, reset0, 1);
                    check(cudaStreamEndCapture(B.stream, &B.graph), "capture");
                    check(cudaGraphInstantiate(&B.exec, B.graph, 0), "graph");
                    B.graph_key = key;
                }
                launches = 1 + (B.ntiles > 0 ? 2 : 0);
                launches = nchunks * launches;
                check(cudaGraphLaunch(B.exec, B.stream), "graph");
            } else {
                launches = enqueue_run(B, nsteps, rcen, reset0, 1);
            }
            check(cudaEventRecord(B.t1, B.stream), "event");
            check(cudaMemcpyAsync(B.status_host, B.status.p, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, B.stream),
                  "status");
            check(cudaStreamSynchronize(B.stream), "advance");
            check(cudaGetLastError(), "advance");
            if (B.status_host->fault) throw std::runtime_error("MVS force failed");
            if (!B.status_host->overflow) break;
            if (attempt > 8) throw std::runtime_error("event buffer growth failed");
            if (B.status_host->overflow & 1) {
                const size_t n = std::max(2 * B.events.n, (size_t)B.status_host->events + 1024);
                B.events.reserve(n);
                B.event_step.reserve(n);
                B.event_sys.reserve(n);
            }
            if (B.status_host->overflow & 2) B.cands.reserve(2 * B.cands.n + 4096);
            ++B.epoch;
            copy(B.pstate[B.cur].p, B.snap.p, sizeof(double) * 9 * B.npcap);
            copy(B.bigbuf[B.cur].p, B.snap.p + 9 * (size_t)B.npcap, sizeof(double) * 9 * bigs);
        }
        check(cudaEventElapsedTime(&B.last_ms, B.t0, B.t1), "timer");
        B.last_launches = launches;
        B.cur = (B.cur + nchunks) & 1;
        B.reset = false;
        const int nev = B.status_host->events;
        B.host_events.resize(nev);
        B.host_sys.resize(nev);
        B.host_step.resize(nev);
        if (nev) {
            check(cudaMemcpy(B.host_events.data(), B.events.p, sizeof(MercuryEvent) * nev, cudaMemcpyDeviceToHost),
                  "events");
            check(cudaMemcpy(B.host_sys.data(), B.event_sys.p, sizeof(int) * nev, cudaMemcpyDeviceToHost), "events");
            check(cudaMemcpy(B.host_step.data(), B.event_step.p, sizeof(int) * nev, cudaMemcpyDeviceToHost),
                  "events");
        }
        // absolute times on each system's own clock (time = time + h per step)
        std::map<int, std::vector<double>> tend;
        for (int k = 0; k < nev; ++k) {
            const int s = B.host_sys[k];
            auto it = tend.find(s);
            if (it == tend.end()) {
                std::vector<double> t(nsteps);
                double tt = time;
                for (int q = 0; q < nsteps; ++q) {
                    tt = tt + B.h[s];
                    t[q] = tt;
                }
                it = tend.emplace(s, std::move(t)).first;
            }
            MercuryEvent& e = B.host_events[k];
            const double te = it->second[B.host_step[k]];
            if (e.kind == EV_CENTRAL) e.time = te - B.h[s] + e.time;
            else e.time = e.time + te;
        }
        sort_batch_events(B);
        *nevents = nev;
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_batch_events(MercuryEvent* events, int* sys, int* steps, int cap) {
    Batch& B = batch();
    const int nev = (int)B.host_events.size();
    const int k = std::min(cap, nev);
    if (k > 0) {
        std::memcpy(events, B.host_events.data(), sizeof(MercuryEvent) * k);
        if (sys) std::memcpy(sys, B.host_sys.data(), sizeof(int) * k);
        if (steps) std::memcpy(steps, B.host_step.data(), sizeof(int) * k);
    }
    return nev;
}

int mercury_b200_batch_download(double* xx, double* vv) {
    Batch& B = batch();
    try {
        if (B.nsys < 1) throw std::runtime_error("no batch uploaded");
        const size_t bigs = B.bm.n;
        std::vector<double> hb(9 * bigs), hp(6 * (size_t)B.npcap);
        check(cudaMemcpy(hb.data(), B.bigbuf[B.cur].p, sizeof(double) * hb.size(), cudaMemcpyDeviceToHost),
              "download");
        check(cudaMemcpy(hp.data(), B.pstate[B.cur].p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost),
              "download");
        for (int s = 0; s < B.nsys; ++s) {
            const int o = B.body_off[s], nb = B.nbig[s];
            const double* base = hb.data() + 9 * (size_t)B.big_off[s];
            for (int k = 0; k < nb; ++k)
                for (int c = 0; c < 3; ++c) {
                    xx[3 * (size_t)(o + k) + c] = base[c * nb + k];
                    vv[3 * (size_t)(o + k) + c] = base[(3 + c) * nb + k];
                }
            for (int q = 0; q < B.np[s]; ++q) {
                const size_t slot = (size_t)B.first_slot[s] + q;
                for (int c = 0; c < 3; ++c) {
                    xx[3 * (size_t)(o + nb + q) + c] = hp[c * (size_t)B.npcap + slot];
                    vv[3 * (size_t)(o + nb + q) + c] = hp[(3 + c) * (size_t)B.npcap + slot];
                }
            }
        }
        return 0;
    } catch (const std::exception& e) {
        return report(e);
    }
}

int mercury_b200_batch_set(int threads, int steps_per_launch, int use_graph) {
    Batch& B = batch();
    if (threads > 0 && threads != 64 && threads != 128 && threads != 256) return 1;
    if (threads >= 0) {
        B.forced_threads = threads;
        B.threads = 0;   // tuned again (over K only when threads is forced)
    }
    if (steps_per_launch >= 0) {
        B.forced_K = std::min(steps_per_launch, 64);
        B.threads = 0;
    }
    if (use_graph >= 0) B.use_graph = use_graph ? 1 : 0;
    return 0;
}

int mercury_b200_batch_timing(double* ms, int* launches, int* threads, int* steps_per_launch) {
    Batch& B = batch();
    if (ms) *ms = B.last_ms;
    if (launches) *launches = B.last_launches;
    if (threads) *threads = B.threads;
    if (steps_per_launch) *steps_per_launch = B.K;
    return 0;
}

void mercury_b200_batch_free(void) { batch().release(); }

}  // extern "C"

// Serving many mesh jobs on one GPU.
//
// BAM's calibration loop issues one mesh job after another (Bam::bamrunner,
// Source/Bam.cpp:13424): each iteration builds a mesh, takes its P(k) and,
// in some iterations, its T-web.  Run one at a time, small meshes leave most
// of a B200 idle and pay several host round trips per job.  This file adds:
//
//   cam_batch_run  -- packs jobs of one shape into CUDA graphs: every job of
//                     a batch gets a slot (its own stream and buffers), the
//                     slots' work is captured once per shape as parallel
//                     branches of one graph, and later batches of that shape
//                     replay the graph after copying their particles into
//                     the slots.  One host synchronisation per batch.
//   cam_server_*   -- continuous batching: worker threads take queued jobs
//                     as soon as a worker and enough of the HBM budget are
//                     free, run single jobs on their own streams (their work
//                     overlaps on the GPU) and pack queued jobs of a common
//                     small shape into graph batches.  Latencies from
//                     submission to completion give p50/p99.
//
// A job gives the same result alone, in a batch and in the server mix: the
// kernels are deterministic and every slot has its own buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cam_internal.h"

namespace cam {
namespace {

constexpr int kMaxBatch = 32;   // jobs per graph in cam_batch_run
constexpr int kMaxGraphs = 16;  // cached graphs per runner (least recently used dropped)

size_t esize(int precision) { return precision == CAM_F64 ? 8 : 4; }

// Pinned host mirror of one job's device results, filled by device->host
// copies at the end of the job's stream work.
struct MirrorHead {
    unsigned long long stats[4];  // lost, max|w| bits, payload records, pad
    double sum[2];                // mesh sum, mean per cell
    unsigned long long tw[8];     // label counts 1..4, ties
};

struct Slot {
    cam_ctx *c = nullptr;
    unsigned char *pin = nullptr;
    size_t pin_bytes = 0;
    float *in[4] = {nullptr, nullptr, nullptr, nullptr};  // scratch of c
    uint64_t local_gen = 0;  // bumped when `pin` is reallocated
    uint64_t gen() const { return c->gen + local_gen; }
    size_t device_bytes() const { return c->used; }
    ~Slot()
    {
        if (!c) return;
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        if (pin) {
            std::lock_guard<std::mutex> lk(alloc_mutex());
            cudaFreeHost(pin);
        }
        cam_ctx_destroy(c);  // takes the allocation mutex itself
    }
};

bool want_pk(const cam_job_desc &d) { return d.pk.nbins > 0 || d.pk.ndel > 0.0; }

void validate_job(const cam_job_desc &d)
{
    for (int a = 0; a < 3; ++a) CAM_REQUIRE(d.grid.n[a] >= 1, CAM_E_INVAL, "grid size must be >= 1");
    CAM_REQUIRE(d.grid.n[0] == d.grid.n[1] && d.grid.n[1] == d.grid.n[2], CAM_E_UNSUPPORTED, "FFT stages need a cubic mesh");
    CAM_REQUIRE(d.precision == CAM_F32 || d.precision == CAM_F64, CAM_E_INVAL, "precision must be CAM_F32 or CAM_F64");
    CAM_REQUIRE(d.scheme >= CAM_NGP && d.scheme <= CAM_TSC, CAM_E_INVAL, "unknown mass assignment scheme");
    CAM_REQUIRE(d.parts.n >= 0 && (d.parts.n == 0 || (d.parts.x && d.parts.y && d.parts.z)), CAM_E_INVAL,
                "invalid particles");
    CAM_REQUIRE(d.parts.mem == CAM_MEM_HOST || d.parts.mem == CAM_MEM_DEVICE, CAM_E_INVAL, "invalid particle memory");
    if (want_pk(d))
        CAM_REQUIRE(d.pk.ndel > 0.0 && d.pk.nbins >= 0 && d.pk.scheme >= 0 && d.pk.scheme <= 2 &&
                        (d.pk.input_type == CAM_INPUT_DENSITY || d.pk.input_type == CAM_INPUT_DELTA),
                    CAM_E_INVAL, "invalid P(k) options");
    if (d.want_tweb)
        CAM_REQUIRE((d.tweb.input_type == CAM_INPUT_DENSITY || d.tweb.input_type == CAM_INPUT_DELTA) &&
                        (d.tweb.method == CAM_TWEB_FFT || d.tweb.method == CAM_TWEB_FD),
                    CAM_E_INVAL, "invalid T-web options");
}

// Upper estimate of the device bytes a job needs (staged inputs, payload at
// its bound, brick tables, mesh, spectrum, T-web components, labels), used
// for admission against the HBM budget.  The 5/4 covers the grow-only
// buffers' rounding.
size_t job_footprint(const cam_job_desc &d)
{
    const size_t n = (size_t)d.grid.n[0], np = (size_t)d.parts.n;
    const size_t es = esize(d.precision), ncell = n * n * n;
    const size_t nh = n * n * (n / 2) + n * n;
    size_t f = np * 16;
    f += np * (d.scheme == CAM_NGP ? 1 : 8) * 16;
    f += (ncell / 8192 + 4096) * ((size_t)kNumSMs * 4 + 32);
    f += ncell * es + nh * 2 * es;
    if (d.want_tweb) f += 6 * nh * 2 * es + ncell;
    return f / 4 * 5 + (32u << 20);
}

Slot *make_slot(int device)
{
    std::unique_ptr<Slot> s(new Slot);
    const int rc = cam_ctx_create(device, 0, &s->c);
    if (rc != CAM_OK) {
        s->c = nullptr;
        throw Error{rc, "cannot create a slot context"};
    }
    return s.release();
}

void ensure_slot(Slot &s, const cam_job_desc &d)
{
    const size_t np = (size_t)std::max<int64_t>(d.parts.n, 1);
    static const char *names[4] = {"slot.x", "slot.y", "slot.z", "slot.w"};
    const uint64_t g0 = s.c->gen;
    for (int a = 0; a < 4; ++a) s.in[a] = static_cast<float *>(scratch(s.c, names[a], np * sizeof(float)));
    // inputs are written on the batch's main stream: let a fresh allocation
    // (ordered on the slot's stream) complete first
    if (s.c->gen != g0) CAM_CUDA_TRY(cudaStreamSynchronize(s.c->stream));
    const int nb = want_pk(d) ? nbins_for(d.pk, d.grid.n[0]) : 0;
    const size_t need = sizeof(MirrorHead) + (size_t)nb * 3 * 8;
    if (s.pin_bytes < need) {
        std::lock_guard<std::mutex> lk(alloc_mutex());
        CAM_CUDA_TRY(cudaStreamSynchronize(s.c->stream));
        s.local_gen++;
        if (s.pin) cudaFreeHost(s.pin);
        s.pin = nullptr;
        s.pin_bytes = 0;
        // one allocation in practice: pinned allocation and release can
        // synchronise the device, so the mirror starts large (64 KB: about
        // 2,700 P(k) bins) rather than growing with each job's bin count
        const size_t bytes = std::max<size_t>(need, 64 << 10);
        CAM_CUDA_TRY(cudaMallocHost(&s.pin, bytes));
        s.pin_bytes = bytes;
    }
}

// Copies the job's particles into the slot's device buffers on `stream`.
void stage_inputs(Slot &s, const cam_job_desc &d, cudaStream_t stream)
{
    if (d.parts.n == 0) return;
    const cudaMemcpyKind k = d.parts.mem == CAM_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const float *src[4] = {d.parts.x, d.parts.y, d.parts.z, d.parts.w};
    for (int a = 0; a < 4; ++a)
        if (src[a]) CAM_CUDA_TRY(cudaMemcpyAsync(s.in[a], src[a], (size_t)d.parts.n * sizeof(float), k, stream));
}

// Enqueues one job on the slot's stream with no host round trip; results
// reach the slot's pinned mirror when the stream gets to the end.  Same
// stages and kernels as cam_job_run.
void enqueue_job(Slot &s, const cam_job_desc &d)
{
    cam_ctx *c = s.c;
    struct SyncFree {
        cam_ctx *c;
        explicit SyncFree(cam_ctx *cc) : c(cc) { c->sync_free = true; }
        ~SyncFree() { c->sync_free = false; }
    } guard(c);
    const cam_grid g = resolved_grid(d.grid);
    const int64_t n = g.n[0];
    FftPlan *plan = get_plan(c, n, d.precision);
    AssignOut out;
    out.precision = d.precision;
    out.mesh = scratch(c, "job.mesh", (size_t)n * n * n * esize(d.precision));
    out.d_sum = static_cast<double *>(scratch(c, "job.sum", 2 * sizeof(double)));
    assign_device(c, s.in[0], s.in[1], s.in[2], d.parts.w ? s.in[3] : nullptr, d.parts.n, g, d.scheme, out);
    Spectrum sp = alloc_spectrum(c, n, d.precision, "job.spec");
    const int nb = want_pk(d) ? nbins_for(d.pk, n) : 0;
    const PkDevice pkd = job_fft_pk(c, plan, out.mesh, out.d_sum + 1, sp, nb ? &d.pk : nullptr, nb, d.want_tweb != 0);
    if (d.want_tweb) tweb_device(c, plan, sp, g.L[0], out.d_sum + 1, d.tweb.input_type, d.tweb, nullptr, nullptr, nullptr);
    auto *m = reinterpret_cast<MirrorHead *>(s.pin);
    CAM_CUDA_TRY(cudaMemcpyAsync(m->stats, scratch(c, "asg.stats", 64), 3 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, c->stream));
    CAM_CUDA_TRY(cudaMemcpyAsync(m->sum, out.d_sum, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (d.want_tweb)
        CAM_CUDA_TRY(cudaMemcpyAsync(m->tw, scratch(c, "tw.cnt", 8 * sizeof(unsigned long long)),
                                     5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    if (nb) {
        double *pk = reinterpret_cast<double *>(s.pin + sizeof(MirrorHead));
        CAM_CUDA_TRY(cudaMemcpyAsync(pk, pkd.sums, (size_t)nb * 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                     c->stream));
        CAM_CUDA_TRY(cudaMemcpyAsync(pk + 2 * nb, pkd.modes, (size_t)nb * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, c->stream));
    }
}

// Fills the caller's result from the slot's mirror (after the stream work).
int collect_job(const Slot &s, const cam_job_desc &d, cam_job_result *r)
{
    const auto *m = reinterpret_cast<const MirrorHead *>(s.pin);
    if (d.parts.w && (unsigned)(m->stats[1] & 0xffffffffu) >= 0x7f800000u) return CAM_E_NONFINITE;
    const int64_t n = d.grid.n[0];
    r->assign.n_lost = (int64_t)m->stats[0];
    r->assign.n_in = d.parts.n - r->assign.n_lost;
    r->assign.sum_mesh = m->sum[0];
    if (want_pk(d)) {
        const int nb = nbins_for(d.pk, n);
        const double *pk = reinterpret_cast<const double *>(s.pin + sizeof(MirrorHead));
        const auto *md = reinterpret_cast<const unsigned long long *>(pk + 2 * nb);
        std::vector<double> sr(nb), ss(nb);
        std::vector<int64_t> mi(nb);
        for (int b = 0; b < nb; ++b) {
            sr[b] = pk[2 * b];
            ss[b] = pk[2 * b + 1];
            mi[b] = (int64_t)md[b];
        }
        const cam_grid g = resolved_grid(d.grid);
        finalize_pk(n, g.L[0], m->sum[0], d.pk, nb, sr.data(), ss.data(), mi.data(), r->pk, r->modes, r->kvector,
                    &r->pk_info);
    }
    if (d.want_tweb) {
        for (int a = 0; a < 4; ++a) r->tweb.counts[a] = (int64_t)m->tw[a];
        r->tweb.ties = (int64_t)m->tw[4];
        r->tweb.mean = m->sum[1];
    }
    return CAM_OK;
}

// Everything a job's captured work depends on besides the particle values.
std::string shape_key(const cam_job_desc &d)
{
    char k[512];
    snprintf(k, sizeof(k),
             "%lld,%lld,%lld|%lld|%d|%d|%d|%d|%.9g,%.9g,%.9g|%.9g,%.9g,%.9g|%.9g,%.9g,%.9g|%d,%d,%d,%d,%d,%.17g,%.17g|"
             "%d|%.9g,%.17g,%.17g,%d,%d",
             (long long)d.grid.n[0], (long long)d.grid.n[1], (long long)d.grid.n[2], (long long)d.parts.n,
             d.parts.w != nullptr, d.parts.mem, d.scheme, d.precision, d.grid.L[0], d.grid.L[1], d.grid.L[2],
             d.grid.d[0], d.grid.d[1], d.grid.d[2], d.grid.min[0], d.grid.min[1], d.grid.min[2], d.pk.scheme,
             d.pk.mas_correction, d.pk.sn_correction, d.pk.input_type, d.pk.nbins, d.pk.DeltaKmin, d.pk.ndel,
             d.want_tweb, d.tweb.smoothing_R, d.tweb.lambda_th, d.tweb.tie_band, d.tweb.input_type,
             d.tweb.method);
    return k;
}

struct GraphEntry {
    std::string key;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> gens;  // slot buffer generations at capture
    uint64_t last_use = 0;
};

}  // namespace

// Graph-packed execution of batches of same-shaped jobs.
struct BatchRunner {
    int device = 0;
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    std::vector<std::unique_ptr<Slot>> slots;
    std::vector<GraphEntry> graphs;
    std::unordered_map<std::string, int> seen;  // uncaptured runs per batch key
    uint64_t clock = 0;
    int64_t replays = 0;

    explicit BatchRunner(int dev) : device(dev)
    {
        CAM_CUDA_TRY(cudaSetDevice(dev));
        CAM_CUDA_TRY(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
        CAM_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    }
    ~BatchRunner()
    {
        cudaSetDevice(device);
        if (main) cudaStreamSynchronize(main);
        for (auto &g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        for (auto e : joins) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        slots.clear();
        if (main) cudaStreamDestroy(main);
    }

    size_t device_bytes() const
    {
        size_t b = 0;
        for (auto &s : slots) b += s->device_bytes();
        return b;
    }

    void ensure_slots(int B)
    {
        while ((int)slots.size() < B) {
            slots.emplace_back(make_slot(device));
            cudaEvent_t e;
            CAM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            joins.push_back(e);
        }
    }

    void fork_join(const cam_job_desc *jobs, int B)
    {
        CAM_CUDA_TRY(cudaEventRecord(fork, main));
        for (int j = 0; j < B; ++j) {
            Slot &s = *slots[j];
            CAM_CUDA_TRY(cudaStreamWaitEvent(s.c->stream, fork, 0));
            enqueue_job(s, jobs[j]);
            CAM_CUDA_TRY(cudaEventRecord(joins[j], s.c->stream));
            CAM_CUDA_TRY(cudaStreamWaitEvent(main, joins[j], 0));
        }
    }

    std::vector<uint64_t> gens(int B) const
    {
        std::vector<uint64_t> g(B);
        for (int j = 0; j < B; ++j) g[j] = slots[j]->gen();
        return g;
    }

    // Runs B jobs concurrently (one slot each) and fills res[] and rc[]
    // (per-job status).  Jobs of one shape are captured into a graph after
    // `capture_after` uncaptured runs of that batch (0 = never) and replayed
    // from then on; jobs of mixed shapes always run uncaptured.
    void run(const cam_job_desc *jobs, int B, cam_job_result *res, int *rc, int capture_after)
    {
        ensure_slots(B);
        for (int j = 0; j < B; ++j) ensure_slot(*slots[j], jobs[j]);
        const std::string key = std::to_string(B) + "#" + shape_key(jobs[0]);
        bool same = true;
        for (int j = 1; j < B && same; ++j) same = shape_key(jobs[j]) == shape_key(jobs[0]);
        if (!same) capture_after = 0;
        // A graph holds the addresses of the slot buffers it was captured
        // with: if any of them was reallocated since, drop the graph.
        GraphEntry *ge = nullptr;
        for (auto it = graphs.begin(); same && it != graphs.end(); ++it) {
            if (it->key != key) continue;
            if (it->gens == gens(B)) {
                ge = &*it;
            } else {
                cudaGraphExecDestroy(it->exec);
                graphs.erase(it);
                seen[key] = 0;
            }
            break;
        }
        for (int j = 0; j < B; ++j) stage_inputs(*slots[j], jobs[j], main);
        if (ge) {
            CAM_CUDA_TRY(cudaGraphLaunch(ge->exec, main));
            ge->last_use = ++clock;
            ++replays;
        } else {
            fork_join(jobs, B);
        }
        CAM_CUDA_TRY(cudaStreamSynchronize(main));
        for (int j = 0; j < B; ++j) rc[j] = collect_job(*slots[j], jobs[j], &res[j]);
        if (!ge && capture_after > 0 && ++seen[key] >= capture_after) capture(jobs, B, key);
    }

    void capture(const cam_job_desc *jobs, int B, const std::string &key)
    {
        // No allocation or free anywhere in the library while this thread
        // captures (allocations in other threads wait on the mutex).
        std::lock_guard<std::mutex> lk(alloc_mutex());
        for (int j = 0; j < B; ++j) slots[j]->c->capturing = true;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = false;
        if (cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            bool enq = true;
            try {
                fork_join(jobs, B);
            } catch (const Error &) {
                enq = false;
            }
            const cudaError_t e = cudaStreamEndCapture(main, &graph);
            ok = enq && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        }
        cudaGetLastError();
        if (graph) cudaGraphDestroy(graph);
        for (int j = 0; j < B; ++j) slots[j]->c->capturing = false;
        if (!ok) {
            if (exec) cudaGraphExecDestroy(exec);
            return;  // this shape stays on the uncaptured path
        }
        if ((int)graphs.size() >= kMaxGraphs) {
            auto it = std::min_element(graphs.begin(), graphs.end(),
                                       [](const GraphEntry &a, const GraphEntry &b) { return a.last_use < b.last_use; });
            cudaGraphExecDestroy(it->exec);
            graphs.erase(it);
        }
        graphs.push_back(GraphEntry{key, exec, gens(B), ++clock});
    }
};

void batch_destroy(void *batch) { delete static_cast<BatchRunner *>(batch); }

}  // namespace cam

using namespace cam;

// ---------------------------------------------------------------- server

struct cam_server {
    struct Job {
        uint64_t id;
        cam_job_desc desc;
        cam_job_result *res;
        std::chrono::steady_clock::time_point t_submit;
        size_t footprint;
        std::string shape;
        bool batchable;  // small mesh, no labels: may share a batch
        bool big;        // fills the GPU alone: at most max_big run at once
    };
    struct Worker {
        int index = 0;
        cam_ctx *ctx = nullptr;
        std::unique_ptr<BatchRunner> br;
        size_t held = 0;      // device bytes cached between jobs
        size_t inflight = 0;  // reservation of the running job(s)
        std::thread t;
    };
    int device = 0;
    size_t budget = 0;
    int max_batch = 16;
    int64_t small_n = 128;  // meshes up to 128^3 are packed into batches
    int max_big = 1;        // large jobs running at once (they contend for L2)
    int big_running = 0;
    // Large jobs run on one shared context (max_big == 1), so their
    // multi-GB buffers exist once instead of once per worker.
    cam_ctx *big_ctx = nullptr;
    size_t big_held = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job> queue;
    std::unordered_map<uint64_t, int> done;  // id -> final status (until read)
    int64_t n_running = 0;
    std::vector<double> lat_ms;
    uint64_t next_id = 1;
    size_t peak_reserved = 0;
    int64_t submitted = 0, completed = 0, failed = 0, batches = 0, batched_jobs = 0, replays = 0;
    std::string last_err;  // message of the most recent failed job
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::vector<cam_server_job_trace> trace;  // completed jobs, oldest first
    bool trim = false;     // the queue head does not fit: idle workers drop caches
    bool stop = false;
    std::vector<std::unique_ptr<Worker>> workers;

    size_t reserved() const
    {
        size_t r = big_held;
        for (auto &w : workers) r += w->held + w->inflight;
        return r;
    }

    void drop_cache(Worker &w)
    {
        w.br.reset();
        release_all(w.ctx);
        w.held = 0;
    }

    // Under `mu`: picks the oldest queued job that may start (a large job
    // waits while max_big large jobs run; smaller jobs may pass it) and, if
    // it is batchable, queued jobs of its own shape up to max_batch (their
    // graph is replayed), as far as the HBM budget allows.  Jobs of distinct
    // shapes run one per worker: batched together they would wait for the
    // slowest of them and gain no graph.
    bool admit(Worker &w, std::vector<Job> &take)
    {
        size_t h = queue.size();
        for (size_t i = 0; i < queue.size() && i < 1024; ++i)
            if (!queue[i].big || big_running < max_big) {
                h = i;
                break;
            }
        if (h == queue.size()) return false;
        const Job &hd = queue[h];
        std::vector<size_t> pick{h};
        if (hd.batchable)
            for (size_t i = h + 1; i < queue.size() && (int)pick.size() < max_batch; ++i)
                if (queue[i].batchable && queue[i].shape == hd.shape) pick.push_back(i);
        size_t need = 0;
        for (size_t i : pick) need += queue[i].footprint;
        const size_t r = reserved();
        while (pick.size() > 1 && r + need > budget) {
            need -= queue[pick.back()].footprint;
            pick.pop_back();
        }
        // a large job reuses the shared context's cached buffers
        if (hd.big) need = need > big_held ? need - big_held : 0;
        if (r + need > budget) {
            if (w.held > 0 && r - w.held + need <= budget) {
                drop_cache(w);
            } else {
                if (!trim) {
                    trim = true;
                    cv_work.notify_all();
                }
                return false;
            }
        }
        for (auto it = pick.rbegin(); it != pick.rend(); ++it) {
            take.push_back(queue[*it]);
            queue.erase(queue.begin() + (long)*it);
        }
        std::reverse(take.begin(), take.end());
        for (auto &j : take) big_running += j.big;
        w.inflight = need;
        n_running += (int64_t)take.size();
        peak_reserved = std::max(peak_reserved, reserved());
        trim = false;
        return true;
    }

    void worker(Worker &w)
    {
        cudaSetDevice(device);
        for (;;) {
            std::vector<Job> take;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (trim && w.held > 0) drop_cache(w);
                    if (trim && big_running == 0 && big_held > 0) {
                        release_all(big_ctx);
                        big_held = 0;
                    }
                    if (!queue.empty() && admit(w, take)) break;
                    if (stop && queue.empty()) break;
                    cv_work.wait(lk);
                }
                if (take.empty()) break;
            }
            std::vector<int> rcs(take.size(), CAM_OK);
            int64_t rp = 0;
            std::string msg;
            const auto t_start = std::chrono::steady_clock::now();
            try {
                if (take.size() == 1) {
                    cam_ctx *c = take[0].big ? big_ctx : w.ctx;
                    rcs[0] = cam_job_run(c, &take[0].desc, take[0].res);
                    if (rcs[0] != CAM_OK) msg = cam_last_error(c);
                } else {
                    if (!w.br) w.br.reset(new BatchRunner(device));
                    std::vector<cam_job_desc> d(take.size());
                    std::vector<cam_job_result> r(take.size());
                    for (size_t i = 0; i < take.size(); ++i) {
                        d[i] = take[i].desc;
                        r[i] = *take[i].res;
                    }
                    const int64_t before = w.br->replays;
                    w.br->run(d.data(), (int)take.size(), r.data(), rcs.data(),
                              (int)take.size() == max_batch ? 1 : 2);
                    rp = w.br->replays - before;
                    for (size_t i = 0; i < take.size(); ++i) {
                        *take[i].res = r[i];
                        if (rcs[i] != CAM_OK) msg = "a particle weight is NaN or infinite";
                    }
                }
            } catch (const Error &e) {
                for (auto &rc : rcs) rc = e.code;
                msg = e.msg;
            } catch (...) {
                for (auto &rc : rcs) rc = CAM_E_CUDA;
                msg = "unexpected exception";
            }
            const auto now = std::chrono::steady_clock::now();
            {
                std::lock_guard<std::mutex> lk(mu);
                w.inflight = 0;
                w.held = w.ctx->used + (w.br ? w.br->device_bytes() : 0);
                if (take.size() == 1 && take[0].big) big_held = big_ctx->used;
                n_running -= (int64_t)take.size();
                for (auto &j : take) big_running -= j.big;
                if (!msg.empty()) last_err = msg;
                auto since = [&](std::chrono::steady_clock::time_point t) {
                    return std::chrono::duration<double, std::milli>(t - t0).count();
                };
                for (size_t i = 0; i < take.size(); ++i) {
                    const double ms = std::chrono::duration<double, std::milli>(now - take[i].t_submit).count();
                    done[take[i].id] = rcs[i];
                    if (trace.size() >= (1u << 20)) trace.erase(trace.begin(), trace.begin() + (1u << 19));
                    trace.push_back(cam_server_job_trace{take[i].id, since(take[i].t_submit), since(t_start), since(now),
                                                         w.index, (int)take.size(), rcs[i], take[i].big ? 1 : 0});
                    if (lat_ms.size() >= (1u << 22)) lat_ms.erase(lat_ms.begin(), lat_ms.begin() + (1u << 21));
                    lat_ms.push_back(ms);
                    ++completed;
                    if (rcs[i] != CAM_OK) ++failed;
                }
                if (take.size() > 1) {
                    ++batches;
                    batched_jobs += (int64_t)take.size();
                    replays += rp;
                }
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }
};

extern "C" {

int cam_batch_run(cam_ctx *ctx, const cam_job_desc *jobs, int njobs, cam_job_result *res)
{
    if (!ctx || njobs < 0 || (njobs > 0 && (!jobs || !res))) return CAM_E_INVAL;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    try {
        CAM_CUDA_TRY(cudaSetDevice(ctx->device));
        std::vector<std::string> keys(njobs);
        for (int i = 0; i < njobs; ++i) {
            validate_job(jobs[i]);
            CAM_REQUIRE(res[i].labels == nullptr, CAM_E_UNSUPPORTED, "batched jobs return label counts, not labels");
            keys[i] = shape_key(jobs[i]);
        }
        if (!ctx->batch) ctx->batch = new BatchRunner(ctx->device);
        auto *br = static_cast<BatchRunner *>(ctx->batch);
        std::vector<int> rc(kMaxBatch);
        int first_err = CAM_OK;
        for (int i = 0; i < njobs;) {
            int k = 1;
            while (i + k < njobs && k < kMaxBatch && keys[i + k] == keys[i]) ++k;
            br->run(jobs + i, k, res + i, rc.data(), k > 1 ? 1 : 0);
            for (int j = 0; j < k; ++j)
                if (rc[j] != CAM_OK && first_err == CAM_OK) first_err = rc[j];
            i += k;
        }
        ctx->err = first_err == CAM_OK ? "" : "a batched job failed (non-finite weight)";
        return first_err;
    } catch (const Error &e) {
        ctx->err = e.msg;
        return e.code;
    } catch (...) {
        ctx->err = "unexpected exception";
        return CAM_E_CUDA;
    }
}

int cam_server_create(int device, size_t hbm_budget, int nworkers, int max_batch, cam_server **out)
{
    if (!out || nworkers < 1 || nworkers > 64 || max_batch < 1 || max_batch > kMaxBatch) return CAM_E_INVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return CAM_E_INVAL;
    }
    std::unique_ptr<cam_server> s(new (std::nothrow) cam_server);
    if (!s) return CAM_E_NOMEM;
    s->device = device;
    if (hbm_budget == 0) {
        size_t fr = 0, tot = 0;
        if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            return CAM_E_CUDA;
        }
        hbm_budget = fr / 10 * 8;
    }
    s->budget = hbm_budget;
    s->max_batch = max_batch;
    {
        const int rc = cam_ctx_create(device, 0, &s->big_ctx);
        if (rc != CAM_OK) return rc;
        s->big_ctx->slabs_off = true;  // admission budgets the exact payload
    }
    for (int i = 0; i < nworkers; ++i) {
        std::unique_ptr<cam_server::Worker> w(new cam_server::Worker);
        w->index = i;
        const int rc = cam_ctx_create(device, 0, &w->ctx);
        if (rc != CAM_OK) {
            for (auto &x : s->workers) cam_ctx_destroy(x->ctx);
            cam_ctx_destroy(s->big_ctx);
            return rc;
        }
        w->ctx->slabs_off = true;
        s->workers.push_back(std::move(w));
    }
    cam_server *sp = s.release();
    for (auto &w : sp->workers) {
        cam_server::Worker *wp = w.get();
        wp->t = std::thread([sp, wp] { sp->worker(*wp); });
    }
    *out = sp;
    return CAM_OK;
}

int cam_server_submit(cam_server *s, const cam_job_desc *job, cam_job_result *res, uint64_t *id)
{
    if (!s || !job || !res || !id) return CAM_E_INVAL;
    try {
        validate_job(*job);
    } catch (const Error &e) {
        return e.code;
    }
    cam_server::Job j;
    j.desc = *job;
    j.res = res;
    j.footprint = job_footprint(*job);
    j.shape = shape_key(*job);
    // a job that moves more than ~0.75 GB through HBM fills the GPU by itself
    const double ncell = (double)job->grid.n[0] * (double)job->grid.n[1] * (double)job->grid.n[2];
    j.big = (double)job->parts.n * 64.0 + ncell * 48.0 > 768.0 * (1 << 20);
    j.batchable = !j.big && job->grid.n[0] <= s->small_n && res->labels == nullptr && s->max_batch > 1;
    j.t_submit = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return CAM_E_BUSY;
        if (j.footprint > s->budget) return CAM_E_NOMEM;
        if (s->queue.size() >= (1u << 20)) return CAM_E_BUSY;
        j.id = s->next_id++;
        *id = j.id;
        s->queue.push_back(std::move(j));
        ++s->submitted;
    }
    s->cv_work.notify_all();
    return CAM_OK;
}

int cam_server_poll(cam_server *s, uint64_t id)
{
    if (!s) return CAM_E_INVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->done.find(id);
    if (it != s->done.end()) {
        const int rc = it->second;
        s->done.erase(it);
        return rc;
    }
    if (id == 0 || id >= s->next_id) return CAM_E_NOTFOUND;
    for (auto &j : s->queue)
        if (j.id == id) return CAM_E_BUSY;
    return s->n_running > 0 ? CAM_E_BUSY : CAM_E_NOTFOUND;
}

int cam_server_wait(cam_server *s, uint64_t id, int64_t timeout_us)
{
    if (!s) return CAM_E_INVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    if (id == 0 || id >= s->next_id) return CAM_E_NOTFOUND;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(timeout_us < 0 ? 0 : timeout_us);
    for (;;) {
        auto it = s->done.find(id);
        if (it != s->done.end()) {
            const int rc = it->second;
            s->done.erase(it);
            return rc;
        }
        bool pending = s->n_running > 0;
        for (auto &j : s->queue)
            if (j.id == id) pending = true;
        if (!pending) return CAM_E_NOTFOUND;  // already collected
        if (timeout_us >= 0) {
            if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && s->done.find(id) == s->done.end())
                return CAM_E_TIMEOUT;
        } else {
            s->cv_done.wait(lk);
        }
    }
}

int cam_server_stats_get(cam_server *s, cam_server_stats *st, int reset)
{
    if (!s || !st) return CAM_E_INVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->queued = (int64_t)s->queue.size();
    st->running = s->n_running;
    st->batches = s->batches;
    st->batched_jobs = s->batched_jobs;
    st->graph_replays = s->replays;
    st->bytes_reserved = s->reserved();
    st->peak_bytes_reserved = s->peak_reserved;
    st->budget = s->budget;
    if (!s->lat_ms.empty()) {
        std::vector<double> v = s->lat_ms;
        std::sort(v.begin(), v.end());
        // nearest-rank percentiles
        auto pct = [&](double p) {
            const size_t r = (size_t)std::ceil(p * (double)v.size());
            return v[std::min(v.size(), std::max<size_t>(r, 1)) - 1];
        };
        st->p50_ms = pct(0.50);
        st->p99_ms = pct(0.99);
        double m = 0.0;
        for (double x : v) m += x;
        st->mean_ms = m / (double)v.size();
        st->max_ms = v.back();
    }
    if (reset) {
        s->lat_ms.clear();
        s->submitted = s->completed = s->failed = s->batches = s->batched_jobs = s->replays = 0;
        s->peak_reserved = s->reserved();
    }
    return CAM_OK;
}

int cam_server_trace(cam_server *s, cam_server_job_trace *out, int max, int *count)
{
    if (!s || !count || max < 0 || (max > 0 && !out)) return CAM_E_INVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    const size_t k = std::min(s->trace.size(), (size_t)max);
    std::copy(s->trace.begin(), s->trace.begin() + (long)k, out);
    s->trace.erase(s->trace.begin(), s->trace.begin() + (long)k);
    *count = (int)k;
    return CAM_OK;
}

const char *cam_server_last_error(cam_server *s)
{
    if (!s) return "null server";
    std::lock_guard<std::mutex> lk(s->mu);
    thread_local std::string copy;
    copy = s->last_err;
    return copy.c_str();
}

int cam_server_destroy(cam_server *s)
{
    if (!s) return CAM_E_INVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &w : s->workers)
        if (w->t.joinable()) w->t.join();
    for (auto &w : s->workers) {
        w->br.reset();
        cam_ctx_destroy(w->ctx);
    }
    cam_ctx_destroy(s->big_ctx);
    delete s;
    return CAM_OK;
}

}  // extern "C"

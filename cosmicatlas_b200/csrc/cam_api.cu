// C ABI of libcam: contexts, scratch memory, deterministic reductions and
// the entry points declared in include/cam.h.
#include <cuda_runtime.h>

#include <cstdlib>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "cam_internal.h"

namespace cam {

// Library-owned stream-ordered memory pool per device.  Scratch buffers
// grow and shrink without cudaMalloc/cudaFree, whose implicit device-wide
// synchronisation would stall every other context's work (the serving
// workers run concurrently).  Freed blocks are kept for reuse (release
// threshold: unlimited) and are only handed out again once their free has
// completed on the GPU (no reuse through stream dependencies), so a buffer
// allocated on one stream is safe to use from any stream.
cudaMemPool_t device_pool(int device)
{
    static std::mutex m;
    static cudaMemPool_t pools[64] = {};
    CAM_REQUIRE(device >= 0 && device < 64, CAM_E_INVAL, "device index out of range");
    std::lock_guard<std::mutex> lk(m);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        CAM_CUDA_TRY(cudaMemPoolCreate(&p, &props));
        uint64_t keep = ~0ull;
        int no = 0;
        CAM_CUDA_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
        CAM_CUDA_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolReuseFollowEventDependencies, &no));
        CAM_CUDA_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolReuseAllowInternalDependencies, &no));
        pools[device] = p;
    }
    return pools[device];
}

// Allocation counters of the process (cam_alloc_stats), all devices.
struct AllocCounters {
    std::atomic<int64_t> allocs{0}, failures{0}, bytes{0}, total_us{0}, max_us{0};
};
AllocCounters &alloc_counters()
{
    static AllocCounters c;
    return c;
}

void *scratch(cam_ctx *ctx, const char *name, size_t bytes)
{
    bytes = std::max<size_t>(bytes, 256);
    DevBuf &b = ctx->bufs[name];
    if (b.cap >= bytes) return b.ptr;
    CAM_REQUIRE(!ctx->capturing, CAM_E_BUSY, std::string("buffer ") + name + " would grow during stream capture");
    const size_t want = std::max(bytes, b.cap + b.cap / 2);
    if (ctx->budget && ctx->used - b.cap + want > ctx->budget)
        throw Error{CAM_E_NOMEM, std::string("HBM budget exceeded allocating ") + name};
    cudaMemPool_t pool = device_pool(ctx->device);
    std::lock_guard<std::mutex> lk(alloc_mutex());
    ctx->gen++;
    if (b.ptr) {
        // stream-ordered: the work already queued on this stream that reads
        // the old buffer completes before the memory is released
        CAM_CUDA_TRY(cudaFreeAsync(b.ptr, ctx->stream));
        ctx->used -= b.cap;
        b.ptr = nullptr;
        b.cap = 0;
    }
    void *p = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaMallocFromPoolAsync(&p, want, pool, ctx->stream);
    if (e != cudaSuccess) {
        // idle pool memory may be fragmented or held for other sizes: hand
        // it back to the device and try once more
        cudaGetLastError();
        alloc_counters().failures++;
        cudaDeviceSynchronize();
        cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocFromPoolAsync(&p, want, pool, ctx->stream);
    }
    {
        AllocCounters &c = alloc_counters();
        const int64_t us =
            std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::steady_clock::now() - t0).count();
        c.allocs++;
        c.bytes += (int64_t)want;
        c.total_us += us;
        int64_t m = c.max_us.load();
        while (us > m && !c.max_us.compare_exchange_weak(m, us)) {
        }
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{CAM_E_NOMEM, std::string("device allocation failed for ") + name + ": " + cudaGetErrorString(e)};
    }
    b.ptr = p;
    b.cap = want;
    ctx->used += want;
    return p;
}

unsigned *device_error_word(cam_ctx *ctx)
{
    if (!ctx->err_word) {
        auto *w = static_cast<unsigned *>(scratch(ctx, "err.word", 16));
        CAM_CUDA_TRY(cudaMemsetAsync(w, 0, 16, ctx->stream));
        ctx->err_word = w;
    }
    return ctx->err_word;
}

void check_device_error(cam_ctx *ctx)
{
    if (!ctx->err_word) return;
    unsigned h = 0;
    CAM_CUDA_TRY(cudaMemcpyAsync(&h, ctx->err_word, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    CAM_REQUIRE(h == 0u, CAM_E_CUDA, "a kernel's bulk copy did not complete within its wait limit");
}

cudaStream_t aux_fork(cam_ctx *ctx)
{
    aux_join(ctx);  // a fork left open by an earlier failure
    CAM_CUDA_TRY(cudaEventRecord(ctx->ev_fork, ctx->stream));
    CAM_CUDA_TRY(cudaStreamWaitEvent(ctx->aux_stream, ctx->ev_fork, 0));
    ctx->aux_open = true;
    return ctx->aux_stream;
}

void aux_join(cam_ctx *ctx)
{
    if (!ctx->aux_open) return;
    ctx->aux_open = false;
    CAM_CUDA_TRY(cudaEventRecord(ctx->ev_join, ctx->aux_stream));
    CAM_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
}

StreamScope::StreamScope(cam_ctx *ctx, cudaStream_t s) : c(ctx), saved(ctx->stream) { ctx->stream = s; }
StreamScope::~StreamScope() { c->stream = saved; }

void prof_begin(cam_ctx *ctx, const char *name)
{
    if (!ctx->prof_on || ctx->capturing) return;
    auto take = [&]() {
        cudaEvent_t e;
        if (!ctx->prof_pool.empty()) {
            e = ctx->prof_pool.back();
            ctx->prof_pool.pop_back();
        } else {
            CAM_CUDA_TRY(cudaEventCreate(&e));
        }
        return e;
    };
    ProfRecord r{name, take(), take(), ctx->stream == ctx->aux_stream};
    CAM_CUDA_TRY(cudaEventRecord(r.start, ctx->stream));
    ctx->prof_pending.push_back(r);
}

void prof_end(cam_ctx *ctx)
{
    if (!ctx->prof_on || ctx->capturing || ctx->prof_pending.empty()) return;
    CAM_CUDA_TRY(cudaEventRecord(ctx->prof_pending.back().stop, ctx->stream));
}

// Folds finished records into the per-name totals (synchronises).
static void prof_collect(cam_ctx *ctx)
{
    if (ctx->prof_pending.empty()) return;
    CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (auto &r : ctx->prof_pending) {
        float ms = 0.f;
        CAM_CUDA_TRY(cudaEventElapsedTime(&ms, r.start, r.stop));
        auto &acc = ctx->prof_acc[r.side ? std::string("side.") + r.name : std::string(r.name)];
        acc.first += 1;
        acc.second += ms;
        ctx->prof_pool.push_back(r.start);
        ctx->prof_pool.push_back(r.stop);
    }
    ctx->prof_pending.clear();
}

void smem_limit(const void *func, size_t bytes)
{
    static std::mutex m;
    static std::map<std::pair<int, const void *>, size_t> cur;
    // the default limit (48 KB) also covers a kernel's static shared memory:
    // sizes near it are raised too
    if (bytes <= 32 * 1024) return;
    int dev = 0;
    CAM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(m);
    size_t &c = cur[{dev, func}];
    if (c >= bytes) return;
    CAM_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    c = bytes;
}

std::mutex &alloc_mutex()
{
    static std::mutex m;
    return m;
}

void release_all(cam_ctx *ctx)
{
    std::lock_guard<std::mutex> lk(alloc_mutex());
    ctx->gen++;
    free_plans(ctx);  // their twiddles live in the buffers freed below
    for (auto &kv : ctx->bufs)
        if (kv.second.ptr) cudaFreeAsync(kv.second.ptr, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    ctx->bufs.clear();
    ctx->err_word = nullptr;
    ctx->used = 0;
    // The freed blocks stay in the device pool: trimming it here made every
    // later growth map new physical memory while other contexts' jobs ran,
    // and jobs running at that moment stalled for 0.4-1 s (served stream).
    // The pool is trimmed on an allocation failure or by cam_pool_trim.
    cudaGetLastError();
}

namespace {

constexpr int kRedBlocks = 8 * kNumSMs;

template <typename T>
__global__ void __launch_bounds__(256) partial_sum_kernel(const T *__restrict__ in, int64_t n, double *__restrict__ part)
{
    __shared__ double red[8];
    // Static contiguous chunk per CTA, a multiple of 4 elements: the
    // summation order is fixed.  16-byte loads when the array is 16-byte
    // aligned, four (float) or two (double) independent accumulators.
    const int64_t chunk = (((n + gridDim.x - 1) / gridDim.x) + 3) & ~(int64_t)3;
    const int64_t beg = min(n, (int64_t)blockIdx.x * chunk), end = min(n, beg + chunk);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int64_t tail = beg;
    if ((reinterpret_cast<uintptr_t>(in) & 15) == 0) {
        if constexpr (sizeof(T) == 4) {
            const int64_t nv = (end - beg) / 4;
            const float4 *v = reinterpret_cast<const float4 *>(in + beg);
            for (int64_t i = threadIdx.x; i < nv; i += blockDim.x) {
                const float4 f = __ldg(v + i);
                a0 += (double)f.x;
                a1 += (double)f.y;
                a2 += (double)f.z;
                a3 += (double)f.w;
            }
            tail = beg + 4 * nv;
        } else {
            const int64_t nv = (end - beg) / 2;
            const double2 *v = reinterpret_cast<const double2 *>(in + beg);
            for (int64_t i = threadIdx.x; i < nv; i += blockDim.x) {
                const double2 f = __ldg(v + i);
                a0 += f.x;
                a1 += f.y;
            }
            tail = beg + 2 * nv;
        }
    }
    for (int64_t i = tail + threadIdx.x; i < end; i += blockDim.x) a0 += (double)in[i];
    double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

// One CTA of kFinalThreads: thread t sums in[t], in[t + kFinalThreads], ...
// in order, then a fixed shuffle tree per warp and the warp sums in order
// (FP64, the same order on every run).  out[0] = sum, out[1] = sum / divisor.
constexpr int kFinalThreads = 1024;
__global__ void __launch_bounds__(kFinalThreads)
final_sum_kernel(const double *__restrict__ part, int np, double *__restrict__ out, double divisor)
{
    __shared__ double red[kFinalThreads / 32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += kFinalThreads) acc += part[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kFinalThreads / 32; ++w) t += red[w];
        out[0] = t;
        out[1] = t / divisor;
    }
}

}  // namespace

// out[0] = sum, out[1] = sum / divisor (FP64, fixed order).  Up to 2^16
// values are summed by one CTA directly.
void reduce_sum_f64(cam_ctx *ctx, const double *in, int64_t n, double *out, double divisor)
{
    if (n <= 65536) {
        CAM_LAUNCH(ctx, final_sum_kernel, 1, kFinalThreads, 0, in, (int)n, out, divisor);
        return;
    }
    auto *part = static_cast<double *>(scratch(ctx, "red.part", kRedBlocks * sizeof(double)));
    CAM_LAUNCH(ctx, partial_sum_kernel<double>, kRedBlocks, 256, 0, in, n, part);
    CAM_LAUNCH(ctx, final_sum_kernel, 1, kFinalThreads, 0, part, kRedBlocks, out, divisor);
}

void mesh_mean(cam_ctx *ctx, const void *mesh, int precision, int64_t ncell, double *d_out)
{
    auto *part = static_cast<double *>(scratch(ctx, "red.part", kRedBlocks * sizeof(double)));
    if (precision == CAM_F32)
        CAM_LAUNCH(ctx, partial_sum_kernel<float>, kRedBlocks, 256, 0, (const float *)mesh, ncell, part);
    else
        CAM_LAUNCH(ctx, partial_sum_kernel<double>, kRedBlocks, 256, 0, (const double *)mesh, ncell, part);
    CAM_LAUNCH(ctx, final_sum_kernel, 1, kFinalThreads, 0, part, kRedBlocks, d_out, (double)ncell);
}

}  // namespace cam

using namespace cam;

namespace {

template <typename F>
int guarded(cam_ctx *ctx, F &&f)
{
    if (!ctx) return CAM_E_INVAL;
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    try {
        CAM_CUDA_TRY(cudaSetDevice(ctx->device));
        f();
        ctx->err.clear();
        return CAM_OK;
    } catch (const Error &e) {
        ctx->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        ctx->err = "host allocation failed";
        return CAM_E_NOMEM;
    } catch (...) {
        ctx->err = "unexpected exception";
        return CAM_E_CUDA;
    }
}

size_t esize(int precision) { return precision == CAM_F64 ? 8 : 4; }

void check_grid_cubic(const cam_grid *g)
{
    CAM_REQUIRE(g, CAM_E_INVAL, "null grid");
    CAM_REQUIRE(g->n[0] == g->n[1] && g->n[1] == g->n[2], CAM_E_UNSUPPORTED, "FFT stages need a cubic mesh");
    CAM_REQUIRE(g->L[0] > 0.f && std::isfinite(g->L[0]), CAM_E_INVAL, "box side must be > 0");
}

void check_prec(int p) { CAM_REQUIRE(p == CAM_F32 || p == CAM_F64, CAM_E_INVAL, "precision must be CAM_F32 or CAM_F64"); }
void check_mem(int m) { CAM_REQUIRE(m == CAM_MEM_HOST || m == CAM_MEM_DEVICE, CAM_E_INVAL, "mem must be CAM_MEM_HOST or CAM_MEM_DEVICE"); }

struct DevParticles {
    const float *x, *y, *z, *w;
    int64_t n;
};

DevParticles stage_particles(cam_ctx *ctx, const cam_particles *p)
{
    CAM_REQUIRE(p, CAM_E_INVAL, "null particles");
    CAM_REQUIRE(p->n >= 0, CAM_E_INVAL, "negative particle count");
    check_mem(p->mem);
    CAM_REQUIRE(p->n == 0 || (p->x && p->y && p->z), CAM_E_INVAL, "null particle coordinates");
    DevParticles d{};
    d.n = p->n;
    d.x = stage_in(ctx, "in.x", p->x, p->n, p->mem);
    d.y = stage_in(ctx, "in.y", p->y, p->n, p->mem);
    d.z = stage_in(ctx, "in.z", p->z, p->n, p->mem);
    d.w = p->w ? stage_in(ctx, "in.w", p->w, p->n, p->mem) : nullptr;
    return d;
}

}  // namespace

namespace cam {

cam_grid resolved_grid(const cam_grid &g)
{
    cam_grid r = g;
    for (int a = 0; a < 3; ++a)
        if (r.d[a] == 0.f) r.d[a] = r.L[a] / (float)r.n[a];
    return r;
}

int nbins_for(const cam_pk_opts &o, int64_t n)
{
    if (o.nbins > 0) return o.nbins;
    return (int)((double)n / o.ndel / 2.0);  // Nnp_data = Nft / ndel_data / 2
}

// P(k) per bin from the FP64 bin sums: normalisation and shot noise of
// PowerSpectrumF::compute_power_spectrum_grid (Source/PowerSpectrumF.cpp:1754-1783)
// and the final division of FftwFunctions::power_spectrum (:1873-1874).
void finalize_pk(int64_t n, float L, double n_obj, const cam_pk_opts &o, int nbins, const double *sr,
                 const double *ss, const int64_t *md, double *pk, int64_t *modes, double *kvec, cam_pk_info *info)
{
    const double vol = (double)L * (double)L * (double)L;
    double normal, ngal;
    if (o.input_type == CAM_INPUT_DENSITY) {
        ngal = n_obj;
        normal = ngal * ngal / vol;  // PowerSpectrumF.cpp:1764
    } else {
        ngal = 1.0;
        const double ng = (double)n * n * n;
        normal = ng * ng / vol;      // PowerSpectrumF.cpp:1775
    }
    const double sn = vol / ngal;   // PowerSpectrumF.cpp:1782
    const double kf = 2.0 * M_PI / (double)L;
    for (int b = 0; b < nbins; ++b) {
        double v = 0.0;
        if (md[b] > 0) {
            v = sr[b] / ((double)md[b] * normal);
            if (o.sn_correction) v -= sn * ss[b] / (double)md[b];
        }
        if (pk) pk[b] = v;
        if (modes) modes[b] = md[b];
        if (kvec) kvec[b] = kf * (o.DeltaKmin + ((double)b + 0.5) * o.ndel);  // PowerSpectrumF.cpp:1792
    }
    if (info) {
        info->n_obj = ngal;
        info->shot_noise = sn;
        info->normal = normal;
        info->kf = kf;
    }
}

Spectrum alloc_spectrum(cam_ctx *ctx, int64_t n, int precision, const char *tag)
{
    Spectrum s;
    s.n = n;
    s.precision = precision;
    const size_t cs = 2 * esize(precision);
    s.main = scratch(ctx, (std::string(tag) + ".main").c_str(), (size_t)n * n * (n / 2) * cs);
    s.nyq = scratch(ctx, (std::string(tag) + ".nyq").c_str(), (size_t)n * n * cs);
    return s;
}

}  // namespace cam

namespace {

// Power spectrum of a spectrum already on the device (split layout).
void power_from_spectrum(cam_ctx *ctx, const Spectrum &s, float L, double n_obj, const cam_pk_opts &o,
                         double *pk, int64_t *modes, double *kvec, cam_pk_info *info)
{
    const int nbins = nbins_for(o, s.n);
    std::vector<double> sr(nbins), ss(nbins);
    std::vector<int64_t> md(nbins);
    power_bin(ctx, s, o, nbins, sr.data(), ss.data(), md.data());
    finalize_pk(s.n, L, n_obj, o, nbins, sr.data(), ss.data(), md.data(), pk, modes, kvec, info);
}

void validate_pk(const cam_pk_opts *o)
{
    CAM_REQUIRE(o, CAM_E_INVAL, "null P(k) options");
    CAM_REQUIRE(o->scheme >= 0 && o->scheme <= 2, CAM_E_INVAL, "unknown window scheme");
    CAM_REQUIRE(o->input_type == CAM_INPUT_DENSITY || o->input_type == CAM_INPUT_DELTA, CAM_E_INVAL, "unknown input type");
    CAM_REQUIRE(o->ndel > 0.0 && std::isfinite(o->ndel), CAM_E_INVAL, "ndel must be > 0");
    CAM_REQUIRE(o->nbins >= 0, CAM_E_INVAL, "nbins must be >= 0");
}

}  // namespace

extern "C" {

const char *cam_version(void) { return "cosmicatlas-b200 0.1 (sm_100a)"; }

int cam_ctx_create(int device, size_t hbm_budget, cam_ctx **out)
{
    if (!out) return CAM_E_INVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return CAM_E_INVAL;
    }
    auto *c = new (std::nothrow) cam_ctx;
    if (!c) return CAM_E_NOMEM;
    c->device = device;
    c->budget = hbm_budget;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (c->ev_fork) cudaEventDestroy(c->ev_fork);
        if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
        delete c;
        return CAM_E_CUDA;
    }
    c->stream = c->own_stream;
    c->no_tma = std::getenv("CAM_NO_TMA") != nullptr;
    *out = c;
    return CAM_OK;
}

int cam_ctx_destroy(cam_ctx *ctx)
{
    if (!ctx) return CAM_E_INVAL;
    {
        std::lock_guard<std::recursive_mutex> lk(ctx->mu);
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto &r : ctx->prof_pending) {
            cudaEventDestroy(r.start);
            cudaEventDestroy(r.stop);
        }
        for (auto e : ctx->prof_pool) cudaEventDestroy(e);
        if (ctx->batch) batch_destroy(ctx->batch);
        ctx->batch = nullptr;
        release_all(ctx);
        if (ctx->job_pin) {
            std::lock_guard<std::mutex> lk(alloc_mutex());
            cudaFreeHost(ctx->job_pin);
            ctx->job_pin = nullptr;
        }
        if (ctx->aux_stream) {
            cudaStreamSynchronize(ctx->aux_stream);
            cudaStreamDestroy(ctx->aux_stream);
        }
        if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
        if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    }
    delete ctx;
    return CAM_OK;
}

int cam_ctx_set_stream(cam_ctx *ctx, void *stream)
{
    return guarded(ctx, [&] { ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream; });
}

int cam_ctx_sync(cam_ctx *ctx)
{
    return guarded(ctx, [&] {
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        check_device_error(ctx);
    });
}

const char *cam_last_error(cam_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int64_t cam_kernel_launches(cam_ctx *ctx) { return ctx ? ctx->launches : -1; }

int cam_alloc_stats_get(cam_alloc_stats *out, int reset)
{
    if (!out) return CAM_E_INVAL;
    AllocCounters &c = alloc_counters();
    out->allocs = c.allocs.load();
    out->failures = c.failures.load();
    out->bytes = c.bytes.load();
    out->total_ms = (double)c.total_us.load() / 1e3;
    out->max_ms = (double)c.max_us.load() / 1e3;
    if (reset) {
        c.allocs = 0;
        c.failures = 0;
        c.bytes = 0;
        c.total_us = 0;
        c.max_us = 0;
    }
    return CAM_OK;
}

int cam_pool_trim(int device)
{
    try {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
            cudaGetLastError();
            return CAM_E_INVAL;
        }
        std::lock_guard<std::mutex> lk(alloc_mutex());
        cudaMemPool_t pool = device_pool(device);
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaDeviceSynchronize();  // frees still in flight complete first
        const cudaError_t e = cudaMemPoolTrimTo(pool, 0);
        cudaSetDevice(prev);
        return e == cudaSuccess ? CAM_OK : CAM_E_CUDA;
    } catch (const Error &e) {
        return e.code;
    }
}

int cam_profile_enable(cam_ctx *ctx, int on)
{
    return guarded(ctx, [&] {
        prof_collect(ctx);
        ctx->prof_on = on != 0;
    });
}

int cam_profile_read(cam_ctx *ctx, char *buf, size_t len, int reset)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(buf && len > 0, CAM_E_INVAL, "null buffer");
        prof_collect(ctx);
        std::string out;
        for (auto &kv : ctx->prof_acc) {
            char line[256];
            snprintf(line, sizeof(line), "%s,%lld,%.6f\n", kv.first.c_str(), (long long)kv.second.first,
                     kv.second.second);
            out += line;
        }
        CAM_REQUIRE(out.size() + 1 <= len, CAM_E_INVAL, "profile buffer too small");
        memcpy(buf, out.c_str(), out.size() + 1);
        if (reset) ctx->prof_acc.clear();
    });
}

int cam_assign(cam_ctx *ctx, const cam_particles *parts, const cam_grid *grid, int scheme,
               int precision, void *mesh_out, int out_mem, cam_assign_stats *stats)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(grid && mesh_out, CAM_E_INVAL, "null grid or output");
        check_prec(precision);
        check_mem(out_mem);
        const DevParticles d = stage_particles(ctx, parts);
        const cam_grid g = resolved_grid(*grid);
        const int64_t ncell = g.n[0] * g.n[1] * g.n[2];
        AssignOut out;
        out.precision = precision;
        out.mesh = out_mem == CAM_MEM_DEVICE ? mesh_out : scratch(ctx, "asg.mesh", ncell * esize(precision));
        out.d_sum = static_cast<double *>(scratch(ctx, "asg.sum", 2 * sizeof(double)));
        assign_device(ctx, d.x, d.y, d.z, d.w, d.n, g, scheme, out);
        if (out_mem == CAM_MEM_HOST)
            CAM_CUDA_TRY(cudaMemcpyAsync(mesh_out, out.mesh, ncell * esize(precision), cudaMemcpyDeviceToHost, ctx->stream));
        double sum = 0.0;
        CAM_CUDA_TRY(cudaMemcpyAsync(&sum, out.d_sum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (stats) {
            stats->n_in = out.n_in;
            stats->n_lost = out.n_lost;
            stats->sum_mesh = sum;
        }
    });
}

int cam_count_ngp(cam_ctx *ctx, const cam_particles *parts, const cam_grid *grid, uint32_t *counts_out,
                  int out_mem, cam_assign_stats *stats)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(grid && counts_out, CAM_E_INVAL, "null grid or output");
        check_mem(out_mem);
        CAM_REQUIRE(parts && parts->w == nullptr, CAM_E_INVAL, "integer counts take unweighted particles");
        const DevParticles d = stage_particles(ctx, parts);
        const cam_grid g = resolved_grid(*grid);
        const int64_t ncell = g.n[0] * g.n[1] * g.n[2];
        AssignOut out;
        out.precision = -1;
        out.mesh = out_mem == CAM_MEM_DEVICE ? (void *)counts_out : scratch(ctx, "asg.mesh", ncell * 4);
        out.d_sum = static_cast<double *>(scratch(ctx, "asg.sum", 2 * sizeof(double)));
        assign_device(ctx, d.x, d.y, d.z, nullptr, d.n, g, CAM_NGP, out);
        if (out_mem == CAM_MEM_HOST)
            CAM_CUDA_TRY(cudaMemcpyAsync(counts_out, out.mesh, ncell * 4, cudaMemcpyDeviceToHost, ctx->stream));
        double sum = 0.0;
        CAM_CUDA_TRY(cudaMemcpyAsync(&sum, out.d_sum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (stats) {
            stats->n_in = out.n_in;
            stats->n_lost = out.n_lost;
            stats->sum_mesh = sum;
        }
    });
}

int cam_cell_keys(cam_ctx *ctx, const cam_particles *parts, const cam_grid *grid, int scheme,
                  int64_t *keys_out, int out_mem)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(grid && keys_out, CAM_E_INVAL, "null grid or output");
        check_mem(out_mem);
        CAM_REQUIRE(scheme >= CAM_NGP && scheme <= CAM_TSC, CAM_E_INVAL, "unknown mass assignment scheme");
        const DevParticles d = stage_particles(ctx, parts);
        const cam_grid g = resolved_grid(*grid);
        int64_t *dk = out_mem == CAM_MEM_DEVICE ? keys_out
                                                : static_cast<int64_t *>(scratch(ctx, "keys.out", std::max<int64_t>(d.n, 1) * 8));
        cell_keys_device(ctx, d.x, d.y, d.z, d.n, g, scheme, dk);
        if (out_mem == CAM_MEM_HOST && d.n > 0)
            CAM_CUDA_TRY(cudaMemcpyAsync(keys_out, dk, d.n * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    });
}

int cam_fft_r2c(cam_ctx *ctx, int64_t n, int precision, const void *in, void *out, int mem)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(in && out, CAM_E_INVAL, "null FFT buffer");
        check_prec(precision);
        check_mem(mem);
        FftPlan *plan = get_plan(ctx, n, precision);
        const size_t es = esize(precision);
        const size_t in_bytes = (size_t)n * n * n * es;
        const size_t out_bytes = (size_t)n * n * (n / 2 + 1) * 2 * es;
        const void *din = mem == CAM_MEM_DEVICE ? in : scratch(ctx, "fft.in", in_bytes);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync((void *)din, in, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
        Spectrum s = alloc_spectrum(ctx, n, precision, "fft.spec");
        fft_r2c_split(ctx, plan, din, nullptr, s);
        void *dout = mem == CAM_MEM_DEVICE ? out : scratch(ctx, "fft.out", out_bytes);
        split_to_fftw(ctx, s, dout);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    });
}

int cam_fft_c2r(cam_ctx *ctx, int64_t n, int precision, const void *in, void *out, int mem)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(in && out, CAM_E_INVAL, "null FFT buffer");
        check_prec(precision);
        check_mem(mem);
        FftPlan *plan = get_plan(ctx, n, precision);
        const size_t es = esize(precision);
        const size_t out_bytes = (size_t)n * n * n * es;
        const size_t in_bytes = (size_t)n * n * (n / 2 + 1) * 2 * es;
        const void *din = mem == CAM_MEM_DEVICE ? in : scratch(ctx, "fft.out", in_bytes);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync((void *)din, in, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
        Spectrum s = alloc_spectrum(ctx, n, precision, "fft.spec");
        fftw_to_split(ctx, din, s);
        void *dout = mem == CAM_MEM_DEVICE ? out : scratch(ctx, "fft.in", out_bytes);
        fft_c2r_split(ctx, plan, s, dout, 1.0 / ((double)n * n * n));
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    });
}

int cam_power(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision, int mem,
              const cam_pk_opts *opts, double *pk, int64_t *modes, double *kvector, cam_pk_info *info)
{
    return cam_power_multipoles(ctx, grid, mesh, precision, mem, opts, -1, pk, nullptr, nullptr, modes, kvector, info);
}

int cam_power_multipoles(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision, int mem,
                         const cam_pk_opts *opts, int los, double *p0, double *p2, double *p4, int64_t *modes,
                         double *kvector, cam_pk_info *info)
{
    double *pk = p0;
    return guarded(ctx, [&] {
        CAM_REQUIRE(los >= -1 && los <= 2, CAM_E_INVAL, "line of sight must be 0 (x), 1 (y) or 2 (z)");
        check_grid_cubic(grid);
        CAM_REQUIRE(mesh, CAM_E_INVAL, "null mesh");
        check_prec(precision);
        check_mem(mem);
        validate_pk(opts);
        const int64_t n = grid->n[0];
        FftPlan *plan = get_plan(ctx, n, precision);
        const size_t bytes = (size_t)n * n * n * esize(precision);
        const void *dm = mem == CAM_MEM_DEVICE ? mesh : scratch(ctx, "pk.mesh", bytes);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync((void *)dm, mesh, bytes, cudaMemcpyHostToDevice, ctx->stream));
        auto *dsum = static_cast<double *>(scratch(ctx, "pk.sum", 2 * sizeof(double)));
        double hs[2] = {0.0, 0.0};
        const double *sub = nullptr;
        if (opts->input_type == CAM_INPUT_DENSITY) {
            mesh_mean(ctx, dm, precision, n * n * n, dsum);
            sub = dsum + 1;  // rho - N_gal / N^3 (PowerSpectrumF.cpp:1756-1762)
        }
        Spectrum s = alloc_spectrum(ctx, n, precision, "job.spec");
        fft_r2c_split(ctx, plan, dm, sub, s);
        if (sub) {
            CAM_CUDA_TRY(cudaMemcpyAsync(hs, dsum, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
            CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        }
        cam_pk_info inf{};
        power_from_spectrum(ctx, s, grid->L[0], hs[0], *opts, pk, modes, kvector, &inf);
        if (info) *info = inf;
        if (los >= 0 && (p2 || p4)) {
            // P_l = (2l + 1) sum L_l(mu) |F|^2 / W^2 / (modes normal), no shot
            // noise for l > 0 (FftwFunctions.cpp:1188-1212, :1614-1625)
            const int nb = nbins_for(*opts, n);
            const PkDevice m = power_multipole_device(ctx, s, *opts, nb, los);
            std::vector<double> hm(2 * (size_t)nb);
            std::vector<unsigned long long> hc(nb);
            CAM_CUDA_TRY(cudaMemcpyAsync(hm.data(), m.sums, hm.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
            CAM_CUDA_TRY(cudaMemcpyAsync(hc.data(), m.modes, (size_t)nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
            CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            for (int b = 0; b < nb; ++b) {
                const double den = (double)hc[b] * inf.normal;
                if (p2) p2[b] = hc[b] ? 5.0 * hm[2 * b] / den : 0.0;
                if (p4) p4[b] = hc[b] ? 9.0 * hm[2 * b + 1] / den : 0.0;
            }
        }
    });
}

int cam_tweb(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision, int mem,
             const cam_tweb_opts *opts, uint8_t *labels, float *lambdas, int out_mem, cam_tweb_stats *stats)
{
    return cam_tweb_invariants(ctx, grid, mesh, precision, mem, opts, labels, lambdas, nullptr, out_mem, stats);
}

int cam_tweb_invariants(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision, int mem,
                        const cam_tweb_opts *opts, uint8_t *labels, float *lambdas, float *invariants, int out_mem,
                        cam_tweb_stats *stats)
{
    return guarded(ctx, [&] {
        check_grid_cubic(grid);
        CAM_REQUIRE(mesh && opts, CAM_E_INVAL, "null mesh or options");
        check_prec(precision);
        check_mem(mem);
        check_mem(out_mem);
        CAM_REQUIRE(opts->input_type == CAM_INPUT_DENSITY || opts->input_type == CAM_INPUT_DELTA ||
                        opts->input_type == CAM_INPUT_POTENTIAL, CAM_E_INVAL,
                    "unknown input type");
        const int64_t n = grid->n[0], ncell = n * n * n;
        FftPlan *plan = get_plan(ctx, n, precision);
        const size_t bytes = (size_t)ncell * esize(precision);
        const void *dm = mem == CAM_MEM_DEVICE ? mesh : scratch(ctx, "pk.mesh", bytes);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync((void *)dm, mesh, bytes, cudaMemcpyHostToDevice, ctx->stream));
        auto *dsum = static_cast<double *>(scratch(ctx, "tw.sum", 2 * sizeof(double)));
        const double *sub = nullptr;
        if (opts->input_type == CAM_INPUT_DENSITY) {
            mesh_mean(ctx, dm, precision, ncell, dsum);
            sub = dsum + 1;
        }
        Spectrum s = alloc_spectrum(ctx, n, precision, "job.spec");
        fft_r2c_split(ctx, plan, dm, sub, s);
        uint8_t *dl = labels ? (out_mem == CAM_MEM_DEVICE ? labels : static_cast<uint8_t *>(scratch(ctx, "tw.labels", ncell))) : nullptr;
        float *dlam = lambdas ? (out_mem == CAM_MEM_DEVICE ? lambdas : static_cast<float *>(scratch(ctx, "tw.lam", 3 * ncell * 4))) : nullptr;
        float *dinv = invariants ? (out_mem == CAM_MEM_DEVICE ? invariants
                                                              : static_cast<float *>(scratch(ctx, "tw.inv", 4 * ncell * 4)))
                                 : nullptr;
        cam_tweb_stats st{};
        tweb_device(ctx, plan, s, grid->L[0], sub, opts->input_type, *opts, dl, dlam, &st, dinv);
        if (out_mem == CAM_MEM_HOST) {
            if (labels) CAM_CUDA_TRY(cudaMemcpyAsync(labels, dl, ncell, cudaMemcpyDeviceToHost, ctx->stream));
            if (lambdas) CAM_CUDA_TRY(cudaMemcpyAsync(lambdas, dlam, 3 * ncell * 4, cudaMemcpyDeviceToHost, ctx->stream));
            if (invariants)
                CAM_CUDA_TRY(cudaMemcpyAsync(invariants, dinv, 4 * ncell * 4, cudaMemcpyDeviceToHost, ctx->stream));
        }
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (stats) *stats = st;
    });
}

int cam_cross_power(cam_ctx *ctx, const cam_grid *grid, const void *mesh_x, const void *mesh_y, int precision,
                    int mem, const cam_pk_opts *opts, int input_type_y, int want_coeff, double *pk, double *pk_x,
                    double *pk_y, int64_t *modes, double *kvector)
{
    return guarded(ctx, [&] {
        check_grid_cubic(grid);
        CAM_REQUIRE(mesh_x && mesh_y, CAM_E_INVAL, "null mesh");
        check_prec(precision);
        check_mem(mem);
        validate_pk(opts);
        CAM_REQUIRE(input_type_y == CAM_INPUT_DENSITY || input_type_y == CAM_INPUT_DELTA, CAM_E_INVAL,
                    "unknown input type of the second mesh");
        const int64_t n = grid->n[0], ncell = n * n * n;
        FftPlan *plan = get_plan(ctx, n, precision);
        const size_t bytes = (size_t)ncell * esize(precision);
        const void *dm[2] = {mesh_x, mesh_y};
        const int kind[2] = {opts->input_type, input_type_y};
        auto *dsum = static_cast<double *>(scratch(ctx, "xpk.sum", 4 * sizeof(double)));
        Spectrum sp[2];
        for (int a = 0; a < 2; ++a) {
            const void *d = dm[a];
            if (mem == CAM_MEM_HOST) {
                void *t = scratch(ctx, a ? "xpk.mesh1" : "xpk.mesh0", bytes);
                CAM_CUDA_TRY(cudaMemcpyAsync(t, dm[a], bytes, cudaMemcpyHostToDevice, ctx->stream));
                d = t;
            }
            const double *sub = nullptr;
            if (kind[a] == CAM_INPUT_DENSITY) {
                mesh_mean(ctx, d, precision, ncell, dsum + 2 * a);  // [2a] = sum, [2a+1] = mean
                sub = dsum + 2 * a + 1;
            }
            sp[a] = alloc_spectrum(ctx, n, precision, a ? "xpk.spec1" : "xpk.spec0");
            fft_r2c_split(ctx, plan, d, sub, sp[a]);  // F(rho - mean), or F(delta)
        }
        const int nb = nbins_for(*opts, n);
        const PkDevice xs = power_cross_device(ctx, sp[0], sp[1], *opts, nb);
        cam_pk_opts oy = *opts;
        oy.sn_correction = 0;
        const PkDevice ys = power_bin_device(ctx, sp[1], oy, nb);
        std::vector<double> hx(2 * (size_t)nb), hy(2 * (size_t)nb), hs(4);
        std::vector<unsigned long long> hm(nb);
        CAM_CUDA_TRY(cudaMemcpyAsync(hx.data(), xs.sums, hx.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaMemcpyAsync(hy.data(), ys.sums, hy.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaMemcpyAsync(hm.data(), xs.modes, (size_t)nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaMemcpyAsync(hs.data(), dsum, 4 * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        // F(delta) = F(rho - mean) / mean for a density; normal = (L^1.5 / N^3)^-2
        // for both fields (PowerSpectrumF.cpp:576-577, :605-606)
        const double fx = kind[0] == CAM_INPUT_DENSITY ? 1.0 / hs[1] : 1.0;
        const double fy = kind[1] == CAM_INPUT_DENSITY ? 1.0 / hs[3] : 1.0;
        const double ng = (double)ncell;
        const double L = grid->L[0];
        const double normal = ng * ng / (L * L * L);
        const double kf = 2.0 * M_PI / L;
        for (int b = 0; b < nb; ++b) {
            const double m = (double)hm[b];
            double px = 0.0, pxx = 0.0, pyy = 0.0;
            if (hm[b] > 0) {
                px = hx[2 * b] * fx * fy / (m * normal);
                pxx = hx[2 * b + 1] * fx * fx / (m * normal);
                pyy = hy[2 * b] * fy * fy / (m * normal);
            }
            if (pk) pk[b] = want_coeff ? (hm[b] > 0 ? px / std::sqrt(pxx * pyy) : 0.0) : px;
            if (pk_x) pk_x[b] = pxx;
            if (pk_y) pk_y[b] = pyy;
            if (modes) modes[b] = (int64_t)hm[b];
            if (kvector) kvector[b] = kf * (opts->DeltaKmin + ((double)b + 0.5) * opts->ndel);
        }
    });
}

int cam_poisson(cam_ctx *ctx, const cam_grid *grid, const void *delta, int precision, int mem, float smoothing_R,
                void *phi, int out_mem)
{
    return guarded(ctx, [&] {
        check_grid_cubic(grid);
        CAM_REQUIRE(delta && phi, CAM_E_INVAL, "null mesh");
        check_prec(precision);
        check_mem(mem);
        check_mem(out_mem);
        CAM_REQUIRE(smoothing_R >= 0.f && std::isfinite(smoothing_R), CAM_E_INVAL, "invalid smoothing radius");
        const int64_t n = grid->n[0];
        FftPlan *plan = get_plan(ctx, n, precision);
        const size_t bytes = (size_t)n * n * n * esize(precision);
        const void *din = mem == CAM_MEM_DEVICE ? delta : scratch(ctx, "fft.in", bytes);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync((void *)din, delta, bytes, cudaMemcpyHostToDevice, ctx->stream));
        Spectrum s = alloc_spectrum(ctx, n, precision, "fft.spec");
        fft_r2c_split(ctx, plan, din, nullptr, s);
        poisson_device(ctx, s, grid->L[0], smoothing_R);
        void *dout = out_mem == CAM_MEM_DEVICE ? phi : scratch(ctx, "fd.out", bytes);
        fft_c2r_split(ctx, plan, s, dout, 1.0 / ((double)n * n * n));
        if (out_mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync(phi, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    });
}

int cam_gradfindif(cam_ctx *ctx, const cam_grid *grid, const void *in, int precision, int mem, int dim, void *out,
                   int out_mem)
{
    return guarded(ctx, [&] {
        check_grid_cubic(grid);
        CAM_REQUIRE(in && out, CAM_E_INVAL, "null mesh");
        check_prec(precision);
        check_mem(mem);
        check_mem(out_mem);
        CAM_REQUIRE(dim >= 1 && dim <= 3, CAM_E_INVAL, "dim must be 1, 2 or 3");
        const int64_t n = grid->n[0];
        const size_t bytes = (size_t)n * n * n * esize(precision);
        const void *din = in;
        if (mem == CAM_MEM_HOST || (out_mem == CAM_MEM_DEVICE && in == out)) {
            // the reference takes `in` by value, so out may be the same array
            void *t = scratch(ctx, "fd.in", bytes);
            CAM_CUDA_TRY(cudaMemcpyAsync(t, in, bytes, mem == CAM_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                         ctx->stream));
            din = t;
        }
        void *dout = out_mem == CAM_MEM_DEVICE ? out : scratch(ctx, "fd.out", bytes);
        gradfindif_device(ctx, din, dout, n, grid->L[0], dim, precision);
        if (out_mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    });
}

int cam_fkp_weights(cam_ctx *ctx, int64_t n, const float *nbar, double nbar_const, const float *w_in, int fkp,
                    double P_est, int mem, float *w_out, int out_mem, double *sums)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(n >= 0 && w_out, CAM_E_INVAL, "invalid object count or null output");
        check_mem(mem);
        check_mem(out_mem);
        CAM_REQUIRE(std::isfinite(nbar_const) && std::isfinite(P_est), CAM_E_INVAL, "non-finite nbar or P_est");
        const float *dn = stage_in(ctx, "fkp.nbar", nbar, (size_t)n, mem);
        const float *dw = stage_in(ctx, "fkp.win", w_in, (size_t)n, mem);
        float *dout = out_mem == CAM_MEM_DEVICE
                          ? w_out
                          : static_cast<float *>(scratch(ctx, "fkp.wout", std::max<size_t>(1, (size_t)n) * sizeof(float)));
        auto *dsum = static_cast<double *>(scratch(ctx, "fkp.sums", 3 * sizeof(double)));
        fkp_weights_device(ctx, n, dn, nbar_const, dw, fkp, P_est, dout, dsum);
        if (out_mem == CAM_MEM_HOST && n > 0)
            CAM_CUDA_TRY(cudaMemcpyAsync(w_out, dout, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        double h[3] = {0.0, 0.0, 0.0};
        CAM_CUDA_TRY(cudaMemcpyAsync(h, dsum, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (sums) {
            sums[0] = (double)n;
            sums[1] = h[0];
            sums[2] = h[1];
            sums[3] = h[2];
        }
    });
}

int cam_bam_kernel_update(cam_ctx *ctx, const cam_grid *grid, int precision, double DeltaKmin, double ndel,
                          int nbins, const double *weight, int mode, void *kernel, int mem, double *kernel_binned,
                          int64_t *modes)
{
    return guarded(ctx, [&] {
        check_grid_cubic(grid);
        check_prec(precision);
        check_mem(mem);
        CAM_REQUIRE(weight && kernel, CAM_E_INVAL, "null weights or kernel");
        CAM_REQUIRE(mode == CAM_KERNEL_SET || mode == CAM_KERNEL_SCALE, CAM_E_INVAL, "unknown kernel update mode");
        CAM_REQUIRE(ndel > 0.0 && std::isfinite(ndel) && DeltaKmin >= 0.0 && std::isfinite(DeltaKmin), CAM_E_INVAL,
                    "invalid binning");
        CAM_REQUIRE(nbins >= 5, CAM_E_INVAL, "the kernel update needs nbins >= 5 (bin 0 is the mean of bins 1..4)");
        const int64_t n = grid->n[0];
        const size_t kbytes = (size_t)n * n * (n / 2 + 1) * esize(precision);
        void *dk = mem == CAM_MEM_DEVICE ? kernel : scratch(ctx, "bamk.kernel", kbytes);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync(dk, kernel, kbytes, cudaMemcpyHostToDevice, ctx->stream));
        auto *dw = static_cast<double *>(scratch(ctx, "bamk.w", (size_t)nbins * sizeof(double)));
        auto *dsum = static_cast<double *>(scratch(ctx, "bamk.sum", (size_t)nbins * sizeof(double)));
        auto *dmod = static_cast<unsigned long long *>(scratch(ctx, "bamk.modes", (size_t)nbins * 8));
        CAM_CUDA_TRY(cudaMemcpyAsync(dw, weight, (size_t)nbins * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        bam_kernel_update_device(ctx, dk, precision, n, grid->L[0], DeltaKmin, ndel, nbins, dw, mode, dsum, dmod);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync(kernel, dk, kbytes, cudaMemcpyDeviceToHost, ctx->stream));
        std::vector<double> hs(nbins);
        std::vector<unsigned long long> hm(nbins);
        CAM_CUDA_TRY(cudaMemcpyAsync(hs.data(), dsum, (size_t)nbins * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaMemcpyAsync(hm.data(), dmod, (size_t)nbins * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (kernel_binned) {
            // kernel_updated[b] /= nmodes[b]; then bin 0 = mean of bins 1..4
            for (int b = 0; b < nbins; ++b) kernel_binned[b] = hs[b] / (double)hm[b];
            kernel_binned[0] = (kernel_binned[1] + kernel_binned[2] + kernel_binned[3] + kernel_binned[4]) / 4.0;
        }
        if (modes)
            for (int b = 0; b < nbins; ++b) modes[b] = (int64_t)hm[b];
    });
}

int cam_konvolve(cam_ctx *ctx, const cam_grid *grid, const void *in, int precision, int mem, const void *kernel,
                 int kernel_mem, void *out, int out_mem)
{
    return guarded(ctx, [&] {
        check_grid_cubic(grid);
        CAM_REQUIRE(in && out && kernel, CAM_E_INVAL, "null mesh or kernel");
        check_prec(precision);
        check_mem(mem);
        check_mem(kernel_mem);
        check_mem(out_mem);
        const int64_t n = grid->n[0], ncell = n * n * n, nh = n * n * (n / 2 + 1);
        FftPlan *plan = get_plan(ctx, n, precision);
        const size_t bytes = (size_t)ncell * esize(precision), kbytes = (size_t)nh * esize(precision);
        const void *din = mem == CAM_MEM_DEVICE ? in : scratch(ctx, "fft.in", bytes);
        if (mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync((void *)din, in, bytes, cudaMemcpyHostToDevice, ctx->stream));
        const void *dk = kernel_mem == CAM_MEM_DEVICE ? kernel : scratch(ctx, "bamk.kernel", kbytes);
        if (kernel_mem == CAM_MEM_HOST)
            CAM_CUDA_TRY(cudaMemcpyAsync((void *)dk, kernel, kbytes, cudaMemcpyHostToDevice, ctx->stream));
        auto *dsum = static_cast<double *>(scratch(ctx, "bamk.ksum", 4 * sizeof(double)));
        mesh_mean(ctx, din, precision, ncell, dsum);     // [0] = sum of in
        mesh_mean(ctx, dk, precision, nh, dsum + 2);     // [2] = w, the kernel sum
        Spectrum s = alloc_spectrum(ctx, n, precision, "fft.spec");
        fft_r2c_split(ctx, plan, din, nullptr, s);
        konvolve_device(ctx, s, dk, dsum + 2);
        void *dout = out_mem == CAM_MEM_DEVICE ? out : scratch(ctx, "fd.out", bytes);
        fft_c2r_split(ctx, plan, s, dout, 1.0 / ((double)n * n * n));
        if (out_mem == CAM_MEM_HOST) CAM_CUDA_TRY(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        double hsum = 0.0;
        CAM_CUDA_TRY(cudaMemcpyAsync(&hsum, dsum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        CAM_REQUIRE(std::isfinite(hsum), CAM_E_NONFINITE, "Konvolve: the input mesh holds a non-finite value");
    });
}

int cam_particles_stage(cam_ctx *ctx, const cam_particles *host, cam_particles *device_out)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(host && device_out, CAM_E_INVAL, "null particles");
        CAM_REQUIRE(host->n >= 0, CAM_E_INVAL, "negative particle count");
        CAM_REQUIRE(host->n == 0 || (host->x && host->y && host->z), CAM_E_INVAL, "null particle coordinates");
        check_mem(host->mem);
        cam_particles d = *host;
        if (host->mem == CAM_MEM_HOST) {
            const size_t bytes = std::max<size_t>((size_t)host->n, 1) * sizeof(float);
            const float *src[4] = {host->x, host->y, host->z, host->w};
            const char *names[4] = {"stage.x", "stage.y", "stage.z", "stage.w"};
            float *dst[4] = {nullptr, nullptr, nullptr, nullptr};
            for (int a = 0; a < 4; ++a) {
                if (!src[a]) continue;
                dst[a] = static_cast<float *>(scratch(ctx, names[a], bytes));
                if (host->n > 0)
                    CAM_CUDA_TRY(cudaMemcpyAsync(dst[a], src[a], (size_t)host->n * sizeof(float),
                                                 cudaMemcpyHostToDevice, ctx->stream));
            }
            d.x = dst[0];
            d.y = dst[1];
            d.z = dst[2];
            d.w = dst[3];
            d.mem = CAM_MEM_DEVICE;
        }
        *device_out = d;
    });
}

int cam_job_run(cam_ctx *ctx, const cam_job_desc *job, cam_job_result *res)
{
    return guarded(ctx, [&] {
        CAM_REQUIRE(job && res, CAM_E_INVAL, "null job or result");
        check_grid_cubic(&job->grid);
        check_prec(job->precision);
        const bool want_pk = job->pk.nbins > 0 || job->pk.ndel > 0.0;
        if (want_pk) validate_pk(&job->pk);
        CAM_REQUIRE(!job->want_tweb || job->tweb.input_type != CAM_INPUT_POTENTIAL, CAM_E_INVAL,
                    "a job's T-web input is its density mesh");
        const cam_grid g = resolved_grid(job->grid);
        const int64_t n = g.n[0], ncell = n * n * n;
        const DevParticles d = stage_particles(ctx, &job->parts);
        FftPlan *plan = get_plan(ctx, n, job->precision);
        const int nb = want_pk ? nbins_for(job->pk, n) : 0;
        // Readback of one run: assignment statistics [6], mesh sum and mean
        // [2], P(k) sums [nb][2] and modes [nb], into a pinned buffer.
        const size_t pin_bytes = 6 * 8 + 2 * 8 + (size_t)nb * 24 + 8;
        if (ctx->job_pin_bytes < pin_bytes) {
            std::lock_guard<std::mutex> lk(alloc_mutex());
            if (ctx->job_pin) CAM_CUDA_TRY(cudaFreeHost(ctx->job_pin));
            ctx->job_pin = nullptr;
            ctx->job_pin_bytes = 0;
            CAM_CUDA_TRY(cudaHostAlloc(reinterpret_cast<void **>(&ctx->job_pin), pin_bytes, cudaHostAllocDefault));
            ctx->job_pin_bytes = pin_bytes;
        }
        auto *hstats = reinterpret_cast<unsigned long long *>(ctx->job_pin);
        auto *hsum = reinterpret_cast<double *>(ctx->job_pin + 48);
        auto *hpk = reinterpret_cast<double *>(ctx->job_pin + 64);
        auto *hmd = reinterpret_cast<unsigned long long *>(ctx->job_pin + 64 + (size_t)nb * 16);
        auto *herr = reinterpret_cast<unsigned *>(ctx->job_pin + 64 + (size_t)nb * 24);
        const unsigned *derr = device_error_word(ctx);
        // One run of the whole job.  defer: the assignment sizes its payload
        // from an estimate and nothing waits for the host until the single
        // readback at the end; returns true if the estimate fell short (the
        // results are then void and the job runs again without defer).
        auto run = [&](bool defer) -> bool {
            AssignOut out;
            out.precision = job->precision;
            out.mesh = scratch(ctx, "job.mesh", ncell * esize(job->precision));
            auto *dsum = static_cast<double *>(scratch(ctx, "job.sum", 2 * sizeof(double)));
            out.d_sum = dsum;
            out.defer = defer;
            assign_device(ctx, d.x, d.y, d.z, d.w, d.n, g, job->scheme, out);
            // FFT of rho - mean, mean from the deposit's exact per-brick sums.
            Spectrum s = alloc_spectrum(ctx, n, job->precision, "job.spec");
            const PkDevice pkd = job_fft_pk(ctx, plan, out.mesh, dsum + 1, s, want_pk ? &job->pk : nullptr, nb,
                                            job->want_tweb != 0);
            CAM_CUDA_TRY(cudaMemcpyAsync(hstats, assign_stats(ctx), 48, cudaMemcpyDeviceToHost, ctx->stream));
            CAM_CUDA_TRY(cudaMemcpyAsync(hsum, dsum, 16, cudaMemcpyDeviceToHost, ctx->stream));
            if (want_pk) {
                CAM_CUDA_TRY(cudaMemcpyAsync(hpk, pkd.sums, (size_t)nb * 16, cudaMemcpyDeviceToHost, ctx->stream));
                CAM_CUDA_TRY(cudaMemcpyAsync(hmd, pkd.modes, (size_t)nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
            }
            CAM_CUDA_TRY(cudaMemcpyAsync(herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
            CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            CAM_REQUIRE(*herr == 0u, CAM_E_CUDA, "a kernel's bulk copy did not complete within its wait limit");
            // An exact run measured its fullest brick: later deferred jobs
            // of this context and mesh shape size their slabs from it.
            const uint64_t bmax = defer ? (hstats[5] & 0xffffffffu) : out.brick_max;
            if (bmax && out.brick_est > 0.0) ctx->slab_clump[out.brick_shape] = slab_clump_of(bmax, out.brick_est);
            // a slab (or the payload estimate) was too small: an exact run,
            // which also measures the bricks again
            if (defer && (hstats[3] & 0xffffffffu)) return true;
            if (d.w) {
                const unsigned wbits = (unsigned)(hstats[1] & 0xffffffffu);
                CAM_REQUIRE(wbits < 0x7f800000u, CAM_E_NONFINITE, "a particle weight is NaN or infinite");
            }
            res->assign.n_lost = (int64_t)hstats[0];
            res->assign.n_in = d.n - res->assign.n_lost;
            res->assign.sum_mesh = hsum[0];
            if (want_pk) {
                std::vector<double> sr(nb), ss(nb);
                std::vector<int64_t> md(nb);
                for (int b = 0; b < nb; ++b) {
                    sr[b] = hpk[2 * b];
                    ss[b] = hpk[2 * b + 1];
                    md[b] = (int64_t)hmd[b];
                }
                finalize_pk(n, g.L[0], hsum[0], job->pk, nb, sr.data(), ss.data(), md.data(), res->pk, res->modes,
                            res->kvector, &res->pk_info);
            }
            if (job->want_tweb) {
                uint8_t *dl = res->labels ? static_cast<uint8_t *>(scratch(ctx, "tw.labels", ncell)) : nullptr;
                cam_tweb_opts to = job->tweb;
                tweb_device(ctx, plan, s, g.L[0], dsum + 1, to.input_type, to, dl, nullptr, &res->tweb);
                if (dl) {
                    CAM_CUDA_TRY(cudaMemcpyAsync(res->labels, dl, ncell, cudaMemcpyDeviceToHost, ctx->stream));
                    CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
                }
            }
            return false;
        };
        if (run(true)) run(false);
    });
}

}  // extern "C"

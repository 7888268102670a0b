// Power-spectrum binning that allocates no device memory.
//
// Callers that cannot call cudaMalloc -- code running under a memory pool
// they do not own, real-time loops that must not touch the allocator, hosts
// whose allocations go through a foreign arena -- still need P(k) of a
// spectrum they already hold on the device.  This entry point bins such a
// spectrum with all of its scratch (per-axis window tables, squared bin
// edges, per-CTA partial bins and the reduced bins) in one file-scope
// device array of fixed size, kNaScratchBytes (about 1.9 MB), that every GPU
// loading the library holds until the process exits.
//
// Limits: N <= kNaMaxN (2048) cells per side, nbins <= kNaMaxBins (512).
// All calls share the one array, and each call overwrites every word it
// reads, so nothing is cleared between calls; two calls that overlap on the
// GPU (different streams or threads) race on it and must be serialised by
// the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/cam.h"

namespace {

constexpr int kNaMaxN = 2048;
constexpr int kNaMaxBins = 512;
constexpr int kNaCtas = 148;
constexpr int kNaThreads = 256;
constexpr int kNaWarps = kNaThreads / 32;
constexpr int kNaMaxDevices = 64;

// Scratch layout (8-byte words):
//   tables   [2 (N/2 + 1) + nbins + 1]   1/W^2 per axis, C/W^2 per axis, E2
//   partials [kNaCtas][nbins][2]         per-CTA sums (|F|^2/W^2, C/W^2)
//   pmodes   [kNaCtas][nbins]            per-CTA mode counts
//   result   [nbins][2] + [nbins]        reduced sums and counts
constexpr size_t kTabWords = 2 * (kNaMaxN / 2 + 1) + kNaMaxBins + 1;
constexpr size_t kPartWords = (size_t)kNaCtas * kNaMaxBins * 2;
constexpr size_t kModeWords = (size_t)kNaCtas * kNaMaxBins;
constexpr size_t kResWords = (size_t)kNaMaxBins * 3;
constexpr size_t kNaScratchBytes = (kTabWords + kPartWords + kModeWords + kResWords) * 8;

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

std::mutex g_na_mu;
// Per device: the CUDA context the scratch address was looked up in, and the
// address.  A context that was torn down and created again (cudaDeviceReset)
// reloads the module, so the address is looked up again when the current
// context differs from the recorded one.
struct NaSlot {
    CUcontext ctx = nullptr;
    void *ptr = nullptr;
};
NaSlot g_na_slot[kNaMaxDevices];

__device__ __forceinline__ bool na_visited(int i, int j, int c, int n)
{
    // Elements the reference's octant loop visits (Source/FftwFunctions.cpp:1731-1869).
    const int h = n >> 1;
    if (i == h || j == h) return false;
    if (c > 0) return true;
    if (i == 0 && j == 0) return false;
    if (j > h) return false;
    if (i > h && j == 0) return false;
    return true;
}

__device__ __forceinline__ int na_bin(double q, const double *E2, int nbins, float m_u, float inv_s)
{
    int b = (int)floorf((sqrtf((float)q) - m_u) * inv_s);
    b = max(-1, min(b, nbins));
    for (int it = 0; it < 8 && b + 1 <= nbins && E2[b + 1] <= q; ++it) ++b;
    for (int it = 0; it < 8 && b >= 0 && E2[b] > q; ++it) --b;
    return b < 0 ? -1 : b;
}

// Spectrum in FFTW r2c layout [i][j][c <= N/2]; rows are split statically
// over the CTAs, each warp walks rows in order and reduces runs of equal
// bins with a fixed shuffle tree (the bin index grows with c).
template <typename C>
__global__ void __launch_bounds__(kNaThreads)
na_bin_kernel(const C *__restrict__ spec, int n, const double *__restrict__ g_tab, int nbins, float m_u,
              float inv_s, int64_t rows_per_cta, double *__restrict__ part, unsigned long long *__restrict__ pmodes)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int h = n / 2, M = h;
    double *tw2 = reinterpret_cast<double *>(smem_raw);
    double *tsn = tw2 + (h + 1);
    double *E2 = tsn + (h + 1);
    double *wsum = E2 + (nbins + 1);
    unsigned long long *wcnt = reinterpret_cast<unsigned long long *>(wsum + (size_t)kNaWarps * nbins * 2);
    for (int t = threadIdx.x; t < 2 * (h + 1) + nbins + 1; t += blockDim.x) tw2[t] = g_tab[t];
    for (int t = threadIdx.x; t < kNaWarps * nbins * 2; t += blockDim.x) wsum[t] = 0.0;
    for (int t = threadIdx.x; t < kNaWarps * nbins; t += blockDim.x) wcnt[t] = 0ull;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *mysum = wsum + (size_t)warp * nbins * 2;
    unsigned long long *mycnt = wcnt + (size_t)warp * nbins;
    const int64_t nrows = (int64_t)n * n;
    const int64_t r_beg = (int64_t)blockIdx.x * rows_per_cta;
    const int64_t r_end = min(nrows, r_beg + rows_per_cta);
    for (int64_t r = r_beg + warp; r < r_end; r += kNaWarps) {
        const int i = (int)(r / n), j = (int)(r % n);
        if (i == h || j == h) continue;
        const int a = i <= h ? i : n - i;
        const int b = j <= h ? j : n - j;
        const double tab_ab = tw2[a] * tw2[b];
        const double sn_ab = tsn[a] * tsn[b];
        const int64_t q0 = (int64_t)a * a + (int64_t)b * b;
        for (int c0 = 0; c0 <= M; c0 += 32) {
            const int c = c0 + lane;
            double vraw = 0.0, vsn = 0.0;
            unsigned long long vcnt = 0;
            int bin = nbins;
            if (c <= M) {
                const double q = (double)(q0 + (int64_t)c * c);
                bin = na_bin(q, E2, nbins, m_u, inv_s);
                if (bin >= 0 && bin < nbins && na_visited(i, j, c, n)) {
                    const C f = spec[r * (M + 1) + c];
                    const double re = (double)f.x, im = (double)f.y;
                    vraw = (re * re + im * im) * (tab_ab * tw2[c]);
                    vsn = sn_ab * tsn[c];
                    vcnt = 1;
                }
            }
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double o0 = __shfl_down_sync(0xffffffffu, vraw, off);
                const double o1 = __shfl_down_sync(0xffffffffu, vsn, off);
                const unsigned long long oc = __shfl_down_sync(0xffffffffu, vcnt, off);
                const int ob = __shfl_down_sync(0xffffffffu, bin, off);
                if (lane + off < 32 && ob == bin) {
                    vraw += o0;
                    vsn += o1;
                    vcnt += oc;
                }
            }
            const int prev = __shfl_up_sync(0xffffffffu, bin, 1);
            if ((lane == 0 || prev != bin) && bin >= 0 && bin < nbins && vcnt) {
                mysum[2 * bin] += vraw;
                mysum[2 * bin + 1] += vsn;
                mycnt[bin] += vcnt;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    for (int bn = threadIdx.x; bn < nbins; bn += blockDim.x) {
        double s0 = 0.0, s1 = 0.0;
        unsigned long long cn = 0;
        for (int w = 0; w < kNaWarps; ++w) {
            s0 += wsum[((size_t)w * nbins + bn) * 2];
            s1 += wsum[((size_t)w * nbins + bn) * 2 + 1];
            cn += wcnt[(size_t)w * nbins + bn];
        }
        part[((size_t)blockIdx.x * nbins + bn) * 2] = s0;
        part[((size_t)blockIdx.x * nbins + bn) * 2 + 1] = s1;
        pmodes[(size_t)blockIdx.x * nbins + bn] = cn;
    }
}

__global__ void __launch_bounds__(kNaThreads)
na_final_kernel(const double *__restrict__ part, const unsigned long long *__restrict__ pmodes, int nbins,
                double *__restrict__ res, unsigned long long *__restrict__ rmodes)
{
    __shared__ double r0[kNaThreads], r1[kNaThreads];
    __shared__ unsigned long long rc[kNaThreads];
    const int bn = blockIdx.x;
    double s0 = 0.0, s1 = 0.0;
    unsigned long long cn = 0;
    for (int p = threadIdx.x; p < kNaCtas; p += blockDim.x) {
        s0 += part[((size_t)p * nbins + bn) * 2];
        s1 += part[((size_t)p * nbins + bn) * 2 + 1];
        cn += pmodes[(size_t)p * nbins + bn];
    }
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    rc[threadIdx.x] = cn;
    __syncthreads();
    for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
        if (threadIdx.x < hh) {
            r0[threadIdx.x] += r0[threadIdx.x + hh];
            r1[threadIdx.x] += r1[threadIdx.x + hh];
            rc[threadIdx.x] += rc[threadIdx.x + hh];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        res[2 * bn] = r0[0];
        res[2 * bn + 1] = r1[0];
        rmodes[bn] = rc[0];
    }
}

double na_sq(int p, double s)
{
    switch (p) {
    case 0: return 1.0;
    case 1: return 1.0 - (2.0 / 3.0) * s * s;
    default: return 1.0 - s * s + (2.0 / 15.0) * s * s * s * s;
    }
}

// Status codes only: the entry point has no context to hold a message.
int na_fail(int code, const char *) { return code; }

// cuCtxGetCurrent through the runtime's driver entry point (the library does
// not link the driver library itself); null if unavailable.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
CtxGetCurrentFn ctx_get_current()
{
    static const CtxGetCurrentFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    return fn;
}

// Device address of the scratch array for the current device, looked up with
// cudaGetSymbolAddress the first time a device (in its current context) is
// used, then reused.  Without cuCtxGetCurrent the address is looked up on
// every call (cheap, and it allocates nothing).
int na_scratch(int dev, void **out)
{
    CUcontext cur = nullptr;
    const CtxGetCurrentFn get = ctx_get_current();
    const bool known = get && get(&cur) == CUDA_SUCCESS && cur;
    std::lock_guard<std::mutex> lk(g_na_mu);
    NaSlot &slot = g_na_slot[dev];
    if (!known || !slot.ptr || slot.ctx != cur) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return na_fail(CAM_E_CUDA, "cudaGetSymbolAddress of the no-allocation scratch failed");
        }
        slot.ptr = p;
        slot.ctx = known ? cur : nullptr;
    }
    *out = slot.ptr;
    return CAM_OK;
}

// The kernels' dynamic shared-memory limit on the current device is only
// ever raised: a concurrent call on another stream or thread may be about to
// launch with a larger size than this one.
cudaError_t raise_smem_limit(int precision, size_t smem)
{
    static std::mutex m;
    static size_t cur[2][64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return e != cudaSuccess ? e : cudaErrorInvalidDevice;
    const int p = precision == CAM_F32 ? 0 : 1;
    std::lock_guard<std::mutex> lk(m);
    if (cur[p][dev] >= smem) return cudaSuccess;
    e = p == 0 ? cudaFuncSetAttribute(na_bin_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
               : cudaFuncSetAttribute(na_bin_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) cur[p][dev] = smem;
    return e;
}

}  // namespace

extern "C" int cam_power_noalloc(const void *spec, int64_t n, int precision, float box, double n_obj,
                                 const cam_pk_opts *opts, double *pk, int64_t *modes, void *stream)
{
    if (!spec || !opts || !pk) return na_fail(CAM_E_INVAL, "null spectrum, options or output");
    if (n < 2 || n % 2 != 0) return na_fail(CAM_E_INVAL, "N must be even and >= 2");
    if (n > kNaMaxN) return na_fail(CAM_E_UNSUPPORTED, "N exceeds the no-allocation maximum of 2048 cells per side");
    if (precision != CAM_F32 && precision != CAM_F64) return na_fail(CAM_E_INVAL, "precision must be CAM_F32 or CAM_F64");
    if (!(box > 0.f) || !std::isfinite(box)) return na_fail(CAM_E_INVAL, "box side must be > 0");
    if (opts->scheme < 0 || opts->scheme > 2) return na_fail(CAM_E_INVAL, "unknown window scheme");
    if (!(opts->ndel > 0.0) || !std::isfinite(opts->ndel) || !std::isfinite(opts->DeltaKmin))
        return na_fail(CAM_E_INVAL, "bin width must be > 0");
    if (opts->input_type != CAM_INPUT_DENSITY && opts->input_type != CAM_INPUT_DELTA)
        return na_fail(CAM_E_INVAL, "unknown input type");
    if (opts->input_type == CAM_INPUT_DENSITY && !(n_obj > 0.0)) return na_fail(CAM_E_INVAL, "density input needs n_obj > 0");
    const int nbins = opts->nbins > 0 ? opts->nbins : (int)((double)n / opts->ndel / 2.0);
    if (nbins < 1) return na_fail(CAM_E_INVAL, "no bins");
    if (nbins > kNaMaxBins) return na_fail(CAM_E_UNSUPPORTED, "nbins exceeds the no-allocation maximum of 512");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) {
        cudaGetLastError();
        return na_fail(CAM_E_CUDA, "no current CUDA device");
    }
    // The host-to-device table copy and the final synchronisation cannot be
    // captured: refuse a capturing stream before touching it, so the
    // caller's capture stays valid.
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs) != cudaSuccess) {
            cudaGetLastError();
            return na_fail(CAM_E_CUDA, "cannot query the stream's capture state");
        }
        if (cs != cudaStreamCaptureStatusNone)
            return na_fail(CAM_E_UNSUPPORTED, "the stream is being captured; call outside a capture");
    }
    void *base = nullptr;
    if (int rc = na_scratch(dev, &base)) return rc;
    double *tab = static_cast<double *>(base);
    double *part = tab + kTabWords;
    auto *pm = reinterpret_cast<unsigned long long *>(part + kPartWords);
    double *res = reinterpret_cast<double *>(pm + kModeWords);
    auto *rmodes = reinterpret_cast<unsigned long long *>(res + 2 * kNaMaxBins);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Host tables on the stack (fixed maximum size).
    const int h = (int)(n / 2), p = opts->scheme;
    double htab[kTabWords];
    for (int a = 0; a <= h; ++a) {
        const double x = M_PI * (double)a / (double)n;
        const double sc = a == 0 ? 1.0 : std::sin(x) / x;
        double w = 1.0;
        if (opts->mas_correction)
            for (int e = 0; e < p + 1; ++e) w *= sc;
        const double iw2 = 1.0 / (w * w);
        htab[a] = iw2;
        htab[h + 1 + a] = (opts->sn_correction ? na_sq(p, std::sin(x)) : 1.0) * iw2;
    }
    for (int b = 0; b <= nbins; ++b) {
        volatile double e = opts->DeltaKmin + (double)b * opts->ndel;
        volatile double e2 = e * e;
        htab[2 * (h + 1) + b] = e2;
    }
    const size_t tab_bytes = (size_t)(2 * (h + 1) + nbins + 1) * sizeof(double);
    const size_t smem = tab_bytes + (size_t)kNaWarps * nbins * (2 * sizeof(double) + sizeof(unsigned long long));
    const int64_t rpc = ((int64_t)n * n + kNaCtas - 1) / kNaCtas;
    const float m_u = (float)opts->DeltaKmin, inv_s = (float)(1.0 / opts->ndel);
    cudaError_t e = cudaMemcpyAsync(tab, htab, tab_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = raise_smem_limit(precision, smem);
    if (e == cudaSuccess) {
        if (precision == CAM_F32) {
            na_bin_kernel<float2><<<kNaCtas, kNaThreads, smem, st>>>(static_cast<const float2 *>(spec), (int)n, tab,
                                                                         nbins, m_u, inv_s, rpc, part, pm);
        } else {
            na_bin_kernel<double2><<<kNaCtas, kNaThreads, smem, st>>>(static_cast<const double2 *>(spec), (int)n,
                                                                          tab, nbins, m_u, inv_s, rpc, part, pm);
        }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) {
        na_final_kernel<<<nbins, kNaThreads, 0, st>>>(part, pm, nbins, res, rmodes);
        e = cudaGetLastError();
    }
    double hres[2 * kNaMaxBins];
    unsigned long long hm[kNaMaxBins];
    if (e == cudaSuccess) e = cudaMemcpyAsync(hres, res, 2 * nbins * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hm, rmodes, nbins * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return CAM_E_CUDA;
    }
    // Normalisation of PowerSpectrumF::compute_power_spectrum_grid
    // (Source/PowerSpectrumF.cpp:1754-1783) and the final division of
    // FftwFunctions::power_spectrum (Source/FftwFunctions.cpp:1873-1874).
    const double vol = (double)box * box * box;
    const double ngal = opts->input_type == CAM_INPUT_DENSITY ? n_obj : 1.0;
    const double ncell = (double)n * n * n;
    const double normal = opts->input_type == CAM_INPUT_DENSITY ? ngal * ngal / vol : ncell * ncell / vol;
    const double sn = vol / ngal;
    for (int b = 0; b < nbins; ++b) {
        double v = 0.0;
        if (hm[b] > 0) {
            v = hres[2 * b] / ((double)hm[b] * normal);
            if (opts->sn_correction) v -= sn * hres[2 * b + 1] / (double)hm[b];
        }
        pk[b] = v;
        if (modes) modes[b] = (int64_t)hm[b];
    }
    return CAM_OK;
}

// BAM kernel: its per-iteration update from the P(k) ratio and the
// convolution of a mesh with it, the two steps that follow P(k) in every
// BAM calibration iteration.
//
//   bamk_update_kernel  Bam::GetKernel, Source/Bam.cpp:529-1025, its 3D part
//                       (:791-905): each element (i, j, k <= N/2) of the
//                       half-complex kernel array gets the bin
//                       b = floor((|k| - kmin) / DeltaK) and, for
//                       0 <= b < nbins, kernel = weight[b] (no rejection,
//                       :863-878) or kernel *= weight[b] (rejection, :829-850).
//                       The bin sums and mode counts of the updated kernel
//                       (kernel_updated, nmodes) come out in FP64.
//   konvolve_mult       Bam::Konvolve, Source/Bam.cpp:1027-1120:
//                       out = c2r(K * r2c(in)) / N^3 * 2 w / N^3, w = the
//                       sum of K over the half-complex array (:1078-1104).
//
// Bin arithmetic: the reference forms |k| with _get_modulo(x, y, z) =
// sqrt(x*x+y*y+z*z) (Headers/def.h:695) where x = coords[i]*deltak, so the
// unparenthesised macro multiplies coords[i]*deltak*coords[i]*deltak left to
// right; every step here is the same IEEE operation in real_prec (no
// contraction), so bins are identical to the reference's.  Along a row
// (fixed i, j) the bin is non-decreasing in k, and the bin sums use the same
// fixed-order warp runs as the P(k) kernel: deterministic, no atomics on
// floating-point values.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "cam_fft_device.cuh"
#include "cam_internal.h"

namespace cam {
namespace {

constexpr int kBkThreads = 256;
constexpr int kBkWarps = kBkThreads / 32;

template <typename T>
__device__ __forceinline__ T rmul(T a, T b);
template <>
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
template <>
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
template <typename T>
__device__ __forceinline__ T radd(T a, T b);
template <>
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
template <>
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rsqrt_(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double rsqrt_(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }

// floor((|k| - kmin) / DeltaK) for coords (ci, cj, ck) in real_prec T.
template <typename T>
__device__ __forceinline__ int bamk_bin(T ci, T cj, T ck, T dk, T kmin, T dK)
{
    const T tx = rmul(rmul(rmul(ci, dk), ci), dk);
    const T ty = rmul(rmul(rmul(cj, dk), cj), dk);
    const T tz = rmul(rmul(rmul(ck, dk), ck), dk);
    const T kv = rsqrt_(radd(radd(tx, ty), tz));
    const T q = rdiv(radd(kv, -kmin), dK);
    return (int)floor(q);
}

// One warp per row (i, j) of the half-complex kernel array (N/2 + 1
// elements, contiguous).  mode 0: K = w[b]; mode 1: K *= w[b].  Per-CTA
// partial bin sums of the updated K and mode counts go to part / part_modes.
template <typename T>
__global__ void __launch_bounds__(kBkThreads)
bamk_update_kernel(T *__restrict__ K, int n, const double *__restrict__ weight, int nbins, int mode, T dk, T kmin,
                   T dK, int64_t rows_per_cta, double *__restrict__ part, unsigned long long *__restrict__ part_modes)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *wsum = reinterpret_cast<double *>(smem_raw);  // [warps][nbins]
    unsigned long long *wcnt = reinterpret_cast<unsigned long long *>(wsum + (size_t)kBkWarps * nbins);
    for (int t = threadIdx.x; t < kBkWarps * nbins; t += blockDim.x) {
        wsum[t] = 0.0;
        wcnt[t] = 0ull;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *mysum = wsum + (size_t)warp * nbins;
    unsigned long long *mycnt = wcnt + (size_t)warp * nbins;
    const int h = n / 2, L1 = h + 1;
    const int64_t nrows = (int64_t)n * n;
    const int64_t r_beg = (int64_t)blockIdx.x * rows_per_cta;
    const int64_t r_end = min(nrows, r_beg + rows_per_cta);
    for (int64_t r = r_beg + warp; r < r_end; r += kBkWarps) {
        const int i = (int)(r / n), j = (int)(r - (int64_t)i * n);
        // coords[i] = i <= N/2 ? i : -(N - i)  (Source/Bam.cpp:791-796)
        const T ci = (T)(i <= h ? i : -(n - i)), cj = (T)(j <= h ? j : -(n - j));
        T *row = K + r * L1;
        for (int c0 = 0; c0 < L1; c0 += 32) {
            const int c = c0 + lane;
            double v = 0.0;
            int bin = nbins;
            if (c < L1) {
                bin = bamk_bin<T>(ci, cj, (T)c, dk, kmin, dK);
                if (bin >= 0 && bin < nbins) {
                    const T w = (T)__ldg(weight + bin);
                    const T nk = mode == 0 ? w : rmul(row[c], w);
                    row[c] = nk;
                    v = (double)nk;
                } else {
                    bin = bin < 0 ? -1 : nbins;
                }
            }
            // runs of equal bins are contiguous lanes: segmented sums with a
            // fixed shuffle tree, added once per run head
            const int prev = __shfl_up_sync(0xffffffffu, bin, 1);
            const bool head = lane == 0 || prev != bin;
            const unsigned heads = __ballot_sync(0xffffffffu, head);
            const unsigned later = heads & ~((2u << lane) - 1u);
            const int end = later ? __ffs((int)later) - 1 : 32;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double o = __shfl_down_sync(0xffffffffu, v, off);
                if (lane + off < end) v += o;
            }
            const bool valid = c < L1 && bin >= 0 && bin < nbins;
            const unsigned vmask = __ballot_sync(0xffffffffu, valid);
            const unsigned run = (end == 32 ? 0xffffffffu : ((1u << end) - 1u)) & ~((1u << lane) - 1u);
            const int cnt = __popc(vmask & run);
            if (head && bin >= 0 && bin < nbins && cnt) {
                mysum[bin] += v;
                mycnt[bin] += (unsigned long long)cnt;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    for (int bn = threadIdx.x; bn < nbins; bn += blockDim.x) {
        double s = 0.0;
        unsigned long long cn = 0;
        for (int w = 0; w < kBkWarps; ++w) {
            s += wsum[(size_t)w * nbins + bn];
            cn += wcnt[(size_t)w * nbins + bn];
        }
        part[(size_t)blockIdx.x * nbins + bn] = s;
        part_modes[(size_t)blockIdx.x * nbins + bn] = cn;
    }
}

// One CTA per bin: strided partial sums, then a fixed-shape tree.
__global__ void __launch_bounds__(256)
bamk_final_kernel(const double *__restrict__ part, const unsigned long long *__restrict__ pm, int nparts, int nbins,
                  double *__restrict__ out, unsigned long long *__restrict__ modes)
{
    __shared__ double r0[256];
    __shared__ unsigned long long rc[256];
    const int bn = blockIdx.x;
    double s = 0.0;
    unsigned long long cn = 0;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) {
        s += part[(size_t)p * nbins + bn];
        cn += pm[(size_t)p * nbins + bn];
    }
    r0[threadIdx.x] = s;
    rc[threadIdx.x] = cn;
    __syncthreads();
    for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
        if (threadIdx.x < hh) {
            r0[threadIdx.x] += r0[threadIdx.x + hh];
            rc[threadIdx.x] += rc[threadIdx.x + hh];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[bn] = r0[0];
        modes[bn] = rc[0];
    }
}

// F(i, j, k) *= K[(i N + j)(N/2 + 1) + k] * 2 w * s2, w = *d_w: the kernel
// product of Konvolve with the factor 2 w / N^3 of its normalisation folded
// in (s2 = 1 / N^3; the c2r applies the other 1 / N^3).  Loops over the
// kernel's half-complex order, so K is read contiguously.
template <typename T>
__global__ void konvolve_mult_kernel(typename fftdev::CT<T>::t *__restrict__ main_, typename fftdev::CT<T>::t *__restrict__ nyq,
                                     const T *__restrict__ K, int n, const double *__restrict__ d_w, double s2)
{
    using C = typename fftdev::CT<T>::t;
    const int M = n / 2, L1 = M + 1;
    const int64_t tot = (int64_t)n * n * L1;
    const T f = (T)(2.0 * (*d_w) * s2);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / L1;
        const int k = (int)(e - r * L1);
        C *p = k < M ? main_ + r * M + k : nyq + r;
        const T m = K[e] * f;
        const C v = *p;
        *p = C{v.x * m, v.y * m};
    }
}

template <typename T>
void bamk_update_impl(cam_ctx *ctx, void *kernel, int64_t n, float L, double kmin_u, double dK_u, int nbins,
                      const double *d_weight, int mode, double *d_sum, unsigned long long *d_modes)
{
    // Params::derived_pars, Source/Params.cpp:4092-4103: deltak = 2 pi / L and
    // kmin, DeltaK = (DeltaKmin, ndel) * deltak_0 in double, read back through
    // real_prec getters (Headers/Params.h:4326, :4350, :4363).
    const double deltak = 2.0 * M_PI / (double)L;
    const double dk2 = deltak * deltak;
    const double deltak0 = std::sqrt((dk2 + dk2) + dk2) / std::sqrt(3.0);
    const T dk = (T)deltak, kmin = (T)(kmin_u * deltak0), dK = (T)(dK_u * deltak0);
    const int64_t nrows = n * n;
    const int64_t target = (int64_t)kNumSMs * 4;
    const int64_t rpc = std::max<int64_t>(kBkWarps, (nrows + target - 1) / target);
    const int grid = (int)((nrows + rpc - 1) / rpc);
    auto *part = static_cast<double *>(scratch(ctx, "bamk.part", (size_t)grid * nbins * sizeof(double)));
    auto *pm = static_cast<unsigned long long *>(scratch(ctx, "bamk.pmodes", (size_t)grid * nbins * 8));
    const size_t smem = (size_t)kBkWarps * nbins * (sizeof(double) + 8);
    auto k = bamk_update_kernel<T>;
    smem_at_least(k, smem);
    CAM_LAUNCH_NAMED(ctx, "bamk_update", k, grid, kBkThreads, smem, static_cast<T *>(kernel), (int)n, d_weight, nbins,
                     mode, dk, kmin, dK, rpc, part, pm);
    CAM_LAUNCH(ctx, bamk_final_kernel, nbins, 256, 0, part, pm, grid, nbins, d_sum, d_modes);
}

}  // namespace

void bam_kernel_update_device(cam_ctx *ctx, void *kernel, int precision, int64_t n, float L, double kmin_u,
                              double dK_u, int nbins, const double *d_weight, int mode, double *d_sum,
                              unsigned long long *d_modes)
{
    CAM_REQUIRE(nbins > 0 && (size_t)kBkWarps * nbins * 16 <= 200 * 1024, CAM_E_UNSUPPORTED,
                "BAM kernel update: 1 <= nbins <= 1600");
    if (precision == CAM_F32)
        bamk_update_impl<float>(ctx, kernel, n, L, kmin_u, dK_u, nbins, d_weight, mode, d_sum, d_modes);
    else
        bamk_update_impl<double>(ctx, kernel, n, L, kmin_u, dK_u, nbins, d_weight, mode, d_sum, d_modes);
}

void konvolve_device(cam_ctx *ctx, Spectrum &s, const void *kernel, const double *d_w)
{
    const int64_t n = s.n;
    const int64_t tot = n * n * (n / 2 + 1);
    const unsigned g = (unsigned)std::min<int64_t>((tot + 255) / 256, (int64_t)kNumSMs * 8);
    const double s2 = 1.0 / ((double)n * (double)n * (double)n);
    if (s.precision == CAM_F32)
        CAM_LAUNCH(ctx, konvolve_mult_kernel<float>, g, 256, 0, static_cast<float2 *>(s.main),
                   static_cast<float2 *>(s.nyq), static_cast<const float *>(kernel), (int)n, d_w, s2);
    else
        CAM_LAUNCH(ctx, konvolve_mult_kernel<double>, g, 256, 0, static_cast<double2 *>(s.main),
                   static_cast<double2 *>(s.nyq), static_cast<const double *>(kernel), (int)n, d_w, s2);
}

}  // namespace cam

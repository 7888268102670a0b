// Potential and finite differences for the reference's default T-web
// variant (_USE_GFINDIFF_EIGENV_, Headers/def.h:2657).
//
//   poisson_device     PoissonSolver, Source/Miscelanious.cpp:1189-1275:
//                      phi_k = -delta_k / k^2 (k = 0 -> 0) on a spectrum in
//                      the split layout, times the Gaussian exp(-k^2 R^2 / 2)
//                      when R > 0 (kernelcomp, Source/NumericalMethods.cpp:2272).
//   gradfindif_device  gradfindif, Source/NumericalMethods.cpp:1123-1218: the
//                      4th-order centred difference along one axis, periodic,
//                      with the reference's own arithmetic (below), so FP32
//                      results are bit-identical to its loops.
//
// The T-web itself does not run these stencils: on a periodic mesh the
// centred difference is the Fourier multiplier i s(k), so the tidal tensor of
// finite differences is made by the separable T-web passes (cam_tweb.cu) with
// s(k) in place of k.  These two kernels serve callers of PoissonSolver and
// gradfindif themselves (LPT, Cwclass, the bias terms).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "cam_fft_device.cuh"
#include "cam_internal.h"

namespace cam {
namespace {

// One pass over the N*N*(N/2) main elements and the N*N Nyquist-plane
// elements (k = N/2) of the split spectrum.  m = -1/(k_f^2 q) exp(-g q),
// q = |f|^2 in units of k_f, formed in FP64 and rounded once to T.
template <typename T>
__global__ void poisson_kernel(typename fftdev::CT<T>::t *__restrict__ main_, typename fftdev::CT<T>::t *__restrict__ nyq,
                               int n, double inv_kf2, double gcoef)
{
    using C = typename fftdev::CT<T>::t;
    const int M = n / 2, h = n / 2;
    const int64_t nmain = (int64_t)n * n * M, ntot = nmain + (int64_t)n * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ntot; e += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
        C *p;
        if (e < nmain) {
            i = (int)(e / ((int64_t)n * M));
            const int64_t r = e - (int64_t)i * n * M;
            j = (int)(r / M);
            k = (int)(r - (int64_t)j * M);
            p = main_ + e;
        } else {
            const int64_t r = e - nmain;
            i = (int)(r / n);
            j = (int)(r - (int64_t)i * n);
            k = M;
            p = nyq + r;
        }
        const int fi = i <= h ? i : i - n, fj = j <= h ? j : j - n;
        const double q = (double)fi * fi + (double)fj * fj + (double)k * k;
        double m = 0.0;
        if (q > 0.0) {
            m = -inv_kf2 / q;
            if (gcoef > 0.0) m *= exp(-gcoef * q);
        }
        const T mt = (T)m;
        const C v = *p;
        *p = C{v.x * mt, v.y * mt};
    }
}

// out = (-in[+2] + 8.0 * in[+1] - 8.0 * in[-1] + in[-2]) * ideltaH along
// `stride` (N*N for dim 1 = x, N for dim 2 = y, 1 for dim 3 = z), periodic.
// The reference's real_prec loop evaluates this in double (8.0 is a double
// literal) and rounds to float on assignment; 8 * v is exact, so fused and
// unfused double arithmetic round alike, and the result matches its bits.
// Grid: x = rows (N*N), y = chunks of blockDim.x cells along z.
template <typename T>
__global__ void gradfindif_kernel(const T *__restrict__ in, T *__restrict__ out, int n, int64_t stride, double ideltaH)
{
    const int z = blockIdx.y * blockDim.x + threadIdx.x;
    if (z >= n) return;
    const int64_t row = blockIdx.x;
    const int64_t c = row * n + z;
    const int a = stride == 1 ? z : (int)((c / stride) % n);  // coordinate along the axis
    const int64_t base = c - (int64_t)a * stride;
    auto at = [&](int o) {
        int b = a + o;
        b += b < 0 ? n : 0;
        b -= b >= n ? n : 0;
        return (double)__ldg(in + base + (int64_t)b * stride);
    };
    const double v = ((-at(2) + 8.0 * at(1)) - 8.0 * at(-1)) + at(-2);
    out[c] = (T)(v * ideltaH);
}

}  // namespace

void poisson_device(cam_ctx *ctx, Spectrum &s, float L, float R)
{
    const int64_t n = s.n;
    const double kf = 2.0 * M_PI / (double)L;
    const double gcoef = R > 0.f ? 0.5 * kf * kf * (double)R * (double)R : 0.0;
    const int64_t tot = n * n * (n / 2 + 1);
    const unsigned g = (unsigned)std::min<int64_t>((tot + 255) / 256, (int64_t)kNumSMs * 8);
    if (s.precision == CAM_F32)
        CAM_LAUNCH(ctx, poisson_kernel<float>, g, 256, 0, static_cast<float2 *>(s.main), static_cast<float2 *>(s.nyq),
                   (int)n, 1.0 / (kf * kf), gcoef);
    else
        CAM_LAUNCH(ctx, poisson_kernel<double>, g, 256, 0, static_cast<double2 *>(s.main),
                   static_cast<double2 *>(s.nyq), (int)n, 1.0 / (kf * kf), gcoef);
}

void gradfindif_device(cam_ctx *ctx, const void *in, void *out, int64_t n, float L, int dim, int precision)
{
    const int64_t stride = dim == 1 ? n * n : (dim == 2 ? n : 1);
    // deltaH = 12.0 * (L1 / N1) and ideltaH = 1.0 / deltaH as the reference
    // rounds them: real_prec quotient, double products, real_prec results.
    double ideltaH;
    if (precision == CAM_F32) {
        const float d = L / (float)n;
        const float deltaH = (float)(12.0 * (double)d);
        ideltaH = (double)(float)(1.0 / (double)deltaH);
    } else {
        ideltaH = 1.0 / (12.0 * ((double)L / (double)n));
    }
    const int bx = (int)std::min<int64_t>(256, ((n + 31) / 32) * 32);
    dim3 grid((unsigned)(n * n), (unsigned)((n + bx - 1) / bx));
    if (precision == CAM_F32)
        CAM_LAUNCH(ctx, gradfindif_kernel<float>, grid, bx, 0, static_cast<const float *>(in), static_cast<float *>(out),
                   (int)n, stride, ideltaH);
    else
        CAM_LAUNCH(ctx, gradfindif_kernel<double>, grid, bx, 0, static_cast<const double *>(in),
                   static_cast<double *>(out), (int)n, stride, ideltaH);
}

}  // namespace cam

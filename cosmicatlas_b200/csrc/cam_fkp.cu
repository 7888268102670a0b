// Per-object weights of the catalogue interpolation with FKP weighting,
// Catalog.cpp's tracer loop, Source/Catalog.cpp:14120-14190:
//   w_i = (product of the object's weights) * 1 / (1 + P_est nbar_i)   (FKP on)
// and the four sums that give the estimator's normalisation and shot noise:
//   n_selected = N,  W_r = sum w,  S_r = sum w^2,  normal = sum nbar w^2.
// The weights feed the mass assignment (the reference passes them to
// grid_assignment_NGP/CIC/TSC, whose OpenMP loop races on the mesh under a
// no-op "#pragma atomic", :14178-14207; the deterministic assignment here
// has no such race).  Sums are FP64 in a fixed order: per-thread strided
// partials, a fixed tree per CTA, then one CTA over the CTA partials.
#include <cuda_runtime.h>

#include <algorithm>

#include "cam_internal.h"

namespace cam {
namespace {

constexpr int kFkpThreads = 256;
constexpr int kFkpBlocks = kNumSMs * 4;

__global__ void __launch_bounds__(kFkpThreads)
fkp_weights_kernel(int64_t n, const float *__restrict__ nbar, double nbar_const, const float *__restrict__ w_in,
                   int fkp, double pest, float *__restrict__ w_out, double *__restrict__ part /* [grid][3] */)
{
    __shared__ double red[3][kFkpThreads];
    double sw = 0.0, sw2 = 0.0, snw2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double nb = nbar ? (double)nbar[i] : nbar_const;
        double w = w_in ? (double)w_in[i] : 1.0;
        if (fkp) w *= 1.0 / (1.0 + pest * nb);
        w_out[i] = (float)w;
        sw += w;
        sw2 += w * w;
        snw2 += nb * w * w;
    }
    red[0][threadIdx.x] = sw;
    red[1][threadIdx.x] = sw2;
    red[2][threadIdx.x] = snw2;
    __syncthreads();
    for (int h = kFkpThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int a = 0; a < 3; ++a) red[a][threadIdx.x] += red[a][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < 3) part[(size_t)blockIdx.x * 3 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void __launch_bounds__(kFkpThreads)
fkp_final_kernel(const double *__restrict__ part, int nparts, double *__restrict__ out /* [3] */)
{
    __shared__ double red[3][kFkpThreads];
    double s[3] = {0.0, 0.0, 0.0};
    for (int p = threadIdx.x; p < nparts; p += blockDim.x)
        for (int a = 0; a < 3; ++a) s[a] += part[(size_t)p * 3 + a];
    for (int a = 0; a < 3; ++a) red[a][threadIdx.x] = s[a];
    __syncthreads();
    for (int h = kFkpThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int a = 0; a < 3; ++a) red[a][threadIdx.x] += red[a][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < 3) out[threadIdx.x] = red[threadIdx.x][0];
}

}  // namespace

void fkp_weights_device(cam_ctx *ctx, int64_t n, const float *nbar, double nbar_const, const float *w_in, int fkp,
                        double pest, float *w_out, double *d_sums)
{
    auto *part = static_cast<double *>(scratch(ctx, "fkp.part", (size_t)kFkpBlocks * 3 * sizeof(double)));
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(kFkpBlocks, (n + kFkpThreads - 1) / kFkpThreads));
    CAM_LAUNCH(ctx, fkp_weights_kernel, grid, kFkpThreads, 0, n, nbar, nbar_const, w_in, fkp, pest, w_out, part);
    CAM_LAUNCH(ctx, fkp_final_kernel, 1, kFkpThreads, 0, part, grid, d_sums);
}

}  // namespace cam

// Device helpers of the power-spectrum estimator shared by the binning
// kernels (cam_power.cu) and the FFT pass that bins its tiles as it
// transforms them (cam_fft.cu).  Mode set and binning of
// FftwFunctions::power_spectrum, Source/FftwFunctions.cpp:1660-1876.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cam {

// Elements (i, j, c) of the half spectrum the reference's octant loop visits:
// planes i = N/2 and j = N/2 never (loop bounds :1731, :1747); in the c = 0
// plane one element of each conjugate pair.
__device__ __forceinline__ bool pk_visited(int i, int j, int c, int n)
{
    const int h = n >> 1;
    if (i == h || j == h) return false;
    if (c > 0) return true;
    if (i == 0 && j == 0) return false;
    if (j > h) return false;
    if (i > h && j == 0) return false;
    return true;
}

// b with E2[b] <= q < E2[b+1]; -1 below the first edge, nbins at or above
// the last.  The initial FP32 estimate is refined by exact comparisons with
// the FP64 squared edges, so the result depends on E2 only.
__device__ __forceinline__ int pk_bin(double q, const double *E2, int nbins, float m_u, float inv_s)
{
    int b = (int)floorf((sqrtf((float)q) - m_u) * inv_s);
    b = max(-1, min(b, nbins));
#pragma unroll 1
    for (int it = 0; it < 8 && b + 1 <= nbins && E2[b + 1] <= q; ++it) ++b;
#pragma unroll 1
    for (int it = 0; it < 8 && b >= 0 && E2[b] > q; ++it) --b;
    return b < 0 ? -1 : b;  // b == nbins: above the last edge
}

}  // namespace cam

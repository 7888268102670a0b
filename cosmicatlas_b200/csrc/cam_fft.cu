// 3D real-to-complex / complex-to-real FFT for sm_100a.
//
// Replaces do_fftw_r2c / do_fftw_c2r, Source/NumericalMethods.cpp:1718-1856
// (a fresh FFTW_ESTIMATE plan per call there; here plans are built once per
// (N, precision) and hold only a twiddle table).
//
// Layout.  Spectra are kept in a "split" layout: main[N][N][N/2] complex
// (k < N/2) plus the Nyquist plane nyq[N][N] (k = N/2).  Every main row is
// N/2 complex, a multiple of 16 bytes, so column tiles are aligned 128-byte
// segments.  split_to_fftw / fftw_to_split convert to FFTW's [i][j][k<=N/2].
//
// Passes (each one HBM read + one HBM write of the array):
//   rows  : along z, real rows of N packed as N/2 complex, half-length
//           complex FFT plus the r2c untangling (or its inverse for c2r);
//   cols  : along y or x, tiles of 16 (float) / 8 (double) consecutive
//           columns x N rows staged in shared memory.
// Inside a CTA the 1D transforms are mixed-radix (16, 8, 4, 2, 3) Stockham
// stages in shared memory.  Each thread keeps its butterflies' inputs in
// registers across a barrier, so a stage reads and writes the same buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "cam_fft_device.cuh"
#include "cam_internal.h"
#include "cam_pk_device.cuh"
#include "cam_tma.cuh"

namespace cam {

struct FftPlan {
    int64_t n = 0;
    int precision = CAM_F32;
    void *tw = nullptr;  // n roots exp(-2 pi i m / n), float2 or double2
    Radices rad_n, rad_m;
};

namespace {

// Rows per CTA of the row kernels: about 4096 (float) / 2048 (double) points.
template <typename T>
constexpr int rows_rpc(int len)
{
    return (sizeof(T) == 4 ? 4096 : 2048) / len > 1 ? (sizeof(T) == 4 ? 4096 : 2048) / len : 1;
}

// Column transforms: element (comp, plane, j, col) at
// base + comp*ccomp + plane*pstride + j*jstride + col, col < ncols.
template <typename T, bool INV, int LEN>
__global__ void __launch_bounds__(1024, 1)
fft_cols_kernel(typename fftdev::CT<T>::t *base, int len, int ncols, int64_t jstride, int64_t pstride,
                int64_t ccomp, Radices rd, const typename fftdev::CT<T>::t *__restrict__ tw, int twmul)
{
    using C = typename fftdev::CT<T>::t;
    constexpr int W = fftdev::CT<T>::kCols;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tile = reinterpret_cast<C *>(smem_raw);
    const int col0 = blockIdx.x * W;
    const int nc = min(W, ncols - col0);
    C *g = base + (int64_t)blockIdx.z * ccomp + (int64_t)blockIdx.y * pstride + col0;
    const int tot = len * W;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const int j = e / W, c = e % W;
        if (c < nc) tile[e] = g[(int64_t)j * jstride + c];
    }
    __syncthreads();
    if constexpr (LEN > 0)
        fftdev::block_fft_fixed<C, INV, false, W, LEN, fftdev::ct_threads(LEN, W, fftdev::CT<T>::kPPT), W, 1, 1, false,
                                fftdev::CT<T>::kMaxR>(
            tile, tw);
    else
        fftdev::block_fft<C, fftdev::CT<T>::kPPT, INV, false, W>(tile, len, W, W, 1, rd, tw, twmul);
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const int j = e / W, c = e % W;
        if (c < nc) g[(int64_t)j * jstride + c] = tile[e];
    }
}

// Column transforms, persistent and double-buffered: each CTA walks the
// column tiles blockIdx.x, blockIdx.x + gridDim.x, ...; while it transforms
// one tile in shared memory, the next tile's rows are already on their way
// (asynchronous 16-byte copies), so the load latency that bounds the
// one-tile-per-CTA kernel overlaps the butterflies.  Full tiles only
// (ncols a multiple of W) and 16-byte aligned rows; the host checks.
// Tile t: column tile t % nct, plane (t / nct) % nplanes, component
// t / (nct * nplanes).
// CTAs per SM the pipelined column kernel is built for: as many as fit
// 1024 threads and two tiles each in 200 KB of shared memory.
template <typename T, int LEN>
constexpr int pipe_min_blocks()
{
    constexpr int nthr = fftdev::ct_threads(LEN, fftdev::CT<T>::kCols, fftdev::CT<T>::kPPT);
    constexpr int by_thr = 1024 / nthr;
    constexpr int by_smem = (200 * 1024) / (2 * LEN * fftdev::CT<T>::kCols * (int)sizeof(typename fftdev::CT<T>::t));
    constexpr int b = by_thr < by_smem ? by_thr : by_smem;
    return b > 1 ? b : 1;
}

template <typename T, bool INV, int LEN>
__global__ void __launch_bounds__(fftdev::ct_threads(LEN, fftdev::CT<T>::kCols, fftdev::CT<T>::kPPT),
                                  pipe_min_blocks<T, LEN>())
fft_cols_pipe_kernel(typename fftdev::CT<T>::t *base, int nct, int nplanes, int64_t ntiles, int64_t jstride,
                     int64_t pstride, int64_t ccomp, const typename fftdev::CT<T>::t *__restrict__ tw)
{
    using C = typename fftdev::CT<T>::t;
    constexpr int W = fftdev::CT<T>::kCols;
    constexpr int NTHR = fftdev::ct_threads(LEN, W, fftdev::CT<T>::kPPT);
    constexpr int CPR = W * (int)sizeof(C) / 16;  // 16-byte chunks per tile row
    constexpr int EPC = 16 / (int)sizeof(C);      // elements per chunk
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *const buf0 = reinterpret_cast<C *>(smem_raw);  // tiles at buf0 and buf0 + LEN * W
    auto tile_ptr = [&](int64_t t) {
        const int64_t ct = t % nct, r = t / nct;
        return base + (r / nplanes) * ccomp + (r % nplanes) * pstride + ct * W;
    };
    auto load = [&](int64_t t, C *dst) {
        const C *g = tile_ptr(t);
        for (int e = threadIdx.x; e < LEN * CPR; e += NTHR) {
            const int j = e / CPR, k = e % CPR;
            fftdev::cp_async16(dst + j * W + k * EPC, g + (int64_t)j * jstride + k * EPC);
        }
    };
    int cur = 0;
    int64_t t = blockIdx.x;
    if (t < ntiles) load(t, buf0);
    fftdev::cp_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        C *const here = buf0 + cur * (LEN * W), *const other = buf0 + (cur ^ 1) * (LEN * W);
        const int64_t tn = t + gridDim.x;
        if (tn < ntiles) load(tn, other);
        fftdev::cp_async_commit();
        fftdev::cp_async_wait<1>();  // this thread's copies of tile t have landed
        __syncthreads();     // ... and everyone's
        fftdev::block_fft_fixed<C, INV, false, W, LEN, NTHR, W, 1, 1, false, fftdev::CT<T>::kMaxR>(here, tw);
        C *g = tile_ptr(t);
        for (int e = threadIdx.x; e < LEN * W; e += NTHR) g[(int64_t)(e / W) * jstride + (e % W)] = here[e];
        __syncthreads();  // buf[cur] is refilled by the next iteration's prefetch
        cur ^= 1;
    }
    fftdev::cp_async_wait<0>();
}

// Column transforms staged by TMA: the persistent, double-buffered column
// pass with its tiles moved by the tensor memory accelerator.  One thread
// issues a tile's loads (boxes of 128-byte rows, at most 256 rows each) on
// the buffer's mbarrier; every thread waits on the mbarrier's phase, the
// block runs the Stockham stages in shared memory, and the same thread
// writes the transformed tile back with TMA stores.  A buffer is reloaded
// only after its previous tile's store has finished reading it.  The tensor
// map covers this GPU's own memory and the loads use no multicast.
// Coordinates: (scalar column 2 W ct, row, plane, component); tile t: column
// tile t % nct, plane (t / nct) % nplanes, component t / (nct * nplanes).
// err: set to 1 if a tile's copies did not land within the wait bound (the
// CTA then stops).
// The tensor map's dimensions 1..3 are (row, plane, component) in order of
// increasing stride; pos = p_row | p_plane << 2 | p_comp << 4 gives each
// one's dimension.
struct TileDims {
    int pos;
};
__device__ __forceinline__ void tile_coords(int pos, int row, int plane, int comp, int &c1, int &c2, int &c3)
{
    const int pr = pos & 3, pp = (pos >> 2) & 3;
    c1 = pr == 1 ? row : (pp == 1 ? plane : comp);
    c2 = pr == 2 ? row : (pp == 2 ? plane : comp);
    c3 = pr == 3 ? row : (pp == 3 ? plane : comp);
}

template <typename T, bool INV, int LEN>
__global__ void __launch_bounds__(fftdev::ct_threads(LEN, fftdev::CT<T>::kCols, fftdev::CT<T>::kPPT),
                                  pipe_min_blocks<T, LEN>())
fft_cols_tma_kernel(const __grid_constant__ CUtensorMap map, TileDims td, int nct, int nplanes, int64_t ntiles,
                    const typename fftdev::CT<T>::t *__restrict__ tw, unsigned *__restrict__ err)
{
    using C = typename fftdev::CT<T>::t;
    constexpr int W = fftdev::CT<T>::kCols;
    constexpr int NTHR = fftdev::ct_threads(LEN, W, fftdev::CT<T>::kPPT);
    constexpr int NBOX = (LEN + 255) / 256;  // boxes of BOXR rows (LEN is a multiple of NBOX)
    constexpr int BOXR = LEN / NBOX;
    constexpr unsigned TILE_BYTES = (unsigned)(LEN * W * sizeof(C));
    extern __shared__ __align__(128) unsigned char smem_tma[];
    __shared__ uint64_t bar[2];
    C *const buf0 = reinterpret_cast<C *>(smem_tma);
    const bool leader = threadIdx.x == 0;
    auto coords = [&](int64_t t, int &x, int &plane, int &comp) {
        const int64_t ct = t % nct, r = t / nct;
        x = (int)(ct * 2 * W);
        plane = (int)(r % nplanes);
        comp = (int)(r / nplanes);
    };
    auto issue_load = [&](int64_t t, int b) {
        int x, plane, comp;
        coords(t, x, plane, comp);
        tma::mbar_arrive_expect_tx(&bar[b], TILE_BYTES);
#pragma unroll
        for (int k = 0; k < NBOX; ++k) {
            int c1, c2, c3;
            tile_coords(td.pos, k * BOXR, plane, comp, c1, c2, c3);
            tma::load_4d(buf0 + b * (LEN * W) + k * BOXR * W, &map, x, c1, c2, c3, &bar[b]);
        }
    };
    if (leader) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_mbar_init();
    }
    __syncthreads();
    unsigned phase = 0;  // bit b: parity of buffer b's next completion
    int cur = 0;
    int64_t t = blockIdx.x;
    if (leader && t < ntiles) issue_load(t, 0);
    bool failed = false;
    for (; t < ntiles; t += gridDim.x) {
        C *const here = buf0 + cur * (LEN * W);
        const int64_t tn = t + gridDim.x;
        if (leader && tn < ntiles) {
            tma::bulk_wait_read0();  // the other buffer's last store has read its tile
            issue_load(tn, cur ^ 1);
        }
        const bool ok = tma::mbar_wait(&bar[cur], (phase >> cur) & 1u);
        phase ^= 1u << cur;
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        fftdev::block_fft_fixed<C, INV, false, W, LEN, NTHR, W, 1, 1, false, fftdev::CT<T>::kMaxR>(here, tw);
        tma::fence_proxy_async_smem();
        __syncthreads();
        if (leader) {
            int x, plane, comp;
            coords(t, x, plane, comp);
#pragma unroll
            for (int k = 0; k < NBOX; ++k) {
                int c1, c2, c3;
                tile_coords(td.pos, k * BOXR, plane, comp, c1, c2, c3);
                tma::store_4d(&map, x, c1, c2, c3, here + k * BOXR * W);
            }
            tma::bulk_commit();
        }
        cur ^= 1;
    }
    if (leader) {
        if (failed) {
            atomicOr(err, 1u);
            // the prefetch of the next tile may still be in flight: give it
            // the same bound before the shared memory is released
            const int64_t tn = t + gridDim.x;
            if (tn < ntiles) tma::mbar_wait(&bar[cur ^ 1], (phase >> (cur ^ 1)) & 1u);
        }
        tma::bulk_wait0();
    }
}

// The x pass of the r2c with the P(k) binning of its tiles (FP32 spectra):
// the TMA column pass above, and after a tile's transform -- while its TMA
// store (if any) reads the tile -- the block bins the tile's modes.  Tile:
// 16 consecutive k (c0 .. c0 + 15) of all rows i, plane j.  A warp takes two
// rows at a time (16 lanes each); along a row the bin is non-decreasing in
// c, so runs of equal bins are contiguous lanes (bins from the table of
// every |k|^2), reduced by a fixed shuffle tree and added by their head lane into the warp's own FP64 bins, the
// first row's heads before the second's.  Warps and tiles are combined in a
// fixed order: part[cta][bin] = this CTA's sum of |F|^2 / W^2.  Mode counts
// and shot-noise sums do not depend on the data; the host takes them from a
// table.  store = 0: the transformed tiles are not written back (a job that
// needs only P(k)).
// Columns per tile: 16 (128-byte rows); 8 from N = 768 on, where two
// 16-column tiles and the warps' bins would not fit one CTA's shared memory
// (8 at N = 512, for two CTAs per SM, measured 0.585 -> 0.600 ms).
template <int LEN>
constexpr int pk_pass_cols()
{
    return LEN >= 768 ? 8 : 16;
}
template <int LEN>
constexpr int pk_pass_threads()
{
    return fftdev::ct_threads(LEN, pk_pass_cols<LEN>(), 16);
}
// CTAs per SM the binning pass is built for: two tiles plus the tables and
// warp bins of N/2 bins in 222 KB (the SM's 228 KB less 1 KB per CTA), at
// most 1024 threads: three CTAs of 80 registers at N = 256 (24 warps per SM
// to hide the binning's latencies), one at 512.
template <int LEN>
constexpr int pk_pass_min_blocks()
{
    constexpr int nthr = pk_pass_threads<LEN>();
    constexpr int by_thr = 1024 / nthr;
    constexpr int bytes = 2 * LEN * pk_pass_cols<LEN>() * 8 + (nthr / 32) * (LEN / 2) * 8 + (LEN / 2 + 1) * 4;
    constexpr int by_smem = (222 * 1024) / bytes;
    constexpr int b = by_thr < by_smem ? by_thr : by_smem;
    return b > 1 ? b : 1;
}

template <int LEN>
__global__ void __launch_bounds__(pk_pass_threads<LEN>(), pk_pass_min_blocks<LEN>())
fft_cols_tma_pk_kernel(const __grid_constant__ CUtensorMap map, TileDims td, int nct, int nplanes, int64_t ntiles,
                       const float2 *__restrict__ tw, unsigned *__restrict__ err,
                       const double *__restrict__ g_tab /* [h+1] 1/W^2, [h+1] C/W^2, [nbins+1] E2 */, int nbins,
                       const short *__restrict__ btab /* bin of q = |k|^2 / k_f^2 */, int store,
                       double *__restrict__ part /* [grid][nbins] */)
{
    using C = float2;
    constexpr int W = pk_pass_cols<LEN>();
    constexpr int RPW = 32 / W;  // rows a warp bins at a time
    constexpr int NTHR = pk_pass_threads<LEN>();
    constexpr int NWARP = NTHR / 32;
    constexpr int NBOX = (LEN + 255) / 256;
    constexpr int BOXR = LEN / NBOX;
    constexpr unsigned TILE_BYTES = (unsigned)(LEN * W * sizeof(C));
    constexpr int N = LEN, H = LEN / 2;
    extern __shared__ __align__(128) unsigned char smem_tma[];
    __shared__ uint64_t bar[2];
    C *const buf0 = reinterpret_cast<C *>(smem_tma);
    double *const wsum = reinterpret_cast<double *>(smem_tma + 2 * (size_t)TILE_BYTES);  // [NWARP][nbins]
    float *const tw2 = reinterpret_cast<float *>(wsum + (size_t)NWARP * nbins);         // [H + 1]
    for (int t = threadIdx.x; t <= H; t += NTHR) tw2[t] = (float)g_tab[t];
    for (int t = threadIdx.x; t < NWARP * nbins; t += NTHR) wsum[t] = 0.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *const mysum = wsum + (size_t)warp * nbins;
    const bool leader = threadIdx.x == 0;
    auto coords = [&](int64_t t, int &x, int &plane, int &comp) {
        const int64_t ct = t % nct, r = t / nct;
        x = (int)(ct * 2 * W);
        plane = (int)(r % nplanes);
        comp = (int)(r / nplanes);
    };
    auto issue_load = [&](int64_t t, int b) {
        int x, plane, comp;
        coords(t, x, plane, comp);
        tma::mbar_arrive_expect_tx(&bar[b], TILE_BYTES);
#pragma unroll
        for (int k = 0; k < NBOX; ++k) {
            int c1, c2, c3;
            tile_coords(td.pos, k * BOXR, plane, comp, c1, c2, c3);
            tma::load_4d(buf0 + b * (LEN * W) + k * BOXR * W, &map, x, c1, c2, c3, &bar[b]);
        }
    };
    if (leader) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_mbar_init();
    }
    __syncthreads();
    unsigned phase = 0;
    int cur = 0;
    int64_t t = blockIdx.x;
    if (leader && t < ntiles) issue_load(t, 0);
    bool failed = false;
    for (; t < ntiles; t += gridDim.x) {
        C *const here = buf0 + cur * (LEN * W);
        const int64_t tn = t + gridDim.x;
        if (leader && tn < ntiles) {
            tma::bulk_wait_read0();
            issue_load(tn, cur ^ 1);
        }
        const bool ok = tma::mbar_wait(&bar[cur], (phase >> cur) & 1u);
        phase ^= 1u << cur;
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        fftdev::block_fft_fixed<C, false, false, W, LEN, NTHR, W, 1, 1, false, 16>(here, tw);
        int x, plane, comp;
        coords(t, x, plane, comp);
        if (store) {
            tma::fence_proxy_async_smem();
            __syncthreads();
            if (leader) {
#pragma unroll
                for (int k = 0; k < NBOX; ++k) {
                    int c1, c2, c3;
                    tile_coords(td.pos, k * BOXR, plane, comp, c1, c2, c3);
                    tma::store_4d(&map, x, c1, c2, c3, here + k * BOXR * W);
                }
                tma::bulk_commit();
            }
        }
        // bin the tile: plane = j, columns c0 .. c0 + W - 1.  A mode's
        // |F|^2 / W^2 is formed in FP32 (one rounding per factor, ~2e-7)
        // and summed over its run of at most W lanes in FP32; each run's
        // sum is added to the warp's FP64 bin, the rows' heads one row at a
        // time (two rows' runs may share a bin).
        const int j = plane, c0 = x / 2;
        if (j != H) {
            const int b = j <= H ? j : N - j;
            const int kk = lane % W;
            const int c = c0 + kk;
            const int qbc = b * b + c * c;
            const float wbc = tw2[b] * tw2[c];
            for (int pr = warp; pr < LEN / RPW; pr += NWARP) {
                const int i = RPW * pr + lane / W;
                const int a = i <= H ? i : N - i;
                const int bin = __ldg(btab + (a * a + qbc));
                float v = 0.0f;
                if (bin >= 0 && bin < nbins && pk_visited(i, j, c, N)) {
                    const C f = here[i * W + kk];
                    v = (f.x * f.x + f.y * f.y) * (tw2[a] * wbc);
                }
                const int prev = __shfl_up_sync(0xffffffffu, bin, 1);
                const bool head = kk == 0 || prev != bin;
                const unsigned heads = __ballot_sync(0xffffffffu, head);
                const unsigned later = heads & ~((2u << lane) - 1u);
                const int end = later ? __ffs((int)later) - 1 : 32;
#pragma unroll
                for (int off = 1; off < W; off <<= 1) {
                    const float o = __shfl_down_sync(0xffffffffu, v, off);
                    if (lane + off < end) v += o;
                }
                const bool add = head && bin >= 0 && bin < nbins;
#pragma unroll
                for (int r = 0; r < RPW; ++r) {
                    if (add && lane / W == r) mysum[bin] += (double)v;
                    __syncwarp();
                }
            }
        }
        __syncthreads();  // the tile is reloaded two iterations on
        cur ^= 1;
    }
    if (leader) {
        if (failed) {
            atomicOr(err, 1u);
            const int64_t tn = t + gridDim.x;
            if (tn < ntiles) tma::mbar_wait(&bar[cur ^ 1], (phase >> (cur ^ 1)) & 1u);
        }
        tma::bulk_wait0();
    }
    __syncthreads();
    for (int bn = threadIdx.x; bn < nbins; bn += NTHR) {
        double sum = 0.0;
        for (int w = 0; w < NWARP; ++w) sum += wsum[(size_t)w * nbins + bn];
        part[(size_t)blockIdx.x * nbins + bn] = sum;
    }
}

// Row transforms along the contiguous axis.
//   MODE 0 (r2c): real rows of n -> main rows of n/2 + nyq element
//   MODE 1 (c2r): main rows + nyq -> real rows of n (times `scale`)
//   MODE 2/3    : complex rows of n, forward / inverse, in place
template <typename T, int MODE, int LEN>
__global__ void __launch_bounds__(1024, 1)
fft_rows_kernel(const void *in, void *out_main, typename fftdev::CT<T>::t *nyq, int n, int64_t nrows,
                int rpc, int64_t ccomp_in, int64_t ccomp_out, Radices rd,
                const typename fftdev::CT<T>::t *__restrict__ tw, const double *__restrict__ d_sub,
                double scale)
{
    using C = typename fftdev::CT<T>::t;
    constexpr bool INV = (MODE == 1 || MODE == 3);
    constexpr bool PAD = LEN > 0;  // row tiles of the compile-time transforms are padded
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tile = reinterpret_cast<C *>(smem_raw);  // element e at slot sidx<PAD>(e)
    auto at = [&](int e) -> C & { return tile[fftdev::sidx<PAD>(e)]; };
    // With a compile-time length, row length, M and rows per CTA are
    // constants (the host passes the same values): index divisions become
    // multiplies.
    const int len = LEN > 0 ? LEN : ((MODE <= 1) ? n / 2 : n);
    const int M = LEN > 0 ? ((MODE <= 1) ? LEN : LEN / 2) : n / 2;
    const int rpcv = LEN > 0 ? rows_rpc<T>(LEN) : rpc;
    const int64_t row0 = (int64_t)blockIdx.x * rpcv;
    const int nr = (int)min((int64_t)rpcv, nrows - row0);
    const int tot = nr * len;
    const int64_t comp = blockIdx.y;

    if (MODE == 0) {
        const C *src = reinterpret_cast<const C *>(static_cast<const T *>(in) + comp * ccomp_in) + row0 * M;
        const T sub = d_sub ? (T)(*d_sub) : (T)0;
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            C v = src[e];
            v.x -= sub;
            v.y -= sub;
            at(e) = v;
        }
    } else if (MODE == 1) {
        const C *srcm = static_cast<const C *>(in) + comp * ccomp_in + row0 * M;
        const C *srcn = nyq + comp * (ccomp_in / M) + row0;  // nyq plane is N*N per component
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            const int r = e / M, k = e % M;
            C xk = srcm[(int64_t)r * M + k];
            C xm = (k == 0) ? srcn[r] : srcm[(int64_t)r * M + (M - k)];
            if (k == 0) {  // imaginary parts of DC and Nyquist are ignored
                xk.y = 0;
                xm.y = 0;
            }
            // Z'[k] = X[k] + conj(X[M-k]) + i e^{+2 pi i k/n} (X[k] - conj(X[M-k]))
            const C a = C{xk.x + xm.x, xk.y - xm.y};
            const C b = C{xk.x - xm.x, xk.y + xm.y};
            C wv = __ldg(tw + k);
            wv.y = -wv.y;
            const C ib = fftdev::rot<C, true>(fftdev::cmul(wv, b));
            at(e) = fftdev::cadd(a, ib);
        }
    } else {
        const C *src = static_cast<const C *>(in) + comp * ccomp_in + row0 * n;
        for (int e = threadIdx.x; e < tot; e += blockDim.x) at(e) = src[e];
    }
    __syncthreads();
    if constexpr (LEN > 0) {
        // all rpc rows (the unused ones of the last CTA hold garbage and are not stored)
        constexpr int RPC = rows_rpc<T>(LEN);
        fftdev::block_fft_fixed<C, INV, true, RPC, LEN, fftdev::ct_threads(LEN, RPC, fftdev::CT<T>::kPPT), 1, LEN,
                                (MODE <= 1) ? 2 : 1, PAD, fftdev::CT<T>::kMaxR>(tile, tw);
    } else {
        fftdev::block_fft<C, fftdev::CT<T>::kPPT, INV, true, 0>(tile, len, nr, 1, len, rd, tw, (MODE <= 1) ? 2 : 1);
    }

    if (MODE == 0) {
        C *dm = static_cast<C *>(out_main) + comp * ccomp_out + row0 * M;
        C *dn = nyq + comp * (ccomp_out / M) + row0;
        const int tot2 = nr * (M + 1);
        for (int e = threadIdx.x; e < tot2; e += blockDim.x) {
            const int r = e / (M + 1), k = e % (M + 1);
            const C zk = at(r * M + (k % M));
            const C zc0 = at(r * M + ((M - k) % M));
            const C zc = C{zc0.x, -zc0.y};
            // X[k] = (Z[k] + conj Z[M-k])/2 - i/2 e^{-2 pi i k/n} (Z[k] - conj Z[M-k])
            const C s = fftdev::cadd(zk, zc), d = fftdev::csub(zk, zc);
            const C wd = fftdev::cmul(__ldg(tw + k), d);
            const C xk = C{(T)0.5 * (s.x + wd.y), (T)0.5 * (s.y - wd.x)};
            if (k < M) dm[(int64_t)r * M + k] = xk;
            else dn[r] = xk;
        }
    } else if (MODE == 1) {
        T *dst = static_cast<T *>(out_main) + comp * ccomp_out + row0 * n;
        const T sc = (T)scale;
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            const C v = at(e);
            reinterpret_cast<C *>(dst)[e] = C{v.x * sc, v.y * sc};
        }
    } else {
        C *dst = static_cast<C *>(out_main) + comp * ccomp_out + row0 * n;
        for (int e = threadIdx.x; e < tot; e += blockDim.x) dst[e] = at(e);
    }
}

// r2c rows (mode 0 of fft_rows_kernel), persistent and pipelined, for one
// component and a compile-time half length LEN: CTAs walk the groups of
// rows_rpc rows blockIdx.x, blockIdx.x + gridDim.x, ...  A group's raw rows
// are consumed when they are copied (minus the mean) into the padded work
// tile, so the next group's copy into the raw buffer starts right after and
// runs while the group is transformed and untangled.
template <typename T, int LEN>
__global__ void __launch_bounds__(fftdev::ct_threads(LEN, rows_rpc<T>(LEN), fftdev::CT<T>::kPPT), 2)
fft_rows_r2c_pipe_kernel(const T *__restrict__ in, typename fftdev::CT<T>::t *__restrict__ out_main,
                         typename fftdev::CT<T>::t *__restrict__ nyq, int64_t nrows,
                         const typename fftdev::CT<T>::t *__restrict__ tw, const double *__restrict__ d_sub)
{
    using C = typename fftdev::CT<T>::t;
    constexpr int M = LEN;
    constexpr int RPC = rows_rpc<T>(LEN);
    constexpr int RAW = RPC * M;
    constexpr int NTHR = fftdev::ct_threads(LEN, RPC, fftdev::CT<T>::kPPT);
    constexpr int EPC = 16 / (int)sizeof(C);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *const raw = reinterpret_cast<C *>(smem_raw);
    C *const tile = raw + RAW;  // element e at slot sidx<true>(e)
    const C *src = reinterpret_cast<const C *>(in);
    const T sub = d_sub ? (T)(*d_sub) : (T)0;
    const int64_t ngroups = (nrows + RPC - 1) / RPC;
    auto load = [&](int64_t gi) {
        const int64_t row0 = gi * RPC;
        const int tot = (int)min((int64_t)RPC, nrows - row0) * M;
        for (int e = threadIdx.x * EPC; e < tot; e += NTHR * EPC) fftdev::cp_async16(raw + e, src + row0 * M + e);
    };
    int64_t gi = blockIdx.x;
    if (gi < ngroups) load(gi);
    fftdev::cp_async_commit();
    for (; gi < ngroups; gi += gridDim.x) {
        fftdev::cp_async_wait<0>();
        __syncthreads();
        const int64_t row0 = gi * RPC;
        const int nr = (int)min((int64_t)RPC, nrows - row0);
        for (int e = threadIdx.x; e < nr * M; e += NTHR) {
            C v = raw[e];
            v.x -= sub;
            v.y -= sub;
            tile[fftdev::sidx<true>(e)] = v;
        }
        __syncthreads();  // raw is consumed: fetch the next group behind the transform
        const int64_t gn = gi + gridDim.x;
        if (gn < ngroups) load(gn);
        fftdev::cp_async_commit();
        // all RPC rows (the unused ones of the last group hold stale data and are not stored)
        fftdev::block_fft_fixed<C, false, true, RPC, LEN, NTHR, 1, LEN, 2, true, fftdev::CT<T>::kMaxR>(tile, tw);
        C *dm = out_main + row0 * M;
        C *dn = nyq + row0;
        for (int e = threadIdx.x; e < nr * (M + 1); e += NTHR) {
            const int r = e / (M + 1), k = e % (M + 1);
            const C zk = tile[fftdev::sidx<true>(r * M + (k % M))];
            const C zc0 = tile[fftdev::sidx<true>(r * M + ((M - k) % M))];
            const C zc = C{zc0.x, -zc0.y};
            // X[k] = (Z[k] + conj Z[M-k])/2 - i/2 e^{-2 pi i k/n} (Z[k] - conj Z[M-k])
            const C s = fftdev::cadd(zk, zc), d = fftdev::csub(zk, zc);
            const C wd = fftdev::cmul(__ldg(tw + k), d);
            const C xk = C{(T)0.5 * (s.x + wd.y), (T)0.5 * (s.y - wd.x)};
            if (k < M) dm[(int64_t)r * M + k] = xk;
            else dn[r] = xk;
        }
        __syncthreads();  // tile is refilled next
    }
    fftdev::cp_async_wait<0>();
}

template <typename T>
__global__ void split_to_fftw_kernel(const typename fftdev::CT<T>::t *__restrict__ main,
                                     const typename fftdev::CT<T>::t *__restrict__ nyq,
                                     typename fftdev::CT<T>::t *__restrict__ dst, int64_t nrows, int M)
{
    const int64_t tot = nrows * (M + 1);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / (M + 1);
        const int k = (int)(e % (M + 1));
        dst[e] = k < M ? main[r * M + k] : nyq[r];
    }
}

template <typename T>
__global__ void fftw_to_split_kernel(const typename fftdev::CT<T>::t *__restrict__ src,
                                     typename fftdev::CT<T>::t *__restrict__ main,
                                     typename fftdev::CT<T>::t *__restrict__ nyq, int64_t nrows, int M)
{
    const int64_t tot = nrows * (M + 1);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / (M + 1);
        const int k = (int)(e % (M + 1));
        if (k < M) main[r * M + k] = src[e];
        else nyq[r] = src[e];
    }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// Dimensions of a column-tile tensor map: dim 0 the scalar columns, then
// (row, plane, component) sorted by increasing byte stride (a component
// count of 1 gets a stride past the others); box: bw scalars x brows rows.
// pos receives each one's dimension (see tile_coords).
void tile_map_layout(int64_t ncol_scalars, int64_t nrows, int64_t rstride, int64_t nplanes, int64_t pstride,
                     int64_t ncomp, int64_t cstride, uint32_t bw, uint32_t brows, uint64_t dims[4],
                     uint64_t strides[3], uint32_t box[4], int &pos)
{
    struct D {
        int role;  // 0 row, 1 plane, 2 component
        int64_t n, st;
    } d[3] = {{0, nrows, rstride}, {1, nplanes, pstride}, {2, ncomp, cstride}};
    if (ncomp == 1) d[2].st = std::max(rstride * nrows, pstride * nplanes);
    if (nplanes == 1) d[1].st = std::max(rstride * nrows, d[2].st * ncomp) + 16;
    std::sort(d, d + 3, [](const D &a, const D &b) { return a.st < b.st; });
    dims[0] = (uint64_t)ncol_scalars;
    box[0] = bw;
    pos = 0;
    for (int i = 0; i < 3; ++i) {
        dims[i + 1] = (uint64_t)d[i].n;
        strides[i] = (uint64_t)((d[i].st + 15) / 16 * 16);
        box[i + 1] = d[i].role == 0 ? brows : 1u;
        pos |= (i + 1) << (2 * d[i].role);
    }
}

int threads_for(int points, int ppt)
{
    int t = (points + ppt - 1) / ppt;
    t = ((t + 31) / 32) * 32;
    return std::max(32, std::min(1024, t));
}

template <typename T>
void cols_impl(cam_ctx *ctx, FftPlan *p, void *base, int64_t len, int64_t ncols, int64_t jstride,
               int64_t nplanes, int64_t pstride, int ncomp, int64_t ccomp, bool inv)
{
    using C = typename fftdev::CT<T>::t;
    constexpr int W = fftdev::CT<T>::kCols;
    const Radices &rd = (len == p->n) ? p->rad_n : p->rad_m;
    const int twmul = (int)(p->n / len);
    const int nthr = threads_for((int)len * W, fftdev::CT<T>::kPPT);  // == ct_threads for compiled lengths
    const size_t smem = (size_t)len * W * sizeof(C);
    dim3 grid((unsigned)((ncols + W - 1) / W), (unsigned)nplanes, (unsigned)ncomp);
    // persistent double-buffered kernel: compile-time length, full tiles,
    // 16-byte aligned rows, two tiles within 200 KB of shared memory
    const size_t es = sizeof(C);
    const bool pipe_ok = ncols % W == 0 && (jstride * es) % 16 == 0 && (pstride * es) % 16 == 0 &&
                         (ccomp * es) % 16 == 0 && ((uintptr_t)base % 16) == 0 && 2 * smem <= 200 * 1024 &&
                         (int64_t)nplanes * ncomp * (ncols / W) < (1ll << 40);
    dispatch_fft_len(len, [&](auto lc) {
        constexpr int LEN = decltype(lc)::value;
        if constexpr (LEN > 0 && 2 * LEN * W * sizeof(C) <= 200 * 1024) {
            // TMA tiles: 128-byte rows of a 4D view (scalar column, row,
            // plane, component) of this GPU's own array
            CUtensorMap map;
            TileDims td{0};
            uint64_t dims[4], strides[3];
            uint32_t box[4];
            tile_map_layout(2 * ncols, len, jstride * es, nplanes, pstride * es, ncomp, ccomp * es,
                            (uint32_t)(2 * W), (uint32_t)(LEN / ((LEN + 255) / 256)), dims, strides, box, td.pos);
            if (pipe_ok && !ctx->no_tma &&
                make_tensor_map_4d(&map, sizeof(T) == 8, base, dims, strides, box)) {
                auto kt = inv ? fft_cols_tma_kernel<T, true, LEN> : fft_cols_tma_kernel<T, false, LEN>;
                smem_at_least(kt, 2 * smem);
                int per_sm = 0;
                CAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kt, nthr, 2 * smem));
                const int64_t ntiles = (int64_t)nplanes * ncomp * (ncols / W);
                const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)kNumSMs * std::max(per_sm, 1)));
                CAM_LAUNCH_NAMED(ctx, "fft_cols", kt, g, nthr, 2 * smem, map, td, (int)(ncols / W), (int)nplanes, ntiles,
                                 static_cast<const C *>(p->tw), device_error_word(ctx));
                return;
            }
            if (pipe_ok) {
                auto kp = inv ? fft_cols_pipe_kernel<T, true, LEN> : fft_cols_pipe_kernel<T, false, LEN>;
                smem_at_least(kp, 2 * smem);
                int per_sm = 0;
                CAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, nthr, 2 * smem));
                const int64_t ntiles = (int64_t)nplanes * ncomp * (ncols / W);
                const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)kNumSMs * std::max(per_sm, 1)));
                CAM_LAUNCH_NAMED(ctx, "fft_cols", kp, g, nthr, 2 * smem, static_cast<C *>(base), (int)(ncols / W),
                                 (int)nplanes, ntiles, jstride, pstride, ccomp, static_cast<const C *>(p->tw));
                return;
            }
        }
        auto kern = inv ? fft_cols_kernel<T, true, LEN> : fft_cols_kernel<T, false, LEN>;
        smem_at_least(kern, smem);
        CAM_LAUNCH_NAMED(ctx, "fft_cols", kern, grid, nthr, smem, static_cast<C *>(base), (int)len, (int)ncols,
                         jstride, pstride, ccomp, rd, static_cast<const C *>(p->tw), twmul);
    });
}

template <typename T, int MODE>
void rows_impl(cam_ctx *ctx, FftPlan *p, const void *in, void *out, void *nyq, int64_t nrows,
               int ncomp, int64_t ccomp_in, int64_t ccomp_out, const double *d_sub, double scale)
{
    using C = typename fftdev::CT<T>::t;
    const int n = (int)p->n;
    const int len = MODE <= 1 ? n / 2 : n;
    const Radices &rd = MODE <= 1 ? p->rad_m : p->rad_n;
    const int rpc = rows_rpc<T>(len);
    const int nthr = threads_for(rpc * len, fftdev::CT<T>::kPPT);  // == ct_threads for compiled lengths
    dim3 grid((unsigned)((nrows + rpc - 1) / rpc), (unsigned)ncomp);
    dispatch_fft_len(len, [&](auto lc) {
    constexpr int LEN = decltype(lc)::value;
    const size_t smem = (size_t)fftdev::padded_len((int64_t)rpc * len, LEN > 0) * sizeof(C);
    if constexpr (MODE == 0 && LEN >= 16 && LEN <= 512 && (LEN & (LEN - 1)) == 0) {
        // pipelined r2c rows for the power-of-two half lengths (their
        // transforms fit the register bound without spilling): one
        // component, 16-byte aligned input, raw + padded tile within 200 KB
        const size_t psmem = (size_t)rpc * len * sizeof(C) + smem;
        if (ncomp == 1 && ((uintptr_t)in % 16) == 0 && (len * sizeof(C)) % 16 == 0 && psmem <= 200 * 1024) {
            auto kp = fft_rows_r2c_pipe_kernel<T, LEN>;
            smem_at_least(kp, psmem);
            int per_sm = 0;
            CAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, nthr, psmem));
            const int64_t ngroups = (nrows + rpc - 1) / rpc;
            const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ngroups, (int64_t)kNumSMs * std::max(per_sm, 1)));
            CAM_LAUNCH_NAMED(ctx, "fft_rows_r2c", kp, g, nthr, psmem, static_cast<const T *>(in), static_cast<C *>(out),
                             static_cast<C *>(nyq), nrows, static_cast<const C *>(p->tw), d_sub);
            return;
        }
    }
    auto kern = fft_rows_kernel<T, MODE, LEN>;
    smem_at_least(kern, smem);
    CAM_LAUNCH_NAMED(ctx, MODE == 0 ? "fft_rows_r2c" : MODE == 1 ? "fft_rows_c2r" : "fft_rows_c2c", kern, grid, nthr, smem, in, out, static_cast<C *>(nyq), n, nrows, rpc,
               ccomp_in, ccomp_out, rd, static_cast<const C *>(p->tw), d_sub, scale);
    });
}

template <typename T>
void r2c_impl(cam_ctx *ctx, FftPlan *p, const void *in, const double *d_sub, Spectrum &s)
{
    const int64_t n = p->n, M = n / 2;
    rows_impl<T, 0>(ctx, p, in, s.main, s.nyq, n * n, 1, 0, 0, d_sub, 1.0);
    cols_impl<T>(ctx, p, s.main, n, M, M, n, n * M, 1, 0, false);        // y
    rows_impl<T, 2>(ctx, p, s.nyq, s.nyq, nullptr, n, 1, 0, 0, nullptr, 1.0);  // nyq, y
    cols_impl<T>(ctx, p, s.main, n, M, n * M, n, M, 1, 0, false);        // x
    cols_impl<T>(ctx, p, s.nyq, n, n, n, 1, 0, 1, 0, false);             // nyq, x
}

template <typename T>
void c2r_impl(cam_ctx *ctx, FftPlan *p, Spectrum &s, void *out, double scale)
{
    const int64_t n = p->n, M = n / 2;
    cols_impl<T>(ctx, p, s.main, n, M, n * M, n, M, 1, 0, true);         // x
    cols_impl<T>(ctx, p, s.nyq, n, n, n, 1, 0, 1, 0, true);              // nyq, x
    cols_impl<T>(ctx, p, s.main, n, M, M, n, n * M, 1, 0, true);         // y
    rows_impl<T, 3>(ctx, p, s.nyq, s.nyq, nullptr, n, 1, 0, 0, nullptr, 1.0);  // nyq, y
    rows_impl<T, 1>(ctx, p, s.main, out, s.nyq, n * n, 1, 0, 0, nullptr, scale);
}

}  // namespace

const void *plan_twiddles(FftPlan *plan) { return plan->tw; }

bool fft_r2c_pk_fused(cam_ctx *ctx, FftPlan *plan, const void *real_in, const double *d_sub, Spectrum &out,
                      const PkTables &pt, bool keep, double **d_part, int *nparts)
{
    if (plan->precision != CAM_F32 || ctx->no_tma) return false;
    const int64_t n = plan->n, M = n / 2;
    if (M % 16 != 0 || ((uintptr_t)out.main % 16) != 0) return false;
    bool done = false;
    dispatch_fft_len(n, [&](auto lc) {
        constexpr int LEN = decltype(lc)::value;
        if constexpr (LEN >= 32 && 2 * LEN * pk_pass_cols<LEN>() * 8 <= 200 * 1024) {
            constexpr int NTHR = pk_pass_threads<LEN>();
            const size_t smem = (size_t)2 * LEN * pk_pass_cols<LEN>() * 8 +
                                (size_t)(NTHR / 32) * pt.nbins * sizeof(double) + (size_t)(LEN / 2 + 1) * sizeof(float);
            if (smem > 220 * 1024) return;
            // x pass over main: 4D view (scalar column, row i, plane j, 1)
            CUtensorMap map;
            TileDims td{0};
            uint64_t dims[4], strides[3];
            uint32_t box[4];
            constexpr int WC = pk_pass_cols<LEN>();
            tile_map_layout(2 * M, n, n * M * 8, n, M * 8, 1, 0, (uint32_t)(2 * WC), (uint32_t)(LEN / ((LEN + 255) / 256)),
                            dims, strides, box, td.pos);
            if (!make_tensor_map_4d(&map, false, out.main, dims, strides, box)) return;
            auto kt = fft_cols_tma_pk_kernel<LEN>;
            smem_at_least(kt, smem);
            int per_sm = 0;
            CAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kt, NTHR, smem));
            if (per_sm < 1) return;
            const int64_t ntiles = n * (M / WC);
            const int g = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)kNumSMs * per_sm));
            // rows [0, g) for the column pass, [g, g + kNumSMs) for the Nyquist plane
            auto *part = static_cast<double *>(
                scratch(ctx, "pkf.part", (size_t)(g + kNumSMs) * pt.nbins * sizeof(double)));
            // r2c rows; then the y columns and the binning x pass, and beside
            // them, on the side stream, the Nyquist plane's y and x
            // transforms (it is independent of the main planes; its binning,
            // also on the side stream, and the join are power_finish_fused's)
            unsigned *errw = device_error_word(ctx);
            rows_impl<float, 0>(ctx, plan, real_in, out.main, out.nyq, n * n, 1, 0, 0, d_sub, 1.0);
            {
                StreamScope side(ctx, aux_fork(ctx));
                rows_impl<float, 2>(ctx, plan, out.nyq, out.nyq, nullptr, n, 1, 0, 0, nullptr, 1.0);
                cols_impl<float>(ctx, plan, out.nyq, n, n, n, 1, 0, 1, 0, false);
            }
            cols_impl<float>(ctx, plan, out.main, n, M, M, n, n * M, 1, 0, false);
            CAM_LAUNCH_NAMED(ctx, "fft_cols_pk", kt, g, NTHR, smem, map, td, (int)(M / WC), (int)n, ntiles,
                             static_cast<const float2 *>(plan->tw), errw, pt.tab, pt.nbins, pt.btab, keep ? 1 : 0,
                             part);
            *d_part = part;
            *nparts = g;
            done = true;
        }
    });
    return done;
}

bool make_tensor_map_4d(CUtensorMap *map, bool fp64, void *base, const uint64_t dims[4], const uint64_t strides[3],
                        const uint32_t box[4])
{
    const EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    for (int a = 0; a < 3; ++a)
        if (strides[a] % 16 != 0 || strides[a] >= (1ull << 40)) return false;
    if (((uintptr_t)base & 15u) != 0) return false;
    const cuuint64_t d[4] = {dims[0], dims[1], dims[2], dims[3]};
    const cuuint64_t st[3] = {strides[0], strides[1], strides[2]};
    const cuuint32_t bx[4] = {box[0], box[1], box[2], box[3]};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = enc(map, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, d, st,
                           bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

void free_plans(cam_ctx *ctx)
{
    for (auto &kv : ctx->plans) delete kv.second;
    ctx->plans.clear();
}

FftPlan *get_plan(cam_ctx *ctx, int64_t n, int precision)
{
    const int64_t key = n * 2 + precision;
    auto it = ctx->plans.find(key);
    if (it != ctx->plans.end()) return it->second;
    CAM_REQUIRE(n >= 8 && n <= 1024 && n % 2 == 0, CAM_E_UNSUPPORTED, "FFT size must be even, 8 <= N <= 1024");
    auto *p = new FftPlan;
    p->n = n;
    p->precision = precision;
    p->rad_n = factor_radices(n);
    p->rad_m = factor_radices(n / 2);
    if (p->rad_n.n < 0 || p->rad_m.n < 0) {
        delete p;
        throw Error{CAM_E_UNSUPPORTED, "FFT size must be 2^a 3^b"};
    }
    // Roots of unity from long double, correctly rounded to the element type.
    std::vector<double> re(n), im(n);
    const long double pi2 = 6.283185307179586476925286766559L;
    for (int64_t m = 0; m < n; ++m) {
        const long double a = pi2 * (long double)m / (long double)n;
        re[m] = (double)cosl(a);
        im[m] = (double)-sinl(a);
    }
    if (precision == CAM_F32) {
        std::vector<float2> h(n);
        for (int64_t m = 0; m < n; ++m) h[m] = make_float2((float)re[m], (float)im[m]);
        p->tw = scratch(ctx, ("fft.tw." + std::to_string(key)).c_str(), n * sizeof(float2));
        CAM_CUDA_TRY(cudaMemcpy(p->tw, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    } else {
        std::vector<double2> h(n);
        for (int64_t m = 0; m < n; ++m) h[m] = make_double2(re[m], im[m]);
        p->tw = scratch(ctx, ("fft.tw." + std::to_string(key)).c_str(), n * sizeof(double2));
        CAM_CUDA_TRY(cudaMemcpy(p->tw, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
    }
    ctx->plans[key] = p;
    return p;
}

void fft_r2c_split(cam_ctx *ctx, FftPlan *plan, const void *real_in, const double *d_sub, Spectrum &out)
{
    if (plan->precision == CAM_F32) r2c_impl<float>(ctx, plan, real_in, d_sub, out);
    else r2c_impl<double>(ctx, plan, real_in, d_sub, out);
}

void fft_c2r_split(cam_ctx *ctx, FftPlan *plan, Spectrum &spec, void *real_out, double scale)
{
    if (plan->precision == CAM_F32) c2r_impl<float>(ctx, plan, spec, real_out, scale);
    else c2r_impl<double>(ctx, plan, spec, real_out, scale);
}

void fft_columns(cam_ctx *ctx, FftPlan *plan, void *base, int64_t len, int64_t ncols, int64_t jstride,
                 int64_t nplanes, int64_t pstride, int ncomp, int64_t ccomp, bool inverse)
{
    if (plan->precision == CAM_F32) cols_impl<float>(ctx, plan, base, len, ncols, jstride, nplanes, pstride, ncomp, ccomp, inverse);
    else cols_impl<double>(ctx, plan, base, len, ncols, jstride, nplanes, pstride, ncomp, ccomp, inverse);
}

void fft_rows_c2c(cam_ctx *ctx, FftPlan *plan, void *base, int64_t len, int64_t nrows, int ncomp,
                  int64_t ccomp, bool inverse)
{
    (void)len;
    if (plan->precision == CAM_F32) {
        if (inverse) rows_impl<float, 3>(ctx, plan, base, base, nullptr, nrows, ncomp, ccomp, ccomp, nullptr, 1.0);
        else rows_impl<float, 2>(ctx, plan, base, base, nullptr, nrows, ncomp, ccomp, ccomp, nullptr, 1.0);
    } else {
        if (inverse) rows_impl<double, 3>(ctx, plan, base, base, nullptr, nrows, ncomp, ccomp, ccomp, nullptr, 1.0);
        else rows_impl<double, 2>(ctx, plan, base, base, nullptr, nrows, ncomp, ccomp, ccomp, nullptr, 1.0);
    }
}

void split_to_fftw(cam_ctx *ctx, const Spectrum &s, void *dst)
{
    const int64_t n = s.n, M = n / 2, rows = n * n;
    const int blocks = (int)std::min<int64_t>((rows * (M + 1) + 255) / 256, kNumSMs * 16);
    if (s.precision == CAM_F32)
        CAM_LAUNCH(ctx, split_to_fftw_kernel<float>, blocks, 256, 0, (const float2 *)s.main,
                   (const float2 *)s.nyq, (float2 *)dst, rows, (int)M);
    else
        CAM_LAUNCH(ctx, split_to_fftw_kernel<double>, blocks, 256, 0, (const double2 *)s.main,
                   (const double2 *)s.nyq, (double2 *)dst, rows, (int)M);
}

void fftw_to_split(cam_ctx *ctx, const void *src, Spectrum &s)
{
    const int64_t n = s.n, M = n / 2, rows = n * n;
    const int blocks = (int)std::min<int64_t>((rows * (M + 1) + 255) / 256, kNumSMs * 16);
    if (s.precision == CAM_F32)
        CAM_LAUNCH(ctx, fftw_to_split_kernel<float>, blocks, 256, 0, (const float2 *)src,
                   (float2 *)s.main, (float2 *)s.nyq, rows, (int)M);
    else
        CAM_LAUNCH(ctx, fftw_to_split_kernel<double>, blocks, 256, 0, (const double2 *)src,
                   (double2 *)s.main, (double2 *)s.nyq, rows, (int)M);
}

}  // namespace cam

// Persistent on-device request loop for small mesh jobs.
//
// BAM's calibration loop issues many small, independent mesh jobs
// (Source/Bam.cpp:13424, Bam::bamrunner; get_BAM_DM per iteration,
// :2102-2303).  Launched per job, each runs a dozen short kernels and the
// GPU spends much of its time between them.  Here one kernel stays resident
// on the GPU, one CTA of 1024 threads per SM, and each CTA runs whole jobs:
// it claims the next job of a queue the host fills, runs the job's
// assignment, r2c FFT and P(k) binning alone, writes the results to the
// host and claims the next job.  Jobs of different sizes and schemes run
// side by side on different SMs.
//
// Scope: FP32 meshes of N in {32, 64, 128} cells per side, NGP/CIC/TSC,
// unit or per-particle weights, density P(k) with up to 128 bins, particles
// already on the device; no T-web.  Larger or other jobs go to cam_job_run,
// cam_batch_run or the job server.
//
// Results: the assignment uses the same device functions, brick geometry
// and 64-bit fixed-point scale as cam_job_run, so the mesh, its sum and the
// lost-particle count are bit-identical to cam_job_run's.  The FFT holds
// 8 points per thread and takes radix-8 stages (cam_job_run's kernels hold
// 16 and take radix-16 stages where that saves a pass), and each mode's
// power is binned in FP64 (cam_job_run: FP32 per mode, FP64 bins), so P(k)
// agrees with cam_job_run's to FP32 rounding (~1e-7 relative).  P(k) bins
// are summed in FP64 in this CTA's fixed order, so a job's results do not
// depend on which CTA ran it or on what ran beside it.
//
// Queue (pinned host memory mapped into the device): a ring of job slots.
// The host writes a slot's job, then raises `submitted`.  CTA thread 0
// takes a sequence number from a device counter, waits until the host has
// submitted that job, runs it, writes its results into the slot and then
// the slot's `done` word (sequence + 1).  Every wait is bounded by the
// global timer: a CTA that sees no job for `idle_ns` leaves the loop, and
// when all have left the kernel ends with status DL_IDLE (cam_devloop_state
// reports CAM_E_TIMEOUT); a later submission relaunches it.  `stop` makes
// the CTAs leave once the submitted jobs are done.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "cam_assign_device.cuh"
#include "cam_fft_device.cuh"
#include "cam_internal.h"
#include "cam_pk_device.cuh"

namespace cam {
namespace {

using namespace asg;

constexpr int kDlThreads = 1024;
constexpr int kDlWarps = kDlThreads / 32;
constexpr int kDlMaxBins = 128;
constexpr int kDlMaxN = 128;
constexpr int kDlMaxBricks = 1024;  // bricks of one job (shared counters)
constexpr int kDlPoints = 8192;     // complex points of one FFT tile (8 per thread)
constexpr size_t kDlSmem = 104 * 1024;

enum : unsigned { DL_RUNNING = 0, DL_STOPPED = 1, DL_IDLE = 2 };

struct DlJob {
    unsigned long long seq;      // the job's sequence number
    const float *x, *y, *z, *w;  // device particle arrays (w null: unit weights)
    int64_t np;
    AssignGeom g;
    int n, scheme;
    int nbins;
    float m_u, inv_s;
    const double *tab;   // P(k) tables: [h+1] 1/W^2, [h+1] C/W^2, [nbins+1] E2
    const float2 *tw;    // FFT twiddles of length n
};

struct DlResult {
    int status;               // CAM_OK, CAM_E_UNSUPPORTED (payload too small)
    unsigned wbits;           // bits of max |w|
    unsigned long long lost;  // particles outside the box
    double sum;               // mesh sum (FP64, from the exact brick sums)
    double raw[kDlMaxBins];   // sum |F|^2 / W^2 per bin
    double sn[kDlMaxBins];    // sum C / W^2 per bin
    unsigned long long modes[kDlMaxBins];
};

struct DlSlot {
    DlJob job;
    DlResult res;
    unsigned long long done;  // sequence + 1 once res is complete
};

struct DlControl {
    unsigned long long submitted;  // jobs the host has published
    unsigned stop;                 // leave once the submitted jobs are done
    unsigned status;               // DL_* of the last kernel
    unsigned exited;               // CTAs that have left the loop
    unsigned closing;              // a CTA ran out of its idle limit: all leave
};

// Per-CTA scratch in device memory.
struct DlScratch {
    uint4 *payload;  // [pcap] records
    float *mesh;     // [N^3]
    float2 *main;    // [N][N][N/2]
    float2 *nyq;     // [N][N]
    uint64_t pcap;
    size_t mesh_stride, main_stride, nyq_stride, payload_stride;  // elements per CTA
};

__device__ __forceinline__ unsigned long long dl_now()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Exclusive scan of v[0, n) in shared memory (n <= kDlMaxBricks), result in
// out[0, n], out[n] = total.  Every thread calls it.
__device__ void dl_scan(const uint32_t *v, int n, uint32_t *out, uint32_t *wsum)
{
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t x = tid < n ? v[tid] : 0u;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const uint32_t ws = wsum[lane];
        uint32_t wi = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        wsum[lane] = wi - ws;
        if (lane == 31) out[n] = wi;
    }
    __syncthreads();
    if (tid < n) out[tid] = wsum[wid] + incl - x;
    __syncthreads();
}

// Shared memory of one job (carved from the dynamic buffer).
struct DlShared {
    uint32_t *hist;     // [kDlMaxBricks]
    uint32_t *start;    // [kDlMaxBricks + 1]
    double *bsum;       // [kDlMaxBricks]
    unsigned *wstat;    // [8]: max |w| bits, negative flag, ..., [6] min-|w| complement
    uint32_t *wsum;     // [32]
    unsigned long long *lost;
    unsigned *ovf;
    unsigned char *big; // the rest: deposit tile, FFT tile, P(k) bins
};

// The assignment of one job by this CTA: counts per brick, scan, records
// in brick order, then brick by brick the haloed fixed-point tile, as the
// multi-CTA passes do.  Writes the FP32 mesh and bsum[brick].
template <int SCHEME>
__device__ void dl_assign(const DlJob &J, const DlScratch &S, uint4 *payload, float *mesh, DlShared &sh, int &nb,
                          bool &ok)
{
    const AssignGeom &g = J.g;
    const int tid = threadIdx.x;
    nb = g.nb[0] * g.nb[1] * g.nb[2];
    for (int b = tid; b < nb; b += kDlThreads) sh.hist[b] = 0u;
    if (tid < 8) sh.wstat[tid] = 0u;
    if (tid == 0) {
        *sh.lost = 0ull;
        *sh.ovf = 0u;
    }
    __syncthreads();
    const bool weighted = J.w != nullptr;
    unsigned long long my_lost = 0;
    unsigned my_wmax = 0, my_neg = 0, my_wminc = 0;
    for (int64_t p = tid; p < J.np; p += kDlThreads)
        count_one<SCHEME, true>(J.x[p], J.y[p], J.z[p], weighted ? J.w[p] : 1.0f, weighted, g, sh.hist, nullptr,
                                my_lost, my_wmax, my_neg, my_wminc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        my_lost += __shfl_down_sync(0xffffffffu, my_lost, off);
        my_wmax = max(my_wmax, __shfl_down_sync(0xffffffffu, my_wmax, off));
        my_neg |= __shfl_down_sync(0xffffffffu, my_neg, off);
        my_wminc = max(my_wminc, __shfl_down_sync(0xffffffffu, my_wminc, off));
    }
    if ((tid & 31) == 0) {
        if (my_lost) atomicAdd(sh.lost, my_lost);
        if (my_wmax) atomicMax(sh.wstat, my_wmax);
        if (my_neg) atomicOr(sh.wstat + 1, 1u);
        if (my_wminc) atomicMax(sh.wstat + 6, my_wminc);
    }
    __syncthreads();
    dl_scan(sh.hist, nb, sh.start, sh.wsum);
    const uint32_t total = sh.start[nb];
    ok = total <= S.pcap;
    if (!ok) return;
    // append cursors (the counts are not needed any more)
    for (int b = tid; b < nb; b += kDlThreads) sh.hist[b] = sh.start[b];
    __syncthreads();
    unsigned dummy_wmax = 0, dummy_neg = 0;
    unsigned long long dummy_lost = 0;
    for (int64_t p = tid; p < J.np; p += kDlThreads)
        bin_one<SCHEME, true, false, 1>(J.x[p], J.y[p], J.z[p], weighted ? J.w[p] : 1.0f, weighted, g, 1, 0, nullptr,
                                        sh.hist, payload, S.pcap, sh.ovf, dummy_lost, dummy_wmax, dummy_neg);
    __syncthreads();
    // deposit, brick by brick (the same tile layout as deposit_kernel)
    const int T2 = g.b[2] + 2, T1 = g.b[1] + 2;
    const int S1 = T2, S0 = T1 * T2;
    const int cap = (g.b[0] + 2) * S0;
    uint32_t *lo = reinterpret_cast<uint32_t *>(sh.big);
    uint32_t *hi = lo + cap;
    long long *red = reinterpret_cast<long long *>(hi + cap);
    const bool whole[3] = {g.nb[0] == 1, g.nb[1] == 1, g.nb[2] == 1};
    const bool nonneg = !weighted || sh.wstat[1] == 0u;
    for (int B = 0; B < nb; ++B) {
        const int B2 = B % g.nb[2];
        const int B1 = (B / g.nb[2]) % g.nb[1];
        const int B0 = B / (g.nb[2] * g.nb[1]);
        const int o[3] = {B0 * g.b[0], B1 * g.b[1], B2 * g.b[2]};
        const int e[3] = {min(g.b[0], g.n[0] - o[0]), min(g.b[1], g.n[1] - o[1]), min(g.b[2], g.n[2] - o[2])};
        {
            uint4 *t4 = reinterpret_cast<uint4 *>(lo);
            const int nw = 2 * cap;
            for (int i = tid; i < nw / 4; i += kDlThreads) t4[i] = make_uint4(0u, 0u, 0u, 0u);
            for (int i = (nw & ~3) + tid; i < nw; i += kDlThreads) lo[i] = 0u;
        }
        __syncthreads();
        const uint32_t beg = sh.start[B], end = sh.start[B + 1];
        const int s = fixed_scale(sh.wstat, weighted ? 1 : 0, end - beg);
        const float f1 = scalbnf(1.0f, s / 2), f2 = scalbnf(1.0f, s - s / 2);
        for (uint32_t p = beg + tid; p < end; p += kDlThreads)
            deposit_record<SCHEME>(payload[p], e, whole, S0, S1, f1, f2, nonneg, lo, hi);
        __syncthreads();
        long long acc = 0;
        const double sc = ldexp(1.0, -s);
        const int ncell = e[0] * e[1] * e[2];
        for (int i = tid; i < ncell; i += kDlThreads) {
            const int lk = i % e[2], row = i / e[2];
            const int lj = row % e[1], li = row / e[1];
            const int c = (li + 1) * S0 + (lj + 1) * S1 + lk + 1;
            const long long q = (long long)(((unsigned long long)hi[c] << 32) | lo[c]);
            acc += q;
            mesh[((int64_t)(o[0] + li) * g.n[1] + (o[1] + lj)) * g.n[2] + (o[2] + lk)] = convert_out<float>(q, s, sc);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if ((tid & 31) == 0) red[tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            long long tot = 0;
            for (int i = 0; i < kDlWarps; ++i) tot += red[i];
            sh.bsum[B] = ldexp((double)tot, -s);
        }
        __syncthreads();
    }
}

// The FP64 sum of bsum[0, nb) in the order of the library's one-CTA
// reduction (1024 threads, strided partial sums, warp trees, warps in
// order), so the mean matches cam_job_run's bit for bit.
__device__ double dl_sum(const double *bsum, int nb, double *wred)
{
    const int tid = threadIdx.x;
    double acc = 0.0;
    for (int i = tid; i < nb; i += kDlThreads) acc += bsum[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((tid & 31) == 0) wred[tid >> 5] = acc;
    __syncthreads();
    double t = 0.0;
    if (tid == 0) {
        for (int w = 0; w < kDlWarps; ++w) t += wred[w];
        wred[0] = t;
    }
    __syncthreads();
    t = wred[0];
    __syncthreads();
    return t;
}

// The r2c FFT of one N^3 mesh by this CTA, into main[N][N][N/2] and
// nyq[N][N]: rows along z (half-length complex transform and untangling),
// columns along y, the Nyquist plane's rows, columns along x and the
// Nyquist plane's columns; each in tiles of kDlPoints points with the same
// Stockham stage lists as the multi-CTA kernels.
template <int N>
__device__ void dl_fft(const float *mesh, float sub, float2 *main, float2 *nyq, const float2 *__restrict__ tw,
                       float2 *tile)
{
    using C = float2;
    constexpr int M = N / 2;
    const int tid = threadIdx.x;
    // rows: RPC rows of M complex per tile (padded slots)
    {
        constexpr int RPC = kDlPoints / M;
        constexpr int NROWS = N * N;
        const C *src = reinterpret_cast<const C *>(mesh);
        for (int row0 = 0; row0 < NROWS; row0 += RPC) {
            const int nr = min(RPC, NROWS - row0);
            for (int e = tid; e < nr * M; e += kDlThreads) {
                C v = src[(int64_t)row0 * M + e];
                v.x -= sub;
                v.y -= sub;
                tile[fftdev::sidx<true>(e)] = v;
            }
            __syncthreads();
            fftdev::block_fft_fixed<C, false, true, RPC, M, kDlThreads, 1, M, 2, true>(tile, tw);
            for (int e = tid; e < nr * (M + 1); e += kDlThreads) {
                const int r = e / (M + 1), k = e % (M + 1);
                const C zk = tile[fftdev::sidx<true>(r * M + (k % M))];
                const C zc0 = tile[fftdev::sidx<true>(r * M + ((M - k) % M))];
                const C zc = C{zc0.x, -zc0.y};
                // X[k] = (Z[k] + conj Z[M-k])/2 - i/2 e^{-2 pi i k/n} (Z[k] - conj Z[M-k])
                const C s = fftdev::cadd(zk, zc), d = fftdev::csub(zk, zc);
                const C wd = fftdev::cmul(__ldg(tw + k), d);
                const C xk = C{0.5f * (s.x + wd.y), 0.5f * (s.y - wd.x)};
                if (k < M) main[(int64_t)(row0 + r) * M + k] = xk;
                else nyq[row0 + r] = xk;
            }
            __syncthreads();
        }
    }
    // columns along y: NCOL columns (i, k) per tile, element j
    constexpr int NCOL = kDlPoints / N;
    {
        constexpr int TOTC = N * M;  // columns (i, k)
        for (int c0 = 0; c0 < TOTC; c0 += NCOL) {
            const int nc = min(NCOL, TOTC - c0);
            for (int e = tid; e < N * NCOL; e += kDlThreads) {
                const int j = e / NCOL, cc = e % NCOL;
                if (cc < nc) {
                    const int c = c0 + cc, i = c / M, k = c % M;
                    tile[e] = main[((int64_t)i * N + j) * M + k];
                }
            }
            __syncthreads();
            fftdev::block_fft_fixed<C, false, false, NCOL, N, kDlThreads, NCOL, 1, 1>(tile, tw);
            for (int e = tid; e < N * NCOL; e += kDlThreads) {
                const int j = e / NCOL, cc = e % NCOL;
                if (cc < nc) {
                    const int c = c0 + cc, i = c / M, k = c % M;
                    main[((int64_t)i * N + j) * M + k] = tile[e];
                }
            }
            __syncthreads();
        }
    }
    // the Nyquist plane's rows (along j), as complex rows of N
    {
        constexpr int RPC = kDlPoints / N;
        for (int r0 = 0; r0 < N; r0 += RPC) {
            const int nr = min(RPC, N - r0);
            for (int e = tid; e < nr * N; e += kDlThreads) tile[fftdev::sidx<true>(e)] = nyq[r0 * N + e];
            __syncthreads();
            fftdev::block_fft_fixed<C, false, true, RPC, N, kDlThreads, 1, N, 1, true>(tile, tw);
            for (int e = tid; e < nr * N; e += kDlThreads) nyq[r0 * N + e] = tile[fftdev::sidx<true>(e)];
            __syncthreads();
        }
    }
    // columns along x: columns c = j * M + k are contiguous within plane i
    {
        constexpr int TOTC = N * M;
        for (int c0 = 0; c0 < TOTC; c0 += NCOL) {
            const int nc = min(NCOL, TOTC - c0);
            for (int e = tid; e < N * NCOL; e += kDlThreads) {
                const int i = e / NCOL, cc = e % NCOL;
                if (cc < nc) tile[e] = main[(int64_t)i * TOTC + c0 + cc];
            }
            __syncthreads();
            fftdev::block_fft_fixed<C, false, false, NCOL, N, kDlThreads, NCOL, 1, 1>(tile, tw);
            for (int e = tid; e < N * NCOL; e += kDlThreads) {
                const int i = e / NCOL, cc = e % NCOL;
                if (cc < nc) main[(int64_t)i * TOTC + c0 + cc] = tile[e];
            }
            __syncthreads();
        }
    }
    // the Nyquist plane's columns (along i): N columns j
    for (int c0 = 0; c0 < N; c0 += NCOL) {
        const int nc = min(NCOL, N - c0);
        for (int e = tid; e < N * NCOL; e += kDlThreads) {
            const int i = e / NCOL, cc = e % NCOL;
            if (cc < nc) tile[e] = nyq[i * N + c0 + cc];
        }
        __syncthreads();
        fftdev::block_fft_fixed<C, false, false, NCOL, N, kDlThreads, NCOL, 1, 1>(tile, tw);
        for (int e = tid; e < N * NCOL; e += kDlThreads) {
            const int i = e / NCOL, cc = e % NCOL;
            if (cc < nc) nyq[i * N + c0 + cc] = tile[e];
        }
        __syncthreads();
    }
}

// P(k) bin sums of one spectrum by this CTA: the estimator's mode set
// (pk_visited), bins by the squared FP64 edges (pk_bin); a warp takes one
// row (i, j) at a time, sums runs of equal bins with a fixed shuffle tree
// and adds them to its own FP64 bins; warps are combined in order.
__device__ void dl_pk(const float2 *main, const float2 *nyq, int n, const double *g_tab, int nbins, float m_u,
                      float inv_s, unsigned char *smem, DlResult *res)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int h = n / 2, M = h;
    double *tw2 = reinterpret_cast<double *>(smem);  // [h+1]
    double *tsn = tw2 + (h + 1);                      // [h+1]
    double *E2 = tsn + (h + 1);                       // [nbins+1]
    double *wsum = E2 + (nbins + 1);                  // [warps][nbins][2]
    unsigned long long *wcnt = reinterpret_cast<unsigned long long *>(wsum + (size_t)kDlWarps * nbins * 2);
    for (int t = tid; t < 2 * (h + 1) + nbins + 1; t += kDlThreads) tw2[t] = g_tab[t];
    for (int t = tid; t < kDlWarps * nbins * 2; t += kDlThreads) wsum[t] = 0.0;
    for (int t = tid; t < kDlWarps * nbins; t += kDlThreads) wcnt[t] = 0ull;
    __syncthreads();
    double *mysum = wsum + (size_t)warp * nbins * 2;
    unsigned long long *mycnt = wcnt + (size_t)warp * nbins;
    for (int r = warp; r < n * n; r += kDlWarps) {
        const int i = r / n, j = r - i * n;
        if (i == h || j == h) continue;
        const int a = i <= h ? i : n - i, b = j <= h ? j : n - j;
        const double tab_ab = tw2[a] * tw2[b], sn_ab = tsn[a] * tsn[b];
        const int q0 = a * a + b * b;
        for (int c0 = 0; c0 < M; c0 += 32) {
            const int c = c0 + lane;
            double vraw = 0.0, vsn = 0.0;
            bool valid = false;
            int bin = nbins;
            if (c < M) {
                const double q = (double)(q0 + c * c);
                bin = pk_bin(q, E2, nbins, m_u, inv_s);
                if (bin >= 0 && bin < nbins && pk_visited(i, j, c, n)) {
                    const float2 f = main[(int64_t)r * M + c];
                    vraw = ((double)f.x * (double)f.x + (double)f.y * (double)f.y) * (tab_ab * tw2[c]);
                    vsn = sn_ab * tsn[c];
                    valid = true;
                }
            }
            const int prev = __shfl_up_sync(0xffffffffu, bin, 1);
            const bool head = lane == 0 || prev != bin;
            const unsigned heads = __ballot_sync(0xffffffffu, head);
            const unsigned later = heads & ~((2u << lane) - 1u);
            const int end = later ? __ffs((int)later) - 1 : 32;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double orr = __shfl_down_sync(0xffffffffu, vraw, off);
                const double os = __shfl_down_sync(0xffffffffu, vsn, off);
                if (lane + off < end) {
                    vraw += orr;
                    vsn += os;
                }
            }
            const unsigned vmask = __ballot_sync(0xffffffffu, valid);
            const unsigned run = (end == 32 ? 0xffffffffu : ((1u << end) - 1u)) & ~((1u << lane) - 1u);
            const int cnt = __popc(vmask & run);
            if (head && bin >= 0 && bin < nbins && cnt) {
                mysum[2 * bin] += vraw;
                mysum[2 * bin + 1] += vsn;
                mycnt[bin] += (unsigned long long)cnt;
            }
            __syncwarp();
        }
        if (lane == 0) {  // the row's Nyquist element (c = N/2)
            const double q = (double)(q0 + M * M);
            const int bin = pk_bin(q, E2, nbins, m_u, inv_s);
            if (bin >= 0 && bin < nbins && pk_visited(i, j, M, n)) {
                const float2 f = nyq[r];
                mysum[2 * bin] += ((double)f.x * (double)f.x + (double)f.y * (double)f.y) * (tab_ab * tw2[M]);
                mysum[2 * bin + 1] += sn_ab * tsn[M];
                mycnt[bin] += 1ull;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int bn = tid; bn < nbins; bn += kDlThreads) {
        double s0 = 0.0, s1 = 0.0;
        unsigned long long cn = 0;
        for (int w = 0; w < kDlWarps; ++w) {
            s0 += wsum[((size_t)w * nbins + bn) * 2];
            s1 += wsum[((size_t)w * nbins + bn) * 2 + 1];
            cn += wcnt[(size_t)w * nbins + bn];
        }
        res->raw[bn] = s0;
        res->sn[bn] = s1;
        res->modes[bn] = cn;
    }
    __threadfence_system();  // the host reads them once `done` is set
    __syncthreads();
}

template <int SCHEME>
__device__ void dl_run_scheme(const DlJob &J, const DlScratch &S, uint4 *payload, float *mesh, float2 *main,
                              float2 *nyq, DlShared &sh, DlResult *res)
{
    int nb = 0;
    bool ok = true;
    dl_assign<SCHEME>(J, S, payload, mesh, sh, nb, ok);
    if (!ok) {
        if (threadIdx.x == 0) res->status = CAM_E_UNSUPPORTED;
        __syncthreads();
        return;
    }
    double *wred = reinterpret_cast<double *>(sh.big);
    const double sum = dl_sum(sh.bsum, nb, wred);
    const double mean = sum / ((double)J.n * J.n * J.n);
    __threadfence_block();
    float2 *tile = reinterpret_cast<float2 *>(sh.big);
    switch (J.n) {
    case 32: dl_fft<32>(mesh, (float)mean, main, nyq, J.tw, tile); break;
    case 64: dl_fft<64>(mesh, (float)mean, main, nyq, J.tw, tile); break;
    default: dl_fft<128>(mesh, (float)mean, main, nyq, J.tw, tile); break;
    }
    if (J.nbins > 0) dl_pk(main, nyq, J.n, J.tab, J.nbins, J.m_u, J.inv_s, sh.big, res);
    if (threadIdx.x == 0) {
        res->status = *sh.ovf ? CAM_E_UNSUPPORTED : CAM_OK;
        res->wbits = sh.wstat[0];
        res->lost = *sh.lost;
        res->sum = sum;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kDlThreads, 1)
devloop_kernel(DlControl *ctl, DlSlot *slots, int nslots, unsigned long long *next, DlScratch S,
               unsigned long long idle_ns)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t s_hist[kDlMaxBricks], s_start[kDlMaxBricks + 1];
    __shared__ double s_bsum[kDlMaxBricks];
    __shared__ unsigned s_wstat[8];
    __shared__ uint32_t s_wsum[32];
    __shared__ unsigned long long s_lost, s_seq;
    __shared__ unsigned s_ovf;
    __shared__ int s_state;  // 0 run the job, 1 leave (stop), 2 leave (idle)
    __shared__ DlJob s_job;
    DlShared sh{s_hist, s_start, s_bsum, s_wstat, s_wsum, &s_lost, &s_ovf, smem_raw};
    const int cta = blockIdx.x;
    uint4 *payload = S.payload + (size_t)cta * S.payload_stride;
    float *mesh = S.mesh + (size_t)cta * S.mesh_stride;
    float2 *main = S.main + (size_t)cta * S.main_stride;
    float2 *nyq = S.nyq + (size_t)cta * S.nyq_stride;
    volatile DlControl *vc = ctl;
    for (;;) {
        if (threadIdx.x == 0) {
            // claim the next sequence number and wait (bounded) for its job
            const unsigned long long seq = atomicAdd(next, 1ull);
            const unsigned long long t0 = dl_now();
            int state = 0;
            for (;;) {
                if (vc->submitted > seq) break;
                if (vc->stop) {
                    state = 1;
                    break;
                }
                if (vc->closing) {
                    state = 2;
                    break;
                }
                if (dl_now() - t0 > idle_ns) {
                    vc->closing = 1u;  // the loop closes as a whole
                    state = 2;
                    break;
                }
                __nanosleep(2000);
            }
            if (state == 0) {
                __threadfence_system();
                const DlSlot *sl = &slots[seq % (unsigned long long)nslots];
                const volatile unsigned *s32 = reinterpret_cast<const volatile unsigned *>(&sl->job);
                unsigned *d32 = reinterpret_cast<unsigned *>(&s_job);
                for (int k = 0; k < (int)(sizeof(DlJob) / 4); ++k) d32[k] = s32[k];
                // a relaunched loop may meet a job that already ran, or a
                // slot that a later job has taken: skip those
                const unsigned long long d = *reinterpret_cast<const volatile unsigned long long *>(&sl->done);
                if (s_job.seq != seq || d == seq + 1) state = 3;
            }
            s_seq = seq;
            s_state = state;
        }
        __syncthreads();
        const int state = s_state;
        if (state == 3) {
            __syncthreads();
            continue;
        }
        if (state != 0) {
            if (threadIdx.x == 0) {
                if (state == 2) atomicMax((unsigned *)&ctl->status, (unsigned)DL_IDLE);
                else atomicMax((unsigned *)&ctl->status, (unsigned)DL_STOPPED);
                __threadfence_system();
                atomicAdd((unsigned *)&ctl->exited, 1u);
            }
            return;
        }
        const DlJob J = s_job;
        DlSlot *slot = &slots[s_seq % (unsigned long long)nslots];
        DlResult *res = &slot->res;
        switch (J.scheme) {
        case CAM_NGP: dl_run_scheme<CAM_NGP>(J, S, payload, mesh, main, nyq, sh, res); break;
        case CAM_CIC: dl_run_scheme<CAM_CIC>(J, S, payload, mesh, main, nyq, sh, res); break;
        default: dl_run_scheme<CAM_TSC>(J, S, payload, mesh, main, nyq, sh, res); break;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence_system();
            *reinterpret_cast<volatile unsigned long long *>(&slot->done) = s_seq + 1;
            __threadfence_system();
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace cam

using namespace cam;

struct cam_devloop {
    int device = 0;
    cam_ctx *ctx = nullptr;  // plans, P(k) tables
    cudaStream_t stream = nullptr;
    int nslots = 0, ctas = 0;
    int64_t max_particles = 0;
    double idle_s = 0;
    DlControl *ctl = nullptr;  // mapped
    DlSlot *slots = nullptr;   // mapped
    DlControl *d_ctl = nullptr;
    DlSlot *d_slots = nullptr;
    unsigned long long *next = nullptr;  // device
    DlScratch scratch{};
    void *scratch_mem = nullptr;
    uint64_t submitted = 0;      // host copy of ctl->submitted
    uint64_t relaunch_seq = 0;   // first sequence of the running kernel
    bool running = false;
    std::vector<uint64_t> slot_seq;  // sequence occupying each slot (0 = free)
    std::mutex mu;
    std::string err;
};

namespace {

int dl_fail(cam_devloop *l, int code, const char *msg)
{
    if (l) l->err = msg;
    return code;
}

// Launches the persistent kernel; sequences from relaunch_seq on.
int dl_launch(cam_devloop *l)
{
    auto *ctl = l->ctl;
    ctl->stop = 0;
    ctl->status = DL_RUNNING;
    ctl->exited = 0;
    ctl->closing = 0;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    cudaError_t e = cudaMemcpyAsync(l->next, &l->relaunch_seq, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                    l->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(l->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return dl_fail(l, CAM_E_CUDA, cudaGetErrorString(e));
    }
    const unsigned long long idle_ns = (unsigned long long)(l->idle_s * 1e9);
    devloop_kernel<<<l->ctas, kDlThreads, kDlSmem, l->stream>>>(l->d_ctl, l->d_slots, l->nslots, l->next, l->scratch,
                                                                idle_ns);
    e = cudaGetLastError();
    if (e != cudaSuccess) return dl_fail(l, CAM_E_CUDA, cudaGetErrorString(e));
    l->running = true;
    return CAM_OK;
}

// True once every CTA of the running kernel has left the loop.
bool dl_exited(cam_devloop *l)
{
    const volatile DlControl *c = l->ctl;
    return c->exited >= (unsigned)l->ctas;
}

bool dl_job_done(cam_devloop *l, uint64_t seq)
{
    const int s = (int)(seq % (uint64_t)l->nslots);
    if (l->slot_seq[s] != seq + 1) return true;  // the slot moved on: the job completed before
    return *reinterpret_cast<volatile unsigned long long *>(&l->slots[s].done) == seq + 1;
}

// After the kernel has left on its idle limit: relaunch it from the oldest
// submitted job that has not completed (or the next one), if any is
// pending or `force`.
int dl_ensure_running(cam_devloop *l, bool force)
{
    if (l->running && dl_exited(l)) {
        cudaStreamSynchronize(l->stream);
        cudaGetLastError();
        l->running = false;
    }
    if (l->running) return CAM_OK;
    uint64_t first = l->submitted;
    const uint64_t lo = l->submitted > (uint64_t)l->nslots ? l->submitted - l->nslots : 0;
    for (uint64_t q = lo; q < l->submitted; ++q)
        if (!dl_job_done(l, q)) {
            first = q;
            break;
        }
    if (first == l->submitted && !force) return CAM_OK;
    l->relaunch_seq = first;
    return dl_launch(l);
}

}  // namespace

extern "C" {

int cam_devloop_create(int device, int64_t max_particles, int nslots, double idle_timeout_s, int max_ctas,
                       cam_devloop **out)
{
    if (!out) return CAM_E_INVAL;
    *out = nullptr;
    if (max_particles < 1 || max_particles > (1ll << 26) || nslots < 1 || nslots > (1 << 16) || max_ctas < 0 ||
        !(idle_timeout_s > 0.0) || !(idle_timeout_s <= 3600.0))
        return CAM_E_INVAL;
    auto *l = new (std::nothrow) cam_devloop;
    if (!l) return CAM_E_NOMEM;
    l->device = device;
    l->nslots = nslots;
    l->max_particles = max_particles;
    l->idle_s = idle_timeout_s;
    l->slot_seq.assign(nslots, 0);
    int rc = cam_ctx_create(device, 0, &l->ctx);
    if (rc != CAM_OK) {
        delete l;
        return rc;
    }
    auto fail = [&](int code) {
        cam_devloop_destroy(l);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(CAM_E_CUDA);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaFuncSetAttribute(devloop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDlSmem) !=
        cudaSuccess) {
        cudaGetLastError();
        return fail(CAM_E_CUDA);
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, devloop_kernel, kDlThreads, kDlSmem) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return fail(CAM_E_CUDA);
    }
    l->ctas = sms * per_sm;
    if (max_ctas > 0) l->ctas = std::min(l->ctas, max_ctas);
    if (cudaStreamCreateWithFlags(&l->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(CAM_E_CUDA);
    if (cudaHostAlloc(reinterpret_cast<void **>(&l->ctl), sizeof(DlControl), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void **>(&l->slots), sizeof(DlSlot) * (size_t)nslots, cudaHostAllocMapped) !=
            cudaSuccess) {
        cudaGetLastError();
        return fail(CAM_E_NOMEM);
    }
    memset(l->ctl, 0, sizeof(DlControl));
    memset(l->slots, 0, sizeof(DlSlot) * (size_t)nslots);
    if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&l->d_ctl), l->ctl, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&l->d_slots), l->slots, 0) != cudaSuccess) {
        cudaGetLastError();
        return fail(CAM_E_CUDA);
    }
    // per-CTA scratch: payload (4 records per particle at most kept), mesh,
    // spectrum for N = 128
    DlScratch &S = l->scratch;
    S.pcap = (uint64_t)max_particles * 4;
    S.payload_stride = (size_t)S.pcap;
    S.mesh_stride = (size_t)kDlMaxN * kDlMaxN * kDlMaxN;
    S.main_stride = (size_t)kDlMaxN * kDlMaxN * (kDlMaxN / 2);
    S.nyq_stride = (size_t)kDlMaxN * kDlMaxN;
    const size_t per_cta = S.payload_stride * 16 + S.mesh_stride * 4 + S.main_stride * 8 + S.nyq_stride * 8 + 1024;
    if (cudaMalloc(&l->scratch_mem, per_cta * l->ctas + 256) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&l->next), 256) != cudaSuccess) {
        cudaGetLastError();
        return fail(CAM_E_NOMEM);
    }
    char *p = static_cast<char *>(l->scratch_mem);
    S.payload = reinterpret_cast<uint4 *>(p);
    p += S.payload_stride * 16 * l->ctas;
    S.main = reinterpret_cast<float2 *>(p);
    p += S.main_stride * 8 * l->ctas;
    S.nyq = reinterpret_cast<float2 *>(p);
    p += S.nyq_stride * 8 * l->ctas;
    S.mesh = reinterpret_cast<float *>(p);
    rc = dl_launch(l);
    if (rc != CAM_OK) return fail(rc);
    *out = l;
    return CAM_OK;
}

int cam_devloop_submit(cam_devloop *l, const cam_job_desc *job, uint64_t *id)
{
    if (!l || !job || !id) return CAM_E_INVAL;
    std::lock_guard<std::mutex> lk(l->mu);
    const int64_t n = job->grid.n[0];
    if (job->grid.n[1] != n || job->grid.n[2] != n || (n != 32 && n != 64 && n != 128))
        return dl_fail(l, CAM_E_UNSUPPORTED, "the device loop runs cubic meshes of N = 32, 64 or 128");
    if (job->precision != CAM_F32 || job->want_tweb)
        return dl_fail(l, CAM_E_UNSUPPORTED, "the device loop runs FP32 meshes without the T-web");
    if (job->parts.mem != CAM_MEM_DEVICE || job->parts.n < 0 || job->parts.n > l->max_particles ||
        (job->parts.n > 0 && (!job->parts.x || !job->parts.y || !job->parts.z)))
        return dl_fail(l, CAM_E_UNSUPPORTED, "device particles, at most the loop's particle limit");
    if (job->scheme < CAM_NGP || job->scheme > CAM_TSC) return dl_fail(l, CAM_E_INVAL, "unknown scheme");
    const bool want_pk = job->pk.nbins > 0 || job->pk.ndel > 0.0;
    if (want_pk && (job->pk.input_type != CAM_INPUT_DENSITY || !(job->pk.ndel > 0.0) ||
                    job->pk.scheme < 0 || job->pk.scheme > 2))
        return dl_fail(l, CAM_E_INVAL, "P(k) of the density mesh with ndel > 0");
    DlJob J{};
    try {
        CAM_CUDA_TRY(cudaSetDevice(l->device));
        const cam_grid g = resolved_grid(job->grid);
        J.g = make_geom(g, job->scheme, job->parts.n);
        CAM_REQUIRE((int64_t)J.g.nb[0] * J.g.nb[1] * J.g.nb[2] <= kDlMaxBricks, CAM_E_UNSUPPORTED, "too many bricks");
        CAM_REQUIRE((size_t)(J.g.b[0] + 2) * (J.g.b[1] + 2) * (J.g.b[2] + 2) * 8 <= kDlSmem, CAM_E_UNSUPPORTED,
                    "brick tile too large");
        J.x = job->parts.x;
        J.y = job->parts.y;
        J.z = job->parts.z;
        J.w = job->parts.w;
        J.np = job->parts.n;
        J.n = (int)n;
        J.scheme = job->scheme;
        FftPlan *plan = get_plan(l->ctx, n, CAM_F32);
        J.tw = static_cast<const float2 *>(plan_twiddles(plan));
        if (want_pk) {
            const int nb = nbins_for(job->pk, n);
            CAM_REQUIRE(nb >= 1 && nb <= kDlMaxBins, CAM_E_UNSUPPORTED, "the device loop bins at most 128 bins");
            CAM_REQUIRE((size_t)(2 * (n / 2 + 1) + nb + 1 + (size_t)kDlWarps * nb * 3) * 8 <= kDlSmem,
                        CAM_E_UNSUPPORTED, "too many bins");
            const PkTables pt = pk_tables(l->ctx, n, job->pk, nb);
            J.nbins = nb;
            J.tab = pt.tab;
            J.m_u = pt.m_u;
            J.inv_s = pt.inv_s;
        }
        CAM_CUDA_TRY(cudaStreamSynchronize(l->ctx->stream));  // plans and tables are on the device
    } catch (const Error &e) {
        return dl_fail(l, e.code, e.msg.c_str());
    }
    // a free slot: its previous job must have completed (bounded wait)
    const uint64_t seq = l->submitted;
    const int s = (int)(seq % (uint64_t)l->nslots);
    if (l->slot_seq[s] != 0) {
        volatile unsigned long long *done = &l->slots[s].done;
        const auto t0 = std::chrono::steady_clock::now();
        while (*done != l->slot_seq[s]) {
            if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(30))
                return dl_fail(l, CAM_E_BUSY, "every slot holds a job that has not completed");
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
    DlSlot *slot = &l->slots[s];
    *reinterpret_cast<volatile unsigned long long *>(&slot->done) = 0;
    J.seq = seq;
    memcpy(&slot->job, &J, sizeof(J));
    std::atomic_thread_fence(std::memory_order_seq_cst);
    l->slot_seq[s] = seq + 1;
    l->submitted = seq + 1;
    *reinterpret_cast<volatile unsigned long long *>(&l->ctl->submitted) = seq + 1;
    *id = seq;
    // relaunch if the kernel left on its idle limit
    return dl_ensure_running(l, false);
}

int cam_devloop_wait(cam_devloop *l, uint64_t id, int64_t timeout_us, const cam_job_desc *job, cam_job_result *res)
{
    if (!l || !job) return CAM_E_INVAL;
    if (id >= l->submitted) return CAM_E_NOTFOUND;
    const int s = (int)(id % (uint64_t)l->nslots);
    if (l->slot_seq[s] != id + 1) return CAM_E_NOTFOUND;  // the slot was reused
    DlSlot *slot = &l->slots[s];
    volatile unsigned long long *done = &slot->done;
    const auto t0 = std::chrono::steady_clock::now();
    while (*done != id + 1) {
        if (timeout_us >= 0 &&
            std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(timeout_us))
            return CAM_E_TIMEOUT;
        if (l->running && dl_exited(l) && *done != id + 1) {
            std::lock_guard<std::mutex> lk(l->mu);
            const int rc = dl_ensure_running(l, false);
            if (rc != CAM_OK) return rc;
        }
        std::this_thread::yield();
    }
    std::atomic_thread_fence(std::memory_order_seq_cst);
    const DlResult &r = slot->res;
    if (r.status != CAM_OK) return dl_fail(l, r.status, "the job's records exceed the loop's payload capacity");
    if (job->parts.w && r.wbits >= 0x7f800000u) return dl_fail(l, CAM_E_NONFINITE, "a particle weight is NaN or infinite");
    if (res) {
        const int64_t n = job->grid.n[0];
        res->assign.n_lost = (int64_t)r.lost;
        res->assign.n_in = job->parts.n - (int64_t)r.lost;
        res->assign.sum_mesh = r.sum;
        const bool want_pk = job->pk.nbins > 0 || job->pk.ndel > 0.0;
        if (want_pk) {
            const int nb = nbins_for(job->pk, n);
            std::vector<int64_t> md(nb);
            for (int b = 0; b < nb; ++b) md[b] = (int64_t)r.modes[b];
            const cam_grid g = resolved_grid(job->grid);
            finalize_pk(n, g.L[0], r.sum, job->pk, nb, r.raw, r.sn, md.data(), res->pk, res->modes, res->kvector,
                        &res->pk_info);
        }
    }
    return CAM_OK;
}

int cam_devloop_state(cam_devloop *l, int *running)
{
    if (!l) return CAM_E_INVAL;
    const bool out = l->running && dl_exited(l);
    if (running) *running = (l->running && !out) ? 1 : 0;
    const volatile DlControl *c = l->ctl;
    if (out && c->status == DL_IDLE) return CAM_E_TIMEOUT;
    return CAM_OK;
}

int cam_devloop_destroy(cam_devloop *l)
{
    if (!l) return CAM_E_INVAL;
    if (l->running && l->ctl) {
        *reinterpret_cast<volatile unsigned *>(&l->ctl->stop) = 1u;
        std::atomic_thread_fence(std::memory_order_seq_cst);
    }
    if (l->stream) cudaStreamSynchronize(l->stream);
    cudaGetLastError();
    if (l->scratch_mem) cudaFree(l->scratch_mem);
    if (l->next) cudaFree(l->next);
    if (l->slots) cudaFreeHost(l->slots);
    if (l->ctl) cudaFreeHost(l->ctl);
    if (l->stream) cudaStreamDestroy(l->stream);
    if (l->ctx) cam_ctx_destroy(l->ctx);
    delete l;
    return CAM_OK;
}

const char *cam_devloop_last_error(cam_devloop *l) { return l ? l->err.c_str() : "null loop"; }

}  // extern "C"

// Particle -> mesh mass assignment (NGP / CIC / TSC) for sm_100a.
//
// Replaces getDensity_NGP / getDensity_CIC / getDensity_TSC,
// Source/massFunctions.cpp:35-98, :678-790, :1050-1165.
//
// Pipeline (no float atomics, bitwise deterministic):
//   1. bin_count   : each CTA takes a contiguous chunk of particles and
//                    computes, per particle, the reference's FP32 home cell
//                    (bit-exact key) and the mesh bricks its stencil
//                    touches; a shared-memory histogram per CTA is added to
//                    per-brick counters.  Also lost particles, max |w|.
//   2. scan        : exclusive scan of the brick counts: every brick owns a
//                    contiguous payload range, its counter becomes its
//                    append cursor.
//   3. bin_scatter : the particles again; one 16-byte payload per touched
//                    brick (home cell relative to the brick, exact
//                    fractional offset in fixed point, weight) at the next
//                    slot of the brick's cursor (one global atomic each).
//   4. deposit     : one CTA per brick accumulates its payloads into a
//                    shared-memory tile of 64-bit fixed-point cell sums kept
//                    as two 32-bit words (32-bit shared atomics, the carry
//                    detected from the returned old value).  Integer sums do
//                    not depend on arrival order, so the result is
//                    deterministic; the tile is written once, coalesced, as
//                    FP32/FP64 (or uint32 counts for NGP).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "cam_assign_device.cuh"
#include "cam_internal.h"

namespace cam {
namespace {

constexpr int kBinThreads = 1024;
constexpr int kDepositThreads = 512;
constexpr int kScatterThreads = 512;  // scatter pass: two CTAs per SM
constexpr int kSmemBricks = 16384;  // per-CTA brick histogram in shared memory (64 KB)
using namespace asg;


// Calls one(x, y, z, w) for the particles [p0, p1), the threads of the CTA
// taking consecutive particles; with VEC (16-byte aligned arrays, p0 a
// multiple of 4) four per thread per iteration from float4 loads.  Unit
// weights when w is null.
template <bool VEC, typename F>
__device__ __forceinline__ void for_chunk(const float *__restrict__ x, const float *__restrict__ y,
                                          const float *__restrict__ z, const float *__restrict__ w, int64_t p0,
                                          int64_t p1, F &one)
{
    const bool weighted = w != nullptr;
    int64_t ptail = p0;
    if (VEC) {
        const int64_t q1 = p0 + ((p1 - p0) & ~(int64_t)3);
        for (int64_t p = p0 + 4 * (int64_t)threadIdx.x; p < q1; p += 4 * (int64_t)blockDim.x) {
            const float4 X = __ldcs(reinterpret_cast<const float4 *>(x + p));
            const float4 Y = __ldcs(reinterpret_cast<const float4 *>(y + p));
            const float4 Z = __ldcs(reinterpret_cast<const float4 *>(z + p));
            const float4 Wt = weighted ? __ldcs(reinterpret_cast<const float4 *>(w + p)) : make_float4(1.f, 1.f, 1.f, 1.f);
            // one copy of the particle body, not four: the inlined body is
            // large and four copies overflowed the instruction cache
#pragma unroll 1
            for (int k = 0; k < 4; ++k) {
                const float px = k == 0 ? X.x : (k == 1 ? X.y : (k == 2 ? X.z : X.w));
                const float py = k == 0 ? Y.x : (k == 1 ? Y.y : (k == 2 ? Y.z : Y.w));
                const float pz = k == 0 ? Z.x : (k == 1 ? Z.y : (k == 2 ? Z.z : Z.w));
                const float pw = k == 0 ? Wt.x : (k == 1 ? Wt.y : (k == 2 ? Wt.z : Wt.w));
                one(px, py, pz, pw);
            }
        }
        ptail = q1;
    }
    for (int64_t p = ptail + threadIdx.x; p < p1; p += blockDim.x)
        one(__ldcs(x + p), __ldcs(y + p), __ldcs(z + p), weighted ? __ldcs(w + p) : 1.0f);
}


// Passes 1 and 3.  Block `blk` handles particles [blk * chunk, (blk+1) * chunk)
// (chunk a multiple of 4).
//   COUNT   : table[brick * kCursorStride] += number of payloads for the
//             brick (through a per-CTA shared-memory histogram when SMEM,
//             nb <= kSmemBricks), plus lost particles and max |w|.
//   SCATTER : table[brick * kCursorStride] is the brick's append cursor (the
//             exclusive scan of the counts); every payload takes the next
//             slot of its brick with one global atomic, and its words are
//             packed while the atomic is in flight.  A brick's records are appended
//             contiguously by all CTAs, so its few open 128-byte lines fill
//             in L2 and are written back whole.  The order of records inside
//             a brick varies from run to run; the deposit's integer sums do
//             not depend on it.
// VEC: 16-byte aligned arrays, four particles per thread per iteration
// (float4 loads).
// SLAB (scatter only): records into per-brick slabs of `slab` records, the
// weight statistics and lost count gathered here (no count pass).
template <int SCHEME, bool SCATTER, bool SMEM, bool VEC, bool SLAB = false>
__global__ void __launch_bounds__(kBinThreads)
bin_kernel(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
           const float *__restrict__ w, int64_t np, int64_t chunk, AssignGeom g, int nb,
           uint32_t *__restrict__ table, uint4 *__restrict__ payload, unsigned long long *__restrict__ lost,
           unsigned int *__restrict__ wmax_bits, uint64_t cap, unsigned int *__restrict__ ovf, uint32_t slab)
{
    extern __shared__ uint32_t hist[];
    constexpr bool kHist = SMEM && !SCATTER;
    const int G = gridDim.x, blk = blockIdx.x;
    const int lane = threadIdx.x & 31;
    if (kHist) {
        for (int i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0u;
        __syncthreads();
    }
    unsigned long long my_lost = 0;
    unsigned int my_wmax = 0, my_neg = 0, my_wminc = 0;
    const bool weighted = w != nullptr;
    auto one = [&](float px, float py, float pz, float wt) {
        if (SCATTER)
            bin_one<SCHEME, true, false>(px, py, pz, wt, weighted, g, G, blk, hist, table, payload, cap, ovf,
                                         my_lost, my_wmax, my_neg, SLAB ? &my_wminc : nullptr, SLAB ? slab : 0u);
        else
            count_one<SCHEME, kHist>(px, py, pz, wt, weighted, g, hist, table, my_lost, my_wmax, my_neg,
                                     my_wminc);
    };
    for_chunk<VEC>(x, y, z, w, (int64_t)blk * chunk, min(np, (int64_t)blk * chunk + chunk), one);
    if (!SCATTER || SLAB) {
        // Warp reductions, one atomic per warp (the scatter's when it writes
        // slabs: there is no count pass then).
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            my_lost += __shfl_down_sync(0xffffffffu, my_lost, off);
            my_wmax = max(my_wmax, __shfl_down_sync(0xffffffffu, my_wmax, off));
            my_neg |= __shfl_down_sync(0xffffffffu, my_neg, off);
            my_wminc = max(my_wminc, __shfl_down_sync(0xffffffffu, my_wminc, off));
        }
        if (lane == 0) {
            if (my_lost) atomicAdd(lost, my_lost);
            if (my_wmax) atomicMax(wmax_bits, my_wmax);
            if (my_neg) atomicOr(wmax_bits + 1, 1u);  // some weight is negative
            if (my_wminc) atomicMax(wmax_bits + 6, my_wminc);  // smallest nonzero |w|
        }
        if (kHist) {
            __syncthreads();
            for (int i = threadIdx.x; i < nb; i += blockDim.x)
                if (hist[i]) atomicAdd(table + (int64_t)i * kCursorStride, hist[i]);
        }
    }
}

// Brick starts in one CTA (nb <= kOffThreads * kOffItems): thread t scans
// the counts of bricks [t * kOffItems, (t + 1) * kOffItems) in order, the
// per-thread sums are scanned across the CTA, and every brick's start goes
// to start[b] and to its padded cursor (which held its count); start[nb] =
// *total = all records.
constexpr int kOffThreads = 1024;
constexpr int kOffItems = 16;
__global__ void __launch_bounds__(kOffThreads)
brick_offsets_kernel(uint32_t *__restrict__ padded, int nb, uint32_t *__restrict__ start, uint32_t *__restrict__ total)
{
    __shared__ uint32_t warp_sums[kOffThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int base = threadIdx.x * kOffItems;
    uint32_t v[kOffItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kOffItems; ++i) {
        v[i] = base + i < nb ? padded[(int64_t)(base + i) * kCursorStride] : 0u;
        s += v[i];
    }
    uint32_t incl = s;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const uint32_t ws = warp_sums[lane];
        uint32_t wi = ws;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += o;
        }
        warp_sums[lane] = wi - ws;
        if (lane == 31) {
            start[nb] = wi;
            *total = wi;
        }
    }
    __syncthreads();
    uint32_t run = warp_sums[wid] + incl - s;
#pragma unroll
    for (int i = 0; i < kOffItems; ++i) {
        if (base + i < nb) {
            start[base + i] = run;
            padded[(int64_t)(base + i) * kCursorStride] = run;
        }
        run += v[i];
    }
}

// The largest brick record count, start[b + 1] - start[b], into *out
// (atomicMax; *out zeroed before).
__global__ void __launch_bounds__(256)
brick_max_kernel(const uint32_t *__restrict__ start, int nb, unsigned int *__restrict__ out)
{
    unsigned m = 0u;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        m = max(m, start[b + 1] - start[b]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// counts[b] = padded[b * kCursorStride] (contiguous, for the scan).
__global__ void compact_counts_kernel(const uint32_t *__restrict__ padded, int nb, uint32_t *__restrict__ counts)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        counts[b] = padded[(int64_t)b * kCursorStride];
}

// start[b] = scanned count of brick b (its first payload), start[nb] = total;
// the padded cursors start there.
__global__ void brick_starts_kernel(const uint32_t *__restrict__ scanned, int nb,
                                    const uint32_t *__restrict__ total, uint32_t *__restrict__ start,
                                    uint32_t *__restrict__ cursor)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nb; b += gridDim.x * blockDim.x) {
        const uint32_t v = b < nb ? scanned[b] : *total;
        start[b] = v;
        if (b < nb) cursor[(int64_t)b * kCursorStride] = v;
    }
}

template <int SCHEME, typename OutT>
__global__ void __launch_bounds__(kDepositThreads, 2)
deposit_kernel(const uint4 *__restrict__ payload, const uint32_t *__restrict__ start, uint32_t nrec,
               AssignGeom g, const unsigned int *__restrict__ wstat, int weighted,
               OutT *__restrict__ mesh, double *__restrict__ brick_sum, uint32_t slab,
               const uint32_t *__restrict__ slab_count)
{
    extern __shared__ uint32_t tile32[];
    __shared__ long long red[kDepositThreads / 32];
    const int B = blockIdx.x;
    const int B2 = B % g.nb[2];
    const int B1 = (B / g.nb[2]) % g.nb[1];
    const int B0 = B / (g.nb[2] * g.nb[1]);
    const int o[3] = {B0 * g.b[0], B1 * g.b[1], B2 * g.b[2]};
    const int e[3] = {min(g.b[0], g.n[0] - o[0]), min(g.b[1], g.n[1] - o[1]),
                      min(g.b[2], g.n[2] - o[2])};
    const bool whole[3] = {g.nb[0] == 1, g.nb[1] == 1, g.nb[2] == 1};
    // haloed tile: (b0 + 2) x (b1 + 2) x (b2 + 2) cells, low words then high words
    const int T2 = g.b[2] + 2, T1 = g.b[1] + 2;
    const int S1 = T2, S0 = T1 * T2;
    const int cap = (g.b[0] + 2) * S0;
    uint32_t *lo = tile32;
    uint32_t *hi = tile32 + cap;
    {
        const int nw = 2 * cap;
        uint4 *t4 = reinterpret_cast<uint4 *>(tile32);
        for (int i = threadIdx.x; i < nw / 4; i += blockDim.x) t4[i] = make_uint4(0u, 0u, 0u, 0u);
        for (int i = (nw & ~3) + threadIdx.x; i < nw; i += blockDim.x) tile32[i] = 0u;
    }
    __syncthreads();

    // records beyond the payload's capacity nrec were not written (overflow
    // flag); with slabs, the brick's records are the first of its slab (the
    // host keeps every slab index below 2^32)
    const uint32_t beg = slab ? (uint32_t)B * slab : min(start[B], nrec);
    const uint32_t end = slab ? beg + min(slab_count[(int64_t)B * kCursorStride], slab) : min(start[B + 1], nrec);
    const bool nonneg = !weighted || wstat[1] == 0u;
    const int s = fixed_scale(wstat, weighted, end - beg);
    // 2^s as two exact factors (s may exceed the float exponent range)
    const float f1 = scalbnf(1.0f, s / 2), f2 = scalbnf(1.0f, s - s / 2);
    // one record per iteration, the next one's load in flight meanwhile; a
    // single inlined copy of the stencil (three conversion paths of up to 27
    // cells each) keeps the loop within the instruction cache
    uint32_t p = beg + threadIdx.x;
    uint4 v = p < end ? payload[p] : make_uint4(0u, 0u, 0u, 0u);
    for (; p < end; p += blockDim.x) {
        const uint32_t pn = p + blockDim.x;
        const uint4 vn = pn < end ? payload[pn] : make_uint4(0u, 0u, 0u, 0u);
        deposit_record<SCHEME>(v, e, whole, S0, S1, f1, f2, nonneg, lo, hi);
        v = vn;
    }
    __syncthreads();

    long long acc = 0;
    const double sc = ldexp(1.0, -s);
    // interior cell i = (li * e1 + lj) * e2 + lk; a brick holds < 2^16 cells
    const int ncell = e[0] * e[1] * e[2];
    const unsigned e2 = (unsigned)e[2], e12 = (unsigned)(e[1] * e[2]);
    const unsigned m2 = e2 > 1u ? (unsigned)((0x100000000ull + e2 - 1) / e2) : 0u;
    const unsigned m12 = e12 > 1u ? (unsigned)((0x100000000ull + e12 - 1) / e12) : 0u;
    const unsigned e1 = (unsigned)e[1];
    for (int i = threadIdx.x; i < ncell; i += blockDim.x) {
        const unsigned row = div_small((unsigned)i, e2, m2);  // li * e1 + lj
        const unsigned lk = (unsigned)i - row * e2;
        const unsigned lii = div_small((unsigned)i, e12, m12);
        const unsigned lj = row - lii * e1;
        const int c = (int)(lii + 1) * S0 + (int)(lj + 1) * S1 + (int)lk + 1;
        const long long q = (long long)(((unsigned long long)hi[c] << 32) | lo[c]);
        acc += q;
        const int64_t gidx = ((int64_t)(o[0] + (int)lii) * g.n[1] + (o[1] + (int)lj)) * g.n[2] + (o[2] + (int)lk);
        mesh[gidx] = convert_out<OutT>(q, s, sc);
    }
    // Deterministic block sum of the integer cell sums.
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long tot = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += red[i];
        brick_sum[B] = ldexp((double)tot, -s);
    }
}

// Keys only (cam_cell_keys).
template <int SCHEME>
__global__ void keys_kernel(const float *__restrict__ x, const float *__restrict__ y,
                            const float *__restrict__ z, int64_t np, AssignGeom g,
                            int64_t *__restrict__ keys)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t ncell = (int64_t)g.n[0] * g.n[1] * g.n[2];
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += stride) {
        const float pos[3] = {x[p], y[p], z[p]};
        int c[3];
        keys[p] = home_cell<SCHEME>(pos, g, c)
                      ? (int64_t)c[2] + (int64_t)g.n[2] * ((int64_t)c[1] + (int64_t)g.n[1] * c[0])
                      : ncell;
    }
}

int grid_for(int64_t work, int threads)
{
    const int64_t blocks = (work + threads - 1) / threads;
    const int64_t cap = (int64_t)kNumSMs * 8;
    return (int)std::max<int64_t>(1, std::min(blocks, cap));
}

}  // namespace

AssignGeom make_geom(const cam_grid &gr, int scheme, int64_t np)
{
    AssignGeom g{};
    for (int a = 0; a < 3; ++a) {
        CAM_REQUIRE(gr.n[a] >= 1 && gr.n[a] <= (1 << 20), CAM_E_INVAL, "grid size out of range");
        CAM_REQUIRE(std::isfinite(gr.L[a]) && gr.L[a] > 0.f, CAM_E_INVAL, "box side must be > 0");
        g.n[a] = (int)gr.n[a];
        g.L[a] = gr.L[a];
        g.d[a] = gr.d[a] != 0.f ? gr.d[a] : gr.L[a] / (float)gr.n[a];
        g.mn[a] = gr.min[a];
        CAM_REQUIRE(std::isfinite(g.d[a]) && g.d[a] > 0.f, CAM_E_INVAL, "cell size must be > 0");
        CAM_REQUIRE(std::isfinite(g.mn[a]), CAM_E_INVAL, "box origin must be finite");
    }
    // Brick extents: z 32 (128-byte rows), y and x 16; shrunk (to 4) while
    // the mesh has too few bricks to fill the GPU.  TSC needs >= 3 cells
    // per brick axis unless one brick spans the axis.
    g.b[2] = std::min(g.n[2], 32);
    g.b[1] = std::min(g.n[1], 16);
    g.b[0] = std::min(g.n[0], 16);
    auto nbricks = [&]() {
        int64_t t = 1;
        for (int a = 0; a < 3; ++a) t *= (g.n[a] + g.b[a] - 1) / g.b[a];
        return t;
    };
    const int64_t want = std::min<int64_t>(4 * kNumSMs, std::max<int64_t>(1, np / 4096));
    while (nbricks() < want && (g.b[0] > 4 || g.b[1] > 4)) {
        if (g.b[0] >= g.b[1] && g.b[0] > 4) g.b[0] = (g.b[0] + 1) / 2;
        else g.b[1] = (g.b[1] + 1) / 2;
    }
    // A stencil of width <= 3 must never span three bricks: a partial last
    // brick keeps at least 2 cells (shrink the brick until it does).
    for (int a = 0; a < 3; ++a) {
        while (g.b[a] < g.n[a] && g.n[a] % g.b[a] != 0 && g.n[a] % g.b[a] < 2 && g.b[a] > 3) --g.b[a];
        g.nb[a] = (g.n[a] + g.b[a] - 1) / g.b[a];
        g.bmagic[a] = (unsigned)(((1ull << 32) + (uint64_t)g.b[a] - 1) / (uint64_t)g.b[a]);
        g.inv_d[a] = 1.0f / g.d[a];
    }
    (void)scheme;
    return g;
}

template <int SCHEME>
static void assign_impl(cam_ctx *ctx, const float *x, const float *y, const float *z,
                        const float *w, int64_t np, const AssignGeom &g, AssignOut &out)
{
    const int64_t nb = (int64_t)g.nb[0] * g.nb[1] * g.nb[2];
    CAM_REQUIRE(nb < (1ll << 31), CAM_E_UNSUPPORTED, "too many mesh bricks");
    // Count pass: one CTA of 1024 threads per SM (its brick histogram in
    // shared memory); scatter pass: two CTAs of 512 threads per SM.  Both
    // take contiguous chunks of >= 4096 particles.
    const int G = (int)std::max<int64_t>(1, std::min<int64_t>(kNumSMs, (np + 4095) / 4096));
    const int64_t chunk = std::max<int64_t>(4, ((np + G - 1) / G + 3) & ~(int64_t)3);
    const int G2 = (int)std::max<int64_t>(1, std::min<int64_t>(2 * kNumSMs, (np + 4095) / 4096));
    const int64_t chunk2 = std::max<int64_t>(4, ((np + G2 - 1) / G2 + 3) & ~(int64_t)3);
    auto aligned = [](const void *p) { return p == nullptr || ((uintptr_t)p & 15u) == 0; };
    const bool vec = aligned(x) && aligned(y) && aligned(z) && aligned(w);
    const bool smem_hist = nb <= kSmemBricks;
    // per-brick counters, one per 128-byte line (counts, then cursors)
    auto *table = static_cast<uint32_t *>(scratch(ctx, "asg.cursor", (size_t)nb * kCursorStride * sizeof(uint32_t)));
    auto *start = static_cast<uint32_t *>(scratch(ctx, "asg.start", (nb + 1) * sizeof(uint32_t)));
    auto *stats = static_cast<unsigned long long *>(scratch(ctx, "asg.stats", 64));
    auto *bsum = static_cast<double *>(scratch(ctx, "asg.bsum", nb * sizeof(double)));
    unsigned long long *d_lost = stats;
    unsigned int *d_wmax = reinterpret_cast<unsigned int *>(stats + 1);
    uint32_t *d_total = reinterpret_cast<uint32_t *>(stats + 2);
    unsigned int *d_ovf = reinterpret_cast<unsigned int *>(stats + 3);
    CAM_CUDA_TRY(cudaMemsetAsync(table, 0, (size_t)nb * kCursorStride * sizeof(uint32_t), ctx->stream));
    CAM_CUDA_TRY(cudaMemsetAsync(stats, 0, 64, ctx->stream));

    // Expected records per particle of a uniform catalogue: a stencil
    // crosses a face of a brick of extent b with probability (W-1)/b per
    // axis; at most two bricks per axis.
    double f = 1.0;
    uint64_t per = 1;
    for (int a = 0; a < 3; ++a) {
        if (SCHEME == CAM_NGP || g.nb[a] == 1) continue;
        f *= 1.0 + std::min(1.0, (double)(Stencil<SCHEME>::W - 1) / g.b[a]);
        per *= 2;
    }
    // Slabs (deferred jobs): every brick gets a fixed slab of the payload,
    // sized from the clumping the last exact job run of this mesh shape
    // measured (a slab that overflows makes the job rerun exactly, which
    // measures again); no count pass and no scan then, and the scatter
    // gathers the statistics.  Only while the slabs stay within twice the
    // expected records (or 2^20 records): the scatter slows as the slabs
    // spread its appends over more memory (256^3: 0.37 ms per job densely
    // packed, 0.48 in slabs of twice, 0.55 of four times the mean brick).
    // A context with an HBM budget keeps the exact path, whose payload the
    // budget was sized for.
    const double est_brick = (double)np * f / (double)nb;
    const int64_t shape = ((int64_t)g.n[0] << 32) | ((int64_t)g.n[1] << 16) | (int64_t)g.n[2];
    uint32_t slab = 0;
    if (out.defer && !ctx->sync_free && !ctx->slabs_off && !ctx->budget && np > 0) {
        const auto it = ctx->slab_clump.find(shape);
        if (it != ctx->slab_clump.end()) {
            const uint64_t cap = slab_capacity(it->second * est_brick);
            const double room = std::max(2.0 * (double)np * f, (double)(1u << 20));
            if ((double)nb * (double)cap <= room && (uint64_t)nb * cap < (1ull << 32)) slab = (uint32_t)cap;
        }
    }

    const size_t hsmem = smem_hist ? (size_t)nb * sizeof(uint32_t) : 0;
    auto count_k = smem_hist ? (vec ? bin_kernel<SCHEME, false, true, true> : bin_kernel<SCHEME, false, true, false>)
                             : (vec ? bin_kernel<SCHEME, false, false, true> : bin_kernel<SCHEME, false, false, false>);
    auto scatter_k = slab ? (vec ? bin_kernel<SCHEME, true, false, true, true> : bin_kernel<SCHEME, true, false, false, true>)
                          : (vec ? bin_kernel<SCHEME, true, false, true> : bin_kernel<SCHEME, true, false, false>);
    if (!slab) {
        smem_at_least(count_k, hsmem);
        CAM_LAUNCH_NAMED(ctx, "assign_bin_count", count_k, G, kBinThreads, hsmem, x, y, z, w, np, chunk, g, (int)nb,
                         table, (uint4 *)nullptr, d_lost, d_wmax, (uint64_t)0, d_ovf, 0u);
        if (nb <= (int64_t)kOffThreads * kOffItems) {
            CAM_LAUNCH_NAMED(ctx, "assign_starts", brick_offsets_kernel, 1, kOffThreads, 0, table, (int)nb, start,
                             d_total);
        } else {
            auto *counts = static_cast<uint32_t *>(scratch(ctx, "asg.counts", (size_t)nb * sizeof(uint32_t)));
            const unsigned sg = (unsigned)std::min<int64_t>((nb + 256) / 256, 1024);
            CAM_LAUNCH_NAMED(ctx, "assign_starts", compact_counts_kernel, sg, 256, 0, table, (int)nb, counts);
            exclusive_scan_u32(ctx, counts, nb, d_total);
            CAM_LAUNCH_NAMED(ctx, "assign_starts", brick_starts_kernel, sg, 256, 0, counts, (int)nb, d_total, start,
                             table);
        }
        // the fullest brick, for the slabs of later deferred jobs
        if (!ctx->sync_free) {
            CAM_LAUNCH_NAMED(ctx, "assign_starts", brick_max_kernel, 64, 256, 0, start, (int)nb,
                             reinterpret_cast<unsigned int *>(stats + 5));
            out.brick_est = est_brick;
            out.brick_shape = shape;
        }
    }

    uint64_t total = 0;
    if (slab) {
        total = (uint64_t)nb * slab;
        out.n_lost = -1;
        out.n_in = -1;
    } else if (ctx->sync_free) {
        // No host round trip (stream capture): size the payload for the
        // provable bound, one record per touched brick and at most two
        // bricks per axis.  Lost count and max |w| stay on the device
        // (asg.stats) for the caller to read back with the results.
        total = (uint64_t)np * per;
        CAM_REQUIRE(total < (1ull << 32), CAM_E_UNSUPPORTED, "payload bound exceeds 2^32 records");
        out.n_lost = -1;
        out.n_in = -1;
    } else if (out.defer) {
        // No host round trip: the expected record count of a uniform
        // catalogue (a stencil crosses a face of a brick of extent b with
        // probability (W-1)/b per axis) with a 25% margin, never below what
        // this context used before nor above the provable bound.  The
        // scatter flags records past it; the caller then reruns.
        const uint64_t bound = (uint64_t)np * per;
        uint64_t est = (uint64_t)((double)np * f * 1.25) + 65536;
        est = std::min(bound, std::max(est, ctx->asg_cap));
        total = std::min<uint64_t>(est, 0xffffffffull);
        ctx->asg_cap = std::max(ctx->asg_cap, total);
        out.n_lost = -1;
        out.n_in = -1;
    } else {
        // Payload size and diagnostics back to the host (one synchronisation),
        // with the fullest brick's record count for later slabs.
        unsigned long long hstats[6] = {0, 0, 0, 0, 0, 0};
        CAM_CUDA_TRY(cudaMemcpyAsync(hstats, stats, sizeof(hstats), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        total = (uint32_t)(hstats[2] & 0xffffffffu);
        ctx->asg_cap = std::max<uint64_t>(ctx->asg_cap, total);  // deferred runs size from it
        out.brick_max = hstats[5] & 0xffffffffu;
        const unsigned int wmax_bits = (unsigned int)(hstats[1] & 0xffffffffu);
        CAM_REQUIRE(!w || wmax_bits < 0x7f800000u, CAM_E_NONFINITE, "a particle weight is NaN or infinite");
        out.n_lost = (int64_t)hstats[0];
        out.n_in = np - out.n_lost;
    }

    uint4 *payload = static_cast<uint4 *>(scratch(ctx, "asg.payload", std::max<size_t>(total, 1) * sizeof(uint4)));
    CAM_LAUNCH_NAMED(ctx, "assign_bin_scatter", scatter_k, G2, kScatterThreads, 0, x, y, z, w, np, chunk2, g, (int)nb,
                     table, payload, d_lost, d_wmax, total, d_ovf, slab);

    const size_t smem = (size_t)(g.b[0] + 2) * (g.b[1] + 2) * (g.b[2] + 2) * 2 * sizeof(uint32_t);
    CAM_REQUIRE(smem <= 110 * 1024, CAM_E_UNSUPPORTED, "brick tile too large");
    const int weighted = w != nullptr;
    auto launch_dep = [&](auto kern, auto *mesh) {
        smem_at_least(kern, smem);
        CAM_LAUNCH_NAMED(ctx, "assign_deposit", kern, (unsigned)nb, kDepositThreads, smem, payload, start,
                         (uint32_t)std::min<uint64_t>(total, 0xffffffffull), g, d_wmax, weighted, mesh, bsum, slab,
                         table);
    };
    if (out.precision == CAM_F32)
        launch_dep(deposit_kernel<SCHEME, float>, static_cast<float *>(out.mesh));
    else if (out.precision == CAM_F64)
        launch_dep(deposit_kernel<SCHEME, double>, static_cast<double *>(out.mesh));
    else
        launch_dep(deposit_kernel<SCHEME, uint32_t>, static_cast<uint32_t *>(out.mesh));
    // out.d_sum[0] = sum of the mesh, out.d_sum[1] = mean per cell
    if (out.d_sum) reduce_sum_f64(ctx, bsum, nb, out.d_sum, (double)g.n[0] * g.n[1] * g.n[2]);
}

unsigned long long *assign_stats(cam_ctx *ctx)
{
    return static_cast<unsigned long long *>(scratch(ctx, "asg.stats", 64));
}

void assign_device(cam_ctx *ctx, const float *x, const float *y, const float *z,
                   const float *w, int64_t np, const cam_grid &grid, int scheme, AssignOut &out)
{
    CAM_REQUIRE(np >= 0, CAM_E_INVAL, "negative particle count");
    CAM_REQUIRE(np == 0 || (x && y && z), CAM_E_INVAL, "null particle coordinates");
    CAM_REQUIRE(np < (1ll << 31), CAM_E_UNSUPPORTED, "more than 2^31 particles per call");
    const AssignGeom g = make_geom(grid, scheme, np);
    if (out.precision == -1)
        CAM_REQUIRE(scheme == CAM_NGP && w == nullptr, CAM_E_INVAL, "integer counts need unweighted NGP");
    switch (scheme) {
    case CAM_NGP: assign_impl<CAM_NGP>(ctx, x, y, z, w, np, g, out); break;
    case CAM_CIC: assign_impl<CAM_CIC>(ctx, x, y, z, w, np, g, out); break;
    case CAM_TSC: assign_impl<CAM_TSC>(ctx, x, y, z, w, np, g, out); break;
    default: throw Error{CAM_E_INVAL, "unknown mass assignment scheme"};
    }
}

void cell_keys_device(cam_ctx *ctx, const float *x, const float *y, const float *z, int64_t np,
                      const cam_grid &grid, int scheme, int64_t *keys)
{
    const AssignGeom g = make_geom(grid, scheme, np);
    if (np == 0) return;
    const int gb = grid_for(np, 256);
    switch (scheme) {
    case CAM_NGP: CAM_LAUNCH(ctx, keys_kernel<CAM_NGP>, gb, 256, 0, x, y, z, np, g, keys); break;
    case CAM_CIC: CAM_LAUNCH(ctx, keys_kernel<CAM_CIC>, gb, 256, 0, x, y, z, np, g, keys); break;
    case CAM_TSC: CAM_LAUNCH(ctx, keys_kernel<CAM_TSC>, gb, 256, 0, x, y, z, np, g, keys); break;
    default: throw Error{CAM_E_INVAL, "unknown mass assignment scheme"};
    }
}

}  // namespace cam

// Particle -> mesh mass assignment (NGP / CIC / TSC) for sm_100a.
//
// Replaces getDensity_NGP / getDensity_CIC / getDensity_TSC,
// Source/massFunctions.cpp:35-98, :678-790, :1050-1165.
//
// Pipeline (no float atomics, bitwise deterministic):
//   1. bin_count   : each CTA takes a contiguous chunk of particles and
//                    computes, per particle, the reference's FP32 home cell
//                    (bit-exact key) and the mesh bricks its stencil
//                    touches; a shared-memory histogram per CTA gives the
//                    table count[brick][cta].  Also lost particles, max |w|.
//   2. scan        : exclusive scan of the table in brick-major order, so
//                    every (brick, cta) pair owns a contiguous payload range.
//   3. bin_scatter : the same CTAs re-read their chunks and write one
//                    16-byte payload per touched brick at their own cursors
//                    (shared-memory atomics only): home cell relative to the
//                    brick, exact fractional offset in fixed point, weight.
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

#include "cam_assign_device.cuh"
#include "cam_internal.h"

namespace cam {
namespace {

constexpr int kBinThreads = 1024;
constexpr int kDepositThreads = 512;
constexpr int kScatterThreads = 512;  // scatter pass: two CTAs per SM
constexpr int kSmemBricks = 16384;  // per-CTA brick histogram in shared memory (64 KB)
using namespace asg;


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
template <int SCHEME, bool SCATTER, bool SMEM, bool VEC>
__global__ void __launch_bounds__(kBinThreads)
bin_kernel(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
           const float *__restrict__ w, int64_t np, int64_t chunk, AssignGeom g, int nb,
           uint32_t *__restrict__ table, uint4 *__restrict__ payload, unsigned long long *__restrict__ lost,
           unsigned int *__restrict__ wmax_bits, uint64_t cap, unsigned int *__restrict__ ovf,
           AssignGeom g1, int nsb, uint32_t *__restrict__ sb_table)
{
    extern __shared__ uint32_t hist[];
    constexpr bool kHist = SMEM && !SCATTER;
    const int G = gridDim.x, blk = blockIdx.x;
    const int lane = threadIdx.x & 31;
    // count pass of the two-level scatter (nsb > 0): also one count per
    // particle for its super-brick, in hist[nb, nb + nsb)
    // (always in shared memory, after the brick histogram if that is too)
    const bool coarse = !SCATTER && nsb > 0;
    uint32_t *sbh = hist + (kHist ? nb : 0);
    if (kHist || coarse) {
        for (int i = threadIdx.x; i < (kHist ? nb : 0) + (coarse ? nsb : 0); i += blockDim.x) hist[i] = 0u;
        __syncthreads();
    }
    unsigned long long my_lost = 0;
    unsigned int my_wmax = 0, my_neg = 0, my_wminc = 0;
    const bool weighted = w != nullptr;
    auto one = [&](float px, float py, float pz, float wt) {
        if (SCATTER)
            bin_one<SCHEME, true, false>(px, py, pz, wt, weighted, g, G, blk, hist, table, payload, cap, ovf,
                                         my_lost, my_wmax, my_neg);
        else
            count_one<SCHEME, kHist>(px, py, pz, wt, weighted, g, hist, table, my_lost, my_wmax, my_neg,
                                     my_wminc, coarse ? &g1 : nullptr, sbh);
    };
    const int64_t p0 = (int64_t)blk * chunk, p1 = min(np, p0 + chunk);
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
    if (!SCATTER) {
        // Warp reductions, one atomic per warp.
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
        if (kHist || coarse) __syncthreads();
        if (kHist)
            for (int i = threadIdx.x; i < nb; i += blockDim.x)
                if (hist[i]) atomicAdd(table + (int64_t)i * kCursorStride, hist[i]);
        if (coarse)
            for (int i = threadIdx.x; i < nsb; i += blockDim.x)
                if (sbh[i]) atomicAdd(sb_table + (int64_t)i * kCursorStride, sbh[i]);
    }
}

// Warp-aggregated reservations in shared memory (every lane of the warp
// calls them): the lanes' n add to *counter with one atomic per warp.
// warp_reserve returns the lane's first slot; warp_add returns nothing.
__device__ __forceinline__ uint32_t warp_reserve(uint32_t *counter, uint32_t n)
{
    const int lane = threadIdx.x & 31;
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    uint32_t base = 0;
    if (lane == 31 && incl) base = atomicAdd(counter, incl);
    base = __shfl_sync(0xffffffffu, base, 31);
    return base + incl - n;
}
__device__ __forceinline__ void warp_add(uint32_t *counter, uint32_t n)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(counter, n);
}

// Pass 3, staged form (nb <= kStageBricks).  Each CTA stages the records of
// a contiguous particle chunk in shared memory and writes them out in
// flushes: a flush ranks its records by brick (shared-memory counts), takes
// one global range per brick it holds (one atomic on the brick's cursor per
// brick and flush instead of one per record) and writes the records in
// brick order, so a warp's stores land in runs of consecutive slots.
// Records past the payload's capacity are flagged, not written.
constexpr int kStageThreads = 1024;
constexpr int kStageCap = 8192;     // staged records per flush (128 KB)
constexpr int kStageBricks = 4096;  // bricks whose counts and ranges fit beside them
constexpr int kStagePer = kStageBricks / 1024;  // scan items per thread of a flush
constexpr int kStageRankBits = 13;  // kStageCap = 2^13

template <int SCHEME>
__global__ void __launch_bounds__(kStageThreads, 1)
scatter_staged_kernel(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                      const float *__restrict__ w, int64_t np, int64_t chunk, AssignGeom g, int nb,
                      uint32_t *__restrict__ table, uint4 *__restrict__ payload, uint64_t cap,
                      unsigned int *__restrict__ ovf)
{
    using St = Stencil<SCHEME>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4 *srec = reinterpret_cast<uint4 *>(smem_raw);                  // [kStageCap]
    uint32_t *skey = reinterpret_cast<uint32_t *>(srec + kStageCap);     // [kStageCap] brick << 13 | rank
    uint16_t *sperm = reinterpret_cast<uint16_t *>(skey + kStageCap);    // [kStageCap] slot -> staged record
    uint32_t *cnt = reinterpret_cast<uint32_t *>(sperm + kStageCap);     // [nb] records per brick, this flush
    uint32_t *off = cnt + kStageBricks;                                  // [nb] first slot of each brick
    uint32_t *gdel = off + kStageBricks;                                 // [nb] global slot - local slot
    __shared__ uint32_t s_fill, s_need, s_wsum[kStageThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int b = tid; b < nb; b += kStageThreads) cnt[b] = 0u;
    if (tid == 0) {
        s_fill = 0u;
        s_need = 0u;
    }
    __syncthreads();
    const bool weighted = w != nullptr;
    const int64_t p0 = (int64_t)blockIdx.x * chunk, p1 = min(np, p0 + chunk);

    // Writes the staged records out (every thread takes part).
    auto flush = [&]() {
        const uint32_t nst = s_fill;
        // exclusive scan of the counts: kStageBricks / kStageThreads per thread
        constexpr int PER = kStageBricks / kStageThreads;
        uint32_t v[PER];
        uint32_t tsum = 0;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int b = tid * PER + k;
            v[k] = b < nb ? cnt[b] : 0u;
            tsum += v[k];
        }
        uint32_t incl = tsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_wsum[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            const uint32_t ws = s_wsum[lane];
            uint32_t wi = ws;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += t;
            }
            s_wsum[lane] = wi - ws;
        }
        __syncthreads();
        uint32_t run = s_wsum[wid] + incl - tsum;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int b = tid * PER + k;
            if (b < nb) {
                off[b] = run;
                // one global range per brick held in this flush
                if (v[k]) gdel[b] = atomicAdd(table + (int64_t)b * kCursorStride, v[k]) - run;
            }
            run += v[k];
        }
        __syncthreads();
        for (uint32_t i = tid; i < nst; i += kStageThreads) {
            const uint32_t key = skey[i];
            sperm[off[key >> kStageRankBits] + (key & ((1u << kStageRankBits) - 1u))] = (uint16_t)i;
        }
        __syncthreads();
        for (uint32_t j = tid; j < nst; j += kStageThreads) {
            const uint32_t i = sperm[j];
            const uint32_t slot = gdel[skey[i] >> kStageRankBits] + j;
            if (slot < cap) payload[slot] = srec[i];
            else atomicOr(ovf, 1u);
        }
        __syncthreads();
        for (int b = tid; b < nb; b += kStageThreads) cnt[b] = 0u;
        if (tid == 0) s_fill = 0u;
        __syncthreads();
    };

    for (int64_t base = p0; base < p1; base += kStageThreads) {
        const int64_t p = base + tid;
        int c[3] = {0, 0, 0}, bl[3] = {0, 0, 0}, nbx[3] = {0, 0, 0};
        float t[3] = {0.f, 0.f, 0.f};
        float wt = 1.0f;
        int nrec = 0;
        if (p < p1) {
            const float pos[3] = {__ldcs(x + p), __ldcs(y + p), __ldcs(z + p)};
            if (weighted) wt = __ldcs(w + p);
            if (home_cell<SCHEME>(pos, g, c)) {
                nrec = 1;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    int lo, hi;
                    stencil_ends<SCHEME>(c[a], g.n[a], lo, hi);
                    bl[a] = brick_of(lo, g.b[a], g.bmagic[a]);
                    nbx[a] = (brick_of(hi, g.b[a], g.bmagic[a]) == bl[a]) ? 1 : 2;
                    if (SCHEME != CAM_NGP) t[a] = exact_offset(pos[a], g.mn[a], g.d[a], g.inv_d[a], c[a], g.n[a]);
                    nrec *= nbx[a];
                }
            }
        }
        // room for this round's records, else flush first
        warp_add(&s_need, (uint32_t)nrec);
        __syncthreads();
        const bool full = s_fill + s_need > (uint32_t)kStageCap;
        __syncthreads();
        if (full) flush();
        if (tid == 0) s_need = 0u;
        uint32_t dst = warp_reserve(&s_fill, (uint32_t)nrec);
        if (nrec) {
#pragma unroll
            for (int i0 = 0; i0 < 2; ++i0) {
                if (i0 >= nbx[0]) break;
                const int b0 = (bl[0] + i0 == g.nb[0]) ? 0 : bl[0] + i0;
#pragma unroll
                for (int i1 = 0; i1 < 2; ++i1) {
                    if (i1 >= nbx[1]) break;
                    const int b1 = (bl[1] + i1 == g.nb[1]) ? 0 : bl[1] + i1;
#pragma unroll
                    for (int i2 = 0; i2 < 2; ++i2) {
                        if (i2 >= nbx[2]) break;
                        const int b2 = (bl[2] + i2 == g.nb[2]) ? 0 : bl[2] + i2;
                        const int key = brick_linear(g, b0, b1, b2);
                        const uint32_t rank = atomicAdd(cnt + key, 1u);
                        const int o[3] = {b0 * g.b[0], b1 * g.b[1], b2 * g.b[2]};
                        uint32_t word[3];
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const int e = min(g.b[a], g.n[a] - o[a]);
                            int cl = c[a] - o[a];
                            if (cl < -1) cl += g.n[a];
                            else if (cl > e) cl -= g.n[a];
                            word[a] = pack_axis(cl, t[a]);
                        }
                        srec[dst] = make_uint4(word[0], word[1], word[2], __float_as_uint(wt));
                        skey[dst] = ((uint32_t)key << kStageRankBits) | rank;
                        ++dst;
                    }
                }
            }
        }
        __syncthreads();
    }
    if (s_fill) flush();
    (void)St::W;
}

// ---- two-level scatter (meshes with more bricks than the staged scatter
// holds).  Level 1 partitions the particles by the super-brick of their
// home cell (one raw 16-byte record per particle, x, y, z, w); level 2
// takes each super-brick's particles and writes their brick records, every
// brick of a window of (sx + 2)(sy + 2)(sz + 2) bricks around the
// super-brick being one bucket.  Both stage records in shared memory and
// write them in bucket order, so stores land in runs.

// Flush of a stage: nst records srec[i] with key skey[i] = bucket << 13 |
// rank, bucket counts cnt[0, nbk); dst(bucket) gives the bucket's global
// cursor.  Takes one range per bucket, writes the records in bucket order
// and clears the counts.  Every thread calls it.
template <typename CursorOf>
__device__ __forceinline__ void stage_flush(uint4 *srec, uint32_t *skey, uint16_t *sperm, uint32_t *cnt, uint32_t *off,
                                            uint32_t *gdel, uint32_t *s_wsum, int nbk, uint32_t nst, CursorOf cursor_of,
                                            uint4 *__restrict__ out, uint64_t cap, unsigned int *__restrict__ ovf)
{
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    constexpr int PER = kStagePer;
    uint32_t v[PER];
    uint32_t tsum = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int b = tid * PER + k;
        v[k] = b < nbk ? cnt[b] : 0u;
        tsum += v[k];
    }
    uint32_t incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const uint32_t ws = s_wsum[lane];
        uint32_t wi = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        s_wsum[lane] = wi - ws;
    }
    __syncthreads();
    uint32_t run = s_wsum[wid] + incl - tsum;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int b = tid * PER + k;
        if (b < nbk) {
            off[b] = run;
            if (v[k]) gdel[b] = atomicAdd(cursor_of(b), v[k]) - run;
        }
        run += v[k];
    }
    __syncthreads();
    for (uint32_t i = tid; i < nst; i += kStageThreads) {
        const uint32_t key = skey[i];
        sperm[off[key >> kStageRankBits] + (key & ((1u << kStageRankBits) - 1u))] = (uint16_t)i;
    }
    __syncthreads();
    for (uint32_t j = tid; j < nst; j += kStageThreads) {
        const uint32_t i = sperm[j];
        const uint32_t slot = gdel[skey[i] >> kStageRankBits] + j;
        if (slot < cap) out[slot] = srec[i];
        else atomicOr(ovf, 1u);
    }
    __syncthreads();
    for (int b = tid; b < nbk; b += kStageThreads) cnt[b] = 0u;
    __syncthreads();
}

constexpr int kL1Cap = 8192;       // staged raw records per flush
constexpr int kL1Buckets = 1024;   // super-bricks at most
constexpr int kL2Cap = 8192;
constexpr int kL2Buckets = 1024;   // window bricks at most

// Level 1: each CTA stages the raw records of a contiguous particle chunk
// by super-brick (g1's bricks) and flushes them in super-brick order.
template <int SCHEME>
__global__ void __launch_bounds__(kStageThreads, 1)
partition_kernel(const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
                 const float *__restrict__ w, int64_t np, int64_t chunk, AssignGeom g, AssignGeom g1, int nsb,
                 uint32_t *__restrict__ sb_cursor, uint4 *__restrict__ out, uint64_t cap,
                 unsigned int *__restrict__ ovf)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4 *srec = reinterpret_cast<uint4 *>(smem_raw);
    uint32_t *skey = reinterpret_cast<uint32_t *>(srec + kL1Cap);
    uint16_t *sperm = reinterpret_cast<uint16_t *>(skey + kL1Cap);
    uint32_t *cnt = reinterpret_cast<uint32_t *>(sperm + kL1Cap);
    uint32_t *off = cnt + kL1Buckets;
    uint32_t *gdel = off + kL1Buckets;
    __shared__ uint32_t s_fill, s_wsum[kStageThreads / 32];
    const int tid = threadIdx.x;
    for (int b = tid; b < nsb; b += kStageThreads) cnt[b] = 0u;
    if (tid == 0) s_fill = 0u;
    __syncthreads();
    const bool weighted = w != nullptr;
    auto cursor_of = [&](int b) { return sb_cursor + (int64_t)b * kCursorStride; };
    const int64_t p0 = (int64_t)blockIdx.x * chunk, p1 = min(np, p0 + chunk);
    for (int64_t base = p0; base < p1; base += kStageThreads) {
        // a round adds at most kStageThreads records
        if (s_fill + kStageThreads > (uint32_t)kL1Cap) {
            stage_flush(srec, skey, sperm, cnt, off, gdel, s_wsum, nsb, s_fill, cursor_of, out, cap, ovf);
            if (tid == 0) s_fill = 0u;
            __syncthreads();
        }
        const int64_t p = base + tid;
        float px = 0.f, py = 0.f, pz = 0.f, pw = 1.0f;
        int c[3] = {0, 0, 0};
        bool ok = false;
        if (p < p1) {
            px = __ldcs(x + p);
            py = __ldcs(y + p);
            pz = __ldcs(z + p);
            if (weighted) pw = __ldcs(w + p);
            const float pos[3] = {px, py, pz};
            ok = home_cell<SCHEME>(pos, g, c);
        }
        const uint32_t dst = warp_reserve(&s_fill, ok ? 1u : 0u);
        if (ok) {
            const int key = brick_linear(g1, brick_of(c[0], g1.b[0], g1.bmagic[0]),
                                         brick_of(c[1], g1.b[1], g1.bmagic[1]),
                                         brick_of(c[2], g1.b[2], g1.bmagic[2]));
            const uint32_t rank = atomicAdd(cnt + key, 1u);
            srec[dst] = make_uint4(__float_as_uint(px), __float_as_uint(py), __float_as_uint(pz),
                                   __float_as_uint(pw));
            skey[dst] = ((uint32_t)key << kStageRankBits) | rank;
        }
        __syncthreads();
    }
    if (s_fill) stage_flush(srec, skey, sperm, cnt, off, gdel, s_wsum, nsb, s_fill, cursor_of, out, cap, ovf);
}

// Work items of level 2: super-brick sb holds ceil(count / R) items;
// items[sb] = the first item of sb, items[nsb] = all items.  One CTA of
// 1024 threads, nsb <= 1024.
__global__ void __launch_bounds__(1024)
refine_items_kernel(const uint32_t *__restrict__ sb_start, int nsb, int R, uint32_t *__restrict__ items)
{
    __shared__ uint32_t wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t v = tid < nsb ? (sb_start[tid + 1] - sb_start[tid] + R - 1) / R : 0u;
    uint32_t incl = v;
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
    }
    __syncthreads();
    if (tid < nsb) items[tid] = wsum[wid] + incl - v;
    if (tid == nsb - 1) items[nsb] = wsum[wid] + incl;
}

// Level 2: CTAs take items (up to R raw records of one super-brick) in
// turn and write every brick record of those particles inside the
// super-brick's window, staged with the window's bricks as buckets.
template <int SCHEME>
__global__ void __launch_bounds__(kStageThreads, 1)
refine_kernel(const uint4 *__restrict__ raw, const uint32_t *__restrict__ sb_start,
              const uint32_t *__restrict__ items, int nsb, int R, AssignGeom g, AssignGeom g1, int ws0, int ws1,
              int ws2, uint32_t *__restrict__ table, uint4 *__restrict__ payload, uint64_t cap,
              unsigned int *__restrict__ ovf)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4 *srec = reinterpret_cast<uint4 *>(smem_raw);
    uint32_t *skey = reinterpret_cast<uint32_t *>(srec + kL2Cap);
    uint16_t *sperm = reinterpret_cast<uint16_t *>(skey + kL2Cap);
    uint32_t *cnt = reinterpret_cast<uint32_t *>(sperm + kL2Cap);
    uint32_t *off = cnt + kL2Buckets;
    uint32_t *gdel = off + kL2Buckets;
    __shared__ uint32_t s_fill, s_need, s_wsum[kStageThreads / 32];
    __shared__ int s_sb;
    const int tid = threadIdx.x;
    const int nwin = ws0 * ws1 * ws2;
    for (int b = tid; b < nwin; b += kStageThreads) cnt[b] = 0u;
    if (tid == 0) {
        s_fill = 0u;
        s_need = 0u;
    }
    __syncthreads();
    const uint32_t nitems = items[nsb];
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        if (tid == 0) {
            int lo = 0, hi = nsb - 1;  // last sb with items[sb] <= it
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (items[mid] <= it) lo = mid;
                else hi = mid - 1;
            }
            s_sb = lo;
        }
        __syncthreads();
        const int sb = s_sb;
        const uint32_t r0 = sb_start[sb] + (it - items[sb]) * (uint32_t)R;
        const uint32_t r1 = min(r0 + (uint32_t)R, sb_start[sb + 1]);
        // window origin (bricks): the super-brick's first brick - 1 per axis
        const int S2 = sb % g1.nb[2], S1 = (sb / g1.nb[2]) % g1.nb[1], S0 = sb / (g1.nb[2] * g1.nb[1]);
        const int w0 = S0 * (g1.b[0] / g.b[0]) - 1, w1 = S1 * (g1.b[1] / g.b[1]) - 1, w2 = S2 * (g1.b[2] / g.b[2]) - 1;
        // global brick of window bucket k
        auto cursor_of = [&](int k) {
            const int l2 = k % ws2, l1 = (k / ws2) % ws1, l0 = k / (ws2 * ws1);
            const int b0 = (w0 + l0 + g.nb[0]) % g.nb[0], b1 = (w1 + l1 + g.nb[1]) % g.nb[1],
                      b2 = (w2 + l2 + g.nb[2]) % g.nb[2];
            return table + (int64_t)brick_linear(g, b0, b1, b2) * kCursorStride;
        };
        for (uint32_t base = r0; base < r1; base += kStageThreads) {
            const uint32_t p = base + tid;
            int c[3] = {0, 0, 0}, bl[3] = {0, 0, 0}, nbx[3] = {0, 0, 0};
            float t[3] = {0.f, 0.f, 0.f};
            float wt = 0.0f;
            int nrec = 0;
            if (p < r1) {
                const uint4 rv = raw[p];
                const float pos[3] = {__uint_as_float(rv.x), __uint_as_float(rv.y), __uint_as_float(rv.z)};
                wt = __uint_as_float(rv.w);
                if (home_cell<SCHEME>(pos, g, c)) {
                    nrec = 1;
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        int lo, hi;
                        stencil_ends<SCHEME>(c[a], g.n[a], lo, hi);
                        bl[a] = brick_of(lo, g.b[a], g.bmagic[a]);
                        nbx[a] = (brick_of(hi, g.b[a], g.bmagic[a]) == bl[a]) ? 1 : 2;
                        if (SCHEME != CAM_NGP) t[a] = exact_offset(pos[a], g.mn[a], g.d[a], g.inv_d[a], c[a], g.n[a]);
                        nrec *= nbx[a];
                    }
                }
            }
            warp_add(&s_need, (uint32_t)nrec);
            __syncthreads();
            const bool full = s_fill + s_need > (uint32_t)kL2Cap;
            __syncthreads();
            if (full) {
                stage_flush(srec, skey, sperm, cnt, off, gdel, s_wsum, nwin, s_fill, cursor_of, payload, cap, ovf);
                if (tid == 0) s_fill = 0u;
                __syncthreads();
            }
            if (tid == 0) s_need = 0u;
            uint32_t dst = warp_reserve(&s_fill, (uint32_t)nrec);
            if (nrec) {
#pragma unroll
                for (int i0 = 0; i0 < 2; ++i0) {
                    if (i0 >= nbx[0]) break;
                    const int b0 = (bl[0] + i0 == g.nb[0]) ? 0 : bl[0] + i0;
#pragma unroll
                    for (int i1 = 0; i1 < 2; ++i1) {
                        if (i1 >= nbx[1]) break;
                        const int b1 = (bl[1] + i1 == g.nb[1]) ? 0 : bl[1] + i1;
#pragma unroll
                        for (int i2 = 0; i2 < 2; ++i2) {
                            if (i2 >= nbx[2]) break;
                            const int b2 = (bl[2] + i2 == g.nb[2]) ? 0 : bl[2] + i2;
                            // window bucket (the stencil's bricks lie within
                            // one brick of the super-brick)
                            const int l0 = (b0 - w0 + g.nb[0]) % g.nb[0], l1 = (b1 - w1 + g.nb[1]) % g.nb[1],
                                      l2 = (b2 - w2 + g.nb[2]) % g.nb[2];
                            const int key = (l0 * ws1 + l1) * ws2 + l2;
                            const uint32_t rank = atomicAdd(cnt + key, 1u);
                            const int o[3] = {b0 * g.b[0], b1 * g.b[1], b2 * g.b[2]};
                            uint32_t word[3];
#pragma unroll
                            for (int a = 0; a < 3; ++a) {
                                const int e = min(g.b[a], g.n[a] - o[a]);
                                int cl = c[a] - o[a];
                                if (cl < -1) cl += g.n[a];
                                else if (cl > e) cl -= g.n[a];
                                word[a] = pack_axis(cl, t[a]);
                            }
                            srec[dst] = make_uint4(word[0], word[1], word[2], __float_as_uint(wt));
                            skey[dst] = ((uint32_t)key << kStageRankBits) | rank;
                            ++dst;
                        }
                    }
                }
            }
            __syncthreads();
        }
        // a window per super-brick: flush before the next item's window
        if (s_fill) {
            stage_flush(srec, skey, sperm, cnt, off, gdel, s_wsum, nwin, s_fill, cursor_of, payload, cap, ovf);
            if (tid == 0) s_fill = 0u;
            __syncthreads();
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
               OutT *__restrict__ mesh, double *__restrict__ brick_sum)
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

    // records beyond the payload's capacity nrec were not written (overflow flag)
    const uint32_t beg = min(start[B], nrec), end = min(start[B + 1], nrec);
    const bool nonneg = !weighted || wstat[1] == 0u;
    const int s = fixed_scale(wstat, weighted, end - beg);
    // 2^s as two exact factors (s may exceed the float exponent range)
    const float f1 = scalbnf(1.0f, s / 2), f2 = scalbnf(1.0f, s - s / 2);
    // two records per thread per iteration: both loads are in flight before
    // the shared-memory atomics of the first one
    for (uint32_t p = beg + threadIdx.x; p < end; p += 2 * blockDim.x) {
        const uint4 va = payload[p];
        const bool has_b = p + blockDim.x < end;
        const uint4 vb = has_b ? payload[p + blockDim.x] : make_uint4(0u, 0u, 0u, 0u);
        deposit_record<SCHEME>(va, e, whole, S0, S1, f1, f2, nonneg, lo, hi);
        if (has_b) deposit_record<SCHEME>(vb, e, whole, S0, S1, f1, f2, nonneg, lo, hi);
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

// Super-bricks of the two-level scatter: groups of s0 x s1 x s2 bricks
// (powers of two), doubled along the axis with the most super-bricks until
// at most kL1Buckets remain.  g1 is the geometry whose "bricks" are the
// super-bricks (c / (b s) = (c / b) / s, so a brick lies in one
// super-brick); ws the window of a super-brick's records in level 2, its
// bricks plus one on every side.
struct Coarse {
    AssignGeom g1;
    int nsb = 0;
    int ws[3] = {1, 1, 1};
};

static Coarse make_coarse(const AssignGeom &g)
{
    Coarse c;
    int s[3] = {1, 1, 1};
    auto nsb_of = [&](int a) { return (g.nb[a] + s[a] - 1) / s[a]; };
    for (;;) {
        const int64_t t = (int64_t)nsb_of(0) * nsb_of(1) * nsb_of(2);
        if (t <= kL1Buckets) break;
        int best = -1;
        for (int a = 0; a < 3; ++a)
            if (s[a] < g.nb[a] && (best < 0 || nsb_of(a) > nsb_of(best))) best = a;
        if (best < 0) break;
        s[best] *= 2;
    }
    c.g1 = g;
    for (int a = 0; a < 3; ++a) {
        c.g1.b[a] = g.b[a] * s[a];
        c.g1.nb[a] = (g.n[a] + c.g1.b[a] - 1) / c.g1.b[a];
        c.g1.bmagic[a] = (unsigned)(((1ull << 32) + (uint64_t)c.g1.b[a] - 1) / (uint64_t)c.g1.b[a]);
        c.ws[a] = s[a] + 2;
    }
    c.nsb = c.g1.nb[0] * c.g1.nb[1] * c.g1.nb[2];
    return c;
}

template <int SCHEME>
static void assign_impl(cam_ctx *ctx, const float *x, const float *y, const float *z,
                        const float *w, int64_t np, const AssignGeom &g, AssignOut &out)
{
    const int64_t nb = (int64_t)g.nb[0] * g.nb[1] * g.nb[2];
    CAM_REQUIRE(nb < (1ll << 31), CAM_E_UNSUPPORTED, "too many mesh bricks");
    // CTAs of the binning passes: one per SM (contiguous chunks of >= 4096
    // particles).  Few CTAs keep the set of partly written payload sectors
    // (CTAs x bricks x 128 B) inside L2, so sectors are complete before they
    // are written back.
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
    // more bricks than the staged scatter holds: the two-level scatter
    Coarse co;
    bool two_level = nb > kStageBricks && !ctx->no_stage;
    if (two_level) {
        co = make_coarse(g);
        two_level = co.nsb <= kL1Buckets && co.ws[0] * co.ws[1] * co.ws[2] <= kL2Buckets;
    }
    uint32_t *sb_table = nullptr;
    if (two_level) {
        sb_table = static_cast<uint32_t *>(
            scratch(ctx, "asg.sbcur", (size_t)co.nsb * kCursorStride * sizeof(uint32_t)));
        CAM_CUDA_TRY(cudaMemsetAsync(sb_table, 0, (size_t)co.nsb * kCursorStride * sizeof(uint32_t), ctx->stream));
    }
    const int nsb = two_level ? co.nsb : 0;

    const size_t hsmem = (size_t)((smem_hist ? nb : 0) + nsb) * sizeof(uint32_t);
    auto count_k = smem_hist ? (vec ? bin_kernel<SCHEME, false, true, true> : bin_kernel<SCHEME, false, true, false>)
                             : (vec ? bin_kernel<SCHEME, false, false, true> : bin_kernel<SCHEME, false, false, false>);
    auto scatter_k = vec ? bin_kernel<SCHEME, true, false, true> : bin_kernel<SCHEME, true, false, false>;
    smem_at_least(count_k, hsmem);
    CAM_LAUNCH_NAMED(ctx, "assign_bin_count", count_k, G, kBinThreads, hsmem, x, y, z, w, np, chunk, g, (int)nb,
                     table, (uint4 *)nullptr, d_lost, d_wmax, (uint64_t)0, d_ovf, two_level ? co.g1 : g, nsb,
                     sb_table);
    if (nb <= (int64_t)kOffThreads * kOffItems) {
        CAM_LAUNCH_NAMED(ctx, "assign_starts", brick_offsets_kernel, 1, kOffThreads, 0, table, (int)nb, start, d_total);
    } else {
        auto *counts = static_cast<uint32_t *>(scratch(ctx, "asg.counts", (size_t)nb * sizeof(uint32_t)));
        const unsigned sg = (unsigned)std::min<int64_t>((nb + 256) / 256, 1024);
        CAM_LAUNCH_NAMED(ctx, "assign_starts", compact_counts_kernel, sg, 256, 0, table, (int)nb, counts);
        exclusive_scan_u32(ctx, counts, nb, d_total);
        CAM_LAUNCH_NAMED(ctx, "assign_starts", brick_starts_kernel, sg, 256, 0, counts, (int)nb, d_total, start,
                         table);
    }

    uint64_t total = 0;
    if (ctx->sync_free) {
        // No host round trip (stream capture): size the payload for the
        // provable bound, one record per touched brick and at most two
        // bricks per axis.  Lost count and max |w| stay on the device
        // (asg.stats) for the caller to read back with the results.
        int per = 1;
        for (int a = 0; a < 3; ++a) per *= (SCHEME == CAM_NGP || g.nb[a] == 1) ? 1 : 2;
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
        double f = 1.0;
        uint64_t per = 1;
        for (int a = 0; a < 3; ++a) {
            if (SCHEME == CAM_NGP || g.nb[a] == 1) continue;
            f *= 1.0 + std::min(1.0, (double)(Stencil<SCHEME>::W - 1) / g.b[a]);
            per *= 2;
        }
        const uint64_t bound = (uint64_t)np * per;
        uint64_t est = (uint64_t)((double)np * f * 1.25) + 65536;
        est = std::min(bound, std::max(est, ctx->asg_cap));
        total = std::min<uint64_t>(est, 0xffffffffull);
        ctx->asg_cap = std::max(ctx->asg_cap, total);
        out.n_lost = -1;
        out.n_in = -1;
    } else {
        // Payload size and diagnostics back to the host (one synchronisation).
        unsigned long long hstats[3] = {0, 0, 0};
        CAM_CUDA_TRY(cudaMemcpyAsync(hstats, stats, sizeof(hstats), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        total = (uint32_t)(hstats[2] & 0xffffffffu);
        ctx->asg_cap = std::max<uint64_t>(ctx->asg_cap, total);  // deferred runs size from it
        const unsigned int wmax_bits = (unsigned int)(hstats[1] & 0xffffffffu);
        CAM_REQUIRE(!w || wmax_bits < 0x7f800000u, CAM_E_NONFINITE, "a particle weight is NaN or infinite");
        out.n_lost = (int64_t)hstats[0];
        out.n_in = np - out.n_lost;
    }

    uint4 *payload = static_cast<uint4 *>(scratch(ctx, "asg.payload", std::max<size_t>(total, 1) * sizeof(uint4)));
    if (two_level) {
        // level 1: particles by super-brick (one raw record each; lost ones
        // are dropped), then level 2: each super-brick's brick records
        auto *sb_start = static_cast<uint32_t *>(scratch(ctx, "asg.sbstart", (size_t)(nsb + 1) * sizeof(uint32_t)));
        auto *sb_total = static_cast<uint32_t *>(scratch(ctx, "asg.sbtotal", 16));
        auto *items = static_cast<uint32_t *>(scratch(ctx, "asg.items", (size_t)(nsb + 1) * sizeof(uint32_t)));
        auto *raw = static_cast<uint4 *>(scratch(ctx, "asg.raw", (size_t)std::max<int64_t>(np, 1) * sizeof(uint4)));
        CAM_LAUNCH_NAMED(ctx, "assign_starts", brick_offsets_kernel, 1, kOffThreads, 0, sb_table, nsb, sb_start,
                         sb_total);
        const int G3 = (int)std::max<int64_t>(1, std::min<int64_t>(kNumSMs, (np + kStageThreads - 1) / kStageThreads));
        const int64_t chunk3 = (np + G3 - 1) / G3;
        const size_t ssmem1 = (size_t)kL1Cap * (16 + 4 + 2) + (size_t)kL1Buckets * 3 * 4;
        auto pk1 = partition_kernel<SCHEME>;
        smem_at_least(pk1, ssmem1);
        CAM_LAUNCH_NAMED(ctx, "assign_partition", pk1, G3, kStageThreads, ssmem1, x, y, z, w, np, chunk3, g, co.g1,
                         nsb, sb_table, raw, (uint64_t)std::max<int64_t>(np, 1), d_ovf);
        const int R = kL2Cap;
        CAM_LAUNCH_NAMED(ctx, "assign_starts", refine_items_kernel, 1, 1024, 0, sb_start, nsb, R, items);
        const size_t ssmem2 = (size_t)kL2Cap * (16 + 4 + 2) + (size_t)kL2Buckets * 3 * 4;
        auto rk = refine_kernel<SCHEME>;
        smem_at_least(rk, ssmem2);
        CAM_LAUNCH_NAMED(ctx, "assign_bin_scatter", rk, kNumSMs, kStageThreads, ssmem2, raw, sb_start, items, nsb, R, g,
                         co.g1, co.ws[0], co.ws[1], co.ws[2], table, payload, total, d_ovf);
    } else if (nb <= kStageBricks && !ctx->no_stage) {
        // staged scatter: one CTA per SM over contiguous chunks
        const int G3 = (int)std::max<int64_t>(1, std::min<int64_t>(kNumSMs, (np + kStageThreads - 1) / kStageThreads));
        const int64_t chunk3 = (np + G3 - 1) / G3;
        const size_t ssmem = (size_t)kStageCap * (16 + 4 + 2) + (size_t)kStageBricks * 3 * 4;
        auto sk = scatter_staged_kernel<SCHEME>;
        smem_at_least(sk, ssmem);
        CAM_LAUNCH_NAMED(ctx, "assign_bin_scatter", sk, G3, kStageThreads, ssmem, x, y, z, w, np, chunk3, g, (int)nb,
                         table, payload, total, d_ovf);
    } else {
        CAM_LAUNCH_NAMED(ctx, "assign_bin_scatter", scatter_k, G2, kScatterThreads, 0, x, y, z, w, np, chunk2, g,
                         (int)nb, table, payload, d_lost, d_wmax, total, d_ovf, g, 0, (uint32_t *)nullptr);
    }

    const size_t smem = (size_t)(g.b[0] + 2) * (g.b[1] + 2) * (g.b[2] + 2) * 2 * sizeof(uint32_t);
    CAM_REQUIRE(smem <= 110 * 1024, CAM_E_UNSUPPORTED, "brick tile too large");
    const int weighted = w != nullptr;
    auto launch_dep = [&](auto kern, auto *mesh) {
        smem_at_least(kern, smem);
        CAM_LAUNCH_NAMED(ctx, "assign_deposit", kern, (unsigned)nb, kDepositThreads, smem, payload, start,
                         (uint32_t)std::min<uint64_t>(total, 0xffffffffull), g, d_wmax, weighted, mesh, bsum);
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

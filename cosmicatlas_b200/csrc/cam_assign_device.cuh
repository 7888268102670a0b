// Device functions of the mass assignment shared by the multi-CTA passes
// (cam_assign.cu) and the one-CTA-per-job pipeline of the device request
// loop (cam_devloop.cu): the reference's FP32 home cell, the exact
// fractional offsets, the payload record format, the stencil deposit into a
// haloed 64-bit fixed-point tile and its conversion.  Both paths use these
// same functions, so a job's mesh is bit-identical whichever runs it.
// Replaces getDensity_NGP / getDensity_CIC / getDensity_TSC,
// Source/massFunctions.cpp:35-98, :678-790, :1050-1165.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cam_internal.h"

namespace cam {
namespace asg {

// Global per-brick counters and append cursors sit one per 128-byte line:
// atomics on one line are serialised in its L2 slice, so packed counters
// would funnel all bricks through a few slices.
constexpr int kCursorStride = 32;

// Reference FP32 home cell (see orc_keys / ref_home in the oracle).
// NGP: x on [min, min+L); CIC: x - d/2 wrapped once by +-L then [min, min+L);
// TSC: x on [min, min+L].  i = floor((x-min)/d) in IEEE float, then mod N.
template <int SCHEME>
__device__ __forceinline__ bool home_cell(const float p[3], const AssignGeom &g, int c[3])
{
    float q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float v = p[a];
        if (SCHEME == CAM_CIC) {
            v = __fsub_rn(v, __fmul_rn(0.5f, g.d[a]));
            if (v < 0.0f) v = __fadd_rn(v, g.L[a]);
            if (v >= g.L[a]) v = __fsub_rn(v, g.L[a]);
        }
        q[a] = v;
    }
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float hi = __fadd_rn(g.mn[a], g.L[a]);
        ok = ok && (SCHEME == CAM_TSC ? (q[a] >= g.mn[a] && q[a] <= hi)
                                      : (q[a] >= g.mn[a] && q[a] < hi));
    }
    if (!ok) return false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // floor of the IEEE quotient fl(t / d).  The product with 1/d is
        // within 2^-22 u of it; unless that product is this close to an
        // integer both have the same floor, otherwise divide exactly.
        const float t = __fsub_rn(q[a], g.mn[a]);
        float u = __fmul_rn(t, g.inv_d[a]);
        if (fabsf(u - rintf(u)) <= fmaxf(u, 1.0f) * 4.0e-7f) u = __fdiv_rn(t, g.d[a]);
        const int i = (int)floorf(u);
        // fmod(float(i), float(N)): i <= N whenever d = L/N; any i >= 0 otherwise
        c[a] = i < g.n[a] ? i : (i == g.n[a] ? 0 : i % g.n[a]);
    }
    return true;
}

// cell / b for the brick extent b (exact for cell < 2^21, b <= 2^11).
__device__ __forceinline__ int brick_of(int cell, int b, unsigned magic)
{
    return b == 1 ? cell : (int)__umulhi((unsigned)cell, magic);
}

// Exact offset t = (x - min)/d - 1/2 - c in cells, nearest periodic image,
// in FP32 with error-free transformations: TwoSum for x - min and a fused
// multiply-add for the subtraction of (c + 1/2) d (the product is exact
// inside the FMA); the residual (|r| <= 1.5 d) is scaled by 1/d.
// |error| <= ~2e-7 cells.
__device__ __forceinline__ float exact_offset(float x, float mn, float d, float inv_d, int c, int n)
{
    const float hi = __fsub_rn(x, mn);
    const float bb = __fsub_rn(hi, x);
    const float lo = __fadd_rn(__fsub_rn(x, __fsub_rn(hi, bb)), __fsub_rn(-mn, bb));
    const float u = hi * inv_d;
    float ci = (float)c + 0.5f;
    const float diff = u - ci;
    if (diff > 0.5f * (float)n) ci += (float)n;
    else if (diff < -0.5f * (float)n) ci -= (float)n;
    const float r = __fadd_rn(__fmaf_rn(-ci, d, hi), lo);
    return r * inv_d;
}

template <int SCHEME>
struct Stencil {
    static constexpr int W = SCHEME == CAM_NGP ? 1 : (SCHEME == CAM_CIC ? 2 : 3);
    static constexpr int FIRST = SCHEME == CAM_TSC ? -1 : 0;
};

// First and last stencil cells of a home cell c in [0, n), wrapped
// periodically: the stencil reaches at most one cell below 0 (TSC) and at
// most one cell at or above n, so one conditional add or subtract each.
template <int SCHEME>
__device__ __forceinline__ void stencil_ends(int c, int n, int &lo, int &hi)
{
    using St = Stencil<SCHEME>;
    lo = c + St::FIRST;
    hi = c + St::FIRST + St::W - 1;
    if constexpr (St::FIRST < 0) lo = lo < 0 ? lo + n : lo;
    if constexpr (St::FIRST + St::W - 1 > 0) hi = hi >= n ? hi - n : hi;
}

// Payload word per axis: bits 26..31 = home cell relative to the brick + 8,
// bits 0..25 = round(t * 2^24) + 2^24 (t in [-1, 3)).
__device__ __forceinline__ uint32_t pack_axis(int cl, float t)
{
    int tq = __float2int_rn(t * 16777216.0f) + 16777216;
    tq = min(max(tq, 0), (1 << 26) - 1);
    return ((uint32_t)(cl + 8) << 26) | (uint32_t)tq;
}
__device__ __forceinline__ void unpack_axis(uint32_t v, int &cl, float &t)
{
    cl = (int)(v >> 26) - 8;
    t = (float)((int)(v & 0x3FFFFFFu) - 16777216) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ int brick_linear(const AssignGeom &g, int b0, int b1, int b2)
{
    return (b0 * g.nb[1] + b1) * g.nb[2] + b2;
}

// One particle of pass 1: the bricks its stencil touches (the brick of its
// first stencil cell and, along each axis whose stencil crosses a brick
// face, the next brick, periodically) each get one count.
template <int SCHEME, bool SMEM>
__device__ __forceinline__ void count_one(float px, float py, float pz, float wt, bool weighted, const AssignGeom &g,
                                          uint32_t *hist, uint32_t *__restrict__ table, unsigned long long &my_lost,
                                          unsigned int &my_wmax, unsigned int &my_neg, unsigned int &my_wminc)
{
    using St = Stencil<SCHEME>;
    const float pos[3] = {px, py, pz};
    int c[3] = {0, 0, 0};
    if (!home_cell<SCHEME>(pos, g, c)) {
        ++my_lost;
        return;
    }
    if (weighted) {
        my_wmax = max(my_wmax, __float_as_uint(fabsf(wt)));
        my_neg |= wt < 0.0f;
        if (wt != 0.0f) my_wminc = max(my_wminc, 0x7fffffffu - __float_as_uint(fabsf(wt)));
    }
    int bl[3];
    bool two[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int lo, hi;
        stencil_ends<SCHEME>(c[a], g.n[a], lo, hi);
        bl[a] = brick_of(lo, g.b[a], g.bmagic[a]);
        two[a] = St::W > 1 && brick_of(hi, g.b[a], g.bmagic[a]) != bl[a];
    }
    const int s1 = g.nb[2], s0 = g.nb[1] * g.nb[2];
    const int k0 = bl[0] * s0 + bl[1] * s1 + bl[2];
    // key step to the next brick along each axis (periodic)
    const int d2 = bl[2] + 1 == g.nb[2] ? -bl[2] : 1;
    const int d1 = (bl[1] + 1 == g.nb[1] ? -bl[1] : 1) * s1;
    const int d0 = (bl[0] + 1 == g.nb[0] ? -bl[0] : 1) * s0;
    auto add = [&](int key) {
        if (SMEM) atomicAdd(hist + key, 1u);
        else atomicAdd(table + (int64_t)key * kCursorStride, 1u);
    };
    add(k0);
    if (two[2]) add(k0 + d2);
    if (two[1]) {
        add(k0 + d1);
        if (two[2]) add(k0 + d1 + d2);
    }
    if (two[0]) {
        add(k0 + d0);
        if (two[2]) add(k0 + d0 + d2);
        if (two[1]) {
            add(k0 + d0 + d1);
            if (two[2]) add(k0 + d0 + d1 + d2);
        }
    }
}

// One particle of pass 3 (see bin_kernel).  slab > 0: the brick's records
// go to its own slab of `slab` records (payload[key * slab + slot], the
// counter starting at 0), and the weight statistics are gathered here
// (there is no count pass); my_wminc then receives the smallest nonzero
// |w| as count_one keeps it.
template <int SCHEME, bool SCATTER, bool SMEM, int CSTRIDE = kCursorStride>
__device__ __forceinline__ void bin_one(float px, float py, float pz, float wt, bool weighted,
                                        const AssignGeom &g, int G, int blk, uint32_t *hist,
                                        uint32_t *__restrict__ table, uint4 *__restrict__ payload, uint64_t cap,
                                        unsigned int *ovf, unsigned long long &my_lost, unsigned int &my_wmax,
                                        unsigned int &my_neg, unsigned int *my_wminc = nullptr, uint32_t slab = 0)
{
    using St = Stencil<SCHEME>;
    const float pos[3] = {px, py, pz};
    int c[3] = {0, 0, 0};
    if (!home_cell<SCHEME>(pos, g, c)) {
        ++my_lost;
        return;
    }
    if (weighted && (!SCATTER || my_wminc)) {
        my_wmax = max(my_wmax, __float_as_uint(fabsf(wt)));
        my_neg |= wt < 0.0f;
        if (SCATTER && wt != 0.0f) *my_wminc = max(*my_wminc, 0x7fffffffu - __float_as_uint(fabsf(wt)));
    }
    // Bricks touched along each axis: 1 or 2.
    int bl[3], nbx[3];
    float t[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int lo, hi;
        stencil_ends<SCHEME>(c[a], g.n[a], lo, hi);
        bl[a] = brick_of(lo, g.b[a], g.bmagic[a]);
        nbx[a] = (brick_of(hi, g.b[a], g.bmagic[a]) == bl[a]) ? 1 : 2;
        if (SCHEME != CAM_NGP && SCATTER) t[a] = exact_offset(pos[a], g.mn[a], g.d[a], g.inv_d[a], c[a], g.n[a]);
    }
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
                // SMEM: the CTA's shared counters (count: its histogram;
                // scatter: its own cursors into each brick's range);
                // otherwise the global counts / the brick's append cursor
                const uint32_t slot = SMEM ? atomicAdd(hist + key, 1u)
                                           : atomicAdd(table + (int64_t)key * CSTRIDE, 1u);
                if (SCATTER) {
                    const int o[3] = {b0 * g.b[0], b1 * g.b[1], b2 * g.b[2]};
                    uint32_t word[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        // Home cell relative to the brick origin: the periodic
                        // image in [-1, e], e = brick extent, which holds
                        // whenever the stencil touches the brick.
                        const int e = min(g.b[a], g.n[a] - o[a]);
                        int cl = c[a] - o[a];
                        if (cl < -1) cl += g.n[a];
                        else if (cl > e) cl -= g.n[a];
                        word[a] = pack_axis(cl, t[a]);
                    }
                    // records past the payload's capacity (a deferred
                    // estimate that fell short) or past a full slab are
                    // flagged, not written
                    const bool fits = slab ? slot < slab : slot < cap;
                    const uint64_t at = slab ? (uint64_t)key * slab + slot : (uint64_t)slot;
                    if (fits) payload[at] = make_uint4(word[0], word[1], word[2], __float_as_uint(wt));
                    else atomicOr(ovf, 1u);
                }
            }
        }
    }
}

// Cell sum q (units of 2^-s) as the output type; sc = 2^-s, so q * sc is
// exact in double (|q| < 2^63, -97 <= s <= 180) and the float output is one
// rounding of the exact value.
template <typename OutT>
__device__ __forceinline__ OutT convert_out(long long q, int s, double sc);
template <>
__device__ __forceinline__ float convert_out<float>(long long q, int, double sc)
{
    return __double2float_rn((double)q * sc);
}
template <>
__device__ __forceinline__ double convert_out<double>(long long q, int, double sc)
{
    return (double)q * sc;
}
template <>
__device__ __forceinline__ uint32_t convert_out<uint32_t>(long long q, int s, double)
{
    return (uint32_t)(q >> s);
}

// floor(i / d) for i, d < 2^16: multiply-high by m = ceil(2^32 / d) (d > 1).
__device__ __forceinline__ unsigned div_small(unsigned i, unsigned d, unsigned m)
{
    return d == 1u ? i : __umulhi(i, m);
}

// Adds round(v) to the 64-bit fixed-point cell (lo, hi) with 32-bit shared
// atomics: the low word's old value tells whether the add carried, and the
// high word takes the upper 32 bits of the two's complement plus the carry.
// |v| < 2^31 converts in 32 bits (the common case); larger contributions
// (heavy particles when light ones set the scale) convert in 64 bits.
__device__ __forceinline__ void add_fixed(uint32_t *lo, uint32_t *hi, float v)
{
    uint32_t ql, qh;
    if (fabsf(v) < 2147483648.0f) {
        const int q = __float2int_rn(v);
        ql = (uint32_t)q;
        qh = q < 0 ? 0xffffffffu : 0u;
    } else {
        const long long q = __float2ll_rn(v);
        ql = (uint32_t)(unsigned long long)q;
        qh = (uint32_t)((unsigned long long)q >> 32);
    }
    const uint32_t old = atomicAdd(lo, ql);
    const uint32_t carry = (uint32_t)(old + ql) < old ? 1u : 0u;
    const uint32_t hadd = qh + carry;
    if (hadd) atomicAdd(hi, hadd);
}

// The brick's tile has a one-cell halo on every side: tile cell
// (li + 1, lj + 1, lk + 1) holds brick cell (li, lj, lk), li in [-1, e].  A
// record deposits its whole stencil with no per-cell test; the halo cells
// take the contributions that belong to neighbouring bricks (which get the
// particle's own record) and are discarded.  Per axis, a stencil point
// further out than the halo (TSC only: home cell -1 or e) gets weight zero
// and the nearest halo index, so it adds nothing.  Along an axis that one
// brick spans (nb = 1) the stencil wraps periodically inside the brick.
template <int SCHEME>
__device__ __forceinline__ void axis_stencil(uint32_t word, int e, bool whole, float wa[3], int ia[3])
{
    using St = Stencil<SCHEME>;
    int cl;
    float t;
    unpack_axis(word, cl, t);
    if (SCHEME == CAM_NGP) {
        wa[0] = 1.0f;
    } else if (SCHEME == CAM_CIC) {
        wa[0] = 1.0f - t;
        wa[1] = t;
    } else {
        const float hm = 0.5f - t, hp = 0.5f + t;
        wa[0] = 0.5f * hm * hm;
        wa[1] = 0.75f - t * t;
        wa[2] = 0.5f * hp * hp;
    }
#pragma unroll
    for (int i = 0; i < St::W; ++i) {
        int lc = cl + St::FIRST + i;
        if (whole) {
            lc += lc < 0 ? e : (lc >= e ? -e : 0);
        } else if (lc < -1 || lc > e) {
            wa[i] = 0.0f;
            lc = lc < -1 ? -1 : e;
        }
        ia[i] = lc + 1;
    }
}

// Adds the non-negative contribution v < 2^32 (units of the quantum) to the
// cell (lo, hi): one 32-bit atomic, and a carry into the high word when the
// low word wraps.  v < 2^22 converts by adding 2^23 (the float's mantissa
// then holds round(v)); larger values convert with cvt.
template <bool SMALL>
__device__ __forceinline__ void add_nonneg(uint32_t *lo, uint32_t *hi, float v)
{
    uint32_t m;
    if (SMALL) m = __float_as_uint(__fadd_rn(v, 8388608.0f)) - 0x4b000000u;
    else m = __float2uint_rn(v);
    const uint32_t old = atomicAdd(lo, m);
    if (old + m < old) atomicAdd(hi, 1u);
}

// TIER 0: every contribution < 2^22 and >= 0; 1: < 2^32 and >= 0; 2: any.
// The whole stencil is written, halo cells included (they are discarded):
// skipping the stencil rows that lie in the halo along x or y saved
// atomics but cost more in branches (TSC deposit 0.257 -> 0.304 ms per
// 256^3 job with the skip).
template <int SCHEME, int TIER>
__device__ __forceinline__ void deposit_stencil(const float wa[3][3], const int ia[3][3], int S0, int S1, float ws,
                                                uint32_t *lo, uint32_t *hi)
{
    using St = Stencil<SCHEME>;
#pragma unroll
    for (int i = 0; i < St::W; ++i) {
#pragma unroll
        for (int j = 0; j < St::W; ++j) {
            const float wij = ws * wa[0][i] * wa[1][j];
            const int row = ia[0][i] * S0 + ia[1][j] * S1;
#pragma unroll
            for (int k = 0; k < St::W; ++k) {
                const int c = row + ia[2][k];
                const float v = wij * wa[2][k];
                if (TIER == 0) add_nonneg<true>(lo + c, hi + c, v);
                else if (TIER == 1) add_nonneg<false>(lo + c, hi + c, v);
                else add_fixed(lo + c, hi + c, v);
            }
        }
    }
}

// One payload record into the haloed tile.  ws = weight * 2^s; the stencil
// weights are <= 1 (a TSC weight can dip below zero by ~1e-7 next to a cell
// face: such records take the signed path), so |ws| bounds every
// contribution and picks the conversion once per record.
template <int SCHEME>
__device__ __forceinline__ void deposit_record(const uint4 v, const int e[3], const bool whole[3], int S0, int S1,
                                               float f1, float f2, bool nonneg, uint32_t *lo, uint32_t *hi)
{
    float wa[3][3];
    int ia[3][3];
    axis_stencil<SCHEME>(v.x, e[0], whole[0], wa[0], ia[0]);
    axis_stencil<SCHEME>(v.y, e[1], whole[1], wa[1], ia[1]);
    axis_stencil<SCHEME>(v.z, e[2], whole[2], wa[2], ia[2]);
    const float ws = (__uint_as_float(v.w) * f1) * f2;
    bool pos = nonneg;
    if (SCHEME == CAM_TSC) {
#pragma unroll
        for (int a = 0; a < 3; ++a) pos = pos && wa[a][0] >= 0.0f && wa[a][2] >= 0.0f;
    } else if (SCHEME == CAM_CIC) {
#pragma unroll
        for (int a = 0; a < 3; ++a) pos = pos && wa[a][0] >= 0.0f && wa[a][1] >= 0.0f;
    }
    // One conversion path for all lanes of the warp here (the most general
    // one any of them needs): lanes of a warp hold unrelated records, and
    // per-lane paths would run one after the other.  Every path gives the
    // same integer sums.
    const int tier = (pos && ws < 4194304.0f) ? 0 : ((pos && ws < 4294967296.0f) ? 1 : 2);
    const unsigned act = __activemask();
    const int wt = __reduce_max_sync(act, (unsigned)tier);
    if (wt == 0) deposit_stencil<SCHEME, 0>(wa, ia, S0, S1, ws, lo, hi);
    else if (wt == 1) deposit_stencil<SCHEME, 1>(wa, ia, S0, S1, ws, lo, hi);
    else deposit_stencil<SCHEME, 2>(wa, ia, S0, S1, ws, lo, hi);
}

// Pass 4: one CTA per brick, cell sums in 64-bit fixed point of quantum
// 2^-s.  The scale puts the heaviest weight just below 2^31 (one 32-bit
// atomic per contribution) unless that leaves the lightest nonzero weight
// fewer than 2^21 quanta; then the lightest sets it (2^-s <= min|w| 2^-21)
// and heavy contributions take the 64-bit path.  Either way every
// contribution of the lightest particle is rounded to within 2.4e-7 of its
// own weight, whatever the heaviest weighs.  The scale is capped so that no
// cell of the brick can overflow: a cell takes at most one contribution
// (stencil weight <= 1) per record of its brick, so max|w| 2^s * nrec <
// 2^62.  Unit weights use s = 30; NGP counts convert by a shift.
// wstat[0] = bits of max |w|, wstat[1] != 0 if some weight is negative,
// wstat[6] = 0x7fffffff - bits of min nonzero |w| (0: no nonzero weight).
__device__ __forceinline__ int fixed_scale(const unsigned int *wstat, int weighted, uint32_t nrec)
{
    float wmax = 1.0f, wmin = 1.0f;
    if (weighted) {
        if (wstat[6] == 0u) return 0;  // every weight is zero
        wmax = __uint_as_float(wstat[0]);
        wmin = __uint_as_float(0x7fffffffu - wstat[6]);
    }
    int emax = 0, emin = 0;
    frexpf(wmax, &emax);
    frexpf(wmin, &emin);
    const int bits = 32 - __clz(nrec | 1u);  // nrec < 2^bits
    return min(max(31 - emax, 22 - emin), 62 - emax - bits);
}

}  // namespace asg
}  // namespace cam

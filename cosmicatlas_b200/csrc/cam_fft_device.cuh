// Device-side FFT building blocks shared by the FFT and T-web kernels:
// complex helpers, radix-2/3/4/8/16 butterflies and a Stockham stage that runs
// over many independent transforms held in shared memory.
//
// Stage (Stockham autosort, radix R, Ns = product of the radices already
// applied): butterfly j of a transform of length len reads elements
// j + r*len/R, multiplies by exp(-+2 pi i r (j mod Ns) / (Ns R)), applies the
// R-point DFT and writes to (j / Ns) * Ns * R + (j mod Ns) + r * Ns.  After
// the last stage the output is in natural order.  Every thread keeps the
// inputs of its butterflies in registers across a barrier, so one buffer is
// read and rewritten in place.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace cam {

// Stage list of one transform length.  Integer divisions by the stage's
// butterfly count nq = len/R and by Ns are done with precomputed
// multipliers: floor(x / d) = umulhi(x, ceil(2^32 / d)), exact for
// x, d < 2^16 (all lengths here are <= 1024).  d = 1 has no 32-bit
// multiplier (2^32); the stage handles it separately.
struct Radices {
    int n = 0;
    int r[16];
    unsigned mq[16];   // ceil(2^32 / (len / r[s]))
    unsigned mns[16];  // ceil(2^32 / Ns[s]), Ns[s] = r[0] * ... * r[s-1]
};

inline unsigned div_magic(int64_t d) { return (unsigned)(((1ull << 32) + (uint64_t)d - 1) / (uint64_t)d); }

// len = 8^a 3^b {1, 2, 4}: radix-8 stages first, then 3s, then one 8/4/2.
inline Radices factor_radices(int64_t len)
{
    Radices rd;
    int64_t m = len;
    while (m % 8 == 0 && m > 8) { rd.r[rd.n++] = 8; m /= 8; }
    while (m % 3 == 0) { rd.r[rd.n++] = 3; m /= 3; }
    if (m == 8) { rd.r[rd.n++] = 8; m = 1; }
    if (m == 4) { rd.r[rd.n++] = 4; m = 1; }
    if (m == 2) { rd.r[rd.n++] = 2; m = 1; }
    if (m != 1 || len > 4096) {
        rd.n = -1;
        return rd;
    }
    int64_t ns = 1;
    for (int s = 0; s < rd.n; ++s) {
        rd.mq[s] = div_magic(len / rd.r[s]);
        rd.mns[s] = div_magic(ns);
        ns *= rd.r[s];
    }
    return rd;
}

namespace fftdev {

template <typename T>
struct CT;
template <>
struct CT<float> {
    using t = float2;
    static constexpr int kCols = 16;  // 128-byte column tiles
    static constexpr int kPPT = 16;   // complex points per thread
    static constexpr int kMaxR = 16;  // largest radix of the compile-time stage lists
};
template <>
struct CT<double> {
    using t = double2;
    static constexpr int kCols = 8;
    static constexpr int kPPT = 8;
    static constexpr int kMaxR = 8;
};

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return C{a.x - b.x, a.y - b.y}; }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) { return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
// multiply by -i (forward) or +i (inverse)
template <typename C, bool INV>
__device__ __forceinline__ C rot(C a) { return INV ? C{-a.y, a.x} : C{a.y, -a.x}; }

// a * exp(-+ i t) given c = cos t, s = sin t (forward: -, inverse: +)
template <typename C, bool INV, typename T>
__device__ __forceinline__ C twid(C a, T c, T s)
{
    return INV ? C{a.x * c - a.y * s, a.x * s + a.y * c} : C{a.x * c + a.y * s, a.y * c - a.x * s};
}

template <typename C, bool INV>
__device__ __forceinline__ void dft2(C &a, C &b)
{
    const C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <typename C, int R, bool INV>
__device__ __forceinline__ void dft(C *v)
{
    using T = decltype(v[0].x);
    if (R == 2) {
        dft2<C, INV>(v[0], v[1]);
    } else if (R == 3) {
        const T s3 = (T)0.86602540378443864676;  // sin(pi/3)
        const C t1 = cadd(v[1], v[2]);
        const C t2 = C{v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y};
        const C d = csub(v[1], v[2]);
        const C t3 = rot<C, INV>(C{s3 * d.x, s3 * d.y});
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    } else if (R == 4) {
        const C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        const C b0 = cadd(v[1], v[3]), b1 = rot<C, INV>(csub(v[1], v[3]));
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    } else if (R == 8) {
        const T h = (T)0.70710678118654752440;
        C e[4] = {v[0], v[2], v[4], v[6]};
        C o[4] = {v[1], v[3], v[5], v[7]};
        dft<C, 4, INV>(e);
        dft<C, 4, INV>(o);
        // o[k] *= W8^k
        o[1] = INV ? C{h * (o[1].x - o[1].y), h * (o[1].x + o[1].y)}
                   : C{h * (o[1].x + o[1].y), h * (o[1].y - o[1].x)};
        o[2] = rot<C, INV>(o[2]);
        o[3] = INV ? C{-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y)}
                   : C{h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y)};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = cadd(e[k], o[k]);
            v[k + 4] = csub(e[k], o[k]);
        }
    } else if (R == 16) {
        // 4 x 4: n = n2 + 4 n1, k = k1 + 4 k2,
        //   X[k1 + 4 k2] = sum_n2 W4^(n2 k2) W16^(n2 k1) sum_n1 x[n2 + 4 n1] W4^(n1 k1)
        const T c1 = (T)0.92387953251128675613;  // cos(pi/8)
        const T s1 = (T)0.38268343236508977173;  // sin(pi/8)
        const T h = (T)0.70710678118654752440;   // cos(pi/4)
        C a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
            for (int n1 = 0; n1 < 4; ++n1) a[n2][n1] = v[n2 + 4 * n1];
            dft<C, 4, INV>(a[n2]);  // a[n2][k1]
        }
        // W16^(n2 k1), angle 2 pi m / 16 for m = n2 k1
        a[1][1] = twid<C, INV>(a[1][1], c1, s1);   // m = 1
        a[1][2] = twid<C, INV>(a[1][2], h, h);     // m = 2
        a[1][3] = twid<C, INV>(a[1][3], s1, c1);   // m = 3
        a[2][1] = twid<C, INV>(a[2][1], h, h);     // m = 2
        a[2][2] = rot<C, INV>(a[2][2]);            // m = 4
        a[2][3] = twid<C, INV>(a[2][3], -h, h);    // m = 6
        a[3][1] = twid<C, INV>(a[3][1], s1, c1);   // m = 3
        a[3][2] = twid<C, INV>(a[3][2], -h, h);    // m = 6
        a[3][3] = twid<C, INV>(a[3][3], -c1, -s1); // m = 9
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            C b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
            dft<C, 4, INV>(b);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
        }
    }
}

// One Stockham stage over `ncol` independent transforms of length `len`
// stored in shared memory at col*cstride + j*jstride.  JFAST: butterflies
// of one transform are consecutive (row layout); otherwise consecutive
// butterflies walk the NCOL columns (column-tile layout).
template <typename C, int R, int PPT, bool INV, bool JFAST, int NCOL>
__device__ __forceinline__ void stage(C *buf, int len, int ncol, int jstride, int cstride, int Ns,
                                      unsigned mq, unsigned mns, const C *__restrict__ tw, int twmul)
{
    constexpr int MAXIT = (PPT + R - 1) / R;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int nq = len / R;
    const int nbf = nq * (JFAST ? ncol : NCOL);
    const int twstep = (len / (Ns * R)) * twmul;
    C v[MAXIT][R];
    int dsto[MAXIT];
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
        const int bi = tid + it * nthr;
        dsto[it] = -1;
        if (bi < nbf) {
            int j, col;
            if (JFAST) {
                col = nq == 1 ? bi : (int)__umulhi((unsigned)bi, mq);
                j = bi - col * nq;
            } else {
                col = bi % NCOL;
                j = bi / NCOL;
            }
            const C *src = buf + col * cstride + j * jstride;
#pragma unroll
            for (int r = 0; r < R; ++r) v[it][r] = src[r * nq * jstride];
            const int q = Ns == 1 ? j : (int)__umulhi((unsigned)j, mns);
            const int k = j - q * Ns;
            if (Ns > 1) {
                const int step = k * twstep;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    C w = __ldg(tw + r * step);
                    if (INV) w.y = -w.y;
                    v[it][r] = cmul(v[it][r], w);
                }
            }
            dft<C, R, INV>(v[it]);
            dsto[it] = col * cstride + (j + q * Ns * (R - 1)) * jstride;
        }
    }
    __syncthreads();
    const int ostride = Ns * jstride;
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
        if (dsto[it] >= 0) {
            C *dst = buf + dsto[it];
#pragma unroll
            for (int r = 0; r < R; ++r) dst[r * ostride] = v[it][r];
        }
    }
    __syncthreads();
}

template <typename C, int PPT, bool INV, bool JFAST, int NCOL>
__device__ __forceinline__ void block_fft(C *buf, int len, int ncol, int jstride, int cstride,
                                          const Radices &rd, const C *__restrict__ tw, int twmul)
{
    int Ns = 1;
    for (int s = 0; s < rd.n; ++s) {
        const unsigned mq = rd.mq[s], mns = rd.mns[s];
        switch (rd.r[s]) {
        case 8: stage<C, 8, PPT, INV, JFAST, NCOL>(buf, len, ncol, jstride, cstride, Ns, mq, mns, tw, twmul); break;
        case 4: stage<C, 4, PPT, INV, JFAST, NCOL>(buf, len, ncol, jstride, cstride, Ns, mq, mns, tw, twmul); break;
        case 3: stage<C, 3, PPT, INV, JFAST, NCOL>(buf, len, ncol, jstride, cstride, Ns, mq, mns, tw, twmul); break;
        default: stage<C, 2, PPT, INV, JFAST, NCOL>(buf, len, ncol, jstride, cstride, Ns, mq, mns, tw, twmul); break;
        }
        Ns *= rd.r[s];
    }
}

// ---- compile-time stage lists -------------------------------------------
// Same factorisation as factor_radices, evaluated at compile time, so that
// each stage of a known length is inlined with constant Ns and len; the
// register allocator then sees one stage at a time (the runtime stage loop
// above spills on sm_100a).  With MAXR = 16 a length takes radix-16 stages
// first when that needs fewer stages than radix 8 (16, 48, 128, 256, 384,
// 768, 1024): every stage is a full pass through shared memory with two
// barriers, so fewer stages is less traffic and fewer barriers.
constexpr int ct_stages_of(int len, int first)
{
    int n = 0, m = len;
    while (m % first == 0 && m > 8) { ++n; m /= first; }
    while (m % 3 == 0) { ++n; m /= 3; }
    if (m == 16 || m == 8 || m == 4 || m == 2) ++n;
    return n;
}
constexpr int ct_first_radix(int len, int maxr)
{
    return maxr >= 16 && len % 16 == 0 && ct_stages_of(len, 16) < ct_stages_of(len, 8) ? 16 : 8;
}
constexpr int ct_num_stages(int len, int maxr = 8)
{
    return ct_stages_of(len, ct_first_radix(len, maxr));
}
constexpr int ct_radix(int len, int s, int maxr = 8)
{
    const int f = ct_first_radix(len, maxr);
    int k = 0, m = len;
    while (m % f == 0 && m > 8) { if (k == s) return f; ++k; m /= f; }
    while (m % 3 == 0) { if (k == s) return 3; ++k; m /= 3; }
    return m;  // the final 16, 8, 4 or 2
}
constexpr unsigned ct_magic(int d) { return d <= 1 ? 0u : (unsigned)(((1ull << 32) + (unsigned long long)d - 1) / (unsigned long long)d); }

// Threads a CTA runs for NCOL transforms of length LEN at PPT points each
// (a multiple of 32); host and device use the same formula.
constexpr int ct_threads(int len, int ncol, int ppt)
{
    return ((len * ncol + ppt - 1) / ppt + 31) / 32 * 32;
}

// 16-byte asynchronous global -> shared copy (LDGSTS, cached in L2 only)
// and its group fences; the waits are hardware waits on this thread's own
// copies.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Shared-memory slot of tile element i.  With PAD one spare element follows
// every 16: row transforms (JSTRIDE 1) store their first stages with a
// stride of R elements, which without padding lands a warp on a few banks.
// One slot in 16 makes every radix-8 stage of the power-of-two lengths
// conflict-free for 8-byte elements (one in 32 still leaves two-way
// conflicts in the first two stages).
template <bool PAD>
__device__ __forceinline__ int sidx(int i)
{
    return PAD ? i + (i >> 4) : i;
}
// Elements a padded tile of n elements occupies.
__host__ __device__ constexpr int64_t padded_len(int64_t n, bool pad)
{
    return pad ? n + n / 16 + 1 : n;
}

// One Stockham stage with every shape parameter known at compile time:
// NCOL transforms of length LEN, element (col, j) at col*CSTRIDE + j*JSTRIDE
// (slot sidx<PAD> of that), NTHR threads; JFAST as in stage().  Index
// arithmetic reduces to shifts, constant multiplies and (for lengths with a
// factor 3) a constant divide.
template <typename C, int R, bool INV, bool JFAST, int NCOL, int LEN, int NS, int NTHR, int JSTRIDE,
          int CSTRIDE, int TWMUL, bool PAD = false>
__device__ __forceinline__ void stage_ct(C *buf, const C *__restrict__ tw)
{
    constexpr int NQ = LEN / R;
    constexpr int NBF = NQ * NCOL;
    constexpr int MAXIT = (NBF + NTHR - 1) / NTHR;
    constexpr bool EXACT = NBF % NTHR == 0;
    constexpr int TWSTEP = (LEN / (NS * R)) * TWMUL;
    const int tid = threadIdx.x;
    C v[MAXIT][R];
    int dsto[MAXIT];
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
        const int bi = tid + it * NTHR;
        dsto[it] = -1;
        if (EXACT || bi < NBF) {
            const int col = JFAST ? bi / NQ : bi % NCOL;
            const int j = JFAST ? bi % NQ : bi / NCOL;
            const int src = col * CSTRIDE + j * JSTRIDE;
#pragma unroll
            for (int r = 0; r < R; ++r) v[it][r] = buf[sidx<PAD>(src + r * NQ * JSTRIDE)];
            const int q = j / NS;
            const int k = j - q * NS;
            if (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    C w = __ldg(tw + r * k * TWSTEP);
                    if (INV) w.y = -w.y;
                    v[it][r] = cmul(v[it][r], w);
                }
            }
            dft<C, R, INV>(v[it]);
            dsto[it] = col * CSTRIDE + (j + q * NS * (R - 1)) * JSTRIDE;
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < MAXIT; ++it) {
        if (EXACT || dsto[it] >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) buf[sidx<PAD>(dsto[it] + r * NS * JSTRIDE)] = v[it][r];
        }
    }
    __syncthreads();
}

// All stages of a length-LEN transform, layout and thread count fixed at
// compile time (the CTA must run exactly NTHR threads).
// MAXR: largest radix (8, or 16 for kernels whose threads hold 16 points).
template <typename C, bool INV, bool JFAST, int NCOL, int LEN, int NTHR, int JSTRIDE, int CSTRIDE, int TWMUL,
          bool PAD = false, int MAXR = 8, int S = 0, int NS = 1>
__device__ __forceinline__ void block_fft_fixed(C *buf, const C *__restrict__ tw)
{
    if constexpr (S < ct_num_stages(LEN, MAXR)) {
        constexpr int R = ct_radix(LEN, S, MAXR);
        stage_ct<C, R, INV, JFAST, NCOL, LEN, NS, NTHR, JSTRIDE, CSTRIDE, TWMUL, PAD>(buf, tw);
        block_fft_fixed<C, INV, JFAST, NCOL, LEN, NTHR, JSTRIDE, CSTRIDE, TWMUL, PAD, MAXR, S + 1, NS * R>(buf, tw);
    }
}

template <typename C, int PPT, bool INV, bool JFAST, int NCOL, int LEN, int S = 0, int NS = 1>
__device__ __forceinline__ void block_fft_ct(C *buf, int ncol, int jstride, int cstride, const C *__restrict__ tw,
                                             int twmul)
{
    if constexpr (S < ct_num_stages(LEN)) {
        constexpr int R = ct_radix(LEN, S);
        stage<C, R, PPT, INV, JFAST, NCOL>(buf, LEN, ncol, jstride, cstride, NS, ct_magic(LEN / R), ct_magic(NS), tw,
                                           twmul);
        block_fft_ct<C, PPT, INV, JFAST, NCOL, LEN, S + 1, NS * R>(buf, ncol, jstride, cstride, tw, twmul);
    }
}

// Lengths with a compile-time stage list; any other 2^a 3^b length uses the
// runtime stage loop.
#define CAM_FFT_CT_LENGTHS(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

// Transform of length LEN (LEN = 0: runtime length `len` with stage list rd).
template <typename C, int PPT, bool INV, bool JFAST, int NCOL, int LEN>
__device__ __forceinline__ void block_fft_any(C *buf, int len, int ncol, int jstride, int cstride, const Radices &rd,
                                              const C *__restrict__ tw, int twmul)
{
    if constexpr (LEN > 0) block_fft_ct<C, PPT, INV, JFAST, NCOL, LEN>(buf, ncol, jstride, cstride, tw, twmul);
    else block_fft<C, PPT, INV, JFAST, NCOL>(buf, len, ncol, jstride, cstride, rd, tw, twmul);
}

}  // namespace fftdev

// Host side: calls f(std::integral_constant<int, LEN>) for a length with a
// compile-time stage list, or with LEN = 0 for any other length.
template <typename F>
inline void dispatch_fft_len(int64_t len, F &&f)
{
    switch (len) {
#define CAM_FFT_CASE(L) \
    case L: f(std::integral_constant<int, L>{}); return;
        CAM_FFT_CT_LENGTHS(CAM_FFT_CASE)
#undef CAM_FFT_CASE
    default: f(std::integral_constant<int, 0>{}); return;
    }
}

}  // namespace cam

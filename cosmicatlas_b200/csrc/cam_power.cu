// Spherically binned power spectrum with window deconvolution and aliased
// shot noise, FP64 bin sums.  Replaces the octant loop of
// FftwFunctions::power_spectrum, Source/FftwFunctions.cpp:1660-1876.
//
// Mode set: the half-spectrum elements the reference's octant loop visits
// (planes i = N/2 and j = N/2 never; in the k = 0 plane one element of each
// conjugate pair), see pk_visited.  Per mode (FP64):
//   raw = |F|^2 / W^2,   sn = C / W^2,
//   W = prod_axes sinc(pi a / N)^(p+1), C = prod_axes Sq(p, sin(pi a / N))
// (Source/Miscelanious.cpp:2532-2577); both are separable, so the kernel
// multiplies per-axis tables.  The fourth octant uses Re^2 + Im^2 (the
// reference's Im*Re + Im*Re at FftwFunctions.cpp:1853 is corrected).
//
// Determinism: along a row (fixed i, j) the bin index is non-decreasing in
// k, so each warp reduces runs of equal bins with a fixed shuffle tree; run
// heads add to warp-private shared bins; warps and CTAs are combined in a
// fixed order.  No atomics on floating-point values.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cmath>
#include <string>
#include <type_traits>
#include <vector>

#include "cam_internal.h"
#include "cam_pk_device.cuh"

namespace cam {
namespace {

constexpr int kPkThreads = 256;
constexpr int kPkWarps = kPkThreads / 32;

// Legendre polynomials of mu^2 = f^2 / q (FftwFunctions.cpp:1152-1153):
// L_2 = (3 mu^2 - 1) / 2, L_4 = (35 mu^4 - 30 mu^2 + 3) / 8, both even in mu.
__device__ __forceinline__ void legendre24(int f, double q, double &l2, double &l4)
{
    const double m2 = (double)f * (double)f / q;
    l2 = 0.5 * (3.0 * m2 - 1.0);
    l4 = ((35.0 * m2 - 30.0) * m2 + 3.0) * 0.125;
}

// MODE 0: P(k) sums |F|^2 / W^2 and C / W^2.
// MODE 1 (cross): a second spectrum (main2, nyq2); the sums become
// Re(F1 conj F2) / W^2 and |F1|^2 / W^2.
// MODE 2 (multipoles): L_2(mu) |F|^2 / W^2 and L_4(mu) |F|^2 / W^2, mu the
// cosine between k and the line of sight (axis `los`: 0 x, 1 y, 2 z).
// Modes 1 and 2 read the table's second half as 1/W^2: the host builds it
// without shot-noise factors.
template <typename C, int MODE = 0>
__global__ void __launch_bounds__(kPkThreads)
pk_bin_kernel(const C *__restrict__ main, const C *__restrict__ nyq, const C *__restrict__ main2,
              const C *__restrict__ nyq2, int los, int n,
              const double *__restrict__ g_tab /* [3][n/2+1]: 1/W^2 axis, C/W^2 axis ; [nbins+1] E2 */,
              int nbins, float m_u, float inv_s, int64_t rows_per_cta,
              double *__restrict__ part /* [grid][nbins][2] */,
              unsigned long long *__restrict__ part_modes /* [grid][nbins] */)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int h = n / 2;
    const int M = h;
    double *tw2 = reinterpret_cast<double *>(smem_raw);  // [h+1]
    double *tsn = tw2 + (h + 1);                          // [h+1]
    double *E2 = tsn + (h + 1);                           // [nbins+1]
    double *wsum = E2 + (nbins + 1);                      // [warps][nbins][2]
    unsigned long long *wcnt = reinterpret_cast<unsigned long long *>(wsum + (size_t)kPkWarps * nbins * 2);
    for (int t = threadIdx.x; t < 2 * (h + 1) + nbins + 1; t += blockDim.x) tw2[t] = g_tab[t];
    for (int t = threadIdx.x; t < kPkWarps * nbins * 2; t += blockDim.x) wsum[t] = 0.0;
    for (int t = threadIdx.x; t < kPkWarps * nbins; t += blockDim.x) wcnt[t] = 0ull;
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // float spectra with an even row length: two elements per lane
    const bool PAIRED = sizeof(C) == 8 && (M & 1) == 0;
    double *mysum = wsum + (size_t)warp * nbins * 2;
    unsigned long long *mycnt = wcnt + (size_t)warp * nbins;
    const int64_t nrows = (int64_t)n * n;
    const int64_t r_beg = (int64_t)blockIdx.x * rows_per_cta;
    const int64_t r_end = min(nrows, r_beg + rows_per_cta);
    for (int64_t r = r_beg + warp; r < r_end; r += kPkWarps) {
        const int i = (int)r / n, j = (int)r - i * n;  // n * n < 2^31 (host check)
        if (i == h || j == h) continue;
        const int a = i <= h ? i : n - i;
        const int b = j <= h ? j : n - j;
        const double tab_ab = tw2[a] * tw2[b];
        const double sn_ab = tsn[a] * tsn[b];
        const int64_t q0 = (int64_t)a * a + (int64_t)b * b;
        // the two sums of one visited element c (FP64)
        auto elem = [&](double re, double im, double gre, double gim, int cc, double q, double &vr, double &vs) {
            if constexpr (MODE == 1) {
                vr = (re * gre + im * gim) * (tab_ab * tw2[cc]);
                vs = (re * re + im * im) * (sn_ab * tsn[cc]);
            } else if constexpr (MODE == 2) {
                double l2, l4;
                legendre24(los == 0 ? a : (los == 1 ? b : cc), q, l2, l4);
                const double pw = (re * re + im * im) * (tab_ab * tw2[cc]);
                vr = pw * l2;
                vs = pw * l4;
            } else {
                vr = (re * re + im * im) * (tab_ab * tw2[cc]);
                vs = sn_ab * tsn[cc];
            }
        };
        if (PAIRED) {
            // Two elements per lane (c, c + 1) from one 16-byte load; M is
            // even, so both exist together.  Each lane's last element (B,
            // bin2) enters the warp's run reduction; its first element (A,
            // bin1 <= bin2), when its bin differs, either joins the previous
            // lane's B (same bin) or is the only element of its bin in this
            // chunk and is added by its own lane.
            for (int c0 = 0; c0 < M; c0 += 64) {
                const int c = c0 + 2 * lane;
                double ra = 0.0, sa = 0.0, rb = 0.0, sb = 0.0;
                int na = 0, nbv = 0;
                int bin1 = nbins, bin2 = nbins;
                if (c < M) {
                    const double q1 = (double)(q0 + (int64_t)c * c);
                    const double q2 = (double)(q0 + (int64_t)(c + 1) * (c + 1));
                    bin1 = pk_bin(q1, E2, nbins, m_u, inv_s);
                    bin2 = pk_bin(q2, E2, nbins, m_u, inv_s);
                    const float4 f4 = __ldg(reinterpret_cast<const float4 *>(main + r * M + c));
                    float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f);
                    if constexpr (MODE == 1) g4 = __ldg(reinterpret_cast<const float4 *>(main2 + r * M + c));
                    if (bin1 >= 0 && bin1 < nbins && pk_visited(i, j, c, n)) {
                        elem(f4.x, f4.y, g4.x, g4.y, c, q1, ra, sa);
                        na = 1;
                    }
                    if (bin2 >= 0 && bin2 < nbins && pk_visited(i, j, c + 1, n)) {
                        elem(f4.z, f4.w, g4.z, g4.w, c + 1, q2, rb, sb);
                        nbv = 1;
                    }
                }
                const bool split = bin1 != bin2;
                double vraw = rb, vsn = sb;
                int cnt = nbv;
                if (!split) {
                    vraw = ra + rb;
                    vsn = sa + sb;
                    cnt = na + nbv;
                }
                // the next lane's A joins this lane's B when their bins agree
                const int nb1 = __shfl_down_sync(0xffffffffu, bin1, 1);
                const int nsplit = __shfl_down_sync(0xffffffffu, (int)split, 1);
                const double nra = __shfl_down_sync(0xffffffffu, ra, 1);
                const double nsa = __shfl_down_sync(0xffffffffu, sa, 1);
                const int nna = __shfl_down_sync(0xffffffffu, na, 1);
                if (lane < 31 && nsplit && nb1 == bin2) {
                    vraw += nra;
                    vsn += nsa;
                    cnt += nna;
                }
                const int prev = __shfl_up_sync(0xffffffffu, bin2, 1);
                const bool a_alone = split && !(lane > 0 && prev == bin1);
                const bool head = lane == 0 || prev != bin2;
                const unsigned heads = __ballot_sync(0xffffffffu, head);
                const unsigned later = heads & ~((2u << lane) - 1u);
                const int end = later ? __ffs((int)later) - 1 : 32;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const double or_ = __shfl_down_sync(0xffffffffu, vraw, off);
                    const double os = __shfl_down_sync(0xffffffffu, vsn, off);
                    const int oc = __shfl_down_sync(0xffffffffu, cnt, off);
                    if (lane + off < end) {
                        vraw += or_;
                        vsn += os;
                        cnt += oc;
                    }
                }
                if (head && bin2 >= 0 && bin2 < nbins && cnt) {
                    mysum[2 * bin2] += vraw;
                    mysum[2 * bin2 + 1] += vsn;
                    mycnt[bin2] += (unsigned long long)cnt;
                }
                if (a_alone && bin1 >= 0 && bin1 < nbins && na) {
                    mysum[2 * bin1] += ra;
                    mysum[2 * bin1 + 1] += sa;
                    mycnt[bin1] += 1ull;
                }
                __syncwarp();
            }
        }
        for (int c0 = 0; !PAIRED && c0 < M; c0 += 32) {
            const int c = c0 + lane;
            double vraw = 0.0, vsn = 0.0;
            bool valid = false;
            int bin = nbins;
            if (c < M) {
                const double q = (double)(q0 + (int64_t)c * c);
                bin = pk_bin(q, E2, nbins, m_u, inv_s);
                if (bin >= 0 && bin < nbins && pk_visited(i, j, c, n)) {
                    const C f = main[r * M + c];
                    C g{};
                    if constexpr (MODE == 1) g = main2[r * M + c];
                    elem((double)f.x, (double)f.y, (double)g.x, (double)g.y, c, q, vraw, vsn);
                    valid = true;
                }
            }
            // Segmented suffix sums over runs of equal bins (bins are
            // non-decreasing in c, so runs are contiguous lanes); a run ends
            // at the next run head.
            const int prev = __shfl_up_sync(0xffffffffu, bin, 1);
            const bool head = lane == 0 || prev != bin;
            const unsigned heads = __ballot_sync(0xffffffffu, head);
            const unsigned later = heads & ~((2u << lane) - 1u);
            const int end = later ? __ffs((int)later) - 1 : 32;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double or_ = __shfl_down_sync(0xffffffffu, vraw, off);
                const double os = __shfl_down_sync(0xffffffffu, vsn, off);
                if (lane + off < end) {
                    vraw += or_;
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
        // c = M, the Nyquist plane element of the row: one lane adds it
        if (lane == 0) {
            const double q = (double)(q0 + (int64_t)M * M);
            const int bin = pk_bin(q, E2, nbins, m_u, inv_s);
            if (bin >= 0 && bin < nbins && pk_visited(i, j, M, n)) {
                const C f = nyq[r];
                const double re = (double)f.x, im = (double)f.y;
                if constexpr (MODE == 1) {
                    const C g = nyq2[r];
                    mysum[2 * bin] += (re * (double)g.x + im * (double)g.y) * (tab_ab * tw2[M]);
                    mysum[2 * bin + 1] += (re * re + im * im) * (sn_ab * tsn[M]);
                } else if constexpr (MODE == 2) {
                    double l2, l4;
                    legendre24(los == 0 ? a : (los == 1 ? b : M), q, l2, l4);
                    const double pw = (re * re + im * im) * (tab_ab * tw2[M]);
                    mysum[2 * bin] += pw * l2;
                    mysum[2 * bin + 1] += pw * l4;
                } else {
                    mysum[2 * bin] += (re * re + im * im) * (tab_ab * tw2[M]);
                    mysum[2 * bin + 1] += sn_ab * tsn[M];
                }
                mycnt[bin] += 1ull;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int bn = threadIdx.x; bn < nbins; bn += blockDim.x) {
        double s0 = 0.0, s1 = 0.0;
        unsigned long long cn = 0;
        for (int w = 0; w < kPkWarps; ++w) {
            s0 += wsum[((size_t)w * nbins + bn) * 2];
            s1 += wsum[((size_t)w * nbins + bn) * 2 + 1];
            cn += wcnt[(size_t)w * nbins + bn];
        }
        part[((size_t)blockIdx.x * nbins + bn) * 2] = s0;
        part[((size_t)blockIdx.x * nbins + bn) * 2 + 1] = s1;
        part_modes[(size_t)blockIdx.x * nbins + bn] = cn;
    }
}

// One CTA per bin: strided partial sums per thread, then a fixed-shape tree
// (deterministic for a given grid size).
__global__ void __launch_bounds__(256)
pk_final_kernel(const double *__restrict__ part, const unsigned long long *__restrict__ pm, int nparts,
                int nbins, double *__restrict__ out /* [nbins][2] */, unsigned long long *__restrict__ modes)
{
    __shared__ double r0[256], r1[256];
    __shared__ unsigned long long rc[256];
    const int bn = blockIdx.x;
    double s0 = 0.0, s1 = 0.0;
    unsigned long long cn = 0;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) {
        s0 += part[((size_t)p * nbins + bn) * 2];
        s1 += part[((size_t)p * nbins + bn) * 2 + 1];
        cn += pm[(size_t)p * nbins + bn];
    }
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    rc[threadIdx.x] = cn;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            r0[threadIdx.x] += r0[threadIdx.x + h];
            r1[threadIdx.x] += r1[threadIdx.x + h];
            rc[threadIdx.x] += rc[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * bn] = r0[0];
        out[2 * bn + 1] = r1[0];
        modes[bn] = rc[0];
    }
}

double sq_factor(int p, double s)
{
    switch (p) {
    case 0: return 1.0;
    case 1: return 1.0 - (2.0 / 3.0) * s * s;
    case 2: return 1.0 - s * s + (2.0 / 15.0) * s * s * s * s;
    default: return 1.0 - (4.0 / 3.0) * s * s + (2.0 / 5.0) * s * s * s * s - (4.0 / 315.0) * s * s * s * s * s * s;
    }
}

}  // namespace

namespace {

// mode 0: P(k) sums of s; 1: the cross sums of s and s2; 2: the multipole
// sums of s about axis los.  Modes 1 and 2 use buffers of their own (tag),
// so that a P(k) can follow.
PkDevice power_bin_impl(cam_ctx *ctx, const Spectrum &s, const Spectrum *s2, const cam_pk_opts &o, int nbins,
                        const char *tag, int mode = 0, int los = 2)
{
    const int n = (int)s.n, h = n / 2;
    CAM_REQUIRE(nbins >= 1 && nbins <= 4096, CAM_E_INVAL, "nbins must be in [1, 4096]");
    CAM_REQUIRE((int64_t)n * n < (1ll << 31), CAM_E_UNSUPPORTED, "mesh too large for P(k)");
    CAM_REQUIRE(o.ndel > 0.0 && std::isfinite(o.ndel) && std::isfinite(o.DeltaKmin), CAM_E_INVAL,
                "bin width must be > 0");
    CAM_REQUIRE(o.scheme >= 0 && o.scheme <= 2, CAM_E_INVAL, "unknown window scheme");
    const PkTables pt = pk_tables(ctx, n, o, nbins);
    const double *d_tab = pt.tab;
    const size_t tab_bytes = (size_t)(2 * (h + 1) + nbins + 1) * sizeof(double);
    // four CTAs per SM where their shared bins fit (<= 56 KB each), two
    // otherwise: the loop is latency-bound, more resident warps hide it
    const size_t smem_need = tab_bytes + (size_t)kPkWarps * nbins * (2 * sizeof(double) + sizeof(unsigned long long));
    const int grid = kNumSMs * (smem_need <= 56 * 1024 ? 4 : 2);
    const int64_t nrows = (int64_t)n * n;
    const int64_t rpc = (nrows + grid - 1) / grid;
    const std::string tg(tag);
    auto *part = static_cast<double *>(scratch(ctx, (tg + ".part").c_str(), (size_t)grid * nbins * 2 * sizeof(double)));
    auto *pm = static_cast<unsigned long long *>(
        scratch(ctx, (tg + ".pm").c_str(), (size_t)grid * nbins * sizeof(unsigned long long)));
    auto *res = static_cast<double *>(scratch(ctx, (tg + ".res").c_str(), (size_t)nbins * 2 * sizeof(double)));
    auto *resm = static_cast<unsigned long long *>(
        scratch(ctx, (tg + ".resm").c_str(), (size_t)nbins * sizeof(unsigned long long)));
    const size_t smem = tab_bytes + (size_t)kPkWarps * nbins * (2 * sizeof(double) + sizeof(unsigned long long));
    CAM_REQUIRE(smem <= 220 * 1024, CAM_E_UNSUPPORTED, "too many bins for one CTA");
    const float m_u = pt.m_u, inv_s = pt.inv_s;
    auto launch = [&](auto cplx, auto md) {
        using C = decltype(cplx);
        constexpr int X = decltype(md)::value;
        auto kern = pk_bin_kernel<C, X>;
        smem_at_least(kern, smem);
        const C *m2 = X == 1 ? (const C *)s2->main : nullptr;
        const C *q2 = X == 1 ? (const C *)s2->nyq : nullptr;
        CAM_LAUNCH_NAMED(ctx, X == 1 ? "pk_cross_bin" : (X == 2 ? "pk_multipole_bin" : "pk_bin"), kern, grid,
                         kPkThreads, smem, (const C *)s.main, (const C *)s.nyq, m2, q2, los, n, d_tab, nbins, m_u,
                         inv_s, rpc, part, pm);
    };
    auto by_mode = [&](auto cplx) {
        if (mode == 1) launch(cplx, std::integral_constant<int, 1>{});
        else if (mode == 2) launch(cplx, std::integral_constant<int, 2>{});
        else launch(cplx, std::integral_constant<int, 0>{});
    };
    if (s.precision == CAM_F32) by_mode(float2{});
    else by_mode(double2{});
    CAM_LAUNCH(ctx, pk_final_kernel, nbins, 256, 0, part, pm, grid, nbins, res, resm);
    return PkDevice{res, resm};
}

}  // namespace

namespace {
// The bin of every q in [0, qmax] by pk_bin itself, so a table lookup gives
// exactly what pk_bin gives.
__global__ void pk_bintab_kernel(const double *__restrict__ E2, int nbins, float m_u, float inv_s, int qmax,
                                 short *__restrict__ out)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= qmax; q += gridDim.x * blockDim.x)
        out[q] = (short)pk_bin((double)q, E2, nbins, m_u, inv_s);
}
}  // namespace

PkTables pk_tables(cam_ctx *ctx, int64_t n_, const cam_pk_opts &o, int nbins)
{
    const int n = (int)n_;
    // Per-axis tables (FP64): 1/W^2 = sinc^(-2(p+1)), C/W^2; squared edges.
    const int p = o.scheme;
    const int h = (int)(n / 2);
    std::vector<double> tab(2 * (h + 1) + nbins + 1);
    for (int a = 0; a <= h; ++a) {
        const double x = M_PI * (double)a / (double)n;
        const double sc = a == 0 ? 1.0 : std::sin(x) / x;
        double w = 1.0;
        if (o.mas_correction)
            for (int e = 0; e < p + 1; ++e) w *= sc;
        const double iw2 = 1.0 / (w * w);
        tab[a] = iw2;
        tab[h + 1 + a] = (o.sn_correction ? sq_factor(p, std::sin(x)) : 1.0) * iw2;
    }
    for (int b = 0; b <= nbins; ++b) {
        volatile double e = o.DeltaKmin + (double)b * o.ndel;  // no contraction: matches the oracle
        volatile double e2 = e * e;
        tab[2 * (h + 1) + b] = e2;
    }
    const size_t tab_bytes = tab.size() * sizeof(double);
    // One table buffer per (N, scheme, corrections, edges), whose contents
    // the key determines: it is uploaded once, when created.  A captured
    // graph keeps reading the buffer it was captured with, and later calls
    // skip the upload (a pageable copy that would wait for the stream).
    char key[160];
    snprintf(key, sizeof(key), "pk.tab.%d.%d.%d.%d.%d.%.17g.%.17g", n, p, o.mas_correction, o.sn_correction, nbins,
             o.DeltaKmin, o.ndel);
    const auto found = ctx->bufs.find(key);
    const bool fresh = found == ctx->bufs.end() || found->second.ptr == nullptr;
    auto *d_tab = static_cast<double *>(scratch(ctx, key, tab_bytes));
    if (fresh) CAM_CUDA_TRY(cudaMemcpyAsync(d_tab, tab.data(), tab_bytes, cudaMemcpyHostToDevice, ctx->stream));
    PkTables pt{d_tab, nbins, (float)o.DeltaKmin, (float)(1.0 / o.ndel), nullptr, 3 * h * h};
    // the bin table depends on N and the edges only
    CAM_REQUIRE(nbins < 32767, CAM_E_UNSUPPORTED, "too many bins");
    char bkey[160];
    snprintf(bkey, sizeof(bkey), "pk.btab.%d.%d.%.17g.%.17g", n, nbins, o.DeltaKmin, o.ndel);
    const auto bf = ctx->bufs.find(bkey);
    const bool bfresh = bf == ctx->bufs.end() || bf->second.ptr == nullptr;
    auto *d_bt = static_cast<short *>(scratch(ctx, bkey, (size_t)(pt.qmax + 1) * sizeof(short)));
    if (bfresh)
        CAM_LAUNCH_NAMED(ctx, "pk_bintab", pk_bintab_kernel, (unsigned)std::min(1024, pt.qmax / 256 + 1), 256, 0,
                         d_tab + 2 * (h + 1), nbins, pt.m_u, pt.inv_s, pt.qmax, d_bt);
    pt.btab = d_bt;
    return pt;
}

namespace {

// Nyquist-plane elements (c = N/2) of a fused P(k): each warp takes 32 rows
// r = i N + j at a time, every lane bins one element, and lane 0 adds the 32
// values to the warp's own bins in lane order.  part[cta][bin] as the fused
// column pass writes it.
constexpr int kNyqThreads = 256;
__global__ void __launch_bounds__(kNyqThreads)
pk_nyq_kernel(const float2 *__restrict__ nyq, int n, const double *__restrict__ g_tab, int nbins,
              const short *__restrict__ btab, double *__restrict__ part)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int h = n / 2;
    double *tw2 = reinterpret_cast<double *>(smem_raw);  // [h+1]
    double *E2 = tw2 + (h + 1);                          // [nbins+1]
    double *wsum = E2 + (nbins + 1);                     // [warps][nbins]
    constexpr int NW = kNyqThreads / 32;
    for (int t = threadIdx.x; t <= h; t += blockDim.x) tw2[t] = g_tab[t];
    for (int t = threadIdx.x; t <= nbins; t += blockDim.x) E2[t] = g_tab[2 * (h + 1) + t];
    for (int t = threadIdx.x; t < NW * nbins; t += blockDim.x) wsum[t] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *mysum = wsum + (size_t)warp * nbins;
    const int64_t nrows = (int64_t)n * n;
    const int64_t chunk = (nrows + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * chunk, r1 = min(nrows, r0 + chunk);
    for (int64_t rb = r0 + 32 * warp; rb < r1; rb += 32 * NW) {
        const int64_t r = rb + lane;
        int bin = -1;
        double v = 0.0;
        if (r < r1) {
            const int i = (int)(r / n), j = (int)(r - (int64_t)i * n);
            const int a = i <= h ? i : n - i, b = j <= h ? j : n - j;
            bin = btab[a * a + b * b + h * h];
            if (bin >= 0 && bin < nbins && pk_visited(i, j, h, n)) {
                const float2 f = nyq[r];
                v = ((double)f.x * (double)f.x + (double)f.y * (double)f.y) * (tw2[a] * tw2[b] * tw2[h]);
            } else {
                bin = -1;
            }
        }
        for (int l = 0; l < 32; ++l) {
            const int bl = __shfl_sync(0xffffffffu, bin, l);
            const double vl = __shfl_sync(0xffffffffu, v, l);
            if (lane == 0 && bl >= 0) mysum[bl] += vl;
        }
    }
    __syncthreads();
    for (int bn = threadIdx.x; bn < nbins; bn += blockDim.x) {
        double sum = 0.0;
        for (int w = 0; w < NW; ++w) sum += wsum[(size_t)w * nbins + bn];
        part[(size_t)blockIdx.x * nbins + bn] = sum;
    }
}

// One CTA per bin: the fused partials [nparts][nbins] summed by a fixed
// tree, with the static shot-noise sums and mode counts of the mode set.
__global__ void __launch_bounds__(256)
pk_final_fused_kernel(const double *__restrict__ part, int nparts, int nbins, const double *__restrict__ stat,
                      const unsigned long long *__restrict__ stat_modes, double *__restrict__ out,
                      unsigned long long *__restrict__ modes)
{
    __shared__ double r0[256];
    const int bn = blockIdx.x;
    double s0 = 0.0;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) s0 += part[(size_t)p * nbins + bn];
    r0[threadIdx.x] = s0;
    __syncthreads();
    for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
        if (threadIdx.x < hh) r0[threadIdx.x] += r0[threadIdx.x + hh];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * bn] = r0[0];
        out[2 * bn + 1] = stat[2 * bn + 1];
        modes[bn] = stat_modes[bn];
    }
}

}  // namespace

PkDevice power_finish_fused(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins, double *part,
                            int nparts)
{
    const int n = (int)s.n, h = n / 2;
    const PkTables pt = pk_tables(ctx, n, o, nbins);  // built before the column pass
    const int g2 = kNumSMs;
    const size_t smem = (size_t)(h + 1 + nbins + 1 + (kNyqThreads / 32) * nbins) * sizeof(double);
    CAM_REQUIRE(smem <= 220 * 1024, CAM_E_UNSUPPORTED, "too many bins for one CTA");
    double *all = part;  // [nparts + kNumSMs][nbins]: the Nyquist rows follow the column pass's
    smem_at_least(pk_nyq_kernel, smem);
    {
        // on the side stream when the Nyquist plane was transformed there
        // (fft_r2c_pk_fused), then joined back before anything else reads it
        StreamScope side(ctx, ctx->aux_open ? ctx->aux_stream : ctx->stream);
        CAM_LAUNCH_NAMED(ctx, "pk_nyq", pk_nyq_kernel, g2, kNyqThreads, smem, static_cast<const float2 *>(s.nyq), n,
                         pt.tab, nbins, pt.btab, all + (size_t)nparts * nbins);
    }
    aux_join(ctx);
    // Mode counts and shot-noise sums depend on N, the options and the bins
    // only: computed once per key by the binning kernel (its sums of |F|^2
    // are discarded, so the spectrum's contents do not matter) and kept.
    char key[176];
    snprintf(key, sizeof(key), "pks.%d.%d.%d.%d.%d.%.17g.%.17g", n, o.scheme, o.mas_correction, o.sn_correction, nbins,
             o.DeltaKmin, o.ndel);
    const std::string k(key);
    const auto found = ctx->bufs.find(k + ".res");
    PkDevice stat;
    if (found == ctx->bufs.end() || found->second.ptr == nullptr) {
        stat = power_bin_impl(ctx, s, nullptr, o, nbins, key);
    } else {
        stat.sums = static_cast<double *>(found->second.ptr);
        stat.modes = static_cast<unsigned long long *>(ctx->bufs[k + ".resm"].ptr);
    }
    auto *res = static_cast<double *>(scratch(ctx, "pkf.res", (size_t)nbins * 2 * sizeof(double)));
    auto *resm = static_cast<unsigned long long *>(scratch(ctx, "pkf.resm", (size_t)nbins * sizeof(unsigned long long)));
    CAM_LAUNCH_NAMED(ctx, "pk_final", pk_final_fused_kernel, nbins, 256, 0, all, nparts + g2, nbins, stat.sums,
                     stat.modes, res, resm);
    return PkDevice{res, resm};
}

PkDevice job_fft_pk(cam_ctx *ctx, FftPlan *plan, const void *mesh, const double *d_sub, Spectrum &s,
                    const cam_pk_opts *pk, int nb, bool keep)
{
    if (pk) {
        const PkTables pt = pk_tables(ctx, s.n, *pk, nb);
        double *part = nullptr;
        int nparts = 0;
        if (fft_r2c_pk_fused(ctx, plan, mesh, d_sub, s, pt, keep, &part, &nparts))
            return power_finish_fused(ctx, s, *pk, nb, part, nparts);
    }
    fft_r2c_split(ctx, plan, mesh, d_sub, s);
    if (!pk) return PkDevice{nullptr, nullptr};
    return power_bin_device(ctx, s, *pk, nb);
}

PkDevice power_bin_device(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins)
{
    return power_bin_impl(ctx, s, nullptr, o, nbins, "pk");
}

PkDevice power_cross_device(cam_ctx *ctx, const Spectrum &s1, const Spectrum &s2, const cam_pk_opts &o, int nbins)
{
    CAM_REQUIRE(s1.n == s2.n && s1.precision == s2.precision, CAM_E_INVAL, "cross spectra differ in size or precision");
    cam_pk_opts ox = o;
    ox.sn_correction = 0;  // the second table half is then 1/W^2
    return power_bin_impl(ctx, s1, &s2, ox, nbins, "pkx", 1);
}

PkDevice power_multipole_device(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins, int los)
{
    CAM_REQUIRE(los >= 0 && los <= 2, CAM_E_INVAL, "line of sight must be 0 (x), 1 (y) or 2 (z)");
    cam_pk_opts ox = o;
    ox.sn_correction = 0;
    return power_bin_impl(ctx, s, nullptr, ox, nbins, "pkm", 2, los);
}

void power_bin(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins, double *h_sum_raw,
               double *h_sum_sn, int64_t *h_modes)
{
    const PkDevice d = power_bin_device(ctx, s, o, nbins);
    if (ctx->sync_free) return;  // sums stay in pk.res / pk.resm for the caller
    double *res = d.sums;
    unsigned long long *resm = d.modes;
    std::vector<double> hres(2 * nbins);
    std::vector<unsigned long long> hm(nbins);
    CAM_CUDA_TRY(cudaMemcpyAsync(hres.data(), res, 2 * nbins * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CAM_CUDA_TRY(cudaMemcpyAsync(hm.data(), resm, nbins * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int b = 0; b < nbins; ++b) {
        if (h_sum_raw) h_sum_raw[b] = hres[2 * b];
        if (h_sum_sn) h_sum_sn[b] = hres[2 * b + 1];
        if (h_modes) h_modes[b] = (int64_t)hm[b];
    }
}

}  // namespace cam

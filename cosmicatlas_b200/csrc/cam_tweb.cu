// T-web cosmic-web classification for sm_100a.
//
// Replaces Cwclass::get_CWC, Source/Cwclass.cpp:235-890, with the FFT tidal
// tensor of EigenValuesTweb, Source/Miscelanious.cpp:1772-1883, and
// calc_LapPhiv, Source/NumericalMethods.cpp:2609-2680:
//   T_ab(x) = c2r( k_a k_b / k^2 * exp(-k^2 R^2 / 2) * delta_k ) / N^3
// with k_a = k_f * (i <= N/2 ? i : i - N) and T = 0 at k = 0; then per cell
// the eigenvalues lambda1 >= lambda2 >= lambda3 and the label
// 4 - #{lambda_a > lambda_th} (Source/Cwclass.cpp:875-890).
//
// Only the six distinct components are made (the reference transforms
// nine), and the multiplier is split into its separable factors:
//   T_ab = IFFT_z[ k_z^r IFFT_y[ k_y^q IFFT_x[ k_x^p phi ] ] ],
//   phi = delta_k exp(-k^2 R^2 / 2) / k^2,  p + q + r = 2,
// so the x pass transforms three fields (p = 0, 1, 2) instead of six.
// Three kernels:
//   tidal_x    : phi times k_x^p and the inverse FFT along x, p = 0, 1, 2;
//                the three CTAs of one delta_k tile run together, so the
//                tile is read from HBM once and from L2 after;
//   tidal_y    : for input field p, the fields (p, q), q = 0 .. 2-p: times
//                k_y^q k_z^r (r = 2-p-q; k_z is constant along y) and the
//                inverse FFT along y; (p, 0) overwrites its input in place,
//                as the last output of the same CTA;
//   tidal_z    : c2r along z of the six fields of a few rows,
//                then the eigenvalues (FP32 trigonometric solution plus one
//                FP64 Newton step) and the label of every cell (uint8).
// Field slots: 0 = (0,0) -> T_zz, 1 = (1,0) -> T_xz, 2 = (2,0) -> T_xx,
// 3 = (0,1) -> T_yz, 4 = (0,2) -> T_yy, 5 = (1,1) -> T_xy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "cam_fft_device.cuh"
#include "cam_internal.h"

namespace cam {
namespace {

template <typename T>
using CTw = fftdev::CT<T>;

// Rows per CTA of the c2r + eigen pass (6 components of each row):
// about 4096 (float) / 2048 (double) points per CTA.
template <typename T>
constexpr int tweb_rpc(int m)
{
    return (sizeof(T) == 4 ? 4096 : 2048) / (6 * m) > 1 ? (sizeof(T) == 4 ? 4096 : 2048) / (6 * m) : 1;
}

// f^e for e = 0, 1, 2 (exact in float for |f| <= 2048).
__device__ __forceinline__ float ipow(int f, int e)
{
    return e == 0 ? 1.0f : (e == 1 ? (float)f : (float)(f * f));
}

// Field slot of (p, q); the y pass gives it the factor k_z^r, r = 2 - p - q.
__host__ __device__ constexpr int slot_of(int p, int q)
{
    return q == 0 ? p : (p == 0 ? 2 + q : 5);
}

// Frequency factor of one axis in units of k_f, for signed frequency f and
// power e = 0, 1, 2: f^e for the FFT tidal tensor; for the finite-difference
// one (FD), s(f)^e with s the Fourier multiplier of the centred difference,
// tabulated as {s, s^2} (each rounded once from FP64) at sf[f + N/2]
// (fd_table_kernel).
template <typename T, bool FD>
__device__ __forceinline__ T kfac(const typename CTw<T>::t *__restrict__ sf, int h, int f, int e)
{
    if constexpr (!FD) {
        return (T)ipow(f, e);
    } else {
        if (e == 0) return (T)1;
        const typename CTw<T>::t s = __ldg(sf + f + h);
        return e == 1 ? s.x : s.y;
    }
}

}  // namespace


namespace {

// Launch bounds of a column kernel for FFT length LEN: its exact thread
// count, and as many CTAs per SM as fit 1024 threads (768 for lengths with
// a factor 3, whose radix-3 stages need up to ~85 registers).
template <typename T, int LEN>
constexpr int col_threads()
{
    return LEN > 0 ? fftdev::ct_threads(LEN, CTw<T>::kCols, CTw<T>::kPPT) : 1024;
}
template <typename T, int LEN>
constexpr int col_min_blocks()
{
    return ((LEN % 3 == 0 ? 768 : 1024) / col_threads<T, LEN>()) > 1
               ? (LEN % 3 == 0 ? 768 : 1024) / col_threads<T, LEN>()
               : 1;
}

// k_x^p phi / delta_k for signed frequencies (fi, fj, fk).  FD: s(k_x)^p
// phi / delta_k, or, for a potential input (pot), -s(k_x)^p (the host folds
// k_f^2 into norm): nabla^2 phi = delta gives phi_k = -delta_k / k^2
// (PoissonSolver, Source/Miscelanious.cpp:1252-1262), and D_a D_b of phi
// has the multiplier -s_a s_b.
template <typename T, bool FD = false>
__device__ __forceinline__ T phi_mult(int p, int fi, int fj, int fk, T gauss_coef, T norm,
                                      const typename CTw<T>::t *__restrict__ sf = nullptr, int h = 0, int pot = 0)
{
    const int q = fi * fi + fj * fj + fk * fk;
    if (q == 0) return (T)0;
    // f^p and q are exact in float up to N = 2048; one rounding each
    T ratio;
    if constexpr (!FD) {
        ratio = (T)(ipow(fi, p) * (1.0f / (float)q));
    } else {
        const T f = kfac<T, true>(sf, h, fi, p);
        ratio = pot ? -f : f * (T)(1.0f / (float)q);
    }
    const T g = gauss_coef != (T)0 ? exp(-gauss_coef * (T)q) : (T)1;
    return ratio * g * norm;
}

// Inverse FFT along x of k_x^p phi, p = blockIdx.x, for one tile of delta_k.
// NYQ = false: main tiles (plane = j, columns = k < N/2, FFT index i with
// stride N*M).  NYQ = true: the Nyquist plane (columns = j, FFT index i with
// stride N, k = N/2).
template <typename T, bool NYQ, int LEN, bool FD>
__global__ void __launch_bounds__(col_threads<T, LEN>(), col_min_blocks<T, LEN>())
tidal_x_kernel(const typename CTw<T>::t *__restrict__ src, typename CTw<T>::t *__restrict__ dst,
               int n, int ncols, int64_t jstride, int64_t pstride, int64_t ccomp, Radices rd,
               const typename CTw<T>::t *__restrict__ tw, double gauss_coef, const double *__restrict__ d_mean,
               int density_input, double scale, const typename CTw<T>::t *__restrict__ sf, int pot)
{
    using C = typename CTw<T>::t;
    constexpr int W = CTw<T>::kCols;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tile = reinterpret_cast<C *>(smem_raw);
    const int comp = blockIdx.x;  // p; fastest: the three CTAs of a tile run together
    const int col0 = blockIdx.y * W;
    const int plane = blockIdx.z;
    const int nc = min(W, ncols - col0);
    const int h = n / 2;
    const C *g = src + (int64_t)plane * pstride + col0;
    C *o = dst + (int64_t)comp * ccomp + (int64_t)plane * pstride + col0;
    double normd = scale;
    if (density_input) normd /= *d_mean;  // delta_k = F(rho - mean) / mean
    const T norm = (T)normd, gc = (T)gauss_coef;
    const int tot = n * W;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const int i = e / W, cc = e % W;
        if (cc < nc) {
            const C v = g[(int64_t)i * jstride + cc];
            const int fi = i <= h ? i : i - n;
            int fj, fk;
            if (NYQ) {
                const int j = col0 + cc;
                fj = j <= h ? j : j - n;
                fk = h;
            } else {
                fj = plane <= h ? plane : plane - n;
                fk = col0 + cc;
            }
            const T m = phi_mult<T, FD>(comp, fi, fj, fk, gc, norm, sf, h, pot);
            tile[e] = C{v.x * m, v.y * m};
        }
    }
    __syncthreads();
    if constexpr (LEN > 0)
        fftdev::block_fft_fixed<C, true, false, W, LEN, fftdev::ct_threads(LEN, W, CTw<T>::kPPT), W, 1, 1, false,
                                    CTw<T>::kMaxR>(tile, tw);
    else
        fftdev::block_fft<C, CTw<T>::kPPT, true, false, W>(tile, n, W, W, 1, rd, tw, 1);
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
        const int i = e / W, cc = e % W;
        if (cc < nc) o[(int64_t)i * jstride + cc] = tile[e];
    }
}

// Inverse FFT along y of k_y^q k_z^r times field p, q = 2-p .. 0,
// r = 2-p-q, for one tile (p = blockIdx.x, columns blockIdx.y * W.., plane
// blockIdx.z).  Element (plane, j, col) of field s sits at base + s*ccomp +
// plane*pstride + j*jstride + col*cstride.  k_z = kz_fixed if >= 0 (the
// Nyquist plane), else the column.  The tile is re-read (from L2) for every
// q, and (p, 0) is written last, over its own input.
template <typename T, int LEN, bool FD>
__global__ void __launch_bounds__(col_threads<T, LEN>(), col_min_blocks<T, LEN>())
tidal_y_kernel(typename CTw<T>::t *__restrict__ base, int n, int ncols, int64_t jstride, int64_t cstride,
               int64_t pstride, int64_t ccomp, Radices rd, const typename CTw<T>::t *__restrict__ tw, int kz_fixed,
               const typename CTw<T>::t *__restrict__ sf)
{
    using C = typename CTw<T>::t;
    constexpr int W = CTw<T>::kCols;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tile = reinterpret_cast<C *>(smem_raw);
    const int p = blockIdx.x;
    const int col0 = blockIdx.y * W;
    const int nc = min(W, ncols - col0);
    const int h = n / 2;
    const int64_t off = (int64_t)blockIdx.z * pstride + (int64_t)col0 * cstride;
    const C *in = base + (int64_t)p * ccomp + off;
    const int tot = n * W;
    for (int q = 2 - p; q >= 0; --q) {
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            const int j = e / W, cc = e % W;
            if (cc < nc) {
                const C v = in[(int64_t)j * jstride + (int64_t)cc * cstride];
                const int kz = kz_fixed >= 0 ? kz_fixed : col0 + cc;
                T m;
                if constexpr (!FD)
                    m = (T)(ipow(j <= h ? j : j - n, q) * ipow(kz, 2 - p - q));
                else
                    m = kfac<T, true>(sf, h, j <= h ? j : j - n, q) * kfac<T, true>(sf, h, kz, 2 - p - q);
                tile[e] = C{v.x * m, v.y * m};
            }
        }
        __syncthreads();
        if constexpr (LEN > 0)
            fftdev::block_fft_fixed<C, true, false, W, LEN, fftdev::ct_threads(LEN, W, CTw<T>::kPPT), W, 1, 1, false,
                                    CTw<T>::kMaxR>(tile, tw);
        else
            fftdev::block_fft<C, CTw<T>::kPPT, true, false, W>(tile, n, W, W, 1, rd, tw, 1);
        C *o = base + (int64_t)slot_of(p, q) * ccomp + off;
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            const int j = e / W, cc = e % W;
            if (cc < nc) o[(int64_t)j * jstride + (int64_t)cc * cstride] = tile[e];
        }
        __syncthreads();
    }
}

// Columns per tile of the pipelined T-web column kernel: the transform
// precision's 128-byte rows, halved (down to 64-byte rows) until its three
// tiles fit 200 KB of shared memory (N = 768: 8 float columns, 144 KB).
// Halving them at N = 512 too, for two CTAs per SM, measured slower (x pass
// 0.87 -> 0.95 ms, y pass 1.60 -> 1.68 ms at 512^3).
template <typename T, int LEN>
constexpr int tpipe_cols()
{
    int w = CTw<T>::kCols;
    while (w * (int)sizeof(typename CTw<T>::t) > 64 && 3 * LEN * w * (int)sizeof(typename CTw<T>::t) > 200 * 1024)
        w /= 2;
    return w;
}
template <typename T, int LEN>
constexpr int tpipe_threads()
{
    return LEN > 0 ? fftdev::ct_threads(LEN, tpipe_cols<T, LEN>(), CTw<T>::kPPT) : 1024;
}
// CTAs per SM the pipelined T-web column kernel is built for: as many as
// fit 1024 threads and three tiles each in 200 KB of shared memory.
template <typename T, int LEN>
constexpr int tpipe_min_blocks()
{
    constexpr int by_thr = 1024 / tpipe_threads<T, LEN>();
    constexpr int by_smem = (200 * 1024) / (3 * LEN * tpipe_cols<T, LEN>() * (int)sizeof(typename CTw<T>::t));
    constexpr int b = by_thr < by_smem ? by_thr : by_smem;
    return b > 1 ? b : 1;
}

// Pipelined T-web column passes over the main planes; persistent CTAs walk
// the work units blockIdx.x, blockIdx.x + gridDim.x, ...  While a unit is
// worked on, the next unit's input tile is already being copied in
// (asynchronous 16-byte copies), and a separate work tile lets one loaded
// input give several outputs.
//   MODE 0 (x pass): unit = (column tile, plane j) of delta_k; it gives the
//     fields k_x^p phi, p = 0, 1, 2, each transformed along x into slot p.
//   MODE 1 (y pass): unit = (p, column tile, plane i); slot p's tile gives
//     the fields (p, q), q = 2-p .. 0, each times k_y^q and transformed
//     along y into slot_of(p, q); (p, 0) goes last, over its own input.
// Element (j, col) of a tile sits at (tile base) + j*jstride + col, the
// unit's tile base at plane*pstride + column tile*W; full tiles only and
// 16-byte aligned rows (the host checks).
template <typename T, int MODE, int LEN, bool FD>
__global__ void __launch_bounds__(tpipe_threads<T, LEN>(), tpipe_min_blocks<T, LEN>())
tidal_pipe_kernel(const typename CTw<T>::t *src, typename CTw<T>::t *dst, int n, int nct, int64_t nunits,
                  int64_t jstride, int64_t pstride, int64_t ccomp, const typename CTw<T>::t *__restrict__ tw,
                  double gauss_coef, const double *__restrict__ d_mean, int density_input, double scale,
                  const typename CTw<T>::t *__restrict__ sf, int pot)
{
    using C = typename CTw<T>::t;
    constexpr int W = tpipe_cols<T, LEN>();
    constexpr int NTHR = tpipe_threads<T, LEN>();
    constexpr int CPR = W * (int)sizeof(C) / 16;  // 16-byte chunks per tile row
    constexpr int EPC = 16 / (int)sizeof(C);
    constexpr int TILE = LEN * W;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *const in0 = reinterpret_cast<C *>(smem_raw);  // input tiles at in0 and in0 + TILE
    C *const work = in0 + 2 * TILE;
    const int h = n / 2;
    T norm = (T)0, gc = (T)0;
    if (MODE == 0) {
        double normd = scale;
        if (density_input) normd /= *d_mean;  // delta_k = F(rho - mean) / mean
        norm = (T)normd;
        gc = (T)gauss_coef;
    }
    // unit -> (p, column tile, plane); p = 0 for the x pass (all three made)
    auto decode = [&](int64_t t, int &p, int &ct, int &plane) {
        if (MODE == 0) {
            p = 0;
            ct = (int)(t % nct);
            plane = (int)(t / nct);
        } else {
            p = (int)(t % 3);
            const int64_t r = t / 3;
            ct = (int)(r % nct);
            plane = (int)(r / nct);
        }
    };
    auto load = [&](int64_t t, C *buf) {
        int p, ct, plane;
        decode(t, p, ct, plane);
        const C *g = src + (MODE == 1 ? (int64_t)p * ccomp : 0) + (int64_t)plane * pstride + (int64_t)ct * W;
        for (int e = threadIdx.x; e < LEN * CPR; e += NTHR) {
            const int j = e / CPR, k = e % CPR;
            fftdev::cp_async16(buf + j * W + k * EPC, g + (int64_t)j * jstride + k * EPC);
        }
    };
    int cur = 0;
    int64_t t = blockIdx.x;
    if (t < nunits) load(t, in0);
    fftdev::cp_async_commit();
    for (; t < nunits; t += gridDim.x) {
        C *const in = in0 + cur * TILE;
        const int64_t tn = t + gridDim.x;
        if (tn < nunits) load(tn, in0 + (cur ^ 1) * TILE);
        fftdev::cp_async_commit();
        fftdev::cp_async_wait<1>();  // this thread's copies of unit t have landed
        __syncthreads();             // ... and everyone's
        int p, ct, plane;
        decode(t, p, ct, plane);
        if (MODE == 0) {
            // phi = delta_k exp(-k^2 R^2 / 2) / k^2, once per input element;
            // each output then only multiplies by k_x^p
            const int fy = plane <= h ? plane : plane - n;
            for (int e = threadIdx.x; e < TILE; e += NTHR) {
                const int j = e / W, cc = e % W;
                const int fj = j <= h ? j : j - n;
                const T m = phi_mult<T, FD>(0, fj, fy, ct * W + cc, gc, norm, sf, h, pot);
                const C v = in[e];
                in[e] = C{v.x * m, v.y * m};
            }
        }
        const int nout = MODE == 0 ? 3 : 3 - p;
        for (int o = 0; o < nout; ++o) {
            const int q = MODE == 0 ? 0 : 2 - p - o;  // y pass: q = 2-p .. 0
            const int pp = MODE == 0 ? o : p;
            // the x pass: k_x^o on this thread's own phi elements (no barrier
            // needed between the two loops);
            // the y pass: k_y^q (k_z^r is applied to the transformed tile)
            for (int e = threadIdx.x; e < TILE; e += NTHR) {
                const int j = e / W;
                const int fj = j <= h ? j : j - n;
                const T m = kfac<T, FD>(sf, h, fj, MODE == 0 ? o : q);
                const C v = in[e];
                work[e] = C{v.x * m, v.y * m};
            }
            __syncthreads();
            fftdev::block_fft_fixed<C, true, false, W, LEN, NTHR, W, 1, 1, false, CTw<T>::kMaxR>(work, tw);
            const int slot = MODE == 0 ? pp : slot_of(p, q);
            C *g = dst + (int64_t)slot * ccomp + (int64_t)plane * pstride + (int64_t)ct * W;
            // the y pass: k_z^r, r = 2 - p - q, k_z = the column (constant
            // along y, so it commutes with the transform)
            for (int e = threadIdx.x; e < TILE; e += NTHR) {
                const C v = work[e];
                const T mz = MODE == 0 ? (T)1 : kfac<T, FD>(sf, h, ct * W + e % W, 2 - p - q);
                g[(int64_t)(e / W) * jstride + (e % W)] = MODE == 0 ? v : C{v.x * mz, v.y * mz};
            }
            __syncthreads();  // work is refilled by the next output
        }
        cur ^= 1;
    }
    fftdev::cp_async_wait<0>();
}

// Trigonometric eigenvalues of a symmetric 3x3 matrix (O.K. Smith, CACM
// 4(4):168, 1961) in FP64 from the FP32 entries, each refined by one Newton
// step on the FP64 characteristic polynomial; returned in descending
// order.  FP64 throughout because acos is ill-conditioned next to r = +-1
// (two equal eigenvalues): an error e in r moves phi by ~sqrt(2e), which
// for FP32 (e ~ 6e-8) is ~3e-4 of the spread; in FP64 it is ~2e-8.  Only
// the eigenvalue planes take this path; labels alone use the sign count.
__device__ __forceinline__ void eig3(float a00f, float a11f, float a22f, float a01f, float a02f, float a12f,
                                     double lam[3])
{
    const double a00 = a00f, a11 = a11f, a22 = a22f, a01 = a01f, a02 = a02f, a12 = a12f;
    const double p1 = a01 * a01 + a02 * a02 + a12 * a12;
    const double q = (a00 + a11 + a22) * (1.0 / 3.0);
    const double b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
    const double p2 = b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * p1;
    double l[3];
    if (!(p2 > 0.0)) {
        l[0] = l[1] = l[2] = q;
    } else {
        const double pp = sqrt(p2 * (1.0 / 6.0));
        const double det = b00 * (b11 * b22 - a12 * a12) - a01 * (a01 * b22 - a12 * a02) +
                           a02 * (a01 * a12 - b11 * a02);
        double r = det / (2.0 * pp * pp * pp);
        r = fmin(1.0, fmax(-1.0, r));
        const double phi = acos(r) * (1.0 / 3.0);  // in [0, pi/3]
        l[0] = q + 2.0 * pp * cos(phi);
        l[2] = q + 2.0 * pp * cos(phi + 2.0943951023931954923);
        l[1] = 3.0 * q - l[0] - l[2];
    }
    // det(x I - A) = x^3 - c2 x^2 + c1 x - c0, coefficients in FP64 from the
    // FP32 entries (products of two floats are exact in double).
    const double c2 = a00 + a11 + a22;
    const double c1 = a00 * a11 + a00 * a22 + a11 * a22 - a01 * a01 - a02 * a02 - a12 * a12;
    const double c0 = a00 * (a11 * a22 - a12 * a12) - a01 * (a01 * a22 - a12 * a02) + a02 * (a01 * a12 - a11 * a02);
    const double sc = fmax(fabs(l[0]), fabs(l[2])) + 1e-30;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double x = l[k];
        const double f = ((x - c2) * x + c1) * x - c0;
        const double fp = (3.0 * x - 2.0 * c2) * x + c1;
        // a Newton step only where the root is simple enough to gain from it
        if (fabs(fp) > 1e-6 * sc * sc) {
            const double dx = f / fp;
            if (fabs(dx) < 1e-4 * sc) x -= dx;
        }
        lam[k] = x;
    }
    // keep descending order after refinement
    if (lam[0] < lam[1]) { const double t = lam[0]; lam[0] = lam[1]; lam[1] = t; }
    if (lam[1] < lam[2]) { const double t = lam[1]; lam[1] = lam[2]; lam[2] = t; }
    if (lam[0] < lam[1]) { const double t = lam[0]; lam[0] = lam[1]; lam[1] = t; }
}

// Coefficients of det(x I - A) = x^3 - c2 x^2 + c1 x - c0 in FP64 from the
// FP32 entries (products of two floats are exact in double).
__device__ __forceinline__ void char_poly(float a00, float a11, float a22, float a01, float a02, float a12,
                                          double &c2, double &c1, double &c0)
{
    const double A00 = a00, A11 = a11, A22 = a22, A01 = a01, A02 = a02, A12 = a12;
    c2 = A00 + A11 + A22;
    c1 = A00 * A11 + A00 * A22 + A11 * A22 - A01 * A01 - A02 * A02 - A12 * A12;
    c0 = A00 * (A11 * A22 - A12 * A12) - A01 * (A01 * A22 - A12 * A02) + A02 * (A01 * A12 - A11 * A02);
}

// Number of eigenvalues greater than t: the sign changes of the coefficients
// of p(x + t) = x^3 + (3t - c2) x^2 + (3t^2 - 2 c2 t + c1) x + p(t), zeros
// skipped.  Descartes' rule of signs is exact here because every root of
// the characteristic polynomial of a symmetric matrix is real.  Takes the
// three lower coefficients.
__device__ __forceinline__ int sign_changes(double a2, double a1, double a0)
{
    int changes = 0;
    bool neg = false;  // sign of the last nonzero coefficient (leading 1 > 0)
    if (a2 != 0.0) {
        changes += a2 < 0.0;
        neg = a2 < 0.0;
    }
    if (a1 != 0.0) {
        changes += (a1 < 0.0) != neg;
        neg = a1 < 0.0;
    }
    if (a0 != 0.0) changes += (a0 < 0.0) != neg;
    return changes;
}
// Taylor coefficients of p at t: p(t + s) = s^3 + a2 s^2 + a1 s + a0.
__device__ __forceinline__ void shifted_poly(double c2, double c1, double c0, double t, double &a2, double &a1,
                                             double &a0)
{
    a2 = 3.0 * t - c2;
    a1 = (3.0 * t - 2.0 * c2) * t + c1;
    a0 = ((t - c2) * t + c1) * t - c0;
}
__device__ __forceinline__ int count_above(double c2, double c1, double c0, double t)
{
    double a2, a1, a0;
    shifted_poly(c2, c1, c0, t, a2, a1, a0);
    return sign_changes(a2, a1, a0);
}

// Screens one cell in FP32 (labels only): the number of eigenvalues of
// the tensor above thf = float(lambda_th), from the signs of the
// coefficients of det(s I - B), B = T - thf I:
//   a2 = -tr B,  a1 = the sum of B's principal 2x2 minors,  a0 = -det B.
// Each coefficient is a sum of products of at most three FP32 numbers, one
// of them rounded once from T - thf, so |fl(a) - a| <= gamma_9 m (gamma_9 =
// 9u/(1-9u) = 5.4e-7, u = 2^-24), m the same sum over absolute values of
// the terms (Higham, Accuracy and Stability of Numerical Algorithms, 2nd
// ed., sec. 3.1); fused multiply-adds only remove roundings.  A sign is
// taken as certain when |fl(a)| > 2e-6 m, so the count is exact for the
// exact coefficients.  The cell is also certified free of ties: no root of
// p within bandp of thf (|p(thf + s) - p(thf)| <= bandp (|a1| + bandp (|a2|
// + bandp)) for |s| <= bandp), with bandp covering lambda_th +- band.
// Returns -1 when any test fails (near-zero coefficients, subnormal or
// non-finite terms, a root near the threshold): the caller then takes the
// FP64 path.  An eigenvalue between thf and lambda_th (|thf - lambda_th|
// <= 2^-24 |lambda_th|) lies inside any positive tie band.
__device__ __forceinline__ int count_above_fp32(const float t6[6], float thf, float bandp)
{
    // (xx, yy, zz, xy, xz, yz) from slots (2, 4, 0, 5, 1, 3)
    const float b0 = t6[2] - thf, b1 = t6[4] - thf, b2 = t6[0] - thf;
    const float d = t6[5], e = t6[1], f = t6[3];
    const float dd = d * d, ee = e * e, ff = f * f;
    const float p01 = b0 * b1, p02 = b0 * b2, p12 = b1 * b2;
    const float a2 = -(b0 + b1 + b2);
    const float m2 = fabsf(b0) + fabsf(b1) + fabsf(b2);
    const float a1 = (p01 + p02 + p12) - (dd + ee + ff);
    const float m1 = (fabsf(p01) + fabsf(p02) + fabsf(p12)) + (dd + ee + ff);
    const float t0 = p01 * b2, tdef = 2.0f * (d * e) * f;
    const float a0 = -(((t0 + tdef) - b0 * ff) - (b1 * ee + b2 * dd));
    const float m0 = ((fabsf(t0) + fabsf(tdef)) + fabsf(b0) * ff) + (fabsf(b1) * ee + fabsf(b2) * dd);
    const float r2 = 2e-6f * m2, r1 = 2e-6f * m1, r0 = 2e-6f * m0;
    // m >= 1e-20: every term's underflow error is far below r
    if (!(m0 >= 1e-20f && m1 >= 1e-20f && m2 >= 1e-20f && m0 < 1e30f && m1 < 1e30f && m2 < 1e30f)) return -1;
    if (!(fabsf(a2) > r2 && fabsf(a1) > r1 && fabsf(a0) > r0)) return -1;
    if (!(fabsf(a0) - r0 > bandp * ((fabsf(a1) + r1) + bandp * ((fabsf(a2) + r2) + bandp)))) return -1;
    // sign changes of (1, a2, a1, a0), all nonzero
    return (int)(a2 < 0.0f) + (int)((a1 < 0.0f) != (a2 < 0.0f)) + (int)((a0 < 0.0f) != (a1 < 0.0f));
}

// Label of one cell from its six field values (slots 0..5 of t6), written
// to labels[cell] (and lambdas when LAMBDAS, and the invariants when
// LAMBDAS and inv != nullptr); the label and tie counters of the calling
// thread are advanced.
template <bool LAMBDAS>
__device__ __forceinline__ void label_cell(const float t6[6], double lth, double band, float thf, float bandp,
                                           int64_t cell, int64_t ncell,
                                           uint8_t *__restrict__ labels, float *__restrict__ lambdas,
                                           float *__restrict__ inv, unsigned &lc0, unsigned &lc1, unsigned &lc2,
                                           unsigned &lc3, unsigned &lties)
{
    // (xx, yy, zz, xy, xz, yz) from slots (2, 4, 0, 5, 1, 3)
    int v = 0, tie = 0;
    if constexpr (LAMBDAS) {
        double lam[3];
        eig3(t6[2], t6[4], t6[0], t6[5], t6[1], t6[3], lam);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            v += lam[a] > lth;
            tie |= fabs(lam[a] - lth) <= band;
        }
        lambdas[cell] = (float)lam[0];
        lambdas[ncell + cell] = (float)lam[1];
        lambdas[2 * ncell + cell] = (float)lam[2];
        if (inv) {
            // invariant_field_I/II/III and tidal_anisotropy, Source/Miscelanious.cpp:1460-1492:
            // I = l1 + l2 + l3, II = l1 l2 + l2 l3 + l1 l3, III = l1 l2 l3 are the
            // characteristic polynomial's coefficients (FP64 from the tensor);
            // ((l3-l1)^2 + (l3-l2)^2 + (l2-l1)^2) / 2 = I^2 - 3 II = 3/2 tr(B^2), B
            // the traceless part of T: a sum of squares, free of cancellation
            double c2, c1, c0;
            char_poly(t6[2], t6[4], t6[0], t6[5], t6[1], t6[3], c2, c1, c0);
            const double q = c2 * (1.0 / 3.0);
            const double bxx = (double)t6[2] - q, byy = (double)t6[4] - q, bzz = (double)t6[0] - q;
            const double o2 = (double)t6[5] * t6[5] + (double)t6[1] * t6[1] + (double)t6[3] * t6[3];
            const double trb2 = bxx * bxx + byy * byy + bzz * bzz + 2.0 * o2;
            inv[cell] = (float)c2;
            inv[ncell + cell] = (float)c1;
            inv[2 * ncell + cell] = (float)c0;
            inv[3 * ncell + cell] = (float)(sqrt(1.5 * trb2) / (2.0 + c2));
        }
    } else {
        v = count_above_fp32(t6, thf, bandp);
        if (v < 0) {
            double c2, c1, c0, a2, a1, a0;
            char_poly(t6[2], t6[4], t6[0], t6[5], t6[1], t6[3], c2, c1, c0);
            shifted_poly(c2, c1, c0, lth, a2, a1, a0);
            v = sign_changes(a2, a1, a0);
            // |p(lth + s) - p(lth)| <= band (|a1| + band (|a2| + band)) for
            // |s| <= band: above that bound p has no root in the band, and the
            // counts at its two ends agree.  Only the other cells count again.
            if (!(fabs(a0) > band * (fabs(a1) + band * (fabs(a2) + band))))
                tie = count_above(c2, c1, c0, lth - band) != count_above(c2, c1, c0, lth + band);
        }
    }
    if (labels) labels[cell] = (uint8_t)(4 - v);
    lc0 += v == 3;  // label 1, knot
    lc1 += v == 2;
    lc2 += v == 1;
    lc3 += v == 0;  // label 4, void
    lties += tie;
}

// Adds the CTA's label and tie counters to counts[0..4] (cnt_s: five shared
// words, zeroed before the first barrier of the kernel).
__device__ __forceinline__ void flush_counts(unsigned lc0, unsigned lc1, unsigned lc2, unsigned lc3, unsigned lties,
                                             unsigned *cnt_s, unsigned long long *__restrict__ counts)
{
#pragma unroll
    for (int a = 0; a < 5; ++a) {
        unsigned v = a == 0 ? lc0 : a == 1 ? lc1 : a == 2 ? lc2 : a == 3 ? lc3 : lties;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&cnt_s[a], v);
    }
    __syncthreads();
    if (threadIdx.x < 5 && cnt_s[threadIdx.x]) atomicAdd(&counts[threadIdx.x], (unsigned long long)cnt_s[threadIdx.x]);
}

// c2r along z of the six components for `rpc` rows, then eigenvalues and
// labels.  Without LAMBDAS the eigenvalues are not formed: the label needs
// only the number of them above lambda_th, and the tie flag whether that
// number differs between lambda_th - band and lambda_th + band.  Component c of row r: main at src + c*ccomp + r*M, Nyquist at
// nyq + c*N*N + r.
template <typename T, int LEN, bool LAMBDAS>
__global__ void __launch_bounds__(256, 2)
tidal_z_kernel(const typename CTw<T>::t *__restrict__ src, const typename CTw<T>::t *__restrict__ nyq,
               int n, int64_t nrows, int rpc, int64_t ccomp, Radices rd,
               const typename CTw<T>::t *__restrict__ tw, double lth, double band,
               uint8_t *__restrict__ labels, float *__restrict__ lambdas, float *__restrict__ inv,
               unsigned long long *__restrict__ counts /* [5] */)
{
    using C = typename CTw<T>::t;
    constexpr bool PAD = LEN > 0;  // row tiles of the compile-time transforms are padded
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tile = reinterpret_cast<C *>(smem_raw);  // [6][rpc][M], element e at slot sidx<PAD>(e)
    __shared__ unsigned int cnt_s[5];
    // With a compile-time length the row length and rows per CTA are
    // constants (the host passes the same values), so the index divisions
    // below become multiplies.
    const int M = LEN > 0 ? LEN : n / 2;
    const int nz = LEN > 0 ? 2 * LEN : n;
    const int rpcv = LEN > 0 ? tweb_rpc<T>(LEN) : rpc;
    const int64_t row0 = (int64_t)blockIdx.x * rpcv;
    const int nr = (int)min((int64_t)rpcv, nrows - row0);
    const int64_t nn = (int64_t)n * n;
    if (threadIdx.x < 5) cnt_s[threadIdx.x] = 0;
    // Load + c2r untangling (see fft_rows_kernel, mode c2r).
    const int per = rpcv * M;
    for (int e = threadIdx.x; e < 6 * per; e += blockDim.x) {
        const int c = e / per, rem = e % per;
        const int r = rem / M, k = rem % M;
        if (r >= nr) continue;
        const C *sm = src + (int64_t)c * ccomp + (row0 + r) * M;
        C xk = sm[k];
        C xm = k == 0 ? nyq[(int64_t)c * nn + row0 + r] : sm[M - k];
        if (k == 0) {
            xk.y = 0;
            xm.y = 0;
        }
        const C a = C{xk.x + xm.x, xk.y - xm.y};
        const C b = C{xk.x - xm.x, xk.y + xm.y};
        C wv = __ldg(tw + k);
        wv.y = -wv.y;
        const C ib = fftdev::rot<C, true>(fftdev::cmul(wv, b));
        tile[fftdev::sidx<PAD>(e)] = fftdev::cadd(a, ib);
    }
    __syncthreads();
    if constexpr (LEN > 0) {
        constexpr int RPCZ = tweb_rpc<T>(LEN);
        fftdev::block_fft_fixed<C, true, true, 6 * RPCZ, LEN, fftdev::ct_threads(LEN, 6 * RPCZ, CTw<T>::kPPT), 1, LEN, 2,
                                true, CTw<T>::kMaxR>(tile, tw);
    } else {
        fftdev::block_fft<C, CTw<T>::kPPT, true, true, 0>(tile, M, 6 * rpc, 1, M, rd, tw, 2);
    }
    // Per cell: 6 components -> eigenvalues -> label.
    unsigned lc0 = 0, lc1 = 0, lc2 = 0, lc3 = 0, lties = 0;
    // FP32 label screen: the threshold in float, the tie band widened by
    // that rounding (and by its own)
    const float thf = (float)lth;
    const float bandp = (float)((band + fabs(lth - (double)thf)) * (1.0 + 1e-3));
    // real value z of row r of comp c: half z & 1 of complex element (c*rpc + r)*M + z/2
    const T *re = reinterpret_cast<const T *>(tile);
    const int64_t ncell = nn * n;
    for (int e = threadIdx.x; e < nr * nz; e += blockDim.x) {
        const int r = e / nz, z = e % nz;
        float t6[6];
#pragma unroll
        for (int c = 0; c < 6; ++c)
            t6[c] = (float)re[2 * fftdev::sidx<PAD>((c * rpcv + r) * M + (z >> 1)) + (z & 1)];
        label_cell<LAMBDAS>(t6, lth, band, thf, bandp, (row0 + r) * nz + z, ncell, labels, lambdas, inv, lc0, lc1, lc2, lc3,
                            lties);
    }
    flush_counts(lc0, lc1, lc2, lc3, lties, cnt_s, counts);
}

// The z pass, persistent and pipelined (compile-time length LEN = N/2):
// CTAs walk the groups of RPC rows blockIdx.x, blockIdx.x + gridDim.x, ...
// A group's raw rows are consumed by the untangling step, so the copy of
// the next group's rows into the same raw buffer (asynchronous 16-byte
// copies) starts right after it and runs while the group is transformed
// and labelled.  Label counts are kept per thread across groups and added
// once per CTA.
template <typename T, int LEN>
constexpr int zpipe_threads()
{
    return fftdev::ct_threads(LEN, 6 * tweb_rpc<T>(LEN), CTw<T>::kPPT);
}
template <typename T, int LEN>
constexpr size_t zpipe_smem()
{
    return ((size_t)6 * tweb_rpc<T>(LEN) * LEN + (size_t)fftdev::padded_len(6 * tweb_rpc<T>(LEN) * LEN, true)) *
           sizeof(typename CTw<T>::t);
}
// CTAs per SM.  Several CTAs per SM hide the latencies of the transform
// stages, barriers and FP64 label arithmetic; the register bound that comes
// with them is one the instantiation fits without spilling (ptxas -v):
// float LEN 256 and double LEN 128/256 in 80 registers (4 CTAs of 192
// threads), float LEN 512 in 96 (3 CTAs); the others need the 2-CTA bound.
// Capped by the shared memory of the CTAs.
template <typename T, int LEN>
constexpr int zpipe_min_blocks()
{
    const int want = sizeof(T) == 4 ? (LEN == 256 ? 4 : (LEN == 512 ? 3 : 2))
                                     : ((LEN == 128 || LEN == 256) ? 4 : 2);
    return (int)std::min<size_t>(want, std::max<size_t>(1, (220 * 1024) / (zpipe_smem<T, LEN>() + 1024)));
}
template <typename T, int LEN, bool LAMBDAS>
__global__ void __launch_bounds__(zpipe_threads<T, LEN>(), zpipe_min_blocks<T, LEN>())
tidal_z_pipe_kernel(const typename CTw<T>::t *__restrict__ src, const typename CTw<T>::t *__restrict__ nyq, int n,
                    int64_t nrows, int64_t ccomp, const typename CTw<T>::t *__restrict__ tw, double lth, double band,
                    uint8_t *__restrict__ labels, float *__restrict__ lambdas, float *__restrict__ inv,
                    unsigned long long *__restrict__ counts /* [5] */)
{
    using C = typename CTw<T>::t;
    constexpr int M = LEN;
    constexpr int RPC = tweb_rpc<T>(LEN);
    constexpr int PER = RPC * M;    // complex elements of one field in a group
    constexpr int RAW = 6 * PER;
    constexpr int NTHR = zpipe_threads<T, LEN>();
    constexpr int EPC = 16 / (int)sizeof(C);
    constexpr int CPRow = M / EPC;  // 16-byte chunks per row
    constexpr int HALF = M / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *const raw = reinterpret_cast<C *>(smem_raw);  // the raw rows of one group
    C *const tile = raw + RAW;                       // padded work tile [6][RPC][M]
    __shared__ unsigned cnt_s[5];
    if (threadIdx.x < 5) cnt_s[threadIdx.x] = 0;
    const int64_t nn = (int64_t)n * n, ncell = nn * n;
    const int64_t ngroups = (nrows + RPC - 1) / RPC;
    auto load = [&](int64_t gi, C *buf) {
        const int64_t row0 = gi * RPC;
        const int nr = (int)min((int64_t)RPC, nrows - row0);
        for (int e = threadIdx.x; e < 6 * RPC * CPRow; e += NTHR) {
            const int c = e / (RPC * CPRow), rem = e % (RPC * CPRow);
            const int r = rem / CPRow, k = rem % CPRow;
            if (r < nr)
                fftdev::cp_async16(buf + c * PER + r * M + k * EPC, src + (int64_t)c * ccomp + (row0 + r) * M + k * EPC);
        }
    };
    unsigned lc0 = 0, lc1 = 0, lc2 = 0, lc3 = 0, lties = 0;
    // FP32 label screen: the threshold in float, the tie band widened by
    // that rounding (and by its own)
    const float thf = (float)lth;
    const float bandp = (float)((band + fabs(lth - (double)thf)) * (1.0 + 1e-3));
    int64_t gi = blockIdx.x;
    if (gi < ngroups) load(gi, raw);
    fftdev::cp_async_commit();
    for (; gi < ngroups; gi += gridDim.x) {
        fftdev::cp_async_wait<0>();  // this thread's copies of group gi have landed
        __syncthreads();             // ... and everyone's
        const int64_t row0 = gi * RPC;
        const int nr = (int)min((int64_t)RPC, nrows - row0);
        // c2r untangling.  Elements k and M - k of a row use the same two
        // inputs X[k], X[M - k]: with a = X[k] + conj(X[M - k]),
        // u = conj(w^k) (X[k] - conj(X[M - k])) and conj(w^(M-k)) = -w^k,
        //   Z[k] = a + i u,   Z[M - k] = conj(a) + i conj(u).
        // Item 0 of a row makes Z[0] (with the Nyquist element X[M]) and
        // Z[M/2].
        for (int e = threadIdx.x; e < 6 * RPC * HALF; e += NTHR) {
            const int row = e / HALF, k = e % HALF;  // row = field * RPC + r
            const int c = row / RPC, r = row % RPC;
            if (r >= nr) continue;
            const C *rr = raw + row * M;
            C *zt = tile + fftdev::sidx<true>(row * M);  // rows start on a 16-element boundary
            const int kk = k == 0 ? HALF : k;
            const C xk = rr[kk], xm = rr[M - kk];
            const C a = C{xk.x + xm.x, xk.y - xm.y};
            const C b = C{xk.x - xm.x, xk.y + xm.y};
            C wv = __ldg(tw + kk);
            wv.y = -wv.y;
            const C u = fftdev::cmul(wv, b);
            zt[fftdev::sidx<true>(kk)] = C{a.x - u.y, a.y + u.x};
            if (k == 0) {
                const T x0 = rr[0].x, xn = nyq[(int64_t)c * nn + row0 + r].x;
                zt[0] = C{x0 + xn, x0 - xn};
            } else {
                zt[fftdev::sidx<true>(M - k)] = C{a.x + u.y, u.x - a.y};
            }
        }
        __syncthreads();  // raw is consumed: fetch the next group behind the transform
        const int64_t gn = gi + gridDim.x;
        if (gn < ngroups) load(gn, raw);
        fftdev::cp_async_commit();
        fftdev::block_fft_fixed<C, true, true, 6 * RPC, LEN, NTHR, 1, LEN, 2, true, CTw<T>::kMaxR>(tile, tw);
        // complex element m of a row holds the real values at z = 2m, 2m + 1
        for (int e = threadIdx.x; e < nr * M; e += NTHR) {
            const int r = e / M, m = e % M;
            float ta[6], tb[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const C v = tile[fftdev::sidx<true>((c * RPC + r) * M + m)];
                ta[c] = (float)v.x;
                tb[c] = (float)v.y;
            }
            const int64_t cell = (row0 + r) * 2 * M + 2 * m;
            label_cell<LAMBDAS>(ta, lth, band, thf, bandp, cell, ncell, labels, lambdas, inv, lc0, lc1, lc2, lc3, lties);
            label_cell<LAMBDAS>(tb, lth, band, thf, bandp, cell + 1, ncell, labels, lambdas, inv, lc0, lc1, lc2, lc3, lties);
        }
        __syncthreads();  // tile is refilled next
    }
    fftdev::cp_async_wait<0>();
    flush_counts(lc0, lc1, lc2, lc3, lties, cnt_s, counts);
}

// sf[i] = s(f) / k_f, f = i - N/2 (i = 0 .. N): the Fourier multiplier of
// the centred difference of gradfindif, Source/NumericalMethods.cpp:1123-1218,
//   D g(x) = (-g(x+2d) + 8 g(x+d) - 8 g(x-d) + g(x-2d)) / (12 d),
// D e^{ikx} = i s(k) e^{ikx},  s(k) = (8 sin kd - sin 2kd) / (6 d).
// With k = k_f f and k_f d = 2 pi / N:  s / k_f = N (8 sin t - sin 2t) / (12 pi),
// t = 2 pi f / N.  s(0) = s(+-N/2) = 0.
// Stored as {s, s^2} in the transform's precision.
template <typename T>
__global__ void fd_table_kernel(typename CTw<T>::t *__restrict__ sf, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    const double t = 2.0 * (double)(i - n / 2) / (double)n;  // sinpi(t) = sin(2 pi f / N)
    const double v = (double)n * (8.0 * sinpi(t) - sinpi(2.0 * t)) / (12.0 * M_PI);
    sf[i] = typename CTw<T>::t{(T)v, (T)(v * v)};
}

int threads_for(int points, int ppt, int cap)
{
    int t = (points + ppt - 1) / ppt;
    t = ((t + 31) / 32) * 32;
    return std::max(32, std::min(cap, t));
}

// Launches the pipelined T-web column kernel for the main planes when it
// applies (compile-time length, full 16-byte aligned tiles, three tiles
// within 200 KB of shared memory); returns false otherwise.
template <typename T, int MODE, int LEN, bool FD>
bool pipe_launch(cam_ctx *ctx, const char *name, const typename CTw<T>::t *src, typename CTw<T>::t *dst, int64_t n,
                 int64_t M, int64_t jstride, int64_t pstride, int64_t ccomp, const typename CTw<T>::t *tw,
                 double gcoef, const double *d_mean, int density, double scale, const typename CTw<T>::t *sf,
                 int pot)
{
    using C = typename CTw<T>::t;
    constexpr int W = LEN > 0 ? tpipe_cols<T, LEN>() : CTw<T>::kCols;
    if constexpr (LEN == 0 || 3 * LEN * W * sizeof(C) > 200 * 1024) {
        return false;
    } else {
        const size_t es = sizeof(C);
        if (M % W != 0 || (jstride * es) % 16 || (pstride * es) % 16 || (ccomp * es) % 16 ||
            ((uintptr_t)src % 16) || ((uintptr_t)dst % 16))
            return false;
        auto k = tidal_pipe_kernel<T, MODE, LEN, FD>;
        const size_t smem = 3 * (size_t)LEN * W * sizeof(C);
        smem_at_least(k, smem);
        int per_sm = 0;
        CAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, tpipe_threads<T, LEN>(), smem));
        const int nct = (int)(M / W);
        const int64_t nunits = (int64_t)nct * n * (MODE == 0 ? 1 : 3);
        const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(nunits, (int64_t)kNumSMs * std::max(per_sm, 1)));
        constexpr int nthr = tpipe_threads<T, LEN>();
        CAM_LAUNCH_NAMED(ctx, name, k, g, nthr, smem, src, dst, (int)n, nct, nunits, jstride, pstride, ccomp, tw, gcoef,
                         d_mean, density, scale, sf, pot);
        return true;
    }
}

template <typename T>
void tweb_impl(cam_ctx *ctx, FftPlan *plan, const Spectrum &dk, float L, const double *d_mean,
               int input_type, const cam_tweb_opts &o, uint8_t *d_labels, float *d_lambdas,
               cam_tweb_stats *stats, float *d_inv)
{
    using C = typename CTw<T>::t;
    constexpr int W = CTw<T>::kCols;
    const int64_t n = dk.n, M = n / 2, nn = n * n;
    const Radices rn = factor_radices(n), rm = factor_radices(M);
    CAM_REQUIRE(rn.n > 0 && rm.n > 0, CAM_E_UNSUPPORTED, "T-web size must be 2^a 3^b");
    const C *tw = static_cast<const C *>(plan_twiddles(plan));
    const int64_t ccomp = nn * M;
    C *cm = static_cast<C *>(scratch(ctx, "tw.main", (size_t)6 * ccomp * sizeof(C)));
    C *cn = static_cast<C *>(scratch(ctx, "tw.nyq", (size_t)6 * nn * sizeof(C)));
    auto *cnt = static_cast<unsigned long long *>(scratch(ctx, "tw.cnt", 8 * sizeof(unsigned long long)));
    CAM_CUDA_TRY(cudaMemsetAsync(cnt, 0, 8 * sizeof(unsigned long long), ctx->stream));

    const double kf = 2.0 * M_PI / (double)L;
    const double R = o.smoothing_R;
    const double gcoef = R > 0 ? 0.5 * kf * kf * R * R : 0.0;
    const int density = input_type == CAM_INPUT_DENSITY;
    const int pot = input_type == CAM_INPUT_POTENTIAL;
    // c2r divides by N^3; a potential input carries the k_f^2 of -k_a k_b
    const double scale = (pot ? kf * kf : 1.0) / ((double)n * (double)n * (double)n);
    const C *sf = nullptr;
    if (o.method == CAM_TWEB_FD) {
        auto *t = static_cast<C *>(scratch(ctx, "tw.sfac", (size_t)(n + 1) * sizeof(C)));
        CAM_LAUNCH_NAMED(ctx, "fd_table_kernel", fd_table_kernel<T>, (unsigned)((n + 1 + 127) / 128), 128, 0, t,
                         (int)n);
        sf = t;
    }
    auto passes = [&](auto fdc) {
    constexpr bool FD = decltype(fdc)::value;
    // 1. x: k_x^p phi + inverse FFT along x, p = 0, 1, 2 (slots 0..2).
    {
        const int nthr = threads_for((int)n * W, CTw<T>::kPPT, 1024);
        const size_t smem = (size_t)n * W * sizeof(C);
        dispatch_fft_len(n, [&](auto lc) {
        constexpr int LEN = decltype(lc)::value;
        auto k0 = tidal_x_kernel<T, false, LEN, FD>;
        auto k1 = tidal_x_kernel<T, true, LEN, FD>;
        smem_at_least(k1, smem);
        if (!pipe_launch<T, 0, LEN, FD>(ctx, "tweb_tidal_x", static_cast<const C *>(dk.main), cm, n, M, n * M,
                                        (int64_t)M, ccomp, tw, gcoef, d_mean, density, scale, sf, pot)) {
            smem_at_least(k0, smem);
            dim3 g0(3, (unsigned)((M + W - 1) / W), (unsigned)n);
            CAM_LAUNCH_NAMED(ctx, "tweb_tidal_x", k0, g0, nthr, smem, static_cast<const C *>(dk.main), cm, (int)n,
                             (int)M, n * M, (int64_t)M, ccomp, rn, tw, gcoef, d_mean, density, scale, sf, pot);
        }
        dim3 g1(3, (unsigned)((n + W - 1) / W), 1);
        CAM_LAUNCH_NAMED(ctx, "tweb_tidal_x_nyq", k1, g1, nthr, smem, static_cast<const C *>(dk.nyq), cn, (int)n, (int)n, n,
                   (int64_t)0, nn, rn, tw, gcoef, d_mean, density, scale, sf, pot);
        });
    }
    // 2. y: k_y^q and the inverse FFT along y: three fields in, six out.
    {
        const int nthr = threads_for((int)n * W, CTw<T>::kPPT, 1024);
        const size_t smem = (size_t)n * W * sizeof(C);
        dispatch_fft_len(n, [&](auto lc) {
        constexpr int LEN = decltype(lc)::value;
        auto ky = tidal_y_kernel<T, LEN, FD>;
        smem_at_least(ky, smem);
        // main: planes i, FFT index j (stride M), columns k (stride 1)
        if (!pipe_launch<T, 1, LEN, FD>(ctx, "tweb_tidal_y", cm, cm, n, M, (int64_t)M, n * M, ccomp, tw, 0.0, nullptr,
                                        0, 1.0, sf, 0)) {
            dim3 g0(3, (unsigned)((M + W - 1) / W), (unsigned)n);
            CAM_LAUNCH_NAMED(ctx, "tweb_tidal_y", ky, g0, nthr, smem, cm, (int)n, (int)M, (int64_t)M, (int64_t)1, n * M,
                             ccomp, rn, tw, -1, sf);
        }
        // Nyquist plane: columns i (stride N), FFT index j (stride 1)
        dim3 g1(3, (unsigned)((n + W - 1) / W), 1);
        CAM_LAUNCH_NAMED(ctx, "tweb_tidal_y_nyq", ky, g1, nthr, smem, cn, (int)n, (int)n, (int64_t)1, n, (int64_t)0,
                         nn, rn, tw, (int)M, sf);
        });
    }
    };
    if (sf) passes(std::true_type{});
    else passes(std::false_type{});
    // 3. z: c2r + eigenvalues + labels.
    {
        // Small tiles (<= 4096 complex, 256 threads) so that several CTAs
        // share an SM: one CTA's loads overlap another's transform and
        // eigen-solve.
        const int rpc = tweb_rpc<T>((int)M);
        const int nthr = threads_for(6 * rpc * (int)M, CTw<T>::kPPT, 256);
        CAM_REQUIRE(6 * rpc * M <= (int64_t)nthr * CTw<T>::kPPT, CAM_E_UNSUPPORTED, "T-web row tile too large");
        dispatch_fft_len(M, [&](auto lc) {
        constexpr int LEN = decltype(lc)::value;
        const size_t smem = (size_t)fftdev::padded_len(6 * rpc * M, LEN > 0) * sizeof(C);
        if constexpr (LEN > 0 && LEN <= 512 && (LEN & (LEN - 1)) == 0 && zpipe_smem<T, LEN>() <= 200 * 1024) {
            // persistent pipelined z pass, for the power-of-two row lengths
            // (whose transforms fit the register bound without spilling)
            auto kp = d_lambdas ? tidal_z_pipe_kernel<T, LEN, true> : tidal_z_pipe_kernel<T, LEN, false>;
            constexpr size_t psmem = zpipe_smem<T, LEN>();
            constexpr int pthr = zpipe_threads<T, LEN>();
            smem_at_least(kp, psmem);
            int per_sm = 0;
            CAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, pthr, psmem));
            const int64_t ngroups = (nn + tweb_rpc<T>(LEN) - 1) / tweb_rpc<T>(LEN);
            const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ngroups, (int64_t)kNumSMs * std::max(per_sm, 1)));
            CAM_LAUNCH_NAMED(ctx, "tweb_tidal_z_eigen", kp, g, pthr, psmem, cm, cn, (int)n, nn, ccomp, tw, o.lambda_th,
                             o.tie_band, d_labels, d_lambdas, d_inv, cnt);
            return;
        }
        auto kz = d_lambdas ? tidal_z_kernel<T, LEN, true> : tidal_z_kernel<T, LEN, false>;
        smem_at_least(kz, smem);
        const unsigned grid = (unsigned)((nn + rpc - 1) / rpc);
        CAM_LAUNCH_NAMED(ctx, "tweb_tidal_z_eigen", kz, grid, nthr, smem, cm, cn, (int)n, nn, rpc, ccomp, rm, tw, o.lambda_th,
                   o.tie_band, d_labels, d_lambdas, d_inv, cnt);
        });
    }
    if (stats) {
        unsigned long long h[5];
        double mean = 0.0;
        CAM_CUDA_TRY(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        if (d_mean) CAM_CUDA_TRY(cudaMemcpyAsync(&mean, d_mean, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CAM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        for (int a = 0; a < 4; ++a) stats->counts[a] = (int64_t)h[a];
        stats->ties = (int64_t)h[4];
        stats->mean = mean;
    }
}

}  // namespace

void tweb_device(cam_ctx *ctx, FftPlan *plan, const Spectrum &dk, float L, const double *d_mean,
                 int input_type, const cam_tweb_opts &o, uint8_t *d_labels, float *d_lambdas,
                 cam_tweb_stats *stats, float *d_inv)
{
    CAM_REQUIRE(std::isfinite(o.lambda_th) && o.tie_band >= 0.0, CAM_E_INVAL, "invalid T-web threshold");
    CAM_REQUIRE(o.smoothing_R >= 0.f && std::isfinite(o.smoothing_R), CAM_E_INVAL, "invalid smoothing radius");
    CAM_REQUIRE(o.method == CAM_TWEB_FFT || o.method == CAM_TWEB_FD, CAM_E_INVAL, "unknown T-web method");
    CAM_REQUIRE(input_type == CAM_INPUT_DENSITY || input_type == CAM_INPUT_DELTA ||
                    (input_type == CAM_INPUT_POTENTIAL && o.method == CAM_TWEB_FD),
                CAM_E_INVAL, "T-web input must be a density or delta mesh (or a potential, finite differences only)");
    CAM_REQUIRE(input_type != CAM_INPUT_DENSITY || d_mean, CAM_E_INVAL, "density input needs the mean");
    // the invariants are formed in the eigenvalue path, which needs lambda planes
    if (d_inv && !d_lambdas) {
        const int64_t ncell = dk.n * dk.n * dk.n;
        d_lambdas = static_cast<float *>(scratch(ctx, "tw.lam", (size_t)3 * ncell * sizeof(float)));
    }
    if (dk.precision == CAM_F32)
        tweb_impl<float>(ctx, plan, dk, L, d_mean, input_type, o, d_labels, d_lambdas, stats, d_inv);
    else
        tweb_impl<double>(ctx, plan, dk, L, d_mean, input_type, o, d_labels, d_lambdas, stats, d_inv);
}

}  // namespace cam

/*
 * CPU oracle for the CosmicAtlas/BAM per-iteration mesh hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file; only the tests, the smoke check and the CPU-baseline leg of
 * the benchmark do, as the checker or as the timed CPU reference.
 *
 * Parity status.  Mass assignment (getDensity_NGP/CIC/TSC) is PINNED: the
 * reference's own functions are compiled from Source/massFunctions.cpp by
 * oracle/Makefile (target ref, stand-in headers in oracle/refstub/), and
 * tests/test_golden_reference.py checks that orc_assign_ref reproduces their
 * meshes bit for bit, that the keys of orc_keys give their NGP counts, and
 * that orc_assign_f64 agrees within 1e-5 (tests/golden/getdensity_ref.npz,
 * written by tests/golden/make_golden.py).  The P(k) estimator and the T-web
 * are UNPINNED: their reference code needs FFTW3, GSL and the FftwFunctions
 * and Cwclass class headers, none of which can be built here, and the
 * reference ships no tests, golden vectors or fixtures; those functions
 * restate the reference source text, each naming the lines it follows.
 *
 * Two families of functions live here:
 *   orc_*_f64  : the FP64 oracle with the pinned semantics the GPU path must
 *                reproduce (integer keys bit-exact, meshes and spectra within
 *                the stated tolerance);
 *   orc_*_ref  : the reference loops as written (FP32, serial scatter, OpenMP
 *                atomics in the power spectrum), used as the timed CPU baseline
 *                and to document where the pinned semantics differ.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).  The FP32 key
 * arithmetic relies on IEEE single precision without contraction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { ORC_NGP = 0, ORC_CIC = 1, ORC_TSC = 2 };

/* ------------------------------------------------------------------------ */
/* Home cell of one particle, reference FP32 semantics.                     */
/* ------------------------------------------------------------------------ */

/* Cell index along one axis, as the reference computes it:
 *   i = floor((x - min)/d) in float, then i = fmod(i, N)
 * Source/massFunctions.cpp:62-68 (NGP), :731-737 (CIC), :1083-1089 (TSC). */
static int64_t ref_cell_index(float x, float mn, float d, int64_t n)
{
    volatile float t = x - mn;
    volatile float u = t / d;
    int64_t i = (int64_t)floorf(u);
    if (i < 0) return -1; /* cannot happen for accepted particles */
    return (int64_t)fmodf((float)i, (float)n);
}

/* Acceptance test and home cell for one particle.  Returns 1 if the particle
 * is assigned, 0 if it is counted as lost.  idx[a] is the home cell in [0,N).
 * The position used for the index is the one the reference uses:
 *   NGP: x itself, accepted on [min, min+L)        massFunctions.cpp:57
 *   CIC: x - d/2 wrapped once by +-L, accepted on [min, min+L)
 *                                                  massFunctions.cpp:700-727
 *        (the reference wraps every axis with L1; the per-axis L is used here,
 *         identical for the cubic boxes the hot path runs on)
 *   TSC: x itself, accepted on [min, min+L] (closed) massFunctions.cpp:1076 */
static int ref_home(int scheme, const float p[3], const int64_t n[3],
                    const float L[3], const float d[3], const float mn[3],
                    int64_t idx[3])
{
    float q[3];
    for (int a = 0; a < 3; ++a) {
        volatile float v = p[a];
        if (scheme == ORC_CIC) {
            volatile float half = 0.5f * d[a];
            v = v - half;
            if (v < 0.0f) v = v + L[a];
            if (v >= L[a]) v = v - L[a];
        }
        q[a] = v;
    }
    for (int a = 0; a < 3; ++a) {
        volatile float hi = mn[a] + L[a];
        int ok = (scheme == ORC_TSC) ? (q[a] >= mn[a] && q[a] <= hi)
                                     : (q[a] >= mn[a] && q[a] < hi);
        if (!ok) return 0;
    }
    for (int a = 0; a < 3; ++a) idx[a] = ref_cell_index(q[a], mn[a], d[a], n[a]);
    return 1;
}

/* Exact fractional offset of the particle from its home node, in cells,
 * reduced to the periodic image nearest the home cell:
 *   t = (x - min)/d - s - c  (mod N),   s = 1/2 for CIC and TSC.
 * CIC: the reference's dx = (xpos-min)/d - i with xpos = x - d/2
 *      (massFunctions.cpp:743-745); TSC: dx = (x-min)/d - (i+1/2)
 *      (massFunctions.cpp:1098-1104).  Here t is computed from the unrounded
 *      position and uses the pre-wrap cell, which removes the reference's
 *      garbage weights when (x-min)/d rounds to N (i wraps to 0 while dx stays
 *      near N). */
static double exact_offset(float x, float mn, float d, int64_t c, int64_t n, double s)
{
    double u = ((double)x - (double)mn) / (double)d - s;
    double t = u - (double)c;
    double hn = 0.5 * (double)n;
    if (t > hn) t -= (double)n;
    if (t < -hn) t += (double)n;
    return t;
}

static inline int64_t wrap(int64_t i, int64_t n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

/* ------------------------------------------------------------------------ */
/* Public oracle entry points                                               */
/* ------------------------------------------------------------------------ */

/* Sort keys: key = k + N3*(j + N2*i) of the home cell (row-major, z fastest,
 * massFunctions.cpp:74), or N1*N2*N3 for a lost particle.  Bit-exact target. */
void orc_keys(int scheme, int64_t np, const float *x, const float *y, const float *z,
              const int64_t n[3], const float L[3], const float d[3], const float mn[3],
              int64_t *keys)
{
    const int64_t ncell = n[0] * n[1] * n[2];
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < np; ++p) {
        float pos[3] = {x[p], y[p], z[p]};
        int64_t idx[3];
        if (!ref_home(scheme, pos, n, L, d, mn, idx)) { keys[p] = ncell; continue; }
        keys[p] = idx[2] + n[2] * (idx[1] + n[1] * idx[0]);
    }
}

/* Per-axis stencil weights in FP64 for offset t.  Returns the stencil width
 * and the first stencil cell relative to the home cell.
 *   NGP: {1} at 0                                  massFunctions.cpp:71-74
 *   CIC: {1-t, t} at 0,+1                          massFunctions.cpp:747-769
 *   TSC: {(1/2-t)^2/2, 3/4-t^2, (1/2+t)^2/2} at -1,0,+1
 *                                                  massFunctions.cpp:1106-1162 */
static int stencil_f64(int scheme, double t, double wt[3], int *first)
{
    switch (scheme) {
    case ORC_NGP: wt[0] = 1.0; *first = 0; return 1;
    case ORC_CIC: wt[0] = 1.0 - t; wt[1] = t; *first = 0; return 2;
    default:
        wt[0] = 0.5 * (0.5 - t) * (0.5 - t);
        wt[1] = 0.75 - t * t;
        wt[2] = 0.5 * (0.5 + t) * (0.5 + t);
        *first = -1;
        return 3;
    }
}

/* FP64 mass assignment with the pinned semantics.  mesh (N1*N2*N3 doubles)
 * is zeroed here, as the reference zeroes delta (massFunctions.cpp:47-50).
 * Serial loop in particle order.  Returns the number of lost particles. */
int64_t orc_assign_f64(int scheme, int64_t np, const float *x, const float *y,
                       const float *z, const float *w, const int64_t n[3],
                       const float L[3], const float d[3], const float mn[3],
                       double *mesh)
{
    const int64_t ncell = n[0] * n[1] * n[2];
    memset(mesh, 0, sizeof(double) * (size_t)ncell);
    int64_t lost = 0;
    for (int64_t p = 0; p < np; ++p) {
        float pos[3] = {x[p], y[p], z[p]};
        int64_t c[3];
        if (!ref_home(scheme, pos, n, L, d, mn, c)) { ++lost; continue; }
        double wa[3][3];
        int first[3], width[3];
        for (int a = 0; a < 3; ++a) {
            double t = (scheme == ORC_NGP) ? 0.0 : exact_offset(pos[a], mn[a], d[a], c[a], n[a], 0.5);
            width[a] = stencil_f64(scheme, t, wa[a], &first[a]);
        }
        const double m = w ? (double)w[p] : 1.0;
        for (int ia = 0; ia < width[0]; ++ia) {
            int64_t ii = wrap(c[0] + first[0] + ia, n[0]);
            for (int ja = 0; ja < width[1]; ++ja) {
                int64_t jj = wrap(c[1] + first[1] + ja, n[1]);
                double wij = m * wa[0][ia] * wa[1][ja];
                for (int ka = 0; ka < width[2]; ++ka) {
                    int64_t kk = wrap(c[2] + first[2] + ka, n[2]);
                    mesh[kk + n[2] * (jj + n[1] * ii)] += wij * wa[2][ka];
                }
            }
        }
    }
    return lost;
}

/* orc_assign_f64 on all threads, for the full-size configurations (16.8 M
 * and 453 M particles): particle chunks per thread, every cell update an
 * atomic FP64 add.  The set of contributions is the serial function's; only
 * the order of the FP64 additions varies (~1e-16 relative), far inside the
 * 1e-5 tolerance the oracle checks against. */
int64_t orc_assign_f64_mt(int scheme, int64_t np, const float *x, const float *y,
                          const float *z, const float *w, const int64_t n[3],
                          const float L[3], const float d[3], const float mn[3],
                          double *mesh)
{
    const int64_t ncell = n[0] * n[1] * n[2];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ncell; ++i) mesh[i] = 0.0;
    int64_t lost = 0;
#pragma omp parallel for schedule(static, 65536) reduction(+ : lost)
    for (int64_t p = 0; p < np; ++p) {
        float pos[3] = {x[p], y[p], z[p]};
        int64_t c[3];
        if (!ref_home(scheme, pos, n, L, d, mn, c)) { ++lost; continue; }
        double wa[3][3];
        int first[3], width[3];
        for (int a = 0; a < 3; ++a) {
            double t = (scheme == ORC_NGP) ? 0.0 : exact_offset(pos[a], mn[a], d[a], c[a], n[a], 0.5);
            width[a] = stencil_f64(scheme, t, wa[a], &first[a]);
        }
        const double m = w ? (double)w[p] : 1.0;
        for (int ia = 0; ia < width[0]; ++ia) {
            int64_t ii = wrap(c[0] + first[0] + ia, n[0]);
            for (int ja = 0; ja < width[1]; ++ja) {
                int64_t jj = wrap(c[1] + first[1] + ja, n[1]);
                double wij = m * wa[0][ia] * wa[1][ja];
                for (int ka = 0; ka < width[2]; ++ka) {
                    int64_t kk = wrap(c[2] + first[2] + ka, n[2]);
#pragma omp atomic update
                    mesh[kk + n[2] * (jj + n[1] * ii)] += wij * wa[2][ka];
                }
            }
        }
    }
    return lost;
}

/* ------------------------------------------------------------------------ */
/* Reference loops as written (FP32) -- the timed CPU baseline.             */
/* ------------------------------------------------------------------------ */

/* One particle of getDensity_NGP / _CIC / _TSC (Gen A) as written, into the
 * float mesh delta: Source/massFunctions.cpp:57-76 (NGP), :700-770 (CIC),
 * :1076-1160 (TSC), including the post-wrap cell used for dx and the float
 * accumulation.  Returns 0 if the particle is assigned, 1 if it is lost. */
static inline int ref_one(int scheme, float px, float py, float pz, float mass, int64_t N1, int64_t N2,
                          int64_t N3, float L1, float L2, float L3, float d1, float d2, float d3, float min1,
                          float min2, float min3, float *delta)
{
#define DELTA(i, j, k) delta[(k) + N3 * ((j) + N2 * (i))]
    if (scheme == ORC_NGP) {
        if ((px >= min1 && px < min1 + L1) && (py >= min2 && py < min2 + L2) && (pz >= min3 && pz < min3 + L3)) {
            uint64_t i = (uint64_t)floorf((px - min1) / d1);
            uint64_t j = (uint64_t)floorf((py - min2) / d2);
            uint64_t k = (uint64_t)floorf((pz - min3) / d3);
            i = (uint64_t)fmodf((float)i, (float)N1);
            j = (uint64_t)fmodf((float)j, (float)N2);
            k = (uint64_t)fmodf((float)k, (float)N3);
            DELTA(i, j, k) += mass;
            return 0;
        }
        return 1;
    }
    if (scheme == ORC_CIC) {
        float xpos = (float)((double)px - 0.5 * (double)d1);
        float ypos = (float)((double)py - 0.5 * (double)d2);
        float zpos = (float)((double)pz - 0.5 * (double)d3);
        if (xpos < 0.f) xpos += L1;
        if (xpos >= L1) xpos -= L1;
        if (ypos < 0.f) ypos += L1;
        if (ypos >= L1) ypos -= L1;
        if (zpos < 0.f) zpos += L1;
        if (zpos >= L1) zpos -= L1;
        if ((xpos >= min1 && xpos < min1 + L1) && (ypos >= min2 && ypos < min2 + L2) &&
            (zpos >= min3 && zpos < min3 + L3)) {
            uint64_t i = (uint64_t)floorf((xpos - min1) / d1);
            uint64_t j = (uint64_t)floorf((ypos - min2) / d2);
            uint64_t k = (uint64_t)floorf((zpos - min3) / d3);
            i = (uint64_t)fmodf((float)i, (float)N1);
            j = (uint64_t)fmodf((float)j, (float)N2);
            k = (uint64_t)fmodf((float)k, (float)N3);
            uint64_t ii = (uint64_t)fmodf((float)(i + 1), (float)N1);
            uint64_t jj = (uint64_t)fmodf((float)(j + 1), (float)N2);
            uint64_t kk = (uint64_t)fmodf((float)(k + 1), (float)N3);
            float dx = (xpos - min1) / d1 - (float)i;
            float dy = (ypos - min2) / d2 - (float)j;
            float dz = (zpos - min3) / d3 - (float)k;
            float tx = 1.0f - dx, ty = 1.0f - dy, tz = 1.0f - dz;
            DELTA(i, j, k) += mass * tx * ty * tz;
            DELTA(ii, j, k) += mass * dx * ty * tz;
            DELTA(i, jj, k) += mass * tx * dy * tz;
            DELTA(i, j, kk) += mass * tx * ty * dz;
            DELTA(ii, jj, k) += mass * dx * dy * tz;
            DELTA(ii, j, kk) += mass * dx * ty * dz;
            DELTA(i, jj, kk) += mass * tx * dy * dz;
            DELTA(ii, jj, kk) += mass * dx * dy * dz;
            return 0;
        }
        return 1;
    }
    if ((px >= min1 && px <= min1 + L1) && (py >= min2 && py <= min2 + L2) && (pz >= min3 && pz <= min3 + L3)) {
        uint64_t i = (uint64_t)floorf((px - min1) / d1);
        uint64_t j = (uint64_t)floorf((py - min2) / d2);
        uint64_t k = (uint64_t)floorf((pz - min3) / d3);
        i = (uint64_t)fmodf((float)i, (float)N1);
        j = (uint64_t)fmodf((float)j, (float)N2);
        k = (uint64_t)fmodf((float)k, (float)N3);
        uint64_t ii = (uint64_t)fmodf((float)(i + 1), (float)N1);
        uint64_t jj = (uint64_t)fmodf((float)(j + 1), (float)N2);
        uint64_t kk = (uint64_t)fmodf((float)(k + 1), (float)N3);
        uint64_t iii = (uint64_t)fmodf((float)(i - 1 + N1), (float)N1);
        uint64_t jjj = (uint64_t)fmodf((float)(j - 1 + N2), (float)N2);
        uint64_t kkk = (uint64_t)fmodf((float)(k - 1 + N3), (float)N3);
        float xc = (float)i + 0.5f, yc = (float)j + 0.5f, zc = (float)k + 0.5f;
        float dx = (px - min1) / d1 - xc;
        float dy = (py - min2) / d2 - yc;
        float dz = (pz - min3) / d3 - zc;
        float hx0 = (float)(0.75 - dx * dx), hy0 = (float)(0.75 - dy * dy), hz0 = (float)(0.75 - dz * dz);
        float hxp1 = (float)(0.5 * (0.5 + dx) * (0.5 + dx));
        float hyp1 = (float)(0.5 * (0.5 + dy) * (0.5 + dy));
        float hzp1 = (float)(0.5 * (0.5 + dz) * (0.5 + dz));
        float hxm1 = (float)(0.5 * (0.5 - dx) * (0.5 - dx));
        float hym1 = (float)(0.5 * (0.5 - dy) * (0.5 - dy));
        float hzm1 = (float)(0.5 * (0.5 - dz) * (0.5 - dz));
        const uint64_t I[3] = {iii, i, ii}, J[3] = {jjj, j, jj}, K[3] = {kkk, k, kk};
        const float hx[3] = {hxm1, hx0, hxp1}, hy[3] = {hym1, hy0, hyp1}, hz[3] = {hzm1, hz0, hzp1};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) DELTA(I[a], J[b], K[c]) += mass * hx[a] * hy[b] * hz[c];
        return 0;
    }
    return 1;
#undef DELTA
}

/* getDensity_NGP / _CIC / _TSC, Gen A, serial particle loop, float mesh.
 * Source/massFunctions.cpp:35-98, :678-790, :1050-1165. */
int64_t orc_assign_ref(int scheme, int64_t np, const float *xp, const float *yp,
                       const float *zp, const float *w, int64_t N1, int64_t N2,
                       int64_t N3, float L1, float L2, float L3, float d1, float d2,
                       float d3, float min1, float min2, float min3, float *delta)
{
    const int64_t ncell = N1 * N2 * N3;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < ncell; ++i) delta[i] = 0.0f;
    int64_t lost = 0;
    for (int64_t n = 0; n < np; ++n)
        lost += ref_one(scheme, xp[n], yp[n], zp[n], w ? w[n] : 1.0f, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1,
                        min2, min3, delta);
    return lost;
}

/* The Gen-B OpenMP form of getDensity_* (Source/Miscelanious.cpp:454-560 CIC,
 * :693 TSC and the NGP twin): every thread accumulates into its own private
 * float grid, and the grids are added into delta one thread at a time under
 * `omp critical`.  As written there, an inner `omp parallel` region wraps the
 * particle loop without a work-sharing `for`, so every thread processes every
 * particle and the mesh comes out NTHREADS times too large; here the loop is
 * shared (`omp for`), which is the fix.  The per-particle arithmetic is Gen
 * A's (ref_one).  nthreads <= 0: all available threads. */
int64_t orc_assign_omp(int scheme, int64_t np, const float *xp, const float *yp, const float *zp,
                       const float *w, int64_t N1, int64_t N2, int64_t N3, float L1, float L2, float L3,
                       float d1, float d2, float d3, float min1, float min2, float min3, float *delta,
                       int nthreads)
{
    const int64_t ncell = N1 * N2 * N3;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t i = 0; i < ncell; ++i) delta[i] = 0.0f;
    int64_t lost = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : lost)
    {
        float *priv = (float *)calloc((size_t)ncell, sizeof(float));
#pragma omp for schedule(static)
        for (int64_t n = 0; n < np; ++n)
            lost += ref_one(scheme, xp[n], yp[n], zp[n], w ? w[n] : 1.0f, N1, N2, N3, L1, L2, L3, d1, d2, d3,
                            min1, min2, min3, priv);
#pragma omp critical
        {
            for (int64_t i = 0; i < ncell; ++i) delta[i] += priv[i];
        }
        free(priv);
    }
    return lost;
}

/* ------------------------------------------------------------------------ */
/* Power spectrum                                                           */
/* ------------------------------------------------------------------------ */

/* Aliased shot-noise factor per axis, Source/Miscelanious.cpp:2532-2549. */
static double sq_factor(int p, double s)
{
    switch (p) {
    case 0: return 1.0;
    case 1: return 1.0 - (2.0 / 3.0) * s * s;
    case 2: return 1.0 - s * s + (2.0 / 15.0) * s * s * s * s;
    default: return 1.0 - (4.0 / 3.0) * s * s + (2.0 / 5.0) * s * s * s * s - (4.0 / 315.0) * s * s * s * s * s * s;
    }
}

static double sinc_pi(int64_t a, int64_t n)
{
    if (a == 0) return 1.0;
    double x = M_PI * (double)a / (double)n;
    return sin(x) / x;
}

/* Whether half-spectrum element (i,j,c) is visited by the reference's octant
 * loop, Source/FftwFunctions.cpp:1731-1869: loop a<N/2, b<N/2, c<=N/2 over
 * (a,b,c), (a,N-b,c) if b,c>0, (N-a,b,c) if a>0 and (b>0 or c>0),
 * (N-a,N-b,c) if a,b,c>0.  Planes i=N/2 and j=N/2 are never visited. */
static int pk_visited(int64_t i, int64_t j, int64_t c, int64_t n)
{
    const int64_t h = n / 2;
    if (i == h || j == h) return 0;
    if (c > 0) return 1;
    if (i == 0 && j == 0) return 0;
    if (j > h) return 0;          /* (a, N-b, 0) is never visited */
    if (i > h && j == 0) return 0; /* (N-a, 0, 0) is never visited */
    return 1;
}

/* Bin of a mode with q = a^2+b^2+c^2 (|k| = sqrt(q) fundamental modes):
 * the b with E2[b] <= q < E2[b+1], E2[b] = (kmin_u + b*dk_u)^2 in FP64, or -1
 * when q < E2[0] or q >= E2[nbins].  This is floor((|k|-kmin)/DeltaK) of
 * FftwFunctions.cpp:1770-1775 evaluated on squared edges, so that a mode lying
 * exactly on an edge goes to the upper bin (the reference's float arithmetic
 * sends such modes either way). */
int64_t orc_bin(double q, double kmin_u, double dk_u, int nbins)
{
    double t = (sqrt(q) - kmin_u) / dk_u;
    if (!(t > -2.0)) return -1;
    int64_t b = (int64_t)floor(t);
    if (b > nbins) b = nbins;
    for (int it = 0; it < 4; ++it) {
        double e = kmin_u + (double)(b + 1) * dk_u;
        if (b + 1 <= nbins && e * e <= q) ++b; else break;
    }
    for (int it = 0; it < 4; ++it) {
        double e = kmin_u + (double)b * dk_u;
        if (b >= 0 && e * e > q) --b; else break;
    }
    if (b < 0 || b >= nbins) return -1;
    return b;
}

/* FP64 binned power spectrum of a half spectrum in FFTW r2c layout
 * [i][j][c<=N/2], interleaved complex128.  Pinned semantics:
 *   bin  = orc_bin(a^2+b^2+c^2), a,b the absolute signed frequencies;
 *   W    = prod sinc(pi a/N)^(p+1)               (Miscelanious.cpp:2557-2562)
 *   C    = prod Sq(p, sin(pi a/N))                (Miscelanious.cpp:2550-2554)
 *   Pk   = (|F|^2 - SN*C*normal) / W^2            (FftwFunctions.cpp:1797-1800)
 *   P[b] = sum Pk / (modes * normal)              (FftwFunctions.cpp:1873-1874)
 * with |F|^2 = Re^2 + Im^2 in every octant (the reference's fourth octant uses
 * Im*Re + Im*Re, FftwFunctions.cpp:1853; corrected here).
 * Outputs per bin: pk, modes, sum_raw = sum |F|^2/W^2, sum_sn = sum C/W^2. */
void orc_power_f64(int64_t n, const double *spec, int p, int mas_corr, int sn_corr,
                   double shot_noise, double normal, double kmin_u, double dk_u,
                   int nbins, double *pk, int64_t *modes, double *sum_raw, double *sum_sn)
{
    const int64_t nz = n / 2 + 1;
    double *sr = calloc((size_t)nbins, sizeof(double));
    double *ss = calloc((size_t)nbins, sizeof(double));
    int64_t *md = calloc((size_t)nbins, sizeof(int64_t));
    double *sx = malloc(sizeof(double) * (size_t)n), *cx = malloc(sizeof(double) * (size_t)n);
    for (int64_t a = 0; a < n; ++a) {
        int64_t aa = a <= n / 2 ? a : n - a;
        sx[a] = sinc_pi(aa, n);
        cx[a] = sq_factor(p, sin(M_PI * (double)aa / (double)n));
    }
    for (int64_t i = 0; i < n; ++i) {
        int64_t a = i <= n / 2 ? i : n - i;
        for (int64_t j = 0; j < n; ++j) {
            int64_t b = j <= n / 2 ? j : n - j;
            for (int64_t c = 0; c < nz; ++c) {
                if (!pk_visited(i, j, c, n)) continue;
                double q = (double)(a * a + b * b + c * c);
                int64_t bin = orc_bin(q, kmin_u, dk_u, nbins);
                if (bin < 0) continue;
                const double *f = spec + 2 * ((i * n + j) * nz + c);
                double raw = f[0] * f[0] + f[1] * f[1];
                double wk = 1.0, ck = 1.0;
                if (mas_corr) wk = pow(sx[i] * sx[j] * sx[c], (double)(p + 1));
                if (sn_corr) ck = cx[i] * cx[j] * cx[c];
                double iw2 = 1.0 / (wk * wk);
                sr[bin] += raw * iw2;
                ss[bin] += sn_corr ? ck * iw2 : 0.0;
                md[bin] += 1;
            }
        }
    }
    for (int b = 0; b < nbins; ++b) {
        modes[b] = md[b];
        sum_raw[b] = sr[b];
        sum_sn[b] = ss[b];
        pk[b] = md[b] == 0 ? 0.0 : sr[b] / ((double)md[b] * normal) - shot_noise * ss[b] / (double)md[b];
    }
    free(sr); free(ss); free(md); free(sx); free(cx);
}

/* Cross power spectrum sums in FP64, FftwFunctions::cross_power_spectrum_fkp,
 * Source/FftwFunctions.cpp:645-893: over the octant loop's mode set
 * (pk_visited) and bins (orc_bin), with icorr2 = 1/W^2 when mas_corr
 * (correction_MAS, :758):
 *   cross[b] = sum Re(F1 conj F2) icorr2   (the reference's Re1 Re2 + Im1 Im2)
 *   a1[b]    = sum |F1|^2 icorr2,  a2[b] = sum |F2|^2 icorr2,  modes[b].
 * No shot noise is subtracted (the reference leaves it out, :653). */
void orc_cross_f64(int64_t n, const double *s1, const double *s2, int p, int mas_corr, double kmin_u,
                   double dk_u, int nbins, double *cross, double *a1, double *a2, int64_t *modes)
{
    const int64_t nz = n / 2 + 1;
    for (int b = 0; b < nbins; ++b) { cross[b] = 0.0; a1[b] = 0.0; a2[b] = 0.0; modes[b] = 0; }
    double *sx = malloc(sizeof(double) * (size_t)n);
    for (int64_t a = 0; a < n; ++a) sx[a] = sinc_pi(a <= n / 2 ? a : n - a, n);
    for (int64_t i = 0; i < n; ++i) {
        int64_t a = i <= n / 2 ? i : n - i;
        for (int64_t j = 0; j < n; ++j) {
            int64_t b = j <= n / 2 ? j : n - j;
            for (int64_t c = 0; c < nz; ++c) {
                if (!pk_visited(i, j, c, n)) continue;
                int64_t bin = orc_bin((double)(a * a + b * b + c * c), kmin_u, dk_u, nbins);
                if (bin < 0) continue;
                const double *f = s1 + 2 * ((i * n + j) * nz + c);
                const double *g = s2 + 2 * ((i * n + j) * nz + c);
                double iw2 = 1.0;
                if (mas_corr) {
                    double wk = pow(sx[i] * sx[j] * sx[c], (double)(p + 1));
                    iw2 = 1.0 / (wk * wk);
                }
                cross[bin] += (f[0] * g[0] + f[1] * g[1]) * iw2;
                a1[bin] += (f[0] * f[0] + f[1] * f[1]) * iw2;
                a2[bin] += (g[0] * g[0] + g[1] * g[1]) * iw2;
                modes[bin] += 1;
            }
        }
    }
    free(sx);
}

/* Multipole sums in FP64, FftwFunctions::power_spectrum_fkp,
 * Source/FftwFunctions.cpp:1125-1212: over the octant loop's mode set and
 * bins, mu = k_los / |k| with los 0 = x, 1 = y, 2 = z (the reference's
 * I_LOSX/Y/Z), L_2 = (3 mu^2 - 1)/2, L_4 = (35 mu^4 - 30 mu^2 + 3)/8:
 *   s2[b] = sum L_2 |F|^2 / W^2,  s4[b] = sum L_4 |F|^2 / W^2,  modes[b]. */
void orc_multipole_f64(int64_t n, const double *spec, int p, int mas_corr, double kmin_u, double dk_u,
                       int nbins, int los, double *s2, double *s4, int64_t *modes)
{
    const int64_t nz = n / 2 + 1;
    for (int b = 0; b < nbins; ++b) { s2[b] = 0.0; s4[b] = 0.0; modes[b] = 0; }
    double *sx = malloc(sizeof(double) * (size_t)n);
    for (int64_t a = 0; a < n; ++a) sx[a] = sinc_pi(a <= n / 2 ? a : n - a, n);
    for (int64_t i = 0; i < n; ++i) {
        int64_t a = i <= n / 2 ? i : n - i;
        for (int64_t j = 0; j < n; ++j) {
            int64_t b = j <= n / 2 ? j : n - j;
            for (int64_t c = 0; c < nz; ++c) {
                if (!pk_visited(i, j, c, n)) continue;
                double q = (double)(a * a + b * b + c * c);
                int64_t bin = orc_bin(q, kmin_u, dk_u, nbins);
                if (bin < 0) continue;
                const double *f = spec + 2 * ((i * n + j) * nz + c);
                double iw2 = 1.0;
                if (mas_corr) {
                    double wk = pow(sx[i] * sx[j] * sx[c], (double)(p + 1));
                    iw2 = 1.0 / (wk * wk);
                }
                double fl = (double)(los == 0 ? a : (los == 1 ? b : c));
                double mu = fl / sqrt(q);
                double pw = (f[0] * f[0] + f[1] * f[1]) * iw2;
                s2[bin] += 0.5 * (3.0 * mu * mu - 1.0) * pw;
                s4[bin] += (35.0 * pow(mu, 4) - 30.0 * mu * mu + 3.0) / 8.0 * pw;
                modes[bin] += 1;
            }
        }
    }
    free(sx);
}

/* The reference's power_spectrum loop as written (FP32, OpenMP atomics,
 * float bins), Source/FftwFunctions.cpp:1660-1876, for the CPU baseline.
 * spec is interleaved complex64.  fix_octant4 selects Re^2+Im^2 for the
 * fourth octant instead of the reference's Im*Re+Im*Re. */
void orc_power_ref(int64_t nft, const float *spec, int p, int mas_corr, int sn_corr,
                   float shot_noise, float normal_power, float deltak, float kmin,
                   float DeltaK, int nbins, int fix_octant4, float *powerk, int *modk)
{
    const int64_t nz = nft / 2 + 1;
    for (int b = 0; b < nbins; ++b) { powerk[b] = 0.f; modk[b] = 0; }
    float rDeltaK = 1.0f / DeltaK;
    float M_PI_rNft = (float)(M_PI * (1.0 / (double)nft));
    float *yy = malloc(sizeof(float) * (size_t)(nft / 2 + 1)), *sy = malloc(sizeof(float) * (size_t)(nft / 2 + 1));
    yy[0] = 1.0f; sy[0] = 0.0f;
    for (int64_t j = 1; j <= nft / 2; ++j) {
        float v = (float)j * M_PI_rNft;
        yy[j] = sinf(v) / v;
        sy[j] = sinf((float)j * M_PI_rNft);
    }
    float sn_aux = sn_corr ? shot_noise : 0.0f;
#define SPEC(ii, jj, kk) (spec + 2 * (((int64_t)(ii) * nft + (int64_t)(jj)) * nz + (int64_t)(kk)))
#define ACC(pkv)                                   \
    if (kmod < nbins) {                            \
        _Pragma("omp atomic update") powerk[kmod] += (pkv); \
        _Pragma("omp atomic update") modk[kmod]++; \
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nft / 2; ++i) {
        float xx = yy[i], sxx = sy[i];
        float i2 = (float)(i * i) * deltak * deltak;
        for (int64_t j = 0; j < nft / 2; ++j) {
            float j2 = (float)(j * j) * deltak * deltak;
            for (int64_t k = 0; k <= nft / 2; ++k) {
                float k2 = (float)(k * k) * deltak * deltak;
                float kv = sqrtf(i2 + j2 + k2);
                int kmod = (int)floorf((kv - kmin) * rDeltaK);
                float corr = mas_corr ? powf(xx * yy[j] * yy[k], (float)(p + 1)) : 1.0f;
                float icorr2 = 1.0f / (corr * corr);
                float sn = sn_aux * (float)(sq_factor(p, sxx) * sq_factor(p, sy[j]) * sq_factor(p, sy[k]));
                if (kmod < 0) continue;
                if (!(i == 0 && j == 0 && k == 0)) {
                    const float *f = SPEC(i, j, k);
                    float pkv = (f[1] * f[1] + f[0] * f[0] - sn * normal_power) * icorr2;
                    ACC(pkv)
                }
                if (j > 0 && k > 0) {
                    const float *f = SPEC(i, nft - j, k);
                    float pkv = (f[1] * f[1] + f[0] * f[0] - sn * normal_power) * icorr2;
                    ACC(pkv)
                }
                if (i > 0 && (j > 0 || k > 0)) {
                    const float *f = SPEC(nft - i, j, k);
                    float pkv = (f[1] * f[1] + f[0] * f[0] - sn * normal_power) * icorr2;
                    ACC(pkv)
                }
                if (i > 0 && j > 0 && k > 0) {
                    const float *f = SPEC(nft - i, nft - j, k);
                    float raw = fix_octant4 ? (f[1] * f[1] + f[0] * f[0]) : (f[1] * f[0] + f[1] * f[0]);
                    float pkv = (raw - sn * normal_power) * icorr2;
                    ACC(pkv)
                }
            }
        }
    }
#undef ACC
#undef SPEC
    for (int b = 0; b < nbins; ++b)
        powerk[b] = modk[b] == 0 ? 0.f : powerk[b] / ((float)modk[b] * normal_power);
    free(yy); free(sy);
}

/* ------------------------------------------------------------------------ */
/* T-web eigenvalues and labels                                             */
/* ------------------------------------------------------------------------ */

/* Eigenvalues (descending) of symmetric 3x3 matrices given as six components
 * t = (xx, yy, zz, xy, xz, yz), FP64 closed form: O.K. Smith, "Eigenvalues of
 * a symmetric 3x3 matrix", CACM 4(4):168 (1961).  Replaces the per-cell
 * gsl_eigen_symmv of get_eigen, Source/NumericalMethods.cpp:572-593, which
 * also sorts descending (GSL_EIGEN_SORT_VAL_DESC). */
void orc_eig3_f64(int64_t ncell, const double *t, double *lam)
{
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < ncell; ++c) {
        const double *m = t + 6 * c;
        double a00 = m[0], a11 = m[1], a22 = m[2], a01 = m[3], a02 = m[4], a12 = m[5];
        double p1 = a01 * a01 + a02 * a02 + a12 * a12;
        double q = (a00 + a11 + a22) / 3.0;
        double b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
        double p2 = b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * p1;
        double l1, l2, l3;
        if (p2 <= 0.0) {
            l1 = l2 = l3 = q;
        } else {
            double pp = sqrt(p2 / 6.0);
            double det = b00 * (b11 * b22 - a12 * a12) - a01 * (a01 * b22 - a12 * a02) + a02 * (a01 * a12 - b11 * a02);
            double r = det / (2.0 * pp * pp * pp);
            if (r < -1.0) r = -1.0;
            if (r > 1.0) r = 1.0;
            double phi = acos(r) / 3.0;
            l1 = q + 2.0 * pp * cos(phi);
            l3 = q + 2.0 * pp * cos(phi + 2.0 * M_PI / 3.0);
            l2 = 3.0 * q - l1 - l3;
        }
        lam[3 * c + 0] = l1;
        lam[3 * c + 1] = l2;
        lam[3 * c + 2] = l3;
    }
}

/* Labels: CWClass = 4 - #{lambda_a > lambda_th} (strict), i.e. 1 knot,
 * 2 filament, 3 sheet, 4 void; Source/Cwclass.cpp:875-890.  counts[l-1]
 * accumulates the cells of label l; ties counts cells with any eigenvalue
 * within band of lambda_th. */
void orc_classify(int64_t ncell, const double *lam, double lth, double band,
                  uint8_t *labels, int64_t counts[4], int64_t *ties)
{
    int64_t cnt[4] = {0, 0, 0, 0}, nt = 0;
    for (int64_t c = 0; c < ncell; ++c) {
        int v = 0, tie = 0;
        for (int a = 0; a < 3; ++a) {
            double l = lam[3 * c + a];
            if (l > lth) ++v;
            if (fabs(l - lth) <= band) tie = 1;
        }
        labels[c] = (uint8_t)(4 - v);
        cnt[3 - v]++;
        nt += tie;
    }
    for (int a = 0; a < 4; ++a) counts[a] = cnt[a];
    *ties = nt;
}

/* Thread count of the OpenMP loops above (CPU-baseline runs at a stated
 * thread count); n <= 0 restores all available threads. */
void orc_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
    (void)n;
#endif
}

/* C entry points over the reference's own getDensity_NGP / getDensity_CIC /
 * getDensity_TSC (Source/massFunctions.cpp:35-98, :678-790, :1050-1165),
 * compiled from the reference source by `make ref` into _ref/libref_mass.so.
 * TEST INFRASTRUCTURE ONLY: the tests pin the oracle's FP32 restatement
 * (orc_assign_ref) and the GPU keys against these, and the CPU baseline of
 * the benchmark times them.  The three helpers below are declared by the
 * reference's NumericalMethods.h and used only by the file's s_Halo variants,
 * which nothing here calls. */
#include <cstdint>
#include <cstdlib>
#include <vector>

#include <omp.h>

typedef float real_prec;
typedef unsigned long ULONG;
using std::vector;

void getDensity_NGP(ULONG, ULONG, ULONG, real_prec, real_prec, real_prec, real_prec, real_prec, real_prec, real_prec,
                    real_prec, real_prec, const vector<real_prec> &, const vector<real_prec> &,
                    const vector<real_prec> &, const vector<real_prec> &, vector<real_prec> &, bool);
void getDensity_CIC(ULONG, ULONG, ULONG, real_prec, real_prec, real_prec, real_prec, real_prec, real_prec, real_prec,
                    real_prec, real_prec, const vector<real_prec> &, const vector<real_prec> &,
                    const vector<real_prec> &, const vector<real_prec> &, vector<real_prec> &, bool);
void getDensity_TSC(ULONG, ULONG, ULONG, real_prec, real_prec, real_prec, real_prec, real_prec, real_prec, real_prec,
                    real_prec, real_prec, const vector<real_prec> &, const vector<real_prec> &,
                    const vector<real_prec> &, const vector<real_prec> &, vector<real_prec> &, bool);

ULONG index_3d(ULONG, ULONG, ULONG, int, int) { std::abort(); }
real_prec get_nobjects(const vector<real_prec> &) { std::abort(); }
int get_bin(real_prec, real_prec, int, real_prec, bool) { std::abort(); }

/* scheme 0 NGP, 1 CIC, 2 TSC; w may be null (unit weights).  delta receives
 * the reference's float mesh (N1*N2*N3).  The reference takes std::vector
 * arguments, so the inputs are copied into vectors first (outside any
 * timing the caller does around ref_assign_timed). */
extern "C" int ref_assign(int scheme, int64_t np, const float *x, const float *y, const float *z, const float *w,
                          int64_t N1, int64_t N2, int64_t N3, float L1, float L2, float L3, float d1, float d2,
                          float d3, float min1, float min2, float min3, float *delta, double *seconds)
{
    vector<real_prec> xp(x, x + np), yp(y, y + np), zp(z, z + np);
    vector<real_prec> mass = w ? vector<real_prec>(w, w + np) : vector<real_prec>();
    vector<real_prec> out((size_t)(N1 * N2 * N3));
    const bool weighted = w != nullptr;
    auto *fn = scheme == 0 ? getDensity_NGP : (scheme == 1 ? getDensity_CIC : getDensity_TSC);
    if (scheme < 0 || scheme > 2) return -1;
    const double t0 = omp_get_wtime();
    fn(N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, mass, out, weighted);
    if (seconds) *seconds = omp_get_wtime() - t0;
    for (size_t i = 0; i < out.size(); ++i) delta[i] = out[i];
    return 0;
}

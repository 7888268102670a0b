/*
 * cam_reference_api.h -- the reference's own hot-path signatures, served by
 * the B200 library (libcam_refapi.so over libcam.so).  A translation unit of
 * the reference that links against libcam_refapi.so instead of
 * massFunctions.o / NumericalMethods.o / Miscelanious.o reaches the GPU path
 * without changing its call sites.
 *
 * Types follow Headers/def.h: real_prec = float (:580), ULONG = unsigned
 * long (:611), complex_prec = float[2] (fftwf_complex, :587).
 */
#ifndef CAM_REFERENCE_API_H
#define CAM_REFERENCE_API_H

#include <vector>

#ifndef CAM_REAL_PREC_DEFINED
typedef float real_prec;
typedef unsigned long ULONG;
typedef float complex_prec[2];
#endif

/* Source/massFunctions.cpp:35 (Headers/massFunctions.h:12).  delta (N1*N2*N3)
 * is zeroed and filled; particles outside the domain are skipped. */
void getDensity_NGP(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3,
                    real_prec d1, real_prec d2, real_prec d3, real_prec min1, real_prec min2,
                    real_prec min3, const std::vector<real_prec> &xp, const std::vector<real_prec> &yp,
                    const std::vector<real_prec> &zp, const std::vector<real_prec> &Par_mass,
                    std::vector<real_prec> &delta, bool weightmass);
/* Source/massFunctions.cpp:678 (Headers/massFunctions.h:18). */
void getDensity_CIC(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3,
                    real_prec d1, real_prec d2, real_prec d3, real_prec min1, real_prec min2,
                    real_prec min3, const std::vector<real_prec> &xp, const std::vector<real_prec> &yp,
                    const std::vector<real_prec> &zp, const std::vector<real_prec> &Par_mass,
                    std::vector<real_prec> &delta, bool weightmass);
/* Source/massFunctions.cpp:1050 (Headers/massFunctions.h:26). */
void getDensity_TSC(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3,
                    real_prec d1, real_prec d2, real_prec d3, real_prec min1, real_prec min2,
                    real_prec min3, const std::vector<real_prec> &xp, const std::vector<real_prec> &yp,
                    const std::vector<real_prec> &zp, const std::vector<real_prec> &Par_mass,
                    std::vector<real_prec> &delta, bool weightmass);

/* Source/NumericalMethods.cpp:1718: unnormalised r2c into out (Nft*Nft*(Nft/2+1)). */
void do_fftw_r2c(ULONG Nft, std::vector<real_prec> &in, complex_prec *out);
/* Source/NumericalMethods.cpp:1818: c2r divided by Nft^3. */
void do_fftw_c2r(int Nft, complex_prec *in, std::vector<real_prec> &out);

/* Source/Miscelanious.cpp:1772 (FFT tidal tensor): eigenvalues of T_ab of
 * delta, descending, into out1..out3 (each Nft^3). */
void EigenValuesTweb(ULONG Nft, real_prec L1, std::vector<real_prec> &delta, std::vector<real_prec> &out1,
                     std::vector<real_prec> &out2, std::vector<real_prec> &out3);

/* Source/Miscelanious.cpp:1663 (finite differences, the reference's default
 * _USE_GFINDIFF_EIGENV_ build): eigenvalues of the gradfindif Hessian of the
 * potential phi, descending, into out1..out3.  delta is not read. */
void EigenValuesTweb(ULONG Nft, real_prec L1, std::vector<real_prec> &delta, std::vector<real_prec> &phi,
                     std::vector<real_prec> &out1, std::vector<real_prec> &out2, std::vector<real_prec> &out3);

/* Source/Miscelanious.cpp:1189: out = the potential of in (nabla^2 out = in). */
void PoissonSolver(real_prec Lbox, ULONG Nft, std::vector<real_prec> &in, std::vector<real_prec> &out);

/* Source/NumericalMethods.cpp:1123: 4th-order centred difference of in along
 * dim (1 = x, 3 = z), periodic, into out (cubic meshes; bit-identical to the
 * reference loop). */
void gradfindif(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3, std::vector<real_prec> in,
                std::vector<real_prec> &out, int dim);

/* Status of the last call on this thread (CAM_OK or a cam.h code); the
 * reference's functions return void and exit on errors, these never exit. */
int cam_refapi_last_status();

#endif

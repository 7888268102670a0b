/* Stand-in for the reference's Headers/NumericalMethods.h when its
 * Source/massFunctions.cpp is compiled on its own (oracle/Makefile, target
 * ref).  TEST INFRASTRUCTURE ONLY.  It declares just what that file uses:
 * the types and constants of Headers/def.h (real_prec = float, :580; ULONG =
 * unsigned long, :611; num_1 / num_0_5 as double constants, :652,:655;
 * _NTHREADS_ = 12, :278), the two structures of
 * Headers/Type_structures_def.h the file names (s_params_box_mas and the
 * s_Halo fields it reads), the weight-property strings and a silent
 * ScreenOutput.  The real header pulls in boost, GSL and gnuplot. */
#pragma once
#include <cmath>
#include <iostream>
#include <string>
#include <vector>
#include <omp.h>

typedef float real_prec;
typedef unsigned long ULONG;
#define num_1 static_cast<double>(1.)
#define num_0_5 static_cast<double>(0.5)
#define _NTHREADS_ 12

#define _MASS_ "_MASS_"
#define _COUNTS_ "_COUNTS_"
#define _SAT_FRACTION_ "_SAT_FRACTION_"
#define _RS_ "_RS_"
#define _VMAX_ "_VMAX_"
#define _VIRIAL_ "_VIRIAL_"
#define _SPIN_ "_SPIN_"

struct s_params_box_mas {
    int masskernel;
    ULONG Nft, NGRID;
    real_prec Lbox, d1, d2, d3, min1, min2, min3;
};

struct s_Halo {
    real_prec coord1, coord2, coord3;
    real_prec mass, number_sub_structures, rs, vmax, virial, spin, bias;
};

// Helpers the file's s_Halo variants call (Headers/NumericalMethods.h:490,564,
// :818); defined in ref_getdensity.cpp.  Not reached by getDensity_NGP/CIC/TSC.
ULONG index_3d(ULONG i, ULONG j, ULONG k, int Nj, int Nk);
real_prec get_nobjects(const std::vector<real_prec> &);
int get_bin(real_prec x, real_prec xmin, int nbins, real_prec delta, bool);

class ScreenOutput {
public:
    template <typename... A>
    void message_screen(A &&...) {}
    void DONE() {}
};


/* Stand-in for the reference's Headers/massFunctions.h (TEST INFRASTRUCTURE
 * ONLY): declarations of the functions Source/massFunctions.cpp defines and
 * calls before their definition, with the reference's signatures
 * (Headers/massFunctions.h:12-32). */
#pragma once
#include <string>
#include <vector>
using std::string;
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
void getDensity_NGPv(s_params_box_mas *, const vector<s_Halo> &, vector<real_prec> &, string);
void getDensity_CICv(s_params_box_mas *, const vector<s_Halo> &, vector<real_prec> &, string);
void getDensity_TSCv(s_params_box_mas *, const vector<s_Halo> &, vector<real_prec> &, string);

// Calls the reference-signature shim the way Bam.cpp / Miscelanious.cpp
// would: getDensity_CIC, do_fftw_r2c, do_fftw_c2r, EigenValuesTweb (both
// overloads), PoissonSolver, gradfindif.
// Usage: shim_check <dir>   (reads <dir>/in.bin, writes <dir>/*.bin)
#include <cstdio>
#include <string>
#include <vector>

#include "../include/cam_reference_api.h"

template <typename T>
static void dump(const std::string &path, const T *p, size_t n)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    std::fwrite(p, sizeof(T), n, f);
    std::fclose(f);
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    FILE *f = std::fopen((dir + "/in.bin").c_str(), "rb");
    if (!f) return 3;
    long np = 0, nft = 0;
    float box = 0.f;
    if (std::fread(&np, sizeof(long), 1, f) != 1 || std::fread(&nft, sizeof(long), 1, f) != 1 ||
        std::fread(&box, sizeof(float), 1, f) != 1)
        return 4;
    std::vector<real_prec> x(np), y(np), z(np), m;
    if (std::fread(x.data(), 4, np, f) != (size_t)np || std::fread(y.data(), 4, np, f) != (size_t)np ||
        std::fread(z.data(), 4, np, f) != (size_t)np)
        return 5;
    std::fclose(f);
    const ULONG N = (ULONG)nft;
    const real_prec d = box / (real_prec)N;
    std::vector<real_prec> delta(N * N * N);
    getDensity_CIC(N, N, N, box, box, box, d, d, d, 0.f, 0.f, 0.f, x, y, z, m, delta, false);
    if (cam_refapi_last_status()) return 10;
    dump(dir + "/mesh.bin", delta.data(), delta.size());
    std::vector<float> spec(2 * N * N * (N / 2 + 1));
    do_fftw_r2c(N, delta, reinterpret_cast<complex_prec *>(spec.data()));
    if (cam_refapi_last_status()) return 11;
    dump(dir + "/spec.bin", spec.data(), spec.size());
    std::vector<real_prec> back;
    do_fftw_c2r((int)N, reinterpret_cast<complex_prec *>(spec.data()), back);
    if (cam_refapi_last_status()) return 12;
    dump(dir + "/back.bin", back.data(), back.size());
    // overdensity, then the tidal eigenvalues
    double s = 0.0;
    for (float v : delta) s += v;
    const float mean = (float)(s / (double)delta.size());
    for (auto &v : delta) v = v / mean - 1.0f;
    std::vector<real_prec> l1, l2, l3;
    EigenValuesTweb(N, box, delta, l1, l2, l3);
    if (cam_refapi_last_status()) return 13;
    dump(dir + "/l1.bin", l1.data(), l1.size());
    dump(dir + "/l3.bin", l3.data(), l3.size());
    // the default build's T-web: the potential, its centred differences and
    // the eigenvalues of their Hessian (Cwclass::get_CWC, EigenValuesTweb
    // with _USE_GFINDIFF_EIGENV_)
    std::vector<real_prec> phi;
    PoissonSolver(box, N, delta, phi);
    if (cam_refapi_last_status()) return 14;
    dump(dir + "/phi.bin", phi.data(), phi.size());
    std::vector<real_prec> gx;
    gradfindif(N, N, N, box, box, box, phi, gx, 1);
    if (cam_refapi_last_status()) return 15;
    dump(dir + "/gx.bin", gx.data(), gx.size());
    EigenValuesTweb(N, box, delta, phi, l1, l2, l3);
    if (cam_refapi_last_status()) return 16;
    dump(dir + "/fd_l1.bin", l1.data(), l1.size());
    dump(dir + "/fd_l3.bin", l3.data(), l3.size());
    return 0;
}

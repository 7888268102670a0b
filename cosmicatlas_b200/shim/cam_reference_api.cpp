// The reference's hot-path signatures (include/cam_reference_api.h) over the
// C ABI of libcam.  One context per thread on device 0; errors are recorded
// in cam_refapi_last_status() instead of exiting.
#include "../../include/cam_reference_api.h"

#include <cstdio>
#include <vector>

#include "../../include/cam.h"

namespace {

thread_local int g_status = CAM_OK;

struct Ctx {
    cam_ctx *c = nullptr;
    Ctx() { cam_ctx_create(0, 0, &c); }
    ~Ctx() {
        if (c) cam_ctx_destroy(c);
    }
};

cam_ctx *ctx()
{
    thread_local Ctx t;
    return t.c;
}

void report(int rc, const char *what)
{
    g_status = rc;
    if (rc != CAM_OK)
        std::fprintf(stderr, "[cam] %s failed (%d): %s\n", what, rc, cam_last_error(ctx()));
}

void density(int scheme, ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3, real_prec d1,
             real_prec d2, real_prec d3, real_prec min1, real_prec min2, real_prec min3,
             const std::vector<real_prec> &xp, const std::vector<real_prec> &yp, const std::vector<real_prec> &zp,
             const std::vector<real_prec> &Par_mass, std::vector<real_prec> &delta, bool weightmass)
{
    cam_particles p{};
    p.n = (int64_t)xp.size();
    p.x = xp.data();
    p.y = yp.data();
    p.z = zp.data();
    p.w = weightmass ? Par_mass.data() : nullptr;
    p.mem = CAM_MEM_HOST;
    cam_grid g{};
    g.n[0] = (int64_t)N1;
    g.n[1] = (int64_t)N2;
    g.n[2] = (int64_t)N3;
    g.L[0] = L1; g.L[1] = L2; g.L[2] = L3;
    g.d[0] = d1; g.d[1] = d2; g.d[2] = d3;
    g.min[0] = min1; g.min[1] = min2; g.min[2] = min3;
    delta.resize(N1 * N2 * N3);
    cam_assign_stats st{};
    report(cam_assign(ctx(), &p, &g, scheme, CAM_F32, delta.data(), CAM_MEM_HOST, &st), "getDensity");
}

}  // namespace

int cam_refapi_last_status() { return g_status; }

void getDensity_NGP(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3, real_prec d1,
                    real_prec d2, real_prec d3, real_prec min1, real_prec min2, real_prec min3,
                    const std::vector<real_prec> &xp, const std::vector<real_prec> &yp,
                    const std::vector<real_prec> &zp, const std::vector<real_prec> &Par_mass,
                    std::vector<real_prec> &delta, bool weightmass)
{
    density(CAM_NGP, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass, delta, weightmass);
}

void getDensity_CIC(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3, real_prec d1,
                    real_prec d2, real_prec d3, real_prec min1, real_prec min2, real_prec min3,
                    const std::vector<real_prec> &xp, const std::vector<real_prec> &yp,
                    const std::vector<real_prec> &zp, const std::vector<real_prec> &Par_mass,
                    std::vector<real_prec> &delta, bool weightmass)
{
    density(CAM_CIC, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass, delta, weightmass);
}

void getDensity_TSC(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3, real_prec d1,
                    real_prec d2, real_prec d3, real_prec min1, real_prec min2, real_prec min3,
                    const std::vector<real_prec> &xp, const std::vector<real_prec> &yp,
                    const std::vector<real_prec> &zp, const std::vector<real_prec> &Par_mass,
                    std::vector<real_prec> &delta, bool weightmass)
{
    density(CAM_TSC, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass, delta, weightmass);
}

void do_fftw_r2c(ULONG Nft, std::vector<real_prec> &in, complex_prec *out)
{
    report(cam_fft_r2c(ctx(), (int64_t)Nft, CAM_F32, in.data(), out, CAM_MEM_HOST), "do_fftw_r2c");
}

void do_fftw_c2r(int Nft, complex_prec *in, std::vector<real_prec> &out)
{
    out.resize((size_t)Nft * Nft * Nft);
    report(cam_fft_c2r(ctx(), (int64_t)Nft, CAM_F32, in, out.data(), CAM_MEM_HOST), "do_fftw_c2r");
}

void EigenValuesTweb(ULONG Nft, real_prec L1, std::vector<real_prec> &delta, std::vector<real_prec> &out1,
                     std::vector<real_prec> &out2, std::vector<real_prec> &out3)
{
    const size_t ng = (size_t)Nft * Nft * Nft;
    cam_grid g{};
    g.n[0] = g.n[1] = g.n[2] = (int64_t)Nft;
    g.L[0] = g.L[1] = g.L[2] = L1;
    cam_tweb_opts o{};
    o.smoothing_R = 0.f;
    o.lambda_th = 0.0;
    o.tie_band = 0.0;
    o.input_type = CAM_INPUT_DELTA;  // EigenValuesTweb transforms delta as given
    std::vector<float> lam(3 * ng);
    cam_tweb_stats st{};
    const int rc = cam_tweb(ctx(), &g, delta.data(), CAM_F32, CAM_MEM_HOST, &o, nullptr, lam.data(), CAM_MEM_HOST, &st);
    report(rc, "EigenValuesTweb");
    out1.assign(lam.begin(), lam.begin() + ng);
    out2.assign(lam.begin() + ng, lam.begin() + 2 * ng);
    out3.assign(lam.begin() + 2 * ng, lam.end());
}

void EigenValuesTweb(ULONG Nft, real_prec L1, std::vector<real_prec> & /*delta*/, std::vector<real_prec> &phi,
                     std::vector<real_prec> &out1, std::vector<real_prec> &out2, std::vector<real_prec> &out3)
{
    const size_t ng = (size_t)Nft * Nft * Nft;
    cam_grid g{};
    g.n[0] = g.n[1] = g.n[2] = (int64_t)Nft;
    g.L[0] = g.L[1] = g.L[2] = L1;
    cam_tweb_opts o{};
    o.input_type = CAM_INPUT_POTENTIAL;  // the Hessian of phi as given
    o.method = CAM_TWEB_FD;
    std::vector<float> lam(3 * ng);
    cam_tweb_stats st{};
    const int rc = cam_tweb(ctx(), &g, phi.data(), CAM_F32, CAM_MEM_HOST, &o, nullptr, lam.data(), CAM_MEM_HOST, &st);
    report(rc, "EigenValuesTweb");
    out1.assign(lam.begin(), lam.begin() + ng);
    out2.assign(lam.begin() + ng, lam.begin() + 2 * ng);
    out3.assign(lam.begin() + 2 * ng, lam.end());
}

void PoissonSolver(real_prec Lbox, ULONG Nft, std::vector<real_prec> &in, std::vector<real_prec> &out)
{
    cam_grid g{};
    g.n[0] = g.n[1] = g.n[2] = (int64_t)Nft;
    g.L[0] = g.L[1] = g.L[2] = Lbox;
    out.resize((size_t)Nft * Nft * Nft);
    report(cam_poisson(ctx(), &g, in.data(), CAM_F32, CAM_MEM_HOST, 0.f, out.data(), CAM_MEM_HOST), "PoissonSolver");
}

void gradfindif(ULONG N1, ULONG N2, ULONG N3, real_prec L1, real_prec L2, real_prec L3, std::vector<real_prec> in,
                std::vector<real_prec> &out, int dim)
{
    cam_grid g{};
    g.n[0] = (int64_t)N1;
    g.n[1] = (int64_t)N2;
    g.n[2] = (int64_t)N3;
    g.L[0] = L1; g.L[1] = L2; g.L[2] = L3;
    out.resize((size_t)N1 * N2 * N3);
    report(cam_gradfindif(ctx(), &g, in.data(), CAM_F32, CAM_MEM_HOST, dim, out.data(), CAM_MEM_HOST), "gradfindif");
}

// Internal declarations shared by the CUDA translation units of libcam.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cam.h"

namespace cam {

constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

// ---------------------------------------------------------------- errors
struct Error {
    int code;
    std::string msg;
};

#define CAM_CUDA_TRY(expr)                                                          \
    do {                                                                            \
        cudaError_t _e = (expr);                                                    \
        if (_e != cudaSuccess)                                                      \
            throw ::cam::Error{CAM_E_CUDA, std::string(#expr) + ": " +              \
                                               cudaGetErrorString(_e)};             \
    } while (0)

#define CAM_REQUIRE(cond, code, msg)                                                \
    do {                                                                            \
        if (!(cond)) throw ::cam::Error{(code), (msg)};                             \
    } while (0)

// Kernel launch with error check, launch accounting and (when enabled)
// CUDA-event timing per kernel name.
#define CAM_LAUNCH_NAMED(ctx, name, kernel, grid, block, smem, ...)                 \
    do {                                                                            \
        ::cam::prof_begin((ctx), (name));                                           \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);            \
        {                                                                           \
            const cudaError_t _le = cudaGetLastError();                             \
            if (_le != cudaSuccess)                                                 \
                throw ::cam::Error{CAM_E_CUDA, std::string("launch of ") + (name) + \
                                                   ": " + cudaGetErrorString(_le)}; \
        }                                                                           \
        ::cam::prof_end(ctx);                                                       \
        (ctx)->launches++;                                                          \
    } while (0)
#define CAM_LAUNCH(ctx, kernel, grid, block, smem, ...) \
    CAM_LAUNCH_NAMED(ctx, #kernel, kernel, grid, block, smem, __VA_ARGS__)

// ------------------------------------------------------ device buffers
// Grow-only device allocation owned by a context, charged to its budget.
struct DevBuf {
    void *ptr = nullptr;
    size_t cap = 0;
};

struct FftPlan;  // cam_fft.cu

struct ProfRecord {
    const char *name;
    cudaEvent_t start, stop;
    bool side;  // launched on the side stream (reported as "side.<name>")
};

}  // namespace cam

struct cam_ctx {
    int device = 0;
    size_t budget = 0;  // 0 = unlimited
    size_t used = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    // Side stream for independent work inside one call (the Nyquist plane
    // of the fused r2c + P(k)), forked from and joined back into `stream`
    // with two events (see aux_fork / aux_join); created with the context.
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool aux_open = false;
    std::string err;
    std::recursive_mutex mu;
    int64_t launches = 0;
    std::map<std::string, cam::DevBuf> bufs;
    std::map<int64_t, cam::FftPlan *> plans;  // key: n * 2 + precision
    // sync_free: enqueue work only (no host round trips, results left in
    // device buffers) -- the mode used under stream capture
    bool sync_free = false;
    bool capturing = false;  // inside stream capture: no allocation, no events
    uint64_t asg_cap = 0;    // payload records of deferred assignments (grow-only)
    // Slabs of deferred assignments (cam_job_run), per mesh shape: the
    // fullest brick's expected records over those of a uniform catalogue,
    // as the last exact job run of that shape measured them (Poisson noise
    // taken out).  No entry until a job of the shape has run exactly.
    // slabs_off: always the exact path (the server's contexts, whose
    // admission budgets the exact payload); so does a context with an HBM
    // budget.
    std::map<int64_t, double> slab_clump;
    bool slabs_off = false;
    unsigned char *job_pin = nullptr;  // pinned readback buffer of cam_job_run
    size_t job_pin_bytes = 0;
    // bumped whenever a scratch buffer is (re)allocated or freed, so that
    // captured graphs holding its old addresses can be recognised as stale
    uint64_t gen = 0;
    void *batch = nullptr;  // cam::BatchRunner of cam_batch_run (cam_serve.cu)
    // Column FFT passes stage tiles with TMA unless CAM_NO_TMA is set in the
    // environment when the context is created (then the cp.async kernels).
    bool no_tma = false;
    unsigned *err_word = nullptr;  // device word: a bounded wait ran out (see device_error_word)
    // per-kernel timing (cam_profile_enable)
    bool prof_on = false;
    std::vector<cam::ProfRecord> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    std::map<std::string, std::pair<int64_t, double>> prof_acc;  // name -> (launches, ms)
};

namespace cam {

void prof_begin(cam_ctx *ctx, const char *name);
void prof_end(cam_ctx *ctx);

// Forks the side stream from the context's stream (the side stream then
// runs after everything enqueued so far) and returns it; aux_join makes the
// context's stream wait for everything enqueued on the side stream since.
// Both are plain event record / wait, so they also work under stream
// capture.
cudaStream_t aux_fork(cam_ctx *ctx);
void aux_join(cam_ctx *ctx);
// Launches made while a StreamScope lives go to `s` instead of the
// context's stream.
struct StreamScope {
    cam_ctx *c;
    cudaStream_t saved;
    StreamScope(cam_ctx *ctx, cudaStream_t s);
    ~StreamScope();
    StreamScope(const StreamScope &) = delete;
    StreamScope &operator=(const StreamScope &) = delete;
};

// Device word of the context where kernels report a bounded wait that ran
// out (TMA copies that did not land within their limit); zero otherwise.
// Allocated and cleared on first use; check_device_error reads it (one
// synchronisation) and throws CAM_E_CUDA if it is set.
unsigned *device_error_word(cam_ctx *ctx);
void check_device_error(cam_ctx *ctx);

// Returns a device buffer of at least `bytes`, reallocating (and
// synchronising the stream) if the cached one is too small.
void *scratch(cam_ctx *ctx, const char *name, size_t bytes);
void release_all(cam_ctx *ctx);
// Serialises device allocation/free against stream capture in other threads.
std::mutex &alloc_mutex();
// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`, never lowering it: another thread may be about to launch
// the same kernel with a larger size.
void smem_limit(const void *func, size_t bytes);
template <typename K>
inline void smem_at_least(K *kern, size_t bytes)
{
    smem_limit(reinterpret_cast<const void *>(kern), bytes);
}
void batch_destroy(void *batch);

// Host <-> device staging helpers for the C ABI.
template <typename T>
inline T *stage_in(cam_ctx *ctx, const char *name, const T *p, size_t count, int mem)
{
    if (mem == CAM_MEM_DEVICE || p == nullptr) return const_cast<T *>(p);
    T *d = static_cast<T *>(scratch(ctx, name, count * sizeof(T)));
    CAM_CUDA_TRY(cudaMemcpyAsync(d, p, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return d;
}

// ------------------------------------------------------ assignment
struct AssignGeom {
    int n[3];
    float L[3], d[3], mn[3];
    float inv_d[3];      // 1/d rounded (offsets only; keys divide exactly)
    int b[3];            // brick extent (cells)
    int nb[3];           // bricks per axis
    unsigned bmagic[3];  // ceil(2^32 / b): cell / b = umulhi(cell, bmagic)
};

struct AssignOut {
    int precision;      // CAM_F32 / CAM_F64, or -1 for uint32 counts
    void *mesh;         // device
    double *d_sum;      // device scalar: sum of the mesh (FP64)
    int64_t n_in = 0, n_lost = 0;
    // defer: no host round trip.  The payload holds an estimate of the
    // record count (grow-only per context); records past it are not
    // written and raise the overflow word of the device statistics, in
    // which case the caller reruns without defer.  n_in / n_lost are -1.
    bool defer = false;
    // Set by exact (non-slab) runs: the records a brick of a uniform
    // catalogue expects, and (without defer) the fullest brick's records;
    // with defer the fullest brick is word [5] of the device statistics.
    double brick_est = 0.0;
    uint64_t brick_max = 0;
    int64_t brick_shape = 0;  // slab_clump key of the mesh
};

// Records per brick (noise included) that hold the fullest brick of a
// catalogue whose fullest brick expects mu records: 9/8 of mu plus 4.5
// Poisson standard deviations plus 16.
inline uint64_t slab_capacity(double mu)
{
    const uint64_t cap = (uint64_t)std::ceil(1.125 * mu + 4.5 * std::sqrt(mu)) + 16;
    return (cap + 3) & ~(uint64_t)3;
}

// The clumping an exact run measured: a fullest brick of m records where a
// uniform brick expects est, less four standard deviations of noise.
inline double slab_clump_of(uint64_t m, double est)
{
    const double md = (double)m;
    return std::max(1.0, (md - 4.0 * std::sqrt(md)) / est);
}

// Device statistics of the last assignment of a context (asg.stats):
// [0] lost particles, [1] low word: bits of max |w|, [2] low word: payload
// records, [3] low word: nonzero if the deferred payload overflowed,
// [5] low word: records of the fullest brick (exact runs; 0 with slabs).
unsigned long long *assign_stats(cam_ctx *ctx);

// Runs the assignment pipeline on device particle arrays.  Writes the mesh
// and, on the device, the FP64 mesh sum.  Synchronises once (payload size)
// unless sync_free or out.defer.
void assign_device(cam_ctx *ctx, const float *x, const float *y, const float *z,
                   const float *w, int64_t np, const cam_grid &grid, int scheme,
                   AssignOut &out);
void cell_keys_device(cam_ctx *ctx, const float *x, const float *y, const float *z,
                      int64_t np, const cam_grid &grid, int scheme, int64_t *keys);
AssignGeom make_geom(const cam_grid &g, int scheme, int64_t np);

// ------------------------------------------------------ FFT
// Internal spectrum layout ("split"): main[N][N][N/2] complex plus the
// Nyquist plane nyq[N][N] (k = N/2).  Row strides are multiples of 16 bytes.
struct Spectrum {
    void *main = nullptr;
    void *nyq = nullptr;
    int64_t n = 0;
    int precision = CAM_F32;
};

FftPlan *get_plan(cam_ctx *ctx, int64_t n, int precision);
void free_plans(cam_ctx *ctx);
// Forward r2c of a real N^3 mesh; `sub` (device scalar, may be null) is
// subtracted from every element on load.
void fft_r2c_split(cam_ctx *ctx, FftPlan *plan, const void *real_in, const double *d_sub,
                   Spectrum &out);
// Inverse c2r (in place on the spectrum), result scaled by `scale`.
void fft_c2r_split(cam_ctx *ctx, FftPlan *plan, Spectrum &spec, void *real_out, double scale);
void split_to_fftw(cam_ctx *ctx, const Spectrum &s, void *dst);
void fftw_to_split(cam_ctx *ctx, const void *src, Spectrum &s);

// Strided complex column FFTs over a batch (used by the T-web passes).
void fft_columns(cam_ctx *ctx, FftPlan *plan, void *base, int64_t len, int64_t ncols,
                 int64_t jstride, int64_t nplanes, int64_t pstride, int ncomp,
                 int64_t cstride_comp, bool inverse);
void fft_rows_c2c(cam_ctx *ctx, FftPlan *plan, void *base, int64_t len, int64_t nrows,
                  int ncomp, int64_t cstride_comp, bool inverse);
const void *plan_twiddles(FftPlan *plan);

// ------------------------------------------------------ power spectrum
// Bin sums of a spectrum left on the device: sums [nbins][2] FP64
// (sum |F|^2/W^2, sum C/W^2), modes [nbins].
struct PkDevice {
    double *sums;
    unsigned long long *modes;
};
PkDevice power_bin_device(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins);
// Cross sums of two spectra of one size: sums [nbins][2] FP64
// (sum Re(F1 conj F2)/W^2, sum |F1|^2/W^2), modes [nbins]; own buffers.
PkDevice power_cross_device(cam_ctx *ctx, const Spectrum &s1, const Spectrum &s2, const cam_pk_opts &o, int nbins);
// Multipole sums about axis los (0 x, 1 y, 2 z): sums [nbins][2] FP64
// (sum L_2(mu) |F|^2/W^2, sum L_4(mu) |F|^2/W^2), modes [nbins]; own buffers.
PkDevice power_multipole_device(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins, int los);
void power_bin(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins,
               double *h_sum_raw, double *h_sum_sn, int64_t *h_modes);

// Binning tables of a P(k) (cam_power.cu): on the device [h+1] 1/W^2 per
// axis, [h+1] C/W^2 per axis, [nbins+1] squared bin edges (units of k_f),
// uploaded once per (N, options, bins); and the FP32 first guess of the bin
// (m_u, inv_s).
struct PkTables {
    const double *tab;
    int nbins;
    float m_u, inv_s;
    // bin of every integer |k|^2 / k_f^2 = q in [0, qmax] (pk_bin's result:
    // -1 below the first edge, nbins at or above the last), int16
    const short *btab;
    int qmax;
};
PkTables pk_tables(cam_ctx *ctx, int64_t n, const cam_pk_opts &o, int nbins);
// Forward r2c of a real N^3 mesh (FP32) whose last column pass also bins
// |F|^2 / W^2 of every main-spectrum mode: *d_part receives [*nparts][nbins]
// partial sums in a fixed order.  keep = false: the x pass does not write
// its output back (only P(k) is wanted; s.main then holds the y pass).
// Returns false, having launched nothing, where this path does not apply
// (FP64, no TMA, sizes without a compile-time stage list, too many bins);
// callers then run fft_r2c_split and power_bin_device.
bool fft_r2c_pk_fused(cam_ctx *ctx, FftPlan *plan, const void *real_in, const double *d_sub, Spectrum &out,
                      const PkTables &pt, bool keep, double **d_part, int *nparts);
// Completes a fused P(k): bins the Nyquist plane s.nyq into the kNumSMs
// rows that follow part's nparts rows (the buffer fft_r2c_pk_fused
// returns has room for them), adds all rows in a fixed order and takes the
// mode counts and shot-noise sums of the estimator's mode set
// (data-independent) from a table built once per key.
PkDevice power_finish_fused(cam_ctx *ctx, const Spectrum &s, const cam_pk_opts &o, int nbins, double *part,
                            int nparts);

// The FFT and P(k) of a job's mesh (cam_job_run and the serving paths use
// the same kernels, so their results are bit-identical): the r2c of
// mesh - *d_sub into s and, if pk is non-null, the P(k) sums of nb bins left
// on the device.  keep = false: the spectrum is not needed after P(k) (no
// T-web), so the fused x pass need not write it back.
PkDevice job_fft_pk(cam_ctx *ctx, FftPlan *plan, const void *mesh, const double *d_sub, Spectrum &s,
                    const cam_pk_opts *pk, int nb, bool keep);

// ------------------------------------------------------ T-web
// d_inv (may be null): 4 planes of N^3 floats, the tidal invariants I, II,
// III and the anisotropy per cell.
void tweb_device(cam_ctx *ctx, FftPlan *plan, const Spectrum &dk, float L, const double *d_mean,
                 int input_type, const cam_tweb_opts &o, uint8_t *d_labels, float *d_lambdas,
                 cam_tweb_stats *stats, float *d_inv = nullptr);

// PoissonSolver's multiplier -1/k^2 (times exp(-k^2 R^2 / 2) if R > 0) on a
// split spectrum, in place (cam_fd.cu).
void poisson_device(cam_ctx *ctx, Spectrum &s, float L, float R);
// gradfindif along dim (1 = x, 2 = y, 3 = z) of a real N^3 mesh; in != out.
void gradfindif_device(cam_ctx *ctx, const void *in, void *out, int64_t n, float L, int dim, int precision);

// FKP object weights and their sums (cam_fkp.cu): d_sums [3] = W_r, S_r, normal.
void fkp_weights_device(cam_ctx *ctx, int64_t n, const float *nbar, double nbar_const, const float *w_in, int fkp,
                        double pest, float *w_out, double *d_sums);

// BAM kernel (cam_bamkernel.cu): the 3D update of GetKernel on a device
// half-complex kernel array, bin sums and counts left in d_sum / d_modes
// [nbins]; and the kernel product of Konvolve on a split spectrum, with the
// factor 2 w / N^3 (w = *d_w, the kernel sum).
void bam_kernel_update_device(cam_ctx *ctx, void *kernel, int precision, int64_t n, float L, double kmin_u,
                              double dK_u, int nbins, const double *d_weight, int mode, double *d_sum,
                              unsigned long long *d_modes);
void konvolve_device(cam_ctx *ctx, Spectrum &s, const void *kernel, const double *d_w);

// In-place exclusive prefix sum of uint32 values; *total (device, may be
// null) receives the sum of all inputs.
void exclusive_scan_u32(cam_ctx *ctx, uint32_t *data, int64_t n, uint32_t *total);
cam_grid resolved_grid(const cam_grid &g);
int nbins_for(const cam_pk_opts &o, int64_t n);
Spectrum alloc_spectrum(cam_ctx *ctx, int64_t n, int precision, const char *tag);
void finalize_pk(int64_t n, float L, double n_obj, const cam_pk_opts &o, int nbins, const double *sr,
                 const double *ss, const int64_t *md, double *pk, int64_t *modes, double *kvec, cam_pk_info *info);

// Deterministic FP64 sum of a device array: out[0] = sum, out[1] = sum / divisor.
void reduce_sum_f64(cam_ctx *ctx, const double *in, int64_t n, double *out, double divisor);
// Mean of a device mesh of precision `prec` into a device scalar (FP64).
void mesh_mean(cam_ctx *ctx, const void *mesh, int precision, int64_t ncell, double *d_mean);

}  // namespace cam

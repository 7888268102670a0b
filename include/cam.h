/*
 * cam.h -- C ABI of the B200 mesh hot path of CosmicAtlas/BAM
 * (particle-to-mesh assignment, 3D r2c/c2r FFT, binned power spectrum, T-web).
 *
 * Every function returns CAM_OK (0) or a negative status and never exits.
 * Pointers are plain host or device pointers; the `mem` field / argument says
 * which (CAM_MEM_HOST or CAM_MEM_DEVICE).  Device pointers must belong to the
 * context's device.  Calls on one context are serialised by the context and
 * run on its stream; results written to host memory are complete when the
 * call returns, results written to device memory are complete when the
 * context's stream reaches the point of the call (cam_ctx_sync waits).
 *
 * Index convention: mesh cell (i, j, k) lives at k + N3*(j + N2*i) (z fastest),
 * Source/massFunctions.cpp:74.  Half spectra use the FFTW r2c layout
 * [i][j][k <= N/2] of complex pairs (re, im).
 */
#ifndef CAM_H
#define CAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
    CAM_OK = 0,
    CAM_E_INVAL = -1,       /* invalid argument, shape or option          */
    CAM_E_NOMEM = -2,       /* device allocation failed / over HBM budget */
    CAM_E_CUDA = -3,        /* CUDA runtime error (see cam_last_error)    */
    CAM_E_TIMEOUT = -4,     /* a bounded wait ran out                      */
    CAM_E_BUSY = -5,        /* queue full or job still running            */
    CAM_E_NOTFOUND = -6,    /* unknown job id                              */
    CAM_E_UNSUPPORTED = -7, /* size or option not implemented              */
    CAM_E_NONFINITE = -8    /* a weight was NaN or infinite                */
};

/* ---- enums ------------------------------------------------------------ */
enum { CAM_NGP = 0, CAM_CIC = 1, CAM_TSC = 2 };       /* mass assignment  */
enum { CAM_F32 = 0, CAM_F64 = 1 };                    /* mesh/FFT precision */
enum { CAM_MEM_HOST = 0, CAM_MEM_DEVICE = 1 };
enum { CAM_INPUT_DENSITY = 0, CAM_INPUT_DELTA = 1 };  /* P(k)/T-web input  */
/* T-web only: the mesh is the potential phi (nabla^2 phi = delta) that
 * Cwclass::get_CWC passes to EigenValuesTweb after PoissonSolver,
 * Source/Cwclass.cpp:259-277. */
enum { CAM_INPUT_POTENTIAL = 2 };
/* Tidal tensor of the T-web:
 *   CAM_TWEB_FFT  T_ab = c2r(k_a k_b / k^2 delta_k)        (_USE_GFFT_EIGENV_,
 *                 calc_LapPhiv, Source/NumericalMethods.cpp:2609-2680);
 *   CAM_TWEB_FD   T_ab = D_b D_a phi, D the 4th-order centred difference
 *                 (-f[+2] + 8 f[+1] - 8 f[-1] + f[-2]) / (12 d) of gradfindif,
 *                 Source/NumericalMethods.cpp:1123-1218, and phi from
 *                 PoissonSolver, Source/Miscelanious.cpp:1189-1275: the
 *                 reference's default (_USE_GFINDIFF_EIGENV_, Headers/def.h:2657). */
enum { CAM_TWEB_FFT = 0, CAM_TWEB_FD = 1 };

typedef struct cam_ctx cam_ctx;

/* Particles in structure-of-arrays form, the reference's xp, yp, zp,
 * Par_mass vectors (Headers/massFunctions.h:12).  w == NULL means unit mass
 * (weightmass == false). */
typedef struct {
    int64_t n;
    const float *x, *y, *z, *w;
    int mem;
} cam_particles;

/* Mesh geometry: N1..N3, L1..L3, d1..d3 and min1..min3 of getDensity_*
 * (Headers/massFunctions.h:12-26).  d[a] == 0 means d = L/N computed in
 * float, as Params::derived_pars does. */
typedef struct {
    int64_t n[3];
    float L[3];
    float d[3];
    float min[3];
} cam_grid;

typedef struct {
    int64_t n_in;    /* particles assigned                         */
    int64_t n_lost;  /* particles outside the domain (NLOSS)        */
    double sum_mesh; /* sum over the mesh, FP64 (get_nobjects)      */
} cam_assign_stats;

/* Binning and corrections of FftwFunctions::power_spectrum.  Edges are in
 * units of the fundamental mode k_f = 2 pi / L: kmin = DeltaKmin * k_f,
 * DeltaK = ndel * k_f (Params::derived_pars, Source/Params.cpp:4099-4104).
 * nbins == 0 selects the reference default N / (2 ndel). */
typedef struct {
    int scheme;         /* window exponent p: NGP 0, CIC 1, TSC 2          */
    int mas_correction; /* divide by W^2                                  */
    int sn_correction;  /* subtract aliased Poisson shot noise            */
    int input_type;     /* CAM_INPUT_DENSITY or CAM_INPUT_DELTA            */
    int nbins;
    double DeltaKmin;   /* kmin in units of k_f                            */
    double ndel;        /* bin width in units of k_f                       */
} cam_pk_opts;

typedef struct {
    double n_obj;       /* N_gal = sum of the mesh (density input) or 1    */
    double shot_noise;  /* V / N_gal                                       */
    double normal;      /* N_gal^2 / V (density) or N^6 / V (delta)        */
    double kf;          /* 2 pi / L                                        */
} cam_pk_info;

/* T-web options (Cwclass::get_CWC, FFT tidal-tensor variant). */
typedef struct {
    float smoothing_R;  /* Gaussian exp(-k^2 R^2 / 2); 0 = none            */
    double lambda_th;   /* label = 4 - #{lambda > lambda_th}               */
    double tie_band;    /* cells with |lambda - lambda_th| <= band counted */
    int input_type;     /* CAM_INPUT_DENSITY (rho -> rho/mean - 1), DELTA
                           or POTENTIAL                                    */
    int method;         /* CAM_TWEB_FFT (0) or CAM_TWEB_FD                 */
} cam_tweb_opts;

typedef struct {
    int64_t counts[4];  /* cells labelled 1 knot, 2 filament, 3 sheet, 4 void */
    int64_t ties;       /* cells with an eigenvalue within tie_band of lambda_th */
    double mean;        /* mean of the input mesh (density input)          */
} cam_tweb_stats;

/* ---- context ---------------------------------------------------------- */

/* Creates a context on `device` with an HBM budget in bytes (0 = no limit
 * beyond the device).  Plans, twiddle tables and scratch buffers are owned
 * by the context and reused across calls. */
int cam_ctx_create(int device, size_t hbm_budget, cam_ctx **out);
int cam_ctx_destroy(cam_ctx *ctx);
/* Device memory of all contexts comes from one stream-ordered pool per
 * device.  Memory a context frees (cam_ctx_destroy, a server dropping its
 * caches) stays in the pool for the next allocation, so a long-running
 * process does not pay the device's allocation cost again; the pool is
 * trimmed automatically when an allocation fails.  cam_pool_trim hands the
 * pool's idle memory back to the device now.  No reference counterpart. */
int cam_pool_trim(int device);
/* Device allocations the library made in this process (all devices): how
 * many, how many first failed and were retried after trimming the pool
 * (that trim waits for the whole device), bytes, and the host time spent in
 * them.  reset != 0 zeroes the counters after reading.  No reference
 * counterpart. */
typedef struct {
    int64_t allocs;
    int64_t failures;
    int64_t bytes;
    double total_ms;
    double max_ms;
} cam_alloc_stats;
int cam_alloc_stats_get(cam_alloc_stats *out, int reset);
/* Sets the CUDA stream (cudaStream_t) the context launches on (NULL = the
 * context's own stream).  Device inputs are read on that stream: data that
 * the caller produced on another stream must be complete before the call,
 * or the caller sets its own stream here. */
int cam_ctx_set_stream(cam_ctx *ctx, void *stream);
int cam_ctx_sync(cam_ctx *ctx);
/* Message of the last failure on this context ("" if none). */
const char *cam_last_error(cam_ctx *ctx);
/* Number of kernels this context has launched so far. */
int64_t cam_kernel_launches(cam_ctx *ctx);
/* Per-kernel timing with CUDA events on the context's stream (no
 * reference counterpart; the reference prints wall-clock banners,
 * Source/ScreenOutput.cpp:466).  cam_profile_read writes lines
 * "kernel,launches,total_ms" and optionally resets the totals. */
int cam_profile_enable(cam_ctx *ctx, int on);
int cam_profile_read(cam_ctx *ctx, char *buf, size_t len, int reset);
const char *cam_version(void);

/* ---- mass assignment --------------------------------------------------
 * Replaces getDensity_NGP / getDensity_CIC / getDensity_TSC,
 * Source/massFunctions.cpp:35, :678, :1050 (declared in
 * Headers/massFunctions.h:12,18,26).  mesh_out (N1*N2*N3 values of the
 * chosen precision) is overwritten (the reference zeroes delta first).
 * Deterministic: integer keys, counting sort into mesh bricks, exact
 * fixed-point accumulation per cell; no float atomics. */
int cam_assign(cam_ctx *ctx, const cam_particles *parts, const cam_grid *grid,
               int scheme, int precision, void *mesh_out, int out_mem,
               cam_assign_stats *stats);

/* Integer NGP counts per cell (uint32), bit-exact with the reference's
 * float cell arithmetic (getDensity_NGP with weightmass == false). */
int cam_count_ngp(cam_ctx *ctx, const cam_particles *parts, const cam_grid *grid,
                  uint32_t *counts_out, int out_mem, cam_assign_stats *stats);

/* Home-cell sort key of every particle: k + N3*(j + N2*i) of the cell the
 * reference indexes for `scheme`, or N1*N2*N3 for a lost particle. */
int cam_cell_keys(cam_ctx *ctx, const cam_particles *parts, const cam_grid *grid,
                  int scheme, int64_t *keys_out, int out_mem);

/* ---- FFT ---------------------------------------------------------------
 * Replace do_fftw_r2c / do_fftw_c2r, Source/NumericalMethods.cpp:1718, :1818.
 * Cubic N^3, N = 2^a 3^b, 8 <= N <= 1024.  r2c is unnormalised; c2r divides
 * by N^3 as the reference does.  `precision` selects float or double
 * elements.  Plans (twiddles) are built once per (N, precision) and cached. */
int cam_fft_r2c(cam_ctx *ctx, int64_t n, int precision, const void *in, void *out, int mem);
int cam_fft_c2r(cam_ctx *ctx, int64_t n, int precision, const void *in, void *out, int mem);

/* ---- power spectrum ----------------------------------------------------
 * Replaces PowerSpectrumF::compute_power_spectrum_grid(const vector&, bool),
 * Source/PowerSpectrumF.cpp:1739, and FftwFunctions::power_spectrum,
 * Source/FftwFunctions.cpp:1660.  mesh is N^3 (cubic) of `precision`.
 * Outputs per bin (host arrays of nbins; any may be NULL): pk, modes,
 * kvector (bin centres kmin + (b + 1/2) DeltaK, PowerSpectrumF.cpp:1792). */
int cam_power(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision,
              int mem, const cam_pk_opts *opts, double *pk, int64_t *modes,
              double *kvector, cam_pk_info *info);

/* cam_power plus the multipoles l = 2, 4 about a fixed line of sight (los:
 * 0 x, 1 y, 2 z; the reference's LOS, Headers/def.h:1714), as
 * FftwFunctions::power_spectrum_fkp computes them for a box,
 * Source/FftwFunctions.cpp:1125-1212 and :1614-1625:
 *   p2[b] = 5 sum L_2(mu) |F|^2 / W^2 / (modes normal),
 *   p4[b] = 9 sum L_4(mu) |F|^2 / W^2 / (modes normal),
 * mu = k_los / |k|, no shot noise subtracted for l > 0; p0 is cam_power's
 * P(k).  Host arrays of nbins; any may be NULL. */
int cam_power_multipoles(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision, int mem,
                         const cam_pk_opts *opts, int los, double *p0, double *p2, double *p4, int64_t *modes,
                         double *kvector, cam_pk_info *info);

/* Cross power spectrum of two meshes: replaces
 * PowerSpectrumF::compute_cross_power_spectrum_grid, Source/PowerSpectrumF.cpp:549,
 * with FftwFunctions::cross_power_spectrum_fkp, Source/FftwFunctions.cpp:645.
 * mesh_x uses opts->input_type, mesh_y input_type_y (a density becomes
 * rho/mean - 1).  Over P(k)'s mode set and bins (opts->scheme and
 * mas_correction give W; no shot noise is subtracted, as in the reference):
 *   pk_x[b] = sum |F_X|^2 / W^2 / (modes N^6 / L^3), pk_y likewise,
 *   pk[b]   = sum Re(F_X conj F_Y) / W^2 / (modes N^6 / L^3),
 *             or, with want_coeff, that divided by sqrt(pk_x pk_y).
 * Host arrays of nbins; any may be NULL. */
int cam_cross_power(cam_ctx *ctx, const cam_grid *grid, const void *mesh_x, const void *mesh_y, int precision,
                    int mem, const cam_pk_opts *opts, int input_type_y, int want_coeff, double *pk,
                    double *pk_x, double *pk_y, int64_t *modes, double *kvector);

/* ---- T-web -------------------------------------------------------------
 * Replaces Cwclass::get_CWC, Source/Cwclass.cpp:235, with the FFT tidal
 * tensor of EigenValuesTweb, Source/Miscelanious.cpp:1772.  labels (N^3
 * uint8, values 1..4) and lambdas (3 x N^3 float, planes lambda1, lambda2,
 * lambda3, descending) may be NULL; out_mem says where they live. */
int cam_tweb(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision,
             int mem, const cam_tweb_opts *opts, uint8_t *labels, float *lambdas,
             int out_mem, cam_tweb_stats *stats);

/* cam_tweb plus the tidal invariants BAM's bias binning reads, per cell:
 * invariants = 4 planes of N^3 floats, I = l1 + l2 + l3, II = l1 l2 + l2 l3
 * + l1 l3, III = l1 l2 l3 (invariant_field_I/II/III,
 * Source/Miscelanious.cpp:1466-1492) and the tidal anisotropy
 * sqrt(((l3-l1)^2 + (l3-l2)^2 + (l2-l1)^2) / 2) / (2 + I) (tidal_anisotropy,
 * :1460), formed in FP64 from the tensor.  labels and lambdas may be NULL. */
int cam_tweb_invariants(cam_ctx *ctx, const cam_grid *grid, const void *mesh, int precision, int mem,
                        const cam_tweb_opts *opts, uint8_t *labels, float *lambdas, float *invariants,
                        int out_mem, cam_tweb_stats *stats);

/* ---- potential and finite differences --------------------------------
 * Replaces PoissonSolver(Lbox, Nft, in, out), Source/Miscelanious.cpp:1189:
 * phi = c2r(-delta_k / k^2) / N^3 (k = 0 mode -> 0), with k from the
 * signed FFT frequencies times 2 pi / L.  smoothing_R > 0 also multiplies
 * delta_k by exp(-k^2 R^2 / 2).  delta and phi are N^3 of `precision`; mem
 * and out_mem say where they live. */
int cam_poisson(cam_ctx *ctx, const cam_grid *grid, const void *delta, int precision, int mem,
                float smoothing_R, void *phi, int out_mem);

/* Replaces gradfindif(N1, N2, N3, L1, L2, L3, in, out, dim),
 * Source/NumericalMethods.cpp:1123: out = (-in[+2] + 8 in[+1] - 8 in[-1] +
 * in[-2]) / (12 L / N) along dim (1 = x, the slowest index; 3 = z),
 * periodic.  FP32 results equal the reference loop's bit for bit.  in may
 * equal out (the reference takes `in` by value). */
int cam_gradfindif(cam_ctx *ctx, const cam_grid *grid, const void *in, int precision, int mem, int dim,
                   void *out, int out_mem);

/* ---- catalogue weights -------------------------------------------------
 * The per-object weights of the catalogue interpolation with FKP weighting,
 * Source/Catalog.cpp:14120-14190: w = w_in * (fkp ? 1 / (1 + P_est nbar) : 1)
 * for n objects, nbar[i] the object's mean density (NULL: nbar_const for
 * all, the catalogue's mean density without a random catalogue), w_in the
 * product of its other weights (NULL: 1).  w_out (float, n) is what the
 * reference passes to grid_assignment_* as the mass; give it to cam_assign
 * as the particles' w.  sums (host, may be NULL): [0] n_selected,
 * [1] W_r = sum w, [2] S_r = sum w^2, [3] normal = sum nbar w^2 (FP64, fixed
 * order).  mem applies to nbar and w_in, out_mem to w_out. */
int cam_fkp_weights(cam_ctx *ctx, int64_t n, const float *nbar, double nbar_const, const float *w_in, int fkp,
                    double P_est, int mem, float *w_out, int out_mem, double *sums);

/* ---- BAM kernel ---------------------------------------------------------
 * The 3D update of Bam::GetKernel, Source/Bam.cpp:529 (:786-910).  kernel is
 * the real half-complex array [N][N][N/2+1] of `precision`.  Each element
 * gets the bin b = floor((|k| - kmin) / DeltaK), kmin = DeltaKmin k_f and
 * DeltaK = ndel k_f, in the reference's real_prec arithmetic; for
 * 0 <= b < nbins it becomes weight[b] (CAM_KERNEL_SET: GetKernel without
 * rejection) or is multiplied by it (CAM_KERNEL_SCALE: with rejection).
 * kernel_binned[b] (may be NULL) = mean of the updated kernel over bin b
 * (kernel_updated, :905-910; bin 0 = the mean of bins 1..4); modes[b] (may
 * be NULL) = its element count.  weight, kernel_binned and modes are host
 * arrays of nbins (1 <= nbins <= 1600). */
enum { CAM_KERNEL_SET = 0, CAM_KERNEL_SCALE = 1 };
int cam_bam_kernel_update(cam_ctx *ctx, const cam_grid *grid, int precision, double DeltaKmin, double ndel,
                          int nbins, const double *weight, int mode, void *kernel, int mem,
                          double *kernel_binned, int64_t *modes);

/* Replaces Bam::Konvolve, Source/Bam.cpp:1027:
 * out = c2r(kernel * r2c(in)) / N^3 * 2 w / N^3, w = the sum of the kernel
 * over its half-complex array.  in may equal out.  A non-finite sum of in
 * returns CAM_E_NONFINITE (the reference exits, :1060-1067). */
int cam_konvolve(cam_ctx *ctx, const cam_grid *grid, const void *in, int precision, int mem,
                 const void *kernel, int kernel_mem, void *out, int out_mem);

/* ---- one mesh job: particles -> mesh -> FFT -> P(k) [-> T-web] ----------
 * The plain per-call GPU path of one BAM iteration: the mesh and its
 * spectrum stay resident on the device between the stages, and the host
 * waits once, for the statistics and P(k) at the end.  A context's first
 * job of a mesh shape sorts the particles into mesh bricks exactly (count,
 * scan, scatter) and measures its fullest brick; later jobs of that shape
 * write every brick's records into a fixed slab sized from it and skip the
 * count.  A job whose records do not fit (its slabs or the payload
 * estimate) runs again exactly, so results never depend on the path. */
typedef struct {
    cam_particles parts;
    cam_grid grid;
    int scheme;
    int precision;
    cam_pk_opts pk;     /* pk.nbins > 0 to compute P(k)            */
    int want_tweb;
    cam_tweb_opts tweb;
} cam_job_desc;

typedef struct {
    double *pk;          /* nbins (host), may be NULL              */
    int64_t *modes;      /* nbins (host), may be NULL              */
    double *kvector;     /* nbins (host), may be NULL              */
    uint8_t *labels;     /* N^3 (host), may be NULL                */
    cam_pk_info pk_info;
    cam_assign_stats assign;
    cam_tweb_stats tweb;
} cam_job_result;

int cam_job_run(cam_ctx *ctx, const cam_job_desc *job, cam_job_result *res);

/* Copies host particles into device buffers owned by the context (one
 * cudaMemcpyAsync per array on the context's stream) and returns them as a
 * CAM_MEM_DEVICE particle set, valid until the next cam_particles_stage on
 * this context.  Lets one upload serve several jobs on the same particles
 * (the reference calls getDensity_* once per scheme on the same vectors,
 * e.g. Source/Catalog.cpp:662-683). */
int cam_particles_stage(cam_ctx *ctx, const cam_particles *host, cam_particles *device_out);

/* ---- many jobs: graph-packed batches and a continuous-batching server ---
 * No single counterpart in the reference: BAM issues its mesh jobs one
 * after another from the calibration loop (Source/Bam.cpp:13424,
 * Bam::bamrunner), one cam_job_run each.  Both entry points below return,
 * per job, exactly what cam_job_run returns for it (the same mesh,
 * transform and binning; every job on its own buffers), except that labels
 * are not returned by batches.
 *
 * cam_batch_run: consecutive jobs of one shape (mesh, particle count,
 * weights or not, scheme, precision, box and all P(k)/T-web options equal)
 * run as batches of up to 32 concurrent jobs.  The first batch of a shape
 * sizes every buffer; its work is then captured into one CUDA graph, and
 * later batches of that shape copy their particles in and replay it: one
 * host synchronisation per batch instead of several per job.
 * res[i].labels must be NULL.  Returns CAM_OK or the first failing job's
 * status (the other jobs' results are still filled in). */
int cam_batch_run(cam_ctx *ctx, const cam_job_desc *jobs, int njobs, cam_job_result *res);

typedef struct cam_server cam_server;

typedef struct {
    int64_t submitted, completed, failed;
    int64_t queued, running;          /* at the time of the call            */
    int64_t batches, batched_jobs;    /* graph-packed batches and their jobs */
    int64_t graph_replays;            /* batches that replayed a graph      */
    size_t bytes_reserved;            /* HBM held or reserved by the workers */
    size_t peak_bytes_reserved;
    size_t budget;
    double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> result latency    */
} cam_server_stats;

/* Starts a server on `device` with `nworkers` worker threads (each runs
 * jobs on its own stream, so their work overlaps on the GPU).  A queued job
 * starts as soon as a worker is free and the server's device memory (held
 * caches plus the reservations of running jobs) stays within hbm_budget
 * (0 = 80% of the free memory); jobs are admitted oldest first.  A large
 * job (one that moves more than ~0.75 GB through HBM, and so fills the GPU
 * by itself) runs on a context shared by the large jobs, one at a time;
 * smaller jobs may start ahead of a large job that waits for that lane.
 * When several queued jobs share a small shape (N <= 128, no labels), a
 * worker takes up to max_batch of them and runs them as one graph-packed
 * batch, as cam_batch_run does. */
int cam_server_create(int device, size_t hbm_budget, int nworkers, int max_batch, cam_server **out);
/* Queues a job.  The descriptor is copied; the particle arrays and the
 * result's output arrays must stay valid until the job completes.
 * CAM_E_NOMEM if the job alone exceeds the budget, CAM_E_INVAL for an
 * invalid job, CAM_E_BUSY if 2^20 jobs are queued. */
int cam_server_submit(cam_server *s, const cam_job_desc *job, cam_job_result *res, uint64_t *id);
/* CAM_E_BUSY while queued or running, else the job's final status (once:
 * later calls for the same id return CAM_E_NOTFOUND). */
int cam_server_poll(cam_server *s, uint64_t id);
/* Waits up to timeout_us (< 0: no limit); CAM_E_TIMEOUT if still running,
 * else as cam_server_poll. */
int cam_server_wait(cam_server *s, uint64_t id, int64_t timeout_us);
/* Counters and latency percentiles; reset != 0 clears the latency record
 * and the counters after reading them. */
int cam_server_stats_get(cam_server *s, cam_server_stats *st, int reset);
/* Per-job trace (no reference counterpart: BAM prints wall-clock banners
 * only, Source/ScreenOutput.cpp:466).  Times in ms since the server started. */
typedef struct {
    uint64_t id;
    double submit_ms, start_ms, end_ms;
    int worker;  /* worker thread that ran the job                    */
    int batch;   /* jobs in the batch it ran in (1 = alone)           */
    int status;
    int big;     /* counted as a large job (at most one runs at once) */
} cam_server_job_trace;
/* Moves up to `max` records of completed jobs (oldest first) into out. */
int cam_server_trace(cam_server *s, cam_server_job_trace *out, int max, int *count);
/* Message of the most recent failed job ("" if none); valid until the next
 * call from this thread. */
const char *cam_server_last_error(cam_server *s);
/* Finishes the queued and running jobs, then stops the workers. */
int cam_server_destroy(cam_server *s);

/* ---- persistent on-device request loop -----------------------------------
 * No single counterpart in the reference: BAM issues its mesh jobs one
 * after another from the calibration loop (Source/Bam.cpp:13424,
 * Bam::bamrunner; get_BAM_DM per iteration, :2102-2303).  Here one kernel
 * stays resident, one CTA of 1024 threads per SM, and every CTA runs whole
 * jobs -- assignment, r2c FFT, P(k) -- taking them from a queue in pinned
 * host memory that the device reads directly, so no kernel is launched per
 * job.  Jobs: FP32 cubic meshes of N = 32, 64 or 128, NGP/CIC/TSC, unit or
 * per-particle weights, particles already on the device (CAM_MEM_DEVICE),
 * density P(k) with at most 128 bins, no T-web (others: CAM_E_UNSUPPORTED).
 * The mesh sum and the lost count equal cam_job_run's bit for bit (same
 * assignment functions and fixed-point scale); P(k) agrees to FP32
 * rounding (its FFT takes radix-8 stages, its binning FP64 per mode); a
 * job's results do not depend on the jobs beside it.
 * Every device-side wait is bounded: with no job for idle_timeout_s the
 * kernel ends (cam_devloop_state then returns CAM_E_TIMEOUT) and the next
 * submission or wait relaunches it.  One host thread per loop. */
typedef struct cam_devloop cam_devloop;
/* Preallocates, per CTA, a record buffer of 4 * max_particles records and
 * the mesh and spectrum of N = 128; launches the kernel.  nslots: queued
 * jobs at most (submit waits, up to 30 s, for a slot).  A CTA holds its
 * SM's whole register file, so other kernels wait for SMs the loop does
 * not use: max_ctas (0 = one per SM) leaves the rest free. */
int cam_devloop_create(int device, int64_t max_particles, int nslots, double idle_timeout_s, int max_ctas,
                       cam_devloop **out);
/* Queues a job; the particle arrays must stay valid until it completes. */
int cam_devloop_submit(cam_devloop *loop, const cam_job_desc *job, uint64_t *id);
/* Waits up to timeout_us (< 0: no limit) for job `id` and fills res's P(k)
 * (pk, modes, kvector, pk_info) and assignment statistics as cam_job_run
 * does; `job` is the descriptor it was submitted with.  CAM_E_TIMEOUT if
 * it has not completed, CAM_E_NOTFOUND for an unknown or overwritten id. */
int cam_devloop_wait(cam_devloop *loop, uint64_t id, int64_t timeout_us, const cam_job_desc *job,
                     cam_job_result *res);
/* CAM_E_TIMEOUT if the kernel has ended on its idle limit, else CAM_OK;
 * *running (may be NULL) = 1 while the kernel is resident. */
int cam_devloop_state(cam_devloop *loop, int *running);
/* Lets the queued jobs finish, ends the kernel and frees everything. */
int cam_devloop_destroy(cam_devloop *loop);
const char *cam_devloop_last_error(cam_devloop *loop);

/* ---- power spectrum without device allocation --------------------------
 * No counterpart in the reference.  For callers that may not allocate
 * device memory -- code running inside a memory pool or arena it does not
 * own, or a latency-critical loop that must never reach cudaMalloc -- this
 * bins a spectrum the caller already holds on the current device, using
 * only a fixed scratch array (about 1.9 MB) built into the library.
 *   spec    device pointer, FFTW r2c layout [i][j][k <= N/2] of an N^3
 *           mesh, complex float (CAM_F32) or complex double (CAM_F64)
 *   n_obj   sum of the density mesh (CAM_INPUT_DENSITY); ignored for delta
 *   pk, modes  host arrays of nbins (modes may be NULL)
 *   stream  cudaStream_t to run on (NULL = the legacy default stream);
 *           the call returns after that stream has finished its work.  It
 *           may not be under stream capture: a capturing stream returns
 *           CAM_E_UNSUPPORTED and the capture is left untouched.
 * Results equal cam_power's binning of the same spectrum.  Limits: N <= 2048
 * and nbins <= 512; larger inputs return CAM_E_UNSUPPORTED.  The first call
 * on a device looks up the scratch array's device address.  All calls share
 * that array and each call overwrites what it uses; calls that overlap on
 * the GPU (other streams, other host threads) race on it, so serialise them. */
int cam_power_noalloc(const void *spec, int64_t n, int precision, float box, double n_obj,
                      const cam_pk_opts *opts, double *pk, int64_t *modes, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CAM_H */

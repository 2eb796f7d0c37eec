/*
 * fc_api.h -- C ABI of the fftcorr_b200 library (B200 / sm_100a).
 *
 * This is the drop-in boundary behind the reference fftcorr API.  Every
 * entry point is `extern "C"`, takes plain pointers and sizes, and returns an
 * fc_status (0 on success, a negative code otherwise; fc_last_error() gives
 * the message).  Host pointers are borrowed for the duration of the call.
 * Device memory is owned by the opaque handles.  Calls are synchronous
 * unless their name ends in _async; handles are not thread-safe (like the
 * reference classes), distinct handles may be used from distinct threads.
 *
 * Reference interfaces replaced (file:line in cshallue/fftcorr):
 *   ConfigSpaceGrid    cc/grid/config_space_grid.h:10-57,
 *                      fftcorr/grid/config_space_grid.pxd:9-14
 *   MassAssignor       cc/particle_mesh/mass_assignor.h:30-234,
 *                      fftcorr/particle_mesh/mass_assignor.pxd:10-29
 *   DistributionScheme cc/particle_mesh/distribution_functions.h:11-15
 *   PeriodicCorrelator cc/correlate/correlator.h:254-358
 *   Correlator         cc/correlate/correlator.h:360-505,
 *                      fftcorr/correlate/correlator.pxd:21-66
 *   WindowCorrection   cc/correlate/window_correct.h:8-12
 *   HistogramList      cc/histogram/histogram_list.h:10-68,
 *                      fftcorr/histogram/histogram_list.pxd:6-13
 *   array_ops sum/sumsq/add_scalar/multiply_by  cc/array/array_ops.h:16-20
 */
#ifndef FC_API_H
#define FC_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
typedef enum fc_status {
  FC_OK = 0,
  FC_ERR_INVALID = -1,     /* std::invalid_argument in the reference     */
  FC_ERR_RANGE = -2,       /* std::out_of_range                           */
  FC_ERR_ALLOC = -3,       /* std::bad_alloc (device or pinned host)      */
  FC_ERR_CUDA = -4,        /* CUDA runtime failure                        */
  FC_ERR_CUFFT = -5,       /* cuFFT plan or execution failure             */
  FC_ERR_STATE = -6,       /* std::logic_error: call out of order         */
  FC_ERR_UNSUPPORTED = -7, /* feature not built into this library         */
  FC_ERR_TIMEOUT = -8,     /* a bounded device wait gave up               */
  FC_ERR_ADMISSION = -9    /* a request does not fit the memory budget    */
} fc_status;

/* Message of the last failing call on this thread (never NULL). */
const char *fc_last_error(void);
/* Library version as 10000*major + 100*minor + patch. */
int fc_version(void);
/* Selects the CUDA device used by handles created afterwards on this thread. */
int fc_set_device(int device);

/* ------------------------------------------------------------- constants */
/* DistributionScheme (distribution_functions.h:11-15); 3 is new: trilinear
 * cloud-in-cell, which the reference does not have. */
enum {
  FC_NEAREST_CELL = 0,
  FC_TRIANGULAR_SHAPED_CLOUD = 1,
  FC_WAVELET = 2,
  FC_CLOUD_IN_CELL = 3
};
/* WindowCorrection (window_correct.h:8-12). */
enum {
  FC_NO_CORRECTION = 0,
  FC_TSC_CORRECTION = 1,
  FC_TSC_ALIASED_CORRECTION = 2
};
/* Arithmetic of the correlator's grids and FFTs.  FC_FP32_MIXED keeps cell
 * coordinates, Y_lm normalisation, subgrids and histograms in FP64. */
enum { FC_FP64 = 0, FC_FP32_MIXED = 1 };
/* Correlator kinds. */
enum { FC_PERIODIC = 0, FC_SURVEY = 1 };

/* ------------------------------------------------------- ConfigSpaceGrid */
typedef struct fc_grid fc_grid;

/* ConfigSpaceGrid(shape, posmin, cell_size): a zeroed FP64 grid in device
 * memory (config_space_grid.h:12-16). */
int fc_grid_create(const int shape[3], const double posmin[3],
                   double cell_size, fc_grid **out);
/* The same grid with a cell type: FC_FP64 (as fc_grid_create) or
 * FC_FP32_MIXED, FP32 cells for the FP32-mixed correlators, which then read
 * the grid without a conversion.  Mass assignment into an FP32 grid sums in
 * FP64 and rounds once per update of a cell; the host copies, sums and
 * arithmetic below work on either, in FP64 per cell.  (A library extension:
 * the reference's grids are always FP64.) */
int fc_grid_create_precision(const int shape[3], const double posmin[3],
                             double cell_size, int precision, fc_grid **out);
int fc_grid_precision(const fc_grid *grid, int *precision);
int fc_grid_destroy(fc_grid *grid);
/* ConfigSpaceGrid::clear (config_space_grid.h:27). */
int fc_grid_clear(fc_grid *grid);
/* Host <-> device copies of the N0*N1*N2 row-major grid, FP64 on the host
 * (an FP32 grid rounds each cell once on upload). */
int fc_grid_upload(fc_grid *grid, const double *host);
int fc_grid_download(const fc_grid *grid, double *host);
/* Device pointer of an FP64 grid's data (valid until fc_grid_destroy);
 * FC_ERR_INVALID for an FP32 grid. */
int fc_grid_device_ptr(const fc_grid *grid, double **device_ptr);
/* Device pointer of the cells of either precision (fc_grid_precision). */
int fc_grid_device_data(const fc_grid *grid, void **device_ptr);
/* ConfigSpaceGrid::get_grid_coords (config_space_grid.h:31-46); *inside is
 * set to 1 or 0 like the reference's bool return. */
int fc_grid_coords(const fc_grid *grid, const double survey[3], int periodic,
                   double grid_coords[3], int *inside);
/* array_ops::sum and sumsq (array_ops.cc:95-137), FP64, deterministic. */
int fc_grid_sum(fc_grid *grid, double *sum, double *sumsq);
/* array_ops::add_scalar / multiply_by (array_ops.cc:55-93). */
int fc_grid_add_scalar(fc_grid *grid, double s);
int fc_grid_multiply_by(fc_grid *grid, double s);
/* y += a * x elementwise (same shapes; precisions may differ, each cell
 * computed in FP64).  Used to form N = D - alpha R from separately
 * assigned catalogs. */
int fc_grid_axpy(fc_grid *y, double a, const fc_grid *x);

/* ---------------------------------------------------------- MassAssignor */
typedef struct fc_assignor fc_assignor;

typedef struct fc_assign_stats {
  uint64_t num_added;
  uint64_t num_skipped;
  double totw;
  double totwsq;
  double sort_time;   /* seconds, device time of the radix sorts */
  double window_time; /* seconds, device time of the stencil scatter */
} fc_assign_stats;

/* MassAssignor(grid, scheme, periodic_wrap, buffer_size)
 * (mass_assignor.h:32-50).  buffer_size 0 assigns every add call at once;
 * otherwise particles are buffered on the device and assigned when at least
 * buffer_size are waiting, or on flush.  The grid must outlive the handle. */
int fc_assignor_create(fc_grid *grid, int scheme, int periodic_wrap,
                       int64_t buffer_size, fc_assignor **out);
int fc_assignor_destroy(fc_assignor *ma);
/* add_particles_to_buffer overloads (mass_assignor.h:72-103):
 * posw is (n, 4) x,y,z,w; pos is (n, 3) with weights (n) or one weight. */
int fc_assignor_add_posw(fc_assignor *ma, const double *posw, int64_t n);
int fc_assignor_add_pos_weights(fc_assignor *ma, const double *pos,
                                const double *weights, int64_t n);
int fc_assignor_add_pos_weight(fc_assignor *ma, const double *pos,
                               double weight, int64_t n);
/* Same as fc_assignor_add_posw but posw is already in device memory. */
int fc_assignor_add_posw_device(fc_assignor *ma, const double *posw_device,
                                int64_t n);
/* MassAssignor::flush (mass_assignor.h:127-191). */
/* add_random_particles (fftcorr/catalog/random_catalog.py:8-87) with the
 * positions generated on the device: n points uniform over the grid's box
 * [posmin, posmin + shape * cell), each of weight particle_weight, displaced
 * by disp (host (N0, N1, N2, 3) FP64 field, as apply_displacement_field;
 * NULL for none), assigned in batches of batch_size (<= 0: 2^26).  The
 * generator is Philox4x32-10 keyed by seed, so the catalog does not depend
 * on batch_size; it differs value by value from numpy's generator.  Fails
 * with FC_ERR_INVALID if a displaced point leaves a non-periodic grid. */
int fc_assignor_add_random(fc_assignor *ma, int64_t n, double particle_weight,
                           const double *disp, uint64_t seed,
                           int64_t batch_size);
int fc_assignor_flush(fc_assignor *ma);
/* MassAssignor::clear (mass_assignor.h:60-70). */
int fc_assignor_clear(fc_assignor *ma);
int fc_assignor_stats(fc_assignor *ma, fc_assign_stats *stats);
int fc_assignor_buffer_size(const fc_assignor *ma, int64_t *buffer_size);

/* ------------------------------------------------------------ Correlator */
typedef struct fc_correlator fc_correlator;

/* PeriodicCorrelator (kind FC_PERIODIC, posmin ignored) or Correlator
 * (kind FC_SURVEY) (correlator.h:20-39, 366-377).  fft_flags is accepted
 * for interface compatibility (the reference passes FFTW planner flags). */
int fc_corr_create(int kind, const int shape[3], double cell_size,
                   const double posmin[3], int window_correct, double rmax,
                   double dr, double kmax, double dk, int maxell,
                   unsigned fft_flags, int precision, fc_correlator **out);
int fc_corr_destroy(fc_correlator *corr);

/* Output geometry: histogram rows (maxell/2+1), r and k bin counts, and the
 * r- and k-subgrid shapes (correlator.h:109-205). */
int fc_corr_dims(const fc_correlator *corr, int *nrows, int *nr, int *nk,
                 int rshape[3], int kshape[3]);

/* BaseCorrelator::set_grid2 / set_grid2_fft (correlator.h:53-77).  The
 * complex grid is N0 x N1 x (N2/2+1) interleaved (re, im) doubles. */
int fc_corr_set_grid2(fc_correlator *corr, const double *host_grid);
int fc_corr_set_grid2_grid(fc_correlator *corr, const fc_grid *grid2);
int fc_corr_set_grid2_fft(fc_correlator *corr, const double *host_complex);

/* autocorrelate(grid) and cross_correlate(grid1) against grid2
 * (correlator.h:262-268, 372-378).  The _grid forms read a device grid. */
int fc_corr_autocorrelate(fc_correlator *corr, const double *host_grid);
int fc_corr_autocorrelate_grid(fc_correlator *corr, const fc_grid *grid);
int fc_corr_cross_correlate(fc_correlator *corr, const double *host_grid1);
int fc_corr_cross_correlate_grid(fc_correlator *corr, const fc_grid *grid1);

/* Results of the last correlation (correlator.h:80-95).  Any pointer may be
 * NULL.  Histograms are (nrows, nbins) row-major; counts are int32. */
int fc_corr_results(const fc_correlator *corr, double *rbins, int *rcounts,
                    double *rhist, double *kbins, int *kcounts, double *khist,
                    double *zerolag);

typedef struct fc_corr_timings {
  double total_time;     /* seconds of device time per phase, last run */
  double fft_time;
  double ylm_time;
  double multiply_time;
  double extract_time;
  double histogram_time;
  double setup_time;
  int n_fft;             /* cuFFT executions in the last run */
} fc_corr_timings;
int fc_corr_timings_get(const fc_correlator *corr, fc_corr_timings *t);

/* Bytes of device memory a correlator of this configuration holds (grids,
 * subgrids, FFT plans); used for admission by HBM footprint. */
int fc_corr_footprint(int kind, const int shape[3], double cell_size,
                      double rmax, double kmax, int maxell, int precision,
                      size_t *bytes);

/* ---------------------------------------------- asynchronous submission */
/* Binds the correlator's work to an existing CUDA stream (a cudaStream_t
 * passed as void*); NULL restores the correlator's own stream. */
int fc_corr_set_stream(fc_correlator *corr, void *cuda_stream);
/* Enqueue a correlation of a device grid without waiting for it; results
 * are valid after fc_corr_synchronize. */
int fc_corr_autocorrelate_grid_async(fc_correlator *corr, const fc_grid *grid);
int fc_corr_synchronize(fc_correlator *corr);

/* Per-kernel device time of the correlator's launches, for roofline
 * accounting.  Off by default; when on, every launch of the correlator is
 * bracketed by CUDA events on its stream. */
typedef struct fc_kernel_time {
  char name[32];   /* kernel family: weight, r2c, c2r, conj_mul, ksub, ... */
  int launches;    /* launches since profiling was (re)enabled */
  double seconds;  /* summed device time of those launches */
} fc_kernel_time;
int fc_corr_set_profiling(fc_correlator *corr, int enable);
/* Splits a survey correlation's (ell, m) terms (the loop of
 * correlator.h:421-489) over `world` ranks: this correlator computes term i
 * (ell ascending, then m) when i % world == rank, and its histograms and
 * zero lag are that share.  The histograms are linear in the terms, so the
 * sum over ranks is the full result; bin counts are the same on every rank.
 * world 1 (the default) computes every term.  FC_ERR_UNSUPPORTED for a
 * periodic correlator with world > 1. */
int fc_corr_set_term_shard(fc_correlator *corr, int rank, int world);
/* Copies up to max entries; *n receives the number of kernel families. */
int fc_corr_profile(fc_correlator *corr, fc_kernel_time *out, int max, int *n);

/* ------------------------------------------------------ device catalogs */
/* Synthetic catalogs written straight into device memory as (n, 4) FP64
 * x, y, z, w rows, from the counter-based Philox4x32-10 generator keyed by
 * seed.  The reference draws such catalogs with numpy on the host
 * (fftcorr/catalog/random_catalog.py); these have no counterpart in it.
 * Uniform: positions uniform in [lo, hi) per axis, w uniform in
 * [wmin, wmax) (wmin == wmax: constant). */
int fc_catalog_uniform(double *posw_device, int64_t n, const double lo[3],
                       const double hi[3], double wmin, double wmax,
                       uint64_t seed);
/* Clustered periodic box [0, boxsize)^3: ncentres uniform centres, each
 * point a uniformly chosen centre plus an isotropic Gaussian offset of
 * width sigma, wrapped into the box. */
int fc_catalog_clustered_box(double *posw_device, int64_t n, double boxsize,
                             int ncentres, double sigma, double wmin,
                             double wmax, uint64_t seed);
/* Uniform in the volume of the shell sector rmin <= r < rmax, |RA| <= ra_half
 * about +x, |Dec| <= dec_half (radians), observer at the origin; weights
 * times wsign (-1 gives the negated randoms of a D - alpha R grid). */
int fc_catalog_sector(double *posw_device, int64_t n, double rmin, double rmax,
                      double ra_half, double dec_half, double wmin, double wmax,
                      double wsign, uint64_t seed);
/* A catalog described by value, for fc_catalog_generate and the serving
 * form: copied from device or host memory, or generated from a seed. */
enum {
  FC_CAT_DEVICE = 0,          /* posw: device (n, 4) array                 */
  FC_CAT_HOST = 1,            /* posw: host (n, 4) array                   */
  FC_CAT_UNIFORM_BOX = 2,     /* uniform in [0, boxsize)^3                 */
  FC_CAT_CLUSTERED_BOX = 3,   /* as fc_catalog_clustered_box               */
  FC_CAT_SECTOR_UNIFORM = 4,  /* as fc_catalog_sector                      */
  FC_CAT_SECTOR_CLUSTERED = 5 /* ncentres uniform in the sector, each point
                                 a centre plus N(0, sigma^2 I), redrawn until
                                 inside the sector                         */
};
typedef struct fc_catalog_spec {
  int kind;
  int64_t n;
  const double *posw;         /* FC_CAT_DEVICE / FC_CAT_HOST               */
  double boxsize;             /* box kinds                                 */
  int ncentres;
  double sigma;
  double rmin, rmax, ra_half, dec_half;  /* sector kinds (radians)       */
  double wmin, wmax, wsign;   /* weights wsign * U[wmin, wmax)             */
  uint64_t seed;
} fc_catalog_spec;
int fc_catalog_generate(const fc_catalog_spec *spec, double *posw_device);
/* apply_displacement_field (fftcorr/grid/utils.pyx:21-55) on the GPU: out =
 * pos + disp[cell of pos] for n host positions (n, 3), host field (N0, N1,
 * N2, 3).  FC_ERR_INVALID if a position has no cell and periodic_wrap is 0. */
int fc_apply_displacement(const fc_grid *grid, const double *pos, int64_t n,
                          const double *disp, int periodic_wrap, double *out);

/* ---------------------------------------------------------- serving form */
/* A request loop over correlation jobs with continuous batching: `slots`
 * workers each take the first queued job that fits the HBM budget, so jobs
 * arriving while others run start as soon as a slot and memory free up and
 * overlap on the device; grids, assignors and correlators (FFT plans, bin
 * indices) stay resident by configuration and are reused, idle ones evicted
 * least recently used first.  A job is one catalog's run of the reference
 * CLI (cc/fftcorr.cc:233-463): periodic: assign, delta = (rho - mean)/mean,
 * autocorrelate; survey: NN = D - alpha R (alpha = sum w_D / sum w_R, the
 * randoms negated as fftcorr/fftcorr.py:538 does), autocorrelate, and with
 * want_rr also the RR grid.  The grids have the job's precision: FP32 cells
 * for FP32-mixed jobs (fc_grid_create_precision).  Results equal a job run
 * alone.  Has no counterpart in the reference. */
typedef struct fc_job {
  int kind;                 /* FC_PERIODIC or FC_SURVEY                    */
  int shape[3];
  double cell;
  double posmin[3];         /* survey: grid origin (observer at 0)         */
  int scheme, window;
  double rmax, dr, kmax, dk;
  int maxell, precision;
  int want_rr;              /* survey: also correlate RR (for xi)          */
  fc_catalog_spec data;     /* host / device catalogs must stay valid until
                               the job completes                           */
  fc_catalog_spec randoms;  /* survey only                                 */
} fc_job;
typedef struct fc_job_info {
  int state;                /* 0 queued, 1 running, 2 done                 */
  int status;               /* fc_status of a finished job                 */
  double queued_s, run_s, latency_s;  /* submit->start, start->end,
                                         submit->end (host clock)          */
  size_t footprint;         /* admission estimate, bytes                   */
  int nrows, nr, nk, has_rr;
  fc_assign_stats data, randoms;
  double phase_s[8];        /* host time per phase: data catalog, data
                               assignment, random catalog, random
                               assignment, combine / normalise, NN
                               correlate, RR correlate, building resident
                               objects                                     */
  char message[256];        /* error message of a failed job               */
} fc_job_info;
typedef struct fc_server_stats {
  int queued, running, peak_running, resident_objects;
  uint64_t completed, admitted_out_of_order, evictions;
  size_t bytes_resident, bytes_transient, peak_bytes, budget;
} fc_server_stats_t;
typedef struct fc_server fc_server;
int fc_job_init(fc_job *job);
/* Device bytes the job needs (FC_ERR_INVALID for a malformed job). */
int fc_job_footprint(const fc_job *job, size_t *bytes);
/* max_bypass: how many times a waiting job may be passed by later jobs
 * that fit when it does not (0: strict arrival order). */
int fc_server_create(size_t hbm_budget, int slots, int max_bypass,
                     fc_server **out);
/* Waits for running jobs and frees everything. */
int fc_server_destroy(fc_server *server);
/* Queues a job; FC_ERR_ADMISSION if it alone exceeds the budget. */
int fc_server_submit(fc_server *server, const fc_job *job, uint64_t *ticket);
/* Waits up to timeout_s (< 0: forever); *done = 1 when it finished.  A
 * wait that runs out sets *done = 0 and returns FC_ERR_TIMEOUT. */
int fc_server_wait(fc_server *server, uint64_t ticket, double timeout_s,
                   int *done);
int fc_server_job_info(fc_server *server, uint64_t ticket, fc_job_info *info);
/* Tables of a finished job: which 0 = NN (or the periodic grid), 1 = RR;
 * arrays as fc_corr_results.  A failed job returns its status. */
int fc_server_job_results(fc_server *server, uint64_t ticket, int which,
                          double *rbins, int *rcounts, double *rhist,
                          double *kbins, int *kcounts, double *khist,
                          double *zerolag);
/* Forgets a finished job's results. */
int fc_server_release(fc_server *server, uint64_t ticket);
int fc_server_stats(fc_server *server, fc_server_stats_t *stats);

/* ---------------------------------------------------------- batched form */
/* Many periodic boxes taken through mass assignment (periodic wrap), the
 * periodic normalisation delta = (rho - mean) / mean of the reference CLI
 * (cc/fftcorr.cc:369-375) and PeriodicCorrelator::correlate_internal
 * (cc/correlate/correlator.h:273-357), captured once into one CUDA graph.
 * Each box's results equal those of MassAssignor + add_scalar/multiply_by +
 * PeriodicCorrelator run on that box alone (same bits for the same
 * precision).  The reference runs such boxes one at a time; this batch has
 * no counterpart in it. */
typedef struct fc_batch fc_batch;
typedef struct fc_batch_box {
  int shape[3];              /* grid cells per axis                       */
  double cell_size;          /* box edge = shape[i] * cell_size, origin 0 */
  const double *posw_device; /* (n, 4) FP64 x, y, z, w in device memory;
                                must stay allocated and unmoved for the
                                batch's lifetime (the graph reads it)    */
  int64_t n;
} fc_batch_box;
typedef struct fc_batch_params {
  int scheme;      /* distribution scheme (FC_CLOUD_IN_CELL, ...)         */
  int window;      /* window correction of the k-subgrid                  */
  double rmax, dr, kmax, dk;
  int maxell;      /* 0, 2 or 4                                           */
  int precision;   /* FC_FP32_MIXED or FC_FP64                            */
  int lanes;       /* streams of the graph; 0 = from the tuning table     */
  int tune;        /* 1: time candidates for entries missing from the
                      tuning table; 0: use fixed defaults for them        */
} fc_batch_params;
typedef struct fc_batch_info_t {
  int nboxes, lanes, hist_blocks;
  int64_t graph_nodes;       /* nodes of the captured graph               */
  int64_t kernel_nodes;      /* its kernel nodes (cuFFT and CUB included) */
  int64_t own_kernel_nodes;  /* of which this library's own kernels      */
  int64_t hist_items;        /* histogram chunk reductions per replay     */
  int64_t device_bytes;      /* device memory the batch holds             */
} fc_batch_info_t;
int fc_batch_params_default(fc_batch_params *p);
/* Allocates everything, tunes, captures and instantiates the graph. */
int fc_batch_create(const fc_batch_box *boxes, int nboxes,
                    const fc_batch_params *params, fc_batch **out);
int fc_batch_destroy(fc_batch *batch);
/* Replays the graph and waits; seconds = its device time. */
int fc_batch_run(fc_batch *batch, double *seconds);
/* The two halves of fc_batch_run. */
int fc_batch_launch(fc_batch *batch);
int fc_batch_wait(fc_batch *batch, double *seconds);
int fc_batch_info(const fc_batch *batch, fc_batch_info_t *info);
int fc_batch_box_dims(const fc_batch *batch, int box, int *nrows, int *nr,
                      int *nk);
/* The box's tables after a run, as fc_corr_results. */
int fc_batch_results(const fc_batch *batch, int box, double *rbins,
                     int *rcounts, double *rhist, double *kbins, int *kcounts,
                     double *khist, double *zerolag);
/* The box's assignment counters, as fc_assignor_stats (times are 0). */
int fc_batch_box_stats(const fc_batch *batch, int box, fc_assign_stats *s);

/* Launch-tuning table of the batched form (thread and wave counts of the
 * grid-stride kernels per grid size, lane count, histogram CTAs): the
 * library's analogue of FFTW wisdom (fftcorr/fftw/fftw.pyx:3-14), written
 * and read as text lines "kernel precision size a b". */
int fc_tune_export(const char *path);
int fc_tune_import(const char *path);
int fc_tune_forget(void);
int fc_tune_count(int *n);

/* --------------------------------------------------------- HistogramList */
typedef struct fc_hist fc_hist;

/* HistogramList(n, minval, maxval, binsize) (histogram_list.h:12-26). */
int fc_hist_create(int n, double minval, double maxval, double binsize,
                   fc_hist **out);
int fc_hist_destroy(fc_hist *h);
int fc_hist_nbins(const fc_hist *h, int *nbins);
/* accumulate(ih, x, y) over len host values (histogram_list.h:33-45):
 * counts are exact, sums are FP64 in a fixed order. */
int fc_hist_accumulate(fc_hist *h, int ih, const double *x, const double *y,
                       int64_t len);
int fc_hist_reset(fc_hist *h);
/* Copies bins (nbins), counts and hist_values ((n, nbins)). */
int fc_hist_get(const fc_hist *h, double *bins, int *counts, double *hist);

/* ----------------------------------------------- allocation-free variant */
/* Sum and sum of squares of n FP64 values already in device memory, like
 * fc_grid_sum, for callers that cannot allocate device memory: code that
 * runs where cudaMalloc is not allowed (it would synchronise the device or
 * draw on memory the host application reserves for itself).  This entry
 * point allocates nothing: its scratch is a fixed 64 KiB array in the
 * library's own device memory, which every GPU that loads the library holds
 * until the process exits.  n may be at most FC_SUM_STATIC_MAX_N; larger n
 * is rejected with FC_ERR_RANGE.  Every call looks up the scratch address
 * in the current context (a query, no allocation), so make calls outside
 * any stream capture.  The work runs on the legacy default stream: it waits
 * for work the caller queued on blocking streams of the device (so data
 * written there is complete), non-blocking streams are not waited for, and
 * a global-mode stream capture in another thread makes the call fail.  All
 * calls share the one scratch array, so calls that overlap on the GPU (from
 * several host threads) race; this call waits for its result before
 * returning.  Has no counterpart in the reference. */
#define FC_SUM_STATIC_MAX_N (1LL << 30)
int fc_sum_sumsq_static(const double *device_data, int64_t n, double *sum,
                        double *sumsq);

/* ------------------------------------------------------------- utilities */
/* Number of this library's own kernel launches issued so far by the host, in
 * all threads (cuFFT's and CUB's kernels are not included; a replayed CUDA
 * graph counts its kernels when it is captured, not when it is replayed).
 * Has no counterpart in the reference. */
int fc_launch_count(unsigned long long *count);
/* Waits for all work on the current device. */
int fc_device_synchronize(void);
/* Marks the start (on != 0) or end of a region for a profiler started with
 * capture off until the region (cudaProfilerStart / cudaProfilerStop), so a
 * launch list can cover one timed step of a longer run.  Has no counterpart
 * in the reference. */
int fc_profiler_range(int on);
/* Page-locks an existing host range so copies from it run at full PCIe
 * speed (cudaHostRegister), and releases it. */
int fc_host_register(void *ptr, size_t bytes);
int fc_host_unregister(void *ptr);
/* ------------------------------------------------- failure injection */
/* Test hooks.  A planned failure is raised on the host where the real one
 * would surface, before the CUDA or cuFFT call, so no GPU faults.  With
 * FC_FAULT_DEVICE_ALLOC, the n-th device allocation of the library from now
 * fails with FC_ERR_ALLOC.  With FC_FAULT_FFT_PLAN, the n-th cuFFT plan
 * creation fails with FC_ERR_CUFFT.  n <= 0 disarms.  The reference fails
 * the same way on an allocation or an FFTW plan that cannot be made
 * (cc/grid/fft_grid.cc:126,153). */
enum { FC_FAULT_DEVICE_ALLOC = 1, FC_FAULT_FFT_PLAN = 2 };
int fc_fault_inject(int kind, int64_t n);
/* Caps the device bytes the library's own allocations may hold (0: no cap).
 * An allocation past the cap fails with FC_ERR_ALLOC. */
int fc_set_device_budget(size_t bytes);
/* Device bytes the library's allocations hold now. */
int fc_device_bytes(size_t *bytes);

/* Plain device allocations for callers that stage inputs themselves. */
int fc_device_malloc(size_t bytes, void **ptr);
int fc_device_free(void *ptr);
int fc_memcpy_htod(void *dst, const void *src, size_t bytes);
int fc_memcpy_dtoh(void *dst, const void *src, size_t bytes);
/* Free and total device memory (cudaMemGetInfo). */
int fc_device_memory(size_t *free_bytes, size_t *total_bytes);
/* Device-timeline stopwatch: start and stop synchronise the device and
 * record an event on the default stream, so the interval covers all work
 * issued in between on any stream. */
typedef struct fc_timer fc_timer;
int fc_timer_create(fc_timer **t);
int fc_timer_start(fc_timer *t);
int fc_timer_stop(fc_timer *t, double *seconds);
int fc_timer_destroy(fc_timer *t);

#ifdef __cplusplus
}
#endif

#endif /* FC_API_H */

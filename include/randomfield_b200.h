/*
 * randomfield_b200.h -- C-ABI of the B200-native spectral-sum random-field
 * generator (the randomFieldND Shinozuka / isotropic path of
 * cottereau/randomField).
 *
 * Plain C types only: pointers, sizes, doubles.  Layouts are Fortran
 * column-major, as the reference's callers hold them:
 *   xPoints   nDim x n   (the coordinates of one point are contiguous)
 *   randField n x Nmc    (one realization is contiguous)
 * The caller allocates everything; the library never frees caller memory.
 * Every entry point returns RF_OK (0) or a negative RF_E* code and never
 * aborts or exits; rf_last_error() gives a one-line reason (thread-local).
 */
#ifndef RANDOMFIELD_B200_H
#define RANDOMFIELD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RF_ABI_VERSION 1

/* Methods, correlation models and marginals: constants_RF.f90:12-21. */
#define RF_ISOTROPIC 1
#define RF_SHINOZUKA 2
#define RF_RANDOMIZATION 3  /* Shinozuka sum over uniformly random wavevectors (randomFieldND.f90:343-361) */
#define RF_FFT 4            /* spectral DCT on a structured grid: rf_generate_fft_grid (randomFieldND.f90:520-763) */
#define RF_CM_GAUSSIAN 1
#define RF_CM_COS 2
#define RF_FOM_GAUSSIAN 1
#define RF_FOM_LOGNORMAL 2

/* Precision forms of the contraction. */
#define RF_PREC_BF16 0      /* BF16 operands on tcgen05 (default): hi/lo BF16 amplitude rows where a trig tile is
                               generated, TF32 on the high-variance K-steps of the outer-group contraction */
#define RF_PREC_FP16 1      /* FP16 trig tiles and scaled FP16 amplitude side, tcgen05     */
#define RF_PREC_FP32 2      /* plain FP32 operands on the FFMA pipes                       */
#define RF_PREC_BF16_FAST 3 /* BF16 trig tiles, single BF16 amplitude side, tcgen05        */
#define RF_PREC_FP8 4       /* FP8 e4m3 trig tiles, hi/lo e4m3 amplitude side, tcgen05 kind::f8f6f4;
                               a stated option: relative-L2 error about 3e-2                */

/* Status codes.  The reference stops or calls MPI_ABORT instead. */
#define RF_OK 0
#define RF_EINVAL_NMC -1        /* Nmc < 1                     (type_inputRF.f90:1159-1206) */
#define RF_EINVAL_NDIM -2       /* nDim outside 1..3, or < 2 for isotropic                   */
#define RF_EINVAL_CORRL -3      /* corrL(i) <= 0               (type_inputRF.f90:1159-1206) */
#define RF_EINVAL_LOGNORMAL -4  /* lognormal with fieldAvg <= 0 (randomFieldND.f90:162-166) */
#define RF_EINVAL_METHOD -5     /* method not 1, 2 or 3                                     */
#define RF_EINVAL_CORRMOD -6    /* corrMod not 1 or 2; cm_COS with 6 or fewer wavevectors    */
#define RF_EINVAL_MARGINAL -7   /* margiFirst not 1 or 2                                    */
#define RF_EINVAL_RANGE -8      /* zero extent along an axis (kDelta would be infinite)      */
#define RF_EINVAL_ARG -9        /* null pointer, n < 1, bad option value                     */
#define RF_ENOTSUP -10          /* valid request outside what this build implements          */
#define RF_ECUDA -20            /* CUDA runtime error                                       */
#define RF_ENOMEM -21           /* device or pinned allocation failed                       */
#define RF_ETIMEDOUT -22        /* a bounded device wait expired; the kernel returned        */
#define RF_ENOMEM_ADMISSION -23 /* request larger than the context's HBM budget              */
#define RF_ESCRATCH -24         /* request larger than rf_generate_device_noalloc's scratch */
#define RF_ENODEV -25           /* no CUDA device                                           */
#define RF_EBOUNDS -26          /* a device index check failed (RF_DEBUG_BOUNDS build only)  */

/*
 * Options.  Zero-initialise (or call rf_options_init) and set what differs;
 * a NULL options pointer means all defaults.
 */
typedef struct rf_options {
  int32_t size;          /* sizeof(rf_options); set by rf_options_init                 */
  int32_t precision;     /* RF_PREC_*                                                   */
  int64_t seed_start;    /* the reference's seedStart (>= 0); rnglib generator 1 seeded */
                         /* with (72 + 18 s, 72 + 18 s + 37), after math_RF.f90:561     */
  int32_t k_nstep[3];    /* Shinozuka: wavenumbers per axis; 0 = reference rule         */
                         /* kNStep = 1 + ceil(kMax / (2 pi / (1.1 xRange))) (spectra_RF.f90:87-92) */
  int32_t iso_n_radial;  /* isotropic: radial points; 0 = 1 + 5 ceil(kMax/kDelta) (:75-80) */
  int32_t iso_n_dir;     /* isotropic: directions per radius; 0 = 32                    */
  int32_t literal;       /* 1: reproduce the reference's deterministic defects B1/B2    */
  int32_t normalize;     /* 1: empirical per-realization normalisation (randomFieldND.f90:820-926) */
  double x_range[3];     /* physical extent per axis; 0 = extent of xPoints             */
  int32_t device;        /* CUDA device ordinal                                         */
  int32_t reserved0;
  /* Optional caller-supplied uniform draws in [0, 1) that replace the rnglib
   * stream: draw p (1-based) of the request is draws[p - 1].  The order is the
   * reference's sequence of random_number calls for the method:
   *   Shinozuka: per realization, K phases in k order (randomFieldND.f90:278)
   *   randomization: nDim * kn base-wavevector draws, axis fastest
   *     (spectra_RF.f90:119-124), then the Shinozuka phases
   *   isotropic: the phi block (3-D only) and the theta block of K draws, then
   *     per realization a gamma block and a psi block of K (:460-468).
   * n_draws must cover every draw the request makes (RF_EINVAL_ARG if not).
   * Host memory.  rf_create_standard_gaussian_field_unstruct and
   * rf_generate_device take it; the batch, serving, blend, grid and
   * no-allocation entry points return RF_ENOTSUP.  NULL: rnglib. */
  const double* draws;
  int64_t n_draws;
  int32_t reserved[2];
} rf_options;

/* Fills defaults: BF16 form, seed_start 0, reference rules, device 0. */
void rf_options_init(rf_options* opt);

/*
 * The drop-in for createStandardGaussianFieldUnstruct(xPoints, corrMod,
 * margiFirst, corrL, fieldAvg, fieldVar, Nmc, method, randField)
 * (README.md:58-92; in code create_RF_Unstruct_Init, randomFieldND.f90:27-38,
 * reached through interface createRandomField, calls_RF.f90:20-22, with
 * gen_Std_Gauss_* :44-132/:184-337/:368-514 and multiVariateTransformation
 * :139-178).  Host buffers; synchronous; the result is FP64 as in the
 * reference.  corrL has nDim entries.
 */
int rf_create_standard_gaussian_field_unstruct(
    const double* xPoints, int nDim, int64_t n, int corrMod, int margiFirst,
    const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method,
    double* randField, const rf_options* opt);

/*
 * Device-resident form of the same call for callers that keep data on the
 * GPU: d_xPoints and d_randField are device pointers; the work is queued on
 * `stream` (a cudaStream_t, 0 = legacy default) and the call returns once it
 * is queued.  The context owns device tables and scratch; one context per
 * host thread (calls on one context are serialised by its stream).
 */
typedef struct rf_context rf_context;
int rf_context_create(int device, rf_context** out);
int rf_context_destroy(rf_context* ctx);
int rf_generate_device(rf_context* ctx, const double* d_xPoints, int nDim, int64_t n,
                       int corrMod, int margiFirst, const double* corrL,
                       double fieldAvg, double fieldVar, int Nmc, int method,
                       double* d_randField, const rf_options* opt, void* stream);
/*
 * Allocation-free variant of rf_generate_device.  No counterpart in the
 * reference (which allocates its work arrays itself); it exists for callers
 * that must not allocate device memory while generating: applications whose
 * allocator (a caching pool, an OpenACC or CUDA Fortran runtime) owns and has
 * reserved nearly all device memory, or latency-critical loops that cannot
 * afford cudaMalloc's implicit synchronisation.  The caller passes device
 * buffers for the points and the field; all other working memory is one
 * fixed 32 MiB device array per GPU, placed by the CUDA runtime on every
 * device where the library is loaded and held until the process exits.
 * Requests whose tables do not fit it fail with RF_ESCRATCH.  The first call
 * on a device resolves the array's address (cudaGetSymbolAddress) and should
 * come before any stream capture on that device.  All calls share the array:
 * calls whose work overlaps on the GPU race, so serialise them.  Runs on
 * opt->device on `stream` (0 = legacy default) and returns when the field is
 * complete: it synchronises `stream` before returning (and once more after
 * the extent pass when the point extent is needed).  Allocates nothing (no
 * cudaMalloc, cudaFree or context).
 */
int rf_generate_device_noalloc(const double* d_xPoints, int nDim, int64_t n, int corrMod, int margiFirst,
                               const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method,
                               double* d_randField, const rf_options* opt, void* stream);

/* Waits for the context's queued work; reports a device-side timeout. */
int rf_context_synchronize(rf_context* ctx);

/* Failure-detection self test: launches a kernel whose bounded device wait
 * (the waits every generation kernel uses) can never complete, on a phase
 * nothing arrives on; after limit_ms the kernel raises the context's error
 * word and returns, and the call reports RF_ETIMEDOUT, as a generation whose
 * wait expired would.  No fault, trap or hang; the context stays usable. */
int rf_context_selftest_timeout(rf_context* ctx, double limit_ms);

/* Self test of the index checks of the RF_DEBUG_BOUNDS build (the library
 * compiled with -DRF_DEBUG_BOUNDS, librf_b200_bounds.so): a kernel computes an
 * index one past a buffer, its check records the failure in the context's
 * error word and skips the access, and the call reports RF_EBOUNDS; the
 * context stays usable.  The normal build returns RF_ENOTSUP and launches
 * nothing. */
int rf_context_selftest_bounds(rf_context* ctx);
/* 1 in the RF_DEBUG_BOUNDS build, 0 otherwise. */
int rf_debug_bounds_build(void);

/* Measured MUFU (sin, cos) pair rate of the device: the SFU bound of the
 * GEN_TABLE generator (one pair per point and wavevector). */
int rf_measure_sfu_rate(int device, double* pairs_per_second);

/*
 * Debug export of the device table builder's rnglib draws (the random_number
 * calls of randomFieldND.f90:278 and :460-468, drawn from rnglib generator 1,
 * RANDLIB/rnglib.f90:548-659), for a bit-exact comparison with a sequential
 * rnglib run.  The request is described without points: opt->k_nstep (or
 * opt->iso_n_radial) or opt->x_range must fix the wavevector count.  Writes
 * *K_out = K; with draws non-NULL also draws[(r * K + k) * D + j], the i4_uni
 * values the builder consumed for realization r and wavevector k in
 * reference order (D = 1: the phase; isotropic D = 2: gamma, psi), and for
 * the isotropic method k_draws[2 k + j] (theta, then phi in 3-D; 0 in 2-D).
 * Uses the same realization blocks as a generation with opt->precision.
 */
int rf_debug_table_draws(int nDim, int method, int Nmc, const rf_options* opt, int64_t* K_out, int32_t* draws,
                         int64_t draws_capacity, int32_t* k_draws, int64_t k_capacity);

/*
 * Field statistics on the device (statistics_RF.f90), for a field already in
 * device memory (rf_generate_device, rf_generate_batch_device): no copy of
 * the field to the host.
 *   - per realization r: mean and standard deviation over the n points
 *     (calculate_average_and_stdVar_MPI, statistics_RF.f90:18-174, "by
 *     event"), and their global values over all n * Nmc values;
 *   - with a structured grid (xNStep, axis 1 fastest, n = prod xNStep): the
 *     directional correlation of realization 1 normalised by the global mean
 *     and deviation, lags 0 .. xNStep_d / 2 - 1 per axis (rebuild_Sk_FFT and
 *     rebuild_Sk, :180-419: |FFT|^2 averaged over the lines, inverse FFT;
 *     here the same circular autocorrelation summed directly), and the
 *     correlation-length estimate 2 (sum R - (R_0 + R_last) / 2) xStep_d
 *     (rebuild_corrL, :425-443).
 * d_randField is n x Nmc column-major (FP64).  evnt_avg / evnt_std (host,
 * Nmc entries each) may be null; with xNStep null only the moments are
 * computed.  sk (host, sum_d xNStep_d / 2 entries, axis 1 first) and corrL_out
 * (host, nDim entries) may be null.  Axis lengths above 4096 give RF_ENOTSUP.
 * Runs on the context's stream and returns when the results are on the host.
 * Sums are formed in FP64 in a fixed order: repeated calls give identical
 * results.
 */
typedef struct rf_field_stats {
  double global_avg;
  double global_std;
  int64_t n;
  int32_t Nmc, nDim;
} rf_field_stats;

int rf_field_statistics(rf_context* ctx, const double* d_randField, int64_t n, int Nmc, int nDim,
                        const int64_t* xNStep, const double* xStep, double* evnt_avg, double* evnt_std,
                        double* sk, double* corrL_out, rf_field_stats* out);

/*
 * The FFT method (method 4; gen_Std_Gauss_FFT, randomFieldND.f90:520-763),
 * which the reference runs on a structured mesh only: the grid has xNStep[d]
 * points spaced xStep[d] along axis d (nDim 2 or 3, axis 1 fastest, 2 to
 * 2048 points per axis).  Random amplitudes on the k grid of set_kPoints'
 * FFT branch (spectra_RF.f90:135-160), the multi-dimensional DCT-III of
 * FFTW's REDFT01 with the reference's scale, then the marginal map.  The
 * reference fills realization 1 only; realization r here uses the rnglib
 * stream of seed_start + r, so realization 1 is the reference's.
 * d_randField (device) is prod(xNStep) x Nmc column-major.  Returns when
 * the field is complete.
 */
int rf_generate_fft_grid(rf_context* ctx, int nDim, const int64_t* xNStep, const double* xStep, int corrMod,
                         int margiFirst, const double* corrL, double fieldAvg, double fieldVar, int Nmc,
                         double* d_randField, const rf_options* opt);

/*
 * The Shinozuka field (method 2) on a structured grid: the points
 * x_d = xMin[d] + j xStep[d], j < xNStep[d], axis 1 fastest (setGrid,
 * math_RF.f90:16-92, as set_XPoints builds them, mesh_RF.f90:17-64), the
 * same field that rf_generate_device computes when given those points in
 * that order (same wavevectors, phases, extent rule and marginal map; the
 * extent is max - min of the coordinates).  Because both the wavevectors
 * and the points are tensor grids, the sum is evaluated axis by axis in
 * FP64 (n1 n2 n3 N3 + n1 n2 N2 N3 + n1 N1 N2 N3 work per realization
 * instead of 4 n1 n2 n3 N1 N2 N3), so the result matches the reference's
 * FP64 sum to rounding whatever opt->precision says.  Limits: method 2, at
 * most 32 wavenumbers per axis, no literal mode (RF_ENOTSUP otherwise:
 * rf_generate_device covers those).  d_randField (device) is
 * prod(xNStep) x Nmc column-major; queued on `stream` (0 = the context's).
 */
int rf_generate_grid(rf_context* ctx, int nDim, const double* xMin, const double* xStep, const int64_t* xNStep,
                     int corrMod, int margiFirst, const double* corrL, double fieldAvg, double fieldVar, int Nmc,
                     int method, double* d_randField, const rf_options* opt, void* stream);
/*
 * Host-buffer form of rf_generate_grid, the structured counterpart of
 * rf_create_standard_gaussian_field_unstruct for callers that would build
 * xPoints with set_XPoints: randField is a host array of prod(xNStep) x Nmc
 * doubles, column-major.  Runs on opt->device's default context and returns
 * when randField is filled.
 */
int rf_create_standard_gaussian_field_grid(int nDim, const double* xMin, const double* xStep, const int64_t* xNStep,
                                           int corrMod, int margiFirst, const double* corrL, double fieldAvg,
                                           double fieldVar, int Nmc, int method, double* randField,
                                           const rf_options* opt);

/*
 * Result files (writeResultFile_RF.f90: write_MONO_proc_result :737-829,
 * write_XMF_Elements :835-938, write_HDF5_attributes :1758-1849).  Writes
 * <folder>/h5/<fileName>.h5 with the dataset "samples": one realization
 * (host array, axis 1 fastest) on the structured grid of
 * nint((xMax - xMin)/xStep) + 1 points per axis, stored with the slowest axis
 * first as the reference's files are; with `attr` non-NULL the run's
 * parameters become attributes of the file's root group (integer scalars,
 * and vectors of nDim entries).  For nDim 2 and 3 it also writes
 * <folder>/xmf/<fileName>.xmf, the XDMF 2.0 description the reference writes
 * (CoRectMesh, origin, step, node-centred scalar RF1 read from
 * ../h5/<fileName>.h5:/samples).  The h5 and xmf folders are created when
 * missing.  The HDF5 file is written without an HDF5 library, in the
 * format's oldest layout (superblock version 0).  Host only: needs no GPU.
 */
typedef struct rf_result_attributes {
  int32_t nb_procs, nDim, Nmc, method, seedStart, corrMod, margiFirst, localizationLevel;
  int32_t kNStep[3], nFields[3];
  double xMinGlob[3], xMaxGlob[3], xStep[3], corrL[3], overlap[3], procExtent[3], kMax_out[3];
} rf_result_attributes;
int rf_write_result_grid(const char* folder, const char* fileName, int nDim, const double* xMin, const double* xMax,
                         const double* xStep, const double* field, const rf_result_attributes* attr);

/* Phase timers.  With timing enabled the context records CUDA events on the
 * launching stream around each phase of a generation; rf_context_last_times
 * waits for the last one and returns the device milliseconds of the table
 * build, the contraction (with its fused epilogue) and the optional
 * normalisation pass, and how many kernels the call launched. */
int rf_context_set_timing(rf_context* ctx, int enable);
int rf_context_last_times(rf_context* ctx, double* tables_ms, double* contract_ms, double* post_ms,
                          int32_t* kernel_launches);

/*
 * Batches.  No counterpart in the reference, whose driver (sample_RF.f90,
 * single_realization :348) generates one field per call; these entry points
 * generate many independent requests in one grouped launch: a persistent
 * tcgen05 kernel whose CTAs run (request realization block, 128-point tile)
 * work items of all requests, balanced across the SMs, replayed from a
 * captured CUDA graph.  Each request carries the arguments of
 * rf_create_standard_gaussian_field_unstruct; its field equals the single-call
 * field within the precision form's tolerance.  Tensor-core forms only (the
 * plain FP32 form runs request by request); literal mode is not supported in
 * a batch (RF_ENOTSUP).  The realization block of the grouped launch is
 * chosen by a tuner on the first batch of each precision form (every
 * candidate computes the same field).
 */
typedef struct rf_request {
  const double* xPoints;  /* nDim x n: host memory (rf_generate_batch) or device memory (_device) */
  double* randField;      /* n x Nmc, the same kind of memory */
  int64_t n;
  int32_t nDim, corrMod, margiFirst, Nmc, method;
  int32_t reserved0;
  double corrL[3];
  double fieldAvg, fieldVar;
  rf_options opt;         /* precision and device must agree across a batch */
} rf_request;

typedef struct rf_batch_stats {
  double tables_ms;           /* device time of the grouped table build */
  double contract_ms;         /* device time of the grouped contraction */
  int64_t units;              /* realization blocks of all requests */
  int64_t work_items;         /* (unit, tile) items */
  int32_t realization_block;  /* chosen by the tuner */
  int32_t stages;             /* pipeline depth of the grouped kernel */
  int32_t graph_replayed;     /* 1: the launch replayed a captured CUDA graph */
  int32_t tuned;              /* 1: this call ran the tuner */
  int32_t outer_stages;       /* pipeline depth of the outer-group kernel (0: not launched) */
  int32_t tune_candidates;    /* configurations the tuner timed for this batch class */
  double tune_default_ms;     /* the default configuration's time in the tuner's search */
  double tune_best_ms;        /* the chosen configuration's time in the tuner's search */
} rf_batch_stats;

/* Host buffers; returns when every field has been copied back. */
int rf_generate_batch(rf_context* ctx, const rf_request* reqs, int32_t count);
/* Device buffers; queued on `stream` (0 = the context's stream). */
int rf_generate_batch_device(rf_context* ctx, const rf_request* reqs, int32_t count, void* stream);
/* Statistics of the last batch on the context (waits for it). */
int rf_batch_last_stats(rf_context* ctx, rf_batch_stats* out);

/*
 * Localization blend (localization_RF.f90:199-263, 705-857; calls_RF.f90:
 * 209-213, 324-369; topography_RF.f90:49-52): one field on a structured group
 * grid assembled from nFields[0] x nFields[1] x nFields[2] overlapping
 * subdomains.  The overlap (units of corrL) is rounded to the grid as the
 * reference does; overlapNPoints = nint((overlap*corrL - 2*xStep)/xStep) + 1
 * points are shared by neighbouring subdomains, each of
 * (xNStep + (nFields-1)*overlapNPoints)/nFields points per axis (this must be
 * an integer: rf_blend_layout reports the subdomain size or RF_EINVAL_RANGE).
 * Subdomain f (fieldNumber 1.., axis 1 fastest) is generated with seed
 * seed_start + fieldNumber (sample_RF.f90:311) on its own grid, multiplied by
 * its cosine partition of unity (all faces ramped) and added into the group
 * field in the grouped launch's epilogue; the group's border faces are then
 * divided by the group's partition (border correction) and the marginal map
 * applied.  randField is xNStep[0]*xNStep[1]*xNStep[2] x Nmc, axis 1 fastest.
 * Tensor-core forms only; the border correction applies to every
 * realization (the reference corrects column 1 only).
 */
typedef struct rf_blend_grid {
  int32_t nDim;
  int32_t xNStep[3];   /* group grid points per axis */
  int32_t nFields[3];  /* subdomains per axis */
  int32_t reserved0;
  double xMin[3];
  double xStep[3];
  double overlap;      /* in units of corrL (the reference's IPT%overlap) */
  int32_t reserved[8];
} rf_blend_grid;
/* Subdomain points per axis and overlapNPoints per axis of a blend grid. */
int rf_blend_layout(const rf_blend_grid* grid, const double* corrL, int32_t* subNStep, int32_t* overlapNPoints);
/* Host randField; returns when it is filled. */
int rf_generate_blended(rf_context* ctx, const rf_blend_grid* grid, int corrMod, int margiFirst, const double* corrL,
                        double fieldAvg, double fieldVar, int Nmc, int method, double* randField,
                        const rf_options* opt);
/* Device randField, queued on `stream` (0 = the context's stream). */
int rf_generate_blended_device(rf_context* ctx, const rf_blend_grid* grid, int corrMod, int margiFirst,
                               const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method,
                               double* d_randField, const rf_options* opt, void* stream);

/*
 * Serving loop.  No counterpart in the reference.  A server owns a worker
 * thread and two batch slots (each a context with its own stream): requests
 * submitted from any thread queue in FIFO order; the worker admits queued
 * requests into a free slot while their device footprint (points, field,
 * operands) fits the slot's share of the HBM budget, launches the slot's
 * grouped batch, and admits the next arrivals into the other slot while the
 * first runs (continuous batching: a request waits for at most the batch in
 * flight).  Points are copied in and fields out through pinned staging, so a
 * request's host buffers must stay valid until rf_server_wait returns.
 * Latency is measured from rf_server_submit to the field being in the
 * caller's buffer.  A request larger than a slot's share fails with
 * RF_ENOMEM_ADMISSION.  The result of a request does not depend on the
 * requests batched with it (each request's tables come from its own seed).
 */
typedef struct rf_server rf_server;
typedef struct rf_server_config {
  int32_t size;              /* sizeof(rf_server_config) */
  int32_t device;
  int32_t precision;         /* RF_PREC_BF16 / FP16 / BF16_FAST */
  int32_t max_batch;         /* requests per grouped launch (0: 512) */
  int64_t hbm_budget_bytes;  /* device memory for requests in flight (0: half the free memory) */
  int32_t reserved[8];
} rf_server_config;
typedef struct rf_server_stats {
  int64_t submitted, completed, failed, batches;
  int64_t admission_waits;   /* batches closed early because the budget was full */
  int64_t peak_bytes;        /* largest footprint admitted to one slot */
  double field_values;       /* sum of n * Nmc over completed requests */
  double busy_ms;            /* device time of the grouped launches */
  double p50_ms, p99_ms, max_ms, mean_ms;  /* submit -> field in the caller's buffer */
} rf_server_stats;

void rf_server_config_init(rf_server_config* cfg);
int rf_server_create(const rf_server_config* cfg, rf_server** out);
/* Queues a request (host buffers); *ticket identifies it for rf_server_wait. */
int rf_server_submit(rf_server* srv, const rf_request* req, int64_t* ticket);
/* Queues a localization blend (rf_generate_blended's arguments, host randField). */
int rf_server_submit_blended(rf_server* srv, const rf_blend_grid* grid, int corrMod, int margiFirst,
                             const double* corrL, double fieldAvg, double fieldVar, int Nmc, int method,
                             double* randField, const rf_options* opt, int64_t* ticket);
/* Waits (timeout_s < 0: forever) for a request; returns its status
 * (RF_ETIMEDOUT when the wait timed out) and its latency in milliseconds. */
int rf_server_wait(rf_server* srv, int64_t ticket, double timeout_s, double* latency_ms);
int rf_server_get_stats(rf_server* srv, rf_server_stats* out);
/* Drains the queue, stops the worker and frees the server. */
int rf_server_destroy(rf_server* srv);

/* Problem geometry exactly as the generator will use it (host only, no GPU):
 * K wavevectors, kNStep, kDelta, ampMult (randomFieldND.f90:260-266). */
int rf_query_geometry(const double* xPoints, int nDim, int64_t n, int corrMod,
                      const double* corrL, int method, const rf_options* opt,
                      int64_t* K, int32_t* kNStep, double* kDelta, double* ampMult);

/* One-line reason for the last error on this thread ("" when none). */
const char* rf_last_error(void);
/* RF_ABI_VERSION of the loaded library. */
int rf_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* RANDOMFIELD_B200_H */

/*
 * rf_oracle.h -- FP64 CPU restatement of the randomField spectral-sum path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product
 * in randomfield_b200/: only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load it.  The product never links, includes or
 * calls anything here.
 *
 * Parity status: the reference (cottereau/randomField, Fortran 90 + MPI +
 * HDF5 + FFTW) ships no golden vectors, known-answer tests or fixtures for
 * this path, and cannot be compiled in this environment (no Fortran
 * compiler).  Parity is therefore UNPINNED against reference output; the
 * restatement is pinned instead by (1) rnglib recurrences cross-checked in
 * 64-bit arithmetic, (2) closed-form known answers (cm_COS single term,
 * single wavenumber), (3) the ensemble variance of the discrete spectral sum
 * and (4) internal identities (direct sum == contraction recast).
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef RF_ORACLE_H
#define RF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* constants_RF.f90:5  PI exactly as the reference spells it */
#define RFO_PI 3.1415926535898
/* constants_RF.f90:12-21 */
#define RFO_ISOTROPIC 1
#define RFO_SHINOZUKA 2
#define RFO_RANDOMIZATION 3
#define RFO_CM_GAUSSIAN 1
#define RFO_CM_COS 2
#define RFO_FOM_GAUSSIAN 1
#define RFO_FOM_LOGNORMAL 2

/* Error codes shared in meaning with the product C-ABI. */
#define RFO_OK 0
#define RFO_EINVAL -1

/* ---- rnglib.f90 (L'Ecuyer-Cote combined MLCG, 32 generators) ----------- */
typedef struct rfo_rnglib {
  int32_t ig1[32], ig2[32];   /* initial seeds   (ig_memory)  */
  int32_t lg1[32], lg2[32];   /* last seeds      (lg_memory)  */
  int32_t cg1[32], cg2[32];   /* current seeds   (cg_memory)  */
  int32_t anti[32];           /* antithetic flags             */
  int32_t g;                  /* current generator, 1-based   */
  int32_t initialized;
} rfo_rnglib;

int32_t rfo_multmod(int32_t a, int32_t s, int32_t m);            /* rnglib.f90:1238-1396 */
void    rfo_rng_initialize(rfo_rnglib* r);                       /* rnglib.f90:909-975   */
void    rfo_rng_set_initial_seed(rfo_rnglib* r, int32_t ig1, int32_t ig2); /* :1521-1622 */
void    rfo_rng_init_generator(rfo_rnglib* r, int32_t t);        /* rnglib.f90:804-908   */
void    rfo_rng_advance_state(rfo_rnglib* r, int32_t k);         /* rnglib.f90:3-91      */
void    rfo_rng_cgn_set(rfo_rnglib* r, int32_t g);               /* rnglib.f90:457-489   */
int32_t rfo_rng_i4_uni(rfo_rnglib* r);                           /* rnglib.f90:548-659   */
double  rfo_rng_r8_uni_01(rfo_rnglib* r);                        /* rnglib.f90:1459-1520 */
/* `count` successive i4_uni calls into out[0..count) (the sequential stream). */
void    rfo_rng_i4_stream(rfo_rnglib* r, int64_t count, int32_t* out);
/* Seed words from seedStart, after math_RF.f90:561 (72 + 18*seedStart + 37*(i-1)). */
void    rfo_seed_words(int64_t seedStart, int32_t* ig1, int32_t* ig2);
/* initialize + set_initial_seed(seed words); generator 1 current. */
int32_t rfo_rng_seed(rfo_rnglib* r, int64_t seedStart);

/* ---- request ------------------------------------------------------------ */
typedef struct rfo_request {
  int32_t nDim;            /* 1..3                                       */
  int64_t n;               /* number of points                          */
  const double* xPoints;   /* nDim x n, Fortran column-major            */
  int32_t corrMod;         /* RFO_CM_*                                  */
  int32_t margiFirst;      /* RFO_FOM_*                                 */
  double corrL[3];
  double fieldAvg, fieldVar;
  int32_t Nmc;
  int32_t method;          /* RFO_ISOTROPIC / RFO_SHINOZUKA             */
  int64_t seedStart;       /* >= 0                                      */
  int32_t kNStep[3];       /* Shinozuka wavenumbers per axis, 0 = rule  */
  int32_t isoNRadial;      /* isotropic radial points, 0 = rule         */
  int32_t isoNDir;         /* isotropic directions per radius, 0 = 32   */
  int32_t literal;         /* 1: reproduce the reference's B1/B2 bugs   */
  int32_t normalize;       /* 1: empirical per-realization normalisation */
  double xRange[3];        /* physical extent per axis, 0 = from points */
} rfo_request;

typedef struct rfo_geometry {
  int32_t nDim;
  int64_t K;               /* number of wavevectors                      */
  int32_t kNStep[3];       /* Shinozuka: per axis; isotropic: [0]=n_r, [1]=n_dir */
  double kDelta[3];        /* Shinozuka: per axis; isotropic: [0]=dr     */
  double kMax;
  double ampMult;          /* Shinozuka overall factor (randomFieldND.f90:265) */
  double xRangeNorm[3];    /* extent / corrL                             */
  int64_t xSlab;           /* literal-mode slab rows (randomFieldND.f90:237) */
} rfo_geometry;

/* Validation rules of type_inputRF.f90:1159-1206 and randomFieldND.f90:162. */
int32_t rfo_validate(const rfo_request* rq);
/* set_kMaxND / set_kPoints sizes (spectra_RF.f90:15-44, :50-133). */
int32_t rfo_geometry_of(const rfo_request* rq, rfo_geometry* g);
/* kPoints (nDim x K column-major) and the per-k amplitude (Shinozuka: sqrt(S_k);
 * isotropic: A_k of the intended amplitude).  S written too (may be NULL). */
int32_t rfo_kpoints(const rfo_request* rq, double* kPoints, double* amp, double* S);
/* Contraction operand: Bc[k + K*r] = amp*gamma*cos(phi), Bs = -amp*gamma*sin(phi). */
int32_t rfo_phase_matrix(const rfo_request* rq, double* Bc, double* Bs);
/* Full path: standard field, optional normalisation, marginal transform.
 * randField n x Nmc column-major.  rows==NULL: all points; else only the listed
 * rows are computed and written compactly (nrows x Nmc).  Tables and xRange
 * always come from the full request.  nthreads<=0: OpenMP default. */
int32_t rfo_generate(const rfo_request* rq, const int64_t* rows, int64_t nrows,
                     double* out, int32_t nthreads);
/* Same standard field through the recast sum_k cos(k.x)Bc + sin(k.x)Bs (FP64). */
int32_t rfo_generate_recast(const rfo_request* rq, const int64_t* rows, int64_t nrows,
                            double* out, int32_t nthreads);
/* multiVariateTransformation (randomFieldND.f90:139-178), in place. */
int32_t rfo_marginal(int32_t margiFirst, double fieldAvg, double fieldVar,
                     double* f, int64_t count);
/* normalize_randField (randomFieldND.f90:820-926) over the given columns. */
void    rfo_normalize(double* f, int64_t n, int32_t ncols);
/* setGrid, axis 1 fastest (math_RF.f90:16-92). */
void    rfo_set_grid(int32_t nDim, const double* xMin, const double* xStep,
                     const int32_t* xNStep, double* xPoints);

/* ---- localization blend ------------------------------------------------- */
/* generateUnityPartition_Matrix (localization_RF.f90:705-857), cosine taper.
 * faceMask bit (2*d + j) set => taper face j (0 low, 1 high) of axis d. */
void    rfo_unity_partition(int32_t nDim, const int32_t* xNStep,
                            const int32_t* overlapNPoints, uint32_t faceMask,
                            double* up);
/* overlapNPoints = nint((overlap*corrL - 2*xStep)/xStep) + 1 (localization_RF.f90:746) */
int32_t rfo_overlap_npoints(double overlap, double corrL, double xStep);

/* ---- CPU baseline: the reference's slab/DGEMM/cos/GEMV structure ------- */
/* gen_Std_Gauss_Shinozuka hot loop (randomFieldND.f90:276-328) with the
 * Netlib DGEMM loop orders (BLAS/dgemm.f90:218-256), for rows [row0,row0+nrows)
 * and realizations [r0, r0+nr); writes out (nrows x nr col-major) before the
 * marginal map.  Returns elapsed seconds (<0 on error). */
double  rfo_baseline_shinozuka(const rfo_request* rq, int64_t row0, int64_t nrows,
                               int32_t r0, int32_t nr, double* out, int32_t nthreads);

#ifdef __cplusplus
}
#endif
#endif

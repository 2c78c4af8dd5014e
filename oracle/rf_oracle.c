/*
 * rf_oracle.c -- FP64 CPU restatement of the randomField spectral-sum path.
 *
 * TEST INFRASTRUCTURE ONLY (see rf_oracle.h): the checker for the CUDA
 * product, never linked by it.  Parity against reference output is
 * unpinned: the reference ships no golden vectors and its Fortran sources
 * cannot be compiled here.  Citations are path:line inside the reference
 * project (cottereau/randomField).
 */
#include "rf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ======================================================================== */
/* rnglib.f90                                                               */
/* ======================================================================== */
#define M1 2147483563
#define M2 2147483399

/* rnglib.f90:1238-1396 -- (a*s) mod m by Schrage's decomposition, h = 2^15.
 * Intermediates are held in 64 bits; the Fortran bounds keep them within
 * 32 bits, so the results are the same. */
int32_t rfo_multmod(int32_t a_in, int32_t s_in, int32_t m_in) {
  const int64_t h = 32768;
  int64_t a = a_in, s = s_in, m = m_in;
  int64_t a0, a1, k, p, q, qh, rh;
  if (a <= 0 || m <= a || s <= 0 || m <= s) return -1; /* the reference stops */
  if (a < h) {
    a0 = a;
    p = 0;
  } else {
    a1 = a / h;
    a0 = a - h * a1;
    qh = m / h;
    rh = m - h * qh;
    if (h <= a1) {
      a1 = a1 - h;
      k = s / qh;
      p = h * (s - k * qh) - k * rh;
      while (p < 0) p += m;
    } else {
      p = 0;
    }
    if (a1 != 0) {
      q = m / a1;
      k = s / q;
      p = p - k * (m - a1 * q);
      if (0 < p) p = p - m;
      p = p + a1 * (s - k * q);
      while (p < 0) p += m;
    }
    k = p / qh;
    p = h * (p - k * qh) - k * rh;
    while (p < 0) p += m;
  }
  if (a0 != 0) {
    q = m / a0;
    k = s / q;
    p = p - k * (m - a0 * q);
    if (0 < p) p = p - m;
    p = p + a0 * (s - k * q);
    while (p < 0) p += m;
  }
  return (int32_t)p;
}

/* rnglib.f90:457-489 */
void rfo_rng_cgn_set(rfo_rnglib* r, int32_t g) { r->g = g; }

/* rnglib.f90:804-908 */
void rfo_rng_init_generator(rfo_rnglib* r, int32_t t) {
  const int32_t a1_w = 1033780774, a2_w = 1494757890;
  int gi;
  if (!r->initialized) rfo_rng_initialize(r);
  gi = r->g - 1;
  if (t == 0) {
    r->lg1[gi] = r->ig1[gi];
    r->lg2[gi] = r->ig2[gi];
  } else if (t == 1) {
    /* restore the last seed: lg unchanged */
  } else if (t == 2) {
    r->lg1[gi] = rfo_multmod(a1_w, r->lg1[gi], M1);
    r->lg2[gi] = rfo_multmod(a2_w, r->lg2[gi], M2);
  } else {
    return; /* the reference stops on T out of bounds */
  }
  r->cg1[gi] = r->lg1[gi];
  r->cg2[gi] = r->lg2[gi];
}

/* rnglib.f90:1521-1622 */
void rfo_rng_set_initial_seed(rfo_rnglib* r, int32_t ig1, int32_t ig2) {
  const int32_t a1_vw = 2082007225, a2_vw = 784306273;
  int32_t g;
  if (ig1 < 1 || M1 <= ig1 || ig2 < 1 || M2 <= ig2) return; /* reference stops */
  r->g = 1;
  r->ig1[0] = ig1;
  r->ig2[0] = ig2;
  rfo_rng_init_generator(r, 0);
  for (g = 2; g <= 32; ++g) {
    r->g = g;
    ig1 = rfo_multmod(a1_vw, ig1, M1);
    ig2 = rfo_multmod(a2_vw, ig2, M2);
    r->ig1[g - 1] = ig1;
    r->ig2[g - 1] = ig2;
    rfo_rng_init_generator(r, 0);
  }
  r->g = 1;
}

/* rnglib.f90:909-975 */
void rfo_rng_initialize(rfo_rnglib* r) {
  memset(r, 0, sizeof(*r));
  r->initialized = 1;
  r->g = 1;
  rfo_rng_set_initial_seed(r, 1234567890, 123456789);
  r->g = 1;
}

/* rnglib.f90:548-659 */
int32_t rfo_rng_i4_uni(rfo_rnglib* r) {
  const int32_t a1 = 40014, a2 = 40692;
  int32_t k, z, cg1, cg2, gi;
  if (!r->initialized) rfo_rng_initialize(r);
  gi = r->g - 1;
  cg1 = r->cg1[gi];
  cg2 = r->cg2[gi];
  k = cg1 / 53668;
  cg1 = a1 * (cg1 - k * 53668) - k * 12211;
  if (cg1 < 0) cg1 = cg1 + M1;
  k = cg2 / 52774;
  cg2 = a2 * (cg2 - k * 52774) - k * 3791;
  if (cg2 < 0) cg2 = cg2 + M2;
  r->cg1[gi] = cg1;
  r->cg2[gi] = cg2;
  z = cg1 - cg2;
  if (z < 1) z = z + M1 - 1;
  if (r->anti[gi]) z = M1 - z;
  return z;
}

void rfo_rng_i4_stream(rfo_rnglib* r, int64_t count, int32_t* out) {
  for (int64_t i = 0; i < count; ++i) out[i] = rfo_rng_i4_uni(r);
}

/* rnglib.f90:1459-1520 */
double rfo_rng_r8_uni_01(rfo_rnglib* r) {
  int32_t i = rfo_rng_i4_uni(r);
  return (double)i * 4.656613057E-10;
}

/* rnglib.f90:3-91 */
void rfo_rng_advance_state(rfo_rnglib* r, int32_t k) {
  int32_t b1 = 40014, b2 = 40692, i, gi;
  if (k < 0) return;
  if (!r->initialized) rfo_rng_initialize(r);
  gi = r->g - 1;
  for (i = 1; i <= k; ++i) {
    b1 = rfo_multmod(b1, b1, M1);
    b2 = rfo_multmod(b2, b2, M2);
  }
  r->cg1[gi] = rfo_multmod(b1, r->cg1[gi], M1);
  r->cg2[gi] = rfo_multmod(b2, r->cg2[gi], M2);
}

/* math_RF.f90:561  seed = 72 + seedStart*18 + 37*(i-1): the first two words
 * become rnglib's (ig1, ig2). */
void rfo_seed_words(int64_t seedStart, int32_t* ig1, int32_t* ig2) {
  *ig1 = (int32_t)(72 + 18 * seedStart);
  *ig2 = (int32_t)(72 + 18 * seedStart + 37);
}

int32_t rfo_rng_seed(rfo_rnglib* r, int64_t seedStart) {
  int32_t ig1, ig2;
  if (seedStart < 0 || 72 + 18 * seedStart + 37 >= M2) return RFO_EINVAL;
  rfo_seed_words(seedStart, &ig1, &ig2);
  rfo_rng_initialize(r);
  rfo_rng_set_initial_seed(r, ig1, ig2);
  return RFO_OK;
}

/* ======================================================================== */
/* tables: spectra_RF.f90, math_RF.f90                                      */
/* ======================================================================== */

/* spectra_RF.f90:15-44 (values cover 99% of the Gaussian spectral area).
 * set_kMaxND assigns kMax only for cm_GAUSSIAN; the restatement uses the
 * same value for cm_COS, whose reference kMax is the -1 of init_RF. */
static double kmax_nd(int32_t nDim) {
  switch (nDim) {
    case 1: return 6.457;
    case 2: return 7.035;
    default: return 7.355;
  }
}

/* math_RF.f90:380-391 */
static int32_t cyclic_mod(int32_t pos, int32_t base) {
  int32_t r = pos % base;
  return r == 0 ? base : r;
}

/* spectra_RF.f90:267-286: rows (+,+,+),(+,+,-),(+,-,+),(+,-,-) in 3D. */
static void ksign(int32_t nDim, double* kSign /* rows x nDim, row-major */) {
  int32_t rows = 1 << (nDim - 1), i, j;
  for (j = 0; j < rows * nDim; ++j) kSign[j] = 1.0;
  for (i = 2; i <= nDim; ++i) {
    int32_t seedStep = 1 << (nDim - i);
    for (j = 1; j <= rows; ++j) {
      int32_t pos = cyclic_mod((int32_t)((j - 0.9) / seedStep), 2);
      if (pos % 2 == 1) kSign[(j - 1) * nDim + (i - 1)] = -1.0;
    }
  }
}

/* math_RF.f90:16-92, non-inverse branch: axis 1 fastest. */
void rfo_set_grid(int32_t nDim, const double* xMin, const double* xStep,
                  const int32_t* xNStep, double* xPoints) {
  int64_t total = 1, p;
  int32_t d;
  for (d = 0; d < nDim; ++d) total *= xNStep[d];
  for (p = 0; p < total; ++p) {
    int64_t rem = p;
    for (d = 0; d < nDim; ++d) {
      int64_t i = rem % xNStep[d];
      rem /= xNStep[d];
      xPoints[p * nDim + d] = xMin[d] + xStep[d] * (double)i;
    }
  }
}

/* type_inputRF.f90:1159-1206 (Nmc, corrL), randomFieldND.f90:162-166
 * (lognormal needs fieldAvg > 0), constants_RF.f90:12-21 (ids). */
int32_t rfo_validate(const rfo_request* rq) {
  int32_t d;
  if (!rq || rq->nDim < 1 || rq->nDim > 3) return RFO_EINVAL;
  if (rq->n < 1 || !rq->xPoints) return RFO_EINVAL;
  if (rq->Nmc < 1) return RFO_EINVAL;
  for (d = 0; d < rq->nDim; ++d)
    if (!(rq->corrL[d] > 0.0)) return RFO_EINVAL;
  if (rq->corrMod != RFO_CM_GAUSSIAN && rq->corrMod != RFO_CM_COS) return RFO_EINVAL;
  if (rq->margiFirst != RFO_FOM_GAUSSIAN && rq->margiFirst != RFO_FOM_LOGNORMAL) return RFO_EINVAL;
  if (rq->margiFirst == RFO_FOM_LOGNORMAL && rq->fieldAvg <= 0.0) return RFO_EINVAL;
  if (rq->method != RFO_SHINOZUKA && rq->method != RFO_ISOTROPIC && rq->method != RFO_RANDOMIZATION) return RFO_EINVAL;
  if (rq->method == RFO_ISOTROPIC && rq->nDim < 2) return RFO_EINVAL;
  if (rq->method == RFO_ISOTROPIC && rq->literal) return RFO_EINVAL;
  if (rq->seedStart < 0) return RFO_EINVAL;
  return RFO_OK;
}

/* randomFieldND.f90:58-73 (x and xRange divided by corrL), spectra_RF.f90:75-118
 * (grid sizes), randomFieldND.f90:237-239 (slab rows), :260-266 (ampMult). */
int32_t rfo_geometry_of(const rfo_request* rq, rfo_geometry* g) {
  int32_t d, rc = rfo_validate(rq);
  const double PI = RFO_PI;
  if (rc) return rc;
  memset(g, 0, sizeof(*g));
  g->nDim = rq->nDim;
  g->kMax = kmax_nd(rq->nDim);
  for (d = 0; d < rq->nDim; ++d) {
    double ext = rq->xRange[d];
    if (!(ext > 0.0)) {
      double lo = rq->xPoints[d], hi = rq->xPoints[d];
      int64_t i;
      for (i = 1; i < rq->n; ++i) {
        double v = rq->xPoints[i * rq->nDim + d];
        if (v < lo) lo = v;
        if (v > hi) hi = v;
      }
      ext = hi - lo;
    }
    if (!(ext > 0.0)) return RFO_EINVAL; /* degenerate extent: kDelta = +inf */
    g->xRangeNorm[d] = ext / rq->corrL[d];
  }
  if (rq->method != RFO_ISOTROPIC) {
    /* Shinozuka and randomization share the grid sizes (spectra_RF.f90:87-124) */
    int64_t kn = 1;
    double prodDelta = 1.0;
    for (d = 0; d < rq->nDim; ++d) {
      double kd = 2.0 * PI / (1.1 * g->xRangeNorm[d]);
      int32_t ns = rq->kNStep[d] > 0 ? rq->kNStep[d]
                                     : 1 + (int32_t)(1.0 * ceil(g->kMax / kd));
      if (ns < 2) return RFO_EINVAL;
      g->kNStep[d] = ns;
      g->kDelta[d] = g->kMax / (double)(ns - 1);
      kn *= ns;
      prodDelta *= g->kDelta[d];
    }
    g->K = kn * ((int64_t)1 << (rq->nDim - 1));
    g->ampMult = 2.0 * sqrt(prodDelta / pow(2.0 * PI, (double)rq->nDim));
    if (rq->method == RFO_RANDOMIZATION) {
      /* randomFieldND.f90:262: 2*sqrt(1/(kNTotal*(2 PI)^nDim)) (literal).  A
       * random wavevector of one quadrant represents kMax^nDim / kn of the
       * spectral volume, which the intended amplitude restores. */
      if (rq->literal) g->ampMult = 2.0 * sqrt(1.0 / ((double)g->K * pow(2.0 * PI, (double)rq->nDim)));
      else g->ampMult = 2.0 * sqrt(pow(g->kMax, (double)rq->nDim) / ((double)kn * pow(2.0 * PI, (double)rq->nDim)));
    }
  } else {
    double r2 = 0.0, kd;
    int32_t nr, nd;
    for (d = 0; d < rq->nDim; ++d) r2 += g->xRangeNorm[d] * g->xRangeNorm[d];
    kd = 2.0 * PI / (1.1 * sqrt(r2));
    nr = rq->isoNRadial > 0 ? rq->isoNRadial : 1 + (int32_t)(5.0 * ceil(g->kMax / kd));
    nd = rq->isoNDir > 0 ? rq->isoNDir : 32;
    if (nr < 2) return RFO_EINVAL;
    g->kNStep[0] = nr;
    g->kNStep[1] = nd;
    g->kDelta[0] = g->kMax / (double)(nr - 1);
    g->K = (int64_t)nr * nd;
    g->ampMult = 1.0;
  }
  g->xSlab = (int64_t)((double)rq->nDim * 1e8 / (double)g->K);
  if (g->xSlab > rq->n) g->xSlab = rq->n;
  if (g->xSlab < 1) g->xSlab = 1;
  return RFO_OK;
}

/* Gaussian spectrum with corrL = 1 after normalisation: spectra_RF.f90:202-208.
 * cm_COS: S = 1 at the 6th wavevector only: spectra_RF.f90:210-220. */
static double spectrum_gauss(const double* k, int32_t nDim) {
  const double PI = RFO_PI;
  double s = 1.0;
  int32_t d;
  for (d = 0; d < nDim; ++d) s = s * 1.0 * exp(-((k[d] * k[d]) * 1.0) / (4.0 * PI));
  return s;
}

/* spectra_RF.f90:87-133 (Shinozuka grid, sign quadrants; B2 in literal mode)
 * and the isotropic intended table (randomFieldND.f90:368-514 restated). */
int32_t rfo_kpoints(const rfo_request* rq, double* kPoints, double* amp, double* S) {
  rfo_geometry g;
  int32_t rc = rfo_geometry_of(rq, &g), d;
  const double PI = RFO_PI;
  int64_t k, K;
  if (rc) return rc;
  K = g.K;
  if (rq->corrMod == RFO_CM_COS && K <= 6) return RFO_EINVAL; /* spectra_RF.f90:218 */
  if (rq->method != RFO_ISOTROPIC) {
    int32_t nq = 1 << (rq->nDim - 1), q;
    int64_t kn = K / nq, b;
    double sign[4 * 3];
    double* ubase = NULL;
    ksign(rq->nDim, sign);
    if (rq->method == RFO_RANDOMIZATION) {
      /* random_number(kPoints_base) then * kMax per axis (spectra_RF.f90:
       * 119-124): nDim x kn draws, axis fastest, before the phases */
      rfo_rnglib rng;
      int64_t t;
      ubase = (double*)malloc(sizeof(double) * kn * rq->nDim);
      if (!ubase) return RFO_EINVAL;
      if (rfo_rng_seed(&rng, rq->seedStart)) { free(ubase); return RFO_EINVAL; }
      for (t = 0; t < kn * rq->nDim; ++t) ubase[t] = rfo_rng_r8_uni_01(&rng);
    }
    for (q = 0; q < nq; ++q) {
      for (b = 0; b < kn; ++b) {
        int64_t rem = b;
        k = q * kn + b;
        for (d = 0; d < rq->nDim; ++d) {
          int64_t i = rem % g.kNStep[d];
          /* setGrid from 0 (spectra_RF.f90:118), then the sign copy :127-133
           * which starts at quadrant 2: the first quadrant stays unwritten. */
          double base = ubase ? ubase[b * rq->nDim + d] * g.kMax : 0.0 + g.kDelta[d] * (double)i;
          rem /= g.kNStep[d];
          kPoints[k * rq->nDim + d] = (rq->literal && q == 0) ? 0.0 : base * sign[q * rq->nDim + d];
        }
      }
    }
    free(ubase);
    for (k = 0; k < K; ++k) {
      double s;
      if (rq->corrMod == RFO_CM_GAUSSIAN) s = spectrum_gauss(&kPoints[k * rq->nDim], rq->nDim);
      else s = (k == 5) ? 1.0 : 0.0;
      if (S) S[k] = s;
      if (amp) amp[k] = sqrt(s);
    }
  } else {
    /* Isotropic, intended maths.  Radial grid r_j = (j-1)*dr from
     * get_Permutation(snapExtremes) (math_RF.f90:98-148) with the loop index
     * of spectra_RF.f90:83 fixed (B3); n_dir directions per radius drawn once
     * per request, uniform on the sphere (circle in 2D); amplitude
     * A = sqrt(2 * |S^{D-1}| r^{D-1} S(r) dr / ((2 pi)^D n_dir)) so that the
     * field has unit variance (the reference's sqrt(S sin(phi) r^2) with
     * phi ~ U[0,pi) has variance 1/(4 pi^2), randomFieldND.f90:480,:500). */
    rfo_rnglib rng;
    int32_t nr = g.kNStep[0], nd = g.kNStep[1], j, dd;
    double dr = g.kDelta[0];
    double* uphi = NULL;
    double* uth = (double*)malloc(sizeof(double) * K);
    if (!uth) return RFO_EINVAL;
    if (rq->nDim == 3) {
      uphi = (double*)malloc(sizeof(double) * K);
      if (!uphi) { free(uth); return RFO_EINVAL; }
    }
    if (rfo_rng_seed(&rng, rq->seedStart)) { free(uth); free(uphi); return RFO_EINVAL; }
    if (uphi) for (k = 0; k < K; ++k) uphi[k] = rfo_rng_r8_uni_01(&rng);
    for (k = 0; k < K; ++k) uth[k] = rfo_rng_r8_uni_01(&rng);
    for (j = 0; j < nr; ++j) {
      double r = (double)j * dr;
      double s, shell;
      if (rq->corrMod == RFO_CM_GAUSSIAN) s = exp(-((r * r) * 1.0) / (4.0 * PI));
      else s = (j == 5) ? 1.0 : 0.0;
      shell = (rq->nDim == 3) ? 4.0 * PI * r * r : 2.0 * PI * r;
      for (dd = 0; dd < nd; ++dd) {
        double th, a;
        k = (int64_t)j * nd + dd;
        th = 2.0 * PI * uth[k];
        if (rq->nDim == 3) {
          double cph = 1.0 - 2.0 * uphi[k];
          double sph = sqrt(fmax(0.0, 1.0 - cph * cph));
          kPoints[k * 3 + 0] = r * (sph * cos(th));
          kPoints[k * 3 + 1] = r * (sph * sin(th));
          kPoints[k * 3 + 2] = r * cph;
        } else {
          kPoints[k * 2 + 0] = r * cos(th);
          kPoints[k * 2 + 1] = r * sin(th);
        }
        a = sqrt(2.0 * shell * s * dr / (pow(2.0 * PI, (double)rq->nDim) * (double)nd));
        if (S) S[k] = s;
        if (amp) amp[k] = a;
      }
    }
    free(uth);
    free(uphi);
  }
  return RFO_OK;
}

/* Per-realization random draws.
 * Shinozuka: phi = 2*pi*U, K draws per realization in k order
 * (randomFieldND.f90:278-279); gamma = 1.
 * Isotropic: after the direction blocks, per realization a gamma block
 * (gamma = sqrt(12.0)*(U - 1/2), randomFieldND.f90:468, with the single
 * precision sqrt(12.0) of the source) then a psi block (psi = 2*pi*U, :465). */
static int32_t draws(const rfo_request* rq, const rfo_geometry* g, double* phi, double* gam) {
  rfo_rnglib rng;
  const double PI = RFO_PI;
  int64_t K = g->K, k;
  int32_t r;
  if (rfo_rng_seed(&rng, rq->seedStart)) return RFO_EINVAL;
  if (rq->method != RFO_ISOTROPIC) {
    if (rq->method == RFO_RANDOMIZATION) /* the wavevector draws come first */
      for (k = 0; k < (K >> (rq->nDim - 1)) * rq->nDim; ++k) (void)rfo_rng_i4_uni(&rng);
    for (r = 0; r < rq->Nmc; ++r)
      for (k = 0; k < K; ++k) {
        phi[k + K * r] = 2.0 * PI * rfo_rng_r8_uni_01(&rng);
        gam[k + K * r] = 1.0;
      }
  } else {
    const double sq12 = (double)sqrtf(12.0f);
    int64_t skip = (rq->nDim == 3 ? 2 : 1) * K;
    for (k = 0; k < skip; ++k) (void)rfo_rng_i4_uni(&rng);
    for (r = 0; r < rq->Nmc; ++r) {
      for (k = 0; k < K; ++k) gam[k + K * r] = sq12 * (rfo_rng_r8_uni_01(&rng) - 0.5);
      for (k = 0; k < K; ++k) phi[k + K * r] = 2.0 * PI * rfo_rng_r8_uni_01(&rng);
    }
  }
  return RFO_OK;
}

int32_t rfo_phase_matrix(const rfo_request* rq, double* Bc, double* Bs) {
  rfo_geometry g;
  int32_t rc = rfo_geometry_of(rq, &g), r;
  int64_t K, k;
  double *kp, *amp, *phi, *gam;
  if (rc) return rc;
  K = g.K;
  kp = (double*)malloc(sizeof(double) * K * rq->nDim);
  amp = (double*)malloc(sizeof(double) * K);
  phi = (double*)malloc(sizeof(double) * K * rq->Nmc);
  gam = (double*)malloc(sizeof(double) * K * rq->Nmc);
  if (!kp || !amp || !phi || !gam) { rc = RFO_EINVAL; goto out; }
  if ((rc = rfo_kpoints(rq, kp, amp, NULL))) goto out;
  if ((rc = draws(rq, &g, phi, gam))) goto out;
  for (r = 0; r < rq->Nmc; ++r)
    for (k = 0; k < K; ++k) {
      double a = amp[k] * gam[k + K * r];
      Bc[k + K * r] = a * cos(phi[k + K * r]);
      Bs[k + K * r] = -a * sin(phi[k + K * r]);
    }
out:
  free(kp); free(amp); free(phi); free(gam);
  return rc;
}

/* ======================================================================== */
/* marginal transform and normalisation                                     */
/* ======================================================================== */

/* randomFieldND.f90:139-178 */
int32_t rfo_marginal(int32_t margiFirst, double fieldAvg, double fieldVar,
                     double* f, int64_t count) {
  double normalVar = 1.0, normalAvg = 0.0, sd;
  int64_t i;
  if (margiFirst == RFO_FOM_GAUSSIAN) {
    normalVar = fieldVar;
    normalAvg = fieldAvg;
  } else if (margiFirst == RFO_FOM_LOGNORMAL) {
    if (fieldAvg <= 0.0) return RFO_EINVAL;
    normalVar = log(1 + fieldVar / (fieldAvg * fieldAvg));
    normalAvg = log(fieldAvg) - normalVar / 2;
  } else {
    return RFO_EINVAL;
  }
  sd = sqrt(normalVar);
  for (i = 0; i < count; ++i) f[i] = f[i] * sd + normalAvg;
  if (margiFirst == RFO_FOM_LOGNORMAL)
    for (i = 0; i < count; ++i) f[i] = exp(f[i]);
  return RFO_OK;
}

/* randomFieldND.f90:820-926: subtract the column mean, divide by the RMS. */
void rfo_normalize(double* f, int64_t n, int32_t ncols) {
  int32_t c;
  int64_t i;
  for (c = 0; c < ncols; ++c) {
    double s = 0.0, s2 = 0.0, avg, sd;
    double* col = f + (int64_t)c * n;
    for (i = 0; i < n; ++i) s += col[i];
    avg = s / (double)n;
    for (i = 0; i < n; ++i) col[i] -= avg;
    for (i = 0; i < n; ++i) s2 += col[i] * col[i];
    sd = sqrt(s2 / (double)n);
    for (i = 0; i < n; ++i) col[i] /= sd;
  }
}

/* ======================================================================== */
/* the field                                                                */
/* ======================================================================== */

typedef struct {
  rfo_geometry g;
  double *kp, *amp, *S, *phi, *gam;
} tables_t;

static void tables_free(tables_t* t) {
  free(t->kp); free(t->amp); free(t->S); free(t->phi); free(t->gam);
}

static int32_t tables_build(const rfo_request* rq, tables_t* t) {
  int32_t rc;
  memset(t, 0, sizeof(*t));
  if ((rc = rfo_geometry_of(rq, &t->g))) return rc;
  t->kp = (double*)malloc(sizeof(double) * t->g.K * rq->nDim);
  t->amp = (double*)malloc(sizeof(double) * t->g.K);
  t->S = (double*)malloc(sizeof(double) * t->g.K);
  t->phi = (double*)malloc(sizeof(double) * t->g.K * rq->Nmc);
  t->gam = (double*)malloc(sizeof(double) * t->g.K * rq->Nmc);
  if (!t->kp || !t->amp || !t->S || !t->phi || !t->gam) { tables_free(t); return RFO_EINVAL; }
  if ((rc = rfo_kpoints(rq, t->kp, t->amp, t->S)) || (rc = draws(rq, &t->g, t->phi, t->gam))) {
    tables_free(t);
    return rc;
  }
  return RFO_OK;
}

/* Literal-mode amplitude (B1): slab m (1-based) of realization n (1-based)
 * uses S^(1/2^t), t = (n-1)*nSlab + m, because SkMat = sqrt(SkMat) runs on
 * every iteration (randomFieldND.f90:312 inside :276 and :284). */
static double literal_amp(double s, int64_t t) {
  int64_t i;
  for (i = 0; i < t; ++i) s = sqrt(s);
  return s;
}

static int32_t finish(const rfo_request* rq, double* out, int64_t nrows) {
  if (rq->normalize) rfo_normalize(out, nrows, rq->literal ? 1 : rq->Nmc);
  return rfo_marginal(rq->margiFirst, rq->fieldAvg, rq->fieldVar, out, nrows * rq->Nmc);
}

/* Shinozuka: f = ampMult * sum_k sqrt(S_k) cos(k.x + phi_k) in the arithmetic
 * order of the reference: DGEMM 'T','N' accumulates x.k over the dimensions
 * from zero and adds phi with beta = 1 (BLAS/dgemm.f90:244-256), cos, then the
 * GEMV accumulates in k order skipping zero weights (:230-238), ampMult last
 * (randomFieldND.f90:330).  Isotropic: sum_k A_k gamma cos(k.x + psi)
 * accumulated in k order (randomFieldND.f90:478-485). */
int32_t rfo_generate(const rfo_request* rq, const int64_t* rows, int64_t nrows,
                     double* out, int32_t nthreads) {
  tables_t t;
  int32_t rc;
  int64_t m, nSlab, K;
  const int32_t D = rq ? rq->nDim : 0;
  if ((rc = tables_build(rq, &t))) return rc;
  K = t.g.K;
  if (!rows) nrows = rq->n;
  nSlab = (rq->n + t.g.xSlab - 1) / t.g.xSlab;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
  for (m = 0; m < nrows; ++m) {
    int64_t i = rows ? rows[m] : m;
    double x[3] = {0, 0, 0};
    int32_t d, r;
    int64_t k;
    for (d = 0; d < D; ++d) x[d] = rq->xPoints[i * D + d] / rq->corrL[d];
    for (r = 0; r < rq->Nmc; ++r) {
      double acc = 0.0;
      if (rq->method != RFO_ISOTROPIC) {
        int64_t slab = i / t.g.xSlab + 1;
        int64_t tt = (int64_t)r * nSlab + slab;
        for (k = 0; k < K; ++k) {
          double temp = 0.0, c, w = t.amp[k];
          for (d = 0; d < D; ++d) temp = temp + x[d] * t.kp[k * D + d];
          c = cos(1.0 * temp + 1.0 * t.phi[k + K * r]);
          if (rq->literal) w = literal_amp(t.S[k], tt);
          if (w != 0.0) acc = acc + w * c;
        }
        out[m + nrows * r] = t.g.ampMult * acc;
      } else {
        for (k = 0; k < K; ++k) {
          double temp = 0.0;
          for (d = 0; d < D; ++d) temp = temp + x[d] * t.kp[k * D + d];
          acc = t.amp[k] * t.gam[k + K * r] * cos(temp + t.phi[k + K * r]) + acc;
        }
        out[m + nrows * r] = acc;
      }
    }
  }
  tables_free(&t);
  return finish(rq, out, nrows);
}

/* The contraction recast of the same sum: f = sum_k cos(k.x) Bc + sin(k.x) Bs
 * with Bc = a cos(phi), Bs = -a sin(phi) (intended mode only). */
int32_t rfo_generate_recast(const rfo_request* rq, const int64_t* rows, int64_t nrows,
                            double* out, int32_t nthreads) {
  tables_t t;
  int32_t rc;
  int64_t m, K;
  double *Bc, *Bs;
  const int32_t D = rq ? rq->nDim : 0;
  if (rq && rq->literal) return RFO_EINVAL;
  if ((rc = tables_build(rq, &t))) return rc;
  K = t.g.K;
  if (!rows) nrows = rq->n;
  Bc = (double*)malloc(sizeof(double) * K * rq->Nmc);
  Bs = (double*)malloc(sizeof(double) * K * rq->Nmc);
  if (!Bc || !Bs) { free(Bc); free(Bs); tables_free(&t); return RFO_EINVAL; }
  for (m = 0; m < K * rq->Nmc; ++m) {
    double a = t.amp[m % K] * t.gam[m];
    Bc[m] = a * cos(t.phi[m]);
    Bs[m] = -a * sin(t.phi[m]);
  }
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
  for (m = 0; m < nrows; ++m) {
    int64_t i = rows ? rows[m] : m;
    double x[3] = {0, 0, 0};
    int32_t d, r;
    int64_t k;
    double* acc = (double*)calloc(rq->Nmc, sizeof(double));
    for (d = 0; d < D; ++d) x[d] = rq->xPoints[i * D + d] / rq->corrL[d];
    for (k = 0; k < K; ++k) {
      double th = 0.0, c, s;
      for (d = 0; d < D; ++d) th += x[d] * t.kp[k * D + d];
      c = cos(th);
      s = sin(th);
      for (r = 0; r < rq->Nmc; ++r) acc[r] += c * Bc[k + K * r] + s * Bs[k + K * r];
    }
    for (r = 0; r < rq->Nmc; ++r) out[m + nrows * r] = t.g.ampMult * acc[r];
    free(acc);
  }
  free(Bc);
  free(Bs);
  tables_free(&t);
  return finish(rq, out, nrows);
}

/* ======================================================================== */
/* localization blend                                                       */
/* ======================================================================== */

int32_t rfo_overlap_npoints(double overlap, double corrL, double xStep) {
  return (int32_t)lround((overlap * corrL - 2 * xStep) / xStep) + 1;
}

/* localization_RF.f90:705-857 with partitionType = 1 (cosine). */
void rfo_unity_partition(int32_t nDim, const int32_t* xNStep,
                         const int32_t* overlapNPoints, uint32_t faceMask,
                         double* up) {
  const double PI = RFO_PI;
  int64_t total = 1, p;
  int32_t j, d;
  for (d = 0; d < nDim; ++d) total *= xNStep[d];
  for (p = 0; p < total; ++p) up[p] = 1.0;
  for (j = 0; j < 2; ++j) {
    for (d = 0; d < nDim; ++d) {
      int32_t N = overlapNPoints[d], s;
      int32_t dlim;
      int64_t stride = 1;
      int32_t e;
      if (N < 1) continue;
      if (!(faceMask & (1u << (2 * d + j)))) continue;
      dlim = (j == 0) ? 1 : xNStep[d] - N + 1;
      for (e = 0; e < d; ++e) stride *= xNStep[e];
      for (s = 1; s <= N; ++s) {
        /* pattern = s/(N+2), reversed on the low face */
        double pat = (j == 0) ? (double)(N + 1 - s) / (double)(N + 2) : (double)s / (double)(N + 2);
        double w = (1.0 + cos(PI * pat)) / 2.0;
        int64_t idx = dlim + s - 2; /* 0-based index along axis d */
        for (p = 0; p < total; ++p) {
          if ((p / stride) % xNStep[d] == idx) up[p] *= w;
        }
      }
    }
  }
}

/* ======================================================================== */
/* CPU baseline                                                             */
/* ======================================================================== */

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#define BASE_SLAB 256

double rfo_baseline_shinozuka(const rfo_request* rq, int64_t row0, int64_t nrows,
                              int32_t r0, int32_t nr, double* out, int32_t nthreads) {
  tables_t t;
  int64_t K, nblk, blk;
  int32_t D;
  double t0, t1;
  if (!rq || rq->method != RFO_SHINOZUKA || rq->literal) return -1.0;
  if (tables_build(rq, &t)) return -1.0;
  if (row0 < 0 || nrows < 1 || row0 + nrows > rq->n || r0 < 0 || nr < 1 || r0 + nr > rq->Nmc) {
    tables_free(&t);
    return -1.0;
  }
  K = t.g.K;
  D = rq->nDim;
  nblk = (nrows + BASE_SLAB - 1) / BASE_SLAB;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  t0 = now_s();
#ifdef _OPENMP
#pragma omp parallel
#endif
  {
    double* kxphi = (double*)malloc(sizeof(double) * BASE_SLAB * K);
    double* xs = (double*)malloc(sizeof(double) * BASE_SLAB * D);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
    for (blk = 0; blk < nblk; ++blk) {
      int64_t s0 = row0 + blk * BASE_SLAB;
      int64_t ns = (s0 + BASE_SLAB <= row0 + nrows) ? BASE_SLAB : row0 + nrows - s0;
      int64_t i, k;
      int32_t r, d;
      for (i = 0; i < ns; ++i)
        for (d = 0; d < D; ++d) xs[i * D + d] = rq->xPoints[(s0 + i) * D + d] / rq->corrL[d];
      for (r = r0; r < r0 + nr; ++r) {
        double* c = out + (s0 - row0) + nrows * (r - r0);
        /* k_x_phi(1:xDelta,:) = phiK(1:xDelta,:)   randomFieldND.f90:304 */
        for (k = 0; k < K; ++k)
          for (i = 0; i < ns; ++i) kxphi[i + ns * k] = t.phi[k + K * r];
        /* DGEMM 'T','N', beta = 1   randomFieldND.f90:307, BLAS/dgemm.f90:244-256 */
        for (k = 0; k < K; ++k)
          for (i = 0; i < ns; ++i) {
            double temp = 0.0;
            for (d = 0; d < D; ++d) temp = temp + xs[i * D + d] * t.kp[k * D + d];
            kxphi[i + ns * k] = 1.0 * temp + 1.0 * kxphi[i + ns * k];
          }
        /* cos   randomFieldND.f90:310 */
        for (k = 0; k < K * ns; ++k) kxphi[k] = cos(kxphi[k]);
        /* DGEMM 'N','N' with one column   randomFieldND.f90:320, BLAS/dgemm.f90:218-238 */
        for (i = 0; i < ns; ++i) c[i] = 0.0;
        for (k = 0; k < K; ++k) {
          if (t.amp[k] != 0.0) {
            double temp = 1.0 * t.amp[k];
            for (i = 0; i < ns; ++i) c[i] = c[i] + temp * kxphi[i + ns * k];
          }
        }
        /* ampMult   randomFieldND.f90:330 */
        for (i = 0; i < ns; ++i) c[i] = t.g.ampMult * c[i];
      }
    }
    free(kxphi);
    free(xs);
  }
  t1 = now_s();
  tables_free(&t);
  return t1 - t0;
}

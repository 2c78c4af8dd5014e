// Host paths of the C-ABI under AddressSanitizer and UBSan (built and run by
// tests/test_sanitizers.py).  Everything here runs on the host: argument
// validation and its status codes, the wavevector geometry, the blend
// layout, the result writer; one valid generation returns RF_OK on a GPU
// box and RF_ENODEV / RF_ECUDA without one.  Prints "harness ok".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "randomfield_b200.h"

static int failures = 0;
#define EXPECT(cond)                                                      \
  do {                                                                    \
    if (!(cond)) {                                                        \
      std::fprintf(stderr, "%s:%d: expected %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                         \
    }                                                                     \
  } while (0)

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  EXPECT(rf_abi_version() == RF_ABI_VERSION);
  rf_options o;
  rf_options_init(&o);
  EXPECT(o.size == (int32_t)sizeof(rf_options) && o.precision == RF_PREC_BF16);

  // points of a 6 x 5 x 4 grid
  std::vector<double> x;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 5; ++j)
      for (int i = 0; i < 6; ++i) {
        x.push_back(0.1 * i);
        x.push_back(0.2 * j);
        x.push_back(0.3 * k);
      }
  const int64_t n = 120;
  const double corrL[3] = {1.0, 2.0, 0.5};
  std::vector<double> field((size_t)n * 3);

  // validation codes of the flat entry point (type_inputRF.f90:1159-1206 and friends)
  struct Bad {
    int nDim, corrMod, margiFirst, Nmc, method;
    double avg;
    int code;
  } bad[] = {{3, 1, 1, 0, 2, 0.0, RF_EINVAL_NMC},  {0, 1, 1, 3, 2, 0.0, RF_EINVAL_NDIM},
             {3, 9, 1, 3, 2, 0.0, RF_EINVAL_CORRMOD}, {3, 1, 9, 3, 2, 0.0, RF_EINVAL_MARGINAL},
             {3, 1, 1, 3, 9, 0.0, RF_EINVAL_METHOD}, {3, 1, 2, 3, 2, -1.0, RF_EINVAL_LOGNORMAL},
             {1, 1, 1, 3, 1, 0.0, RF_EINVAL_NDIM}};
  for (const Bad& b : bad) {
    const int rc = rf_create_standard_gaussian_field_unstruct(x.data(), b.nDim, n, b.corrMod, b.margiFirst, corrL,
                                                              b.avg, 1.0, b.Nmc, b.method, field.data(), nullptr);
    EXPECT(rc == b.code);
    EXPECT(std::strlen(rf_last_error()) > 0);
  }
  const double badL[3] = {1.0, 0.0, 1.0};
  EXPECT(rf_create_standard_gaussian_field_unstruct(x.data(), 3, n, 1, 1, badL, 0.0, 1.0, 3, 2, field.data(),
                                                    nullptr) == RF_EINVAL_CORRL);
  EXPECT(rf_create_standard_gaussian_field_unstruct(nullptr, 3, n, 1, 1, corrL, 0.0, 1.0, 3, 2, field.data(),
                                                    nullptr) == RF_EINVAL_ARG);
  // a valid request: generated on a GPU box, refused without one
  {
    rf_options g;
    rf_options_init(&g);
    g.precision = RF_PREC_FP32;
    g.k_nstep[0] = g.k_nstep[1] = g.k_nstep[2] = 4;
    const int rc = rf_create_standard_gaussian_field_unstruct(x.data(), 3, n, 1, 1, corrL, 0.0, 1.0, 3, 2,
                                                              field.data(), &g);
    EXPECT(rc == RF_OK || rc == RF_ENODEV || rc == RF_ECUDA);
  }

  // geometry (host only)
  for (int method = 1; method <= 3; ++method) {
    int64_t K = 0;
    int32_t kn[3] = {0, 0, 0};
    double kd[3] = {0, 0, 0}, amp = 0;
    EXPECT(rf_query_geometry(x.data(), 3, n, 1, corrL, method, nullptr, &K, kn, kd, &amp) == RF_OK);
    EXPECT(K > 0 && amp > 0);
  }

  // blend layout (host only)
  {
    rf_blend_grid gr;
    std::memset(&gr, 0, sizeof(gr));
    gr.nDim = 3;
    for (int d = 0; d < 3; ++d) {
      gr.xNStep[d] = 256;
      gr.nFields[d] = 2;
      gr.xStep[d] = 0.05;
    }
    gr.overlap = 0.65;
    const double cl[3] = {1.0, 1.0, 1.0};
    int32_t sub[3], ov[3];
    const int rc = rf_blend_layout(&gr, cl, sub, ov);
    EXPECT(rc == RF_OK || rc == RF_EINVAL_RANGE);
  }

  // structured-grid entry point: host-side refusals
  {
    const double xmin[3] = {0, 0, 0}, h[3] = {0.1, 0.1, 0.1}, hbad[3] = {0.1, -0.1, 0.1};
    const int64_t ns[3] = {8, 8, 8};
    std::vector<double> out(512 * 2);
    EXPECT(rf_create_standard_gaussian_field_grid(3, xmin, h, ns, 1, 1, corrL, 0.0, 1.0, 2, 1, out.data(),
                                                  nullptr) == RF_ENOTSUP);
    EXPECT(rf_create_standard_gaussian_field_grid(3, xmin, hbad, ns, 1, 1, corrL, 0.0, 1.0, 2, 2, out.data(),
                                                  nullptr) == RF_EINVAL_ARG);
    EXPECT(rf_create_standard_gaussian_field_grid(3, xmin, h, ns, 1, 1, corrL, 0.0, 1.0, 0, 2, out.data(),
                                                  nullptr) == RF_EINVAL_NMC);
    EXPECT(rf_generate_fft_grid(nullptr, 3, ns, h, 1, 1, corrL, 0.0, 1.0, 1, out.data(), nullptr) == RF_EINVAL_ARG);
  }

  // result writer (host only)
  {
    const double xmin[3] = {0.0, -1.0, 2.0}, xmax[3] = {0.4, 0.5, 2.6}, h[3] = {0.1, 0.25, 0.2};
    std::vector<double> f(5 * 7 * 4);
    for (size_t i = 0; i < f.size(); ++i) f[i] = 0.01 * (double)i - 1.0;
    rf_result_attributes at;
    std::memset(&at, 0, sizeof(at));
    at.nb_procs = 1;
    at.nDim = 3;
    at.Nmc = 4;
    for (int d = 0; d < 3; ++d) {
      at.kNStep[d] = 24;
      at.corrL[d] = corrL[d];
    }
    EXPECT(rf_write_result_grid(dir.c_str(), "h3", 3, xmin, xmax, h, f.data(), &at) == RF_OK);
    EXPECT(rf_write_result_grid(dir.c_str(), "h2", 2, xmin, xmax, h, f.data(), nullptr) == RF_OK);
    EXPECT(rf_write_result_grid(dir.c_str(), "h1", 1, xmin, xmax, h, f.data(), nullptr) == RF_OK);
    EXPECT(rf_write_result_grid((dir + "/no/such/dir").c_str(), "x", 3, xmin, xmax, h, f.data(), nullptr) ==
           RF_EINVAL_ARG);
    EXPECT(rf_write_result_grid(dir.c_str(), "x", 4, xmin, xmax, h, f.data(), nullptr) == RF_EINVAL_NDIM);
  }

  if (failures) {
    std::fprintf(stderr, "%d expectation(s) failed\n", failures);
    return 1;
  }
  std::printf("harness ok\n");
  return 0;
}

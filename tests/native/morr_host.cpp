// The library's Morrison column and radar reflectivity column (thunderengine-web_b200/
// csrc/te_morr.cuh, te_refl.cuh) compiled for the host, with the tape-player kernel ABI of
// the CPU oracle (fn(uint32_t *M, const uint32_t *ARG): ARG[0..2] grid in threads,
// ARG[4 + n] word offset of binding n).  TEST
// INFRASTRUCTURE: it lets the CPU suite compare the library's restatement with the
// reference's own kernel (oracle/_ref) word for word without a GPU; the WGSL builtins are
// the binary64 evaluations of liboracle (te_*_f64), the same operations the CUDA build uses.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

extern "C" float te_pow_f64(float x, float y);
extern "C" float te_exp_f64(float x);
extern "C" float te_log_f64(float x);
extern "C" float te_log2_f64(float x);
extern "C" float te_atan2_f64(float y, float x);

namespace te {
#define TE_MORR_HD inline
inline float morr_div(float a, float b) { return a / b; }
inline float morr_min(float a, float b) { return (b < a || a != a) ? b : a; }
inline float morr_max(float a, float b) { return (a < b || a != a) ? b : a; }
inline float morr_pow(float x, float y) { return te_pow_f64(x, y); }
inline float morr_exp(float x) { return te_exp_f64(x); }
inline float morr_log(float x) { return te_log_f64(x); }
inline float morr_sin(float x) { return sinf(x); }
inline float morr_sqrt(float x) { return sqrtf(x); }
inline float morr_log2(float x) { return te_log2_f64(x); }
inline float morr_atan2(float y, float x) { return te_atan2_f64(y, x); }
}  // namespace te
#include "../../thunderengine-web_b200/csrc/te_morr.cuh"
#include "../../thunderengine-web_b200/csrc/te_refl.cuh"

extern "C" void temh_morr_column(uint32_t* M, const uint32_t* ARG) {
  using namespace te::morr;
  Params p;
  std::memcpy(&p, M + ARG[4 + 0], sizeof p);
  auto fld = [&](int b) { return reinterpret_cast<float*>(M + ARG[4 + b]); };
  Fields F;
  F.T3 = fld(1); F.QV = fld(2); F.QC = fld(3); F.QR = fld(4); F.QI = fld(5); F.QS = fld(6); F.QG = fld(7);
  F.NI = fld(8); F.NS = fld(9); F.NR = fld(10); F.NG = fld(11);
  F.P3 = fld(12); F.RH3 = fld(13); F.DZQ = fld(14);
  F.sfc = fld(15); F.EFFC = fld(16); F.EFFI = fld(17); F.EFFS = fld(18);
  int dorad;
  std::memcpy(&dorad, M + ARG[4 + 19], 4);
  const int gx = (int)ARG[0], gy = (int)ARG[1];
#pragma omp parallel
  {
    std::vector<float> scr((size_t)29 * (p.nz > 0 ? p.nz : 1));
#pragma omp for schedule(dynamic, 16)
    for (int t = 0; t < gx * gy; t++) {
      const int x = t % gx, y = t / gx;
      if (x >= p.nx || y >= p.ny) continue;
      Scratch S{scr.data(), 1u, p.nz};
      column(p, F, S, x, y, dorad);
    }
  }
}

extern "C" void temh_morr_refl10cm(uint32_t* M, const uint32_t* ARG) {
  using namespace te::morr;
  Params p;
  std::memcpy(&p, M + ARG[4 + 0], sizeof p);
  RadarHead h;
  std::memcpy(&h, M + ARG[4 + 1], sizeof h);
  auto fld = [&](int b) { return reinterpret_cast<float*>(M + ARG[4 + b]); };
  RadarFields F;
  F.bs = fld(2); F.bg = fld(3); F.simpson = fld(4);
  F.T = fld(5); F.QR = fld(6); F.QS = fld(7); F.QG = fld(8); F.NR = fld(9); F.NS = fld(10); F.NG = fld(11);
  F.RH = fld(12); F.dbz = fld(13);
  const int gx = (int)ARG[0], gy = (int)ARG[1];
#pragma omp parallel
  {
    std::vector<float> scr((size_t)11 * (p.nz > 0 ? p.nz : 1));
#pragma omp for schedule(dynamic, 16)
    for (int t = 0; t < gx * gy; t++) {
      const int x = t % gx, y = t / gx;
      if (x >= p.nx || y >= p.ny) continue;
      Scratch S{scr.data(), 1u, p.nz};
      refl_column(p, h, F, S, x, y);
    }
  }
}

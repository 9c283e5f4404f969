// Radar reflectivity at 10 cm of the Morrison hydrometeors, one column
// (data/kernels/morr_refl10cm.wgsl), the display diagnostic the reference's encodeDiag
// plays after a step (web/core/micro.js:388-395: grid nx x ny, one thread per column).  As
// te_morr.cuh, it is a function the CUDA kernel runs on the device and a host test build
// runs against the reference's kernel.
//
// Arithmetic: the binary32 operations of the reference kernel in its order, built with
// -fmad=false (fmaf where the WGSL has fma).  Besides te_morr.cuh's functions the includer
// provides, as TE_MORR_HD functions:
//   morr_sqrt(x)      the correctly rounded square root (the kernel's sqrt_cr)
//   morr_log2(x), morr_atan2(y, x)   the WGSL builtins, evaluated in binary64, rounded once
//
// Per-column scratch: 11 arrays of 128 levels in the reference's 1408 words (array
// a = offset / 128, laid out as te_morr.cuh's Scratch).  The reference clears the 1408
// words first; every word read here is written earlier in the same call, so the clears
// are left out.
#pragma once

namespace te {
namespace morr {

// S_MorrRadarHead (morr_refl10cm.wgsl:148-161): the refractive indices of water and ice,
// |K_w|^2, pi^5, lambda^4 and the Rayleigh factors of snow and graupel.
struct RadarHead {
  float mw_re, mw_im, mi_re, mi_im, kw, pi5, lamda4, zfac_s, zfac_g, ocms, obms, ocmg, obmg, pad;
};
static_assert(sizeof(RadarHead) == 14 * 4, "RadarHead mirrors the 14 words of the head buffer");

// S_MorrRadarBin (morr_refl10cm.wgsl:163-170): 6 words per diameter bin.
enum : int { kBinD = 0, kBinDt = 1, kBinX = 2, kBinVg = 3, kBinRhog = 4, kBinGrenz = 5, kBinWords = 6, kBins = 100 };

struct RadarFields {
  const float *T, *QR, *QS, *QG, *NR, *NS, *NG, *RH;
  const float *bs, *bg, *simpson;  // snow and graupel bins, Simpson weights
  float* dbz;
};

struct cplx {
  float re, im;
};

// f_c_mul, f_c_div, f_c_log, f_c_sqrt (morr_refl10cm.wgsl:428-458); |a| is WGSL length.
TE_MORR_HD cplx c_mul(cplx a, cplx b) { return {fmaf(a.re, b.re, -(a.im * b.im)), fmaf(a.re, b.im, a.im * b.re)}; }
TE_MORR_HD cplx c_div(cplx a, cplx b) {
  const float d = fmaf(b.re, b.re, b.im * b.im);
  return {morr_div(fmaf(a.re, b.re, a.im * b.im), d), morr_div(fmaf(a.im, b.re, -(a.re * b.im)), d)};
}
TE_MORR_HD float c_abs(cplx a) { return morr_sqrt(a.re * a.re + a.im * a.im); }
TE_MORR_HD cplx c_log(cplx a) { return {morr_log(c_abs(a)), morr_atan2(a.im, a.re)}; }
TE_MORR_HD cplx c_sqrt(cplx a) {
  const float r = c_abs(a);
  if (r == 0.0f) return {0.0f, 0.0f};
  if (a.re >= 0.0f) {
    const float t = morr_sqrt(0.5f * (r + a.re));
    return {t, morr_div(a.im, 2.0f * t)};
  }
  const float t = morr_sqrt(0.5f * (r - a.re));
  return {morr_div(fabsf(a.im), 2.0f * t), copysignf(t, a.im)};
}

// One Maxwell-Garnett coefficient b_n = 2 m1^2 / (mn^2 - m1^2) *
// (mn^2 / (mn^2 - m1^2) * log(mn^2 / m1^2) - 1), with m1t = m1^2 and mt = mn^2.
TE_MORR_HD cplx mg_coef(cplx m1t, cplx mt) {
  const cplx dm = {mt.re - m1t.re, mt.im - m1t.im};
  const cplx l = c_mul(c_div(mt, dm), c_log(c_div(mt, m1t)));
  return c_mul(c_div({2.0f * m1t.re, 2.0f * m1t.im}, dm), {l.re - 1.0f, l.im - 0.0f});
}

// f_c_mg (morr_refl10cm.wgsl:406-426): the Maxwell-Garnett effective refractive index of
// a three-component mixture with volume fractions v1..v3 (false unless they sum to 1).
TE_MORR_HD bool c_mg(float v1, float v2, float v3, cplx m1, cplx m2, cplx m3, cplx& out) {
  if (fabsf(((v1 + v2) + v3) - 1.0f) > 1e-06f) return false;
  const cplx m1t = c_mul(m1, m1), m2t = c_mul(m2, m2), m3t = c_mul(m3, m3);
  const cplx b2 = mg_coef(m1t, m2t), b3 = mg_coef(m1t, m3t);
  const float w1 = (1.0f - v2) - v3;
  const cplx b3m = c_mul(b3, m3t), b2m = c_mul(b2, m2t);
  const cplx num = {fmaf(v3, b3m.re, fmaf(w1, m1t.re, v2 * b2m.re)), fmaf(v3, b3m.im, fmaf(w1, m1t.im, v2 * b2m.im))};
  const cplx den = {fmaf(v3, b3.re, fmaf(v2, b2.re, w1)), fmaf(v3, b3.im, fmaf(v2, b2.im, 0.0f))};
  out = c_sqrt(c_div(num, den));
  return true;
}

// f_morr_cbrt_cr (morr_refl10cm.wgsl:340-356): x^(1/3) from pow with the binary32 third,
// corrected by one Newton step on the exact residual x - y0^3 (split products) and by
// the exponent's own error, 1/3 - 0.33333334f, times ln x.
TE_MORR_HD float cbrt_cr(float x) {
  const float y0 = morr_pow(x, morr_div(1.0f, 3.0f));
  if (!(x > 0.0f) || fabsf(x) == INFINITY) return y0;
  const float p1 = y0 * y0;
  const float e1 = fmaf(y0, y0, -p1);
  const float p2 = p1 * y0;
  const float e2 = fmaf(p1, y0, -p2);
  const float e3 = e1 * y0;
  const float r = ((x - p2) - e2) - e3;
  const float c = morr_div(r, 3.0f * p1);
  const float t = 9.934107e-09f * morr_log(x);
  return y0 + fmaf(y0, t, c);
}

// f_morr_soak (morr_refl10cm.wgsl:364-404): backscatter of one melting particle of bin b
// (mass x, air-ice volume vg, density rhog, limit grenz) at melted fraction fmelt: the
// water/ice/air volumes, an ice-in-water matrix (Maxwell-Garnett) mixed with air, and the
// Rayleigh term |K|^2 pi^5 D^6 / lambda^4.
TE_MORR_HD float soak(const RadarHead& h, const float* b, float fmelt) {
  const float rho_i = 900.0f, rho_w = 1000.0f;
  const float fm = morr_max(morr_min(fmelt, 1.0f), 0.0f);
  float mra = 0.7f;
  mra = fmaf(1.0f - mra, fm, mra);
  const float x_w = b[kBinX] * fm;
  float volg;
  if (mra <= b[kBinGrenz]) {
    volg = b[kBinVg] * fmaf(-mra, fm, 1.0f);
  } else {
    const float fmgrenz = morr_div(rho_i - b[kBinRhog],
                                   fmaf(mra, rho_i, -b[kBinRhog]) + morr_div(rho_i * b[kBinRhog], rho_w));
    if (fm <= fmgrenz) volg = fmaf(-mra, fm, 1.0f) * b[kBinVg];
    else volg = morr_div(b[kBinX] - x_w, rho_i) + morr_div(x_w, rho_w);
  }
  const float dlarge = morr_pow(morr_div(6.0f, 3.1415927f) * volg, morr_div(1.0f, 3.0f));
  const float volice = morr_div(b[kBinX] - x_w, volg * rho_i);
  const float volwater = morr_div(x_w, rho_w * volg);
  const float volair = (1.0f - volice) - volwater;
  const float v1 = morr_div(volice, morr_max(volice + volwater, 1e-10f));
  const float v2 = 1.0f - v1;
  const cplx ma = {1.0f, 0.0f};
  cplx mtmp, mcore;
  if (!c_mg(v2, 0.0f, v1, {h.mw_re, h.mw_im}, ma, {h.mi_re, h.mi_im}, mtmp)) return 0.0f;
  if (!c_mg(1.0f - volair, volair, 0.0f, mtmp, ma, {2.0f * ma.re, 2.0f * ma.im}, mcore)) return 0.0f;
  const cplx m2 = c_mul(mcore, mcore);
  const cplx k = c_div({m2.re - 1.0f, m2.im - 0.0f}, {m2.re + 2.0f, m2.im + 0.0f});
  const float d3 = (dlarge * dlarge) * dlarge;
  return morr_div(((k.re * k.re + k.im * k.im) * h.pi5) * (d3 * d3), h.lamda4);
}

// Slope 1/lambda and intercept n0 of one species' exponential size distribution from its
// mass and number densities (the reference's three copies for snow, graupel and rain):
// lambda = cbrt(c n / q) clamped to [lmin, lmax], n0 = n lambda / rho, or from q at a clamp.
TE_MORR_HD void slope(float c, float n, float q, float rho, float lmin, float lmax, float& lam, float& n0) {
  lam = cbrt_cr(morr_div(c * n, q));
  n0 = morr_div(n * lam, rho);
  if (lam < lmin) {
    lam = lmin;
    n0 = morr_div(pow4(lam) * q, c);
  } else if (lam > lmax) {
    lam = lmax;
    n0 = morr_div(pow4(lam) * q, c);
  }
}

TE_MORR_HD float pow7(float s) {
  const float s2 = s * s, s4 = s2 * s2;
  return (s4 * s2) * s;
}

// main of morr_refl10cm.wgsl (:464-657) for column (i, j): the Rayleigh reflectivities
// of rain, snow and graupel per level (Z = 720 n0 / lambda^7), in a melting layer (below
// the lowest level k0 over rain above 0 C with snow and graupel above it) the snow and
// graupel terms replaced by the melting-particle integral over 100 bins, then
// dbz = 10 log10((Zr + Zs + Zg) 1e18).
TE_MORR_HD void refl_column(const Params& p, const RadarHead& h, const RadarFields& F, const Scratch& S, int i, int j) {
  const int nk = p.nz;
  const float R1 = 1e-12f, T_0 = 273.15f;
  enum { kQr = 0, kQs = 128, kQg = 256, kT = 384, kIls = 512, kN0s = 640, kIlg = 768, kN0g = 896, kZr = 1024,
         kZs = 1152, kZg = 1280 };
  for (int k = 0; k < nk; k++) {
    const int c = mi(p, i, j, k);
    const float rho = F.RH[c];
    S(kT, k) = F.T[c];
    const float qr = F.QR[c], qs = F.QS[c], qg = F.QG[c], nr = F.NR[c], ns = F.NS[c], ng = F.NG[c];
    const bool lr = qr > R1, ls = qs > R1, lg = qg > R1;
    const float rqr = lr ? qr * rho : R1, rqs = ls ? qs * rho : R1, rqg = lg ? qg * rho : R1;
    S(kQr, k) = rqr;
    S(kQs, k) = rqs;
    S(kQg, k) = rqg;
    const float rnr = nr > R1 ? nr * rho : R1, rns = ns > R1 ? ns * rho : R1, rng = ng > R1 ? ng * rho : R1;
    float lam, n0;
    slope(p.cons[1], rns, rqs, rho, p.lammins, p.lammaxs, lam, n0);
    const float ils = morr_div(1.0f, lam), n0s = n0;
    S(kIls, k) = ils;
    S(kN0s, k) = n0s;
    slope(p.cons[2], rng, rqg, rho, p.lamming, p.lammaxg, lam, n0);
    const float ilg = morr_div(1.0f, lam), n0g = n0;
    S(kIlg, k) = ilg;
    S(kN0g, k) = n0g;
    slope(p.pi * p.rhow, rnr, rqr, rho, p.lamminr, p.lammaxr, lam, n0);
    S(kZr, k) = lr ? (n0 * 720.0f) * pow7(morr_div(1.0f, lam)) : 1e-22f;
    S(kZs, k) = ls ? ((h.zfac_s * n0s) * 720.0f) * pow7(ils) : 1e-22f;
    S(kZg, k) = lg ? ((h.zfac_g * n0g) * 720.0f) * pow7(ilg) : 1e-22f;
  }
  // the melting layer: the first level from the top with rain above 0 C under snow or
  // graupel
  int k0 = 0;
  bool melti = false;
  for (int k = nk - 2; k >= 0; k--) {
    if (S(kT, k) > T_0 && S(kQr, k) > 1e-06f && S(kQs, k + 1) + S(kQg, k + 1) > 1e-05f) {
      k0 = k + 1 > k0 ? k + 1 : k0;
      melti = true;
      break;
    }
  }
  if (melti && k0 >= 1) {
    const float kfac = morr_div(h.lamda4, h.pi5 * h.kw);
    for (int k = k0 - 1; k >= 0; k--) {
      const float fs = morr_min(1.0f - morr_div(S(kQs, k), S(kQs, k0)), 1.0f);
      if (fs > 0.01f && fs < 0.99f && S(kQs, k) > R1) {
        const float n0s = S(kN0s, k), ils = S(kIls, k);
        float eta = 0.0f;
        for (int n = 0; n < kBins; n++) {
          const float* b = F.bs + n * kBinWords;
          const float cb = soak(h, b, fs);
          const float fd = n0s * morr_exp(morr_div(-b[kBinD], ils));
          eta = fmaf((fd * cb) * F.simpson[n], b[kBinDt], eta);
        }
        S(kZs, k) = kfac * eta;
      }
      const float fg = morr_min(1.0f - morr_div(S(kQg, k), S(kQg, k0)), 1.0f);
      if (fg > 0.01f && fg < 0.99f && S(kQg, k) > R1) {
        const float n0g = S(kN0g, k), lamg = morr_div(1.0f, S(kIlg, k));
        float eta = 0.0f;
        for (int n = 0; n < kBins; n++) {
          const float* b = F.bg + n * kBinWords;
          const float cb = soak(h, b, fg);
          const float fd = n0g * morr_exp((-lamg) * b[kBinD]);
          eta = fmaf((fd * cb) * F.simpson[n], b[kBinDt], eta);
        }
        S(kZg, k) = kfac * eta;
      }
    }
  }
  for (int k = 0; k < nk; k++) {
    const float z = (S(kZr, k) + S(kZs, k)) + S(kZg, k);
    F.dbz[mi(p, i, j, k)] = 10.0f * (morr_log2(z * 1e+18f) * 0.30103f);
  }
}

}  // namespace morr
}  // namespace te

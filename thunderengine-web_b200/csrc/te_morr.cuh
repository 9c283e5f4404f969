// Morrison two-moment microphysics, one column (data/kernels/morr_column.wgsl), as a
// function the CUDA kernel (te_kernels.cu, one thread per column) runs on the device; the
// same source compiles for the host, where a test runs it against the reference build.
//
// Arithmetic: the binary32 operations of the reference kernel in its order (the WGSL
// keeps every operation separate with opq(); here the expressions are written with the
// same parenthesisation and built with -fmad=false, so each + - * is one rounding and
// fmaf appears where the WGSL has fma).  The includer provides, as TE_MORR_HD functions:
//   morr_div(a, b)   correctly rounded quotient (div_cr)
//   morr_min/max     WGSL min/max
//   morr_pow, morr_exp, morr_log   the WGSL builtins (evaluated in binary64, rounded once)
//   morr_sin         the WGSL sin builtin (only reached by the gamma function for
//                    non-positive arguments, which no caller passes)
//
// Per-column scratch: the reference gives each column 3712 words, arrays of 128 levels at
// fixed offsets.  Here array a = offset / 128 holds level k at (a * nz + k) * stride of a
// caller-provided buffer (stride = columns of the launch, so a warp's accesses are
// consecutive words); only levels below nz exist.  The reference clears all 3712 words
// first; every word read here is written earlier in the same call (the per-level clears
// of the first loop and the sedimentation's own writes), so those bulk clears are left out.
#pragma once

namespace te {
namespace morr {

// S_MorrParams (morr_column.wgsl:74-146): 5 integers, 64 reals, cons[42], dnu[16], the
// order of the setBytes words.
struct Params {
  int nx, ny, nz, sJ, sK;
  float dt, rdt, tsmall, ai, ac, as_, ar, ag, bi, bc, bs, br, bg, r, rv, cp, ep2, cv, cvv, cpv, cpl, cpi, lv1, lv2,
      ls1, ls2, tmelt, rhosu, rhow, rhoi, rhosn, rhog, aimm, bimm, dcs, mi0, mg0, f1s, f2s, f1r, f2r, g, qsmall, qthr,
      cpw, ci, di, cs, ds, cg, dg, mmult, lammaxi, lammini, lammaxr, lamminr, lammaxs, lammins, lammaxg, lamming, dB,
      ndcnst, pi, drizzleVt;
  float cons[42];
  float dnu[16];
};
static_assert(sizeof(Params) == 127 * 4, "Params mirrors the 127 setBytes words");

struct Fields {
  float *T3, *QV, *QC, *QR, *QI, *QS, *QG, *NI, *NS, *NR, *NG;
  const float *P3, *RH3, *DZQ;
  float *sfc, *EFFC, *EFFI, *EFFS;
};

struct Scratch {
  float* p;
  unsigned stride;
  int nz;
  TE_MORR_HD float& operator()(int off, int k) const { return p[(size_t)((off >> 7) * nz + k) * stride]; }
};

TE_MORR_HD float sq(float x) { return x * x; }
TE_MORR_HD float cube(float x) { return (x * x) * x; }
TE_MORR_HD float pow4(float x) {
  const float t = x * x;
  return t * t;
}

// f_morr_gamma (morr_column.wgsl:340-476): the rational approximation of Cody's gamma in
// binary32, with the reflection for non-positive arguments.
TE_MORR_HD float gamma(float x) {
  const float one = 1.0f, chalf = 0.5f, twelve = 12.0f, two = 2.0f, zero = 0.0f, xbig = 35.04f, xminin = 1.18e-38f,
              eps = 1.19e-07f, xinf = 3.4e+38f, PI = 3.1415927f, xxx = 0.9189385f;
  const float P[8] = {-1.7161851f, 24.765652f, -379.80426f, 629.3312f, 866.9662f, -31451.273f, -36144.414f, 66456.14f};
  const float Q[8] = {-30.84023f, 315.35062f, -1015.1564f, -3107.7717f, 22538.12f, 4755.846f, -134659.95f, -115132.26f};
  const float C[7] = {-0.0019104441f, 0.00084171386f, -0.000595238f, 0.0007936508f, -0.0027777778f, 0.083333336f,
                      0.0057083834f};
  bool parity = false;
  float fact = one, res;
  int n = 0;
  float y = x;
  if (y <= zero) {
    y = -x;
    const float y1 = truncf(y);
    res = y - y1;
    if (res != zero) {
      if (y1 != truncf(y1 * chalf) * two) parity = true;
      fact = morr_div(-PI, morr_sin(PI * res));
      y = y + one;
    } else {
      return xinf;
    }
  }
  if (y < eps) {
    if (y >= xminin) res = morr_div(one, y);
    else return xinf;
  } else if (y < twelve) {
    const float y1 = y;
    float z;
    if (y < one) {
      z = y;
      y = y + one;
    } else {
      n = (int)y - 1;
      y = y - (float)n;
      z = y - one;
    }
    float xnum = zero, xden = one;
    for (int i = 0; i < 8; i++) {
      xnum = (xnum + P[i]) * z;
      xden = fmaf(xden, z, Q[i]);
    }
    res = morr_div(xnum, xden) + one;
    if (y1 < y) {
      res = morr_div(res, y1);
    } else if (y1 > y) {
      for (int i = 0; i < n; i++) {
        res = res * y;
        y = y + one;
      }
    }
  } else {
    if (y <= xbig) {
      const float ysq = y * y;
      float sum = C[6];
      for (int i = 0; i < 6; i++) sum = morr_div(sum, ysq) + C[i];
      sum = (morr_div(sum, y) - y) + xxx;
      sum = fmaf(y - chalf, morr_log(y), sum);
      res = morr_exp(sum);
    } else {
      return xinf;
    }
  }
  if (parity) res = -res;
  if (fact != one) res = morr_div(fact, res);
  return res;
}

// f_morr_lamr (morr_column.wgsl:293-309)
TE_MORR_HD void lamr_of(const Params& p, float q, float& n, float& lam, float& n0) {
  lam = morr_pow(morr_div((p.pi * p.rhow) * n, q), 1.0f / 3.0f);
  n0 = n * lam;
  if (lam < p.lamminr) {
    lam = p.lamminr;
    n0 = morr_div(pow4(lam) * q, p.pi * p.rhow);
    n = morr_div(n0, lam);
  } else if (lam > p.lammaxr) {
    lam = p.lammaxr;
    n0 = morr_div(pow4(lam) * q, p.pi * p.rhow);
    n = morr_div(n0, lam);
  }
}

// f_morr_lamc (morr_column.wgsl:317-338)
TE_MORR_HD void lamc_of(const Params& p, float qc, float& nc, float rho, float& pgam, float& lamc, float& cdist1) {
  pgam = fmaf(0.0005714f, morr_div(nc, 1e+06f) * rho, 0.2714f);
  pgam = morr_div(1.0f, sq(pgam)) - 1.0f;
  pgam = morr_max(pgam, 2.0f);
  pgam = morr_min(pgam, 1e+01f);
  lamc = morr_pow(morr_div((p.cons[26] * nc) * gamma(pgam + 4.0f), qc * gamma(pgam + 1.0f)), 1.0f / 3.0f);
  const float lammin = morr_div(pgam + 1.0f, 6e-05f);
  const float lammax = morr_div(pgam + 1.0f, 1e-06f);
  if (lamc < lammin || lamc > lammax) {
    lamc = lamc < lammin ? lammin : lammax;
    nc = morr_div(morr_exp((fmaf(3.0f, morr_log(lamc), morr_log(qc)) + morr_log(gamma(pgam + 1.0f))) -
                           morr_log(gamma(pgam + 4.0f))),
                  p.cons[26]);
  }
  cdist1 = morr_div(nc, gamma(pgam + 1.0f));
}

// f_morr_lam3 (morr_column.wgsl:478-497)
TE_MORR_HD void lam3_of(float q, float& n, float cons, float d, float lmin, float lmax, float& lam, float& n0) {
  lam = morr_pow(morr_div(cons * n, q), morr_div(1.0f, d));
  n0 = n * lam;
  if (lam < lmin || lam > lmax) {
    lam = lam < lmin ? lmin : lmax;
    n0 = morr_div(morr_pow(lam, d + 1.0f) * q, cons);
    n = morr_div(n0, lam);
  }
}

TE_MORR_HD float esat_liquid(float prs, float t) {
  return morr_min(prs * 0.5f, 611.2f * morr_exp(morr_div(17.67f * (t - 273.15f), t - 29.65f)));
}
TE_MORR_HD float esat_ice(float prs, float t) {
  return morr_min(prs * 0.5f, 611.2f * morr_exp(morr_div(21.874557f * (t - 273.15f), t - 7.66f)));
}

// f_morr_satadj2 (morr_column.wgsl:504-552): saturation adjustment, at most 100 iterations.
TE_MORR_HD void satadj2(const Params& p, float& tnew, float& prs, float& qvnew, float& qcnew, float qrnew, float qinew,
                        float qsnew, float qgnew, float rho) {
  const float converge = 2.0f * p.tsmall;
  float esl = esat_liquid(prs, tnew);
  float qvs = morr_div(p.ep2 * esl, prs - esl);
  if (qcnew > p.qsmall || qvnew > qvs) {
    const float ql = morr_max(0.0f, qcnew + qrnew);
    const float qi = morr_max(0.0f, (qinew + qsnew) + qgnew);
    const float cvml = fmaf(p.cpi, qi, fmaf(p.cpl, ql, fmaf(p.cvv, qvnew, p.cv)));
    const float lhv = fmaf(-p.lv2, tnew, p.lv1);
    const float t1 = morr_div(fmaf(-p.rv, tnew, lhv), cvml);
    const float d1 = (t1 * 17.67f) * 243.5f;
    int n = 0;
    float tlast = tnew;
    bool doit = true;
    while (doit) {
      n = n + 1;
      float dqv = morr_div(qvs - qvnew, 1.0f + morr_div(d1 * qvs, sq(tnew - 29.65f)));
      dqv = morr_min(dqv, qcnew);
      if (qvnew + dqv < 1e-20f) dqv = 1e-20f - qvnew;
      qvnew = qvnew + dqv;
      qcnew = qcnew - dqv;
      tnew = fmaf(-dqv, t1, tnew);
      prs = (rho * fmaf(p.rv, qvnew, p.r)) * tnew;
      doit = false;
      if (fabsf(tnew - tlast) > converge) {
        tlast = tnew;
        esl = esat_liquid(prs, tnew);
        qvs = morr_div(p.ep2 * esl, prs - esl);
        doit = true;
      }
      if (n == 100) doit = false;
    }
  }
}

// Collection rates of rain with snow or graupel (the pracs / pracg forms of the reference):
// cons41 * (((sqrt-term * rho) * n0r) * n0x / lamr^3) * (5/(lamr^3 lamx) + 2/(lamr^2 lamx^2)
// + 0.5/(lamr lamx^3)), with the fall-speed difference term of the reference.
TE_MORR_HD float rain_collect(const Params& p, float umx, float umr, float rho, float n0rr, float n0x, float lamr,
                              float lamx) {
  return p.cons[41] * (morr_div(((morr_pow(fmaf(0.08f * umx, umr, sq(fmaf(1.2f, umr, -(0.95f * umx)))), 0.5f) * rho) *
                                 n0rr) * n0x,
                                cube(lamr)) *
                       ((morr_div(5.0f, cube(lamr) * lamx) + morr_div(2.0f, sq(lamr) * sq(lamx))) +
                        morr_div(0.5f, lamr * cube(lamx))));
}
TE_MORR_HD float rain_collect_n(const Params& p, float unr, float unx, float rho, float n0rr, float n0x, float lamr,
                                float lamx) {
  return (((p.cons[32] * rho) * morr_pow(fmaf(1.7f, sq(unr - unx), (0.3f * unr) * unx), 0.5f)) * n0rr) * n0x *
         ((morr_div(1.0f, cube(lamr) * lamx) + morr_div(1.0f, sq(lamr) * sq(lamx))) + morr_div(1.0f, lamr * cube(lamx)));
}

// The ventilation bracket f1/lam^2 + f2 (a rho/mu)^(1/2) scn^(1/3) cons[ci] / lam^cons[ce]
// of rain (f1r, f2r), snow and graupel (f1s, f2s); the depositional growth factors are
// 2 pi n0 rho dv times it, the melting rates 2 pi n0 kap (T0 - T) / Lf times it.
TE_MORR_HD float vent_y(float f1, float f2, float a, float rho, float mu, float scn, float consi, float lam, float conse) {
  return morr_div(f1, lam * lam) +
         morr_div(((f2 * morr_pow(morr_div(a * rho, mu), 0.5f)) * morr_pow(scn, 1.0f / 3.0f)) * consi, morr_pow(lam, conse));
}

TE_MORR_HD int mi(const Params& p, int i, int j, int k) { return (i + 3) + p.sJ * ((j + 3) + p.sK * k); }

// The column (i, j): morr_column.wgsl main, in its order.  Phase 1 (levels 0..nz-1): the
// process rates of every level and their tendencies (warm branch for T >= T0, cold branch
// below), the saturation adjustment of the provisional state; phase 2 (if any level was
// active): sedimentation of rain, ice, cloud water, snow and graupel with the substep count
// of each species; phase 3: the tendencies applied, the instantaneous processes and the
// effective radii; last, the surface precipitation.
TE_MORR_HD void column(const Params& p, const Fields& F, const Scratch& S, int i, int j, int dorad) {
  const int nk = p.nz;
  if (dorad != 0) {
    for (int k = 0; k < nk; k++) {
      const int c = mi(p, i, j, k);
      F.EFFC[c] = 25.0f * 1e-06f;
      F.EFFI[c] = morr_min(1.4e+02f, 25.0f) * 1e-06f;
      F.EFFS[c] = 25.0f * 1e-06f;
    }
  }
  const float DT = p.dt, RDT = p.rdt, QSMALL = p.qsmall, TMELT = p.tmelt;
  for (int k = 0; k < nk; k++) {
    for (int a = 0; a <= 1408; a += 128) S(a, k) = 0.0f;
    S(1920, k) = 0.0f;
    S(2048, k) = 0.0f;
    for (int s = 0; s < 5; s++) S(2304 + s * 128, k) = 0.0f;
  }
  bool ltrue = false;
  for (int k = 0; k < nk; k++) {
    const int c = mi(p, i, j, k);
    float t3 = F.T3[c], qv3 = F.QV[c], qc3 = F.QC[c], qr3 = F.QR[c], qi3 = F.QI[c], qni3 = F.QS[c], qg3 = F.QG[c];
    float ni3 = F.NI[c], ns3 = F.NS[c], nr3 = F.NR[c], ng3 = F.NG[c];
    float nc3 = S(2048, k);
    float pres = F.P3[c];
    const float rho = F.RH3[c];
    const float xxlv = fmaf(-p.lv2, t3, p.lv1);
    const float xxls = fmaf(-p.ls2, t3, p.ls1);
    const float cpm = p.cp * fmaf(0.887f, qv3, 1.0f);
    const float cvm = morr_div(1.0f, fmaf(p.cpi, (qi3 + qni3) + qg3, fmaf(p.cpl, qc3 + qr3, fmaf(p.cvv, qv3, p.cv))));
    const float ecnd = fmaf(-p.rv, t3, xxlv) * cvm;
    const float edep = fmaf(-p.rv, t3, xxls) * cvm;
    const float efrz = (xxls - xxlv) * cvm;
    S(1536, k) = ecnd;
    S(1664, k) = edep;
    S(1792, k) = efrz;
    const float evs = esat_liquid(pres, t3);
    float eis = esat_ice(pres, t3);
    if (eis > evs) eis = evs;
    const float qvs = morr_div(p.ep2 * evs, pres - evs);
    const float qvi = morr_div(p.ep2 * eis, pres - eis);
    const float qvqvs = morr_div(qv3, qvs);
    const float qvqvsi = morr_div(qv3, qvi);
    if (qvqvs < 0.9f) {
      if (qr3 < p.qthr) {
        qv3 = qv3 + qr3;
        t3 = fmaf(-qr3, ecnd, t3);
        qr3 = 0.0f;
      }
      if (qc3 < p.qthr) {
        qv3 = qv3 + qc3;
        t3 = fmaf(-qc3, ecnd, t3);
        qc3 = 0.0f;
      }
    }
    if (qvqvsi < 0.9f) {
      if (qi3 < p.qthr) {
        qv3 = qv3 + qi3;
        t3 = fmaf(-qi3, edep, t3);
        qi3 = 0.0f;
      }
      if (qni3 < p.qthr) {
        qv3 = qv3 + qni3;
        t3 = fmaf(-qni3, edep, t3);
        qni3 = 0.0f;
      }
      if (qg3 < p.qthr) {
        qv3 = qv3 + qg3;
        t3 = fmaf(-qg3, edep, t3);
        qg3 = 0.0f;
      }
    }
    const float xlf = xxls - xxlv;
    if (qc3 < QSMALL) { qc3 = 0.0f; nc3 = 0.0f; }
    if (qr3 < QSMALL) { qr3 = 0.0f; nr3 = 0.0f; }
    if (qi3 < QSMALL) { qi3 = 0.0f; ni3 = 0.0f; }
    if (qni3 < QSMALL) { qni3 = 0.0f; ns3 = 0.0f; }
    if (qg3 < QSMALL) { qg3 = 0.0f; ng3 = 0.0f; }
    const float mu = morr_div(1.496e-06f * morr_pow(t3, 1.5f), t3 + 1.2e+02f);
    const float dum = morr_pow(morr_div(p.rhosu, rho), 0.54f);
    const float ain = morr_pow(morr_div(p.rhosu, rho), 0.35f) * p.ai;
    const float arn = dum * p.ar;
    const float asn = dum * p.as_;
    const float acn = morr_div(p.g * p.rhow, 18.0f * mu);
    const float agn = dum * p.ag;
    S(2176, k) = acn;
    float lami = 0.0f;
    bool skip200 = false;
    if (qc3 < QSMALL && qi3 < QSMALL && qni3 < QSMALL && qr3 < QSMALL && qg3 < QSMALL) {
      if (t3 < TMELT && qvqvsi < 0.999f) skip200 = true;
      if (t3 >= TMELT && qvqvs < 0.999f) skip200 = true;
    }
    if (!skip200) {
      const float kap = 1414.0f * mu;
      const float dv = morr_div(8.794e-05f * morr_pow(t3, 1.81f), pres);
      const float scn = morr_div(mu, rho * dv);
      const float dumr = p.rv * sq(t3);
      const float dqsdt = morr_div(xxlv * qvs, dumr);
      const float dqsidt = morr_div(xxls * qvi, dumr);
      const float abi = 1.0f + morr_div(dqsidt * xxls, cpm);
      const float ab = 1.0f + morr_div(dqsdt * xxlv, cpm);
      if (t3 >= TMELT) {
        // ---------------------------------------------------------------- warm branch
        nc3 = morr_div(p.ndcnst * 1e+06f, rho);
        if (qni3 < 1e-06f) {
          qr3 = qr3 + qni3;
          nr3 = nr3 + ns3;
          t3 = fmaf(-qni3, efrz, t3);
          qni3 = 0.0f;
          ns3 = 0.0f;
        }
        if (qg3 < 1e-06f) {
          qr3 = qr3 + qg3;
          nr3 = nr3 + ng3;
          t3 = fmaf(-qg3, efrz, t3);
          qg3 = 0.0f;
          ng3 = 0.0f;
        }
        const bool goto300 = qc3 < QSMALL && qni3 < 1e-08f && qr3 < QSMALL && qg3 < 1e-08f;
        if (!goto300) {
          ns3 = morr_max(0.0f, ns3);
          nr3 = morr_max(0.0f, nr3);
          ng3 = morr_max(0.0f, ng3);
          float lamr = 0.0f, n0rr = 0.0f, lamc = 0.0f, pgam = 0.0f, cdist1 = 0.0f, lams = 0.0f, n0s = 0.0f, lamg = 0.0f,
                n0g = 0.0f;
          if (qr3 >= QSMALL) lamr_of(p, qr3, nr3, lamr, n0rr);
          if (qc3 >= QSMALL) lamc_of(p, qc3, nc3, rho, pgam, lamc, cdist1);
          if (qni3 >= QSMALL) lam3_of(qni3, ns3, p.cons[1], p.ds, p.lammins, p.lammaxs, lams, n0s);
          if (qg3 >= QSMALL) lam3_of(qg3, ng3, p.cons[2], p.dg, p.lamming, p.lammaxg, lamg, n0g);
          float prc = 0.0f, nprc = 0.0f, nprc1 = 0.0f, pra = 0.0f, npra = 0.0f, nragg = 0.0f, nsmlts = 0.0f,
                nsmltr = 0.0f, evpms = 0.0f, pre = 0.0f, nsubr = 0.0f, pracg = 0.0f, npracg = 0.0f, psmlt = 0.0f,
                pgmlt = 0.0f, evpmg = 0.0f, pracs = 0.0f, ngmltg = 0.0f, ngmltr = 0.0f;
          if (qc3 >= 1e-06f) {
            prc = (1.35e+03f * morr_pow(qc3, 2.47f)) * morr_pow(morr_div(nc3, 1e+06f) * rho, -1.79f);
            nprc1 = morr_div(prc, p.cons[29]);
            nprc = morr_div(prc, morr_div(qc3, nc3));
            nprc = morr_min(nprc, morr_div(nc3, DT));
            nprc1 = morr_min(nprc1, nprc);
          }
          if (qr3 >= 1e-08f && qni3 >= 1e-08f) {
            float ums = morr_div(asn * p.cons[3], morr_pow(lams, p.bs));
            float umr = morr_div(arn * p.cons[4], morr_pow(lamr, p.br));
            float uns = morr_div(asn * p.cons[5], morr_pow(lams, p.bs));
            float unr = morr_div(arn * p.cons[6], morr_pow(lamr, p.br));
            const float d = morr_pow(morr_div(p.rhosu, rho), 0.54f);
            ums = morr_min(ums, 1.2f * d);
            uns = morr_min(uns, 1.2f * d);
            umr = morr_min(umr, 9.1f * d);
            unr = morr_min(unr, 9.1f * d);
            (void)uns;
            (void)unr;
            pracs = rain_collect(p, ums, umr, rho, n0rr, n0s, lamr, lams);
          }
          if (qr3 >= 1e-08f && qg3 >= 1e-08f) {
            float umg = morr_div(agn * p.cons[7], morr_pow(lamg, p.bg));
            float umr = morr_div(arn * p.cons[4], morr_pow(lamr, p.br));
            float ung = morr_div(agn * p.cons[8], morr_pow(lamg, p.bg));
            float unr = morr_div(arn * p.cons[6], morr_pow(lamr, p.br));
            const float d = morr_pow(morr_div(p.rhosu, rho), 0.54f);
            umg = morr_min(umg, 2e+01f * d);
            ung = morr_min(ung, 2e+01f * d);
            umr = morr_min(umr, 9.1f * d);
            unr = morr_min(unr, 9.1f * d);
            pracg = rain_collect(p, umg, umr, rho, n0rr, n0g, lamr, lamg);
            const float dd = morr_div(pracg, 5.2e-07f);
            npracg = rain_collect_n(p, unr, ung, rho, n0rr, n0g, lamr, lamg);
            npracg = npracg - dd;
          }
          if (qr3 >= 1e-08f && qc3 >= 1e-08f) {
            const float d = qc3 * qr3;
            pra = 67.0f * morr_pow(d, 1.15f);
            npra = morr_div(pra, morr_div(qc3, nc3));
          }
          if (qr3 >= 1e-08f) {
            const float dum1 = p.dB;
            float d = 0.0f;
            if (morr_div(1.0f, lamr) < dum1) {
              d = 1.0f;
            } else if (morr_div(1.0f, lamr) >= dum1) {
              d = 2.0f - morr_exp(2.3e+03f * (morr_div(1.0f, lamr) - dum1));
            }
            nragg = (((-5.78f) * d) * qr3) * nr3 * rho;
          }
          float epsr;
          if (qr3 >= QSMALL) {
            epsr = ((((2.0f * p.pi) * n0rr) * rho) * dv) * vent_y(p.f1r, p.f2r, arn, rho, mu, scn, p.cons[9], lamr, p.cons[34]);
          } else {
            epsr = 0.0f;
          }
          if (qv3 < qvs) {
            pre = morr_div(epsr * (qv3 - qvs), ab);
            pre = morr_min(pre, 0.0f);
            const float d = fmaf(-pre, DT, qv3);
            if (d > qvs) pre = morr_div(qv3 - qvs, DT);
          } else {
            pre = 0.0f;
          }
          if (qni3 >= 1e-08f) {
            const float d = (morr_div(-p.cpw, xlf) * (t3 - 273.15f)) * pracs;
            psmlt = fmaf(morr_div((((2.0f * p.pi) * n0s) * kap) * (TMELT - t3), xlf),
                         vent_y(p.f1s, p.f2s, asn, rho, mu, scn, p.cons[10], lams, p.cons[35]), d);
            if (qvqvs < 1.0f) {
              const float epss =
                  ((((2.0f * p.pi) * n0s) * rho) * dv) * vent_y(p.f1s, p.f2s, asn, rho, mu, scn, p.cons[10], lams, p.cons[35]);
              evpms = morr_div((qv3 - qvs) * epss, ab);
              evpms = morr_max(evpms, psmlt);
              psmlt = psmlt - evpms;
            }
          }
          if (qg3 >= 1e-08f) {
            const float d = (morr_div(-p.cpw, xlf) * (t3 - 273.15f)) * pracg;
            pgmlt = fmaf(morr_div((((2.0f * p.pi) * n0g) * kap) * (TMELT - t3), xlf),
                         vent_y(p.f1s, p.f2s, agn, rho, mu, scn, p.cons[11], lamg, p.cons[36]), d);
            if (qvqvs < 1.0f) {
              const float epsg =
                  ((((2.0f * p.pi) * n0g) * rho) * dv) * vent_y(p.f1s, p.f2s, agn, rho, mu, scn, p.cons[11], lamg, p.cons[36]);
              evpmg = morr_div((qv3 - qvs) * epsg, ab);
              evpmg = morr_max(evpmg, pgmlt);
              pgmlt = pgmlt - evpmg;
            }
          }
          pracg = 0.0f;
          pracs = 0.0f;
          float d = (prc + pra) * DT;
          if (d > qc3 && qc3 >= QSMALL) {
            const float ratio = morr_div(qc3, d);
            prc = prc * ratio;
            pra = pra * ratio;
          }
          d = ((-psmlt - evpms) + pracs) * DT;
          if (d > qni3 && qni3 >= QSMALL) {
            const float ratio = morr_div(qni3, d);
            psmlt = psmlt * ratio;
            evpms = evpms * ratio;
            pracs = pracs * ratio;
          }
          d = ((-pgmlt - evpmg) + pracg) * DT;
          if (d > qg3 && qg3 >= QSMALL) {
            const float ratio = morr_div(qg3, d);
            pgmlt = pgmlt * ratio;
            evpmg = evpmg * ratio;
            pracg = pracg * ratio;
          }
          d = ((((((-pracs - pracg) - pre) - pra) - prc) + psmlt) + pgmlt) * DT;
          if (d > qr3 && qr3 >= QSMALL) {
            const float ratio = morr_div((((((morr_div(qr3, DT) + pracs) + pracg) + pra) + prc) - psmlt) - pgmlt, -pre);
            pre = pre * ratio;
          }
          S(0, k) = S(0, k) + ((-pre - evpms) - evpmg);
          S(128, k) = S(128, k) + fmaf(((psmlt + pgmlt) - pracs) - pracg, efrz, fmaf(pre, ecnd, (evpms + evpmg) * edep));
          S(256, k) = S(256, k) + (-pra - prc);
          S(640, k) = S(640, k) + (((((pre + pra) + prc) - psmlt) - pgmlt) + pracs) + pracg;
          S(512, k) = S(512, k) + ((psmlt + evpms) - pracs);
          S(768, k) = S(768, k) + ((pgmlt + evpmg) - pracg);
          S(1408, k) = S(1408, k) + (-npra - nprc);
          S(1152, k) = S(1152, k) + ((nprc1 + nragg) - npracg);
          if (pre < 0.0f) {
            float dd = morr_div(pre * DT, qr3);
            dd = morr_max(-1.0f, dd);
            nsubr = morr_div(dd * nr3, DT);
          }
          if (evpms + psmlt < 0.0f) {
            float dd = morr_div((evpms + psmlt) * DT, qni3);
            dd = morr_max(-1.0f, dd);
            nsmlts = morr_div(dd * ns3, DT);
          }
          if (psmlt < 0.0f) {
            float dd = morr_div(psmlt * DT, qni3);
            dd = morr_max(-1.0f, dd);
            nsmltr = morr_div(dd * ns3, DT);
          }
          if (evpmg + pgmlt < 0.0f) {
            float dd = morr_div((evpmg + pgmlt) * DT, qg3);
            dd = morr_max(-1.0f, dd);
            ngmltg = morr_div(dd * ng3, DT);
          }
          if (pgmlt < 0.0f) {
            float dd = morr_div(pgmlt * DT, qg3);
            dd = morr_max(-1.0f, dd);
            ngmltr = morr_div(dd * ng3, DT);
          }
          S(1024, k) = S(1024, k) + nsmlts;
          S(1280, k) = S(1280, k) + ngmltg;
          S(1152, k) = S(1152, k) + ((nsubr - nsmltr) - ngmltr);
        }
        {
          float dumt = fmaf(DT, S(128, k), t3);
          float dumqv = fmaf(DT, S(0, k), qv3);
          float dumqc = fmaf(DT, S(256, k), qc3);
          const float dumqr = fmaf(DT, S(640, k), qr3);
          const float dummqs = fmaf(DT, S(512, k), qni3);
          const float dumqg = fmaf(DT, S(768, k), qg3);
          const float dumqi = 0.0f;
          pres = (rho * dumt) * fmaf(p.rv, dumqv, p.r);
          const float saveqc = dumqc, savet = dumt;
          satadj2(p, dumt, pres, dumqv, dumqc, dumqr, dumqi, dummqs, dumqg, rho);
          if (fabsf(dumt - savet) >= 0.0001f) {
            const float pccv = (dumqc - saveqc) * RDT;
            S(0, k) = S(0, k) - pccv;
            S(256, k) = S(256, k) + pccv;
            S(128, k) = fmaf(dumt - savet, RDT, S(128, k));
          }
        }
      } else {
        // ---------------------------------------------------------------- cold branch
        nc3 = morr_div(p.ndcnst * 1e+06f, rho);
        ni3 = morr_max(0.0f, ni3);
        ns3 = morr_max(0.0f, ns3);
        nr3 = morr_max(0.0f, nr3);
        ng3 = morr_max(0.0f, ng3);
        float n0i = 0.0f, lamr = 0.0f, n0rr = 0.0f, lamc = 0.0f, pgam = 0.0f, cdist1 = 0.0f, lams = 0.0f, n0s = 0.0f,
              lamg = 0.0f, n0g = 0.0f;
        if (qi3 >= QSMALL) lam3_of(qi3, ni3, p.cons[12], p.di, p.lammini, p.lammaxi, lami, n0i);
        if (qr3 >= QSMALL) lamr_of(p, qr3, nr3, lamr, n0rr);
        if (qc3 >= QSMALL) lamc_of(p, qc3, nc3, rho, pgam, lamc, cdist1);
        if (qni3 >= QSMALL) lam3_of(qni3, ns3, p.cons[1], p.ds, p.lammins, p.lammaxs, lams, n0s);
        if (qg3 >= QSMALL) lam3_of(qg3, ng3, p.cons[2], p.dg, p.lamming, p.lammaxg, lamg, n0g);
        float mnuccc = 0.0f, nnuccc = 0.0f, prc = 0.0f, nprc = 0.0f, nprc1 = 0.0f, nsagg = 0.0f, psacws = 0.0f,
              npsacws = 0.0f, psacwi = 0.0f, npsacwi = 0.0f, pracs = 0.0f, npracs = 0.0f, nmults = 0.0f, qmults = 0.0f,
              nmultr = 0.0f, qmultr = 0.0f, nmultg = 0.0f, qmultg = 0.0f, nmultrg = 0.0f, qmultrg = 0.0f, mnuccr = 0.0f,
              nnuccr = 0.0f, pra = 0.0f, npra = 0.0f, nragg = 0.0f, prci = 0.0f, nprci = 0.0f, prai = 0.0f, nprai = 0.0f,
              nnuccd = 0.0f, mnuccd = 0.0f, pcc = 0.0f, pre = 0.0f, prd = 0.0f, prds = 0.0f, eprd = 0.0f, eprds = 0.0f,
              nsubi = 0.0f, nsubs = 0.0f, nsubr = 0.0f, piacr = 0.0f, niacr = 0.0f, praci = 0.0f, piacrs = 0.0f,
              niacrs = 0.0f, pracis = 0.0f, pracg = 0.0f, psacr = 0.0f, psacwg = 0.0f, pgsacw = 0.0f, pgracs = 0.0f,
              prdg = 0.0f, eprdg = 0.0f, npracg = 0.0f, npsacwg = 0.0f, nscng = 0.0f, ngracs = 0.0f, nsubg = 0.0f;
        if (qc3 >= QSMALL && t3 < 269.15f) {
          const float nacnt = morr_exp(fmaf(0.262f, TMELT - t3, -2.8f)) * 1e+03f;
          const float d = morr_div(morr_div(7.37f * t3, (288.0f * 1e+01f) * pres), 1e+02f);
          const float dap = morr_div((p.cons[37] * t3) * (1.0f + morr_div(d, 1e-07f)), mu);
          mnuccc = ((p.cons[38] * dap) * nacnt) *
                   morr_exp(fmaf(-4.0f, morr_log(lamc), morr_log(cdist1) + morr_log(gamma(pgam + 5.0f))));
          nnuccc = morr_div(((((2.0f * p.pi) * dap) * nacnt) * cdist1) * gamma(pgam + 2.0f), lamc);
          mnuccc = fmaf(p.cons[39] * morr_exp(fmaf(-6.0f, morr_log(lamc), morr_log(cdist1) + morr_log(gamma(7.0f + pgam)))),
                        morr_exp(p.aimm * (273.15f - t3)) - 1.0f, mnuccc);
          nnuccc = fmaf(p.cons[40] * morr_exp(fmaf(-3.0f, morr_log(lamc), morr_log(cdist1) + morr_log(gamma(pgam + 4.0f)))),
                        morr_exp(p.aimm * (273.15f - t3)) - 1.0f, nnuccc);
          nnuccc = morr_min(nnuccc, morr_div(nc3, DT));
        }
        if (qc3 >= 1e-06f) {
          prc = (1.35e+03f * morr_pow(qc3, 2.47f)) * morr_pow(morr_div(nc3, 1e+06f) * rho, -1.79f);
          nprc1 = morr_div(prc, p.cons[29]);
          nprc = morr_div(prc, morr_div(qc3, nc3));
          nprc = morr_min(nprc, morr_div(nc3, DT));
          nprc1 = morr_min(nprc1, nprc);
        }
        if (qni3 >= 1e-08f) {
          nsagg = morr_div(((p.cons[15] * asn) * morr_pow(rho, morr_div(2.0f + p.bs, 3.0f))) *
                               morr_pow(qni3, morr_div(2.0f + p.bs, 3.0f)) *
                               morr_pow(ns3 * rho, morr_div(4.0f - p.bs, 3.0f)),
                           rho);
        }
        if (qni3 >= 1e-08f && qc3 >= QSMALL) {
          psacws = morr_div((((p.cons[13] * asn) * qc3) * rho) * n0s, morr_pow(lams, p.bs + 3.0f));
          npsacws = morr_div((((p.cons[13] * asn) * nc3) * rho) * n0s, morr_pow(lams, p.bs + 3.0f));
        }
        if (qg3 >= 1e-08f && qc3 >= QSMALL) {
          psacwg = morr_div((((p.cons[14] * agn) * qc3) * rho) * n0g, morr_pow(lamg, p.bg + 3.0f));
          npsacwg = morr_div((((p.cons[14] * agn) * nc3) * rho) * n0g, morr_pow(lamg, p.bg + 3.0f));
        }
        if (qi3 >= 1e-08f && qc3 >= QSMALL) {
          if (morr_div(1.0f, lami) >= 0.0001f) {
            psacwi = morr_div((((p.cons[16] * ain) * qc3) * rho) * n0i, morr_pow(lami, p.bi + 3.0f));
            npsacwi = morr_div((((p.cons[16] * ain) * nc3) * rho) * n0i, morr_pow(lami, p.bi + 3.0f));
          }
        }
        if (qr3 >= 1e-08f && qni3 >= 1e-08f) {
          float ums = morr_div(asn * p.cons[3], morr_pow(lams, p.bs));
          float umr = morr_div(arn * p.cons[4], morr_pow(lamr, p.br));
          float uns = morr_div(asn * p.cons[5], morr_pow(lams, p.bs));
          float unr = morr_div(arn * p.cons[6], morr_pow(lamr, p.br));
          const float d = morr_pow(morr_div(p.rhosu, rho), 0.54f);
          ums = morr_min(ums, 1.2f * d);
          uns = morr_min(uns, 1.2f * d);
          umr = morr_min(umr, 9.1f * d);
          unr = morr_min(unr, 9.1f * d);
          pracs = rain_collect(p, ums, umr, rho, n0rr, n0s, lamr, lams);
          npracs = rain_collect_n(p, unr, uns, rho, n0rr, n0s, lamr, lams);
          pracs = morr_min(pracs, morr_div(qr3, DT));
          if (qni3 >= 0.0001f && qr3 >= 0.0001f) {
            psacr = p.cons[31] *
                    (morr_div(((morr_pow(fmaf(0.08f * ums, umr, sq(fmaf(1.2f, umr, -(0.95f * ums)))), 0.5f) * rho) * n0rr) *
                                  n0s,
                              cube(lams)) *
                     ((morr_div(5.0f, cube(lams) * lamr) + morr_div(2.0f, sq(lams) * sq(lamr))) +
                      morr_div(0.5f, lams * cube(lamr))));
          }
        }
        if (qr3 >= 1e-08f && qg3 >= 1e-08f) {
          float umg = morr_div(agn * p.cons[7], morr_pow(lamg, p.bg));
          float umr = morr_div(arn * p.cons[4], morr_pow(lamr, p.br));
          float ung = morr_div(agn * p.cons[8], morr_pow(lamg, p.bg));
          float unr = morr_div(arn * p.cons[6], morr_pow(lamr, p.br));
          const float d = morr_pow(morr_div(p.rhosu, rho), 0.54f);
          umg = morr_min(umg, 2e+01f * d);
          ung = morr_min(ung, 2e+01f * d);
          umr = morr_min(umr, 9.1f * d);
          unr = morr_min(unr, 9.1f * d);
          pracg = rain_collect(p, umg, umr, rho, n0rr, n0g, lamr, lamg);
          npracg = rain_collect_n(p, unr, ung, rho, n0rr, n0g, lamr, lamg);
          pracg = morr_min(pracg, morr_div(qr3, DT));
        }
        // rime splintering (Hallett-Mossop) on snow, then on graupel
        if (qni3 >= 0.0001f && (qc3 >= 0.0005f || qr3 >= 0.0001f) && (psacws > 0.0f || pracs > 0.0f) && t3 < 270.16f &&
            t3 > 265.16f) {
          float fmult = 0.0f;
          if (t3 > 270.16f) fmult = 0.0f;
          else if (t3 <= 270.16f && t3 > 268.16f) fmult = morr_div(270.16f - t3, 2.0f);
          else if (t3 >= 265.16f && t3 <= 268.16f) fmult = morr_div(t3 - 265.16f, 3.0f);
          else if (t3 < 265.16f) fmult = 0.0f;
          if (psacws > 0.0f) {
            nmults = ((3.5e+05f * psacws) * fmult) * 1e+03f;
            qmults = nmults * p.mmult;
            qmults = morr_min(qmults, psacws);
            psacws = psacws - qmults;
          }
          if (pracs > 0.0f) {
            nmultr = ((3.5e+05f * pracs) * fmult) * 1e+03f;
            qmultr = nmultr * p.mmult;
            qmultr = morr_min(qmultr, pracs);
            pracs = pracs - qmultr;
          }
        }
        if (qg3 >= 0.0001f && (qc3 >= 0.0005f || qr3 >= 0.0001f) && (psacwg > 0.0f || pracg > 0.0f) && t3 < 270.16f &&
            t3 > 265.16f) {
          float fmult = 0.0f;
          if (t3 > 270.16f) fmult = 0.0f;
          else if (t3 <= 270.16f && t3 > 268.16f) fmult = morr_div(270.16f - t3, 2.0f);
          else if (t3 >= 265.16f && t3 <= 268.16f) fmult = morr_div(t3 - 265.16f, 3.0f);
          else if (t3 < 265.16f) fmult = 0.0f;
          if (psacwg > 0.0f) {
            nmultg = ((3.5e+05f * psacwg) * fmult) * 1e+03f;
            qmultg = nmultg * p.mmult;
            qmultg = morr_min(qmultg, psacwg);
            psacwg = psacwg - qmultg;
          }
          if (pracg > 0.0f) {
            nmultrg = ((3.5e+05f * pracg) * fmult) * 1e+03f;
            qmultrg = nmultrg * p.mmult;
            qmultrg = morr_min(qmultrg, pracg);
            pracg = pracg - qmultrg;
          }
        }
        if (psacws > 0.0f && qni3 >= 0.0001f && qc3 >= 0.0005f) {
          pgsacw = morr_min(psacws, morr_div(((((p.cons[17] * DT) * n0s) * qc3) * qc3) * asn * asn,
                                             rho * morr_pow(lams, fmaf(2.0f, p.bs, 2.0f))));
          const float d = morr_max(morr_div(p.rhosn, p.rhog - p.rhosn) * pgsacw, 0.0f);
          nscng = morr_div(d, p.mg0) * rho;
          nscng = morr_min(nscng, morr_div(ns3, DT));
          psacws = psacws - pgsacw;
        }
        if (pracs > 0.0f && qni3 >= 0.0001f && qr3 >= 0.0001f) {
          const float cs4 = cube(morr_div(4.0f, lams)), cr4 = cube(morr_div(4.0f, lamr));
          float d = morr_div((p.cons[18] * cs4) * cs4, fmaf(p.cons[18] * cs4, cs4, (p.cons[19] * cr4) * cr4));
          d = morr_min(d, 1.0f);
          d = morr_max(d, 0.0f);
          pgracs = (1.0f - d) * pracs;
          ngracs = (1.0f - d) * npracs;
          ngracs = morr_min(ngracs, morr_div(nr3, DT));
          ngracs = morr_min(ngracs, morr_div(ns3, DT));
          pracs = pracs - pgracs;
          npracs = npracs - ngracs;
          psacr = psacr * (1.0f - d);
        }
        if (t3 < 269.15f && qr3 >= QSMALL) {
          mnuccr = (p.cons[20] * nr3) * morr_div(morr_div(morr_exp(p.aimm * (273.15f - t3)) - 1.0f, cube(lamr)), cube(lamr));
          nnuccr = morr_div(((p.pi * nr3) * p.bimm) * (morr_exp(p.aimm * (273.15f - t3)) - 1.0f), cube(lamr));
          nnuccr = morr_min(nnuccr, morr_div(nr3, DT));
        }
        if (qr3 >= 1e-08f && qc3 >= 1e-08f) {
          const float d = qc3 * qr3;
          pra = 67.0f * morr_pow(d, 1.15f);
          npra = morr_div(pra, morr_div(qc3, nc3));
        }
        if (qr3 >= 1e-08f) {
          const float dum1 = p.dB;
          float d = 0.0f;
          if (morr_div(1.0f, lamr) < dum1) {
            d = 1.0f;
          } else if (morr_div(1.0f, lamr) >= dum1) {
            d = 2.0f - morr_exp(2.3e+03f * (morr_div(1.0f, lamr) - dum1));
          }
          nragg = (((-5.78f) * d) * qr3) * nr3 * rho;
        }
        if (qi3 >= 1e-08f && qvqvsi >= 1.0f) {
          nprci = morr_div(((((p.cons[21] * (qv3 - qvi)) * rho) * n0i) * morr_exp(-lami * p.dcs)) * dv, abi);
          prci = p.cons[22] * nprci;
          nprci = morr_min(nprci, morr_div(ni3, DT));
        }
        if (qni3 >= 1e-08f && qi3 >= QSMALL) {
          prai = morr_div((((p.cons[23] * asn) * qi3) * rho) * n0s, morr_pow(lams, p.bs + 3.0f));
          nprai = morr_div((((p.cons[23] * asn) * ni3) * rho) * n0s, morr_pow(lams, p.bs + 3.0f));
          nprai = morr_min(nprai, morr_div(ni3, DT));
        }
        if (qr3 >= 1e-08f && qi3 >= 1e-08f && t3 <= TMELT) {
          const float lr3 = morr_pow(lamr, p.br + 3.0f);
          if (qr3 >= 0.0001f) {
            niacr = morr_div(((p.cons[24] * ni3) * n0rr) * arn, lr3) * rho;
            piacr = morr_div(morr_div(((p.cons[25] * ni3) * n0rr) * arn, lr3), cube(lamr)) * rho;
            praci = morr_div(((p.cons[24] * qi3) * n0rr) * arn, lr3) * rho;
            niacr = morr_min(niacr, morr_div(nr3, DT));
            niacr = morr_min(niacr, morr_div(ni3, DT));
          } else {
            niacrs = morr_div(((p.cons[24] * ni3) * n0rr) * arn, lr3) * rho;
            piacrs = morr_div(morr_div(((p.cons[25] * ni3) * n0rr) * arn, lr3), cube(lamr)) * rho;
            pracis = morr_div(((p.cons[24] * qi3) * n0rr) * arn, lr3) * rho;
            niacrs = morr_min(niacrs, morr_div(nr3, DT));
            niacrs = morr_min(niacrs, morr_div(ni3, DT));
          }
        }
        if ((qvqvs >= 0.999f && t3 <= 265.15f) || qvqvsi >= 1.25f) {
          float kc2 = (0.005f * morr_exp(0.304f * (TMELT - t3))) * 1e+03f;
          kc2 = morr_min(kc2, 5e+05f);
          kc2 = morr_max(morr_div(kc2, rho), 0.0f);
          if (kc2 > (ni3 + ns3) + ng3) {
            nnuccd = morr_div(((kc2 - ni3) - ns3) - ng3, DT);
            mnuccd = nnuccd * p.mi0;
          }
        }
        float epsi, epss, epsg, epsr;
        if (qi3 >= QSMALL) epsi = morr_div((((2.0f * p.pi) * n0i) * rho) * dv, lami * lami);
        else epsi = 0.0f;
        if (qni3 >= QSMALL)
          epss = ((((2.0f * p.pi) * n0s) * rho) * dv) * vent_y(p.f1s, p.f2s, asn, rho, mu, scn, p.cons[10], lams, p.cons[35]);
        else epss = 0.0f;
        if (qg3 >= QSMALL)
          epsg = ((((2.0f * p.pi) * n0g) * rho) * dv) * vent_y(p.f1s, p.f2s, agn, rho, mu, scn, p.cons[11], lamg, p.cons[36]);
        else epsg = 0.0f;
        if (qr3 >= QSMALL)
          epsr = ((((2.0f * p.pi) * n0rr) * rho) * dv) * vent_y(p.f1r, p.f2r, arn, rho, mu, scn, p.cons[9], lamr, p.cons[34]);
        else epsr = 0.0f;
        float dd;
        if (qi3 >= QSMALL) {
          dd = fmaf(-morr_exp(-lami * p.dcs), fmaf(lami, p.dcs, 1.0f), 1.0f);
          prd = morr_div(epsi * (qv3 - qvi), abi) * dd;
        } else {
          dd = 0.0f;
        }
        if (qni3 >= QSMALL) {
          prds = fmaf(morr_div(epsi * (qv3 - qvi), abi), 1.0f - dd, morr_div(epss * (qv3 - qvi), abi));
        } else {
          prd = fmaf(morr_div(epsi * (qv3 - qvi), abi), 1.0f - dd, prd);
        }
        prdg = morr_div(epsg * (qv3 - qvi), abi);
        if (qv3 < qvs) {
          pre = morr_div(epsr * (qv3 - qvs), ab);
          pre = morr_min(pre, 0.0f);
          const float d = fmaf(-pre, DT, qv3);
          if (d > qvs) pre = morr_div(qv3 - qvs, DT);
        } else {
          pre = 0.0f;
        }
        {
          const float d = morr_div(qv3 - qvi, DT);
          const float fudgef = 0.9999f;
          const float sum_dep = ((prd + prds) + mnuccd) + prdg;
          if ((d > 0.0f && sum_dep > d * fudgef) || (d < 0.0f && sum_dep < d * fudgef)) {
            mnuccd = morr_div((fudgef * mnuccd) * d, sum_dep);
            prd = morr_div((fudgef * prd) * d, sum_dep);
            prds = morr_div((fudgef * prds) * d, sum_dep);
            prdg = morr_div((fudgef * prdg) * d, sum_dep);
          }
        }
        if (prd < 0.0f) {
          eprd = prd;
          prd = 0.0f;
        }
        if (prds < 0.0f) {
          eprds = prds;
          prds = 0.0f;
        }
        if (prdg < 0.0f) {
          eprdg = prdg;
          prdg = 0.0f;
        }
        float d = ((((((((prc + pra) + mnuccc) + psacws) + psacwi) + qmults) + psacwg) + pgsacw) + qmultg) * DT;
        if (d > qc3 && qc3 >= QSMALL) {
          const float ratio = morr_div(qc3, d);
          prc = prc * ratio;
          pra = pra * ratio;
          mnuccc = mnuccc * ratio;
          psacws = psacws * ratio;
          psacwi = psacwi * ratio;
          qmults = qmults * ratio;
          qmultg = qmultg * ratio;
          psacwg = psacwg * ratio;
          pgsacw = pgsacw * ratio;
        }
        d = ((((((((((((-prd - mnuccc) + prci) + prai) - qmults) - qmultg) - qmultr) - qmultrg) - mnuccd) + praci) + pracis) -
              eprd) -
             psacwi) *
            DT;
        if (d > qi3 && qi3 >= QSMALL) {
          const float ratio =
              morr_div((((((((morr_div(qi3, DT) + prd) + mnuccc) + qmults) + qmultg) + qmultr) + qmultrg) + mnuccd) + psacwi,
                       ((((prci + prai) + praci) + pracis) - eprd));
          prci = prci * ratio;
          prai = prai * ratio;
          praci = praci * ratio;
          pracis = pracis * ratio;
          eprd = eprd * ratio;
        }
        d = (((((((pracs - pre) + ((qmultr + qmultrg) - prc)) + (mnuccr - pra)) + piacr) + piacrs) + pgracs) + pracg) * DT;
        if (d > qr3 && qr3 >= QSMALL) {
          const float ratio =
              morr_div((morr_div(qr3, DT) + prc) + pra,
                       ((((((((-pre + qmultr) + qmultrg) + pracs) + mnuccr) + piacr) + piacrs) + pgracs) + pracg));
          pre = pre * ratio;
          pracs = pracs * ratio;
          qmultr = qmultr * ratio;
          qmultrg = qmultrg * ratio;
          mnuccr = mnuccr * ratio;
          piacr = piacr * ratio;
          piacrs = piacrs * ratio;
          pgracs = pgracs * ratio;
          pracg = pracg * ratio;
        }
        d = (((((((((-prds - psacws) - prai) - prci) - pracs) - eprds) + psacr) - piacrs) - pracis)) * DT;
        if (d > qni3 && qni3 >= QSMALL) {
          const float ratio =
              morr_div((((((((morr_div(qni3, DT) + prds) + psacws) + prai) + prci) + pracs) + piacrs) + pracis), -eprds + psacr);
          eprds = eprds * ratio;
          psacr = psacr * ratio;
        }
        d = ((((((((((-psacwg - pracg) - pgsacw) - pgracs) - prdg) - mnuccr) - eprdg) - piacr) - praci) - psacr)) * DT;
        if (d > qg3 && qg3 >= QSMALL) {
          const float ratio = morr_div(
              (((((((((morr_div(qg3, DT) + psacwg) + pracg) + pgsacw) + pgracs) + prdg) + mnuccr) + psacr) + piacr) + praci),
              -eprdg);
          eprdg = eprdg * ratio;
        }
        S(0, k) = S(0, k) + (((((((-pre - prd) - prds) - mnuccd) - eprd) - eprds) - prdg) - eprdg);
        S(128, k) =
            S(128, k) +
            fmaf(((((((((((((psacws + psacwi) + mnuccc) + mnuccr) + qmults) + qmultg) + qmultr) + qmultrg) + pracs) +
                       psacwg) +
                      pracg) +
                     pgsacw) +
                    pgracs) +
                       piacr +
                   piacrs,
                 efrz, fmaf(pre, ecnd, ((((((prd + prds) + mnuccd) + eprd) + eprds) + prdg) + eprdg) * edep));
        S(256, k) = S(256, k) + ((((((((-pra - prc) - mnuccc) + pcc) - psacws) - psacwi) - qmults) - qmultg) - psacwg) - pgsacw;
        S(384, k) = S(384, k) + ((((((((((((prd + eprd) + psacwi) + mnuccc) - prci) - prai) + qmults) + qmultg) + qmultr) +
                                      qmultrg) +
                                     mnuccd) -
                                    praci) -
                                   pracis);
        S(640, k) =
            S(640, k) + (((((((((pre + pra) + prc) - pracs) - mnuccr) - qmultr) - qmultrg) - piacr) - piacrs) - pracg) - pgracs;
        S(512, k) = S(512, k) + (((((((prai + psacws) + prds) + pracs) + prci) + eprds) - psacr) + piacrs) + pracis;
        S(1024, k) = S(1024, k) + ((((nsagg + nprci) - nscng) - ngracs) + niacrs);
        S(768, k) = S(768, k) + (((((((((pracg + psacwg) + pgsacw) + pgracs) + prdg) + eprdg) + mnuccr) + piacr) + praci) + psacr);
        S(1280, k) = S(1280, k) + (((nscng + ngracs) + nnuccr) + niacr);
        S(1408, k) = S(1408, k) + (((((-nnuccc - npsacws) - npra) - nprc) - npsacwi) - npsacwg);
        S(896, k) = S(896, k) + (((((((((nnuccc - nprci) - nprai) + nmults) + nmultg) + nmultr) + nmultrg) + nnuccd) - niacr) -
                                 niacrs);
        S(1152, k) = S(1152, k) + (((((((nprc1 - npracs) - nnuccr) + nragg) - niacr) - niacrs) - npracg) - ngracs);
        if (eprd < 0.0f) {
          float q = morr_div(eprd * DT, qi3);
          q = morr_max(-1.0f, q);
          nsubi = morr_div(q * ni3, DT);
        }
        if (eprds < 0.0f) {
          float q = morr_div(eprds * DT, qni3);
          q = morr_max(-1.0f, q);
          nsubs = morr_div(q * ns3, DT);
        }
        if (pre < 0.0f) {
          float q = morr_div(pre * DT, qr3);
          q = morr_max(-1.0f, q);
          nsubr = morr_div(q * nr3, DT);
        }
        if (eprdg < 0.0f) {
          float q = morr_div(eprdg * DT, qg3);
          q = morr_max(-1.0f, q);
          nsubg = morr_div(q * ng3, DT);
        }
        S(896, k) = S(896, k) + nsubi;
        S(1024, k) = S(1024, k) + nsubs;
        S(1280, k) = S(1280, k) + nsubg;
        S(1152, k) = S(1152, k) + nsubr;
        {
          float dumt = fmaf(DT, S(128, k), t3);
          float dumqv = fmaf(DT, S(0, k), qv3);
          float dumqc = fmaf(DT, S(256, k), qc3);
          const float dumqr = fmaf(DT, S(640, k), qr3);
          const float dummqs = fmaf(DT, S(512, k), qni3);
          const float dumqg = fmaf(DT, S(768, k), qg3);
          const float dumqi = fmaf(DT, S(384, k), qi3);
          pres = (rho * dumt) * fmaf(p.rv, dumqv, p.r);
          const float saveqc = dumqc, savet = dumt;
          satadj2(p, dumt, pres, dumqv, dumqc, dumqr, dumqi, dummqs, dumqg, rho);
          if (fabsf(dumt - savet) >= 0.0001f) {
            const float pccv = (dumqc - saveqc) * RDT;
            S(0, k) = S(0, k) - pccv;
            S(256, k) = S(256, k) + pccv;
            S(128, k) = fmaf(dumt - savet, RDT, S(128, k));
          }
        }
      }
      ltrue = true;
    }
    S(1920, k) = lami;
    S(2048, k) = nc3;
    F.T3[c] = t3;
    F.QV[c] = qv3;
    F.QC[c] = qc3;
    F.QR[c] = qr3;
    F.QI[c] = qi3;
    F.QS[c] = qni3;
    F.QG[c] = qg3;
    F.NI[c] = ni3;
    F.NS[c] = ns3;
    F.NR[c] = nr3;
    F.NG[c] = ng3;
  }
  float precrt = 0.0f;
  if (!ltrue) return;
  // ------------------------------------------------------------------ sedimentation
  for (int s = 0; s < 5; s++) {
    int nstep = 1;
    for (int k = nk - 1; k >= 0; k--) {
      const int c = mi(p, i, j, k);
      const float rho = F.RH3[c];
      float um = 0.0f, un = 0.0f, dq, dn;
      if (s == 0) {
        dq = fmaf(S(640, k), DT, F.QR[c]);
        dn = fmaf(S(1152, k), DT, F.NR[c]);
      } else if (s == 1) {
        dq = fmaf(S(384, k), DT, F.QI[c]);
        dn = fmaf(S(896, k), DT, F.NI[c]);
      } else if (s == 2) {
        dq = fmaf(S(256, k), DT, F.QC[c]);
        dn = S(2048, k);
      } else if (s == 3) {
        dq = fmaf(S(512, k), DT, F.QS[c]);
        dn = fmaf(S(1024, k), DT, F.NS[c]);
      } else {
        dq = fmaf(S(768, k), DT, F.QG[c]);
        dn = fmaf(S(1280, k), DT, F.NG[c]);
      }
      dn = morr_max(0.0f, dn);
      const float d = morr_pow(morr_div(p.rhosu, rho), 0.54f);
      if (s == 0) {
        if (dq >= QSMALL) {
          float dlamr = morr_pow(morr_div((p.pi * p.rhow) * dn, dq), 1.0f / 3.0f);
          dlamr = morr_max(dlamr, p.lamminr);
          dlamr = morr_min(dlamr, p.lammaxr);
          const float arn = d * p.ar;
          un = morr_div(arn * p.cons[6], morr_pow(dlamr, p.br));
          um = morr_div(arn * p.cons[4], morr_pow(dlamr, p.br));
        }
        um = morr_min(um, 9.1f * d);
        un = morr_min(un, 9.1f * d);
      } else if (s == 1) {
        if (dq >= QSMALL) {
          float dlami = morr_pow(morr_div(p.cons[12] * dn, dq), morr_div(1.0f, p.di));
          dlami = morr_max(dlami, p.lammini);
          dlami = morr_min(dlami, p.lammaxi);
          const float ain = morr_pow(morr_div(p.rhosu, rho), 0.35f) * p.ai;
          un = morr_div(ain * p.cons[27], morr_pow(dlami, p.bi));
          um = morr_div(ain * p.cons[28], morr_pow(dlami, p.bi));
        }
        um = morr_min(um, 1.2f * morr_pow(morr_div(p.rhosu, rho), 0.35f));
        un = morr_min(un, 1.2f * morr_pow(morr_div(p.rhosu, rho), 0.35f));
      } else if (s == 2) {
        if (dq >= QSMALL) {
          float pgam = fmaf(0.0005714f, morr_div(S(2048, k), 1e+06f) * rho, 0.2714f);
          pgam = morr_div(1.0f, sq(pgam)) - 1.0f;
          pgam = morr_max(pgam, 2.0f);
          pgam = morr_min(pgam, 1e+01f);
          float dlamc = morr_pow(morr_div((p.cons[26] * dn) * gamma(pgam + 4.0f), dq * gamma(pgam + 1.0f)), 1.0f / 3.0f);
          const float lmin = morr_div(pgam + 1.0f, 6e-05f);
          const float lmax = morr_div(pgam + 1.0f, 1e-06f);
          dlamc = morr_max(dlamc, lmin);
          dlamc = morr_min(dlamc, lmax);
          const float acn = S(2176, k);
          un = morr_div(acn * gamma((1.0f + p.bc) + pgam), morr_pow(dlamc, p.bc) * gamma(pgam + 1.0f));
          um = morr_div(acn * gamma((4.0f + p.bc) + pgam), morr_pow(dlamc, p.bc) * gamma(pgam + 4.0f));
        }
        if (p.drizzleVt != 0.0f) {
          if (dq >= QSMALL) {
            um = ((1.19e+08f * morr_pow(morr_div(3.0f, (((4.0f * p.pi) * p.rhow) * p.ndcnst) * 1e+06f), 2.0f / 3.0f)) *
                  morr_pow(rho * dq, 2.0f / 3.0f)) *
                 morr_exp(5.0f * sq(morr_log(1.5f)));
          } else {
            um = 0.0f;
          }
        }
      } else if (s == 3) {
        if (dq >= QSMALL) {
          float dlams = morr_pow(morr_div(p.cons[1] * dn, dq), morr_div(1.0f, p.ds));
          dlams = morr_max(dlams, p.lammins);
          dlams = morr_min(dlams, p.lammaxs);
          const float asn = d * p.as_;
          um = morr_div(asn * p.cons[3], morr_pow(dlams, p.bs));
          un = morr_div(asn * p.cons[5], morr_pow(dlams, p.bs));
        }
        um = morr_min(um, 1.2f * d);
        un = morr_min(un, 1.2f * d);
      } else {
        if (dq >= QSMALL) {
          float dlamg = morr_pow(morr_div(p.cons[2] * dn, dq), morr_div(1.0f, p.dg));
          dlamg = morr_max(dlamg, p.lamming);
          dlamg = morr_min(dlamg, p.lammaxg);
          const float agn = d * p.ag;
          um = morr_div(agn * p.cons[7], morr_pow(dlamg, p.bg));
          un = morr_div(agn * p.cons[8], morr_pow(dlamg, p.bg));
        }
        um = morr_min(um, 2e+01f * d);
        un = morr_min(un, 2e+01f * d);
      }
      S(2944, k) = um;
      S(3072, k) = un;
      if (k <= nk - 2) {
        if (S(2944, k) < 1e-10f) S(2944, k) = S(2944, k + 1);
        if (S(3072, k) < 1e-10f) S(3072, k) = S(3072, k + 1);
      }
      const float temz = morr_div(1.0f, F.DZQ[k]);
      const float rgvm = morr_max(S(2944, k), S(3072, k));
      const int nst = (int)fmaf(rgvm * DT, temz, 1.0f);
      nstep = nst > nstep ? nst : nstep;
      S(3200, k) = dq * rho;
      S(3328, k) = dn * rho;
    }
    const float dttmp = morr_div(DT, (float)nstep);
    const int ntend = s == 0 ? 1152 : s == 1 ? 896 : s == 2 ? 1408 : s == 3 ? 1024 : 1280;
    for (int n = 0; n < nstep; n++) {
      for (int k = 0; k < nk; k++) {
        S(3456, k) = S(2944, k) * S(3200, k);
        S(3584, k) = S(3072, k) * S(3328, k);
      }
      int k = nk - 1;
      int c = mi(p, i, j, k);
      float temr = morr_div(1.0f, (float)nstep * F.RH3[c]);
      float temz = morr_div(1.0f, F.DZQ[k]);
      float faltnd = S(3456, k) * temz;
      float faltndn = S(3584, k) * temz;
      S(2304 + s * 128, k) = fmaf(-faltnd, temr, S(2304 + s * 128, k));
      S(ntend, k) = fmaf(-faltndn, temr, S(ntend, k));
      S(3200, k) = fmaf(-faltnd, dttmp, S(3200, k));
      S(3328, k) = fmaf(-faltndn, dttmp, S(3328, k));
      for (k = nk - 2; k >= 0; k--) {
        c = mi(p, i, j, k);
        temr = morr_div(1.0f, (float)nstep * F.RH3[c]);
        temz = morr_div(1.0f, F.DZQ[k]);
        faltnd = (S(3456, k + 1) - S(3456, k)) * temz;
        faltndn = (S(3584, k + 1) - S(3584, k)) * temz;
        S(2304 + s * 128, k) = fmaf(faltnd, temr, S(2304 + s * 128, k));
        S(ntend, k) = fmaf(faltndn, temr, S(ntend, k));
        S(3200, k) = fmaf(faltnd, dttmp, S(3200, k));
        S(3328, k) = fmaf(faltndn, dttmp, S(3328, k));
      }
      precrt = fmaf(S(3456, 0), dttmp, precrt);
    }
  }
  // ------------------------------------------------------------------ update
  for (int k = 0; k < nk; k++) {
    const int c = mi(p, i, j, k);
    const float rho = F.RH3[c];
    S(640, k) = S(640, k) + S(2304, k);
    S(384, k) = S(384, k) + S(2304 + 128, k);
    S(256, k) = S(256, k) + S(2304 + 2 * 128, k);
    S(768, k) = S(768, k) + S(2304 + 4 * 128, k);
    S(512, k) = S(512, k) + S(2304 + 3 * 128, k);
    float t3 = F.T3[c], qv3 = F.QV[c], qc3 = F.QC[c], qr3 = F.QR[c], qi3 = F.QI[c], qni3 = F.QS[c], qg3 = F.QG[c];
    float ni3 = F.NI[c], ns3 = F.NS[c], nr3 = F.NR[c], ng3 = F.NG[c];
    float nc3 = S(2048, k);
    const float lami_k = S(1920, k);
    if (qi3 >= QSMALL && t3 < TMELT && lami_k >= 1e-10f) {
      if (morr_div(1.0f, lami_k) >= 2.0f * p.dcs) {
        S(512, k) = (S(512, k) + morr_div(qi3, DT)) + S(384, k);
        S(1024, k) = (S(1024, k) + morr_div(ni3, DT)) + S(896, k);
        S(384, k) = morr_div(-qi3, DT);
        S(896, k) = morr_div(-ni3, DT);
      }
    }
    qc3 = fmaf(S(256, k), DT, qc3);
    qi3 = fmaf(S(384, k), DT, qi3);
    qni3 = fmaf(S(512, k), DT, qni3);
    qr3 = fmaf(S(640, k), DT, qr3);
    nc3 = fmaf(S(1408, k), DT, nc3);
    ni3 = fmaf(S(896, k), DT, ni3);
    ns3 = fmaf(S(1024, k), DT, ns3);
    nr3 = fmaf(S(1152, k), DT, nr3);
    qg3 = fmaf(S(768, k), DT, qg3);
    ng3 = fmaf(S(1280, k), DT, ng3);
    t3 = fmaf(S(128, k), DT, t3);
    qv3 = fmaf(S(0, k), DT, qv3);
    const float pres = (rho * t3) * fmaf(p.rv, qv3, p.r);
    const float evs = esat_liquid(pres, t3);
    float eis = esat_ice(pres, t3);
    if (eis > evs) eis = evs;
    const float qvs = morr_div(p.ep2 * evs, pres - evs);
    const float qvi = morr_div(p.ep2 * eis, pres - eis);
    const float qvqvs = morr_div(qv3, qvs);
    const float qvqvsi = morr_div(qv3, qvi);
    const float ecnd = S(1536, k), edep = S(1664, k), efrz = S(1792, k);
    if (qvqvs < 0.9f) {
      if (qr3 < p.qthr) {
        qv3 = qv3 + qr3;
        t3 = fmaf(-qr3, ecnd, t3);
        qr3 = 0.0f;
      }
      if (qc3 < p.qthr) {
        qv3 = qv3 + qc3;
        t3 = fmaf(-qc3, ecnd, t3);
        qc3 = 0.0f;
      }
    }
    if (qvqvsi < 0.9f) {
      if (qi3 < p.qthr) {
        qv3 = qv3 + qi3;
        t3 = fmaf(-qi3, edep, t3);
        qi3 = 0.0f;
      }
      if (qni3 < p.qthr) {
        qv3 = qv3 + qni3;
        t3 = fmaf(-qni3, edep, t3);
        qni3 = 0.0f;
      }
      if (qg3 < p.qthr) {
        qv3 = qv3 + qg3;
        t3 = fmaf(-qg3, edep, t3);
        qg3 = 0.0f;
      }
    }
    if (qc3 < QSMALL) { qc3 = 0.0f; nc3 = 0.0f; }
    if (qr3 < QSMALL) { qr3 = 0.0f; nr3 = 0.0f; }
    if (qi3 < QSMALL) { qi3 = 0.0f; ni3 = 0.0f; }
    if (qni3 < QSMALL) { qni3 = 0.0f; ns3 = 0.0f; }
    if (qg3 < QSMALL) { qg3 = 0.0f; ng3 = 0.0f; }
    const bool goto500 = qc3 < QSMALL && qi3 < QSMALL && qni3 < QSMALL && qr3 < QSMALL && qg3 < QSMALL;
    if (!goto500) {
      if (qi3 >= QSMALL && t3 >= TMELT) {
        qr3 = qr3 + qi3;
        t3 = fmaf(-qi3, efrz, t3);
        qi3 = 0.0f;
        nr3 = nr3 + ni3;
        ni3 = 0.0f;
      }
      if (t3 <= 233.15f && qc3 >= QSMALL) {
        qi3 = qi3 + qc3;
        t3 = fmaf(qc3, efrz, t3);
        qc3 = 0.0f;
        ni3 = ni3 + nc3;
        nc3 = 0.0f;
      }
      if (t3 <= 233.15f && qr3 >= QSMALL) {
        qg3 = qg3 + qr3;
        t3 = fmaf(qr3, efrz, t3);
        qr3 = 0.0f;
        ng3 = ng3 + nr3;
        nr3 = 0.0f;
      }
      ni3 = morr_max(0.0f, ni3);
      ns3 = morr_max(0.0f, ns3);
      nc3 = morr_max(0.0f, nc3);
      nr3 = morr_max(0.0f, nr3);
      ng3 = morr_max(0.0f, ng3);
      float lam = 0.0f, n0 = 0.0f, lami = 0.0f, lams = 0.0f, lamcF = 0.0f, pgamF = 0.0f;
      if (qi3 >= QSMALL) {
        lam3_of(qi3, ni3, p.cons[12], p.di, p.lammini, p.lammaxi, lam, n0);
        lami = lam;
      }
      if (qr3 >= QSMALL) lamr_of(p, qr3, nr3, lam, n0);
      if (qc3 >= QSMALL) {
        float cd;
        lamc_of(p, qc3, nc3, rho, pgamF, lamcF, cd);
      }
      if (qni3 >= QSMALL) {
        lam3_of(qni3, ns3, p.cons[1], p.ds, p.lammins, p.lammaxs, lam, n0);
        lams = lam;
      }
      if (qg3 >= QSMALL) lam3_of(qg3, ng3, p.cons[2], p.dg, p.lamming, p.lammaxg, lam, n0);
      if (dorad != 0) {
        const float effi = qi3 >= QSMALL ? morr_div(morr_div(3.0f, lami), 2.0f) * 1e+06f : 25.0f;
        const float effs = qni3 >= QSMALL ? morr_div(morr_div(3.0f, lams), 2.0f) * 1e+06f : 25.0f;
        float effc;
        if (qc3 >= QSMALL)
          effc = morr_div(morr_div(morr_div(gamma(pgamF + 4.0f), gamma(pgamF + 3.0f)), lamcF), 2.0f) * 1e+06f;
        else
          effc = 25.0f;
        F.EFFC[c] = effc * 1e-06f;
        F.EFFI[c] = morr_min(1.4e+02f, effi) * 1e-06f;
        F.EFFS[c] = effs * 1e-06f;
      }
    }
    ni3 = morr_min(ni3, morr_div(3e+05f, rho));
    nc3 = morr_div(p.ndcnst * 1e+06f, rho);
    F.T3[c] = t3;
    F.QV[c] = qv3;
    F.QC[c] = qc3;
    F.QR[c] = qr3;
    F.QI[c] = qi3;
    F.QS[c] = qni3;
    F.QG[c] = qg3;
    F.NI[c] = ni3;
    F.NS[c] = ns3;
    F.NR[c] = nr3;
    F.NG[c] = ng3;
  }
  const int c0 = mi(p, i, j, 0);
  F.sfc[c0] = F.sfc[c0] + precrt;
}

}  // namespace morr
}  // namespace te

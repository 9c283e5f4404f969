/* Oracle: hand-written CPU restatement of the reference's CM1 dynamics kernels.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each kernel cites the WGSL file of the
 * reference (data/kernels/<name>.wgsl, main() body) whose arithmetic it restates, in
 * the same operation order: every binary32 operation rounds once, fmaf() exactly where
 * the reference writes fma, IEEE division (the reference's div_cr is a correctly
 * rounded division, adv_flux_x_weno.wgsl:29-50, restated as te_div_cr below).
 * Build: oracle/Makefile (-ffp-contract=off, no fast-math, -fwrapv).
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <string.h>
#include <xmmintrin.h>

/* ------------------------------------------------------------------ utilities */

uint32_t te_fnv1a(const uint32_t *w, size_t n) {
  /* FNV-1a over u32 words (web/view.js:1063-1068) */
  uint32_t h = 0x811c9dc5u;
  for (size_t i = 0; i < n; i++) h = (h ^ w[i]) * 0x01000193u;
  return h;
}

void te_set_ftz(int on) {
  /* flush-to-zero + denormals-are-zero on every OpenMP worker and on the caller */
  unsigned bits = 0x8000u | 0x0040u;
#pragma omp parallel
  {
    unsigned c = _mm_getcsr();
    _mm_setcsr(on ? (c | bits) : (c & ~bits));
  }
  unsigned c = _mm_getcsr();
  _mm_setcsr(on ? (c | bits) : (c & ~bits));
}

static inline uint32_t fbits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static inline float bitsf(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

/* div_core / div_cr (adv_flux_x_weno.wgsl:29-50): quotient, then up to four
 * neighbour corrections by exact fma residual; tiny numerators are scaled by 2^64. */
static float div_core(float a, float b) {
  float q0 = a / b;
  int special = q0 == 0.0f || fabsf(q0) > 3.0e38f || q0 != q0 || fabsf(q0) < 1.0e-37f;
  float q = q0;
  float r = fabsf(fmaf(-q, b, a));
  for (int k = 0; k < 4; k++) {
    float qu = bitsf(fbits(q) + 1u);
    float qd = bitsf(fbits(q) - 1u);
    float ru = fabsf(fmaf(-qu, b, a));
    float rd = fabsf(fmaf(-qd, b, a));
    int up = ru < r;
    int dn = !up && rd < r;
    q = up ? qu : (dn ? qd : q);
    r = up ? ru : (dn ? rd : r);
  }
  return special ? q0 : q;
}

float te_div_cr(float a, float b) {
  int small = fabsf(a) < 8.67361738e-19f && a != 0.0f;
  float q = div_core(small ? a * 1.8446744e19f : a, b);
  return small ? q * 5.42101086e-20f : q;
}
#define DCR te_div_cr

/* sqrt_core / sqrt_cr (adv_flux_x_weno.wgsl:53-71) */
static float sqrt_core(float x) {
  float s = sqrtf(x);
  if (!(x > 1.0e-30f) || x > 3.0e38f) return s;
  for (int k = 0; k < 4; k++) {
    float r = fmaf(-s, s, x);
    float su = bitsf(fbits(s) + 1u);
    float sd = bitsf(fbits(s) - 1u);
    if (r > s * (su - s)) s = su;
    else if (r <= -(s * (s - sd))) s = sd;
    else break;
  }
  return s;
}

float te_sqrt_cr(float x) {
  if (x < 8.67361738e-19f && x > 0.0f) return sqrt_core(x * 1.8446744e19f) * 2.32830644e-10f;
  return sqrt_core(x);
}

#ifdef TE_ORACLE_F64
/* Binary64 twin (oracle/oracle64.c compiles this file with TE_ORACLE_F64): every
 * kernel below evaluates the same formulas in binary64.  Field values live in a double
 * array parallel to the word memory (te64_D, set by te64_bind); parameter structs are
 * still read from the words.  Division and square root are the binary64 operations;
 * fma is the binary64 fma; the reference's two-float pow becomes pow().  Constants keep
 * the binary32 values the step is defined with. */
double *te64_D;
void te64_bind(double *D) { te64_D = D; }
#undef DCR
#define DCR(a, b) ((double)(a) / (double)(b))
#define float double
#define fmaf fma
#define fabsf fabs
#define sqrtf sqrt
#define powf pow
#define nearbyintf nearbyint
#define ldexpf ldexp
#define frexpf frexp
#define te_sqrt_cr sqrt
#define te_weno5 te64_weno5
#define te_rr_pow_cr te64_rr_pow_cr
#define te_pow_f64 pow
#define te_exp_f64 exp
#define te_log_f64 log
#endif

/* WGSL min/max on f32: min(a, b) is b if b < a, else a; max(a, b) is b if a < b,
 * else a; a NaN operand yields the other one.  This fixes the sign of a zero result
 * when the operands are +0 and -0. */
static inline float fmin_(float a, float b) { return (b < a || a != a) ? b : a; }
static inline float fmax_(float a, float b) { return (a < b || a != a) ? b : a; }

/* --------------------------------------------------------------- grid access */

typedef struct {
  int nx, ny, nz, sJ, sK;
  float rdx, rdy, rdz;
} Dims;

static Dims dims_at(const uint32_t *M, uint32_t off) {
  /* GridDims (timestep.js:88-90; ld_GridDims in every kernel) */
  Dims g;
  g.nx = (int)M[off + 0];
  g.ny = (int)M[off + 1];
  g.nz = (int)M[off + 2];
  g.sJ = (int)M[off + 3];
  g.sK = (int)M[off + 4];
  g.rdx = bitsf(M[off + 5]);
  g.rdy = bitsf(M[off + 6]);
  g.rdz = bitsf(M[off + 7]);
  return g;
}

typedef struct {
  float dts, alph, beta, kdiv, smeps;
} Acoustic;

static Acoustic acoustic_at(const uint32_t *M, uint32_t off) {
  /* AcousticParamsGPU (timestep.js:46-52) */
  Acoustic a;
  a.dts = bitsf(M[off + 0]);
  a.alph = bitsf(M[off + 1]);
  a.beta = bitsf(M[off + 2]);
  a.kdiv = bitsf(M[off + 3]);
  a.smeps = bitsf(M[off + 4]);
  return a;
}

#define B(n) (ARG[4 + (n)])
#ifdef TE_ORACLE_F64
#define FPTR(n) (te64_D + B(n))
#else
#define FPTR(n) ((float *)(M + B(n)))
#endif
#define FVAL(n) (bitsf(M[B(n)]))
#define IVAL(n) ((int32_t)M[B(n)])
#define GIDX(g, i, j, k) (((i) + 3) + (g).sJ * (((j) + 3) + (g).sK * (k)))
#define CP_ 1005.7f

/* horizontal metric planes (grid.js:200-214; f_hm_* helpers of the kernels) */
static inline float hm_uh(const Dims *g, const float *hm, int i) { return hm[i + 3]; }
static inline float hm_uf(const Dims *g, const float *hm, int i) { return hm[g->sJ + i + 3]; }
static inline float hm_vh(const Dims *g, const float *hm, int j) { return hm[2 * g->sJ + j + 3]; }
static inline float hm_vf(const Dims *g, const float *hm, int j) { return hm[2 * g->sJ + g->sK + j + 3]; }

/* loop over the dispatch grid in threads (ARG[0..2]) */
#define FOR_GRID                                                   \
  const long GX = ARG[0], GY = ARG[1], GZ = ARG[2];                \
  _Pragma("omp parallel for collapse(2) schedule(static)")          \
  for (long tz = 0; tz < GZ; tz++)                                  \
    for (long ty = 0; ty < GY; ty++)                                \
      for (long tx = 0; tx < GX; tx++)

/* --------------------------------------------------------- reconstructions */

/* f_flx5 (adv_flux_x.wgsl:106-143): 5th-order upwind-biased (2,-13,47,27,-3)/60 */
static inline float flx5(float s1, float s2, float s3, float s4, float s5) {
  return fmaf(DCR(-3.0f, 60.0f), s5,
              fmaf(DCR(27.0f, 60.0f), s4, fmaf(DCR(47.0f, 60.0f), s3, fmaf(DCR(2.0f, 60.0f), s1, DCR(-13.0f, 60.0f) * s2))));
}

/* f_flx3 (adv_flux_z.wgsl:106-113): 3rd-order (-1,5,2)/6 */
static inline float flx3(float s1, float s2, float s3) {
  return fmaf(DCR(2.0f, 6.0f), s3, fmaf(DCR(-1.0f, 6.0f), s1, DCR(5.0f, 6.0f) * s2));
}

/* f_weno5 (adv_flux_x_weno.wgsl:121-151): WENO-JS with clipped ratios */
float te_weno5(float s1, float s2, float s3, float s4, float s5, float weps) {
  const float c13 = DCR(13.0f, 12.0f);
  float e1 = fmaf(-2.0f, s2, s1) + s3;
  float d1 = fmaf(3.0f, s3, fmaf(-4.0f, s2, s1));
  float b1 = fmaf(c13 * e1, e1, (0.25f * d1) * d1);
  float e2 = fmaf(-2.0f, s3, s2) + s4;
  float d2 = s2 - s4;
  float b2 = fmaf(c13 * e2, e2, (0.25f * d2) * d2);
  float e3 = fmaf(-2.0f, s4, s3) + s5;
  float d3 = fmaf(3.0f, s3, -(4.0f * s4)) + s5;
  float b3 = fmaf(c13 * e3, e3, (0.25f * d3) * d3);
  float tau = fabsf(b1 - b3);
  float r1 = fmin_(1e30f, DCR(tau, b1 + weps));
  float r2 = fmin_(1e30f, DCR(tau, b2 + weps));
  float r3 = fmin_(1e30f, DCR(tau, b3 + weps));
  float m = fmax_(r1, fmax_(r2, r3));
  float one = 1.0f;
  if (m > 1e15f) {
    float im = DCR(1.0f, m);
    r1 = r1 * im;
    r2 = r2 * im;
    r3 = r3 * im;
    one = im * im;
  }
  float w1 = 0.1f * fmaf(r1, r1, one);
  float w2 = 0.6f * fmaf(r2, r2, one);
  float w3 = 0.3f * fmaf(r3, r3, one);
  float p1 = fmaf(DCR(11.0f, 6.0f), s3, fmaf(DCR(2.0f, 6.0f), s1, DCR(-7.0f, 6.0f) * s2));
  float p2 = fmaf(DCR(2.0f, 6.0f), s4, fmaf(DCR(-1.0f, 6.0f), s2, DCR(5.0f, 6.0f) * s3));
  float p3 = fmaf(DCR(-1.0f, 6.0f), s5, fmaf(DCR(2.0f, 6.0f), s3, DCR(5.0f, 6.0f) * s4));
  return DCR(fmaf(w3, p3, fmaf(w1, p1, w2 * p2)), (w1 + w2) + w3);
}
#define WENO te_weno5

/* f_weno_pdef_ok (adv_flux_x_weno.wgsl:106-119) */
static inline int weno_pdef_ok(float s1, float s2, float s3, float s4, float s5, float weps, int pdef) {
  if (!pdef) return 1;
  float bmax = fmax_(fmax_(fmax_(fabsf(s1), fabsf(s2)), fmax_(fabsf(s3), fabsf(s4))), fabsf(s5));
  return bmax > weps;
}

/* f_upstrpd (adv_flux_z_weno.wgsl:111-120): 3rd-order limited upstream value */
static inline float upstrpd(float s1, float s2, float s3, float weps) {
  float dd = s2 - s1;
  float sgn = bitsf((fbits(weps) & 0x7fffffffu) | (fbits(dd) & 0x80000000u));
  float rr = DCR(s3 - s2, sgn + dd);
  float phi = fmax_(0.0f, fmin_(rr, fmin_(fmaf(DCR(2.0f, 6.0f), rr, DCR(1.0f, 6.0f)), 1.0f)));
  return fmaf(phi, s2 - s1, s2);
}

/* ------------------------------------------------- linear upwind fluxes (RK 1-2) */

static void flux_lin_h(uint32_t *M, const uint32_t *ARG, int dir) {
  /* adv_flux_x.wgsl / adv_flux_y.wgsl main: f = rr * flx5(upwind stencil) */
  Dims g = dims_at(M, B(0));
  const float *s = FPTR(1), *rr = FPTR(2);
  float *fo = FPTR(3);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (dir == 0 ? (i > g.nx || j >= g.ny || k >= g.nz) : (i >= g.nx || j > g.ny || k >= g.nz)) continue;
    int c = GIDX(g, i, j, k);
    int d = dir == 0 ? 1 : g.sJ;
    float u = rr[c];
    float f = u >= 0.0f ? flx5(s[c - 3 * d], s[c - 2 * d], s[c - d], s[c], s[c + d])
                        : flx5(s[c + 2 * d], s[c + d], s[c], s[c - d], s[c - 2 * d]);
    fo[c] = u * f;
  }
}
void teor_adv_flux_x(uint32_t *M, const uint32_t *ARG) { flux_lin_h(M, ARG, 0); }
void teor_adv_flux_y(uint32_t *M, const uint32_t *ARG) { flux_lin_h(M, ARG, 1); }

void teor_adv_flux_z(uint32_t *M, const uint32_t *ARG) {
  /* adv_flux_z.wgsl main: 2nd order at k=1 / nz-1 (upwind side), 3rd next to them */
  Dims g = dims_at(M, B(0));
  const float *s = FPTR(1), *rrw = FPTR(2), *c1 = FPTR(3), *c2 = FPTR(4);
  float *fz = FPTR(5);
  const int sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k > g.nz) continue;
    int c = GIDX(g, i, j, k);
    if (k == 0 || k == g.nz) { fz[c] = 0.0f; continue; }
    float w = rrw[c];
    int up = w >= 0.0f;
    float f;
    if (k == 1) f = up ? fmaf(c1[k], s[c - sk], c2[k] * s[c]) : flx3(s[c + sk], s[c], s[c - sk]);
    else if (k == 2) f = up ? flx3(s[c - 2 * sk], s[c - sk], s[c]) : flx5(s[c + 2 * sk], s[c + sk], s[c], s[c - sk], s[c - 2 * sk]);
    else if (k == g.nz - 2) f = up ? flx5(s[c - 3 * sk], s[c - 2 * sk], s[c - sk], s[c], s[c + sk]) : flx3(s[c + sk], s[c], s[c - sk]);
    else if (k == g.nz - 1) f = up ? flx3(s[c - 2 * sk], s[c - sk], s[c]) : fmaf(c1[k], s[c - sk], c2[k] * s[c]);
    else f = up ? flx5(s[c - 3 * sk], s[c - 2 * sk], s[c - sk], s[c], s[c + sk])
                : flx5(s[c + 2 * sk], s[c + sk], s[c], s[c - sk], s[c - 2 * sk]);
    fz[c] = w * f;
  }
}

/* f_flx5_upwind (adv_flux_x_stag.wgsl:106-129): stencil shifted by one when the
 * variable is staggered along the flux direction */
static inline float flx5_upwind(const float *a, int c, int s, int up, int shifted) {
  if (shifted) return up ? flx5(a[c - 2 * s], a[c - s], a[c], a[c + s], a[c + 2 * s])
                         : flx5(a[c + 3 * s], a[c + 2 * s], a[c + s], a[c], a[c - s]);
  return up ? flx5(a[c - 3 * s], a[c - 2 * s], a[c - s], a[c], a[c + s])
            : flx5(a[c + 2 * s], a[c + s], a[c], a[c - s], a[c - 2 * s]);
}

static void flux_stag_h(uint32_t *M, const uint32_t *ARG, int dir) {
  /* adv_flux_x_stag.wgsl / adv_flux_y_stag.wgsl main */
  Dims g = dims_at(M, B(0));
  int stag = IVAL(1);
  const float *a = FPTR(2), *rr = dir == 0 ? FPTR(3) : FPTR(4), *c2 = FPTR(7);
  float *fo = FPTR(8);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx - 1, j = (int)ty - 1, k = (int)tz;
    if (i > g.nx || j > g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    if (stag == 4 && k == 0) { fo[c] = 0.0f; continue; }
    float m;
    if (dir == 0) {
      if (stag == 2) m = 0.5f * (rr[c] + rr[c + 1]);
      else if (stag == 3) m = 0.5f * (rr[c] + rr[c - sj]);
      else if (stag == 4) { float cc2 = c2[k]; m = fmaf(cc2, rr[c], (1.0f - cc2) * rr[c - sk]); }
      else m = rr[c];
      fo[c] = m * flx5_upwind(a, c, 1, m >= 0.0f, stag == 2);
    } else {
      if (stag == 2) m = 0.5f * (rr[c] + rr[c - 1]);
      else if (stag == 3) m = 0.5f * (rr[c] + rr[c + sj]);
      else if (stag == 4) { float cc2 = c2[k]; m = fmaf(cc2, rr[c], (1.0f - cc2) * rr[c - sk]); }
      else m = rr[c];
      fo[c] = m * flx5_upwind(a, c, sj, m >= 0.0f, stag == 3);
    }
  }
}
void teor_adv_flux_x_stag(uint32_t *M, const uint32_t *ARG) { flux_stag_h(M, ARG, 0); }
void teor_adv_flux_y_stag(uint32_t *M, const uint32_t *ARG) { flux_stag_h(M, ARG, 1); }

void teor_adv_flux_z_stag(uint32_t *M, const uint32_t *ARG) {
  /* adv_flux_z_stag.wgsl main (momentum, RK stages 1-2) */
  Dims g = dims_at(M, B(0));
  int stag = IVAL(1);
  const float *a = FPTR(2), *rrw = FPTR(5), *c1 = FPTR(6), *c2 = FPTR(7);
  float *fz = FPTR(8);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > g.nx || j > g.ny || k > g.nz) continue;
    int c = GIDX(g, i, j, k);
    float m;
    if (stag == 2) m = 0.5f * (rrw[c] + rrw[c - 1]);
    else if (stag == 3) m = 0.5f * (rrw[c] + rrw[c - sj]);
    else m = 0.5f * (rrw[c] + (k < g.nz ? rrw[c + sk] : 0.0f));
    int up = m >= 0.0f;
    float f;
    if (stag == 4) {
      if (k > g.nz - 1) { fz[c] = 0.0f; continue; }
      if (k == 0) f = up ? 0.5f * (a[c] + a[c + sk]) : flx3(a[c + 2 * sk], a[c + sk], a[c]);
      else if (k == 1) f = up ? flx3(a[c - sk], a[c], a[c + sk]) : flx5(a[c + 3 * sk], a[c + 2 * sk], a[c + sk], a[c], a[c - sk]);
      else if (k == g.nz - 2) f = up ? flx5(a[c - 2 * sk], a[c - sk], a[c], a[c + sk], a[c + 2 * sk]) : flx3(a[c + 2 * sk], a[c + sk], a[c]);
      else if (k == g.nz - 1) f = up ? flx3(a[c - sk], a[c], a[c + sk]) : 0.5f * (a[c] + a[c + sk]);
      else f = up ? flx5(a[c - 2 * sk], a[c - sk], a[c], a[c + sk], a[c + 2 * sk])
                  : flx5(a[c + 3 * sk], a[c + 2 * sk], a[c + sk], a[c], a[c - sk]);
    } else {
      if (k == 0 || k == g.nz) { fz[c] = 0.0f; continue; }
      if (k == 1) f = up ? fmaf(c1[k], a[c - sk], c2[k] * a[c]) : flx3(a[c + sk], a[c], a[c - sk]);
      else if (k == 2) f = up ? flx3(a[c - 2 * sk], a[c - sk], a[c]) : flx5(a[c + 2 * sk], a[c + sk], a[c], a[c - sk], a[c - 2 * sk]);
      else if (k == g.nz - 2) f = up ? flx5(a[c - 3 * sk], a[c - 2 * sk], a[c - sk], a[c], a[c + sk]) : flx3(a[c + sk], a[c], a[c - sk]);
      else if (k == g.nz - 1) f = up ? flx3(a[c - 2 * sk], a[c - sk], a[c]) : fmaf(c1[k], a[c - sk], c2[k] * a[c]);
      else f = up ? flx5(a[c - 3 * sk], a[c - 2 * sk], a[c - sk], a[c], a[c + sk])
                  : flx5(a[c + 2 * sk], a[c + sk], a[c], a[c - sk], a[c - 2 * sk]);
    }
    fz[c] = m * f;
  }
}

/* ------------------------------------------------------ WENO fluxes (RK stage 3) */

static void flux_weno_h(uint32_t *M, const uint32_t *ARG, int dir) {
  /* adv_flux_x_weno.wgsl / adv_flux_y_weno.wgsl main (scalars, optional pdef gate) */
  Dims g = dims_at(M, B(0));
  const float *a = FPTR(1), *rr = FPTR(2);
  float weps = FVAL(3);
  int pdef = IVAL(4);
  float *fo = FPTR(5);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (dir == 0 ? (i > g.nx || j >= g.ny || k >= g.nz) : (i >= g.nx || j > g.ny || k >= g.nz)) continue;
    int c = GIDX(g, i, j, k);
    int d = dir == 0 ? 1 : g.sJ;
    float s1, s2, s3, s4, s5;
    if (rr[c] >= 0.0f) { s1 = a[c - 3 * d]; s2 = a[c - 2 * d]; s3 = a[c - d]; s4 = a[c]; s5 = a[c + d]; }
    else { s1 = a[c + 2 * d]; s2 = a[c + d]; s3 = a[c]; s4 = a[c - d]; s5 = a[c - 2 * d]; }
    fo[c] = weno_pdef_ok(s1, s2, s3, s4, s5, weps, pdef == 1) ? rr[c] * WENO(s1, s2, s3, s4, s5, weps) : 0.0f;
  }
}
void teor_adv_flux_x_weno(uint32_t *M, const uint32_t *ARG) { flux_weno_h(M, ARG, 0); }
void teor_adv_flux_y_weno(uint32_t *M, const uint32_t *ARG) { flux_weno_h(M, ARG, 1); }

void teor_adv_flux_z_weno(uint32_t *M, const uint32_t *ARG) {
  /* adv_flux_z_weno.wgsl main: face kf = k+1; c1/c2 interpolation and upstrpd next
   * to the boundaries, positive-definite gating by pdefweno */
  Dims g = dims_at(M, B(0));
  const float *a = FPTR(1), *rrw = FPTR(2), *c1 = FPTR(3), *c2 = FPTR(4);
  float weps = FVAL(5);
  int pdefweno = IVAL(7);
  float *fz = FPTR(8);
  const int sk = g.sJ * g.sK, nk = g.nz;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, kf = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || kf > g.nz + 1) continue;
    int k = kf - 1;
    int c = GIDX(g, i, j, k);
    if (kf == 1 || kf == g.nz + 1) { fz[c] = 0.0f; continue; }
#define A(o) a[c + (o) * sk]
    float w = rrw[c];
    if (kf == 2) {
      fz[c] = w >= 0.0f ? w * fmaf(c1[k], A(-1), c2[k] * A(0)) : w * upstrpd(A(1), A(0), A(-1), weps);
      continue;
    }
    if (kf == nk) {
      fz[c] = w > 0.0f ? w * upstrpd(A(-2), A(-1), A(0), weps) : w * fmaf(c1[k], A(-1), c2[k] * A(0));
      continue;
    }
    float s1, s2, s3, s4, s5;
    if (w >= 0.0f) { s1 = A(-3); s2 = A(-2); s3 = A(-1); s4 = A(0); s5 = A(1); }
    else { s1 = A(2); s2 = A(1); s3 = A(0); s4 = A(-1); s5 = A(-2); }
    if (pdefweno == 1) {
      int doit = weno_pdef_ok(s1, s2, s3, s4, s5, weps, 1);
      if (kf == 3 && w > 0.0f) doit = 0;
      if (kf == nk - 1 && w < 0.0f) doit = 0;
      if (doit) { fz[c] = w * WENO(s1, s2, s3, s4, s5, weps); continue; }
      if (kf != 3 && kf != nk - 1) { fz[c] = 0.0f; continue; }
    }
    if (kf == 3) {
      fz[c] = w >= 0.0f ? w * upstrpd(A(-2), A(-1), A(0), weps) : w * WENO(A(2), A(1), A(0), A(-1), A(-2), weps);
      continue;
    }
    if (kf == nk - 1) {
      fz[c] = w >= 0.0f ? w * WENO(A(-3), A(-2), A(-1), A(0), A(1), weps) : w * upstrpd(A(1), A(0), A(-1), weps);
      continue;
    }
    fz[c] = w * WENO(s1, s2, s3, s4, s5, weps);
#undef A
  }
}

/* f_weno5_upwind (adv_flux_x_weno_uv.wgsl:106-129) */
static inline float weno5_upwind(const float *a, int c, int s, int up, int shifted, float weps) {
  if (shifted) return up ? WENO(a[c - 2 * s], a[c - s], a[c], a[c + s], a[c + 2 * s], weps)
                         : WENO(a[c + 3 * s], a[c + 2 * s], a[c + s], a[c], a[c - s], weps);
  return up ? WENO(a[c - 3 * s], a[c - 2 * s], a[c - s], a[c], a[c + s], weps)
            : WENO(a[c + 2 * s], a[c + s], a[c], a[c - s], a[c - 2 * s], weps);
}

static void flux_weno_uv_h(uint32_t *M, const uint32_t *ARG, int dir) {
  /* adv_flux_x_weno_uv.wgsl / adv_flux_y_weno_uv.wgsl main (u, v momentum) */
  Dims g = dims_at(M, B(0));
  int stag = IVAL(1);
  const float *a = FPTR(2), *rr = FPTR(3);
  float weps = FVAL(4);
  float *fo = FPTR(5);
  const int sj = g.sJ;
  FOR_GRID {
    int i = (int)tx - 1, j = (int)ty - 1, k = (int)tz;
    if (i > g.nx || j > g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float m;
    if (dir == 0) {
      m = stag == 2 ? 0.5f * (rr[c] + rr[c + 1]) : 0.5f * (rr[c] + rr[c - sj]);
      fo[c] = m * weno5_upwind(a, c, 1, m >= 0.0f, stag == 2, weps);
    } else {
      m = stag == 2 ? 0.5f * (rr[c] + rr[c - 1]) : 0.5f * (rr[c] + rr[c + sj]);
      fo[c] = m * weno5_upwind(a, c, sj, m >= 0.0f, stag == 3, weps);
    }
  }
}
void teor_adv_flux_x_weno_uv(uint32_t *M, const uint32_t *ARG) { flux_weno_uv_h(M, ARG, 0); }
void teor_adv_flux_y_weno_uv(uint32_t *M, const uint32_t *ARG) { flux_weno_uv_h(M, ARG, 1); }

void teor_adv_flux_z_weno_uv(uint32_t *M, const uint32_t *ARG) {
  /* adv_flux_z_weno_uv.wgsl main: order reduction at k = 1, 2, nz-2, nz-1 */
  Dims g = dims_at(M, B(0));
  int stag = IVAL(1);
  const float *a = FPTR(2), *rrw = FPTR(3), *c1 = FPTR(4), *c2 = FPTR(5);
  float weps = FVAL(6);
  float *fz = FPTR(7);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > g.nx || j > g.ny || k > g.nz) continue;
    int c = GIDX(g, i, j, k);
    if (k == 0 || k == g.nz) { fz[c] = 0.0f; continue; }
#define A(o) a[c + (o) * sk]
    float m = stag == 2 ? 0.5f * (rrw[c] + rrw[c - 1]) : 0.5f * (rrw[c] + rrw[c - sj]);
    int up = m >= 0.0f;
    float f;
    if (k == 1) f = up ? fmaf(c1[k], A(-1), c2[k] * A(0)) : upstrpd(A(1), A(0), A(-1), weps);
    else if (k == 2) f = up ? upstrpd(A(-2), A(-1), A(0), weps) : WENO(A(2), A(1), A(0), A(-1), A(-2), weps);
    else if (k == g.nz - 2) f = up ? WENO(A(-3), A(-2), A(-1), A(0), A(1), weps) : upstrpd(A(1), A(0), A(-1), weps);
    else if (k == g.nz - 1) f = up ? upstrpd(A(-2), A(-1), A(0), weps) : fmaf(c1[k], A(-1), c2[k] * A(0));
    else f = up ? WENO(A(-3), A(-2), A(-1), A(0), A(1), weps) : WENO(A(2), A(1), A(0), A(-1), A(-2), weps);
    fz[c] = m * f;
#undef A
  }
}

static void flux_weno_w_h(uint32_t *M, const uint32_t *ARG, int dir) {
  /* adv_flux_x_weno_w.wgsl / adv_flux_y_weno_w.wgsl main (w momentum) */
  Dims g = dims_at(M, B(0));
  const float *a = FPTR(1), *rr = FPTR(2), *c2 = FPTR(3);
  float weps = FVAL(4);
  float *fo = FPTR(5);
  const int sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx - 1, j = (int)ty - 1, k = (int)tz;
    if (i < 0 || j < 0 || i > g.nx || j > g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    if (k == 0) { fo[c] = 0.0f; continue; }
    int d = dir == 0 ? 1 : g.sJ;
    float cc2 = c2[k];
    float cc1 = 1.0f - cc2;
    float ub = fmaf(cc2, rr[c], cc1 * rr[c - sk]);
    fo[c] = ub >= 0.0f ? ub * WENO(a[c - 3 * d], a[c - 2 * d], a[c - d], a[c], a[c + d], weps)
                       : ub * WENO(a[c + 2 * d], a[c + d], a[c], a[c - d], a[c - 2 * d], weps);
  }
}
void teor_adv_flux_x_weno_w(uint32_t *M, const uint32_t *ARG) { flux_weno_w_h(M, ARG, 0); }
void teor_adv_flux_y_weno_w(uint32_t *M, const uint32_t *ARG) { flux_weno_w_h(M, ARG, 1); }

void teor_adv_flux_z_weno_w(uint32_t *M, const uint32_t *ARG) {
  /* adv_flux_z_weno_w.wgsl main: w flux at cell centres, wbar = (rrw_k + rrw_k+1)/2 */
  Dims g = dims_at(M, B(0));
  const float *a = FPTR(1), *rrw = FPTR(2);
  float weps = FVAL(3);
  float *fz = FPTR(4);
  const int sk = g.sJ * g.sK, nz = g.nz;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > g.nx || j > g.ny || k > g.nz) continue;
    int c = GIDX(g, i, j, k);
    if (k > g.nz - 1) { fz[c] = 0.0f; continue; }
#define A(o) a[c + (o) * sk]
    float wb = 0.5f * (rrw[c] + rrw[c + sk]);
    float f;
    if (k == 0) f = wb >= 0.0f ? 0.5f * (A(0) + A(1)) : upstrpd(A(2), A(1), A(0), weps);
    else if (k == nz - 1) f = wb > 0.0f ? upstrpd(A(-1), A(0), A(1), weps) : 0.5f * (A(0) + A(1));
    else if (k == 1) f = wb >= 0.0f ? upstrpd(A(-1), A(0), A(1), weps) : WENO(A(3), A(2), A(1), A(0), A(-1), weps);
    else if (k == nz - 2) f = wb > 0.0f ? WENO(A(-2), A(-1), A(0), A(1), A(2), weps) : upstrpd(A(2), A(1), A(0), weps);
    else f = wb >= 0.0f ? WENO(A(-2), A(-1), A(0), A(1), A(2), weps) : WENO(A(3), A(2), A(1), A(0), A(-1), weps);
    fz[c] = wb * f;
#undef A
  }
}

/* ------------------------------------------------------------- flux assembly */

void teor_adv_assemble(uint32_t *M, const uint32_t *ARG) {
  /* adv_assemble.wgsl main (periodic/closed branches; open-boundary inflow branches
   * restated too): t = (s*dv - sum dF*rd*m) / rho, optional accumulation */
  Dims g = dims_at(M, B(0));
  int stag = IVAL(1);
  const float *s = FPTR(2), *fx = FPTR(3), *fy = FPTR(4), *fz = FPTR(5), *divx = FPTR(6);
  const float *rho0 = FPTR(7), *rf0 = FPTR(8), *mh = FPTR(9), *mf = FPTR(10);
  float *tend = FPTR(11);
  int accumulate = IVAL(12);
  const float *rru = FPTR(13), *rrv = FPTR(14), *c1 = FPTR(15), *c2 = FPTR(16);
  int openx = (int)M[B(17)], openy = (int)M[B(17) + 1];
  const float *hm = FPTR(30);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  int st = stag < 0 ? -stag : stag;
  int iMax = st == 2 ? g.nx : g.nx - 1, jMax = st == 3 ? g.ny : g.ny - 1;
  int kLo = st == 4 ? 1 : 0, kMax = g.nz - 1;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > iMax || j > jMax || k < kLo || k > kMax) continue;
    if (openx != 0 && st == 2 && (i == 0 || i == g.nx)) continue;
    if (openy != 0 && st == 3 && (j == 0 || j == g.ny)) continue;
    int c = GIDX(g, i, j, k);
    float dFx = st == 2 ? fx[c] - fx[c - 1] : fx[c + 1] - fx[c];
    float dFy = st == 3 ? fy[c] - fy[c - sj] : fy[c + sj] - fy[c];
    float dFz = st == 4 ? fz[c] - fz[c - sk] : fz[c + sk] - fz[c];
    float mz = stag < 0 ? 1.0f : (stag == 4 ? mf[k] : mh[k]);
    float dv;
    if (st == 2) dv = 0.5f * (divx[c] + divx[c - 1]);
    else if (st == 3) dv = 0.5f * (divx[c] + divx[c - sj]);
    else if (st == 4) dv = fmaf(c2[k], divx[c], c1[k] * divx[c - sk]);
    else dv = divx[c];
    if (openx != 0 && st != 2) {
      int west = i == 0, east = i == g.nx - 1;
      if (west || east) {
        int cf = west ? c : c + 1;
        float un, piece;
        if (st == 3) {
          un = rru[cf] + rru[cf - sj];
          piece = ((0.5f * ((rru[c + 1 - sj] - rru[c - sj]) + (rru[c + 1] - rru[c]))) * g.rdx) * hm_uh(&g, hm, i);
        } else if (st == 4) {
          float cc2 = 0.5f * (c2[k - 1] + c2[k]);
          float cc1 = 1.0f - cc2;
          un = fmaf(cc2, rru[cf], cc1 * rru[cf - sk]);
          piece = (fmaf(c1[k], rru[c + 1 - sk] - rru[c - sk], c2[k] * (rru[c + 1] - rru[c])) * g.rdx) * hm_uh(&g, hm, i);
        } else {
          un = rru[cf];
          piece = ((rru[c + 1] - rru[c]) * g.rdx) * hm_uh(&g, hm, i);
        }
        int inflow = west ? un >= 0.0f : un <= 0.0f;
        if (inflow) { dFx = 0.0f; dv = dv - piece; }
      }
    }
    if (openy != 0 && st != 3) {
      int south = j == 0, north = j == g.ny - 1;
      if (south || north) {
        int cf = south ? c : c + sj;
        float vn, piece;
        if (st == 2) {
          vn = rrv[cf] + rrv[cf - 1];
          piece = ((0.5f * ((rrv[c + sj - 1] - rrv[c - 1]) + (rrv[c + sj] - rrv[c]))) * g.rdy) * hm_vh(&g, hm, j);
        } else if (st == 4) {
          float cc2 = 0.5f * (c2[k - 1] + c2[k]);
          float cc1 = 1.0f - cc2;
          vn = fmaf(cc2, rrv[cf], cc1 * rrv[cf - sk]);
          piece = (fmaf(c1[k], rrv[c + sj - sk] - rrv[c - sk], c2[k] * (rrv[c + sj] - rrv[c])) * g.rdy) * hm_vh(&g, hm, j);
        } else {
          vn = rrv[cf];
          piece = ((rrv[c + sj] - rrv[c]) * g.rdy) * hm_vh(&g, hm, j);
        }
        int inflow = south ? vn >= 0.0f : vn <= 0.0f;
        if (inflow) { dFy = 0.0f; dv = dv - piece; }
      }
    }
    float mx = st == 2 ? hm_uf(&g, hm, i) : hm_uh(&g, hm, i);
    float my = st == 3 ? hm_vf(&g, hm, j) : hm_vh(&g, hm, j);
    float divF = fmaf(dFz * g.rdz, mz, fmaf(dFx * g.rdx, mx, (dFy * g.rdy) * my));
    float rho = st == 4 ? rf0[k] : rho0[k];
    float t = DCR(fmaf(s[c], dv, -divF), rho);
    tend[c] = accumulate != 0 ? tend[c] + t : t;
  }
}

void teor_rk_update(uint32_t *M, const uint32_t *ARG) {
  /* rk_update.wgsl main: phi = fma(dttmp, tend, phi_a) */
  Dims g = dims_at(M, B(0));
  int stag = IVAL(1);
  const float *phiA = FPTR(2), *tend = FPTR(3);
  float *phi = FPTR(4);
  float dttmp = FVAL(5);
  int iMax = stag == 2 ? g.nx : g.nx - 1, jMax = stag == 3 ? g.ny : g.ny - 1, kLo = stag == 4 ? 1 : 0;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > iMax || j > jMax || k < kLo || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    phi[c] = fmaf(dttmp, tend[c], phiA[c]);
  }
}

/* f_pdef_inflow (pdef_dum.wgsl:108-134) */
static inline int pdef_inflow(const Dims *g, int dir, int i, int j, int c, int step, const float *rr, int ox, int oy) {
  if (dir == 0 && ox != 0) {
    if (i == 0 && rr[c] >= 0.0f) return 1;
    if (i == g->nx - 1 && rr[c + step] <= 0.0f) return 1;
  }
  if (dir == 1 && oy != 0) {
    if (j == 0 && rr[c] >= 0.0f) return 1;
    if (j == g->ny - 1 && rr[c + step] <= 0.0f) return 1;
  }
  return 0;
}

void teor_pdef_dum(uint32_t *M, const uint32_t *ARG) {
  /* pdef_dum.wgsl main: provisional mass after advection along one direction */
  Dims g = dims_at(M, B(0));
  int dir = IVAL(1);
  const float *s = FPTR(2), *s0 = FPTR(3), *f = FPTR(4), *rr = FPTR(5), *rho0 = FPTR(6), *mh = FPTR(7);
  float dt = FVAL(8);
  int ox = (int)M[B(9)], oy = (int)M[B(9) + 1];
  float *dum = FPTR(10);
  const float *hm = FPTR(30);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    int step = dir == 0 ? 1 : (dir == 1 ? g.sJ : g.sJ * g.sK);
    float rd = dir == 0 ? g.rdx : (dir == 1 ? g.rdy : g.rdz);
    float base = rho0[k] * s0[c];
    if (pdef_inflow(&g, dir, i, j, c, step, rr, ox, oy)) { dum[c] = base; continue; }
    float adv = (-(f[c + step] - f[c])) * rd;
    float sdiv = (s[c] * (rr[c + step] - rr[c])) * rd;
    float m = dir == 0 ? hm_uh(&g, hm, i) : (dir == 1 ? hm_vh(&g, hm, j) : mh[k]);
    adv = adv * m;
    sdiv = sdiv * m;
    dum[c] = fmaf(dt, adv + sdiv, base);
  }
}

/* f_pdef_cell / f_pdef_mass (pdef_apply.wgsl:115-158), K_PDEF_SMEPS = 1e-30 */
typedef struct { int neg; float f1, f2, foo3; } PdefCell;
static inline PdefCell pdef_cell(float d, float dm, float dp) {
  PdefCell r = {0, 0.0f, 0.0f, 0.0f};
  if (d < 0.0f) {
    float f1 = fmax_(0.0f, dm), f2 = fmax_(0.0f, dp);
    if (f1 + f2 > 1e-30f) {
      r.neg = 1;
      r.f1 = f1;
      r.f2 = f2;
      r.foo3 = DCR(fmax_(d, -(f1 + f2)), f1 + f2);
    }
  }
  return r;
}
static inline float pdef_mass(float dm2, float dm1, float d0, float dp1, float dp2, int *flag) {
  PdefCell l = pdef_cell(dm1, dm2, d0), c = pdef_cell(d0, dm1, dp1), r = pdef_cell(dp1, d0, dp2);
  float mass = 0.0f;
  if (l.neg) mass = fmaf(l.f2, l.foo3, mass);
  if (c.neg) mass = fmaf(-(c.f1 + c.f2), c.foo3, mass);
  if (r.neg) mass = fmaf(r.f1, r.foo3, mass);
  *flag = c.neg || (l.neg && d0 > 1e-30f) || (r.neg && d0 > 1e-30f);
  return mass;
}

void teor_pdef_apply(uint32_t *M, const uint32_t *ARG) {
  /* pdef_apply.wgsl main: replace the advective tendency where the provisional mass
   * would go negative */
  Dims g = dims_at(M, B(0));
  const float *s = FPTR(1), *s0 = FPTR(2), *fx = FPTR(3), *fy = FPTR(4), *fz = FPTR(5);
  const float *rru = FPTR(6), *rrv = FPTR(7), *rrw = FPTR(8), *dumx = FPTR(9), *dumy = FPTR(10), *dumz = FPTR(11);
  const float *rho0 = FPTR(12), *mh = FPTR(13);
  float dt = FVAL(14);
  int ox = (int)M[B(15)], oy = (int)M[B(15) + 1];
  float *tend = FPTR(16);
  const float *hm = FPTR(30);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float rdt = DCR(1.0f, dt);
    float base = rho0[k] * s0[c];
    float delta = 0.0f;
    int flag;
    float mx = pdef_mass(dumx[c - 2], dumx[c - 1], dumx[c], dumx[c + 1], dumx[c + 2], &flag);
    if (flag) {
      float sdiv = ((s[c] * (rru[c + 1] - rru[c])) * g.rdx) * hm_uh(&g, hm, i);
      float advOld = pdef_inflow(&g, 0, i, j, c, 1, rru, ox, oy) ? -sdiv : ((-(fx[c + 1] - fx[c])) * g.rdx) * hm_uh(&g, hm, i);
      float advNew = fmaf((dumx[c] + mx) - base, rdt, -sdiv);
      delta = delta + (advNew - advOld);
    }
    float my = pdef_mass(dumy[c - 2 * sj], dumy[c - sj], dumy[c], dumy[c + sj], dumy[c + 2 * sj], &flag);
    if (flag) {
      float sdiv = ((s[c] * (rrv[c + sj] - rrv[c])) * g.rdy) * hm_vh(&g, hm, j);
      float advOld = pdef_inflow(&g, 1, i, j, c, sj, rrv, ox, oy) ? -sdiv : ((-(fy[c + sj] - fy[c])) * g.rdy) * hm_vh(&g, hm, j);
      float advNew = fmaf((dumy[c] + my) - base, rdt, -sdiv);
      delta = delta + (advNew - advOld);
    }
    float zm2 = k >= 2 ? dumz[c - 2 * sk] : 0.0f;
    float zm1 = k >= 1 ? dumz[c - sk] : 0.0f;
    float zp1 = k + 1 < g.nz ? dumz[c + sk] : 0.0f;
    float zp2 = k + 2 < g.nz ? dumz[c + 2 * sk] : 0.0f;
    float mz = pdef_mass(zm2, zm1, dumz[c], zp1, zp2, &flag);
    if (flag) {
      float sdiv = ((s[c] * (rrw[c + sk] - rrw[c])) * g.rdz) * mh[k];
      float advOld = ((-(fz[c + sk] - fz[c])) * g.rdz) * mh[k];
      float advNew = fmaf((dumz[c] + mz) - base, rdt, -sdiv);
      delta = delta + (advNew - advOld);
    }
    tend[c] = tend[c] + DCR(delta, rho0[k]);
  }
}

/* ----------------------------------------------------------- whole-grid glue */

#define FOR_WHOLE(kcond)                                    \
  FOR_GRID {                                                \
    int i = (int)tx - 3, j = (int)ty - 3, k = (int)tz;      \
    if (i > g.nx + 3 || j > g.ny + 3 || !(kcond)) continue; \
    int c = GIDX(g, i, j, k);

void teor_build_sadv(uint32_t *M, const uint32_t *ARG) {
  /* build_sadv.wgsl main: sadv = (th0 - 300) + th' */
  Dims g = dims_at(M, B(0));
  const float *th0 = FPTR(1), *thp = FPTR(2);
  float *sadv = FPTR(3);
  FOR_WHOLE(k < g.nz)
    sadv[c] = (th0[k] - 300.0f) + thp[c];
  }
}

void teor_massflux_from_state(uint32_t *M, const uint32_t *ARG) {
  /* massflux_from_state.wgsl main: rru = rho0 u, rrv = rho0 v, rrw = rf0 w (0 at k=0, nz) */
  Dims g = dims_at(M, B(0));
  const float *u = FPTR(1), *v = FPTR(2), *w = FPTR(3), *rho0 = FPTR(4), *rf0 = FPTR(5);
  float *rru = FPTR(6), *rrv = FPTR(7), *rrw = FPTR(8);
  FOR_WHOLE(k <= g.nz)
    if (k < g.nz) {
      rru[c] = rho0[k] * u[c];
      rrv[c] = rho0[k] * v[c];
    }
    rrw[c] = (k == 0 || k == g.nz) ? 0.0f : rf0[k] * w[c];
  }
}

void teor_div_massflux(uint32_t *M, const uint32_t *ARG) {
  /* div_massflux.wgsl main */
  Dims g = dims_at(M, B(0));
  const float *rru = FPTR(1), *rrv = FPTR(2), *rrw = FPTR(3), *mh = FPTR(4);
  float *divx = FPTR(5);
  const float *hm = FPTR(30);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx - 3, j = (int)ty - 3, k = (int)tz;
    if (i > g.nx + 2 || j > g.ny + 2 || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    divx[c] = fmaf((rrw[c + sk] - rrw[c]) * g.rdz, mh[k],
                   fmaf((rru[c + 1] - rru[c]) * g.rdx, hm_uh(&g, hm, i), ((rrv[c + sj] - rrv[c]) * g.rdy) * hm_vh(&g, hm, j)));
  }
}

void teor_velocity_to_massflux(uint32_t *M, const uint32_t *ARG) {
  /* velocity_to_massflux.wgsl main */
  Dims g = dims_at(M, B(0));
  const float *rho0 = FPTR(1), *rf0 = FPTR(2);
  float *rru = FPTR(3), *rrv = FPTR(4), *rrw = FPTR(5);
  FOR_WHOLE(k <= g.nz)
    if (k < g.nz) {
      rru[c] = rru[c] * rho0[k];
      rrv[c] = rrv[c] * rho0[k];
    }
    rrw[c] = (k == 0 || k == g.nz) ? 0.0f : rrw[c] * rf0[k];
  }
}

void teor_stage_state_reset(uint32_t *M, const uint32_t *ARG) {
  /* stage_state_reset.wgsl main */
  Dims g = dims_at(M, B(0));
  const float *ua = FPTR(1), *va = FPTR(2), *wa = FPTR(3), *ppi = FPTR(4);
  float *u = FPTR(5), *v = FPTR(6), *w = FPTR(7), *pp3d = FPTR(8), *ppd = FPTR(9);
  const float *ppx = FPTR(10);
  FOR_WHOLE(k <= g.nz)
    u[c] = ua[c];
    v[c] = va[c];
    w[c] = wa[c];
    pp3d[c] = ppi[c];
    ppd[c] = ppx[c];
  }
}

void teor_stage_tendency_reset(uint32_t *M, const uint32_t *ARG) {
  /* stage_tendency_reset.wgsl main */
  Dims g = dims_at(M, B(0));
  float *uten = FPTR(1), *vten = FPTR(2), *wten = FPTR(3);
  FOR_WHOLE(k <= g.nz)
    uten[c] = 0.0f;
    vten[c] = 0.0f;
    wten[c] = 0.0f;
  }
}

void teor_buoyancy_apply(uint32_t *M, const uint32_t *ARG) {
  /* buoyancy_apply.wgsl main: wten += c1 buoy(k-1) + c2 buoy(k) on interior faces */
  Dims g = dims_at(M, B(0));
  const float *buoy = FPTR(1), *c1 = FPTR(2), *c2 = FPTR(3);
  float *wten = FPTR(4);
  const int sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k);
    wten[c] = wten[c] + fmaf(c1[k], buoy[c - sk], c2[k] * buoy[c]);
  }
}

void teor_apply_thterm(uint32_t *M, const uint32_t *ARG) {
  /* apply_thterm.wgsl main: tend -= div * thterm */
  Dims g = dims_at(M, B(0));
  const float *div = FPTR(1), *thterm = FPTR(2);
  float *tend = FPTR(3);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    tend[c] = fmaf(-div[c], thterm[c], tend[c]);
  }
}

/* ---------------------------------------------------------- acoustic substep */

void teor_acoustic_prepare(uint32_t *M, const uint32_t *ARG) {
  /* acoustic_prepare.wgsl main: qk, pk1, pk2, mm; the pk fma order depends on
   * whether i falls in CM1's vectorised part of the loop (vec_v) */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *ppterm = FPTR(2), *piadv = FPTR(3), *thv = FPTR(4), *rr0 = FPTR(5), *rf0 = FPTR(6);
  const float *mh = FPTR(7), *mf = FPTR(8), *c1 = FPTR(9), *c2 = FPTR(10);
  float *qk = FPTR(11), *pk1 = FPTR(12), *pk2 = FPTR(13), *mm = FPTR(14);
  const int sk = g.sJ * g.sK;
  const float cp = CP_;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float tem = (a.dts * g.rdz) * mh[k];
    float r2 = (tem * rr0[k]) * rf0[k + 1];
    float r1 = (tem * rr0[k]) * rf0[k];
    float tem1 = ((a.dts * g.rdz) * cp) * mf[k];
    float c1a = c1[k], c1b = c1[k + 1], c2a = c2[k], c2b = c2[k + 1];
    int vec_v = g.nx > 3 && i < (g.nx / 4) * 4;
    qk[c] = tem * ppterm[c];
    float p2 = 0.0f, p1 = 0.0f;
    if (k != g.nz - 1)
      p2 = vec_v ? fmaf(-c2b, piadv[c + sk], (1.0f - c1b) * piadv[c])
                 : fmaf(1.0f - c1b, piadv[c], -(c2b * piadv[c + sk]));
    if (k != 0)
      p1 = vec_v ? fmaf(c2a - 1.0f, piadv[c], c1a * piadv[c - sk])
                 : fmaf(c1a, piadv[c - sk], (c2a - 1.0f) * piadv[c]);
    pk2[c] = k == g.nz - 1 ? 0.0f : r2 * p2;
    pk1[c] = k == 0 ? 0.0f : r1 * p1;
    mm[c] = tem1 * fmaf(c2a, thv[c], c1a * (k == 0 ? thv[c] : thv[c - sk]));
  }
}

void teor_acoustic_begin(uint32_t *M, const uint32_t *ARG) {
  /* acoustic_begin.wgsl main: rru = rrv = 0, rrw = beta w */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *w = FPTR(2);
  float *rru = FPTR(3), *rrv = FPTR(4), *rrw = FPTR(5);
  FOR_WHOLE(k <= g.nz)
    rru[c] = 0.0f;
    rrv[c] = 0.0f;
    rrw[c] = w[c] * a.beta;
  }
}

void teor_acoustic_uv(uint32_t *M, const uint32_t *ARG) {
  /* acoustic_uv.wgsl main: horizontal pi'-gradient update of u and v */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *ppd = FPTR(2), *thv = FPTR(3), *uten = FPTR(4), *vten = FPTR(5);
  float *u = FPTR(6), *v = FPTR(7);
  int ox = (int)M[B(8)], oy = (int)M[B(8) + 1];
  const float *hm = FPTR(30);
  const int sj = g.sJ;
  const float cp = CP_;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > g.nx || j > g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float tem1 = (g.rdx * cp) * 0.5f;
    float tem2 = (g.rdy * cp) * 0.5f;
    int uEdge = ox != 0 && (i == 0 || i == g.nx);
    int vEdge = oy != 0 && (j == 0 || j == g.ny);
    if (!uEdge)
      u[c] = fmaf(a.dts, fmaf(-((tem1 * (ppd[c] - ppd[c - 1])) * hm_uf(&g, hm, i)), thv[c] + thv[c - 1], uten[c]), u[c]);
    if (!vEdge)
      v[c] = fmaf(a.dts, fmaf(-((tem2 * (ppd[c] - ppd[c - sj])) * hm_vf(&g, hm, j)), thv[c] + thv[c - sj], vten[c]), v[c]);
  }
}

void teor_acoustic_fpk(uint32_t *M, const uint32_t *ARG) {
  /* acoustic_fpk.wgsl main: explicit forcing of the pi' equation */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *u = FPTR(2), *v = FPTR(3), *w = FPTR(4), *piadv = FPTR(5), *ppten = FPTR(6), *ppterm = FPTR(7);
  const float *pk1 = FPTR(8), *pk2 = FPTR(9), *qk = FPTR(10);
  float *fpk = FPTR(11);
  const float *hm = FPTR(30);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float temx = (a.dts * 0.5f) * g.rdx;
    float temy = (a.dts * 0.5f) * g.rdy;
    float div = fmaf((u[c + 1] - u[c]) * g.rdx, hm_uh(&g, hm, i), ((v[c + sj] - v[c]) * g.rdy) * hm_vh(&g, hm, j));
    if (fabsf(div) < a.smeps) div = 0.0f;
    float advPi = fmaf((-fmaf(u[c], piadv[c] - piadv[c - 1], u[c + 1] * (piadv[c + 1] - piadv[c]))) * temx, hm_uh(&g, hm, i),
                       -((fmaf(v[c], piadv[c] - piadv[c - sj], v[c + sj] * (piadv[c + sj] - piadv[c])) * temy) * hm_vh(&g, hm, j)));
    fpk[c] = fmaf(a.beta, fmaf(w[c], pk1[c] + qk[c], w[c + sk] * (pk2[c] - qk[c])),
                  fmaf(a.dts, fmaf(-ppterm[c], div, ppten[c]), advPi));
  }
}

void teor_acoustic_w_solve(uint32_t *M, const uint32_t *ARG) {
  /* acoustic_w_solve.wgsl main + lam_1 (:124-139): per column, tridiagonal Thomas solve
   * for w on faces k = 1..nz-1 with w(0) = w(nz) = 0; forward sweep stores cA, cB */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *pk1 = FPTR(2), *pk2 = FPTR(3), *qk = FPTR(4), *mm = FPTR(5), *fpk = FPTR(6), *wten = FPTR(7), *pp3d = FPTR(8);
  float *w = FPTR(9), *cA = FPTR(10), *cB = FPTR(11);
  const int sk = g.sJ * g.sK;
  const long GX = ARG[0], GY = ARG[1];
#pragma omp parallel for collapse(2) schedule(static)
  for (long ty = 0; ty < GY; ty++)
    for (long tx = 0; tx < GX; tx++) {
      int i = (int)tx, j = (int)ty;
      if (i >= g.nx || j >= g.ny) continue;
      float asq = a.alph * a.alph;
      w[GIDX(g, i, j, 0)] = 0.0f;
      w[GIDX(g, i, j, g.nz)] = 0.0f;
      float aa, bb, cc, dd;
#define LAM(kk)                                                                     \
  do {                                                                              \
    int c_ = GIDX(g, i, j, (kk)), cm_ = c_ - sk;                                    \
    float m_ = mm[c_];                                                              \
    aa = (-asq) * (m_ * (pk1[cm_] + qk[cm_]));                                      \
    cc = (-asq) * ((-m_) * (pk2[c_] - qk[c_]));                                     \
    bb = fmaf(-asq, m_ * ((-(pk1[c_] + qk[c_])) + (pk2[cm_] - qk[cm_])), 1.0f);     \
    float fw_ = fmaf(a.dts, wten[c_], a.beta * ((-m_) * (pp3d[c_] - pp3d[cm_])));   \
    dd = fmaf(a.alph, (-m_) * ((pp3d[c_] + fpk[c_]) - (pp3d[cm_] + fpk[cm_])), w[c_] + fw_); \
  } while (0)
      {
        int c = GIDX(g, i, j, 1);
        LAM(1);
        float r = DCR(1.0f, bb);
        cA[c] = (-cc) * r;
        cB[c] = dd * r;
      }
      for (int k = 2; k < g.nz - 1; k++) {
        int c = GIDX(g, i, j, k);
        LAM(k);
        float r = DCR(1.0f, fmaf(aa, cA[c - sk], bb));
        cA[c] = (-cc) * r;
        cB[c] = fmaf(-aa, cB[c - sk], dd) * r;
      }
      {
        int k = g.nz - 1, c = GIDX(g, i, j, k);
        LAM(k);
        float r = DCR(1.0f, fmaf(aa, cA[c - sk], bb));
        w[c] = fmaf(-aa, cB[c - sk], dd) * r;
      }
#undef LAM
      for (int k = g.nz - 2; k >= 1; k--) {
        int c = GIDX(g, i, j, k);
        w[c] = fmaf(cA[c], w[c + sk], cB[c]);
      }
    }
}

void teor_acoustic_pp(uint32_t *M, const uint32_t *ARG) {
  /* acoustic_pp.wgsl main: pi' update, divergence damping ppd, ppx on stage 3 */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *w = FPTR(2), *pk1 = FPTR(3), *pk2 = FPTR(4), *qk = FPTR(5), *fpk = FPTR(6);
  float *pp3d = FPTR(7), *ppd = FPTR(8), *ppx = FPTR(9);
  int saveX = IVAL(10);
  const int sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float prev = pp3d[c];
    float w1 = w[c], w2 = w[c + sk];
    float p = fmaf(a.alph, fmaf(w1, pk1[c] + qk[c], w2 * (pk2[c] - qk[c])), prev + fpk[c]);
    if (fabsf(p) < a.smeps) p = 0.0f;
    pp3d[c] = p;
    float dum1 = a.kdiv * (p - prev);
    ppd[c] = p + dum1;
    if (saveX != 0) ppx[c] = dum1;
  }
}

void teor_acoustic_accumulate(uint32_t *M, const uint32_t *ARG) {
  /* acoustic_accumulate.wgsl main: substep sums, averaged on the last substep */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *u = FPTR(2), *v = FPTR(3), *w = FPTR(4);
  float *rru = FPTR(5), *rrv = FPTR(6), *rrw = FPTR(7);
  float tavg = FVAL(8);
  FOR_WHOLE(k <= g.nz)
    if (tavg > 0.0f) {
      rru[c] = (rru[c] + u[c]) * tavg;
      rrv[c] = (rrv[c] + v[c]) * tavg;
      rrw[c] = fmaf(w[c], a.alph, rrw[c]) * tavg;
    } else {
      rru[c] = rru[c] + u[c];
      rrv[c] = rrv[c] + v[c];
      rrw[c] = rrw[c] + w[c];
    }
  }
}

/* --------------------------------------------------------- periodic halos */

void teor_bc_periodic_x(uint32_t *M, const uint32_t *ARG) {
  /* bc_periodic_x.wgsl main: i = -1-h <- nx-1-h (h < 3), i = nx+h <- h (h <= 3) */
  Dims g = dims_at(M, B(0));
  float *f = FPTR(1);
  FOR_GRID {
    int h = (int)tx, jj = (int)ty - 3, k = (int)tz;
    if (h > 3 || jj > g.ny + 3 || k > g.nz) continue;
    int lo = (((-1 - h) % g.nx) + g.nx) % g.nx;
    int hi = (((g.nx + h) % g.nx) + g.nx) % g.nx;
    if (h < 3) f[GIDX(g, -1 - h, jj, k)] = f[GIDX(g, lo, jj, k)];
    f[GIDX(g, g.nx + h, jj, k)] = f[GIDX(g, hi, jj, k)];
  }
}

void teor_bc_periodic_y(uint32_t *M, const uint32_t *ARG) {
  /* bc_periodic_y.wgsl main */
  Dims g = dims_at(M, B(0));
  float *f = FPTR(1);
  FOR_GRID {
    int h = (int)tx, i = (int)ty - 3, k = (int)tz;
    if (h > 3 || i > g.nx + 3 || k > g.nz) continue;
    int lo = (((-1 - h) % g.ny) + g.ny) % g.ny;
    int hi = (((g.ny + h) % g.ny) + g.ny) % g.ny;
    if (h < 3) f[GIDX(g, i, -1 - h, k)] = f[GIDX(g, i, lo, k)];
    f[GIDX(g, i, g.ny + h, k)] = f[GIDX(g, i, hi, k)];
  }
}

/* ------------------------------------------------------ thermodynamic glue */

void teor_update_diagnostics(uint32_t *M, const uint32_t *ARG) {
  /* update_diagnostics.wgsl main (dry step): thv = th0 + th', piadv = pi, ppterm = pi rd/(cp-rd),
   * buoy = (g th') / th0 */
  Dims g = dims_at(M, B(0));
  const float *thp = FPTR(1), *ppp = FPTR(2), *th0 = FPTR(3), *pi0 = FPTR(4), *rth0 = FPTR(8);
  float *thv = FPTR(5), *ppterm = FPTR(6), *piadv = FPTR(7), *buoy = FPTR(9);
  FOR_WHOLE(k < g.nz)
    float rd = 287.04f, cp = 1005.7f;
    float rddcv = DCR(rd, cp - rd);
    float pi = pi0[k] + ppp[c];
    thv[c] = th0[k] + thp[c];
    piadv[c] = pi;
    ppterm[c] = pi * rddcv;
    buoy[c] = (9.81f * thp[c]) * rth0[k];
  }
}

void teor_stability_max(uint32_t *M, const uint32_t *ARG) {
  /* stability_max.wgsl main: max over interior points of the squared Courant number and of
   * the diffusion number (bit patterns of non-negative floats, atomicMax into out[0..1]) */
  Dims g = dims_at(M, B(0));
  const uint32_t pw = B(1);
  const float dtdx = bitsf(M[pw]), dtdy = bitsf(M[pw + 1]), dtdz = bitsf(M[pw + 2]);
  const float ksdx = bitsf(M[pw + 3]), ksdy = bitsf(M[pw + 4]);
  const int twoD = (int)M[pw + 5], withKs = (int)M[pw + 6];
  const float *u = FPTR(2), *v = FPTR(3), *w = FPTR(4), *mh = FPTR(5), *kmh = FPTR(6), *kmv = FPTR(7), *khh = FPTR(8);
  const float *hm = FPTR(30);
  uint32_t *out = M + B(9);
  const long GX = ARG[0], GY = ARG[1], GZ = ARG[2];
  uint32_t cbmax = 0, kbmax = 0;
  for (long tz = 0; tz < GZ; tz++)
    for (long ty = 0; ty < GY; ty++)
      for (long tx = 0; tx < GX; tx++) {
        int i = (int)tx, j = (int)ty, k = (int)tz;
        if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
        int c = GIDX(g, i, j, k);
        float uh = hm_uh(&g, hm, i), vh = hm_vh(&g, hm, j);
        float x = ((u[c] + u[GIDX(g, i + 1, j, k)]) * dtdx) * uh;
        float z = ((w[c] + w[GIDX(g, i, j, k + 1)]) * dtdz) * mh[k];
        float c2, m = 0.0f;
        if (twoD != 0) c2 = fmaf(x, x, z * z);
        else {
          float y = ((v[c] + v[GIDX(g, i, j + 1, k)]) * dtdy) * vh;
          c2 = fmaf(z, z, fmaf(x, x, y * y));
        }
        if (withKs != 0 && k >= 1) {
          float K[3] = {kmh[c], khh[c], kmv[c]};
          for (int n = 0; n < 3; n++) {
            float a = ((K[n] * ksdx) * uh) * uh;
            float t;
            if (twoD != 0) t = a;
            else {
              float b = ((K[n] * ksdy) * vh) * vh;
              t = fmaf(a, a, b * b);
            }
            m = fmax_(m, t);
          }
        }
        if (fbits(c2) > cbmax) cbmax = fbits(c2);
        if (fbits(m) > kbmax) kbmax = fbits(m);
      }
  if (cbmax > out[0]) out[0] = cbmax;
  if (kbmax > out[1]) out[1] = kbmax;
}

void teor_update_diagnostics_moist(uint32_t *M, const uint32_t *ARG) {
  /* update_diagnostics_moist.wgsl main: thv, piadv, ppterm, thterm, buoy */
  Dims g = dims_at(M, B(0));
  const float *thp = FPTR(1), *ppp = FPTR(2), *th0 = FPTR(3), *pi0 = FPTR(4), *qv0 = FPTR(5), *qc0 = FPTR(6);
  const float *qi0 = FPTR(7), *rth0 = FPTR(8), *qv = FPTR(9), *qc = FPTR(10), *qr = FPTR(11), *qi = FPTR(12);
  const float *qs = FPTR(13), *qg = FPTR(14);
  float *thv = FPTR(15), *ppterm = FPTR(16), *piadv = FPTR(17), *thterm = FPTR(18), *buoy = FPTR(19);
  const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, cv = 718.66003f, cpv = 1870.0f, cvv = 1408.5f;
  const float rovcp = 0.28541315f, cpl = 4190.0f, cpi = 2106.0f;
  FOR_WHOLE(k < g.nz)
    float reps = DCR(rv, rd);
    float repsm1 = reps - 1.0f;
    float gacc = 9.81f;
    float qvv = fmax_(qv[c], 0.0f);
    float liq = qc[c] + qr[c];
    float ice = (qi[c] + qs[c]) + qg[c];
    float qli = fmax_(0.0f, liq + ice);
    float cpli = fmaf(cpl, fmax_(0.0f, liq), cpi * fmax_(0.0f, ice));
    float th = th0[k] + thp[c];
    float pi = pi0[k] + ppp[c];
    float cpm = fmaf(cpv, qvv, cp) + cpli;
    float cvm = DCR(1.0f, fmaf(cvv, qvv, cv) + cpli);
    thv[c] = DCR(th * fmaf(reps, qvv, 1.0f), (1.0f + qvv) + qli);
    piadv[c] = pi;
    ppterm[c] = ((pi * rovcp) * cpm) * cvm;
    thterm[c] = (th * fmaf(-rovcp, cpm, fmaf(rv, qvv, rd))) * cvm;
    buoy[c] = gacc * (fmaf(thp[c], rth0[k], repsm1 * (qvv - qv0[k])) - ((qli - qc0[k]) - qi0[k]));
  }
}

/* f_rr_* double-float helpers (pressure_tendency.wgsl:114-226): a correctly rounded
 * powf built from a two-float log and exp */
typedef struct { float x, y; } F2;
static inline F2 two_sum(float a, float b) {
  float s = a + b, bb = s - a;
  F2 r = {s, (a - (s - bb)) + (b - bb)};
  return r;
}
static inline F2 quick_two_sum(float a, float b) {
  float s = a + b;
  F2 r = {s, b - (s - a)};
  return r;
}
static inline F2 mul_ff(F2 a, F2 b) {
  float p = a.x * b.x;
  float e = fmaf(a.x, b.x, -p);
  e = fmaf(a.x, b.y, e);
  e = fmaf(a.y, b.x, e);
  return quick_two_sum(p, e);
}
static inline F2 add_ff(F2 a, F2 b) {
  F2 s = two_sum(a.x, b.x), t = two_sum(a.y, b.y);
  F2 u = quick_two_sum(s.x, s.y + t.x);
  return quick_two_sum(u.x, u.y + t.y);
}
static inline F2 mkf2(float x, float y) { F2 r = {x, y}; return r; }
static F2 rr_log_ff(float x) {
  int e;
  float m = frexpf(x, &e);
  if (m < 0.70710677f) { m = m * 2.0f; e = e - 1; }
  float f = m - 1.0f;
  F2 d = two_sum(2.0f, f);
  float sh = DCR(f, d.x);
  float r = fmaf(-sh, d.x, f);
  r = fmaf(-sh, d.y, r);
  F2 sf = quick_two_sum(sh, DCR(r, d.x));
  F2 s2 = mul_ff(sf, sf), s3 = mul_ff(s2, sf);
  F2 P = mkf2(0.11764706f, -4.3826945e-10f);
  P = add_ff(mul_ff(P, s2), mkf2(0.13333334f, -6.9538753e-09f));
  P = add_ff(mul_ff(P, s2), mkf2(0.15384616f, -5.731216e-09f));
  P = add_ff(mul_ff(P, s2), mkf2(0.18181819f, -5.4186042e-09f));
  P = add_ff(mul_ff(P, s2), mkf2(0.22222222f, -1.6556846e-09f));
  P = add_ff(mul_ff(P, s2), mkf2(0.2857143f, -1.2772424e-08f));
  P = add_ff(mul_ff(P, s2), mkf2(0.4f, -5.9604646e-09f));
  P = add_ff(mul_ff(P, s2), mkf2(0.6666667f, -1.9868216e-08f));
  F2 l1p = add_ff(mkf2(2.0f * sf.x, 2.0f * sf.y), mul_ff(s3, P));
  const float ln2h = 0.69314575f, ln2m = 1.4285906e-06f, ln2l = 1.6198487e-11f;
  float fe = (float)e;
  F2 a = add_ff(mkf2(fe * ln2h, fe * ln2m), l1p);
  return add_ff(a, mkf2(fe * ln2l, 0.0f));
}
static float rr_exp_ff(F2 y) {
  const float ln2h = 0.69314575f, ln2m = 1.4285906e-06f, ln2l = 1.6198487e-11f;
  float k = nearbyintf(DCR(y.x, 0.6931472f));
  F2 r = add_ff(y, mkf2((-k) * ln2h, (-k) * ln2m));
  r = add_ff(r, mkf2((-k) * ln2l, 0.0f));
  F2 P = mkf2(2.5052108e-08f, 4.417623e-16f);
  P = add_ff(mul_ff(P, r), mkf2(2.755732e-07f, -7.575112e-15f));
  P = add_ff(mul_ff(P, r), mkf2(2.7557319e-06f, 3.7935712e-14f));
  P = add_ff(mul_ff(P, r), mkf2(2.4801588e-05f, -3.406996e-13f));
  P = add_ff(mul_ff(P, r), mkf2(0.0001984127f, -2.7255969e-12f));
  P = add_ff(mul_ff(P, r), mkf2(0.0013888889f, -3.3631094e-11f));
  P = add_ff(mul_ff(P, r), mkf2(0.008333334f, -4.346172e-10f));
  P = add_ff(mul_ff(P, r), mkf2(0.041666668f, -1.2417635e-09f));
  P = add_ff(mul_ff(P, r), mkf2(0.16666667f, -4.967054e-09f));
  P = add_ff(mul_ff(P, r), mkf2(0.5f, 0.0f));
  P = add_ff(mul_ff(P, r), mkf2(1.0f, 0.0f));
  F2 Q = mul_ff(P, r);
  float s = 1.0f + Q.x;
  float t = (1.0f - s) + Q.x;
  F2 ur = two_sum(t, Q.y);
  float res = s + ur.x;
  float bb = res - s;
  float e3 = (s - (res - bb)) + (ur.x - bb);
  if (e3 != 0.0f && ur.y != 0.0f && (e3 > 0.0f) == (ur.y > 0.0f)) {
    float nb = bitsf(fbits(res) + (e3 > 0.0f ? 1u : 4294967295u));
    if (e3 + e3 == nb - res) res = nb;
  }
  return ldexpf(res, (int)k);
}
float te_rr_pow_cr(float x, float p) {
#ifdef TE_ORACLE_F64
  if (1) return pow(x, p);
#endif
  if (!(x > 0.0f) || (fbits(x) & 0x7fffffffu) == 0x7f800000u) return powf(x, p);
  F2 L = rr_log_ff(x);
  float yh = L.x * p;
  return rr_exp_ff(quick_two_sum(yh, fmaf(L.y, p, fmaf(L.x, p, -yh))));
}

void teor_pressure_tendency(uint32_t *M, const uint32_t *ARG) {
  /* pressure_tendency.wgsl main: pi' forcing from the step tendencies of th and qv */
  Dims g = dims_at(M, B(0));
  const float *th = FPTR(1), *qv = FPTR(2), *rho = FPTR(3), *ppi = FPTR(4), *thten = FPTR(5), *qpten = FPTR(6);
  const float *th0 = FPTR(7), *pi0 = FPTR(8);
  float dt = FVAL(9);
  int hasDiabatic = IVAL(10);
  float *ppten = FPTR(11);
  int hasStepTend = IVAL(12);
  const float *qvt = FPTR(13);
  int moist = IVAL(14);
  const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, p00 = 1e5f;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float rp00 = DCR(1.0f, p00);
    float rddcv = DCR(rd, cp - rd);
    float tem = 0.0001f * 0.0001f;
    float qsmall = 1e-14f;
    float tht = hasStepTend != 0 ? thten[c] : 0.0f;
    if (moist == 0) {
      float p = 0.0f;
      if (fabsf(dt * tht) > tem) {
        float thnew = fmaf(dt, tht, th[c]);
        float pinew = te_rr_pow_cr(((rho[c] * (th0[k] + thnew)) * rd) * rp00, rddcv) - pi0[k];
        p = DCR(pinew - ppi[c], dt);
      }
      ppten[c] = p;
      continue;
    }
    float qvten = qvt[c];
    float p = 0.0f;
    if (fabsf(dt * tht) > tem || fabsf(dt * qvten) > qsmall) {
      float thnew = fmaf(dt, tht, th[c]);
      float qvnew = fmaf(dt, qvten, qv[c]);
      float pinew = te_rr_pow_cr(((rho[c] * (th0[k] + thnew)) * fmaf(rv, qvnew, rd)) * rp00, rddcv) - pi0[k];
      p = DCR(pinew - ppi[c], dt);
    }
    if (hasDiabatic != 0) p = p + qpten[c];
    ppten[c] = p;
  }
}

void teor_divergence3d(uint32_t *M, const uint32_t *ARG) {
  /* divergence3d.wgsl main (|d| < 1e-30 -> 0) */
  Dims g = dims_at(M, B(0));
  const float *u = FPTR(1), *v = FPTR(2), *w = FPTR(3), *mh = FPTR(4);
  float *div = FPTR(5);
  const float *hm = FPTR(30);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float d = fmaf((w[c + sk] - w[c]) * g.rdz, mh[k],
                   fmaf((u[c + 1] - u[c]) * g.rdx, hm_uh(&g, hm, i), ((v[c + sj] - v[c]) * g.rdy) * hm_vh(&g, hm, j)));
    div[c] = fabsf(d) < 1e-30f ? 0.0f : d;
  }
}

void teor_update_rho_prs(uint32_t *M, const uint32_t *ARG) {
  /* update_rho_prs.wgsl main: prs = p00 pi^(cp/rd), rho = prs / (th pi rmix) */
  Dims g = dims_at(M, B(0));
  int moist = IVAL(1);
  const float *thp = FPTR(2), *ppp = FPTR(3), *th0 = FPTR(4), *pi0 = FPTR(5), *qv = FPTR(6);
  float *prs = FPTR(7), *rho = FPTR(8);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float cpdrd = DCR(1005.7f, 287.04f);
    float pi = pi0[k] + ppp[c];
    float th = th0[k] + thp[c];
    float p = 1e5f * te_rr_pow_cr(pi, cpdrd);
    prs[c] = p;
    float rmix = moist != 0 ? fmaf(fmax_(0.0f, qv[c]), 461.5f, 287.04f) : 287.04f;
    rho[c] = DCR(p, (th * pi) * rmix);
  }
}

void teor_diabatic_unapply(uint32_t *M, const uint32_t *ARG) {
  /* diabatic_unapply.wgsl main: remove last step's diabatic tendencies, keep values */
  Dims g = dims_at(M, B(0));
  float dt = FVAL(1);
  float *pp3d = FPTR(2), *th = FPTR(3), *qv = FPTR(4), *qc = FPTR(5);
  float *qpten = FPTR(6), *qtten = FPTR(7), *qvten = FPTR(8), *qcten = FPTR(9);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    pp3d[c] = fmaf(-dt, qpten[c], pp3d[c]);
    qpten[c] = pp3d[c];
    th[c] = fmaf(-dt, qtten[c], th[c]);
    qtten[c] = th[c];
    qv[c] = fmaf(-dt, qvten[c], qv[c]);
    qvten[c] = qv[c];
    qc[c] = fmaf(-dt, qcten[c], qc[c]);
    qcten[c] = qc[c];
  }
}

void teor_diabatic_rates(uint32_t *M, const uint32_t *ARG) {
  /* diabatic_rates.wgsl main */
  Dims g = dims_at(M, B(0));
  float dt = FVAL(1);
  const float *pp3d = FPTR(2), *th = FPTR(3), *qv = FPTR(4), *qc = FPTR(5);
  float *qpten = FPTR(6), *qtten = FPTR(7), *qvten = FPTR(8), *qcten = FPTR(9);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float rdt = DCR(1.0f, dt);
    qpten[c] = (pp3d[c] - qpten[c]) * rdt;
    qtten[c] = (th[c] - qtten[c]) * rdt;
    qvten[c] = (qv[c] - qvten[c]) * rdt;
    qcten[c] = (qc[c] - qcten[c]) * rdt;
  }
}

void teor_ppx_finish(uint32_t *M, const uint32_t *ARG) {
  /* ppx_finish.wgsl main: ppx = pp3d + ppx */
  Dims g = dims_at(M, B(0));
  const float *pp3d = FPTR(1);
  float *ppx = FPTR(2);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    ppx[c] = pp3d[c] + ppx[c];
  }
}

/* ------------------------------------------------------ open lateral boundaries */

void teor_bc_open_x(uint32_t *M, const uint32_t *ARG) {
  /* bc_open_x.wgsl main: zero-gradient x halos, i = -1-h <- 0 and i = last+1+h <- last
   * (h < 3, last = nx + stagX - 1) over rows j in [-3, ny+3] and levels k <= nz */
  Dims g = dims_at(M, B(0));
  float *f = FPTR(1);
  const int stagX = IVAL(2);
  FOR_GRID {
    int h = (int)tx, jj = (int)ty - 3, k = (int)tz;
    if (h >= 3 || jj > g.ny + 3 || k > g.nz) continue;
    int last = g.nx + stagX - 1;
    f[GIDX(g, -1 - h, jj, k)] = f[GIDX(g, 0, jj, k)];
    f[GIDX(g, last + 1 + h, jj, k)] = f[GIDX(g, last, jj, k)];
  }
}

void teor_bc_open_y(uint32_t *M, const uint32_t *ARG) {
  /* bc_open_y.wgsl main: the same along y, columns i in [-3, nx+3] */
  Dims g = dims_at(M, B(0));
  float *f = FPTR(1);
  const int stagY = IVAL(2);
  FOR_GRID {
    int h = (int)tx, ii = (int)ty - 3, k = (int)tz;
    if (h >= 3 || ii > g.nx + 3 || k > g.nz) continue;
    int last = g.ny + stagY - 1;
    f[GIDX(g, ii, -1 - h, k)] = f[GIDX(g, ii, 0, k)];
    f[GIDX(g, ii, last + 1 + h, k)] = f[GIDX(g, ii, last, k)];
  }
}

/* copysign(1e-10, x) as the reference builds it from bits */
static inline float tiny_signed(float x) { return bitsf((fbits(1e-10f) & 0x7fffffffu) | (fbits(x) & 0x80000000u)); }

/* one boundary's radiation speed at a point (radbc_ew.wgsl / radbc_ns.wgsl loop body):
 * dx (a - b) / (dt (tiny_signed(foo) + foo)) with foo = a2 - a1 */
static inline float radbc_speed(float dx, float a, float b, float foo, float dt) {
  return DCR(dx * (a - b), dt * (tiny_signed(foo) + foo));
}

void teor_radbc_ew(uint32_t *M, const uint32_t *ARG) {
  /* radbc_ew.wgsl main: per row j < ny, the level mean of the west (i = 1, clipped to
   * [-umax, 0]) and east (i = nx-1, clipped to [0, umax]) radiation speeds of u */
  Dims g = dims_at(M, B(0));
  const float *ua = FPTR(1), *u3d = FPTR(2), *hm = FPTR(30);
  const float dt = FVAL(3);
  float *radbcw = FPTR(4), *radbce = FPTR(5);
  FOR_GRID {
    int j = (int)tx;
    if (j >= g.ny) continue;
    const float umax = 350.0f;
    float dxw = DCR(DCR(1.0f, g.rdx), hm_uf(&g, hm, 1));
    float dxe = DCR(DCR(1.0f, g.rdx), hm_uf(&g, hm, g.nx - 1));
    float avgw = 0.0f, avge = 0.0f;
    for (int k = 0; k < g.nz; k++) {
      int c1 = GIDX(g, 1, j, k), c2 = GIDX(g, 2, j, k);
      float foo = ua[c2] - ua[c1];
      float cbcw = radbc_speed(dxw, ua[c1], u3d[c1], foo, dt);
      cbcw = fmax_(fmin_(cbcw, 0.0f), -umax);
      avgw = avgw + cbcw;
      int ce = GIDX(g, g.nx - 1, j, k), ce2 = GIDX(g, g.nx - 2, j, k);
      foo = ua[ce] - ua[ce2];
      float cbce = radbc_speed(dxe, ua[ce], u3d[ce], foo, dt);
      cbce = fmin_(fmax_(cbce, 0.0f), umax);
      avge = avge + cbce;
    }
    radbcw[j] = DCR(avgw, (float)g.nz);
    radbce[j] = DCR(avge, (float)g.nz);
  }
}

void teor_radbc_ns(uint32_t *M, const uint32_t *ARG) {
  /* radbc_ns.wgsl main: per column i < nx, the same for v at j = 1 (south) and
   * j = ny-1 (north) */
  Dims g = dims_at(M, B(0));
  const float *va = FPTR(1), *v3d = FPTR(2), *hm = FPTR(30);
  const float dt = FVAL(3);
  float *radbcs = FPTR(4), *radbcn = FPTR(5);
  FOR_GRID {
    int i = (int)tx;
    if (i >= g.nx) continue;
    const float umax = 350.0f;
    float dys = DCR(DCR(1.0f, g.rdy), hm_vf(&g, hm, 1));
    float dyn = DCR(DCR(1.0f, g.rdy), hm_vf(&g, hm, g.ny - 1));
    float avgs = 0.0f, avgn = 0.0f;
    for (int k = 0; k < g.nz; k++) {
      int c1 = GIDX(g, i, 1, k), c2 = GIDX(g, i, 2, k);
      float foo = va[c2] - va[c1];
      float cbcs = radbc_speed(dys, va[c1], v3d[c1], foo, dt);
      cbcs = fmax_(fmin_(cbcs, 0.0f), -umax);
      avgs = avgs + cbcs;
      int cn = GIDX(g, i, g.ny - 1, k), cn2 = GIDX(g, i, g.ny - 2, k);
      foo = va[cn] - va[cn2];
      float cbcn = radbc_speed(dyn, va[cn], v3d[cn], foo, dt);
      cbcn = fmin_(fmax_(cbcn, 0.0f), umax);
      avgn = avgn + cbcn;
    }
    radbcs[i] = DCR(avgs, (float)g.nz);
    radbcn[i] = DCR(avgn, (float)g.nz);
  }
}

void teor_openbc_uv_tendency(uint32_t *M, const uint32_t *ARG) {
  /* openbc_uv_tendency.wgsl main: on open x boundaries the u faces i = 0 and i = nx
   * (and on open y boundaries the v faces j = 0, j = ny) advance by the radiation term
   * u = fma(dts, fma((-c * du) * rdx, uh, uten), u), du the one-sided difference */
  Dims g = dims_at(M, B(0));
  Acoustic a = acoustic_at(M, B(1));
  const float *radbcw = FPTR(2), *radbce = FPTR(3), *radbcs = FPTR(4), *radbcn = FPTR(5);
  const float *uten = FPTR(6), *vten = FPTR(7), *hm = FPTR(30);
  float *u3d = FPTR(8), *v3d = FPTR(9);
  const int openx = (int32_t)M[B(10)], openy = (int32_t)M[B(10) + 1];
  FOR_GRID {
    int n = (int)tx, k = (int)ty;
    if (k >= g.nz) continue;
    if (openx != 0 && n < g.ny) {
      int j = n;
      int cw = GIDX(g, 0, j, k);
      u3d[cw] = fmaf(a.dts, fmaf(((-radbcw[j]) * (u3d[cw + 1] - u3d[cw])) * g.rdx, hm_uh(&g, hm, 0), uten[cw]), u3d[cw]);
      int ce = GIDX(g, g.nx, j, k);
      u3d[ce] = fmaf(a.dts, fmaf(((-radbce[j]) * (u3d[ce] - u3d[ce - 1])) * g.rdx, hm_uh(&g, hm, g.nx - 1), uten[ce]),
                     u3d[ce]);
    }
    if (openy != 0 && n < g.nx) {
      int i = n, sj = g.sJ;
      int cs = GIDX(g, i, 0, k);
      v3d[cs] = fmaf(a.dts, fmaf(((-radbcs[i]) * (v3d[cs + sj] - v3d[cs])) * g.rdy, hm_vh(&g, hm, 0), vten[cs]), v3d[cs]);
      int cn = GIDX(g, i, g.ny, k);
      v3d[cn] = fmaf(a.dts, fmaf(((-radbcn[i]) * (v3d[cn] - v3d[cn - sj])) * g.rdy, hm_vh(&g, hm, g.ny - 1), vten[cn]),
                     v3d[cn]);
    }
  }
}

/* ------------------------------------------------------- turbulence bookkeeping */

void teor_turb_zero(uint32_t *M, const uint32_t *ARG) {
  /* turb_zero.wgsl main: f[i + strideJ (j + strideK k)] = 0 for i < strideJ, j < strideK,
   * k <= nz + 1 (one level above the field's nz + 1: the reference's own range) */
  Dims g = dims_at(M, B(0));
  float *f = FPTR(1);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.sJ || j >= g.sK || k > g.nz + 1) continue;
    f[i + g.sJ * (j + g.sK * k)] = 0.0f;
  }
}

void teor_turb_add_tendency(uint32_t *M, const uint32_t *ARG) {
  /* turb_add_tendency.wgsl main: dst = fma(scale, src, dst) over the whole field */
  Dims g = dims_at(M, B(0));
  const float *src = FPTR(1);
  float *dst = FPTR(2);
  const float scale = FVAL(3);
  FOR_GRID {
    int i = (int)tx - 3, j = (int)ty - 3, k = (int)tz;
    if (i > g.nx + 3 || j > g.ny + 3 || k > g.nz) continue;
    int c = GIDX(g, i, j, k);
    dst[c] = fmaf(scale, src[c], dst[c]);
  }
}

/* turbulence fluxes and TKE bookkeeping (the reference's subgrid turbulence kernels) */

void teor_turb_scalar_flux_h(uint32_t *M, const uint32_t *ARG) {
  /* turb_scalar_flux_h.wgsl main: horizontal subgrid scalar fluxes at the x and y faces
   * fx = ((((-1/8 (rho + rho_w)) le) ((kh + kh_w) + (kh_up + kh_w,up))) (s - s_w)) rdx uf */
  Dims g = dims_at(M, B(0));
  const float *s = FPTR(1), *rho = FPTR(2), *khh = FPTR(3), *hm = FPTR(30);
  const float leNum = FVAL(4);
  float *fx = FPTR(5), *fy = FPTR(6);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > g.nx || j > g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
    fx[c] = ((((((-0.125f) * (rho[c] + rho[c - 1])) * leNum) * ((khh[c] + khh[c - 1]) + (khh[c + sk] + khh[c - 1 + sk]))) *
              (s[c] - s[c - 1])) * g.rdx) * hm_uf(&g, hm, i);
    fy[c] = ((((((-0.125f) * (rho[c] + rho[c - sj])) * leNum) * ((khh[c] + khh[c - sj]) + (khh[c + sk] + khh[c - sj + sk]))) *
              (s[c] - s[c - sj])) * g.rdy) * hm_vf(&g, hm, j);
  }
}

void teor_turb_openbc_flux(uint32_t *M, const uint32_t *ARG) {
  /* turb_openbc_flux.wgsl main: on open boundaries the edge fluxes copy their inner
   * neighbours (x: 0 <- 1, nx <- nx-1; y: 0 <- 1, ny <- ny-1), levels k <= nz */
  Dims g = dims_at(M, B(0));
  float *fx = FPTR(1), *fy = FPTR(2);
  const int openx = (int32_t)M[B(3)], openy = (int32_t)M[B(3) + 1];
  FOR_GRID {
    int n = (int)tx, k = (int)ty;
    if (k > g.nz) continue;
    if (openx != 0 && n <= g.ny) {
      fx[GIDX(g, 0, n, k)] = fx[GIDX(g, 1, n, k)];
      fx[GIDX(g, g.nx, n, k)] = fx[GIDX(g, g.nx - 1, n, k)];
    }
    if (openy != 0 && n <= g.nx) {
      fy[GIDX(g, n, 0, k)] = fy[GIDX(g, n, 1, k)];
      fy[GIDX(g, n, g.ny, k)] = fy[GIDX(g, n, g.ny - 1, k)];
    }
  }
}

void teor_turb_openbc_stress_x(uint32_t *M, const uint32_t *ARG) {
  /* turb_openbc_stress_x.wgsl main: s11 halo columns -1 <- 0, nx <- nx-1 (rows j >= -1);
   * s12 columns 0 <- 1, nx <- nx-1 (rows j >= 0) */
  Dims g = dims_at(M, B(0));
  float *s11 = FPTR(1), *s12 = FPTR(2);
  FOR_GRID {
    int j = (int)tx - 1, k = (int)ty;
    if (j > g.ny || k >= g.nz) continue;
    s11[GIDX(g, -1, j, k)] = s11[GIDX(g, 0, j, k)];
    s11[GIDX(g, g.nx, j, k)] = s11[GIDX(g, g.nx - 1, j, k)];
    if (j >= 0) {
      s12[GIDX(g, 0, j, k)] = s12[GIDX(g, 1, j, k)];
      s12[GIDX(g, g.nx, j, k)] = s12[GIDX(g, g.nx - 1, j, k)];
    }
  }
}

void teor_turb_openbc_stress_y(uint32_t *M, const uint32_t *ARG) {
  /* turb_openbc_stress_y.wgsl main: the same along y for s22 and s12 */
  Dims g = dims_at(M, B(0));
  float *s22 = FPTR(1), *s12 = FPTR(2);
  FOR_GRID {
    int i = (int)tx - 1, k = (int)ty;
    if (i > g.nx || k >= g.nz) continue;
    s22[GIDX(g, i, -1, k)] = s22[GIDX(g, i, 0, k)];
    s22[GIDX(g, i, g.ny, k)] = s22[GIDX(g, i, g.ny - 1, k)];
    if (i >= 0) {
      s12[GIDX(g, i, 0, k)] = s12[GIDX(g, i, 1, k)];
      s12[GIDX(g, i, g.ny, k)] = s12[GIDX(g, i, g.ny - 1, k)];
    }
  }
}

void teor_tke_advance(uint32_t *M, const uint32_t *ARG) {
  /* tke_advance.wgsl main: tke = fma(dttmp, tketen, tkea), flushed to 0 below 1e-10,
   * interior w levels 1 .. nz-1 */
  Dims g = dims_at(M, B(0));
  const float *tkea = FPTR(1), *tketen = FPTR(2);
  const float dttmp = FVAL(3);
  float *tke = FPTR(4);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k);
    float v = fmaf(dttmp, tketen[c], tkea[c]);
    tke[c] = v < 1e-10f ? 0.0f : v;
  }
}

void teor_tke_sources(uint32_t *M, const uint32_t *ARG) {
  /* tke_sources.wgsl main: tketen = fma(-khv, nm, -dissten) + epst */
  Dims g = dims_at(M, B(0));
  const float *khv = FPTR(1), *nm = FPTR(2), *dissten = FPTR(3), *epst = FPTR(4);
  float *tketen = FPTR(5);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k);
    tketen[c] = fmaf(-khv[c], nm[c], -dissten[c]) + epst[c];
  }
}

void teor_tke_flux_h(uint32_t *M, const uint32_t *ARG) {
  /* tke_flux_h.wgsl main: horizontal TKE fluxes at the x and y faces of w levels 1..nz-1
   * fx = (((((-1/4 (rf + rf_w)) 2) (km + km_w)) (t - t_w)) rdx) uf */
  Dims g = dims_at(M, B(0));
  const float *t = FPTR(1), *rf = FPTR(2), *kmh = FPTR(3), *hm = FPTR(30);
  float *fx = FPTR(4), *fy = FPTR(5);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i > g.nx || j > g.ny || k > g.nz - 1) continue;
    int sj = g.sJ, c = GIDX(g, i, j, k);
    fx[c] = ((((((-0.25f) * (rf[c] + rf[c - 1])) * 2.0f) * (kmh[c] + kmh[c - 1])) * (t[c] - t[c - 1])) * g.rdx) *
            hm_uf(&g, hm, i);
    fy[c] = ((((((-0.25f) * (rf[c] + rf[c - sj])) * 2.0f) * (kmh[c] + kmh[c - sj])) * (t[c] - t[c - sj])) * g.rdy) *
            hm_vf(&g, hm, j);
  }
}

void teor_mp_pdefq(uint32_t *M, const uint32_t *ARG) {
  /* mp_pdefq.wgsl main: per column, t1 = sum rho q; q below rmax set to 0; t2 = sum rho q
   * after the clip; every q of the column scaled by (t1 + 1e-20) / (t2 + 1e-20), 1 when
   * that ratio is negative (a column-mass-preserving positive-definite fix) */
  Dims g = dims_at(M, B(0));
  const float *rho = FPTR(1);
  float *q = FPTR(2);
  const float rmax = FVAL(3);
  const int sk = g.sJ * g.sK;
  const long GX = ARG[0], GY = ARG[1];
#pragma omp parallel for collapse(2) schedule(static)
  for (long ty = 0; ty < GY; ty++)
    for (long tx = 0; tx < GX; tx++) {
      int i = (int)tx, j = (int)ty;
      if (i >= g.nx || j >= g.ny) continue;
      const int base = GIDX(g, i, j, 0);
      float t1 = 0.0f, t2 = 0.0f;
      for (int k = 0; k < g.nz; k++) {
        int c = base + k * sk;
        t1 = fmaf(rho[c], q[c], t1);
        if (q[c] < rmax) q[c] = 0.0f;
        t2 = fmaf(rho[c], q[c], t2);
      }
      float t3 = DCR(t1 + 1e-20f, t2 + 1e-20f);
      if (t3 < 0.0f) t3 = 1.0f;
      for (int k = 0; k < g.nz; k++) q[base + k * sk] = q[base + k * sk] * t3;
    }
}

/* Vertical subgrid flux of a scalar at w level kf of a column (turb_scalar_vert_implicit.wgsl
 * lam_1 and lam_2): interior levels -khv ds/dz mf rf; the bottom and top levels follow the
 * wall setting (w = 0: surface flux or the bcturbs == 2 inner gradient; w = 2: a prescribed
 * flux; otherwise a drag towards the wall values y (bottom) and z (top)) */
static float tsvi_vflux(const Dims *g, int base, int sk, int kf, const float *khv, const float *s, const float *mf,
                        const float *rf, const float *wall, int useFlux, const float *sflux, int bcturbs) {
  const int c = base + kf * sk;
  if (kf == 0 || kf == g->nz) {
    int inner = kf == 0 ? 1 : g->nz - 1;
    if (wall[3] == 0.0f) {
      if (kf == 0 && useFlux != 0) return sflux[base] * rf[c];
      if (bcturbs != 2) return 0.0f;
      int cc = base + inner * sk;
      return ((((-khv[cc]) * (s[cc] - s[cc - sk])) * g->rdz) * mf[inner]) * rf[cc];
    }
    if (wall[3] == 2.0f) return (wall[0] * (kf == 0 ? wall[1] : wall[2])) * rf[c];
    if (kf == 0) return (((((-wall[0]) * 2.0f) * (s[c] - wall[1])) * g->rdz) * mf[0]) * rf[c];
    return (((((-wall[0]) * 2.0f) * (wall[2] - s[base + (g->nz - 1) * sk])) * g->rdz) * mf[g->nz]) * rf[c];
  }
  return ((((-khv[c]) * (s[c] - s[c - sk])) * g->rdz) * mf[kf]) * rf[c];
}

/* sten += ((fx/fy divergence) + turbz) rr at point c (turb_scalar_vert_implicit.wgsl lam_5) */
static void tsvi_tend(const Dims *g, int c, int i, int j, float turbz, const float *fx, const float *fy,
                      const float *hm, const float *rr, float *sten) {
  float h = ((-(fx[c + 1] - fx[c])) * g->rdx) * hm_uh(g, hm, i) + ((-(fy[c + g->sJ] - fy[c])) * g->rdy) * hm_vh(g, hm, j);
  sten[c] = fmaf(h + turbz, rr[c], sten[c]);
}

void teor_turb_scalar_vert_implicit(uint32_t *M, const uint32_t *ARG) {
  /* turb_scalar_vert_implicit.wgsl main: subgrid tendency of a scalar, horizontal flux
   * divergence plus either the explicit vertical flux divergence (explicitZ) or the
   * implicit one: per column a tridiagonal Thomas solve of s_new - dt d/dz(K ds_new/dz)
   * = s (cA, cB: forward sweep; cB ends as s_new), tendency rho (s_new - s) / dt.
   * lam_3 / lam_4 are the coefficients khv mf rf (face above / below) mh rr. */
  Dims g = dims_at(M, B(0));
  const float *s = FPTR(1), *rho = FPTR(2), *rr = FPTR(3), *rf = FPTR(4), *khv = FPTR(5), *mh = FPTR(6), *mf = FPTR(7);
  const float *fx = FPTR(8), *fy = FPTR(9), *sflux = FPTR(14), *hm = FPTR(30);
  float *cA = FPTR(11), *cB = FPTR(12), *sten = FPTR(13);
  const float dt = FVAL(10);
  const int useFlux = IVAL(15), explicitZ = IVAL(16), bcturbs = IVAL(18);
  float wall[4];
  for (int q = 0; q < 4; q++) wall[q] = bitsf(M[B(17) + q]);
  const int sk = g.sJ * g.sK;
  const long GX = ARG[0], GY = ARG[1];
#pragma omp parallel for collapse(2) schedule(static)
  for (long ty = 0; ty < GY; ty++)
    for (long tx = 0; tx < GX; tx++) {
      int i = (int)tx, j = (int)ty;
      if (i >= g.nx || j >= g.ny) continue;
      const int base = GIDX(g, i, j, 0);
      if (explicitZ != 0) {
        float below = tsvi_vflux(&g, base, sk, 0, khv, s, mf, rf, wall, useFlux, sflux, bcturbs);
        for (int k = 0; k < g.nz; k++) {
          float above = tsvi_vflux(&g, base, sk, k + 1, khv, s, mf, rf, wall, useFlux, sflux, bcturbs);
          tsvi_tend(&g, base + k * sk, i, j, ((-(above - below)) * g.rdz) * mh[k], fx, fy, hm, rr, sten);
          below = above;
        }
        continue;
      }
#define LAM3(k) ((((khv[base + (k) * sk + sk] * mf[(k) + 1]) * rf[base + (k) * sk + sk]) * mh[k]) * rr[base + (k) * sk])
#define LAM4(k) ((((khv[base + (k) * sk] * mf[k]) * rf[base + (k) * sk]) * mh[k]) * rr[base + (k) * sk])
      const float tema = ((-dt) * g.rdz) * g.rdz, rdt = DCR(1.0f, dt), temc = dt * g.rdz;
      {
        float cfc = tema * LAM3(0), t = DCR(1.0f, 1.0f - cfc);
        cA[base] = (-cfc) * t;
        float cfd = s[base];
        if (useFlux != 0 || bcturbs == 2) {
          int c1 = base + sk;
          float dumz = useFlux != 0 ? sflux[base] * rf[base]
                                    : ((((-khv[c1]) * (s[c1] - s[base])) * g.rdz) * mf[1]) * rf[c1];
          cfd = fmaf((temc * dumz) * mh[0], rr[base], s[base]);
        }
        cB[base] = cfd * t;
      }
      for (int k = 1; k < g.nz - 1; k++) {
        int c = base + k * sk;
        float cfa = tema * LAM4(k), cfc = tema * LAM3(k), cfb = (1.0f - cfa) - cfc;
        float t = DCR(1.0f, fmaf(cfa, cA[c - sk], cfb));
        cA[c] = (-cfc) * t;
        cB[c] = fmaf(-cfa, cB[c - sk], s[c]) * t;
      }
      {
        int kt = g.nz - 1, ct = base + kt * sk;
        float cfa = tema * LAM4(kt), t = DCR(1.0f, fmaf(cfa, cA[ct - sk], 1.0f - cfa));
        float cfd = s[ct];
        if (bcturbs == 2) {
          float dumz = ((((-khv[ct]) * (s[ct] - s[ct - sk])) * g.rdz) * mf[kt]) * rf[ct];
          cfd = fmaf(-((temc * dumz) * mh[kt]), rr[ct], s[ct]);
        }
        float snew = fmaf(-cfa, cB[ct - sk], cfd) * t;
        cB[ct] = snew;
        tsvi_tend(&g, ct, i, j, (rho[ct] * (snew - s[ct])) * rdt, fx, fy, hm, rr, sten);
      }
#undef LAM3
#undef LAM4
      for (int k = g.nz - 2; k >= 0; k--) {
        int c = base + k * sk;
        float snew = fmaf(cA[c], cB[c + sk], cB[c]);
        cB[c] = snew;
        tsvi_tend(&g, c, i, j, (rho[c] * (snew - s[c])) * rdt, fx, fy, hm, rr, sten);
      }
    }
}

void teor_rayleigh_damping(uint32_t *M, const uint32_t *ARG) {
  /* rayleigh_damping.wgsl main: tendencies -rdalpha tau (phi - phi_ref) for u, v, th
   * (reference profiles u0/v0/th, or the level averages avg[k], avg[nz + k], avg[2 nz + k]
   * when toAverage), and -rdalpha tauf w for w, tauf raised to the lateral sponge hdx/hdy */
  Dims g = dims_at(M, B(0));
  const float *u = FPTR(1), *v = FPTR(2), *w = FPTR(3), *th = FPTR(4), *u0 = FPTR(5), *v0 = FPTR(6);
  const float *tauh = FPTR(7), *tauf = FPTR(8), *hdx = FPTR(14), *hdy = FPTR(15), *avg = FPTR(18), *th0 = FPTR(19);
  float *uten = FPTR(10), *vten = FPTR(11), *wten = FPTR(12), *thten = FPTR(13);
  const float rdalpha = FVAL(9);
  const int lateral = IVAL(16), toAverage = IVAL(17);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i > g.nx || j > g.ny || k > g.nz) continue;
    int c = GIDX(g, i, j, k);
    if (k < g.nz) {
      float t = tauh[k];
      float ur = toAverage != 0 ? avg[k] : u0[k];
      float vr = toAverage != 0 ? avg[g.nz + k] : v0[k];
      if (j < g.ny) uten[c] = ((-rdalpha) * t) * (u[c] - ur);
      if (i < g.nx) vten[c] = ((-rdalpha) * t) * (v[c] - vr);
      if (i < g.nx && j < g.ny) {
        float d = toAverage != 0 ? (th0[k] - avg[2 * g.nz + k]) + th[c] : th[c];
        thten[c] = ((-rdalpha) * t) * d;
      }
    }
    if (i < g.nx && j < g.ny) {
      float tf = tauf[k];
      if (lateral != 0 && k < g.nz) tf = fmax_(fmax_(tf, hdx[i]), hdy[j]);
      wten[c] = ((-rdalpha) * tf) * w[c];
    }
  }
}

void teor_turb_rho_faces(uint32_t *M, const uint32_t *ARG) {
  /* turb_rho_faces.wgsl main: rr = 1 / rho at levels k < nz; rf on w levels: interior
   * c1 rho(k-1) + c2 rho(k), bottom and top extrapolated with the weights cgs / cgt
   * (third weight only when nz >= 3); columns -2..nx+1, rows -2..ny+1 */
  Dims g = dims_at(M, B(0));
  const float *rho = FPTR(1), *c1 = FPTR(2), *c2 = FPTR(3);
  float *rr = FPTR(4), *rf = FPTR(5);
  float cgs[3], cgt[3];
  for (int q = 0; q < 3; q++) {
    cgs[q] = bitsf(M[B(6) + q]);
    cgt[q] = bitsf(M[B(7) + q]);
  }
  const int sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx - 2, j = (int)ty - 2, k = (int)tz;
    if (i > g.nx + 1 || j > g.ny + 1 || k > g.nz) continue;
    int c = GIDX(g, i, j, k);
    if (k < g.nz) rr[c] = DCR(1.0f, rho[c]);
    if (k == 0) {
      float r = fmaf(cgs[0], rho[c], cgs[1] * rho[c + sk]);
      if (g.nz >= 3) r = fmaf(cgs[2], rho[c + 2 * sk], r);
      rf[c] = r;
    } else if (k == g.nz) {
      float r = fmaf(cgt[0], rho[c - sk], cgt[1] * rho[c - 2 * sk]);
      if (g.nz >= 3) r = fmaf(cgt[2], rho[c - 3 * sk], r);
      rf[c] = r;
    } else {
      rf[c] = fmaf(c1[k], rho[c - sk], c2[k] * rho[c]);
    }
  }
}

void teor_turb_def_centers(uint32_t *M, const uint32_t *ARG) {
  /* turb_def_centers.wgsl main: rho-weighted strain rates at cell centres (s11, s22, s33)
   * and at the (i-1/2, j-1/2) edges (s12, with the four-point corner density) */
  Dims g = dims_at(M, B(0));
  const float *u = FPTR(1), *v = FPTR(2), *w = FPTR(3), *rho = FPTR(4), *mh = FPTR(5), *hm = FPTR(30);
  float *s11 = FPTR(6), *s22 = FPTR(7), *s33 = FPTR(8), *s12 = FPTR(9);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx - 1, j = (int)ty - 1, k = (int)tz;
    if (i > g.nx + 1 || j > g.ny + 1 || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    s11[c] = ((rho[c] * (u[c + 1] - u[c])) * g.rdx) * hm_uh(&g, hm, i);
    s22[c] = ((rho[c] * (v[c + sj] - v[c])) * g.rdy) * hm_vh(&g, hm, j);
    s33[c] = ((rho[c] * (w[c + sk] - w[c])) * g.rdz) * mh[k];
    float rcorner = 0.25f * ((rho[c - 1 - sj] + rho[c]) + (rho[c - 1] + rho[c - sj]));
    s12[c] = (0.5f * fmaf((u[c] - u[c - sj]) * g.rdy, hm_vf(&g, hm, j), ((v[c] - v[c - 1]) * g.rdx) * hm_uf(&g, hm, i))) * rcorner;
  }
}

void teor_turb_def_faces(uint32_t *M, const uint32_t *ARG) {
  /* turb_def_faces.wgsl main: strain rates s13, s23 on the w levels 1..nz-1 at the x and y
   * faces, weighted by the face-averaged rf */
  Dims g = dims_at(M, B(0));
  const float *u = FPTR(1), *v = FPTR(2), *w = FPTR(3), *rf = FPTR(4), *mf = FPTR(5), *hm = FPTR(30);
  float *s13 = FPTR(6), *s23 = FPTR(7);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i > g.nx + 1 || j > g.ny + 1 || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k);
    float mfk = 0.5f * (mf[k] + mf[k]);
    s13[c] = ((0.5f * fmaf((w[c] - w[c - 1]) * g.rdx, hm_uf(&g, hm, i), ((u[c] - u[c - sk]) * g.rdz) * mfk)) * 0.5f) * (rf[c - 1] + rf[c]);
    s23[c] = ((0.5f * fmaf((w[c] - w[c - sj]) * g.rdy, hm_vf(&g, hm, j), ((v[c] - v[c - sk]) * g.rdz) * mfk)) * 0.5f) * (rf[c - sj] + rf[c]);
  }
}

void teor_turb_def_assemble(uint32_t *M, const uint32_t *ARG) {
  /* turb_def_assemble.wgsl main: deformation on w levels 1..nz-1, defv = 4 (t13 + t23) / rf^2,
   * defh = (2 (t11 + t22 + t33) + 4 t12) / rf^2, with t11..t33 the squared centre rates
   * interpolated by c1/c2 and t12, t13, t23 averaged over the surrounding edges and faces */
  Dims g = dims_at(M, B(0));
  const float *s11 = FPTR(1), *s22 = FPTR(2), *s33 = FPTR(3), *s12 = FPTR(4), *s13 = FPTR(5), *s23 = FPTR(6);
  const float *c1 = FPTR(7), *c2 = FPTR(8), *rf = FPTR(9);
  float *defv = FPTR(10), *defh = FPTR(11);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k);
    float a = c1[k], b = c2[k];
#define SQ2(s) fmaf(a * s[c - sk], s[c - sk], (b * s[c]) * s[c])
    float t11 = SQ2(s11), t22 = SQ2(s22), t33 = SQ2(s33);
#undef SQ2
#define PAIR(p, q) fmaf(s12[p], s12[p], s12[q] * s12[q])
    float lo = PAIR(c - sk, c + 1 + sj - sk) + PAIR(c + sj - sk, c + 1 - sk);
    float hi = PAIR(c, c + 1 + sj) + PAIR(c + sj, c + 1);
#undef PAIR
    float t12 = 0.25f * fmaf(a, lo, b * hi);
    float t13 = 0.5f * fmaf(s13[c], s13[c], s13[c + 1] * s13[c + 1]);
    float t23 = 0.5f * fmaf(s23[c], s23[c], s23[c + sj] * s23[c + sj]);
    float rrf = DCR(1.0f, rf[c] * rf[c]);
    defv[c] = (4.0f * (t13 + t23)) * rrf;
    defh[c] = fmaf(2.0f, (t11 + t22) + t33, 4.0f * t12) * rrf;
  }
}

void teor_turb_gettau(uint32_t *M, const uint32_t *ARG) {
  /* turb_gettau.wgsl main: stresses from the strain rates, t = s (kmh + kmh above) at
   * centres, t12 with the 8-point edge average of kmh, t13 / t23 with the face sums of kmv
   * (levels 1..nz-1, columns and rows >= 0); columns and rows -1..n */
  Dims g = dims_at(M, B(0));
  const float *kmh = FPTR(1), *kmv = FPTR(2);
  float *t11 = FPTR(3), *t22 = FPTR(4), *t33 = FPTR(5), *t12 = FPTR(6), *t13 = FPTR(7), *t23 = FPTR(8);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx - 1, j = (int)ty - 1, k = (int)tz;
    if (i > g.nx || j > g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float tem = kmh[c] + kmh[c + sk];
    t11[c] = t11[c] * tem;
    t22[c] = t22[c] * tem;
    t33[c] = t33[c] * tem;
    int d = c + sk;
    t12[c] = t12[c] * (0.25f * (((kmh[c - 1 - sj] + kmh[c]) + (kmh[c - 1] + kmh[c - sj])) +
                                ((kmh[d - 1 - sj] + kmh[d]) + (kmh[d - 1] + kmh[d - sj]))));
    if (k >= 1 && k <= g.nz - 1 && i >= 0 && j >= 0) {
      t13[c] = t13[c] * (kmv[c - 1] + kmv[c]);
      t23[c] = t23[c] * (kmv[c - sj] + kmv[c]);
    }
  }
}

/* The reference's WGSL pow, exp and log builtins (turb_km_kh.wgsl, turb_nm.wgsl,
 * turb_dissipative_heating.wgsl), whose precision WGSL leaves to the implementation, are
 * evaluated in binary64 with plain operations and rounded once to binary32:
 *   ln x = e ln 2 + 2 atanh(s) for x = 2^e m, m in [sqrt(1/2), sqrt(2)), s = (m - 1) / (m + 1),
 *          atanh by its odd power series to s^23;
 *   2^t  = 2^n e^r, n = rint(t), r = (t - n) ln 2, e^r by its Taylor series to r^14;
 *   x^y = 2^(y log2 x), e^x = 2^(x / ln 2).
 * The binary64 error is far below half a binary32 ulp, so each is the correctly rounded
 * value except within that error of a rounding boundary.  The CUDA kernels evaluate the
 * same operations in the same order. */
#ifndef TE_ORACLE_F64
static double ln_mantissa(float x, int *e) {   /* x > 0 normal: returns ln(m), sets e */
  uint32_t b = fbits(x);
  double m = (double)bitsf((b & 0x7fffffu) | 0x3f800000u);
  *e = (int)(b >> 23) - 127;
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    *e = *e + 1;
  }
  double s = (m - 1.0) / (m + 1.0), s2 = s * s, p = 1.0 / 23;
  for (int k = 21; k >= 1; k -= 2) p = p * s2 + 1.0 / k;
  return 2.0 * s * p;
}
static float exp2_rounded(double t) {
  if (t > 128.0) return INFINITY;
  if (t < -126.0) return 0.0f;
  double n = nearbyint(t), r = (t - n) * 0.6931471805599453, q = 1.0;
  for (int k = 14; k >= 1; k--) q = 1.0 + (r * (1.0 / k)) * q;
  return (float)ldexp(q, (int)n);
}
float te_pow_f64(float x, float y) {
  if (!(x > 0.0f) || x == INFINITY) return x == 0.0f ? (y > 0.0f ? 0.0f : INFINITY) : (x == INFINITY ? (y > 0.0f ? INFINITY : 0.0f) : NAN);
  int e;
  double lm = ln_mantissa(x, &e);
  return exp2_rounded((double)y * ((double)e + lm * 1.4426950408889634));
}
float te_exp_f64(float x) {
  if (x != x) return x;
  return exp2_rounded((double)x * 1.4426950408889634);
}
float te_log_f64(float x) {
  if (x != x || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return INFINITY;
  int e;
  double lm = ln_mantissa(x, &e);
  return (float)((double)e * 0.6931471805599453 + lm);
}
/* log2 x = e + ln(m) / ln 2 from the same ln(m); atan2 in binary64: octant reduction to
 * a = min/max in [0, 1], atan a = pi/6 + atan((a sqrt3 - 1) / (a + sqrt3)) above
 * tan(pi/12), the odd power series to u^29, then the octant and the sign of y (zeros and
 * infinities as C's atan2f).  WGSL leaves both precisions to the implementation; these are
 * the CUDA kernels' (te_math.cuh log2_f64, atan2_f64), operation for operation. */
float te_log2_f64(float x) {
  if (x != x || x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return INFINITY;
  int e;
  double lm = ln_mantissa(x, &e);
  return (float)((double)e + lm * 1.4426950408889634);
}
float te_atan2_f64(float y, float x) {
  if (x != x || y != y) return x + y;
  double ax = fabs((double)x), ay = fabs((double)y), r;
  int neg = (int)(fbits(y) >> 31), xneg = (int)(fbits(x) >> 31);
  if (ax == INFINITY && ay == INFINITY) {
    r = xneg ? 2.356194490192345 : 0.7853981633974483;
  } else if (ax == 0.0 && ay == 0.0) {
    r = xneg ? 3.141592653589793 : 0.0;
  } else {
    int swap = ay > ax;
    double a = swap ? ax / ay : ay / ax, u = a, base = 0.0;
    if (a > 0.2679491924311227) {
      u = (a * 1.7320508075688772 - 1.0) / (a + 1.7320508075688772);
      base = 0.5235987755982988;
    }
    double w = -(u * u), p = 1.0 / 29;
    for (int k = 27; k >= 1; k -= 2) p = p * w + 1.0 / k;
    r = base + u * p;
    if (swap) r = 1.5707963267948966 - r;
    if (xneg) r = 3.141592653589793 - r;
  }
  float f = (float)r;
  return neg ? -f : f;
}
#endif /* !TE_ORACLE_F64 */

void teor_turb_km_kh(uint32_t *M, const uint32_t *ARG) {
  /* turb_km_kh.wgsl main: TKE closure on w levels 1..nz-1.  Grid scale (dx dy dz)^(1/3),
   * mixing length (stability-limited by c_l sqrt(tke / N^2)), dissipation added to dissten,
   * km = cmz sqrt(tke) len kmScale (or kmFixed), kh = km / Pr with 1/Pr = min(1 + 2 len /
   * grid scale, 3) */
  Dims g = dims_at(M, B(0));
  const float *tkea = FPTR(1), *nm = FPTR(2), *mf = FPTR(3), *hm = FPTR(30);
  float *kmh = FPTR(4), *kmv = FPTR(5), *khh = FPTR(6), *khv = FPTR(7), *lenscl = FPTR(8), *dissten = FPTR(9);
  const float kmScale = FVAL(10), kmFixed = FVAL(11), turbfac = FVAL(12);
  const float c_m = 0.1f, c_l = 0.8165f, ri_c = 0.25f, tke_min = 1e-10f, nm_min = 1e-06f, small_len_frac = 0.001f;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k);
    float cmz = fmax_(0.001f, turbfac * c_m);
    float ce1z = ((cmz * c_l) * c_l) * (DCR(1.0f, ri_c) - 1.0f);
    float ce2z = fmax_(0.0f, fmaf(cmz * 3.1415927f, 3.1415927f, -ce1z));
    float dzk = DCR(DCR(1.0f, g.rdz), mf[k]);
    float grdscl = te_pow_f64((DCR(DCR(1.0f, g.rdx), hm_uh(&g, hm, i)) * DCR(DCR(1.0f, g.rdy), hm_vh(&g, hm, j))) * dzk, 0.33333334f);
    float rgrdscl = DCR(1.0f, grdscl);
    float tk, len;
    if (tkea[c] <= tke_min) {
      tk = tke_min;
      len = small_len_frac * grdscl;
    } else {
      tk = tkea[c];
      len = grdscl;
      if (nm[c] > nm_min) {
        len = c_l * sqrtf(DCR(tk, nm[c]));
        len = fmin_(len, grdscl);
        len = fmax_(len, small_len_frac * grdscl);
      }
    }
    lenscl[c] = len;
    dissten[c] = dissten[c] + DCR((fmaf(ce2z * len, rgrdscl, ce1z) * tk) * sqrtf(tk), len);
    float km = kmFixed > 0.0f ? kmFixed : ((cmz * sqrtf(tk)) * len) * kmScale;
    kmh[c] = km;
    kmv[c] = km;
    float prinv = 3.0f;
    if (nm[c] > nm_min) prinv = fmin_(fmaf(2.0f * len, rgrdscl, 1.0f), 3.0f);
    khh[c] = km * prinv;
    khv[c] = khh[c];
  }
}

void teor_tke_epst(uint32_t *M, const uint32_t *ARG) {
  /* tke_epst.wgsl main: shear production of TKE on w levels 1..nz-1, the stresses t_ij
   * times the strain rates, interpolated (c1/c2) or averaged to the w point, divided by rf */
  Dims g = dims_at(M, B(0));
  const float *u = FPTR(1), *v = FPTR(2), *w = FPTR(3), *t11 = FPTR(4), *t12 = FPTR(5), *t13 = FPTR(6);
  const float *t22 = FPTR(7), *t23 = FPTR(8), *t33 = FPTR(9), *rf = FPTR(10), *mh = FPTR(11), *mf = FPTR(12);
  const float *c1 = FPTR(13), *c2 = FPTR(14), *hm = FPTR(30);
  float *epst = FPTR(15);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k), cd = c - sk;
    const float uh = hm_uh(&g, hm, i), vh = hm_vh(&g, hm, j), mfk = mf[k];
#define L1(cc) fmaf(((u[(cc) + 1] - u[cc]) * g.rdx) * uh, t11[cc], (((v[(cc) + sj] - v[cc]) * g.rdy) * vh) * t22[cc])
#define L2(cc, ii, jj) (t12[cc] * fmaf((u[cc] - u[(cc) - sj]) * g.rdy, hm_vf(&g, hm, jj), ((v[cc] - v[(cc) - 1]) * g.rdx) * hm_uf(&g, hm, ii)))
#define L3(cc, ii) (fmaf((w[cc] - w[(cc) - 1]) * g.rdx, hm_uf(&g, hm, ii), ((u[cc] - u[(cc) - sk]) * g.rdz) * mfk) * t13[cc])
#define L4(cc, jj) (fmaf((w[cc] - w[(cc) - sj]) * g.rdy, hm_vf(&g, hm, jj), ((v[cc] - v[(cc) - sk]) * g.rdz) * mfk) * t23[cc])
#define L5(cc, kk) ((((w[(cc) + sk] - w[cc]) * g.rdz) * mh[kk]) * t33[cc])
    float e = fmaf(c1[k], L1(cd), c2[k] * L1(c));
    float hi = (L2(c, i, j) + L2(c + 1 + sj, i + 1, j + 1)) + (L2(c + sj, i, j + 1) + L2(c + 1, i + 1, j));
    float lo = (L2(cd, i, j) + L2(cd + 1 + sj, i + 1, j + 1)) + (L2(cd + sj, i, j + 1) + L2(cd + 1, i + 1, j));
    e = fmaf(0.25f, fmaf(c2[k], hi, c1[k] * lo), e);
    e = fmaf(0.5f, (L3(c, i) + L3(c + 1, i + 1)) + (L4(c, j) + L4(c + sj, j + 1)), e);
    e = e + fmaf(c1[k], L5(cd, k - 1), c2[k] * L5(c, k));
#undef L1
#undef L2
#undef L3
#undef L4
#undef L5
    epst[c] = DCR(e, rf[c]);
  }
}

/* turb_nm.wgsl f_rr_log_cr: the reference's correctly rounded log (two-float log, summed);
 * non-positive, infinite and NaN arguments take the log builtin's special values */
static float rr_log_cr(float x) {
  if (!(x > 0.0f) || x == INFINITY) return x == 0.0f ? -INFINITY : (x == INFINITY ? INFINITY : NAN);
  F2 a = rr_log_ff(x);
  return a.x + a.y;
}

/* saturation mixing ratios over liquid (f_mp_rslf) and ice (f_mp_rsif), turb_nm.wgsl */
static float mp_rs(float p, float t, float a, float b) {
  float es = 611.2f * te_exp_f64(DCR(a * (t - 273.15f), t - b));
  es = fmin_(es, p * 0.5f);
  return DCR(DCR(287.04f, 461.5f) * es, p - es);
}

void teor_turb_nm(uint32_t *M, const uint32_t *ARG) {
  /* turb_nm.wgsl main: squared Brunt-Vaisala frequency on w levels 1..nz-1.  Dry: g dln(th)/dz.
   * Moist: g dln(thv)/dz, or in saturated air (liquid above 0 C, ice below -40 C, a linear
   * blend between) the moist-adiabatic form of lam_1; sat marks saturated points */
  Dims g = dims_at(M, B(0));
  const float *thPert = FPTR(1), *ppPert = FPTR(2), *th0 = FPTR(3), *pi0 = FPTR(4), *prs = FPTR(5);
  const float *qv = FPTR(6), *qc = FPTR(7), *qr = FPTR(8), *qi = FPTR(9), *qs = FPTR(10), *qg = FPTR(11);
  const float *c1 = FPTR(12), *c2 = FPTR(13), *mf = FPTR(14);
  float *nm = FPTR(15), *sat = FPTR(17);
  const int moist = IVAL(16), wantSat = IVAL(18);
  const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, cpv = 1870.0f, cpl = 4190.0f, cpi = 2106.0f;
  const float lv1 = 3134708.0f, lv2 = 2320.0f, ls1 = 2898463.5f, ls2 = 236.0f, nmsat = 1e-10f, gAcc = 9.81f;
  const int sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz + 1;
    if (i >= g.nx || j >= g.ny || k > g.nz - 1) continue;
    int c = GIDX(g, i, j, k), d = c - sk;
    if (wantSat != 0) sat[c] = 0.0f;
    float eps = DCR(rd, rv), reps = DCR(rv, rd);
    float thA = th0[k - 1] + thPert[d], thB = th0[k] + thPert[c];
    if (moist == 0) {
      nm[c] = ((rr_log_cr(DCR(thB, thA)) * gAcc) * g.rdz) * mf[k];
      continue;
    }
    float piA = pi0[k - 1] + ppPert[d], piB = pi0[k] + ppPert[c];
    float tA = thA * piA, tB = thB * piB;
    float qtA = ((((qv[d] + qc[d]) + qr[d]) + qi[d]) + qs[d]) + qg[d];
    float qtB = ((((qv[c] + qc[c]) + qr[c]) + qi[c]) + qs[c]) + qg[c];
    float qciA = (qv[d] + qc[d]) + qi[d], qciB = (qv[c] + qc[c]) + qi[c];
    float thvA = DCR(thA * fmaf(reps, qv[d], 1.0f), 1.0f + qtA);
    float thvB = DCR(thB * fmaf(reps, qv[c], 1.0f), 1.0f + qtB);
    float rmf = g.rdz * mf[k];
    float dlnT = rr_log_cr(DCR(tB, tA)) * rmf;
    float dlnQt = rr_log_cr(DCR(1.0f + qtB, 1.0f + qtA)) * rmf;
    float out = (gAcc * rr_log_cr(DCR(thvB, thvA))) * rmf;
    float a = c1[k], b = c2[k];
    float pavg = fmaf(a, prs[d], b * prs[c]), tavg = fmaf(a, tA, b * tB);
    float qtavg = fmaf(a, qtA, b * qtB), qciavg = fmaf(a, qciA, b * qciB);
    /* lam_1: moist-adiabatic N^2 for saturation ratio qvs, latent heat lh, dqvs/dT drdt */
#define LAM1(qvs, lh, drdt, cpml)                                                                    \
  (gAcc * fmaf(dlnT + DCR(DCR((gAcc * (1.0f + qtavg)) * (1.0f + DCR((lh) * (qvs), rd * tavg)),          \
                              fmaf((lh), (drdt), (cpml))), tavg),                                      \
               1.0f + DCR(tavg * (drdt), eps + (qvs)), -dlnQt))
    const float al = 17.67f, bl = 29.65f, ai = 21.874557f, bi = 7.66f;
    if (tavg >= 273.15f) {
      float qvs = mp_rs(pavg, tavg, al, bl);
      float ql = fmax_(qciavg - qvs, 0.0f);
      if (ql > nmsat) {
        if (wantSat != 0) sat[c] = 1.0f;
        float qvl = fmax_(qciavg - ql, 0.0f);
        float cpml = fmaf(cpl, ql, fmaf(cpv, qvl, cp));
        float lh = fmaf(-lv2, tavg, lv1);
        float drdt = DCR((al * (273.15f - bl)) * qvs, (tavg - bl) * (tavg - bl));
        out = LAM1(qvs, lh, drdt, cpml);
      }
    } else if (tavg <= 233.15f) {
      float qvs = mp_rs(pavg, tavg, ai, bi);
      float qice = fmax_(qciavg - qvs, 0.0f);
      if (qice > nmsat) {
        if (wantSat != 0) sat[c] = 1.0f;
        float qvl = fmax_(qciavg - qice, 0.0f);
        float cpml = fmaf(cpi, qice, fmaf(cpv, qvl, cp));
        float lh = fmaf(-ls2, tavg, ls1);
        float drdt = DCR((ai * (273.15f - bi)) * qvs, (tavg - bi) * (tavg - bi));
        out = LAM1(qvs, lh, drdt, cpml);
      }
    } else {
      float ff = DCR(tavg - 233.15f, 273.15f - 233.15f);
      float qvsl = mp_rs(pavg, tavg, al, bl), qvsi = mp_rs(pavg, tavg, ai, bi);
      float qvs = fmaf(ff, qvsl, (1.0f - ff) * qvsi);
      float qice = fmax_(0.0f, (1.0f - ff) * (qciavg - qvs));
      float ql = fmax_(0.0f, ff * (qciavg - qvs));
      if (ql + qice > nmsat) {
        if (wantSat != 0) sat[c] = 1.0f;
        float qvl = fmax_(0.0f, (qciavg - ql) - qice);
        float cpml = fmaf(cpi, qice, fmaf(cpl, ql, fmaf(cpv, qvl, cp)));
        float lhl = fmaf(-lv2, tavg, lv1);
        float drdtl = DCR((al * (273.15f - bl)) * qvsl, (tavg - bl) * (tavg - bl));
        float nml = LAM1(qvsl, lhl, drdtl, cpml);
        float lhi = fmaf(-ls2, tavg, ls1);
        float drdti = DCR((ai * (273.15f - bi)) * qvsi, (tavg - bi) * (tavg - bi));
        float nmi = LAM1(qvsi, lhi, drdti, cpml);
        out = fmaf(ff, nml, (1.0f - ff) * nmi);
      }
    }
#undef LAM1
    nm[c] = out;
  }
}

void teor_turb_sfcstress(uint32_t *M, const uint32_t *ARG) {
  /* turb_sfcstress.wgsl main: boundary stresses t13, t23 per column (i <= nx, j <= ny).
   * Top (level nz): no-slip drag, or a copy of level nz-1.  Bottom (level 0) by mode:
   * 0 copy of level 1; 4 no-slip drag; 2 constant drag coefficient 0.001229 with the
   * surface wind speed s1 (plane 2 of sfc); 3 the drag against the domain-mean wind
   * (planes 14..16 at the origin, lam_1); otherwise u*^2 w1 / max(s1, 0.01) (lam_2) */
  Dims g = dims_at(M, B(0));
  const float *sfc = FPTR(1), *rf = FPTR(2), *u = FPTR(6), *v = FPTR(7), *kmv = FPTR(9), *mf = FPTR(11);
  float *t13 = FPTR(3), *t23 = FPTR(4);
  const int mode = IVAL(5), topNoSlip = IVAL(10);
  const float mx = bitsf(M[B(8)]), my = bitsf(M[B(8) + 1]);
  const int plane = g.sJ * g.sK, sj = g.sJ;
  const long GX = ARG[0], GY = ARG[1];
#pragma omp parallel for collapse(2) schedule(static)
  for (long ty = 0; ty < GY; ty++)
    for (long tx = 0; tx < GX; tx++) {
      int i = (int)tx, j = (int)ty;
      if (i > g.nx || j > g.ny) continue;
      int ct = GIDX(g, i, j, g.nz);
      if (topNoSlip != 0) {
        int cu = ct - plane;
        float mft = 0.5f * (mf[g.nz] + mf[g.nz]);
        t13[ct] = ((((((-2.0f) * (u[cu] + mx)) * g.rdz) * mft) * 0.5f) * (rf[ct - 1] + rf[ct])) * 0.5f * (kmv[cu - 1] + kmv[cu]);
        t23[ct] = ((((((-2.0f) * (v[cu] + my)) * g.rdz) * mft) * 0.5f) * (rf[ct - sj] + rf[ct])) * 0.5f * (kmv[cu - sj] + kmv[cu]);
      } else {
        t13[ct] = t13[ct - plane];
        t23[ct] = t23[ct - plane];
      }
      int c = GIDX(g, i, j, 0);
      if (mode == 0) {
        t13[c] = t13[c + plane];
        t23[c] = t23[c + plane];
      } else if (mode == 4) {
        float mfb = 0.5f * (mf[0] + mf[0]);
        t13[c] = ((((((2.0f * (u[c] + mx)) * g.rdz) * mfb) * 0.5f) * (rf[c - 1] + rf[c])) * 0.5f) * (kmv[c - 1 + plane] + kmv[c + plane]);
        t23[c] = ((((((2.0f * (v[c] + my)) * g.rdz) * mfb) * 0.5f) * (rf[c - sj] + rf[c])) * 0.5f) * (kmv[c - sj + plane] + kmv[c + plane]);
      } else if (mode == 2) {
        float s1w = sfc[2 * plane + GIDX(g, i - 1, j, 0)], s1c = sfc[2 * plane + c], s1s = sfc[2 * plane + GIDX(g, i, j - 1, 0)];
        t13[c] = ((((0.001229f * 0.5f) * (s1w + s1c)) * (u[c] + mx)) * 0.5f) * (rf[c - 1] + rf[c]);
        t23[c] = ((((0.001229f * 0.5f) * (s1s + s1c)) * (v[c] + my)) * 0.5f) * (rf[c - sj] + rf[c]);
      } else if (mode == 3) {
        int o0 = GIDX(g, 0, 0, 0);
        float au = sfc[14 * plane + o0], av = sfc[15 * plane + o0], as = sfc[16 * plane + o0];
        float den = fmax_(0.0001f, as * sqrtf(fmaf(au, au, av * av)));
#define L1(ii, jj, comp)                                                                                  \
  DCR((sfc[3 * plane + GIDX(g, ii, jj, 0)] * sfc[3 * plane + GIDX(g, ii, jj, 0)]) *                        \
          fmaf(sfc[2 * plane + GIDX(g, ii, jj, 0)], (comp) == 0 ? au : av,                                 \
               as * (sfc[(comp) * plane + GIDX(g, ii, jj, 0)] - ((comp) == 0 ? au : av))),                 \
      den)
        t13[c] = (0.25f * (L1(i - 1, j, 0) + L1(i, j, 0))) * (rf[c - 1] + rf[c]);
        t23[c] = (0.25f * (L1(i, j - 1, 1) + L1(i, j, 1))) * (rf[c - sj] + rf[c]);
#undef L1
      } else {
#define L2(ii, jj, comp)                                                                                  \
  DCR((sfc[3 * plane + GIDX(g, ii, jj, 0)] * sfc[3 * plane + GIDX(g, ii, jj, 0)]) *                        \
          sfc[(comp) * plane + GIDX(g, ii, jj, 0)],                                                        \
      fmax_(sfc[2 * plane + GIDX(g, ii, jj, 0)], 0.01f))
        t13[c] = (0.25f * (L2(i - 1, j, 0) + L2(i, j, 0))) * (rf[c - 1] + rf[c]);
        t23[c] = (0.25f * (L2(i, j - 1, 1) + L2(i, j, 1))) * (rf[c - sj] + rf[c]);
#undef L2
      }
    }
}

void teor_turb_dissipative_heating(uint32_t *M, const uint32_t *ARG) {
  /* turb_dissipative_heating.wgsl main: thten += eps / (cp_m/cv_m... pi): the dissipation
   * averaged to the cell centre (at the surface with bbc3, u*^3 ln((dz1 + z0) / z0) / (k dz1)),
   * divided by cp pi (dry) or (cp/cv) cv_m pi (moist) */
  Dims g = dims_at(M, B(0));
  const float *dissten = FPTR(1), *pi0 = FPTR(2), *ppi = FPTR(3), *qv = FPTR(4), *qc = FPTR(5), *qr = FPTR(6);
  const float *qi = FPTR(7), *qs = FPTR(8), *qg = FPTR(9), *sfc = FPTR(12);
  float *thten = FPTR(10);
  const uint32_t pw = B(11);
  const int moist = (int32_t)M[pw], bbc3 = (int32_t)M[pw + 1], zntField = (int32_t)M[pw + 4];
  const float znt = bitsf(M[pw + 2]), dz1 = bitsf(M[pw + 3]);
  const float cpd = 1005.7f, rd = 287.04f, cpv = 1870.0f, rv = 461.5f, karman = 0.4f;
  const int sk = g.sJ * g.sK;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float cv = cpd - rd, cvv = cpv - rv, cpl = 4190.0f, cpi = 2106.0f, cpdcv = DCR(cpd, cv);
    float epsd;
    if (k == 0 && bbc3 != 0) {
      float ust = sfc[3 * sk + GIDX(g, i, j, 0)];
      float z0 = zntField != 0 ? sfc[4 * sk + GIDX(g, i, j, 0)] : znt;
      epsd = DCR(((ust * ust) * ust) * te_log_f64(DCR(dz1 + z0, z0)), karman * dz1);
    } else {
      epsd = 0.5f * (dissten[c] + dissten[c + sk]);
    }
    float pi = pi0[k] + ppi[c], dheat;
    if (moist != 0) {
      float cvm = fmaf(cpi, (qi[c] + qs[c]) + qg[c], fmaf(cpl, qc[c] + qr[c], fmaf(cvv, qv[c], cv)));
      dheat = DCR(epsd, (cpdcv * cvm) * pi);
    } else {
      dheat = DCR(epsd, cpd * pi);
    }
    thten[c] = thten[c] + dheat;
  }
}

/* turb_u_tendency.wgsl / turb_v_tendency.wgsl main (axis 0: u, axis 1: v; the v kernel is
 * the u kernel with x and y exchanged): subgrid momentum tendency.  Horizontal stress
 * divergence (zero on open edges) plus either the explicit vertical one or, per column, an
 * implicit vertical diffusion solved by a Thomas sweep (cA, cB; cB ends as the new
 * velocity), its tendency rho (new - old) / dt, and the dw/dx (dw/dy) cross term dwd */
static void turb_uv_tendency(uint32_t *M, const uint32_t *ARG, int axis) {
  Dims g = dims_at(M, B(0));
  const float *X = FPTR(1), *w = FPTR(2), *rho = FPTR(3), *rf = FPTR(4), *kmv = FPTR(5);
  const float *A1 = FPTR(6), *A2 = FPTR(7), *A3 = FPTR(8), *mh = FPTR(9), *mf = FPTR(10), *hm = FPTR(30);
  float *cA = FPTR(12), *cB = FPTR(13), *dwd = FPTR(14), *ten = FPTR(15);
  const float dt = FVAL(11);
  const int openx = (int32_t)M[B(16)], openy = (int32_t)M[B(16) + 1], explicitZ = IVAL(17);
  const int sj = g.sJ, sk = g.sJ * g.sK, s = axis == 0 ? 1 : sj;
  const long GX = ARG[0], GY = ARG[1];
#pragma omp parallel for collapse(2) schedule(static)
  for (long ty = 0; ty < GY; ty++)
    for (long tx = 0; tx < GX; tx++) {
      int i = (int)tx, j = (int)ty;
      if (axis == 0 ? (i > g.nx || j >= g.ny) : (i >= g.nx || j > g.ny)) continue;
      int zeroX = openx != 0 && (i == 0 || i == (axis == 0 ? g.nx : g.nx - 1));
      int zeroY = openy != 0 && (j == 0 || j == (axis == 0 ? g.ny - 1 : g.ny));
      const int base = GIDX(g, i, j, 0);
#define HORIZ(c)                                                                                         \
  ((zeroX ? 0.0f : axis == 0 ? ((A1[c] - A1[(c) - 1]) * g.rdx) * hm_uf(&g, hm, i)                        \
                             : ((A1[(c) + 1] - A1[c]) * g.rdx) * hm_uh(&g, hm, i)) +                     \
   (zeroY ? 0.0f : axis == 0 ? ((A2[(c) + sj] - A2[c]) * g.rdy) * hm_vh(&g, hm, j)                       \
                             : ((A2[c] - A2[(c) - sj]) * g.rdy) * hm_vf(&g, hm, j)))
#define RINV(k) DCR(1.0f, 0.5f * (rho[base + (k) * sk - s] + rho[base + (k) * sk]))
      if (explicitZ != 0) {
        for (int k = 0; k < g.nz; k++) {
          int c = base + k * sk;
          float turbz = (((A3[c + sk] - A3[c]) * g.rdz) * 0.5f) * (mh[k] + mh[k]);
          ten[c] = ten[c] + DCR(HORIZ(c) + turbz, 0.5f * (rho[c - s] + rho[c]));
        }
        continue;
      }
      const float tema = (((-0.0625f) * dt) * g.rdz) * g.rdz, temc = (0.5f * dt) * g.rdz, rdt = DCR(0.5f, dt);
      for (int k = 0; k <= g.nz; k++) {
        int c = base + k * sk;
        float dwx = axis == 0 ? ((w[c] - w[c - 1]) * g.rdx) * hm_uf(&g, hm, i) : ((w[c] - w[c - sj]) * g.rdy) * hm_vf(&g, hm, j);
        dwd[c] = ((dwx * 0.25f) * (kmv[c - s] + kmv[c])) * (rf[c - s] + rf[c]);
      }
      /* lam_1: coefficient of the face at level lev for the cell at level k */
#define LAM1(k, lev) \
  ((((kmv[base + (lev) * sk - s] + kmv[base + (lev) * sk]) * (mf[lev] + mf[lev])) * (rf[base + (lev) * sk - s] + rf[base + (lev) * sk])) * ((mh[k] + mh[k]) * RINV(k)))
      {
        float cfc = tema * LAM1(0, 1), cfb = 1.0f - cfc;
        float cfd = fmaf(-((temc * A3[base]) * (mh[0] + mh[0])), RINV(0), X[base]);
        float t = DCR(1.0f, cfb);
        cA[base] = (-cfc) * t;
        cB[base] = cfd * t;
      }
      for (int k = 1; k < g.nz - 1; k++) {
        int c = base + k * sk;
        float cfa = tema * LAM1(k, k), cfc = tema * LAM1(k, k + 1), cfb = (1.0f - cfa) - cfc;
        float t = DCR(1.0f, fmaf(cfa, cA[c - sk], cfb));
        cA[c] = (-cfc) * t;
        cB[c] = fmaf(-cfa, cB[c - sk], X[c]) * t;
      }
      {
        int kt = g.nz - 1, ct = base + kt * sk;
        float cfa = tema * LAM1(kt, kt), cfb = 1.0f - cfa;
        float cfd = fmaf((temc * A3[base + g.nz * sk]) * (mh[kt] + mh[kt]), RINV(kt), X[ct]);
        float t = DCR(1.0f, fmaf(cfa, cA[ct - sk], cfb));
        cB[ct] = fmaf(-cfa, cB[ct - sk], cfd) * t;
      }
#undef LAM1
      for (int k = g.nz - 2; k >= 0; k--) {
        int c = base + k * sk;
        cB[c] = fmaf(cA[c], cB[c + sk], cB[c]);
      }
      for (int k = 0; k < g.nz; k++) {
        int c = base + k * sk;
        float turbz = ((rho[c - s] + rho[c]) * (cB[c] - X[c])) * rdt;
        turbz = fmaf(((dwd[c + sk] - dwd[c]) * g.rdz) * 0.5f, mh[k] + mh[k], turbz);
        ten[c] = fmaf(HORIZ(c) + turbz, RINV(k), ten[c]);
      }
#undef HORIZ
#undef RINV
    }
}
void teor_turb_u_tendency(uint32_t *M, const uint32_t *ARG) { turb_uv_tendency(M, ARG, 0); }
void teor_turb_v_tendency(uint32_t *M, const uint32_t *ARG) { turb_uv_tendency(M, ARG, 1); }

/* turb_w_tendency.wgsl and tke_transport.wgsl main (tke = 1): tendency of a w-level
 * quantity q (w, or TKE) on levels 1..nz-1.  Horizontal divergence (w: of the stresses
 * t13, t23; TKE: of -fx, -fy), zero on open edges, plus the explicit vertical divergence
 * or, per column, the implicit vertical diffusion (Thomas sweep over levels 1..nz-1 with
 * the boundary fluxes folded into the right-hand side), tendency rf (new - old) / dt */
static void turb_wlevel_tendency(uint32_t *M, const uint32_t *ARG, int tke) {
  Dims g = dims_at(M, B(0));
  const float *q, *rho, *rf, *kmh, *kmv = 0, *h1, *h2, *t33 = 0, *mh, *mf, *hm = FPTR(30);
  float *cA, *cB, *ten;
  float dt;
  int ob;
  if (tke) {
    q = FPTR(1); rho = FPTR(2); rf = FPTR(3); kmh = FPTR(4); kmv = FPTR(5); mh = FPTR(6); mf = FPTR(7);
    dt = FVAL(8); cA = FPTR(9); cB = FPTR(10); h1 = FPTR(11); h2 = FPTR(12); ten = FPTR(13); ob = 14;
  } else {
    q = FPTR(1); rho = FPTR(2); rf = FPTR(3); kmh = FPTR(4); h1 = FPTR(5); h2 = FPTR(6); t33 = FPTR(7);
    mh = FPTR(8); mf = FPTR(9); dt = FVAL(10); cA = FPTR(11); cB = FPTR(12); ten = FPTR(13); ob = 14;
  }
  const int openx = (int32_t)M[B(ob)], openy = (int32_t)M[B(ob) + 1], explicitZ = IVAL(ob + 1);
  const int sj = g.sJ, sk = g.sJ * g.sK;
  const long GX = ARG[0], GY = ARG[1];
#pragma omp parallel for collapse(2) schedule(static)
  for (long ty = 0; ty < GY; ty++)
    for (long tx = 0; tx < GX; tx++) {
      int i = (int)tx, j = (int)ty;
      if (i >= g.nx || j >= g.ny) continue;
      int zeroX = openx != 0 && (i == 0 || i == g.nx - 1), zeroY = openy != 0 && (j == 0 || j == g.ny - 1);
      const int base = GIDX(g, i, j, 0);
#define HORIZ(c)                                                                                          \
  ((zeroX ? 0.0f : tke ? ((-(h1[(c) + 1] - h1[c])) * g.rdx) * hm_uh(&g, hm, i) : ((h1[(c) + 1] - h1[c]) * g.rdx) * hm_uh(&g, hm, i)) + \
   (zeroY ? 0.0f : tke ? ((-(h2[(c) + sj] - h2[c])) * g.rdy) * hm_vh(&g, hm, j) : ((h2[(c) + sj] - h2[c]) * g.rdy) * hm_vh(&g, hm, j)))
      /* TKE vertical flux at cell level k (lam_1 of tke_transport.wgsl) */
#define TFLUX(k) \
  (((((-(kmv[base + (k) * sk] + kmv[base + (k) * sk + sk])) * (q[base + (k) * sk + sk] - q[base + (k) * sk])) * g.rdz) * mh[k]) * rho[base + (k) * sk])
      if (explicitZ != 0) {
        float below = tke ? TFLUX(0) : 0.0f;
        for (int k = 1; k < g.nz; k++) {
          int c = base + k * sk;
          float turbz;
          if (tke) {
            float here = TFLUX(k);
            turbz = ((-(here - below)) * g.rdz) * mf[k];
            below = here;
          } else {
            turbz = ((t33[c] - t33[c - sk]) * g.rdz) * mf[k];
          }
          ten[c] = ten[c] + DCR(HORIZ(c) + turbz, rf[c]);
        }
        continue;
      }
      const float tema = (((-1.0f) * dt) * g.rdz) * g.rdz, temc = dt * g.rdz, rdt = DCR(1.0f, dt);
      /* coefficients of the faces above (UP) and below (DN) w level k */
#define MFR(k) DCR(mf[k], rf[base + (k) * sk])
#define UP(k) ((((kmh[base + (k) * sk] + kmh[base + (k) * sk + sk]) * mh[k]) * rho[base + (k) * sk]) * MFR(k))
#define DN(k) ((((kmh[base + (k) * sk - sk] + kmh[base + (k) * sk]) * mh[(k) - 1]) * rho[base + (k) * sk - sk]) * MFR(k))
      {
        int c = base + sk;
        float cfc = tema * UP(1), cfb = 1.0f - cfc, cfd;
        if (tke)
          cfd = fmaf(temc * ((((-(kmv[c - sk] + kmv[c])) * (q[c] - q[c - sk])) * g.rdz) * mh[0]) * rho[c - sk], MFR(1), q[c]);
        else
          cfd = fmaf(-(temc * t33[c - sk]), MFR(1), q[c]);
        float t = DCR(1.0f, cfb);
        cA[c] = (-cfc) * t;
        cB[c] = cfd * t;
      }
      for (int k = 2; k < g.nz - 1; k++) {
        int c = base + k * sk;
        float cfa = tema * DN(k), cfc = tema * UP(k), cfb = (1.0f - cfa) - cfc;
        float t = DCR(1.0f, fmaf(cfa, cA[c - sk], cfb));
        cA[c] = (-cfc) * t;
        cB[c] = fmaf(-cfa, cB[c - sk], q[c]) * t;
      }
      {
        int kt = g.nz - 1, ct = base + kt * sk;
        float cfa = tema * DN(kt), cfb = 1.0f - cfa, cfd;
        if (tke)
          cfd = fmaf(-(temc * (((((-(kmv[ct] + kmv[ct + sk])) * (q[ct + sk] - q[ct])) * g.rdz) * mh[kt]) * rho[ct])), MFR(kt), q[ct]);
        else
          cfd = fmaf(temc * t33[ct], MFR(kt), q[ct]);
        float t = DCR(1.0f, fmaf(cfa, cA[ct - sk], cfb));
        cB[ct] = fmaf(-cfa, cB[ct - sk], cfd) * t;
      }
#undef UP
#undef DN
#undef MFR
#undef TFLUX
      for (int k = g.nz - 2; k >= 1; k--) {
        int c = base + k * sk;
        cB[c] = fmaf(cA[c], cB[c + sk], cB[c]);
      }
      for (int k = 1; k < g.nz; k++) {
        int c = base + k * sk;
        float turbz = (rf[c] * (cB[c] - q[c])) * rdt;
        ten[c] = ten[c] + DCR(HORIZ(c) + turbz, rf[c]);
      }
#undef HORIZ
    }
}
void teor_turb_w_tendency(uint32_t *M, const uint32_t *ARG) { turb_wlevel_tendency(M, ARG, 0); }
void teor_tke_transport(uint32_t *M, const uint32_t *ARG) { turb_wlevel_tendency(M, ARG, 1); }

/* two-float accumulation of the mass sums (f_df_add / f_df_add_pair, mass_row_sums.wgsl):
 * acc.x + x by an error-free sum, the error accumulated in acc.y */
static inline void df_add(F2 *acc, float x) {
  float s = acc->x + x, bb = s - acc->x;
  float err = (acc->x - (s - bb)) + (x - bb);
  acc->x = s;
  acc->y = acc->y + err;
}
static inline void df_add_pair(F2 *acc, float vx, float vy) {
  df_add(acc, vx);
  acc->y = acc->y + vy;
}

void teor_mass_row_sums(uint32_t *M, const uint32_t *ARG) {
  /* mass_row_sums.wgsl main: per (j, k) row, the two-float sums over i of the cell mass
   * rho / (uh vh mh) (rows1) and of pi0 + pp3d (rows2), stored at (k strideK + j) pairs */
  Dims g = dims_at(M, B(0));
  const float *rho = FPTR(1), *pi0 = FPTR(2), *pp3d = FPTR(3), *mh = FPTR(4), *hm = FPTR(30);
  float *rows1 = FPTR(5), *rows2 = FPTR(6);
  const long GX = ARG[0], GY = ARG[1];
#pragma omp parallel for collapse(2) schedule(static)
  for (long ty = 0; ty < GY; ty++)
    for (long tx = 0; tx < GX; tx++) {
      int j = (int)tx, k = (int)ty;
      if (j >= g.ny || k >= g.nz) continue;
      F2 s1 = {0.0f, 0.0f}, s2 = {0.0f, 0.0f};
      float rvh = DCR(1.0f, hm_vh(&g, hm, j));
      for (int i = 0; i < g.nx; i++) {
        int c = GIDX(g, i, j, k);
        float rmh = DCR(1.0f, mh[k]);
        df_add(&s1, ((rho[c] * DCR(1.0f, hm_uh(&g, hm, i))) * rvh) * rmh);
        df_add(&s2, pi0[k] + pp3d[c]);
      }
      long o = 2L * ((long)k * g.sK + j);
      rows1[o] = s1.x;
      rows1[o + 1] = s1.y;
      rows2[o] = s2.x;
      rows2[o + 1] = s2.y;
    }
}

void teor_mass_level_sums(uint32_t *M, const uint32_t *ARG) {
  /* mass_level_sums.wgsl main: per level k, the two-float sums over j of the row pairs */
  Dims g = dims_at(M, B(0));
  const float *rows1 = FPTR(1), *rows2 = FPTR(2);
  float *levels1 = FPTR(3), *levels2 = FPTR(4);
  const long GX = ARG[0];
#pragma omp parallel for schedule(static)
  for (long tx = 0; tx < GX; tx++) {
    int k = (int)tx;
    if (k >= g.nz) continue;
    F2 s1 = {0.0f, 0.0f}, s2 = {0.0f, 0.0f};
    for (int j = 0; j < g.ny; j++) {
      long o = 2L * ((long)k * g.sK + j);
      df_add_pair(&s1, rows1[o], rows1[o + 1]);
      df_add_pair(&s2, rows2[o], rows2[o + 1]);
    }
    levels1[2 * k] = s1.x;
    levels1[2 * k + 1] = s1.y;
    levels2[2 * k] = s2.x;
    levels2[2 * k + 1] = s2.y;
  }
}

void teor_mass_reference_init(uint32_t *M, const uint32_t *ARG) {
  /* mass_reference_init.wgsl main: on its first run (ref[2] == 0) thread 0 stores the total
   * mass (two-float sum of the level sums) as the reference and sets ref[2] = 1 */
  Dims g = dims_at(M, B(0));
  const float *levels1 = FPTR(1);
  float *ref = FPTR(2);
  if (ARG[0] == 0 || ref[2] != 0.0f) return;
  F2 s = {0.0f, 0.0f};
  for (int k = 0; k < g.nz; k++) df_add_pair(&s, levels1[2 * k], levels1[2 * k + 1]);
  ref[0] = s.x;
  ref[1] = s.y;
  ref[2] = 1.0f;
}

/* (1 + r)^a - 1 (f_powm1, mass_correction_apply.wgsl): the WGSL pow for |r| > 0.05, else
 * its third-order expansion */
static float powm1(float r, float a) {
  if (fabsf(r) > 0.05f) return te_pow_f64(1.0f + r, a) - 1.0f;
  return r * fmaf(r, fmaf(a * (a - 1.0f), 0.5f, DCR(((r * a) * (a - 1.0f)) * (a - 2.0f), 6.0f)), a);
}

void teor_mass_correction_apply(uint32_t *M, const uint32_t *ARG) {
  /* mass_correction_apply.wgsl main: the relative mass change r against the reference,
   * turned into a uniform pi' correction tem = ((1 + r)^(rd/cv) - 1) sum(pi) / (nx ny nz),
   * added to pp3d; prs and rho recomputed from the corrected pi; thread (0,0,0) records
   * tem, the mass, the pi sum, r and the mass's low part in out[0..4] */
  Dims g = dims_at(M, B(0));
  const float *levels1 = FPTR(2), *levels2 = FPTR(3), *ref = FPTR(4), *thPert = FPTR(5);
  const float *th0 = FPTR(7), *pi0 = FPTR(8), *qv = FPTR(9);
  float *pp3d = FPTR(6), *prs = FPTR(10), *rho = FPTR(11), *out = FPTR(12);
  const int moist = IVAL(1);
  const float rd = 287.04f, cp = 1005.7f, rv = 461.5f, p00 = 1e+05f;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    F2 m2 = {0.0f, 0.0f}, pp2 = {0.0f, 0.0f};
    for (int kk = 0; kk < g.nz; kk++) {
      df_add_pair(&m2, levels1[2 * kk], levels1[2 * kk + 1]);
      df_add_pair(&pp2, levels2[2 * kk], levels2[2 * kk + 1]);
    }
    float rddcv = DCR(rd, cp - rd);
    float r = DCR((ref[0] - m2.x) + (ref[1] - m2.y), m2.x);
    float p2 = pp2.x + pp2.y;
    float tem = DCR(powm1(r, rddcv) * p2, (float)((g.nx * g.ny) * g.nz));
    if (i == 0 && j == 0 && k == 0) {
      out[0] = tem;
      out[1] = m2.x;
      out[2] = p2;
      out[3] = r;
      out[4] = m2.y;
    }
    int c = GIDX(g, i, j, k);
    float pp = pp3d[c] + tem;
    pp3d[c] = pp;
    float cpdrd = DCR(cp, rd);
    float pi = pi0[k] + pp, th = th0[k] + thPert[c];
    float p = p00 * te_rr_pow_cr(pi, cpdrd);
    prs[c] = p;
    float rmix = moist != 0 ? fmaf(fmax_(0.0f, qv[c]), rv, rd) : rd;
    rho[c] = DCR(p, (th * pi) * rmix);
  }
}

void teor_morr_prep(uint32_t *M, const uint32_t *ARG) {
  /* morr_prep.wgsl main: temperature T = (th0 + th) (pi0 + pp) and a copy qv0 of qv before
   * the microphysics column */
  Dims g = dims_at(M, B(0));
  const float *th0 = FPTR(1), *pi0 = FPTR(2), *th = FPTR(3), *pp = FPTR(4), *qv = FPTR(5);
  float *T = FPTR(6), *qv0 = FPTR(7);
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    T[c] = (th0[k] + th[c]) * (pi0[k] + pp[c]);
    qv0[c] = qv[c];
  }
}

void teor_morr_post(uint32_t *M, const uint32_t *ARG) {
  /* morr_post.wgsl main: where the column changed T (by >= 1e-4) or qv (by >= 1e-14),
   * pressure from the equation of state, pi' from it (the reference's correctly rounded
   * pow) and th from T and the new pi */
  Dims g = dims_at(M, B(0));
  const float *th0 = FPTR(1), *pi0 = FPTR(2), *rho = FPTR(3), *T = FPTR(4), *qv0 = FPTR(5), *qv = FPTR(6);
  float *th = FPTR(7), *pp = FPTR(8), *prs = FPTR(9);
  const float rd = 287.04f, cp = 1005.7f, rv = 461.5f;
  FOR_GRID {
    int i = (int)tx, j = (int)ty, k = (int)tz;
    if (i >= g.nx || j >= g.ny || k >= g.nz) continue;
    int c = GIDX(g, i, j, k);
    float rp00 = DCR(1.0f, 1e+05f), rovcp = DCR(rd, cp);
    float told = (th0[k] + th[c]) * (pi0[k] + pp[c]);
    float t = T[c], q = qv[c];
    if (fabsf(t - told) >= 0.0001f || fabsf(q - qv0[c]) >= 1e-14f) {
      float p = (rho[c] * fmaf(rv, q, rd)) * t;
      float ppn = te_rr_pow_cr(p * rp00, rovcp) - pi0[k];
      prs[c] = p;
      pp[c] = ppn;
      th[c] = DCR(t, pi0[k] + ppn) - th0[k];
    }
  }
}

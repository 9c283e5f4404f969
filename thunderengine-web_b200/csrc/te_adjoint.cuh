// Discrete adjoint of the dynamics-core step: per-kernel adjoint operators.
//
// Every kernel of the dynamics-core step (the large step of timestep.js:797-2201 restricted
// to the WENO / upwind advection, the acoustic substeps and the buoyancy coupling, with
// the thermodynamic coefficients held at their window-start values) has here an adjoint
// operator for ONE dispatch thread of the forward kernel.  Given the memory before the op
// (forward values, `p`) and the adjoints of the values after it (`l`), the operator leaves
// in `l` the adjoints of the values before the op:
//   * an output that the op overwrites has its adjoint read, then cleared (its old value
//     does not reach the result), and the contributions go to the inputs;
//   * an output updated in place (u = u + ..., tend += ...) keeps the adjoint of the
//     identity part and passes the rest on.
// Contributions to other points are added through the `Acc` policy (atomic adds on the GPU,
// OpenMP atomics on the host), so the operators can run one thread per dispatch thread.
// `Acc::skip_zero` says whether an operator returns early when the adjoint it reads is 0
// (all it would add is 0): worth it on the host; on the GPU the branch would make every
// thread wait for that load before issuing its other loads, so there it is off.
//
// The arithmetic is generic in the real type R: the library instantiates it in binary32
// (te_adjoint.cu), the binary64 CPU adjoint of the test suite in binary64.  The local
// Jacobian of a flux face (stencil values and mass fluxes -> face flux, through the WENO
// weights, their clipping and rescaling and the upwind choice) is taken by forward-mode
// dual numbers over the same formula as the forward kernel; everything else is written
// out by hand.  Branch decisions (upwind side, WENO rescaling, limiter cases) follow the
// forward values, as the discrete adjoint of the branch taken.
#pragma once
#include <cmath>
#include <cstdint>

#include "te_dims.cuh"

#ifdef __CUDACC__
#define TE_HD __host__ __device__ __forceinline__
#else
#define TE_HD inline
#endif

namespace te {
namespace adj {

constexpr int kMaxBindA = 40;

template <class R>
struct AdjArgs {
  Dims g;
  Acoustic a;
  int gx, gy, gz;
  const R* p[kMaxBindA];  // values before the op
  R* l[kMaxBindA];        // adjoints
  float f[kMaxBindA];     // f32 word of a setBytes struct bound at n
  int iv[kMaxBindA];      // i32 word
  int iv2[kMaxBindA];     // second i32 word
};

TE_HD float rfma(float a, float b, float c) { return fmaf(a, b, c); }
TE_HD double rfma(double a, double b, double c) { return fma(a, b, c); }
TE_HD float rabs(float a) { return fabsf(a); }
TE_HD double rabs(double a) { return fabs(a); }

// ------------------------------------------------------------ dual numbers

template <int N, class R>
struct Dual {
  R v;
  R d[N];
  TE_HD Dual() {}
  TE_HD Dual(R x) : v(x) {
#pragma unroll
    for (int q = 0; q < N; q++) d[q] = R(0);
  }
  TE_HD static Dual seed(R x, int slot) {
    Dual r(x);
#pragma unroll
    for (int q = 0; q < N; q++) r.d[q] = q == slot ? R(1) : R(0);
    return r;
  }
};

#define TE_DUAL template <int N, class R> TE_HD Dual<N, R>
TE_DUAL operator+(const Dual<N, R>& a, const Dual<N, R>& b) {
  Dual<N, R> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a.d[q] + b.d[q];
  return r;
}
TE_DUAL operator-(const Dual<N, R>& a, const Dual<N, R>& b) {
  Dual<N, R> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a.d[q] - b.d[q];
  return r;
}
TE_DUAL operator-(const Dual<N, R>& a) {
  Dual<N, R> r;
  r.v = -a.v;
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = -a.d[q];
  return r;
}
TE_DUAL operator*(const Dual<N, R>& a, const Dual<N, R>& b) {
  Dual<N, R> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a.d[q] * b.v + a.v * b.d[q];
  return r;
}
TE_DUAL operator*(R a, const Dual<N, R>& b) {
  Dual<N, R> r;
  r.v = a * b.v;
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a * b.d[q];
  return r;
}
TE_DUAL operator*(const Dual<N, R>& b, R a) { return a * b; }
TE_DUAL operator+(const Dual<N, R>& a, R b) {
  Dual<N, R> r = a;
  r.v = a.v + b;
  return r;
}
TE_DUAL operator+(R b, const Dual<N, R>& a) { return a + b; }
TE_DUAL operator/(const Dual<N, R>& a, const Dual<N, R>& b) {
  Dual<N, R> r;
  r.v = a.v / b.v;
  const R ib = R(1) / b.v;
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = (a.d[q] - r.v * b.d[q]) * ib;
  return r;
}
TE_DUAL operator/(const Dual<N, R>& a, R b) {
  Dual<N, R> r;
  r.v = a.v / b;
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a.d[q] / b;
  return r;
}
TE_DUAL gfma(const Dual<N, R>& a, const Dual<N, R>& b, const Dual<N, R>& c) {
  Dual<N, R> r;
  r.v = rfma(a.v, b.v, c.v);
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a.d[q] * b.v + a.v * b.d[q] + c.d[q];
  return r;
}
TE_DUAL gfma(R a, const Dual<N, R>& b, const Dual<N, R>& c) {
  Dual<N, R> r;
  r.v = rfma(a, b.v, c.v);
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a * b.d[q] + c.d[q];
  return r;
}
TE_DUAL gfma(const Dual<N, R>& a, const Dual<N, R>& b, R c) {
  Dual<N, R> r;
  r.v = rfma(a.v, b.v, c);
#pragma unroll
  for (int q = 0; q < N; q++) r.d[q] = a.d[q] * b.v + a.v * b.d[q];
  return r;
}
// WGSL min / max and abs, by value (the branch the forward takes)
TE_DUAL gmin(const Dual<N, R>& a, const Dual<N, R>& b) { return (b.v < a.v || a.v != a.v) ? b : a; }
TE_DUAL gmax(const Dual<N, R>& a, const Dual<N, R>& b) { return (a.v < b.v || a.v != a.v) ? b : a; }
TE_DUAL gabs(const Dual<N, R>& a) { return a.v < R(0) ? -a : a; }
#undef TE_DUAL

// An adjoint update of the thread's own point: no other thread of the op touches it, so a
// plain add (the point-wise operators below use it; stencil operators go through Acc).
template <class R>
TE_HD void own(R* p, R v) { *p += v; }

// ------------------------------------------------------------ face reconstructions
// The forward formulas of te_flux.cuh / te_math.cuh (adv_flux_x.wgsl:106-143,
// adv_flux_z.wgsl:106-113, adv_flux_x_weno.wgsl:106-151, adv_flux_z_weno.wgsl:111-120)
// over dual numbers.  Constant quotients (2/60, ...) are formed in R.

template <class T, class R>
TE_HD T g_flx5(const T& s1, const T& s2, const T& s3, const T& s4, const T& s5) {
  return gfma(R(-3) / R(60), s5,
              gfma(R(27) / R(60), s4, gfma(R(47) / R(60), s3, gfma(R(2) / R(60), s1, (R(-13) / R(60)) * s2))));
}

template <class T, class R>
TE_HD T g_flx3(const T& s1, const T& s2, const T& s3) {
  return gfma(R(2) / R(6), s3, gfma(R(-1) / R(6), s1, (R(5) / R(6)) * s2));
}

template <class T, class R>
TE_HD T g_weno5(const T& s1, const T& s2, const T& s3, const T& s4, const T& s5, R weps) {
  const R c13 = R(13) / R(12);
  const T e1 = gfma(R(-2), s2, s1) + s3;
  const T d1 = gfma(R(3), s3, gfma(R(-4), s2, s1));
  const T b1 = gfma(c13 * e1, e1, (R(0.25) * d1) * d1);
  const T e2 = gfma(R(-2), s3, s2) + s4;
  const T d2 = s2 - s4;
  const T b2 = gfma(c13 * e2, e2, (R(0.25) * d2) * d2);
  const T e3 = gfma(R(-2), s4, s3) + s5;
  const T d3 = gfma(R(3), s3, -(R(4) * s4)) + s5;
  const T b3 = gfma(c13 * e3, e3, (R(0.25) * d3) * d3);
  const T tau = gabs(b1 - b3);
  const T big(R(1e30f));
  T r1 = gmin(big, tau / (b1 + weps));
  T r2 = gmin(big, tau / (b2 + weps));
  T r3 = gmin(big, tau / (b3 + weps));
  const T m = gmax(r1, gmax(r2, r3));
  T one(R(1));
  if (m.v > R(1e15f)) {
    const T im = T(R(1)) / m;
    r1 = r1 * im;
    r2 = r2 * im;
    r3 = r3 * im;
    one = im * im;
  }
  const T w1 = R(0.1f) * gfma(r1, r1, one);
  const T w2 = R(0.6f) * gfma(r2, r2, one);
  const T w3 = R(0.3f) * gfma(r3, r3, one);
  const T p1 = gfma(R(11) / R(6), s3, gfma(R(2) / R(6), s1, (R(-7) / R(6)) * s2));
  const T p2 = gfma(R(2) / R(6), s4, gfma(R(-1) / R(6), s2, (R(5) / R(6)) * s3));
  const T p3 = gfma(R(-1) / R(6), s5, gfma(R(2) / R(6), s3, (R(5) / R(6)) * s4));
  return gfma(w3, p3, gfma(w1, p1, w2 * p2)) / ((w1 + w2) + w3);
}

template <class T, class R>
TE_HD T g_upstrpd(const T& s1, const T& s2, const T& s3, R weps) {
  const T dd = s2 - s1;
  const R sgn = dd.v < R(0) || (dd.v == R(0) && std::signbit(dd.v)) ? -rabs(weps) : rabs(weps);
  const T rr = (s3 - s2) / (dd + sgn);
  const T phi = gmax(T(R(0)), gmin(rr, gmin(gfma(R(2) / R(6), rr, T(R(1) / R(6))), T(R(1)))));
  return gfma(phi, s2 - s1, s2);
}

// metric planes (grid.js:200-214)
template <class R>
TE_HD R hm_uh_(const Dims& g, const R* hm, int i) { return hm[i + 3]; }
template <class R>
TE_HD R hm_uf_(const Dims& g, const R* hm, int i) { return hm[g.sJ + i + 3]; }
template <class R>
TE_HD R hm_vh_(const Dims& g, const R* hm, int j) { return hm[2 * g.sJ + j + 3]; }
template <class R>
TE_HD R hm_vf_(const Dims& g, const R* hm, int j) { return hm[2 * g.sJ + g.sK + j + 3]; }

// ------------------------------------------------------------ flux faces
// A face's inputs: the advected field at up to 7 offsets o = -3..3 along the flux
// direction (slots 0..6) and up to two mass-flux values (slots 7, 8).
constexpr int kFaceSlots = 9;

template <class R>
struct Face {
  typedef Dual<kFaceSlots, R> T;
  T s[7];
  T m0, m1;
};

// Loads the 7-point window around c along stride d; offsets whose coordinate `pos + o`
// leaves [lo, hi] (the halo-3 field) are not read and enter as constants.
template <class Q, class R>
TE_HD void load_face(Face<Q>& F, const R* a, int c, int d, int pos, int lo, int hi) {
#pragma unroll
  for (int o = -3; o <= 3; o++)
    F.s[o + 3] = (pos + o >= lo && pos + o <= hi) ? Face<Q>::T::seed(Q(a[c + o * d]), o + 3) : typename Face<Q>::T(Q(0));
}

// Adds lam * d(flux)/d(input) to the adjoints of the inputs: field `la` at c + o d, mass
// fluxes lm0 at c + m0off and lm1 at c + m1off (either may be null).
template <class R, class Acc, class TT>
TE_HD void scatter_face(const TT& f, R lam, R* la, int c, int d, R* lm0, int m0off, R* lm1, int m1off) {
#pragma unroll
  for (int o = -3; o <= 3; o++)
    if (f.d[o + 3] != 0) Acc::add(&la[c + o * d], lam * R(f.d[o + 3]));
  if (lm0 && f.d[7] != 0) Acc::add(&lm0[c + m0off], lam * R(f.d[7]));
  if (lm1 && f.d[8] != 0) Acc::add(&lm1[c + m1off], lam * R(f.d[8]));
}

#define S(o) F.s[(o) + 3]

// adv_flux_x / adv_flux_y (adv_flux_x.wgsl main): f = rr flx5(upwind stencil)
template <class R, class Acc>
TE_HD void adj_flux_lin_h(const AdjArgs<R>& A, int tx, int ty, int tz, int dir) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (dir == 0 ? (i > g.nx || j >= g.ny || k >= g.nz) : (i >= g.nx || j > g.ny || k >= g.nz)) return;
  const int c = gidx(g, i, j, k), d = dir == 0 ? 1 : g.sJ;
  const R lam = A.l[3][c];
  A.l[3][c] = R(0);
  if (Acc::skip_zero && lam == R(0)) return;
  Face<Q> F;
  load_face(F, A.p[1], c, d, dir == 0 ? i : j, -3, dir == 0 ? g.nx + 3 : g.ny + 3);
  typedef typename Face<Q>::T T;
  const T rr = T::seed(Q(A.p[2][c]), 7);
  const T f = rr.v >= 0 ? rr * g_flx5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1))
                           : rr * g_flx5<T, Q>(S(2), S(1), S(0), S(-1), S(-2));
  scatter_face<R, Acc>(f, lam, A.l[1], c, d, A.l[2], 0, (R*)nullptr, 0);
}

// adv_flux_z (adv_flux_z.wgsl main)
template <class R, class Acc>
TE_HD void adj_flux_lin_z(const AdjArgs<R>& A, int tx, int ty, int tz) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k > g.nz) return;
  const int c = gidx(g, i, j, k), sk = g.sJ * g.sK;
  const R lam = A.l[5][c];
  A.l[5][c] = R(0);
  if (k == 0 || k == g.nz || (Acc::skip_zero && lam == R(0))) return;
  const R *c1 = A.p[3], *c2 = A.p[4];
  Face<Q> F;
  typedef typename Face<Q>::T T;
#pragma unroll
  for (int o = -3; o <= 3; o++) F.s[o + 3] = (k + o >= 0 && k + o <= g.nz) ? T::seed(Q(A.p[1][c + o * sk]), o + 3) : T(Q(0));
  const T w = T::seed(Q(A.p[2][c]), 7);
  const bool up = w.v >= 0;
  T f;
  if (k == 1) f = up ? gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0)) : g_flx3<T, Q>(S(1), S(0), S(-1));
  else if (k == 2) f = up ? g_flx3<T, Q>(S(-2), S(-1), S(0)) : g_flx5<T, Q>(S(2), S(1), S(0), S(-1), S(-2));
  else if (k == g.nz - 2) f = up ? g_flx5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1)) : g_flx3<T, Q>(S(1), S(0), S(-1));
  else if (k == g.nz - 1) f = up ? g_flx3<T, Q>(S(-2), S(-1), S(0)) : gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0));
  else f = up ? g_flx5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1)) : g_flx5<T, Q>(S(2), S(1), S(0), S(-1), S(-2));
  f = w * f;
  scatter_face<R, Acc>(f, lam, A.l[1], c, sk, A.l[2], 0, (R*)nullptr, 0);
}

template <class T, class R>
TE_HD T flx5_up(const Face<R>& F, bool up, bool shifted) {
  if (shifted) return up ? g_flx5<T, R>(S(-2), S(-1), S(0), S(1), S(2)) : g_flx5<T, R>(S(3), S(2), S(1), S(0), S(-1));
  return up ? g_flx5<T, R>(S(-3), S(-2), S(-1), S(0), S(1)) : g_flx5<T, R>(S(2), S(1), S(0), S(-1), S(-2));
}
template <class T, class R>
TE_HD T weno5_up(const Face<R>& F, bool up, bool shifted, R weps) {
  if (shifted)
    return up ? g_weno5<T, R>(S(-2), S(-1), S(0), S(1), S(2), weps) : g_weno5<T, R>(S(3), S(2), S(1), S(0), S(-1), weps);
  return up ? g_weno5<T, R>(S(-3), S(-2), S(-1), S(0), S(1), weps) : g_weno5<T, R>(S(2), S(1), S(0), S(-1), S(-2), weps);
}

// adv_flux_x_stag / adv_flux_y_stag (adv_flux_x_stag.wgsl main)
template <class R, class Acc>
TE_HD void adj_flux_stag_h(const AdjArgs<R>& A, int tx, int ty, int tz, int dir) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx - 1, j = ty - 1, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  const int stag = A.iv[1];
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  const R lam = A.l[8][c];
  A.l[8][c] = R(0);
  if ((stag == 4 && k == 0) || (Acc::skip_zero && lam == R(0))) return;
  const int rb = dir == 0 ? 3 : 4;  // rru or rrv binding
  const R* rr = A.p[rb];
  R* lr = A.l[rb];
  const int d = dir == 0 ? 1 : sj;
  Face<Q> F;
  load_face(F, A.p[2], c, d, dir == 0 ? i : j, -3, dir == 0 ? g.nx + 3 : g.ny + 3);
  typedef typename Face<Q>::T T;
  int off1 = 0;
  T m;
  const T r0 = T::seed(Q(rr[c]), 7);
  if (dir == 0) {
    if (stag == 2) off1 = 1;
    else if (stag == 3) off1 = -sj;
    else if (stag == 4) off1 = -sk;
  } else {
    if (stag == 2) off1 = -1;
    else if (stag == 3) off1 = sj;
    else if (stag == 4) off1 = -sk;
  }
  if (stag == 2 || stag == 3) m = Q(0.5) * (r0 + T::seed(Q(rr[c + off1]), 8));
  else if (stag == 4) {
    const Q cc2 = A.p[7][k];
    m = gfma(T(cc2), r0, (Q(1) - cc2) * T::seed(Q(rr[c + off1]), 8));
  } else m = r0;
  const bool shifted = dir == 0 ? stag == 2 : stag == 3;
  const T f = m * flx5_up<T, Q>(F, m.v >= 0, shifted);
  scatter_face<R, Acc>(f, lam, A.l[2], c, d, lr, 0, off1 ? lr : (R*)nullptr, off1);
}

// adv_flux_z_stag (adv_flux_z_stag.wgsl main)
template <class R, class Acc>
TE_HD void adj_flux_stag_z(const AdjArgs<R>& A, int tx, int ty, int tz) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const int stag = A.iv[1];
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  const R lam = A.l[8][c];
  A.l[8][c] = R(0);
  if (Acc::skip_zero && lam == R(0)) return;
  if (stag == 4 ? k > g.nz - 1 : (k == 0 || k == g.nz)) return;
  const R *rrw = A.p[5], *c1 = A.p[6], *c2 = A.p[7];
  R* lw = A.l[5];
  typedef typename Face<Q>::T T;
  Face<Q> F;
#pragma unroll
  for (int o = -3; o <= 3; o++) F.s[o + 3] = (k + o >= 0 && k + o <= g.nz) ? T::seed(Q(A.p[2][c + o * sk]), o + 3) : T(Q(0));
  int off1;
  T m;
  const T r0 = T::seed(Q(rrw[c]), 7);
  if (stag == 2) {
    off1 = -1;
    m = Q(0.5) * (r0 + T::seed(Q(rrw[c - 1]), 8));
  } else if (stag == 3) {
    off1 = -sj;
    m = Q(0.5) * (r0 + T::seed(Q(rrw[c - sj]), 8));
  } else {
    off1 = sk;
    m = Q(0.5) * (r0 + (k < g.nz ? T::seed(Q(rrw[c + sk]), 8) : T(Q(0))));
  }
  const bool up = m.v >= 0;
  T f;
  if (stag == 4) {
    if (k == 0) f = up ? Q(0.5) * (S(0) + S(1)) : g_flx3<T, Q>(S(2), S(1), S(0));
    else if (k == 1) f = up ? g_flx3<T, Q>(S(-1), S(0), S(1)) : g_flx5<T, Q>(S(3), S(2), S(1), S(0), S(-1));
    else if (k == g.nz - 2) f = up ? g_flx5<T, Q>(S(-2), S(-1), S(0), S(1), S(2)) : g_flx3<T, Q>(S(2), S(1), S(0));
    else if (k == g.nz - 1) f = up ? g_flx3<T, Q>(S(-1), S(0), S(1)) : Q(0.5) * (S(0) + S(1));
    else f = up ? g_flx5<T, Q>(S(-2), S(-1), S(0), S(1), S(2)) : g_flx5<T, Q>(S(3), S(2), S(1), S(0), S(-1));
  } else {
    if (k == 1) f = up ? gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0)) : g_flx3<T, Q>(S(1), S(0), S(-1));
    else if (k == 2) f = up ? g_flx3<T, Q>(S(-2), S(-1), S(0)) : g_flx5<T, Q>(S(2), S(1), S(0), S(-1), S(-2));
    else if (k == g.nz - 2) f = up ? g_flx5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1)) : g_flx3<T, Q>(S(1), S(0), S(-1));
    else if (k == g.nz - 1) f = up ? g_flx3<T, Q>(S(-2), S(-1), S(0)) : gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0));
    else f = up ? g_flx5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1)) : g_flx5<T, Q>(S(2), S(1), S(0), S(-1), S(-2));
  }
  f = m * f;
  scatter_face<R, Acc>(f, lam, A.l[2], c, sk, lw, 0, lw, off1);
}

// pdef gate of the scalar WENO fluxes (adv_flux_x_weno.wgsl:106-119), by value
template <class R>
TE_HD bool pdef_ok(R s1, R s2, R s3, R s4, R s5, R weps, bool pdef) {
  if (!pdef) return true;
  R b = rabs(s1);
  b = b < rabs(s2) ? rabs(s2) : b;
  b = b < rabs(s3) ? rabs(s3) : b;
  b = b < rabs(s4) ? rabs(s4) : b;
  b = b < rabs(s5) ? rabs(s5) : b;
  return b > weps;
}

// adv_flux_x_weno / adv_flux_y_weno (scalars)
template <class R, class Acc>
TE_HD void adj_flux_weno_h(const AdjArgs<R>& A, int tx, int ty, int tz, int dir) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (dir == 0 ? (i > g.nx || j >= g.ny || k >= g.nz) : (i >= g.nx || j > g.ny || k >= g.nz)) return;
  const int c = gidx(g, i, j, k), d = dir == 0 ? 1 : g.sJ;
  const R lam = A.l[5][c];
  A.l[5][c] = R(0);
  if (Acc::skip_zero && lam == R(0)) return;
  const Q weps = (Q)A.f[3];
  const bool pdef = A.iv[4] == 1;
  Face<Q> F;
  load_face(F, A.p[1], c, d, dir == 0 ? i : j, -3, dir == 0 ? g.nx + 3 : g.ny + 3);
  typedef typename Face<Q>::T T;
  const T rr = T::seed(Q(A.p[2][c]), 7);
  const bool up = rr.v >= 0;
  const T s1 = up ? S(-3) : S(2), s2 = up ? S(-2) : S(1), s3 = up ? S(-1) : S(0), s4 = up ? S(0) : S(-1),
          s5 = up ? S(1) : S(-2);
  if (!pdef_ok<Q>(s1.v, s2.v, s3.v, s4.v, s5.v, weps, pdef)) return;
  const T f = rr * g_weno5<T, Q>(s1, s2, s3, s4, s5, weps);
  scatter_face<R, Acc>(f, lam, A.l[1], c, d, A.l[2], 0, (R*)nullptr, 0);
}

// adv_flux_z_weno (scalars; face kf = k + 1)
template <class R, class Acc>
TE_HD void adj_flux_weno_z(const AdjArgs<R>& A, int tx, int ty, int tz) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx, j = ty, kf = tz + 1;
  if (i >= g.nx || j >= g.ny || kf > g.nz + 1) return;
  const int k = kf - 1, nk = g.nz;
  const int c = gidx(g, i, j, k), sk = g.sJ * g.sK;
  const R lam = A.l[8][c];
  A.l[8][c] = R(0);
  if (kf == 1 || kf == g.nz + 1 || (Acc::skip_zero && lam == R(0))) return;
  const R *c1 = A.p[3], *c2 = A.p[4];
  const Q weps = (Q)A.f[5];
  const bool pdefweno = A.iv[7] == 1;
  typedef typename Face<Q>::T T;
  Face<Q> F;
#pragma unroll
  for (int o = -3; o <= 3; o++) F.s[o + 3] = (k + o >= 0 && k + o <= g.nz) ? T::seed(Q(A.p[1][c + o * sk]), o + 3) : T(Q(0));
  const T w = T::seed(Q(A.p[2][c]), 7);
  T f;
  bool have = false;
  if (kf == 2) {
    f = w.v >= 0 ? gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0)) : g_upstrpd<T, Q>(S(1), S(0), S(-1), weps);
    have = true;
  } else if (kf == nk) {
    f = w.v > 0 ? g_upstrpd<T, Q>(S(-2), S(-1), S(0), weps) : gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0));
    have = true;
  }
  if (!have) {
    const bool up = w.v >= 0;
    const T s1 = up ? S(-3) : S(2), s2 = up ? S(-2) : S(1), s3 = up ? S(-1) : S(0), s4 = up ? S(0) : S(-1),
            s5 = up ? S(1) : S(-2);
    if (pdefweno) {
      bool doit = pdef_ok<Q>(s1.v, s2.v, s3.v, s4.v, s5.v, weps, true);
      if (kf == 3 && w.v > 0) doit = false;
      if (kf == nk - 1 && w.v < 0) doit = false;
      if (doit) {
        f = g_weno5<T, Q>(s1, s2, s3, s4, s5, weps);
        have = true;
      } else if (kf != 3 && kf != nk - 1) {
        return;  // flux 0
      }
    }
    if (!have) {
      if (kf == 3)
        f = w.v >= 0 ? g_upstrpd<T, Q>(S(-2), S(-1), S(0), weps) : g_weno5<T, Q>(S(2), S(1), S(0), S(-1), S(-2), weps);
      else if (kf == nk - 1)
        f = w.v >= 0 ? g_weno5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1), weps) : g_upstrpd<T, Q>(S(1), S(0), S(-1), weps);
      else f = g_weno5<T, Q>(s1, s2, s3, s4, s5, weps);
    }
  }
  f = w * f;
  scatter_face<R, Acc>(f, lam, A.l[1], c, sk, A.l[2], 0, (R*)nullptr, 0);
}

// adv_flux_x_weno_uv / adv_flux_y_weno_uv (u, v momentum)
template <class R, class Acc>
TE_HD void adj_flux_weno_uv_h(const AdjArgs<R>& A, int tx, int ty, int tz, int dir) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx - 1, j = ty - 1, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  const int stag = A.iv[1];
  const int c = gidx(g, i, j, k), sj = g.sJ;
  const R lam = A.l[5][c];
  A.l[5][c] = R(0);
  if (Acc::skip_zero && lam == R(0)) return;
  const Q weps = (Q)A.f[4];
  const R* rr = A.p[3];
  R* lr = A.l[3];
  typedef typename Face<Q>::T T;
  Face<Q> F;
  const int d = dir == 0 ? 1 : sj;
  load_face(F, A.p[2], c, d, dir == 0 ? i : j, -3, dir == 0 ? g.nx + 3 : g.ny + 3);
  int off1;
  if (dir == 0) off1 = stag == 2 ? 1 : -sj;
  else off1 = stag == 2 ? -1 : sj;
  const T m = Q(0.5) * (T::seed(Q(rr[c]), 7) + T::seed(Q(rr[c + off1]), 8));
  const bool shifted = dir == 0 ? stag == 2 : stag == 3;
  const T f = m * weno5_up<T, Q>(F, m.v >= 0, shifted, weps);
  scatter_face<R, Acc>(f, lam, A.l[2], c, d, lr, 0, lr, off1);
}

// adv_flux_z_weno_uv
template <class R, class Acc>
TE_HD void adj_flux_weno_uv_z(const AdjArgs<R>& A, int tx, int ty, int tz) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const int stag = A.iv[1];
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  const R lam = A.l[7][c];
  A.l[7][c] = R(0);
  if (k == 0 || k == g.nz || (Acc::skip_zero && lam == R(0))) return;
  const R *rrw = A.p[3], *c1 = A.p[4], *c2 = A.p[5];
  R* lw = A.l[3];
  const Q weps = (Q)A.f[6];
  typedef typename Face<Q>::T T;
  Face<Q> F;
#pragma unroll
  for (int o = -3; o <= 3; o++) F.s[o + 3] = (k + o >= 0 && k + o <= g.nz) ? T::seed(Q(A.p[2][c + o * sk]), o + 3) : T(Q(0));
  const int off1 = stag == 2 ? -1 : -sj;
  const T m = Q(0.5) * (T::seed(Q(rrw[c]), 7) + T::seed(Q(rrw[c + off1]), 8));
  const bool up = m.v >= 0;
  T f;
  if (k == 1) f = up ? gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0)) : g_upstrpd<T, Q>(S(1), S(0), S(-1), weps);
  else if (k == 2) f = up ? g_upstrpd<T, Q>(S(-2), S(-1), S(0), weps) : g_weno5<T, Q>(S(2), S(1), S(0), S(-1), S(-2), weps);
  else if (k == g.nz - 2)
    f = up ? g_weno5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1), weps) : g_upstrpd<T, Q>(S(1), S(0), S(-1), weps);
  else if (k == g.nz - 1) f = up ? g_upstrpd<T, Q>(S(-2), S(-1), S(0), weps) : gfma(T(Q(c1[k])), S(-1), Q(c2[k]) * S(0));
  else
    f = up ? g_weno5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1), weps) : g_weno5<T, Q>(S(2), S(1), S(0), S(-1), S(-2), weps);
  f = m * f;
  scatter_face<R, Acc>(f, lam, A.l[2], c, sk, lw, 0, lw, off1);
}

// adv_flux_x_weno_w / adv_flux_y_weno_w (w momentum)
template <class R, class Acc>
TE_HD void adj_flux_weno_w_h(const AdjArgs<R>& A, int tx, int ty, int tz, int dir) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx - 1, j = ty - 1, k = tz;
  if (i < 0 || j < 0 || i > g.nx || j > g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k), sk = g.sJ * g.sK;
  const R lam = A.l[5][c];
  A.l[5][c] = R(0);
  if (k == 0 || (Acc::skip_zero && lam == R(0))) return;
  const Q weps = (Q)A.f[4];
  const R* rr = A.p[2];
  R* lr = A.l[2];
  const Q cc2 = A.p[3][k], cc1 = Q(1) - cc2;
  typedef typename Face<Q>::T T;
  Face<Q> F;
  const int d = dir == 0 ? 1 : g.sJ;
  load_face(F, A.p[1], c, d, dir == 0 ? i : j, -3, dir == 0 ? g.nx + 3 : g.ny + 3);
  const T ub = gfma(T(cc2), T::seed(Q(rr[c]), 7), cc1 * T::seed(Q(rr[c - sk]), 8));
  const T f = ub.v >= 0 ? ub * g_weno5<T, Q>(S(-3), S(-2), S(-1), S(0), S(1), weps)
                           : ub * g_weno5<T, Q>(S(2), S(1), S(0), S(-1), S(-2), weps);
  scatter_face<R, Acc>(f, lam, A.l[1], c, d, lr, 0, lr, -sk);
}

// adv_flux_z_weno_w: w flux at cell centres
template <class R, class Acc>
TE_HD void adj_flux_weno_w_z(const AdjArgs<R>& A, int tx, int ty, int tz) {
  typedef double Q;  // the face Jacobian in binary64 whatever R is
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz, nz = g.nz;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const int c = gidx(g, i, j, k), sk = g.sJ * g.sK;
  const R lam = A.l[4][c];
  A.l[4][c] = R(0);
  if (k > g.nz - 1 || (Acc::skip_zero && lam == R(0))) return;
  const Q weps = (Q)A.f[3];
  const R* rrw = A.p[2];
  R* lw = A.l[2];
  typedef typename Face<Q>::T T;
  Face<Q> F;
#pragma unroll
  for (int o = -3; o <= 3; o++) F.s[o + 3] = (k + o >= 0 && k + o <= g.nz) ? T::seed(Q(A.p[1][c + o * sk]), o + 3) : T(Q(0));
  const T wb = Q(0.5) * (T::seed(Q(rrw[c]), 7) + T::seed(Q(rrw[c + sk]), 8));
  T f;
  if (k == 0) f = wb.v >= 0 ? Q(0.5) * (S(0) + S(1)) : g_upstrpd<T, Q>(S(2), S(1), S(0), weps);
  else if (k == nz - 1) f = wb.v > 0 ? g_upstrpd<T, Q>(S(-1), S(0), S(1), weps) : Q(0.5) * (S(0) + S(1));
  else if (k == 1)
    f = wb.v >= 0 ? g_upstrpd<T, Q>(S(-1), S(0), S(1), weps) : g_weno5<T, Q>(S(3), S(2), S(1), S(0), S(-1), weps);
  else if (k == nz - 2)
    f = wb.v > 0 ? g_weno5<T, Q>(S(-2), S(-1), S(0), S(1), S(2), weps) : g_upstrpd<T, Q>(S(2), S(1), S(0), weps);
  else
    f = wb.v >= 0 ? g_weno5<T, Q>(S(-2), S(-1), S(0), S(1), S(2), weps)
                     : g_weno5<T, Q>(S(3), S(2), S(1), S(0), S(-1), weps);
  f = wb * f;
  scatter_face<R, Acc>(f, lam, A.l[1], c, sk, lw, 0, lw, sk);
}
#undef S

// ------------------------------------------------------------ assembly and updates

// adv_assemble (adv_assemble.wgsl:139-279), periodic / closed lateral boundaries:
// t = (s dv - divF) / rho; dest = t or dest + t
template <class R, class Acc>
TE_HD void adj_assemble(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int stag = A.iv[1];
  const int st = stag < 0 ? -stag : stag;
  const int iMax = st == 2 ? g.nx : g.nx - 1, jMax = st == 3 ? g.ny : g.ny - 1;
  const int kLo = st == 4 ? 1 : 0, kMax = g.nz - 1;
  const int i = tx, j = ty, k = tz;
  if (i > iMax || j > jMax || k < kLo || k > kMax) return;
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  R* ldest = A.l[11];
  const R lt = ldest[c];
  if (A.iv[12] == 0) ldest[c] = R(0);  // dest overwritten
  if (Acc::skip_zero && lt == R(0)) return;
  const R *s = A.p[2], *divx = A.p[6], *rho0 = A.p[7], *rf0 = A.p[8], *mh = A.p[9], *mf = A.p[10];
  const R *c1 = A.p[15], *c2 = A.p[16], *hm = A.p[30];
  R dv;
  if (st == 2) dv = R(0.5) * (divx[c] + divx[c - 1]);
  else if (st == 3) dv = R(0.5) * (divx[c] + divx[c - sj]);
  else if (st == 4) dv = rfma(c2[k], divx[c], c1[k] * divx[c - sk]);
  else dv = divx[c];
  const R mz = stag < 0 ? R(1) : (stag == 4 ? mf[k] : mh[k]);
  const R mx = st == 2 ? hm_uf_(g, hm, i) : hm_uh_(g, hm, i);
  const R my = st == 3 ? hm_vf_(g, hm, j) : hm_vh_(g, hm, j);
  const R rho = st == 4 ? rf0[k] : rho0[k];
  // the values read after the first atomic add, loaded before it
  const R sc = s[c], c1k = st == 4 ? c1[k] : R(0), c2k = st == 4 ? c2[k] : R(0);
  const R ln = lt / rho;  // adjoint of the numerator s dv - divF
  Acc::add(&A.l[2][c], ln * dv);
  const R lsdv = ln * sc;
  R* ld = A.l[6];
  if (st == 2) {
    Acc::add(&ld[c], R(0.5) * lsdv);
    Acc::add(&ld[c - 1], R(0.5) * lsdv);
  } else if (st == 3) {
    Acc::add(&ld[c], R(0.5) * lsdv);
    Acc::add(&ld[c - sj], R(0.5) * lsdv);
  } else if (st == 4) {
    Acc::add(&ld[c], c2k * lsdv);
    Acc::add(&ld[c - sk], c1k * lsdv);
  } else {
    Acc::add(&ld[c], lsdv);
  }
  // divF = dFz rdz mz + dFx rdx mx + dFy rdy my, entering with a minus sign
  const R ax = -ln * (R)g.rdx * mx, ay = -ln * (R)g.rdy * my, az = -ln * (R)g.rdz * mz;
  R *lx = A.l[3], *ly = A.l[4], *lz = A.l[5];
  if (st == 2) {
    Acc::add(&lx[c], ax);
    Acc::add(&lx[c - 1], -ax);
  } else {
    Acc::add(&lx[c + 1], ax);
    Acc::add(&lx[c], -ax);
  }
  if (st == 3) {
    Acc::add(&ly[c], ay);
    Acc::add(&ly[c - sj], -ay);
  } else {
    Acc::add(&ly[c + sj], ay);
    Acc::add(&ly[c], -ay);
  }
  if (st == 4) {
    Acc::add(&lz[c], az);
    Acc::add(&lz[c - sk], -az);
  } else {
    Acc::add(&lz[c + sk], az);
    Acc::add(&lz[c], -az);
  }
}

// rk_update: phi = fma(dttmp, tend, phi_a)
template <class R, class Acc>
TE_HD void adj_rk_update(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int stag = A.iv[1];
  const int iMax = stag == 2 ? g.nx : g.nx - 1, jMax = stag == 3 ? g.ny : g.ny - 1, kLo = stag == 4 ? 1 : 0;
  const int i = tx, j = ty, k = tz;
  if (i > iMax || j > jMax || k < kLo || k >= g.nz) return;
  const int c = gidx(g, i, j, k);
  const R lp = A.l[4][c], l2 = A.l[2][c], l3 = A.l[3][c];
  A.l[4][c] = R(0);
  A.l[2][c] = l2 + lp;
  A.l[3][c] = l3 + (R)A.f[5] * lp;
}

// apply_thterm: tend = fma(-div, thterm, tend)
template <class R, class Acc>
TE_HD void adj_apply_thterm(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k);
  const R lt = A.l[3][c], l1 = A.l[1][c];
  A.l[1][c] = l1 + -A.p[2][c] * lt;  // thterm is a constant of the core step
}

// buoyancy_apply: wten += c1 buoy(k-1) + c2 buoy(k) on interior faces
template <class R, class Acc>
TE_HD void adj_buoyancy_apply(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  const int c = gidx(g, i, j, k), sk = g.sJ * g.sK;
  const R lw = A.l[4][c];
  Acc::add(&A.l[1][c - sk], A.p[2][k] * lw);
  Acc::add(&A.l[1][c], A.p[3][k] * lw);
}

// whole-field loops (FOR_WHOLE: i, j from -3, levels by kcond)
#define TE_ADJ_WHOLE(kcond)                        \
  const Dims& g = A.g;                             \
  const int i = tx - 3, j = ty - 3, k = tz;        \
  if (i > g.nx + 3 || j > g.ny + 3 || !(kcond)) return; \
  const int c = gidx(g, i, j, k);

// update_diagnostics_moist (update_diagnostics_moist.wgsl main): the derivatives of thv,
// ppterm, piadv, thterm and buoy with respect to th' and pi' (the moisture fields are
// constants of the core step)
template <class R, class Acc>
TE_HD void adj_update_diagnostics_moist(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k < g.nz)
  const R rd = R(287.04f), rv = R(461.5f), cp = R(1005.7f), cv = R(718.66003f), cpv = R(1870.0f), cvv = R(1408.5f);
  const R rovcp = R(0.28541315f), cpl = R(4190.0f), cpi = R(2106.0f);
  const R reps = rv / rd, gacc = R(9.81f);
  const R *th0 = A.p[3], *pi0 = A.p[4], *rth0 = A.p[8];
  const R qvr = A.p[9][c];
  const R qvv = qvr > R(0) ? qvr : R(0);
  const R liq = A.p[10][c] + A.p[11][c];
  const R ice = (A.p[12][c] + A.p[13][c]) + A.p[14][c];
  const R qli = R(0) < liq + ice ? liq + ice : R(0);
  const R cpli = rfma(cpl, liq > R(0) ? liq : R(0), cpi * (ice > R(0) ? ice : R(0)));
  const R cpm = rfma(cpv, qvv, cp) + cpli;
  const R cvm = R(1) / (rfma(cvv, qvv, cv) + cpli);
  // every adjoint this thread reads, before any of its stores (the bindings are distinct
  // fields, so the loads need not wait for the stores)
  const R l15 = A.l[15][c], l16 = A.l[16][c], l17 = A.l[17][c], l18 = A.l[18][c], l19 = A.l[19][c];
  const R l1 = A.l[1][c], l2 = A.l[2][c];
  R lth = R(0), lpi = R(0);
  lth += l15 * (rfma(reps, qvv, R(1)) / ((R(1) + qvv) + qli));
  lpi += l16 * ((rovcp * cpm) * cvm);
  lpi += l17;
  lth += l18 * (rfma(-rovcp, cpm, rfma(rv, qvv, rd)) * cvm);
  lth += l19 * (gacc * rth0[k]);
  A.l[15][c] = R(0);
  A.l[16][c] = R(0);
  A.l[17][c] = R(0);
  A.l[18][c] = R(0);
  A.l[19][c] = R(0);
  A.l[1][c] = l1 + lth;
  A.l[2][c] = l2 + lpi;
}

// stage_tendency_reset: uten = vten = wten = 0
template <class R, class Acc>
TE_HD void adj_stage_tendency_reset(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k <= g.nz)
  A.l[1][c] = R(0);
  A.l[2][c] = R(0);
  A.l[3][c] = R(0);
}

// massflux_from_state: rru = rho0 u, rrv = rho0 v, rrw = rf0 w (0 at k = 0, nz)
template <class R, class Acc>
TE_HD void adj_massflux_from_state(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k <= g.nz)
  const R *rho0 = A.p[4], *rf0 = A.p[5];
  const bool wk = k != 0 && k != g.nz;
  const R l8 = wk ? A.l[8][c] : R(0), l3 = wk ? A.l[3][c] : R(0);
  if (k < g.nz) {
    const R l6 = A.l[6][c], l7 = A.l[7][c], l1 = A.l[1][c], l2 = A.l[2][c];
    A.l[1][c] = l1 + rho0[k] * l6;
    A.l[2][c] = l2 + rho0[k] * l7;
    A.l[6][c] = R(0);
    A.l[7][c] = R(0);
  }
  if (wk) A.l[3][c] = l3 + rf0[k] * l8;
  A.l[8][c] = R(0);
}

// div_massflux: divx = d(rrw)/dz mh + d(rru)/dx uh + d(rrv)/dy vh
template <class R, class Acc>
TE_HD void adj_div_massflux(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx - 3, j = ty - 3, k = tz;
  if (i > g.nx + 2 || j > g.ny + 2 || k >= g.nz) return;
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  const R ld = A.l[5][c];
  A.l[5][c] = R(0);
  if (Acc::skip_zero && ld == R(0)) return;
  const R* hm = A.p[30];
  const R az = ld * (R)g.rdz * A.p[4][k], ax = ld * (R)g.rdx * hm_uh_(g, hm, i), ay = ld * (R)g.rdy * hm_vh_(g, hm, j);
  Acc::add(&A.l[3][c + sk], az);
  Acc::add(&A.l[3][c], -az);
  Acc::add(&A.l[1][c + 1], ax);
  Acc::add(&A.l[1][c], -ax);
  Acc::add(&A.l[2][c + sj], ay);
  Acc::add(&A.l[2][c], -ay);
}

// divergence3d: the same form from the averaged velocities (|d| < 1e-30 -> 0)
template <class R, class Acc>
TE_HD void adj_divergence3d(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  const R ld = A.l[5][c];
  A.l[5][c] = R(0);
  if (Acc::skip_zero && ld == R(0)) return;
  const R *u = A.p[1], *v = A.p[2], *w = A.p[3], *mh = A.p[4], *hm = A.p[30];
  const R d = rfma((w[c + sk] - w[c]) * (R)g.rdz, mh[k],
                   rfma((u[c + 1] - u[c]) * (R)g.rdx, hm_uh_(g, hm, i), ((v[c + sj] - v[c]) * (R)g.rdy) * hm_vh_(g, hm, j)));
  if (rabs(d) < R(1e-30f)) return;
  const R az = ld * (R)g.rdz * mh[k], ax = ld * (R)g.rdx * hm_uh_(g, hm, i), ay = ld * (R)g.rdy * hm_vh_(g, hm, j);
  Acc::add(&A.l[3][c + sk], az);
  Acc::add(&A.l[3][c], -az);
  Acc::add(&A.l[1][c + 1], ax);
  Acc::add(&A.l[1][c], -ax);
  Acc::add(&A.l[2][c + sj], ay);
  Acc::add(&A.l[2][c], -ay);
}

// velocity_to_massflux: rru *= rho0, rrv *= rho0, rrw *= rf0 (0 at k = 0, nz)
template <class R, class Acc>
TE_HD void adj_velocity_to_massflux(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k <= g.nz)
  const R *rho0 = A.p[1], *rf0 = A.p[2];
  const R l5 = A.l[5][c];
  if (k < g.nz) {
    const R l3 = A.l[3][c], l4 = A.l[4][c];
    A.l[3][c] = l3 * rho0[k];
    A.l[4][c] = l4 * rho0[k];
  }
  A.l[5][c] = (k == 0 || k == g.nz) ? R(0) : l5 * rf0[k];
}

// build_sadv: sadv = (th0 - 300) + th'
template <class R, class Acc>
TE_HD void adj_build_sadv(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k < g.nz)
  const R l3 = A.l[3][c], l2 = A.l[2][c];
  A.l[2][c] = l2 + l3;
  A.l[3][c] = R(0);
}

// stage_state_reset: u, v, w, pp3d, ppd <- u_a, v_a, w_a, ppi, ppx
template <class R, class Acc>
TE_HD void adj_stage_state_reset(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k <= g.nz)
  const R l5 = A.l[5][c], l6 = A.l[6][c], l7 = A.l[7][c], l8 = A.l[8][c], l9 = A.l[9][c];
  const R l1 = A.l[1][c], l2 = A.l[2][c], l3 = A.l[3][c], l4 = A.l[4][c], l10 = A.l[10][c];
  A.l[1][c] = l1 + l5;
  A.l[2][c] = l2 + l6;
  A.l[3][c] = l3 + l7;
  A.l[4][c] = l4 + l8;
  A.l[10][c] = l10 + l9;
  A.l[5][c] = R(0);
  A.l[6][c] = R(0);
  A.l[7][c] = R(0);
  A.l[8][c] = R(0);
  A.l[9][c] = R(0);
}

// acoustic_prepare (acoustic_prepare.wgsl:131-184): qk, pk1, pk2, mm are formed from
// ppterm, piadv, thv and the profiles, which the core step holds fixed: the operator only
// clears the adjoints of the four overwritten outputs.
template <class R, class Acc>
TE_HD void adj_acoustic_prepare(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k);
  A.l[11][c] = R(0);
  A.l[12][c] = R(0);
  A.l[13][c] = R(0);
  A.l[14][c] = R(0);
}

// acoustic_begin: rru = rrv = 0, rrw = beta w
template <class R, class Acc>
TE_HD void adj_acoustic_begin(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k <= g.nz)
  const R l5 = A.l[5][c], l2 = A.l[2][c];
  A.l[3][c] = R(0);
  A.l[4][c] = R(0);
  A.l[2][c] = l2 + (R)A.a.beta * l5;
  A.l[5][c] = R(0);
}

// acoustic_uv (acoustic_uv.wgsl:145-181): u += dts (uten - tem1 uf (thv + thv_w) d(ppd)/dx)
template <class R, class Acc>
TE_HD void adj_acoustic_uv(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k), sj = g.sJ;
  const int ox = A.iv[8], oy = A.iv2[8];
  const R *thv = A.p[3], *hm = A.p[30];
  const R dts = (R)A.a.dts, cp = R(1005.7f);
  const R tem1 = ((R)g.rdx * cp) * R(0.5), tem2 = ((R)g.rdy * cp) * R(0.5);
  const bool uEdge = ox != 0 && (i == 0 || i == g.nx);
  const bool vEdge = oy != 0 && (j == 0 || j == g.ny);
  // u' = u + dts (uten - tem1 uf (thv + thv_w) (ppd - ppd_w)); thv is a constant of the
  // core step (no adjoint); u and uten updated at the thread's own point
  R gc = R(0);
  // the adjoints and values this thread reads, before any of its stores
  const R lu = uEdge ? R(0) : A.l[6][c], lv = vEdge ? R(0) : A.l[7][c];
  const R l4 = uEdge ? R(0) : A.l[4][c], l5 = vEdge ? R(0) : A.l[5][c];
  const R tc = thv[c], tw = uEdge ? R(0) : thv[c - 1], ts = vEdge ? R(0) : thv[c - sj];
  if (!uEdge && !(Acc::skip_zero && lu == R(0))) {
    const R gp = lu * dts * (tc + tw) * (-(tem1 * hm_uf_(g, hm, i)));
    gc += gp;
    Acc::add(&A.l[2][c - 1], -gp);
    A.l[4][c] = l4 + lu * dts;
  }
  if (!vEdge && !(Acc::skip_zero && lv == R(0))) {
    const R gp = lv * dts * (tc + ts) * (-(tem2 * hm_vf_(g, hm, j)));
    gc += gp;
    Acc::add(&A.l[2][c - sj], -gp);
    A.l[5][c] = l5 + lv * dts;
  }
  if (!(Acc::skip_zero && gc == R(0))) Acc::add(&A.l[2][c], gc);
}

// acoustic_fpk (acoustic_fpk.wgsl:167-207): the explicit pi' forcing from u, v, w (pk1,
// pk2, qk, piadv, ppterm are constants of the core step)
template <class R, class Acc>
TE_HD void adj_acoustic_fpk(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  const R lf = A.l[11][c];
  if (Acc::skip_zero && lf == R(0)) {
    A.l[11][c] = R(0);
    return;
  }
  const R *u = A.p[2], *v = A.p[3], *piadv = A.p[5], *ppterm = A.p[7], *pk1 = A.p[8], *pk2 = A.p[9], *qk = A.p[10];
  const R *hm = A.p[30];
  const R dts = (R)A.a.dts, beta = (R)A.a.beta;
  // every value this thread reads, before any of its stores
  const R uh = hm_uh_(g, hm, i), vh = hm_vh_(g, hm, j);
  const R du = u[c + 1] - u[c], dv = v[c + sj] - v[c];
  const R a1 = pk1[c] + qk[c], a2 = pk2[c] - qk[c], pt = ppterm[c];
  const R pc = piadv[c], pxp = piadv[c + 1], pxm = piadv[c - 1], pyp = piadv[c + sj], pym = piadv[c - sj];
  const R l6 = A.l[6][c];
  A.l[11][c] = R(0);
  const R temx = (dts * R(0.5)) * (R)g.rdx, temy = (dts * R(0.5)) * (R)g.rdy;
  const R div = rfma(du * (R)g.rdx, uh, (dv * (R)g.rdy) * vh);
  const bool clipped = rabs(div) < (R)A.a.smeps;
  Acc::add(&A.l[4][c], lf * beta * a1);
  Acc::add(&A.l[4][c + sk], lf * beta * a2);
  A.l[6][c] = l6 + lf * dts;  // ppten, read at the thread's own point only
  const R ldiv = clipped ? R(0) : lf * dts * (-pt);
  const R lu1 = ldiv * (R)g.rdx * uh - lf * (pxp - pc) * temx * uh;
  const R lu0 = -ldiv * (R)g.rdx * uh - lf * (pc - pxm) * temx * uh;
  const R lv1 = ldiv * (R)g.rdy * vh - lf * (pyp - pc) * temy * vh;
  const R lv0 = -ldiv * (R)g.rdy * vh - lf * (pc - pym) * temy * vh;
  Acc::add(&A.l[2][c + 1], lu1);
  Acc::add(&A.l[2][c], lu0);
  Acc::add(&A.l[3][c + sj], lv1);
  Acc::add(&A.l[3][c], lv0);
}

// acoustic_pp (acoustic_pp.wgsl:131-167)
template <class R, class Acc>
TE_HD void adj_acoustic_pp(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k), sk = g.sJ * g.sK;
  const R *w = A.p[2], *pk1 = A.p[3], *pk2 = A.p[4], *qk = A.p[5], *fpk = A.p[6], *pp3d = A.p[7];
  const R alph = (R)A.a.alph, kdiv = (R)A.a.kdiv;
  const bool saveX = A.iv[10] != 0;
  const R prev = pp3d[c];
  const R a1 = pk1[c] + qk[c], a2 = pk2[c] - qk[c];
  const R p = rfma(alph, rfma(w[c], a1, w[c + sk] * a2), prev + fpk[c]);
  const bool clipped = rabs(p) < (R)A.a.smeps;
  const R lpp = A.l[7][c], lppd = A.l[8][c], lpx = saveX ? A.l[9][c] : R(0);
  A.l[8][c] = R(0);
  if (saveX) A.l[9][c] = R(0);
  // pp3d = p, ppd = p + kdiv (p - prev), ppx = kdiv (p - prev)
  R lp = lpp + (R(1) + kdiv) * lppd + kdiv * lpx;
  R lprev = -kdiv * lppd - kdiv * lpx;
  if (clipped) lp = R(0);
  A.l[7][c] = lprev + lp;  // pp3d before the op: prev, and through p
  Acc::add(&A.l[6][c], lp);
  Acc::add(&A.l[2][c], lp * alph * a1);
  Acc::add(&A.l[2][c + sk], lp * alph * a2);
}

// acoustic_accumulate: rr += u (averaged on the last substep; w weighted by alph)
template <class R, class Acc>
TE_HD void adj_acoustic_accumulate(const AdjArgs<R>& A, int tx, int ty, int tz) {
  TE_ADJ_WHOLE(k <= g.nz)
  const R tavg = (R)A.f[8];
  const R lu = A.l[5][c], lv = A.l[6][c], lw = A.l[7][c];
  const R l2 = A.l[2][c], l3 = A.l[3][c], l4 = A.l[4][c];
  if (tavg > R(0)) {
    A.l[5][c] = lu * tavg;
    A.l[6][c] = lv * tavg;
    A.l[7][c] = lw * tavg;
    A.l[2][c] = l2 + lu * tavg;
    A.l[3][c] = l3 + lv * tavg;
    A.l[4][c] = l4 + lw * tavg * (R)A.a.alph;
  } else {
    A.l[2][c] = l2 + lu;
    A.l[3][c] = l3 + lv;
    A.l[4][c] = l4 + lw;
  }
}

// bc_periodic_x / bc_periodic_y: halo points copy interior points
template <class R, class Acc>
TE_HD void adj_bc_periodic(const AdjArgs<R>& A, int tx, int ty, int tz, int dir) {
  const Dims& g = A.g;
  const int h = tx, t = ty - 3, k = tz;
  const int n = dir == 0 ? g.nx : g.ny;
  if (h > 3 || t > (dir == 0 ? g.ny : g.nx) + 3 || k > g.nz) return;
  const int lo = (((-1 - h) % n) + n) % n;
  const int hi = (((n + h) % n) + n) % n;
  R* lf = A.l[1];
  // with n >= 7 the 7 source points of a row are distinct (h and n - 1 - h): each is
  // updated by one thread, so a plain add; narrower domains need the atomic
  const bool distinct = n >= 7;
  // the forward writes the low halo, then the high one: the adjoint takes them in reverse
  {
    const int dst = dir == 0 ? gidx(g, n + h, t, k) : gidx(g, t, n + h, k);
    const int src = dir == 0 ? gidx(g, hi, t, k) : gidx(g, t, hi, k);
    const R x = lf[dst];
    lf[dst] = R(0);
    if (distinct) own(&lf[src], x);
    else Acc::add(&lf[src], x);
  }
  if (h < 3) {
    const int dst = dir == 0 ? gidx(g, -1 - h, t, k) : gidx(g, t, -1 - h, k);
    const int src = dir == 0 ? gidx(g, lo, t, k) : gidx(g, t, lo, k);
    const R x = lf[dst];
    lf[dst] = R(0);
    if (distinct) own(&lf[src], x);
    else Acc::add(&lf[src], x);
  }
}

// ppx_finish: ppx = pp3d + ppx
template <class R, class Acc>
TE_HD void adj_ppx_finish(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k);
  own(&A.l[1][c], A.l[2][c]);
}

// acoustic_w_solve (acoustic_w_solve.wgsl:124-212), one column per dispatch thread.
// The forward solves T w = d for w(1..nz-1), with T tridiagonal (sub aa_k, diagonal bb_k,
// super cc_k: constants of the core step) and d_k = w_old(k) + dts wten(k)
// - beta m_k (pp(k) - pp(k-1)) - alph m_k (s(k) - s(k-1)), s = pp3d + fpk.  The adjoint
// solves T^T mu = lambda_w by a Thomas sweep (scratch: the column of the cA adjoint
// field, whose forward values are step scratch) and distributes mu.
template <class R, class Acc>
TE_HD void adj_acoustic_w_solve(const AdjArgs<R>& A, int tx, int ty, int tz) {
  const Dims& g = A.g;
  const int i = tx, j = ty;
  if (i >= g.nx || j >= g.ny || tz != 0) return;
  const int nz = g.nz, sk = g.sJ * g.sK, c0 = gidx(g, i, j, 0);
  const R *pk1 = A.p[2], *pk2 = A.p[3], *qk = A.p[4], *mm = A.p[5];
  R *lfpk = A.l[6], *lwten = A.l[7], *lpp = A.l[8], *lw = A.l[9], *lcA = A.l[10], *lcB = A.l[11];
  const R asq = (R)A.a.alph * (R)A.a.alph, alph = (R)A.a.alph, beta = (R)A.a.beta, dts = (R)A.a.dts;
  // coefficients of row k (k = 1..nz-1)
  auto Acol = [&](int k) { return pk1[c0 + k * sk] + qk[c0 + k * sk]; };
  auto Bcol = [&](int k) { return pk2[c0 + k * sk] - qk[c0 + k * sk]; };
  auto aa = [&](int k) { return (-asq) * (mm[c0 + k * sk] * Acol(k - 1)); };
  auto cc = [&](int k) { return (-asq) * ((-mm[c0 + k * sk]) * Bcol(k)); };
  auto bb = [&](int k) { return rfma(-asq, mm[c0 + k * sk] * ((-Acol(k)) + Bcol(k - 1)), R(1)); };
  // T^T: row k has sub T(k-1,k) = cc(k-1), diagonal bb(k), super T(k+1,k) = aa(k+1).
  // Forward sweep of T^T mu = lam, keeping the modified super-diagonal in lcA and the
  // modified right-hand side in lcB (their own adjoint values are cleared: cA, cB are
  // step scratch that nothing reads after the solve).
  R cp = R(0), dp = R(0);
  for (int k = 1; k <= nz - 1; k++) {
    const R sub = k > 1 ? cc(k - 1) : R(0);
    const R sup = k < nz - 1 ? aa(k + 1) : R(0);
    const R den = bb(k) - sub * cp;
    const R rhs = lw[c0 + k * sk];
    cp = sup / den;
    dp = (rhs - sub * dp) / den;
    lcA[c0 + k * sk] = cp;
    lcB[c0 + k * sk] = dp;
  }
  R mu_next = R(0);
  for (int k = nz - 1; k >= 1; k--) {
    const R mu = lcB[c0 + k * sk] - lcA[c0 + k * sk] * mu_next;
    lcB[c0 + k * sk] = mu;  // mu(k), read by the distribution below
    mu_next = mu;
  }
  for (int k = 0; k <= nz; k++) {
    lcA[c0 + k * sk] = R(0);
  }
  // d_k = w_old(k) + dts wten(k) + beta (-m_k) (pp(k) - pp(k-1)) + alph (-m_k) (s(k) - s(k-1))
  for (int k = 1; k <= nz - 1; k++) {
    const int c = c0 + k * sk;
    const R mu = lcB[c];
    const R m = mm[c];
    lwten[c] += dts * mu;
    lpp[c] += mu * (beta * (-m) + alph * (-m));
    lfpk[c] += mu * (alph * (-m));
    lpp[c - sk] -= mu * (beta * (-m) + alph * (-m));
    lfpk[c - sk] -= mu * (alph * (-m));
  }
  // w is overwritten in place: its adjoint before the op is mu at levels 1..nz-1 and 0 at
  // levels 0, nz (w(0) = w(nz) = 0 whatever w held)
  lw[c0] = R(0);
  lw[c0 + nz * sk] = R(0);
  for (int k = 1; k <= nz - 1; k++) {
    lw[c0 + k * sk] = lcB[c0 + k * sk];
    lcB[c0 + k * sk] = R(0);
  }
  lcB[c0] = R(0);
  lcB[c0 + nz * sk] = R(0);
}

}  // namespace adj
}  // namespace te

// Per-face advective fluxes of the flux kernels (data/kernels/adv_flux_*.wgsl) and the
// cell assembly of adv_assemble, as device functions shared by the per-dispatch kernels
// (te_kernels.cu) and the fused advection kernel (te_fused.cu): both run this code, so
// both produce the same bits.  face_*(A, i, j, k) is the value the reference kernel
// stores at index (i, j, k) of its output field; A holds that kernel's bindings.
#pragma once
#include "te_kernels.cuh"
#include "te_math.cuh"

namespace te {

// Index box [lo, hi] (inclusive) of faces or cells.
struct FaceRange {
  int ilo, ihi, jlo, jhi, klo, khi;
};

// The five values of an upwind-biased stencil at face index c along stride s: on the
// upwind side (up) c-3s .. c+s, else c+2s .. c-2s (reversed), both moved by `shift`
// points along the axis.  The six points of both sides are loaded before the side is
// known (the loads do not wait for the mass flux that decides it), then the side is
// chosen, so each face evaluates one reconstruction whatever the flow direction.
struct Sten5 {
  float s1, s2, s3, s4, s5;
};
__device__ __forceinline__ Sten5 sten5(const float* a, int c, int s, bool up, int shift) {
  const int b = c + (shift - 3) * s;
  const float v0 = a[b], v1 = a[b + s], v2 = a[b + 2 * s], v3 = a[b + 3 * s], v4 = a[b + 4 * s], v5 = a[b + 5 * s];
  return up ? Sten5{v0, v1, v2, v3, v4} : Sten5{v5, v4, v3, v2, v1};
}
__device__ __forceinline__ float flx5(const Sten5& t) { return flx5(t.s1, t.s2, t.s3, t.s4, t.s5); }
__device__ __forceinline__ float weno5(const Sten5& t, float weps) { return weno5(t.s1, t.s2, t.s3, t.s4, t.s5, weps); }

__device__ __forceinline__ float flx5_upwind(const float* a, int c, int s, bool up, bool shifted) {
  return flx5(sten5(a, c, s, up, shifted ? 1 : 0));
}

__device__ __forceinline__ float weno5_upwind(const float* a, int c, int s, bool up, bool shifted, float weps) {
  return weno5(sten5(a, c, s, up, shifted ? 1 : 0), weps);
}

// Horizontal faces come in two forms: face_X_h_at reads the advected field's stencil
// through (a, ca, sa) - values a[ca + n * sa] along the face's axis - so that a caller
// may stage the field elsewhere (shared memory); face_X_h reads it from the tape field.
//
// The *_c forms take the face's linear index c (and the grid g it was formed on) from
// the caller, so that a caller that walks many faces forms each index once; stagger
// dependent forms take the stagger as a template argument SG (0: read it from the
// bindings).  Every form evaluates the same operations as the reference kernel.
template <int DIR>
__device__ __forceinline__ float face_lin_h_c(const KArgs& A, int c, const float* a, int ca, int sa) {
  const float* rr = A.p[2];
  float u = rr[c];
  float f = flx5(sten5(a, ca, sa, u >= 0.0f, 0));
  return u * f;
}
template <int DIR>
__device__ __forceinline__ float face_lin_h_at(const KArgs& A, int i, int j, int k, const float* a, int ca, int sa) {
  return face_lin_h_c<DIR>(A, gidx(A.g, i, j, k), a, ca, sa);
}
template <int DIR>
__device__ __forceinline__ float face_lin_h(const KArgs& A, int i, int j, int k) {
  return face_lin_h_at<DIR>(A, i, j, k, A.p[1], gidx(A.g, i, j, k), DIR == 0 ? 1 : A.g.sJ);
}

__device__ __forceinline__ float face_lin_z_c(const KArgs& A, const Dims& g, int c, int k) {
  const float *s = A.p[1], *rrw = A.p[2], *c1 = A.p[3], *c2 = A.p[4];
  const int sk = g.sJ * g.sK;
  if (k > 2 && k < g.nz - 2) {  // the interior stencil, tested first (the common case)
    float w = rrw[c];
    return w * flx5(sten5(s, c, sk, w >= 0.0f, 0));
  }
  if (k == 0 || k == g.nz) {
    return 0.0f;
  }
  float w = rrw[c];
  bool up = w >= 0.0f;
  float f;
  if (k == 1) f = up ? fmaf(c1[k], s[c - sk], c2[k] * s[c]) : flx3(s[c + sk], s[c], s[c - sk]);
  else if (k == 2) f = up ? flx3(s[c - 2 * sk], s[c - sk], s[c]) : flx5(s[c + 2 * sk], s[c + sk], s[c], s[c - sk], s[c - 2 * sk]);
  else if (k == g.nz - 2) f = up ? flx5(s[c - 3 * sk], s[c - 2 * sk], s[c - sk], s[c], s[c + sk]) : flx3(s[c + sk], s[c], s[c - sk]);
  else if (k == g.nz - 1) f = up ? flx3(s[c - 2 * sk], s[c - sk], s[c]) : fmaf(c1[k], s[c - sk], c2[k] * s[c]);
  else f = flx5(sten5(s, c, sk, up, 0));
  return w * f;
}
__device__ __forceinline__ float face_lin_z(const KArgs& A, int i, int j, int k) {
  return face_lin_z_c(A, A.g, gidx(A.g, i, j, k), k);
}

template <int DIR, int SG = 0>
__device__ __forceinline__ float face_stag_h_c(const KArgs& A, const Dims& g, int c, int k, const float* a, int ca, int sa) {
  const int stag = SG ? SG : A.iv[1];
  const float *rr = DIR == 0 ? A.p[3] : A.p[4], *c2 = A.p[7];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  if (stag == 4 && k == 0) {
    return 0.0f;
  }
  float m;
  if (DIR == 0) {
    if (stag == 2) m = 0.5f * (rr[c] + rr[c + 1]);
    else if (stag == 3) m = 0.5f * (rr[c] + rr[c - sj]);
    else if (stag == 4) { float cc2 = c2[k]; m = fmaf(cc2, rr[c], (1.0f - cc2) * rr[c - sk]); }
    else m = rr[c];
    return m * flx5_upwind(a, ca, sa, m >= 0.0f, stag == 2);
  } else {
    if (stag == 2) m = 0.5f * (rr[c] + rr[c - 1]);
    else if (stag == 3) m = 0.5f * (rr[c] + rr[c + sj]);
    else if (stag == 4) { float cc2 = c2[k]; m = fmaf(cc2, rr[c], (1.0f - cc2) * rr[c - sk]); }
    else m = rr[c];
    return m * flx5_upwind(a, ca, sa, m >= 0.0f, stag == 3);
  }
}
template <int DIR>
__device__ __forceinline__ float face_stag_h_at(const KArgs& A, int i, int j, int k, const float* a, int ca, int sa) {
  return face_stag_h_c<DIR>(A, A.g, gidx(A.g, i, j, k), k, a, ca, sa);
}
template <int DIR>
__device__ __forceinline__ float face_stag_h(const KArgs& A, int i, int j, int k) {
  return face_stag_h_at<DIR>(A, i, j, k, A.p[2], gidx(A.g, i, j, k), DIR == 0 ? 1 : A.g.sJ);
}

template <int SG = 0>
__device__ __forceinline__ float face_stag_z_c(const KArgs& A, const Dims& g, int c, int k) {
  const int stag = SG ? SG : A.iv[1];
  const float *a = A.p[2], *rrw = A.p[5], *c1 = A.p[6], *c2 = A.p[7];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  float m;
  if (stag == 2) m = 0.5f * (rrw[c] + rrw[c - 1]);
  else if (stag == 3) m = 0.5f * (rrw[c] + rrw[c - sj]);
  else m = 0.5f * (rrw[c] + (k < g.nz ? rrw[c + sk] : 0.0f));
  bool up = m >= 0.0f;
  float f;
  // the interior stencils, tested first (the common case)
  if (stag == 4 && k >= 2 && k < g.nz - 2) return m * flx5(sten5(a, c, sk, up, 1));
  if (stag != 4 && k > 2 && k < g.nz - 2) return m * flx5(sten5(a, c, sk, up, 0));
  if (stag == 4) {
    if (k > g.nz - 1) {
      return 0.0f;
    }
    if (k == 0) f = up ? 0.5f * (a[c] + a[c + sk]) : flx3(a[c + 2 * sk], a[c + sk], a[c]);
    else if (k == 1) f = up ? flx3(a[c - sk], a[c], a[c + sk]) : flx5(a[c + 3 * sk], a[c + 2 * sk], a[c + sk], a[c], a[c - sk]);
    else if (k == g.nz - 2) f = up ? flx5(a[c - 2 * sk], a[c - sk], a[c], a[c + sk], a[c + 2 * sk]) : flx3(a[c + 2 * sk], a[c + sk], a[c]);
    else if (k == g.nz - 1) f = up ? flx3(a[c - sk], a[c], a[c + sk]) : 0.5f * (a[c] + a[c + sk]);
    else f = flx5(sten5(a, c, sk, up, 1));
  } else {
    if (k == 0 || k == g.nz) {
      return 0.0f;
    }
    if (k == 1) f = up ? fmaf(c1[k], a[c - sk], c2[k] * a[c]) : flx3(a[c + sk], a[c], a[c - sk]);
    else if (k == 2) f = up ? flx3(a[c - 2 * sk], a[c - sk], a[c]) : flx5(a[c + 2 * sk], a[c + sk], a[c], a[c - sk], a[c - 2 * sk]);
    else if (k == g.nz - 2) f = up ? flx5(a[c - 3 * sk], a[c - 2 * sk], a[c - sk], a[c], a[c + sk]) : flx3(a[c + sk], a[c], a[c - sk]);
    else if (k == g.nz - 1) f = up ? flx3(a[c - 2 * sk], a[c - sk], a[c]) : fmaf(c1[k], a[c - sk], c2[k] * a[c]);
    else f = flx5(sten5(a, c, sk, up, 0));
  }
  return m * f;
}
__device__ __forceinline__ float face_stag_z(const KArgs& A, int i, int j, int k) {
  return face_stag_z_c(A, A.g, gidx(A.g, i, j, k), k);
}

template <int DIR>
__device__ __forceinline__ float face_weno_h_c(const KArgs& A, int c, const float* a, int ca, int sa) {
  const float* rr = A.p[2];
  const float weps = A.f[3];
  const int pdef = A.iv[4];
  float r = rr[c];
  const Sten5 t = sten5(a, ca, sa, r >= 0.0f, 0);
  bool ok = pdef != 1 || weno_pdef_ok(t.s1, t.s2, t.s3, t.s4, t.s5, weps);
  return ok ? r * weno5(t, weps) : 0.0f;
}
template <int DIR>
__device__ __forceinline__ float face_weno_h_at(const KArgs& A, int i, int j, int k, const float* a, int ca, int sa) {
  return face_weno_h_c<DIR>(A, gidx(A.g, i, j, k), a, ca, sa);
}
template <int DIR>
__device__ __forceinline__ float face_weno_h(const KArgs& A, int i, int j, int k) {
  return face_weno_h_at<DIR>(A, i, j, k, A.p[1], gidx(A.g, i, j, k), DIR == 0 ? 1 : A.g.sJ);
}

__device__ __forceinline__ float face_weno_z_c(const KArgs& A, const Dims& g, int c, int k) {
  const int kf = k + 1;
  const float *a = A.p[1], *rrw = A.p[2], *c1 = A.p[3], *c2 = A.p[4];
  const float weps = A.f[5];
  const int pdefweno = A.iv[7];
  const int sk = g.sJ * g.sK, nk = g.nz;
#define AZ(o) a[c + (o) * sk]
  if (kf > 3 && kf < nk - 1) {  // the interior stencil, tested first (the common case)
    const float w = rrw[c];
    float s1, s2, s3, s4, s5;
    if (w >= 0.0f) { s1 = AZ(-3); s2 = AZ(-2); s3 = AZ(-1); s4 = AZ(0); s5 = AZ(1); }
    else { s1 = AZ(2); s2 = AZ(1); s3 = AZ(0); s4 = AZ(-1); s5 = AZ(-2); }
    if (pdefweno == 1 && !weno_pdef_ok(s1, s2, s3, s4, s5, weps)) return 0.0f;
    return w * weno5(s1, s2, s3, s4, s5, weps);
  }
  if (kf == 1 || kf == g.nz + 1) {
    return 0.0f;
  }
  float w = rrw[c];
  if (kf == 2) {
    return w >= 0.0f ? w * fmaf(c1[k], AZ(-1), c2[k] * AZ(0)) : w * upstrpd(AZ(1), AZ(0), AZ(-1), weps);
  }
  if (kf == nk) {
    return w > 0.0f ? w * upstrpd(AZ(-2), AZ(-1), AZ(0), weps) : w * fmaf(c1[k], AZ(-1), c2[k] * AZ(0));
  }
  float s1, s2, s3, s4, s5;
  if (w >= 0.0f) { s1 = AZ(-3); s2 = AZ(-2); s3 = AZ(-1); s4 = AZ(0); s5 = AZ(1); }
  else { s1 = AZ(2); s2 = AZ(1); s3 = AZ(0); s4 = AZ(-1); s5 = AZ(-2); }
  if (pdefweno == 1) {
    bool doit = weno_pdef_ok(s1, s2, s3, s4, s5, weps);
    if (kf == 3 && w > 0.0f) doit = false;
    if (kf == nk - 1 && w < 0.0f) doit = false;
    if (doit) {
      return w * weno5(s1, s2, s3, s4, s5, weps);
    }
    if (kf != 3 && kf != nk - 1) {
      return 0.0f;
    }
  }
  if (kf == 3) {
    return w >= 0.0f ? w * upstrpd(AZ(-2), AZ(-1), AZ(0), weps) : w * weno5(AZ(2), AZ(1), AZ(0), AZ(-1), AZ(-2), weps);
  }
  if (kf == nk - 1) {
    return w >= 0.0f ? w * weno5(AZ(-3), AZ(-2), AZ(-1), AZ(0), AZ(1), weps) : w * upstrpd(AZ(1), AZ(0), AZ(-1), weps);
  }
  return w * weno5(s1, s2, s3, s4, s5, weps);
#undef AZ
}
__device__ __forceinline__ float face_weno_z(const KArgs& A, int i, int j, int k) {
  return face_weno_z_c(A, A.g, gidx(A.g, i, j, k), k);
}

template <int DIR, int SG = 0>
__device__ __forceinline__ float face_weno_uv_h_c(const KArgs& A, const Dims& g, int c, const float* a, int ca, int sa) {
  const int stag = SG ? SG : A.iv[1];
  const float* rr = A.p[3];
  const float weps = A.f[4];
  const int sj = g.sJ;
  if (DIR == 0) {
    float m = stag == 2 ? 0.5f * (rr[c] + rr[c + 1]) : 0.5f * (rr[c] + rr[c - sj]);
    return m * weno5_upwind(a, ca, sa, m >= 0.0f, stag == 2, weps);
  } else {
    float m = stag == 2 ? 0.5f * (rr[c] + rr[c - 1]) : 0.5f * (rr[c] + rr[c + sj]);
    return m * weno5_upwind(a, ca, sa, m >= 0.0f, stag == 3, weps);
  }
}
template <int DIR>
__device__ __forceinline__ float face_weno_uv_h_at(const KArgs& A, int i, int j, int k, const float* a, int ca, int sa) {
  return face_weno_uv_h_c<DIR>(A, A.g, gidx(A.g, i, j, k), a, ca, sa);
}
template <int DIR>
__device__ __forceinline__ float face_weno_uv_h(const KArgs& A, int i, int j, int k) {
  return face_weno_uv_h_at<DIR>(A, i, j, k, A.p[2], gidx(A.g, i, j, k), DIR == 0 ? 1 : A.g.sJ);
}

template <int SG = 0>
__device__ __forceinline__ float face_weno_uv_z_c(const KArgs& A, const Dims& g, int c, int k) {
  const int stag = SG ? SG : A.iv[1];
  const float *a = A.p[2], *rrw = A.p[3], *c1 = A.p[4], *c2 = A.p[5];
  const float weps = A.f[6];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  if (k > 2 && k < g.nz - 2) {  // the interior stencil, tested first (the common case)
    const float m = stag == 2 ? 0.5f * (rrw[c] + rrw[c - 1]) : 0.5f * (rrw[c] + rrw[c - sj]);
    return m * weno5(sten5(a, c, sk, m >= 0.0f, 0), weps);
  }
  if (k == 0 || k == g.nz) {
    return 0.0f;
  }
#define AZ(o) a[c + (o) * sk]
  float m = stag == 2 ? 0.5f * (rrw[c] + rrw[c - 1]) : 0.5f * (rrw[c] + rrw[c - sj]);
  bool up = m >= 0.0f;
  float f;
  if (k == 1) f = up ? fmaf(c1[k], AZ(-1), c2[k] * AZ(0)) : upstrpd(AZ(1), AZ(0), AZ(-1), weps);
  else if (k == 2) f = up ? upstrpd(AZ(-2), AZ(-1), AZ(0), weps) : weno5(AZ(2), AZ(1), AZ(0), AZ(-1), AZ(-2), weps);
  else if (k == g.nz - 2) f = up ? weno5(AZ(-3), AZ(-2), AZ(-1), AZ(0), AZ(1), weps) : upstrpd(AZ(1), AZ(0), AZ(-1), weps);
  else if (k == g.nz - 1) f = up ? upstrpd(AZ(-2), AZ(-1), AZ(0), weps) : fmaf(c1[k], AZ(-1), c2[k] * AZ(0));
  else f = weno5(sten5(a, c, sk, up, 0), weps);
  return m * f;
#undef AZ
}
__device__ __forceinline__ float face_weno_uv_z(const KArgs& A, int i, int j, int k) {
  return face_weno_uv_z_c(A, A.g, gidx(A.g, i, j, k), k);
}

template <int DIR>
__device__ __forceinline__ float face_weno_w_h_c(const KArgs& A, const Dims& g, int c, int k, const float* a, int ca, int sa) {
  const float *rr = A.p[2], *c2 = A.p[3];
  const float weps = A.f[4];
  const int sk = g.sJ * g.sK;
  if (k == 0) {
    return 0.0f;
  }
  float cc2 = c2[k];
  float cc1 = 1.0f - cc2;
  float ub = fmaf(cc2, rr[c], cc1 * rr[c - sk]);
  return ub * weno5(sten5(a, ca, sa, ub >= 0.0f, 0), weps);
}
template <int DIR>
__device__ __forceinline__ float face_weno_w_h_at(const KArgs& A, int i, int j, int k, const float* a, int ca, int sa) {
  return face_weno_w_h_c<DIR>(A, A.g, gidx(A.g, i, j, k), k, a, ca, sa);
}
template <int DIR>
__device__ __forceinline__ float face_weno_w_h(const KArgs& A, int i, int j, int k) {
  return face_weno_w_h_at<DIR>(A, i, j, k, A.p[1], gidx(A.g, i, j, k), DIR == 0 ? 1 : A.g.sJ);
}

__device__ __forceinline__ float face_weno_w_z_c(const KArgs& A, const Dims& g, int c, int k) {
  const float *a = A.p[1], *rrw = A.p[2];
  const float weps = A.f[3];
  const int sk = g.sJ * g.sK, nz = g.nz;
  if (k >= 2 && k < nz - 2) {  // the interior stencil, tested first (the common case)
    const float wb = 0.5f * (rrw[c] + rrw[c + sk]);
    return wb * weno5(sten5(a, c, sk, wb >= 0.0f, 1), weps);
  }
  if (k > g.nz - 1) {
    return 0.0f;
  }
#define AZ(o) a[c + (o) * sk]
  float wb = 0.5f * (rrw[c] + rrw[c + sk]);
  float f;
  if (k == 0) f = wb >= 0.0f ? 0.5f * (AZ(0) + AZ(1)) : upstrpd(AZ(2), AZ(1), AZ(0), weps);
  else if (k == nz - 1) f = wb > 0.0f ? upstrpd(AZ(-1), AZ(0), AZ(1), weps) : 0.5f * (AZ(0) + AZ(1));
  else if (k == 1) f = wb >= 0.0f ? upstrpd(AZ(-1), AZ(0), AZ(1), weps) : weno5(AZ(3), AZ(2), AZ(1), AZ(0), AZ(-1), weps);
  else if (k == nz - 2) f = wb > 0.0f ? weno5(AZ(-2), AZ(-1), AZ(0), AZ(1), AZ(2), weps) : upstrpd(AZ(2), AZ(1), AZ(0), weps);
  else f = weno5(sten5(a, c, sk, wb >= 0.0f, 1), weps);
  return wb * f;
#undef AZ
}
__device__ __forceinline__ float face_weno_w_z(const KArgs& A, int i, int j, int k) {
  return face_weno_w_z_c(A, A.g, gidx(A.g, i, j, k), k);
}

// Pieces of adv_assemble (adv_assemble.wgsl:139-279), shared by the per-dispatch kernel
// and the fused advection kernel.  assemble_dv_off: offset of the second divergence
// value the cell's stagger averages (0 for a scalar); assemble_dv: the divergence at the
// cell from divx[c] and divx[c - off]; assemble_core: the tendency from the advected
// value s[c], that divergence and the flux differences.
template <int SG = 0>
__device__ __forceinline__ int assemble_dv_off(const KArgs& A) {
  const int stag = SG ? SG : A.iv[1], st = stag < 0 ? -stag : stag;
  return st == 2 ? 1 : (st == 3 ? A.g.sJ : (st == 4 ? A.g.sJ * A.g.sK : 0));
}
template <int SG = 0>
__device__ __forceinline__ float assemble_dv(const KArgs& A, int k, float d0, float d1) {
  const int stag = SG ? SG : A.iv[1], st = stag < 0 ? -stag : stag;
  const float *c1 = A.p[15], *c2 = A.p[16];
  if (st == 2 || st == 3) return 0.5f * (d0 + d1);
  if (st == 4) return fmaf(c2[k], d0, c1[k] * d1);
  return d0;
}
template <int SG = 0>
__device__ __forceinline__ float assemble_core(const KArgs& A, int i, int j, int k, float sc, float dv, float dFx,
                                               float dFy, float dFz) {
  const Dims& g = A.g;
  const int stag = SG ? SG : A.iv[1], st = stag < 0 ? -stag : stag;
  const float *rho0 = A.p[7], *rf0 = A.p[8], *mh = A.p[9], *mf = A.p[10];
  const float* hm = A.p[30];
  const float mz = stag < 0 ? 1.0f : (stag == 4 ? mf[k] : mh[k]);
  const float mx = st == 2 ? hm_uf(g, hm, i) : hm_uh(g, hm, i);
  const float my = st == 3 ? hm_vf(g, hm, j) : hm_vh(g, hm, j);
  const float divF = fmaf(dFz * g.rdz, mz, fmaf(dFx * g.rdx, mx, (dFy * g.rdy) * my));
  const float rho = st == 4 ? rf0[k] : rho0[k];
  return dcr(fmaf(sc, dv, -divF), rho);
}

// The open lateral boundary branches of adv_assemble (adv_assemble.wgsl:139-279): at a cell
// on an open edge whose boundary face is an inflow face, the face flux is dropped and the
// divergence term loses the boundary piece.  Cells off the open edges are left alone.
template <int SG = 0>
__device__ __forceinline__ void assemble_open(const KArgs& A, int i, int j, int k, int c, float& dFx, float& dFy,
                                              float& dv) {
  const Dims& g = A.g;
  const int stag = SG ? SG : A.iv[1];
  const float *rru = A.p[13], *rrv = A.p[14], *c1 = A.p[15], *c2 = A.p[16];
  const int openx = A.iv[17], openy = A.iv2[17];
  const float* hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  const int st = stag < 0 ? -stag : stag;
  if (openx != 0 && st != 2) {
    bool west = i == 0, east = i == g.nx - 1;
    if (west || east) {
      int cf = west ? c : c + 1;
      float un, piece;
      if (st == 3) {
        un = rru[cf] + rru[cf - sj];
        piece = ((0.5f * ((rru[c + 1 - sj] - rru[c - sj]) + (rru[c + 1] - rru[c]))) * g.rdx) * hm_uh(g, hm, i);
      } else if (st == 4) {
        float cc2 = 0.5f * (c2[k - 1] + c2[k]);
        float cc1 = 1.0f - cc2;
        un = fmaf(cc2, rru[cf], cc1 * rru[cf - sk]);
        piece = (fmaf(c1[k], rru[c + 1 - sk] - rru[c - sk], c2[k] * (rru[c + 1] - rru[c])) * g.rdx) * hm_uh(g, hm, i);
      } else {
        un = rru[cf];
        piece = ((rru[c + 1] - rru[c]) * g.rdx) * hm_uh(g, hm, i);
      }
      bool inflow = west ? un >= 0.0f : un <= 0.0f;
      if (inflow) {
        dFx = 0.0f;
        dv = dv - piece;
      }
    }
  }
  if (openy != 0 && st != 3) {
    bool south = j == 0, north = j == g.ny - 1;
    if (south || north) {
      int cf = south ? c : c + sj;
      float vn, piece;
      if (st == 2) {
        vn = rrv[cf] + rrv[cf - 1];
        piece = ((0.5f * ((rrv[c + sj - 1] - rrv[c - 1]) + (rrv[c + sj] - rrv[c]))) * g.rdy) * hm_vh(g, hm, j);
      } else if (st == 4) {
        float cc2 = 0.5f * (c2[k - 1] + c2[k]);
        float cc1 = 1.0f - cc2;
        vn = fmaf(cc2, rrv[cf], cc1 * rrv[cf - sk]);
        piece = (fmaf(c1[k], rrv[c + sj - sk] - rrv[c - sk], c2[k] * (rrv[c + sj] - rrv[c])) * g.rdy) * hm_vh(g, hm, j);
      } else {
        vn = rrv[cf];
        piece = ((rrv[c + sj] - rrv[c]) * g.rdy) * hm_vh(g, hm, j);
      }
      bool inflow = south ? vn >= 0.0f : vn <= 0.0f;
      if (inflow) {
        dFy = 0.0f;
        dv = dv - piece;
      }
    }
  }
}

// adv_assemble (adv_assemble.wgsl:139-279) at cell (i, j, k) from the flux differences:
// returns the advective tendency t (before the accumulate/store).
__device__ __forceinline__ float assemble_t(const KArgs& A, int i, int j, int k, int c, float dFx, float dFy, float dFz) {
  const float *s = A.p[2], *divx = A.p[6];
  float dv = assemble_dv(A, k, divx[c], divx[c - assemble_dv_off(A)]);
  assemble_open(A, i, j, k, c, dFx, dFy, dv);
  return assemble_core(A, i, j, k, s[c], dv, dFx, dFy, dFz);
}

}  // namespace te

// Per-dispatch CUDA kernels of the CM1 large-step dynamics path (sm_100a).
//
// One kernel per reference kernel name (data/kernels/<name>.wgsl of ThunderEngine),
// with the reference's dispatch semantics: the launch covers the tape's grid in
// threads, each thread applies the kernel's own range check, and computes the same
// binary32 operations in the same order (te_math.cuh).  These are the "exact" path of
// the player: every dispatch of a tape runs here when the caller asks for per-dispatch
// hashes; the fused step kernels (te_fused.cu) are checked against them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "te_flux.cuh"
#include "te_kernels.cuh"
#include "te_math.cuh"

// The Morrison column's arithmetic on the device (te_morr.cuh): WGSL builtins evaluated in
// binary64 and rounded once, like every other kernel here (te_math.cuh).
#define TE_MORR_HD __device__ __forceinline__
namespace te {
__device__ __forceinline__ float morr_div(float a, float b) { return dcr(a, b); }
__device__ __forceinline__ float morr_min(float a, float b) { return wmin(a, b); }
__device__ __forceinline__ float morr_max(float a, float b) { return wmax(a, b); }
__device__ __forceinline__ float morr_pow(float x, float y) { return pow_f64(x, y); }
__device__ __forceinline__ float morr_exp(float x) { return exp_f64(x); }
__device__ __forceinline__ float morr_log(float x) { return log_f64(x); }
// WGSL sin: only the gamma function's reflection for non-positive arguments reaches it,
// and no caller passes one; CUDA's sinf.
__device__ __forceinline__ float morr_sin(float x) { return sinf(x); }
// The reflectivity column's (te_refl.cuh): the correctly rounded square root and the
// binary64 log2 and atan2.
__device__ __forceinline__ float morr_sqrt(float x) { return __fsqrt_rn(x); }
__device__ __forceinline__ float morr_log2(float x) { return log2_f64(x); }
__device__ __forceinline__ float morr_atan2(float y, float x) { return atan2_f64(y, x); }
}  // namespace te
#include "te_morr.cuh"
#include "te_refl.cuh"

// TE_R qualifies every field pointer a kernel takes from its bindings.  Built as is it
// is empty; te_kernels_fast.cu compiles this file again with TE_R = __restrict__ into
// te::fast, which the player uses for ops whose bound regions do not overlap (the
// compiler may then issue all of a thread's loads before its stores).
#ifndef TE_R
#define TE_R
#endif

namespace te {
#ifdef TE_KERNELS_FAST
namespace fast {
#endif

#define TE_K3                                                   \
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;         \
  const int ty = blockIdx.y * blockDim.y + threadIdx.y;         \
  const int tz = blockIdx.z;                                    \
  if (tx >= A.gx || ty >= A.gy || tz >= A.gz) return;           \
  const Dims& g = A.g;                                          \
  (void)g;

static void launch3(void (*k)(KArgs), const KArgs& A, cudaStream_t s) {
  const dim3 b = tile_of(A);
  dim3 gr((A.gx + b.x - 1) / b.x, (A.gy + b.y - 1) / b.y, A.gz);
  launch_kernel(k, dim3(gr), dim3(b), 0, s, A);
}

#define TE_LAUNCH3(name) \
  static void launch_##name(const KArgs& A, cudaStream_t s) { launch3(k_##name, A, s); }

// Halo kernels dispatch 3-4 threads along x (the halo depth) per row: blocks of 4 x 64
// threads keep their warps full (the per-thread work is the same)
static void launch_halo3(void (*k)(KArgs), const KArgs& A, cudaStream_t s) {
  dim3 b(4, 64, 1);
  dim3 gr((A.gx + 3) / 4, (A.gy + 63) / 64, A.gz);
  launch_kernel(k, dim3(gr), dim3(b), 0, s, A);
}
#define TE_LAUNCH_HALO(name) \
  static void launch_##name(const KArgs& A, cudaStream_t s) { launch_halo3(k_##name, A, s); }

// Point-wise kernels in the __restrict__ build: a thread takes kRowVec dispatch threads
// of the same (tx, ty) on consecutive levels, loads the inputs of all of them, then
// computes and stores each (the loads of a warp stay 128-byte rows).  Op::active is the
// kernel's range check, Op::load reads one point's inputs, Op::store computes and
// writes it; the operations of a point are the per-dispatch kernel's, and distinct
// points share no written word, so the results are those of one thread per point.
enum { kRowVec = 4 };

template <class Op>
__global__ void __launch_bounds__(128) k_rowvec(KArgs A) {
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y * blockDim.y + threadIdx.y;
  const int tz0 = blockIdx.z * kRowVec;
  if (tx >= A.gx || ty >= A.gy) return;
  typename Op::In in[kRowVec];
  bool on[kRowVec];
#pragma unroll
  for (int q = 0; q < kRowVec; q++) {
    on[q] = tz0 + q < A.gz && Op::active(A, tx, ty, tz0 + q);
    if (on[q]) in[q] = Op::load(A, tx, ty, tz0 + q);
  }
#pragma unroll
  for (int q = 0; q < kRowVec; q++)
    if (on[q]) Op::store(A, tx, ty, tz0 + q, in[q]);
}

template <class Op>
static void launch_rowvec(const KArgs& A, cudaStream_t s) {
  const dim3 b = tile_of(A);
  dim3 gr((A.gx + b.x - 1) / b.x, (A.gy + b.y - 1) / b.y, (A.gz + kRowVec - 1) / kRowVec);
  launch_kernel(k_rowvec<Op>, dim3(gr), dim3(b), 0, s, A);
}

// ------------------------------------------------------------------ fluxes

// Each flux kernel stores face_*(A, i, j, k) (te_flux.cuh) over its dispatch range.

// adv_flux_x / adv_flux_y: f = rr * flx5(upwind stencil)
template <int DIR>
__global__ void k_flux_lin_h(KArgs A) {
  TE_K3
  int i = tx, j = ty, k = tz;
  if (DIR == 0 ? (i > g.nx || j >= g.ny || k >= g.nz) : (i >= g.nx || j > g.ny || k >= g.nz)) return;
  A.p[3][gidx(g, i, j, k)] = face_lin_h<DIR>(A, i, j, k);
}
static void launch_adv_flux_x(const KArgs& A, cudaStream_t s) { launch3(k_flux_lin_h<0>, A, s); }
static void launch_adv_flux_y(const KArgs& A, cudaStream_t s) { launch3(k_flux_lin_h<1>, A, s); }

__global__ void k_adv_flux_z(KArgs A) {
  TE_K3
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k > g.nz) return;
  A.p[5][gidx(g, i, j, k)] = face_lin_z(A, i, j, k);
}
TE_LAUNCH3(adv_flux_z)


// adv_flux_x_stag / adv_flux_y_stag (momentum, RK stages 1-2)
template <int DIR>
__global__ void k_flux_stag_h(KArgs A) {
  TE_K3
  int i = tx - 1, j = ty - 1, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  A.p[8][gidx(g, i, j, k)] = face_stag_h<DIR>(A, i, j, k);
}
static void launch_adv_flux_x_stag(const KArgs& A, cudaStream_t s) { launch3(k_flux_stag_h<0>, A, s); }
static void launch_adv_flux_y_stag(const KArgs& A, cudaStream_t s) { launch3(k_flux_stag_h<1>, A, s); }

__global__ void k_adv_flux_z_stag(KArgs A) {
  TE_K3
  int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  A.p[8][gidx(g, i, j, k)] = face_stag_z(A, i, j, k);
}
TE_LAUNCH3(adv_flux_z_stag)

// adv_flux_x_weno / adv_flux_y_weno (scalars, positive-definite gate)
template <int DIR>
__global__ void k_flux_weno_h(KArgs A) {
  TE_K3
  int i = tx, j = ty, k = tz;
  if (DIR == 0 ? (i > g.nx || j >= g.ny || k >= g.nz) : (i >= g.nx || j > g.ny || k >= g.nz)) return;
  A.p[5][gidx(g, i, j, k)] = face_weno_h<DIR>(A, i, j, k);
}
static void launch_adv_flux_x_weno(const KArgs& A, cudaStream_t s) { launch3(k_flux_weno_h<0>, A, s); }
static void launch_adv_flux_y_weno(const KArgs& A, cudaStream_t s) { launch3(k_flux_weno_h<1>, A, s); }

__global__ void k_adv_flux_z_weno(KArgs A) {
  TE_K3
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k > g.nz) return;
  A.p[8][gidx(g, i, j, k)] = face_weno_z(A, i, j, k);
}
TE_LAUNCH3(adv_flux_z_weno)


// adv_flux_x_weno_uv / adv_flux_y_weno_uv (u, v momentum, RK stage 3)
template <int DIR>
__global__ void k_flux_weno_uv_h(KArgs A) {
  TE_K3
  int i = tx - 1, j = ty - 1, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  A.p[5][gidx(g, i, j, k)] = face_weno_uv_h<DIR>(A, i, j, k);
}
static void launch_adv_flux_x_weno_uv(const KArgs& A, cudaStream_t s) { launch3(k_flux_weno_uv_h<0>, A, s); }
static void launch_adv_flux_y_weno_uv(const KArgs& A, cudaStream_t s) { launch3(k_flux_weno_uv_h<1>, A, s); }

__global__ void k_adv_flux_z_weno_uv(KArgs A) {
  TE_K3
  int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  A.p[7][gidx(g, i, j, k)] = face_weno_uv_z(A, i, j, k);
}
TE_LAUNCH3(adv_flux_z_weno_uv)

// adv_flux_x_weno_w / adv_flux_y_weno_w (w momentum, RK stage 3)
template <int DIR>
__global__ void k_flux_weno_w_h(KArgs A) {
  TE_K3
  int i = tx - 1, j = ty - 1, k = tz;
  if (i < 0 || j < 0 || i > g.nx || j > g.ny || k >= g.nz) return;
  A.p[5][gidx(g, i, j, k)] = face_weno_w_h<DIR>(A, i, j, k);
}
static void launch_adv_flux_x_weno_w(const KArgs& A, cudaStream_t s) { launch3(k_flux_weno_w_h<0>, A, s); }
static void launch_adv_flux_y_weno_w(const KArgs& A, cudaStream_t s) { launch3(k_flux_weno_w_h<1>, A, s); }

__global__ void k_adv_flux_z_weno_w(KArgs A) {
  TE_K3
  int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  A.p[4][gidx(g, i, j, k)] = face_weno_w_z(A, i, j, k);
}
TE_LAUNCH3(adv_flux_z_weno_w)

// ------------------------------------------------------------ assembly

__global__ void k_adv_assemble(KArgs A) {
  TE_K3
  const int stag = A.iv[1];
  const float *TE_R fx = A.p[3], *TE_R fy = A.p[4], *TE_R fz = A.p[5];
  float* TE_R tend = A.p[11];
  const int accumulate = A.iv[12];
  const int openx = A.iv[17], openy = A.iv2[17];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  const int st = stag < 0 ? -stag : stag;
  const int iMax = st == 2 ? g.nx : g.nx - 1, jMax = st == 3 ? g.ny : g.ny - 1;
  const int kLo = st == 4 ? 1 : 0, kMax = g.nz - 1;
  int i = tx, j = ty, k = tz;
  if (i > iMax || j > jMax || k < kLo || k > kMax) return;
  if (openx != 0 && st == 2 && (i == 0 || i == g.nx)) return;
  if (openy != 0 && st == 3 && (j == 0 || j == g.ny)) return;
  int c = gidx(g, i, j, k);
  float dFx = st == 2 ? fx[c] - fx[c - 1] : fx[c + 1] - fx[c];
  float dFy = st == 3 ? fy[c] - fy[c - sj] : fy[c + sj] - fy[c];
  float dFz = st == 4 ? fz[c] - fz[c - sk] : fz[c + sk] - fz[c];
  float t = assemble_t(A, i, j, k, c, dFx, dFy, dFz);
  tend[c] = accumulate != 0 ? tend[c] + t : t;
}
TE_LAUNCH3(adv_assemble)

__global__ void k_rk_update(KArgs A) {
  TE_K3
  const int stag = A.iv[1];
  const float *TE_R phiA = A.p[2], *TE_R tend = A.p[3];
  float* TE_R phi = A.p[4];
  const float dttmp = A.f[5];
  const int iMax = stag == 2 ? g.nx : g.nx - 1, jMax = stag == 3 ? g.ny : g.ny - 1, kLo = stag == 4 ? 1 : 0;
  int i = tx, j = ty, k = tz;
  if (i > iMax || j > jMax || k < kLo || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  phi[c] = fmaf(dttmp, tend[c], phiA[c]);
}
TE_LAUNCH3(rk_update)

__device__ __forceinline__ bool pdef_inflow(const Dims& g, int dir, int i, int j, int c, int step, const float* rr, int ox, int oy) {
  if (dir == 0 && ox != 0) {
    if (i == 0 && rr[c] >= 0.0f) return true;
    if (i == g.nx - 1 && rr[c + step] <= 0.0f) return true;
  }
  if (dir == 1 && oy != 0) {
    if (j == 0 && rr[c] >= 0.0f) return true;
    if (j == g.ny - 1 && rr[c + step] <= 0.0f) return true;
  }
  return false;
}

__global__ void k_pdef_dum(KArgs A) {
  TE_K3
  const int dir = A.iv[1];
  const float *TE_R s = A.p[2], *TE_R s0 = A.p[3], *TE_R f = A.p[4], *TE_R rr = A.p[5], *TE_R rho0 = A.p[6], *TE_R mh = A.p[7];
  const float dt = A.f[8];
  const int ox = A.iv[9], oy = A.iv2[9];
  float* TE_R dum = A.p[10];
  const float* TE_R hm = A.p[30];
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  int step = dir == 0 ? 1 : (dir == 1 ? g.sJ : g.sJ * g.sK);
  float rd = dir == 0 ? g.rdx : (dir == 1 ? g.rdy : g.rdz);
  float base = rho0[k] * s0[c];
  if (pdef_inflow(g, dir, i, j, c, step, rr, ox, oy)) {
    dum[c] = base;
    return;
  }
  float adv = (-(f[c + step] - f[c])) * rd;
  float sdiv = (s[c] * (rr[c + step] - rr[c])) * rd;
  float m = dir == 0 ? hm_uh(g, hm, i) : (dir == 1 ? hm_vh(g, hm, j) : mh[k]);
  adv = adv * m;
  sdiv = sdiv * m;
  dum[c] = fmaf(dt, adv + sdiv, base);
}
TE_LAUNCH3(pdef_dum)

struct PdefCell {
  bool neg;
  float f1, f2, foo3;
};
__device__ __forceinline__ PdefCell pdef_cell(float d, float dm, float dp) {
  PdefCell r{false, 0.0f, 0.0f, 0.0f};
  if (d < 0.0f) {
    float f1 = wmax(0.0f, dm), f2 = wmax(0.0f, dp);
    if (f1 + f2 > 1e-30f) {
      r.neg = true;
      r.f1 = f1;
      r.f2 = f2;
      r.foo3 = dcr(wmax(d, -(f1 + f2)), f1 + f2);
    }
  }
  return r;
}
__device__ __forceinline__ float pdef_mass(float dm2, float dm1, float d0, float dp1, float dp2, bool* flag) {
  PdefCell l = pdef_cell(dm1, dm2, d0), c = pdef_cell(d0, dm1, dp1), r = pdef_cell(dp1, d0, dp2);
  float mass = 0.0f;
  if (l.neg) mass = fmaf(l.f2, l.foo3, mass);
  if (c.neg) mass = fmaf(-(c.f1 + c.f2), c.foo3, mass);
  if (r.neg) mass = fmaf(r.f1, r.foo3, mass);
  *flag = c.neg || (l.neg && d0 > 1e-30f) || (r.neg && d0 > 1e-30f);
  return mass;
}

__global__ void k_pdef_apply(KArgs A) {
  TE_K3
  const float *TE_R s = A.p[1], *TE_R s0 = A.p[2], *TE_R fx = A.p[3], *TE_R fy = A.p[4], *TE_R fz = A.p[5];
  const float *TE_R rru = A.p[6], *TE_R rrv = A.p[7], *TE_R rrw = A.p[8], *TE_R dumx = A.p[9], *TE_R dumy = A.p[10], *TE_R dumz = A.p[11];
  const float *TE_R rho0 = A.p[12], *TE_R mh = A.p[13];
  const float dt = A.f[14];
  const int ox = A.iv[15], oy = A.iv2[15];
  float* TE_R tend = A.p[16];
  const float* TE_R hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float rdt = dcr(1.0f, dt);
  float base = rho0[k] * s0[c];
  float delta = 0.0f;
  bool flag;
  float mx = pdef_mass(dumx[c - 2], dumx[c - 1], dumx[c], dumx[c + 1], dumx[c + 2], &flag);
  if (flag) {
    float sdiv = ((s[c] * (rru[c + 1] - rru[c])) * g.rdx) * hm_uh(g, hm, i);
    float advOld = pdef_inflow(g, 0, i, j, c, 1, rru, ox, oy) ? -sdiv : ((-(fx[c + 1] - fx[c])) * g.rdx) * hm_uh(g, hm, i);
    float advNew = fmaf((dumx[c] + mx) - base, rdt, -sdiv);
    delta = delta + (advNew - advOld);
  }
  float my = pdef_mass(dumy[c - 2 * sj], dumy[c - sj], dumy[c], dumy[c + sj], dumy[c + 2 * sj], &flag);
  if (flag) {
    float sdiv = ((s[c] * (rrv[c + sj] - rrv[c])) * g.rdy) * hm_vh(g, hm, j);
    float advOld = pdef_inflow(g, 1, i, j, c, sj, rrv, ox, oy) ? -sdiv : ((-(fy[c + sj] - fy[c])) * g.rdy) * hm_vh(g, hm, j);
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
  tend[c] = tend[c] + dcr(delta, rho0[k]);
}
TE_LAUNCH3(pdef_apply)

// --------------------------------------------------------- whole-grid glue

#define TE_WHOLE(kcond)                                          \
  int i = tx - 3, j = ty - 3, k = tz;                            \
  if (i > g.nx + 3 || j > g.ny + 3 || !(kcond)) return;          \
  int c = gidx(g, i, j, k);

__global__ void k_build_sadv(KArgs A) {
  TE_K3
  const float *TE_R th0 = A.p[1], *TE_R thp = A.p[2];
  float* TE_R sadv = A.p[3];
  TE_WHOLE(k < g.nz)
  sadv[c] = (th0[k] - 300.0f) + thp[c];
}
TE_LAUNCH3(build_sadv)

__global__ void k_massflux_from_state(KArgs A) {
  TE_K3
  const float *TE_R u = A.p[1], *TE_R v = A.p[2], *TE_R w = A.p[3], *TE_R rho0 = A.p[4], *TE_R rf0 = A.p[5];
  float *TE_R rru = A.p[6], *TE_R rrv = A.p[7], *TE_R rrw = A.p[8];
  TE_WHOLE(k <= g.nz)
  if (k < g.nz) {
    rru[c] = rho0[k] * u[c];
    rrv[c] = rho0[k] * v[c];
  }
  rrw[c] = (k == 0 || k == g.nz) ? 0.0f : rf0[k] * w[c];
}
TE_LAUNCH3(massflux_from_state)

__global__ void k_div_massflux(KArgs A) {
  TE_K3
  const float *TE_R rru = A.p[1], *TE_R rrv = A.p[2], *TE_R rrw = A.p[3], *TE_R mh = A.p[4];
  float* TE_R divx = A.p[5];
  const float* TE_R hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  int i = tx - 3, j = ty - 3, k = tz;
  if (i > g.nx + 2 || j > g.ny + 2 || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  divx[c] = fmaf((rrw[c + sk] - rrw[c]) * g.rdz, mh[k],
                 fmaf((rru[c + 1] - rru[c]) * g.rdx, hm_uh(g, hm, i), ((rrv[c + sj] - rrv[c]) * g.rdy) * hm_vh(g, hm, j)));
}
TE_LAUNCH3(div_massflux)

struct OpDivMassflux {  // div_massflux as a row-vector op (same operations)
  struct In {
    float ru0, ru1, rv0, rv1, rw0, rw1;
  };
  static __device__ __forceinline__ bool active(const KArgs& A, int tx, int ty, int tz) {
    return tx - 3 <= A.g.nx + 2 && ty - 3 <= A.g.ny + 2 && tz < A.g.nz;
  }
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    const Dims& g = A.g;
    const float *TE_R rru = A.p[1], *TE_R rrv = A.p[2], *TE_R rrw = A.p[3];
    const int c = gidx(g, tx - 3, ty - 3, tz), sj = g.sJ, sk = g.sJ * g.sK;
    return In{rru[c], rru[c + 1], rrv[c], rrv[c + sj], rrw[c], rrw[c + sk]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    const Dims& g = A.g;
    const float *TE_R mh = A.p[4], *TE_R hm = A.p[30];
    float* TE_R divx = A.p[5];
    const int i = tx - 3, j = ty - 3, k = tz, c = gidx(g, i, j, k);
    divx[c] = fmaf((v.rw1 - v.rw0) * g.rdz, mh[k],
                   fmaf((v.ru1 - v.ru0) * g.rdx, hm_uh(g, hm, i), ((v.rv1 - v.rv0) * g.rdy) * hm_vh(g, hm, j)));
  }
};

__global__ void k_velocity_to_massflux(KArgs A) {
  TE_K3
  const float *TE_R rho0 = A.p[1], *TE_R rf0 = A.p[2];
  float *TE_R rru = A.p[3], *TE_R rrv = A.p[4], *TE_R rrw = A.p[5];
  TE_WHOLE(k <= g.nz)
  if (k < g.nz) {
    rru[c] = rru[c] * rho0[k];
    rrv[c] = rrv[c] * rho0[k];
  }
  rrw[c] = (k == 0 || k == g.nz) ? 0.0f : rrw[c] * rf0[k];
}
TE_LAUNCH3(velocity_to_massflux)

struct OpVelocityToMassflux {  // velocity_to_massflux as a row-vector op
  struct In {
    float ru, rv, rw;
  };
  static __device__ __forceinline__ bool active(const KArgs& A, int tx, int ty, int tz) {
    return tx - 3 <= A.g.nx + 3 && ty - 3 <= A.g.ny + 3 && tz <= A.g.nz;
  }
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    const int c = gidx(A.g, tx - 3, ty - 3, tz);
    const float *TE_R rru = A.p[3], *TE_R rrv = A.p[4], *TE_R rrw = A.p[5];
    const int k = tz;
    return In{k < A.g.nz ? rru[c] : 0.0f, k < A.g.nz ? rrv[c] : 0.0f, (k == 0 || k == A.g.nz) ? 0.0f : rrw[c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    const Dims& g = A.g;
    const float *TE_R rho0 = A.p[1], *TE_R rf0 = A.p[2];
    float *TE_R rru = A.p[3], *TE_R rrv = A.p[4], *TE_R rrw = A.p[5];
    const int k = tz, c = gidx(g, tx - 3, ty - 3, k);
    if (k < g.nz) {
      rru[c] = v.ru * rho0[k];
      rrv[c] = v.rv * rho0[k];
    }
    rrw[c] = (k == 0 || k == g.nz) ? 0.0f : v.rw * rf0[k];
  }
};

// Words of one field when the dispatch covers every point of the first `levels` levels of
// a field, halos included (TE_WHOLE(k < levels)), and the layout has no row padding, so
// that the points are the field's first sJ * sK * levels words, in order; 0 otherwise.  Kernels that copy or
// clear whole fields then walk them as aligned 16-byte vectors (whole 32-byte sectors; the
// per-point form leaves the sectors at row ends half-written by two warps).
static unsigned long long whole_field_words(const KArgs& A, const int* fields, int n, int levels) {
  const Dims& g = A.g;
  const unsigned long long words = (unsigned long long)g.sJ * g.sK * levels;
  if (!(g.sJ == g.nx + 7 && g.sK == g.ny + 7 && A.gx >= g.nx + 7 && A.gy >= g.ny + 7 && A.gz >= levels)) return 0;
  if (words >= (1ull << 32)) return 0;
  for (int q = 0; q < n; q++)
    if ((reinterpret_cast<uintptr_t>(A.p[fields[q]]) & 15) != 0) return 0;
  return words;
}

// stage_state_reset over whole fields: dst[n] = src[n] for the five (src, dst) pairs.
__global__ void k_stage_state_reset_v4(KArgs A, unsigned words) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n4 = words / 4;
  const float *TE_R s0 = A.p[1], *TE_R s1 = A.p[2], *TE_R s2 = A.p[3], *TE_R s3 = A.p[4], *TE_R s4 = A.p[10];
  float *TE_R d0 = A.p[5], *TE_R d1 = A.p[6], *TE_R d2 = A.p[7], *TE_R d3 = A.p[8], *TE_R d4 = A.p[9];
  if (q < n4) {
    const float4 a = reinterpret_cast<const float4*>(s0)[q], b = reinterpret_cast<const float4*>(s1)[q];
    const float4 c = reinterpret_cast<const float4*>(s2)[q], d = reinterpret_cast<const float4*>(s3)[q];
    const float4 e = reinterpret_cast<const float4*>(s4)[q];
    reinterpret_cast<float4*>(d0)[q] = a;
    reinterpret_cast<float4*>(d1)[q] = b;
    reinterpret_cast<float4*>(d2)[q] = c;
    reinterpret_cast<float4*>(d3)[q] = d;
    reinterpret_cast<float4*>(d4)[q] = e;
  }
  if (q < words - 4 * n4) {
    const unsigned w = 4 * n4 + q;
    d0[w] = s0[w];
    d1[w] = s1[w];
    d2[w] = s2[w];
    d3[w] = s3[w];
    d4[w] = s4[w];
  }
}

__global__ void k_stage_state_reset(KArgs A) {
  TE_K3
  const float *TE_R ua = A.p[1], *TE_R va = A.p[2], *TE_R wa = A.p[3], *TE_R ppi = A.p[4];
  float *TE_R u = A.p[5], *TE_R v = A.p[6], *TE_R w = A.p[7], *TE_R pp3d = A.p[8], *TE_R ppd = A.p[9];
  const float* TE_R ppx = A.p[10];
  TE_WHOLE(k <= g.nz)
  u[c] = ua[c];
  v[c] = va[c];
  w[c] = wa[c];
  pp3d[c] = ppi[c];
  ppd[c] = ppx[c];
}

static void launch_stage_state_reset(const KArgs& A, cudaStream_t s) {
  // the vector form loads all five sources before it stores: only for disjoint bindings
  // (the __restrict__ build), where that order cannot change a result
  static const int fields[10] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10};
#ifdef TE_KERNELS_FAST
  const unsigned long long words = whole_field_words(A, fields, 10, A.g.nz + 1);
#else
  const unsigned long long words = 0;
  (void)fields;
#endif
  if (words) {
    const unsigned n4 = (unsigned)(words / 4);
    launch_kernel(k_stage_state_reset_v4, dim3((n4 + 255) / 256), dim3(256), 0, s, A, (unsigned)words);
  } else {
    launch3(k_stage_state_reset, A, s);
  }
}

__global__ void k_stage_tendency_reset(KArgs A) {
  TE_K3
  float *TE_R uten = A.p[1], *TE_R vten = A.p[2], *TE_R wten = A.p[3];
  TE_WHOLE(k <= g.nz)
  uten[c] = 0.0f;
  vten[c] = 0.0f;
  wten[c] = 0.0f;
}

// The same zeros over whole fields (whole_field_words): 16-byte stores, then the last
// words % 4 words one by one.
__global__ void k_stage_tendency_reset_v4(float* TE_R a, float* TE_R b, float* TE_R c, unsigned words) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n4 = words / 4;
  if (q < n4) {
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    reinterpret_cast<float4*>(a)[q] = z;
    reinterpret_cast<float4*>(b)[q] = z;
    reinterpret_cast<float4*>(c)[q] = z;
  }
  if (q < words - 4 * n4) {
    a[4 * n4 + q] = 0.0f;
    b[4 * n4 + q] = 0.0f;
    c[4 * n4 + q] = 0.0f;
  }
}

static void launch_stage_tendency_reset(const KArgs& A, cudaStream_t s) {
  static const int fields[3] = {1, 2, 3};
  const unsigned long long words = whole_field_words(A, fields, 3, A.g.nz + 1);
  if (words) {
    const unsigned n4 = (unsigned)(words / 4);
    launch_kernel(k_stage_tendency_reset_v4, dim3((n4 + 255) / 256), dim3(256), 0, s, A.p[1], A.p[2], A.p[3], (unsigned)words);
  } else {
    launch3(k_stage_tendency_reset, A, s);
  }
}

__global__ void k_buoyancy_apply(KArgs A) {
  TE_K3
  const float *TE_R buoy = A.p[1], *TE_R c1 = A.p[2], *TE_R c2 = A.p[3];
  float* TE_R wten = A.p[4];
  const int sk = g.sJ * g.sK;
  int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  int c = gidx(g, i, j, k);
  wten[c] = wten[c] + fmaf(c1[k], buoy[c - sk], c2[k] * buoy[c]);
}
TE_LAUNCH3(buoyancy_apply)

__global__ void k_apply_thterm(KArgs A) {
  TE_K3
  const float *TE_R div = A.p[1], *TE_R thterm = A.p[2];
  float* TE_R tend = A.p[3];
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  tend[c] = fmaf(-div[c], thterm[c], tend[c]);
}
TE_LAUNCH3(apply_thterm)

// ------------------------------------------------------ acoustic substep

__global__ void k_acoustic_prepare(KArgs A) {
  TE_K3
  const Acoustic a = A.a;
  const float *TE_R ppterm = A.p[2], *TE_R piadv = A.p[3], *TE_R thv = A.p[4], *TE_R rr0 = A.p[5], *TE_R rf0 = A.p[6];
  const float *TE_R mh = A.p[7], *TE_R mf = A.p[8], *TE_R c1 = A.p[9], *TE_R c2 = A.p[10];
  float *TE_R qk = A.p[11], *TE_R pk1 = A.p[12], *TE_R pk2 = A.p[13], *TE_R mm = A.p[14];
  const int sk = g.sJ * g.sK;
  const float cp = 1005.7f;
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float tem = (a.dts * g.rdz) * mh[k];
  float r2 = (tem * rr0[k]) * rf0[k + 1];
  float r1 = (tem * rr0[k]) * rf0[k];
  float tem1 = ((a.dts * g.rdz) * cp) * mf[k];
  float c1a = c1[k], c1b = c1[k + 1], c2a = c2[k], c2b = c2[k + 1];
  bool vec_v = g.nx > 3 && i < (g.nx / 4) * 4;
  qk[c] = tem * ppterm[c];
  float p2 = 0.0f, p1 = 0.0f;
  if (k != g.nz - 1)
    p2 = vec_v ? fmaf(-c2b, piadv[c + sk], (1.0f - c1b) * piadv[c]) : fmaf(1.0f - c1b, piadv[c], -(c2b * piadv[c + sk]));
  if (k != 0)
    p1 = vec_v ? fmaf(c2a - 1.0f, piadv[c], c1a * piadv[c - sk]) : fmaf(c1a, piadv[c - sk], (c2a - 1.0f) * piadv[c]);
  pk2[c] = k == g.nz - 1 ? 0.0f : r2 * p2;
  pk1[c] = k == 0 ? 0.0f : r1 * p1;
  mm[c] = tem1 * fmaf(c2a, thv[c], c1a * (k == 0 ? thv[c] : thv[c - sk]));
}
TE_LAUNCH3(acoustic_prepare)

__global__ void k_acoustic_begin(KArgs A) {
  TE_K3
  const float* TE_R w = A.p[2];
  float *TE_R rru = A.p[3], *TE_R rrv = A.p[4], *TE_R rrw = A.p[5];
  TE_WHOLE(k <= g.nz)
  rru[c] = 0.0f;
  rrv[c] = 0.0f;
  rrw[c] = w[c] * A.a.beta;
}
TE_LAUNCH3(acoustic_begin)

__global__ void k_acoustic_uv(KArgs A) {
  TE_K3
  const Acoustic a = A.a;
  const float *TE_R ppd = A.p[2], *TE_R thv = A.p[3], *TE_R uten = A.p[4], *TE_R vten = A.p[5];
  float *TE_R u = A.p[6], *TE_R v = A.p[7];
  const int ox = A.iv[8], oy = A.iv2[8];
  const float* TE_R hm = A.p[30];
  const int sj = g.sJ;
  const float cp = 1005.7f;
  int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float tem1 = (g.rdx * cp) * 0.5f;
  float tem2 = (g.rdy * cp) * 0.5f;
  bool uEdge = ox != 0 && (i == 0 || i == g.nx);
  bool vEdge = oy != 0 && (j == 0 || j == g.ny);
  if (!uEdge) u[c] = fmaf(a.dts, fmaf(-((tem1 * (ppd[c] - ppd[c - 1])) * hm_uf(g, hm, i)), thv[c] + thv[c - 1], uten[c]), u[c]);
  if (!vEdge) v[c] = fmaf(a.dts, fmaf(-((tem2 * (ppd[c] - ppd[c - sj])) * hm_vf(g, hm, j)), thv[c] + thv[c - sj], vten[c]), v[c]);
}
TE_LAUNCH3(acoustic_uv)

__global__ void k_acoustic_fpk(KArgs A) {
  TE_K3
  const Acoustic a = A.a;
  const float *TE_R u = A.p[2], *TE_R v = A.p[3], *TE_R w = A.p[4], *TE_R piadv = A.p[5], *TE_R ppten = A.p[6], *TE_R ppterm = A.p[7];
  const float *TE_R pk1 = A.p[8], *TE_R pk2 = A.p[9], *TE_R qk = A.p[10];
  float* TE_R fpk = A.p[11];
  const float* TE_R hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float temx = (a.dts * 0.5f) * g.rdx;
  float temy = (a.dts * 0.5f) * g.rdy;
  float div = fmaf((u[c + 1] - u[c]) * g.rdx, hm_uh(g, hm, i), ((v[c + sj] - v[c]) * g.rdy) * hm_vh(g, hm, j));
  if (fabsf(div) < a.smeps) div = 0.0f;
  float advPi = fmaf((-fmaf(u[c], piadv[c] - piadv[c - 1], u[c + 1] * (piadv[c + 1] - piadv[c]))) * temx, hm_uh(g, hm, i),
                     -((fmaf(v[c], piadv[c] - piadv[c - sj], v[c + sj] * (piadv[c + sj] - piadv[c])) * temy) * hm_vh(g, hm, j)));
  fpk[c] = fmaf(a.beta, fmaf(w[c], pk1[c] + qk[c], w[c + sk] * (pk2[c] - qk[c])), fmaf(a.dts, fmaf(-ppterm[c], div, ppten[c]), advPi));
}
TE_LAUNCH3(acoustic_fpk)

// Vertically implicit w-pi' solve: one column per thread, columns of a warp adjacent
// in i (coalesced), the Thomas recurrence sequential in k as in the reference.
__global__ void k_acoustic_w_solve(KArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const Dims& g = A.g;
  if (i >= A.gx || j >= A.gy) return;
  if (i >= g.nx || j >= g.ny) return;
  const Acoustic a = A.a;
  const float *TE_R pk1 = A.p[2], *TE_R pk2 = A.p[3], *TE_R qk = A.p[4], *TE_R mm = A.p[5], *TE_R fpk = A.p[6], *TE_R wten = A.p[7], *TE_R pp3d = A.p[8];
  float *TE_R w = A.p[9], *TE_R cA = A.p[10], *TE_R cB = A.p[11];
  const int sk = g.sJ * g.sK;
  const float asq = a.alph * a.alph;
  w[gidx(g, i, j, 0)] = 0.0f;
  w[gidx(g, i, j, g.nz)] = 0.0f;
  float aa, bb, cc, dd;
  auto lam = [&](int kk) {
    int c = gidx(g, i, j, kk), cm = c - sk;
    float m = mm[c];
    aa = (-asq) * (m * (pk1[cm] + qk[cm]));
    cc = (-asq) * ((-m) * (pk2[c] - qk[c]));
    bb = fmaf(-asq, m * ((-(pk1[c] + qk[c])) + (pk2[cm] - qk[cm])), 1.0f);
    float fw = fmaf(a.dts, wten[c], a.beta * ((-m) * (pp3d[c] - pp3d[cm])));
    dd = fmaf(a.alph, (-m) * ((pp3d[c] + fpk[c]) - (pp3d[cm] + fpk[cm])), w[c] + fw);
  };
  {
    int c = gidx(g, i, j, 1);
    lam(1);
    float r = dcr(1.0f, bb);
    cA[c] = (-cc) * r;
    cB[c] = dd * r;
  }
  for (int k = 2; k < g.nz - 1; k++) {
    int c = gidx(g, i, j, k);
    lam(k);
    float r = dcr(1.0f, fmaf(aa, cA[c - sk], bb));
    cA[c] = (-cc) * r;
    cB[c] = fmaf(-aa, cB[c - sk], dd) * r;
  }
  {
    int k = g.nz - 1, c = gidx(g, i, j, k);
    lam(k);
    float r = dcr(1.0f, fmaf(aa, cA[c - sk], bb));
    w[c] = fmaf(-aa, cB[c - sk], dd) * r;
  }
  for (int k = g.nz - 2; k >= 1; k--) {
    int c = gidx(g, i, j, k);
    w[c] = fmaf(cA[c], w[c + sk], cB[c]);
  }
}
static void launch_acoustic_w_solve_columns(const KArgs& A, cudaStream_t s) {
  dim3 b(32, 4, 1);
  dim3 gr((A.gx + 31) / 32, (A.gy + 3) / 4, 1);
  launch_kernel(k_acoustic_w_solve, dim3(gr), dim3(b), 0, s, A);
}
#ifndef TE_KERNELS_FAST
static void launch_acoustic_w_solve(const KArgs& A, cudaStream_t s) { launch_acoustic_w_solve_columns(A, s); }
#endif

__global__ void k_acoustic_pp(KArgs A) {
  TE_K3
  const Acoustic a = A.a;
  const float *TE_R w = A.p[2], *TE_R pk1 = A.p[3], *TE_R pk2 = A.p[4], *TE_R qk = A.p[5], *TE_R fpk = A.p[6];
  float *TE_R pp3d = A.p[7], *TE_R ppd = A.p[8], *TE_R ppx = A.p[9];
  const int saveX = A.iv[10];
  const int sk = g.sJ * g.sK;
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float prev = pp3d[c];
  float p = fmaf(a.alph, fmaf(w[c], pk1[c] + qk[c], w[c + sk] * (pk2[c] - qk[c])), prev + fpk[c]);
  if (fabsf(p) < a.smeps) p = 0.0f;
  pp3d[c] = p;
  float dum1 = a.kdiv * (p - prev);
  ppd[c] = p + dum1;
  if (saveX != 0) ppx[c] = dum1;
}
TE_LAUNCH3(acoustic_pp)

__global__ void k_acoustic_accumulate(KArgs A) {
  TE_K3
  const float *TE_R u = A.p[2], *TE_R v = A.p[3], *TE_R w = A.p[4];
  float *TE_R rru = A.p[5], *TE_R rrv = A.p[6], *TE_R rrw = A.p[7];
  const float tavg = A.f[8];
  TE_WHOLE(k <= g.nz)
  if (tavg > 0.0f) {
    rru[c] = (rru[c] + u[c]) * tavg;
    rrv[c] = (rrv[c] + v[c]) * tavg;
    rrw[c] = fmaf(w[c], A.a.alph, rrw[c]) * tavg;
  } else {
    rru[c] = rru[c] + u[c];
    rrv[c] = rrv[c] + v[c];
    rrw[c] = rrw[c] + w[c];
  }
}
TE_LAUNCH3(acoustic_accumulate)

// ------------------------------------------------------- periodic halos

__global__ void k_bc_periodic_x(KArgs A) {
  TE_K3
  float* TE_R f = A.p[1];
  int h = tx, jj = ty - 3, k = tz;
  if (h > 3 || jj > g.ny + 3 || k > g.nz) return;
  int lo = (((-1 - h) % g.nx) + g.nx) % g.nx;
  int hi = (((g.nx + h) % g.nx) + g.nx) % g.nx;
  if (h < 3) f[gidx(g, -1 - h, jj, k)] = f[gidx(g, lo, jj, k)];
  f[gidx(g, g.nx + h, jj, k)] = f[gidx(g, hi, jj, k)];
}
TE_LAUNCH_HALO(bc_periodic_x)

__global__ void k_bc_periodic_y(KArgs A) {
  TE_K3
  float* TE_R f = A.p[1];
  int h = tx, i = ty - 3, k = tz;
  if (h > 3 || i > g.nx + 3 || k > g.nz) return;
  int lo = (((-1 - h) % g.ny) + g.ny) % g.ny;
  int hi = (((g.ny + h) % g.ny) + g.ny) % g.ny;
  if (h < 3) f[gidx(g, i, -1 - h, k)] = f[gidx(g, i, lo, k)];
  f[gidx(g, i, g.ny + h, k)] = f[gidx(g, i, hi, k)];
}
TE_LAUNCH_HALO(bc_periodic_y)

// ------------------------------------------------------ open lateral boundaries

// bc_open_x.wgsl / bc_open_y.wgsl: zero-gradient halos, -1-h <- 0 and last+1+h <- last
// (h < 3, last = n + stagger - 1)
__global__ void k_bc_open_x(KArgs A) {
  TE_K3
  float* TE_R f = A.p[1];
  const int stagX = A.iv[2];
  const int h = tx, jj = ty - 3, k = tz;
  if (h >= 3 || jj > g.ny + 3 || k > g.nz) return;
  const int last = g.nx + stagX - 1;
  f[gidx(g, -1 - h, jj, k)] = f[gidx(g, 0, jj, k)];
  f[gidx(g, last + 1 + h, jj, k)] = f[gidx(g, last, jj, k)];
}
TE_LAUNCH_HALO(bc_open_x)

__global__ void k_bc_open_y(KArgs A) {
  TE_K3
  float* TE_R f = A.p[1];
  const int stagY = A.iv[2];
  const int h = tx, ii = ty - 3, k = tz;
  if (h >= 3 || ii > g.nx + 3 || k > g.nz) return;
  const int last = g.ny + stagY - 1;
  f[gidx(g, ii, -1 - h, k)] = f[gidx(g, ii, 0, k)];
  f[gidx(g, ii, last + 1 + h, k)] = f[gidx(g, ii, last, k)];
}
TE_LAUNCH_HALO(bc_open_y)

// copysign(1e-10, x) as the reference forms it from bits
__device__ __forceinline__ float tiny_signed(float x) {
  return __uint_as_float((__float_as_uint(1e-10f) & 0x7fffffffu) | (__float_as_uint(x) & 0x80000000u));
}
__device__ __forceinline__ float radbc_speed(float dx, float a, float b, float foo, float dt) {
  return dcr(dx * (a - b), dt * (tiny_signed(foo) + foo));
}

// radbc_ew.wgsl: per row j < ny, the level mean of the clipped radiation speeds of u at
// the west (i = 1) and east (i = nx - 1) faces.  One thread per row; the level loop is
// sequential as in the reference (the sum's rounding order).
__global__ void k_radbc_ew(KArgs A) {
  TE_K3
  const float *TE_R ua = A.p[1], *TE_R u3d = A.p[2], *TE_R hm = A.p[30];
  const float dt = A.f[3];
  float *TE_R radbcw = A.p[4], *TE_R radbce = A.p[5];
  const int j = tx;
  if (j >= g.ny) return;
  const float umax = 350.0f;
  const float dxw = dcr(dcr(1.0f, g.rdx), hm_uf(g, hm, 1));
  const float dxe = dcr(dcr(1.0f, g.rdx), hm_uf(g, hm, g.nx - 1));
  float avgw = 0.0f, avge = 0.0f;
  for (int k = 0; k < g.nz; k++) {
    const int c1 = gidx(g, 1, j, k), c2 = gidx(g, 2, j, k);
    float foo = ua[c2] - ua[c1];
    float cbcw = radbc_speed(dxw, ua[c1], u3d[c1], foo, dt);
    cbcw = wmax(wmin(cbcw, 0.0f), -umax);
    avgw = avgw + cbcw;
    const int ce = gidx(g, g.nx - 1, j, k), ce2 = gidx(g, g.nx - 2, j, k);
    foo = ua[ce] - ua[ce2];
    float cbce = radbc_speed(dxe, ua[ce], u3d[ce], foo, dt);
    cbce = wmin(wmax(cbce, 0.0f), umax);
    avge = avge + cbce;
  }
  radbcw[j] = dcr(avgw, (float)g.nz);
  radbce[j] = dcr(avge, (float)g.nz);
}
#ifndef TE_KERNELS_FAST
TE_LAUNCH3(radbc_ew)
#endif

// radbc_ns.wgsl: the same for v at the south (j = 1) and north (j = ny - 1) faces
__global__ void k_radbc_ns(KArgs A) {
  TE_K3
  const float *TE_R va = A.p[1], *TE_R v3d = A.p[2], *TE_R hm = A.p[30];
  const float dt = A.f[3];
  float *TE_R radbcs = A.p[4], *TE_R radbcn = A.p[5];
  const int i = tx;
  if (i >= g.nx) return;
  const float umax = 350.0f;
  const float dys = dcr(dcr(1.0f, g.rdy), hm_vf(g, hm, 1));
  const float dyn = dcr(dcr(1.0f, g.rdy), hm_vf(g, hm, g.ny - 1));
  float avgs = 0.0f, avgn = 0.0f;
  for (int k = 0; k < g.nz; k++) {
    const int c1 = gidx(g, i, 1, k), c2 = gidx(g, i, 2, k);
    float foo = va[c2] - va[c1];
    float cbcs = radbc_speed(dys, va[c1], v3d[c1], foo, dt);
    cbcs = wmax(wmin(cbcs, 0.0f), -umax);
    avgs = avgs + cbcs;
    const int cn = gidx(g, i, g.ny - 1, k), cn2 = gidx(g, i, g.ny - 2, k);
    foo = va[cn] - va[cn2];
    float cbcn = radbc_speed(dyn, va[cn], v3d[cn], foo, dt);
    cbcn = wmin(wmax(cbcn, 0.0f), umax);
    avgn = avgn + cbcn;
  }
  radbcs[i] = dcr(avgs, (float)g.nz);
  radbcn[i] = dcr(avgn, (float)g.nz);
}
#ifndef TE_KERNELS_FAST
TE_LAUNCH3(radbc_ns)
#endif

enum { kLineWarps = 8 };

#ifdef TE_KERNELS_FAST
// Line sums in the __restrict__ build: a warp per line.  Its lanes evaluate the terms of 32
// consecutive levels (or columns) at a time, and every lane adds them in the reference's
// order, taking each term from the lane that computed it (__shfl_sync), so the sum is the
// one-thread-per-line kernel's; those kernels ran 40-4800 threads.

// radbc_ew (NS 0: line j, the u columns i = 1, 2 and nx - 1, nx - 2) and radbc_ns (NS 1:
// line i, the v rows j = 1, 2 and ny - 1, ny - 2)
template <int NS>
__global__ void __launch_bounds__(32 * kLineWarps) k_radbc_warp(KArgs A) {
  const Dims& g = A.g;
  const int lane = threadIdx.x & 31, line = blockIdx.x * kLineWarps + (threadIdx.x >> 5);
  if (line >= A.gx || A.gy <= 0 || A.gz <= 0 || line >= (NS ? g.nx : g.ny)) return;
  const float *TE_R a3 = A.p[1], *TE_R b3 = A.p[2], *TE_R hm = A.p[30];
  const float dt = A.f[3];
  const float umax = 350.0f;
  const float d0 = NS ? dcr(dcr(1.0f, g.rdy), hm_vf(g, hm, 1)) : dcr(dcr(1.0f, g.rdx), hm_uf(g, hm, 1));
  const float d1 = NS ? dcr(dcr(1.0f, g.rdy), hm_vf(g, hm, g.ny - 1)) : dcr(dcr(1.0f, g.rdx), hm_uf(g, hm, g.nx - 1));
  float avg0 = 0.0f, avg1 = 0.0f;
  for (int k0 = 0; k0 < g.nz; k0 += 32) {
    const int k = k0 + lane;
    float t0 = 0.0f, t1 = 0.0f;
    if (k < g.nz) {
      const int c1 = NS ? gidx(g, line, 1, k) : gidx(g, 1, line, k), c2 = NS ? gidx(g, line, 2, k) : gidx(g, 2, line, k);
      t0 = radbc_speed(d0, a3[c1], b3[c1], a3[c2] - a3[c1], dt);
      t0 = wmax(wmin(t0, 0.0f), -umax);
      const int e1 = NS ? gidx(g, line, g.ny - 1, k) : gidx(g, g.nx - 1, line, k);
      const int e2 = NS ? gidx(g, line, g.ny - 2, k) : gidx(g, g.nx - 2, line, k);
      t1 = radbc_speed(d1, a3[e1], b3[e1], a3[e1] - a3[e2], dt);
      t1 = wmin(wmax(t1, 0.0f), umax);
    }
    const int n = min(32, g.nz - k0);
    for (int l = 0; l < n; l++) {
      avg0 = avg0 + __shfl_sync(0xffffffffu, t0, l);
      avg1 = avg1 + __shfl_sync(0xffffffffu, t1, l);
    }
  }
  if (lane == 0) {
    A.p[4][line] = dcr(avg0, (float)g.nz);
    A.p[5][line] = dcr(avg1, (float)g.nz);
  }
}
static void launch_radbc_ew(const KArgs& A, cudaStream_t s) {
  if (A.gx > 0) launch_kernel(k_radbc_warp<0>, dim3((A.gx + kLineWarps - 1) / kLineWarps), dim3(32 * kLineWarps), 0, s, A);
}
static void launch_radbc_ns(const KArgs& A, cudaStream_t s) {
  if (A.gx > 0) launch_kernel(k_radbc_warp<1>, dim3((A.gx + kLineWarps - 1) / kLineWarps), dim3(32 * kLineWarps), 0, s, A);
}
#endif

// openbc_uv_tendency.wgsl: on open x boundaries the u faces i = 0 and i = nx, on open y
// boundaries the v faces j = 0 and j = ny, advance by the radiation term
__global__ void k_openbc_uv_tendency(KArgs A) {
  TE_K3
  const Acoustic a = A.a;
  const float *TE_R radbcw = A.p[2], *TE_R radbce = A.p[3], *TE_R radbcs = A.p[4], *TE_R radbcn = A.p[5];
  const float *TE_R uten = A.p[6], *TE_R vten = A.p[7], *TE_R hm = A.p[30];
  float *TE_R u3d = A.p[8], *TE_R v3d = A.p[9];
  const int openx = A.iv[10], openy = A.iv2[10];
  const int n = tx, k = ty;
  if (k >= g.nz) return;
  if (openx != 0 && n < g.ny) {
    const int j = n, cw = gidx(g, 0, j, k);
    u3d[cw] = fmaf(a.dts, fmaf(((-radbcw[j]) * (u3d[cw + 1] - u3d[cw])) * g.rdx, hm_uh(g, hm, 0), uten[cw]), u3d[cw]);
    const int ce = gidx(g, g.nx, j, k);
    u3d[ce] = fmaf(a.dts, fmaf(((-radbce[j]) * (u3d[ce] - u3d[ce - 1])) * g.rdx, hm_uh(g, hm, g.nx - 1), uten[ce]),
                   u3d[ce]);
  }
  if (openy != 0 && n < g.nx) {
    const int i = n, sj = g.sJ, cs = gidx(g, i, 0, k);
    v3d[cs] = fmaf(a.dts, fmaf(((-radbcs[i]) * (v3d[cs + sj] - v3d[cs])) * g.rdy, hm_vh(g, hm, 0), vten[cs]), v3d[cs]);
    const int cn = gidx(g, i, g.ny, k);
    v3d[cn] = fmaf(a.dts, fmaf(((-radbcn[i]) * (v3d[cn] - v3d[cn - sj])) * g.rdy, hm_vh(g, hm, g.ny - 1), vten[cn]),
                   v3d[cn]);
  }
}
TE_LAUNCH3(openbc_uv_tendency)

// ------------------------------------------------------- turbulence bookkeeping

// turb_zero.wgsl: zero f[i + strideJ (j + strideK k)] for i < strideJ, j < strideK and
// k <= nz + 1 (the reference's range, one level above a field's nz + 1)
__global__ void k_turb_zero(KArgs A) {
  TE_K3
  float* TE_R f = A.p[1];
  if (tx >= g.sJ || ty >= g.sK || tz > g.nz + 1) return;
  f[tx + g.sJ * (ty + g.sK * tz)] = 0.0f;
}
TE_LAUNCH3(turb_zero)

// turb_add_tendency.wgsl: dst = fma(scale, src, dst) over the whole field
__global__ void k_turb_add_tendency(KArgs A) {
  TE_K3
  const float* TE_R src = A.p[1];
  float* TE_R dst = A.p[2];
  TE_WHOLE(k <= g.nz)
  dst[c] = fmaf(A.f[3], src[c], dst[c]);
}
TE_LAUNCH3(turb_add_tendency)

// turb_scalar_flux_h.wgsl: horizontal subgrid scalar fluxes at the x and y faces
__global__ void k_turb_scalar_flux_h(KArgs A) {
  TE_K3
  const float *TE_R s = A.p[1], *TE_R rho = A.p[2], *TE_R khh = A.p[3], *TE_R hm = A.p[30];
  const float leNum = A.f[4];
  float *TE_R fx = A.p[5], *TE_R fy = A.p[6];
  const int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k), sj = g.sJ, sk = g.sJ * g.sK;
  fx[c] = ((((((-0.125f) * (rho[c] + rho[c - 1])) * leNum) * ((khh[c] + khh[c - 1]) + (khh[c + sk] + khh[c - 1 + sk]))) *
            (s[c] - s[c - 1])) * g.rdx) * hm_uf(g, hm, i);
  fy[c] = ((((((-0.125f) * (rho[c] + rho[c - sj])) * leNum) * ((khh[c] + khh[c - sj]) + (khh[c + sk] + khh[c - sj + sk]))) *
            (s[c] - s[c - sj])) * g.rdy) * hm_vf(g, hm, j);
}
TE_LAUNCH3(turb_scalar_flux_h)

// turb_openbc_flux.wgsl: edge fluxes copy their inner neighbours on open boundaries
__global__ void k_turb_openbc_flux(KArgs A) {
  TE_K3
  float *TE_R fx = A.p[1], *TE_R fy = A.p[2];
  const int openx = A.iv[3], openy = A.iv2[3];
  const int n = tx, k = ty;
  if (k > g.nz) return;
  if (openx != 0 && n <= g.ny) {
    fx[gidx(g, 0, n, k)] = fx[gidx(g, 1, n, k)];
    fx[gidx(g, g.nx, n, k)] = fx[gidx(g, g.nx - 1, n, k)];
  }
  if (openy != 0 && n <= g.nx) {
    fy[gidx(g, n, 0, k)] = fy[gidx(g, n, 1, k)];
    fy[gidx(g, n, g.ny, k)] = fy[gidx(g, n, g.ny - 1, k)];
  }
}
TE_LAUNCH3(turb_openbc_flux)

// turb_openbc_stress_x.wgsl / _y.wgsl: edge stresses copy their inner neighbours
__global__ void k_turb_openbc_stress_x(KArgs A) {
  TE_K3
  float *TE_R s11 = A.p[1], *TE_R s12 = A.p[2];
  const int j = tx - 1, k = ty;
  if (j > g.ny || k >= g.nz) return;
  s11[gidx(g, -1, j, k)] = s11[gidx(g, 0, j, k)];
  s11[gidx(g, g.nx, j, k)] = s11[gidx(g, g.nx - 1, j, k)];
  if (j >= 0) {
    s12[gidx(g, 0, j, k)] = s12[gidx(g, 1, j, k)];
    s12[gidx(g, g.nx, j, k)] = s12[gidx(g, g.nx - 1, j, k)];
  }
}
TE_LAUNCH3(turb_openbc_stress_x)

__global__ void k_turb_openbc_stress_y(KArgs A) {
  TE_K3
  float *TE_R s22 = A.p[1], *TE_R s12 = A.p[2];
  const int i = tx - 1, k = ty;
  if (i > g.nx || k >= g.nz) return;
  s22[gidx(g, i, -1, k)] = s22[gidx(g, i, 0, k)];
  s22[gidx(g, i, g.ny, k)] = s22[gidx(g, i, g.ny - 1, k)];
  if (i >= 0) {
    s12[gidx(g, i, 0, k)] = s12[gidx(g, i, 1, k)];
    s12[gidx(g, i, g.ny, k)] = s12[gidx(g, i, g.ny - 1, k)];
  }
}
TE_LAUNCH3(turb_openbc_stress_y)

// tke_advance.wgsl: tke = fma(dttmp, tketen, tkea), flushed to 0 below 1e-10
__global__ void k_tke_advance(KArgs A) {
  TE_K3
  const float *TE_R tkea = A.p[1], *TE_R tketen = A.p[2];
  float* TE_R tke = A.p[4];
  const int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  const int c = gidx(g, i, j, k);
  const float v = fmaf(A.f[3], tketen[c], tkea[c]);
  tke[c] = v < 1e-10f ? 0.0f : v;
}
TE_LAUNCH3(tke_advance)

// tke_sources.wgsl: tketen = fma(-khv, nm, -dissten) + epst
__global__ void k_tke_sources(KArgs A) {
  TE_K3
  const float *TE_R khv = A.p[1], *TE_R nm = A.p[2], *TE_R dissten = A.p[3], *TE_R epst = A.p[4];
  float* TE_R tketen = A.p[5];
  const int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  const int c = gidx(g, i, j, k);
  tketen[c] = fmaf(-khv[c], nm[c], -dissten[c]) + epst[c];
}
TE_LAUNCH3(tke_sources)

// tke_flux_h.wgsl: horizontal TKE fluxes at the x and y faces of w levels 1..nz-1
__global__ void k_tke_flux_h(KArgs A) {
  TE_K3
  const float *TE_R t = A.p[1], *TE_R rf = A.p[2], *TE_R kmh = A.p[3], *TE_R hm = A.p[30];
  float *TE_R fx = A.p[4], *TE_R fy = A.p[5];
  const int i = tx, j = ty, k = tz + 1;
  if (i > g.nx || j > g.ny || k > g.nz - 1) return;
  const int sj = g.sJ, c = gidx(g, i, j, k);
  fx[c] = ((((((-0.25f) * (rf[c] + rf[c - 1])) * 2.0f) * (kmh[c] + kmh[c - 1])) * (t[c] - t[c - 1])) * g.rdx) *
          hm_uf(g, hm, i);
  fy[c] = ((((((-0.25f) * (rf[c] + rf[c - sj])) * 2.0f) * (kmh[c] + kmh[c - sj])) * (t[c] - t[c - sj])) * g.rdy) *
          hm_vf(g, hm, j);
}
TE_LAUNCH3(tke_flux_h)

// Column kernels (one thread per (i, j) column, columns of a warp adjacent in i) share
// the acoustic solve's launch shape.
static void launch_columns(void (*k)(KArgs), const KArgs& A, cudaStream_t s) {
  dim3 b(32, 4, 1);
  dim3 gr((A.gx + 31) / 32, (A.gy + 3) / 4, 1);
  launch_kernel(k, dim3(gr), dim3(b), 0, s, A);
}
#define TE_LAUNCH_COLUMNS(name) \
  static void launch_##name(const KArgs& A, cudaStream_t s) { launch_columns(k_##name, A, s); }

// mp_pdefq.wgsl: per column, q below rmax set to 0 and the column rescaled so that
// sum rho q keeps its value before the clip ((t1 + 1e-20) / (t2 + 1e-20), 1 if negative)
__global__ void k_mp_pdefq(KArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const Dims& g = A.g;
  if (i >= A.gx || j >= A.gy || i >= g.nx || j >= g.ny) return;
  const float* TE_R rho = A.p[1];
  float* TE_R q = A.p[2];
  const float rmax = A.f[3];
  const int sk = g.sJ * g.sK, base = gidx(g, i, j, 0);
  float t1 = 0.0f, t2 = 0.0f;
  for (int k = 0; k < g.nz; k++) {
    const int c = base + k * sk;
    const float r = rho[c];
    float v = q[c];
    t1 = fmaf(r, v, t1);
    if (v < rmax) {
      v = 0.0f;
      q[c] = 0.0f;
    }
    t2 = fmaf(r, v, t2);
  }
  float t3 = dcr(t1 + 1e-20f, t2 + 1e-20f);
  if (t3 < 0.0f) t3 = 1.0f;
  for (int k = 0; k < g.nz; k++) q[base + k * sk] = q[base + k * sk] * t3;
}
#ifndef TE_KERNELS_FAST
TE_LAUNCH_COLUMNS(mp_pdefq)
#endif

// turb_scalar_vert_implicit.wgsl: subgrid tendency of a scalar s.  sten gains
// ((fx, fy divergence) + turbz) rr at every level; turbz is the explicit vertical flux
// divergence (explicitZ), or rho (s_new - s) / dt with s_new from a per-column Thomas
// solve of the implicit vertical diffusion (cA, cB as the forward sweep; cB ends as s_new).
struct TsviCol {
  const Dims& g;
  int i, j, base, sk, useFlux, bcturbs;
  const float *TE_R s, *TE_R khv, *TE_R mf, *TE_R rf, *TE_R sflux, *TE_R fx, *TE_R fy, *TE_R hm, *TE_R rr;
  float* TE_R sten;
  const float* wall;
  // vertical flux at w level kf (lam_1 / lam_2 of the reference kernel)
  __device__ float vflux(int kf) const {
    const int c = base + kf * sk;
    if (kf == 0 || kf == g.nz) {
      const int inner = kf == 0 ? 1 : g.nz - 1;
      if (wall[3] == 0.0f) {
        if (kf == 0 && useFlux != 0) return sflux[base] * rf[c];
        if (bcturbs != 2) return 0.0f;
        const int cc = base + inner * sk;
        return ((((-khv[cc]) * (s[cc] - s[cc - sk])) * g.rdz) * mf[inner]) * rf[cc];
      }
      if (wall[3] == 2.0f) return (wall[0] * (kf == 0 ? wall[1] : wall[2])) * rf[c];
      if (kf == 0) return (((((-wall[0]) * 2.0f) * (s[c] - wall[1])) * g.rdz) * mf[0]) * rf[c];
      return (((((-wall[0]) * 2.0f) * (wall[2] - s[base + (g.nz - 1) * sk])) * g.rdz) * mf[g.nz]) * rf[c];
    }
    return ((((-khv[c]) * (s[c] - s[c - sk])) * g.rdz) * mf[kf]) * rf[c];
  }
  // sten += ((fx, fy divergence) + turbz) rr at point c (lam_5)
  __device__ void tend(int c, float turbz) const {
    const float h = ((-(fx[c + 1] - fx[c])) * g.rdx) * hm_uh(g, hm, i) + ((-(fy[c + g.sJ] - fy[c])) * g.rdy) * hm_vh(g, hm, j);
    sten[c] = fmaf(h + turbz, rr[c], sten[c]);
  }
};

__global__ void k_turb_scalar_vert_implicit(KArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const Dims& g = A.g;
  if (i >= A.gx || j >= A.gy || i >= g.nx || j >= g.ny) return;
  const float *TE_R s = A.p[1], *TE_R rho = A.p[2], *TE_R rr = A.p[3], *TE_R rf = A.p[4], *TE_R khv = A.p[5];
  const float *TE_R mh = A.p[6], *TE_R mf = A.p[7];
  float *TE_R cA = A.p[11], *TE_R cB = A.p[12];
  const float dt = A.f[10];
  const int sk = g.sJ * g.sK, base = gidx(g, i, j, 0);
  const TsviCol col{g, i, j, base, sk, A.iv[15], A.iv[18], s, khv, mf, rf, A.p[14], A.p[8], A.p[9], A.p[30], rr, A.p[13], A.sw[0]};
  if (A.iv[16] != 0) {
    float below = col.vflux(0);
    for (int k = 0; k < g.nz; k++) {
      const float above = col.vflux(k + 1);
      col.tend(base + k * sk, ((-(above - below)) * g.rdz) * mh[k]);
      below = above;
    }
    return;
  }
  // lam_3 (coefficient of the face above level k) and lam_4 (the face below)
  auto lam3 = [&](int k) {
    const int c = base + k * sk;
    return (((khv[c + sk] * mf[k + 1]) * rf[c + sk]) * mh[k]) * rr[c];
  };
  auto lam4 = [&](int k) {
    const int c = base + k * sk;
    return (((khv[c] * mf[k]) * rf[c]) * mh[k]) * rr[c];
  };
  const float tema = ((-dt) * g.rdz) * g.rdz, rdt = dcr(1.0f, dt), temc = dt * g.rdz;
  const int useFlux = A.iv[15], bcturbs = A.iv[18];
  {
    const float cfc = tema * lam3(0), t = dcr(1.0f, 1.0f - cfc);
    cA[base] = (-cfc) * t;
    float cfd = s[base];
    if (useFlux != 0 || bcturbs == 2) {
      const int c1 = base + sk;
      const float dumz = useFlux != 0 ? A.p[14][base] * rf[base] : ((((-khv[c1]) * (s[c1] - s[base])) * g.rdz) * mf[1]) * rf[c1];
      cfd = fmaf((temc * dumz) * mh[0], rr[base], s[base]);
    }
    cB[base] = cfd * t;
  }
  for (int k = 1; k < g.nz - 1; k++) {
    const int c = base + k * sk;
    const float cfa = tema * lam4(k), cfc = tema * lam3(k), cfb = (1.0f - cfa) - cfc;
    const float t = dcr(1.0f, fmaf(cfa, cA[c - sk], cfb));
    cA[c] = (-cfc) * t;
    cB[c] = fmaf(-cfa, cB[c - sk], s[c]) * t;
  }
  {
    const int kt = g.nz - 1, ct = base + kt * sk;
    const float cfa = tema * lam4(kt), t = dcr(1.0f, fmaf(cfa, cA[ct - sk], 1.0f - cfa));
    float cfd = s[ct];
    if (bcturbs == 2) {
      const float dumz = ((((-khv[ct]) * (s[ct] - s[ct - sk])) * g.rdz) * mf[kt]) * rf[ct];
      cfd = fmaf(-((temc * dumz) * mh[kt]), rr[ct], s[ct]);
    }
    const float snew = fmaf(-cfa, cB[ct - sk], cfd) * t;
    cB[ct] = snew;
    col.tend(ct, (rho[ct] * (snew - s[ct])) * rdt);
  }
  for (int k = g.nz - 2; k >= 0; k--) {
    const int c = base + k * sk;
    const float snew = fmaf(cA[c], cB[c + sk], cB[c]);
    cB[c] = snew;
    col.tend(c, (rho[c] * (snew - s[c])) * rdt);
  }
}
#ifdef TE_KERNELS_FAST
// Column solves in the __restrict__ build (no bound region overlaps another): a block per
// 32 columns.  Its 8 warps build the tridiagonal rows of all levels in parallel (warp w:
// levels w, w + 8, ...; lanes on consecutive columns), one warp runs the Thomas sweep and
// back-substitution of the 32 columns from shared memory (coop_thomas), and the 8 warps
// then form the tendencies level-parallel.  Every value is computed by the operations of
// the one-thread-per-column kernel, and the recurrence in its order, so every written word
// is the same; the one-thread-per-column kernels walk 40-80 dependent levels per column.
enum { kCoopCols = 32, kCoopWarps = 8 };

// Thomas sweep over levels klo..khi of a block's 32 columns.  Row k: sA = sub-diagonal
// coefficient (k > klo), sC = super-diagonal (k < khi), sD = right-hand side; the diagonal
// is 1 - sA - sC as the reference forms it.  Writes the forward coefficient cA (levels
// klo..khi-1) and the solution into cB (levels klo..khi), in memory and in scA / scB,
// which may be sC / sD themselves (each row is read before its slot is rewritten).
__device__ __forceinline__ void coop_thomas(const float* sA, const float* sC, const float* sD, float* scA, float* scB,
                                            int klo, int khi, int lane, float* TE_R cA, float* TE_R cB, int base, int sk) {
  int e = klo * kCoopCols + lane;
  float t = dcr(1.0f, 1.0f - sC[e]);
  float a = (-sC[e]) * t, b = sD[e] * t;
  scA[e] = a;
  scB[e] = b;
  cA[base + klo * sk] = a;
  for (int k = klo + 1; k < khi; k++) {
    e = k * kCoopCols + lane;
    const float cfa = sA[e], cfc = sC[e];
    t = dcr(1.0f, fmaf(cfa, a, (1.0f - cfa) - cfc));
    a = (-cfc) * t;
    b = fmaf(-cfa, b, sD[e]) * t;
    scA[e] = a;
    scB[e] = b;
    cA[base + k * sk] = a;
  }
  e = khi * kCoopCols + lane;
  const float cfa = sA[e];
  t = dcr(1.0f, fmaf(cfa, a, 1.0f - cfa));
  b = fmaf(-cfa, b, sD[e]) * t;
  scB[e] = b;
  cB[base + khi * sk] = b;
  for (int k = khi - 1; k >= klo; k--) {
    e = k * kCoopCols + lane;
    b = fmaf(scA[e], b, scB[e]);
    scB[e] = b;
    cB[base + k * sk] = b;
  }
}

struct CoopCol {
  int lane, wq, i, j, base, sk;
  bool on;
  float *sA, *sC, *sD, *scA, *scB;
};

// the block's column (lane): cx x cy columns of the dispatch, x fastest
__device__ __forceinline__ CoopCol coop_col(const KArgs& A, float* smem, int cx, int cy) {
  CoopCol q;
  const Dims& g = A.g;
  const int nz = g.nz;
  q.lane = threadIdx.x & 31;
  q.wq = threadIdx.x >> 5;
  const int col = blockIdx.x * kCoopCols + q.lane;
  q.i = col % cx;
  q.j = col / cx;
  q.on = col < cx * cy && q.i < A.gx && q.j < A.gy;
  q.sk = g.sJ * g.sK;
  q.base = gidx(g, q.on ? q.i : 0, q.on ? q.j : 0, 0);
  q.sA = smem;
  q.sC = smem + nz * kCoopCols;
  q.sD = smem + 2 * nz * kCoopCols;
  q.scA = q.sC;  // the forward sweep overwrites each row's sC / sD after reading them
  q.scB = q.sD;
  return q;
}

static size_t coop_bytes(int nz) { return (size_t)3 * nz * kCoopCols * sizeof(float); }

template <class K>
static void launch_coop(K kernel, const KArgs& A, cudaStream_t st, int cx, int cy) {
  const size_t bytes = coop_bytes(A.g.nz);
  if (A.gx <= 0 || A.gy <= 0 || A.gz <= 0) return;
  if (opt_in_smem((const void*)kernel, bytes) != cudaSuccess) return;  // error left pending for the player
  launch_kernel(kernel, dim3((cx * cy + kCoopCols - 1) / kCoopCols), dim3(kCoopCols * kCoopWarps), bytes, st, A);
}

// mp_pdefq: the column sums run by one warp from shared memory in the reference's order,
// the clipped and rescaled q stored level-parallel
__global__ void __launch_bounds__(kCoopCols * kCoopWarps) k_pdefq_coop(KArgs A) {
  extern __shared__ float tsm[];
  const Dims& g = A.g;
  const int nz = g.nz;
  const CoopCol cq = coop_col(A, tsm, g.nx, g.ny);
  const float* TE_R rho = A.p[1];
  float* TE_R q = A.p[2];
  const float rmax = A.f[3];
  if (cq.on)
    for (int k = cq.wq; k < nz; k += kCoopWarps) {
      const int c = cq.base + k * cq.sk, e = k * kCoopCols + cq.lane;
      cq.sA[e] = rho[c];
      cq.sC[e] = q[c];
    }
  __syncthreads();
  if (cq.wq == 0 && cq.on) {
    float t1 = 0.0f, t2 = 0.0f;
    for (int k = 0; k < nz; k++) {
      const int e = k * kCoopCols + cq.lane;
      const float r = cq.sA[e];
      float v = cq.sC[e];
      t1 = fmaf(r, v, t1);
      if (v < rmax) {
        v = 0.0f;
        cq.sC[e] = 0.0f;
      }
      t2 = fmaf(r, v, t2);
    }
    float t3 = dcr(t1 + 1e-20f, t2 + 1e-20f);
    if (t3 < 0.0f) t3 = 1.0f;
    cq.sD[cq.lane] = t3;
  }
  __syncthreads();
  if (!cq.on) return;
  const float t3 = cq.sD[cq.lane];
  for (int k = cq.wq; k < nz; k += kCoopWarps) q[cq.base + k * cq.sk] = cq.sC[k * kCoopCols + cq.lane] * t3;
}

static void launch_mp_pdefq(const KArgs& A, cudaStream_t st) {
  if (A.g.nz < 1 || coop_bytes(A.g.nz) > 200 * 1024) {
    launch_columns(k_mp_pdefq, A, st);
    return;
  }
  launch_coop(k_pdefq_coop, A, st, A.g.nx, A.g.ny);
}

// acoustic_w_solve: the rows (aa, bb, cc, dd of every w level) level-parallel, the
// Thomas sweep and back-substitution of the 32 columns by one warp from shared memory
__global__ void __launch_bounds__(kCoopCols * kCoopWarps) k_wsolve_coop(KArgs A) {
  extern __shared__ float tsm[];
  const Dims& g = A.g;
  const int nz = g.nz;
  const CoopCol q = coop_col(A, tsm, g.nx, g.ny);
  float* sB = tsm + 3 * nz * kCoopCols;
  const Acoustic a = A.a;
  const float asq = a.alph * a.alph;
  const float *TE_R pk1 = A.p[2], *TE_R pk2 = A.p[3], *TE_R qk = A.p[4], *TE_R mm = A.p[5], *TE_R fpk = A.p[6];
  const float *TE_R wten = A.p[7], *TE_R pp3d = A.p[8];
  float *TE_R w = A.p[9], *TE_R cA = A.p[10], *TE_R cB = A.p[11];
  const int sk = q.sk, base = q.base;
  if (q.on)
#pragma unroll 2
    for (int k = 1 + q.wq; k <= nz - 1; k += kCoopWarps) {
      const int c = base + k * sk, cm = c - sk, e = k * kCoopCols + q.lane;
      const float m = mm[c];
      q.sA[e] = (-asq) * (m * (pk1[cm] + qk[cm]));
      q.sC[e] = (-asq) * ((-m) * (pk2[c] - qk[c]));
      sB[e] = fmaf(-asq, m * ((-(pk1[c] + qk[c])) + (pk2[cm] - qk[cm])), 1.0f);
      const float fw = fmaf(a.dts, wten[c], a.beta * ((-m) * (pp3d[c] - pp3d[cm])));
      q.sD[e] = fmaf(a.alph, (-m) * ((pp3d[c] + fpk[c]) - (pp3d[cm] + fpk[cm])), w[c] + fw);
    }
  __syncthreads();
  if (q.wq != 0 || !q.on) return;
  const int ln = q.lane;
  w[base] = 0.0f;
  w[base + nz * sk] = 0.0f;
  int e = kCoopCols + ln;
  float r = dcr(1.0f, sB[e]);
  float ca = (-q.sC[e]) * r, cb = q.sD[e] * r;
  q.scA[e] = ca;
  q.scB[e] = cb;
  cA[base + sk] = ca;
  cB[base + sk] = cb;
  for (int k = 2; k < nz - 1; k++) {
    e = k * kCoopCols + ln;
    const float aa = q.sA[e];
    r = dcr(1.0f, fmaf(aa, ca, sB[e]));
    ca = (-q.sC[e]) * r;
    cb = fmaf(-aa, cb, q.sD[e]) * r;
    q.scA[e] = ca;
    q.scB[e] = cb;
    cA[base + k * sk] = ca;
    cB[base + k * sk] = cb;
  }
  e = (nz - 1) * kCoopCols + ln;
  const float aa = q.sA[e];
  r = dcr(1.0f, fmaf(aa, ca, sB[e]));
  float wk = fmaf(-aa, cb, q.sD[e]) * r;
  w[base + (nz - 1) * sk] = wk;
  for (int k = nz - 2; k >= 1; k--) {
    e = k * kCoopCols + ln;
    wk = fmaf(q.scA[e], wk, q.scB[e]);
    w[base + k * sk] = wk;
  }
}

static void launch_acoustic_w_solve(const KArgs& A, cudaStream_t st) {
  const int nz = A.g.nz;
  const size_t bytes = (size_t)4 * nz * kCoopCols * sizeof(float);
  if (nz < 3 || bytes > 200 * 1024) {
    launch_acoustic_w_solve_columns(A, st);
    return;
  }
  if (A.gx <= 0 || A.gy <= 0) return;
  if (opt_in_smem((const void*)k_wsolve_coop, bytes) != cudaSuccess) return;  // error left pending
  launch_kernel(k_wsolve_coop, dim3((A.g.nx * A.g.ny + kCoopCols - 1) / kCoopCols), dim3(kCoopCols * kCoopWarps), bytes, st, A);
}

// turb_scalar_vert_implicit, implicit branch
__global__ void __launch_bounds__(kCoopCols * kCoopWarps) k_tsvi_coop(KArgs A) {
  extern __shared__ float tsm[];
  const Dims& g = A.g;
  const int nz = g.nz;
  const CoopCol q = coop_col(A, tsm, g.nx, g.ny);
  const int sk = q.sk, base = q.base;
  const float *TE_R s = A.p[1], *TE_R rho = A.p[2], *TE_R rr = A.p[3], *TE_R rf = A.p[4], *TE_R khv = A.p[5];
  const float *TE_R mh = A.p[6], *TE_R mf = A.p[7];
  const float dt = A.f[10];
  const int useFlux = A.iv[15], bcturbs = A.iv[18];
  const float tema = ((-dt) * g.rdz) * g.rdz, temc = dt * g.rdz;
  if (q.on)
#pragma unroll 2
    for (int k = q.wq; k < nz; k += kCoopWarps) {
      const int c = base + k * sk, e = k * kCoopCols + q.lane;
      if (k < nz - 1) q.sC[e] = tema * ((((khv[c + sk] * mf[k + 1]) * rf[c + sk]) * mh[k]) * rr[c]);
      if (k > 0) q.sA[e] = tema * ((((khv[c] * mf[k]) * rf[c]) * mh[k]) * rr[c]);
      float d = s[c];
      if (k == 0 && (useFlux != 0 || bcturbs == 2)) {
        const int c1 = base + sk;
        const float dumz = useFlux != 0 ? A.p[14][base] * rf[base] : ((((-khv[c1]) * (s[c1] - s[base])) * g.rdz) * mf[1]) * rf[c1];
        d = fmaf((temc * dumz) * mh[0], rr[base], s[base]);
      } else if (k == nz - 1 && bcturbs == 2) {
        const float dumz = ((((-khv[c]) * (s[c] - s[c - sk])) * g.rdz) * mf[k]) * rf[c];
        d = fmaf(-((temc * dumz) * mh[k]), rr[c], s[c]);
      }
      q.sD[e] = d;
    }
  __syncthreads();
  if (q.wq == 0 && q.on) coop_thomas(q.sA, q.sC, q.sD, q.scA, q.scB, 0, nz - 1, q.lane, A.p[11], A.p[12], base, sk);
  __syncthreads();
  if (!q.on) return;
  const float rdt = dcr(1.0f, dt);
  const float uh = hm_uh(g, A.p[30], q.i), vh = hm_vh(g, A.p[30], q.j);
  const float *TE_R fx = A.p[8], *TE_R fy = A.p[9];
  float* TE_R sten = A.p[13];
  for (int k = q.wq; k < nz; k += kCoopWarps) {
    const int c = base + k * sk;
    const float snew = q.scB[k * kCoopCols + q.lane];
    const float h = ((-(fx[c + 1] - fx[c])) * g.rdx) * uh + ((-(fy[c + g.sJ] - fy[c])) * g.rdy) * vh;
    sten[c] = fmaf(h + (rho[c] * (snew - s[c])) * rdt, rr[c], sten[c]);
  }
}

static void launch_turb_scalar_vert_implicit(const KArgs& A, cudaStream_t st) {
  if (A.iv[16] != 0 || A.g.nz < 2 || coop_bytes(A.g.nz) > 200 * 1024) {  // explicit branch, degenerate columns
    launch_columns(k_turb_scalar_vert_implicit, A, st);
    return;
  }
  launch_coop(k_tsvi_coop, A, st, A.g.nx, A.g.ny);
}
#else
TE_LAUNCH_COLUMNS(turb_scalar_vert_implicit)
#endif

// rayleigh_damping.wgsl: -rdalpha tau (phi - phi_ref) for u, v, th (profiles, or level
// averages when toAverage) and -rdalpha tauf w, tauf raised to the lateral sponge
__global__ void k_rayleigh_damping(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz;
  if (i > g.nx || j > g.ny || k > g.nz) return;
  const float *TE_R u = A.p[1], *TE_R v = A.p[2], *TE_R w = A.p[3], *TE_R th = A.p[4];
  float *TE_R uten = A.p[10], *TE_R vten = A.p[11], *TE_R wten = A.p[12], *TE_R thten = A.p[13];
  const float rdalpha = A.f[9];
  const int toAverage = A.iv[17];
  const int c = gidx(g, i, j, k);
  if (k < g.nz) {
    const float t = A.p[7][k];
    const float ur = toAverage != 0 ? A.p[18][k] : A.p[5][k];
    const float vr = toAverage != 0 ? A.p[18][g.nz + k] : A.p[6][k];
    if (j < g.ny) uten[c] = ((-rdalpha) * t) * (u[c] - ur);
    if (i < g.nx) vten[c] = ((-rdalpha) * t) * (v[c] - vr);
    if (i < g.nx && j < g.ny) {
      const float d = toAverage != 0 ? (A.p[19][k] - A.p[18][2 * g.nz + k]) + th[c] : th[c];
      thten[c] = ((-rdalpha) * t) * d;
    }
  }
  if (i < g.nx && j < g.ny) {
    float tf = A.p[8][k];
    if (A.iv[16] != 0 && k < g.nz) tf = wmax(wmax(tf, A.p[14][i]), A.p[15][j]);
    wten[c] = ((-rdalpha) * tf) * w[c];
  }
}
TE_LAUNCH3(rayleigh_damping)

// turb_rho_faces.wgsl: rr = 1 / rho (k < nz); rf on w levels, interior c1/c2 weights,
// bottom and top extrapolated with cgs / cgt; columns -2..nx+1, rows -2..ny+1
__global__ void k_turb_rho_faces(KArgs A) {
  TE_K3
  const int i = tx - 2, j = ty - 2, k = tz;
  if (i > g.nx + 1 || j > g.ny + 1 || k > g.nz) return;
  const float* TE_R rho = A.p[1];
  float *TE_R rr = A.p[4], *TE_R rf = A.p[5];
  const float *cgs = A.sw[0], *cgt = A.sw[1];
  const int sk = g.sJ * g.sK, c = gidx(g, i, j, k);
  if (k < g.nz) rr[c] = dcr(1.0f, rho[c]);
  float r;
  if (k == 0) {
    r = fmaf(cgs[0], rho[c], cgs[1] * rho[c + sk]);
    if (g.nz >= 3) r = fmaf(cgs[2], rho[c + 2 * sk], r);
  } else if (k == g.nz) {
    r = fmaf(cgt[0], rho[c - sk], cgt[1] * rho[c - 2 * sk]);
    if (g.nz >= 3) r = fmaf(cgt[2], rho[c - 3 * sk], r);
  } else {
    r = fmaf(A.p[2][k], rho[c - sk], A.p[3][k] * rho[c]);
  }
  rf[c] = r;
}
TE_LAUNCH3(turb_rho_faces)

// turb_def_centers.wgsl: rho-weighted strain rates s11, s22, s33 at cell centres and s12
// at the (i-1/2, j-1/2) edges; columns -1..nx+1, rows -1..ny+1
__global__ void k_turb_def_centers(KArgs A) {
  TE_K3
  const int i = tx - 1, j = ty - 1, k = tz;
  if (i > g.nx + 1 || j > g.ny + 1 || k >= g.nz) return;
  const float *TE_R u = A.p[1], *TE_R v = A.p[2], *TE_R w = A.p[3], *TE_R rho = A.p[4], *TE_R hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK, c = gidx(g, i, j, k);
  A.p[6][c] = ((rho[c] * (u[c + 1] - u[c])) * g.rdx) * hm_uh(g, hm, i);
  A.p[7][c] = ((rho[c] * (v[c + sj] - v[c])) * g.rdy) * hm_vh(g, hm, j);
  A.p[8][c] = ((rho[c] * (w[c + sk] - w[c])) * g.rdz) * A.p[5][k];
  const float rcorner = 0.25f * ((rho[c - 1 - sj] + rho[c]) + (rho[c - 1] + rho[c - sj]));
  A.p[9][c] = (0.5f * fmaf((u[c] - u[c - sj]) * g.rdy, hm_vf(g, hm, j), ((v[c] - v[c - 1]) * g.rdx) * hm_uf(g, hm, i))) * rcorner;
}
TE_LAUNCH3(turb_def_centers)

// turb_def_faces.wgsl: s13, s23 on w levels 1..nz-1 at the x and y faces
__global__ void k_turb_def_faces(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz + 1;
  if (i > g.nx + 1 || j > g.ny + 1 || k > g.nz - 1) return;
  const float *TE_R u = A.p[1], *TE_R v = A.p[2], *TE_R w = A.p[3], *TE_R rf = A.p[4], *TE_R hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK, c = gidx(g, i, j, k);
  const float mfk = 0.5f * (A.p[5][k] + A.p[5][k]);
  A.p[6][c] = ((0.5f * fmaf((w[c] - w[c - 1]) * g.rdx, hm_uf(g, hm, i), ((u[c] - u[c - sk]) * g.rdz) * mfk)) * 0.5f) * (rf[c - 1] + rf[c]);
  A.p[7][c] = ((0.5f * fmaf((w[c] - w[c - sj]) * g.rdy, hm_vf(g, hm, j), ((v[c] - v[c - sk]) * g.rdz) * mfk)) * 0.5f) * (rf[c - sj] + rf[c]);
}
TE_LAUNCH3(turb_def_faces)

// turb_def_assemble.wgsl: defv = 4 (t13 + t23) / rf^2, defh = (2 (t11 + t22 + t33) + 4 t12)
// / rf^2 on w levels 1..nz-1 (squared rates interpolated by c1/c2, edge/face averages)
__global__ void k_turb_def_assemble(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  const float *TE_R s11 = A.p[1], *TE_R s22 = A.p[2], *TE_R s33 = A.p[3], *TE_R s12 = A.p[4], *TE_R s13 = A.p[5];
  const float *TE_R s23 = A.p[6], *TE_R rf = A.p[9];
  const int sj = g.sJ, sk = g.sJ * g.sK, c = gidx(g, i, j, k);
  const float a = A.p[7][k], b = A.p[8][k];
  auto sq2 = [&](const float* s) { return fmaf(a * s[c - sk], s[c - sk], (b * s[c]) * s[c]); };
  auto pair = [&](int p, int q) { return fmaf(s12[p], s12[p], s12[q] * s12[q]); };
  const float t11 = sq2(s11), t22 = sq2(s22), t33 = sq2(s33);
  const float lo = pair(c - sk, c + 1 + sj - sk) + pair(c + sj - sk, c + 1 - sk);
  const float hi = pair(c, c + 1 + sj) + pair(c + sj, c + 1);
  const float t12 = 0.25f * fmaf(a, lo, b * hi);
  const float t13 = 0.5f * fmaf(s13[c], s13[c], s13[c + 1] * s13[c + 1]);
  const float t23 = 0.5f * fmaf(s23[c], s23[c], s23[c + sj] * s23[c + sj]);
  const float rrf = dcr(1.0f, rf[c] * rf[c]);
  A.p[10][c] = (4.0f * (t13 + t23)) * rrf;
  A.p[11][c] = fmaf(2.0f, (t11 + t22) + t33, 4.0f * t12) * rrf;
}
TE_LAUNCH3(turb_def_assemble)

// turb_gettau.wgsl: stresses t = s (kmh + kmh above) at centres, t12 by the 8-point edge
// average of kmh, t13 / t23 by the face sums of kmv (levels 1..nz-1, i, j >= 0); the
// dispatch covers columns and rows -1..n
__global__ void k_turb_gettau(KArgs A) {
  TE_K3
  const int i = tx - 1, j = ty - 1, k = tz;
  if (i > g.nx || j > g.ny || k >= g.nz) return;
  const float *TE_R kmh = A.p[1], *TE_R kmv = A.p[2];
  float *TE_R t11 = A.p[3], *TE_R t22 = A.p[4], *TE_R t33 = A.p[5], *TE_R t12 = A.p[6];
  const int sj = g.sJ, sk = g.sJ * g.sK, c = gidx(g, i, j, k), d = c + sk;
  const float tem = kmh[c] + kmh[d];
  t11[c] = t11[c] * tem;
  t22[c] = t22[c] * tem;
  t33[c] = t33[c] * tem;
  t12[c] = t12[c] * (0.25f * (((kmh[c - 1 - sj] + kmh[c]) + (kmh[c - 1] + kmh[c - sj])) +
                              ((kmh[d - 1 - sj] + kmh[d]) + (kmh[d - 1] + kmh[d - sj]))));
  if (k >= 1 && k <= g.nz - 1 && i >= 0 && j >= 0) {
    float *TE_R t13 = A.p[7], *TE_R t23 = A.p[8];
    t13[c] = t13[c] * (kmv[c - 1] + kmv[c]);
    t23[c] = t23[c] * (kmv[c - sj] + kmv[c]);
  }
}
TE_LAUNCH3(turb_gettau)

// turb_km_kh.wgsl: TKE closure on w levels 1..nz-1: grid scale (dx dy dz)^(1/3), mixing
// length (limited by c_l sqrt(tke / N^2) in stable air), dissipation added to dissten,
// km = cmz sqrt(tke) len kmScale (or kmFixed > 0), kh = km min(1 + 2 len / scale, 3)
__global__ void k_turb_km_kh(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  const float *TE_R tkea = A.p[1], *TE_R nm = A.p[2], *TE_R hm = A.p[30];
  float *TE_R kmh = A.p[4], *TE_R kmv = A.p[5], *TE_R khh = A.p[6], *TE_R khv = A.p[7];
  float *TE_R lenscl = A.p[8], *TE_R dissten = A.p[9];
  const float kmScale = A.f[10], kmFixed = A.f[11], turbfac = A.f[12];
  const float c_m = 0.1f, c_l = 0.8165f, ri_c = 0.25f, tke_min = 1e-10f, nm_min = 1e-06f, small_len_frac = 0.001f;
  const int c = gidx(g, i, j, k);
  const float cmz = wmax(0.001f, turbfac * c_m);
  const float ce1z = ((cmz * c_l) * c_l) * (dcr(1.0f, ri_c) - 1.0f);
  const float ce2z = wmax(0.0f, fmaf(cmz * 3.1415927f, 3.1415927f, -ce1z));
  const float dzk = dcr(dcr(1.0f, g.rdz), A.p[3][k]);
  const float grdscl = pow_f64((dcr(dcr(1.0f, g.rdx), hm_uh(g, hm, i)) * dcr(dcr(1.0f, g.rdy), hm_vh(g, hm, j))) * dzk, 0.33333334f);
  const float rgrdscl = dcr(1.0f, grdscl);
  const float tka = tkea[c], nmc = nm[c];
  float tk, len;
  if (tka <= tke_min) {
    tk = tke_min;
    len = small_len_frac * grdscl;
  } else {
    tk = tka;
    len = grdscl;
    if (nmc > nm_min) {
      len = c_l * sqrtf(dcr(tk, nmc));
      len = wmin(len, grdscl);
      len = wmax(len, small_len_frac * grdscl);
    }
  }
  lenscl[c] = len;
  dissten[c] = dissten[c] + dcr((fmaf(ce2z * len, rgrdscl, ce1z) * tk) * sqrtf(tk), len);
  const float km = kmFixed > 0.0f ? kmFixed : ((cmz * sqrtf(tk)) * len) * kmScale;
  kmh[c] = km;
  kmv[c] = km;
  float prinv = 3.0f;
  if (nm[c] > nm_min) prinv = wmin(fmaf(2.0f * len, rgrdscl, 1.0f), 3.0f);
  khh[c] = km * prinv;
  khv[c] = khh[c];
}
TE_LAUNCH3(turb_km_kh)

// tke_epst.wgsl: shear production on w levels 1..nz-1, stresses times strain rates
// interpolated (c1/c2) or averaged to the w point, divided by rf
__global__ void k_tke_epst(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  const float *TE_R u = A.p[1], *TE_R v = A.p[2], *TE_R w = A.p[3], *TE_R t11 = A.p[4], *TE_R t12 = A.p[5];
  const float *TE_R t13 = A.p[6], *TE_R t22 = A.p[7], *TE_R t23 = A.p[8], *TE_R t33 = A.p[9], *TE_R rf = A.p[10];
  const float *TE_R mh = A.p[11], *TE_R hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK, c = gidx(g, i, j, k), cd = c - sk;
  const float uh = hm_uh(g, hm, i), vh = hm_vh(g, hm, j), mfk = A.p[12][k], c1 = A.p[13][k], c2 = A.p[14][k];
  auto l1 = [&](int cc) {
    return fmaf(((u[cc + 1] - u[cc]) * g.rdx) * uh, t11[cc], (((v[cc + sj] - v[cc]) * g.rdy) * vh) * t22[cc]);
  };
  auto l2 = [&](int cc, int ii, int jj) {
    return t12[cc] * fmaf((u[cc] - u[cc - sj]) * g.rdy, hm_vf(g, hm, jj), ((v[cc] - v[cc - 1]) * g.rdx) * hm_uf(g, hm, ii));
  };
  auto l3 = [&](int cc, int ii) {
    return fmaf((w[cc] - w[cc - 1]) * g.rdx, hm_uf(g, hm, ii), ((u[cc] - u[cc - sk]) * g.rdz) * mfk) * t13[cc];
  };
  auto l4 = [&](int cc, int jj) {
    return fmaf((w[cc] - w[cc - sj]) * g.rdy, hm_vf(g, hm, jj), ((v[cc] - v[cc - sk]) * g.rdz) * mfk) * t23[cc];
  };
  auto l5 = [&](int cc, int kk) { return (((w[cc + sk] - w[cc]) * g.rdz) * mh[kk]) * t33[cc]; };
  float e = fmaf(c1, l1(cd), c2 * l1(c));
  const float hi = (l2(c, i, j) + l2(c + 1 + sj, i + 1, j + 1)) + (l2(c + sj, i, j + 1) + l2(c + 1, i + 1, j));
  const float lo = (l2(cd, i, j) + l2(cd + 1 + sj, i + 1, j + 1)) + (l2(cd + sj, i, j + 1) + l2(cd + 1, i + 1, j));
  e = fmaf(0.25f, fmaf(c2, hi, c1 * lo), e);
  e = fmaf(0.5f, (l3(c, i) + l3(c + 1, i + 1)) + (l4(c, j) + l4(c + sj, j + 1)), e);
  e = e + fmaf(c1, l5(cd, k - 1), c2 * l5(c, k));
  A.p[15][c] = dcr(e, rf[c]);
}
TE_LAUNCH3(tke_epst)

// saturation mixing ratio over liquid (a, b = 17.67, 29.65: f_mp_rslf) or ice (21.874557,
// 7.66: f_mp_rsif), turb_nm.wgsl
__device__ __forceinline__ float mp_rs(float p, float t, float a, float b) {
  float es = 611.2f * exp_f64(dcr(a * (t - 273.15f), t - b));
  es = wmin(es, p * 0.5f);
  return dcr(dcr(287.04f, 461.5f) * es, p - es);
}

// turb_nm.wgsl: squared Brunt-Vaisala frequency on w levels 1..nz-1.  Dry: g dln(th)/dz;
// moist: g dln(thv)/dz, or in saturated air (liquid above 0 C, ice below -40 C, a linear
// blend between) the moist-adiabatic form (lam_1); sat marks saturated points
__global__ void k_turb_nm(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz + 1;
  if (i >= g.nx || j >= g.ny || k > g.nz - 1) return;
  const float *TE_R thPert = A.p[1], *TE_R ppPert = A.p[2], *TE_R th0 = A.p[3], *TE_R pi0 = A.p[4], *TE_R prs = A.p[5];
  const float *TE_R qv = A.p[6], *TE_R qc = A.p[7], *TE_R qr = A.p[8], *TE_R qi = A.p[9], *TE_R qs = A.p[10], *TE_R qg = A.p[11];
  const float *TE_R mf = A.p[14];
  float *TE_R nm = A.p[15], *TE_R sat = A.p[17];
  const int moist = A.iv[16], wantSat = A.iv[18];
  const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, cpv = 1870.0f, cpl = 4190.0f, cpi = 2106.0f;
  const float lv1 = 3134708.0f, lv2 = 2320.0f, ls1 = 2898463.5f, ls2 = 236.0f, nmsat = 1e-10f, gAcc = 9.81f;
  const float al = 17.67f, bl = 29.65f, ai = 21.874557f, bi = 7.66f;
  const int sk = g.sJ * g.sK, c = gidx(g, i, j, k), d = c - sk;
  if (wantSat != 0) sat[c] = 0.0f;
  const float eps = dcr(rd, rv), reps = dcr(rv, rd);
  const float thA = th0[k - 1] + thPert[d], thB = th0[k] + thPert[c];
  if (moist == 0) {
    nm[c] = ((rr_log_cr(dcr(thB, thA)) * gAcc) * g.rdz) * mf[k];
    return;
  }
  const float piA = pi0[k - 1] + ppPert[d], piB = pi0[k] + ppPert[c];
  const float tA = thA * piA, tB = thB * piB;
  const float qtA = ((((qv[d] + qc[d]) + qr[d]) + qi[d]) + qs[d]) + qg[d];
  const float qtB = ((((qv[c] + qc[c]) + qr[c]) + qi[c]) + qs[c]) + qg[c];
  const float qciA = (qv[d] + qc[d]) + qi[d], qciB = (qv[c] + qc[c]) + qi[c];
  const float thvA = dcr(thA * fmaf(reps, qv[d], 1.0f), 1.0f + qtA);
  const float thvB = dcr(thB * fmaf(reps, qv[c], 1.0f), 1.0f + qtB);
  const float rmf = g.rdz * mf[k];
  const float dlnT = rr_log_cr(dcr(tB, tA)) * rmf;
  const float dlnQt = rr_log_cr(dcr(1.0f + qtB, 1.0f + qtA)) * rmf;
  float out = (gAcc * rr_log_cr(dcr(thvB, thvA))) * rmf;
  const float a = A.p[12][k], b = A.p[13][k];
  const float pavg = fmaf(a, prs[d], b * prs[c]), tavg = fmaf(a, tA, b * tB);
  const float qtavg = fmaf(a, qtA, b * qtB), qciavg = fmaf(a, qciA, b * qciB);
  // lam_1: moist-adiabatic N^2 for saturation ratio qvs, latent heat lh, dqvs/dT drdt
  auto lam1 = [&](float qvs, float lh, float drdt, float cpml) {
    const float gamma = dcr((gAcc * (1.0f + qtavg)) * (1.0f + dcr(lh * qvs, rd * tavg)), fmaf(lh, drdt, cpml));
    return gAcc * fmaf(dlnT + dcr(gamma, tavg), 1.0f + dcr(tavg * drdt, eps + qvs), -dlnQt);
  };
  if (tavg >= 273.15f) {
    const float qvs = mp_rs(pavg, tavg, al, bl);
    const float ql = wmax(qciavg - qvs, 0.0f);
    if (ql > nmsat) {
      if (wantSat != 0) sat[c] = 1.0f;
      const float qvl = wmax(qciavg - ql, 0.0f);
      const float cpml = fmaf(cpl, ql, fmaf(cpv, qvl, cp));
      const float lh = fmaf(-lv2, tavg, lv1);
      const float drdt = dcr((al * (273.15f - bl)) * qvs, (tavg - bl) * (tavg - bl));
      out = lam1(qvs, lh, drdt, cpml);
    }
  } else if (tavg <= 233.15f) {
    const float qvs = mp_rs(pavg, tavg, ai, bi);
    const float qice = wmax(qciavg - qvs, 0.0f);
    if (qice > nmsat) {
      if (wantSat != 0) sat[c] = 1.0f;
      const float qvl = wmax(qciavg - qice, 0.0f);
      const float cpml = fmaf(cpi, qice, fmaf(cpv, qvl, cp));
      const float lh = fmaf(-ls2, tavg, ls1);
      const float drdt = dcr((ai * (273.15f - bi)) * qvs, (tavg - bi) * (tavg - bi));
      out = lam1(qvs, lh, drdt, cpml);
    }
  } else {
    const float ff = dcr(tavg - 233.15f, 273.15f - 233.15f);
    const float qvsl = mp_rs(pavg, tavg, al, bl), qvsi = mp_rs(pavg, tavg, ai, bi);
    const float qvs = fmaf(ff, qvsl, (1.0f - ff) * qvsi);
    const float qice = wmax(0.0f, (1.0f - ff) * (qciavg - qvs));
    const float ql = wmax(0.0f, ff * (qciavg - qvs));
    if (ql + qice > nmsat) {
      if (wantSat != 0) sat[c] = 1.0f;
      const float qvl = wmax(0.0f, (qciavg - ql) - qice);
      const float cpml = fmaf(cpi, qice, fmaf(cpl, ql, fmaf(cpv, qvl, cp)));
      const float lhl = fmaf(-lv2, tavg, lv1);
      const float drdtl = dcr((al * (273.15f - bl)) * qvsl, (tavg - bl) * (tavg - bl));
      const float nml = lam1(qvsl, lhl, drdtl, cpml);
      const float lhi = fmaf(-ls2, tavg, ls1);
      const float drdti = dcr((ai * (273.15f - bi)) * qvsi, (tavg - bi) * (tavg - bi));
      const float nmi = lam1(qvsi, lhi, drdti, cpml);
      out = fmaf(ff, nml, (1.0f - ff) * nmi);
    }
  }
  nm[c] = out;
}
TE_LAUNCH3(turb_nm)

// turb_sfcstress.wgsl: boundary stresses t13, t23 per column (i <= nx, j <= ny).  Top:
// no-slip drag or a copy of level nz-1.  Bottom by mode: 0 copy of level 1; 4 no-slip drag;
// 2 drag coefficient 0.001229 with the surface wind speed (plane 2 of sfc); 3 drag against
// the domain-mean wind (planes 14..16 at the origin, lam_1); else u*^2 w1 / max(s1, 0.01)
__global__ void k_turb_sfcstress(KArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const Dims& g = A.g;
  if (i >= A.gx || j >= A.gy || i > g.nx || j > g.ny) return;
  const float *TE_R sfc = A.p[1], *TE_R rf = A.p[2], *TE_R u = A.p[6], *TE_R v = A.p[7], *TE_R kmv = A.p[9];
  const float *TE_R mf = A.p[11];
  float *TE_R t13 = A.p[3], *TE_R t23 = A.p[4];
  const int mode = A.iv[5];
  const float mx = A.f[8], my = __int_as_float(A.iv2[8]);
  const int plane = g.sJ * g.sK, sj = g.sJ;
  const int ct = gidx(g, i, j, g.nz);
  if (A.iv[10] != 0) {
    const int cu = ct - plane;
    const float mft = 0.5f * (mf[g.nz] + mf[g.nz]);
    t13[ct] = ((((((-2.0f) * (u[cu] + mx)) * g.rdz) * mft) * 0.5f) * (rf[ct - 1] + rf[ct])) * 0.5f * (kmv[cu - 1] + kmv[cu]);
    t23[ct] = ((((((-2.0f) * (v[cu] + my)) * g.rdz) * mft) * 0.5f) * (rf[ct - sj] + rf[ct])) * 0.5f * (kmv[cu - sj] + kmv[cu]);
  } else {
    t13[ct] = t13[ct - plane];
    t23[ct] = t23[ct - plane];
  }
  const int c = gidx(g, i, j, 0);
  if (mode == 0) {
    t13[c] = t13[c + plane];
    t23[c] = t23[c + plane];
  } else if (mode == 4) {
    const float mfb = 0.5f * (mf[0] + mf[0]);
    t13[c] = ((((((2.0f * (u[c] + mx)) * g.rdz) * mfb) * 0.5f) * (rf[c - 1] + rf[c])) * 0.5f) * (kmv[c - 1 + plane] + kmv[c + plane]);
    t23[c] = ((((((2.0f * (v[c] + my)) * g.rdz) * mfb) * 0.5f) * (rf[c - sj] + rf[c])) * 0.5f) * (kmv[c - sj + plane] + kmv[c + plane]);
  } else if (mode == 2) {
    const float s1w = sfc[2 * plane + c - 1], s1c = sfc[2 * plane + c], s1s = sfc[2 * plane + c - sj];
    t13[c] = ((((0.001229f * 0.5f) * (s1w + s1c)) * (u[c] + mx)) * 0.5f) * (rf[c - 1] + rf[c]);
    t23[c] = ((((0.001229f * 0.5f) * (s1s + s1c)) * (v[c] + my)) * 0.5f) * (rf[c - sj] + rf[c]);
  } else if (mode == 3) {
    const int o0 = gidx(g, 0, 0, 0);
    const float au = sfc[14 * plane + o0], av = sfc[15 * plane + o0], as = sfc[16 * plane + o0];
    const float den = wmax(0.0001f, as * sqrtf(fmaf(au, au, av * av)));
    auto lam1 = [&](int q, int comp) {
      const float us = sfc[3 * plane + q], am = comp == 0 ? au : av;
      return dcr((us * us) * fmaf(sfc[2 * plane + q], am, as * (sfc[comp * plane + q] - am)), den);
    };
    t13[c] = (0.25f * (lam1(c - 1, 0) + lam1(c, 0))) * (rf[c - 1] + rf[c]);
    t23[c] = (0.25f * (lam1(c - sj, 1) + lam1(c, 1))) * (rf[c - sj] + rf[c]);
  } else {
    auto lam2 = [&](int q, int comp) {
      const float us = sfc[3 * plane + q];
      return dcr((us * us) * sfc[comp * plane + q], wmax(sfc[2 * plane + q], 0.01f));
    };
    t13[c] = (0.25f * (lam2(c - 1, 0) + lam2(c, 0))) * (rf[c - 1] + rf[c]);
    t23[c] = (0.25f * (lam2(c - sj, 1) + lam2(c, 1))) * (rf[c - sj] + rf[c]);
  }
}
static void launch_turb_sfcstress(const KArgs& A, cudaStream_t s) { launch_columns(k_turb_sfcstress, A, s); }

// turb_dissipative_heating.wgsl: thten += dissipation / (cp pi) (dry) or / ((cp/cv) cv_m pi)
// (moist); the dissipation averaged to the cell centre, at the surface with bbc3
// u*^3 ln((dz1 + z0) / z0) / (k dz1)
__global__ void k_turb_dissipative_heating(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const float *TE_R dissten = A.p[1], *TE_R ppi = A.p[3], *TE_R sfc = A.p[12];
  float* TE_R thten = A.p[10];
  const float* pw = A.sw[0];
  const int moist = __float_as_int(pw[0]), bbc3 = __float_as_int(pw[1]), zntField = __float_as_int(pw[4]);
  const float znt = pw[2], dz1 = pw[3];
  const float cpd = 1005.7f, rd = 287.04f, cpv = 1870.0f, rv = 461.5f, karman = 0.4f;
  const int sk = g.sJ * g.sK, c = gidx(g, i, j, k);
  const float cv = cpd - rd, cvv = cpv - rv, cpl = 4190.0f, cpi = 2106.0f, cpdcv = dcr(cpd, cv);
  float epsd;
  if (k == 0 && bbc3 != 0) {
    const float ust = sfc[3 * sk + c];
    const float z0 = zntField != 0 ? sfc[4 * sk + c] : znt;
    epsd = dcr(((ust * ust) * ust) * log_f64(dcr(dz1 + z0, z0)), karman * dz1);
  } else {
    epsd = 0.5f * (dissten[c] + dissten[c + sk]);
  }
  const float pi = A.p[2][k] + ppi[c];
  float dheat;
  if (moist != 0) {
    const float cvm = fmaf(cpi, (A.p[7][c] + A.p[8][c]) + A.p[9][c], fmaf(cpl, A.p[5][c] + A.p[6][c], fmaf(cvv, A.p[4][c], cv)));
    dheat = dcr(epsd, (cpdcv * cvm) * pi);
  } else {
    dheat = dcr(epsd, cpd * pi);
  }
  thten[c] = thten[c] + dheat;
}
TE_LAUNCH3(turb_dissipative_heating)

// turb_u_tendency.wgsl (AX 0) and turb_v_tendency.wgsl (AX 1, x and y exchanged): subgrid
// momentum tendency per column.  Horizontal stress divergence (zero on open edges) plus
// the explicit vertical divergence, or an implicit vertical diffusion by a Thomas sweep
// (cA, cB; cB ends as the new velocity) with tendency rho (new - old) / dt and the dw/dx
// (dw/dy) cross term dwd.  s is the offset of the staggered neighbour (1 or strideJ).
template <int AX>
__global__ void k_turb_uv_tendency(KArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const Dims& g = A.g;
  if (i >= A.gx || j >= A.gy) return;
  if (AX == 0 ? (i > g.nx || j >= g.ny) : (i >= g.nx || j > g.ny)) return;
  const float *TE_R X = A.p[1], *TE_R w = A.p[2], *TE_R rho = A.p[3], *TE_R rf = A.p[4], *TE_R kmv = A.p[5];
  const float *TE_R A1 = A.p[6], *TE_R A2 = A.p[7], *TE_R A3 = A.p[8], *TE_R mh = A.p[9], *TE_R mf = A.p[10];
  const float* TE_R hm = A.p[30];
  float *TE_R cA = A.p[12], *TE_R cB = A.p[13], *TE_R dwd = A.p[14], *TE_R ten = A.p[15];
  const float dt = A.f[11];
  const bool zeroX = A.iv[16] != 0 && (i == 0 || i == (AX == 0 ? g.nx : g.nx - 1));
  const bool zeroY = A.iv2[16] != 0 && (j == 0 || j == (AX == 0 ? g.ny - 1 : g.ny));
  const int sj = g.sJ, sk = g.sJ * g.sK, s = AX == 0 ? 1 : sj, base = gidx(g, i, j, 0);
  auto horiz = [&](int c) {
    const float tx = zeroX ? 0.0f
                           : (AX == 0 ? ((A1[c] - A1[c - 1]) * g.rdx) * hm_uf(g, hm, i) : ((A1[c + 1] - A1[c]) * g.rdx) * hm_uh(g, hm, i));
    const float ty = zeroY ? 0.0f
                           : (AX == 0 ? ((A2[c + sj] - A2[c]) * g.rdy) * hm_vh(g, hm, j) : ((A2[c] - A2[c - sj]) * g.rdy) * hm_vf(g, hm, j));
    return tx + ty;
  };
  auto rinv = [&](int k) { return dcr(1.0f, 0.5f * (rho[base + k * sk - s] + rho[base + k * sk])); };
  if (A.iv[17] != 0) {
    for (int k = 0; k < g.nz; k++) {
      const int c = base + k * sk;
      const float turbz = (((A3[c + sk] - A3[c]) * g.rdz) * 0.5f) * (mh[k] + mh[k]);
      ten[c] = ten[c] + dcr(horiz(c) + turbz, 0.5f * (rho[c - s] + rho[c]));
    }
    return;
  }
  const float tema = (((-0.0625f) * dt) * g.rdz) * g.rdz, temc = (0.5f * dt) * g.rdz, rdt = dcr(0.5f, dt);
  for (int k = 0; k <= g.nz; k++) {
    const int c = base + k * sk;
    const float dwx = AX == 0 ? ((w[c] - w[c - 1]) * g.rdx) * hm_uf(g, hm, i) : ((w[c] - w[c - sj]) * g.rdy) * hm_vf(g, hm, j);
    dwd[c] = ((dwx * 0.25f) * (kmv[c - s] + kmv[c])) * (rf[c - s] + rf[c]);
  }
  // lam_1: coefficient of the face at level lev for the cell at level k
  auto lam1 = [&](int k, int lev) {
    const int cl = base + lev * sk;
    return (((kmv[cl - s] + kmv[cl]) * (mf[lev] + mf[lev])) * (rf[cl - s] + rf[cl])) * ((mh[k] + mh[k]) * rinv(k));
  };
  {
    const float cfc = tema * lam1(0, 1), cfb = 1.0f - cfc;
    const float cfd = fmaf(-((temc * A3[base]) * (mh[0] + mh[0])), rinv(0), X[base]);
    const float t = dcr(1.0f, cfb);
    cA[base] = (-cfc) * t;
    cB[base] = cfd * t;
  }
  for (int k = 1; k < g.nz - 1; k++) {
    const int c = base + k * sk;
    const float cfa = tema * lam1(k, k), cfc = tema * lam1(k, k + 1), cfb = (1.0f - cfa) - cfc;
    const float t = dcr(1.0f, fmaf(cfa, cA[c - sk], cfb));
    cA[c] = (-cfc) * t;
    cB[c] = fmaf(-cfa, cB[c - sk], X[c]) * t;
  }
  {
    const int kt = g.nz - 1, ct = base + kt * sk;
    const float cfa = tema * lam1(kt, kt), cfb = 1.0f - cfa;
    const float cfd = fmaf((temc * A3[base + g.nz * sk]) * (mh[kt] + mh[kt]), rinv(kt), X[ct]);
    const float t = dcr(1.0f, fmaf(cfa, cA[ct - sk], cfb));
    cB[ct] = fmaf(-cfa, cB[ct - sk], cfd) * t;
  }
  for (int k = g.nz - 2; k >= 0; k--) {
    const int c = base + k * sk;
    cB[c] = fmaf(cA[c], cB[c + sk], cB[c]);
  }
  for (int k = 0; k < g.nz; k++) {
    const int c = base + k * sk;
    float turbz = ((rho[c - s] + rho[c]) * (cB[c] - X[c])) * rdt;
    turbz = fmaf(((dwd[c + sk] - dwd[c]) * g.rdz) * 0.5f, mh[k] + mh[k], turbz);
    ten[c] = fmaf(horiz(c) + turbz, rinv(k), ten[c]);
  }
}
#ifdef TE_KERNELS_FAST
// implicit branch of turb_u_tendency / turb_v_tendency, a block per 32 columns (coop_thomas)
template <int AX>
__global__ void __launch_bounds__(kCoopCols * kCoopWarps) k_turb_uv_coop(KArgs A) {
  extern __shared__ float tsm[];
  const Dims& g = A.g;
  const int nz = g.nz;
  const CoopCol q = coop_col(A, tsm, g.nx + (AX == 0), g.ny + (AX == 1));
  const int i = q.i, j = q.j;
  const bool on = q.on;
  const float *TE_R X = A.p[1], *TE_R w = A.p[2], *TE_R rho = A.p[3], *TE_R rf = A.p[4], *TE_R kmv = A.p[5];
  const float *TE_R A1 = A.p[6], *TE_R A2 = A.p[7], *TE_R A3 = A.p[8], *TE_R mh = A.p[9], *TE_R mf = A.p[10];
  const float* TE_R hm = A.p[30];
  float *TE_R dwd = A.p[14], *TE_R ten = A.p[15];
  const float dt = A.f[11];
  const int sj = g.sJ, sk = q.sk, s = AX == 0 ? 1 : sj, base = q.base;
  const float tema = (((-0.0625f) * dt) * g.rdz) * g.rdz, temc = (0.5f * dt) * g.rdz;
  auto rinv = [&](int k) { return dcr(1.0f, 0.5f * (rho[base + k * sk - s] + rho[base + k * sk])); };
  auto lam1 = [&](int k, int lev) {
    const int cl = base + lev * sk;
    return (((kmv[cl - s] + kmv[cl]) * (mf[lev] + mf[lev])) * (rf[cl - s] + rf[cl])) * ((mh[k] + mh[k]) * rinv(k));
  };
  if (on) {
#pragma unroll 2
    for (int k = q.wq; k <= nz; k += kCoopWarps) {
      const int c = base + k * sk;
      const float dwx = AX == 0 ? ((w[c] - w[c - 1]) * g.rdx) * hm_uf(g, hm, i) : ((w[c] - w[c - sj]) * g.rdy) * hm_vf(g, hm, j);
      dwd[c] = ((dwx * 0.25f) * (kmv[c - s] + kmv[c])) * (rf[c - s] + rf[c]);
      if (k == nz) continue;
      const int e = k * kCoopCols + q.lane;
      if (k < nz - 1) q.sC[e] = tema * lam1(k, k + 1);
      if (k > 0) q.sA[e] = tema * lam1(k, k);
      float d = X[c];
      if (k == 0) d = fmaf(-((temc * A3[base]) * (mh[0] + mh[0])), rinv(0), X[base]);
      else if (k == nz - 1) d = fmaf((temc * A3[base + nz * sk]) * (mh[k] + mh[k]), rinv(k), X[c]);
      q.sD[e] = d;
    }
  }
  __syncthreads();
  if (q.wq == 0 && on) coop_thomas(q.sA, q.sC, q.sD, q.scA, q.scB, 0, nz - 1, q.lane, A.p[12], A.p[13], base, sk);
  __syncthreads();
  if (!on) return;
  const bool zeroX = A.iv[16] != 0 && (i == 0 || i == (AX == 0 ? g.nx : g.nx - 1));
  const bool zeroY = A.iv2[16] != 0 && (j == 0 || j == (AX == 0 ? g.ny - 1 : g.ny));
  const float rdt = dcr(0.5f, dt);
  for (int k = q.wq; k < nz; k += kCoopWarps) {
    const int c = base + k * sk;
    const float tx = zeroX ? 0.0f
                           : (AX == 0 ? ((A1[c] - A1[c - 1]) * g.rdx) * hm_uf(g, hm, i) : ((A1[c + 1] - A1[c]) * g.rdx) * hm_uh(g, hm, i));
    const float ty = zeroY ? 0.0f
                           : (AX == 0 ? ((A2[c + sj] - A2[c]) * g.rdy) * hm_vh(g, hm, j) : ((A2[c] - A2[c - sj]) * g.rdy) * hm_vf(g, hm, j));
    float turbz = ((rho[c - s] + rho[c]) * (q.scB[k * kCoopCols + q.lane] - X[c])) * rdt;
    turbz = fmaf(((dwd[c + sk] - dwd[c]) * g.rdz) * 0.5f, mh[k] + mh[k], turbz);
    ten[c] = fmaf((tx + ty) + turbz, rinv(k), ten[c]);
  }
}

template <int AX>
static void launch_turb_uv(const KArgs& A, cudaStream_t st) {
  if (A.iv[17] != 0 || A.g.nz < 2 || coop_bytes(A.g.nz) > 200 * 1024) {
    launch_columns(k_turb_uv_tendency<AX>, A, st);
    return;
  }
  launch_coop(k_turb_uv_coop<AX>, A, st, A.g.nx + (AX == 0), A.g.ny + (AX == 1));
}
static void launch_turb_u_tendency(const KArgs& A, cudaStream_t s) { launch_turb_uv<0>(A, s); }
static void launch_turb_v_tendency(const KArgs& A, cudaStream_t s) { launch_turb_uv<1>(A, s); }
#else
static void launch_turb_u_tendency(const KArgs& A, cudaStream_t s) { launch_columns(k_turb_uv_tendency<0>, A, s); }
static void launch_turb_v_tendency(const KArgs& A, cudaStream_t s) { launch_columns(k_turb_uv_tendency<1>, A, s); }
#endif

// turb_w_tendency.wgsl (TKE 0) and tke_transport.wgsl (TKE 1): tendency of a w-level
// quantity q on levels 1..nz-1 per column.  Horizontal divergence (w: of t13, t23; TKE: of
// -fx, -fy), zero on open edges, plus the explicit vertical divergence or the implicit
// vertical diffusion (Thomas sweep over levels 1..nz-1, boundary fluxes folded into the
// right-hand side), tendency rf (new - old) / dt.
template <int TKE>
__global__ void k_turb_wlevel(KArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const Dims& g = A.g;
  if (i >= A.gx || j >= A.gy || i >= g.nx || j >= g.ny) return;
  const float *TE_R q = A.p[1], *TE_R rho = A.p[2], *TE_R rf = A.p[3], *TE_R kmh = A.p[4];
  const float *TE_R kmv = TKE ? A.p[5] : nullptr, *TE_R h1 = TKE ? A.p[11] : A.p[5], *TE_R h2 = TKE ? A.p[12] : A.p[6];
  const float *TE_R t33 = TKE ? nullptr : A.p[7], *TE_R mh = TKE ? A.p[6] : A.p[8], *TE_R mf = TKE ? A.p[7] : A.p[9];
  const float* TE_R hm = A.p[30];
  float *TE_R cA = TKE ? A.p[9] : A.p[11], *TE_R cB = TKE ? A.p[10] : A.p[12], *TE_R ten = A.p[13];
  const float dt = TKE ? A.f[8] : A.f[10];
  const bool zeroX = A.iv[14] != 0 && (i == 0 || i == g.nx - 1), zeroY = A.iv2[14] != 0 && (j == 0 || j == g.ny - 1);
  const int sj = g.sJ, sk = g.sJ * g.sK, base = gidx(g, i, j, 0);
  auto horiz = [&](int c) {
    const float tx = zeroX ? 0.0f : (TKE ? ((-(h1[c + 1] - h1[c])) * g.rdx) * hm_uh(g, hm, i) : ((h1[c + 1] - h1[c]) * g.rdx) * hm_uh(g, hm, i));
    const float ty = zeroY ? 0.0f : (TKE ? ((-(h2[c + sj] - h2[c])) * g.rdy) * hm_vh(g, hm, j) : ((h2[c + sj] - h2[c]) * g.rdy) * hm_vh(g, hm, j));
    return tx + ty;
  };
  // TKE vertical flux at cell level k (lam_1 of tke_transport.wgsl)
  auto tflux = [&](int k) {
    const int c = base + k * sk;
    return ((((-(kmv[c] + kmv[c + sk])) * (q[c + sk] - q[c])) * g.rdz) * mh[k]) * rho[c];
  };
  if (A.iv[15] != 0) {
    float below = TKE ? tflux(0) : 0.0f;
    for (int k = 1; k < g.nz; k++) {
      const int c = base + k * sk;
      float turbz;
      if (TKE) {
        const float here = tflux(k);
        turbz = ((-(here - below)) * g.rdz) * mf[k];
        below = here;
      } else {
        turbz = ((t33[c] - t33[c - sk]) * g.rdz) * mf[k];
      }
      ten[c] = ten[c] + dcr(horiz(c) + turbz, rf[c]);
    }
    return;
  }
  const float tema = (((-1.0f) * dt) * g.rdz) * g.rdz, temc = dt * g.rdz, rdt = dcr(1.0f, dt);
  auto mfr = [&](int k) { return dcr(mf[k], rf[base + k * sk]); };
  auto up = [&](int k) {
    const int c = base + k * sk;
    return (((kmh[c] + kmh[c + sk]) * mh[k]) * rho[c]) * mfr(k);
  };
  auto dn = [&](int k) {
    const int c = base + k * sk;
    return (((kmh[c - sk] + kmh[c]) * mh[k - 1]) * rho[c - sk]) * mfr(k);
  };
  {
    const int c = base + sk;
    const float cfc = tema * up(1), cfb = 1.0f - cfc;
    const float cfd = TKE ? fmaf(temc * ((((-(kmv[c - sk] + kmv[c])) * (q[c] - q[c - sk])) * g.rdz) * mh[0]) * rho[c - sk], mfr(1), q[c])
                          : fmaf(-(temc * t33[c - sk]), mfr(1), q[c]);
    const float t = dcr(1.0f, cfb);
    cA[c] = (-cfc) * t;
    cB[c] = cfd * t;
  }
  for (int k = 2; k < g.nz - 1; k++) {
    const int c = base + k * sk;
    const float cfa = tema * dn(k), cfc = tema * up(k), cfb = (1.0f - cfa) - cfc;
    const float t = dcr(1.0f, fmaf(cfa, cA[c - sk], cfb));
    cA[c] = (-cfc) * t;
    cB[c] = fmaf(-cfa, cB[c - sk], q[c]) * t;
  }
  {
    const int kt = g.nz - 1, ct = base + kt * sk;
    const float cfa = tema * dn(kt), cfb = 1.0f - cfa;
    const float cfd = TKE ? fmaf(-(temc * (((((-(kmv[ct] + kmv[ct + sk])) * (q[ct + sk] - q[ct])) * g.rdz) * mh[kt]) * rho[ct])), mfr(kt), q[ct])
                          : fmaf(temc * t33[ct], mfr(kt), q[ct]);
    const float t = dcr(1.0f, fmaf(cfa, cA[ct - sk], cfb));
    cB[ct] = fmaf(-cfa, cB[ct - sk], cfd) * t;
  }
  for (int k = g.nz - 2; k >= 1; k--) {
    const int c = base + k * sk;
    cB[c] = fmaf(cA[c], cB[c + sk], cB[c]);
  }
  for (int k = 1; k < g.nz; k++) {
    const int c = base + k * sk;
    const float turbz = (rf[c] * (cB[c] - q[c])) * rdt;
    ten[c] = ten[c] + dcr(horiz(c) + turbz, rf[c]);
  }
}
#ifdef TE_KERNELS_FAST
// implicit branch of turb_w_tendency (TKE 0) / tke_transport (TKE 1) over w levels
// 1..nz-1, a block per 32 columns (coop_thomas)
template <int TKE>
__global__ void __launch_bounds__(kCoopCols * kCoopWarps) k_turb_wlevel_coop(KArgs A) {
  extern __shared__ float tsm[];
  const Dims& g = A.g;
  const int nz = g.nz;
  const CoopCol cq = coop_col(A, tsm, g.nx, g.ny);
  const int i = cq.i, j = cq.j, sj = g.sJ, sk = cq.sk, base = cq.base;
  const float *TE_R q = A.p[1], *TE_R rho = A.p[2], *TE_R rf = A.p[3], *TE_R kmh = A.p[4];
  const float *TE_R kmv = TKE ? A.p[5] : nullptr, *TE_R h1 = TKE ? A.p[11] : A.p[5], *TE_R h2 = TKE ? A.p[12] : A.p[6];
  const float *TE_R t33 = TKE ? nullptr : A.p[7], *TE_R mh = TKE ? A.p[6] : A.p[8], *TE_R mf = TKE ? A.p[7] : A.p[9];
  const float* TE_R hm = A.p[30];
  float* TE_R ten = A.p[13];
  const float dt = TKE ? A.f[8] : A.f[10];
  const float tema = (((-1.0f) * dt) * g.rdz) * g.rdz, temc = dt * g.rdz;
  auto mfr = [&](int k) { return dcr(mf[k], rf[base + k * sk]); };
  if (cq.on)
#pragma unroll 2
    for (int k = 1 + cq.wq; k <= nz - 1; k += kCoopWarps) {
      const int c = base + k * sk, e = k * kCoopCols + cq.lane;
      if (k < nz - 1) cq.sC[e] = tema * ((((kmh[c] + kmh[c + sk]) * mh[k]) * rho[c]) * mfr(k));
      if (k > 1) cq.sA[e] = tema * ((((kmh[c - sk] + kmh[c]) * mh[k - 1]) * rho[c - sk]) * mfr(k));
      float d = q[c];
      if (k == 1)
        d = TKE ? fmaf(temc * ((((-(kmv[c - sk] + kmv[c])) * (q[c] - q[c - sk])) * g.rdz) * mh[0]) * rho[c - sk], mfr(1), q[c])
                : fmaf(-(temc * t33[c - sk]), mfr(1), q[c]);
      else if (k == nz - 1)
        d = TKE ? fmaf(-(temc * (((((-(kmv[c] + kmv[c + sk])) * (q[c + sk] - q[c])) * g.rdz) * mh[k]) * rho[c])), mfr(k), q[c])
                : fmaf(temc * t33[c], mfr(k), q[c]);
      cq.sD[e] = d;
    }
  __syncthreads();
  float* TE_R cA = TKE ? A.p[9] : A.p[11];
  float* TE_R cB = TKE ? A.p[10] : A.p[12];
  if (cq.wq == 0 && cq.on) coop_thomas(cq.sA, cq.sC, cq.sD, cq.scA, cq.scB, 1, nz - 1, cq.lane, cA, cB, base, sk);
  __syncthreads();
  if (!cq.on) return;
  const bool zeroX = A.iv[14] != 0 && (i == 0 || i == g.nx - 1), zeroY = A.iv2[14] != 0 && (j == 0 || j == g.ny - 1);
  const float rdt = dcr(1.0f, dt);
  for (int k = 1 + cq.wq; k <= nz - 1; k += kCoopWarps) {
    const int c = base + k * sk;
    const float tx = zeroX ? 0.0f : (TKE ? ((-(h1[c + 1] - h1[c])) * g.rdx) * hm_uh(g, hm, i) : ((h1[c + 1] - h1[c]) * g.rdx) * hm_uh(g, hm, i));
    const float ty = zeroY ? 0.0f : (TKE ? ((-(h2[c + sj] - h2[c])) * g.rdy) * hm_vh(g, hm, j) : ((h2[c + sj] - h2[c]) * g.rdy) * hm_vh(g, hm, j));
    const float turbz = (rf[c] * (cq.scB[k * kCoopCols + cq.lane] - q[c])) * rdt;
    ten[c] = ten[c] + dcr((tx + ty) + turbz, rf[c]);
  }
}

template <int TKE>
static void launch_turb_wlevel(const KArgs& A, cudaStream_t st) {
  if (A.iv[15] != 0 || A.g.nz < 3 || coop_bytes(A.g.nz) > 200 * 1024) {
    launch_columns(k_turb_wlevel<TKE>, A, st);
    return;
  }
  launch_coop(k_turb_wlevel_coop<TKE>, A, st, A.g.nx, A.g.ny);
}
static void launch_turb_w_tendency(const KArgs& A, cudaStream_t s) { launch_turb_wlevel<0>(A, s); }
static void launch_tke_transport(const KArgs& A, cudaStream_t s) { launch_turb_wlevel<1>(A, s); }
#else
static void launch_turb_w_tendency(const KArgs& A, cudaStream_t s) { launch_columns(k_turb_wlevel<0>, A, s); }
static void launch_tke_transport(const KArgs& A, cudaStream_t s) { launch_columns(k_turb_wlevel<1>, A, s); }
#endif

// Two-float accumulation of the mass sums (f_df_add / f_df_add_pair, mass_row_sums.wgsl):
// acc.x + x by an error-free sum, the error accumulated in acc.y.  The sums run in the
// reference's order (row by row in i, level by level in j, total in k), so the results
// are its words.
__device__ __forceinline__ void df_add(F2& acc, float x) {
  const float s = acc.x + x, bb = s - acc.x;
  const float err = (acc.x - (s - bb)) + (x - bb);
  acc.x = s;
  acc.y = acc.y + err;
}
__device__ __forceinline__ void df_add_pair(F2& acc, float vx, float vy) {
  df_add(acc, vx);
  acc.y = acc.y + vy;
}

// mass_row_sums with a warp per (j, k) row: the lanes form 32 consecutive terms, every
// lane accumulates them in order of i (two-float sums are order-dependent).  A row's
// inputs are all read before lane 0 writes its two pairs, in the reference's order, so
// this form serves aliased bindings too.
__global__ void __launch_bounds__(32 * kLineWarps) k_mass_rows_warp(KArgs A) {
  const Dims& g = A.g;
  const int lane = threadIdx.x & 31, j = blockIdx.x * kLineWarps + (threadIdx.x >> 5), k = blockIdx.y;
  if (j >= A.gx || k >= A.gy || A.gz <= 0 || j >= g.ny || k >= g.nz) return;
  const float *TE_R rho = A.p[1], *TE_R pp3d = A.p[3], *TE_R hm = A.p[30];
  const float pik = A.p[2][k], mhk = A.p[4][k];
  const float rvh = dcr(1.0f, hm_vh(g, hm, j));
  F2 s1{0.0f, 0.0f}, s2{0.0f, 0.0f};
  for (int i0 = 0; i0 < g.nx; i0 += 32) {
    const int i = i0 + lane;
    float w = 0.0f, p = 0.0f;
    if (i < g.nx) {
      const int c = gidx(g, i, j, k);
      w = ((rho[c] * dcr(1.0f, hm_uh(g, hm, i))) * rvh) * dcr(1.0f, mhk);
      p = pik + pp3d[c];
    }
    const int n = min(32, g.nx - i0);
    for (int l = 0; l < n; l++) {
      df_add(s1, __shfl_sync(0xffffffffu, w, l));
      df_add(s2, __shfl_sync(0xffffffffu, p, l));
    }
  }
  if (lane == 0) {
    const long o = 2L * ((long)k * g.sK + j);
    A.p[5][o] = s1.x;
    A.p[5][o + 1] = s1.y;
    A.p[6][o] = s2.x;
    A.p[6][o + 1] = s2.y;
  }
}
static void launch_mass_row_sums(const KArgs& A, cudaStream_t s) {
  if (A.gx > 0 && A.gy > 0)
    launch_kernel(k_mass_rows_warp, dim3((A.gx + kLineWarps - 1) / kLineWarps, A.gy), dim3(32 * kLineWarps), 0, s, A);
}

// mass_level_sums with a warp per level, the row pairs added in order of j
__global__ void __launch_bounds__(32 * kLineWarps) k_mass_levels_warp(KArgs A) {
  const Dims& g = A.g;
  const int lane = threadIdx.x & 31, k = blockIdx.x * kLineWarps + (threadIdx.x >> 5);
  if (k >= A.gx || A.gy <= 0 || A.gz <= 0 || k >= g.nz) return;
  const float *TE_R rows1 = A.p[1], *TE_R rows2 = A.p[2];
  F2 s1{0.0f, 0.0f}, s2{0.0f, 0.0f};
  for (int j0 = 0; j0 < g.ny; j0 += 32) {
    const int j = j0 + lane;
    float a0 = 0.0f, a1 = 0.0f, b0 = 0.0f, b1 = 0.0f;
    if (j < g.ny) {
      const long o = 2L * ((long)k * g.sK + j);
      a0 = rows1[o];
      a1 = rows1[o + 1];
      b0 = rows2[o];
      b1 = rows2[o + 1];
    }
    const int n = min(32, g.ny - j0);
    for (int l = 0; l < n; l++) {
      df_add_pair(s1, __shfl_sync(0xffffffffu, a0, l), __shfl_sync(0xffffffffu, a1, l));
      df_add_pair(s2, __shfl_sync(0xffffffffu, b0, l), __shfl_sync(0xffffffffu, b1, l));
    }
  }
  if (lane == 0) {
    A.p[3][2 * k] = s1.x;
    A.p[3][2 * k + 1] = s1.y;
    A.p[4][2 * k] = s2.x;
    A.p[4][2 * k + 1] = s2.y;
  }
}
static void launch_mass_level_sums(const KArgs& A, cudaStream_t s) {
  if (A.gx > 0) launch_kernel(k_mass_levels_warp, dim3((A.gx + kLineWarps - 1) / kLineWarps), dim3(32 * kLineWarps), 0, s, A);
}

// mass_reference_init.wgsl: on its first run (ref[2] == 0) thread 0 stores the total mass
// (the sum of the level pairs) as the reference and sets ref[2] = 1
__global__ void k_mass_reference_init(KArgs A) {
  TE_K3
  if (tx != 0 || ty != 0) return;
  const float* TE_R levels1 = A.p[1];
  float* TE_R ref = A.p[2];
  if (ref[2] != 0.0f) return;
  F2 s{0.0f, 0.0f};
  for (int k = 0; k < g.nz; k++) df_add_pair(s, levels1[2 * k], levels1[2 * k + 1]);
  ref[0] = s.x;
  ref[1] = s.y;
  ref[2] = 1.0f;
}
TE_LAUNCH3(mass_reference_init)

// mass_correction_apply.wgsl: relative mass change r against the reference turned into a
// uniform pi' correction tem = ((1 + r)^(rd/cv) - 1) sum(pi) / (nx ny nz) (f_powm1: the pow
// builtin for |r| > 0.05, else its third-order expansion), added to pp3d; prs and rho from
// the corrected pi; thread (0,0,0) records tem, the mass, the pi sum, r and the mass's low part
__global__ void k_mass_correction_apply(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const float *TE_R levels1 = A.p[2], *TE_R levels2 = A.p[3], *TE_R ref = A.p[4], *TE_R thPert = A.p[5];
  float *TE_R pp3d = A.p[6], *TE_R prs = A.p[10], *TE_R rho = A.p[11];
  const float rd = 287.04f, cp = 1005.7f, rv = 461.5f, p00 = 1e+05f;
  F2 m2{0.0f, 0.0f}, pp2{0.0f, 0.0f};
  for (int kk = 0; kk < g.nz; kk++) {
    df_add_pair(m2, levels1[2 * kk], levels1[2 * kk + 1]);
    df_add_pair(pp2, levels2[2 * kk], levels2[2 * kk + 1]);
  }
  const float rddcv = dcr(rd, cp - rd);
  const float r = dcr((ref[0] - m2.x) + (ref[1] - m2.y), m2.x);
  const float p2 = pp2.x + pp2.y;
  const float pm1 = fabsf(r) > 0.05f ? pow_f64(1.0f + r, rddcv) - 1.0f
                                     : r * fmaf(r, fmaf(rddcv * (rddcv - 1.0f), 0.5f, dcr(((r * rddcv) * (rddcv - 1.0f)) * (rddcv - 2.0f), 6.0f)), rddcv);
  const float tem = dcr(pm1 * p2, (float)((g.nx * g.ny) * g.nz));
  if (i == 0 && j == 0 && k == 0) {
    float* out = A.p[12];
    out[0] = tem;
    out[1] = m2.x;
    out[2] = p2;
    out[3] = r;
    out[4] = m2.y;
  }
  const int c = gidx(g, i, j, k);
  const float pp = pp3d[c] + tem;
  pp3d[c] = pp;
  const float cpdrd = dcr(cp, rd);
  const float pi = A.p[8][k] + pp, th = A.p[7][k] + thPert[c];
  const float p = p00 * rr_pow_cr(pi, cpdrd);
  prs[c] = p;
  const float rmix = A.iv[1] != 0 ? fmaf(wmax(0.0f, A.p[9][c]), rv, rd) : rd;
  rho[c] = dcr(p, (th * pi) * rmix);
}
TE_LAUNCH3(mass_correction_apply)

// morr_prep.wgsl: temperature T = (th0 + th)(pi0 + pp) and a copy qv0 of qv before the
// microphysics column
__global__ void k_morr_prep(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const int c = gidx(g, i, j, k);
  A.p[6][c] = (A.p[1][k] + A.p[3][c]) * (A.p[2][k] + A.p[4][c]);
  A.p[7][c] = A.p[5][c];
}
TE_LAUNCH3(morr_prep)

// morr_column.wgsl: one thread per column (te_morr.cuh morr::column), the dispatch's rows
// taken scr_rows at a time (the reference's y tiles: the planned per-thread scratch holds
// that many rows); each launch lays the scratch out by array, level, then column of the
// tile, so the threads of a warp touch consecutive words.
__global__ void __launch_bounds__(128) k_morr_column(KArgs A, int y0, int rows) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int ncol = A.gx * rows;
  if (t >= ncol) return;
  const int i = t % A.gx, j = y0 + t / A.gx;
  if (j >= A.gy) return;
  morr::Params p;
  {
    uint32_t* w = reinterpret_cast<uint32_t*>(&p);
    for (int q = 0; q < (int)(sizeof(morr::Params) / 4); q++) w[q] = A.ref0[q];
  }
  if (i >= p.nx || j >= p.ny) return;
  morr::Fields F;
  F.T3 = A.p[1];
  F.QV = A.p[2];
  F.QC = A.p[3];
  F.QR = A.p[4];
  F.QI = A.p[5];
  F.QS = A.p[6];
  F.QG = A.p[7];
  F.NI = A.p[8];
  F.NS = A.p[9];
  F.NR = A.p[10];
  F.NG = A.p[11];
  F.P3 = A.p[12];
  F.RH3 = A.p[13];
  F.DZQ = A.p[14];
  F.sfc = A.p[15];
  F.EFFC = A.p[16];
  F.EFFI = A.p[17];
  F.EFFS = A.p[18];
  const morr::Scratch S{A.scr + t, (unsigned)ncol, p.nz};
  morr::column(p, F, S, i, j, A.iv[19]);
}

// (nz <= 128 and a one-level dispatch grid are checked at plan time, Plan::finalize_args)
static void launch_morr_column(const KArgs& A, cudaStream_t s) {
  const int rows = A.scr_rows > 0 ? (int)A.scr_rows : A.gy;
  for (int y0 = 0; y0 < A.gy; y0 += rows) {
    const int r = std::min(rows, A.gy - y0);
    const int ncol = A.gx * r;
    launch_kernel(k_morr_column, dim3((ncol + 127) / 128), dim3(128), 0, s, A, y0, r);
  }
}

// morr_refl10cm.wgsl: one thread per column (te_refl.cuh morr::refl_column), the
// dispatch's rows taken scr_rows at a time like morr_column, the 11 per-level arrays in the
// planned scratch laid out by array, level, then column of the tile.
__global__ void __launch_bounds__(128) k_morr_refl10cm(KArgs A, int y0, int rows) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int ncol = A.gx * rows;
  if (t >= ncol) return;
  const int i = t % A.gx, j = y0 + t / A.gx;
  if (j >= A.gy) return;
  morr::Params p;
  {
    uint32_t* w = reinterpret_cast<uint32_t*>(&p);
    for (int q = 0; q < (int)(sizeof(morr::Params) / 4); q++) w[q] = A.ref0[q];
  }
  if (i >= p.nx || j >= p.ny) return;
  morr::RadarHead h;
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(A.p[1]);
    uint32_t* w = reinterpret_cast<uint32_t*>(&h);
    for (int q = 0; q < (int)(sizeof(morr::RadarHead) / 4); q++) w[q] = src[q];
  }
  morr::RadarFields F;
  F.bs = A.p[2];
  F.bg = A.p[3];
  F.simpson = A.p[4];
  F.T = A.p[5];
  F.QR = A.p[6];
  F.QS = A.p[7];
  F.QG = A.p[8];
  F.NR = A.p[9];
  F.NS = A.p[10];
  F.NG = A.p[11];
  F.RH = A.p[12];
  F.dbz = A.p[13];
  const morr::Scratch S{A.scr + t, (unsigned)ncol, p.nz};
  morr::refl_column(p, h, F, S, i, j);
}

// (nz <= 128, a one-level dispatch grid and bound head, bins and weights are checked at
// plan time, Plan::finalize_args)
static void launch_morr_refl10cm(const KArgs& A, cudaStream_t s) {
  const int rows = A.scr_rows > 0 ? (int)A.scr_rows : A.gy;
  for (int y0 = 0; y0 < A.gy; y0 += rows) {
    const int r = std::min(rows, A.gy - y0);
    const int ncol = A.gx * r;
    launch_kernel(k_morr_refl10cm, dim3((ncol + 127) / 128), dim3(128), 0, s, A, y0, r);
  }
}

// morr_post.wgsl: where the column changed T (by >= 1e-4) or qv (by >= 1e-14), pressure
// from the equation of state, pi' from it (the reference's correctly rounded pow) and th
__global__ void k_morr_post(KArgs A) {
  TE_K3
  const int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  const float *TE_R th0 = A.p[1], *TE_R pi0 = A.p[2], *TE_R rho = A.p[3], *TE_R T = A.p[4], *TE_R qv0 = A.p[5];
  const float* TE_R qv = A.p[6];
  float *TE_R th = A.p[7], *TE_R pp = A.p[8], *TE_R prs = A.p[9];
  const float rd = 287.04f, cp = 1005.7f, rv = 461.5f;
  const int c = gidx(g, i, j, k);
  const float rp00 = dcr(1.0f, 1e+05f), rovcp = dcr(rd, cp);
  const float told = (th0[k] + th[c]) * (pi0[k] + pp[c]);
  const float t = T[c], q = qv[c];
  if (fabsf(t - told) >= 0.0001f || fabsf(q - qv0[c]) >= 1e-14f) {
    const float p = (rho[c] * fmaf(rv, q, rd)) * t;
    const float ppn = rr_pow_cr(p * rp00, rovcp) - pi0[k];
    prs[c] = p;
    pp[c] = ppn;
    th[c] = dcr(t, pi0[k] + ppn) - th0[k];
  }
}
TE_LAUNCH3(morr_post)

// -------------------------------------------------- thermodynamic glue

__global__ void k_update_diagnostics_moist(KArgs A) {
  TE_K3
  const float *TE_R thp = A.p[1], *TE_R ppp = A.p[2], *TE_R th0 = A.p[3], *TE_R pi0 = A.p[4], *TE_R qv0 = A.p[5], *TE_R qc0 = A.p[6];
  const float *TE_R qi0 = A.p[7], *TE_R rth0 = A.p[8], *TE_R qv = A.p[9], *TE_R qc = A.p[10], *TE_R qr = A.p[11], *TE_R qi = A.p[12];
  const float *TE_R qs = A.p[13], *TE_R qg = A.p[14];
  float *TE_R thv = A.p[15], *TE_R ppterm = A.p[16], *TE_R piadv = A.p[17], *TE_R thterm = A.p[18], *TE_R buoy = A.p[19];
  const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, cv = 718.66003f, cpv = 1870.0f, cvv = 1408.5f;
  const float rovcp = 0.28541315f, cpl = 4190.0f, cpi = 2106.0f;
  TE_WHOLE(k < g.nz)
  float reps = dcr(rv, rd);
  float repsm1 = reps - 1.0f;
  float gacc = 9.81f;
  float qvv = wmax(qv[c], 0.0f);
  float liq = qc[c] + qr[c];
  float ice = (qi[c] + qs[c]) + qg[c];
  float qli = wmax(0.0f, liq + ice);
  float cpli = fmaf(cpl, wmax(0.0f, liq), cpi * wmax(0.0f, ice));
  float th = th0[k] + thp[c];
  float pi = pi0[k] + ppp[c];
  float cpm = fmaf(cpv, qvv, cp) + cpli;
  float cvm = dcr(1.0f, fmaf(cvv, qvv, cv) + cpli);
  thv[c] = dcr(th * fmaf(reps, qvv, 1.0f), (1.0f + qvv) + qli);
  piadv[c] = pi;
  ppterm[c] = ((pi * rovcp) * cpm) * cvm;
  thterm[c] = (th * fmaf(-rovcp, cpm, fmaf(rv, qvv, rd))) * cvm;
  buoy[c] = gacc * (fmaf(thp[c], rth0[k], repsm1 * (qvv - qv0[k])) - ((qli - qc0[k]) - qi0[k]));
}
TE_LAUNCH3(update_diagnostics_moist)

// update_diagnostics (update_diagnostics.wgsl main; encoded timestep.js:1548-1556): the dry
// step's thv = th0 + th', piadv = pi0 + pi', ppterm = pi rd / (cp - rd), buoy = g th' / th0
__global__ void k_update_diagnostics(KArgs A) {
  TE_K3
  const float *TE_R thp = A.p[1], *TE_R ppp = A.p[2], *TE_R th0 = A.p[3], *TE_R pi0 = A.p[4], *TE_R rth0 = A.p[8];
  float *TE_R thv = A.p[5], *TE_R ppterm = A.p[6], *TE_R piadv = A.p[7], *TE_R buoy = A.p[9];
  TE_WHOLE(k < g.nz)
  const float rd = 287.04f, cp = 1005.7f;
  const float rddcv = dcr(rd, cp - rd);
  const float pi = pi0[k] + ppp[c];
  thv[c] = th0[k] + thp[c];
  piadv[c] = pi;
  ppterm[c] = pi * rddcv;
  buoy[c] = (9.81f * thp[c]) * rth0[k];
}
TE_LAUNCH3(update_diagnostics)

// stability_max (stability_max.wgsl main; encoded timestep.js:742-762): per interior point
// the squared advective Courant number c2 = x^2 + y^2 + z^2 (x = (u + u_e) dt/2dx uh, ...)
// and, with the eddy viscosities (withKs, k >= 1), the largest diffusion number m; the
// bit patterns (non-negative floats order like their u32 words) reach out[0], out[1] by
// atomic max.  A warp forms its maxima first, so one atomic per warp and word.
__global__ void k_stability_max(KArgs A) {
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y * blockDim.y + threadIdx.y;
  const int tz = blockIdx.z;
  const Dims& g = A.g;
  const float dtdx = A.sw[0][0], dtdy = A.sw[0][1], dtdz = A.sw[0][2], ksdx = A.sw[0][3], ksdy = A.sw[0][4];
  const int twoD = __float_as_int(A.sw[0][5]), withKs = __float_as_int(A.sw[0][6]);
  const float *TE_R u = A.p[2], *TE_R v = A.p[3], *TE_R w = A.p[4], *TE_R mh = A.p[5];
  const float *TE_R kmh = A.p[6], *TE_R kmv = A.p[7], *TE_R khh = A.p[8], *TE_R hm = A.p[30];
  const int i = tx, j = ty, k = tz;
  const bool inside = tx < A.gx && ty < A.gy && tz < A.gz && i < g.nx && j < g.ny && k < g.nz;
  float c2 = 0.0f, m = 0.0f;
  if (inside) {
    const int c = gidx(g, i, j, k);
    const float uh = hm_uh(g, hm, i), vh = hm_vh(g, hm, j);
    const float x = ((u[c] + u[gidx(g, i + 1, j, k)]) * dtdx) * uh;
    const float z = ((w[c] + w[gidx(g, i, j, k + 1)]) * dtdz) * mh[k];
    if (twoD != 0) {
      c2 = fmaf(x, x, z * z);
    } else {
      const float y = ((v[c] + v[gidx(g, i, j + 1, k)]) * dtdy) * vh;
      c2 = fmaf(z, z, fmaf(x, x, y * y));
    }
    if (withKs != 0 && k >= 1) {
      const float K[3] = {kmh[c], khh[c], kmv[c]};
#pragma unroll
      for (int n = 0; n < 3; n++) {
        const float a = ((K[n] * ksdx) * uh) * uh;
        float t;
        if (twoD != 0) {
          t = a;
        } else {
          const float b = ((K[n] * ksdy) * vh) * vh;
          t = fmaf(a, a, b * b);
        }
        m = wmax(m, t);
      }
    }
  }
  unsigned cb = __float_as_uint(c2), kb = __float_as_uint(m);
  for (int o = 16; o > 0; o >>= 1) {
    cb = max(cb, __shfl_xor_sync(0xffffffffu, cb, o));
    kb = max(kb, __shfl_xor_sync(0xffffffffu, kb, o));
  }
  if ((threadIdx.x & 31) == 0) {
    unsigned* out = reinterpret_cast<unsigned*>(A.p[9]);
    atomicMax(out, cb);
    atomicMax(out + 1, kb);
  }
}
static void launch_stability_max(const KArgs& A, cudaStream_t s) {
  // blocks of 32 x 4: every warp is one full row of 32 threads, as the shuffle reduction needs
  dim3 b(32, 4, 1);
  dim3 gr((A.gx + 31) / 32, (A.gy + 3) / 4, A.gz);
  launch_kernel(k_stability_max, dim3(gr), dim3(b), 0, s, A);
}

__global__ void k_pressure_tendency(KArgs A) {
  TE_K3
  const float *TE_R th = A.p[1], *TE_R qv = A.p[2], *TE_R rho = A.p[3], *TE_R ppi = A.p[4], *TE_R thten = A.p[5], *TE_R qpten = A.p[6];
  const float *TE_R th0 = A.p[7], *TE_R pi0 = A.p[8];
  const float dt = A.f[9];
  const int hasDiabatic = A.iv[10];
  float* TE_R ppten = A.p[11];
  const int hasStepTend = A.iv[12];
  const float* TE_R qvt = A.p[13];
  const int moist = A.iv[14];
  const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, p00 = 1e5f;
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float rp00 = dcr(1.0f, p00);
  float rddcv = dcr(rd, cp - rd);
  float tem = 0.0001f * 0.0001f;
  float qsmall = 1e-14f;
  float tht = hasStepTend != 0 ? thten[c] : 0.0f;
  if (moist == 0) {
    float p = 0.0f;
    if (fabsf(dt * tht) > tem) {
      float thnew = fmaf(dt, tht, th[c]);
      float pinew = rr_pow_cr(((rho[c] * (th0[k] + thnew)) * rd) * rp00, rddcv) - pi0[k];
      p = dcr(pinew - ppi[c], dt);
    }
    ppten[c] = p;
    return;
  }
  float qvten = qvt[c];
  float p = 0.0f;
  if (fabsf(dt * tht) > tem || fabsf(dt * qvten) > qsmall) {
    float thnew = fmaf(dt, tht, th[c]);
    float qvnew = fmaf(dt, qvten, qv[c]);
    float pinew = rr_pow_cr(((rho[c] * (th0[k] + thnew)) * fmaf(rv, qvnew, rd)) * rp00, rddcv) - pi0[k];
    p = dcr(pinew - ppi[c], dt);
  }
  if (hasDiabatic != 0) p = p + qpten[c];
  ppten[c] = p;
}
TE_LAUNCH3(pressure_tendency)

__global__ void k_divergence3d(KArgs A) {
  TE_K3
  const float *TE_R u = A.p[1], *TE_R v = A.p[2], *TE_R w = A.p[3], *TE_R mh = A.p[4];
  float* TE_R div = A.p[5];
  const float* TE_R hm = A.p[30];
  const int sj = g.sJ, sk = g.sJ * g.sK;
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float d = fmaf((w[c + sk] - w[c]) * g.rdz, mh[k],
                 fmaf((u[c + 1] - u[c]) * g.rdx, hm_uh(g, hm, i), ((v[c + sj] - v[c]) * g.rdy) * hm_vh(g, hm, j)));
  div[c] = fabsf(d) < 1e-30f ? 0.0f : d;
}
TE_LAUNCH3(divergence3d)

__global__ void k_update_rho_prs(KArgs A) {
  TE_K3
  const int moist = A.iv[1];
  const float *TE_R thp = A.p[2], *TE_R ppp = A.p[3], *TE_R th0 = A.p[4], *TE_R pi0 = A.p[5], *TE_R qv = A.p[6];
  float *TE_R prs = A.p[7], *TE_R rho = A.p[8];
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float cpdrd = dcr(1005.7f, 287.04f);
  float pi = pi0[k] + ppp[c];
  float th = th0[k] + thp[c];
  float p = 1e5f * rr_pow_fast(pi, cpdrd);
  prs[c] = p;
  float rmix = moist != 0 ? fmaf(wmax(0.0f, qv[c]), 461.5f, 287.04f) : 287.04f;
  rho[c] = dcr(p, (th * pi) * rmix);
}
TE_LAUNCH3(update_rho_prs)

__global__ void k_diabatic_unapply(KArgs A) {
  TE_K3
  const float dt = A.f[1];
  float *TE_R pp3d = A.p[2], *TE_R th = A.p[3], *TE_R qv = A.p[4], *TE_R qc = A.p[5];
  float *TE_R qpten = A.p[6], *TE_R qtten = A.p[7], *TE_R qvten = A.p[8], *TE_R qcten = A.p[9];
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float x;
  x = fmaf(-dt, qpten[c], pp3d[c]);
  pp3d[c] = x;
  qpten[c] = x;
  x = fmaf(-dt, qtten[c], th[c]);
  th[c] = x;
  qtten[c] = x;
  x = fmaf(-dt, qvten[c], qv[c]);
  qv[c] = x;
  qvten[c] = x;
  x = fmaf(-dt, qcten[c], qc[c]);
  qc[c] = x;
  qcten[c] = x;
}
TE_LAUNCH3(diabatic_unapply)

__global__ void k_diabatic_rates(KArgs A) {
  TE_K3
  const float dt = A.f[1];
  const float *TE_R pp3d = A.p[2], *TE_R th = A.p[3], *TE_R qv = A.p[4], *TE_R qc = A.p[5];
  float *TE_R qpten = A.p[6], *TE_R qtten = A.p[7], *TE_R qvten = A.p[8], *TE_R qcten = A.p[9];
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  float rdt = dcr(1.0f, dt);
  qpten[c] = (pp3d[c] - qpten[c]) * rdt;
  qtten[c] = (th[c] - qtten[c]) * rdt;
  qvten[c] = (qv[c] - qvten[c]) * rdt;
  qcten[c] = (qc[c] - qcten[c]) * rdt;
}
TE_LAUNCH3(diabatic_rates)

__global__ void k_ppx_finish(KArgs A) {
  TE_K3
  const float* TE_R pp3d = A.p[1];
  float* TE_R ppx = A.p[2];
  int i = tx, j = ty, k = tz;
  if (i >= g.nx || j >= g.ny || k >= g.nz) return;
  int c = gidx(g, i, j, k);
  ppx[c] = pp3d[c] + ppx[c];
}
TE_LAUNCH3(ppx_finish)

// ------------------------------------------------------------ registry
// Parameter tables: binding index, ptr/ref, written (the reference kernel ABI,
// data/kernels/kernels.json); the write order defines the per-dispatch hash slots.

#define R(i) {i, kRef, 0}
#define P(i) {i, kPtr, 0}
#define W(i) {i, kPtr, 1}

// ------------------------------------------ row-vector forms of point-wise kernels
// (the __restrict__ build; see k_rowvec).  Each Op restates its kernel above: the same
// range check (active), the same loads (load) and the same operations (store).

#define TE_OP_WHOLE(kcond)                                                            \
  static __device__ __forceinline__ bool active(const KArgs& A, int tx, int ty, int tz) { \
    const Dims& g = A.g;                                                              \
    const int k = tz;                                                                 \
    return tx - 3 <= g.nx + 3 && ty - 3 <= g.ny + 3 && (kcond);                       \
  }
#define TE_OP_INTERIOR                                                                \
  static __device__ __forceinline__ bool active(const KArgs& A, int tx, int ty, int tz) { \
    return tx < A.g.nx && ty < A.g.ny && tz < A.g.nz;                                 \
  }
#define TE_OP_C(ioff) const Dims& g = A.g; const int i = tx - (ioff), j = ty - (ioff), k = tz; \
  const int c = gidx(g, i, j, k); (void)i; (void)j; (void)k

struct OpBuildSadv {
  struct In { float thp; };
  TE_OP_WHOLE(k < g.nz)
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(3);
    return In{A.p[2][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(3);
    A.p[3][c] = (A.p[1][k] - 300.0f) + v.thp;
  }
};

struct OpAcousticBegin {
  struct In { float w; };
  TE_OP_WHOLE(k <= g.nz)
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(3);
    return In{A.p[2][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(3);
    A.p[3][c] = 0.0f;
    A.p[4][c] = 0.0f;
    A.p[5][c] = v.w * A.a.beta;
  }
};

struct OpMassfluxFromState {
  struct In { float u, v, w; };
  TE_OP_WHOLE(k <= g.nz)
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(3);
    In r{0.0f, 0.0f, 0.0f};
    if (k < g.nz) {
      r.u = A.p[1][c];
      r.v = A.p[2][c];
    }
    if (!(k == 0 || k == g.nz)) r.w = A.p[3][c];
    return r;
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(3);
    const float *TE_R rho0 = A.p[4], *TE_R rf0 = A.p[5];
    if (k < g.nz) {
      A.p[6][c] = rho0[k] * v.u;
      A.p[7][c] = rho0[k] * v.v;
    }
    A.p[8][c] = (k == 0 || k == g.nz) ? 0.0f : rf0[k] * v.w;
  }
};

struct OpAcousticAccumulate {
  struct In { float u, v, w, ru, rv, rw; };
  TE_OP_WHOLE(k <= g.nz)
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(3);
    return In{A.p[2][c], A.p[3][c], A.p[4][c], A.p[5][c], A.p[6][c], A.p[7][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(3);
    const float tavg = A.f[8];
    if (tavg > 0.0f) {
      A.p[5][c] = (v.ru + v.u) * tavg;
      A.p[6][c] = (v.rv + v.v) * tavg;
      A.p[7][c] = fmaf(v.w, A.a.alph, v.rw) * tavg;
    } else {
      A.p[5][c] = v.ru + v.u;
      A.p[6][c] = v.rv + v.v;
      A.p[7][c] = v.rw + v.w;
    }
  }
};

struct OpUpdateDiagnosticsMoist {
  struct In { float thp, ppp, qv, qc, qr, qi, qs, qg; };
  TE_OP_WHOLE(k < g.nz)
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(3);
    return In{A.p[1][c], A.p[2][c], A.p[9][c], A.p[10][c], A.p[11][c], A.p[12][c], A.p[13][c], A.p[14][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(3);
    float o[5];
    point(A, k, v, o);
    A.p[15][c] = o[0];
    A.p[17][c] = o[2];
    A.p[16][c] = o[1];
    A.p[18][c] = o[3];
    A.p[19][c] = o[4];
  }
  // thv, ppterm, pi, thterm, buoy (bindings 15..19) of one point at level k
  static __device__ __forceinline__ void point(const KArgs& A, int k, const In& v, float* o) {
    const float *TE_R th0 = A.p[3], *TE_R pi0 = A.p[4], *TE_R qv0 = A.p[5], *TE_R qc0 = A.p[6];
    const float *TE_R qi0 = A.p[7], *TE_R rth0 = A.p[8];
    const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, cv = 718.66003f, cpv = 1870.0f, cvv = 1408.5f;
    const float rovcp = 0.28541315f, cpl = 4190.0f, cpi = 2106.0f;
    float reps = dcr(rv, rd);
    float repsm1 = reps - 1.0f;
    float gacc = 9.81f;
    float qvv = wmax(v.qv, 0.0f);
    float liq = v.qc + v.qr;
    float ice = (v.qi + v.qs) + v.qg;
    float qli = wmax(0.0f, liq + ice);
    float cpli = fmaf(cpl, wmax(0.0f, liq), cpi * wmax(0.0f, ice));
    float th = th0[k] + v.thp;
    float pi = pi0[k] + v.ppp;
    float cpm = fmaf(cpv, qvv, cp) + cpli;
    float cvm = dcr(1.0f, fmaf(cvv, qvv, cv) + cpli);
    o[0] = dcr(th * fmaf(reps, qvv, 1.0f), (1.0f + qvv) + qli);
    o[2] = pi;
    o[1] = ((pi * rovcp) * cpm) * cvm;
    o[3] = (th * fmaf(-rovcp, cpm, fmaf(rv, qvv, rd))) * cvm;
    o[4] = gacc * (fmaf(v.thp, rth0[k], repsm1 * (qvv - qv0[k])) - ((qli - qc0[k]) - qi0[k]));
  }
};

struct OpRkUpdate {
  struct In { float phiA, tend; };
  static __device__ __forceinline__ bool active(const KArgs& A, int tx, int ty, int tz) {
    const Dims& g = A.g;
    const int stag = A.iv[1];
    const int iMax = stag == 2 ? g.nx : g.nx - 1, jMax = stag == 3 ? g.ny : g.ny - 1, kLo = stag == 4 ? 1 : 0;
    return tx <= iMax && ty <= jMax && tz >= kLo && tz < g.nz;
  }
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    return In{A.p[2][c], A.p[3][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    A.p[4][c] = fmaf(A.f[5], v.tend, v.phiA);
  }
};

struct OpApplyThterm {
  struct In { float div, thterm, tend; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    return In{A.p[1][c], A.p[2][c], A.p[3][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    A.p[3][c] = fmaf(-v.div, v.thterm, v.tend);
  }
};

struct OpDiabaticUnapply {
  struct In { float pp, th, qv, qc, qp_t, qt_t, qv_t, qc_t; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    return In{A.p[2][c], A.p[3][c], A.p[4][c], A.p[5][c], A.p[6][c], A.p[7][c], A.p[8][c], A.p[9][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    const float dt = A.f[1];
    float x;
    x = fmaf(-dt, v.qp_t, v.pp);
    A.p[2][c] = x;
    A.p[6][c] = x;
    x = fmaf(-dt, v.qt_t, v.th);
    A.p[3][c] = x;
    A.p[7][c] = x;
    x = fmaf(-dt, v.qv_t, v.qv);
    A.p[4][c] = x;
    A.p[8][c] = x;
    x = fmaf(-dt, v.qc_t, v.qc);
    A.p[5][c] = x;
    A.p[9][c] = x;
  }
};

struct OpDiabaticRates {
  struct In { float pp, th, qv, qc, qp_t, qt_t, qv_t, qc_t; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    return In{A.p[2][c], A.p[3][c], A.p[4][c], A.p[5][c], A.p[6][c], A.p[7][c], A.p[8][c], A.p[9][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    float rdt = dcr(1.0f, A.f[1]);
    A.p[6][c] = (v.pp - v.qp_t) * rdt;
    A.p[7][c] = (v.th - v.qt_t) * rdt;
    A.p[8][c] = (v.qv - v.qv_t) * rdt;
    A.p[9][c] = (v.qc - v.qc_t) * rdt;
  }
};

struct OpPpxFinish {
  struct In { float pp, ppx; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    return In{A.p[1][c], A.p[2][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    A.p[2][c] = v.pp + v.ppx;
  }
};

struct OpDivergence3d {
  struct In { float u0, u1, v0, v1, w0, w1; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    const float *TE_R u = A.p[1], *TE_R v = A.p[2], *TE_R w = A.p[3];
    return In{u[c], u[c + 1], v[c], v[c + g.sJ], w[c], w[c + g.sJ * g.sK]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    const float *TE_R mh = A.p[4], *TE_R hm = A.p[30];
    float d = fmaf((v.w1 - v.w0) * g.rdz, mh[k],
                   fmaf((v.u1 - v.u0) * g.rdx, hm_uh(g, hm, i), ((v.v1 - v.v0) * g.rdy) * hm_vh(g, hm, j)));
    A.p[5][c] = fabsf(d) < 1e-30f ? 0.0f : d;
  }
};

struct OpAcousticPrepare {
  struct In { float ppterm, pa, pa_up, pa_dn, thv, thv_dn; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    const float *TE_R ppterm = A.p[2], *TE_R piadv = A.p[3], *TE_R thv = A.p[4];
    const int sk = g.sJ * g.sK;
    In r;
    r.ppterm = ppterm[c];
    r.pa = piadv[c];
    r.pa_up = k != g.nz - 1 ? piadv[c + sk] : 0.0f;
    r.pa_dn = k != 0 ? piadv[c - sk] : 0.0f;
    r.thv = thv[c];
    r.thv_dn = k == 0 ? r.thv : thv[c - sk];
    return r;
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    const Acoustic a = A.a;
    const float *TE_R rr0 = A.p[5], *TE_R rf0 = A.p[6], *TE_R mh = A.p[7], *TE_R mf = A.p[8];
    const float *TE_R c1 = A.p[9], *TE_R c2 = A.p[10];
    const float cp = 1005.7f;
    float tem = (a.dts * g.rdz) * mh[k];
    float r2 = (tem * rr0[k]) * rf0[k + 1];
    float r1 = (tem * rr0[k]) * rf0[k];
    float tem1 = ((a.dts * g.rdz) * cp) * mf[k];
    float c1a = c1[k], c1b = c1[k + 1], c2a = c2[k], c2b = c2[k + 1];
    bool vec_v = g.nx > 3 && i < (g.nx / 4) * 4;
    A.p[11][c] = tem * v.ppterm;
    float p2 = 0.0f, p1 = 0.0f;
    if (k != g.nz - 1) p2 = vec_v ? fmaf(-c2b, v.pa_up, (1.0f - c1b) * v.pa) : fmaf(1.0f - c1b, v.pa, -(c2b * v.pa_up));
    if (k != 0) p1 = vec_v ? fmaf(c2a - 1.0f, v.pa, c1a * v.pa_dn) : fmaf(c1a, v.pa_dn, (c2a - 1.0f) * v.pa);
    A.p[13][c] = k == g.nz - 1 ? 0.0f : r2 * p2;
    A.p[12][c] = k == 0 ? 0.0f : r1 * p1;
    A.p[14][c] = tem1 * fmaf(c2a, v.thv, c1a * v.thv_dn);
  }
};

struct OpBuoyancyApply {
  struct In { float wten, b_dn, b; };
  static __device__ __forceinline__ bool active(const KArgs& A, int tx, int ty, int tz) {
    return tx < A.g.nx && ty < A.g.ny && tz + 1 <= A.g.nz - 1;
  }
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    const Dims& g = A.g;
    const int c = gidx(g, tx, ty, tz + 1), sk = g.sJ * g.sK;
    return In{A.p[4][c], A.p[1][c - sk], A.p[1][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    const Dims& g = A.g;
    const int k = tz + 1, c = gidx(g, tx, ty, k);
    const float *TE_R c1 = A.p[2], *TE_R c2 = A.p[3];
    A.p[4][c] = v.wten + fmaf(c1[k], v.b_dn, c2[k] * v.b);
  }
};

struct OpPdefDum {
  struct In { float s0, s, f0, f1, r0, r1; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ int step(const KArgs& A) {
    const int dir = A.iv[1];
    return dir == 0 ? 1 : (dir == 1 ? A.g.sJ : A.g.sJ * A.g.sK);
  }
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    const int st = step(A);
    const float *TE_R sf = A.p[2], *TE_R s0 = A.p[3], *TE_R f = A.p[4], *TE_R rr = A.p[5];
    return In{s0[c], sf[c], f[c], f[c + st], rr[c], rr[c + st]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    const int dir = A.iv[1], ox = A.iv[9], oy = A.iv2[9];
    const float *TE_R rho0 = A.p[6], *TE_R mh = A.p[7], *TE_R hm = A.p[30];
    const float dt = A.f[8];
    float rd = dir == 0 ? g.rdx : (dir == 1 ? g.rdy : g.rdz);
    float base = rho0[k] * v.s0;
    // pdef_inflow on the loaded mass fluxes (rr[c], rr[c + step])
    bool inflow = false;
    if (dir == 0 && ox != 0) inflow = (i == 0 && v.r0 >= 0.0f) || (i == g.nx - 1 && v.r1 <= 0.0f);
    if (dir == 1 && oy != 0) inflow = (j == 0 && v.r0 >= 0.0f) || (j == g.ny - 1 && v.r1 <= 0.0f);
    if (inflow) {
      A.p[10][c] = base;
      return;
    }
    float adv = (-(v.f1 - v.f0)) * rd;
    float sdiv = (v.s * (v.r1 - v.r0)) * rd;
    float m = dir == 0 ? hm_uh(g, hm, i) : (dir == 1 ? hm_vh(g, hm, j) : mh[k]);
    adv = adv * m;
    sdiv = sdiv * m;
    A.p[10][c] = fmaf(dt, adv + sdiv, base);
  }
};

struct OpMorrPrep {
  struct In { float th, pp, qv; };
  TE_OP_INTERIOR
  static __device__ __forceinline__ In load(const KArgs& A, int tx, int ty, int tz) {
    TE_OP_C(0);
    return In{A.p[3][c], A.p[4][c], A.p[5][c]};
  }
  static __device__ __forceinline__ void store(const KArgs& A, int tx, int ty, int tz, const In& v) {
    TE_OP_C(0);
    A.p[6][c] = (A.p[1][k] + v.th) * (A.p[2][k] + v.pp);
    A.p[7][c] = v.qv;
  }
};

#ifdef TE_KERNELS_FAST
// update_diagnostics_moist over whole fields (whole_field_words, levels 0..nz-1): the eight
// inputs and five outputs of four consecutive words as 16-byte vectors, each word's level
// from its offset; the arithmetic of OpUpdateDiagnosticsMoist::point word by word.
__global__ void k_update_diagnostics_moist_v4(KArgs A, unsigned words, unsigned sk) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n4 = words / 4;
  static constexpr int in_f[8] = {1, 2, 9, 10, 11, 12, 13, 14};
  using Op = OpUpdateDiagnosticsMoist;
  if (q < n4) {
    float4 a[8];
#pragma unroll
    for (int f = 0; f < 8; f++) a[f] = reinterpret_cast<const float4*>(A.p[in_f[f]])[q];
    float4 o4[5];
    const unsigned c0 = 4 * q, k0 = c0 / sk;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int k = (int)(c0 + e >= (k0 + 1) * sk ? k0 + 1 : k0);
      const Op::In v{reinterpret_cast<const float*>(&a[0])[e], reinterpret_cast<const float*>(&a[1])[e],
                     reinterpret_cast<const float*>(&a[2])[e], reinterpret_cast<const float*>(&a[3])[e],
                     reinterpret_cast<const float*>(&a[4])[e], reinterpret_cast<const float*>(&a[5])[e],
                     reinterpret_cast<const float*>(&a[6])[e], reinterpret_cast<const float*>(&a[7])[e]};
      float o[5];
      Op::point(A, k, v, o);
#pragma unroll
      for (int f = 0; f < 5; f++) reinterpret_cast<float*>(&o4[f])[e] = o[f];
    }
#pragma unroll
    for (int f = 0; f < 5; f++) reinterpret_cast<float4*>(A.p[15 + f])[q] = o4[f];
  }
  if (q < words - 4 * n4) {
    const unsigned c = 4 * n4 + q;
    const Op::In v{A.p[1][c], A.p[2][c], A.p[9][c], A.p[10][c], A.p[11][c], A.p[12][c], A.p[13][c], A.p[14][c]};
    float o[5];
    Op::point(A, (int)(c / sk), v, o);
#pragma unroll
    for (int f = 0; f < 5; f++) A.p[15 + f][c] = o[f];
  }
}

static void launch_update_diagnostics_moist_whole(const KArgs& A, cudaStream_t s) {
  static const int fields[13] = {1, 2, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19};
  const unsigned long long words = whole_field_words(A, fields, 13, A.g.nz);
  if (words) {
    const unsigned n4 = (unsigned)(words / 4);
    launch_kernel(k_update_diagnostics_moist_v4, dim3((n4 + 255) / 256), dim3(256), 0, s, A, (unsigned)words,
                  (unsigned)(A.g.sJ * A.g.sK));
  } else {
    launch_rowvec<OpUpdateDiagnosticsMoist>(A, s);
  }
}

// massflux_from_state over whole fields: levels 0..nz-1 of rru = rho0 u, rrv = rho0 v,
// rrw = rf0 w (0 at level 0) as 16-byte vectors, each word's level from its offset; level
// nz of rrw is 0 (rru, rrv have no level nz and are not written there).
__global__ void k_massflux_from_state_v4(KArgs A, unsigned words, unsigned sk) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n4 = words / 4;
  const float *TE_R rho0 = A.p[4], *TE_R rf0 = A.p[5];
  if (q < n4) {
    const float4 u = reinterpret_cast<const float4*>(A.p[1])[q], v = reinterpret_cast<const float4*>(A.p[2])[q];
    const float4 w = reinterpret_cast<const float4*>(A.p[3])[q];
    float4 ru, rv, rw;
    const unsigned c0 = 4 * q, k0 = c0 / sk;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int k = (int)(c0 + e >= (k0 + 1) * sk ? k0 + 1 : k0);
      reinterpret_cast<float*>(&ru)[e] = rho0[k] * reinterpret_cast<const float*>(&u)[e];
      reinterpret_cast<float*>(&rv)[e] = rho0[k] * reinterpret_cast<const float*>(&v)[e];
      reinterpret_cast<float*>(&rw)[e] = k == 0 ? 0.0f : rf0[k] * reinterpret_cast<const float*>(&w)[e];
    }
    reinterpret_cast<float4*>(A.p[6])[q] = ru;
    reinterpret_cast<float4*>(A.p[7])[q] = rv;
    reinterpret_cast<float4*>(A.p[8])[q] = rw;
  }
  if (q < words - 4 * n4) {
    const unsigned c = 4 * n4 + q;
    const int k = (int)(c / sk);
    A.p[6][c] = rho0[k] * A.p[1][c];
    A.p[7][c] = rho0[k] * A.p[2][c];
    A.p[8][c] = k == 0 ? 0.0f : rf0[k] * A.p[3][c];
  }
  if (q < sk) A.p[8][words + q] = 0.0f;
}

static void launch_massflux_from_state_whole(const KArgs& A, cudaStream_t s) {
  static const int fields[6] = {1, 2, 3, 6, 7, 8};
  const unsigned long long all = whole_field_words(A, fields, 6, A.g.nz + 1);
  if (all) {
    const unsigned sk = (unsigned)(A.g.sJ * A.g.sK), words = (unsigned)(all - sk);
    const unsigned n = std::max(words / 4, sk);
    launch_kernel(k_massflux_from_state_v4, dim3((n + 255) / 256), dim3(256), 0, s, A, words, sk);
  } else {
    launch_rowvec<OpMassfluxFromState>(A, s);
  }
}

// build_sadv over whole fields (levels 0..nz-1): sadv = (th0[k] - 300) + th', 16-byte vectors
__global__ void k_build_sadv_v4(KArgs A, unsigned words, unsigned sk) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n4 = words / 4;
  const float* TE_R th0 = A.p[1];
  if (q < n4) {
    const float4 t = reinterpret_cast<const float4*>(A.p[2])[q];
    float4 o;
    const unsigned c0 = 4 * q, k0 = c0 / sk;
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int k = (int)(c0 + e >= (k0 + 1) * sk ? k0 + 1 : k0);
      reinterpret_cast<float*>(&o)[e] = (th0[k] - 300.0f) + reinterpret_cast<const float*>(&t)[e];
    }
    reinterpret_cast<float4*>(A.p[3])[q] = o;
  }
  if (q < words - 4 * n4) {
    const unsigned c = 4 * n4 + q;
    A.p[3][c] = (th0[c / sk] - 300.0f) + A.p[2][c];
  }
}

static void launch_build_sadv_whole(const KArgs& A, cudaStream_t s) {
  static const int fields[2] = {2, 3};
  const unsigned long long words = whole_field_words(A, fields, 2, A.g.nz);
  if (words) {
    const unsigned n4 = (unsigned)(words / 4);
    launch_kernel(k_build_sadv_v4, dim3((n4 + 255) / 256), dim3(256), 0, s, A, (unsigned)words, (unsigned)(A.g.sJ * A.g.sK));
  } else {
    launch_rowvec<OpBuildSadv>(A, s);
  }
}

// acoustic_begin over whole fields (whole_field_words): rru = rrv = 0, rrw = beta w, as
// 16-byte vectors (disjoint bindings only: the vector loads w before any store)
__global__ void k_acoustic_begin_v4(KArgs A, unsigned words) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n4 = words / 4;
  const float beta = A.a.beta;
  const float* TE_R w = A.p[2];
  float *TE_R ru = A.p[3], *TE_R rv = A.p[4], *TE_R rw = A.p[5];
  if (q < n4) {
    const float4 x = reinterpret_cast<const float4*>(w)[q];
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    reinterpret_cast<float4*>(ru)[q] = z;
    reinterpret_cast<float4*>(rv)[q] = z;
    reinterpret_cast<float4*>(rw)[q] = make_float4(x.x * beta, x.y * beta, x.z * beta, x.w * beta);
  }
  if (q < words - 4 * n4) {
    const unsigned e = 4 * n4 + q;
    const float x = w[e];
    ru[e] = 0.0f;
    rv[e] = 0.0f;
    rw[e] = x * beta;
  }
}

static void launch_acoustic_begin_whole(const KArgs& A, cudaStream_t s) {
  static const int fields[4] = {2, 3, 4, 5};
  const unsigned long long words = whole_field_words(A, fields, 4, A.g.nz + 1);
  if (words) {
    const unsigned n4 = (unsigned)(words / 4);
    launch_kernel(k_acoustic_begin_v4, dim3((n4 + 255) / 256), dim3(256), 0, s, A, (unsigned)words);
  } else {
    launch_rowvec<OpAcousticBegin>(A, s);
  }
}
#endif

// the __restrict__ build launches the row-vector form where a kernel has one
#ifdef TE_KERNELS_FAST
#define TE_ROWVEC(name, op) launch_rowvec<op>
#else
#define TE_ROWVEC(name, op) launch_##name
#endif

static const KernelSpec kTable[] = {
    {"adv_flux_x", 4, {R(0), P(1), P(2), W(3)}, false, launch_adv_flux_x},
    {"adv_flux_y", 4, {R(0), P(1), P(2), W(3)}, false, launch_adv_flux_y},
    {"adv_flux_z", 6, {R(0), P(1), P(2), P(3), P(4), W(5)}, false, launch_adv_flux_z},
    {"adv_flux_x_stag", 9, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), W(8)}, false, launch_adv_flux_x_stag},
    {"adv_flux_y_stag", 9, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), W(8)}, false, launch_adv_flux_y_stag},
    {"adv_flux_z_stag", 10, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), W(8), P(30)}, false, launch_adv_flux_z_stag},
    {"adv_flux_x_weno", 6, {R(0), P(1), P(2), R(3), R(4), W(5)}, false, launch_adv_flux_x_weno},
    {"adv_flux_y_weno", 6, {R(0), P(1), P(2), R(3), R(4), W(5)}, false, launch_adv_flux_y_weno},
    {"adv_flux_z_weno", 9, {R(0), P(1), P(2), P(3), P(4), R(5), R(6), R(7), W(8)}, false, launch_adv_flux_z_weno},
    {"adv_flux_x_weno_uv", 6, {R(0), R(1), P(2), P(3), R(4), W(5)}, false, launch_adv_flux_x_weno_uv},
    {"adv_flux_y_weno_uv", 6, {R(0), R(1), P(2), P(3), R(4), W(5)}, false, launch_adv_flux_y_weno_uv},
    {"adv_flux_z_weno_uv", 9, {R(0), R(1), P(2), P(3), P(4), P(5), R(6), W(7), P(30)}, false, launch_adv_flux_z_weno_uv},
    {"adv_flux_x_weno_w", 6, {R(0), P(1), P(2), P(3), R(4), W(5)}, false, launch_adv_flux_x_weno_w},
    {"adv_flux_y_weno_w", 6, {R(0), P(1), P(2), P(3), R(4), W(5)}, false, launch_adv_flux_y_weno_w},
    {"adv_flux_z_weno_w", 5, {R(0), P(1), P(2), R(3), W(4)}, false, launch_adv_flux_z_weno_w},
    {"adv_assemble", 24, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), W(11), R(12), P(13), P(14),
                          P(15), P(16), R(17), P(30), P(18), W(19), R(27), P(24), P(25)}, false, launch_adv_assemble},
    {"rk_update", 6, {R(0), R(1), P(2), P(3), W(4), R(5)}, false, TE_ROWVEC(rk_update, OpRkUpdate)},
    {"pdef_dum", 12, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), R(8), R(9), W(10), P(30)}, false, TE_ROWVEC(pdef_dum, OpPdefDum)},
    {"pdef_apply", 18, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), P(11), P(12), P(13), R(14),
                        R(15), W(16), P(30)}, false, launch_pdef_apply},
#ifdef TE_KERNELS_FAST
    {"build_sadv", 4, {R(0), P(1), P(2), W(3)}, false, launch_build_sadv_whole},
#else
    {"build_sadv", 4, {R(0), P(1), P(2), W(3)}, false, launch_build_sadv},
#endif
#ifdef TE_KERNELS_FAST
    {"massflux_from_state", 10, {R(0), P(1), P(2), P(3), P(4), P(5), W(6), W(7), W(8), P(24)}, false, launch_massflux_from_state_whole},
#else
    {"massflux_from_state", 10, {R(0), P(1), P(2), P(3), P(4), P(5), W(6), W(7), W(8), P(24)}, false, launch_massflux_from_state},
#endif
    {"div_massflux", 8, {R(0), P(1), P(2), P(3), P(4), W(5), P(30), P(25)}, false, TE_ROWVEC(div_massflux, OpDivMassflux)},
    {"velocity_to_massflux", 7, {R(0), P(1), P(2), W(3), W(4), W(5), P(24)}, false,
     TE_ROWVEC(velocity_to_massflux, OpVelocityToMassflux)},
    {"stage_state_reset", 11, {R(0), P(1), P(2), P(3), P(4), W(5), W(6), W(7), W(8), W(9), P(10)}, false, launch_stage_state_reset},
    {"stage_tendency_reset", 4, {R(0), W(1), W(2), W(3)}, false, launch_stage_tendency_reset},
    {"buoyancy_apply", 5, {R(0), P(1), P(2), P(3), W(4)}, false, TE_ROWVEC(buoyancy_apply, OpBuoyancyApply)},
    {"apply_thterm", 4, {R(0), P(1), P(2), W(3)}, false, TE_ROWVEC(apply_thterm, OpApplyThterm)},
    {"acoustic_prepare", 17, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), W(11), W(12), W(13),
                              W(14), P(24), P(25)}, true, TE_ROWVEC(acoustic_prepare, OpAcousticPrepare)},
#ifdef TE_KERNELS_FAST
    {"acoustic_begin", 6, {R(0), R(1), P(2), W(3), W(4), W(5)}, true, launch_acoustic_begin_whole},
#else
    {"acoustic_begin", 6, {R(0), R(1), P(2), W(3), W(4), W(5)}, true, launch_acoustic_begin},
#endif
    {"acoustic_uv", 13, {R(0), R(1), P(2), P(3), P(4), P(5), W(6), W(7), R(8), P(30), P(21), P(23), P(25)}, true, launch_acoustic_uv},
    {"acoustic_fpk", 19, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), W(11), P(30), P(15), P(16),
                          P(17), P(24), P(25), R(26)}, true, launch_acoustic_fpk},
    {"acoustic_w_solve", 12, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), W(9), W(10), W(11)}, true, launch_acoustic_w_solve},
    {"acoustic_pp", 11, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), W(7), W(8), W(9), R(10)}, true, launch_acoustic_pp},
    {"acoustic_accumulate", 9, {R(0), R(1), P(2), P(3), P(4), W(5), W(6), W(7), R(8)}, true, TE_ROWVEC(acoustic_accumulate, OpAcousticAccumulate)},
    {"bc_periodic_x", 2, {R(0), W(1)}, false, launch_bc_periodic_x},
    {"bc_periodic_y", 2, {R(0), W(1)}, false, launch_bc_periodic_y},
    {"bc_open_x", 3, {R(0), W(1), R(2)}, false, launch_bc_open_x},
    {"bc_open_y", 3, {R(0), W(1), R(2)}, false, launch_bc_open_y},
    {"radbc_ew", 7, {R(0), P(1), P(2), R(3), W(4), W(5), P(30)}, false, launch_radbc_ew},
    {"radbc_ns", 7, {R(0), P(1), P(2), R(3), W(4), W(5), P(30)}, false, launch_radbc_ns},
    {"openbc_uv_tendency", 17, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), W(8), W(9), R(10), P(30), P(20), P(22),
                                P(24), P(25), R(26)}, true, launch_openbc_uv_tendency},
    {"turb_zero", 2, {R(0), W(1)}, false, launch_turb_zero},
    {"turb_add_tendency", 4, {R(0), P(1), W(2), R(3)}, false, launch_turb_add_tendency},
    {"turb_scalar_flux_h", 8, {R(0), P(1), P(2), P(3), R(4), W(5), W(6), P(30)}, false, launch_turb_scalar_flux_h},
    {"turb_openbc_flux", 4, {R(0), W(1), W(2), R(3)}, false, launch_turb_openbc_flux},
    {"turb_openbc_stress_x", 3, {R(0), W(1), W(2)}, false, launch_turb_openbc_stress_x},
    {"turb_openbc_stress_y", 3, {R(0), W(1), W(2)}, false, launch_turb_openbc_stress_y},
    {"tke_advance", 5, {R(0), P(1), P(2), R(3), W(4)}, false, launch_tke_advance},
    {"tke_sources", 6, {R(0), P(1), P(2), P(3), P(4), W(5)}, false, launch_tke_sources},
    {"tke_flux_h", 7, {R(0), P(1), P(2), P(3), W(4), W(5), P(30)}, false, launch_tke_flux_h},
    {"mp_pdefq", 4, {R(0), P(1), W(2), R(3)}, false, launch_mp_pdefq},
    {"turb_scalar_vert_implicit", 20, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), R(10), W(11), W(12), W(13), P(14), R(15), R(16), {17, kRefS, 0}, R(18), P(30)}, false, launch_turb_scalar_vert_implicit},
    {"rayleigh_damping", 20, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), R(9), W(10), W(11), W(12), W(13), P(14), P(15), R(16), R(17), P(18), P(19)}, false, launch_rayleigh_damping},
    {"turb_rho_faces", 8, {R(0), P(1), P(2), P(3), W(4), W(5), {6, kRefS, 0}, {7, kRefS, 0}}, false, launch_turb_rho_faces},
    {"turb_def_centers", 11, {R(0), P(1), P(2), P(3), P(4), P(5), W(6), W(7), W(8), W(9), P(30)}, false, launch_turb_def_centers},
    {"turb_def_faces", 9, {R(0), P(1), P(2), P(3), P(4), P(5), W(6), W(7), P(30)}, false, launch_turb_def_faces},
    {"turb_def_assemble", 12, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), W(10), W(11)}, false, launch_turb_def_assemble},
    {"turb_gettau", 10, {R(0), P(1), P(2), W(3), W(4), W(5), W(6), W(7), W(8), P(30)}, false, launch_turb_gettau},
    {"turb_km_kh", 14, {R(0), P(1), P(2), P(3), W(4), W(5), W(6), W(7), W(8), W(9), R(10), R(11), R(12), P(30)}, false, launch_turb_km_kh},
    {"tke_epst", 17, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), P(11), P(12), P(13), P(14), W(15), P(30)}, false, launch_tke_epst},
    {"turb_nm", 19, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), P(11), P(12), P(13), P(14), W(15), R(16), W(17), R(18)}, false, launch_turb_nm},
    {"turb_sfcstress", 13, {R(0), P(1), P(2), W(3), W(4), R(5), P(6), P(7), R(8), P(9), R(10), P(11), P(30)}, false, launch_turb_sfcstress},
    {"turb_dissipative_heating", 13, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), W(10), {11, kRefS, 0}, P(12)}, false, launch_turb_dissipative_heating},
    {"turb_u_tendency", 19, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), R(11), W(12), W(13), W(14), W(15), R(16), R(17), P(30)}, false, launch_turb_u_tendency},
    {"turb_v_tendency", 19, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), R(11), W(12), W(13), W(14), W(15), R(16), R(17), P(30)}, false, launch_turb_v_tendency},
    {"turb_w_tendency", 17, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), R(10), W(11), W(12), W(13), R(14), R(15), P(30)}, false, launch_turb_w_tendency},
    {"tke_transport", 17, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), R(8), W(9), W(10), W(11), W(12), W(13), R(14), R(15), P(30)}, false, launch_tke_transport},
    {"mass_row_sums", 8, {R(0), P(1), P(2), P(3), P(4), W(5), W(6), P(30)}, false, launch_mass_row_sums},
    {"mass_level_sums", 5, {R(0), P(1), P(2), W(3), W(4)}, false, launch_mass_level_sums},
    {"mass_reference_init", 3, {R(0), P(1), W(2)}, false, launch_mass_reference_init},
    {"mass_correction_apply", 13, {R(0), R(1), P(2), P(3), P(4), P(5), W(6), P(7), P(8), P(9), W(10), W(11), W(12)}, false, launch_mass_correction_apply},
    {"morr_prep", 8, {R(0), P(1), P(2), P(3), P(4), P(5), W(6), W(7)}, false, TE_ROWVEC(morr_prep, OpMorrPrep)},
    {"morr_column", 20, {R(0), W(1), W(2), W(3), W(4), W(5), W(6), W(7), W(8), W(9), W(10), W(11), P(12), P(13), P(14),
                         W(15), W(16), W(17), W(18), R(19)}, false, launch_morr_column},
    {"morr_refl10cm", 14, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), P(11), P(12), W(13)},
     false, launch_morr_refl10cm},
    {"morr_post", 10, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), W(7), W(8), W(9)}, false, launch_morr_post},
    {"update_diagnostics", 10, {R(0), P(1), P(2), P(3), P(4), W(5), W(6), W(7), P(8), W(9)}, false, launch_update_diagnostics},
    {"stability_max", 11, {R(0), {1, kRefS, 0}, P(2), P(3), P(4), P(5), P(6), P(7), P(8), W(9), P(30)}, false, launch_stability_max},
#ifdef TE_KERNELS_FAST
    {"update_diagnostics_moist", 20, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), P(11), P(12),
                                      P(13), P(14), W(15), W(16), W(17), W(18), W(19)}, false, launch_update_diagnostics_moist_whole},
#else
    {"update_diagnostics_moist", 20, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), P(9), P(10), P(11), P(12),
                                      P(13), P(14), W(15), W(16), W(17), W(18), W(19)}, false, launch_update_diagnostics_moist},
#endif
    {"pressure_tendency", 15, {R(0), P(1), P(2), P(3), P(4), P(5), P(6), P(7), P(8), R(9), R(10), R(12), P(13), R(14), W(11)},
     false, launch_pressure_tendency},
    {"divergence3d", 7, {R(0), P(1), P(2), P(3), P(4), W(5), P(30)}, false, TE_ROWVEC(divergence3d, OpDivergence3d)},
    {"update_rho_prs", 9, {R(0), R(1), P(2), P(3), P(4), P(5), P(6), W(7), W(8)}, false, launch_update_rho_prs},
    {"diabatic_unapply", 10, {R(0), R(1), W(2), W(3), W(4), W(5), W(6), W(7), W(8), W(9)}, false, TE_ROWVEC(diabatic_unapply, OpDiabaticUnapply)},
    {"diabatic_rates", 10, {R(0), R(1), P(2), P(3), P(4), P(5), W(6), W(7), W(8), W(9)}, false, TE_ROWVEC(diabatic_rates, OpDiabaticRates)},
    {"ppx_finish", 3, {R(0), P(1), W(2)}, false, TE_ROWVEC(ppx_finish, OpPpxFinish)},
};

#undef R
#undef P
#undef W

const KernelSpec* kernel_table(int* count) {
  *count = (int)(sizeof(kTable) / sizeof(kTable[0]));
  return kTable;
}

const KernelSpec* find_kernel(const char* name) {
  int n;
  const KernelSpec* t = kernel_table(&n);
  for (int i = 0; i < n; i++)
    if (std::strcmp(t[i].name, name) == 0) return &t[i];
  return nullptr;
}

#ifdef TE_KERNELS_FAST
}  // namespace fast
#endif
}  // namespace te

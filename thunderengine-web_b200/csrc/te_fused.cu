// Fused step phases (TE_MODE_FUSED) for sm_100a.
//
// The planner scans a step's op list for phases it can run as fewer, larger kernels
// whose results are bit-identical on every field the step keeps; everything else runs
// the exact per-dispatch kernels.  Recognised phases:
//
//  * acoustic substep (timestep.js:1997-2060): acoustic_uv, acoustic_fpk,
//    acoustic_w_solve, acoustic_pp, halo(ppd), acoustic_accumulate, halo(u, v, w)
//    -> K1 (u/v update + u/v accumulation), K2 (pi' forcing + implicit w solve + pi'
//       update + w accumulation, 32-column tiles staged in shared memory), K3 (the
//       four halo fills, with the w accumulation of the halo points).
//  * runs of periodic halo fills (bc_periodic_x then bc_periodic_y per field)
//    -> one launch for up to four fields.
//
// Contract: every field that is not step scratch (fpk, cA, cB are not written in fused
// mode) ends bit-identical to the exact sequence.  Arithmetic per point is the
// same sequence of binary32 operations as te_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/thunderstep.h"
#include "te_flux.cuh"
#include "te_fused.cuh"
#include "te_math.cuh"
#include "te_player.hpp"

namespace te {

// ------------------------------------------------------------ acoustic K1

struct AcuArgs {
  Dims g;
  Acoustic a;
  const float *ppd, *thv, *uten, *vten, *hm;
  float *u, *v, *w, *rru, *rrv, *rrw;
  const float *piadv, *ppten, *ppterm, *pk1, *pk2, *qk, *mm, *wten;
  float *pp3d, *ppdw, *ppx, *cA, *cB, *sbuf;
  float tavg;
  int saveX;
};

// u, v at (i, j, k) after acoustic_uv (acoustic_uv.wgsl:145-181); a point outside the
// update range keeps its value.
__device__ __forceinline__ float uv_u(const AcuArgs& A, int i, int j, int c) {
  const Dims& g = A.g;
  const float tem1 = (g.rdx * 1005.7f) * 0.5f;
  return fmaf(A.a.dts, fmaf(-((tem1 * (A.ppd[c] - A.ppd[c - 1])) * hm_uf(g, A.hm, i)), A.thv[c] + A.thv[c - 1], A.uten[c]),
              A.u[c]);
}
__device__ __forceinline__ float uv_v(const AcuArgs& A, int i, int j, int c) {
  const Dims& g = A.g;
  const float tem2 = (g.rdy * 1005.7f) * 0.5f;
  const int sj = g.sJ;
  return fmaf(A.a.dts, fmaf(-((tem2 * (A.ppd[c] - A.ppd[c - sj])) * hm_vf(g, A.hm, j)), A.thv[c] + A.thv[c - sj], A.vten[c]),
              A.v[c]);
}

// Exact unsigned division by a divisor d >= 2 fixed for a launch: q = floor(n * m / 2^64)
// with m = floor(2^64 / d) + 1 equals floor(n / d) for every n < 2^32 (the error term
// n (m - 2^64/d) / 2^64 is below 2^-32, less than the distance 1/d from n/d to the
// next integer).
struct FastDiv {
  unsigned long long m;
  unsigned d;
};
static FastDiv fast_div(unsigned d) { return FastDiv{~0ull / d + 1ull, d}; }
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) { return (unsigned)__umul64hi(n, f.m); }

// K1: every point of the field (halos and k = nz included, as acoustic_accumulate):
// u, v updated where acoustic_uv updates them, then rru += u, rrv += v (averaged on the
// last substep, acoustic_accumulate.wgsl:129-158).  The points are numbered by their
// linear index c (the field's word offset) and thread t takes c = t + q S, q < kUvLevels
// (S a multiple of 32), so every warp reads and writes whole aligned 128-byte lines of
// each field rather than a row segment straddling two (measured at 256x256x80: 51.5 us
// per launch against 57.8 us for 32 x 8 blocks of two levels per thread); (i, j, k)
// follow from c by exact division.  A thread issues all its loads before its first store
// (the points are distinct, so nothing it stores is read by it or by another thread).
// Row padding of aligned-row layouts (x > nx + 6) belongs to no point.
#ifndef TE_UV_POINTS
#define TE_UV_POINTS 1   // points per thread (2 and 4 measured slower)
#endif
constexpr int kUvLevels = TE_UV_POINTS;

__global__ void __launch_bounds__(256) k_acu_uv_lin(AcuArgs A, FastDiv dJ, FastDiv dK, unsigned S, unsigned total) {
  const Dims& g = A.g;
  const unsigned t = blockIdx.x * 256u + threadIdx.x;
  if (t >= S) return;  // every point is some thread's t + q S
  float un[kUvLevels], vn[kUvLevels], ru[kUvLevels], rv[kUvLevels];
  bool on[kUvLevels], upd[kUvLevels];
#pragma unroll
  for (int q = 0; q < kUvLevels; q++) {
    const unsigned c = t + q * S;
    const unsigned kk = fdiv(c, dK);                 // level (dK: sJ * sK)
    const unsigned r = c - kk * dK.d;
    const unsigned jj = fdiv(r, dJ);                 // row (dJ: sJ)
    const int x = (int)(r - jj * dJ.d);
    const int i = x - 3, j = (int)jj - 3, k = (int)kk;
    on[q] = c < total && x <= g.nx + 6 && j <= g.ny + 3;
    upd[q] = on[q] && i >= 0 && j >= 0 && i <= g.nx && j <= g.ny && k < g.nz;
    if (on[q]) {
      un[q] = upd[q] ? uv_u(A, i, j, (int)c) : A.u[c];
      vn[q] = upd[q] ? uv_v(A, i, j, (int)c) : A.v[c];
      ru[q] = A.rru[c];
      rv[q] = A.rrv[c];
    }
  }
#pragma unroll
  for (int q = 0; q < kUvLevels; q++) {
    if (!on[q]) continue;
    const unsigned c = t + q * S;
    if (upd[q]) {
      A.u[c] = un[q];
      A.v[c] = vn[q];
    }
    if (A.tavg > 0.0f) {
      A.rru[c] = (ru[q] + un[q]) * A.tavg;
      A.rrv[c] = (rv[q] + vn[q]) * A.tavg;
    } else {
      A.rru[c] = ru[q] + un[q];
      A.rrv[c] = rv[q] + vn[q];
    }
  }
}

static void launch_acu_uv(const AcuArgs& A, cudaStream_t s) {
  const Dims& g = A.g;
  const unsigned total = (unsigned)g.sJ * (unsigned)g.sK * (unsigned)(g.nz + 1);
  const unsigned S = ((total + kUvLevels - 1) / kUvLevels + 31u) / 32u * 32u;
  launch_kernel(k_acu_uv_lin, dim3((S + 255u) / 256u), dim3(256), 0, s, A, fast_div((unsigned)g.sJ),
                fast_div((unsigned)g.sJ * (unsigned)g.sK), S, total);
}

// ------------------------------------------------------------ acoustic K2

// Explicit pi' forcing at an interior point (acoustic_fpk.wgsl:167-207).
__device__ __forceinline__ float fpk_at(const AcuArgs& A, int i, int j, int c, const float* w_old) {
  const Dims& g = A.g;
  const Acoustic& a = A.a;
  const int sj = g.sJ, sk = g.sJ * g.sK;
  const float temx = (a.dts * 0.5f) * g.rdx;
  const float temy = (a.dts * 0.5f) * g.rdy;
  const float *u = A.u, *v = A.v, *piadv = A.piadv;
  float div = fmaf((u[c + 1] - u[c]) * g.rdx, hm_uh(g, A.hm, i), ((v[c + sj] - v[c]) * g.rdy) * hm_vh(g, A.hm, j));
  if (fabsf(div) < a.smeps) div = 0.0f;
  float advPi = fmaf((-fmaf(u[c], piadv[c] - piadv[c - 1], u[c + 1] * (piadv[c + 1] - piadv[c]))) * temx, hm_uh(g, A.hm, i),
                     -((fmaf(v[c], piadv[c] - piadv[c - sj], v[c + sj] * (piadv[c + sj] - piadv[c])) * temy) * hm_vh(g, A.hm, j)));
  return fmaf(a.beta, fmaf(w_old[c], A.pk1[c] + A.qk[c], w_old[c + sk] * (A.pk2[c] - A.qk[c])),
              fmaf(a.dts, fmaf(-A.ppterm[c], div, A.ppten[c]), advPi));
}

// K2: a CTA owns 32 interior columns (i0..i0+31, row j) and runs their implicit w-pi'
// solve with warp specialisation.  kLevels worker warps (one level each per pass) load
// the 19 inputs of their level, form fpk (acoustic_fpk.wgsl:167-207) and the tridiagonal
// coefficients aa, bb, cc, dd of the level (lam_1, acoustic_w_solve.wgsl:124-139) into a
// double-buffered pass store; the recurrence warp (one lane per column) runs the
// sequential Thomas forward recurrence over the previous pass while the workers prepare
// the next one, then back-substitutes w.  Shared memory holds only cA, cB and
// s = pi' + fpk for the whole column (3 nz floats per column): the level-(k-1) values
// the coefficients need come through a per-pass exchange store, and the pi' update
// (acoustic_pp.wgsl:131-167) re-reads pk1, qk, pk2 and pi' — those loads, with rrw, are
// issued before the back substitution so that their latency overlaps it.  Finally the
// workers store pi', ppd, ppx, w and accumulate rrw (acoustic_accumulate.wgsl:129-158)
// for levels 0..nz.  Every value is produced by the same binary32 operations as the
// per-dispatch kernels; sums the reference forms twice (pk1+qk, pp3d+fpk, ...) are formed
// with the same rounding each time.
//
// Sized for three resident CTAs per SM (416 threads, 52 KB of shared memory at nz = 80):
// more columns in flight hide the per-pass load latency better than a deeper pass.
#ifndef TE_COL_LEVELS
#define TE_COL_LEVELS 12   // worker warps = levels per pass
#endif
#ifndef TE_COL_MINB
#define TE_COL_MINB 3      // resident CTAs per SM the register budget is sized for
#endif
#ifndef TE_COL_EPI
#define TE_COL_EPI 7       // epilogue levels per worker per chunk
#endif
constexpr int kColTile = 32;
constexpr int kLevels = TE_COL_LEVELS;
constexpr int kWorkers = kColTile * kLevels;     // 384
constexpr int kColThreads = kWorkers + kColTile; // + the recurrence warp
constexpr int kEpiChunk = TE_COL_EPI;

// [nz][32] cA, cB, s; [2][4][kLevels][32] aa, bb, cc, dd per pass; [2][3][kLevels][32]
// the exchange store (pk1 + qk, pk2 - qk, pi') per pass
static size_t col_smem_bytes(int nz) { return (size_t)(3 * nz + 14 * kLevels) * kColTile * sizeof(float); }

__device__ __forceinline__ int co_at(int b, int term, int q, int lane) {
  return ((b * 4 + term) * kLevels + q) * kColTile + lane;
}
__device__ __forceinline__ int xs_at(int b, int term, int q, int lane) {
  return ((b * 3 + term) * kLevels + q) * kColTile + lane;
}

__device__ __forceinline__ void workers_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kWorkers) : "memory");
}
// The CTA-wide barrier; workers and the recurrence warp reach it from separate code paths
// (whole warps each), the same number of times.
__device__ __forceinline__ void block_sync() { asm volatile("bar.sync 0;" ::: "memory"); }

// The 19 inputs of one level of one column, loaded ahead of use.
struct LevelIn {
  float u0, u1, v0, v1, pa0, paw, pae, pas, pan, ppten, ppterm, pk1, pk2, qk, w0, w1, pp, mm, wt;
};

__device__ __forceinline__ LevelIn load_level(const AcuArgs& A, int c) {
  const int sj = A.g.sJ, sk = A.g.sJ * A.g.sK;
  LevelIn L;
  L.u0 = A.u[c];
  L.u1 = A.u[c + 1];
  L.v0 = A.v[c];
  L.v1 = A.v[c + sj];
  L.pa0 = __ldg(A.piadv + c);
  L.paw = __ldg(A.piadv + c - 1);
  L.pae = __ldg(A.piadv + c + 1);
  L.pas = __ldg(A.piadv + c - sj);
  L.pan = __ldg(A.piadv + c + sj);
  L.ppten = __ldg(A.ppten + c);
  L.ppterm = __ldg(A.ppterm + c);
  L.pk1 = __ldg(A.pk1 + c);
  L.pk2 = __ldg(A.pk2 + c);
  L.qk = __ldg(A.qk + c);
  L.w0 = A.w[c];
  L.w1 = A.w[c + sk];
  L.pp = A.pp3d[c];
  L.mm = __ldg(A.mm + c);
  L.wt = __ldg(A.wten + c);
  return L;
}

// fpk from loaded values: the operations of acoustic_fpk.wgsl:167-207 in their order
__device__ __forceinline__ float fpk_of(const AcuArgs& A, const LevelIn& L, float uh, float vh) {
  const Dims& g = A.g;
  const Acoustic& a = A.a;
  const float temx = (a.dts * 0.5f) * g.rdx;
  const float temy = (a.dts * 0.5f) * g.rdy;
  float div = fmaf((L.u1 - L.u0) * g.rdx, uh, ((L.v1 - L.v0) * g.rdy) * vh);
  if (fabsf(div) < a.smeps) div = 0.0f;
  float advPi = fmaf((-fmaf(L.u0, L.pa0 - L.paw, L.u1 * (L.pae - L.pa0))) * temx, uh,
                     -((fmaf(L.v0, L.pa0 - L.pas, L.v1 * (L.pan - L.pa0)) * temy) * vh));
  return fmaf(a.beta, fmaf(L.w0, L.pk1 + L.qk, L.w1 * (L.pk2 - L.qk)), fmaf(a.dts, fmaf(-L.ppterm, div, L.ppten), advPi));
}

// Forward recurrence over one pass of kLevels levels (acoustic_w_solve.wgsl:150-190): the
// coefficients of four levels are read from the pass store before the chain reaches them.
__device__ __forceinline__ void forward_pass(const float* co, float* cA, float* cB, int pp, int nz, int lane, float& cAm,
                                             float& cBm, float& wtop) {
  const int b = pp & 1, base = pp * kLevels;
  float ca[4], cb[4], cc[4], cd[4];
#pragma unroll
  for (int t = 0; t < 4; t++) {
    ca[t] = co[co_at(b, 0, t, lane)];
    cb[t] = co[co_at(b, 1, t, lane)];
    cc[t] = co[co_at(b, 2, t, lane)];
    cd[t] = co[co_at(b, 3, t, lane)];
  }
#pragma unroll
  for (int g4 = 0; g4 < kLevels / 4; g4++) {
    float na[4], nb[4], nc[4], nd[4];
    if (g4 + 1 < kLevels / 4) {
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const int qq = 4 * (g4 + 1) + t;
        na[t] = co[co_at(b, 0, qq, lane)];
        nb[t] = co[co_at(b, 1, qq, lane)];
        nc[t] = co[co_at(b, 2, qq, lane)];
        nd[t] = co[co_at(b, 3, qq, lane)];
      }
    }
    float oA[4], oB[4];
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int kk = base + 4 * g4 + t;
      if (kk == 1) {
        const float r = dcr(1.0f, cb[t]);
        cAm = (-cc[t]) * r;
        cBm = cd[t] * r;
      } else if (kk >= 2 && kk < nz - 1) {
        const float r = dcr(1.0f, fmaf(ca[t], cAm, cb[t]));
        const float cAk = (-cc[t]) * r, cBk = fmaf(-ca[t], cBm, cd[t]) * r;
        cAm = cAk;
        cBm = cBk;
      } else if (kk == nz - 1) {
        const float r = dcr(1.0f, fmaf(ca[t], cAm, cb[t]));
        wtop = fmaf(-ca[t], cBm, cd[t]) * r;
      }
      oA[t] = cAm;
      oB[t] = cBm;
    }
#pragma unroll
    for (int t = 0; t < 4; t++) {
      const int kk = base + 4 * g4 + t;
      if (kk >= 1 && kk < nz - 1) {
        cA[kk * kColTile + lane] = oA[t];
        cB[kk * kColTile + lane] = oB[t];
      }
    }
    if (g4 + 1 < kLevels / 4) {
#pragma unroll
      for (int t = 0; t < 4; t++) {
        ca[t] = na[t];
        cb[t] = nb[t];
        cc[t] = nc[t];
        cd[t] = nd[t];
      }
    }
  }
}

// Back substitution: w(k) overwrites cA(k); w(0) = w(nz) = 0.  Eight levels of cA, cB are
// read ahead of the chain.
__device__ __forceinline__ void back_substitute(float* cA, const float* cB, int nz, int lane, float wtop) {
  float wk1 = wtop;
  cA[(nz - 1) * kColTile + lane] = wtop;
  for (int k0 = nz - 2; k0 >= 1; k0 -= 8) {
    float xa[8], xb[8], wv[8];
#pragma unroll
    for (int t = 0; t < 8; t++) {
      const int k = k0 - t;
      if (k >= 1) {
        xa[t] = cA[k * kColTile + lane];
        xb[t] = cB[k * kColTile + lane];
      }
    }
#pragma unroll
    for (int t = 0; t < 8; t++) {
      if (k0 - t >= 1) {
        wv[t] = fmaf(xa[t], wk1, xb[t]);
        wk1 = wv[t];
      }
    }
#pragma unroll
    for (int t = 0; t < 8; t++) {
      const int k = k0 - t;
      if (k >= 1) cA[k * kColTile + lane] = wv[t];
    }
  }
  cA[lane] = 0.0f;
}

// The pi' update inputs of a worker's epilogue levels k0, k0 + kLevels, ...
struct EpiIn {
  float rr[kEpiChunk], pk1[kEpiChunk], qk[kEpiChunk], pk2[kEpiChunk], pp[kEpiChunk];
};

__device__ __forceinline__ void load_epi(const AcuArgs& A, EpiIn& E, int c0, int k0, int nz, int sk) {
#pragma unroll
  for (int t = 0; t < kEpiChunk; t++) {
    const int k = k0 + t * kLevels;
    if (k <= nz) {
      const int c = c0 + k * sk;
      E.rr[t] = A.rrw[c];
      if (k < nz) {
        E.pk1[t] = __ldg(A.pk1 + c);
        E.qk[t] = __ldg(A.qk + c);
        E.pk2[t] = __ldg(A.pk2 + c);
        E.pp[t] = A.pp3d[c];
      }
    }
  }
}

__global__ void __launch_bounds__(kColThreads, TE_COL_MINB) k_acu_column(AcuArgs A) {
  extern __shared__ float smem[];
  const Dims& g = A.g;
  const Acoustic& a = A.a;
  const int nz = g.nz;
  float* cA = smem;
  float* cB = smem + nz * kColTile;
  float* sS = smem + 2 * nz * kColTile;
  float* co = smem + 3 * nz * kColTile;
  float* xs = co + 8 * kLevels * kColTile;
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
  const int i = blockIdx.x * kColTile + lane;
  const int j = blockIdx.y;
  const bool col = i < g.nx;
  const int sk = g.sJ * g.sK;
  const int c0 = gidx(g, col ? i : 0, j, 0);
  const int npass = (nz + kLevels - 1) / kLevels;
  if (q == kLevels) {
    // recurrence warp: pass p - 1 while the workers prepare pass p, then the last pass
    // and the back substitution
    float cAm = 0.0f, cBm = 0.0f, wtop = 0.0f;
    for (int p = 0; p < npass; p++) {
      if (p >= 1 && col) forward_pass(co, cA, cB, p - 1, nz, lane, cAm, cBm, wtop);
      block_sync();
    }
    if (col) {
      forward_pass(co, cA, cB, npass - 1, nz, lane, cAm, cBm, wtop);
      back_substitute(cA, cB, nz, lane, wtop);
    }
    block_sync();
    return;
  }
  const float asq = a.alph * a.alph;
  const float uh = hm_uh(g, A.hm, col ? i : 0), vh = hm_vh(g, A.hm, j);
  for (int p = 0; p < npass; p++) {
    const int k = p * kLevels + q;
    const bool ok = col && k < nz;
    const int b = p & 1;
    float m = 0.0f, wt = 0.0f, w0 = 0.0f, vA = 0.0f, vB = 0.0f, vP = 0.0f, vS = 0.0f;
    if (ok) {
      const LevelIn cur = load_level(A, c0 + k * sk);
      const float fk = fpk_of(A, cur, uh, vh);
      vA = cur.pk1 + cur.qk;
      vB = cur.pk2 - cur.qk;
      vP = cur.pp;
      vS = cur.pp + fk;
      sS[k * kColTile + lane] = vS;
      xs[xs_at(b, 0, q, lane)] = vA;
      xs[xs_at(b, 1, q, lane)] = vB;
      xs[xs_at(b, 2, q, lane)] = vP;
      m = cur.mm;
      wt = cur.wt;
      w0 = cur.w0;
    }
    workers_sync();
    if (ok && k >= 1) {
      // level k - 1: the previous warp of this pass, or the last warp of the previous one
      const int bp = q > 0 ? b : b ^ 1, qp = q > 0 ? q - 1 : kLevels - 1;
      const float pA = xs[xs_at(bp, 0, qp, lane)], pB = xs[xs_at(bp, 1, qp, lane)], pP = xs[xs_at(bp, 2, qp, lane)];
      const float pS = sS[(k - 1) * kColTile + lane];
      co[co_at(b, 0, q, lane)] = (-asq) * (m * pA);
      co[co_at(b, 2, q, lane)] = (-asq) * ((-m) * vB);
      co[co_at(b, 1, q, lane)] = fmaf(-asq, m * ((-vA) + pB), 1.0f);
      const float fw = fmaf(a.dts, wt, a.beta * ((-m) * (vP - pP)));
      co[co_at(b, 3, q, lane)] = fmaf(a.alph, (-m) * (vS - pS), w0 + fw);
    }
    block_sync();
  }
  // the epilogue's first loads fly during the last forward pass and the back substitution
  EpiIn E;
  if (col) load_epi(A, E, c0, q, nz, sk);
  block_sync();
  if (!col) return;
  // pi' update and stores, levels q, q + kLevels, ... (acoustic_pp.wgsl:131-167,
  // acoustic_accumulate.wgsl:129-158)
  for (int k0 = q; k0 <= nz; k0 += kEpiChunk * kLevels) {
    if (k0 != q) load_epi(A, E, c0, k0, nz, sk);
#pragma unroll
    for (int t = 0; t < kEpiChunk; t++) {
      const int k = k0 + t * kLevels;
      if (k > nz) break;
      const int c = c0 + k * sk;
      if (k < nz) {
        const int e = k * kColTile + lane;
        const float vA = E.pk1[t] + E.qk[t], vB = E.pk2[t] - E.qk[t];
        const float wk = cA[e];
        const float wk1 = k + 1 < nz ? cA[e + kColTile] : 0.0f;
        float p = fmaf(a.alph, fmaf(wk, vA, wk1 * vB), sS[e]);
        if (fabsf(p) < a.smeps) p = 0.0f;
        A.pp3d[c] = p;
        const float dum1 = a.kdiv * (p - E.pp[t]);
        A.ppdw[c] = p + dum1;
        if (A.saveX != 0) A.ppx[c] = dum1;
        A.w[c] = wk;
        A.rrw[c] = A.tavg > 0.0f ? fmaf(wk, a.alph, E.rr[t]) * A.tavg : E.rr[t] + wk;
      } else {
        A.w[c] = 0.0f;
        A.rrw[c] = A.tavg > 0.0f ? fmaf(0.0f, a.alph, E.rr[t]) * A.tavg : E.rr[t] + 0.0f;
      }
    }
  }
}

static void launch_acu_column(const AcuArgs& A, cudaStream_t s) {
  const size_t bytes = col_smem_bytes(A.g.nz);
  if (opt_in_smem((const void*)k_acu_column, bytes) != cudaSuccess) return;  // error left pending
  dim3 b(kColThreads), gr((A.g.nx + kColTile - 1) / kColTile, A.g.ny);
  launch_kernel(k_acu_column, dim3(gr), dim3(b), bytes, s, A);
}

// ------------------------------------------------------------ periodic halos

struct HaloArgs {
  Dims g;
  float* f[4];
  int nf;
  // acoustic substep: before the fill, halo points accumulate w into rrw
  // (acoustic_accumulate covers halos with the values they hold before the fill)
  float* acc_w;
  float* acc_rrw;
  float tavg, alph;
};

// Final state of bc_periodic_x followed by bc_periodic_y (bc_periodic_x.wgsl,
// bc_periodic_y.wgsl): every halo point of levels 0..nz holds the interior value at
// (i mod nx, j mod ny).  Two kinds of warps:
//  * x-halo rows: one warp per (j, k) row, lane = (field, halo column) for the 7 halo
//    columns of up to 4 fields, so a row's reads and writes are a few sectors per warp;
//  * y-halo rows: one thread per interior column of the 7 halo rows, all fields.
// Every halo point is written by exactly one thread, after that thread has read what it
// needs (a halo point is never an interior point read by another thread).
constexpr int kHaloX = 7;
constexpr int kHaloLevels = 3;  // levels per thread: their loads are issued together

__global__ void __launch_bounds__(256) k_halo_periodic(HaloArgs H) {
  const Dims& g = H.g;
  const int k0 = blockIdx.y * kHaloLevels;
  const int sk = g.sJ * g.sK;
  const int xrows = g.sK;                       // x-halo rows of a level (j = -3 .. ny + 3)
  const int xwarps = (xrows + 7) / 8;           // blocks of 8 warps
  if ((int)blockIdx.x < xwarps) {
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    const int f = lane / kHaloX, col = lane % kHaloX;
    if (row >= xrows || f >= H.nf) return;
    const int j = row - 3;
    const int i = col < 3 ? col - 3 : g.nx + (col - 3);
    const int ii = ((i % g.nx) + g.nx) % g.nx, jj = ((j % g.ny) + g.ny) % g.ny;
    const int dst0 = gidx(g, i, j, 0), src0 = gidx(g, ii, jj, 0);
    const bool acc = H.acc_rrw && H.f[f] == H.acc_w;
    float v[kHaloLevels], wv[kHaloLevels], rr[kHaloLevels];
#pragma unroll
    for (int q = 0; q < kHaloLevels; q++) {
      if (k0 + q > g.nz) break;
      v[q] = H.f[f][src0 + (k0 + q) * sk];
      if (acc) {
        wv[q] = H.acc_w[dst0 + (k0 + q) * sk];
        rr[q] = H.acc_rrw[dst0 + (k0 + q) * sk];
      }
    }
#pragma unroll
    for (int q = 0; q < kHaloLevels; q++) {
      if (k0 + q > g.nz) break;
      const int dst = dst0 + (k0 + q) * sk;
      if (acc) H.acc_rrw[dst] = H.tavg > 0.0f ? fmaf(wv[q], H.alph, rr[q]) * H.tavg : rr[q] + wv[q];
      H.f[f][dst] = v[q];
    }
    return;
  }
  const int t = (blockIdx.x - xwarps) * blockDim.x + threadIdx.x;
  if (t >= kHaloX * g.nx) return;
  const int r = t / g.nx, i = t % g.nx;
  const int j = r < 3 ? r - 3 : g.ny + (r - 3);
  const int jj = ((j % g.ny) + g.ny) % g.ny;
  const int dst0 = gidx(g, i, j, 0), src0 = gidx(g, i, jj, 0);
  // all loads of the thread's levels before the first store
  float v[kHaloLevels][4], wv[kHaloLevels], rr[kHaloLevels];
#pragma unroll
  for (int q = 0; q < kHaloLevels; q++) {
    if (k0 + q > g.nz) break;
#pragma unroll
    for (int f = 0; f < 4; f++)
      if (f < H.nf) v[q][f] = H.f[f][src0 + (k0 + q) * sk];
    if (H.acc_rrw) {
      wv[q] = H.acc_w[dst0 + (k0 + q) * sk];
      rr[q] = H.acc_rrw[dst0 + (k0 + q) * sk];
    }
  }
#pragma unroll
  for (int q = 0; q < kHaloLevels; q++) {
    if (k0 + q > g.nz) break;
    const int dst = dst0 + (k0 + q) * sk;
    if (H.acc_rrw) H.acc_rrw[dst] = H.tavg > 0.0f ? fmaf(wv[q], H.alph, rr[q]) * H.tavg : rr[q] + wv[q];
#pragma unroll
    for (int f = 0; f < 4; f++)
      if (f < H.nf) H.f[f][dst] = v[q][f];
  }
}

static void launch_halo(const HaloArgs& H, cudaStream_t s) {
  const int xblocks = (H.g.sK + 7) / 8, yblocks = (kHaloX * H.g.nx + 255) / 256;
  dim3 b(256), gr(xblocks + yblocks, (H.g.nz + kHaloLevels) / kHaloLevels);
  launch_kernel(k_halo_periodic, dim3(gr), dim3(b), 0, s, H);
}

// ------------------------------------------------------------ planner helpers

enum SegKind { kExact = 0, kAcoustic = 1, kHalo = 2, kAdvect = 3 };

static bool is_name(const Op& o, const char* n) { return !o.copy && o.name == n; }

static bool same_dims(const Dims& a, const Dims& b) {
  return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.sJ == b.sJ && a.sK == b.sK && a.rdx == b.rdx &&
         a.rdy == b.rdy && a.rdz == b.rdz;
}
static bool same_acoustic(const Acoustic& a, const Acoustic& b) {
  return a.dts == b.dts && a.alph == b.alph && a.beta == b.beta && a.kdiv == b.kdiv && a.smeps == b.smeps;
}

// ------------------------------------------------------------ fused advection

// Advection of one variable (timestep.js:1629-1900): the three face-flux dispatches and
// adv_assemble, optionally followed by apply_thterm and rk_update, as one kernel.  The
// per-face arithmetic is face_* of te_flux.cuh and the assembly assemble_t, i.e. the
// per-dispatch kernels' own code; the fx, fy, fz fields are never read, and written only
// where a later op of the step reads them (then every face the flux dispatches write is
// stored once, by the tile that computes it).
enum FaceKind { kLin = 0, kStag, kWeno, kWenoUV, kWenoW };

struct AdvArgs {
  KArgs fx, fy, fz, as;              // bindings of the four dispatches
  int ilo, ihi, jlo, jhi, klo, khi;  // cells adv_assemble writes
  FaceRange rx, ry, rz;              // faces each flux dispatch produces
  int accumulate, write_dest;
  int open;                          // the tape has open lateral edges (adv_assemble's branches)
  float* dest;                       // adv_assemble's tendency output
  const float *div3d, *thterm;       // apply_thterm (null if not fused)
  const float* phiA;                 // rk_update (null if not fused)
  float* phi;
  float dttmp;
  float *fxo, *fyo, *fzo;            // flux outputs when a later op reads them (else null)
};

// Face (i, j, k) of direction DIR whose linear index c on the common grid g is known.
template <int KIND, int DIR, int ST>
__device__ __forceinline__ float adv_face(const KArgs& A, const Dims& g, int c, int k) {
  const int sa = DIR == 0 ? 1 : g.sJ;
  if (KIND == kLin) return DIR == 2 ? face_lin_z_c(A, g, c, k) : face_lin_h_c<DIR>(A, c, A.p[1], c, sa);
  if (KIND == kStag) return DIR == 2 ? face_stag_z_c<ST>(A, g, c, k) : face_stag_h_c<DIR, ST>(A, g, c, k, A.p[2], c, sa);
  if (KIND == kWeno) return DIR == 2 ? face_weno_z_c(A, g, c, k) : face_weno_h_c<DIR>(A, c, A.p[1], c, sa);
  if (KIND == kWenoUV)
    return DIR == 2 ? face_weno_uv_z_c<ST>(A, g, c, k) : face_weno_uv_h_c<DIR, ST>(A, g, c, A.p[2], c, sa);
  return DIR == 2 ? face_weno_w_z_c(A, g, c, k) : face_weno_w_h_c<DIR>(A, g, c, k, A.p[1], c, sa);
}

__device__ __forceinline__ bool in_range(const FaceRange& r, int i, int j, int k) {
  return i >= r.ilo && i <= r.ihi && j >= r.jlo && j <= r.jhi && k >= r.klo && k <= r.khi;
}
// the box [i0, i1] x [j0, j1] x [k0, k1] lies inside r
__device__ __forceinline__ bool box_in(const FaceRange& r, int i0, int i1, int j0, int j1, int k0, int k1) {
  return i0 >= r.ilo && i1 <= r.ihi && j0 >= r.jlo && j1 <= r.jhi && k0 >= r.klo && k1 <= r.khi;
}

constexpr int kAdvTX = 32, kAdvTY = 8;

// ST = |stagger| of the advected variable: cell (i, j, k) takes the faces i + dx and
// i + dx + 1 (dx = -1 along its own staggered axis, else 0), likewise in j and k.  A CTA
// covers a 32 x 8 tile of KZ consecutive levels and walks up them: per level the
// 33 x 8 x-faces and 32 x 9 y-faces of the tile are computed once into shared memory
// (double-buffered, one barrier per level; the faces beyond 256 by warps 0 and 1), and
// each cell computes the z-face above it, reusing the one below from the level before.
// KZ = 4 where the z-face is a WENO reconstruction of momentum (the saved face pays for
// the shorter grid), 2 for scalar WENO; KZ = 1 (most parallel) where faces are cheap.  Every index is
// formed once per thread on the assembly's grid (the four dispatches share it) and
// advanced by a level stride; a tile whose faces and cells all lie inside the dispatch
// ranges (all but the edge tiles) skips the per-face range tests.
#ifndef TE_ADV_KZ_FAST
#define TE_ADV_KZ_FAST 1   // levels per CTA, linear and staggered-linear kinds
#endif
#ifndef TE_ADV_KZ_WENO
#define TE_ADV_KZ_WENO 2   // levels per CTA, scalar WENO (158 -> 155 us per launch against 1)
#endif
#ifndef TE_ADV_KZ_WENO_MOM
#define TE_ADV_KZ_WENO_MOM 4   // levels per CTA, momentum WENO
#endif
#ifndef TE_ADV_MINB_FAST
#define TE_ADV_MINB_FAST 8   // resident CTAs per SM the register budget is sized for
#endif
#ifndef TE_ADV_MINB_WENO
#define TE_ADV_MINB_WENO 8
#endif
#ifndef TE_ADV_MINB_WENO_MOM
#define TE_ADV_MINB_WENO_MOM 6
#endif
template <int KIND>
struct AdvKZ {
  static constexpr int value = KIND == kWenoUV || KIND == kWenoW ? TE_ADV_KZ_WENO_MOM
                               : KIND == kWeno                   ? TE_ADV_KZ_WENO
                                                                 : TE_ADV_KZ_FAST;
};
template <int KIND>
struct AdvMinBlocks {
  static constexpr int value = KIND == kLin || KIND == kStag ? TE_ADV_MINB_FAST
                               : KIND == kWeno                 ? TE_ADV_MINB_WENO
                                                               : TE_ADV_MINB_WENO_MOM;
};

template <int KIND, int ST, bool FULL, bool OPEN>
__device__ __forceinline__ void adv_tile(const AdvArgs& A, float (*fxs)[kAdvTY][kAdvTX + 1], float (*fys)[kAdvTY + 1][kAdvTX]) {
  constexpr int kAdvKZ = AdvKZ<KIND>::value;
  constexpr int dx = ST == 2 ? -1 : 0, dy = ST == 3 ? -1 : 0, dz = ST == 4 ? -1 : 0;
  const Dims& g = A.as.g;
  const int sk = g.sJ * g.sK;
  const int lx = threadIdx.x, ly = threadIdx.y, t = ly * kAdvTX + lx;
  const int i0 = A.ilo + (int)blockIdx.x * kAdvTX, j0 = A.jlo + (int)blockIdx.y * kAdvTY;
  const int i = i0 + lx, j = j0 + ly;
  const int kb = A.klo + (int)blockIdx.z * kAdvKZ, ke = min(A.khi, kb + kAdvKZ - 1);
  const bool cell = FULL || (i <= A.ihi && j <= A.jhi);
  const int xr = t / (kAdvTX + 1), xq = t % (kAdvTX + 1);                       // x-face of this thread
  const int e2 = kAdvTX * kAdvTY + lx, xr2 = e2 / (kAdvTX + 1), xq2 = e2 % (kAdvTX + 1);  // 256..263, warp 0
  // level-0 indices: the cell, its x-face, y-face and the extra faces of warps 0 and 1
  const int cc0 = gidx(g, i, j, 0);
  const int cx0 = gidx(g, i0 + dx + xq, j0 + xr, 0), cy0 = gidx(g, i, j0 + dy + ly, 0);
  const int cx20 = gidx(g, i0 + dx + xq2, j0 + xr2, 0), cy20 = gidx(g, i, j0 + dy + kAdvTY, 0);
  float fzb = cell ? adv_face<KIND, 2, ST>(A.fz, g, cc0 + (kb + dz) * sk, kb + dz) : 0.0f;
  const int dvoff = assemble_dv_off<ST>(A.as);
  for (int k = kb, b = 0; k <= ke; k++, b ^= 1) {
    // the cell's own inputs first, so their loads overlap the face computations
    const int c = cc0 + k * sk;
    float sc = 0.0f, d0 = 0.0f, d1 = 0.0f, dst = 0.0f, dv3 = 0.0f, tht = 0.0f, pa = 0.0f;
    if (cell) {
      sc = A.as.p[2][c];
      d0 = A.as.p[6][c];
      d1 = A.as.p[6][c - dvoff];
      if (A.accumulate) dst = A.dest[c];
      if (A.thterm) {
        dv3 = A.div3d[c];
        tht = A.thterm[c];
      }
      if (A.phi) pa = A.phiA[c];
    }
    const int ko = k * sk;
    // a tile stores the faces it shares with the next tile only when there is none
    const bool last_x = i0 + kAdvTX > A.ihi, last_y = j0 + kAdvTY > A.jhi;
    if (FULL || in_range(A.rx, i0 + dx + xq, j0 + xr, k)) {
      const float f = adv_face<KIND, 0, ST>(A.fx, g, cx0 + ko, k);
      fxs[b][xr][xq] = f;
      if (A.fxo && (xq < kAdvTX || last_x)) A.fxo[cx0 + ko] = f;
    }
    if (FULL || in_range(A.ry, i, j0 + dy + ly, k)) {
      const float f = adv_face<KIND, 1, ST>(A.fy, g, cy0 + ko, k);
      fys[b][ly][lx] = f;
      if (A.fyo) A.fyo[cy0 + ko] = f;
    }
    if (ly == 0 && lx < kAdvTY && (FULL || in_range(A.rx, i0 + dx + xq2, j0 + xr2, k))) {
      const float f = adv_face<KIND, 0, ST>(A.fx, g, cx20 + ko, k);
      fxs[b][xr2][xq2] = f;
      if (A.fxo && (xq2 < kAdvTX || last_x)) A.fxo[cx20 + ko] = f;
    }
    if (ly == 1 && (FULL || in_range(A.ry, i, j0 + dy + kAdvTY, k))) {
      const float f = adv_face<KIND, 1, ST>(A.fy, g, cy20 + ko, k);
      fys[b][kAdvTY][lx] = f;
      if (A.fyo && last_y) A.fyo[cy20 + ko] = f;
    }
    const float fzt = cell ? adv_face<KIND, 2, ST>(A.fz, g, c + (dz + 1) * sk, k + dz + 1) : 0.0f;
    if (A.fzo && cell) {
      A.fzo[c + (dz + 1) * sk] = fzt;
      if (k == A.klo) A.fzo[c + dz * sk] = fzb;  // the lowest face of the column
    }
    __syncthreads();
    // adv_assemble leaves the boundary faces of u (v) on an open x (y) edge alone: no
    // tendency there; a fused rk_update uses the tendency the field already holds
    const bool edge = !OPEN ? false
                    : ST == 2 ? A.as.iv[17] != 0 && (i == 0 || i == g.nx)
                    : ST == 3 ? A.as.iv2[17] != 0 && (j == 0 || j == g.ny) : false;
    if (cell && edge) {
      if (!A.accumulate && A.phi) A.phi[c] = fmaf(A.dttmp, A.dest[c], pa);   // rk_update.wgsl
    } else if (cell) {
      const float dFx = fxs[b][ly][lx + 1] - fxs[b][ly][lx];
      const float dFy = fys[b][ly + 1][lx] - fys[b][ly][lx];
      // adv_assemble, with its open-boundary branches where the tape has open edges
      float dv = assemble_dv<ST>(A.as, k, d0, d1), gx = dFx, gy = dFy;
      if (OPEN) assemble_open<ST>(A.as, i, j, k, c, gx, gy, dv);
      float tn = assemble_core<ST>(A.as, i, j, k, sc, dv, gx, gy, fzt - fzb);
      if (A.accumulate) {
        A.dest[c] = dst + tn;
      } else {
        if (A.thterm) tn = fmaf(-dv3, tht, tn);                 // apply_thterm.wgsl
        if (A.write_dest) A.dest[c] = tn;
        if (A.phi) A.phi[c] = fmaf(A.dttmp, tn, pa);            // rk_update.wgsl
      }
    }
    fzb = fzt;
  }
}

// OPEN: the tape has open lateral edges (adv_assemble's open branches compiled in)
template <int KIND, int ST, bool OPEN>
__global__ void __launch_bounds__(kAdvTX* kAdvTY, AdvMinBlocks<KIND>::value) k_adv_fused(AdvArgs A) {
  constexpr int kAdvKZ = AdvKZ<KIND>::value;
  constexpr int dx = ST == 2 ? -1 : 0, dy = ST == 3 ? -1 : 0, dz = ST == 4 ? -1 : 0;
  __shared__ float fxs[2][kAdvTY][kAdvTX + 1];
  __shared__ float fys[2][kAdvTY + 1][kAdvTX];
  const int i0 = A.ilo + (int)blockIdx.x * kAdvTX, j0 = A.jlo + (int)blockIdx.y * kAdvTY;
  const int kb = A.klo + (int)blockIdx.z * kAdvKZ, ke = min(A.khi, kb + kAdvKZ - 1);
  const int i1 = i0 + kAdvTX - 1, j1 = j0 + kAdvTY - 1;
  const bool full = i1 <= A.ihi && j1 <= A.jhi && box_in(A.rx, i0 + dx, i1 + dx + 1, j0, j1, kb, ke) &&
                    box_in(A.ry, i0, i1, j0 + dy, j1 + dy + 1, kb, ke) && box_in(A.rz, i0, i1, j0, j1, kb + dz, ke + dz + 1);
  if (full)
    adv_tile<KIND, ST, true, OPEN>(A, fxs, fys);
  else
    adv_tile<KIND, ST, false, OPEN>(A, fxs, fys);
}

template <int KIND, int ST>
static void launch_adv_t(const AdvArgs& A, cudaStream_t s) {
  const dim3 b(kAdvTX, kAdvTY, 1);
  constexpr int kz = AdvKZ<KIND>::value;
  const dim3 gr((A.ihi - A.ilo + kAdvTX) / kAdvTX, (A.jhi - A.jlo + kAdvTY) / kAdvTY, (A.khi - A.klo + kz) / kz);
  if (A.open)
    launch_kernel(k_adv_fused<KIND, ST, true>, dim3(gr), dim3(b), 0, s, A);
  else
    launch_kernel(k_adv_fused<KIND, ST, false>, dim3(gr), dim3(b), 0, s, A);
}

static void launch_adv(const AdvArgs& A, int kind, int st, cudaStream_t s) {
  switch (kind * 10 + st) {
    case kLin * 10 + 1: launch_adv_t<kLin, 1>(A, s); break;
    case kWeno * 10 + 1: launch_adv_t<kWeno, 1>(A, s); break;
    case kStag * 10 + 2: launch_adv_t<kStag, 2>(A, s); break;
    case kStag * 10 + 3: launch_adv_t<kStag, 3>(A, s); break;
    case kStag * 10 + 4: launch_adv_t<kStag, 4>(A, s); break;
    case kWenoUV * 10 + 2: launch_adv_t<kWenoUV, 2>(A, s); break;
    case kWenoUV * 10 + 3: launch_adv_t<kWenoUV, 3>(A, s); break;
    case kWenoW * 10 + 4: launch_adv_t<kWenoW, 4>(A, s); break;
    default: throw std::runtime_error("fused advection: no kernel for this flux kind / stagger");
  }
}

struct FluxNames {
  const char *x, *y, *z;
  int kind;
  int out_h, out_z;  // output binding of the horizontal / vertical flux dispatches
  int src;           // binding of the advected field
};
static const FluxNames kFluxSets[] = {
    {"adv_flux_x", "adv_flux_y", "adv_flux_z", kLin, 3, 5, 1},
    {"adv_flux_x_stag", "adv_flux_y_stag", "adv_flux_z_stag", kStag, 8, 8, 2},
    {"adv_flux_x_weno", "adv_flux_y_weno", "adv_flux_z_weno", kWeno, 5, 8, 1},
    {"adv_flux_x_weno_uv", "adv_flux_y_weno_uv", "adv_flux_z_weno_uv", kWenoUV, 5, 7, 2},
    {"adv_flux_x_weno_w", "adv_flux_y_weno_w", "adv_flux_z_weno_w", kWenoW, 5, 4, 1},
};

// Face indices a flux dispatch writes: its dispatch grid mapped to indices (the staggered
// horizontal kernels start at -1), cut by the kernel's own range check (te_kernels.cu).
static FaceRange flux_range(int kind, int dir, const Op& o) {
  const Dims& g = o.args.g;
  const bool centred = kind == kLin || kind == kWeno;
  const int off = !centred && dir != 2 ? -1 : 0;
  FaceRange r;
  r.ilo = off;
  r.jlo = off;
  r.klo = 0;
  r.ihi = o.grid[0] - 1 + off;
  r.jhi = o.grid[1] - 1 + off;
  r.khi = o.grid[2] - 1;
  int gi, gj, gk;
  if (dir == 0) { gi = g.nx; gj = centred ? g.ny - 1 : g.ny; gk = g.nz - 1; }
  else if (dir == 1) { gi = centred ? g.nx - 1 : g.nx; gj = g.ny; gk = g.nz - 1; }
  else { gi = centred ? g.nx - 1 : g.nx; gj = centred ? g.ny - 1 : g.ny; gk = g.nz; }
  if (kind == kWenoW && dir != 2) {
    r.ilo = std::max(r.ilo, 0);
    r.jlo = std::max(r.jlo, 0);
  }
  r.ihi = std::min(r.ihi, gi);
  r.jhi = std::min(r.jhi, gj);
  r.khi = std::min(r.khi, gk);
  return r;
}

static bool covers(const FaceRange& r, int ilo, int ihi, int jlo, int jhi, int klo, int khi) {
  return r.ilo <= ilo && r.ihi >= ihi && r.jlo <= jlo && r.jhi >= jhi && r.klo <= klo && r.khi >= khi;
}

static bool references(const Op& o, const float* f) {
  if (o.copy || !o.spec) return false;
  for (int q = 0; q < o.spec->nparams; q++)
    if (o.spec->params[q].kind == kPtr && o.args.p[o.spec->params[q].index] == f) return true;
  return false;
}

// Does op o overwrite f everywhere it matters without reading it first?  Only the
// flux kernels (their output binding) and adv_assemble without accumulation (its
// tendency) are known to; any other kernel that names f counts as a reader.
static bool writes_first(const Op& o, const float* f) {
  const std::string& n = o.name;
  for (auto& fs : kFluxSets) {
    const bool h = n == fs.x || n == fs.y, z = n == fs.z;
    if (!h && !z) continue;
    const int out = h ? fs.out_h : fs.out_z;
    for (int q = 0; q < o.spec->nparams; q++) {
      const ParamSpec& ps = o.spec->params[q];
      if (ps.kind == kPtr && ps.index != out && o.args.p[ps.index] == f) return false;
    }
    return o.args.p[out] == f;
  }
  if (n == "adv_assemble" && o.args.iv[12] == 0) {
    for (int q = 0; q < o.spec->nparams; q++) {
      const ParamSpec& ps = o.spec->params[q];
      if (ps.kind == kPtr && ps.index != 11 && o.args.p[ps.index] == f) return false;
    }
    return o.args.p[11] == f;
  }
  return false;
}

// The values ops [first, last] leave in field f are never read afterwards: scanning the
// step cyclically from last + 1 (steps repeat), f is next fully rewritten by a kernel
// that does not read it, or never named again.
static bool dead_after(const std::vector<Op>& ops, int first, int last, const float* f, uint32_t* M) {
  const int n = (int)ops.size();
  for (int s = 1; s < n; s++) {
    const int q = (last + s) % n;
    if (q >= first && q <= last) break;
    const Op& o = ops[q];
    if (o.copy) {  // a blit that touches f: not proven dead
      const float *s0 = reinterpret_cast<const float*>(M + o.src), *d0 = reinterpret_cast<const float*>(M + o.dst);
      if ((f >= s0 && f < s0 + o.n) || (f >= d0 && f < d0 + o.n)) return false;
      continue;
    }
    if (!references(o, f)) continue;
    return writes_first(o, f);
  }
  return true;
}

// flux_x, flux_y, flux_z of one kind on one field, then adv_assemble of their fluxes;
// optionally apply_thterm and rk_update of the fresh tendency.
static bool match_advect(const std::vector<Op>& ops, size_t i, uint32_t* M, FusedSegment& s, AdvArgs& A) {
  if (i + 4 > ops.size() || ops[i].copy) return false;
  const FluxNames* fs = nullptr;
  for (auto& c : kFluxSets)
    if (ops[i].name == c.x) fs = &c;
  if (!fs) return false;
  const Op &ox = ops[i], &oy = ops[i + 1], &oz = ops[i + 2], &oa = ops[i + 3];
  if (!is_name(oy, fs->y) || !is_name(oz, fs->z) || !is_name(oa, "adv_assemble")) return false;
  const Dims& g = oa.args.g;
  if (!same_dims(g, ox.args.g) || !same_dims(g, oy.args.g) || !same_dims(g, oz.args.g)) return false;
  if (g.nz < 3) return false;
  const int stag = oa.args.iv[1];
  if (stag < 1 || stag > 4) return false;
  if ((fs->kind == kLin || fs->kind == kWeno) && stag != 1) return false;
  if (fs->kind == kStag && stag == 1) return false;
  if (fs->kind == kWenoUV && stag != 2 && stag != 3) return false;
  if (fs->kind == kWenoW && stag != 4) return false;
  if (fs->kind == kStag || fs->kind == kWenoUV)
    if (ox.args.iv[1] != stag || oy.args.iv[1] != stag || oz.args.iv[1] != stag) return false;
  float* src = ox.args.p[fs->src];
  if (oy.args.p[fs->src] != src || oz.args.p[fs->src] != src || oa.args.p[2] != src) return false;
  float *fx = ox.args.p[fs->out_h], *fy = oy.args.p[fs->out_h], *fz = oz.args.p[fs->out_z];
  if (oa.args.p[3] != fx || oa.args.p[4] != fy || oa.args.p[5] != fz) return false;
  if (fx == fy || fx == fz || fy == fz) return false;
  std::memset(&A, 0, sizeof(A));
  A.fx = ox.args;
  A.fy = oy.args;
  A.fz = oz.args;
  A.as = oa.args;
  A.ilo = 0;
  A.ihi = stag == 2 ? g.nx : g.nx - 1;
  A.jlo = 0;
  A.jhi = stag == 3 ? g.ny : g.ny - 1;
  A.klo = stag == 4 ? 1 : 0;
  A.khi = g.nz - 1;
  if (oa.grid[0] <= A.ihi || oa.grid[1] <= A.jhi || oa.grid[2] <= A.khi) return false;
  A.rx = flux_range(fs->kind, 0, ox);
  A.ry = flux_range(fs->kind, 1, oy);
  A.rz = flux_range(fs->kind, 2, oz);
  const int dx = stag == 2 ? -1 : 0, dy = stag == 3 ? -1 : 0, dz = stag == 4 ? -1 : 0;
  if (!covers(A.rx, A.ilo + dx, A.ihi + dx + 1, A.jlo, A.jhi, A.klo, A.khi)) return false;
  if (!covers(A.ry, A.ilo, A.ihi, A.jlo + dy, A.jhi + dy + 1, A.klo, A.khi)) return false;
  if (!covers(A.rz, A.ilo, A.ihi, A.jlo, A.jhi, A.klo + dz, A.khi + dz + 1)) return false;
  A.accumulate = oa.args.iv[12] != 0;
  A.open = oa.args.iv[17] != 0 || oa.args.iv2[17] != 0;
  A.dest = oa.args.p[11];
  A.write_dest = 1;
  // fields the kernel reads at other cells than the one it writes: nothing it writes may
  // be among them
  std::vector<const float*> reads;
  for (int b = 0; b < kMaxBind; b++) {
    if (b != fs->out_h && A.fx.p[b]) reads.push_back(A.fx.p[b]);
    if (b != fs->out_h && A.fy.p[b]) reads.push_back(A.fy.p[b]);
    if (b != fs->out_z && A.fz.p[b]) reads.push_back(A.fz.p[b]);
    if (b != 11 && b != 19 && A.as.p[b]) reads.push_back(A.as.p[b]);
  }
  auto is_read = [&](const float* f) {
    for (auto* r : reads)
      if (r == f) return true;
    return false;
  };
  if (is_read(A.dest)) return false;
  int last = (int)i + 3;
  if (!A.accumulate) {
    size_t q = i + 4;
    if (stag == 1 && q < ops.size() && is_name(ops[q], "apply_thterm") && ops[q].args.p[3] == A.dest &&
        same_dims(g, ops[q].args.g) && ops[q].grid[0] >= g.nx && ops[q].grid[1] >= g.ny && ops[q].grid[2] >= g.nz &&
        ops[q].args.p[1] != A.dest && ops[q].args.p[2] != A.dest && !is_read(ops[q].args.p[3])) {
      A.div3d = ops[q].args.p[1];
      A.thterm = ops[q].args.p[2];
      q++;
    }
    if (q < ops.size() && is_name(ops[q], "rk_update") && ops[q].args.p[3] == A.dest && ops[q].args.iv[1] == stag &&
        same_dims(g, ops[q].args.g) && ops[q].grid[0] > A.ihi && ops[q].grid[1] > A.jhi && ops[q].grid[2] > A.khi) {
      float* phi = ops[q].args.p[4];
      const float* phiA = ops[q].args.p[2];
      bool clash = is_read(phi) || phi == A.dest || phiA == A.dest || phi == fx || phi == fy || phi == fz;
      if (A.thterm) clash |= A.div3d == phi || A.thterm == phi;
      if (!clash) {
        A.phi = phi;
        A.phiA = phiA;
        A.dttmp = ops[q].args.f[5];
        last = (int)q;
      }
    }
    if (A.thterm && !A.phi) return false;  // apply_thterm only together with its rk_update
    if (A.phi) A.write_dest = dead_after(ops, (int)i, last, A.dest, M) ? 0 : 1;
  }
  bool live = false;
  for (float* f : {fx, fy, fz}) live |= !dead_after(ops, (int)i, last, f, M);
  if (live) {
    // a later op reads the fluxes: the kernel stores them, which is the flux dispatches'
    // result only if they write exactly the faces the tiles compute and read none of them
    if (!(A.rx.ilo == A.ilo + dx && A.rx.ihi == A.ihi + dx + 1 && A.rx.jlo == A.jlo && A.rx.jhi == A.jhi &&
          A.rx.klo == A.klo && A.rx.khi == A.khi))
      return false;
    if (!(A.ry.ilo == A.ilo && A.ry.ihi == A.ihi && A.ry.jlo == A.jlo + dy && A.ry.jhi == A.jhi + dy + 1 &&
          A.ry.klo == A.klo && A.ry.khi == A.khi))
      return false;
    if (!(A.rz.ilo == A.ilo && A.rz.ihi == A.ihi && A.rz.jlo == A.jlo && A.rz.jhi == A.jhi &&
          A.rz.klo == A.klo + dz && A.rz.khi == A.khi + dz + 1))
      return false;
    for (float* f : {fx, fy, fz}) {
      for (int b = 0; b < kMaxBind; b++) {
        if ((b != fs->out_h && A.fx.p[b] == f) || (b != fs->out_h && A.fy.p[b] == f) || (b != fs->out_z && A.fz.p[b] == f))
          return false;
        if (b != 3 && b != 4 && b != 5 && b != 11 && b != 19 && A.as.p[b] == f) return false;
      }
      if (f == A.dest || f == A.phi || f == A.phiA || f == A.div3d || f == A.thterm) return false;
    }
    A.fxo = fx;
    A.fyo = fy;
    A.fzo = fz;
  }
  s.kind = kAdvect;
  s.first = (int)i;
  s.last = last;
  s.aux[1] = fs->kind;
  s.aux[2] = stag;
  return true;
}

// ------------------------------------------------------------ planner


// bc_periodic_x(f) followed by bc_periodic_y(f) over the standard halo grid
static bool halo_pair(const std::vector<Op>& ops, size_t i, float** f) {
  if (i + 1 >= ops.size()) return false;
  const Op &x = ops[i], &y = ops[i + 1];
  if (!is_name(x, "bc_periodic_x") || !is_name(y, "bc_periodic_y")) return false;
  const Dims& g = x.args.g;
  if (!same_dims(g, y.args.g) || x.args.p[1] != y.args.p[1]) return false;
  if (x.grid[0] != 4 || x.grid[1] != g.ny + 7 || x.grid[2] != g.nz + 1) return false;
  if (y.grid[0] != 4 || y.grid[1] != g.nx + 7 || y.grid[2] != g.nz + 1) return false;
  *f = x.args.p[1];
  return true;
}

bool periodic_halo_pair(const std::vector<Op>& ops, size_t i, float** f) { return halo_pair(ops, i, f); }

void launch_periodic_halos(const Dims& g, float* const* f, int nf, cudaStream_t s) {
  HaloArgs H;
  std::memset(&H, 0, sizeof H);
  H.g = g;
  H.nf = nf;
  for (int q = 0; q < nf && q < 4; q++) H.f[q] = f[q];
  launch_halo(H, s);
}

static const char* kSubstep[] = {"acoustic_uv", "acoustic_fpk", "acoustic_w_solve", "acoustic_pp"};

static bool match_substep(const std::vector<Op>& ops, size_t i, FusedSegment& s, AcuArgs& A) {
  if (i + 13 > ops.size()) return false;
  for (int q = 0; q < 4; q++)
    if (!is_name(ops[i + q], kSubstep[q])) return false;
  const Op &uv = ops[i], &fp = ops[i + 1], &ws = ops[i + 2], &pp = ops[i + 3];
  const Op& acc = ops[i + 6];
  if (!is_name(acc, "acoustic_accumulate")) return false;
  const Dims& g = uv.args.g;
  if (g.nx < 1 || g.ny < 1 || g.nz < 3 || col_smem_bytes(g.nz) > 200 * 1024)
    return false;
  for (const Op* o : {&fp, &ws, &pp, &acc})
    if (!same_dims(g, o->args.g) || !same_acoustic(uv.args.a, o->args.a)) return false;
  // periodic (closed) lateral boundaries only
  if (uv.args.iv[8] != 0 || uv.args.iv2[8] != 0) return false;
  // dispatch grids as the encoder emits them
  if (uv.grid[0] != g.nx + 1 || uv.grid[1] != g.ny + 1 || uv.grid[2] != g.nz) return false;
  for (const Op* o : {&fp, &pp})
    if (o->grid[0] != g.nx || o->grid[1] != g.ny || o->grid[2] != g.nz) return false;
  if (ws.grid[0] != g.nx || ws.grid[1] != g.ny || ws.grid[2] != 1) return false;
  if (acc.grid[0] != g.sJ || acc.grid[1] != g.sK || acc.grid[2] != g.nz + 1) return false;
  // bindings: one set of fields across the seven kernels
  float *ppd = uv.args.p[2], *u = uv.args.p[6], *v = uv.args.p[7];
  float* w = fp.args.p[4];
  float *pk1 = fp.args.p[8], *pk2 = fp.args.p[9], *qk = fp.args.p[10], *fpk = fp.args.p[11];
  bool ok = fp.args.p[2] == u && fp.args.p[3] == v && ws.args.p[2] == pk1 && ws.args.p[3] == pk2 && ws.args.p[4] == qk &&
            ws.args.p[6] == fpk && ws.args.p[9] == w && pp.args.p[2] == w && pp.args.p[3] == pk1 && pp.args.p[4] == pk2 &&
            pp.args.p[5] == qk && pp.args.p[6] == fpk && pp.args.p[7] == ws.args.p[8] && pp.args.p[8] == ppd &&
            acc.args.p[2] == u && acc.args.p[3] == v && acc.args.p[4] == w && uv.args.p[30] == fp.args.p[30];
  if (!ok) return false;
  // halo fills: ppd after pp, then u, v, w after the accumulation
  float* f;
  if (!halo_pair(ops, i + 4, &f) || f != ppd) return false;
  const float* want[3] = {u, v, w};
  for (int q = 0; q < 3; q++)
    if (!halo_pair(ops, i + 7 + 2 * q, &f) || f != want[q]) return false;
  // the three fields K2 uses for its intermediate values must be distinct scratch
  float *cA = ws.args.p[10], *cB = ws.args.p[11];
  if (cA == cB || cA == fpk || cB == fpk) return false;
  for (float* p : {ppd, u, v, w, pk1, pk2, qk, acc.args.p[5], acc.args.p[6], acc.args.p[7], pp.args.p[7], pp.args.p[9],
                   fp.args.p[5], fp.args.p[6], fp.args.p[7], ws.args.p[5], ws.args.p[7], uv.args.p[3], uv.args.p[4],
                   uv.args.p[5]})
    if (p == cA || p == cB || p == fpk) return false;
  std::memset(&A, 0, sizeof(A));
  A.g = g;
  A.a = uv.args.a;
  A.ppd = ppd;
  A.thv = uv.args.p[3];
  A.uten = uv.args.p[4];
  A.vten = uv.args.p[5];
  A.hm = uv.args.p[30];
  A.u = u;
  A.v = v;
  A.w = w;
  A.piadv = fp.args.p[5];
  A.ppten = fp.args.p[6];
  A.ppterm = fp.args.p[7];
  A.pk1 = pk1;
  A.pk2 = pk2;
  A.qk = qk;
  A.mm = ws.args.p[5];
  A.wten = ws.args.p[7];
  A.pp3d = ws.args.p[8];
  A.ppdw = ppd;
  A.ppx = pp.args.p[9];
  A.saveX = pp.args.iv[10];
  A.cA = cA;
  A.cB = cB;
  A.sbuf = fpk;
  A.rru = acc.args.p[5];
  A.rrv = acc.args.p[6];
  A.rrw = acc.args.p[7];
  A.tavg = acc.args.f[8];
  s.kind = kAcoustic;
  s.first = (int)i;
  s.last = (int)i + 12;
  return true;
}

struct FusedData {
  std::vector<AcuArgs> acu;
  std::vector<HaloArgs> halo;
  std::vector<AdvArgs> adv;
};

void FusedStep::build(Plan& P, std::vector<Op>& ops) {
  segs.clear();
  if (!data) data = new FusedData();
  FusedData& D = *static_cast<FusedData*>(data);
  D.acu.clear();
  D.halo.clear();
  D.adv.clear();
  size_t i = 0;
  auto exact_to = [&](size_t e) {
    if (!segs.empty() && segs.back().kind == kExact && segs.back().last + 1 == (int)i) segs.back().last = (int)e;
    else {
      FusedSegment s;
      s.kind = kExact;
      s.first = (int)i;
      s.last = (int)e;
      segs.push_back(s);
    }
  };
  while (i < ops.size()) {
    FusedSegment s;
    AcuArgs A;
    if (match_substep(ops, i, s, A)) {
      s.aux[0] = (int)D.acu.size();
      D.acu.push_back(A);
      segs.push_back(s);
      i += 13;
      continue;
    }
    AdvArgs V;
    if (match_advect(ops, i, P.M, s, V)) {
      s.aux[0] = (int)D.adv.size();
      D.adv.push_back(V);
      segs.push_back(s);
      i = s.last + 1;
      continue;
    }
    float* f;
    if (halo_pair(ops, i, &f)) {
      HaloArgs H;
      std::memset(&H, 0, sizeof(H));
      H.g = ops[i].args.g;
      H.f[0] = f;
      H.nf = 1;
      size_t e = i + 2;
      float* f2;
      while (H.nf < 4 && halo_pair(ops, e, &f2) && same_dims(H.g, ops[e].args.g)) {
        bool dup = false;
        for (int q = 0; q < H.nf; q++) dup |= H.f[q] == f2;
        if (dup) break;
        H.f[H.nf++] = f2;
        e += 2;
      }
      s.kind = kHalo;
      s.first = (int)i;
      s.last = (int)e - 1;
      s.aux[0] = (int)D.halo.size();
      D.halo.push_back(H);
      segs.push_back(s);
      i = e;
      continue;
    }
    exact_to(i);
    i++;
  }
}

void FusedStep::launch(Plan& P, std::vector<Op>& ops) {
  for (int q = 0; q < (int)segs.size(); q++) launch_segment(P, ops, q, -1);
}

void FusedStep::launch_segment(Plan& P, std::vector<Op>& ops, int seg, int part) {
  FusedData& D = *static_cast<FusedData*>(data);
  const FusedSegment& s = segs.at(seg);
  if (s.kind == kExact) {
    P.launch_exact(ops, s.first, s.last, false);
  } else if (s.kind == kHalo) {
    launch_halo(D.halo[s.aux[0]], P.stream);
  } else if (s.kind == kAdvect) {
    launch_adv(D.adv[s.aux[0]], s.aux[1], s.aux[2], P.stream);
  } else {
    const AcuArgs& A = D.acu[s.aux[0]];
    const Dims& g = A.g;
    if (part < 0 || part == 0) launch_acu_uv(A, P.stream);
    if (part < 0 || part == 1) launch_acu_column(A, P.stream);
    if (part < 0 || part == 2) {
      HaloArgs H;
      std::memset(&H, 0, sizeof(H));
      H.g = g;
      H.f[0] = A.ppdw;
      H.f[1] = A.u;
      H.f[2] = A.v;
      H.f[3] = A.w;
      H.nf = 4;
      H.acc_w = A.w;
      H.acc_rrw = A.rrw;
      H.tavg = A.tavg;
      H.alph = A.a.alph;
      launch_halo(H, P.stream);
    }
  }
}

int FusedStep::launches_per_step() const {
  if (!data) return 0;
  int n = 0;
  for (auto& s : segs) n += s.kind == kExact ? 0 : (s.kind == kAcoustic ? 3 : 1);
  return n;
}

void FusedStep::release() {
  segs.clear();
  delete static_cast<FusedData*>(data);
  data = nullptr;
}

}  // namespace te

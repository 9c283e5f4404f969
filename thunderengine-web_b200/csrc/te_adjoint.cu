// Discrete adjoint of a planned step (te_adjoint_* in include/thunderstep.h).
//
// The forward (te_adjoint_forward) runs N steps of the active step, keeping a copy of the
// tape buffers every K steps (checkpoints).  The backward (te_adjoint_backward) walks the
// blocks of K steps from the last: it restores the block's checkpoint and replays its steps
// op by op, saving every region an op is about to write into an undo log; then it walks the
// block's ops in reverse, restoring each op's written regions (so memory holds the values
// before the op, in every field an adjoint operator reads; regions of the others are not
// logged) and running the op's adjoint operator (te_adjoint.cuh), which turns the
// adjoints of the values after the op into the adjoints of the values before it.  At the
// end memory holds the state of step 0 and the adjoint memory the gradient with respect
// to it.  Each block position has its own CUDA graph for the logged replay and for the
// reverse walk, so a step costs two graph launches.
//
// The adjoint memory has the layout of the player's word memory: the adjoint of the value
// at word w is the float at word w.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/thunderstep.h"
#include "te_adjoint.cuh"
#include "te_fused.cuh"
#include "te_kernels.cuh"
#include "te_player.hpp"

namespace te {
namespace adj {

struct AccDevice {
  static constexpr bool skip_zero = false;
  __device__ static void add(float* p, float v) { atomicAdd(p, v); }
};

#define TE_ADJ_OP(Name, call)                                                           \
  struct Name {                                                                         \
    __device__ static void run(const AdjArgs<float>& A, int tx, int ty, int tz) { call; } \
  };

TE_ADJ_OP(OpFluxX, (adj_flux_lin_h<float, AccDevice>(A, tx, ty, tz, 0)))
TE_ADJ_OP(OpFluxY, (adj_flux_lin_h<float, AccDevice>(A, tx, ty, tz, 1)))
TE_ADJ_OP(OpFluxZ, (adj_flux_lin_z<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpStagX, (adj_flux_stag_h<float, AccDevice>(A, tx, ty, tz, 0)))
TE_ADJ_OP(OpStagY, (adj_flux_stag_h<float, AccDevice>(A, tx, ty, tz, 1)))
TE_ADJ_OP(OpStagZ, (adj_flux_stag_z<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpWenoX, (adj_flux_weno_h<float, AccDevice>(A, tx, ty, tz, 0)))
TE_ADJ_OP(OpWenoY, (adj_flux_weno_h<float, AccDevice>(A, tx, ty, tz, 1)))
TE_ADJ_OP(OpWenoZ, (adj_flux_weno_z<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpWenoUvX, (adj_flux_weno_uv_h<float, AccDevice>(A, tx, ty, tz, 0)))
TE_ADJ_OP(OpWenoUvY, (adj_flux_weno_uv_h<float, AccDevice>(A, tx, ty, tz, 1)))
TE_ADJ_OP(OpWenoUvZ, (adj_flux_weno_uv_z<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpWenoWX, (adj_flux_weno_w_h<float, AccDevice>(A, tx, ty, tz, 0)))
TE_ADJ_OP(OpWenoWY, (adj_flux_weno_w_h<float, AccDevice>(A, tx, ty, tz, 1)))
TE_ADJ_OP(OpWenoWZ, (adj_flux_weno_w_z<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpAssemble, (adj_assemble<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpRk, (adj_rk_update<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpThterm, (adj_apply_thterm<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpBuoy, (adj_buoyancy_apply<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpDiag, (adj_update_diagnostics_moist<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpTendReset, (adj_stage_tendency_reset<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpMassflux, (adj_massflux_from_state<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpDivMassflux, (adj_div_massflux<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpDiv3d, (adj_divergence3d<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpVelMassflux, (adj_velocity_to_massflux<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpSadv, (adj_build_sadv<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpStateReset, (adj_stage_state_reset<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpBegin, (adj_acoustic_begin<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpPrepare, (adj_acoustic_prepare<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpUv, (adj_acoustic_uv<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpFpk, (adj_acoustic_fpk<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpPp, (adj_acoustic_pp<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpAccum, (adj_acoustic_accumulate<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpHaloX, (adj_bc_periodic<float, AccDevice>(A, tx, ty, tz, 0)))
TE_ADJ_OP(OpHaloY, (adj_bc_periodic<float, AccDevice>(A, tx, ty, tz, 1)))
TE_ADJ_OP(OpPpxFinish, (adj_ppx_finish<float, AccDevice>(A, tx, ty, tz)))
TE_ADJ_OP(OpWSolve, (adj_acoustic_w_solve<float, AccDevice>(A, tx, ty, tz)))

// One thread per dispatch thread of the forward op (its grid in threads).
template <class Op>
__global__ void __launch_bounds__(128) k_adj(AdjArgs<float> A) {
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y * blockDim.y + threadIdx.y;
  const int tz = blockIdx.z;
  if (tx >= A.gx || ty >= A.gy || tz >= A.gz) return;
  Op::run(A, tx, ty, tz);
}

typedef void (*AdjLaunch)(const AdjArgs<float>&, cudaStream_t);

template <class Op>
static void launch_adj(const AdjArgs<float>& A, cudaStream_t s) {
  if (A.gx <= 0 || A.gy <= 0 || A.gz <= 0) return;
  launch_kernel(k_adj<Op>, dim3((A.gx + 31) / 32, (A.gy + 3) / 4, A.gz), dim3(32, 4, 1), 0, s, A);
}

// Per kernel: the adjoint operator and the bindings whose values BEFORE the op the
// operator reads (bit n = binding n).  Only fields some operator of the step reads need
// their overwritten values kept in the undo log.
// The halo operators' dispatch has 4 threads along x (the halo depth) per row: blocks of
// 4 x 32 (k_adj is compiled for 128 threads) keep every thread of a block busy.
template <class Op>
static void launch_adj_halo(const AdjArgs<float>& A, cudaStream_t s) {
  if (A.gx <= 0 || A.gy <= 0 || A.gz <= 0) return;
  launch_kernel(k_adj<Op>, dim3((A.gx + 3) / 4, (A.gy + 31) / 32, A.gz), dim3(4, 32, 1), 0, s, A);
}

// acoustic_w_solve, a block per 32 columns (lanes on consecutive i) and 8 warps: the rows
// of the transposed system T^T mu = lambda_w of all levels are formed level-parallel into
// shared memory, one warp runs the Thomas sweep of the 32 columns, and the 8 warps
// distribute mu level-parallel (each level's adjoint updates come from rows k and k + 1
// of its own column: no atomics).  The same operations as adj_acoustic_w_solve.
constexpr int kAdjCols = 32, kAdjWarps = 8;

__global__ void __launch_bounds__(kAdjCols * kAdjWarps) k_adj_wsolve_coop(AdjArgs<float> A) {
  extern __shared__ float asm_[];
  const Dims& g = A.g;
  const int nz = g.nz, sk = g.sJ * g.sK;
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int col = blockIdx.x * kAdjCols + lane;
  const bool on = col < g.nx * g.ny;
  const int c0 = gidx(g, on ? col % g.nx : 0, on ? col / g.nx : 0, 0);
  float* sSub = asm_;
  float* sDia = asm_ + nz * kAdjCols;
  float* sSup = asm_ + 2 * nz * kAdjCols;
  float* sRhs = asm_ + 3 * nz * kAdjCols;
  const float *pk1 = A.p[2], *pk2 = A.p[3], *qk = A.p[4], *mm = A.p[5];
  float *lfpk = A.l[6], *lwten = A.l[7], *lpp = A.l[8], *lw = A.l[9], *lcA = A.l[10], *lcB = A.l[11];
  const float alph = A.a.alph, beta = A.a.beta, dts = A.a.dts, asq = alph * alph;
  if (on)
    for (int k = 1 + wq; k <= nz - 1; k += kAdjWarps) {
      const int c = c0 + k * sk, e = k * kAdjCols + lane;
      const float Ak = pk1[c] + qk[c];
      const float Bm = pk2[c - sk] - qk[c - sk];
      const float m = mm[c];
      sDia[e] = fmaf(-asq, m * ((-Ak) + Bm), 1.0f);
      sSub[e] = k > 1 ? (-asq) * ((-mm[c - sk]) * Bm) : 0.0f;          // cc(k - 1)
      sSup[e] = k < nz - 1 ? (-asq) * (mm[c + sk] * Ak) : 0.0f;         // aa(k + 1)
      sRhs[e] = lw[c];
    }
  __syncthreads();
  if (wq == 0 && on) {
    // Thomas sweep of the transposed system: one correctly rounded reciprocal per level on
    // the serial chain instead of two divisions
    float cp = 0.0f, dp = 0.0f;
    for (int k = 1; k <= nz - 1; k++) {
      const int e = k * kAdjCols + lane;
      const float sub = sSub[e];
      const float r = __frcp_rn(sDia[e] - sub * cp);
      cp = sSup[e] * r;
      dp = (sRhs[e] - sub * dp) * r;
      sSup[e] = cp;
      sRhs[e] = dp;
    }
    float mu = 0.0f;
    for (int k = nz - 1; k >= 1; k--) {
      const int e = k * kAdjCols + lane;
      mu = sRhs[e] - sSup[e] * mu;
      sRhs[e] = mu;
    }
  }
  __syncthreads();
  if (!on) return;
  for (int k = wq; k <= nz; k += kAdjWarps) {
    const int c = c0 + k * sk;
    const float mu = (k >= 1 && k <= nz - 1) ? sRhs[k * kAdjCols + lane] : 0.0f;
    const float mu1 = (k + 1 <= nz - 1) ? sRhs[(k + 1) * kAdjCols + lane] : 0.0f;
    const float m = k <= nz - 1 ? mm[c] : 0.0f;
    const float m1 = k + 1 <= nz - 1 ? mm[c + sk] : 0.0f;
    if (k <= nz - 1) {
      lwten[c] += dts * mu;
      lpp[c] += mu * (beta * (-m) + alph * (-m)) - mu1 * (beta * (-m1) + alph * (-m1));
      lfpk[c] += mu * (alph * (-m)) - mu1 * (alph * (-m1));
    }
    lw[c] = mu;
    lcA[c] = 0.0f;
    lcB[c] = 0.0f;
  }
}

static void launch_adj_wsolve(const AdjArgs<float>& A, cudaStream_t s) {
  const int nz = A.g.nz;
  const size_t bytes = (size_t)4 * nz * kAdjCols * sizeof(float);
  if (nz < 3 || bytes > 200 * 1024) {
    launch_adj<OpWSolve>(A, s);
    return;
  }
  if (A.gx <= 0 || A.gy <= 0) return;
  if (opt_in_smem((const void*)k_adj_wsolve_coop, bytes) != cudaSuccess) return;  // error left pending
  launch_kernel(k_adj_wsolve_coop, dim3((A.g.nx * A.g.ny + kAdjCols - 1) / kAdjCols), dim3(kAdjCols * kAdjWarps),
                bytes, s, A);
}

struct AdjEntry {
  const char* name;
  AdjLaunch launch;
  uint64_t reads;
};

#define B1(n) (uint64_t(1) << (n))
static const AdjEntry kAdjTable[] = {
    {"adv_flux_x", launch_adj<OpFluxX>, B1(1) | B1(2)},
    {"adv_flux_y", launch_adj<OpFluxY>, B1(1) | B1(2)},
    {"adv_flux_z", launch_adj<OpFluxZ>, B1(1) | B1(2) | B1(3) | B1(4)},
    {"adv_flux_x_stag", launch_adj<OpStagX>, B1(2) | B1(3) | B1(4) | B1(7)},
    {"adv_flux_y_stag", launch_adj<OpStagY>, B1(2) | B1(3) | B1(4) | B1(7)},
    {"adv_flux_z_stag", launch_adj<OpStagZ>, B1(2) | B1(5) | B1(6) | B1(7)},
    {"adv_flux_x_weno", launch_adj<OpWenoX>, B1(1) | B1(2)},
    {"adv_flux_y_weno", launch_adj<OpWenoY>, B1(1) | B1(2)},
    {"adv_flux_z_weno", launch_adj<OpWenoZ>, B1(1) | B1(2) | B1(3) | B1(4)},
    {"adv_flux_x_weno_uv", launch_adj<OpWenoUvX>, B1(2) | B1(3)},
    {"adv_flux_y_weno_uv", launch_adj<OpWenoUvY>, B1(2) | B1(3)},
    {"adv_flux_z_weno_uv", launch_adj<OpWenoUvZ>, B1(2) | B1(3) | B1(4) | B1(5)},
    {"adv_flux_x_weno_w", launch_adj<OpWenoWX>, B1(1) | B1(2) | B1(3)},
    {"adv_flux_y_weno_w", launch_adj<OpWenoWY>, B1(1) | B1(2) | B1(3)},
    {"adv_flux_z_weno_w", launch_adj<OpWenoWZ>, B1(1) | B1(2)},
    {"adv_assemble", launch_adj<OpAssemble>, B1(2) | B1(6) | B1(7) | B1(8) | B1(9) | B1(10) | B1(15) | B1(16) | B1(30)},
    {"rk_update", launch_adj<OpRk>, 0},
    {"apply_thterm", launch_adj<OpThterm>, B1(1) | B1(2)},
    {"buoyancy_apply", launch_adj<OpBuoy>, B1(2) | B1(3)},
    {"update_diagnostics_moist", launch_adj<OpDiag>,
     B1(3) | B1(4) | B1(8) | B1(9) | B1(10) | B1(11) | B1(12) | B1(13) | B1(14)},
    {"stage_tendency_reset", launch_adj<OpTendReset>, 0},
    {"massflux_from_state", launch_adj<OpMassflux>, B1(4) | B1(5)},
    {"div_massflux", launch_adj<OpDivMassflux>, B1(4) | B1(30)},
    {"divergence3d", launch_adj<OpDiv3d>, B1(1) | B1(2) | B1(3) | B1(4) | B1(30)},
    {"velocity_to_massflux", launch_adj<OpVelMassflux>, B1(1) | B1(2)},
    {"build_sadv", launch_adj<OpSadv>, 0},
    {"stage_state_reset", launch_adj<OpStateReset>, 0},
    {"acoustic_begin", launch_adj<OpBegin>, 0},
    {"acoustic_prepare", launch_adj<OpPrepare>, 0},
    {"acoustic_uv", launch_adj<OpUv>, B1(2) | B1(3) | B1(30)},
    {"acoustic_fpk", launch_adj<OpFpk>, B1(2) | B1(3) | B1(5) | B1(7) | B1(8) | B1(9) | B1(10) | B1(30)},
    {"acoustic_pp", launch_adj<OpPp>, B1(2) | B1(3) | B1(4) | B1(5) | B1(6) | B1(7)},
    {"acoustic_accumulate", launch_adj<OpAccum>, 0},
    {"bc_periodic_x", launch_adj_halo<OpHaloX>, 0},
    {"bc_periodic_y", launch_adj_halo<OpHaloY>, 0},
    {"ppx_finish", launch_adj<OpPpxFinish>, 0},
    {"acoustic_w_solve", launch_adj_wsolve, B1(2) | B1(3) | B1(4) | B1(5)},
};
#undef B1

static const AdjEntry* find_adjoint(const std::string& name) {
  for (const AdjEntry& e : kAdjTable)
    if (name == e.name) return &e;
  return nullptr;
}

// adjoint of a copy dst <- src (disjoint ranges): lambda_src += lambda_dst, lambda_dst = 0;
// one word per thread, both loads before the stores
__global__ void __launch_bounds__(256) k_adj_copy(float* L, uint64_t src, uint64_t dst, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = L[dst + i], y = L[src + i];
  L[dst + i] = 0.0f;
  L[src + i] = y + x;
}

// Adjoint of a run of periodic halo pairs (bc_periodic_x(f) then bc_periodic_y(f)) on up
// to 4 distinct fields.  The pair leaves every halo point of the box [-3, nx + 3] x
// [-3, ny + 3] (levels 0..nz) with the value of its interior image (i mod nx, j mod ny), so
// its adjoint moves each halo point's adjoint onto that image and clears it.  As a gather:
// one thread per (interior point that has images, level, field) — the points with images
// are the 7 columns i < 4, i >= nx - 3 and the 7 rows j < 4, j >= ny - 3 of the interior;
// every halo point has exactly one image, so it is read and cleared by one thread and no
// update needs an atomic.  A thread reads all its halo points before its first store.
struct HaloRunArgs {
  Dims g;
  float* l[4];
  int nf;
};

__global__ void __launch_bounds__(128) k_adj_halo_run(HaloRunArgs H) {
  const Dims& g = H.g;
  const int nx = g.nx, ny = g.ny;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int i, j;
  if (t < 7 * ny) {  // the x band, every row
    j = t / 7;
    const int c = t % 7;
    i = c < 4 ? c : nx - 3 + (c - 4);
    if (i < 0 || i >= nx || (c >= 4 && i < 4)) return;
  } else {  // the y band, columns outside the x band
    const int u = t - 7 * ny;
    if (u >= 7 * nx) return;
    const int r = u / nx;
    i = u % nx;
    j = r < 4 ? r : ny - 3 + (r - 4);
    if (j < 0 || j >= ny || (r >= 4 && j < 4)) return;
    if (i < 4 || i >= nx - 3) return;
  }
  const int k = blockIdx.y, f = blockIdx.z;
  if (k > g.nz || f >= H.nf) return;
  // images i + a nx in [-3, nx + 3], j + b ny in [-3, ny + 3]
  const int alo = -((i + 3) / nx), ahi = (nx + 3 - i) / nx;
  const int blo = -((j + 3) / ny), bhi = (ny + 3 - j) / ny;
  float* L = H.l[f] + (size_t)k * g.sJ * g.sK;
  float acc = 0.0f;
  for (int a = alo; a <= ahi; a++)
    for (int b = blo; b <= bhi; b++)
      if (a != 0 || b != 0) acc += L[gidx(g, i + a * nx, j + b * ny, 0)];
  const int c0 = gidx(g, i, j, 0);
  const float own = L[c0];
  for (int a = alo; a <= ahi; a++)
    for (int b = blo; b <= bhi; b++)
      if (a != 0 || b != 0) L[gidx(g, i + a * nx, j + b * ny, 0)] = 0.0f;
  L[c0] = own + acc;
}

static void launch_adj_halo_run(const HaloRunArgs& H, cudaStream_t s) {
  const int threads = 7 * H.g.ny + 7 * H.g.nx;
  launch_kernel(k_adj_halo_run, dim3((threads + 127) / 128, H.g.nz + 1, H.nf), dim3(128), 0, s, H);
}

// The undo log's copies of one op's regions in one launch: region q is `rows` rows of
// `width` words, `pitch` words apart, at word `off` of the memory, packed at word `log` of
// the undo log; `start` holds the prefix sums of the regions' sizes.  save: memory -> log,
// restore: log -> memory.
constexpr int kCopyBatch = 8;
struct CopyBatch {
  uint64_t off[kCopyBatch], pitch[kCopyBatch], log[kCopyBatch];
  uint32_t width[kCopyBatch], rows[kCopyBatch];
  uint32_t start[kCopyBatch + 1];
  int n;
};

__global__ void __launch_bounds__(256) k_batch_copy(uint32_t* M, uint32_t* L, CopyBatch B, int restore) {
  const uint32_t total = B.start[B.n];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int q = 0;
    while (q + 1 < B.n && t >= B.start[q + 1]) q++;
    const uint32_t e = t - B.start[q];
    uint64_t m;
    if (B.rows[q] == 1) {
      m = B.off[q] + e;
    } else {
      const uint32_t r = e / B.width[q], col = e - r * B.width[q];
      m = B.off[q] + (uint64_t)r * B.pitch[q] + col;
    }
    const uint64_t l = B.log[q] + e;
    if (restore) M[m] = L[l];
    else L[l] = M[m];
  }
}

}  // namespace adj

// A written region in words: `rows` rows of `width` words, `pitch` words apart.
struct Region {
  uint64_t off, width, pitch, rows;
  uint64_t field;  // word offset of the field (binding) the region belongs to
  uint64_t size() const { return width * rows; }
  uint64_t last() const { return off + (rows - 1) * pitch + width - 1; }
  // every word of r lies in this region (a contiguous region, or the same pitched strip)
  bool covers(const Region& r) const {
    if (rows == 1) return off <= r.off && r.last() <= off + width - 1;
    return off == r.off && width == r.width && pitch == r.pitch && rows == r.rows;
  }
};

struct AdjointState {
  float* L = nullptr;  // adjoint memory, mem_words floats
  std::vector<uint32_t*> ckpt;
  uint64_t ckpt_words = 0;
  int nsteps = 0, every = 0;
  const Step* step = nullptr;  // the step the tables below were built for
  std::vector<std::vector<Region>> regions;  // per op: the regions it writes
  std::vector<adj::AdjArgs<float>> args;     // per op
  std::vector<adj::AdjLaunch> launch;        // per op (nullptr for copies)
  uint64_t step_undo_words = 0;
  uint32_t* undo = nullptr;
  uint64_t undo_cap = 0;  // words
  std::vector<cudaGraphExec_t> fwd_graph, rev_graph;  // per position in a block
  // runs of periodic halo pairs (ops first..last) replayed and reversed as one launch each
  struct HaloRun {
    int first = 0, last = 0, nf = 0;
    float* f[4] = {nullptr, nullptr, nullptr, nullptr};
    adj::HaloRunArgs adj{};
    std::vector<Region> regions;  // the undo-log regions of ops first..last, in op order
  };
  std::vector<HaloRun> runs;
  std::vector<int> run_from, run_to;  // per op: the run it starts / ends, or -1

  void drop_graphs() {
    for (auto g : fwd_graph)
      if (g) cudaGraphExecDestroy(g);
    for (auto g : rev_graph)
      if (g) cudaGraphExecDestroy(g);
    fwd_graph.clear();
    rev_graph.clear();
  }
};

void release_adjoint(Plan& P) {
  AdjointState* S = P.adjoint;
  if (!S) return;
  S->drop_graphs();
  for (auto p : S->ckpt) cudaFree(p);
  if (S->L) cudaFree(S->L);
  if (S->undo) cudaFree(S->undo);
  delete S;
  P.adjoint = nullptr;
}

namespace {

struct AdjError : std::runtime_error {
  int code;
  AdjError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define ACU(x)                                                                                  \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) throw te::AdjError(TE_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

AdjointState& state(Plan& P) {
  if (!P.adjoint) P.adjoint = new AdjointState();
  return *P.adjoint;
}

uint64_t regions_words(const std::vector<Region>& regs);

// Per-op tables of the active step: written regions, adjoint arguments and operators.
void build_tables(Plan& P, AdjointState& S) {
  if (S.step == P.active && !S.args.empty()) return;
  S.drop_graphs();
  const std::vector<Op>& ops = P.active->ops;
  S.regions.assign(ops.size(), {});
  S.args.assign(ops.size(), adj::AdjArgs<float>());
  S.launch.assign(ops.size(), nullptr);
  S.step_undo_words = 0;
  const uint32_t* M = P.M;
  // the memory regions whose values before an op some adjoint operator reads
  std::set<uint64_t> read;
  std::vector<std::vector<uint64_t>> reads(ops.size());  // per op: the fields its adjoint reads
  for (size_t i = 0; i < ops.size(); i++) {
    const Op& o = ops[i];
    if (o.copy) continue;
    if (!o.spec) throw AdjError(TE_ENOKERNEL, "no CUDA kernel for " + o.name);
    const adj::AdjEntry* e = adj::find_adjoint(o.name);
    if (!e) throw AdjError(TE_ENOKERNEL, "no adjoint operator for " + o.name);
    for (auto& kv : o.bind)
      if (kv.first < 64 && (e->reads >> kv.first & 1u)) {
        read.insert(kv.second);
        reads[i].push_back(kv.second);
      }
  }
  for (size_t i = 0; i < ops.size(); i++) {
    const Op& o = ops[i];
    if (o.copy) {
      if (read.count(o.dst)) {
        S.regions[i].push_back({o.dst, o.n, o.n, 1, o.dst});
        S.step_undo_words += o.n;
      }
      continue;
    }
    S.launch[i] = adj::find_adjoint(o.name)->launch;
    const bool halo_x = o.name == "bc_periodic_x", halo_y = o.name == "bc_periodic_y";
    for (int q = 0; q < o.spec->nparams; q++) {
      const ParamSpec& ps = o.spec->params[q];
      if (ps.kind != kPtr || !ps.write) continue;
      auto it = o.bind.find(ps.index);
      if (it == o.bind.end() || !read.count(it->second)) continue;
      const uint64_t f0 = it->second;
      const Dims& g = o.args.g;
      if (halo_x || halo_y) {
        // the halo points only: 3 columns (rows) below the interior and 4 above
        const uint64_t sJ = g.sJ, sK = g.sK, lv = (uint64_t)g.nz + 1;
        if (halo_x) {
          S.regions[i].push_back({f0, 3, sJ, sK * lv, f0});
          S.regions[i].push_back({f0 + (uint64_t)g.nx + 3, 4, sJ, sK * lv, f0});
        } else {
          S.regions[i].push_back({f0, 3 * sJ, sJ * sK, lv, f0});
          S.regions[i].push_back({f0 + ((uint64_t)g.ny + 3) * sJ, 4 * sJ, sJ * sK, lv, f0});
        }
        S.step_undo_words += S.regions[i][S.regions[i].size() - 2].size() + S.regions[i].back().size();
        continue;
      }
      const uint64_t len = P.region_len(f0);
      S.regions[i].push_back({f0, len, len, 1, f0});
      S.step_undo_words += len;
    }
    adj::AdjArgs<float>& a = S.args[i];
    std::memset(&a, 0, sizeof a);
    a.g = o.args.g;
    a.a = o.args.a;
    a.gx = o.args.gx;
    a.gy = o.args.gy;
    a.gz = o.args.gz;
    for (int n = 0; n < adj::kMaxBindA && n < kMaxBind; n++) {
      a.p[n] = o.args.p[n];
      a.l[n] = o.args.p[n] ? S.L + (reinterpret_cast<const uint32_t*>(o.args.p[n]) - M) : nullptr;
      a.f[n] = o.args.f[n];
      a.iv[n] = o.args.iv[n];
      a.iv2[n] = o.args.iv2[n];
    }
  }
  // A region's values before op i are needed only if some adjoint reads its field between
  // the previous op that wrote all of the region (whose own restore then brings the field
  // back for the adjoints before it) and op i, op i's own adjoint included.  The ops of a
  // step repeat every step, so that previous writer is searched cyclically; the block's
  // first step ends its reverse walk with fields some adjoint no longer reads left at later
  // values, which the next block's checkpoint (or the final restore) replaces.
  {
    const size_t n = ops.size();
    auto reads_field = [&](size_t k, uint64_t f) {
      return std::find(reads[k].begin(), reads[k].end(), f) != reads[k].end();
    };
    std::vector<std::vector<Region>> kept(n);
    for (size_t i = 0; i < n; i++)
      for (const Region& r : S.regions[i]) {
        bool need = reads_field(i, r.field);
        for (size_t step = 1; step < n && !need; step++) {
          const size_t k = (i + n - step) % n;
          bool covered = false;
          for (const Region& w : S.regions[k])
            if (w.field == r.field && w.covers(r)) covered = true;
          if (covered) break;
          need = reads_field(k, r.field);
        }
        if (need) kept[i].push_back(r);
      }
    S.regions.swap(kept);
    S.step_undo_words = 0;
    for (const auto& rs : S.regions) S.step_undo_words += regions_words(rs);
  }
  // runs of bc_periodic_x/y pairs on up to 4 distinct fields of the same grid
  S.runs.clear();
  S.run_from.assign(ops.size(), -1);
  S.run_to.assign(ops.size(), -1);
  for (size_t i = 0; i < ops.size();) {
    float* f = nullptr;
    if (!periodic_halo_pair(ops, i, &f)) {
      i++;
      continue;
    }
    AdjointState::HaloRun R;
    R.first = (int)i;
    const Dims& g = ops[i].args.g;
    size_t e = i;
    while (R.nf < 4 && periodic_halo_pair(ops, e, &f) && std::memcmp(&ops[e].args.g, &g, sizeof g) == 0 &&
           std::find(R.f, R.f + R.nf, f) == R.f + R.nf) {
      R.f[R.nf++] = f;
      e += 2;
    }
    R.last = (int)e - 1;
    for (int q = R.first; q <= R.last; q++) R.regions.insert(R.regions.end(), S.regions[q].begin(), S.regions[q].end());
    R.adj.g = g;
    R.adj.nf = R.nf;
    for (int q = 0; q < R.nf; q++) R.adj.l[q] = S.L + (reinterpret_cast<const uint32_t*>(R.f[q]) - M);
    S.run_from[R.first] = (int)S.runs.size();
    S.run_to[R.last] = (int)S.runs.size();
    S.runs.push_back(R);
    i = e;
  }
  S.step = P.active;
}

// Saves the regions of op `i` of the memory in the undo log from word `cur` on, or restores
// them from there (k_batch_copy: one launch for up to kCopyBatch regions).
void copy_regions(Plan& P, const std::vector<Region>& regs, uint32_t* log, uint64_t cur, bool restore) {
  for (size_t q0 = 0; q0 < regs.size(); q0 += adj::kCopyBatch) {
    adj::CopyBatch B;
    std::memset(&B, 0, sizeof B);
    uint64_t total = 0;
    for (size_t q = q0; q < regs.size() && B.n < adj::kCopyBatch; q++) {
      const Region& r = regs[q];
      B.off[B.n] = r.off;
      B.pitch[B.n] = r.pitch;
      B.log[B.n] = cur;
      B.width[B.n] = (uint32_t)r.width;
      B.rows[B.n] = (uint32_t)r.rows;
      B.start[B.n] = (uint32_t)total;
      if (r.width >= (1ull << 32) || r.rows >= (1ull << 32)) throw AdjError(TE_ERANGE, "undo-log region too large");
      total += r.size();
      cur += r.size();
      B.n++;
    }
    if (total >= (1ull << 32)) throw AdjError(TE_ERANGE, "undo-log regions of one op of 2^32 words or more");
    B.start[B.n] = (uint32_t)total;
    const int blocks = (int)std::min<uint64_t>(148 * 8, (total + 255) / 256);
    launch_kernel(adj::k_batch_copy, dim3(blocks), dim3(256), 0, P.stream, P.M, log, B, restore ? 1 : 0);
    ACU(cudaGetLastError());
  }
}

// The undo-log words of one op's regions.
uint64_t regions_words(const std::vector<Region>& regs) {
  uint64_t n = 0;
  for (const Region& r : regs) n += r.size();
  return n;
}

// Replays the active step op by op, saving each op's written regions at log + cursor.
void logged_step(Plan& P, AdjointState& S, uint32_t* log) {
  std::vector<Op>& ops = P.active->ops;
  uint64_t cur = 0;
  for (size_t i = 0; i < ops.size(); i++) {
    const int run = S.run_from[i];
    if (run >= 0) {
      // the pairs' halo fills leave the same memory as the per-dispatch kernels; the
      // intermediate state between them is never read (their adjoints read no values), so
      // every op's regions are saved before the run
      const AdjointState::HaloRun& R = S.runs[run];
      copy_regions(P, R.regions, log, cur, false);
      cur += regions_words(R.regions);
      launch_periodic_halos(ops[i].args.g, R.f, R.nf, P.stream);
      ACU(cudaGetLastError());
      i = (size_t)R.last;
      continue;
    }
    copy_regions(P, S.regions[i], log, cur, false);
    cur += regions_words(S.regions[i]);
    P.launch_exact(ops, (int)i, (int)i, false);
  }
}

// Walks the active step's ops in reverse: restore the op's written regions, run its adjoint.
// An op's regions are disjoint, except the x and y halo strips of one field in a halo run,
// whose shared corner words were saved at the same moment and restore the same value.
void reverse_step(Plan& P, AdjointState& S, const uint32_t* log) {
  std::vector<Op>& ops = P.active->ops;
  uint32_t* lg = const_cast<uint32_t*>(log);
  uint64_t cur = S.step_undo_words;
  for (size_t ii = ops.size(); ii-- > 0;) {
    const Op& o = ops[ii];
    if (S.run_to[ii] >= 0) {
      const AdjointState::HaloRun& R = S.runs[S.run_to[ii]];
      cur -= regions_words(R.regions);
      copy_regions(P, R.regions, lg, cur, true);
      adj::launch_adj_halo_run(R.adj, P.stream);
      ACU(cudaGetLastError());
      ii = (size_t)R.first;
      continue;
    }
    cur -= regions_words(S.regions[ii]);
    copy_regions(P, S.regions[ii], lg, cur, true);
    if (o.copy) {
      if ((o.n + 255) / 256 > 0x7fffffffu) throw AdjError(TE_ERANGE, "copy of 2^39 words or more");
      launch_kernel(adj::k_adj_copy, dim3((unsigned)((o.n + 255) / 256)), dim3(256), 0, P.stream, S.L, o.src, o.dst,
                    o.n);
    } else {
      S.launch[ii](S.args[ii], P.stream);
    }
  }
}

template <class F>
cudaGraphExec_t capture(cudaStream_t s, F body) {
  cudaGraph_t graph = nullptr;
  ACU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    body();
  } catch (...) {
    cudaStreamEndCapture(s, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  ACU(cudaStreamEndCapture(s, &graph));
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ex, graph, 0);
  cudaGraphDestroy(graph);
  ACU(e);
  return ex;
}

int fail(te_ctx* ctx, int code, const std::string& m) {
  ctx->err = m;
  return code;
}

}  // namespace
}  // namespace te

#define ADJ_BEGIN(ctx) \
  if (!ctx) return TE_EINVAL; \
  try {
#define ADJ_END(ctx)                                                        \
  }                                                                         \
  catch (const te::AdjError& e) { return te::fail(ctx, e.code, e.what()); } \
  catch (const std::exception& e) { return te::fail(ctx, TE_EINVAL, e.what()); } \
  return TE_OK;

extern "C" {

int te_adjoint_forward(te_ctx* ctx, int nsteps, int checkpoint_every) {
  ADJ_BEGIN(ctx)
  te::Plan& P = ctx->plan;
  if (!P.M) throw te::AdjError(TE_ESTATE, "te_plan has not been called");
  if (nsteps < 1 || checkpoint_every < 1) throw te::AdjError(TE_EINVAL, "nsteps and checkpoint_every must be >= 1");
  ACU(cudaSetDevice(ctx->device));
  te::AdjointState& S = te::state(P);
  if (!S.L) {
    ACU(cudaMalloc(&S.L, P.mem_words * 4));
  }
  ACU(cudaMemsetAsync(S.L, 0, P.mem_words * 4, P.stream));
  te::build_tables(P, S);
  const int nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
  S.ckpt_words = P.buffers_end;
  while ((int)S.ckpt.size() < nck) {
    uint32_t* p = nullptr;
    ACU(cudaMalloc(&p, S.ckpt_words * 4));
    S.ckpt.push_back(p);
  }
  const uint64_t need = (uint64_t)checkpoint_every * S.step_undo_words;
  if (need > S.undo_cap) {
    if (S.undo) cudaFree(S.undo);
    S.undo = nullptr;
    S.undo_cap = 0;
    ACU(cudaMalloc(&S.undo, need * 4));
    S.undo_cap = need;
  }
  if (S.every != checkpoint_every) S.drop_graphs();
  S.every = checkpoint_every;
  S.nsteps = nsteps;
  for (int s = 0; s < nsteps; s++) {
    if (s % checkpoint_every == 0)
      ACU(cudaMemcpyAsync(S.ckpt[s / checkpoint_every], P.M, S.ckpt_words * 4, cudaMemcpyDeviceToDevice, P.stream));
    P.launch_step_graph();
  }
  ACU(cudaGetLastError());
  ADJ_END(ctx)
}

int te_adjoint_backward(te_ctx* ctx) {
  ADJ_BEGIN(ctx)
  te::Plan& P = ctx->plan;
  te::AdjointState* Sp = P.adjoint;
  if (!P.M || !Sp || Sp->nsteps < 1) throw te::AdjError(TE_ESTATE, "te_adjoint_forward has not been called");
  te::AdjointState& S = *Sp;
  ACU(cudaSetDevice(ctx->device));
  te::build_tables(P, S);
  const int K = S.every;
  if ((uint64_t)K * S.step_undo_words > S.undo_cap) throw te::AdjError(TE_ESTATE, "step changed since te_adjoint_forward");
  if ((int)S.fwd_graph.size() != K) {
    S.drop_graphs();
    S.fwd_graph.assign(K, nullptr);
    S.rev_graph.assign(K, nullptr);
  }
  const int nb = (S.nsteps + K - 1) / K;
  for (int b = nb - 1; b >= 0; b--) {
    const int s0 = b * K, s1 = std::min(s0 + K, S.nsteps);
    ACU(cudaMemcpyAsync(P.M, S.ckpt[b], S.ckpt_words * 4, cudaMemcpyDeviceToDevice, P.stream));
    for (int s = s0; s < s1; s++) {
      const int j = s - s0;
      if (!S.fwd_graph[j])
        S.fwd_graph[j] = te::capture(P.stream, [&] { te::logged_step(P, S, S.undo + (uint64_t)j * S.step_undo_words); });
      ACU(cudaGraphLaunch(S.fwd_graph[j], P.stream));
    }
    for (int s = s1 - 1; s >= s0; s--) {
      const int j = s - s0;
      if (!S.rev_graph[j])
        S.rev_graph[j] = te::capture(P.stream, [&] { te::reverse_step(P, S, S.undo + (uint64_t)j * S.step_undo_words); });
      ACU(cudaGraphLaunch(S.rev_graph[j], P.stream));
    }
  }
  // fields that no adjoint operator reads are not logged: memory returns to the start
  // state from its checkpoint
  ACU(cudaMemcpyAsync(P.M, S.ckpt[0], S.ckpt_words * 4, cudaMemcpyDeviceToDevice, P.stream));
  ACU(cudaGetLastError());
  ADJ_END(ctx)
}

int te_adjoint_write_words(te_ctx* ctx, uint64_t word_off, const void* data, size_t bytes) {
  ADJ_BEGIN(ctx)
  te::Plan& P = ctx->plan;
  if (!P.adjoint || !P.adjoint->L) throw te::AdjError(TE_ESTATE, "te_adjoint_forward has not been called");
  if (word_off + (bytes + 3) / 4 > P.mem_words) throw te::AdjError(TE_ERANGE, "write past the end of memory");
  ACU(cudaSetDevice(ctx->device));
  ACU(cudaMemcpyAsync(P.adjoint->L + word_off, data, bytes, cudaMemcpyHostToDevice, P.stream));
  ACU(cudaStreamSynchronize(P.stream));
  ADJ_END(ctx)
}

int te_adjoint_read(te_ctx* ctx, uint64_t word_off, uint64_t words, void* out) {
  ADJ_BEGIN(ctx)
  te::Plan& P = ctx->plan;
  if (!P.adjoint || !P.adjoint->L) throw te::AdjError(TE_ESTATE, "te_adjoint_forward has not been called");
  if (word_off + words > P.mem_words) throw te::AdjError(TE_ERANGE, "read past the end of memory");
  ACU(cudaSetDevice(ctx->device));
  ACU(cudaMemcpyAsync(out, P.adjoint->L + word_off, words * 4, cudaMemcpyDeviceToHost, P.stream));
  ACU(cudaStreamSynchronize(P.stream));
  ADJ_END(ctx)
}

int te_adjoint_zero(te_ctx* ctx) {
  ADJ_BEGIN(ctx)
  te::Plan& P = ctx->plan;
  if (!P.adjoint || !P.adjoint->L) throw te::AdjError(TE_ESTATE, "te_adjoint_forward has not been called");
  ACU(cudaSetDevice(ctx->device));
  ACU(cudaMemsetAsync(P.adjoint->L, 0, P.mem_words * 4, P.stream));
  ADJ_END(ctx)
}

int te_adjoint_device_ptr(te_ctx* ctx, uint64_t word_off, void** out) {
  ADJ_BEGIN(ctx)
  te::Plan& P = ctx->plan;
  if (!P.adjoint || !P.adjoint->L) throw te::AdjError(TE_ESTATE, "te_adjoint_forward has not been called");
  if (word_off >= P.mem_words) throw te::AdjError(TE_ERANGE, "offset outside memory");
  *out = P.adjoint->L + word_off;
  ADJ_END(ctx)
}

int te_adjoint_memory(te_ctx* ctx, uint64_t* bytes) {
  ADJ_BEGIN(ctx)
  te::Plan& P = ctx->plan;
  const te::AdjointState* S = P.adjoint;
  *bytes = S ? (S->L ? P.mem_words * 4 : 0) + S->ckpt.size() * S->ckpt_words * 4 + S->undo_cap * 4 : 0;
  ADJ_END(ctx)
}

}  // extern "C"

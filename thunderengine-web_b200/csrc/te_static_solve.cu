// te_w_solve_static_scratch: the vertically implicit w-pi' column solve with its
// forward-sweep coefficients held in a library-owned device array.
//
// For callers that cannot allocate device memory at the point where they run the solve
// (a custom allocator owns the pool, or an embedding forbids allocation): the caller
// passes only its input and output fields; the Thomas coefficients cA, cB that the tape
// kernel keeps in two arena fields live in kScratch below.  No cudaMalloc, cudaFree or
// allocating library routine is called.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/thunderstep.h"
#include "te_math.cuh"

namespace te {
namespace {

// 64 MiB, held by every GPU that loads this library until the process exits.
constexpr size_t kScratchFloats = size_t(16) << 20;
static __device__ __align__(256) float kScratch[kScratchFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_scratch[kMaxDevices] = {nullptr};

// One thread per column, lanes on consecutive i.  The arithmetic is the tape kernel's
// (acoustic_w_solve.wgsl:124-212, k_acoustic_w_solve in te_kernels.cu); cA, cB of level k
// sit at scratch[(k - 1) * ncol + col] and scratch[(nz - 2 + k - 1) * ncol + col].
__global__ void __launch_bounds__(128) k_w_solve_static(te_wsolve_fields f, Dims g, float dts, float alph,
                                                        float beta, float* scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int ncol = g.nx * g.ny, col = i + g.nx * j;
  float* cA = scratch + col;
  float* cB = scratch + (size_t)(g.nz - 2) * ncol + col;
  const int sk = g.sJ * g.sK;
  const float asq = alph * alph;
  float* w = f.w;
  w[gidx(g, i, j, 0)] = 0.0f;
  w[gidx(g, i, j, g.nz)] = 0.0f;
  float aa, bb, cc, dd;
  auto lam = [&](int kk) {
    const int c = gidx(g, i, j, kk), cm = c - sk;
    const float m = f.mm[c];
    aa = (-asq) * (m * (f.pk1[cm] + f.qk[cm]));
    cc = (-asq) * ((-m) * (f.pk2[c] - f.qk[c]));
    bb = fmaf(-asq, m * ((-(f.pk1[c] + f.qk[c])) + (f.pk2[cm] - f.qk[cm])), 1.0f);
    const float fw = fmaf(dts, f.wten[c], beta * ((-m) * (f.pp3d[c] - f.pp3d[cm])));
    dd = fmaf(alph, (-m) * ((f.pp3d[c] + f.fpk[c]) - (f.pp3d[cm] + f.fpk[cm])), w[c] + fw);
  };
  lam(1);
  {
    const float r = dcr(1.0f, bb);
    cA[0] = (-cc) * r;
    cB[0] = dd * r;
  }
  for (int k = 2; k < g.nz - 1; k++) {
    lam(k);
    const size_t q = (size_t)(k - 1) * ncol, p = q - ncol;
    const float r = dcr(1.0f, fmaf(aa, cA[p], bb));
    cA[q] = (-cc) * r;
    cB[q] = fmaf(-aa, cB[p], dd) * r;
  }
  {
    const int k = g.nz - 1, c = gidx(g, i, j, k);
    lam(k);
    const size_t p = (size_t)(k - 2) * ncol;
    const float r = dcr(1.0f, fmaf(aa, cA[p], bb));
    w[c] = fmaf(-aa, cB[p], dd) * r;
  }
  for (int k = g.nz - 2; k >= 1; k--) {
    const int c = gidx(g, i, j, k);
    const size_t q = (size_t)(k - 1) * ncol;
    w[c] = fmaf(cA[q], w[c + sk], cB[q]);
  }
}

int fail(char* err, size_t len, int code, const char* msg) {
  if (err && len) std::snprintf(err, len, "%s", msg);
  return code;
}

}  // namespace
}  // namespace te

extern "C" int te_w_solve_static_scratch(const te_wsolve_fields* f, int nx, int ny, int nz, float dts, float alph,
                                         float beta, void* cuda_stream, char* err, size_t err_len) {
  using namespace te;
  if (!f || !f->pk1 || !f->pk2 || !f->qk || !f->mm || !f->fpk || !f->wten || !f->pp3d || !f->w)
    return fail(err, err_len, TE_EINVAL, "te_w_solve_static_scratch: a field pointer is NULL");
  if (nx < 1 || ny < 1 || nz < 3)
    return fail(err, err_len, TE_EINVAL, "te_w_solve_static_scratch: needs nx >= 1, ny >= 1, nz >= 3");
  const size_t need = 2 * (size_t)nx * (size_t)ny * (size_t)(nz - 2);
  if (need > kScratchFloats) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "te_w_solve_static_scratch: %d x %d columns of %d levels need %zu scratch floats; the "
                  "library holds %zu (nx * ny * (nz - 2) must be <= %zu)",
                  nx, ny, nz, need, kScratchFloats, kScratchFloats / 2);
    return fail(err, err_len, TE_ERANGE, msg);
  }
  if (ny > 4 * 65535) {
    char msg[160];
    std::snprintf(msg, sizeof msg, "te_w_solve_static_scratch: ny = %d exceeds the launch limit of 262140 rows", ny);
    return fail(err, err_len, TE_ERANGE, msg);
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(err, err_len, TE_ECUDA, "te_w_solve_static_scratch: no usable current CUDA device");
  float* scratch;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
      // first call on this device: translate the array's host-side name into its device
      // address (the host symbol itself is not a device pointer).  The address belongs to
      // the device's primary context, the one the CUDA runtime uses; it stays valid until
      // that context is destroyed (cudaDeviceReset), after which this cache is stale.
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, kScratch);
      if (e != cudaSuccess) {
        char msg[200];
        std::snprintf(msg, sizeof msg, "te_w_solve_static_scratch: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
        return fail(err, err_len, TE_ECUDA, msg);
      }
      g_scratch[dev] = static_cast<float*>(p);
    }
    scratch = g_scratch[dev];
  }
  Dims g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.sJ = nx + 7;
  g.sK = ny + 7;
  g.rdx = g.rdy = g.rdz = 0.0f;
  dim3 b(32, 4, 1);
  dim3 gr((nx + 31) / 32, (ny + 3) / 4, 1);
  k_w_solve_static<<<gr, b, 0, static_cast<cudaStream_t>(cuda_stream)>>>(*f, g, dts, alph, beta, scratch);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[200];
    std::snprintf(msg, sizeof msg, "te_w_solve_static_scratch: launch failed: %s", cudaGetErrorString(e));
    return fail(err, err_len, TE_ECUDA, msg);
  }
  return TE_OK;
}

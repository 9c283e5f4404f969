// Kernel registry: one CUDA kernel per reference kernel name on the dynamics path.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "te_math.cuh"

namespace te {

constexpr int kMaxBind = 40;

// Decoded arguments of one dispatch.  `p[n]` is the device address of binding n
// (memory word offset of the tape player), `f[n]`/`iv[n]`/`iv2[n]` are the f32 / i32 /
// second i32 word of a setBytes struct bound at n.
struct KArgs {
  Dims g;
  Acoustic a;
  int gx, gy, gz;
  float* p[kMaxBind];
  float f[kMaxBind];
  int iv[kMaxBind];
  int iv2[kMaxBind];
  float sw[2][8];  // the first 8 words of the kernel's first and second struct bindings (kRefS)
  short bx, by;    // thread-block shape of the generic launchers (0: 32 x 4), set by te_autotune
  const uint32_t* ref0;  // device address of binding 0's words (a kernel's parameter struct)
  float* scr;            // the planned per-thread kernel scratch (kernels with scratch)
  unsigned scr_rows;     // dispatch rows that share that scratch per launch (the reference's y tile)
};

// Thread-block shape of a generic launch: the op's tuned shape, else 32 x 4.
inline dim3 tile_of(const KArgs& A) { return dim3(A.bx > 0 ? A.bx : 32, A.by > 0 ? A.by : 4, 1); }

enum ParamKind : uint8_t { kPtr = 0, kRef = 1, kRefS = 2 };

struct ParamSpec {
  int8_t index;
  uint8_t kind;
  uint8_t write;
};

typedef void (*LaunchFn)(const KArgs&, cudaStream_t);

struct KernelSpec {
  const char* name;
  int nparams;
  ParamSpec params[24];
  bool acoustic;  // binding 1 is AcousticParams
  LaunchFn launch;
};

// Launches kernel k on stream s (cudaLaunchKernelEx: one call for every kernel of the
// library, dynamic shared memory included).
template <typename... P, typename... Args>
inline cudaError_t launch_kernel(void (*k)(P...), dim3 gr, dim3 b, size_t smem, cudaStream_t s, Args... a) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = gr;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  return cudaLaunchKernelEx(&cfg, k, a...);
}

// Opts kernel `k` into `bytes` of dynamic shared memory on the CURRENT device.  The
// attribute belongs to the device, so it is set once per (kernel, device) — a process
// with contexts on several GPUs sets it on each — under a lock.  On failure the CUDA
// error stays pending for the caller's cudaGetLastError check and is also returned.
cudaError_t opt_in_smem(const void* k, size_t bytes);

// All kernels this library implements (te_kernels.cu).
const KernelSpec* kernel_table(int* count);
const KernelSpec* find_kernel(const char* name);

// The same kernels with __restrict__ field pointers (te_kernels_fast.cu), for ops whose
// bound regions do not overlap.
namespace fast {
const KernelSpec* kernel_table(int* count);
const KernelSpec* find_kernel(const char* name);
}  // namespace fast

}  // namespace te

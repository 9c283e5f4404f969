// Ensembles of independent runs and the launch-shape autotuner (no counterpart in the
// reference).
//
// te_autotune: for every per-dispatch op of the active step whose launcher takes its thread
// block from the op (the generic point-wise and row-vector launchers), times each
// candidate block shape with CUDA events on the context's stream and keeps the fastest;
// memory is restored afterwards, so tuning leaves the state as it found it.
//
// te_ensemble: members are planned contexts on one device, of any grid size, time step
// and substep count.  Each member's step (in its current mode) is captured as a graph and
// becomes a child node of one ensemble graph with no edges between members, so one graph
// launch advances every member by one large step and the members' kernels run
// concurrently: small members no longer leave the GPU idle between launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/thunderstep.h"
#include "te_kernels.cuh"
#include "te_player.hpp"

struct te_ensemble {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<te_ctx*> members;
  cudaGraphExec_t exec = nullptr;
  std::string err;
};

namespace te {
namespace {

struct EnsError : std::runtime_error {
  int code;
  EnsError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define ECU(x)                                                                                     \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) throw te::EnsError(TE_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// candidate thread-block shapes (at most 128 threads: the row-vector kernels are
// compiled for 128)
const short kShapes[][2] = {{32, 4}, {32, 2}, {64, 2}, {128, 1}, {16, 8}, {64, 1}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

}  // namespace
}  // namespace te

extern "C" {

int te_autotune(te_ctx* ctx, int reps, int* tuned_ops) {
  if (!ctx) return TE_EINVAL;
  try {
    te::Plan& P = ctx->plan;
    if (!P.M) throw te::EnsError(TE_ESTATE, "te_plan has not been called");
    ECU(cudaSetDevice(ctx->device));
    reps = std::max(1, reps);
    std::vector<te::Op>& ops = P.active->ops;
    uint32_t* save = nullptr;
    ECU(cudaMalloc(&save, P.buffers_end * 4));
    ECU(cudaMemcpyAsync(save, P.M, P.buffers_end * 4, cudaMemcpyDeviceToDevice, P.stream));
    cudaEvent_t e0, e1;
    ECU(cudaEventCreate(&e0));
    ECU(cudaEventCreate(&e1));
    int changed = 0;
    for (size_t i = 0; i < ops.size(); i++) {
      te::Op& o = ops[i];
      if (o.copy || !o.spec) continue;
      float best = 1e30f, base_ms = 0.0f;
      int best_q = 0;
      for (int q = 0; q < te::kNumShapes; q++) {
        o.args.bx = te::kShapes[q][0];
        o.args.by = te::kShapes[q][1];
        P.launch_exact(ops, (int)i, (int)i, false);  // warm-up
        if (cudaGetLastError() != cudaSuccess) continue;  // shape not launchable for this kernel
        ECU(cudaEventRecord(e0, P.stream));
        for (int r = 0; r < reps; r++) P.launch_exact(ops, (int)i, (int)i, false);
        ECU(cudaEventRecord(e1, P.stream));
        ECU(cudaEventSynchronize(e1));
        float ms = 0.0f;
        ECU(cudaEventElapsedTime(&ms, e0, e1));
        if (q == 0) base_ms = ms;
        if (ms < best) {
          best = ms;
          best_q = q;
        }
      }
      // keep the default unless another shape is clearly faster (timing noise otherwise)
      if (best_q != 0 && best > 0.97f * base_ms) best_q = 0;
      o.tile[0] = best_q ? te::kShapes[best_q][0] : 0;
      o.tile[1] = best_q ? te::kShapes[best_q][1] : 0;
      o.args.bx = o.tile[0];
      o.args.by = o.tile[1];
      changed += best_q != 0;
    }
    ECU(cudaMemcpyAsync(P.M, save, P.buffers_end * 4, cudaMemcpyDeviceToDevice, P.stream));
    ECU(cudaStreamSynchronize(P.stream));
    cudaFree(save);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P.invalidate_graphs();
    if (tuned_ops) *tuned_ops = changed;
  } catch (const te::EnsError& e) {
    ctx->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return TE_EINVAL;
  }
  return TE_OK;
}

int te_ensemble_create(te_ctx* const* members, int n, te_ensemble** out) {
  if (!out || !members || n < 1) return TE_EINVAL;
  *out = nullptr;
  te_ensemble* E = new te_ensemble();
  try {
    E->device = members[0]->device;
    for (int m = 0; m < n; m++) {
      if (!members[m] || !members[m]->plan.M) throw te::EnsError(TE_ESTATE, "member " + std::to_string(m) + " is not planned");
      if (members[m]->device != E->device) throw te::EnsError(TE_EINVAL, "members must share one device");
      E->members.push_back(members[m]);
    }
    ECU(cudaSetDevice(E->device));
    ECU(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
    cudaGraph_t root = nullptr;
    ECU(cudaGraphCreate(&root, 0));
    try {
      for (te_ctx* c : E->members) {
        cudaGraph_t g = c->plan.capture_step();
        cudaGraphNode_t node;
        const cudaError_t e = cudaGraphAddChildGraphNode(&node, root, nullptr, 0, g);
        cudaGraphDestroy(g);
        ECU(e);
      }
      ECU(cudaGraphInstantiate(&E->exec, root, 0));
    } catch (...) {
      cudaGraphDestroy(root);
      throw;
    }
    cudaGraphDestroy(root);
  } catch (const te::EnsError& e) {
    E->err = e.what();
    *out = E;
    return e.code;
  } catch (const std::exception& e) {
    E->err = e.what();
    *out = E;
    return TE_EINVAL;
  }
  *out = E;
  return TE_OK;
}

int te_ensemble_run(te_ensemble* E, int nsteps) {
  if (!E || !E->exec) return TE_ESTATE;
  cudaError_t e = cudaSetDevice(E->device);
  for (int s = 0; s < nsteps && e == cudaSuccess; s++) e = cudaGraphLaunch(E->exec, E->stream);
  if (e != cudaSuccess) {
    E->err = std::string("te_ensemble_run: ") + cudaGetErrorString(e);
    return TE_ECUDA;
  }
  return TE_OK;
}

int te_ensemble_stream(te_ensemble* E, void** stream) {
  if (!E || !stream) return TE_EINVAL;
  *stream = E->stream;
  return TE_OK;
}

int te_ensemble_sync(te_ensemble* E) {
  if (!E) return TE_EINVAL;
  cudaSetDevice(E->device);
  const cudaError_t e = cudaStreamSynchronize(E->stream);
  if (e != cudaSuccess) {
    E->err = std::string("te_ensemble_sync: ") + cudaGetErrorString(e);
    return TE_ECUDA;
  }
  return TE_OK;
}

const char* te_ensemble_last_error(te_ensemble* E) { return E ? E->err.c_str() : "no ensemble"; }

void te_ensemble_destroy(te_ensemble* E) {
  if (!E) return;
  cudaSetDevice(E->device);
  if (E->stream) cudaStreamSynchronize(E->stream);
  if (E->exec) cudaGraphExecDestroy(E->exec);
  if (E->stream) cudaStreamDestroy(E->stream);
  delete E;
}

}  // extern "C"

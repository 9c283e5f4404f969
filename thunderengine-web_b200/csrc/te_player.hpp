// Host-side state of one tape player context.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "te_fused.cuh"
#include "te_json.hpp"
#include "te_kernels.cuh"

namespace te {

struct HashReq {
  uint32_t slot = 0;
  bool bound = false;
  uint64_t off = 0, len = 0;
};

// One op of a step: a kernel dispatch or a blit copy (replay.js:95-118).
struct Op {
  bool copy = false;
  std::string name;
  uint64_t src = 0, dst = 0, n = 0;
  const KernelSpec* spec = nullptr;
  LaunchFn launch = nullptr;  // spec->launch, or its __restrict__ twin when the bound regions are disjoint
  int grid[3] = {0, 0, 0}, tg[3] = {0, 0, 0};
  std::map<int, uint64_t> bind;  // binding index -> memory word offset
  std::vector<HashReq> hashes;
  KArgs args;
  short tile[2] = {0, 0};  // thread-block shape chosen by te_autotune (0: the launcher's default)
  uint64_t tile_y = 0;     // dispatch rows per scratch tile (replay.js:104-108)
};

struct Step {
  std::vector<Op> ops;
  std::map<int, uint64_t> offs;    // command index -> word offset of its setBytes payload
  std::map<int, std::string> data;  // command index -> last payload written
};

struct KParam {
  int index;
  bool ref;
  bool write;
};
struct KMeta {
  uint64_t scratch = 0;
  std::vector<KParam> params;
};

struct BufInfo {
  uint64_t length;  // bytes
  bool arena;
};

struct AdjointState;  // te_adjoint.cu

struct Plan {
  cudaStream_t stream = nullptr;
  int mode = 0;
  int flags = 0;
  // layout (replay.js:46-66)
  std::vector<BufInfo> buffers;
  std::vector<uint64_t> base;
  uint64_t field_stride = 0;  // bytes
  uint64_t buffers_end = 0, bytes_top = 0, bytes_spare_end = 0, scratch_base = 0, scratch_need = 0, mem_words = 0;
  uint32_t hash_count = 0;
  bool with_hashes = false;
  std::vector<std::pair<uint64_t, std::vector<uint8_t>>> bytes_init;
  std::vector<uint32_t> host_bytes;  // host copy of words [buffers_end, bytes_spare_end), word-indexed
  std::map<std::string, KMeta> kmeta;
  std::map<std::string, Step> cache;
  Step* active = nullptr;
  std::vector<Op> diag_ops;
  // device
  uint32_t* M = nullptr;
  uint32_t* H = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  FusedStep fused;
  bool fused_dirty = true;
  AdjointState* adjoint = nullptr;  // checkpoints, undo log and adjoint memory of te_adjoint_*

  void load_kernel_meta(const char* kjson, size_t klen);
  std::map<int, uint64_t> layout_bytes(const JValue& cmds);
  uint64_t region_len(uint64_t off) const;
  std::vector<Op> build_ops(const JValue& cmds, const std::map<int, uint64_t>& offs, bool hashes);
  void plan(const char* tj, size_t tl, bool with_hashes);
  void finalize_args(std::vector<Op>& ops);
  void launch_exact(std::vector<Op>& ops, int first, int last, bool hashes);
  void launch_step_graph();
  cudaGraph_t capture_step();  // the active step (current mode) as a graph, not instantiated
  void invalidate_graphs();
  void release();
};

void release_adjoint(Plan& P);  // te_adjoint.cu

}  // namespace te

// One player context (include/thunderstep.h te_ctx).
struct te_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  te::Plan plan;
};

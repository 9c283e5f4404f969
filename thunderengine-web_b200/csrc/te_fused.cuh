// Fused execution of recognised step phases (TE_MODE_FUSED).
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace te {

struct Op;
struct Plan;

// A step's op list rewritten into segments: runs of exact per-dispatch kernels and
// fused phase kernels that produce bit-identical prognostic fields.
struct FusedSegment {
  int kind = 0;  // 0 = exact ops [first, last]; >0 = a fused phase
  int first = 0, last = 0;
  int aux[16] = {0};
};

struct FusedStep {
  std::vector<FusedSegment> segs;
  void* data = nullptr;  // kernel arguments of the fused segments
  void build(Plan& P, std::vector<Op>& ops);
  void launch(Plan& P, std::vector<Op>& ops);
  // one segment; part = -1 for all of its kernels, else the index of one of them
  void launch_segment(Plan& P, std::vector<Op>& ops, int seg, int part);
  int launches_per_step() const;
  void release();
};

}  // namespace te

// Fused execution of recognised step phases (TE_MODE_FUSED).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "te_dims.cuh"

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

// ops[i], ops[i + 1] are bc_periodic_x(f) then bc_periodic_y(f) over the standard halo
// grids (4 x (ny + 7) x (nz + 1), 4 x (nx + 7) x (nz + 1)): sets *f, returns true.
bool periodic_halo_pair(const std::vector<Op>& ops, size_t i, float** f);

// The final state of such pairs for nf <= 4 distinct fields in one launch: every halo point
// of levels 0..nz holds the interior value at (i mod nx, j mod ny).
void launch_periodic_halos(const Dims& g, float* const* f, int nf, cudaStream_t s);

}  // namespace te

// Fused step phases (TE_MODE_FUSED).  Segments not recognised run the exact kernels.
#include "te_fused.cuh"
#include "te_player.hpp"

namespace te {

void FusedStep::build(Plan& P, std::vector<Op>& ops) {
  segs.clear();
  FusedSegment s;
  s.kind = 0;
  s.first = 0;
  s.last = (int)ops.size() - 1;
  segs.push_back(s);
}

void FusedStep::launch(Plan& P, std::vector<Op>& ops) {
  for (auto& s : segs) {
    if (s.kind == 0) P.launch_exact(ops, s.first, s.last, false);
  }
}

}  // namespace te

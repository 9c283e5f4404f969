// The per-dispatch kernels again, with every field pointer __restrict__-qualified, in
// namespace te::fast.  Same arithmetic, same results; used only for ops whose bound
// field regions are pairwise disjoint (Plan::finalize_args checks), where the
// qualifier is true.
#define TE_R __restrict__
#define TE_KERNELS_FAST 1
#include "te_kernels.cu"

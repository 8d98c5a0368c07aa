// kernels_multi.cu -- multi-pass forward kernels (reads longer than 32*8 rows).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<kMaxRowsPerLane, true>(Precision, bool, bool, int);
}  // namespace rodv

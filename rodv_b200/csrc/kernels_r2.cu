// kernels_r2.cu -- forward kernels with 2 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<2, false>(Precision, bool, bool, int);
}  // namespace rodv

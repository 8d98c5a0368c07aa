// kernels_r4.cu -- forward kernels with 4 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<4, false>(Precision, bool, bool, int);
}  // namespace rodv

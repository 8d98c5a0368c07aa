// kernels_r8.cu -- forward kernels with 8 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<8, false>(Precision, bool, bool, int);
}  // namespace rodv

// kernels_r7.cu -- forward kernels with 7 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<7, false>(Precision, bool, bool, int);
}  // namespace rodv

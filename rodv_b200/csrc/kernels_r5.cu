// kernels_r5.cu -- forward kernels with 5 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<5, false>(Precision, bool, bool, int);
}  // namespace rodv

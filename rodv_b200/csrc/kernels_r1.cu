// kernels_r1.cu -- forward kernels with 1 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<1, false>(Precision, bool, bool, int);
}  // namespace rodv

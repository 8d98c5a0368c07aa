// kernels_r3.cu -- forward kernels with 3 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<3, false>(Precision, bool, bool, int);
}  // namespace rodv

// kernels_r6.cu -- forward kernels with 6 read rows per lane (single pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo info_for<6, false>(Precision, bool, bool, int);
}  // namespace rodv

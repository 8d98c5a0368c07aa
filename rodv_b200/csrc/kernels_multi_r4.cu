// kernels_multi_r4.cu -- multi-pass forward kernels with a strip height of 4
// rows per lane (128 read rows per pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo pipe_info_for<4>(Precision, bool, bool, int);
}  // namespace rodv

// kernels_multi_r8.cu -- multi-pass forward kernels with a strip height of 8
// rows per lane (256 read rows per pass).
#include "kernel_table.cuh"

namespace rodv {
template KernelInfo pipe_info_for<8>(Precision, bool, bool, int);
}  // namespace rodv

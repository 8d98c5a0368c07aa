// kernel_table.cuh -- KernelInfo of every forward-kernel instantiation.
//
// Each rows-per-lane value R is instantiated in its own translation unit
// (kernels_r<R>.cu, kernels_multi.cu) so the ~100 kernels compile in parallel.
#pragma once
#include <type_traits>

#include "kernels.h"
#include "pairhmm_fwd.cuh"

namespace rodv {

template <class P, int R, bool U, bool MU, bool SAME, int MINB, int GROUP = 32>
KernelInfo make_info(int variant) {
  using F = Forward<P, R, U, MU, SAME, MINB, GROUP>;
  KernelInfo k;
  k.fn = reinterpret_cast<const void*>(&forward_kernel<P, R, U, MU, SAME, MINB, GROUP>);
  k.threads = F::kWarpsPerBlock * kWarp;
  k.warps_per_block = F::kWarpsPerBlock;
  k.smem_bytes = F::kWarpsPerBlock * F::kSmemPerWarp;
  k.rows_per_lane = R;
  k.multi = MU;
  k.same_hap = SAME || P::kSlots == 1;
  k.chain = F::kChain;
  k.items_per_warp = F::kGroups;
  k.min_blocks = MINB;
  k.variant = variant;
  return k;
}

// Same-haplotype FP32 kernels come in occupancy targets (kVariantMinBlocks);
// the chain kernels of reads up to 128 bases (R <= 4) also in a lane-grouped
// form: two 16-lane groups per warp, each sweeping its own chain item with
// 2R rows per lane, so that each lane's per-step overhead (shuffles, code and
// table loads, row-0 selects) covers twice the rows (faster at R <= 2 on B200,
// slower at R >= 3, where the longer per-step dependency chain shows; the
// autotuner picks).  Every other kernel has one variant.
template <class P, int R, bool U, bool MU, bool SAME>
KernelInfo variant_info(int variant) {
  if constexpr (!(std::is_same<P, F32x2>::value && SAME)) {
    (void)variant;
    return make_info<P, R, U, MU, SAME, 1>(0);
  } else {
    if constexpr (!MU && R <= kMaxGroupedRows) {
      switch (variant) {
        case 4: return make_info<P, 2 * R, U, MU, SAME, kVariantMinBlocks[4], 16>(4);
        case 5: return make_info<P, 2 * R, U, MU, SAME, kVariantMinBlocks[5], 16>(5);
        case 6: return make_info<P, 2 * R, U, MU, SAME, kVariantMinBlocks[6], 16>(6);
        case 7: return make_info<P, 2 * R, U, MU, SAME, kVariantMinBlocks[7], 16>(7);
        default: break;
      }
    }
    switch (variant) {
      case 0: return make_info<P, R, U, MU, SAME, kVariantMinBlocks[0]>(0);
      case 1: return make_info<P, R, U, MU, SAME, kVariantMinBlocks[1]>(1);
      case 2: return make_info<P, R, U, MU, SAME, kVariantMinBlocks[2]>(2);
      default: return make_info<P, R, U, MU, SAME, kVariantMinBlocks[3]>(3);
    }
  }
}

template <int R, bool MU>
KernelInfo info_for(Precision prec, bool uniform, bool same, int variant) {
  if (prec == Precision::kF64)
    return uniform ? variant_info<F64, R, true, MU, false>(0)
                   : variant_info<F64, R, false, MU, false>(0);
  if (same)
    return uniform ? variant_info<F32x2, R, true, MU, true>(variant)
                   : variant_info<F32x2, R, false, MU, true>(variant);
  // Two-haplotype items: multi-pass leftovers, and the odd single-pass read
  // of a region against each of its haplotypes.
  return uniform ? variant_info<F32x2, R, true, MU, false>(0)
                 : variant_info<F32x2, R, false, MU, false>(0);
}

}  // namespace rodv

// kernel_table.cuh -- KernelInfo of every forward-kernel instantiation.
//
// Each rows-per-lane value R is instantiated in its own translation unit
// (kernels_r<R>.cu; multi-pass strip heights in kernels_multi_r<R>.cu) so the
// ~150 kernels compile in parallel.
#pragma once
#include <type_traits>

#include "kernels.h"
#include "pairhmm_fwd.cuh"
#include "pairhmm_pipe.cuh"

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
  k.items_per_block = F::kWarpsPerBlock * F::kGroups;
  k.min_blocks = MINB;
  k.variant = variant;
  return k;
}

// Multi-pass kernels: the passes of one item on the W warps of a block.
template <class P, int R, bool U, bool SAME, int W>
KernelInfo make_pipe_info(int variant) {
  using F = PipeForward<P, R, U, SAME, 1, W>;
  KernelInfo k;
  k.fn = reinterpret_cast<const void*>(&forward_pipe_kernel<P, R, U, SAME, 1, W>);
  k.threads = W * kWarp;
  k.warps_per_block = W;
  k.smem_bytes = W * F::kSmemPerWarp;
  k.rows_per_lane = R;
  k.multi = true;
  k.same_hap = SAME || P::kSlots == 1;
  k.chain = false;
  k.items_per_warp = 1;
  k.items_per_block = 1;
  k.min_blocks = 1;
  k.boundary_rows = F::kRows;
  k.variant = variant;
  return k;
}

// The multi-pass variants of strip height R (pipe_variant_rows) for one
// precision and item kind: W = 2 or 4 warps per item.
template <int R>
KernelInfo pipe_info_for(Precision prec, bool uniform, bool same, int variant) {
  const bool w4 = pipe_variant_warps(variant) == 4;
  if (prec == Precision::kF64) {
    if (uniform)
      return w4 ? make_pipe_info<F64, R, true, false, 4>(variant)
                : make_pipe_info<F64, R, true, false, 2>(variant);
    return w4 ? make_pipe_info<F64, R, false, false, 4>(variant)
              : make_pipe_info<F64, R, false, false, 2>(variant);
  }
  if (same) {
    if (uniform)
      return w4 ? make_pipe_info<F32x2, R, true, true, 4>(variant)
                : make_pipe_info<F32x2, R, true, true, 2>(variant);
    return w4 ? make_pipe_info<F32x2, R, false, true, 4>(variant)
              : make_pipe_info<F32x2, R, false, true, 2>(variant);
  }
  if (uniform)
    return w4 ? make_pipe_info<F32x2, R, true, false, 4>(variant)
              : make_pipe_info<F32x2, R, true, false, 2>(variant);
  return w4 ? make_pipe_info<F32x2, R, false, false, 4>(variant)
            : make_pipe_info<F32x2, R, false, false, 2>(variant);
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

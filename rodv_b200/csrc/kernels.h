// kernels.h -- host-visible handles to the device kernels.
#pragma once
#include <cuda_runtime.h>

namespace rodv {

enum class Precision { kF32x2 = 0, kF64 = 1 };

struct KernelInfo {
  const void* fn = nullptr;   // __global__ forward_kernel<...>(BatchView, ClassLaunch)
  int threads = 0;            // threads per block
  int warps_per_block = 0;
  int smem_bytes = 0;         // dynamic shared memory per block
  int rows_per_lane = 0;      // R
  bool multi = false;         // sweeps reads longer than 32*R rows in passes
  bool same_hap = false;      // both pairs of an item share the haplotype
  bool chain = false;         // takes ChainItem work (single-pass same-haplotype FP32)
  int items_per_warp = 1;     // chain items a warp sweeps at once (one per lane group)
  int items_per_block = 1;    // work items a block has in flight
  int min_blocks = 1;         // launch-bounds occupancy target (caps registers)
  int boundary_rows = 0;      // multi-pass: boundary rows of scratch per block of the grid
  int variant = 0;
};

// Multi-pass (pipelined) kernels: a variant is a strip height R (rows per
// lane per pass: 8 or 4) and the warps W of a block that sweep one item's
// passes concurrently (2 or 4).
constexpr int kPipeVariants = 4;
inline int pipe_variant_rows(int variant) { return (variant & 2) ? 4 : 8; }
inline int pipe_variant_warps(int variant) { return (variant & 1) ? 4 : 2; }

// Variants of the tunable (same-haplotype FP32) kernels: an occupancy target
// (blocks per SM, which caps registers) and, for the chain kernels of reads
// up to 128 bases (R <= 4), the lane grouping: variants 0-3 sweep one chain
// item per warp with R rows per lane, 4-7 two items per warp in 16-lane
// groups with 2R rows per lane.
constexpr int kTuneVariants = 8;
constexpr int kOccupancyTargets = 4;
constexpr int kVariantMinBlocks[kTuneVariants] = {4, 5, 6, 8, 4, 5, 6, 8};
constexpr int kMaxGroupedRows = 4;  // classes with R <= 4 have the grouped variants

// Forward kernel for one work class.  rows_per_lane in 1..8 for single-pass
// kernels; multi-pass kernels take their strip height from the variant.
// same: FP32 items whose reads share the haplotypes -- ChainItem for
// single-pass classes, SameItem for multi-pass ones; !same: DiffItem
// (multi-pass leftovers; in a single-pass class, the pairs of each region's
// odd read).  FP64 kernels take PairRef lists.  variant <
// forward_kernel_variants(...) selects the variant: of same-haplotype FP32
// single-pass kernels, and of every multi-pass kernel (FP32 same and
// two-haplotype items share the class's variant, so they agree on the pass
// count; FP64 ones have their own).
KernelInfo forward_kernel_info(Precision prec, int rows_per_lane, bool uniform, bool multi,
                               bool same = true, int variant = 0);
inline int forward_kernel_variants(Precision prec, bool same, int rows_per_lane = 8,
                                   bool multi = true) {
  if (multi) return kPipeVariants;
  if (prec != Precision::kF32x2 || !same) return 1;
  return rows_per_lane <= kMaxGroupedRows ? kTuneVariants : kOccupancyTargets;
}

// Peak microbenchmarks: kind 0 = FP32 FFMA, 1 = FP32x2 FFMA2, 2 = FP64 DFMA.
// scratch must hold kPeakScratchBytes; the FFMA run stores the SM cycles its
// first block spent at byte offset kPeakCyclesOffset.
constexpr int kPeakCyclesOffset = 32768;
constexpr int kPeakScratchBytes = 65536;
cudaError_t run_peak(int kind, int blocks, int threads, int iters, cudaStream_t st, void* scratch);
double peak_flops_per_launch(int kind, int blocks, int threads, int iters);

}  // namespace rodv

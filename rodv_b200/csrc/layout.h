// layout.h -- device-side data layout shared by the host packer and kernels.
//
// A batch is packed once on the host into these flat arrays (one H2D copy
// each) and stays resident in HBM while the kernels run:
//
//   hap_codes  u8   the haplotypes in batch order as base codes A0 C1 G2 T3
//                   N4, one separator code (kSep) between consecutive
//                   haplotypes, kHapPad code-0 bytes before the first; the
//                   tail holds kHapPad + max_hap_len + kHapPad more, so a warp
//                   whose shorter slot runs past its haplotype end still
//                   reads in bounds.  Any run of consecutive haplotypes is
//                   therefore one column sequence [h0][sep][h1][sep]...
//   read_rows  u32  one word per read base:
//                     bits 0-2 base code, 3-9 q, 10-16 ins, 17-23 del,
//                     24-30 gcp (quals masked with &127 as the reference
//                     does, pairhmm_inter.cpp:85-88); each read starts on a
//                     16-byte boundary.
//   haps       HapDesc[], reads ReadDesc[]
//   items      the FP32 kernels' work, two reads per warp (the two float
//              halves of every f32x2 instruction): ChainItem (read pairs
//              stacked down the lanes against all haplotypes of their
//              region, single-pass reads; their read lists follow the
//              class's items),
//              SameItem (two reads against one haplotype, multi-pass reads) or
//              DiffItem (two PairRef, the multi-pass leftovers)
//   lists      PairRef[] per work class: the FP64 kernels' work (pairs the
//              FP32 kernels rescued, or every pair when FP64 is forced)
//   out        f64[num_pairs]  final log10 likelihood, in the reference's
//              result order (region, hap-major, read-minor)
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define RODV_HD __host__ __device__
#else
#define RODV_HD
#endif

namespace rodv {

constexpr int kWarp = 32;
constexpr int kHapPad = 32;          // code bytes before the first haplotype
constexpr int kChainHaps = 32;       // haplotypes per chain item (one per lane)
constexpr int kMaxRowsPerLane = 8;   // R: read rows held in registers per lane
constexpr int kPassRows = kWarp * kMaxRowsPerLane;  // rows per multi-pass sweep
constexpr uint32_t kNoPair = 0xffffffffu;

// Base codes.  'N' on either side matches every base (common.h:42-56,
// pairhmm_impl.cpp:26-42).
// kSep is the column between two haplotypes of a chain: its emission is 0 for
// every row.
enum BaseCode : uint8_t { kA = 0, kC = 1, kG = 2, kT = 3, kN = 4, kSep = 5 };
constexpr int kNumCodes = 6;

struct HapDesc {
  uint64_t code_off;  // index in hap_codes of the first base
  uint32_t len;
  uint32_t pad_;
};

struct ReadDesc {
  uint64_t row_off;   // index in read_rows of the first row word
  uint32_t len;
  uint32_t flags;     // kReadUniformGaps: ins, del and gcp constant over the read
};
constexpr uint32_t kReadUniformGaps = 1u;

// One (haplotype, read) pair and where its result goes.
struct PairRef {
  uint32_t hap;
  uint32_t read;      // kNoPair marks an empty slot
  uint32_t out;       // index in the output array
};

// Two reads of one region against one haplotype.  The result index of read y
// is out_x + (read_y - read_x): reads of a region are contiguous and results
// are hap-major.  read_y may be kNoPair.
struct SameItem {
  uint32_t hap;
  uint32_t read_x;
  uint32_t read_y;
  uint32_t out_x;
};

// Reads of one region against consecutive haplotypes of the region (up to
// kChainHaps), swept in one pass over their concatenated columns.  The item
// holds `pairs` read pairs, entries [stack, stack + 2 * pairs) of the
// class's stack list (x read, then y read or kNoPair), one pair per run of
// lanes down the warp: a pair takes floor(len / R) + 1 lanes of R rows for
// its longer read (its rows, then at least one pass-through row), x in the
// low float half of the f32x2 lanes and y in the high one, and each pair's
// first lane starts at the chain's first column.  The result of (haplotype
// hap_start + i, read r) goes to out0 + i * stride + (r - read_base): reads
// of a region are contiguous and results are hap-major.  norm_len is the
// length of the region's longest haplotype: row 0 of the sweep is scaled by
// 2^120/norm_len, which depends on the region only, so a pair's result does
// not depend on how the region was cut into chains, nor on the lanes, item
// or kernel its read was given.
struct alignas(16) ChainItem {
  uint32_t hap_start;
  uint32_t num_haps;
  uint32_t stack;     // first entry of the item's read pairs in the class's stack list
  uint32_t pairs;     // read pairs stacked down the lanes
  uint32_t out0;      // out index of (hap_start, read_base)
  uint32_t stride;    // the region's read count
  uint32_t norm_len;
  uint32_t read_base; // the region's first read
};

// Two arbitrary pairs; x has the longer (or equal) haplotype; y.read may be
// kNoPair.
struct DiffItem {
  PairRef x;
  PairRef y;
};

// Passes of a multi-pass sweep of a read of `len` rows with R rows per lane:
// floor(len / 32R) + 1, so the last pass always ends in pass-through rows.
RODV_HD inline uint32_t pipe_passes(uint32_t len, int rows_per_lane) {
  return len / (uint32_t)(kWarp * rows_per_lane) + 1u;
}

RODV_HD inline uint32_t row_word(uint32_t code, uint32_t q, uint32_t ins,
                                             uint32_t del, uint32_t gcp) {
  return (code & 7u) | ((q & 127u) << 3) | ((ins & 127u) << 10) | ((del & 127u) << 17) |
         ((gcp & 127u) << 24);
}
RODV_HD inline uint32_t rw_code(uint32_t w) { return w & 7u; }
RODV_HD inline uint32_t rw_q(uint32_t w) { return (w >> 3) & 127u; }
RODV_HD inline uint32_t rw_ins(uint32_t w) { return (w >> 10) & 127u; }
RODV_HD inline uint32_t rw_del(uint32_t w) { return (w >> 17) & 127u; }
RODV_HD inline uint32_t rw_gcp(uint32_t w) { return (w >> 24) & 127u; }

// Prior tables in the two precisions (Context<float>/Context<double>,
// context.h:22-166): ph2pr[q] and the match-to-match table indexed by
// (max*(max+1))/2 + min of the (ins, del) quals.
constexpr int kMmTableSize = 128 * 129 / 2;
struct PriorTables {
  const float* ph2pr_f;
  const float* mm_f;
  const double* ph2pr_d;
  const double* mm_d;
};

// Everything a forward kernel needs about the resident batch.
struct BatchView {
  const uint8_t* hap_codes;
  const uint32_t* read_rows;
  const HapDesc* haps;
  const ReadDesc* reads;
  double* out;
  // Raw mode (null otherwise): out[] receives the scaled likelihood itself
  // and raw_prec[] the precision that produced it -- 0: FP32, scaled by
  // 2^120/haplen; 1: FP64, scaled by 2^1020/haplen.
  uint8_t* raw_prec;
  PriorTables tab;
};

// One launch of a forward kernel over one class of work.
struct ClassLaunch {
  const void* work;            // SameItem[] / DiffItem[] (FP32) or PairRef[] (FP64)
  const uint32_t* work_count;  // device count (FP64 rescue lists) or null
  uint32_t static_count;       // item count when work_count is null
  uint32_t* counter;           // work counter, zeroed before launch
  PairRef* rescue_list;        // FP32 only: pairs whose result fell below 1e-28
  uint32_t* rescue_count;
  float* scratch;              // MULTI: per resident warp boundary-row buffer
  uint32_t scratch_cols;       // columns per warp buffer (max hap len + 40)
  uint32_t* error_flags;       // bit set by a kernel that hit a bad descriptor
  uint32_t flags;              // kLaunch* bits
  uint32_t wait_polls;         // pipelined sweeps: polls before a wait gives up (0: default)
  uint32_t rescue_base;        // kLaunchRescueByItem: list position of item 0's first pair
  const uint32_t* stack;       // chain items: their read pairs (read indices)
};

// ClassLaunch::flags.  Testing hook: the producers of a pipelined sweep
// publish no progress, so every consumer's wait runs out (its expiry path is
// tested without a fault).
constexpr uint32_t kLaunchNoPublish = 1u;
// FP32 multi-pass launches: the rescue of slot s of item i goes to list
// position rescue_base + 2i + s (the list is cleared to kNoPair entries
// first) instead of the next free one, so the FP64 sweep takes the rescues in
// the items' order -- longest first, as packed -- and not in the order the
// FP32 sweeps rejected them, shortest first.
constexpr uint32_t kLaunchRescueByItem = 2u;

enum ErrorFlag : uint32_t {
  kErrBadLength = 1u,   // a pair with zero or over-limit length reached a kernel
  kErrPassLimit = 2u,   // a read longer than the pass limit reached a kernel
  kErrChain = 4u,       // a chain item with no haplotypes
  kErrNonFinite = 8u,   // a likelihood came out NaN or infinite (an arithmetic fault)
  kErrWaitTimeout = 16u,  // a pipelined sweep waited too long for another warp's progress
};

}  // namespace rodv

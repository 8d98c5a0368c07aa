// engine.h -- the engine behind the C ABI (include/rodv_pairhmm.h).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/rodv_pairhmm.h"
#include "kernels.h"
#include "layout.h"

namespace rodv {

// Work classes: single-pass kernels for R = 1..8 rows per lane (reads up to
// 32*R bases), times {per-row, uniform} gap priors, plus the multi-pass
// kernels for longer reads.
constexpr int kSinglePassClasses = kMaxRowsPerLane * 2;
constexpr int kNumClasses = kSinglePassClasses + 2;

// The single-pass class of R rows per lane and the given gap form.
inline int single_pass_class(int R, bool uniform) { return (R - 1) * 2 + (uniform ? 1 : 0); }
// A single-pass sweep holds a read's rows, then at least one pass-through
// row (so one running sum gives the result) and, in the uniform-gap (scaled)
// form, the row whose D sums that pass-through row over each haplotype's
// columns: a class of R rows per lane holds reads of up to 32R - 1 bases
// with per-row gaps and 32R - 2 with uniform gaps.  Longer reads are
// multi-pass.
inline int class_of(uint32_t read_len, bool uniform) {
  const uint32_t rows = read_len + (uniform ? 2u : 1u);
  if (rows <= (uint32_t)kPassRows)
    return single_pass_class((int)((rows + kWarp - 1) / kWarp), uniform);
  return kSinglePassClasses + (uniform ? 1 : 0);
}
inline int class_rows(int cls) { return cls < kSinglePassClasses ? cls / 2 + 1 : kMaxRowsPerLane; }
inline bool class_uniform(int cls) { return (cls & 1) != 0; }
inline bool class_multi(int cls) { return cls >= kSinglePassClasses; }

// Device counters of one packed batch: per class the work counters of the
// same-haplotype, two-haplotype and FP64 launches and the rescue count, then
// one error word.
enum CounterBlock : int {
  kCtrSame = 0,
  kCtrDiff = kNumClasses,
  kCtrF64 = 2 * kNumClasses,
  kCtrRescue = 3 * kNumClasses,
  kCtrError = 4 * kNumClasses,
  kCountWords = 4 * kNumClasses + 1,
};

// Testing hooks behind rodv_fault_inject_alloc / rodv_debug_live_allocations:
// kind 0 = device (cudaMalloc), 1 = pinned host (cudaMallocHost).
void set_alloc_fault(int kind, int64_t nth);
void set_wait_fault(bool on);
void live_allocations(uint64_t* device, uint64_t* pinned);

struct DeviceMem {
  void* ptr = nullptr;
  size_t bytes = 0;
  ~DeviceMem();
  cudaError_t ensure(size_t n);
};

struct PinnedMem {
  void* ptr = nullptr;
  size_t bytes = 0;
  ~PinnedMem();
  cudaError_t ensure(size_t n);
};

// Host-side description of one packed batch (sizes, per-class counts and the
// byte offsets of every array in the staging buffer / device arena).
struct PackedPlan {
  uint64_t num_pairs = 0, cells = 0;
  uint64_t hap_code_bytes = 0, read_rows = 0;
  uint32_t num_haps = 0, num_reads = 0;
  uint32_t max_hap_len = 0;
  uint32_t multi_max_hap = 0;
  bool fp64 = false;                       // every pair computed in FP64
  bool raw = false;                        // raw likelihoods and their precision
  // FP32 same-haplotype items: ChainItem for single-pass classes, SameItem
  // for the multi-pass ones
  uint32_t same_items[kNumClasses] = {};
  uint32_t diff_items[kNumClasses] = {};   // FP32 two-haplotype items (multi-pass leftovers)
  uint32_t chain_haps[kNumClasses] = {};   // haplotypes per chain item (single-pass classes)
  int variant[kNumClasses] = {};           // kernel variant per class the items were packed for
  int variant64[kNumClasses] = {};         // FP64 kernel variant per class
  uint32_t pairs[kNumClasses] = {};        // pairs per class
  // FP64 list capacity per class: the pairs, or for a multi-pass class in an
  // FP32 run two positions per FP32 item (kLaunchRescueByItem)
  uint32_t list_cap[kNumClasses] = {};
  size_t off_hap_codes = 0, off_read_rows = 0, off_haps = 0, off_reads = 0;
  size_t off_same[kNumClasses] = {};
  size_t off_stack[kNumClasses] = {};      // chain items' bins: read indices (uint32)
  size_t off_diff[kNumClasses] = {};
  size_t off_lists[kNumClasses] = {};      // FP64 work lists (rescued or forced)
  size_t off_preset = 0;                   // forced FP64: list lengths (uploaded)
  size_t upload_bytes = 0;                 // the H2D part starts at 0
  size_t off_out = 0, off_counts = 0, off_scratch = 0;
  size_t off_prec = 0;                     // raw mode: precision byte per pair
  size_t total_bytes = 0;
  size_t scratch_bytes = 0;
  uint32_t scratch_cols = 0;
  // host copies kept for the plain per-pair form
  std::vector<rodv_region> regions;
  std::vector<uint32_t> hap_len;
  std::vector<uint8_t> read_class;
};

// Records the message rodv_last_error(NULL) returns (a failed engine creation).
void set_create_error(const std::string& msg);

// Checks a batch's regions, lengths, limits and (check_bases) every base;
// the status and message the engine would fail the batch with.
rodv_status validate_batch(const rodv_batch& b, bool check_bases, uint64_t* num_pairs,
                           std::string* msg);

class Service;

class Engine {
  friend class Service;

 public:
  explicit Engine(const rodv_options& opt);
  ~Engine();
  rodv_status init();
  // Loads every forward kernel variant now instead of at its first launch.
  rodv_status load_kernels();

  // prec: null, or raw mode (rodv_pairhmm_batch_raw): out receives raw
  // likelihoods and prec the precision of each.
  rodv_status run_host(const rodv_batch& b, double* out, rodv_stats* st, bool force_fp64 = false,
                       uint8_t* prec = nullptr);
  rodv_status upload(const rodv_batch& b, rodv_device_batch** out);
  rodv_status run_device(rodv_device_batch* db, rodv_stats* st);
  rodv_status download(rodv_device_batch* db, double* out);
  rodv_status plain(rodv_device_batch* db, double* out, rodv_stats* st);
  rodv_status measure_peaks(double* f32, double* f32x2, double* f64, double* mhz);
  rodv_status autotune(const char* cache_path, int force, int32_t* variants_out);
  // The current FP32 and FP64 kernel variant of every class (either may be null).
  void variants(int32_t* fp32, int32_t* fp64) const {
    for (int c = 0; c < kNumClasses; ++c) {
      if (fp32) fp32[c] = variant_[c];
      if (fp64) fp64[c] = variant64_[c];
    }
  }

  std::mutex& mutex() { return mu_; }
  // One stage of the chunked host-buffer path: a region range packed,
  // uploaded, computed and downloaded on its own stream while the host packs
  // the following ranges into the other lanes.
  struct HostLane {
    PackedPlan plan;
    PinnedMem staging, out;
    DeviceMem arena;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {};        // FP32 start, FP32 end, FP64 end, upload start
    cudaEvent_t done = nullptr;    // after the result download
    std::vector<rodv_region> regs;
    uint64_t out_off = 0;
    bool busy = false;
  };
  const char* last_error() const { return last_error_.c_str(); }
  rodv_status fail(rodv_status s, const std::string& msg);
  rodv_status cuda_fail(cudaError_t e, const char* where);

 private:
  // stack_uniform: uniform-gap reads may stack into bins of the R = 8 class
  // (off: one read per bin, every class keeps its own reads; the autotuner's
  // per-class batches)
  rodv_status pack(const rodv_batch& b, PackedPlan& plan, PinnedMem& staging, bool fp64,
                   bool raw = false, bool stack_uniform = true);
  // parts: 1 = counter reset and FP32 launches, 2 = FP64 launches.  ev: null,
  // or three events recorded before the FP32 launches, between the two parts
  // and after the FP64 launches.  fan_out: each class's launches go to its own
  // side stream (forked from and joined back into `stream`), so that class
  // kernels fill each other's tails.  The side streams are the engine's: the
  // captured resident path, the host-buffer ranges and the service's batches
  // use them from the one thread that launches for the engine at a time.
  rodv_status launch_all(const PackedPlan& plan, uint8_t* dbase, rodv_stats* st,
                         cudaStream_t stream, cudaEvent_t* ev, int parts,
                         bool fan_out = false);
  rodv_status launch_fp32_class(const PackedPlan& plan, uint8_t* dbase, int cls, bool same,
                                int variant, int blocks_cap, cudaStream_t stream);
  rodv_status launch_fp64_class(const PackedPlan& plan, uint8_t* dbase, int cls, int variant,
                                cudaStream_t stream);
  rodv_status check_errors(const PackedPlan& plan, uint8_t* dbase);
  rodv_status run_host_single(const rodv_batch& b, double* out, rodv_stats* st, bool fp64,
                              uint8_t* prec);
  rodv_status run_host_chunked(const rodv_batch& b, double* out, rodv_stats* st, bool fp64,
                               const std::vector<uint32_t>& bounds, uint8_t* prec);
  rodv_status finish_lane(HostLane& lane, double* out, rodv_stats* st, uint8_t* prec);
  int persistent_blocks(const KernelInfo& k) const;
  size_t multi_scratch_rows() const;
  std::string device_key() const;
  bool load_tuning(const std::string& path);
  bool save_tuning(const std::string& path) const;

  rodv_options opt_;
  mutable std::mutex occ_mu_;
  mutable std::unordered_map<const void*, int> occ_cache_;  // kernel -> resident blocks
  int device_ = 0;
  int num_sms_ = 0;
  std::string device_name_;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[4] = {};
  cudaStream_t side_[kNumClasses] = {};  // launch_all fan-out, one per class
  cudaEvent_t fork_ev_ = nullptr, join_ev_[kNumClasses] = {};
  DeviceMem tables_;
  PriorTables tab_{};
  int variant_[kNumClasses] = {};          // tuned FP32 kernel variant per class
  int variant64_[kNumClasses] = {};        // tuned FP64 kernel variant per class
  bool tuned_ = false;
  // buffers of the one-call path (rodv_pairhmm_batch), reused across calls
  PinnedMem staging_;
  PinnedMem out_staging_;
  DeviceMem arena_;
  static constexpr int kHostLanes = 3;
  HostLane lanes_[kHostLanes];
  std::mutex mu_;
  std::string last_error_;
  bool ready_ = false;
};

}  // namespace rodv

// Opaque handles of the C ABI.
struct rodv_engine {
  rodv::Engine* impl;
};

struct rodv_device_batch {
  rodv::PackedPlan plan;
  rodv::DeviceMem arena;
  // The per-step launch sequence (counter reset, FP32 and FP64 class
  // launches) captured once as two CUDA graphs and replayed by every run.
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // FP32 part, FP64 part
  uint32_t graph_launches = 0;
  ~rodv_device_batch() {
    for (cudaGraphExec_t g : graph)
      if (g) cudaGraphExecDestroy(g);
  }
};

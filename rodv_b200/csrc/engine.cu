// engine.cu -- host side of the PairHMM engine: validation, packing, class
// planning, persistent launches, FP64 rescue, autotuning, results.
//
// Control flow of one batch (the B200 counterpart of schedule_pairhmm,
// src/core/pairhmm_schedule.cpp:116-340):
//   1. validate and pack on the host (threads over regions and reads) into one
//      pinned staging buffer laid out exactly like the device arena;
//   2. one H2D copy of the staging buffer;
//   3. per work class, one persistent FP32 launch over its chain items (two
//      reads of a region against all its haplotypes per warp; reads of up to
//      256 bases) or, for longer reads, over same-haplotype items (two reads
//      against one haplotype) and leftover two-haplotype items; pairs whose
//      scaled FP32 result is below 1e-28 are appended to the class's FP64
//      list on the device;
//   4. per work class, one persistent FP64 launch that drains that list (its
//      length is read by the kernel, never by the host);
//   5. one D2H copy of the log10 results.
// The reference instead groups pairs into SIMD-width groups by padded area
// (greedy_grouping, :46-105) and sends leftovers to a per-pair kernel; here
// work classes (rows per lane) and per-region chains play that part.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <functional>
#include <memory>
#include <mutex>
#include <random>
#include <sstream>
#include <thread>

#include "engine.h"
#include "chain_plan.h"
#include "tables.h"
#include "trace.h"
#include "worker_pool.h"

namespace rodv {

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v, size_t a = kAlign) { return (v + a - 1) / a * a; }

// A0 C1 G2 T3 N4; 0xff marks a base outside the engine's domain.
struct CodeTable {
  uint8_t v[256];
  CodeTable() {
    std::memset(v, 0xff, sizeof(v));
    v['A'] = kA; v['C'] = kC; v['G'] = kG; v['T'] = kT; v['N'] = kN;
  }
};
const CodeTable kCodes;

// Section timer of the packer, printed at verbose level 2.
struct PackTimer {
  bool on;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  std::string line;
  explicit PackTimer(bool enabled) : on(enabled) {}
  void mark(const char* what) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    char buf[64];
    snprintf(buf, sizeof(buf), " %s %.2f", what,
             std::chrono::duration<double, std::milli>(now - t).count());
    line += buf;
    t = now;
  }
  ~PackTimer() {
    if (on) fprintf(stderr, "rodv: pack ms:%s\n", line.c_str());
  }
};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Device-arena views of a packed plan.
struct ArenaView {
  BatchView view;
  uint32_t* counts;
  float* scratch;
};

ArenaView arena_view(const PackedPlan& p, uint8_t* base, const PriorTables& tab) {
  ArenaView a;
  a.view.hap_codes = base + p.off_hap_codes;
  a.view.read_rows = reinterpret_cast<const uint32_t*>(base + p.off_read_rows);
  a.view.haps = reinterpret_cast<const HapDesc*>(base + p.off_haps);
  a.view.reads = reinterpret_cast<const ReadDesc*>(base + p.off_reads);
  a.view.out = reinterpret_cast<double*>(base + p.off_out);
  a.view.raw_prec = p.raw ? base + p.off_prec : nullptr;
  a.view.tab = tab;
  a.counts = reinterpret_cast<uint32_t*>(base + p.off_counts);
  a.scratch = p.scratch_bytes ? reinterpret_cast<float*>(base + p.off_scratch) : nullptr;
  return a;
}

// Boundary rows of multi-pass class c (each multi-pass class has its own
// region: the two classes' kernels run as parallel graph branches).
float* class_scratch(const PackedPlan& p, const ArenaView& a, int c) {
  if (!a.scratch || !class_multi(c)) return a.scratch;
  return reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(a.scratch) +
                                  (size_t)(c - kSinglePassClasses) * p.scratch_bytes);
}

// Occupancy variant used before (or without) tuning: the register budget
// measured best for each rows-per-lane value on B200.
int default_variant(int cls) {
  const int R = class_rows(cls);
  if (class_multi(cls)) return 1;            // strip height 8, 4 warps per item
  if (R >= 3) return 0;                      // one chain per warp, 4 blocks/SM (128 registers)
  if (R == 2) return 4;                      // two 16-lane groups, 4 blocks/SM
  return 6;                                  // two 16-lane groups, 6 blocks/SM (80 registers)
}
// FP64 kernels: multi-pass classes have the pipelined variants, the others one.
int default_variant64(int cls) { return class_multi(cls) ? 1 : 0; }

}  // namespace

// Every device and pinned-host allocation of the engine and the service goes
// through DeviceMem / PinnedMem.  Testing hooks (rodv_fault_inject_alloc,
// rodv_debug_live_allocations): a countdown per kind makes the n-th next
// allocation fail on the host, as cudaMalloc / cudaMallocHost fail when memory
// is exhausted, and live counters show that a failed call released what it
// had allocated.
namespace {
std::atomic<int64_t> g_fail_countdown[2];  // 0: device, 1: pinned host
std::atomic<int64_t> g_live[2];

bool injected_failure(int kind) {
  int64_t v = g_fail_countdown[kind].load();
  while (v > 0)
    if (g_fail_countdown[kind].compare_exchange_weak(v, v - 1)) return v == 1;
  return false;
}
}  // namespace

void set_alloc_fault(int kind, int64_t nth) { g_fail_countdown[kind].store(nth > 0 ? nth : 0); }

// Testing hook (rodv_fault_inject_wait): multi-pass launches made while it is
// set publish no progress and give up a wait after kTestWaitPolls polls.
namespace {
std::atomic<bool> g_wait_fault{false};
constexpr uint32_t kTestWaitPolls = 1u << 12;
void apply_wait_fault(ClassLaunch& cl, int cls) {
  if (class_multi(cls) && g_wait_fault.load()) {
    cl.flags |= kLaunchNoPublish;
    cl.wait_polls = kTestWaitPolls;
  }
}
}  // namespace
void set_wait_fault(bool on) { g_wait_fault.store(on); }
void live_allocations(uint64_t* device, uint64_t* pinned) {
  if (device) *device = (uint64_t)g_live[0].load();
  if (pinned) *pinned = (uint64_t)g_live[1].load();
}

DeviceMem::~DeviceMem() {
  if (ptr) {
    cudaFree(ptr);
    --g_live[0];
  }
}
cudaError_t DeviceMem::ensure(size_t n) {
  if (n <= bytes && ptr) return cudaSuccess;
  if (ptr) {
    cudaFree(ptr);
    --g_live[0];
  }
  ptr = nullptr;
  bytes = 0;
  if (injected_failure(0)) return cudaErrorMemoryAllocation;
  cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(n, 1));
  if (e == cudaSuccess) {
    bytes = n;
    ++g_live[0];
  } else {
    ptr = nullptr;
  }
  return e;
}
PinnedMem::~PinnedMem() {
  if (ptr) {
    cudaFreeHost(ptr);
    --g_live[1];
  }
}
cudaError_t PinnedMem::ensure(size_t n) {
  if (n <= bytes && ptr) return cudaSuccess;
  if (ptr) {
    cudaFreeHost(ptr);
    --g_live[1];
  }
  ptr = nullptr;
  bytes = 0;
  if (injected_failure(1)) return cudaErrorMemoryAllocation;
  cudaError_t e = cudaMallocHost(&ptr, std::max<size_t>(n, 1));
  if (e == cudaSuccess) {
    bytes = n;
    ++g_live[1];
  } else {
    ptr = nullptr;
  }
  return e;
}

Engine::Engine(const rodv_options& opt) : opt_(opt) {
  for (int c = 0; c < kNumClasses; ++c) {
    variant_[c] = default_variant(c);
    variant64_[c] = default_variant64(c);
  }
}

Engine::~Engine() {
  if (ready_) {
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    for (auto& e : ev_) cudaEventDestroy(e);
    cudaStreamDestroy(stream_);
    for (int c = 0; c < kNumClasses; ++c) {
      if (side_[c]) cudaStreamSynchronize(side_[c]);
      if (side_[c]) cudaStreamDestroy(side_[c]);
      if (join_ev_[c]) cudaEventDestroy(join_ev_[c]);
    }
    if (fork_ev_) cudaEventDestroy(fork_ev_);
    for (HostLane& l : lanes_) {
      if (l.stream) cudaStreamSynchronize(l.stream);
      for (cudaEvent_t e : l.ev)
        if (e) cudaEventDestroy(e);
      if (l.done) cudaEventDestroy(l.done);
      if (l.stream) cudaStreamDestroy(l.stream);
    }
  }
}

rodv_status Engine::fail(rodv_status s, const std::string& msg) {
  last_error_ = msg;
  if (opt_.verbose) fprintf(stderr, "rodv: %s\n", msg.c_str());
  return s;
}

rodv_status Engine::cuda_fail(cudaError_t e, const char* where) {
  const rodv_status s = (e == cudaErrorMemoryAllocation) ? RODV_ERR_OUT_OF_MEMORY : RODV_ERR_CUDA;
  return fail(s, std::string(where) + ": " + cudaGetErrorString(e));
}

#define RODV_CUDA(call)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

rodv_status Engine::init() {
  cudaGetLastError();  // clear a stale error of an earlier call on this thread
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return fail(RODV_ERR_NO_DEVICE, "no CUDA device visible");
  if (opt_.device < 0 || opt_.device >= n)
    return fail(RODV_ERR_NO_DEVICE, "device ordinal out of range");
  device_ = opt_.device;
  RODV_CUDA(cudaSetDevice(device_));
  cudaDeviceProp prop;
  RODV_CUDA(cudaGetDeviceProperties(&prop, device_));
  if (prop.major != 10 || prop.minor != 0)
    return fail(RODV_ERR_NO_DEVICE, std::string("engine is built for sm_100a; device is ") +
                                        prop.name);
  num_sms_ = prop.multiProcessorCount;
  device_name_ = prop.name;
  RODV_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  for (auto& e : ev_) RODV_CUDA(cudaEventCreate(&e));
  ready_ = true;  // the destructor releases what was created
  RODV_CUDA(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
  for (int c = 0; c < kNumClasses; ++c) {
    RODV_CUDA(cudaStreamCreateWithFlags(&side_[c], cudaStreamNonBlocking));
    RODV_CUDA(cudaEventCreateWithFlags(&join_ev_[c], cudaEventDisableTiming));
  }
  for (HostLane& l : lanes_) {
    RODV_CUDA(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking));
    for (auto& e : l.ev) RODV_CUDA(cudaEventCreate(&e));
    RODV_CUDA(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming));
  }
  const HostPriorTables& t = host_prior_tables();
  const size_t bytes = 128 * 4 + kMmTableSize * 4 + 128 * 8 + kMmTableSize * 8 + 4 * kAlign;
  RODV_CUDA(tables_.ensure(bytes));
  uint8_t* base = static_cast<uint8_t*>(tables_.ptr);
  size_t o = 0;
  cudaError_t ce = cudaSuccess;
  auto put = [&](const void* src, size_t n) -> void* {
    void* dst = base + o;
    if (ce == cudaSuccess) ce = cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice);
    o = align_up(o + n);
    return dst;
  };
  tab_.ph2pr_f = static_cast<const float*>(put(t.ph2pr_f.data(), 128 * 4));
  tab_.mm_f = static_cast<const float*>(put(t.mm_f.data(), kMmTableSize * 4));
  tab_.ph2pr_d = static_cast<const double*>(put(t.ph2pr_d.data(), 128 * 8));
  tab_.mm_d = static_cast<const double*>(put(t.mm_d.data(), kMmTableSize * 8));
  RODV_CUDA(ce);
  // Kernels whose tables exceed the default 48 KB of dynamic shared memory
  // per block opt in to their size.
  for (int c = 0; c < kNumClasses; ++c)
    for (int p = 0; p < 3; ++p)
      for (int v = 0; v < kTuneVariants; ++v) {
        const Precision pr = p == 2 ? Precision::kF64 : Precision::kF32x2;
        if (v >= forward_kernel_variants(pr, p == 0, class_rows(c), class_multi(c))) continue;
        const KernelInfo k =
            forward_kernel_info(pr, class_rows(c), class_uniform(c), class_multi(c), p == 0, v);
        if (k.fn && k.smem_bytes > 48 * 1024)
          RODV_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         k.smem_bytes));
      }
  ready_ = true;
  if (opt_.tune_cache && opt_.tune_cache[0]) load_tuning(opt_.tune_cache);
  if (opt_.autotune) {
    rodv_status s = autotune(opt_.tune_cache, opt_.autotune > 1, nullptr);
    if (s != RODV_OK) return s;
  }
  return RODV_OK;
}

// Every forward kernel the engine can launch, loaded now: with CUDA's lazy
// module loading a kernel's first launch loads it, which stalls that launch
// for milliseconds (the occupancy query both loads it and fills the cache
// persistent_blocks uses).
rodv_status Engine::load_kernels() {
  RODV_CUDA(cudaSetDevice(device_));
  for (int c = 0; c < kNumClasses; ++c)
    for (int p = 0; p < 3; ++p) {
      const Precision pr = p == 2 ? Precision::kF64 : Precision::kF32x2;
      const int nv = forward_kernel_variants(pr, p == 0, class_rows(c), class_multi(c));
      for (int v = 0; v < nv; ++v) {
        const KernelInfo k =
            forward_kernel_info(pr, class_rows(c), class_uniform(c), class_multi(c), p == 0, v);
        if (k.fn) persistent_blocks(k);
      }
    }
  RODV_CUDA(cudaGetLastError());
  return RODV_OK;
}

// Boundary rows a multi-pass class's kernels need: per block of the largest
// grid any multi-pass kernel variant launches (the autotuner runs every
// variant on its batches).
size_t Engine::multi_scratch_rows() const {
  size_t rows = 0;
  for (int u = 0; u < 2; ++u)
    for (int p = 0; p < 3; ++p)
      for (int v = 0; v < kPipeVariants; ++v) {
        const Precision pr = p == 2 ? Precision::kF64 : Precision::kF32x2;
        const KernelInfo k = forward_kernel_info(pr, kMaxRowsPerLane, u != 0, true, p == 0, v);
        rows = std::max(rows, (size_t)persistent_blocks(k) * k.boundary_rows);
      }
  return rows;
}

// Resident blocks of a kernel on the whole device, queried once per kernel
// (the occupancy query costs more than a launch).
int Engine::persistent_blocks(const KernelInfo& k) const {
  {
    std::lock_guard<std::mutex> lk(occ_mu_);
    auto it = occ_cache_.find(k.fn);
    if (it != occ_cache_.end()) return it->second;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, k.smem_bytes) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  std::lock_guard<std::mutex> lk(occ_mu_);
  occ_cache_[k.fn] = per_sm * num_sms_;
  return per_sm * num_sms_;
}

// ---------------------------------------------------------------------------
// Packing
// ---------------------------------------------------------------------------
rodv_status validate_batch(const rodv_batch& b, bool check_bases, uint64_t* num_pairs,
                           std::string* msg) {
  auto bad = [&](rodv_status st, const std::string& m) {
    if (msg) *msg = m;
    return st;
  };
  if (b.num_regions == 0 || !b.regions) return bad(RODV_ERR_EMPTY, "batch has no regions");
  if (!b.hap_bases || !b.hap_offsets || !b.hap_lengths || !b.read_bases || !b.base_quals ||
      !b.ins_quals || !b.del_quals || !b.gcp_quals || !b.read_offsets || !b.read_lengths)
    return bad(RODV_ERR_INVALID_ARG, "null array in batch");
  uint64_t pairs = 0;
  for (uint32_t g = 0; g < b.num_regions; ++g) {
    const rodv_region& r = b.regions[g];
    if (r.num_haps == 0 || r.num_reads == 0)
      return bad(RODV_ERR_EMPTY, "region " + std::to_string(g) + " has no haplotypes or reads");
    if ((uint64_t)r.hap_start + r.num_haps > b.num_haps ||
        (uint64_t)r.read_start + r.num_reads > b.num_reads)
      return bad(RODV_ERR_INVALID_ARG, "region " + std::to_string(g) + " indexes out of range");
    pairs += (uint64_t)r.num_haps * r.num_reads;
  }
  if (pairs >= 0xffffffffull) return bad(RODV_ERR_TOO_LONG, "batch has 2^32 or more pairs");
  for (uint32_t h = 0; h < b.num_haps; ++h) {
    const uint32_t len = b.hap_lengths[h];
    if (len == 0) return bad(RODV_ERR_INVALID_ARG, "haplotype " + std::to_string(h) + " is empty");
    if (len > RODV_MAX_HAP_LEN) return bad(RODV_ERR_TOO_LONG, "haplotype longer than limit");
    if (check_bases)
      for (uint32_t k = 0; k < len; ++k)
        if (kCodes.v[b.hap_bases[b.hap_offsets[h] + k]] == 0xff)
          return bad(RODV_ERR_INVALID_BASE, "haplotype base is not one of A, C, G, T, N");
  }
  for (uint32_t r = 0; r < b.num_reads; ++r) {
    const uint32_t len = b.read_lengths[r];
    if (len == 0) return bad(RODV_ERR_INVALID_ARG, "read " + std::to_string(r) + " is empty");
    if (len > RODV_MAX_READ_LEN) return bad(RODV_ERR_TOO_LONG, "read longer than limit");
    if (check_bases)
      for (uint32_t k = 0; k < len; ++k)
        if (kCodes.v[b.read_bases[b.read_offsets[r] + k]] == 0xff)
          return bad(RODV_ERR_INVALID_BASE, "read base is not one of A, C, G, T, N");
  }
  if (num_pairs) *num_pairs = pairs;
  return RODV_OK;
}

namespace {

// Whether every byte of p[0, n) has low 7 bits v (a quality array of one
// value), eight bytes at a time.
bool low7_all_equal(const uint8_t* p, uint32_t n, uint8_t v) {
  const uint64_t pat = 0x0101010101010101ull * v, mask = 0x7f7f7f7f7f7f7f7full;
  uint32_t k = 0;
  for (; k + 8 <= n; k += 8) {
    uint64_t w;
    std::memcpy(&w, p + k, 8);
    if ((w & mask) != pat) return false;
  }
  for (; k < n; ++k)
    if ((p[k] & 127) != v) return false;
  return true;
}

}  // namespace

rodv_status Engine::pack(const rodv_batch& b, PackedPlan& plan, PinnedMem& staging, bool fp64,
                         bool raw, bool stack_uniform) {
  TraceRange trace("rodv: pack");
  PackTimer timer(opt_.verbose >= 2);
  plan = PackedPlan{};
  plan.fp64 = fp64;
  plan.raw = raw;
  uint64_t pairs = 0;
  {
    std::string msg;
    const rodv_status vs = validate_batch(b, false, &pairs, &msg);
    if (vs != RODV_OK) return fail(vs, msg);
  }
  const uint32_t G = b.num_regions;
  plan.num_pairs = pairs;
  plan.num_haps = b.num_haps;
  plan.num_reads = b.num_reads;
  plan.regions.assign(b.regions, b.regions + G);
  plan.hap_len.assign(b.hap_lengths, b.hap_lengths + b.num_haps);

  // haplotype code buffer: [pad][hap 0][sep][hap 1][sep]...[hap n-1][sep]
  // [pad + max len + pad]; any run of consecutive haplotypes is one chain.
  std::vector<uint64_t> hap_code_off(b.num_haps);
  uint64_t hb = kHapPad;
  uint32_t max_h = 0;
  for (uint32_t h = 0; h < b.num_haps; ++h) {
    const uint32_t len = b.hap_lengths[h];
    if (len == 0) return fail(RODV_ERR_INVALID_ARG, "haplotype " + std::to_string(h) + " is empty");
    if (len > RODV_MAX_HAP_LEN) return fail(RODV_ERR_TOO_LONG, "haplotype longer than limit");
    hap_code_off[h] = hb;
    hb += len + 1;
    max_h = std::max(max_h, len);
  }
  const uint64_t tail_begin = hb;
  hb += kHapPad + max_h + kHapPad;
  plan.hap_code_bytes = hb;
  plan.max_hap_len = max_h;

  std::vector<uint64_t> row_off(b.num_reads);
  uint64_t rows = 0;
  for (uint32_t r = 0; r < b.num_reads; ++r) {
    const uint32_t len = b.read_lengths[r];
    if (len == 0) return fail(RODV_ERR_INVALID_ARG, "read " + std::to_string(r) + " is empty");
    if (len > RODV_MAX_READ_LEN) return fail(RODV_ERR_TOO_LONG, "read longer than limit");
    row_off[r] = rows;
    rows += (len + 3) & ~3u;
  }
  plan.read_rows = rows;

  timer.mark("validate+offsets");
  // ---- read flags (uniform gaps) and class of every read ----
  std::vector<uint8_t>& read_class = plan.read_class;
  read_class.resize(b.num_reads);
  const HostPriorTables& pt = host_prior_tables();
  parallel_for(b.num_reads, 512, [&](size_t lo, size_t hi) {
    for (size_t r = lo; r < hi; ++r) {
      const uint64_t off = b.read_offsets[r];
      const uint32_t n = b.read_lengths[r];
      const uint8_t i0 = b.ins_quals[off] & 127, d0 = b.del_quals[off] & 127,
                    c0 = b.gcp_quals[off] & 127;
      const bool u = low7_all_equal(b.ins_quals + off, n, i0) &&
                     low7_all_equal(b.del_quals + off, n, d0) &&
                     low7_all_equal(b.gcp_quals + off, n, c0);
      // Uniform-gap classes: ins, del and gcp constant, ins == del (the
      // single-pass kernels' scaled form needs mi == md), gcp quality not 0
      // (gapm = 0), and c = mi*gapm >= 1e-6, so that M/gapm*c -- which the
      // scaled form keeps -- stays far from the FP32 denormal range for any
      // likelihood the FP32 pass accepts.  Other reads take the per-row
      // kernels.
      const bool uniform = u && c0 != 0 && i0 == d0 &&
                           (double)pt.ph2pr_f[i0] * (1.0 - (double)pt.ph2pr_f[c0]) >= 1e-6;
      read_class[r] = (uint8_t)class_of(n, uniform);
    }
  });

  timer.mark("classes");
  // ---- per region and class: reads, chain items, same items, leftovers ----
  // Single-pass reads of a region are sorted by (uniform gaps, length).
  // Reads with per-row gap priors pair neighbour by neighbour, one read per
  // bin of a chain item, the pair in the class of its longer read (an odd
  // last one pairs with the shortest uniform read, in a per-row class).
  // Uniform reads either do the same or, where the cost model below finds it
  // cheaper, stack into bins of the R = 8 uniform class (stack_uniform).
  // Each item takes ceil(haps / chain_haps[class]) chain items.  An odd last
  // read is a leftover: its pairs (one per haplotype) go into two-haplotype
  // items with other regions' leftover pairs of its class, so that both
  // halves of the f32x2 lanes work (a one-read chain leaves one half idle; a
  // batch of one-read regions ran at half the FP32 rate).  Whether a read is
  // a leftover depends on its region only, and a pair's arithmetic does not
  // depend on its partner, bin, lanes or kernel, so results do not depend on
  // the rest of the batch.
  // Multi-pass reads keep their own class: same-haplotype items per
  // haplotype, leftovers in two-haplotype items.
  const uint32_t K = kNumClasses;
  auto sorted_single = [&](const rodv_region& rg, std::vector<uint32_t>& out_reads) {
    sort_single_pass(b.read_lengths, read_class.data(), rg.read_start, rg.num_reads, out_reads);
  };
  // the uniform classes' item geometry, from the kernel variants packed for
  int chain_ipw[kMaxRowsPerLane + 1] = {};
  for (int R = 1; R <= kMaxRowsPerLane; ++R)
    chain_ipw[R] = forward_kernel_info(Precision::kF32x2, R, true, false, true,
                                       variant_[single_pass_class(R, true)])
                       .items_per_warp;
  ChainGeom geom[kMaxRowsPerLane + 1];
  chain_geometry(chain_ipw, geom);
  auto region_chains = [&](const std::vector<uint32_t>& sr, RegionChains& rc) {
    plan_region_chains(b.read_lengths, read_class.data(), geom, stack_uniform, sr, rc);
  };
  std::vector<uint32_t> rc((size_t)G * K, 0);      // reads of class c in region g
  std::vector<uint32_t> rpairs((size_t)G * K, 0);  // bin pairs of chain class c in region g
  std::vector<uint32_t> chains((size_t)G * K, 0);  // chain items of class c in region g
  std::vector<uint64_t> cpairs((size_t)G * K, 0);  // pairs those chains compute
  std::vector<uint32_t> nstack((size_t)G * K, 0);  // reads in those bins (stack list entries)
  std::vector<uint64_t> hsum(G, 0);
  std::vector<uint32_t> hmax(G, 0);
  // multi-pass leftovers: the last read of each multi-pass class in the region
  std::vector<uint32_t> left_read((size_t)G * 2, kNoPair);
  // single-pass leftover: the odd last read of the region's sorted single-pass reads
  std::vector<uint32_t> single_read(G, kNoPair);
  std::atomic<bool> chain_class_bad{false};  // a chain item outside the single-pass classes
  parallel_for(G, 16, [&](size_t lo, size_t hi) {
    std::vector<uint32_t> sr;
    RegionChains chs;
    for (size_t g = lo; g < hi; ++g) {
      const rodv_region& rg = b.regions[g];
      for (uint32_t r = 0; r < rg.num_reads; ++r) {
        const uint32_t read = rg.read_start + r;
        const int c = read_class[read];
        rc[g * K + c]++;
        if (class_multi(c)) left_read[g * 2 + (c - kSinglePassClasses)] = read;
      }
      for (int u = 0; u < 2; ++u)
        if (!(rc[g * K + kSinglePassClasses + u] & 1)) left_read[g * 2 + u] = kNoPair;
      for (uint32_t h = 0; h < rg.num_haps; ++h) {
        hsum[g] += b.hap_lengths[rg.hap_start + h];
        hmax[g] = std::max(hmax[g], b.hap_lengths[rg.hap_start + h]);
      }
      if (fp64) continue;
      sorted_single(rg, sr);
      region_chains(sr, chs);
      for (const ChainPairs& ci : chs.items) {
        if (ci.cls < 0 || ci.cls >= kSinglePassClasses) {
          chain_class_bad.store(true);
          break;
        }
        rpairs[g * K + ci.cls] += 1;
        nstack[g * K + ci.cls] += 2 * ci.pairs;
        cpairs[g * K + ci.cls] += (uint64_t)rg.num_haps * 2 * ci.pairs;
      }
      if (chs.leftover != kNoPair) {
        single_read[g] = chs.leftover;
        cpairs[g * K + read_class[chs.leftover]] += rg.num_haps;
      }
    }
  });
  if (chain_class_bad.load())
    return fail(RODV_ERR_INTERNAL, "packer placed a chain item outside the single-pass classes");
  // Haplotypes per chain item, per class: the longest chains (up to
  // kChainHaps) that still leave every resident warp of the class's launch
  // (16 per SM at most) two items; a small batch gets short chains (down to
  // one haplotype).
  for (int c = 0; c < kNumClasses; ++c) {
    plan.variant[c] = variant_[c];
    plan.variant64[c] = variant64_[c];
  }
  for (int c = 0; c < kSinglePassClasses; ++c) {
    // chain items a warp of this class's kernel sweeps at once
    const int ipw = forward_kernel_info(Precision::kF32x2, class_rows(c), class_uniform(c),
                                        false, true, plan.variant[c]).items_per_warp;
    const uint64_t target_items = (uint64_t)num_sms_ * 16 * 2 * ipw;
    plan.chain_haps[c] = 1;
    for (uint32_t cap = kChainHaps / ipw; cap >= 1; cap /= 2) {
      uint64_t items = 0;
      for (uint32_t g = 0; g < G; ++g)
        items += (uint64_t)rpairs[(size_t)g * K + c] * ((b.regions[g].num_haps + cap - 1) / cap);
      if (items >= target_items || cap == 1) {
        plan.chain_haps[c] = cap;
        break;
      }
    }
  }
  for (uint32_t g = 0; g < G; ++g)
    for (int c = 0; c < kSinglePassClasses; ++c)
      chains[(size_t)g * K + c] = rpairs[(size_t)g * K + c] *
          ((b.regions[g].num_haps + plan.chain_haps[c] - 1) / plan.chain_haps[c]);
  // Chain items are laid out region by region in decreasing order of the
  // region's haplotype-length sum (a chain's cost), so the persistent
  // kernels take the longest chains first.
  std::vector<uint32_t> order(G);
  for (uint32_t g = 0; g < G; ++g) order[g] = g;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t x, uint32_t y) { return hsum[x] > hsum[y]; });
  // prefix offsets (within each class) of same/chain items, leftovers, FP64 list entries
  std::vector<uint64_t> same_off((size_t)G * K), left_off((size_t)G * K), list_off((size_t)G * K),
      stack_off((size_t)G * K);
  uint64_t same_tot[kNumClasses] = {}, left_tot[kNumClasses] = {}, list_tot[kNumClasses] = {},
           cap_tot[kNumClasses] = {}, stack_tot[kNumClasses] = {};
  for (uint32_t i = 0; i < G; ++i) {
    const uint32_t g = order[i];
    const uint64_t H = b.regions[g].num_haps;
    for (int c = 0; c < kNumClasses; ++c) {
      const uint64_t n = rc[(size_t)g * K + c];
      same_off[(size_t)g * K + c] = same_tot[c];
      left_off[(size_t)g * K + c] = left_tot[c];
      list_off[(size_t)g * K + c] = list_tot[c];
      stack_off[(size_t)g * K + c] = stack_tot[c];
      stack_tot[c] += nstack[(size_t)g * K + c];
      list_tot[c] += H * n;
      if (class_multi(c)) {
        same_tot[c] += H * (n / 2);
        left_tot[c] += H * (n & 1);
        cap_tot[c] += H * n;
      } else {
        same_tot[c] += chains[(size_t)g * K + c];
        cap_tot[c] += cpairs[(size_t)g * K + c];
        if (single_read[g] != kNoPair && read_class[single_read[g]] == c) left_tot[c] += H;
      }
    }
  }
  // Multi-pass leftovers are paired with leftovers of the same pass count at
  // the class's strip height, so neither slot of an item sweeps passes of
  // pass-through rows only.  (A result does not depend on the partner: the
  // last pass always ends in pass-through rows, pipe_passes.)
  auto passes_of = [&](uint32_t read) -> uint32_t {
    const int c = read_class[read];
    if (!class_multi(c)) return 1u;  // single-pass leftovers: one group
    return pipe_passes(b.read_lengths[read], pipe_variant_rows(plan.variant[c]));
  };
  std::vector<uint64_t> left_by_passes[2];
  for (int u = 0; u < 2; ++u) left_by_passes[u].assign(RODV_MAX_READ_LEN / (kWarp * 4) + 2, 0);
  for (uint32_t g = 0; g < G; ++g)
    for (int u = 0; u < 2; ++u)
      if (left_read[g * 2 + u] != kNoPair)
        left_by_passes[u][passes_of(left_read[g * 2 + u])] += b.regions[g].num_haps;
  for (int c = 0; c < kNumClasses; ++c) {
    // FP64 list capacity: every pair whose FP32 work is in class c (or, FP64
    // forced, every pair whose read is of class c)
    plan.pairs[c] = (uint32_t)(fp64 ? list_tot[c] : cap_tot[c]);
    plan.same_items[c] = fp64 ? 0u : (uint32_t)same_tot[c];
    uint64_t diff = (left_tot[c] + 1) / 2;  // single-pass leftovers pair freely
    if (class_multi(c)) {
      diff = 0;
      for (uint64_t n : left_by_passes[c - kSinglePassClasses]) diff += (n + 1) / 2;
    }
    plan.diff_items[c] = fp64 ? 0u : (uint32_t)diff;
  }
  for (uint32_t g = 0; g < G; ++g) {
    const rodv_region& rg = b.regions[g];
    if (rc[(size_t)g * K + kSinglePassClasses] || rc[(size_t)g * K + kSinglePassClasses + 1])
      for (uint32_t h = 0; h < rg.num_haps; ++h)
        plan.multi_max_hap = std::max(plan.multi_max_hap, b.hap_lengths[rg.hap_start + h]);
  }

  timer.mark("pairing");
  // ---- arena layout ----
  size_t o = 0;
  plan.off_hap_codes = o; o = align_up(o + hb);
  plan.off_read_rows = o; o = align_up(o + rows * 4);
  plan.off_haps = o; o = align_up(o + (size_t)b.num_haps * sizeof(HapDesc));
  plan.off_reads = o; o = align_up(o + (size_t)b.num_reads * sizeof(ReadDesc));
  for (int c = 0; c < kNumClasses; ++c) {
    plan.off_same[c] = o;
    const size_t item = class_multi(c) ? sizeof(SameItem) : sizeof(ChainItem);
    o = align_up(o + (size_t)plan.same_items[c] * item);
    plan.off_stack[c] = o;  // chain items' bins
    if (!fp64 && !class_multi(c)) o = align_up(o + (size_t)stack_tot[c] * 4);
  }
  for (int c = 0; c < kNumClasses; ++c) {
    plan.off_diff[c] = o;
    o = align_up(o + (size_t)plan.diff_items[c] * sizeof(DiffItem));
  }
  const size_t lists_begin = o;
  for (int c = 0; c < kNumClasses; ++c) {
    plan.list_cap[c] = plan.pairs[c];
    if (!fp64 && class_multi(c))
      plan.list_cap[c] = std::max(plan.pairs[c], 2u * (plan.same_items[c] + plan.diff_items[c]));
    plan.off_lists[c] = o;
    o = align_up(o + (size_t)plan.list_cap[c] * sizeof(PairRef));
  }
  // forced FP64: the lists are full from the start; their lengths are uploaded
  // too and copied into the counters at every run
  plan.off_preset = o;
  if (fp64) o = align_up(o + kNumClasses * 4);
  // FP32 runs fill the lists on the device; only forced-FP64 lists are uploaded.
  plan.upload_bytes = fp64 ? o : lists_begin;
  plan.off_out = o; o = align_up(o + pairs * 8);
  plan.off_counts = o; o = align_up(o + kCountWords * 4);
  plan.off_prec = o;
  if (raw) o = align_up(o + pairs);
  plan.scratch_cols = plan.multi_max_hap ? plan.multi_max_hap + 40 : 0;
  plan.off_scratch = o;
  if (plan.scratch_cols) {
    // one region per multi-pass class: the two classes' kernels run as
    // parallel graph branches and must not share boundary rows
    plan.scratch_bytes = align_up(multi_scratch_rows() * plan.scratch_cols * 24);
    o = align_up(o + 2 * plan.scratch_bytes);
  }
  plan.total_bytes = o;

  cudaError_t e = staging.ensure(std::max<size_t>(plan.upload_bytes, 1));
  if (e != cudaSuccess) return cuda_fail(e, "pinned staging allocation");
  uint8_t* s = static_cast<uint8_t*>(staging.ptr);

  timer.mark("layout+staging");
  // ---- haplotype codes ----
  std::atomic<int> bad_base{-1};
  uint8_t* codes = s + plan.off_hap_codes;
  HapDesc* hd = reinterpret_cast<HapDesc*>(s + plan.off_haps);
  parallel_for(b.num_haps, 64, [&](size_t lo, size_t hi) {
    for (size_t h = lo; h < hi; ++h) {
      const uint8_t* src = b.hap_bases + b.hap_offsets[h];
      uint8_t* dst = codes + hap_code_off[h];
      const uint32_t n = b.hap_lengths[h];
      for (uint32_t k = 0; k < n; ++k) {
        const uint8_t c = kCodes.v[src[k]];
        if (c == 0xff) bad_base.store((int)src[k]);
        dst[k] = c;
      }
      dst[n] = kSep;
      hd[h].code_off = hap_code_off[h];
      hd[h].len = n;
      hd[h].pad_ = 0;
    }
  });
  std::memset(codes, 0, kHapPad);
  std::memset(codes + tail_begin, 0, hb - tail_begin);
  timer.mark("haps");
  // ---- read rows ----
  uint32_t* rw = reinterpret_cast<uint32_t*>(s + plan.off_read_rows);
  ReadDesc* rdesc = reinterpret_cast<ReadDesc*>(s + plan.off_reads);
  parallel_for(b.num_reads, 256, [&](size_t lo, size_t hi) {
    for (size_t r = lo; r < hi; ++r) {
      const uint64_t off = b.read_offsets[r];
      const uint32_t n = b.read_lengths[r];
      uint32_t* dst = rw + row_off[r];
      const uint8_t* base = b.read_bases + off;
      const uint8_t* q = b.base_quals + off;
      if (read_class[r] & 1) {
        // uniform gaps: insertion, deletion and gcp qualities are the same
        // on every row, so their fields are one constant
        const uint32_t gaps = row_word(0, 0, b.ins_quals[off], b.del_quals[off], b.gcp_quals[off]);
        for (uint32_t k = 0; k < n; ++k) {
          const uint8_t c = kCodes.v[base[k]];
          if (c == 0xff) bad_base.store((int)base[k]);
          dst[k] = gaps | (c & 7u) | ((uint32_t)(q[k] & 127) << 3);
        }
      } else {
        for (uint32_t k = 0; k < n; ++k) {
          const uint8_t c = kCodes.v[base[k]];
          if (c == 0xff) bad_base.store((int)base[k]);
          dst[k] = row_word(c, q[k], b.ins_quals[off + k], b.del_quals[off + k],
                            b.gcp_quals[off + k]);
        }
      }
      for (uint32_t k = n; k < ((n + 3) & ~3u); ++k) dst[k] = 0;
      rdesc[r].row_off = row_off[r];
      rdesc[r].len = n;
      rdesc[r].flags = (read_class[r] & 1) ? kReadUniformGaps : 0u;
    }
  });
  if (bad_base.load() >= 0) {
    char msg[96];
    snprintf(msg, sizeof(msg), "base 0x%02x is not one of A, C, G, T, N", bad_base.load());
    return fail(RODV_ERR_INVALID_BASE, msg);
  }

  if (fp64) {
    uint32_t* preset = reinterpret_cast<uint32_t*>(s + plan.off_preset);
    for (int c = 0; c < kNumClasses; ++c) preset[c] = plan.pairs[c];
  }
  timer.mark("rows");
  // ---- work: chain items, same-haplotype items, leftovers, forced-FP64 lists ----
  std::vector<uint64_t> region_out(G);
  for (uint32_t g = 0, acc = 0; g < G; ++g) {
    region_out[g] = acc;
    acc += b.regions[g].num_haps * b.regions[g].num_reads;
  }
  std::vector<PairRef> leftovers[kNumClasses];
  for (int c = 0; c < kNumClasses; ++c) leftovers[c].resize(left_tot[c]);
  parallel_for(G, 16, [&](size_t lo, size_t hi) {
    std::vector<uint32_t> byclass[kNumClasses];
    std::vector<uint32_t> sr;
    RegionChains chs;
    for (size_t g = lo; g < hi; ++g) {
      const rodv_region& rg = b.regions[g];
      const uint32_t N = rg.num_reads;
      // out index of (haplotype h of the region, read rr)
      auto out_of = [&](uint32_t h, uint32_t rr) {
        return (uint32_t)(region_out[g] + (uint64_t)h * N + (rr - rg.read_start));
      };
      if (!fp64) {
        sorted_single(rg, sr);
        region_chains(sr, chs);
        uint64_t next[kNumClasses], snext[kNumClasses];
        for (int c = 0; c < kNumClasses; ++c) {
          next[c] = same_off[g * K + c];
          snext[c] = stack_off[g * K + c];
        }
        for (const ChainPairs& cb : chs.items) {
          const int c = cb.cls;
          ChainItem* ci = reinterpret_cast<ChainItem*>(s + plan.off_same[c]);
          uint32_t* stk = reinterpret_cast<uint32_t*>(s + plan.off_stack[c]);
          const uint32_t e0 = (uint32_t)snext[c];
          for (uint32_t j = 0; j < 2 * cb.pairs; ++j) stk[snext[c]++] = chs.reads[cb.first + j];
          const uint32_t cap = plan.chain_haps[c];
          for (uint32_t h0 = 0; h0 < rg.num_haps; h0 += cap)
            ci[next[c]++] = ChainItem{rg.hap_start + h0, std::min(cap, rg.num_haps - h0), e0,
                                      cb.pairs, out_of(h0, rg.read_start), N, hmax[g],
                                      rg.read_start};
        }
        if (single_read[g] != kNoPair) {
          const uint32_t rr = single_read[g];
          const int c = read_class[rr];
          PairRef* lf = leftovers[c].data() + left_off[g * K + c];
          for (uint32_t h = 0; h < rg.num_haps; ++h)
            lf[h] = PairRef{rg.hap_start + h, rr, out_of(h, rr)};
        }
      }
      for (auto& v : byclass) v.clear();
      for (uint32_t r = 0; r < N; ++r) byclass[read_class[rg.read_start + r]].push_back(rg.read_start + r);
      for (int c = 0; c < kNumClasses; ++c) {
        const std::vector<uint32_t>& rd = byclass[c];
        if (rd.empty() || (!fp64 && !class_multi(c))) continue;
        SameItem* si = reinterpret_cast<SameItem*>(s + plan.off_same[c]) + same_off[g * K + c];
        PairRef* lf = leftovers[c].data() + left_off[g * K + c];
        PairRef* li = reinterpret_cast<PairRef*>(s + plan.off_lists[c]) + list_off[g * K + c];
        for (uint32_t h = 0; h < rg.num_haps; ++h) {
          const uint32_t hap = rg.hap_start + h;
          if (fp64) {
            for (uint32_t rr : rd) *li++ = PairRef{hap, rr, out_of(h, rr)};
            continue;
          }
          size_t k = 0;
          for (; k + 1 < rd.size(); k += 2)
            *si++ = SameItem{hap, rd[k], rd[k + 1], out_of(h, rd[k])};
          if (k < rd.size()) *lf++ = PairRef{hap, rd[k], out_of(h, rd[k])};
        }
      }
    }
  });
  if (!fp64) {
    // leftovers: grouped by pass count (single-pass classes: one group),
    // sorted by haplotype length within a group (slot x takes the longer
    // haplotype), paired longest-first within the group
    for (int c = 0; c < kNumClasses; ++c) {
      std::vector<PairRef>& lv = leftovers[c];
      std::stable_sort(lv.begin(), lv.end(), [&](const PairRef& x, const PairRef& y) {
        const uint32_t px = passes_of(x.read), py = passes_of(y.read);
        if (px != py) return px > py;
        return b.hap_lengths[x.hap] > b.hap_lengths[y.hap];
      });
      DiffItem* di = reinterpret_cast<DiffItem*>(s + plan.off_diff[c]);
      size_t n = 0;
      for (size_t k = 0; k < lv.size();) {
        const bool two = k + 1 < lv.size() && passes_of(lv[k].read) == passes_of(lv[k + 1].read);
        di[n].x = lv[k];
        di[n].y = two ? lv[k + 1] : PairRef{0, kNoPair, 0};
        ++n;
        k += two ? 2 : 1;
      }
      if (n != plan.diff_items[c])
        return fail(RODV_ERR_INTERNAL, "leftover pairing count mismatch");
      // Multi-pass items go out in decreasing sweep length (passes x columns)
      // across pass-count groups, so the persistent grids -- and, through the
      // rescue positions, the FP64 sweep -- take the longest first.
      if (class_multi(c))
        std::stable_sort(di, di + n, [&](const DiffItem& x, const DiffItem& y) {
          return (uint64_t)passes_of(x.x.read) * (b.hap_lengths[x.x.hap] + kWarp) >
                 (uint64_t)passes_of(y.x.read) * (b.hap_lengths[y.x.hap] + kWarp);
        });
    }
    // the same for the multi-pass classes' same-haplotype items
    for (int c = kSinglePassClasses; c < kNumClasses; ++c) {
      SameItem* si = reinterpret_cast<SameItem*>(s + plan.off_same[c]);
      auto cost = [&](const SameItem& it) {
        return (uint64_t)std::max(passes_of(it.read_x), passes_of(it.read_y)) *
               (b.hap_lengths[it.hap] + kWarp);
      };
      std::stable_sort(si, si + plan.same_items[c],
                       [&](const SameItem& x, const SameItem& y) { return cost(x) > cost(y); });
    }
  }
  timer.mark("work");
  // cells
  uint64_t cells = 0;
  for (uint32_t g = 0; g < G; ++g) {
    const rodv_region& rg = b.regions[g];
    uint64_t rs = 0;
    for (uint32_t r = 0; r < rg.num_reads; ++r) rs += b.read_lengths[rg.read_start + r];
    cells += hsum[g] * rs;
  }
  plan.cells = cells;
  return RODV_OK;
}

// ---------------------------------------------------------------------------
// Launches
// ---------------------------------------------------------------------------
rodv_status Engine::launch_fp32_class(const PackedPlan& plan, uint8_t* dbase, int c, bool same,
                                      int variant, int blocks_cap, cudaStream_t stream) {
  ArenaView a = arena_view(plan, dbase, tab_);
  const uint32_t n = same ? plan.same_items[c] : plan.diff_items[c];
  if (!n) return RODV_OK;
  // the multi-pass two-haplotype kernel shares the class's variant (strip
  // height), which the packer paired its items by
  const KernelInfo k = forward_kernel_info(Precision::kF32x2, class_rows(c), class_uniform(c),
                                           class_multi(c), same,
                                           (same || class_multi(c)) ? variant : 0);
  ClassLaunch cl{};
  cl.work = dbase + (same ? plan.off_same[c] : plan.off_diff[c]);
  cl.work_count = nullptr;
  cl.static_count = n;
  cl.counter = a.counts + (same ? kCtrSame : kCtrDiff) + c;
  cl.rescue_list = reinterpret_cast<PairRef*>(dbase + plan.off_lists[c]);
  cl.rescue_count = a.counts + kCtrRescue + c;
  cl.scratch = class_scratch(plan, a, c);
  cl.scratch_cols = plan.scratch_cols;
  cl.error_flags = a.counts + kCtrError;
  cl.stack = reinterpret_cast<const uint32_t*>(dbase + plan.off_stack[c]);
  if (class_multi(c)) {  // rescues at their items' positions: same items, then two-haplotype
    cl.flags |= kLaunchRescueByItem;
    cl.rescue_base = same ? 0u : 2u * plan.same_items[c];
  }
  apply_wait_fault(cl, c);
  const int per_block = k.items_per_block;
  const int need = (int)((n + per_block - 1) / per_block);
  int blocks = std::max(1, std::min(persistent_blocks(k), need));
  if (blocks_cap > 0) blocks = std::min(blocks, blocks_cap);
  void* args[] = {&a.view, &cl};
  RODV_CUDA(cudaLaunchKernel(k.fn, dim3(blocks), dim3(k.threads), args, k.smem_bytes, stream));
  return RODV_OK;
}

// FP64 launch of class c over its list (rescued pairs, or every pair when
// FP64 is forced); the list's length is read by the kernel.
rodv_status Engine::launch_fp64_class(const PackedPlan& plan, uint8_t* dbase, int c,
                                      int variant, cudaStream_t stream) {
  ArenaView a = arena_view(plan, dbase, tab_);
  const KernelInfo k = forward_kernel_info(Precision::kF64, class_rows(c), class_uniform(c),
                                           class_multi(c), false, variant);
  ClassLaunch cl{};
  cl.work = dbase + plan.off_lists[c];
  cl.work_count = a.counts + kCtrRescue + c;
  cl.static_count = 0;
  if (class_multi(c) && !plan.fp64) {
    // rescues sit at their FP32 items' positions (longest items first); the
    // kernel passes over the empty positions
    cl.work_count = nullptr;
    cl.static_count = 2u * (plan.same_items[c] + plan.diff_items[c]);
  }
  cl.counter = a.counts + kCtrF64 + c;
  cl.scratch = class_scratch(plan, a, c);
  cl.scratch_cols = plan.scratch_cols;
  cl.error_flags = a.counts + kCtrError;
  apply_wait_fault(cl, c);
  const int need = (int)((plan.pairs[c] + k.items_per_block - 1) / k.items_per_block);
  const int blocks = std::max(1, std::min(persistent_blocks(k), need));
  void* args[] = {&a.view, &cl};
  RODV_CUDA(cudaLaunchKernel(k.fn, dim3(blocks), dim3(k.threads), args, k.smem_bytes, stream));
  return RODV_OK;
}

rodv_status Engine::launch_all(const PackedPlan& plan, uint8_t* dbase, rodv_stats* st,
                               cudaStream_t stream, cudaEvent_t* ev, int parts, bool fan_out) {
  ArenaView a = arena_view(plan, dbase, tab_);
  uint32_t launches = 0;
  // fan-out: the first launch of class c waits on the fork point on side_[c];
  // join() brings every used side stream back into `stream`
  bool forked[kNumClasses] = {};
  auto lane = [&](int c) -> cudaStream_t {
    if (!fan_out) return stream;
    if (!forked[c]) {
      if (cudaStreamWaitEvent(side_[c], fork_ev_, 0) != cudaSuccess) return nullptr;
      forked[c] = true;
    }
    return side_[c];
  };
  auto fork = [&]() -> cudaError_t {
    for (bool& f : forked) f = false;
    return fan_out ? cudaEventRecord(fork_ev_, stream) : cudaSuccess;
  };
  auto join = [&]() -> cudaError_t {
    for (int c = 0; c < kNumClasses && fan_out; ++c) {
      if (!forked[c]) continue;
      cudaError_t e = cudaEventRecord(join_ev_[c], side_[c]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, join_ev_[c], 0);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  if (parts & 1) {
    RODV_CUDA(cudaMemsetAsync(a.counts, 0, kCountWords * 4, stream));
    if (plan.fp64)  // every pair goes to the FP64 kernels: the uploaded lists are full
      RODV_CUDA(cudaMemcpyAsync(a.counts + kCtrRescue, dbase + plan.off_preset,
                                kNumClasses * 4, cudaMemcpyDeviceToDevice, stream));
    // multi-pass classes' lists: every position empty (kNoPair) until a
    // rescue fills it (kLaunchRescueByItem)
    for (int c = kSinglePassClasses; c < kNumClasses && !plan.fp64; ++c)
      if (plan.same_items[c] + plan.diff_items[c])
        RODV_CUDA(cudaMemsetAsync(dbase + plan.off_lists[c], 0xff,
                                  (size_t)plan.list_cap[c] * sizeof(PairRef), stream));
  }
  if (ev) RODV_CUDA(cudaEventRecord(ev[0], stream));
  if (!plan.fp64 && (parts & 1)) {
    RODV_CUDA(fork());
    for (int c = 0; c < kNumClasses; ++c) {
      for (int same = 1; same >= 0; --same) {
        if (!(same ? plan.same_items[c] : plan.diff_items[c])) continue;
        const cudaStream_t ls = lane(c);
        if (!ls) return cuda_fail(cudaErrorUnknown, "class stream fork");
        rodv_status s = launch_fp32_class(plan, dbase, c, same != 0, plan.variant[c], 0, ls);
        if (s != RODV_OK) return s;
        ++launches;
      }
    }
    RODV_CUDA(join());
  }
  if (ev) RODV_CUDA(cudaEventRecord(ev[1], stream));
  if (parts & 2) RODV_CUDA(fork());
  for (int c = 0; c < kNumClasses && (parts & 2); ++c) {
    if (!plan.pairs[c]) continue;
    const cudaStream_t ls = lane(c);
    if (!ls) return cuda_fail(cudaErrorUnknown, "class stream fork");
    const rodv_status s = launch_fp64_class(plan, dbase, c, plan.variant64[c], ls);
    if (s != RODV_OK) return s;
    ++launches;
  }
  if (parts & 2) RODV_CUDA(join());
  if (ev) RODV_CUDA(cudaEventRecord(ev[2], stream));
  if (st) st->kernel_launches += launches;
  return RODV_OK;
}

rodv_status Engine::check_errors(const PackedPlan& plan, uint8_t* dbase) {
  uint32_t err = 0;
  RODV_CUDA(cudaMemcpy(&err, dbase + plan.off_counts + kCtrError * 4, 4, cudaMemcpyDeviceToHost));
  if (err != 0)
    return fail(RODV_ERR_DEVICE_CHECK, "kernel reported error flags " + std::to_string(err));
  return RODV_OK;
}

static void fill_stats(rodv_stats* st, const PackedPlan& plan, const uint32_t* counts) {
  if (!st) return;
  st->pairs = plan.num_pairs;
  st->cells = plan.cells;
  uint64_t n = 0;
  for (int c = 0; c < kNumClasses; ++c) n += plan.fp64 ? plan.pairs[c] : counts[kCtrRescue + c];
  st->fp64_pairs = n;
}

// Host buffers in and out.  A large batch is cut into region ranges that go
// through three lanes: while ranges compute, the host packs the next into a
// free lane's staging buffer and its upload runs on the copy engine, so
// packing and transfers hide behind the kernels (with two lanes the host
// could only start a range once the range two back had finished, which left
// the GPU idle between ranges).  Range sizes start small
// (the first range's packing and upload are not hidden) and double up to
// kChunkCells cells.  Results do not depend on the cut (a pair's arithmetic
// depends on its own region only).  Measured on the 10,000-region uneven
// batch (5.1e11 cells): 3e10-cell ranges 171 ms, 6e10 158 ms, 1.2e11 150 ms
// per call, against 139 ms of resident compute (with later kernels: 146-148
// ms against 133).  Running every range's kernels on one stream was slower
// (159 ms): concurrent ranges fill each other's per-class tails.
constexpr double kChunkCells = 1.2e11;
constexpr double kFirstChunkCells = 4e9;
// first range: 1/32 of the batch's cells, at least 4e9 (1/64 measured the
// same on the uneven batch: 121.2-121.7 ms per call either way)
constexpr double kFirstChunkDiv = 32;
constexpr double kMinChunkedCells = 2e10;

// Range sizes, overridable for tuning (RODV_CHUNK_CELLS, RODV_FIRST_CHUNK_CELLS,
// RODV_FIRST_CHUNK_DIV).
double env_cells(const char* name, double fallback) {
  const char* v = std::getenv(name);
  if (!v || !*v) return fallback;
  const double x = std::atof(v);
  return x > 0 ? x : fallback;
}

rodv_status Engine::run_host(const rodv_batch& b, double* out, rodv_stats* st, bool force_fp64,
                             uint8_t* prec) {
  if (!out) return fail(RODV_ERR_INVALID_ARG, "null output");
  RODV_CUDA(cudaSetDevice(device_));
  const bool fp64 = force_fp64 || opt_.force_fp64 != 0;
  {
    std::string msg;
    const rodv_status vs = validate_batch(b, false, nullptr, &msg);
    if (vs != RODV_OK) return fail(vs, msg);
  }
  const uint32_t G = b.num_regions;
  std::vector<double> cum(G + 1, 0.0);
  for (uint32_t g = 0; g < G; ++g) {
    const rodv_region& rg = b.regions[g];
    double hs = 0, rs = 0;
    for (uint32_t h = 0; h < rg.num_haps; ++h) hs += b.hap_lengths[rg.hap_start + h];
    for (uint32_t r = 0; r < rg.num_reads; ++r) rs += b.read_lengths[rg.read_start + r];
    cum[g + 1] = cum[g] + hs * rs;
  }
  static const double chunk_cells = env_cells("RODV_CHUNK_CELLS", kChunkCells);
  static const double first_cells = env_cells("RODV_FIRST_CHUNK_CELLS", kFirstChunkCells);
  static const double first_div = env_cells("RODV_FIRST_CHUNK_DIV", kFirstChunkDiv);
  if (cum[G] < kMinChunkedCells || G < 4) return run_host_single(b, out, st, fp64, prec);
  std::vector<uint32_t> bounds{0};
  double target = std::min(chunk_cells, std::max(first_cells, cum[G] / first_div));
  for (uint32_t g = 1; g < G; ++g) {
    if (cum[g] - cum[bounds.back()] >= target) {
      bounds.push_back(g);
      target = std::min(chunk_cells, 2 * target);
    }
  }
  bounds.push_back(G);
  if (bounds.size() < 3) return run_host_single(b, out, st, fp64, prec);
  return run_host_chunked(b, out, st, fp64, bounds, prec);
}

rodv_status Engine::finish_lane(HostLane& l, double* out, rodv_stats* st, uint8_t* prec) {
  TraceRange trace("rodv: finish range");
  l.busy = false;
  RODV_CUDA(cudaEventSynchronize(l.done));
  if (opt_.verbose >= 2) {
    float a = 0.f, k0 = 0.f, k1 = 0.f;
    cudaEventElapsedTime(&a, ev_[3], l.ev[3]);
    cudaEventElapsedTime(&k0, ev_[3], l.ev[0]);
    cudaEventElapsedTime(&k1, ev_[3], l.ev[2]);
    fprintf(stderr, "rodv:   device: upload from %.2f, kernels %.2f-%.2f ms\n", a, k0, k1);
  }
  const PackedPlan& p = l.plan;
  const uint8_t* h = static_cast<const uint8_t*>(l.out.ptr);
  const uint32_t* counts = reinterpret_cast<const uint32_t*>(h + p.num_pairs * 8);
  if (counts[kCtrError] != 0)
    return fail(RODV_ERR_DEVICE_CHECK,
                "kernel reported error flags " + std::to_string(counts[kCtrError]));
  // results into the caller's (pageable) buffer, 128K pairs per task: the
  // last range's copy is on the call's critical path
  const uint8_t* hp = h + p.num_pairs * 8 + kCountWords * 4;  // raw mode: precisions
  parallel_for(p.num_pairs, 1u << 17, [&](size_t lo, size_t hi) {
    std::memcpy(out + l.out_off + lo, h + lo * 8, (hi - lo) * 8);
    if (prec) std::memcpy(prec + l.out_off + lo, hp + lo, hi - lo);
  });
  if (st) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, l.ev[0], l.ev[2]);
    st->device_ms += ms;
    cudaEventElapsedTime(&ms, l.ev[0], l.ev[1]);
    st->fp32_ms += ms;
    cudaEventElapsedTime(&ms, l.ev[3], l.ev[0]);
    st->h2d_ms += ms;
    st->h2d_bytes += p.upload_bytes;
    st->d2h_bytes += p.num_pairs * 8 + kCountWords * 4;
    st->pairs += p.num_pairs;
    st->cells += p.cells;
    for (int c = 0; c < kNumClasses; ++c)
      st->fp64_pairs += p.fp64 ? p.pairs[c] : counts[kCtrRescue + c];
  }
  return RODV_OK;
}

rodv_status Engine::run_host_chunked(const rodv_batch& b, double* out, rodv_stats* st,
                                     bool fp64, const std::vector<uint32_t>& bounds,
                                     uint8_t* prec) {
  const auto t0 = std::chrono::steady_clock::now();
  const bool timeline = opt_.verbose >= 2;
  if (timeline) RODV_CUDA(cudaEventRecord(ev_[3], lanes_[0].stream));
  rodv_stats acc{};
  const size_t nchunks = bounds.size() - 1;
  rodv_status result = RODV_OK;
  uint64_t out_off = 0;
  for (size_t k = 0; k < nchunks && result == RODV_OK; ++k) {
    HostLane& l = lanes_[k % kHostLanes];
    if (l.busy) {
      result = finish_lane(l, out, &acc, prec);
      if (result != RODV_OK) break;
    }
    // the range's regions over the batch's arrays, rebased to the range's
    // first haplotype and read
    const uint32_t g0 = bounds[k], g1 = bounds[k + 1];
    uint32_t h0 = UINT32_MAX, h1 = 0, r0 = UINT32_MAX, r1 = 0;
    uint64_t pairs = 0;
    for (uint32_t g = g0; g < g1; ++g) {
      const rodv_region& rg = b.regions[g];
      h0 = std::min(h0, rg.hap_start);
      h1 = std::max(h1, rg.hap_start + rg.num_haps);
      r0 = std::min(r0, rg.read_start);
      r1 = std::max(r1, rg.read_start + rg.num_reads);
      pairs += (uint64_t)rg.num_haps * rg.num_reads;
    }
    l.regs.assign(b.regions + g0, b.regions + g1);
    for (rodv_region& rg : l.regs) {
      rg.hap_start -= h0;
      rg.read_start -= r0;
    }
    const rodv_batch v{g1 - g0, l.regs.data(), h1 - h0, b.hap_bases, b.hap_offsets + h0,
                       b.hap_lengths + h0, r1 - r0, b.read_bases, b.base_quals, b.ins_quals,
                       b.del_quals, b.gcp_quals, b.read_offsets + r0, b.read_lengths + r0};
    {
      // Upper bound of the upload (codes, row words, descriptors, items, lists),
      // reserved with headroom: regrowing pinned memory synchronises the device.
      uint64_t est = 1u << 20;
      for (uint32_t x = h0; x < h1; ++x) est += b.hap_lengths[x] + 1 + 16;
      for (uint32_t x = r0; x < r1; ++x) est += ((b.read_lengths[x] + 3) & ~3u) * 4 + 16;
      est += pairs * (fp64 ? 12 : 16);
      if (l.staging.bytes < est) {
        const cudaError_t e = l.staging.ensure(est + est / 4);
        if (e != cudaSuccess) {
          result = cuda_fail(e, "chunk staging");
          break;
        }
      }
    }
    const double t_pack0 = ms_since(t0);
    result = pack(v, l.plan, l.staging, fp64, prec != nullptr);
    if (result != RODV_OK) break;
    if (timeline)
      fprintf(stderr, "rodv: range %zu (%u regions, %.2e cells): pack %.2f-%.2f ms\n", k, g1 - g0,
              (double)l.plan.cells, t_pack0, ms_since(t0));
    const PackedPlan& p = l.plan;
    cudaError_t e = cudaSuccess;
    if (l.arena.bytes < p.total_bytes) e = l.arena.ensure(p.total_bytes + p.total_bytes / 4);
    const size_t ob = p.num_pairs * 8 + kCountWords * 4 + (p.raw ? p.num_pairs : 0);
    if (e == cudaSuccess && l.out.bytes < ob) e = l.out.ensure(ob + ob / 4);
    uint8_t* d = static_cast<uint8_t*>(l.arena.ptr);
    uint8_t* h = static_cast<uint8_t*>(l.out.ptr);
    if (e == cudaSuccess) e = cudaEventRecord(l.ev[3], l.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d, l.staging.ptr, p.upload_bytes, cudaMemcpyHostToDevice, l.stream);
    if (e != cudaSuccess) {
      result = cuda_fail(e, "chunk upload");
      break;
    }
    // the range's classes as parallel branches (their tails overlap; 130 ms
    // per call of the uneven batch against 132-134 without)
    result = launch_all(p, d, &acc, l.stream, l.ev, 3, /*fan_out=*/true);
    if (result != RODV_OK) break;
    e = cudaMemcpyAsync(h, d + p.off_out, p.num_pairs * 8, cudaMemcpyDeviceToHost, l.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h + p.num_pairs * 8, d + p.off_counts, kCountWords * 4,
                          cudaMemcpyDeviceToHost, l.stream);
    if (e == cudaSuccess && p.raw)
      e = cudaMemcpyAsync(h + p.num_pairs * 8 + kCountWords * 4, d + p.off_prec, p.num_pairs,
                          cudaMemcpyDeviceToHost, l.stream);
    if (e == cudaSuccess) e = cudaEventRecord(l.done, l.stream);
    if (e != cudaSuccess) {
      result = cuda_fail(e, "chunk download");
      break;
    }
    l.out_off = out_off;
    l.busy = true;
    out_off += pairs;
  }
  // collect what is still in flight, oldest first (on error too: no lane may
  // be left with work that writes into buffers reused by the next call)
  for (size_t k = nchunks; k < nchunks + kHostLanes; ++k) {
    HostLane& l = lanes_[k % kHostLanes];
    if (!l.busy) continue;
    if (result == RODV_OK) {
      result = finish_lane(l, out, &acc, prec);
    } else {
      cudaStreamSynchronize(l.stream);
      l.busy = false;
    }
  }
  if (result != RODV_OK) return result;
  if (st) {
    const uint32_t launches = st->kernel_launches + acc.kernel_launches;
    *st = acc;
    st->kernel_launches = launches;
    st->total_ms = ms_since(t0);
  }
  return RODV_OK;
}

rodv_status Engine::run_host_single(const rodv_batch& b, double* out, rodv_stats* st,
                                    bool fp64, uint8_t* prec) {
  const auto t0 = std::chrono::steady_clock::now();
  PackedPlan plan;
  rodv_status s = pack(b, plan, staging_, fp64, prec != nullptr);
  if (s != RODV_OK) return s;
  RODV_CUDA(arena_.ensure(plan.total_bytes));
  RODV_CUDA(out_staging_.ensure(plan.num_pairs * 8 + kCountWords * 4 +
                                (prec ? plan.num_pairs : 0)));
  uint8_t* d = static_cast<uint8_t*>(arena_.ptr);
  RODV_CUDA(cudaEventRecord(ev_[3], stream_));
  RODV_CUDA(cudaMemcpyAsync(d, staging_.ptr, plan.upload_bytes, cudaMemcpyHostToDevice, stream_));
  s = launch_all(plan, d, st, stream_, ev_, 3);
  if (s != RODV_OK) return s;
  uint8_t* hs = static_cast<uint8_t*>(out_staging_.ptr);
  RODV_CUDA(cudaMemcpyAsync(hs, d + plan.off_out, plan.num_pairs * 8, cudaMemcpyDeviceToHost,
                            stream_));
  RODV_CUDA(cudaMemcpyAsync(hs + plan.num_pairs * 8, d + plan.off_counts, kCountWords * 4,
                            cudaMemcpyDeviceToHost, stream_));
  if (prec)
    RODV_CUDA(cudaMemcpyAsync(hs + plan.num_pairs * 8 + kCountWords * 4, d + plan.off_prec,
                              plan.num_pairs, cudaMemcpyDeviceToHost, stream_));
  RODV_CUDA(cudaStreamSynchronize(stream_));
  const uint32_t* counts = reinterpret_cast<const uint32_t*>(hs + plan.num_pairs * 8);
  if (counts[kCtrError] != 0)
    return fail(RODV_ERR_DEVICE_CHECK,
                "kernel reported error flags " + std::to_string(counts[kCtrError]));
  const uint8_t* hp = hs + plan.num_pairs * 8 + kCountWords * 4;
  parallel_for(plan.num_pairs, 1u << 17, [&](size_t lo, size_t hi) {
    std::memcpy(out + lo, hs + lo * 8, (hi - lo) * 8);
    if (prec) std::memcpy(prec + lo, hp + lo, hi - lo);
  });
  if (st) {
    fill_stats(st, plan, counts);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev_[0], ev_[2]);
    st->device_ms = ms;
    cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
    st->fp32_ms = ms;
    cudaEventElapsedTime(&ms, ev_[3], ev_[0]);
    st->h2d_ms = ms;
    st->h2d_bytes = plan.upload_bytes;
    st->d2h_bytes = plan.num_pairs * 8 + kCountWords * 4;
    st->total_ms = ms_since(t0);
  }
  return RODV_OK;
}

rodv_status Engine::upload(const rodv_batch& b, rodv_device_batch** out) {
  RODV_CUDA(cudaSetDevice(device_));
  auto* db = new rodv_device_batch();
  PinnedMem staging;
  rodv_status s = pack(b, db->plan, staging, opt_.force_fp64 != 0);
  if (s != RODV_OK) {
    delete db;
    return s;
  }
  cudaError_t e = db->arena.ensure(db->plan.total_bytes);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(db->arena.ptr, staging.ptr, db->plan.upload_bytes,
                        cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    delete db;
    return cuda_fail(e, "device batch upload");
  }
  *out = db;
  return RODV_OK;
}

rodv_status Engine::run_device(rodv_device_batch* db, rodv_stats* st) {
  RODV_CUDA(cudaSetDevice(device_));
  uint8_t* d = static_cast<uint8_t*>(db->arena.ptr);
  const auto t0 = std::chrono::steady_clock::now();
  if (!db->graph[0]) {
    // Capture once, as two graphs (FP32 part: counter reset and the FP32 class
    // launches; FP64 part: the rescue launches) so that an event between them
    // times the FP32 pass; later runs are two graph launches.  Within each
    // graph the classes are parallel branches (independent items, counters
    // and rescue lists), so one class's kernel starts in another's tail.
    for (int part = 0; part < 2; ++part) {
      rodv_stats cap{};
      RODV_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      rodv_status s =
          launch_all(db->plan, d, &cap, stream_, nullptr, part == 0 ? 1 : 2, /*fan_out=*/true);
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(stream_, &g);
      if (s != RODV_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
      }
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      const cudaError_t ie = cudaGraphInstantiate(&db->graph[part], g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate");
      db->graph_launches += cap.kernel_launches;
    }
  }
  RODV_CUDA(cudaEventRecord(ev_[0], stream_));
  RODV_CUDA(cudaGraphLaunch(db->graph[0], stream_));
  RODV_CUDA(cudaEventRecord(ev_[1], stream_));
  RODV_CUDA(cudaGraphLaunch(db->graph[1], stream_));
  RODV_CUDA(cudaEventRecord(ev_[2], stream_));
  RODV_CUDA(cudaStreamSynchronize(stream_));
  uint32_t counts[kCountWords];
  RODV_CUDA(cudaMemcpy(counts, d + db->plan.off_counts, sizeof(counts), cudaMemcpyDeviceToHost));
  if (st) {
    fill_stats(st, db->plan, counts);
    st->kernel_launches += db->graph_launches;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev_[0], ev_[2]);
    st->device_ms = ms;
    cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
    st->fp32_ms = ms;
    st->total_ms = ms_since(t0);
  }
  if (counts[kCtrError] != 0)
    return fail(RODV_ERR_DEVICE_CHECK,
                "kernel reported error flags " + std::to_string(counts[kCtrError]));
  return RODV_OK;
}

rodv_status Engine::download(rodv_device_batch* db, double* out) {
  RODV_CUDA(cudaSetDevice(device_));
  RODV_CUDA(cudaMemcpy(out, static_cast<uint8_t*>(db->arena.ptr) + db->plan.off_out,
                       db->plan.num_pairs * 8, cudaMemcpyDeviceToHost));
  return RODV_OK;
}

// The plain GPU form: every pair is its own FP32 launch (one warp, second slot
// empty), its result is read back, and a pair below 1e-28 gets a second,
// FP64 launch.  Same kernels as the batched path; no batching.
rodv_status Engine::plain(rodv_device_batch* db, double* out, rodv_stats* st) {
  RODV_CUDA(cudaSetDevice(device_));
  const PackedPlan& plan = db->plan;
  uint8_t* d = static_cast<uint8_t*>(db->arena.ptr);
  ArenaView a = arena_view(plan, d, tab_);
  // control block: [0,32) ChainItem (one haplotype, one read pair) or
  // SameItem (multi-pass), [32,44) rescue PairRef, words 12..15: fp32
  // counter, fp64 counter, rescue count, error flags, words 16..17: the
  // chain item's pair (the read, kNoPair)
  DeviceMem ctl;
  RODV_CUDA(ctl.ensure(72));
  uint8_t* w = static_cast<uint8_t*>(ctl.ptr);
  uint32_t* wc = reinterpret_cast<uint32_t*>(w + 48);
  PinnedMem host;
  RODV_CUDA(host.ensure(72));
  uint8_t* hw = static_cast<uint8_t*>(host.ptr);
  uint32_t* hc = reinterpret_cast<uint32_t*>(hw + 48);
  uint32_t launches = 0;
  uint64_t rescued = 0;
  const auto t0 = std::chrono::steady_clock::now();
  RODV_CUDA(cudaEventRecord(ev_[0], stream_));
  uint64_t p = 0;
  for (const rodv_region& rg : plan.regions) {
    for (uint32_t h = 0; h < rg.num_haps; ++h) {
      for (uint32_t r = 0; r < rg.num_reads; ++r, ++p) {
        const uint32_t read = rg.read_start + r;
        const int c = plan.read_class[read];
        if (class_multi(c)) {
          const SameItem item{rg.hap_start + h, read, kNoPair, (uint32_t)p};
          std::memcpy(hw, &item, sizeof(item));
        } else {
          const ChainItem item{rg.hap_start + h, 1, 0, 1, (uint32_t)p, 0,
                               plan.hap_len[rg.hap_start + h], read};
          std::memcpy(hw, &item, sizeof(item));
        }
        const PairRef ref{rg.hap_start + h, read, (uint32_t)p};
        std::memcpy(hw + 32, &ref, sizeof(ref));
        const uint32_t pair[2] = {read, kNoPair};
        std::memcpy(hw + 64, pair, sizeof(pair));
        hc[0] = hc[1] = hc[2] = hc[3] = 0;
        RODV_CUDA(cudaMemcpyAsync(w, hw, 72, cudaMemcpyHostToDevice, stream_));
        for (int pass = 0; pass < 2; ++pass) {
          const bool f64 = pass == 1 || plan.fp64;
          const KernelInfo k =
              forward_kernel_info(f64 ? Precision::kF64 : Precision::kF32x2, class_rows(c),
                                  class_uniform(c), class_multi(c), true,
                                  f64 ? variant64_[c] : variant_[c]);
          ClassLaunch cl{};
          cl.work = f64 ? static_cast<const void*>(w + 32) : static_cast<const void*>(w);
          cl.work_count = nullptr;
          cl.static_count = 1;
          cl.counter = f64 ? wc + 1 : wc;
          cl.rescue_list = reinterpret_cast<PairRef*>(w + 32);
          cl.rescue_count = wc + 2;
          cl.scratch = class_scratch(plan, a, c);
          cl.scratch_cols = plan.scratch_cols;
          cl.error_flags = wc + 3;
          cl.stack = reinterpret_cast<const uint32_t*>(w + 64);
          void* args[] = {&a.view, &cl};
          RODV_CUDA(
              cudaLaunchKernel(k.fn, dim3(1), dim3(k.threads), args, k.smem_bytes, stream_));
          ++launches;
          if (f64) break;
          RODV_CUDA(cudaMemcpyAsync(hc + 2, wc + 2, 8, cudaMemcpyDeviceToHost, stream_));
          RODV_CUDA(cudaStreamSynchronize(stream_));
          if (hc[3]) return fail(RODV_ERR_DEVICE_CHECK, "plain kernel reported an error");
          if (hc[2] == 0) break;
          ++rescued;
        }
      }
    }
  }
  RODV_CUDA(cudaEventRecord(ev_[1], stream_));
  RODV_CUDA(cudaStreamSynchronize(stream_));
  if (st) {
    st->pairs = plan.num_pairs;
    st->cells = plan.cells;
    st->fp64_pairs = plan.fp64 ? plan.num_pairs : rescued;
    st->kernel_launches += launches;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
    st->device_ms = ms;
    st->total_ms = ms_since(t0);
  }
  if (out) return download(db, out);
  return RODV_OK;
}

// ---------------------------------------------------------------------------
// Autotuning.  Per work class, every variant of the class's FP32 kernel is
// timed on a synthetic batch of that class and the fastest kept:
//   single-pass classes: the occupancy target (blocks per SM, which caps the
//     registers) and, for reads up to 128 bases, one or two chain items per
//     warp (16-lane groups with twice the rows per lane);
//   multi-pass classes: the strip height (4 or 8 rows per lane per pass) and
//     the warps that sweep one item's passes concurrently (2 or 4), for the
//     FP32 kernel and, on a batch forced to FP64, for the FP64 kernel.
// Synthetic batches: reads of 32R-5 bases against four 400-base haplotypes
// per region (single-pass), or 1,500-base reads against 3,000-base
// haplotypes (multi-pass).  Results are cached per device.
// ---------------------------------------------------------------------------
std::string Engine::device_key() const {
  std::string k = device_name_;
  for (char& ch : k)
    if (ch == ' ') ch = '_';
  return k + "_sm" + std::to_string(num_sms_);
}

bool Engine::load_tuning(const std::string& path) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line, key = device_key();
  int found = 0;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string k;
    int c, v, v64;
    if (!(ss >> k >> c >> v >> v64) || k != key) continue;
    if (c < 0 || c >= kNumClasses) continue;
    if (v < 0 ||
        v >= forward_kernel_variants(Precision::kF32x2, true, class_rows(c), class_multi(c)))
      continue;
    if (v64 < 0 ||
        v64 >= forward_kernel_variants(Precision::kF64, false, class_rows(c), class_multi(c)))
      continue;
    variant_[c] = v;
    variant64_[c] = v64;
    ++found;
  }
  tuned_ = found == kNumClasses;
  return tuned_;
}

bool Engine::save_tuning(const std::string& path) const {
  std::ofstream out(path, std::ios::trunc);
  if (!out) return false;
  for (int c = 0; c < kNumClasses; ++c)
    out << device_key() << ' ' << c << ' ' << variant_[c] << ' ' << variant64_[c] << '\n';
  return (bool)out;
}

namespace {
// What a kernel variant is, for the tuner's log.
std::string variant_name(int cls, int v, bool fp64) {
  char buf[96];
  if (class_multi(cls))
    snprintf(buf, sizeof(buf), "strip height %d, %d warps per item", pipe_variant_rows(v),
             pipe_variant_warps(v));
  else if (fp64)
    snprintf(buf, sizeof(buf), "one variant");
  else
    snprintf(buf, sizeof(buf), "%d blocks/SM%s", kVariantMinBlocks[v],
             v >= kOccupancyTargets ? ", two 16-lane chains per warp" : "");
  return buf;
}

// A synthetic batch of one work class (the tuner's input).
struct TuneBatch {
  std::vector<uint8_t> hb, rb, q, ins, del, gcp;
  std::vector<uint64_t> ho, ro;
  std::vector<uint32_t> hl, rl;
  std::vector<rodv_region> rg;
  rodv_batch view() const {
    return rodv_batch{(uint32_t)rg.size(), rg.data(), (uint32_t)hl.size(), hb.data(),
                      ho.data(), hl.data(), (uint32_t)rl.size(), rb.data(), q.data(),
                      ins.data(), del.data(), gcp.data(), ro.data(), rl.data()};
  }
};

// one_in: one base in `one_in` of a read differs from its haplotype.
void make_tune_batch(TuneBatch& tb, std::mt19937& rng, int regions, int haps, int reads,
                     uint32_t H, uint32_t L, bool uni, uint32_t one_in = 100) {
  const char* acgt = "ACGT";
  for (int g = 0; g < regions; ++g) {
    rodv_region r{(uint32_t)tb.ho.size(), (uint32_t)haps, (uint32_t)tb.ro.size(),
                  (uint32_t)reads};
    std::string base;
    for (uint32_t j = 0; j < H; ++j) base += acgt[rng() % 4];
    for (int h = 0; h < haps; ++h) {
      tb.ho.push_back(tb.hb.size());
      tb.hl.push_back(H);
      for (uint32_t j = 0; j < H; ++j) tb.hb.push_back(rng() % 100 ? base[j] : acgt[rng() % 4]);
    }
    for (int k = 0; k < reads; ++k) {
      tb.ro.push_back(tb.rb.size());
      tb.rl.push_back(L);
      const uint32_t st = rng() % (H - std::min(L, H) + 1);
      for (uint32_t j = 0; j < L; ++j) {
        tb.rb.push_back(j + st < H && rng() % one_in ? base[j + st] : acgt[rng() % 4]);
        tb.q.push_back(10 + rng() % 31);
        tb.ins.push_back(uni ? 45 : 20 + rng() % 26);
        tb.del.push_back(uni ? 45 : 20 + rng() % 26);
        tb.gcp.push_back(uni ? 10 : 5 + rng() % 11);
      }
    }
    tb.rg.push_back(r);
  }
}
}  // namespace

rodv_status Engine::autotune(const char* cache_path, int force, int32_t* variants_out) {
  const std::string path = cache_path ? cache_path : "";
  if (!force && !path.empty() && load_tuning(path)) {
    if (variants_out)
      for (int c = 0; c < kNumClasses; ++c) variants_out[c] = variant_[c];
    return RODV_OK;
  }
  RODV_CUDA(cudaSetDevice(device_));
  std::mt19937 rng(12345);
  // Times `launch` (three runs, the first discarded) after a counter reset.
  auto time_launch = [&](const PackedPlan& plan, uint8_t* d, const auto& launch,
                         float* best) -> rodv_status {
    *best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      RODV_CUDA(cudaMemsetAsync(d + plan.off_counts, 0, kCountWords * 4, stream_));
      if (plan.fp64)
        RODV_CUDA(cudaMemcpyAsync(d + plan.off_counts + kCtrRescue * 4, d + plan.off_preset,
                                  kNumClasses * 4, cudaMemcpyDeviceToDevice, stream_));
      RODV_CUDA(cudaEventRecord(ev_[0], stream_));
      const rodv_status s = launch();
      if (s != RODV_OK) return s;
      RODV_CUDA(cudaEventRecord(ev_[1], stream_));
      RODV_CUDA(cudaEventSynchronize(ev_[1]));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
      if (rep > 0) *best = std::min(*best, ms);
    }
    return check_errors(plan, d);
  };
  for (int c = 0; c < kNumClasses; ++c) {
    const int R = class_rows(c);
    const bool multi = class_multi(c), uni = class_uniform(c);
    TuneBatch tb;
    if (multi) {
      // long pairs, several waves of the largest grid of one item per block:
      // half the regions with reads of 1% differences (the FP32 sweep runs
      // every pass), half with 8% (it stops after the first passes and the
      // pairs go to FP64), so the choice weighs both kinds of long read
      make_tune_batch(tb, rng, num_sms_ * 2, 1, 2, 3000, 1500, uni, 100);
      make_tune_batch(tb, rng, num_sms_ * 2, 1, 2, 3000, 1500, uni, 12);
    } else {
      // Enough items that every warp of the largest grid takes several (chain
      // items of 4 haplotypes: ~8), so the timing reflects per-item throughput
      // and not the tail of the work queue.
      const uint64_t max_warps = (uint64_t)num_sms_ * kVariantMinBlocks[kTuneVariants - 1] * 4;
      const int regions = 16;
      const int reads = (int)std::max<uint64_t>(2, 2 * max_warps * 8 / regions + 1);
      make_tune_batch(tb, rng, regions, 4, reads, 400, (uint32_t)std::max(1, 32 * R - 5), uni);
    }
    const rodv_batch b = tb.view();
    for (int prec = 0; prec < (multi ? 2 : 1); ++prec) {
      const bool f64 = prec == 1;
      auto* db = new rodv_device_batch();
      PinnedMem staging;
      // one read per bin: each class's batch stays in its class
      rodv_status s = pack(b, db->plan, staging, f64, false, false);
      cudaError_t e = s == RODV_OK ? db->arena.ensure(db->plan.total_bytes) : cudaSuccess;
      if (s == RODV_OK && e == cudaSuccess)
        e = cudaMemcpyAsync(db->arena.ptr, staging.ptr, db->plan.upload_bytes,
                            cudaMemcpyHostToDevice, stream_);
      if (s != RODV_OK || e != cudaSuccess) {
        delete db;
        return s != RODV_OK ? s : cuda_fail(e, "tuning batch upload");
      }
      uint8_t* d = static_cast<uint8_t*>(db->arena.ptr);
      const Precision pr = f64 ? Precision::kF64 : Precision::kF32x2;
      const int nvar = forward_kernel_variants(pr, !f64, R, multi);
      int* slot = f64 ? &variant64_[c] : &variant_[c];
      float best_ms = 1e30f;
      int best_v = *slot;
      for (int v = 0; v < nvar; ++v) {
        float ms = 0.f;
        s = time_launch(
            db->plan, d,
            [&]() {
              return f64 ? launch_fp64_class(db->plan, d, c, v, stream_)
                         : launch_fp32_class(db->plan, d, c, true, v, 0, stream_);
            },
            &ms);
        if (s != RODV_OK) {
          delete db;
          return s;
        }
        if (opt_.verbose)
          fprintf(stderr, "rodv: tune %s class %d (R=%d%s%s) variant %d (%s): %.3f ms\n",
                  f64 ? "FP64" : "FP32", c, R, uni ? ", uniform" : "",
                  multi ? ", multi-pass" : "", v, variant_name(c, v, f64).c_str(), ms);
        if (ms < best_ms) {
          best_ms = ms;
          best_v = v;
        }
      }
      delete db;
      *slot = best_v;
      if (opt_.verbose)
        fprintf(stderr, "rodv: tuned %s class %d (R=%d%s%s): variant %d (%s), %.3f ms\n",
                f64 ? "FP64" : "FP32", c, R, uni ? ", uniform" : "",
                multi ? ", multi-pass" : "", best_v, variant_name(c, best_v, f64).c_str(),
                best_ms);
    }
  }
  tuned_ = true;
  if (!path.empty()) save_tuning(path);
  if (variants_out)
    for (int c = 0; c < kNumClasses; ++c) variants_out[c] = variant_[c];
  return RODV_OK;
}

rodv_status Engine::measure_peaks(double* f32, double* f32x2, double* f64, double* mhz) {
  RODV_CUDA(cudaSetDevice(device_));
  DeviceMem scratch;
  RODV_CUDA(scratch.ensure(kPeakScratchBytes));
  // 8 blocks of 256 threads per SM (all resident); ~20-40 ms per launch
  const int threads = 256, blocks = num_sms_ * 8, iters = 262144;
  double res[3] = {0, 0, 0};
  double clock_mhz = 0;
  for (int kind = 0; kind < 3; ++kind) {
    RODV_CUDA(run_peak(kind, blocks, threads, iters / 8, stream_, scratch.ptr));  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      if (kind == 0)
        RODV_CUDA(cudaMemsetAsync(static_cast<char*>(scratch.ptr) + kPeakCyclesOffset, 0, 8,
                                  stream_));
      RODV_CUDA(cudaEventRecord(ev_[0], stream_));
      RODV_CUDA(run_peak(kind, blocks, threads, iters, stream_, scratch.ptr));
      RODV_CUDA(cudaEventRecord(ev_[1], stream_));
      RODV_CUDA(cudaEventSynchronize(ev_[1]));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
      if (ms < best) {
        best = ms;
        if (kind == 0) {
          long long cyc = 0;
          RODV_CUDA(cudaMemcpy(&cyc, static_cast<char*>(scratch.ptr) + kPeakCyclesOffset,
                               sizeof(cyc), cudaMemcpyDeviceToHost));
          clock_mhz = (double)cyc / (ms * 1e3);
        }
      }
    }
    res[kind] = peak_flops_per_launch(kind, blocks, threads, iters) / (best * 1e-3) / 1e9;
  }
  if (f32) *f32 = res[0];
  if (f32x2) *f32x2 = res[1];
  if (f64) *f64 = res[2];
  if (mhz) *mhz = clock_mhz;
  return RODV_OK;
}

}  // namespace rodv

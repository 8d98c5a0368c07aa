// noalloc.cu -- rodv_pairhmm_batch_noalloc: the batch call for callers that
// cannot allocate device memory.
//
// Who needs it.  Some callers own every byte of device memory themselves (a
// framework's caching allocator, a memory pool reserved at start-up) or run
// where a cudaMalloc/cudaFree would synchronise the device or may fail (a
// latency-critical loop, a process whose device memory is fully reserved by
// others).  They allocate the batch's input and output buffers their own way
// and need a compute call that allocates nothing.  This entry point is that
// call: every byte of scratch it needs -- the packed batch, the work lists and
// counters, the boundary rows of multi-pass sweeps and the prior tables --
// lives in one file-scope __device__ array of fixed size (kScratchBytes, about
// 12 MB), which every GPU that loads this library holds until the process
// exits.  It calls no cudaMalloc, cudaFree, cudaMallocHost or other allocating
// routine.
//
// How it works.  The caller passes a rodv_batch whose array pointers are
// device memory, and a device output array.  On the caller's stream:
//   na_prefix_kernel   validates sizes and computes offsets (one block);
//   na_pack_kernel     packs bases and qualities into the scratch layout;
//   na_pairs_kernel    builds the two-pair work items (and FP64 lists);
//   forward_kernel     the multi-pass FP32 kernel (8 rows per lane, per-row
//                      gap priors) and its FP64 rescue -- the same kernel
//                      template as the batched engine -- with the boundary rows
//                      in the scratch array.
// Then it reads the error word back and synchronises the stream.
//
// Set-up.  Host code cannot use the array's name as a device address: in host
// code it names a host-side stand-in.  The first call on each device (with
// that device current) obtains the real address with cudaGetSymbolAddress,
// copies the prior tables into the array and raises the two forward kernels'
// dynamic shared-memory limit (their tables and boundary ring take more than
// the default 48 KB per block; a function attribute, not an allocation); that
// first call synchronises the device and must come before any stream capture.
//
// The array is shared by every call in the process on that device and keeps
// the last call's contents; each call clears the counters and pads it depends
// on.  Calls that overlap on the GPU (two streams, two threads) race on it and
// must be serialised by the caller.
#include <cuda_runtime.h>

#include <cub/block/block_scan.cuh>
#include <mutex>

#include "../../include/rodv_pairhmm.h"
#include "layout.h"
#include "pairhmm_fwd.cuh"
#include "tables.h"

namespace rodv {
namespace {

// ---- limits (stated in include/rodv_pairhmm.h) -----------------------------
constexpr uint32_t kNaMaxRegions = RODV_NOALLOC_MAX_REGIONS;
constexpr uint32_t kNaMaxHaps = RODV_NOALLOC_MAX_HAPS;
constexpr uint32_t kNaMaxReads = RODV_NOALLOC_MAX_READS;
constexpr uint32_t kNaMaxPairs = RODV_NOALLOC_MAX_PAIRS;
constexpr uint32_t kNaMaxHapLen = RODV_NOALLOC_MAX_HAP_LEN;
constexpr uint64_t kNaMaxHapBases = RODV_NOALLOC_MAX_HAP_BASES;
constexpr uint64_t kNaMaxReadBases = RODV_NOALLOC_MAX_READ_BASES;
// The two forward kernels of this call: the multi-pass FP32 kernel with
// per-row gap priors and its FP64 rescue.
using NaF32 = Forward<F32x2, kMaxRowsPerLane, false, true, false, 1>;
using NaF64 = Forward<F64, kMaxRowsPerLane, false, true, false, 1>;
constexpr int kNaBlocks = 32;                    // forward kernels' fixed grid
// resident warps owning boundary rows
constexpr int kNaWarps = kNaBlocks * (NaF32::kWarpsPerBlock > NaF64::kWarpsPerBlock
                                          ? NaF32::kWarpsPerBlock
                                          : NaF64::kWarpsPerBlock);
constexpr uint32_t kNaCols = kNaMaxHapLen + 40;  // boundary columns per warp

constexpr size_t al(size_t v) { return (v + 255) / 256 * 256; }

// ---- scratch layout (byte offsets) -----------------------------------------
constexpr size_t kOffPh2prF = 0;
constexpr size_t kOffMmF = al(kOffPh2prF + 128 * 4);
constexpr size_t kOffPh2prD = al(kOffMmF + kMmTableSize * 4);
constexpr size_t kOffMmD = al(kOffPh2prD + 128 * 8);
constexpr size_t kTablesEnd = al(kOffMmD + kMmTableSize * 8);
constexpr size_t kOffCounters = kTablesEnd;
constexpr size_t kOffRegOff = al(kOffCounters + 64 * 4);
constexpr size_t kOffHapCodes = al(kOffRegOff + (kNaMaxRegions + 1) * 8);
// haplotype bases + one pad per haplotype + the tail pad after the last one
constexpr size_t kHapCodeUsedMax = kNaMaxHapBases + (size_t)kNaMaxHaps * kHapPad;
constexpr size_t kHapTail = 2 * kHapPad + kNaMaxHapLen + kHapPad;
constexpr size_t kOffHaps = al(kOffHapCodes + kHapCodeUsedMax + kHapTail);
constexpr size_t kOffRows = al(kOffHaps + kNaMaxHaps * sizeof(HapDesc));
constexpr size_t kRowWords = kNaMaxReadBases + 3 * (size_t)kNaMaxReads;
constexpr size_t kOffReads = al(kOffRows + kRowWords * 4);
constexpr size_t kOffItems = al(kOffReads + kNaMaxReads * sizeof(ReadDesc));
constexpr size_t kOffList = al(kOffItems + (kNaMaxPairs / 2 + 1) * sizeof(DiffItem));
constexpr size_t kOffBoundary = al(kOffList + kNaMaxPairs * sizeof(PairRef));
constexpr size_t kScratchBytes = al(kOffBoundary + (size_t)kNaWarps * kNaCols * 24);

// counter words
enum : int { kCItems = 0, kCCtr32 = 1, kCCtr64 = 2, kCRescue = 3, kCErr = 4, kCPairs = 5,
             kCHapBytes = 6 };
// device-side validation bits (the low bits are the forward kernels' ErrorFlag)
enum : uint32_t {
  kNaErrTooMany = 1u << 8,   // pairs / bases / one read's length above the limits
  kNaErrHapLen = 1u << 9,    // a haplotype above RODV_NOALLOC_MAX_HAP_LEN
  kNaErrEmpty = 1u << 10,    // a region without haplotypes or reads
  kNaErrIndex = 1u << 11,    // a region indexes outside the batch
  kNaErrZeroLen = 1u << 12,  // an empty haplotype or read
  kNaErrBase = 1u << 13,     // a base other than A, C, G, T, N
};

// The scratch array.  In host code this name is a host-side stand-in, not a
// device address; host code uses the pointer from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct NaArgs {
  rodv_batch b;        // array pointers are device memory
  unsigned char* s;    // scratch base (device address)
  int use_double;
};

__device__ __forceinline__ uint32_t* counters(unsigned char* s) {
  return reinterpret_cast<uint32_t*>(s + kOffCounters);
}

__device__ __forceinline__ uint8_t code_of(uint8_t c, uint32_t* err) {
  switch (c) {
    case 'A': return kA;
    case 'C': return kC;
    case 'G': return kG;
    case 'T': return kT;
    case 'N': return kN;
    default: *err |= kNaErrBase; return kA;
  }
}

// Exclusive prefix sums over regions, haplotypes and reads, with validation.
// One block of 1024 threads.
__global__ void __launch_bounds__(1024) na_prefix_kernel(NaArgs a) {
  using Scan = cub::BlockScan<unsigned long long, 1024>;
  __shared__ typename Scan::TempStorage tmp;
  __shared__ unsigned long long running;
  __shared__ uint32_t err_s;
  uint32_t* c = counters(a.s);
  const rodv_batch& b = a.b;
  if (threadIdx.x == 0) { running = 0; err_s = 0; }
  __syncthreads();
  uint32_t err = 0;

  unsigned long long* reg_off = reinterpret_cast<unsigned long long*>(a.s + kOffRegOff);
  for (uint32_t base = 0; base < b.num_regions; base += 1024) {
    const uint32_t g = base + threadIdx.x;
    unsigned long long v = 0;
    if (g < b.num_regions) {
      const rodv_region r = b.regions[g];
      if (r.num_haps == 0 || r.num_reads == 0) err |= kNaErrEmpty;
      if ((unsigned long long)r.hap_start + r.num_haps > b.num_haps ||
          (unsigned long long)r.read_start + r.num_reads > b.num_reads)
        err |= kNaErrIndex;
      v = (unsigned long long)r.num_haps * r.num_reads;
    }
    unsigned long long ex, agg;
    Scan(tmp).ExclusiveSum(v, ex, agg);
    if (g < b.num_regions) reg_off[g] = running + ex;
    __syncthreads();
    if (threadIdx.x == 0) running += agg;
    __syncthreads();
  }
  const unsigned long long total_pairs = running;
  __syncthreads();
  if (threadIdx.x == 0) { reg_off[b.num_regions] = total_pairs; running = 0; }
  if (total_pairs > kNaMaxPairs) err |= kNaErrTooMany;
  __syncthreads();

  HapDesc* hd = reinterpret_cast<HapDesc*>(a.s + kOffHaps);
  for (uint32_t base = 0; base < b.num_haps; base += 1024) {
    const uint32_t h = base + threadIdx.x;
    unsigned long long v = 0;
    if (h < b.num_haps) {
      const uint32_t len = b.hap_lengths[h];
      if (len == 0) err |= kNaErrZeroLen;
      if (len > kNaMaxHapLen) err |= kNaErrHapLen;
      v = (unsigned long long)len + kHapPad;
    }
    unsigned long long ex, agg;
    Scan(tmp).ExclusiveSum(v, ex, agg);
    if (h < b.num_haps) {
      hd[h].code_off = running + ex + kHapPad;
      hd[h].len = b.hap_lengths[h];
      hd[h].pad_ = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) running += agg;
    __syncthreads();
  }
  const unsigned long long hap_bytes = running;
  __syncthreads();
  if (threadIdx.x == 0) running = 0;
  if (hap_bytes > kHapCodeUsedMax) err |= kNaErrTooMany;
  __syncthreads();

  ReadDesc* rd = reinterpret_cast<ReadDesc*>(a.s + kOffReads);
  for (uint32_t base = 0; base < b.num_reads; base += 1024) {
    const uint32_t r = base + threadIdx.x;
    unsigned long long v = 0;
    if (r < b.num_reads) {
      const uint32_t len = b.read_lengths[r];
      if (len == 0) err |= kNaErrZeroLen;
      // a read above the engine's read limit is refused before its padded
      // length is formed (64-bit, so no length wraps to a small value)
      if (len > RODV_MAX_READ_LEN) err |= kNaErrTooMany;
      v = ((unsigned long long)len + 3ull) & ~3ull;
    }
    unsigned long long ex, agg;
    Scan(tmp).ExclusiveSum(v, ex, agg);
    if (r < b.num_reads) {
      rd[r].row_off = running + ex;
      rd[r].len = b.read_lengths[r];
      rd[r].flags = 0;  // the per-row gap-prior kernel serves every read
    }
    __syncthreads();
    if (threadIdx.x == 0) running += agg;
    __syncthreads();
  }
  if (running > kRowWords) err |= kNaErrTooMany;
  atomicOr(&err_s, err);
  __syncthreads();
  const uint32_t e = err_s;
  if (threadIdx.x == 0) {
    c[kCErr] = e;
    const uint32_t np = e ? 0u : (uint32_t)total_pairs;
    c[kCPairs] = np;
    c[kCItems] = a.use_double ? 0u : (np + 1) / 2;
    c[kCRescue] = a.use_double ? np : 0u;
    c[kCCtr32] = 0;
    c[kCCtr64] = 0;
    c[kCHapBytes] = e ? 0u : (uint32_t)hap_bytes;
  }
  // the tail pad after the last haplotype reads as code 0
  if (!e) {
    unsigned char* codes = a.s + kOffHapCodes;
    for (size_t k = hap_bytes + threadIdx.x; k < hap_bytes + kHapTail; k += 1024) codes[k] = 0;
  }
}

// Bases to codes and read rows to row words; one warp per haplotype or read.
__global__ void na_pack_kernel(NaArgs a) {
  uint32_t* c = counters(a.s);
  if (c[kCErr]) return;
  const rodv_batch& b = a.b;
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const uint32_t nwarps = gridDim.x * blockDim.x / 32;
  uint32_t err = 0;
  unsigned char* codes = a.s + kOffHapCodes;
  const HapDesc* hd = reinterpret_cast<const HapDesc*>(a.s + kOffHaps);
  for (uint32_t h = warp; h < b.num_haps; h += nwarps) {
    const uint64_t off = hd[h].code_off;
    const uint32_t len = hd[h].len;
    const uint8_t* src = b.hap_bases + b.hap_offsets[h];
    if (lane < kHapPad) codes[off - kHapPad + lane] = 0;
    for (uint32_t k = lane; k < len; k += 32) codes[off + k] = code_of(src[k], &err);
  }
  uint32_t* rows = reinterpret_cast<uint32_t*>(a.s + kOffRows);
  const ReadDesc* rd = reinterpret_cast<const ReadDesc*>(a.s + kOffReads);
  for (uint32_t r = warp; r < b.num_reads; r += nwarps) {
    const uint64_t off = rd[r].row_off;
    const uint32_t len = rd[r].len;
    const uint64_t src = b.read_offsets[r];
    const uint64_t padded = ((uint64_t)len + 3u) & ~3ull;
    for (uint64_t k = lane; k < padded; k += 32) {
      uint32_t w = 0;
      if (k < len)
        w = row_word(code_of(b.read_bases[src + k], &err), b.base_quals[src + k],
                     b.ins_quals[src + k], b.del_quals[src + k], b.gcp_quals[src + k]);
      rows[off + k] = w;
    }
  }
  if (err) atomicOr(&c[kCErr], err);
}

// Pair p (result order) as a PairRef: its region by binary search over the
// region offsets, then hap-major position inside the region.
__device__ __forceinline__ PairRef pair_ref(const NaArgs& a, uint32_t p) {
  const unsigned long long* reg_off =
      reinterpret_cast<const unsigned long long*>(a.s + kOffRegOff);
  uint32_t lo = 0, hi = a.b.num_regions;  // reg_off[lo] <= p < reg_off[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (reg_off[mid] <= p) lo = mid; else hi = mid;
  }
  const rodv_region r = a.b.regions[lo];
  const uint32_t local = p - (uint32_t)reg_off[lo];
  return PairRef{r.hap_start + local / r.num_reads, r.read_start + local % r.num_reads, p};
}

// Two-pair FP32 items over consecutive pairs (longer haplotype in slot x),
// and the FP64 list when every pair is forced to FP64.
__global__ void na_pairs_kernel(NaArgs a) {
  uint32_t* c = counters(a.s);
  const uint32_t np = c[kCPairs];
  DiffItem* items = reinterpret_cast<DiffItem*>(a.s + kOffItems);
  PairRef* list = reinterpret_cast<PairRef*>(a.s + kOffList);
  const uint32_t stride = gridDim.x * blockDim.x;
  if (a.use_double)
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += stride)
      list[p] = pair_ref(a, p);
  const uint32_t ni = c[kCItems];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ni; k += stride) {
    const PairRef x = pair_ref(a, 2 * k);
    if (2 * k + 1 >= np) {
      items[k].x = x;
      items[k].y = PairRef{0, kNoPair, 0};
      continue;
    }
    const PairRef y = pair_ref(a, 2 * k + 1);
    const bool swap = a.b.hap_lengths[y.hap] > a.b.hap_lengths[x.hap];
    items[k].x = swap ? y : x;
    items[k].y = swap ? x : y;
  }
}

// Dynamic shared memory per block of the two kernels.
constexpr int kSmemF32 = NaF32::kWarpsPerBlock * NaF32::kSmemPerWarp;
constexpr int kSmemF64 = NaF64::kWarpsPerBlock * NaF64::kSmemPerWarp;
static_assert(kSmemF32 <= 227 * 1024 && kSmemF64 <= 227 * 1024, "tables too large");

// Per-device set-up: the scratch array's device address, tables copied in,
// the kernels' shared-memory limit raised.  Only a successful set-up is kept:
// a failed one (say, a call made before the device could be used) is tried
// again by the next call.
struct DeviceSlot {
  unsigned char* ptr = nullptr;
};
constexpr int kMaxDevices = 64;
DeviceSlot g_slots[kMaxDevices];
std::mutex g_setup_mu;

cudaError_t setup_device(int dev, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  DeviceSlot& slot = g_slots[dev];
  cudaError_t e = cudaSuccess;
  if (!slot.ptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e == cudaSuccess) {
      const HostPriorTables& t = host_prior_tables();
      unsigned char* s = static_cast<unsigned char*>(p);
      e = cudaMemcpy(s + kOffPh2prF, t.ph2pr_f.data(), 128 * 4, cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(s + kOffMmF, t.mm_f.data(), kMmTableSize * 4, cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(s + kOffPh2prD, t.ph2pr_d.data(), 128 * 8, cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(s + kOffMmD, t.mm_d.data(), kMmTableSize * 8, cudaMemcpyHostToDevice);
      // the two kernels' shared memory (tables and boundary ring) may exceed
      // the default 48 KB per block
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(&forward_kernel<F32x2, kMaxRowsPerLane, false, true, false, 1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemF32);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(&forward_kernel<F64, kMaxRowsPerLane, false, true, false, 1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemF64);
    }
    if (e == cudaSuccess) slot.ptr = static_cast<unsigned char*>(p);
  }
  *out = slot.ptr;
  return e;
}

// True when p is memory of the current device (device or managed).
bool on_device(const void* p, int dev) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // an unregistered host pointer; clear the error it left
    return false;
  }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) &&
         at.device == dev;
}

rodv_status status_of_flags(uint32_t f) {
  if (f & (kNaErrTooMany | kNaErrHapLen)) return RODV_ERR_TOO_LONG;
  if (f & kNaErrEmpty) return RODV_ERR_EMPTY;
  if (f & (kNaErrIndex | kNaErrZeroLen)) return RODV_ERR_INVALID_ARG;
  if (f & kNaErrBase) return RODV_ERR_INVALID_BASE;
  return RODV_ERR_DEVICE_CHECK;
}

}  // namespace
}  // namespace rodv

extern "C" rodv_status rodv_pairhmm_batch_noalloc(const rodv_batch* batch, int32_t use_double,
                                                  double* out_log10, void* stream) {
  using namespace rodv;
  if (!batch || !out_log10 || !batch->regions || !batch->hap_bases || !batch->hap_offsets ||
      !batch->hap_lengths || !batch->read_bases || !batch->base_quals || !batch->ins_quals ||
      !batch->del_quals || !batch->gcp_quals || !batch->read_offsets || !batch->read_lengths)
    return RODV_ERR_INVALID_ARG;
  if (batch->num_regions == 0) return RODV_ERR_EMPTY;
  if (batch->num_regions > kNaMaxRegions || batch->num_haps > kNaMaxHaps ||
      batch->num_reads > kNaMaxReads)
    return RODV_ERR_TOO_LONG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RODV_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return RODV_ERR_NO_DEVICE;
  int major = 0, minor = 0, sms = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return RODV_ERR_NO_DEVICE;
  if (major != 10 || minor != 0) return RODV_ERR_NO_DEVICE;
  // An error left pending by earlier work on this thread is not this call's
  // to clear or report as its own: refuse to launch on top of it.
  if (cudaPeekAtLastError() != cudaSuccess) return RODV_ERR_CUDA;
  // Every array must be memory of this device: a host pointer read by a
  // kernel is an illegal access that ends the caller's context.
  const void* arrays[] = {batch->regions,    batch->hap_bases,  batch->hap_offsets,
                          batch->hap_lengths, batch->read_bases, batch->base_quals,
                          batch->ins_quals,  batch->del_quals,  batch->gcp_quals,
                          batch->read_offsets, batch->read_lengths, out_log10};
  for (const void* p : arrays)
    if (!on_device(p, dev)) return RODV_ERR_INVALID_ARG;
  unsigned char* s = nullptr;
  if (setup_device(dev, &s) != cudaSuccess || !s) return RODV_ERR_CUDA;

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  NaArgs a;
  a.b = *batch;
  a.s = s;
  a.use_double = use_double ? 1 : 0;
  na_prefix_kernel<<<1, 1024, 0, st>>>(a);
  na_pack_kernel<<<sms * 4, 256, 0, st>>>(a);
  na_pairs_kernel<<<sms * 2, 256, 0, st>>>(a);

  BatchView v;
  v.hap_codes = s + kOffHapCodes;
  v.read_rows = reinterpret_cast<const uint32_t*>(s + kOffRows);
  v.haps = reinterpret_cast<const HapDesc*>(s + kOffHaps);
  v.reads = reinterpret_cast<const ReadDesc*>(s + kOffReads);
  v.out = out_log10;
  v.raw_prec = nullptr;
  v.tab.ph2pr_f = reinterpret_cast<const float*>(s + kOffPh2prF);
  v.tab.mm_f = reinterpret_cast<const float*>(s + kOffMmF);
  v.tab.ph2pr_d = reinterpret_cast<const double*>(s + kOffPh2prD);
  v.tab.mm_d = reinterpret_cast<const double*>(s + kOffMmD);
  uint32_t* cnt = reinterpret_cast<uint32_t*>(s + kOffCounters);

  using F32 = NaF32;
  using D64 = NaF64;
  ClassLaunch c32{};
  c32.work = s + kOffItems;
  c32.work_count = cnt + kCItems;
  c32.counter = cnt + kCCtr32;
  c32.rescue_list = reinterpret_cast<PairRef*>(s + kOffList);
  c32.rescue_count = cnt + kCRescue;
  c32.scratch = reinterpret_cast<float*>(s + kOffBoundary);
  c32.scratch_cols = kNaCols;
  c32.error_flags = cnt + kCErr;
  forward_kernel<F32x2, kMaxRowsPerLane, false, true, false, 1>
      <<<kNaBlocks, F32::kWarpsPerBlock * kWarp,
         F32::kWarpsPerBlock * F32::kSmemPerWarp, st>>>(
          v, c32);
  ClassLaunch c64 = c32;
  c64.work = s + kOffList;
  c64.work_count = cnt + kCRescue;
  c64.counter = cnt + kCCtr64;
  c64.rescue_list = nullptr;
  c64.rescue_count = nullptr;
  forward_kernel<F64, kMaxRowsPerLane, false, true, false, 1>
      <<<kNaBlocks, D64::kWarpsPerBlock * kWarp,
         D64::kWarpsPerBlock * D64::kSmemPerWarp, st>>>(
          v, c64);
  // nothing was pending on entry, so a launch error now is this call's own
  if (cudaGetLastError() != cudaSuccess) return RODV_ERR_CUDA;

  uint32_t flags = 0;
  if (cudaMemcpyAsync(&flags, cnt + kCErr, sizeof(flags), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return RODV_ERR_CUDA;
  return flags ? status_of_flags(flags) : RODV_OK;
}

/*
 * rodv_pairhmm.h -- C ABI of the B200 PairHMM engine.
 *
 * The engine computes, for every (haplotype, read) pair of every region in a
 * batch, the PairHMM forward log10 likelihood that roDV's src/core batch API
 * computes on the CPU.  All functions are plain C: caller-owned host
 * buffers, engine-owned device state, integer status codes, no exceptions
 * across the boundary.  One engine may be shared by several host threads;
 * calls on one engine are serialised internally.
 *
 * Reference interfaces replaced (paths relative to the roDV repository):
 *   pairhmm::schedule::schedule_pairhmm     src/core/pairhmm_schedule.h:14-25
 *       -> rodv_pairhmm_batch (and the C++ shim of the same name in
 *          rodv_b200/csrc/schedule_shim.cpp, declared in
 *          include/rodv_pairhmm_schedule.h)
 *   pairhmm::intra::computeLikelihoodsAVX2/AVX512
 *                                           src/core/pairhmm/intra/pairhmm_api.h:17-20
 *       -> rodv_pairhmm_pair
 *   pairhmm::inter::compute_inter_pairhmm_{AVX2,AVX512}_{float,double}
 *                                           src/core/pairhmm/inter/pairhmm_inter_api.h:17-24
 *       -> rodv_pairhmm_batch with one single-pair region per test case
 *          (islog10 = true), rodv_pairhmm_batch_raw (islog10 = false)
 * Base comparison: the engine applies the intra kernel's rule everywhere
 * ('N' on either side matches any base, pairhmm_impl.cpp:26-42), also where
 * roDV's inter kernel compares raw bytes (inter/simd_traits_avx2.h:61-63);
 * roDV's scheduler never sends a pair with 'N' to the inter kernel, so the
 * two agree on every pair schedule_pairhmm computes.
 */
#ifndef RODV_PAIRHMM_H_
#define RODV_PAIRHMM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RODV_ABI_VERSION 2

typedef int32_t rodv_status;
enum {
  RODV_OK = 0,
  RODV_ERR_INVALID_ARG = 1,   /* null pointer, bad index, zero length, quals length mismatch */
  RODV_ERR_EMPTY = 2,         /* a region with no haplotypes or no reads (reference returns
                                 false, pairhmm_schedule.cpp:130-132) */
  RODV_ERR_INVALID_BASE = 3,  /* a base other than A, C, G, T, N */
  RODV_ERR_NO_DEVICE = 4,     /* no CUDA device, or the library was built for another arch */
  RODV_ERR_CUDA = 5,          /* a CUDA runtime call failed */
  RODV_ERR_OUT_OF_MEMORY = 6, /* device or pinned host allocation failed */
  RODV_ERR_TOO_LONG = 7,      /* read or haplotype above the engine limits */
  RODV_ERR_DEVICE_CHECK = 8,  /* a kernel reported a bad descriptor or an expired wait */
  RODV_ERR_ADMISSION = 9,     /* streaming: region does not fit the device memory budget */
  RODV_ERR_NOT_FOUND = 10,    /* streaming: unknown ticket */
  RODV_ERR_NOT_READY = 11,    /* streaming: result not yet available */
  RODV_ERR_SHUTDOWN = 12,     /* streaming: service stopped */
  RODV_ERR_INTERNAL = 13      /* an internal consistency check failed (a bug; please report) */
};

/* Engine limits (inputs beyond them are rejected with RODV_ERR_TOO_LONG). */
#define RODV_MAX_READ_LEN 65536u
#define RODV_MAX_HAP_LEN 65536u

/* A region is roDV's schedule_pairhmm call: haplotypes [hap_start,
 * hap_start+num_haps) against reads [read_start, read_start+num_reads). */
typedef struct rodv_region {
  uint32_t hap_start;
  uint32_t num_haps;
  uint32_t read_start;
  uint32_t num_reads;
} rodv_region;

/* A batch of regions over flat host arrays.  Bases are ASCII A/C/G/T/N;
 * qualities are raw Phred integers (not +33), one per read base in each of
 * the four arrays (base, insertion, deletion, gap continuation), masked with
 * &127 as the reference does.  Results of region g are written hap-major
 * (result[h][r] of schedule_pairhmm) starting at sum over g' < g of
 * num_haps*num_reads. */
typedef struct rodv_batch {
  uint32_t num_regions;
  const rodv_region* regions;
  uint32_t num_haps;
  const uint8_t* hap_bases;
  const uint64_t* hap_offsets;
  const uint32_t* hap_lengths;
  uint32_t num_reads;
  const uint8_t* read_bases;
  const uint8_t* base_quals;
  const uint8_t* ins_quals;
  const uint8_t* del_quals;
  const uint8_t* gcp_quals;
  const uint64_t* read_offsets; /* shared by read_bases and the four quality arrays */
  const uint32_t* read_lengths;
} rodv_batch;

typedef struct rodv_options {
  int32_t device;               /* CUDA device ordinal */
  int32_t force_fp64;           /* 1: every pair in FP64 (schedule_pairhmm use_double) */
  uint64_t device_memory_budget;/* bytes the streaming service may hold; 0 = 50% of free */
  uint32_t max_inflight;        /* streaming: regions admitted at once; 0 = 4096 */
  int32_t verbose;              /* 1: print per-batch statistics to stderr */
  int32_t autotune;             /* 0: cached or default kernel variants; 1: tune at creation
                                   unless the cache has this device; 2: always tune */
  const char* tune_cache;       /* file of tuned variants (read, and written after tuning);
                                   NULL = none */
} rodv_options;

typedef struct rodv_stats {
  uint64_t pairs;               /* pairs computed */
  uint64_t cells;               /* sum of read_len * hap_len over pairs */
  uint64_t fp64_pairs;          /* pairs computed in FP64 (rescued or forced) */
  uint64_t fp64_cells;
  uint32_t kernel_launches;     /* forward/pack kernels launched by this call */
  uint32_t pad_;
  double total_ms;              /* wall time of the call */
  double device_ms;             /* device time of the forward kernels (CUDA events) */
  double fp32_ms;               /* device time of the FP32 pass */
  double h2d_ms;
  double d2h_ms;
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
} rodv_stats;

typedef struct rodv_engine rodv_engine;
typedef struct rodv_device_batch rodv_device_batch;

/* Fills opts with defaults (device 0, FP32 with FP64 rescue). */
void rodv_default_options(rodv_options* opts);

rodv_status rodv_engine_create(const rodv_options* opts, rodv_engine** out);
void rodv_engine_destroy(rodv_engine* engine);

/* Whole batch, host buffers in and out: pack, upload, compute, download.
 * Replaces schedule_pairhmm (pairhmm_schedule.h:14-25) for many regions at
 * once; out_log10 holds rodv_batch_num_pairs(batch) doubles.  use_double != 0
 * computes every pair in FP64 (schedule_pairhmm's use_double); otherwise
 * FP32 with FP64 rescue below 1e-28.  stats may be null. */
rodv_status rodv_pairhmm_batch(rodv_engine* engine, const rodv_batch* batch, int32_t use_double,
                               double* out_log10, rodv_stats* stats);

/* The same computation returning raw likelihoods instead of log10, as
 * compute_inter_pairhmm_*(..., islog10 = false) does
 * (pairhmm_inter_api.h:17-24, pairhmm_schedule.cpp:229-248): out_raw[i] is
 * the pair's scaled likelihood sum(M + I) of the last row and
 * out_precision[i] the precision that produced it: 0 = FP32 with row 0 at
 * 2^120/haplen (log10 = log10(raw) - 36.1236000061f; raw >= 1e-28 always),
 * 1 = FP64 with row 0 at 2^1020/haplen (log10 = log10(raw) -
 * 307.050595577260822; 0 where the reference's flush-to-zero gives -inf).
 * FP32 results below the acceptance bound are recomputed in FP64 as in
 * rodv_pairhmm_batch; use_double != 0 makes every result FP64.  Both arrays
 * hold rodv_batch_num_pairs(batch) entries. */
rodv_status rodv_pairhmm_batch_raw(rodv_engine* engine, const rodv_batch* batch,
                                   int32_t use_double, double* out_raw, uint8_t* out_precision,
                                   rodv_stats* stats);

/* Number of results of a batch (sum of num_haps*num_reads). */
uint64_t rodv_batch_num_pairs(const rodv_batch* batch);

/* Checks a batch on the host, without a device, by the rules the compute
 * calls apply: at least one region; every region with haplotypes and reads
 * and indexing inside the arrays; no empty sequence; lengths within the
 * limits above; fewer than 2^32 pairs; bases A, C, G, T or N.  Returns
 * RODV_OK or the status a compute call would return for the batch; msg (may
 * be null) receives a description, at most msg_len bytes including the
 * terminating zero.  No counterpart in the reference: schedule_pairhmm checks
 * only for M == 0 or N == 0 (pairhmm_schedule.cpp:130-132) and reads other
 * invalid input out of bounds. */
rodv_status rodv_batch_validate(const rodv_batch* batch, char* msg, size_t msg_len);

/* One pair (computeLikelihoodsAVX512(tc, use_double), pairhmm_api.h:17-20):
 * FP32 with FP64 rescue below 1e-28, or FP64 when use_double != 0. */
rodv_status rodv_pairhmm_pair(rodv_engine* engine, const uint8_t* hap, uint32_t hap_len,
                              const uint8_t* read, const uint8_t* base_quals,
                              const uint8_t* ins_quals, const uint8_t* del_quals,
                              const uint8_t* gcp_quals, uint32_t read_len, int32_t use_double,
                              double* out_log10);

/* Device-resident batches: upload once, run many times, read results.
 * rodv_device_batch_run computes with inputs already in HBM (no host
 * copies); results stay on the device until rodv_device_batch_download. */
rodv_status rodv_device_batch_upload(rodv_engine* engine, const rodv_batch* batch,
                                     rodv_device_batch** out);
rodv_status rodv_device_batch_run(rodv_engine* engine, rodv_device_batch* dbatch,
                                  rodv_stats* stats);
rodv_status rodv_device_batch_download(rodv_engine* engine, rodv_device_batch* dbatch,
                                       double* out_log10);
void rodv_device_batch_free(rodv_engine* engine, rodv_device_batch* dbatch);

/* The plain GPU form: one kernel launch per pair (plus one FP64 launch for a
 * pair below the threshold) over a device-resident batch, results downloaded
 * to out_log10.  Kept as the comparison point for the batched engine. */
rodv_status rodv_pairhmm_plain(rodv_engine* engine, rodv_device_batch* dbatch,
                               double* out_log10, rodv_stats* stats);

/* Arithmetic peak of the device, measured by FMA-chain kernels: FP32 FFMA,
 * FP32x2 FFMA2 and FP64 DFMA, in GFLOP/s, and the SM clock in MHz seen
 * during the FP32 run (from clock64 against CUDA events). */
rodv_status rodv_measure_peaks(rodv_engine* engine, double* fp32_gflops, double* fp32x2_gflops,
                               double* fp64_gflops, double* sm_mhz);

/* ---- One batch over several GPUs -------------------------------------------
 * roDV runs schedule_pairhmm (pairhmm_schedule.cpp:116-340) once per region on
 * one thread; regions are independent, so a batch splits over GPUs by region
 * with no exchange between them.  rodv_shard_plan assigns every region to one
 * of num_shards shards, longest processing time first by cells (sum of
 * haplotype lengths x sum of read lengths): regions in decreasing cell count,
 * each to the shard with the fewest cells so far, lowest index on a tie.  The
 * plan depends only on the batch and num_shards, so every process of a
 * multi-process job computes the same plan.  Host only: no device is needed.
 * region_shard receives num_regions shard indices; shard_cells (may be NULL)
 * num_shards cell counts.
 * rodv_shard_merge is the inverse step: shard_results[k] holds the results of
 * shard k's regions, in batch order, as rodv_pairhmm_batch returns them for a
 * batch of just those regions; they are copied into out_log10 in the batch's
 * result order.  Host only.
 * rodv_multi_create makes one engine per listed device (a device may be
 * listed twice: two engines share it); rodv_multi_batch plans the shards,
 * runs each device's shard through its engine on its own host thread (host
 * buffers in and out, as rodv_pairhmm_batch) and merges the results.  Results
 * are bitwise those of rodv_pairhmm_batch on one device.  stats: pairs,
 * cells and bytes summed over devices, device times the maximum. */
rodv_status rodv_shard_plan(const rodv_batch* batch, uint32_t num_shards, uint32_t* region_shard,
                            uint64_t* shard_cells);
rodv_status rodv_shard_merge(const rodv_batch* batch, uint32_t num_shards,
                             const uint32_t* region_shard, const double* const* shard_results,
                             double* out_log10);
typedef struct rodv_multi rodv_multi;
rodv_status rodv_multi_create(const rodv_options* opts, const int32_t* devices,
                              uint32_t num_devices, rodv_multi** out);
void rodv_multi_destroy(rodv_multi* multi);
rodv_status rodv_multi_batch(rodv_multi* multi, const rodv_batch* batch, int32_t use_double,
                             double* out_log10, rodv_stats* stats);
/* Details of the last failure of rodv_multi_batch (valid until the next call). */
const char* rodv_multi_last_error(rodv_multi* multi);

/* ---- Allocation-free batch call ------------------------------------------
 * No counterpart in the reference (roDV computes on the CPU and allocates per
 * call).  For callers that cannot call cudaMalloc: code that owns all device
 * memory through its own allocator or a pool reserved at start-up, or that
 * runs where an allocation would synchronise the device or may fail.  The
 * caller allocates the inputs and the output its own way; this call
 * allocates nothing (no cudaMalloc, cudaFree or cudaMallocHost).  Its
 * scratch is one fixed array of about 12 MB in the library's device memory,
 * held by every GPU that loads the library until the process exits.
 *
 * batch: a rodv_batch whose array pointers (regions included) are DEVICE
 * (or managed) memory on the current device, checked before any launch:
 * anything else returns RODV_ERR_INVALID_ARG; out_log10: device array of
 * rodv_batch_num_pairs() doubles; stream: a cudaStream_t (NULL = default).
 * Results equal rodv_pairhmm_batch's within 1e-5 log10, not bitwise: this
 * call sends every pair through the per-row-prior multi-pass kernels, the
 * batched engine through the scaled and chain kernels.  Returns after the
 * work on `stream` has finished.  A CUDA error already pending on the
 * calling thread is left in place and the call returns RODV_ERR_CUDA
 * without launching.
 * The first call on a device sets that device up (obtains the scratch
 * address, copies the prior tables, raises its two kernels' shared-memory
 * limit per block) and synchronises it: make it before any stream capture.  All calls in a process share the scratch array: calls
 * that overlap on the GPU race and must be serialised by the caller.
 * Sizes beyond the limits below return RODV_ERR_TOO_LONG; on any error the
 * output contents are unspecified. */
#define RODV_NOALLOC_MAX_REGIONS 4096u
#define RODV_NOALLOC_MAX_HAPS 4096u
#define RODV_NOALLOC_MAX_READS 16384u
#define RODV_NOALLOC_MAX_PAIRS 16384u
#define RODV_NOALLOC_MAX_HAP_LEN 2048u      /* bases per haplotype */
#define RODV_NOALLOC_MAX_HAP_BASES 1048576u /* bases over all haplotypes */
#define RODV_NOALLOC_MAX_READ_BASES 1048576u /* bases over all reads; one read at most
                                                RODV_MAX_READ_LEN bases */
rodv_status rodv_pairhmm_batch_noalloc(const rodv_batch* batch, int32_t use_double,
                                       double* out_log10, void* stream);

/* Autotuner: per work class (read-length bucket and gap-prior form), times
 * every variant of the class's kernels on a synthetic batch of that class
 * and keeps the fastest.  Single-pass classes: the FP32 kernel's occupancy
 * target (register budget) and, for reads up to 128 bases, one or two chain
 * items per warp.  Multi-pass classes (reads of 255 bases and more): the strip
 * height (4 or 8 read rows per lane per pass) and the warps that sweep one
 * item's passes concurrently (2 or 4), for the FP32 and the FP64 kernel.
 * Results do not depend on the variants.  No counterpart in the reference,
 * whose only tunables are the grouping idle ratios of schedule_pairhmm
 * (pairhmm_schedule.h:23-24), accepted and ignored by the engine's shim.
 * With cache_path, a cached result for this device is used unless force !=
 * 0, and new results are written there.  variants_out (may be NULL) receives
 * the RODV_TUNE_CLASSES FP32 variant indices; rodv_tuned_variants reads the
 * engine's current FP32 and FP64 variants (either pointer may be NULL). */
#define RODV_TUNE_CLASSES 18
rodv_status rodv_autotune(rodv_engine* engine, const char* cache_path, int32_t force,
                          int32_t* variants_out);
rodv_status rodv_tuned_variants(rodv_engine* engine, int32_t* fp32_variants,
                                int32_t* fp64_variants);

/* ---- Streaming service -----------------------------------------------------
 * No single counterpart in the reference: it stands for a caller that runs
 * schedule_pairhmm (pairhmm_schedule.cpp:116-340) once per region as regions
 * arrive.  rodv_submit_region copies one or more regions (a rodv_batch; the
 * caller's buffers may be reused as soon as it returns) into the service's
 * queue and returns a ticket.  A worker thread puts everything submitted while
 * the GPU was busy into the next device batch (continuous batching over three
 * streams: the next batches are packed and uploaded while earlier ones
 * compute).  A region's results are bitwise identical whatever it was
 * batched with.
 * Admission: opts->device_memory_budget bytes (0 = half of the free device
 * memory) are split between the three batch slots; a request that cannot fit
 * one slot is refused with RODV_ERR_ADMISSION; rodv_submit_region blocks while
 * opts->max_inflight requests (0 = 4096) are queued or computing.
 * rodv_poll returns RODV_ERR_NOT_READY until the results are available, then
 * copies them (hap-major per region, regions in submission order, as
 * rodv_pairhmm_batch writes them) and forgets the ticket; a later call returns
 * RODV_ERR_NOT_FOUND.  rodv_wait blocks up to timeout_ms (< 0: no limit).
 * A request whose batch failed returns that failure's status.
 * rodv_service_destroy finishes all submitted work, then stops. */
typedef struct rodv_service rodv_service;

typedef struct rodv_request_stats {
  uint64_t pairs;
  uint64_t cells;
  uint64_t fp64_pairs;          /* pairs of the request's device batch computed in FP64 */
  uint64_t batch_id;            /* device batch the request was computed in */
  uint32_t batch_regions;       /* regions in that batch */
  uint32_t pad_;
  double queue_ms;              /* submit -> its batch started packing */
  double latency_ms;            /* submit -> results available */
} rodv_request_stats;

typedef struct rodv_service_stats {
  uint64_t submitted;           /* requests since the last reset */
  uint64_t completed;
  uint64_t failed;
  uint64_t batches;
  uint64_t regions;
  uint64_t pairs;
  uint64_t cells;
  uint64_t fp64_pairs;
  double latency_p50_ms;        /* over completed requests (nearest rank) */
  double latency_p99_ms;
  double latency_max_ms;
  double latency_mean_ms;
  double device_ms;             /* sum of the batches' kernel times */
  double wall_ms;               /* first submit -> last completion */
  double mean_batch_regions;
  double host_launch_ms;        /* worker time forming, packing and enqueueing batches */
  double host_finish_ms;        /* worker time handing results to requests */
} rodv_service_stats;

rodv_status rodv_service_create(const rodv_options* opts, rodv_service** out);
void rodv_service_destroy(rodv_service* service);
rodv_status rodv_submit_region(rodv_service* service, const rodv_batch* regions,
                               uint64_t* ticket);
rodv_status rodv_poll(rodv_service* service, uint64_t ticket, double* out_log10,
                      rodv_request_stats* stats);
rodv_status rodv_wait(rodv_service* service, uint64_t ticket, int32_t timeout_ms,
                      double* out_log10, rodv_request_stats* stats);
rodv_status rodv_service_get_stats(rodv_service* service, rodv_service_stats* out);
void rodv_service_reset_stats(rodv_service* service);
/* Details of the service's last failure (valid until this thread's next call). */
const char* rodv_service_last_error(rodv_service* service);

/* ---- Testing hooks -----------------------------------------------------------
 * No counterpart in the reference (whose only failure report is the bool of
 * schedule_pairhmm, pairhmm_schedule.cpp:130-132).  For tests of the engine's
 * failure paths without a real out-of-memory condition.
 * rodv_fault_inject_alloc makes the nth next allocation of one kind fail on
 * the host exactly as an exhausted cudaMalloc / cudaMallocHost would (kind 0:
 * device memory, 1: pinned host memory; nth = 0 disarms it).  Process-wide;
 * affects every engine and service.  rodv_debug_live_allocations reports how
 * many device and pinned-host allocations of the library are live, so a test
 * can check that a failed call released what it had allocated. */
rodv_status rodv_fault_inject_alloc(int32_t kind, int64_t nth);
/* While enabled, long reads' multi-pass sweeps (whose warps wait for one
 * another's progress, each wait bounded) run with progress publication off
 * and a short wait limit: every wait runs out, the kernel records it and
 * returns, and the call fails with RODV_ERR_DEVICE_CHECK.  Tests the expiry
 * path with no hang and no fault; the device stays usable. */
rodv_status rodv_fault_inject_wait(int32_t enable);
void rodv_debug_live_allocations(uint64_t* device, uint64_t* pinned_host);
/* The chain items the packer makes of one region's reads, on the host only
 * (no device call; for tests of the placement rules).  Reads 0..num_reads-1
 * have read_lengths[r] bases and uniform[r] != 0 when their gap priors are
 * uniform (constant ins/del/gcp, ins == del, as the packer decides from the
 * qualities); items_per_warp[R - 1] (R = 1..8) is 1, or 2 for the
 * lane-grouped variant of the uniform class of R rows per lane; stack != 0
 * lets uniform reads stack (every batch call does).  out receives
 * [items, leftover read or 0xFFFFFFFF], then per item [class, pairs, then
 * x read and y read (or 0xFFFFFFFF) of each pair]; *words_written is set
 * even when out_words is too small (RODV_ERR_INVALID_ARG then).  Multi-pass
 * reads are not placed in chain items and appear nowhere. */
rodv_status rodv_debug_chain_plan(const uint32_t* read_lengths, const uint8_t* uniform,
                                  uint32_t num_reads, const int32_t* items_per_warp,
                                  int32_t stack, uint32_t* out, uint32_t out_words,
                                  uint32_t* words_written);

/* Human-readable name of a status code (static storage). */
const char* rodv_status_string(rodv_status status);

/* Details of the last failure on this engine (static until the next call);
 * with engine == NULL, of the last failed rodv_engine_create. */
const char* rodv_last_error(rodv_engine* engine);

#ifdef __cplusplus
}
#endif

#endif /* RODV_PAIRHMM_H_ */

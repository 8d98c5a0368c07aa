// schedule_shim.cpp -- pairhmm::schedule::schedule_pairhmm on the B200 engine.
//
// Same symbol and signature as roDV's src/core/pairhmm_schedule.h:14-25; see
// include/rodv_pairhmm_schedule.h for the semantics kept and changed.  The
// region is flattened into one rodv_batch and computed by a process-wide
// engine on the current CUDA device (created on first use; the environment
// variable RODV_DEVICE overrides the device).
#include "../../include/rodv_pairhmm_schedule.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "../../include/rodv_pairhmm.h"

namespace {

rodv_engine* shared_engine(rodv_status* status) {
  static std::once_flag once;
  static rodv_engine* engine = nullptr;
  static rodv_status st = RODV_OK;
  std::call_once(once, [] {
    rodv_options o;
    rodv_default_options(&o);
    int dev = 0;
    if (const char* env = std::getenv("RODV_DEVICE")) dev = std::atoi(env);
    else if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    o.device = dev;
    st = rodv_engine_create(&o, &engine);
  });
  *status = st;
  return engine;
}

}  // namespace

namespace pairhmm {
namespace schedule {

bool schedule_pairhmm(const std::vector<std::vector<uint8_t>>& haplotypes,
                      const std::vector<std::vector<uint8_t>>& reads,
                      std::vector<std::vector<double>>& result,
                      const std::vector<std::vector<uint8_t>>& quality,
                      const std::vector<std::vector<uint8_t>>& insertion_qualities,
                      const std::vector<std::vector<uint8_t>>& deletion_qualities,
                      const std::vector<std::vector<uint8_t>>& gap_contiguous_qualities,
                      bool use_double, double /*max_idle_ratio_float*/,
                      double /*max_idle_ratio_double*/, bool verbose) {
  const size_t M = haplotypes.size(), N = reads.size();
  if (M == 0 || N == 0) return false;
  result.resize(M);
  for (auto& row : result) row.assign(N, 0.0);
  if (quality.size() < N || insertion_qualities.size() < N || deletion_qualities.size() < N ||
      gap_contiguous_qualities.size() < N)
    return false;

  std::vector<uint8_t> hap_bases, read_bases, q, ins, del, gcp;
  std::vector<uint64_t> hap_off(M), read_off(N);
  std::vector<uint32_t> hap_len(M), read_len(N);
  for (size_t h = 0; h < M; ++h) {
    hap_off[h] = hap_bases.size();
    hap_len[h] = (uint32_t)haplotypes[h].size();
    hap_bases.insert(hap_bases.end(), haplotypes[h].begin(), haplotypes[h].end());
  }
  for (size_t r = 0; r < N; ++r) {
    const size_t n = reads[r].size();
    if (quality[r].size() != n || insertion_qualities[r].size() != n ||
        deletion_qualities[r].size() != n || gap_contiguous_qualities[r].size() != n)
      return false;
    read_off[r] = read_bases.size();
    read_len[r] = (uint32_t)n;
    read_bases.insert(read_bases.end(), reads[r].begin(), reads[r].end());
    q.insert(q.end(), quality[r].begin(), quality[r].end());
    ins.insert(ins.end(), insertion_qualities[r].begin(), insertion_qualities[r].end());
    del.insert(del.end(), deletion_qualities[r].begin(), deletion_qualities[r].end());
    gcp.insert(gcp.end(), gap_contiguous_qualities[r].begin(),
               gap_contiguous_qualities[r].end());
  }
  rodv_region region{0, (uint32_t)M, 0, (uint32_t)N};
  rodv_batch b{};
  b.num_regions = 1;
  b.regions = &region;
  b.num_haps = (uint32_t)M;
  b.hap_bases = hap_bases.data();
  b.hap_offsets = hap_off.data();
  b.hap_lengths = hap_len.data();
  b.num_reads = (uint32_t)N;
  b.read_bases = read_bases.data();
  b.base_quals = q.data();
  b.ins_quals = ins.data();
  b.del_quals = del.data();
  b.gcp_quals = gcp.data();
  b.read_offsets = read_off.data();
  b.read_lengths = read_len.data();

  rodv_status st = RODV_OK;
  rodv_engine* engine = shared_engine(&st);
  if (!engine) {
    if (verbose) std::fprintf(stderr, "schedule_pairhmm: %s\n", rodv_status_string(st));
    return false;
  }
  std::vector<double> flat(M * N);
  rodv_stats stats;
  st = rodv_pairhmm_batch(engine, &b, use_double ? 1 : 0, flat.data(), &stats);
  if (st != RODV_OK) {
    if (verbose)
      std::fprintf(stderr, "schedule_pairhmm: %s (%s)\n", rodv_status_string(st),
                   rodv_last_error(engine));
    return false;
  }
  for (size_t h = 0; h < M; ++h)
    for (size_t r = 0; r < N; ++r) result[h][r] = flat[h * N + r];
  if (verbose)
    std::fprintf(stderr, "schedule_pairhmm: %llu pairs, %llu cells, %llu in FP64, %.3f ms\n",
                 (unsigned long long)stats.pairs, (unsigned long long)stats.cells,
                 (unsigned long long)stats.fp64_pairs, stats.total_ms);
  return true;
}

}  // namespace schedule
}  // namespace pairhmm

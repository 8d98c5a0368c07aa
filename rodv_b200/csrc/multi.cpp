// multi.cpp -- one batch over several GPUs: region sharding, per-device
// engines on their own host threads, results merged back into batch order.
//
// roDV computes one schedule_pairhmm call per region on one thread
// (src/core/pairhmm_schedule.cpp:116-340); regions are independent, so the
// B200 engine splits a batch by regions: no pair's arithmetic depends on
// another region, and no data moves between GPUs.  Each device runs a full
// engine (its own streams, arenas and host lanes) on the regions of its
// shard; the shards' results are scattered back to the batch's result order.
// There is no collective and no peer memory access on this path.
//
// Sharding is longest-processing-time first by cells (sum of haplotype
// lengths x sum of read lengths per region): regions in decreasing cell
// count, each to the shard with the fewest cells so far (lowest index on a
// tie).  The plan depends only on the batch and the shard count, so every
// process of a multi-process job computes the same plan.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"

namespace rodv {
namespace {

uint64_t region_cells(const rodv_batch& b, uint32_t g) {
  const rodv_region& rg = b.regions[g];
  uint64_t hs = 0, rs = 0;
  for (uint32_t h = 0; h < rg.num_haps; ++h) hs += b.hap_lengths[rg.hap_start + h];
  for (uint32_t r = 0; r < rg.num_reads; ++r) rs += b.read_lengths[rg.read_start + r];
  return hs * rs;
}

// Region indices must stay inside the batch's arrays before any of them is
// followed (the cell count reads lengths through them).
rodv_status check_regions(const rodv_batch& b) {
  if (!b.regions || !b.hap_lengths || !b.read_lengths) return RODV_ERR_INVALID_ARG;
  if (b.num_regions == 0) return RODV_ERR_EMPTY;
  for (uint32_t g = 0; g < b.num_regions; ++g) {
    const rodv_region& rg = b.regions[g];
    if (rg.num_haps == 0 || rg.num_reads == 0) return RODV_ERR_EMPTY;
    if ((uint64_t)rg.hap_start + rg.num_haps > b.num_haps ||
        (uint64_t)rg.read_start + rg.num_reads > b.num_reads)
      return RODV_ERR_INVALID_ARG;
  }
  return RODV_OK;
}

}  // namespace

rodv_status shard_plan(const rodv_batch& b, uint32_t num_shards, uint32_t* region_shard,
                       uint64_t* shard_cells) {
  if (num_shards == 0 || !region_shard) return RODV_ERR_INVALID_ARG;
  const rodv_status s = check_regions(b);
  if (s != RODV_OK) return s;
  const uint32_t G = b.num_regions;
  std::vector<uint64_t> cells(G);
  for (uint32_t g = 0; g < G; ++g) cells[g] = region_cells(b, g);
  std::vector<uint32_t> order(G);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t x, uint32_t y) { return cells[x] > cells[y]; });
  std::vector<uint64_t> load(num_shards, 0);
  for (uint32_t g : order) {
    uint32_t best = 0;
    for (uint32_t k = 1; k < num_shards; ++k)
      if (load[k] < load[best]) best = k;
    region_shard[g] = best;
    load[best] += cells[g];
  }
  if (shard_cells)
    for (uint32_t k = 0; k < num_shards; ++k) shard_cells[k] = load[k];
  return RODV_OK;
}

// The sub-batch of one shard: its regions in batch order, over compacted
// offset and length arrays that point into the batch's own base and quality
// buffers (no base or quality byte is copied).
struct SubBatch {
  std::vector<rodv_region> regions;
  std::vector<uint64_t> hap_offsets, read_offsets;
  std::vector<uint32_t> hap_lengths, read_lengths;
  std::vector<uint32_t> members;  // batch region index of each sub-batch region
  rodv_batch view{};
  uint64_t pairs = 0;
};

void make_sub_batch(const rodv_batch& b, const uint32_t* region_shard, uint32_t shard,
                    SubBatch& sb) {
  for (uint32_t g = 0; g < b.num_regions; ++g) {
    if (region_shard[g] != shard) continue;
    const rodv_region& rg = b.regions[g];
    rodv_region r{(uint32_t)sb.hap_lengths.size(), rg.num_haps, (uint32_t)sb.read_lengths.size(),
                  rg.num_reads};
    for (uint32_t h = 0; h < rg.num_haps; ++h) {
      sb.hap_offsets.push_back(b.hap_offsets[rg.hap_start + h]);
      sb.hap_lengths.push_back(b.hap_lengths[rg.hap_start + h]);
    }
    for (uint32_t k = 0; k < rg.num_reads; ++k) {
      sb.read_offsets.push_back(b.read_offsets[rg.read_start + k]);
      sb.read_lengths.push_back(b.read_lengths[rg.read_start + k]);
    }
    sb.regions.push_back(r);
    sb.members.push_back(g);
    sb.pairs += (uint64_t)rg.num_haps * rg.num_reads;
  }
  rodv_batch& v = sb.view;
  v = b;
  v.num_regions = (uint32_t)sb.regions.size();
  v.regions = sb.regions.data();
  v.num_haps = (uint32_t)sb.hap_lengths.size();
  v.hap_offsets = sb.hap_offsets.data();
  v.hap_lengths = sb.hap_lengths.data();
  v.num_reads = (uint32_t)sb.read_lengths.size();
  v.read_offsets = sb.read_offsets.data();
  v.read_lengths = sb.read_lengths.data();
}

rodv_status shard_merge(const rodv_batch& b, uint32_t num_shards, const uint32_t* region_shard,
                        const double* const* shard_results, double* out) {
  if (num_shards == 0 || !region_shard || !shard_results || !out) return RODV_ERR_INVALID_ARG;
  const rodv_status s = check_regions(b);
  if (s != RODV_OK) return s;
  std::vector<uint64_t> pos(num_shards, 0);  // next result of each shard
  uint64_t o = 0;
  for (uint32_t g = 0; g < b.num_regions; ++g) {
    const uint32_t k = region_shard[g];
    if (k >= num_shards || !shard_results[k]) return RODV_ERR_INVALID_ARG;
    const uint64_t n = (uint64_t)b.regions[g].num_haps * b.regions[g].num_reads;
    std::memcpy(out + o, shard_results[k] + pos[k], n * sizeof(double));
    pos[k] += n;
    o += n;
  }
  return RODV_OK;
}

}  // namespace rodv

// One engine per device, each driven by its own host thread during a call.
struct rodv_multi {
  std::vector<std::unique_ptr<rodv::Engine>> engines;
  std::mutex mu;
  std::string last_error;
};

extern "C" {

rodv_status rodv_shard_plan(const rodv_batch* batch, uint32_t num_shards, uint32_t* region_shard,
                            uint64_t* shard_cells) {
  if (!batch) return RODV_ERR_INVALID_ARG;
  return rodv::shard_plan(*batch, num_shards, region_shard, shard_cells);
}

rodv_status rodv_shard_merge(const rodv_batch* batch, uint32_t num_shards,
                             const uint32_t* region_shard, const double* const* shard_results,
                             double* out_log10) {
  if (!batch) return RODV_ERR_INVALID_ARG;
  return rodv::shard_merge(*batch, num_shards, region_shard, shard_results, out_log10);
}

rodv_status rodv_multi_create(const rodv_options* opts, const int32_t* devices,
                              uint32_t num_devices, rodv_multi** out) {
  if (!out || !devices || num_devices == 0) return RODV_ERR_INVALID_ARG;
  *out = nullptr;
  std::unique_ptr<rodv_multi> m(new (std::nothrow) rodv_multi());
  if (!m) return RODV_ERR_OUT_OF_MEMORY;
  for (uint32_t k = 0; k < num_devices; ++k) {
    rodv_options o;
    rodv_default_options(&o);
    if (opts) o = *opts;
    o.device = devices[k];
    std::unique_ptr<rodv::Engine> e(new (std::nothrow) rodv::Engine(o));
    if (!e) return RODV_ERR_OUT_OF_MEMORY;
    const rodv_status s = e->init();
    if (s != RODV_OK) {
      rodv::set_create_error("device " + std::to_string(devices[k]) + ": " + e->last_error());
      return s;
    }
    m->engines.push_back(std::move(e));
  }
  *out = m.release();
  return RODV_OK;
}

void rodv_multi_destroy(rodv_multi* multi) { delete multi; }

rodv_status rodv_multi_batch(rodv_multi* multi, const rodv_batch* batch, int32_t use_double,
                             double* out_log10, rodv_stats* stats) {
  using namespace rodv;
  if (!multi || !batch || !out_log10) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(multi->mu);
  const auto t0 = std::chrono::steady_clock::now();
  if (stats) std::memset(stats, 0, sizeof(*stats));
  const uint32_t n = (uint32_t)multi->engines.size();
  std::vector<uint32_t> region_shard(batch->num_regions);
  rodv_status s = shard_plan(*batch, n, region_shard.data(), nullptr);
  if (s != RODV_OK) {
    multi->last_error = "shard plan: invalid batch";
    return s;
  }
  std::vector<SubBatch> subs(n);
  for (uint32_t k = 0; k < n; ++k) make_sub_batch(*batch, region_shard.data(), k, subs[k]);
  std::vector<std::vector<double>> results(n);
  std::vector<rodv_stats> st(n);
  std::vector<rodv_status> status(n, RODV_OK);
  std::vector<std::thread> threads;
  for (uint32_t k = 0; k < n; ++k) {
    if (subs[k].regions.empty()) continue;
    threads.emplace_back([&, k] {
      try {
        results[k].resize(subs[k].pairs);
      } catch (const std::bad_alloc&) {
        status[k] = RODV_ERR_OUT_OF_MEMORY;
        return;
      }
      std::memset(&st[k], 0, sizeof(st[k]));
      Engine& e = *multi->engines[k];
      std::lock_guard<std::mutex> elk(e.mutex());
      status[k] = e.run_host(subs[k].view, results[k].data(), &st[k], use_double != 0);
    });
  }
  for (std::thread& t : threads) t.join();
  for (uint32_t k = 0; k < n; ++k) {
    if (status[k] != RODV_OK) {
      multi->last_error = "device " + std::to_string(k) + ": " + multi->engines[k]->last_error();
      return status[k];
    }
  }
  std::vector<const double*> ptrs(n);
  for (uint32_t k = 0; k < n; ++k) ptrs[k] = results[k].data();
  s = shard_merge(*batch, n, region_shard.data(), ptrs.data(), out_log10);
  if (s != RODV_OK) return s;
  if (stats) {
    for (uint32_t k = 0; k < n; ++k) {
      stats->pairs += st[k].pairs;
      stats->cells += st[k].cells;
      stats->fp64_pairs += st[k].fp64_pairs;
      stats->fp64_cells += st[k].fp64_cells;
      stats->kernel_launches += st[k].kernel_launches;
      stats->device_ms = std::max(stats->device_ms, st[k].device_ms);
      stats->fp32_ms = std::max(stats->fp32_ms, st[k].fp32_ms);
      stats->h2d_ms = std::max(stats->h2d_ms, st[k].h2d_ms);
      stats->d2h_ms = std::max(stats->d2h_ms, st[k].d2h_ms);
      stats->h2d_bytes += st[k].h2d_bytes;
      stats->d2h_bytes += st[k].d2h_bytes;
    }
    stats->total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  return RODV_OK;
}

const char* rodv_multi_last_error(rodv_multi* multi) {
  return multi ? multi->last_error.c_str() : "";
}

}  // extern "C"

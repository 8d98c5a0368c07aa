// capi.cpp -- extern "C" entry points of include/rodv_pairhmm.h.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "chain_plan.h"
#include "engine.h"
#include "service.h"

using rodv::Engine;
using rodv::Service;

static_assert(RODV_TUNE_CLASSES == rodv::kNumClasses, "tuning classes out of sync");

extern "C" {

void rodv_default_options(rodv_options* opts) {
  if (!opts) return;
  std::memset(opts, 0, sizeof(*opts));
  opts->device = 0;
  opts->force_fp64 = 0;
  opts->device_memory_budget = 0;
  opts->max_inflight = 0;
  opts->verbose = 0;
  opts->autotune = 0;
  opts->tune_cache = nullptr;
}

// Message of the last failed rodv_engine_create (rodv_last_error(NULL)).
static std::mutex g_create_mu;
static std::string g_create_error;

}  // extern "C"

namespace rodv {
void set_create_error(const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_create_mu);
  g_create_error = msg;
}
}  // namespace rodv

extern "C" {

rodv_status rodv_engine_create(const rodv_options* opts, rodv_engine** out) {
  if (!out) return RODV_ERR_INVALID_ARG;
  *out = nullptr;
  rodv_options o;
  rodv_default_options(&o);
  if (opts) o = *opts;
  Engine* e = new (std::nothrow) Engine(o);
  if (!e) return RODV_ERR_OUT_OF_MEMORY;
  rodv_status s = e->init();
  if (s != RODV_OK) {
    {
      std::lock_guard<std::mutex> lk(g_create_mu);
      g_create_error = e->last_error();
    }
    delete e;
    return s;
  }
  *out = new (std::nothrow) rodv_engine{e};
  if (!*out) {
    delete e;
    return RODV_ERR_OUT_OF_MEMORY;
  }
  return RODV_OK;
}

void rodv_engine_destroy(rodv_engine* engine) {
  if (!engine) return;
  delete engine->impl;
  delete engine;
}

uint64_t rodv_batch_num_pairs(const rodv_batch* b) {
  if (!b || !b->regions) return 0;
  uint64_t n = 0;
  for (uint32_t g = 0; g < b->num_regions; ++g)
    n += (uint64_t)b->regions[g].num_haps * b->regions[g].num_reads;
  return n;
}

rodv_status rodv_batch_validate(const rodv_batch* b, char* msg, size_t msg_len) {
  if (msg && msg_len) msg[0] = '\0';
  if (!b) {
    if (msg && msg_len) snprintf(msg, msg_len, "%s", "null batch");
    return RODV_ERR_INVALID_ARG;
  }
  std::string m;
  const rodv_status s = rodv::validate_batch(*b, /*check_bases=*/true, nullptr, &m);
  if (msg && msg_len && s != RODV_OK) snprintf(msg, msg_len, "%s", m.c_str());
  return s;
}

rodv_status rodv_pairhmm_batch(rodv_engine* engine, const rodv_batch* batch, int32_t use_double,
                               double* out, rodv_stats* stats) {
  if (!engine || !batch) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  if (stats) std::memset(stats, 0, sizeof(*stats));
  return engine->impl->run_host(*batch, out, stats, use_double != 0);
}

rodv_status rodv_pairhmm_batch_raw(rodv_engine* engine, const rodv_batch* batch,
                                   int32_t use_double, double* out_raw, uint8_t* out_precision,
                                   rodv_stats* stats) {
  if (!engine || !batch || !out_raw || !out_precision) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  if (stats) std::memset(stats, 0, sizeof(*stats));
  return engine->impl->run_host(*batch, out_raw, stats, use_double != 0, out_precision);
}

rodv_status rodv_pairhmm_pair(rodv_engine* engine, const uint8_t* hap, uint32_t hap_len,
                              const uint8_t* read, const uint8_t* q, const uint8_t* ins,
                              const uint8_t* del, const uint8_t* gcp, uint32_t read_len,
                              int32_t use_double, double* out) {
  if (!engine || !hap || !read || !q || !ins || !del || !gcp || !out)
    return RODV_ERR_INVALID_ARG;
  if (read_len == 0 || hap_len == 0) return RODV_ERR_INVALID_ARG;
  // One region, one haplotype, one read; the read's four quality arrays
  // are separate buffers, so the batch's shared read_offsets is 0 for each.
  rodv_region rg{0, 1, 0, 1};
  const uint64_t zero = 0;
  rodv_batch b{};
  b.num_regions = 1;
  b.regions = &rg;
  b.num_haps = 1;
  b.hap_bases = hap;
  b.hap_offsets = &zero;
  b.hap_lengths = &hap_len;
  b.num_reads = 1;
  b.read_bases = read;
  b.base_quals = q;
  b.ins_quals = ins;
  b.del_quals = del;
  b.gcp_quals = gcp;
  b.read_offsets = &zero;
  b.read_lengths = &read_len;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  return engine->impl->run_host(b, out, nullptr, use_double != 0);
}

rodv_status rodv_device_batch_upload(rodv_engine* engine, const rodv_batch* batch,
                                     rodv_device_batch** out) {
  if (!engine || !batch || !out) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  return engine->impl->upload(*batch, out);
}

rodv_status rodv_device_batch_run(rodv_engine* engine, rodv_device_batch* db, rodv_stats* stats) {
  if (!engine || !db) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  if (stats) std::memset(stats, 0, sizeof(*stats));
  return engine->impl->run_device(db, stats);
}

rodv_status rodv_device_batch_download(rodv_engine* engine, rodv_device_batch* db, double* out) {
  if (!engine || !db || !out) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  return engine->impl->download(db, out);
}

void rodv_device_batch_free(rodv_engine* engine, rodv_device_batch* db) {
  if (!db) return;
  if (engine) {
    std::lock_guard<std::mutex> lk(engine->impl->mutex());
    delete db;
  } else {
    delete db;
  }
}

rodv_status rodv_pairhmm_plain(rodv_engine* engine, rodv_device_batch* db, double* out,
                               rodv_stats* stats) {
  if (!engine || !db) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  if (stats) std::memset(stats, 0, sizeof(*stats));
  return engine->impl->plain(db, out, stats);
}

rodv_status rodv_measure_peaks(rodv_engine* engine, double* f32, double* f32x2, double* f64,
                               double* mhz) {
  if (!engine) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  return engine->impl->measure_peaks(f32, f32x2, f64, mhz);
}

rodv_status rodv_autotune(rodv_engine* engine, const char* cache_path, int32_t force,
                          int32_t* variants_out) {
  if (!engine) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  return engine->impl->autotune(cache_path, force, variants_out);
}

rodv_status rodv_tuned_variants(rodv_engine* engine, int32_t* fp32, int32_t* fp64) {
  if (!engine) return RODV_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(engine->impl->mutex());
  engine->impl->variants(fp32, fp64);
  return RODV_OK;
}

const char* rodv_status_string(rodv_status s) {
  switch (s) {
    case RODV_OK: return "ok";
    case RODV_ERR_INVALID_ARG: return "invalid argument";
    case RODV_ERR_EMPTY: return "region without haplotypes or reads";
    case RODV_ERR_INVALID_BASE: return "base outside A, C, G, T, N";
    case RODV_ERR_NO_DEVICE: return "no usable CUDA device";
    case RODV_ERR_CUDA: return "CUDA runtime error";
    case RODV_ERR_OUT_OF_MEMORY: return "out of memory";
    case RODV_ERR_TOO_LONG: return "input above engine limits";
    case RODV_ERR_DEVICE_CHECK: return "device-side check failed";
    case RODV_ERR_ADMISSION: return "region does not fit the device memory budget";
    case RODV_ERR_NOT_FOUND: return "unknown ticket";
    case RODV_ERR_NOT_READY: return "result not ready";
    case RODV_ERR_SHUTDOWN: return "service stopped";
    case RODV_ERR_INTERNAL: return "internal consistency check failed";
    default: return "unknown status";
  }
}

rodv_status rodv_fault_inject_alloc(int32_t kind, int64_t nth) {
  if (kind != 0 && kind != 1) return RODV_ERR_INVALID_ARG;
  rodv::set_alloc_fault(kind, nth);
  return RODV_OK;
}

rodv_status rodv_fault_inject_wait(int32_t enable) {
  rodv::set_wait_fault(enable != 0);
  return RODV_OK;
}

void rodv_debug_live_allocations(uint64_t* device, uint64_t* pinned_host) {
  rodv::live_allocations(device, pinned_host);
}

rodv_status rodv_debug_chain_plan(const uint32_t* read_lengths, const uint8_t* uniform,
                                  uint32_t num_reads, const int32_t* items_per_warp,
                                  int32_t stack, uint32_t* out, uint32_t out_words,
                                  uint32_t* words_written) {
  if (words_written) *words_written = 0;
  if ((num_reads && (!read_lengths || !uniform)) || !items_per_warp || !words_written ||
      (out_words && !out))
    return RODV_ERR_INVALID_ARG;
  std::vector<uint8_t> cls(num_reads);
  for (uint32_t r = 0; r < num_reads; ++r) {
    if (read_lengths[r] == 0 || read_lengths[r] > RODV_MAX_READ_LEN) return RODV_ERR_INVALID_ARG;
    cls[r] = (uint8_t)rodv::class_of(read_lengths[r], uniform[r] != 0);
  }
  int ipw[rodv::kMaxRowsPerLane + 1] = {};
  for (int R = 1; R <= rodv::kMaxRowsPerLane; ++R) {
    if (items_per_warp[R - 1] != 1 && items_per_warp[R - 1] != 2) return RODV_ERR_INVALID_ARG;
    ipw[R] = items_per_warp[R - 1];
  }
  rodv::ChainGeom geom[rodv::kMaxRowsPerLane + 1];
  rodv::chain_geometry(ipw, geom);
  std::vector<uint32_t> sr;
  rodv::sort_single_pass(read_lengths, cls.data(), 0, num_reads, sr);
  rodv::RegionChains rc;
  rodv::plan_region_chains(read_lengths, cls.data(), geom, stack != 0, sr, rc);
  std::vector<uint32_t> words{(uint32_t)rc.items.size(), rc.leftover};
  for (const rodv::ChainPairs& it : rc.items) {
    words.push_back((uint32_t)it.cls);
    words.push_back(it.pairs);
    for (uint32_t j = 0; j < 2 * it.pairs; ++j) words.push_back(rc.reads[it.first + j]);
  }
  *words_written = (uint32_t)words.size();
  if (words.size() > out_words) return RODV_ERR_INVALID_ARG;
  std::memcpy(out, words.data(), words.size() * 4);
  return RODV_OK;
}

const char* rodv_last_error(rodv_engine* engine) {
  if (!engine) {
    std::lock_guard<std::mutex> lk(g_create_mu);
    return g_create_error.c_str();
  }
  return engine->impl->last_error();
}

// ---- streaming service ----------------------------------------------------
rodv_status rodv_service_create(const rodv_options* opts, rodv_service** out) {
  if (!out) return RODV_ERR_INVALID_ARG;
  *out = nullptr;
  rodv_options o;
  rodv_default_options(&o);
  if (opts) o = *opts;
  Service* sv = new (std::nothrow) Service(o);
  if (!sv) return RODV_ERR_OUT_OF_MEMORY;
  const rodv_status s = sv->init();
  if (s != RODV_OK) {
    {
      std::lock_guard<std::mutex> lk(g_create_mu);
      g_create_error = sv->last_error();
    }
    delete sv;
    return s;
  }
  *out = new (std::nothrow) rodv_service{sv};
  if (!*out) {
    delete sv;
    return RODV_ERR_OUT_OF_MEMORY;
  }
  return RODV_OK;
}

void rodv_service_destroy(rodv_service* service) {
  if (!service) return;
  delete service->impl;
  delete service;
}

rodv_status rodv_submit_region(rodv_service* service, const rodv_batch* regions,
                               uint64_t* ticket) {
  if (!service || !regions || !ticket) return RODV_ERR_INVALID_ARG;
  return service->impl->submit(*regions, ticket);
}

rodv_status rodv_poll(rodv_service* service, uint64_t ticket, double* out_log10,
                      rodv_request_stats* stats) {
  if (!service) return RODV_ERR_INVALID_ARG;
  return service->impl->result(ticket, 0, out_log10, stats);
}

rodv_status rodv_wait(rodv_service* service, uint64_t ticket, int32_t timeout_ms,
                      double* out_log10, rodv_request_stats* stats) {
  if (!service) return RODV_ERR_INVALID_ARG;
  return service->impl->result(ticket, timeout_ms, out_log10, stats);
}

rodv_status rodv_service_get_stats(rodv_service* service, rodv_service_stats* out) {
  if (!service) return RODV_ERR_INVALID_ARG;
  return service->impl->stats(out);
}

void rodv_service_reset_stats(rodv_service* service) {
  if (service) service->impl->reset_stats();
}

const char* rodv_service_last_error(rodv_service* service) {
  static thread_local std::string msg;
  msg = service ? service->impl->last_error() : std::string();
  return msg.c_str();
}

}  // extern "C"

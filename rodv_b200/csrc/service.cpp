// service.cpp -- streaming PairHMM service: continuous batching of submitted
// regions over three device batch slots (see service.h).
#include "service.h"
#include "trace.h"
#include "worker_pool.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace rodv {

namespace {

constexpr uint64_t kMaxBatchPairs = 1ull << 31;
// A batch holds up to this many estimated device bytes (~600 regions of
// 1-32 haplotypes x 1-300 reads; tens of ms of GPU work), unless one request
// alone is larger.  Each slot's buffers are reserved for it at creation, so
// steady-state batches never reallocate (a pinned or device reallocation
// synchronises the device and costs far more than packing a batch).
constexpr uint64_t kBatchBytes = 128ull << 20;

// Grows a buffer to at least n bytes, at least doubling it.
template <class Mem>
cudaError_t grow(Mem& m, size_t n) {
  if (m.ptr && m.bytes >= n) return cudaSuccess;
  return m.ensure(std::max(n + n / 4, 2 * m.bytes));
}

double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

Service::Service(const rodv_options& opt) : opt_(opt), engine_(opt) {}

Service::~Service() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  if (ring_) ring_->stop();
  cv_work_.notify_all();
  cv_space_.notify_all();
  cv_done_.notify_all();
  if (thread_.joinable()) thread_.join();  // the worker finishes all submitted work first
  if (ready_) {
    for (Slot& s : slots_) {
      for (cudaEvent_t e : s.ev)
        if (e) cudaEventDestroy(e);
      if (s.done) cudaEventDestroy(s.done);
      if (s.stream) cudaStreamDestroy(s.stream);
    }
  }
}

rodv_status Service::init() {
  rodv_status st = engine_.init();
  if (st != RODV_OK) {
    err_ = engine_.last_error();
    return st;
  }
  // A kernel's first launch would otherwise load it in the middle of a batch
  // (a stall of milliseconds for every request of that batch and the ones
  // queued behind it).
  st = engine_.load_kernels();
  if (st != RODV_OK) {
    err_ = engine_.last_error();
    return st;
  }
  ready_ = true;  // streams and events created below are released by the destructor
  cudaError_t e = cudaSetDevice(engine_.device_);
  for (Slot& s : slots_) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
    for (cudaEvent_t& ev : s.ev)
      if (e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
  }
  size_t free_b = 0, total_b = 0;
  if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) {
    st = engine_.cuda_fail(e, "service setup");
    err_ = engine_.last_error();
    return st;
  }
  const uint64_t budget = opt_.device_memory_budget ? opt_.device_memory_budget : free_b / 2;
  slot_budget_ = budget / kSlots;
  batch_bytes_ = std::min<uint64_t>(slot_budget_, kBatchBytes);
  max_inflight_ = opt_.max_inflight ? opt_.max_inflight : 4096;
  // Each of the ring's five arrays holds about a batch's bases (a batch's
  // device estimate counts 4 bytes per read base); requests above half of it
  // keep their own copy.
  ring_.reset(new HostRing(std::max<uint64_t>(batch_bytes_, 1ull << 20)));
  // Touched once now, so that no request's copy takes the ring's first-use
  // page faults.
  for (int k = 0; k < HostRing::kArrays; ++k) std::memset(ring_->array(k), 0, ring_->capacity());
  for (Slot& s : slots_) {
    // staging holds at most the estimate; results are 8 of its ~36 bytes per pair
    if (e == cudaSuccess) e = s.staging.ensure(batch_bytes_);
    if (e == cudaSuccess) e = s.arena.ensure(batch_bytes_);
    if (e == cudaSuccess) e = s.out_host.ensure(batch_bytes_ / 4 + kCountWords * 4);
  }
  if (e != cudaSuccess) {
    st = engine_.cuda_fail(e, "service buffers");
    err_ = engine_.last_error();
    return st;
  }
  thread_ = std::thread([this] { worker(); });
  return RODV_OK;
}

// Upper bound of the device bytes one request adds to a batch (the packed
// layout of engine.cu: codes, row words, descriptors, work items, FP64
// lists, results, alignment, and the multi-pass boundary scratch when a read
// needs more than one pass).
uint64_t Service::estimate_bytes(const rodv_batch& b, uint64_t pairs) const {
  uint64_t bytes = 4096 + 3 * kNumClasses * 256;
  uint32_t max_h = 0;
  bool multi = false;
  for (uint32_t h = 0; h < b.num_haps; ++h) {
    bytes += b.hap_lengths[h] + 1;
    max_h = std::max(max_h, b.hap_lengths[h]);
  }
  bytes += 3 * kHapPad + max_h;
  for (uint32_t r = 0; r < b.num_reads; ++r) {
    bytes += (uint64_t)((b.read_lengths[r] + 3) & ~3u) * 4;
    multi = multi || b.read_lengths[r] + 2 > (uint32_t)kPassRows;  // class_of, either form
  }
  bytes += (uint64_t)(b.num_haps + b.num_reads) * 16;
  bytes += pairs * (16 + 12 + 8);
  // boundary scratch: 24 bytes per column per boundary row of the multi-pass
  // kernels, one region per multi-pass class
  if (multi) bytes += 2 * (uint64_t)engine_.multi_scratch_rows() * (max_h + 40) * 24 + 512;
  return bytes;
}

rodv_status Service::submit(const rodv_batch& b, uint64_t* ticket) {
  if (!ticket) return RODV_ERR_INVALID_ARG;
  uint64_t pairs = 0;
  std::string msg;
  const rodv_status st = validate_batch(b, true, &pairs, &msg);
  auto refuse = [&](rodv_status s, const std::string& m) {
    std::lock_guard<std::mutex> lk(mu_);
    err_ = m;
    return s;
  };
  if (st != RODV_OK) return refuse(st, msg);
  auto r = std::make_shared<Request>();
  r->pairs = pairs;
  r->bytes = estimate_bytes(b, pairs);
  if (r->bytes > slot_budget_ || pairs >= kMaxBatchPairs)
    return refuse(RODV_ERR_ADMISSION, "request needs ~" + std::to_string(r->bytes) +
                                          " device bytes; a batch slot holds " +
                                          std::to_string(slot_budget_));
  // Copy of the bases and qualities: into the ring when the request fits in
  // half of it (haplotypes, then reads, at the same position in every
  // array), else into the request's own arrays.
  uint64_t hb = 0, rb = 0;
  for (uint32_t h = 0; h < b.num_haps; ++h) hb += b.hap_lengths[h];
  for (uint32_t k = 0; k < b.num_reads; ++k) rb += b.read_lengths[k];
  r->hap_bytes = hb;
  r->read_bytes = rb;
  r->hap_off.resize(b.num_haps);
  r->hap_len.assign(b.hap_lengths, b.hap_lengths + b.num_haps);
  r->read_off.resize(b.num_reads);
  r->read_len.assign(b.read_lengths, b.read_lengths + b.num_reads);
  uint8_t* hap_dst;
  uint8_t* read_dst[HostRing::kArrays];
  uint64_t hap_base = 0, read_base = 0;  // offsets of the copies in their arrays
  if (hb + rb <= ring_->capacity() / 2) {
    const uint64_t pos = ring_->acquire(hb + rb);
    if (pos == HostRing::kNone) return RODV_ERR_SHUTDOWN;
    r->ring_pos = pos;
    hap_base = pos;
    read_base = pos + hb;
    hap_dst = ring_->array(0) + hap_base;
    for (int k = 0; k < HostRing::kArrays; ++k) read_dst[k] = ring_->array(k) + read_base;
  } else {
    r->hap_bases.resize(hb);
    r->read_bases.resize(rb);
    for (auto& q : r->quals) q.resize(rb);
    hap_dst = r->hap_bases.data();
    read_dst[0] = r->read_bases.data();
    for (int q = 0; q < 4; ++q) read_dst[q + 1] = r->quals[q].data();
  }
  for (uint64_t h = 0, o = 0; h < b.num_haps; ++h) {
    std::memcpy(hap_dst + o, b.hap_bases + b.hap_offsets[h], b.hap_lengths[h]);
    r->hap_off[h] = hap_base + o;
    o += b.hap_lengths[h];
  }
  const uint8_t* src[HostRing::kArrays] = {b.read_bases, b.base_quals, b.ins_quals, b.del_quals,
                                           b.gcp_quals};
  for (uint64_t k = 0, o = 0; k < b.num_reads; ++k) {
    const uint64_t off = b.read_offsets[k];
    const uint32_t n = b.read_lengths[k];
    for (int a = 0; a < HostRing::kArrays; ++a) std::memcpy(read_dst[a] + o, src[a] + off, n);
    r->read_off[k] = read_base + o;
    o += n;
  }
  r->regions.assign(b.regions, b.regions + b.num_regions);
  for (const rodv_region& rg : r->regions) {
    uint64_t hs = 0, rs = 0;
    for (uint32_t h = 0; h < rg.num_haps; ++h) hs += b.hap_lengths[rg.hap_start + h];
    for (uint32_t k = 0; k < rg.num_reads; ++k) rs += b.read_lengths[rg.read_start + k];
    r->cells += hs * rs;
  }
  {
    std::unique_lock<std::mutex> lk(mu_);
    cv_space_.wait(lk, [&] { return stop_ || inflight_ < max_inflight_; });
    if (stop_) {
      lk.unlock();
      if (r->ring_pos != HostRing::kNone) ring_->release(r->ring_pos);
      return RODV_ERR_SHUTDOWN;
    }
    r->ticket = next_ticket_++;
    r->submitted = Clock::now();
    if (!st_any_) {
      st_first_submit_ = r->submitted;
      st_any_ = true;
    }
    ++st_submitted_;
    ++inflight_;
    table_[r->ticket] = r;
    pending_.push_back(r);
    *ticket = r->ticket;
  }
  cv_work_.notify_one();
  return RODV_OK;
}

void Service::worker() {
  cudaSetDevice(engine_.device_);
  std::deque<int> busy;  // slots with a batch in flight, oldest first
  for (;;) {
    // Collect every batch that is done, in whatever order they finish (a
    // small batch launched after a large one often finishes first, and its
    // slot is then free for what queued meanwhile).
    for (auto it = busy.begin(); it != busy.end();) {
      if (cudaEventQuery(slots_[*it].done) != cudaErrorNotReady) {
        complete(slots_[*it]);
        it = busy.erase(it);
      } else {
        ++it;
      }
    }
    // A new batch is formed only once every batch in flight has started on
    // the GPU: at most one batch waits behind the running one, and what
    // arrives meanwhile goes into the next batch instead of one queued two
    // batches ahead.
    bool all_started = true;
    for (int i : busy)
      all_started = all_started && cudaEventQuery(slots_[i].ev[0]) != cudaErrorNotReady;
    const bool can_launch = busy.size() < (size_t)kSlots && all_started;
    int slot = -1;
    std::vector<std::shared_ptr<Request>> batch;
    {
      std::unique_lock<std::mutex> lk(mu_);
      if (busy.empty()) cv_work_.wait(lk, [&] { return stop_ || !pending_.empty(); });
      if (busy.empty() && pending_.empty() && stop_) break;
      if (can_launch && !pending_.empty()) {
        // everything queued, up to one batch's size, goes into the next batch
        for (int i = 0; i < kSlots && slot < 0; ++i)
          if (std::find(busy.begin(), busy.end(), i) == busy.end()) slot = i;
        uint64_t bytes = 0, pairs = 0;
        while (!pending_.empty()) {
          const std::shared_ptr<Request>& r = pending_.front();
          if (!batch.empty() &&
              (bytes + r->bytes > batch_bytes_ || pairs + r->pairs >= kMaxBatchPairs))
            break;
          bytes += r->bytes;
          pairs += r->pairs;
          batch.push_back(r);
          pending_.pop_front();
        }
      } else {
        // Batches in flight, and no launch due or nothing queued: look again
        // in 50 us, or as soon as something arrives while a launch is due.
        cv_work_.wait_for(lk, std::chrono::microseconds(50),
                          [&] { return can_launch && !pending_.empty(); });
        continue;
      }
    }
    Slot& s = slots_[slot];
    s.reqs = std::move(batch);
    s.batch_id = next_batch_++;
    const Clock::time_point t0 = Clock::now();
    const rodv_status st = launch(s);
    release_ring(s);  // packed into the slot's staging: the ring ranges are free
    {
      std::lock_guard<std::mutex> lk(mu_);
      st_launch_ms_ += ms_between(t0, Clock::now());
    }
    if (st != RODV_OK) {
      // the slot's stream may still hold part of the batch
      cudaStreamSynchronize(s.stream);
      fail_slot(s, st);
    } else {
      busy.push_back(slot);
    }
  }
}

rodv_status Service::launch(Slot& s) {
  TraceRange trace("rodv service: form and launch batch");
  const Clock::time_point t0 = Clock::now();
  // The combined batch: the requests' regions, haplotype and read tables
  // back to back in the slot's arrays (resized below; every element is
  // overwritten).  When every request's bases are in the ring (the usual
  // case), the batch's base and quality arrays are the ring's and its offsets
  // the requests' ring positions: no base is copied.  Otherwise the bases go
  // to the slot's arrays too.  Each request's part goes to offsets known in
  // advance, so the copies run on the worker pool.
  struct Off {
    uint64_t reg, hap, read, hb, rb;
  };
  std::vector<Off> offs(s.reqs.size() + 1);
  uint64_t est = 0;
  bool in_ring = true;
  for (size_t k = 0; k < s.reqs.size(); ++k) {
    const auto& r = s.reqs[k];
    r->started = t0;
    est += r->bytes;
    in_ring = in_ring && r->ring_pos != HostRing::kNone;
    offs[k + 1] = Off{offs[k].reg + r->regions.size(), offs[k].hap + r->hap_len.size(),
                      offs[k].read + r->read_len.size(), offs[k].hb + r->hap_bytes,
                      offs[k].rb + r->read_bytes};
  }
  const Off& tot = offs.back();
  s.regions.resize(tot.reg);
  if (!in_ring) {
    s.hap_bases.resize(tot.hb);
    s.read_bases.resize(tot.rb);
    for (auto& q : s.quals) q.resize(tot.rb);
  }
  s.hap_off.resize(tot.hap);
  s.read_off.resize(tot.read);
  s.hap_len.resize(tot.hap);
  s.read_len.resize(tot.read);
  const size_t grain = in_ring ? 64 : 1;
  parallel_for(s.reqs.size(), grain, [&](size_t lo, size_t hi) {
    for (size_t k = lo; k < hi; ++k) {
      const Request& r = *s.reqs[k];
      const Off& o = offs[k];
      for (size_t g = 0; g < r.regions.size(); ++g) {
        rodv_region rg = r.regions[g];
        rg.hap_start += (uint32_t)o.hap;
        rg.read_start += (uint32_t)o.read;
        s.regions[o.reg + g] = rg;
      }
      std::memcpy(s.hap_len.data() + o.hap, r.hap_len.data(), r.hap_len.size() * 4);
      std::memcpy(s.read_len.data() + o.read, r.read_len.data(), r.read_len.size() * 4);
      if (in_ring) {
        std::memcpy(s.hap_off.data() + o.hap, r.hap_off.data(), r.hap_off.size() * 8);
        std::memcpy(s.read_off.data() + o.read, r.read_off.data(), r.read_off.size() * 8);
        continue;
      }
      // the request's bases, wherever submit put them, to the slot's arrays
      const bool ring = r.ring_pos != HostRing::kNone;
      const uint64_t hap_base = ring ? r.ring_pos : 0, read_base = hap_base + (ring ? r.hap_bytes : 0);
      const uint8_t* hsrc = ring ? ring_->array(0) + hap_base : r.hap_bases.data();
      const uint8_t* rsrc[HostRing::kArrays] = {
          ring ? ring_->array(0) + read_base : r.read_bases.data(),
          ring ? ring_->array(1) + read_base : r.quals[0].data(),
          ring ? ring_->array(2) + read_base : r.quals[1].data(),
          ring ? ring_->array(3) + read_base : r.quals[2].data(),
          ring ? ring_->array(4) + read_base : r.quals[3].data()};
      uint8_t* rdst[HostRing::kArrays] = {s.read_bases.data(), s.quals[0].data(), s.quals[1].data(),
                                          s.quals[2].data(), s.quals[3].data()};
      std::memcpy(s.hap_bases.data() + o.hb, hsrc, r.hap_bytes);
      for (int a = 0; a < HostRing::kArrays; ++a) std::memcpy(rdst[a] + o.rb, rsrc[a], r.read_bytes);
      for (size_t h = 0; h < r.hap_off.size(); ++h)
        s.hap_off[o.hap + h] = r.hap_off[h] - hap_base + o.hb;
      for (size_t j = 0; j < r.read_off.size(); ++j)
        s.read_off[o.read + j] = r.read_off[j] - read_base + o.rb;
    }
  });
  const Clock::time_point t_comb = Clock::now();
  const uint8_t* arr[HostRing::kArrays + 1];
  if (in_ring) {
    arr[0] = ring_->array(0);
    for (int a = 0; a < HostRing::kArrays; ++a) arr[a + 1] = ring_->array(a);
  } else {
    arr[0] = s.hap_bases.data();
    arr[1] = s.read_bases.data();
    for (int q = 0; q < 4; ++q) arr[q + 2] = s.quals[q].data();
  }
  const rodv_batch b{(uint32_t)s.regions.size(), s.regions.data(), (uint32_t)s.hap_len.size(),
                     arr[0], s.hap_off.data(), s.hap_len.data(), (uint32_t)s.read_len.size(),
                     arr[1], arr[2], arr[3], arr[4], arr[5], s.read_off.data(),
                     s.read_len.data()};
  // Buffers grow with headroom: reallocating device or pinned memory
  // synchronises the device, which would stall the other slot's batch.
  {
    const cudaError_t e = grow(s.staging, est);
    if (e != cudaSuccess) return engine_.cuda_fail(e, "service staging");
  }
  const Clock::time_point t_stage = Clock::now();
  rodv_status st;
  {
    TraceRange pack("rodv service: pack");
    st = engine_.pack(b, s.plan, s.staging, opt_.force_fp64 != 0);
  }
  if (st != RODV_OK) return st;
  const Clock::time_point t_pack = Clock::now();
  const PackedPlan& p = s.plan;
  cudaError_t e = grow(s.arena, p.total_bytes);
  if (e == cudaSuccess) e = grow(s.out_host, p.num_pairs * 8 + kCountWords * 4);
  if (e != cudaSuccess) return engine_.cuda_fail(e, "service buffers");
  uint8_t* d = static_cast<uint8_t*>(s.arena.ptr);
  uint8_t* h = static_cast<uint8_t*>(s.out_host.ptr);
  e = cudaMemcpyAsync(d, s.staging.ptr, p.upload_bytes, cudaMemcpyHostToDevice, s.stream);
  if (e != cudaSuccess) return engine_.cuda_fail(e, "service upload");
  // Batches compute one after the other: this batch's kernels wait for the
  // previous batch's (its upload overlaps them), and its classes run as
  // parallel branches, whose tails overlap.  Run side by side, the batches in
  // flight shared the GPU and each took about as long as all of them
  // together, which is what a request waited for.
  if (prev_kernels_) {
    e = cudaStreamWaitEvent(s.stream, prev_kernels_, 0);
    if (e != cudaSuccess) return engine_.cuda_fail(e, "service batch order");
  }
  st = engine_.launch_all(p, d, nullptr, s.stream, s.ev, 3, /*fan_out=*/true);
  if (st != RODV_OK) return st;
  prev_kernels_ = s.ev[2];
  e = cudaMemcpyAsync(h, d + p.off_out, p.num_pairs * 8, cudaMemcpyDeviceToHost, s.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h + p.num_pairs * 8, d + p.off_counts, kCountWords * 4,
                        cudaMemcpyDeviceToHost, s.stream);
  if (e == cudaSuccess) e = cudaEventRecord(s.done, s.stream);
  if (e != cudaSuccess) return engine_.cuda_fail(e, "service download");
  if (opt_.verbose >= 2)
    fprintf(stderr,
            "rodv service: batch %llu launch ms: combine %.2f staging %.2f pack %.2f "
            "enqueue %.2f (%zu regions)\n",
            (unsigned long long)s.batch_id, ms_between(t0, t_comb), ms_between(t_comb, t_stage),
            ms_between(t_stage, t_pack), ms_between(t_pack, Clock::now()), s.regions.size());
  return RODV_OK;
}

void Service::complete(Slot& s) {
  cudaError_t e;
  {
    TraceRange wait("rodv service: wait for batch");
    e = cudaEventSynchronize(s.done);
  }
  TraceRange trace("rodv service: finish batch");
  if (e != cudaSuccess) {
    fail_slot(s, engine_.cuda_fail(e, "service batch"));
    return;
  }
  const Clock::time_point t0 = Clock::now();
  const PackedPlan& p = s.plan;
  const uint8_t* h = static_cast<const uint8_t*>(s.out_host.ptr);
  const uint32_t* counts = reinterpret_cast<const uint32_t*>(h + p.num_pairs * 8);
  if (counts[kCtrError] != 0) {
    fail_slot(s, engine_.fail(RODV_ERR_DEVICE_CHECK, "kernel reported error flags " +
                                                         std::to_string(counts[kCtrError])));
    return;
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s.ev[0], s.ev[2]);
  uint64_t fp64 = 0;
  for (int c = 0; c < kNumClasses; ++c) fp64 += p.fp64 ? p.pairs[c] : counts[kCtrRescue + c];
  const double* res = reinterpret_cast<const double*>(h);
  uint64_t off = 0;
  for (const auto& r : s.reqs) {
    r->out.assign(res + off, res + off + r->pairs);
    off += r->pairs;
    r->fp64_pairs = fp64;
    r->batch_id = s.batch_id;
    r->batch_regions = (uint32_t)s.regions.size();
  }
  const Clock::time_point now = Clock::now();
  {
    std::lock_guard<std::mutex> lk(mu_);
    for (const auto& r : s.reqs) {
      r->finished = now;
      r->status = RODV_OK;
      r->done = true;
      latencies_.push_back(ms_between(r->submitted, now));
      ++st_completed_;
      st_pairs_ += r->pairs;
      st_cells_ += r->cells;
      st_regions_ += r->regions.size();
      --inflight_;
    }
    st_fp64_ += fp64;
    st_device_ms_ += ms;
    st_finish_ms_ += ms_between(t0, now);
    ++st_batches_;
    st_last_done_ = now;
  }
  if (opt_.verbose)
    fprintf(stderr, "rodv service: batch %llu: %zu requests, %zu regions, %llu pairs, %.3f ms\n",
            (unsigned long long)s.batch_id, s.reqs.size(), s.regions.size(),
            (unsigned long long)p.num_pairs, ms);
  s.reqs.clear();
  cv_done_.notify_all();
  cv_space_.notify_all();
}

void Service::release_ring(Slot& s) {
  for (const auto& r : s.reqs)
    if (r->ring_pos != HostRing::kNone) {
      ring_->release(r->ring_pos);
      r->ring_pos = HostRing::kNone;
    }
}

void Service::fail_slot(Slot& s, rodv_status st) {
  const Clock::time_point now = Clock::now();
  {
    std::lock_guard<std::mutex> lk(mu_);
    err_ = engine_.last_error();
    for (const auto& r : s.reqs) {
      r->finished = now;
      r->status = st;
      r->done = true;
      ++st_failed_;
      --inflight_;
    }
  }
  s.reqs.clear();
  cv_done_.notify_all();
  cv_space_.notify_all();
}

rodv_status Service::result(uint64_t ticket, int32_t wait_ms, double* out,
                            rodv_request_stats* st) {
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = table_.find(ticket);
    if (it == table_.end()) return RODV_ERR_NOT_FOUND;
    r = it->second;
    if (!r->done) {
      if (wait_ms == 0) return RODV_ERR_NOT_READY;
      auto ready = [&] { return r->done; };
      if (wait_ms < 0)
        cv_done_.wait(lk, ready);
      else if (!cv_done_.wait_for(lk, std::chrono::milliseconds(wait_ms), ready))
        return RODV_ERR_NOT_READY;
    }
    table_.erase(ticket);
  }
  if (r->status != RODV_OK) return r->status;
  if (out) std::memcpy(out, r->out.data(), r->pairs * sizeof(double));
  if (st) {
    *st = rodv_request_stats{};
    st->pairs = r->pairs;
    st->cells = r->cells;
    st->fp64_pairs = r->fp64_pairs;
    st->batch_id = r->batch_id;
    st->batch_regions = r->batch_regions;
    st->queue_ms = ms_between(r->submitted, r->started);
    st->latency_ms = ms_between(r->submitted, r->finished);
  }
  return RODV_OK;
}

rodv_status Service::stats(rodv_service_stats* out) {
  if (!out) return RODV_ERR_INVALID_ARG;
  std::vector<double> lat;
  *out = rodv_service_stats{};
  {
    std::lock_guard<std::mutex> lk(mu_);
    lat = latencies_;
    out->submitted = st_submitted_;
    out->completed = st_completed_;
    out->failed = st_failed_;
    out->batches = st_batches_;
    out->regions = st_regions_;
    out->pairs = st_pairs_;
    out->cells = st_cells_;
    out->fp64_pairs = st_fp64_;
    out->device_ms = st_device_ms_;
    out->wall_ms = (st_any_ && st_completed_) ? ms_between(st_first_submit_, st_last_done_) : 0.0;
    out->mean_batch_regions = st_batches_ ? (double)st_regions_ / st_batches_ : 0.0;
    out->host_launch_ms = st_launch_ms_;
    out->host_finish_ms = st_finish_ms_;
  }
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {  // nearest rank
      const size_t k = (size_t)std::ceil(q * (double)lat.size());
      return lat[std::min(lat.size(), std::max<size_t>(k, 1)) - 1];
    };
    out->latency_p50_ms = pct(0.50);
    out->latency_p99_ms = pct(0.99);
    out->latency_max_ms = lat.back();
    double sum = 0;
    for (double v : lat) sum += v;
    out->latency_mean_ms = sum / (double)lat.size();
  }
  return RODV_OK;
}

std::string Service::last_error() {
  std::lock_guard<std::mutex> lk(mu_);
  return err_;
}

void Service::reset_stats() {
  std::lock_guard<std::mutex> lk(mu_);
  latencies_.clear();
  st_submitted_ = st_completed_ = st_failed_ = st_batches_ = 0;
  st_pairs_ = st_cells_ = st_fp64_ = st_regions_ = 0;
  st_device_ms_ = st_launch_ms_ = st_finish_ms_ = 0;
  st_any_ = false;
}

}  // namespace rodv

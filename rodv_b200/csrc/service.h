// service.h -- the streaming PairHMM service behind rodv_service_* (C ABI).
//
// Callers submit regions (one rodv_batch each) at any time and poll or wait
// for their results.  One worker thread batches whatever has been submitted
// while the GPU was busy into the next device batch (continuous batching) on
// kSlots slots, each with its own stream, pinned staging and device arena, so
// the host packs and uploads the next batches while earlier ones compute.
// Submit copies a request's bases and qualities into the service's host ring
// (host_ring.h), so forming a batch copies no bases: the batch's arrays are
// the ring's, and the packer reads each request where submit put it.
// Admission: a request larger than a slot's share of the device-memory
// budget is refused (RODV_ERR_ADMISSION); submit blocks while max_inflight
// requests are queued or running.  A batch takes queued requests up to a
// fixed size (or one larger request alone) so that its buffers, reserved at
// creation, are reused without reallocation.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "host_ring.h"

namespace rodv {

class Service {
 public:
  explicit Service(const rodv_options& opt);
  ~Service();
  rodv_status init();
  rodv_status submit(const rodv_batch& b, uint64_t* ticket);
  // wait_ms < 0: wait without limit; 0: poll.
  rodv_status result(uint64_t ticket, int32_t wait_ms, double* out, rodv_request_stats* st);
  rodv_status stats(rodv_service_stats* out);
  void reset_stats();
  std::string last_error();

 private:
  using Clock = std::chrono::steady_clock;
  struct Request {
    uint64_t ticket = 0;
    // copy of the caller's regions: bases and qualities in the service's
    // ring (ring_pos != kNone; hap_off and read_off are ring positions) or,
    // for a request too large for it, in the request's own arrays
    std::vector<rodv_region> regions;
    uint64_t ring_pos = HostRing::kNone;
    std::vector<uint8_t> hap_bases, read_bases, quals[4];
    std::vector<uint64_t> hap_off, read_off;
    uint64_t hap_bytes = 0, read_bytes = 0;
    std::vector<uint32_t> hap_len, read_len;
    uint64_t pairs = 0, cells = 0, bytes = 0;
    Clock::time_point submitted, started, finished;
    std::vector<double> out;
    rodv_status status = RODV_OK;
    uint64_t fp64_pairs = 0;
    uint64_t batch_id = 0;
    uint32_t batch_regions = 0;
    bool done = false;
  };
  struct Slot {
    PackedPlan plan;
    PinnedMem staging, out_host;
    DeviceMem arena;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[3] = {};        // FP32 start, FP32 end, FP64 end
    cudaEvent_t done = nullptr;    // after the result download
    std::vector<std::shared_ptr<Request>> reqs;
    // the combined batch's host arrays
    std::vector<rodv_region> regions;
    std::vector<uint8_t> hap_bases, read_bases, quals[4];
    std::vector<uint64_t> hap_off, read_off;
    std::vector<uint32_t> hap_len, read_len;
    uint64_t batch_id = 0;
  };

  void worker();
  rodv_status launch(Slot& s);
  void complete(Slot& s);
  void fail_slot(Slot& s, rodv_status st);
  void release_ring(Slot& s);
  uint64_t estimate_bytes(const rodv_batch& b, uint64_t pairs) const;

  rodv_options opt_;
  Engine engine_;
  static constexpr int kSlots = 3;
  Slot slots_[kSlots];
  uint64_t slot_budget_ = 0;   // largest request (device bytes) a slot admits
  uint64_t batch_bytes_ = 0;   // batches are formed up to this size
  uint32_t max_inflight_ = 0;
  cudaEvent_t prev_kernels_ = nullptr;  // end of the last launched batch's kernels
  std::unique_ptr<HostRing> ring_;

  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_, cv_space_;
  std::deque<std::shared_ptr<Request>> pending_;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> table_;
  uint32_t inflight_ = 0;      // queued or running requests
  uint64_t next_ticket_ = 1;
  uint64_t next_batch_ = 1;
  bool stop_ = false;
  std::string err_;            // last failure
  bool ready_ = false;
  std::thread thread_;

  // statistics since the last reset
  std::vector<double> latencies_;
  uint64_t st_submitted_ = 0, st_completed_ = 0, st_failed_ = 0, st_batches_ = 0;
  uint64_t st_pairs_ = 0, st_cells_ = 0, st_fp64_ = 0, st_regions_ = 0;
  double st_device_ms_ = 0, st_launch_ms_ = 0, st_finish_ms_ = 0;
  bool st_any_ = false;
  Clock::time_point st_first_submit_, st_last_done_;
};

}  // namespace rodv

struct rodv_service {
  rodv::Service* impl;
};

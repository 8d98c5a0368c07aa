// host_ring.h -- the streaming service's host copy of submitted requests.
//
// A request's bases and qualities are copied at submit into five parallel
// byte rings (read bases, base, insertion, deletion and gap-continuation
// qualities; haplotype bases share the first): one range of the same
// position in every ring.  A batch of requests is then one rodv_batch whose
// arrays are the rings themselves, with each request's haplotype and read
// offsets pointing at its range, so forming a batch copies no bases.  Ranges
// are released when the request's batch completes or fails, in any order;
// the ring's free space starts after the oldest range still held.
#pragma once
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>

namespace rodv {

class HostRing {
 public:
  static constexpr int kArrays = 5;
  static constexpr uint64_t kNone = ~0ull;

  explicit HostRing(uint64_t capacity) : cap_(capacity) {
    for (auto& a : arr_) a.reset(new uint8_t[cap_ ? cap_ : 1]);
  }
  uint64_t capacity() const { return cap_; }
  uint8_t* array(int k) const { return arr_[k].get(); }

  // A range of n bytes (1 <= n <= capacity / 2), waiting while the ring is
  // full; kNone once stop() was called.
  uint64_t acquire(uint64_t n) {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      if (stopped_) return kNone;
      const uint64_t pos = place(n);
      if (pos != kNone) {
        held_.push_back(Range{pos, n, false});
        tail_ = pos + n;
        return pos;
      }
      cv_.wait(lk);
    }
  }
  // Releases the range that starts at pos.
  void release(uint64_t pos) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (Range& r : held_)
        if (r.pos == pos && !r.released) {
          r.released = true;
          break;
        }
      while (!held_.empty() && held_.front().released) held_.pop_front();
      if (held_.empty()) tail_ = 0;
    }
    cv_.notify_all();
  }
  void stop() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stopped_ = true;
    }
    cv_.notify_all();
  }
  // Ranges held (testing).
  size_t held() {
    std::lock_guard<std::mutex> lk(mu_);
    return held_.size();
  }

 private:
  struct Range {
    uint64_t pos, n;
    bool released;
  };
  // Where n bytes fit after the newest range, wrapping to the ring's start
  // when the end is too short; kNone if they do not fit before the oldest.
  uint64_t place(uint64_t n) const {
    if (held_.empty()) return n <= cap_ ? 0 : kNone;
    const uint64_t head = held_.front().pos;
    if (tail_ > head) {  // used: [head, tail)
      if (tail_ + n <= cap_) return tail_;
      return n <= head ? 0 : kNone;
    }
    // wrapped, used: [head, cap) and [0, tail)
    return tail_ + n <= head ? tail_ : kNone;
  }

  uint64_t cap_;
  std::unique_ptr<uint8_t[]> arr_[kArrays];
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Range> held_;  // in acquisition order
  uint64_t tail_ = 0;       // end of the newest range
  bool stopped_ = false;
};

}  // namespace rodv

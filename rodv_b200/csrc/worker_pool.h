// worker_pool.h -- a process-wide pool of host worker threads, used by the
// packer and the streaming service.
#pragma once
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace rodv {

// A process-wide pool of host worker threads for the packer.  parallel_for
// splits [0, n) into chunks of `grain`; the calling thread and up to
// (chunks - 1) pool workers take chunks until none is left.  Threads are
// created once: spawning them per call cost more than packing a small batch.
class WorkerPool {
 public:
  static inline WorkerPool& get() {
    static WorkerPool pool;
    return pool;
  }
  unsigned size() const { return (unsigned)threads_.size(); }
  void submit(std::function<void()> task) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      tasks_.push_back(std::move(task));
    }
    cv_.notify_one();
  }

 private:
  WorkerPool() {
    const unsigned n = std::max(1u, std::thread::hardware_concurrency()) - 1;
    for (unsigned i = 0; i < n; ++i)
      threads_.emplace_back([this] {
        for (;;) {
          std::function<void()> task;
          {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !tasks_.empty(); });
            if (stop_ && tasks_.empty()) return;
            task = std::move(tasks_.front());
            tasks_.pop_front();
          }
          task();
        }
      });
  }
  ~WorkerPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<void()>> tasks_;
  std::vector<std::thread> threads_;
  bool stop_ = false;
};

template <class F>
void parallel_for(size_t n, size_t grain, F&& f) {
  const size_t chunks = (n + grain - 1) / grain;
  const unsigned helpers = (unsigned)std::min<size_t>(WorkerPool::get().size(), chunks ? chunks - 1 : 0);
  if (helpers == 0) {
    if (n) f(0, n);
    return;
  }
  struct Job {
    std::atomic<size_t> next{0};
    std::atomic<unsigned> running{0};
    std::mutex mu;
    std::condition_variable cv;
  };
  auto job = std::make_shared<Job>();
  auto work = [job, chunks, grain, n, &f] {
    for (;;) {
      const size_t c = job->next.fetch_add(1);
      if (c >= chunks) break;
      f(c * grain, std::min(n, (c + 1) * grain));
    }
  };
  job->running = helpers;
  for (unsigned t = 0; t < helpers; ++t)
    WorkerPool::get().submit([job, work] {
      work();
      if (job->running.fetch_sub(1) == 1) {
        std::lock_guard<std::mutex> lk(job->mu);
        job->cv.notify_all();
      }
    });
  work();
  std::unique_lock<std::mutex> lk(job->mu);
  job->cv.wait(lk, [&] { return job->running.load() == 0; });
}

}  // namespace rodv

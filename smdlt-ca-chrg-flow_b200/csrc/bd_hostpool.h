// Process-wide pool of host worker threads for the Krylov convergence checks
// (one tridiagonal square root per open right-hand side of a noise block).
// The workers are created once, at the first parallel call, so a check costs
// a wake-up instead of a thread spawn and join per worker; the device waits
// for the host at every check, so this is on the step's critical path.
//
// HostPool::run(n, f) calls f(0) .. f(n - 1) once each, on the calling thread
// and on the workers, and returns when every call has finished.  The caller
// takes indices itself, so a run completes even when no worker picks it up
// (no worker threads in a forked child, all workers busy with the runs of
// other replicas): the workers only add parallelism.  Concurrent callers
// share the workers; f must not throw.
//
// The pool is never destroyed: its workers sleep on a condition variable and
// end with the process, so no exit-time join can wait on them.
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>

namespace bd {

class HostPool {
 public:
  static HostPool& get() {
    static HostPool* pool = new HostPool();
    return *pool;
  }

  template <class F>
  void run(int n, F&& f) {
    if (n <= 0) return;
    if (n == 1 || nworkers_ == 0) {
      for (int i = 0; i < n; i++) f(i);
      return;
    }
    auto job = std::make_shared<Job>();
    // f is held by reference and lives on this frame.  That is safe only
    // because of the order in work(): a thread calls f only for an index it
    // claimed below n, and counts the call down after it returns; run returns
    // once every claimed call has been counted, so no call of f can start or
    // still run after that.  Keep claim -> call -> count down in that order
    // (never count down first, never retry an index).
    job->f = std::function<void(int)>(std::ref(f));
    job->n = n;
    job->left.store(n);
    {
      std::lock_guard<std::mutex> lk(mu_);
      q_.push_back(job);
    }
    if (n - 1 >= nworkers_)
      cv_.notify_all();
    else
      for (int w = 0; w < n - 1; w++) cv_.notify_one();
    work(*job);
    {
      std::unique_lock<std::mutex> lk(job->mu);
      job->done.wait(lk, [&] { return job->left.load() == 0; });
    }
    drop(job);
  }

  int workers() const { return nworkers_; }

 private:
  struct Job {
    std::function<void(int)> f;
    int n = 0;
    std::atomic<int> next{0};
    std::atomic<int> left{0};
    std::mutex mu;
    std::condition_variable done;
  };

  HostPool() {
    unsigned hw = std::thread::hardware_concurrency();
    nworkers_ = (int)std::min(15u, hw > 1 ? hw - 1 : 0u);
    for (int w = 0; w < nworkers_; w++) std::thread([this] { loop(); }).detach();
  }

  // Takes indices of the job until none is left; the thread that finishes
  // the last call wakes the job's caller.
  static void work(Job& j) {
    for (int i; (i = j.next.fetch_add(1)) < j.n;) {
      j.f(i);
      if (j.left.fetch_sub(1) == 1) {
        std::lock_guard<std::mutex> lk(j.mu);
        j.done.notify_all();
      }
    }
  }

  // Removes an exhausted job from the queue (by whichever thread sees it
  // first: a worker or the job's caller).
  void drop(const std::shared_ptr<Job>& job) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = std::find(q_.begin(), q_.end(), job);
    if (it != q_.end()) q_.erase(it);
  }

  void loop() {
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !q_.empty(); });
        job = q_.front();
        if (job->next.load() >= job->n) {  // exhausted: drop it, look again
          q_.pop_front();
          continue;
        }
      }
      work(*job);
      drop(job);
    }
  }

  int nworkers_ = 0;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::shared_ptr<Job>> q_;
};

}  // namespace bd

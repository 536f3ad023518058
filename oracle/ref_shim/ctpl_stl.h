// Test infrastructure only: a project-written stand-in for the CTPL thread-pool
// header (github.com/vit-vit/CTPL, `ctpl_stl.h`, branch master, commit not pinned
// by the reference's .gitmodules) that the reference's CPU code includes
// (src/ThreadPool/ThreadPool.h:4) but whose submodule is empty in the mount.
//
// Only the three calls the reference makes are provided, with CTPL's published
// semantics:
//   push(f, args...)  queue f(threadId, args...) on a worker thread
//   resize(n)         make n workers available
//   size()            number of workers requested
// The scheduling order does not affect the reference's arithmetic: every task
// writes its own output slots (src/Coil/Fields/CalculateAllFieldsMT.cxx:26-40).
#ifndef CCOIL_ORACLE_CTPL_SHIM_H
#define CCOIL_ORACLE_CTPL_SHIM_H

#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace ctpl
{
class thread_pool
{
  public:
    thread_pool() = default;
    explicit thread_pool(int n) { resize(n); }
    ~thread_pool()
    {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : workers_)
            if (t.joinable())
                t.join();
    }

    int size() const { return requested_; }

    void resize(int n)
    {
        if (n < 1)
            n = 1;
        std::lock_guard<std::mutex> lock(mutex_);
        requested_ = n;
        // workers are only ever added; idle extra workers cost nothing
        while (static_cast<int>(workers_.size()) < n)
        {
            int id = static_cast<int>(workers_.size());
            workers_.emplace_back([this, id] { run(id); });
        }
    }

    template <class F, class... Rest>
    void push(F &&f, Rest &&...rest)
    {
        auto bound = std::bind(std::forward<F>(f), std::placeholders::_1, std::forward<Rest>(rest)...);
        {
            std::lock_guard<std::mutex> lock(mutex_);
            if (workers_.empty())
            {
                requested_ = 1;
                workers_.emplace_back([this] { run(0); });
            }
            queue_.emplace_back([bound](int id) mutable { bound(id); });
        }
        cv_.notify_one();
    }

  private:
    void run(int id)
    {
        for (;;)
        {
            std::function<void(int)> task;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                cv_.wait(lock, [this] { return stop_ || !queue_.empty(); });
                if (stop_ && queue_.empty())
                    return;
                task = std::move(queue_.front());
                queue_.pop_front();
            }
            task(id);
        }
    }

    std::vector<std::thread> workers_;
    std::deque<std::function<void(int)>> queue_;
    std::mutex mutex_;
    std::condition_variable cv_;
    bool stop_ = false;
    int requested_ = 0;
};
} // namespace ctpl

#endif

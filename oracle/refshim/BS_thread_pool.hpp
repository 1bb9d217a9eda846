// Stand-in for the bshoshany thread-pool header that the reference fetches at
// configure time (not vendored, no network here).  It provides only the three
// members the reference calls on BS::light_thread_pool: detach_task, wait and
// get_thread_ids (include/core/container/ThreadLocalWrapper.h:46,
// source/core/utility/MultiThreading.cpp:9-13).  It is a plain
// mutex/condition-variable FIFO pool written for this oracle build; it only
// changes scheduling, never what a task computes.
#pragma once
#include <condition_variable>
#include <cstddef>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace BS {
class light_thread_pool {
  public:
    explicit light_thread_pool(std::size_t n = 0) {
        if (n == 0) n = 1;
        for (std::size_t i = 0; i < n; ++i) workers_.emplace_back([this] { run(); });
    }
    ~light_thread_pool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    template <typename F>
    void detach_task(F&& f) {
        {
            std::lock_guard<std::mutex> g(m_);
            q_.emplace_back(std::forward<F>(f));
            ++pending_;
        }
        cv_.notify_one();
    }
    void wait() {
        std::unique_lock<std::mutex> g(m_);
        done_.wait(g, [this] { return pending_ == 0; });
    }
    std::vector<std::thread::id> get_thread_ids() const {
        std::vector<std::thread::id> ids;
        for (auto& t : workers_) ids.push_back(t.get_id());
        return ids;
    }
    std::size_t get_thread_count() const { return workers_.size(); }

  private:
    void run() {
        for (;;) {
            std::function<void()> task;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [this] { return stop_ || !q_.empty(); });
                if (stop_ && q_.empty()) return;
                task = std::move(q_.front());
                q_.pop_front();
            }
            task();
            {
                std::lock_guard<std::mutex> g(m_);
                if (--pending_ == 0) done_.notify_all();
            }
        }
    }
    std::vector<std::thread> workers_;
    std::deque<std::function<void()>> q_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    std::size_t pending_ = 0;
    bool stop_ = false;
};
}  // namespace BS

// Request scheduler of the serving loop: continuous admission of fit and predict requests
// by device-memory budget.
//
// A request carries its estimated device working set and a piece of work.  Requests
// start in arrival order (FIFO): the head of the queue is admitted as soon as a slot is
// free and its working set fits into what the running requests leave of the budget.  A
// request that arrives while others run is admitted the moment they free enough slots
// and memory, and runs beside them.  On the device each request has its own stream, so
// the kernels of concurrent requests overlap.  A request larger than the whole budget is
// refused when it is submitted.  Requests with the same key (the model they fit or
// predict with) never run at once: a predict submitted after its model's fit starts
// after that fit ends.  Latency is measured from submission to completion, so it
// includes the time spent waiting for admission.
//
// The scheduler knows nothing about the device: the work is a callable, so the tests
// drive it with host-only work.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace tgb {

class Scheduler {
public:
    enum Kind { kFit = 0, kPredict = 1 };
    enum Status { kQueued = 0, kRunning = 1, kDone = 2, kFailed = 3 };

    struct Stats {
        long long completed = 0, failed = 0;
        double p50_s = 0, p99_s = 0;                  // latency (submit -> done), all requests
        double p50_fit_s = 0, p99_fit_s = 0;          // fit requests
        double p50_predict_s = 0, p99_predict_s = 0;  // predict requests
        double mean_wait_s = 0;                       // submit -> start
        size_t peak_bytes = 0;                        // largest admitted working set total
        int peak_running = 0;                         // most requests running at once
        double busy_s = 0;                            // first submit -> last completion
    };

    Scheduler(size_t budget_bytes, int slots) : budget_(budget_bytes), slots_(std::max(1, slots)) {
        for (int w = 0; w < slots_; ++w) workers_.emplace_back([this] { worker(); });
    }

    ~Scheduler() {
        {
            std::unique_lock<std::mutex> lk(mu_);
            done_cv_.wait(lk, [&] { return queue_.empty() && running_ == 0; });
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

    Scheduler(const Scheduler&) = delete;
    Scheduler& operator=(const Scheduler&) = delete;

    // Queues a request; returns its id.  key: requests with the same nonzero key run one at
    // a time.  Throws when bytes exceed the whole budget.
    long long submit(Kind kind, size_t bytes, std::function<void()> work, uintptr_t key = 0) {
        if (bytes > budget_) throw std::runtime_error("request needs more device memory than the serving budget");
        std::lock_guard<std::mutex> lk(mu_);
        const long long id = next_id_++;
        Req& r = reqs_[id];
        r.kind = kind;
        r.bytes = bytes;
        r.key = key;
        r.work = std::move(work);
        r.t_submit = now();
        if (first_submit_ < 0) first_submit_ = r.t_submit;
        queue_.push_back(id);
        cv_.notify_all();
        return id;
    }

    // Waits up to timeout_s (< 0: no limit) for request id; returns its status (kDone or
    // kFailed when finished, else kQueued / kRunning).  error receives a failure's message.
    int wait(long long id, double timeout_s, std::string* error = nullptr) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) throw std::runtime_error("unknown request id");
        auto finished = [&] { return it->second.status == kDone || it->second.status == kFailed; };
        if (timeout_s < 0) done_cv_.wait(lk, finished);
        else done_cv_.wait_for(lk, std::chrono::duration<double>(timeout_s), finished);
        if (error) *error = it->second.error;
        return it->second.status;
    }

    Stats stats() const {
        std::lock_guard<std::mutex> lk(mu_);
        Stats s;
        std::vector<double> all, fit, pred;
        double wait_sum = 0;
        for (const auto& kv : reqs_) {
            const Req& r = kv.second;
            if (r.status != kDone && r.status != kFailed) continue;
            if (r.status == kFailed) ++s.failed;
            else ++s.completed;
            const double lat = r.t_done - r.t_submit;
            all.push_back(lat);
            (r.kind == kFit ? fit : pred).push_back(lat);
            wait_sum += r.t_start - r.t_submit;
        }
        s.p50_s = quantile(all, 0.50);
        s.p99_s = quantile(all, 0.99);
        s.p50_fit_s = quantile(fit, 0.50);
        s.p99_fit_s = quantile(fit, 0.99);
        s.p50_predict_s = quantile(pred, 0.50);
        s.p99_predict_s = quantile(pred, 0.99);
        s.mean_wait_s = all.empty() ? 0.0 : wait_sum / static_cast<double>(all.size());
        s.peak_bytes = peak_bytes_;
        s.peak_running = peak_running_;
        s.busy_s = first_submit_ < 0 ? 0.0 : last_done_ - first_submit_;
        return s;
    }

    // Start order of the requests admitted so far (ids), for tests of the FIFO rule.
    std::vector<long long> start_order() const {
        std::lock_guard<std::mutex> lk(mu_);
        return started_;
    }

    size_t budget() const { return budget_; }

    // Nearest-rank quantile (the smallest value with at least q of the sample at or below it).
    static double quantile(std::vector<double> v, double q) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        size_t k = static_cast<size_t>(std::ceil(q * static_cast<double>(v.size())));
        k = std::min(std::max<size_t>(k, 1), v.size());
        return v[k - 1];
    }

private:
    struct Req {
        Kind kind = kFit;
        size_t bytes = 0;
        uintptr_t key = 0;
        std::function<void()> work;
        int status = kQueued;
        std::string error;
        double t_submit = 0, t_start = 0, t_done = 0;
    };

    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }

    // The head of the queue may start now (caller holds mu_).
    bool head_admissible() const {
        if (queue_.empty() || running_ >= slots_) return false;
        const Req& r = reqs_.at(queue_.front());
        if (r.key != 0 && busy_.count(r.key)) return false;
        return used_ + r.bytes <= budget_;
    }

    void worker() {
        for (;;) {
            long long id;
            std::function<void()> work;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || head_admissible(); });
                if (stop_) return;
                id = queue_.front();
                queue_.pop_front();
                Req& r = reqs_[id];
                used_ += r.bytes;
                if (r.key != 0) busy_.insert(r.key);
                ++running_;
                peak_bytes_ = std::max(peak_bytes_, used_);
                peak_running_ = std::max(peak_running_, running_);
                r.status = kRunning;
                r.t_start = now();
                started_.push_back(id);
                work = std::move(r.work);
            }
            cv_.notify_all();  // the next head may fit beside this one
            std::string err;
            try {
                work();
            } catch (const std::exception& e) {
                err = e.what();
                if (err.empty()) err = "request failed";
            } catch (...) {
                err = "request failed";
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                Req& r = reqs_[id];
                r.t_done = now();
                last_done_ = std::max(last_done_, r.t_done);
                r.status = err.empty() ? kDone : kFailed;
                r.error = err;
                used_ -= r.bytes;
                if (r.key != 0) busy_.erase(r.key);
                --running_;
            }
            cv_.notify_all();
            done_cv_.notify_all();
        }
    }

    const size_t budget_;
    const int slots_;
    mutable std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::deque<long long> queue_;
    std::map<long long, Req> reqs_;
    std::vector<long long> started_;
    std::set<uintptr_t> busy_;  // keys of running requests
    std::vector<std::thread> workers_;
    long long next_id_ = 1;
    size_t used_ = 0, peak_bytes_ = 0;
    int running_ = 0, peak_running_ = 0;
    double first_submit_ = -1, last_done_ = 0;
    bool stop_ = false;
};

}  // namespace tgb

// Host pipeline that produces each tree's GOSS draw positions ahead of the GPU.
//
// Per tree the booster's generator makes one std::shuffle of the m-row GOSS remainder
// (cpp/src/booster.cpp:572) and one draw for grow_tree's seed (booster.cpp:588).  The
// positions a tree needs depend only on the generator state at the tree's start, so:
//   producer  walks the stream once (skip_shuffle: exact, no positions) and snapshots
//             the generator at every tree start;
//   workers   take trees in order, restart from the snapshot and compute the kept
//             positions (shuffled_prefix) into a pinned slot, in parallel;
//   consumer  (the fit loop) waits for tree t, enqueues the H2D copy, records an event
//             and releases the slot; a worker reuses a slot only after that copy ends.
// The producer starts with the object, so it runs ahead while the fit uploads and bins
// the data; the workers start on start_workers() (or the first wait).
#pragma once

#include <chrono>
#include <condition_variable>
#include <cuda_runtime.h>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "sampling.h"

namespace tgb {

// Pinned host blocks kept for reuse across fits of the process (cudaMallocHost and
// cudaFreeHost cost milliseconds each).
inline std::mutex& pinned_cache_mutex() {
    static std::mutex mu;
    return mu;
}
inline std::vector<std::pair<size_t, void*>>& pinned_cache() {
    static std::vector<std::pair<size_t, void*>> cache;
    return cache;
}
inline void* pinned_take(size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(pinned_cache_mutex());
        auto& c = pinned_cache();
        for (size_t k = 0; k < c.size(); ++k)
            if (c[k].first == bytes) {
                void* p = c[k].second;
                c.erase(c.begin() + static_cast<long>(k));
                return p;
            }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) throw std::runtime_error("cudaMallocHost (GOSS positions)");
    return p;
}
inline void pinned_give(size_t bytes, void* p) {
    std::lock_guard<std::mutex> lk(pinned_cache_mutex());
    auto& c = pinned_cache();
    if (c.size() < 64) c.emplace_back(bytes, p);
    else cudaFreeHost(p);
}

class GossSampler {
public:
    GossSampler(uint32_t seed, int64_t m, int64_t keep, int n_trees, int n_slots, int n_workers)
        : m_(m), keep_(std::max<int64_t>(1, keep)), T_(n_trees), S_(std::max(1, n_slots)),
          snaps_(n_trees), min_pos_(n_trees, 0), produced_(n_trees, 0), ready_(n_trees, 0), released_(n_trees, 0),
          slot_(S_, nullptr), slot_ev_(S_, nullptr) {
        for (int k = 0; k < S_; ++k) {
            slot_[k] = static_cast<int32_t*>(pinned_take(sizeof(int32_t) * keep_));
            if (cudaEventCreateWithFlags(&slot_ev_[k], cudaEventDisableTiming) != cudaSuccess)
                throw std::runtime_error("cudaEventCreate (GOSS positions)");
        }
        n_workers_ = std::max(1, n_workers);
        threads_.emplace_back([this, seed] { produce(seed); });
    }

    // Starts the workers.  The producer runs from construction (it walks the stream
    // sequentially and is the long pole); the workers can start once the host has
    // finished its other parallel work.
    void start_workers() {
        if (workers_started_) return;
        workers_started_ = true;
        for (int w = 0; w < n_workers_; ++w) threads_.emplace_back([this] { work(); });
    }

    // Stops the threads (all trees consumed, or an error path) and joins them.
    void stop() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            abort_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_)
            if (t.joinable()) t.join();
    }

    ~GossSampler() {
        stop();
        for (int k = 0; k < S_; ++k) {
            if (slot_[k]) pinned_give(sizeof(int32_t) * keep_, slot_[k]);
            if (slot_ev_[k]) cudaEventDestroy(slot_ev_[k]);
        }
    }

    // Blocks until tree t's positions are ready; returns the pinned slot holding them.
    const int32_t* wait(int t) {
        start_workers();
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return ready_[t] || abort_ || !error_.empty(); });
        if (!error_.empty()) throw std::runtime_error(error_);
        return slot_[t % S_];
    }

    // Smallest position of tree t's draw (valid once wait(t) returned): the sampled row of
    // the remainder with the largest |g|.
    int32_t min_pos(int t) const { return min_pos_[t]; }

    // After the consumer enqueued the copy of tree t's slot on `stream`.
    void release(int t, cudaStream_t stream) {
        if (cudaEventRecord(slot_ev_[t % S_], stream) != cudaSuccess) throw std::runtime_error("cudaEventRecord");
        {
            std::lock_guard<std::mutex> lk(mu_);
            released_[t] = 1;
        }
        cv_.notify_all();
    }

private:
    void produce(uint32_t seed) {
        Mt32 rng(seed);
        for (int t = 0; t < T_; ++t) {
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (abort_) return;
                snaps_[t] = rng;
                produced_[t] = 1;
            }
            cv_.notify_all();
            const auto t0 = std::chrono::steady_clock::now();
            skip_shuffle(m_, rng);
            (void)rng();  // grow_tree's seed draw
            producer_s_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
    }

public:
    // Seconds the producer spent walking the stream (its per-tree cost bounds throughput).
    double producer_seconds() const { return producer_s_; }

private:
    double producer_s_ = 0.0;

    void work() {
        for (;;) {
            int t;
            {
                std::unique_lock<std::mutex> lk(mu_);
                if (next_ >= T_ || abort_) return;
                t = next_++;
                cv_.wait(lk, [&] { return abort_ || (produced_[t] && (t < S_ || released_[t - S_])); });
                if (abort_) return;
            }
            const int k = t % S_;
            if (t >= S_ && cudaEventSynchronize(slot_ev_[k]) != cudaSuccess) {
                std::lock_guard<std::mutex> lk(mu_);
                error_ = "cudaEventSynchronize (GOSS positions)";
                cv_.notify_all();
                return;
            }
            Mt32 rng = snaps_[t];
            shuffled_prefix(m_, keep_, rng, slot_[k]);
            min_pos_[t] = *std::min_element(slot_[k], slot_[k] + keep_);
            {
                std::lock_guard<std::mutex> lk(mu_);
                ready_[t] = 1;
            }
            cv_.notify_all();
        }
    }

    int64_t m_, keep_;
    int T_, S_;
    std::vector<Mt32> snaps_;
    std::vector<int32_t> min_pos_;
    std::vector<char> produced_, ready_, released_;
    std::vector<int32_t*> slot_;
    std::vector<cudaEvent_t> slot_ev_;
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_;
    int next_ = 0;
    int n_workers_ = 1;
    bool workers_started_ = false;
    bool abort_ = false;
    std::string error_;
};

}  // namespace tgb

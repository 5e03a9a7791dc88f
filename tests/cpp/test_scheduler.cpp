// Host-only checks of the serving scheduler (tidegbm_b200/csrc/serving.h) with timed
// sleeps as the work.  Built and run by tests/test_cpu_serving.py; prints "ok".
#include "serving.h"

#include <atomic>
#include <cstdio>
#include <cstdlib>

using tgb::Scheduler;

#define CHECK(c)                                                        \
    do {                                                                \
        if (!(c)) {                                                     \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #c); \
            std::exit(1);                                               \
        }                                                               \
    } while (0)

static void sleep_ms(int ms) { std::this_thread::sleep_for(std::chrono::milliseconds(ms)); }

int main() {
    // budget: 40% requests, two fit at once although four slots are free
    {
        Scheduler s(100, 4);
        std::atomic<int> live{0}, most{0};
        std::vector<long long> ids;
        for (int k = 0; k < 8; ++k)
            ids.push_back(s.submit(Scheduler::kFit, 40, [&] {
                const int v = ++live;
                int m = most.load();
                while (v > m && !most.compare_exchange_weak(m, v)) {}
                sleep_ms(60);
                --live;
            }));
        for (long long id : ids) CHECK(s.wait(id, -1) == Scheduler::kDone);
        const auto st = s.stats();
        CHECK(st.peak_bytes <= 100 && st.peak_running == 2 && most.load() == 2);
        CHECK(st.completed == 8 && st.failed == 0);
    }
    // slots: small requests, at most three at once, and three do overlap
    {
        Scheduler s(1000, 3);
        std::vector<long long> ids;
        for (int k = 0; k < 9; ++k) ids.push_back(s.submit(Scheduler::kPredict, 1, [] { sleep_ms(60); }));
        for (long long id : ids) CHECK(s.wait(id, -1) == Scheduler::kDone);
        CHECK(s.stats().peak_running == 3);
    }
    // FIFO: a small request behind a large one that does not fit waits for it
    {
        Scheduler s(100, 4);
        const long long a = s.submit(Scheduler::kFit, 70, [] { sleep_ms(80); });
        sleep_ms(10);
        const long long b = s.submit(Scheduler::kFit, 70, [] { sleep_ms(10); });  // does not fit beside a
        const long long c = s.submit(Scheduler::kPredict, 10, [] { sleep_ms(10); });  // would fit, but queues behind b
        CHECK(s.wait(c, -1) == Scheduler::kDone);
        const auto order = s.start_order();
        CHECK(order.size() == 3 && order[0] == a && order[1] == b && order[2] == c);
        CHECK(s.wait(a, -1) == Scheduler::kDone && s.wait(b, -1) == Scheduler::kDone);
    }
    // continuous admission: a request arriving while another runs starts beside it
    {
        Scheduler s(100, 4);
        std::atomic<bool> a_running{false}, b_saw_a{false};
        const long long a = s.submit(Scheduler::kFit, 60, [&] {
            a_running = true;
            sleep_ms(200);
            a_running = false;
        });
        sleep_ms(30);
        const long long b = s.submit(Scheduler::kPredict, 30, [&] { b_saw_a = a_running.load(); });
        CHECK(s.wait(b, 1.0) == Scheduler::kDone);
        CHECK(b_saw_a.load());  // b ran while a was still on
        // c does not fit beside a (60 + 50): it starts only once a finishes
        std::atomic<bool> c_saw_a{true};
        const long long c = s.submit(Scheduler::kFit, 50, [&] { c_saw_a = a_running.load(); });
        CHECK(s.wait(c, -1) == Scheduler::kDone);
        CHECK(!c_saw_a.load());
        CHECK(s.wait(a, -1) == Scheduler::kDone);
    }
    // one key at a time: a predict queued behind its model's fit starts after the fit ends,
    // and the queue keeps arrival order
    {
        Scheduler s(100, 4);
        std::atomic<bool> fit_running{false}, predict_saw_fit{true};
        int model = 0;
        const uintptr_t key = reinterpret_cast<uintptr_t>(&model);
        const long long f = s.submit(Scheduler::kFit, 10, [&] {
            fit_running = true;
            sleep_ms(100);
            fit_running = false;
        }, key);
        const long long p = s.submit(Scheduler::kPredict, 10, [&] { predict_saw_fit = fit_running.load(); }, key);
        const long long o = s.submit(Scheduler::kPredict, 10, [] {});  // other key: behind p in the queue
        CHECK(s.wait(p, -1) == Scheduler::kDone && !predict_saw_fit.load());
        CHECK(s.wait(f, -1) == Scheduler::kDone && s.wait(o, -1) == Scheduler::kDone);
        const auto order = s.start_order();
        CHECK(order.size() == 3 && order[0] == f && order[1] == p && order[2] == o);
    }
    // failures are reported per request; the others complete
    {
        Scheduler s(100, 2);
        const long long a = s.submit(Scheduler::kFit, 10, [] { throw std::runtime_error("bad config"); });
        const long long b = s.submit(Scheduler::kFit, 10, [] { sleep_ms(5); });
        std::string err;
        CHECK(s.wait(a, -1, &err) == Scheduler::kFailed && err == "bad config");
        CHECK(s.wait(b, -1) == Scheduler::kDone);
        const auto st = s.stats();
        CHECK(st.failed == 1 && st.completed == 1);
    }
    // a request larger than the whole budget is refused at submission
    {
        Scheduler s(100, 2);
        bool threw = false;
        try {
            s.submit(Scheduler::kFit, 101, [] {});
        } catch (const std::runtime_error&) {
            threw = true;
        }
        CHECK(threw);
    }
    // wait with a timeout reports a request still running
    {
        Scheduler s(100, 1);
        const long long a = s.submit(Scheduler::kFit, 10, [] { sleep_ms(300); });
        const long long b = s.submit(Scheduler::kFit, 10, [] {});
        for (int k = 0; k < 1000 && s.start_order().empty(); ++k) sleep_ms(1);  // a has started
        CHECK(s.wait(b, 0.01) == Scheduler::kQueued);
        CHECK(s.wait(a, 0.01) == Scheduler::kRunning);
        CHECK(s.wait(b, -1) == Scheduler::kDone);
    }
    // latency quantiles: nearest rank
    {
        std::vector<double> v;
        for (int k = 1; k <= 100; ++k) v.push_back(k);
        CHECK(Scheduler::quantile(v, 0.5) == 50 && Scheduler::quantile(v, 0.99) == 99);
        CHECK(Scheduler::quantile({7.0}, 0.99) == 7.0 && Scheduler::quantile({}, 0.5) == 0.0);
        Scheduler s(100, 2);
        std::vector<long long> ids;
        for (int k = 0; k < 6; ++k) ids.push_back(s.submit(k % 2 ? Scheduler::kPredict : Scheduler::kFit, 10,
                                                           [k] { sleep_ms(5 + 5 * k); }));
        for (long long id : ids) s.wait(id, -1);
        const auto st = s.stats();
        CHECK(st.completed == 6 && st.p99_s >= st.p50_s && st.p50_s > 0 && st.p99_fit_s > 0 && st.p99_predict_s > 0);
        CHECK(st.busy_s >= st.p99_s * 0.99);
    }
    std::printf("ok\n");
    return 0;
}

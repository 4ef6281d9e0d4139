// The host codec's thread pool (see pool.h).
#include "pool.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace gb {

namespace {

struct Call {
    const std::function<void(int)>* fn;
    int n;
    std::atomic<int> next{0}, done{0};
    std::mutex m;
    std::condition_variable cv;
    std::exception_ptr error;
    // runs items until none is left to take; true when this thread ran the last one
    void work() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) return;
            try {
                (*fn)(i);
            } catch (...) {
                std::lock_guard<std::mutex> lock(m);
                if (!error) error = std::current_exception();
            }
            if (done.fetch_add(1) + 1 == n) {
                std::lock_guard<std::mutex> lock(m);
                cv.notify_all();
            }
        }
    }
};

class Pool {
public:
    Pool() {
        const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
        resize((int)std::min(4u, hw / 4));
    }
    ~Pool() { resize(0); }
    void resize(int n) {
        {
            std::lock_guard<std::mutex> lock(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
        threads_.clear();
        stop_ = false;
        for (int i = 0; i < n; ++i) threads_.emplace_back([this] { loop(); });
    }
    int size() const { return (int)threads_.size(); }
    void run(Call& c) {
        const int helpers = std::min((int)threads_.size(), c.n - 1);
        if (helpers > 0) {
            std::lock_guard<std::mutex> lock(m_);
            for (int i = 0; i < helpers; ++i) q_.push_back(&c);
        }
        cv_.notify_all();
        c.work();
        {
            std::unique_lock<std::mutex> lock(c.m);
            c.cv.wait(lock, [&] { return c.done.load() == c.n; });
        }  // released: the helper that ran the last item may still be taking it to notify
        // entries of the call still queued come out, and helpers still inside the call are
        // waited for, before the call's storage goes away
        std::unique_lock<std::mutex> ql(m_);
        q_.erase(std::remove(q_.begin(), q_.end(), &c), q_.end());
        while (busyWith(&c)) {
            ql.unlock();
            std::this_thread::yield();
            ql.lock();
        }
    }

private:
    bool busyWith(Call* c) { return std::count(active_.begin(), active_.end(), c) > 0; }
    void loop() {
        for (;;) {
            Call* c;
            {
                std::unique_lock<std::mutex> lock(m_);
                cv_.wait(lock, [&] { return stop_ || !q_.empty(); });
                if (stop_) return;
                c = q_.front();
                q_.pop_front();
                active_.push_back(c);
            }
            c->work();
            std::lock_guard<std::mutex> lock(m_);
            active_.erase(std::find(active_.begin(), active_.end(), c));
        }
    }
    std::mutex m_;
    std::condition_variable cv_;
    std::deque<Call*> q_;
    std::vector<Call*> active_;
    std::vector<std::thread> threads_;
    bool stop_ = false;
};

Pool& pool() {
    static Pool p;
    return p;
}

}  // namespace

void parallelFor(int n, const std::function<void(int)>& fn) {
    if (n <= 0) return;
    if (n == 1 || pool().size() == 0) {
        for (int i = 0; i < n; ++i) fn(i);
        return;
    }
    Call c;
    c.fn = &fn;
    c.n = n;
    pool().run(c);
    if (c.error) std::rethrow_exception(c.error);
}

void setPoolThreads(int n) { pool().resize(std::max(0, std::min(n, 64))); }
int poolThreads() { return pool().size(); }

}  // namespace gb

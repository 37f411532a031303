// WorkPool: a fixed team of host threads that runs one function on every member and waits for
// all of them -- the parallel host passes of the resolver reuse it batch after batch instead of
// starting threads each time.
#pragma once

#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace xkb {

class WorkPool {
public:
    explicit WorkPool(unsigned members) : n_(members ? members : 1)
    {
        for (unsigned k = 1; k < n_; ++k) th_.emplace_back([this, k] { loop(k); });
    }
    ~WorkPool()
    {
        { std::lock_guard<std::mutex> lk(mu_); stop_ = true; }
        cv_.notify_all();
        for (auto & t : th_) t.join();
    }
    WorkPool(const WorkPool &) = delete;
    WorkPool & operator=(const WorkPool &) = delete;

    unsigned size() const { return n_; }

    // fn(k) for every member k in [0, size()); member 0 is the calling thread. Returns when all
    // have returned.
    void run(const std::function<void(unsigned)> & fn)
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            fn_ = &fn;
            left_ = n_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        fn(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [this] { return left_ == 0; });
        fn_ = nullptr;
    }

private:
    void loop(unsigned k)
    {
        unsigned long long seen = 0;
        for (;;)
        {
            const std::function<void(unsigned)> * fn;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                fn = fn_;
            }
            (*fn)(k);
            std::lock_guard<std::mutex> lk(mu_);
            if (--left_ == 0) done_.notify_one();
        }
    }

    unsigned n_;
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(unsigned)> * fn_ = nullptr;
    unsigned left_ = 0;
    unsigned long long gen_ = 0;
    bool stop_ = false;
};

} // namespace xkb

// Host threads for the library's parallel host loops (table totals,
// rarefied replicates, statistics jobs).
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <exception>
#include <mutex>
#include <sched.h>
#include <system_error>
#include <thread>
#include <vector>

namespace ssu {

// Host threads for the library's own parallel loops: OMP_NUM_THREADS when
// set (the reference's OpenMP loops honour it), else the CPUs this process
// may run on (affinity mask, so cgroup/taskset limits hold), at most `cap`.
inline unsigned host_threads(unsigned cap) {
    unsigned n = 0;
    if (const char *v = std::getenv("OMP_NUM_THREADS")) {
        const long x = std::strtol(v, nullptr, 10);
        if (x > 0) n = static_cast<unsigned>(x);
    }
    if (n == 0) {
        cpu_set_t set;
        CPU_ZERO(&set);
        if (sched_getaffinity(0, sizeof(set), &set) == 0) n = static_cast<unsigned>(CPU_COUNT(&set));
    }
    if (n == 0) n = std::thread::hardware_concurrency();
    return std::max(1u, std::min(n, std::max(1u, cap)));
}

// Run fn(i) for i in [0, n) on up to `threads` threads (the caller's included)
// pulling indices from a shared counter.  A thread that cannot be started
// leaves its share to the others; every started thread is joined, also when
// fn throws; the first exception is rethrown on the calling thread.
template <class F>
inline void parallel_for(unsigned n, unsigned threads, F &&fn) {
    std::atomic<unsigned> next{0};
    std::mutex err_mu;
    std::exception_ptr err;
    auto work = [&] {
        try {
            for (unsigned i = next.fetch_add(1); i < n; i = next.fetch_add(1)) fn(i);
        } catch (...) {
            std::lock_guard<std::mutex> lock(err_mu);
            if (!err) err = std::current_exception();
            next.store(n);  // the others stop at their next index
        }
    };
    struct Joiner {
        std::vector<std::thread> v;
        ~Joiner() {
            for (std::thread &t : v)
                if (t.joinable()) t.join();
        }
    } pool;
    for (unsigned t = 1; t < std::min(threads, n); t++) {
        try {
            pool.v.emplace_back(work);
        } catch (const std::system_error &) {
            break;
        }
    }
    work();
    for (std::thread &t : pool.v) t.join();
    if (err) std::rethrow_exception(err);
}

}  // namespace ssu

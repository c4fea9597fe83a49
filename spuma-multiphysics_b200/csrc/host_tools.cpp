// Host-side helpers for callers of the host-array entry points: the
// bookkeeping the reference solver does in its own parallel loops between the
// library calls (src/reactiveFoam/ReactiveFoam.C:419-420 compact, :651-661 the
// transport stage's states, :732-751 the recovery's inputs), here as
// multi-threaded C++ over a persistent worker pool, so a Python or C caller
// does not pay interpreter-speed array passes. No device work.
#include "../../include/reactive_b200_host.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace {

// A fixed pool of workers running one parallel-for at a time over contiguous
// chunks (the calling thread takes a share too).
class Pool {
public:
    Pool() {
        const unsigned n = std::max(1u, std::thread::hardware_concurrency());
        for (unsigned i = 1; i < n; ++i) workers_.emplace_back([this, i] { loop(i); });
        size_ = n;
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> lock(mutex_);
            stop_ = true;
        }
        wake_.notify_all();
        for (auto& t : workers_) t.join();
    }
    // f(begin, end) over [0, count) in size_ chunks.
    void run(size_t count, const std::function<void(size_t, size_t)>& f) {
        if (count < 65536 || size_ == 1) {
            f(0, count);
            return;
        }
        std::lock_guard<std::mutex> serial(serial_);
        {
            std::lock_guard<std::mutex> lock(mutex_);
            task_ = &f;
            count_ = count;
            pending_ = size_ - 1;
            ++generation_;
        }
        wake_.notify_all();
        chunk(0, f);
        std::unique_lock<std::mutex> lock(mutex_);
        done_.wait(lock, [this] { return pending_ == 0; });
        task_ = nullptr;
    }

private:
    void chunk(unsigned i, const std::function<void(size_t, size_t)>& f) {
        const size_t per = (count_ + size_ - 1) / size_, begin = std::min(count_, i * per),
                     end = std::min(count_, begin + per);
        if (begin < end) f(begin, end);
    }
    void loop(unsigned i) {
        unsigned long long seen = 0;
        for (;;) {
            const std::function<void(size_t, size_t)>* task;
            {
                std::unique_lock<std::mutex> lock(mutex_);
                wake_.wait(lock, [&] { return stop_ || generation_ != seen; });
                if (stop_) return;
                seen = generation_;
                task = task_;
            }
            chunk(i, *task);
            {
                std::lock_guard<std::mutex> lock(mutex_);
                if (--pending_ == 0) done_.notify_one();
            }
        }
    }
    std::vector<std::thread> workers_;
    unsigned size_ = 1;
    std::mutex mutex_, serial_;
    std::condition_variable wake_, done_;
    const std::function<void(size_t, size_t)>* task_ = nullptr;
    size_t count_ = 0;
    unsigned pending_ = 0;
    unsigned long long generation_ = 0;
    bool stop_ = false;
};

Pool& pool() {
    static Pool p;
    return p;
}

}  // namespace

extern "C" {

int reactive_b200_host_threads_v3(void) { return int(std::max(1u, std::thread::hardware_concurrency())); }

int reactive_b200_host_copy_v3(void* dst, const void* src, size_t bytes) {
    if (!bytes) return 0;
    if (!dst || !src) return 1;
    auto* d = static_cast<unsigned char*>(dst);
    const auto* s = static_cast<const unsigned char*>(src);
    const size_t blocks = (bytes + 4095) / 4096;
    pool().run(blocks, [&](size_t b, size_t e) {
        const size_t from = b * 4096, to = std::min(bytes, e * 4096);
        std::memcpy(d + from, s + from, to - from);
    });
    return 0;
}

int reactive_b200_host_transport_states_v3(const ReactiveThermoState* thermo, size_t count, const double* q,
                                           size_t qStride, size_t species, ReactiveTransportState* states,
                                           ReactiveTransportPrimitive* primitives) {
    if (!count) return 0;
    if (!thermo || !states || (primitives && (!q || qStride < species + 3 || !species))) return 1;
    pool().run(count, [&](size_t b, size_t e) {
        for (size_t c = b; c < e; ++c) {
            const ReactiveThermoState& s = thermo[c];
            ReactiveTransportState& t = states[c];
            t.p = s.p;
            t.T = s.T;
            t.rho = s.rho;
            t.cv = s.cv;
            t.sound = s.soundFrozen;
            t.gasMass = s.gasMass;
            t.dilatation = 0.0;
            if (primitives) {
                const double* row = q + c * qStride;
                ReactiveTransportPrimitive& p = primitives[c];
                p.rho = s.rho;
                for (int d = 0; d < 3; ++d) p.u[d] = row[species + d] / s.rho;
            }
        }
    });
    return 0;
}

int reactive_b200_host_recovery_inputs_v3(const double* q, size_t count, size_t qStride, size_t species,
                                          double* masses, double* energy) {
    if (!count) return 0;
    if (!q || !energy || !species || qStride < species + 4) return 1;
    pool().run(count, [&](size_t b, size_t e) {
        for (size_t c = b; c < e; ++c) {
            const double* row = q + c * qStride;
            double rho = 0;
            for (size_t k = 0; k < species; ++k) {
                rho += row[k];
                if (masses) masses[c * species + k] = row[k];
            }
            const double mx = row[species], my = row[species + 1], mz = row[species + 2];
            energy[c] = row[species + 3] - .5 * (mx * mx + my * my + mz * mz) / rho;
        }
    });
    return 0;
}

}  // extern "C"

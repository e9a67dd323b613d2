// Host side of qpd_run_host: worker threads that pack the reference's float64 host arrays into the
// kernel input layout, so only the packed bytes cross PCIe.
//
// The reference hands diffraction() float64 planes (src/python/diffraction.py:62-74): 8 bytes per
// value, 72 bytes per cell with two phases and a region.  The kernels read P and u in the plan
// precision, an int8 phase index and one weight per cell: 29 bytes per cell in float32.  Packing on
// the host, chunk by chunk into a pinned ring while earlier chunks are copied, moves 2.5x fewer
// bytes over the link.  The arithmetic is the GPU pack kernel's (pack_kernel): every packed value
// is bit-identical to what qpd_pack_device would write.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace qpd {

// A fixed set of threads running one parallel-for at a time.
class Workers {
   public:
    explicit Workers(int n) {
        for (int i = 0; i < n; i++) th_.emplace_back([this] { loop(); });
    }
    ~Workers() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    int size() const { return (int)th_.size(); }

    // f(i) for i in [0, count), spread over the workers and the calling thread; returns when done.
    void parallel(int count, const std::function<void(int)>& f) {
        if (count <= 0) return;
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &f;
            count_ = count;
            next_.store(0);
            left_ = count;
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> g(m_);
        done_.wait(g, [this] { return left_ == 0; });
        job_ = nullptr;
    }

   private:
    void work() {
        for (;;) {
            const int i = next_.fetch_add(1);
            if (i >= count_) return;
            (*job_)(i);
            std::lock_guard<std::mutex> g(m_);
            if (--left_ == 0) done_.notify_all();
        }
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return stop_ || (gen_ != seen && job_ != nullptr); });
                if (stop_) return;
                seen = gen_;
            }
            work();
        }
    }
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    std::atomic<int> next_{0};
    int count_ = 0, left_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

// Planes of one packed chunk in a pinned slot: P[3], U[3], weight, then either the phase index
// (single mode) or nPhase dense weight planes (dense mode) in the space after the weight.
template <typename T> struct HostChunk {
    T* P;
    T* U;
    T* W;
    int8_t* ph;
    T* WD;       // nPhase planes, dense mode only
    int64_t cap;  // cells per plane
    static size_t bytes(int64_t cap, int nPhase, bool dense) {
        return (sizeof(T) * 7 + 1) * (size_t)cap + (dense ? sizeof(T) * nPhase * (size_t)cap : 0) + 64;
    }
    static HostChunk at(void* base, int64_t cap) {
        HostChunk h;
        h.cap = cap;
        h.P = static_cast<T*>(base);
        h.U = h.P + 3 * cap;
        h.W = h.U + 3 * cap;
        h.WD = h.W + cap;
        h.ph = reinterpret_cast<int8_t*>(h.WD);
        return h;
    }
};

// Pack cells [g0 + i0, g0 + i1) of the float64 planes into chunk slot positions [i0, i1); returns
// the pack flags (bit 0: a cell has several phases with weight, bit 1: a weight other than 0, 1).
// Same arithmetic as pack_kernel: T(value), weight = T(oPhase_p * region) in double.
template <typename T>
uint32_t host_pack(const HostChunk<T>& h, int64_t n, int64_t g0, int64_t i0, int64_t i1, int nStruc, int nPhase,
                   const double* oPhase, const double* oStruc, const double* u, const double* region, bool dense) {
    uint32_t f = 0;
    for (int k = 0; k < 3; k++) {
        T* dp = h.P + k * h.cap;
        T* du = h.U + k * h.cap;
        const double* sp = k < nStruc ? oStruc + k * n + g0 : nullptr;
        const double* su = u + k * n + g0;
        for (int64_t i = i0; i < i1; i++) {
            dp[i] = sp ? T(sp[i]) : T(0);
            du[i] = T(su[i]);
        }
    }
    if (dense) {
        for (int p = 0; p < nPhase; p++) {
            const double* op = oPhase + p * n + g0;
            T* dw = h.WD + p * h.cap;
            for (int64_t i = i0; i < i1; i++) dw[i] = T(op[i] * (region ? region[g0 + i] : 1.0));
        }
        return 0;
    }
    for (int64_t i = i0; i < i1; i++) {
        const double r = region ? region[g0 + i] : 1.0;
        int which = -1;
        double w = 0.0;
        for (int p = 0; p < nPhase; p++) {
            const double wp = oPhase[p * n + g0 + i] * r;
            if (wp != 0.0) {
                if (which >= 0) f |= 1u;
                else {
                    which = p;
                    w = wp;
                }
            }
        }
        if (which >= 0 && w != 1.0) f |= 2u;
        h.ph[i] = (int8_t)which;
        h.W[i] = T(w);
    }
    return f;
}

}  // namespace qpd

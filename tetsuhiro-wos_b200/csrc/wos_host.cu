// wos_host.cu -- host-side staging of pageable fields.
//
// A Go caller passes its fields as ordinary (pageable) slices.  The driver
// copies pageable memory through its own small bounce buffer, one direction at
// a time, at a fraction of the PCIe rate (2048^2 complex128: 107 fields/s
// against 650 from page-locked memory).  For such fields the host batch
// instead converts on a pool of host threads into page-locked staging owned
// by the context, in the context's precision: complex64 for a WOS_FP32
// context, which the pipeline rounds to anyway (IEEE round to nearest, the
// same rounding the first sweep applies), so half the bytes cross PCIe and
// the results are bit-identical; complex128 copies for WOS_FP64.  The
// conversions of one field run on the host while the GPU works on the others.
#include <condition_variable>
#include <functional>
#include <thread>

#include "wos_api_internal.cuh"

namespace wapi {

// A fixed set of worker threads running one job at a time: run(f) calls
// f(k) for k in [0, size()), k = 0 on the calling thread.
class HostPool {
  public:
    explicit HostPool(int n) : n_(n < 1 ? 1 : n) {
        for (int i = 1; i < n_; i++) th_.emplace_back([this, i] { loop(i); });
    }
    ~HostPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    int size() const { return n_; }
    void run(const std::function<void(int)>& f) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &f;
            left_ = n_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        f(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return left_ == 0; });
        job_ = nullptr;
    }

  private:
    void loop(int i) {
        long long seen = 0;
        for (;;) {
            const std::function<void(int)>* f;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                f = job_;
            }
            (*f)(i);
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (--left_ == 0) done_.notify_one();
            }
        }
    }
    int n_;
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int left_ = 0;
    long long gen_ = 0;
    bool stop_ = false;
};

HostPool& pool_of(wos_ctx c) {
    if (!c->host_pool) {
        int n = env_int("WOS_HOST_THREADS", 0);
        if (n <= 0) n = std::min(16, std::max(1, (int)std::thread::hardware_concurrency()));
        c->host_pool = new HostPool(n);
    }
    return *static_cast<HostPool*>(c->host_pool);
}

void host_release(wos_ctx c) {
    delete static_cast<HostPool*>(c->host_pool);
    c->host_pool = nullptr;
    for (int i = 0; i < wos_ctx_s::kSlots; i++) {
        if (c->hst[i]) cudaFreeHost(c->hst[i]);
        c->hst[i] = nullptr;
        c->hst_n[i] = 0;
    }
}

bool host_pageable(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

int host_stage(wos_ctx c, int slot, size_t bytes) {
    if (c->hst_n[slot] >= bytes && c->hst[slot]) return WOS_OK;
    if (c->hst[slot]) cudaFreeHost(c->hst[slot]);
    c->hst[slot] = nullptr;
    c->hst_n[slot] = 0;
    CK(cudaHostAlloc(&c->hst[slot], bytes, cudaHostAllocDefault));
    c->hst_n[slot] = bytes;
    return WOS_OK;
}

// Components of f, complex128, into dst in the context's complex type
// ([ncomp][ny][nx]), or back (to_host), on the context's host threads.
void host_convert(wos_ctx c, wos_field& f, void* dst, bool to_host) {
    HostPool& pool = pool_of(c);
    const size_t np = (size_t)f.ny * f.nx;
    const int ncomp = f.polarized ? 2 : 1;
    const int nt = pool.size();
    const size_t chunk = ((np + nt - 1) / nt + 63) / 64 * 64;
    pool.run([&](int k) {
        const size_t b = std::min(np, (size_t)k * chunk), e = std::min(np, b + chunk);
        for (int q = 0; q < ncomp; q++) {
            wos_c128* h = q == 0 ? f.ex : f.ey;
            if (c->fp64) {
                wos_c128* s = static_cast<wos_c128*>(dst) + q * np;
                if (to_host) std::memcpy(h + b, s + b, (e - b) * sizeof(wos_c128));
                else std::memcpy(s + b, h + b, (e - b) * sizeof(wos_c128));
            } else {
                float2* s = static_cast<float2*>(dst) + q * np;
                if (to_host) {
                    for (size_t i = b; i < e; i++) h[i] = wos_c128{(double)s[i].x, (double)s[i].y};
                } else {
                    for (size_t i = b; i < e; i++) s[i] = make_float2((float)h[i].re, (float)h[i].im);
                }
            }
        }
    });
}

}  // namespace wapi

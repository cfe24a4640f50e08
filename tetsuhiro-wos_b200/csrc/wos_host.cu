// wos_host.cu -- the host-field batch (wos_propagate_batch) and the
// host-side staging of pageable fields.
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
#include <emmintrin.h>

#include <condition_variable>
#include <cstdint>
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

// complex128 [b, e) -> complex64 and back, two values per SSE2 step; the
// stores bypass the caches (streaming stores: the staging and the caller's
// field are each written once and read by someone else next), which saves
// the read-for-ownership traffic of an ordinary store.  Both conversions
// round or widen exactly as the scalar casts do.
void narrow_c128(const wos_c128* h, float2* s, size_t b, size_t e) {
    size_t i = b;
    const bool al = ((reinterpret_cast<uintptr_t>(h) | reinterpret_cast<uintptr_t>(s)) & 15) == 0;
    if (al && (i & 1)) {
        s[i] = make_float2((float)h[i].re, (float)h[i].im);
        i++;
    }
    if (al) {
        for (; i + 2 <= e; i += 2) {
            const __m128 lo = _mm_cvtpd_ps(_mm_load_pd(&h[i].re));
            const __m128 hi = _mm_cvtpd_ps(_mm_load_pd(&h[i + 1].re));
            _mm_stream_ps(reinterpret_cast<float*>(s + i), _mm_movelh_ps(lo, hi));
        }
        _mm_sfence();
    }
    for (; i < e; i++) s[i] = make_float2((float)h[i].re, (float)h[i].im);
}

void widen_c64(const float2* s, wos_c128* h, size_t b, size_t e) {
    size_t i = b;
    const bool al = ((reinterpret_cast<uintptr_t>(h) | reinterpret_cast<uintptr_t>(s)) & 15) == 0;
    if (al && (i & 1)) {
        h[i] = wos_c128{(double)s[i].x, (double)s[i].y};
        i++;
    }
    if (al) {
        for (; i + 2 <= e; i += 2) {
            const __m128 v = _mm_load_ps(reinterpret_cast<const float*>(s + i));
            _mm_stream_pd(&h[i].re, _mm_cvtps_pd(v));
            _mm_stream_pd(&h[i + 1].re, _mm_cvtps_pd(_mm_movehl_ps(v, v)));
        }
        _mm_sfence();
    }
    for (; i < e; i++) h[i] = wos_c128{(double)s[i].x, (double)s[i].y};
}

// complex128 [b, e) copied with streaming stores (one value per SSE2 step),
// the complex128 pipeline's staging in both directions: like the conversions,
// it writes memory that the DMA engine or the caller reads next
void copy_c128(const wos_c128* src, wos_c128* dst, size_t b, size_t e) {
    if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) != 0) {
        std::memcpy(dst + b, src + b, (e - b) * sizeof(wos_c128));
        return;
    }
    for (size_t i = b; i < e; i++) _mm_stream_pd(&dst[i].re, _mm_load_pd(&src[i].re));
    _mm_sfence();
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
                if (to_host) copy_c128(s, h, b, e);
                else copy_c128(h, s, b, e);
            } else {
                float2* s = static_cast<float2*>(dst) + q * np;
                if (to_host) widen_c64(s, h, b, e);
                else narrow_c128(h, s, b, e);
            }
        }
    });
}

}  // namespace wapi

extern "C" {

// PropagateBatch over host fields (no counterpart in the reference, which
// propagates one field per call): copies and sweeps of consecutive fields
// overlap; pageable fields go through the context's page-locked staging.
int wos_propagate_batch(wos_ctx c, int nfields, wos_field* fields, double z, int method, const wos_context* cci,
                        wos_diag* diags) {
    if (!c || nfields < 0 || (nfields > 0 && !fields)) return fail(WOS_INVALID_ARG, "batch arguments");
    if (method < WOS_ASM || method > WOS_FRAUNHOFER) return fail(WOS_UNKNOWN_METHOD, "unknown propagation method");
    for (int i = 0; i < nfields; i++) TRY(check_field(&fields[i]));
    if (nfields == 0) return WOS_OK;
    const wos_context cc = cci ? *cci : default_context();
    if (z == 0) {
        for (int i = 0; i < nfields && diags; i++) {
            std::memset(&diags[i], 0, sizeof(diags[i]));
            diags[i].dx_out = fields[i].dx;
        }
        return WOS_OK;
    }
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    if (!c->pipe_made) {
        CK(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
        for (int i = 0; i < wos_ctx_s::kSlots; i++) {
            CK(cudaEventCreateWithFlags(&c->in_ev[i], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&c->done_ev[i], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&c->free_ev[i], cudaEventDisableTiming));
            CK(cudaEventRecord(c->free_ev[i], c->d2h));
        }
        c->pipe_made = true;
    }
    bool staged = false;
    for (int i = 0; i < nfields; i++)
        staged = staged || host_pageable(fields[i].ex) || (fields[i].polarized && host_pageable(fields[i].ey));
    if (staged) {
        // pageable fields: host threads convert field i into the slot's
        // page-locked staging (context precision), then copy, sweep and copy
        // back; field i - kSlots is converted back when its slot comes round,
        // so the host converts while the GPU runs the fields before it
        const size_t esz = c->csz();
        auto drain = [&](int j) -> int {
            const int sl = j % wos_ctx_s::kSlots;
            CK(cudaEventSynchronize(c->free_ev[sl]));
            host_convert(c, fields[j], c->hst[sl], true);
            return WOS_OK;
        };
        int rc = WOS_OK;
        for (int i = 0; i < nfields && rc == WOS_OK; i++) {
            const int sl = i % wos_ctx_s::kSlots;
            if (i >= wos_ctx_s::kSlots && (rc = drain(i - wos_ctx_s::kSlots)) != WOS_OK) break;
            wos_field& f = fields[i];
            const int ncomp = f.polarized ? 2 : 1;
            const size_t bytes = (size_t)f.ny * f.nx * ncomp * esz;
            if ((rc = host_stage(c, sl, bytes)) != WOS_OK || (rc = ensure(c->slot[sl], bytes)) != WOS_OK) break;
            host_convert(c, f, c->hst[sl], false);
            CK(cudaMemcpyAsync(c->slot[sl].p, c->hst[sl], bytes, cudaMemcpyHostToDevice, c->h2d));
            CK(cudaEventRecord(c->in_ev[sl], c->h2d));
            CK(cudaStreamWaitEvent(c->st, c->in_ev[sl], 0));
            wos_diag local;
            wos_diag* d = diags ? &diags[i] : (method == WOS_FRAUNHOFER ? &local : nullptr);
            Prop p{f.ny, f.nx, f.dx, ncomp, c->slot[sl].p, 0, c->slot[sl].p, 0, z, method, cc, d};
            if ((rc = run_propagate(c, p)) != WOS_OK) break;
            if (method == WOS_FRAUNHOFER) f.dx = d->dx_out;
            CK(cudaEventRecord(c->done_ev[sl], c->st));
            CK(cudaStreamWaitEvent(c->d2h, c->done_ev[sl], 0));
            CK(cudaMemcpyAsync(c->hst[sl], c->slot[sl].p, bytes, cudaMemcpyDeviceToHost, c->d2h));
            CK(cudaEventRecord(c->free_ev[sl], c->d2h));
        }
        for (int j = std::max(0, nfields - wos_ctx_s::kSlots); j < nfields && rc == WOS_OK; j++) rc = drain(j);
        cudaStreamSynchronize(c->h2d);
        cudaStreamSynchronize(c->d2h);
        CK(cudaMemcpyAsync(c->err_host, c->err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        if (rc != WOS_OK) return rc;
        return check_err_word(c);
    }
    // field i lives in slot i % kSlots from its upload to its download; the
    // upload of the next field is queued before field i's sweeps, so the two
    // copy directions and the sweeps overlap (the sweeps stay in order on the
    // context stream and share its workspace)
    auto bytes_of = [&](int i) {
        return (size_t)fields[i].ny * fields[i].nx * 16 * (fields[i].polarized ? 2 : 1);
    };
    auto upload = [&](int i) -> int {
        const int sl = i % wos_ctx_s::kSlots;
        const wos_field& f = fields[i];
        const size_t np = (size_t)f.ny * f.nx;
        CK(cudaStreamWaitEvent(c->h2d, c->free_ev[sl], 0));
        TRY(ensure(c->slot[sl], bytes_of(i)));
        CK(cudaMemcpyAsync(c->slot[sl].p, f.ex, np * 16, cudaMemcpyHostToDevice, c->h2d));
        if (f.polarized)
            CK(cudaMemcpyAsync(reinterpret_cast<char*>(c->slot[sl].p) + np * 16, f.ey, np * 16,
                               cudaMemcpyHostToDevice, c->h2d));
        CK(cudaEventRecord(c->in_ev[sl], c->h2d));
        return WOS_OK;
    };
    int rc = upload(0);
    for (int i = 0; i < nfields && rc == WOS_OK; i++) {
        const int sl = i % wos_ctx_s::kSlots;
        if (i + 1 < nfields) {
            rc = upload(i + 1);
            if (rc != WOS_OK) break;
        }
        wos_field& f = fields[i];
        const size_t np = (size_t)f.ny * f.nx;
        const int ncomp = f.polarized ? 2 : 1;
        CK(cudaStreamWaitEvent(c->st, c->in_ev[sl], 0));
        wos_diag local;
        wos_diag* d = diags ? &diags[i] : (method == WOS_FRAUNHOFER ? &local : nullptr);
        Prop p{f.ny, f.nx, f.dx, ncomp, c->slot[sl].p, 1, c->slot[sl].p, 1, z, method, cc, d};
        rc = run_propagate(c, p);
        if (rc != WOS_OK) break;
        if (method == WOS_FRAUNHOFER) f.dx = d->dx_out;
        CK(cudaEventRecord(c->done_ev[sl], c->st));
        CK(cudaStreamWaitEvent(c->d2h, c->done_ev[sl], 0));
        CK(cudaMemcpyAsync(f.ex, c->slot[sl].p, np * 16, cudaMemcpyDeviceToHost, c->d2h));
        if (ncomp == 2)
            CK(cudaMemcpyAsync(f.ey, reinterpret_cast<char*>(c->slot[sl].p) + np * 16, np * 16,
                               cudaMemcpyDeviceToHost, c->d2h));
        CK(cudaEventRecord(c->free_ev[sl], c->d2h));
    }
    cudaStreamSynchronize(c->h2d);
    cudaStreamSynchronize(c->d2h);
    CK(cudaMemcpyAsync(c->err_host, c->err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (rc != WOS_OK) return rc;
    return check_err_word(c);
}

}  // extern "C"

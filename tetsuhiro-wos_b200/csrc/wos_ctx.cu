// wos_ctx.cu -- contexts (device, precision, stream, workspaces), their
// settings and profiling counters, CUDA graphs of device-resident calls and
// the launch-configuration tuner of the specialised sweeps.
#include <algorithm>

#include "wos_api_internal.cuh"

extern "C" {

// A captured CUDA graph of device-resident calls and its executable.
struct wos_graph_s {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
};

const char* wos_backend_info(void) { return "B200 native (sm_100a): hand-written Stockham/Bluestein FFT, fused ASM sweeps"; }

int wos_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int wos_device_name(int device, char* buf, int buflen) {
    if (!buf || buflen <= 0) return fail(WOS_INVALID_ARG, "null buffer");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    std::snprintf(buf, (size_t)buflen, "%s", prop.name);
    return WOS_OK;
}

int wos_ctx_create(int device, int precision, wos_ctx* out) {
    if (!out) return fail(WOS_INVALID_ARG, "null out");
    *out = nullptr;
    if (precision != WOS_FP32 && precision != WOS_FP64) return fail(WOS_INVALID_ARG, "precision");
    int n = wos_device_count();
    if (n <= 0) return fail(WOS_NOT_INITIALISED, "no CUDA device");
    if (device < 0 || device >= n) return fail(WOS_INVALID_ARG, "device index");
    wos_ctx c = new wos_ctx_s();
    c->device = device;
    c->fp64 = precision == WOS_FP64;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return fail(WOS_CUDA_ERROR, std::string("context creation: ") + cudaGetErrorString(e));
    }
    c->own_stream = true;
    e = cudaMalloc(&c->err_dev, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(c->err_dev, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMallocHost(&c->err_host, sizeof(unsigned));
    if (e != cudaSuccess) {
        if (c->err_dev) cudaFree(c->err_dev);
        cudaStreamDestroy(c->st);
        delete c;
        return fail(WOS_CUDA_ERROR, std::string("context creation: ") + cudaGetErrorString(e));
    }
    *c->err_host = 0;
    c->col_pair = env_int("WOS_COLPAIR", 0);
    c->tiled = env_int("WOS_TILED", 1);
    c->bpm_comp = env_int("WOS_BPM_COMP", 1);
    c->htab_on = env_int("WOS_HTAB", 1);
    c->htab_reg = env_int("WOS_HTAB_REG", 1);
    c->out_stream = env_int("WOS_OUT_STREAM", 1);
    *out = c;
    return WOS_OK;
}

// A context destroyed in the middle of a capture: a branch leaves its
// owner's list (the owner's capture then fails at its end); an owner ends its
// capture (discarding the graph) and releases its branches, which keep no
// pointer to it.
static void capture_release(wos_ctx c) {
    wos_ctx owner = nullptr;
    std::vector<wos_ctx> open;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        owner = c->cap_owner;
        open.swap(c->cap_open);
        if (c->capturing && !owner) {
            cudaSetDevice(c->device);
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(c->st, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
        }
        c->capturing = false;
        c->cap_owner = nullptr;
    }
    if (owner) {
        std::lock_guard<std::mutex> lk(owner->mu);
        owner->cap_open.erase(std::remove(owner->cap_open.begin(), owner->cap_open.end(), c), owner->cap_open.end());
    }
    for (wos_ctx b : open) {
        std::lock_guard<std::mutex> lk(b->mu);
        b->capturing = false;
        b->cap_owner = nullptr;
    }
}

int wos_ctx_destroy(wos_ctx c) {
    if (!c) return WOS_OK;
    comm_release(c);
    capture_release(c);
    {
        std::lock_guard<std::mutex> lk(c->mu);
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->st);
        if (c->pipe_made) {
            cudaStreamSynchronize(c->h2d);
            cudaStreamSynchronize(c->d2h);
        }
        host_release(c);
        for (int pr = 0; pr < 2; pr++)
            for (auto& kv : c->axes[pr]) {
                cudaFree(kv.second.tw);
                if (kv.second.chirp) cudaFree(kv.second.chirp);
                if (kv.second.bf) cudaFree(kv.second.bf);
                if (kv.second.bi) cudaFree(kv.second.bi);
                for (void* t : kv.second.ftw)
                    if (t) cudaFree(t);
                for (void* t : kv.second.ftw_lo)
                    if (t) cudaFree(t);
                if (kv.second.ptw) cudaFree(kv.second.ptw);
            }
        for (auto& h : c->htab)
            if (h.buf.p) cudaFree(h.buf.p);
        for (auto& ps : c->pslot)
            if (ps.buf.p) cudaFree(ps.buf.p);
        DevBuf* bufs[] = {&c->stage, &c->scratch, &c->scratch2, &c->scratch3, &c->red, &c->redout, &c->tmp,
                          &c->maps, &c->params, &c->vol, &c->accum, &c->aux};
        for (DevBuf* b : bufs)
            if (b->p) cudaFree(b->p);
        for (DevBuf& b : c->tsc)
            if (b.p) cudaFree(b.p);
        if (c->bpm_tab.p) cudaFree(c->bpm_tab.p);
        if (c->hred) cudaFreeHost(c->hred);
        if (c->err_dev) cudaFree(c->err_dev);
        if (c->err_host) cudaFreeHost(c->err_host);
        for (int i = 0; i < c->naux; i++) {
            cudaStreamDestroy(c->side[i]);
            cudaEventDestroy(c->join_ev[i]);
        }
        if (c->fork_ev) cudaEventDestroy(c->fork_ev);
        if (c->cap_ev) cudaEventDestroy(c->cap_ev);
        if (c->pipe_made) {
            cudaStreamDestroy(c->h2d);
            cudaStreamDestroy(c->d2h);
            for (int i = 0; i < wos_ctx_s::kSlots; i++) {
                if (c->slot[i].p) cudaFree(c->slot[i].p);
                cudaEventDestroy(c->in_ev[i]);
                cudaEventDestroy(c->done_ev[i]);
                cudaEventDestroy(c->free_ev[i]);
            }
        }
        if (c->prof_made)
            for (int i = 0; i < wos_ctx_s::kRing; i++) {
                cudaEventDestroy(c->ev0[i]);
                cudaEventDestroy(c->ev1[i]);
            }
        if (c->own_stream) cudaStreamDestroy(c->st);
    }
    delete c;
    return WOS_OK;
}

int wos_ctx_set_stream(wos_ctx c, void* stream) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->own_stream) {
        cudaStreamSynchronize(c->st);
        cudaStreamDestroy(c->st);
        c->own_stream = false;
    }
    c->st = reinterpret_cast<cudaStream_t>(stream);
    return WOS_OK;
}

void* wos_ctx_get_stream(wos_ctx c) { return c ? reinterpret_cast<void*>(c->st) : nullptr; }

int wos_ctx_precision(wos_ctx c) { return c ? (c->fp64 ? WOS_FP64 : WOS_FP32) : -1; }

int wos_ctx_set_col_width(wos_ctx c, int w) {
    if (!c || w < 0 || (w > 0 && (w & (w - 1)))) return fail(WOS_INVALID_ARG, "column width must be 0 or a power of two");
    c->colw = w;
    return WOS_OK;
}

int wos_ctx_set_profiling(wos_ctx c, int on) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    if (on && !c->prof_made) {
        CK(cudaSetDevice(c->device));
        for (int i = 0; i < wos_ctx_s::kRing; i++) {
            CK(cudaEventCreate(&c->ev0[i]));
            CK(cudaEventCreate(&c->ev1[i]));
            c->ev_used[i] = false;
        }
        c->prof_made = true;
    }
    c->prof_on = on != 0;
    return WOS_OK;
}

int wos_ctx_profile(wos_ctx c, int kind, double* total_ms, long long* launches) {
    if (!c || kind < 0 || kind > 7) return fail(WOS_INVALID_ARG, "profile kind");
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->prof_made)
        for (int i = 0; i < wos_ctx_s::kRing; i++) prof_fold(c, i);
    if (total_ms) *total_ms = c->prof_ms[kind];
    if (launches) *launches = c->prof_n[kind];
    return WOS_OK;
}

int wos_ctx_profile_reset(wos_ctx c) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->prof_made)
        for (int i = 0; i < wos_ctx_s::kRing; i++) prof_fold(c, i);
    for (int k = 0; k < 8; k++) {
        c->prof_ms[k] = 0;
        c->prof_n[k] = 0;
    }
    c->launches = 0;
    return WOS_OK;
}

long long wos_ctx_launch_count(wos_ctx c) { return c ? c->launches : -1; }

int wos_ctx_synchronize(wos_ctx c) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    CK(cudaMemcpyAsync(c->err_host, c->err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_err_word(c);
}

// ---- FFTs for the remaining fft2D / fft1DAny users

int wos_graph_capture_begin(wos_ctx c) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->capturing) return fail(WOS_INVALID_ARG, "capture begin: ctx is already capturing");
    TRY(set_device(c));
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
    c->capturing = true;  // tables and parameter lists used from here on stay as the graph reads them
    return WOS_OK;
}

// A branch of a capture: the other context's stream waits on an event of the
// capturing stream, which makes it part of the same capture (its calls are
// recorded as nodes that depend only on what ctx recorded before the fork);
// the join records an event on the branch and has the capturing stream wait
// on it.  Contexts are locked one at a time, capturing context first.
int wos_graph_capture_fork(wos_ctx c, wos_ctx o) {
    if (!c || !o || c == o) return fail(WOS_INVALID_ARG, "capture fork: two distinct contexts");
    if (c->device != o->device) return fail(WOS_INVALID_ARG, "capture fork: contexts on different devices");
    cudaStream_t cst;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        if (!c->capturing || c->cap_owner) return fail(WOS_INVALID_ARG, "capture fork: ctx is not capturing");
        TRY(set_device(c));
        if (!c->cap_ev) CK(cudaEventCreateWithFlags(&c->cap_ev, cudaEventDisableTiming));
        CK(cudaEventRecord(c->cap_ev, c->st));
        cst = c->st;
    }
    {
        std::lock_guard<std::mutex> lk(o->mu);
        if (o->capturing) return fail(WOS_INVALID_ARG, "capture fork: the other context is already capturing");
        if (o->st == cst) return fail(WOS_INVALID_ARG, "capture fork: both contexts use one stream");
        TRY(set_device(o));
        CK(cudaStreamWaitEvent(o->st, c->cap_ev, 0));
        o->capturing = true;
        o->cap_owner = c;
    }
    std::lock_guard<std::mutex> lk(c->mu);
    c->cap_open.push_back(o);
    return WOS_OK;
}

int wos_graph_capture_join(wos_ctx c, wos_ctx o) {
    if (!c || !o || c == o) return fail(WOS_INVALID_ARG, "capture join: two distinct contexts");
    {
        std::lock_guard<std::mutex> lk(o->mu);
        if (!o->capturing || o->cap_owner != c) return fail(WOS_INVALID_ARG, "capture join: not a branch of ctx");
        TRY(set_device(o));
        if (!o->cap_ev) CK(cudaEventCreateWithFlags(&o->cap_ev, cudaEventDisableTiming));
        CK(cudaEventRecord(o->cap_ev, o->st));
        o->capturing = false;
        o->cap_owner = nullptr;
    }
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    CK(cudaStreamWaitEvent(c->st, o->cap_ev, 0));
    c->cap_open.erase(std::remove(c->cap_open.begin(), c->cap_open.end(), o), c->cap_open.end());
    return WOS_OK;
}

int wos_graph_capture_end(wos_ctx c, wos_graph* out) {
    if (!c || !out) return fail(WOS_INVALID_ARG, "null argument");
    *out = nullptr;
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->cap_owner) return fail(WOS_INVALID_ARG, "capture end: ctx is a branch; join it to its capture instead");
    if (!c->cap_open.empty()) return fail(WOS_INVALID_ARG, "capture end: join every forked context first");
    TRY(set_device(c));
    cudaGraph_t g = nullptr;
    c->capturing = false;
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (e != cudaSuccess || !g) {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        return fail(WOS_CUDA_ERROR, std::string("graph capture failed (a call inside it synchronised or failed): ") +
                                        cudaGetErrorString(e));
    }
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        return fail(WOS_CUDA_ERROR, std::string("graph instantiation: ") + cudaGetErrorString(e));
    }
    wos_graph h = new wos_graph_s();
    h->graph = g;
    h->exec = x;
    h->device = c->device;
    *out = h;
    return WOS_OK;
}

int wos_graph_launch(wos_ctx c, wos_graph g) {
    if (!c || !g) return fail(WOS_INVALID_ARG, "null argument");
    if (g->device != c->device) return fail(WOS_INVALID_ARG, "graph captured on another device");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    CK(cudaGraphLaunch(g->exec, c->st));
    return WOS_OK;
}

int wos_graph_destroy(wos_graph g) {
    if (!g) return WOS_OK;
    cudaSetDevice(g->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return WOS_OK;
}

int wos_ctx_set_fast_path(wos_ctx c, int enabled) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    if (enabled < 0 || enabled > 3) return fail(WOS_INVALID_ARG, "fast path mode is 0, 1, 2 or 3");
    std::lock_guard<std::mutex> lk(c->mu);
    c->no_fast = enabled == 0;
    c->sweep_mode = enabled == 0 ? 1 : enabled;
    return WOS_OK;
}

int wos_ctx_set_tune(wos_ctx c, int ny, int nx, int row_e, int col_e, int col_w) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    if (!fast_supported(c->fp64, nx, row_e) || !fast_supported(c->fp64, ny, col_e) || col_w < 1 ||
        (col_w & (col_w - 1)))
        return fail(WOS_INVALID_ARG, "unsupported launch configuration");
    std::lock_guard<std::mutex> lk(c->mu);
    c->tune[tune_key(c->fp64, ny, nx)] = Tune{row_e, col_e, col_w};
    return WOS_OK;
}

// Times every launch configuration of the specialised ASM sweeps for an
// ny x nx grid on this device (in-place propagations of a scratch field,
// CUDA events on the context stream) and keeps the fastest for the context.
int wos_autotune(wos_ctx c, int ny, int nx, int* row_e, int* col_e, int* col_w) {
    if (!c || ny < 2 || nx < 2) return fail(WOS_INVALID_ARG, "autotune arguments");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long key = tune_key(c->fp64, ny, nx);
    c->tune.erase(key);
    const Tune def = get_tune(c, ny, nx);
    if (!is_pow2(nx) || !is_pow2(ny)) {
        if (row_e) *row_e = def.rowE;
        if (col_e) *col_e = def.colE;
        if (col_w) *col_w = def.colW;
        return WOS_OK;
    }
    const long long np = (long long)ny * nx;
    TRY(ensure(c->aux, (size_t)np * c->csz()));
    CK(cudaMemsetAsync(c->aux.p, 0, (size_t)np * c->csz(), c->st));
    wos_context cc = default_context();
    cc.wavelength = 0.5e-6;
    Prop p{ny, nx, 1e-6, 1, c->aux.p, 0, c->aux.p, 0, 1e-3, WOS_ASM, cc, nullptr};
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // each configuration: two warm-up propagations, then the best of three
    // rounds of ten (single-field timings vary by a few percent from round to
    // round); the default is kept unless another is faster by more than 2 %
    auto time_cfg = [&](const Tune& tn, float* out) {
        c->tune[key] = tn;
        bool ok = true;
        for (int it = 0; it < 2 && ok; it++) ok = run_propagate(c, p) == WOS_OK;
        float bestr = 1e30f;
        for (int round = 0; round < 3 && ok; round++) {
            cudaEventRecord(e0, c->st);
            for (int it = 0; it < 10 && ok; it++) ok = run_propagate(c, p) == WOS_OK;
            cudaEventRecord(e1, c->st);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            bestr = std::min(bestr, ms);
        }
        if (!ok) cudaGetLastError();
        *out = bestr;
        return ok;
    };
    float best = 1e30f, tdef = 1e30f;
    Tune bt = def;
    const int es[2] = {8, 16};
    for (int re : es)
        for (int ce : es)
            for (int w = 1; w <= 16; w <<= 1) {
                if (!fast_supported(c->fp64, nx, re) || !fast_supported(c->fp64, ny, ce)) continue;
                if (fast_col_width(c->fp64, ny, ce, w) != w || fast_col_smem(c->fp64, ny, ce, w) > 220 * 1024) continue;
                float ms = 0;
                if (!time_cfg(Tune{re, ce, w}, &ms)) continue;
                if (re == def.rowE && ce == def.colE && w == def.colW) tdef = ms;
                if (ms < best) {
                    best = ms;
                    bt = Tune{re, ce, w};
                }
            }
    if (tdef <= best * 1.02f) bt = def;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tune[key] = bt;
    if (row_e) *row_e = bt.rowE;
    if (col_e) *col_e = bt.colE;
    // the width the ASM column sweep runs with: tiles of kTileW columns when
    // the tiled intermediate applies (the tuned width then serves the other
    // column sweeps of this grid, such as split-step slices)
    const bool tiled = c->tiled && !c->fp64 && nx % kTileW == 0 && fast_col_width(c->fp64, ny, bt.colE, kTileW) == kTileW;
    if (col_w) *col_w = tiled ? kTileW : bt.colW;
    return WOS_OK;
}

}  // extern "C"

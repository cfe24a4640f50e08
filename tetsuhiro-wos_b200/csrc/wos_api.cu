// wos_api.cu -- the C ABI of libwosgpu.so (include/wos_gpu.h).
//
// Each entry point restates one function of the reference's Go `optics`
// package as a sequence of sm_100a sweeps (wos_kernels.cu).  Host-visible
// behaviour (z == 0 early return, nil-context defaults, evanescent policy,
// warning codes and values) follows the cited reference lines; the numerics
// run on the device, with no CPU fallback.
#include "wos_api_internal.cuh"

namespace wapi {

thread_local std::string g_err;

int fail(int st, const std::string& msg) {
    g_err = msg;
    return st;
}

int ensure(DevBuf& b, size_t bytes) {
    if (b.n >= bytes && b.p) return WOS_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
    if (bytes == 0) return WOS_OK;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(WOS_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    b.n = bytes;
    return WOS_OK;
}

int next_pow2(int n) {
    int m = 1;
    while (m < n) m <<= 1;
    return m;
}

int set_device(wos_ctx c) {
    CK(cudaSetDevice(c->device));
    return WOS_OK;
}

// The pipelined sweeps bound every wait on a copy; one that expired left a bit
// in the context's error word.  Read after a synchronisation that copied the
// word to its pinned mirror; the word is cleared for the calls that follow.
int check_err_word(wos_ctx c) {
    const unsigned w = *c->err_host;
    if (w == 0) return WOS_OK;
    *c->err_host = 0;
    cudaMemsetAsync(c->err_dev, 0, sizeof(unsigned), c->st);
    return fail(WOS_TIMEOUT, "a pipelined sweep gave up waiting for a bulk copy (device error word " +
                                 std::to_string(w) + "); its output is incomplete");
}

void prof_fold(wos_ctx c, int slot) {
    if (!c->ev_used[slot]) return;
    float ms = 0;
    if (cudaEventSynchronize(c->ev1[slot]) == cudaSuccess &&
        cudaEventElapsedTime(&ms, c->ev0[slot], c->ev1[slot]) == cudaSuccess) {
        c->prof_ms[c->ev_kind[slot]] += ms;
        c->prof_n[c->ev_kind[slot]] += 1;
    }
    cudaGetLastError();
    c->ev_used[slot] = false;
}

cudaError_t prof_rows(wos_ctx c, int fp64, const RowArgs& a) {
    return timed_launch(c, a.mode & 3, [&] { return launch_rows(fp64, a, c->st); });
}

cudaError_t prof_cols(wos_ctx c, int fp64, const ColArgs& a) {
    return timed_launch(c, 4 + (a.mode & 3), [&] { return launch_cols(fp64, a, c->st); });
}

bool mixed_radix_ok(int n) {
    if (n < 4 || (n & 1)) return false;
    int m = n;
    for (int f : {2, 3, 5})
        while (m % f == 0) m /= f;
    return m == 1 && !is_pow2(n);
}

int build_axis(wos_ctx c, int n, int fp64, Axis& ax) {
    const size_t cs = fp64 ? 16 : 8;
    ax.n = n;
    // power-of-two lines and 2^a 3^b 5^c lines (a >= 1, a mixed-radix plan)
    // are transformed directly; any other length through Bluestein's chirp
    // convolution on a power-of-two length M >= 2n - 1
    // a mixed-radix line must fit one CTA: n / E threads, and two shared-memory
    // buffers of the line (its passes alternate between them)
    bool mixed = mixed_radix_ok(n);
    if (mixed) {
        const int E = pick_E(fp64, n);
        mixed = n % E == 0 && n / E <= max_threads_for(fp64, E) &&
                2 * row_smem_bytes(fp64, n, E, 1) <= (size_t)227 * 1024;
    }
    ax.blue = (is_pow2(n) || mixed) ? 0 : 1;
    ax.L = ax.blue ? next_pow2(2 * n - 1) : n;
    if (n < 2) return fail(WOS_UNSUPPORTED_SIZE, "line length must be >= 2");
    if (ax.L > (fp64 ? kMaxL64 : kMaxL32))
        return fail(WOS_UNSUPPORTED_SIZE, "line length " + std::to_string(n) + " exceeds the on-chip limit (" +
                                              std::to_string(fp64 ? kMaxL64 : kMaxL32) + " transform points)");
    // mixed-radix lines: the L-point table, then the per-pass tables of the plan
    const size_t ntw = (size_t)ax.L + (mixed ? (size_t)mixed_table_len(ax.L) : 0);
    CK(cudaMalloc(&ax.tw, cs * ntw));
    CK(launch_twiddles(fp64, ax.tw, ax.L, c->st));
    if (mixed) CK(launch_mixed_twiddles(fp64, reinterpret_cast<char*>(ax.tw) + cs * ax.L, ax.L, c->st));
    if (!ax.blue) return WOS_OK;
    CK(cudaMalloc(&ax.chirp, cs * n));
    CK(cudaMalloc(&ax.bf, cs * ax.L));
    CK(cudaMalloc(&ax.bi, cs * ax.L));
    // b0 kernels in FP64, transformed with the FP64 power-of-two axis of M
    Axis* m64 = nullptr;
    TRY(get_axis(c, ax.L, 1, &m64));
    double2* b0 = nullptr;
    CK(cudaMalloc(&b0, sizeof(double2) * 2 * ax.L));
    CK(launch_chirp_b0(fp64, ax.chirp, b0, b0 + ax.L, n, ax.L, c->st));
    RowArgs r{};
    r.mode = ROW_FWD;
    r.rows = 2;
    r.L = ax.L;
    r.ny_grid = 2;
    r.nx_grid = ax.L;
    r.dx = 1;
    r.in = b0;
    r.in_ld = ax.L;
    r.in_off = 0;
    r.in_n = ax.L;
    r.out = b0;
    r.out_ld = ax.L;
    r.out_off = 0;
    r.out_n = ax.L;
    r.out_scale = 1;
    r.tw = m64->tw;
    r.batch = 1;
    CK(prof_rows(c, 1, r));
    CK(launch_bhat_finish(fp64, ax.bf, ax.bi, b0, b0 + ax.L, ax.L, c->st));
    CK(cudaStreamSynchronize(c->st));
    cudaFree(b0);
    return WOS_OK;
}

int get_axis(wos_ctx c, int n, int fp64, Axis** out) {
    auto& m = c->axes[fp64];
    auto it = m.find(n);
    if (it != m.end()) {
        *out = &it->second;
        return WOS_OK;
    }
    Axis ax;
    int rc = build_axis(c, n, fp64, ax);
    if (rc != WOS_OK) {
        if (ax.tw) cudaFree(ax.tw);
        if (ax.chirp) cudaFree(ax.chirp);
        if (ax.bf) cudaFree(ax.bf);
        if (ax.bi) cudaFree(ax.bi);
        return rc;
    }
    auto res = m.emplace(n, ax);
    *out = &res.first->second;
    return WOS_OK;
}

void fill_axis(RowArgs& r, const Axis* a) {
    r.L = a->L;
    r.blue_n = a->blue ? a->n : 0;
    r.tw = a->tw;
    r.chirp = a->chirp;
    r.bhat_f = a->bf;
    r.bhat_i = a->bi;
}

void fill_axis(ColArgs& r, const Axis* a) {
    r.L = a->L;
    r.blue_n = a->blue ? a->n : 0;
    r.tw = a->tw;
    r.chirp = a->chirp;
    r.bhat_f = a->bf;
    r.bhat_i = a->bi;
}

RowArgs row_defaults(int ny, int nx, double dx) {
    RowArgs r{};
    r.ny_grid = ny;
    r.nx_grid = nx;
    r.dx = dx;
    r.out_scale = 1.0;
    r.pre_amp = 1.0;
    r.weight = 1.0;
    r.batch = 1;
    return r;
}

ColArgs col_defaults(wos_ctx c, double dx) {
    ColArgs a{};
    a.h.scale = 1.0;
    a.h.dx = dx;
    a.h.c_re = 1.0;
    a.h.exact = c->fp64;
    a.hist_dx = dx;
    a.out_scale = 1.0;
    a.batch = 1;
    a.W = c->colw;
    return a;
}

// Columns per CTA of the fused pass.  Adjacent columns give 64 B row segments
// (8 x complex64, 4 x complex128) while the tile stays within shared memory.
int auto_colw_p(wos_ctx c, int fp64, int L) {
    if (c->colw > 0) return c->colw;
    const int E = pick_E(fp64, L);
    const int T = L / E;
    const int maxt = max_threads_for(fp64, E);
    // complex64 mixed-radix lines take 4 columns (the lean column sweep at
    // 768 points: 2.21 ms with 8 for 128 planes, 2.03 ms with 4)
    const bool mixed = (L & (L - 1)) != 0;
    int W = (fp64 || mixed) ? 4 : 8;
    // mixed-radix columns run between two tile buffers
    const size_t bufs = mixed ? 2 : 1;
    while (W > 1 && (W * T > maxt || bufs * col_smem_bytes(fp64, L, W) > 200 * 1024)) W >>= 1;
    return W;
}

int auto_colw(wos_ctx c, int L) { return auto_colw_p(c, c->fp64, L); }

int red_prepare(wos_ctx c, size_t max_blocks) {
    const size_t per = max_blocks * RS_COUNT;
    TRY(ensure(c->red, per * kRegions * sizeof(double)));
    TRY(ensure(c->redout, (size_t)kRegions * RS_COUNT * sizeof(double) * 1));
    if (!c->hred || c->hred_n < (size_t)kRegions * RS_COUNT) {
        if (c->hred) cudaFreeHost(c->hred);
        CK(cudaMallocHost(&c->hred, sizeof(double) * kRegions * RS_COUNT));
        c->hred_n = kRegions * RS_COUNT;
    }
    return WOS_OK;
}

double* red_region(wos_ctx c, int r) {
    const size_t per = c->red.n / sizeof(double) / kRegions;
    return reinterpret_cast<double*>(c->red.p) + per * r;
}

size_t red_region_blocks(wos_ctx c) { return c->red.n / sizeof(double) / kRegions / RS_COUNT; }

double* redout_region(wos_ctx c, int r) { return reinterpret_cast<double*>(c->redout.p) + (size_t)RS_COUNT * r; }

// blocks of a row launch (mirrors launch_rows_t) and of a column launch
size_t row_blocks(int fp64, int L, int rows, int batch) {
    const int E = pick_E(fp64, L);
    const int T = L / E;
    int lines = 1;
    while (lines * 2 * T <= 256 && lines * 2 <= rows) lines *= 2;
    while (lines * T < 32) lines *= 2;
    return (size_t)((rows + lines - 1) / lines) * std::max(batch, 1);
}

size_t col_blocks(int fp64, int L, int W, int ncols, int batch) {
    const int E = pick_E(fp64, L);
    const int T = L / E;
    const int maxt = max_threads_for(fp64, E);
    while (W * T < 32) W *= 2;
    while (W > 1 && W * T > maxt) W /= 2;
    return (size_t)((ncols + W - 1) / W) * std::max(batch, 1);
}

Policy ev_policy(const wos_context& c, double z) {
    Policy p;
    p.limit = c.evanescent_limit;
    if (z < 0) {
        if (c.backward_regularize) {
            p.alpha = c.tikhonov_alpha;
            if (p.alpha <= 0) p.alpha = 1e-3;
            p.reg = 1;
            return p;
        }
        p.zero = 1;
        return p;
    }
    p.zero = c.evanescent_zero;
    return p;
}

void warn_add(wos_diag* d, int bit, double value) {
    if (!d) return;
    d->warn_count[bit]++;
    if (value != 0) d->warn_value[bit] = value;
}

// asmWarn (optics/propagate.go:203-218)
void asm_warn(wos_diag* d, double z, double pin, double pout, const Policy& p) {
    if (pin > 0 && pout < pin * (1 - 1e-8) && z > 0)
        warn_add(d, WOS_W_EVANESCENT_FILTERED, (pin - pout) / pin);
    if (z < 0) {
        if (p.reg) warn_add(d, WOS_W_BACKWARD_REGULARIZED, 0);
        else if (p.zero) warn_add(d, WOS_W_BACKWARD_EVANESCENT, 0);
    }
}

// spectralRadius tail (optics/propagate.go:309-319) from the 97-bin histogram
double spectral_radius_from_hist(const double* hist, double dx, double frac) {
    const int bins = 96;
    const double fnyq = 1 / (2 * dx);
    double tot = 0;
    for (int b = 0; b <= bins; b++) tot += hist[b];
    if (tot <= 0) return 0;
    double run = 0;
    for (int b = 0; b <= bins; b++) {
        run += hist[b];
        if (run >= frac * tot) return (double)b / bins * fnyq;
    }
    return fnyq;
}

// asmWrapWarn decision (optics/propagate.go:247-264); carry = min(nx,ny)*dx
bool wrap_needed(const wos_context& c, int ny, int nx, double dx, double z) {
    const double carry = (double)std::min(nx, ny) * dx;
    if (!c.diagnostics || z == 0 || carry <= 0) return false;
    return std::fabs(z) * c.wavelength / (2 * dx) > carry;
}

void wrap_finish(wos_diag* d, const wos_context& c, int ny, int nx, double dx, double z, const double* hist) {
    const double carry = (double)std::min(nx, ny) * dx;
    const double fsig = spectral_radius_from_hist(hist, dx, 0.90);
    if (d) {
        d->wrap_checked = 1;
        d->spectral_radius = fsig;
    }
    if (fsig <= 0) return;
    const double walk = std::fabs(z) * c.wavelength * fsig;
    if (walk > carry) warn_add(d, WOS_W_ASM_ALIAS_WRAP, walk / carry);
}

// Fetch finished reduction regions [0, n) to the host (one synchronisation).
int fetch_red(wos_ctx c, int nreg) {
    CK(cudaMemcpyAsync(c->hred, c->redout.p, sizeof(double) * RS_COUNT * nreg, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

HArgs asm_h(wos_ctx c, const wos_context& cc, double z, const Policy& p, double dx, int lfx, int lfy) {
    HArgs h{};
    h.kind = H_ASM;
    h.exact = c->fp64;
    h.wl = cc.wavelength;
    h.k = 2 * M_PI / cc.wavelength;
    h.z = z;
    h.kz = h.k * z;
    h.kaz = h.k * std::fabs(z);
    h.zero_ev = p.zero;
    h.reg = p.reg;
    h.alpha = p.alpha;
    h.limit = p.limit;
    h.dx = dx;
    h.lfx = lfx;
    h.lfy = lfy;
    h.scale = 1.0 / ((double)lfx * (double)lfy);
    h.c_re = 1;
    return h;
}

// Forward row pass of an unpadded field into `dst` (native), plus a column
// reduction: spectral centroid sums and/or the radial histogram.
int spectrum_stats(wos_ctx c, const Prop& p, void* dst, bool centroid, bool hist, int shift, double fxc,
                   double fyc, int region, int* blocks_out) {
    Axis *ax, *ay;
    TRY(get_axis(c, p.nx, c->fp64, &ax));
    TRY(get_axis(c, p.ny, c->fp64, &ay));
    const long long np = (long long)p.ny * p.nx;
    RowArgs r = row_defaults(p.ny, p.nx, p.dx);
    r.mode = ROW_FWD;
    r.rows = p.ny;
    fill_axis(r, ax);
    r.in = p.in;
    r.in_c128 = p.in_c128;
    r.in_ld = p.nx;
    r.in_bstride = np;
    r.in_off = 0;
    r.in_n = p.nx;
    r.out = dst;
    r.out_ld = p.nx;
    r.out_bstride = np;
    r.out_off = 0;
    r.out_n = p.nx;
    r.pre_shift = shift;
    r.fxc = fxc;
    r.fyc = fyc;
    r.batch = p.ncomp;
    const int W = auto_colw(c, ay->L);
    const size_t nbc = col_blocks(c->fp64, ay->L, W, p.nx, p.ncomp);
    TRY(red_prepare(c, nbc));
    CK(prof_rows(c, c->fp64, r));
    ColArgs a = col_defaults(c, p.dx);
    a.mode = COL_REDUCE;
    a.ncols = p.nx;
    fill_axis(a, ay);
    a.W = W;
    a.src = dst;
    a.src_ld = p.nx;
    a.src_bstride = np;
    a.in_off = 0;
    a.in_n = p.ny;
    a.red = red_region(c, region);
    a.red_spec = centroid;
    a.red_hist = hist;
    a.hist_lx = p.nx;
    a.hist_ly = p.ny;
    a.hist_dx = p.dx;
    a.batch = p.ncomp;
    CK(prof_cols(c, c->fp64, a));
    const int nb = (int)nbc;
    if (centroid) {
        CK(launch_reduce_finish(a.red, nb, 1, RS_SW, 3, redout_region(c, region), c->st));
        CK(launch_reduce_finish(a.red, nb, 1, RS_SLO, 3, redout_region(c, region), c->st));
    }
    if (hist) CK(launch_reduce_finish(a.red, nb, 1, RS_HIST, 97, redout_region(c, region), c->st));
    if (blocks_out) *blocks_out = nb;
    return WOS_OK;
}

int env_int(const char* name, int def) {
    const char* v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : def;
}

Tune get_tune(wos_ctx c, int ny, int nx) {
    auto it = c->tune.find(tune_key(c->fp64, ny, nx));
    if (it != c->tune.end()) return it->second;
    Tune t;
    // complex64 1024-point rows: E = 8, twice the threads per line of E = 16
    // (1024^2 split-step runs 9.45 -> 8.89 ms); 512 and 2048 points are faster
    // with E = 16 (12.3 vs 16.1 us per propagation, 20.3k vs 17.8k props/s)
    t.rowE = env_int("WOS_ROWE", c->fp64 ? (nx >= 8192 ? 16 : 8) : (nx == 1024 ? 8 : 16));
    t.colE = env_int("WOS_COLE", c->fp64 ? (ny >= 8192 ? 16 : 8) : 16);
    t.colW = env_int("WOS_COLW", c->fp64 ? 2 : 8);
    if (c->colw > 0) t.colW = c->colw;
    return t;
}

size_t fast_row_blocks(int L, int E, int rows, int batch) {
    const int lines = fast_row_lines(L, E, rows);
    return (size_t)((rows + lines - 1) / lines) * std::max(batch, 1);
}

// (an upper bound: the split tiles of fast_cols_pair launch two CTAs per tile)
size_t fast_col_blocks(int fp64, int L, int E, int W, int ncols, int batch) {
    W = fast_col_width(fp64, L, E, W);
    if (W < 1) W = 1;
    const size_t per = fast_cols_pair_case(fp64, L, E, W) ? 2 : 1;
    return per * (size_t)((ncols + W - 1) / W) * std::max(batch, 1);
}

// Per-pass twiddle table of the specialised sweeps for a power-of-two axis.
int fast_tw(wos_ctx c, Axis* a, int E, const void** out) {
    const int slot = E == 16 ? 1 : 0;
    if (!a->ftw[slot]) {
        const size_t bytes = (size_t)fast_table_len(a->L, E) * c->csz();
        CK(cudaMalloc(&a->ftw[slot], bytes));
        CK(fast_build_twiddles(c->fp64, a->L, E, a->ftw[slot], c->st));
    }
    *out = a->ftw[slot];
    return WOS_OK;
}

// Residual table of the complex64 per-pass twiddles (compensated sweeps).
int fast_tw_lo(wos_ctx c, Axis* a, int E, const void** out) {
    const int slot = E == 16 ? 1 : 0;
    if (!a->ftw_lo[slot]) {
        CK(cudaMalloc(&a->ftw_lo[slot], (size_t)fast_table_len(a->L, E) * sizeof(float2)));
        CK(fast_build_twiddles_lo(a->L, E, a->ftw_lo[slot], c->st));
    }
    *out = a->ftw_lo[slot];
    return WOS_OK;
}

// Transfer-function table of a complex64 column sweep (FastCols::htab) for
// columns of L points, when the sweep can use one: the split-step's column
// sweeps (precise phase), no loss sums, one wavelength and distance, W
// columns per CTA dividing ncols / 2, and the table rows fitting beside the
// tile in shared memory.  Sets k.htab / k.htab_ld (left null otherwise); the
// entries are hi + lo pairs when the sweep runs the compensated transforms
// (k.tw_lo set).  Measured: the split-step's plain complex64 run 9.87 ->
// 8.60 ms (1024^2, 400 slices; its H takes sin/cos to ~1 ulp); the 2048^2
// ASM column sweep unchanged at 35.1 us, its evaluation of H running under
// the sweep's memory latency, while the 33 KB of table rows per CTA took the
// shared memory that the other stream's row sweeps overlap in (two-stream
// batch 20.4k -> 17.1k props/s), so the plain ASM does not use it.
// The table of k's transfer function for columns of L points, from the
// context's cache or built now on the context stream.  A new table is waited
// for before returning (outside stream capture), so that sweeps on other
// streams (the batch's side streams, a stream the caller switches to) can use
// it at once.
int htab_of(wos_ctx c, FastCols& k, int L, int hilo) {
    const int ld = htab_ld_for(L);
    const double key[9] = {k.wl, k.dx, k.kz, k.kaz, k.scale, k.alpha, k.limit, (double)k.zero_ev,
                           (double)(k.reg + 2 * k.backward + 4 * hilo)};
    for (auto& h : c->htab)
        if (h.valid && h.L == L && h.ncols == k.ncols && std::memcmp(h.key, key, sizeof key) == 0) {
            if (c->capturing) h.frozen = true;
            k.htab = reinterpret_cast<const float2*>(h.buf.p);
            k.htab_ld = ld;
            return WOS_OK;
        }
    // the next slot round robin that no captured graph reads, else a new one
    int slot = -1;
    for (size_t i = 0; i < c->htab.size() && slot < 0; i++) {
        const int j = (int)((c->htab_next + i) % c->htab.size());
        if (!c->htab[j].frozen) slot = j;
    }
    if (slot < 0) {
        c->htab.emplace_back();
        slot = (int)c->htab.size() - 1;
    }
    c->htab_next = (slot + 1) % (int)c->htab.size();
    wos_ctx_s::HTab& h = c->htab[slot];
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(c->st, &cs));
    // a table being replaced may still be read by sweeps on another stream
    if (h.valid && cs == cudaStreamCaptureStatusNone) CK(cudaDeviceSynchronize());
    h.valid = false;
    TRY(ensure(h.buf, (size_t)(k.ncols / 2 + 1) * ld * sizeof(float2) * (hilo ? 2 : 1)));
    CK(fast_build_htab(k, L, reinterpret_cast<float2*>(h.buf.p), ld, hilo, c->st));
    if (cs == cudaStreamCaptureStatusNone) CK(cudaStreamSynchronize(c->st));
    h.valid = true;
    h.frozen = c->capturing;
    h.L = L;
    h.ncols = k.ncols;
    std::memcpy(h.key, key, sizeof key);
    k.htab = reinterpret_cast<const float2*>(h.buf.p);
    k.htab_ld = ld;
    return WOS_OK;
}

int attach_htab(wos_ctx c, FastCols& k, int L, int E) {
    k.htab_global = 0;
    if (c->fp64 || !c->htab_on || !k.precise_phase || k.red || k.batch_wl || k.batch_z || L < 32) return WOS_OK;
    if (c->htab_reg && !k.hist) {
        // in registers from global memory (FastCols::htab_global), at the
        // widths that variant is built for
        const int Wg = fast_col_width(0, L, E, k.W);
        if (Wg == 4 || (Wg == 8 && k.tw_lo)) {
            TRY(htab_of(c, k, L, k.tw_lo != nullptr));
            k.htab_global = 1;
            return WOS_OK;
        }
    }
    const int W = fast_col_width(0, L, E, k.tiled ? kTileW : k.W);
    const int ld = htab_ld_for(L);
    if (W < 1 || k.ncols < 2 * W || k.ncols % (2 * W) != 0) return WOS_OK;
    const int hilo = k.tw_lo != nullptr;
    if (fast_col_smem_htab(L, E, W, ld, hilo) + 2048 > 227 * 1024) return WOS_OK;
    return htab_of(c, k, L, hilo);
}

// The same table read from global memory into registers (FastCols::htab_global)
// by the plain complex64 ASM column sweep on the tiled intermediate (no loss
// sums, histogram, per-unit wavelengths or distances).  Measured at 2048^2
// (two-stream batch): column sweep 37.2 -> 33.1 us, 19.8k -> 20.4k props/s,
// one call per field 15.9k -> 16.8k; FP32 against the oracle 4.6e-7 -> 3.3e-7
// (H rounded once from its FP64 value).
int attach_htab_global(wos_ctx c, FastCols& k, int L) {
    if (c->fp64 || !c->htab_reg || k.red || k.hist || k.batch_wl || k.batch_z || k.tw_lo || L < 32) return WOS_OK;
    TRY(htab_of(c, k, L, 0));
    k.htab_global = 1;
    return WOS_OK;
}

// The complex128 table (FP64 values of H, 16-byte entries) for the pipelined
// complex128 column sweep, which reads it into registers; its entries are the
// values the sweep would evaluate, so the results do not change.
int attach_htab64(wos_ctx c, FastCols& k, int L) {
    if (!c->fp64 || !c->htab_reg || c->sweep_mode == 2 || k.red || k.hist || k.batch_wl || k.batch_z || L < 32)
        return WOS_OK;
    TRY(htab_of(c, k, L, 2));
    k.htab_global = 1;
    return WOS_OK;
}

// Plain band-limited ASM on power-of-two grids through the specialised
// sweeps.  Returns -1 when the grid is not covered (the general sweeps run).
// One specialised sweep: the pipelined kernel where the sweep mode asks for it
// and it accepts the layout, else the one-shot kernel; *nb receives the number
// of per-CTA records.  By default FP32 rows are one-shot (four resident
// register-bound CTAs beat three pipelined ones; in the two-stream 2048^2
// batch the persistent forward rows, storing the tiled intermediate, took
// 21.6k -> 18.8k props/s: they hold every SM, so the other stream's sweeps
// no longer run beside them), FP64 rows and all columns pipelined where the
// tile fits two stages.
cudaError_t sweep_rows(wos_ctx c, int L, int E, bool inv, const FastRows& a, int* nb) {
    if ((c->sweep_mode == 3 || (c->sweep_mode == 1 && c->fp64)) && !a.in_tiled && (!a.out_tiled || !inv)) {
        FastRows b = a;
        b.err = c->err_dev;
        const cudaError_t e = pipe_rows(c->fp64, L, E, inv, b, c->st, nb);
        if (e != cudaErrorNotSupported) return e;
    }
    return fast_rows(c->fp64, L, E, inv, a, c->st, nb);
}

// Tables of the split column tiles: per-pass twiddles of L/2 and W_L^n.
bool pair_tables(wos_ctx c, int L, int E, const void** twh, const void** twp) {
    Axis *ah, *af;
    if (get_axis(c, L / 2, c->fp64, &ah) != WOS_OK || get_axis(c, L, c->fp64, &af) != WOS_OK) return false;
    if (fast_tw(c, ah, E, twh) != WOS_OK) return false;
    if (!af->ptw) {
        if (cudaMalloc(&af->ptw, (size_t)(L / 2) * c->csz()) != cudaSuccess) {
            cudaGetLastError();
            af->ptw = nullptr;
            return false;
        }
        if (fast_build_pair_twiddles(c->fp64, L, af->ptw, c->st) != cudaSuccess) return false;
    }
    *twp = af->ptw;
    return true;
}

bool pair_eligible(wos_ctx c, int L, int E, const FastCols& a) {
    return c->col_pair && !a.hist && !a.tiled && !a.tw_lo && !a.htab &&
           fast_cols_pair_case(c->fp64, L, E, fast_col_width(c->fp64, L, E, a.W));
}

cudaError_t sweep_cols(wos_ctx c, int L, int E, const FastCols& a, int* nb) {
    if (pair_eligible(c, L, E, a)) {
        FastCols b = a;
        if (pair_tables(c, L, E, &b.tw_half, &b.tw_pair)) {
            const cudaError_t e = fast_cols_pair(c->fp64, L, E, b, c->st, nb);
            if (e != cudaErrorNotSupported) return e;
        }
    }
    // (complex64 table or compensated: one-shot kernels; the complex128
    // pipelined sweep reads its table itself)
    if (c->sweep_mode != 2 && !a.tiled && !a.tw_lo && (!a.htab || (c->fp64 && a.htab_global))) {
        FastCols b = a;
        b.err = c->err_dev;
        const cudaError_t e = pipe_cols(c->fp64, L, E, b, c->st, nb);
        if (e != cudaErrorNotSupported) return e;
    }
    return fast_cols(c->fp64, L, E, a, c->st, nb);
}

// The transfer-function fields of a specialised column sweep from the H of a
// plain ASM step.
void fill_asm_h(FastCols& k, const HArgs& h) {
    k.wl = h.wl;
    k.dx = h.dx;
    k.kz = h.kz;
    k.kaz = h.kaz;
    k.scale = h.scale;
    k.alpha = h.alpha;
    k.limit = h.limit;
    k.zero_ev = h.zero_ev;
    k.reg = h.reg;
    k.backward = h.z < 0;
    k.conj = h.conj;
    k.krev = h.kz / (2 * M_PI);
}

// Whether the three-sweep ASM of an ny x nx grid goes through the tiled
// intermediate (complex64: contiguous column tiles of kTileW).
bool asm_tiled(wos_ctx c, int ny, int nx, const Tune& t) {
    return c->tiled && !c->fp64 && nx % kTileW == 0 && fast_col_width(c->fp64, ny, t.colE, kTileW) == kTileW;
}

int try_fast_sweep3(wos_ctx c, const Prop& p, Sweep3& s) {
    if (!is_pow2(p.nx) || !is_pow2(p.ny)) return -1;
    // the FP32 column sweep reduces the phase in revolutions: |kz / 2 pi| < 2^28
    if (!c->fp64 && !(std::fabs(s.h.kz / (2 * M_PI)) < 268435456.0)) return -1;
    const Tune t = get_tune(c, p.ny, p.nx);
    if (!fast_supported(c->fp64, p.nx, t.rowE) || !fast_supported(c->fp64, p.ny, t.colE)) return -1;
    Axis *ax, *ay;
    TRY(get_axis(c, p.nx, c->fp64, &ax));
    TRY(get_axis(c, p.ny, c->fp64, &ay));
    const void *twx, *twy;
    TRY(fast_tw(c, ax, t.rowE, &twx));
    TRY(fast_tw(c, ay, t.colE, &twy));
    const long long np = (long long)p.ny * p.nx;
    // tiled intermediate (FP32): the column sweep reads contiguous tiles of
    // kTileW columns; the intermediate is then a buffer of its own (the last
    // sweep changes the layout, so it cannot run in place in the output)
    const bool tiled = asm_tiled(c, p.ny, p.nx, t);
    void* S;
    if (p.out_c128) {
        TRY(ensure(c->scratch, (size_t)np * p.ncomp * c->csz()));
        S = c->scratch.p;
    } else if (tiled) {
        DevBuf& b = c->tsc[std::max(0, std::min(c->cur_slot, wos_ctx_s::kMaxAux))];
        TRY(ensure(b, (size_t)np * p.ncomp * c->csz()));
        S = b.p;
    } else {
        S = p.out;
    }
    const size_t nbr = fast_row_blocks(p.nx, t.rowE, p.ny, p.ncomp);
    const size_t nbc = fast_col_blocks(c->fp64, p.ny, t.colE, t.colW, p.nx, p.ncomp);
    if (s.red_pin || s.red_pout || s.red_loss || s.hist) TRY(red_prepare(c, std::max(nbr, nbc)));
    int nb = 0;
    FastRows r{};
    r.rows = p.ny;
    r.in = p.in;
    r.in_c128 = p.in_c128;
    r.in_ld = p.nx;
    r.in_bstride = np;
    r.out = S;
    r.out_ld = p.nx;
    r.out_bstride = np;
    r.tw = twx;
    r.out_scale = 1.0;
    r.red = s.red_pin ? red_region(c, 0) + RS_P : nullptr;
    r.red_stride = RS_COUNT;
    r.batch = p.ncomp;
    r.out_tiled = tiled;
    r.tile_len = p.ny;
    CK(timed_launch(c, 0, [&] { return sweep_rows(c, p.nx, t.rowE, false, r, &nb); }));
    if (s.red_pin) CK(launch_reduce_finish(red_region(c, 0), nb, 1, RS_P, 1, redout_region(c, 0), c->st));
    FastCols k{};
    k.ncols = p.nx;
    k.W = tiled ? kTileW : t.colW;
    k.data = S;
    k.ld = tiled ? kTileW : p.nx;
    k.tiled = tiled;
    k.bstride = np;
    k.tw = twy;
    k.batch = p.ncomp;
    fill_asm_h(k, s.h);
    k.red = s.red_loss ? red_region(c, 1) + RS_SW : nullptr;
    k.red_stride = RS_COUNT;
    if (s.hist) {
        k.hist = red_region(c, 1) + RS_HIST;
        k.hist_dx = p.dx;
    }
    if (tiled) TRY(attach_htab_global(c, k, p.ny));
    else TRY(attach_htab64(c, k, p.ny));
    CK(timed_launch(c, 4, [&] { return sweep_cols(c, p.ny, t.colE, k, &nb); }));
    if (s.red_loss) CK(launch_reduce_finish(red_region(c, 1), nb, 1, RS_SW, 2, redout_region(c, 1), c->st));
    if (s.hist) CK(launch_reduce_finish(red_region(c, 1), nb, 1, RS_HIST, 97, redout_region(c, 1), c->st));
    FastRows q{};
    q.rows = p.ny;
    q.in = S;
    q.in_ld = p.nx;
    q.in_bstride = np;
    q.out = p.out;
    q.out_c128 = p.out_c128;
    q.out_ld = p.nx;
    q.out_bstride = np;
    q.tw = twx;
    q.out_scale = 1.0;
    q.red = s.red_pout ? red_region(c, 2) + RS_P : nullptr;
    q.red_stride = RS_COUNT;
    q.batch = p.ncomp;
    q.in_tiled = tiled;
    q.tile_len = p.ny;
    // the result with evict-first stores: L2 stays with the intermediates of
    // the fields in flight (2048^2 batch 21.2k -> 21.5k props/s)
    q.out_stream = c->out_stream;
    CK(timed_launch(c, 1, [&] { return sweep_rows(c, p.nx, t.rowE, true, q, &nb); }));
    if (s.red_pout) CK(launch_reduce_finish(red_region(c, 2), nb, 1, RS_P, 1, redout_region(c, 2), c->st));
    s.fast = true;
    return WOS_OK;
}

int run_sweep3(wos_ctx c, const Prop& p, Sweep3& s) {
    if (!s.pad && !s.shift && s.h.kind == H_ASM && s.h.fxoff == 0 && s.h.fyoff == 0 && !c->no_fast) {
        const int rc = try_fast_sweep3(c, p, s);
        if (rc != -1) return rc;
    }
    const int mx = s.pad ? 2 * p.nx : p.nx;
    const int my = s.pad ? 2 * p.ny : p.ny;
    const int offx = s.pad ? p.nx / 2 : 0, offy = s.pad ? p.ny / 2 : 0;
    Axis *ax, *ay;
    TRY(get_axis(c, mx, c->fp64, &ax));
    TRY(get_axis(c, my, c->fp64, &ay));
    const long long np_in = (long long)p.ny * p.nx;
    const long long np_s = (long long)p.ny * mx;
    // scratch: the output buffer itself when it is native and unpadded
    void* S;
    if (!s.pad && !p.out_c128) {
        S = p.out;
    } else {
        TRY(ensure(c->scratch, (size_t)np_s * p.ncomp * c->csz()));
        S = c->scratch.p;
    }
    const int W = auto_colw(c, ay->L);
    const size_t nbr = row_blocks(c->fp64, ax->L, p.ny, p.ncomp);
    const size_t nbc = col_blocks(c->fp64, ay->L, W, mx, p.ncomp);
    TRY(red_prepare(c, std::max(nbr, nbc)));

    RowArgs r = row_defaults(p.ny, p.nx, p.dx);
    r.mode = ROW_FWD;
    r.rows = p.ny;
    fill_axis(r, ax);
    r.in = p.in;
    r.in_c128 = p.in_c128;
    r.in_ld = p.nx;
    r.in_bstride = np_in;
    r.in_off = offx;
    r.in_n = p.nx;
    r.out = S;
    r.out_ld = mx;
    r.out_bstride = np_s;
    r.out_off = 0;
    r.out_n = ax->n;
    r.pre_shift = s.shift;
    r.fxc = s.fxc;
    r.fyc = s.fyc;
    r.batch = p.ncomp;
    if (s.red_pin) {
        r.red = red_region(c, 0);
        r.red_pre = 1;
    }
    CK(prof_rows(c, c->fp64, r));
    if (s.red_pin) CK(launch_reduce_finish(r.red, (int)nbr, 1, RS_P, 1, redout_region(c, 0), c->st));

    ColArgs a = col_defaults(c, p.dx);
    a.mode = COL_FUSED;
    a.ncols = mx;
    fill_axis(a, ay);
    a.W = W;
    a.src = S;
    a.src_ld = mx;
    a.src_bstride = np_s;
    a.in_off = offy;
    a.in_n = p.ny;
    a.dst = S;
    a.dst_ld = mx;
    a.dst_bstride = np_s;
    a.out_off = offy;
    a.out_n = p.ny;
    a.h = s.h;
    a.batch = p.ncomp;
    if (s.hist || s.red_loss) a.red = red_region(c, 1);
    if (s.hist) {
        a.red_hist = 1;
        a.hist_lx = p.nx;
        a.hist_ly = p.ny;
        a.hist_dx = p.dx;
    }
    a.red_bpm = s.red_loss;
    CK(prof_cols(c, c->fp64, a));
    if (s.hist) CK(launch_reduce_finish(a.red, (int)nbc, 1, RS_HIST, 97, redout_region(c, 1), c->st));
    if (s.red_loss) CK(launch_reduce_finish(a.red, (int)nbc, 1, RS_SW, 4, redout_region(c, 1), c->st));

    RowArgs q = row_defaults(p.ny, p.nx, p.dx);
    q.mode = ROW_INV;
    q.rows = p.ny;
    fill_axis(q, ax);
    q.in = S;
    q.in_c128 = 0;
    q.in_ld = mx;
    q.in_bstride = np_s;
    q.in_off = 0;
    q.in_n = ax->n;
    q.out = p.out;
    q.out_c128 = p.out_c128;
    q.out_ld = p.nx;
    q.out_bstride = np_in;
    q.out_off = offx;
    q.out_n = p.nx;
    q.post_shift = s.shift;
    q.fxc = s.fxc;
    q.fyc = s.fyc;
    q.batch = p.ncomp;
    if (s.red_pout) {
        q.red = red_region(c, 2);
        q.red_post = 1;
    }
    CK(prof_rows(c, c->fp64, q));
    if (s.red_pout) CK(launch_reduce_finish(q.red, (int)nbr, 1, RS_P, 2, redout_region(c, 2), c->st));
    return WOS_OK;
}

int copy_field(wos_ctx c, const Prop& p) {
    // z == 0: Propagate returns the field unchanged (optics/propagate.go:66-68)
    const long long n = (long long)p.ny * p.nx * p.ncomp;
    if (p.in == p.out && p.in_c128 == p.out_c128) return WOS_OK;
    if (p.in_c128 == p.out_c128) {
        CK(cudaMemcpyAsync(p.out, p.in, n * (p.in_c128 ? 16 : c->csz()), cudaMemcpyDeviceToDevice, c->st));
        return WOS_OK;
    }
    if (c->fp64) {
        CK(cudaMemcpyAsync(p.out, p.in, n * 16, cudaMemcpyDeviceToDevice, c->st));
        return WOS_OK;
    }
    CK(launch_convert(p.out_c128, p.in, p.out, n, c->st));
    return WOS_OK;
}

int run_propagate(wos_ctx c, const Prop& p0) {
    Prop p = p0;
    wos_diag* d = p.diag;
    if (d) {
        std::memset(d, 0, sizeof(*d));
        d->dx_out = p.dx;
    }
    if (p.ny < 2 || p.nx < 2 || p.ncomp < 1 || p.ncomp > 2 || !(p.dx > 0))
        return fail(WOS_INVALID_ARG, "invalid field geometry");
    if (!p.in || !p.out) return fail(WOS_INVALID_ARG, "null field pointer");
    if (p.z == 0) return copy_field(c, p);
    if (!(p.c.wavelength > 0) && p.method != WOS_FRESNEL_IR)
        return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    const bool diag = d != nullptr;
    const Policy pol = ev_policy(p.c, p.z);
    const double z = p.z;
    const double dx = p.dx;
    switch (p.method) {
    case WOS_ASM:
    case WOS_ASM_SHIFT:
    case WOS_ASM_PAD:
    case WOS_ASM_SHIFT_PAD: {
        const bool shift_m = (p.method == WOS_ASM_SHIFT || p.method == WOS_ASM_SHIFT_PAD);
        const bool pad_m = (p.method == WOS_ASM_PAD || p.method == WOS_ASM_SHIFT_PAD);
        const bool wrap = wrap_needed(p.c, p.ny, p.nx, dx, z);
        Sweep3 s;
        s.pad = pad_m;
        if (shift_m) {
            // spectralCentroid (optics/propagate.go:391-416) over all components
            const long long np = (long long)p.ny * p.nx;
            TRY(ensure(c->scratch2, (size_t)np * p.ncomp * c->csz()));
            const bool hist_here = wrap && p.method == WOS_ASM_SHIFT;
            TRY(spectrum_stats(c, p, c->scratch2.p, true, hist_here, 0, 0, 0, 3, nullptr));
            TRY(fetch_red(c, 4));
            // compensated sums: the centroid is exact to the last bits (the
            // reference accumulates it in sequence, whose rounding the
            // carrier-shift output amplifies ~1e4-fold)
            const double* rr = c->hred + RS_COUNT * 3;
            const double sw = rr[RS_SW] + rr[RS_SLO];
            double fxc = 0, fyc = 0;
            if (sw > 0) {
                fxc = (rr[RS_SFX] + rr[RS_SLO + 1]) / sw;
                fyc = (rr[RS_SFY] + rr[RS_SLO + 2]) / sw;
            }
            if (d) {
                d->centroid_fx = fxc;
                d->centroid_fy = fyc;
            }
            const double fbx = 1 / ((double)p.nx * dx), fby = 1 / ((double)p.ny * dx);
            if (!(std::fabs(fxc) < 0.5 * fbx && std::fabs(fyc) < 0.5 * fby)) {
                s.shift = 1;
                s.fxc = fxc;
                s.fyc = fyc;
                if (d) d->carrier_applied = 1;
                if (wrap) {
                    if (p.method == WOS_ASM_SHIFT) {
                        std::vector<double> h(c->hred + RS_COUNT * 3 + RS_HIST, c->hred + RS_COUNT * 3 + RS_HIST + 97);
                        wrap_finish(d, p.c, p.ny, p.nx, dx, z, h.data());
                    } else {
                        // propASMPadCore checks the carrier-free field
                        TRY(spectrum_stats(c, p, c->scratch2.p, false, true, 1, fxc, fyc, 3, nullptr));
                        TRY(fetch_red(c, 4));
                        std::vector<double> h(c->hred + RS_COUNT * 3 + RS_HIST, c->hred + RS_COUNT * 3 + RS_HIST + 97);
                        wrap_finish(d, p.c, p.ny, p.nx, dx, z, h.data());
                    }
                }
            }
        }
        const int mx = pad_m ? 2 * p.nx : p.nx, my = pad_m ? 2 * p.ny : p.ny;
        s.h = asm_h(c, p.c, z, pol, dx, mx, my);
        s.h.fxoff = s.fxc;
        s.h.fyoff = s.fyc;
        s.red_pin = diag;
        s.red_pout = diag;
        s.red_loss = diag;
        // wrap check when no carrier branch ran: the plain field's spectrum
        if (wrap && !s.shift) {
            if (!pad_m) {
                s.hist = true;
            } else {
                TRY(ensure(c->scratch2, (size_t)p.ny * p.nx * p.ncomp * c->csz()));
                TRY(spectrum_stats(c, p, c->scratch2.p, false, true, 0, 0, 0, 3, nullptr));
                TRY(fetch_red(c, 4));
                std::vector<double> h(c->hred + RS_COUNT * 3 + RS_HIST, c->hred + RS_COUNT * 3 + RS_HIST + 97);
                wrap_finish(d, p.c, p.ny, p.nx, dx, z, h.data());
            }
        }
        TRY(run_sweep3(c, p, s));
        if (diag) {
            TRY(fetch_red(c, 3));
            const double pin = c->hred[RS_P] * dx * dx;
            d->p_in = pin;
            d->p_out = c->hred[2 * RS_COUNT + RS_P] * dx * dx;
            if (s.hist) wrap_finish(d, p.c, p.ny, p.nx, dx, z, c->hred + RS_COUNT + RS_HIST);
            // loss fraction of the step, from sums of positive terms only:
            // spectral sum |F|^2 (1 - |H|^2) / sum |F|^2, plus the energy the
            // zero-padded methods crop away in the column (mx * Dy) and row (Dx) passes
            const double p0 = c->hred[RS_COUNT + RS_SW], l1 = c->hred[RS_COUNT + RS_SW + 1];
            const double dy = s.fast ? 0.0 : c->hred[RS_COUNT + RS_SW + 3];
            const double dxr = s.fast ? 0.0 : c->hred[2 * RS_COUNT + RS_P + 1];
            const double pin_sp = c->hred[RS_P];
            const int mx = pad_m ? 2 * p.nx : p.nx;
            double frac = p0 > 0 ? l1 / p0 : 0.0;
            if (pin_sp > 0) frac += ((double)mx * dy + dxr) / pin_sp;
            asm_warn(d, z, pin, pin - pin * frac, pol);
        }
        return WOS_OK;
    }
    case WOS_FRESNEL_TF: {
        // propFresnelTF (optics/propagate.go:507-519)
        Sweep3 s;
        s.h = asm_h(c, p.c, z, pol, dx, p.nx, p.ny);
        s.h.kind = H_FRESNEL_TF;
        const double kz = (2 * M_PI / p.c.wavelength) * z;
        s.h.c_re = std::cos(kz);
        s.h.c_im = std::sin(kz);
        s.red_pin = diag;
        s.red_pout = diag;
        TRY(run_sweep3(c, p, s));
        if (diag) {
            TRY(fetch_red(c, 3));
            d->p_in = c->hred[RS_P] * dx * dx;
            d->p_out = c->hred[2 * RS_COUNT + RS_P] * dx * dx;
        }
        const int n = std::min(p.nx, p.ny);
        if (std::fabs(z) > (double)n * dx * dx / p.c.wavelength) warn_add(d, WOS_W_FRESNEL_TF_ALIAS, 0);
        return WOS_OK;
    }
    case WOS_FRESNEL_IR: {
        // propFresnelIR (optics/propagate.go:533-590): FFT2D of the 2N chirp
        // kernel is separable, FFT(hx) (x) FFT(hy), built in FP64 per axis.
        const double wl = p.c.wavelength;
        if (!(wl > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
        const int mx = 2 * p.nx, my = 2 * p.ny;
        Axis *ax64, *ay64;
        TRY(get_axis(c, mx, 1, &ax64));
        TRY(get_axis(c, my, 1, &ay64));
        TRY(ensure(c->tmp, sizeof(double2) * (size_t)(mx + my) + c->csz() * (size_t)(mx + my)));
        double2* hx = reinterpret_cast<double2*>(c->tmp.p);
        double2* hy = hx + mx;
        void* tx = hy + my;
        void* ty = reinterpret_cast<char*>(tx) + c->csz() * mx;
        CK(launch_fresnel_ir_axis(hx, mx, dx, wl, z, c->st));
        CK(launch_fresnel_ir_axis(hy, my, dx, wl, z, c->st));
        for (int ax = 0; ax < 2; ax++) {
            Axis* A = ax ? ay64 : ax64;
            RowArgs r = row_defaults(1, A->n, dx);
            r.mode = ROW_FWD;
            r.rows = 1;
            fill_axis(r, A);
            r.in = ax ? hy : hx;
            r.in_ld = A->n;
            r.in_n = A->n;
            r.out = ax ? hy : hx;
            r.out_ld = A->n;
            r.out_n = A->n;
            CK(prof_rows(c, 1, r));
        }
        CK(launch_scale_copy(c->fp64, hx, tx, mx, 1.0, 0.0, c->st));
        CK(launch_scale_copy(c->fp64, hy, ty, my, 1.0, 0.0, c->st));
        Sweep3 s;
        s.pad = 1;
        s.h = asm_h(c, p.c, z, pol, dx, mx, my);
        s.h.kind = H_TABLE_XY;
        s.h.tx = tx;
        s.h.ty = ty;
        // pre = complex(0, -1/(wl z)) * cexpI(k z) * complex(dx^2, 0)
        const double k = 2 * M_PI / wl;
        const double a0 = -1 / (wl * z);
        const double cr = std::cos(k * z), ci = std::sin(k * z);
        const double pr = -a0 * ci, pi_ = a0 * cr;  // (0 + i a0)(cr + i ci)
        s.h.c_re = pr * (dx * dx);
        s.h.c_im = pi_ * (dx * dx);
        s.red_pin = diag;
        s.red_pout = diag;
        TRY(run_sweep3(c, p, s));
        if (diag) {
            TRY(fetch_red(c, 3));
            d->p_in = c->hred[RS_P] * dx * dx;
            d->p_out = c->hred[2 * RS_COUNT + RS_P] * dx * dx;
        }
        const int n = std::max(p.nx, p.ny);
        if (std::fabs(z) < (double)n * dx * dx / wl) warn_add(d, WOS_W_FRESNEL_IR_ALIAS, 0);
        return WOS_OK;
    }
    case WOS_FRAUNHOFER: {
        // propFraunhofer (optics/propagate.go:603-662), square grids
        if (p.nx != p.ny) return fail(WOS_UNSUPPORTED_SIZE, "fraunhofer needs a square grid (nx == ny)");
        const int n = p.nx;
        const double wl = p.c.wavelength;
        const double k = 2 * M_PI / wl;
        const double dxout = wl * std::fabs(z) / ((double)n * dx);
        Axis* A;
        TRY(get_axis(c, n, c->fp64, &A));
        const long long np = (long long)n * n;
        TRY(ensure(c->scratch, (size_t)np * p.ncomp * c->csz()));
        void* S = c->scratch.p;
        void* O = p.out;
        if (p.out_c128 && !c->fp64) {
            TRY(ensure(c->scratch3, (size_t)np * p.ncomp * c->csz()));
            O = c->scratch3.p;
        }
        const size_t nbr = row_blocks(c->fp64, A->L, n, p.ncomp);
        TRY(red_prepare(c, nbr));
        RowArgs r = row_defaults(n, n, dx);
        r.mode = ROW_FWD;
        r.rows = n;
        fill_axis(r, A);
        r.in = p.in;
        r.in_c128 = p.in_c128;
        r.in_ld = n;
        r.in_bstride = np;
        r.in_n = n;
        r.out = S;
        r.out_ld = n;
        r.out_bstride = np;
        r.out_n = n;
        r.batch = p.ncomp;
        if (diag) {
            r.red = red_region(c, 0);
            r.red_pre = 1;
            r.red_moments = 1;
        }
        CK(prof_rows(c, c->fp64, r));
        if (diag) CK(launch_reduce_finish(r.red, (int)nbr, 1, RS_P, 4, redout_region(c, 0), c->st));
        ColArgs a = col_defaults(c, dx);
        a.mode = COL_FRAUNHOFER;
        a.ncols = n;
        fill_axis(a, A);
        a.W = auto_colw(c, A->L);
        a.src = S;
        a.src_ld = n;
        a.src_bstride = np;
        a.in_n = n;
        a.dst = O;
        a.dst_ld = n;
        a.dst_bstride = np;
        a.h.k = k;
        a.h.z = z;
        a.h.wl = wl;
        // cexpI(k z) * complex(0, -1/(wl z)), times the dx^2 of the transform
        const double cr = std::cos(k * z), ci = std::sin(k * z);
        const double a0 = -1 / (wl * z);
        a.fr_c_re = (-a0 * ci) * (dx * dx);
        a.fr_c_im = (a0 * cr) * (dx * dx);
        a.fr_dxout = dxout;
        a.fr_n = n;
        a.batch = p.ncomp;
        CK(prof_cols(c, c->fp64, a));
        if (O != p.out) CK(launch_convert(1, O, p.out, np * p.ncomp, c->st));
        if (d) {
            d->dx_out = dxout;
            TRY(fetch_red(c, 1));
            const double* m = c->hred;
            const double pw = m[RS_P];
            double din = 0;
            if (pw > 0) {
                const double cx = m[RS_PX] / pw, cy = m[RS_PY] / pw;
                double vr = m[RS_PR2] - pw * (cx * cx + cy * cy);
                if (vr < 0) vr = 0;
                din = 2 * std::sqrt(vr / pw);
            }
            d->rms_radius_in = din;
            d->p_in = pw * dx * dx;
            if (din > 0) {
                const double nf = din * din / (wl * std::fabs(z));
                if (nf > 0.5) warn_add(d, WOS_W_FRAUNHOFER_NEARFIELD, nf);
            }
        }
        return WOS_OK;
    }
    default:
        return fail(WOS_UNKNOWN_METHOD, "unknown propagation method " + std::to_string(p.method));
    }
}

// Host field staging: [ncomp][ny][nx] complex128 in c->stage.
int stage_in(wos_ctx c, const wos_field* f, int ncomp) {
    const size_t np = (size_t)f->ny * f->nx;
    TRY(ensure(c->stage, np * ncomp * 16));
    CK(cudaMemcpyAsync(c->stage.p, f->ex, np * 16, cudaMemcpyHostToDevice, c->st));
    if (ncomp == 2)
        CK(cudaMemcpyAsync(reinterpret_cast<char*>(c->stage.p) + np * 16, f->ey, np * 16, cudaMemcpyHostToDevice, c->st));
    return WOS_OK;
}

int stage_out(wos_ctx c, wos_field* f, int ncomp) {
    const size_t np = (size_t)f->ny * f->nx;
    CK(cudaMemcpyAsync(f->ex, c->stage.p, np * 16, cudaMemcpyDeviceToHost, c->st));
    if (ncomp == 2)
        CK(cudaMemcpyAsync(f->ey, reinterpret_cast<char*>(c->stage.p) + np * 16, np * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(c->err_host, c->err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return check_err_word(c);
}

int check_field(const wos_field* f) {
    if (!f || !f->ex || f->ny < 2 || f->nx < 2 || !(f->dx > 0) || (f->polarized && !f->ey))
        return fail(WOS_INVALID_ARG, "invalid wos_field");
    return WOS_OK;
}

wos_context default_context() {
    // nil *Context -> &Context{Evanescent: "decay"} (optics/propagate.go:72-74)
    wos_context c{};
    return c;
}

// fft2DCPU semantics (optics/fft.go:219-242): rows then columns, inverse
// scaled by 1/n per axis; `a` holds `batch` arrays in precision fp64.
int fft2d_impl(wos_ctx c, int fp64, int ny, int nx, int batch, void* a, int inverse) {
    Axis *ax, *ay;
    TRY(get_axis(c, nx, fp64, &ax));
    TRY(get_axis(c, ny, fp64, &ay));
    const long long np = (long long)ny * nx;
    RowArgs r = row_defaults(ny, nx, 1.0);
    r.mode = inverse ? ROW_INV : ROW_FWD;
    r.rows = ny;
    fill_axis(r, ax);
    r.in = a;
    r.in_ld = nx;
    r.in_bstride = np;
    r.in_n = nx;
    r.out = a;
    r.out_ld = nx;
    r.out_bstride = np;
    r.out_n = nx;
    r.out_scale = inverse ? 1.0 / (double)nx : 1.0;
    r.batch = batch;
    CK(prof_rows(c, fp64, r));
    ColArgs k = col_defaults(c, 1.0);
    k.h.exact = fp64;
    k.mode = COL_FFT;
    k.col_inverse = inverse;
    k.ncols = nx;
    fill_axis(k, ay);
    k.W = auto_colw_p(c, fp64, ay->L);
    k.src = a;
    k.src_ld = nx;
    k.src_bstride = np;
    k.in_n = ny;
    k.dst = a;
    k.dst_ld = nx;
    k.dst_bstride = np;
    k.out_n = ny;
    k.out_scale = inverse ? 1.0 / (double)ny : 1.0;
    k.batch = batch;
    CK(prof_cols(c, fp64, k));
    return WOS_OK;
}

// One plane view into the device float buffer `out` (see wos_plane_view);
// planes of precision fp64 (complex128) or complex64.
int plane_view_dev(wos_ctx c, int fp64, const void* ex, const void* ey, const void* ez, int pol, long long np,
                   int view, double mask_cut, void* out) {
    const double cut = mask_cut > 0 ? mask_cut : 2e-3;
    const double* peak = nullptr;
    if (view >= WOS_VIEW_PHASE_X) {
        const int nb = norm2_max_blocks(np);
        TRY(red_prepare(c, (size_t)(nb + RS_COUNT - 1) / RS_COUNT + 1));
        const void* comp = view == WOS_VIEW_PHASE_X ? ex : (view == WOS_VIEW_PHASE_Y ? ey : ez);
        double* o = redout_region(c, 0);
        CK(launch_norm2_max(fp64, comp, np, red_region(c, 0), o, c->st));
        peak = o;
    }
    CK(launch_plane_view(fp64, ex, ey, ez, pol, np, view, peak, cut, out, c->st));
    return WOS_OK;
}

void diag_merge(wos_diag* into, const wos_diag& d) {
    if (!into) return;
    for (int b = 0; b < WOS_W_COUNT; b++) {
        into->warn_count[b] += d.warn_count[b];
        if (d.warn_count[b] && d.warn_value[b] != 0) into->warn_value[b] = d.warn_value[b];
    }
}

}  // namespace wapi

// ====================================================================== ABI
extern "C" {

const char* wos_status_string(int s) {
    switch (s) {
    case WOS_OK: return "ok";
    case WOS_INVALID_ARG: return "invalid argument";
    case WOS_UNSUPPORTED_SIZE: return "unsupported size";
    case WOS_OOM: return "out of device memory";
    case WOS_CUDA_ERROR: return "CUDA error";
    case WOS_TIMEOUT: return "timeout";
    case WOS_NOT_INITIALISED: return "not initialised";
    case WOS_UNKNOWN_METHOD: return "unknown method";
    }
    return "unknown status";
}

const char* wos_last_error(void) { return g_err.c_str(); }
}  // extern "C"

namespace wos {
// error text of entry points defined in other translation units
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace wos

extern "C" {

int wos_fft2d_dev(wos_ctx c, int ny, int nx, int batch, void* a, int inverse) {
    if (!c || !a || ny < 2 || nx < 2 || batch < 1) return fail(WOS_INVALID_ARG, "fft2d_dev arguments");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    return fft2d_impl(c, c->fp64, ny, nx, batch, a, inverse);
}

int wos_fft2d(wos_ctx c, int ny, int nx, wos_c128* a, int inverse) {
    if (!c || !a || ny < 2 || nx < 2) return fail(WOS_INVALID_ARG, "fft2d arguments");
    const size_t np = (size_t)ny * nx;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        TRY(set_device(c));
        TRY(ensure(c->stage, np * 16));
        if (!c->fp64) TRY(ensure(c->scratch, np * 8));
        CK(cudaMemcpyAsync(c->stage.p, a, np * 16, cudaMemcpyHostToDevice, c->st));
        if (!c->fp64) CK(launch_convert(0, c->stage.p, c->scratch.p, (long long)np, c->st));
    }
    void* buf = c->fp64 ? c->stage.p : c->scratch.p;
    TRY(wos_fft2d_dev(c, ny, nx, 1, buf, inverse));
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->fp64) CK(launch_convert(1, c->scratch.p, c->stage.p, (long long)np, c->st));
    CK(cudaMemcpyAsync(a, c->stage.p, np * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

int wos_fft1d(wos_ctx c, int n, wos_c128* a, int inverse) {
    if (!c || !a || n < 2) return fail(WOS_INVALID_ARG, "fft1d arguments");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    Axis* ax;
    TRY(get_axis(c, n, c->fp64, &ax));
    TRY(ensure(c->stage, (size_t)n * 16));
    CK(cudaMemcpyAsync(c->stage.p, a, (size_t)n * 16, cudaMemcpyHostToDevice, c->st));
    RowArgs r = row_defaults(1, n, 1.0);
    r.mode = inverse ? ROW_INV : ROW_FWD;
    r.rows = 1;
    fill_axis(r, ax);
    r.in = c->stage.p;
    r.in_c128 = 1;
    r.in_ld = n;
    r.in_n = n;
    r.out = c->stage.p;
    r.out_c128 = 1;
    r.out_ld = n;
    r.out_n = n;
    r.out_scale = inverse ? 1.0 / (double)n : 1.0;
    CK(prof_rows(c, c->fp64, r));
    CK(cudaMemcpyAsync(a, c->stage.p, (size_t)n * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

// ---- Propagate
int wos_propagate_dev(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* in, void* out, double z,
                      int method, const wos_context* cc, wos_diag* diag) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    Prop p{ny, nx, dx, ncomp, in, 0, out, 0, z, method, cc ? *cc : default_context(), diag};
    return run_propagate(c, p);
}

int wos_propagate_dev_c128(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* in, void* out, double z,
                           int method, const wos_context* cc, wos_diag* diag) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    Prop p{ny, nx, dx, ncomp, in, 1, out, 1, z, method, cc ? *cc : default_context(), diag};
    return run_propagate(c, p);
}

int wos_propagate_batch_dev(wos_ctx c, int nfields, int ny, int nx, double dx, int ncomp, const void* const* in,
                            void* const* out, double z, int method, const wos_context* cci) {
    if (!c || nfields < 0 || (nfields > 0 && (!in || !out))) return fail(WOS_INVALID_ARG, "batch arguments");
    if (nfields == 0) return WOS_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    wos_context cc = cci ? *cci : default_context();
    cc.diagnostics = 0;
    for (int i = 0; i < nfields; i++)
        if (!in[i] || !out[i]) return fail(WOS_INVALID_ARG, "null field pointer in batch");
    // Independent fields on the specialised power-of-two ASM path touch no
    // context workspace (the sweeps run in place in each output), so they can
    // run concurrently on the context's side streams; the tables they share
    // are built first, on the context stream.  Two streams measured best at
    // 2048^2 complex64 (two 32 MiB fields in flight stay in L2; three thrash),
    // three for smaller fields.
    const bool concurrent = method == WOS_ASM && z != 0 && !c->no_fast && is_pow2(nx) && is_pow2(ny) &&
                            (c->fp64 || std::fabs(z / cc.wavelength) < 268435456.0) && nfields > 1;
    int nstreams = 0;
    if (concurrent) {
        const Tune t = get_tune(c, ny, nx);
        if (fast_supported(c->fp64, nx, t.rowE) && fast_supported(c->fp64, ny, t.colE)) {
            Axis *ax, *ay;
            const void *twx, *twy;
            TRY(get_axis(c, nx, c->fp64, &ax));
            TRY(get_axis(c, ny, c->fp64, &ay));
            TRY(fast_tw(c, ax, t.rowE, &twx));
            TRY(fast_tw(c, ay, t.colE, &twy));
            FastCols probe{};
            probe.W = t.colW;
            if (pair_eligible(c, ny, t.colE, probe)) {  // shared tables of the split column tiles
                const void *th, *tp;
                if (!pair_tables(c, ny, t.colE, &th, &tp)) return fail(WOS_CUDA_ERROR, "split-tile tables");
            }
            // the transfer-function table the (tiled) column sweeps read
            {
                FastCols hk{};
                hk.ncols = nx;
                fill_asm_h(hk, asm_h(c, cc, z, ev_policy(cc, z), dx, nx, ny));
                if (asm_tiled(c, ny, nx, t)) TRY(attach_htab_global(c, hk, ny));
                else TRY(attach_htab64(c, hk, ny));
            }
            // three streams for fields up to 16 MiB (1024^2 +4-5 %, 512^2
            // complex128 +20-30 %), two above (2048^2 complex64: 21.3k
            // against 18.9k props/s with three)
            const size_t fbytes = (size_t)ny * nx * ncomp * c->csz();
            const int def_streams = fbytes <= ((size_t)16 << 20) ? 3 : 2;
            nstreams = std::max(1, std::min(wos_ctx_s::kMaxAux, env_int("WOS_STREAMS", def_streams)));
        }
    }
    if (nstreams <= 1) {
        for (int i = 0; i < nfields; i++) {
            Prop p{ny, nx, dx, ncomp, in[i], 0, out[i], 0, z, method, cc, nullptr};
            TRY(run_propagate(c, p));
        }
        return WOS_OK;
    }
    if (!c->fork_ev) CK(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    while (c->naux < nstreams) {
        CK(cudaStreamCreateWithFlags(&c->side[c->naux], cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->join_ev[c->naux], cudaEventDisableTiming));
        c->naux++;
    }
    CK(cudaEventRecord(c->fork_ev, c->st));
    for (int k = 0; k < nstreams; k++) CK(cudaStreamWaitEvent(c->side[k], c->fork_ev, 0));
    const cudaStream_t home = c->st;
    int rc = WOS_OK;
    for (int i = 0; i < nfields && rc == WOS_OK; i++) {
        c->st = c->side[i % nstreams];
        c->cur_slot = 1 + i % nstreams;
        Prop p{ny, nx, dx, ncomp, in[i], 0, out[i], 0, z, method, cc, nullptr};
        rc = run_propagate(c, p);
    }
    c->st = home;
    c->cur_slot = 0;
    for (int k = 0; k < nstreams; k++) {
        CK(cudaEventRecord(c->join_ev[k], c->side[k]));
        CK(cudaStreamWaitEvent(c->st, c->join_ev[k], 0));
    }
    return rc;
}

int wos_propagate(wos_ctx c, wos_field* f, double z, int method, const wos_context* cc, wos_diag* diag) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    TRY(check_field(f));
    if (method < WOS_ASM || method > WOS_FRAUNHOFER) return fail(WOS_UNKNOWN_METHOD, "unknown propagation method");
    if (z == 0) {
        if (diag) {
            std::memset(diag, 0, sizeof(*diag));
            diag->dx_out = f->dx;
        }
        return WOS_OK;
    }
    // a pageable field goes through the host batch's page-locked staging
    if (host_pageable(f->ex) || (f->polarized && host_pageable(f->ey)))
        return wos_propagate_batch(c, 1, f, z, method, cc, diag);
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int ncomp = f->polarized ? 2 : 1;
    TRY(stage_in(c, f, ncomp));
    Prop p{f->ny, f->nx, f->dx, ncomp, c->stage.p, 1, c->stage.p, 1, z, method, cc ? *cc : default_context(), diag};
    wos_diag local;
    if (!p.diag && method == WOS_FRAUNHOFER) p.diag = &local;  // the new pitch is needed below
    TRY(run_propagate(c, p));
    TRY(stage_out(c, f, ncomp));
    if (method == WOS_FRAUNHOFER) f->dx = p.diag->dx_out;
    return WOS_OK;
}

}  // extern "C"

// wos_batch.cu -- batches of units sharing a geometry: PropagatePolychromatic
// (optics/polychromatic.go:18-44), Propagate3D (optics/volume.go:8-18) and
// the Gaussian-Schell source (optics/coherence.go:22-116), on one row
// spectrum and per-chunk column launches.
#include "wos_api_internal.cuh"

namespace wapi {

// FFT2D of a complex128 device array in FP64, whatever the context precision
// (one-time source synthesis).
int fft2d_fp64(wos_ctx c, int n, int batch, double2* a, int inverse) {
    return fft2d_impl(c, 1, n, n, batch, a, inverse);
}

// GenerateSchellRealizations (optics/coherence.go:22-80) into modes (device, complex128)
int schell_generate(wos_ctx c, int n, double dx, double width, double coh, int m, const void* noise, bool noise_dev,
                    double2* modes) {
    const long long nn = (long long)n * n;
    TRY(ensure(c->aux, (size_t)nn * (16 + 8)));
    double2* mu = reinterpret_cast<double2*>(c->aux.p);
    double* sqs = reinterpret_cast<double*>(mu + nn);
    CK(launch_schell_mu(mu, n, dx, coh, c->st));
    TRY(fft2d_fp64(c, n, 1, mu, 0));
    CK(launch_sqrt_re(sqs, mu, nn, c->st));
    CK(cudaMemcpyAsync(modes, noise, (size_t)nn * m * 16, noise_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       c->st));
    CK(launch_mul_map(modes, sqs, nn, m, c->st));
    TRY(fft2d_fp64(c, n, m, modes, 1));
    CK(launch_schell_env(modes, n, dx, width, m, c->st));
    return WOS_OK;
}

// Batched ASM over units that share a geometry (polychromatic wavelengths,
// volume distances, coherent modes): one row sweep per unit set, one column
// launch per chunk with gridDim.y = units, then either a batched inverse row
// sweep (planes out) or an accumulating one (intensity out).
struct Batch {
    int ny, nx, ncomp;
    double dx;
    const void* in;       // complex128 device input [ncomp or units][ny][nx]
    long long in_unit_stride;  // elements between units of the input (0: shared input)
    int units;
    const double* wl_dev;  // per-unit wavelength (device) or null
    const double* z_dev;   // per-unit z (device) or null
    std::vector<double> wl, z;  // host copies
    const double* w_dev;   // per-unit intensity weight (device) or null
    double* out_int;       // device [ny][nx] FP64 intensity accumulation, or null
    void* out_planes;      // device complex128 [units][ncomp][ny][nx], or null
    wos_context cc;
    wos_diag* diag;
    int in_native = 0;     // in holds the context's complex type, not complex128
    int out_native = 0;    // out_planes of the context's complex type
    // Gaussian-Schell realizations synthesised inside the sweeps: in holds the
    // units' noise (complex128), schell_sq the map sqrt(S) and schell_g the
    // envelope factor exp(-t^2/w^2)/n of one axis (square grid; the 1/n of
    // each inverse axis folded in).  Only the specialised sweeps run it.
    const double* schell_sq = nullptr;
    const double* schell_g = nullptr;
    size_t in_esz(wos_ctx c) const { return in_native ? c->csz() : 16; }
    size_t out_esz(wos_ctx c) const { return out_native ? c->csz() : 16; }
};

// Grid sizes of the fused Gaussian-Schell sweeps (wos_schell.cu).
bool schell_fast_size(int n) { return is_pow2(n) && n >= 256 && n <= 4096; }

// Batched ASM on the specialised sweeps (power-of-two grids): the forward row
// sweep once per component for a shared input, then per chunk of units one
// column sweep (gridDim.y = units, per-unit wavelength / distance, the shared
// row spectrum as its source) and one row sweep that either accumulates the
// weighted intensity of the chunk in registers or writes each unit's plane.
// Diagnostics: per-unit spectral loss sums and histograms from the column
// records, input power from the row records.  -1: not eligible.
int try_fast_batch(wos_ctx c, Batch& b, std::vector<double>& sums, std::vector<double>& pin_unit,
                   double& pin_total) {
    const int ny = b.ny, nx = b.nx, ncomp = b.ncomp;
    if (c->no_fast || !is_pow2(nx) || !is_pow2(ny)) return -1;
    if (!c->fp64) {
        for (int u = 0; u < b.units; u++) {
            const double wl = b.wl.empty() ? b.cc.wavelength : b.wl[u];
            const double z = b.z.empty() ? 0.0 : b.z[u];
            if (!(std::fabs(z / wl) < 268435456.0)) return -1;
        }
    }
    const Tune t = get_tune(c, ny, nx);
    if (!fast_supported(c->fp64, nx, t.rowE) || !fast_supported(c->fp64, ny, t.colE)) return -1;
    const double dx = b.dx;
    const long long np = (long long)ny * nx;
    const bool shared_in = b.in_unit_stride == 0;
    const bool diag = b.diag != nullptr;
    const bool schell = b.schell_sq != nullptr;
    if (schell && (diag || shared_in || ncomp != 1 || !schell_fast_size(nx) || nx != ny)) return -1;
    // a shared input is column-transformed once; every unit's column sweep
    // then starts from that spectrum (H, inverse)
    const bool spec = shared_in && !diag && !schell && schell_fast_size(ny);
    Axis *ax, *ay;
    TRY(get_axis(c, nx, c->fp64, &ax));
    TRY(get_axis(c, ny, c->fp64, &ay));
    const void *twx, *twy, *twx8 = nullptr, *twy8 = nullptr;
    TRY(fast_tw(c, ax, t.rowE, &twx));
    TRY(fast_tw(c, ay, t.colE, &twy));
    if (schell || spec) {
        TRY(fast_tw(c, ax, 8, &twx8));
        TRY(fast_tw(c, ay, 8, &twy8));
    }
    // all units of a batch in one launch per sweep, up to 4 GiB of
    // intermediates: chunks small enough to stay in L2 (16 - 64 MiB) measured
    // slower (cfg4 3.69 -> 4.31 ms at 16 MiB): the launches lose parallelism
    const size_t per = (size_t)np * c->csz();
    int B = (int)std::max<size_t>(1, ((size_t)4 << 30) / per);
    B = std::min(B, b.units);
    B = std::min(B, 65535);
    const size_t nbr = fast_row_blocks(nx, t.rowE, ny, shared_in ? 1 : B);
    const size_t nbc = fast_col_blocks(c->fp64, ny, t.colE, t.colW, nx, 1);
    TRY(red_prepare(c, std::max(nbr, nbc * (size_t)B)));
    if (diag) TRY(ensure(c->tmp, sizeof(double) * RS_COUNT * (size_t)B));
    TRY(ensure(c->scratch, (size_t)(shared_in ? 1 : B) * per));
    TRY(ensure(c->scratch2, (size_t)B * per));
    void* S0 = c->scratch.p;
    void* S1 = c->scratch2.p;
    const Policy pol = ev_policy(b.cc, b.z.empty() ? 1.0 : b.z[0]);
    const HArgs h = asm_h(c, b.cc, b.z.empty() ? 0.0 : b.z[0], pol, dx, nx, ny);
    double* o = reinterpret_cast<double*>(c->tmp.p);
    int nb = 0;
    for (int comp = 0; comp < ncomp; comp++) {
        for (int k0 = 0; k0 < b.units; k0 += B) {
            const int nu = std::min(B, b.units - k0);
            if (k0 == 0 || !shared_in) {
                FastRows r{};
                r.rows = ny;
                r.in = reinterpret_cast<const char*>(b.in) +
                       b.in_esz(c) * (shared_in ? comp * np : ((long long)k0 * ncomp + comp) * np);
                r.in_c128 = !b.in_native;
                r.in_ld = nx;
                r.in_bstride = shared_in ? 0 : ncomp * np;
                r.out = S0;
                r.out_ld = nx;
                r.out_bstride = np;
                r.tw = twx;
                r.out_scale = 1.0;
                r.batch = shared_in ? 1 : nu;
                if (diag) {
                    r.red = red_region(c, 0) + RS_P;
                    r.red_stride = RS_COUNT;
                }
                if (schell) {
                    r.tw = twx8;
                    r.pre_map = b.schell_sq;
                    r.env_x = b.schell_g;
                    CK(timed_launch(c, 0, [&] { return fast_rows_schell(c->fp64, nx, 8, r, c->st, &nb); }));
                } else {
                    CK(timed_launch(c, 0, [&] { return fast_rows(c->fp64, nx, t.rowE, false, r, c->st, &nb); }));
                }
                if (spec) {  // the column spectrum of the shared input, once
                    Axis* ag;
                    TRY(get_axis(c, ny, c->fp64, &ag));
                    ColArgs f = col_defaults(c, dx);
                    f.mode = COL_FFT;
                    f.ncols = nx;
                    fill_axis(f, ag);
                    f.W = auto_colw(c, ag->L);
                    f.src = S0;
                    f.src_ld = nx;
                    f.in_n = ny;
                    f.dst = S0;
                    f.dst_ld = nx;
                    f.out_n = ny;
                    CK(prof_cols(c, c->fp64, f));
                }
                if (diag) {
                    const int per_unit = nb / r.batch;
                    CK(launch_reduce_finish(red_region(c, 0), per_unit, r.batch, RS_P, 1, o, c->st));
                    std::vector<double> hh((size_t)r.batch * RS_COUNT);
                    CK(cudaMemcpyAsync(hh.data(), o, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, c->st));
                    CK(cudaStreamSynchronize(c->st));
                    for (int u = 0; u < r.batch; u++) {
                        const double p = hh[(size_t)u * RS_COUNT + RS_P] * dx * dx;
                        if (shared_in) pin_total += p;
                        else pin_unit[k0 + u] += p;
                    }
                }
            }
            FastCols k{};
            k.ncols = nx;
            k.W = t.colW;
            k.data = S1;
            k.ld = nx;
            k.bstride = np;
            k.src = S0;
            k.src_bstride = shared_in ? 0 : np;
            k.tw = twy;
            k.batch = nu;
            k.wl = b.cc.wavelength;
            k.dx = dx;
            k.z = b.z.empty() ? 0.0 : b.z[0];
            k.kz = h.kz;
            k.kaz = h.kaz;
            k.krev = h.kz / (2 * M_PI);
            k.batch_wl = b.wl_dev ? b.wl_dev + k0 : nullptr;
            k.batch_z = b.z_dev ? b.z_dev + k0 : nullptr;
            k.scale = h.scale;
            k.alpha = h.alpha;
            k.limit = h.limit;
            k.zero_ev = h.zero_ev;
            k.reg = h.reg;
            k.backward = h.z < 0;
            if (diag) {
                k.red = red_region(c, 1) + RS_SW;
                k.red_stride = RS_COUNT;
                k.hist = red_region(c, 1) + RS_HIST;
                k.hist_dx = dx;
            }
            if (schell) {
                k.tw = twy8;
                k.W = 4;
                k.env_y = b.schell_g;
                CK(timed_launch(c, 4, [&] { return fast_cols_env(c->fp64, ny, 8, k, c->st, &nb); }));
            } else if (spec) {
                k.tw = twy8;
                k.W = 4;
                CK(timed_launch(c, 4, [&] { return fast_cols_spec(c->fp64, ny, 8, k, c->st, &nb); }));
            } else {
                CK(timed_launch(c, 4, [&] { return sweep_cols(c, ny, t.colE, k, &nb); }));
            }
            if (diag) {
                const int per_unit = nb / nu;
                CK(launch_reduce_finish(red_region(c, 1), per_unit, nu, RS_SW, 2, o, c->st));
                CK(launch_reduce_finish(red_region(c, 1), per_unit, nu, RS_HIST, 97, o, c->st));
                std::vector<double> hh((size_t)nu * RS_COUNT);
                CK(cudaMemcpyAsync(hh.data(), o, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, c->st));
                CK(cudaStreamSynchronize(c->st));
                for (int u = 0; u < nu; u++)
                    for (int sl = RS_SW; sl < RS_COUNT; sl++)
                        sums[((size_t)(k0 + u) * ncomp + comp) * RS_COUNT + sl] = hh[(size_t)u * RS_COUNT + sl];
            }
            FastRows q{};
            q.rows = ny;
            q.in = S1;
            q.in_ld = nx;
            q.in_bstride = np;
            q.tw = twx;
            q.out_scale = 1.0;
            if (b.out_int) {
                AccArgs acc{nu, b.w_dev ? b.w_dev + k0 : nullptr, b.out_int, 1};
                CK(timed_launch(c, 1, [&] { return fast_rows_acc(c->fp64, nx, t.rowE, q, acc, c->st, &nb); }));
            } else {
                q.out = reinterpret_cast<char*>(b.out_planes) + b.out_esz(c) * (((long long)k0 * ncomp + comp) * np);
                q.out_c128 = !b.out_native;
                q.out_ld = nx;
                q.out_bstride = ncomp * np;
                q.batch = nu;
                CK(timed_launch(c, 1, [&] { return fast_rows(c->fp64, nx, t.rowE, true, q, c->st, &nb); }));
            }
        }
    }
    return WOS_OK;
}

int run_batch_asm(wos_ctx c, Batch& b) {
    const int ny = b.ny, nx = b.nx, ncomp = b.ncomp;
    const double dx = b.dx;
    const long long np = (long long)ny * nx;
    Axis *ax, *ay;
    TRY(get_axis(c, nx, c->fp64, &ax));
    TRY(get_axis(c, ny, c->fp64, &ay));
    const int W = auto_colw(c, ay->L);
    const bool shared_in = b.in_unit_stride == 0;
    // chunk the units so the per-chunk spectra stay within ~4 GiB
    const size_t per = (size_t)np * c->csz();
    int B = (int)std::max<size_t>(1, ((size_t)4 << 30) / per);
    B = std::min(B, b.units);
    B = std::min(B, 65535);
    const size_t nbr1 = row_blocks(c->fp64, ax->L, ny, shared_in ? 1 : B);
    const size_t nbc1 = col_blocks(c->fp64, ay->L, W, nx, 1);
    TRY(red_prepare(c, std::max(nbr1, nbc1 * (size_t)B)));
    const bool diag = b.diag != nullptr;
    // spectral sums per unit and component, plus a histogram per unit
    std::vector<double> sums((size_t)b.units * RS_COUNT * ncomp, 0.0);
    if (diag) TRY(ensure(c->tmp, sizeof(double) * RS_COUNT * (size_t)B));
    TRY(ensure(c->scratch, (size_t)(shared_in ? 1 : B) * per));
    TRY(ensure(c->scratch2, (size_t)B * per));
    void* S0 = c->scratch.p;
    void* S1 = c->scratch2.p;
    const Policy pol = ev_policy(b.cc, b.z.empty() ? 1.0 : b.z[0]);
    double pin_total = 0;
    std::vector<double> pin_unit(b.units, 0.0);
    const int fast = try_fast_batch(c, b, sums, pin_unit, pin_total);
    if (fast != -1 && fast != WOS_OK) return fast;
    if (fast == -1 && b.schell_sq) return -1;  // the caller synthesises the realizations first
    // a shared input is column-transformed once and every unit's column sweep
    // starts from that spectrum (H, inverse), where the lines need no Bluestein
    bool spec = false;
    if (shared_in && !diag) {
        ColArgs probe = col_defaults(c, dx);
        fill_axis(probe, ay);
        spec = probe.blue_n == 0;
    }
    for (int comp = 0; comp < ncomp && fast == -1; comp++) {
        for (int k0 = 0; k0 < b.units; k0 += B) {
            const int nb = std::min(B, b.units - k0);
            // rows forward (the shared input once per component, else per unit)
            if (k0 == 0 || !shared_in) {
                RowArgs r = row_defaults(ny, nx, dx);
                r.mode = ROW_FWD;
                r.rows = ny;
                fill_axis(r, ax);
                r.in = reinterpret_cast<const char*>(b.in) +
                       b.in_esz(c) * (shared_in ? comp * np : ((long long)k0 * ncomp + comp) * np);
                r.in_c128 = !b.in_native;
                r.in_ld = nx;
                r.in_bstride = shared_in ? 0 : ncomp * np;
                r.in_n = nx;
                r.out = S0;
                r.out_ld = nx;
                r.out_bstride = np;
                r.out_n = nx;
                r.batch = shared_in ? 1 : nb;
                if (diag) {
                    r.red = red_region(c, 0);
                    r.red_pre = 1;
                }
                CK(prof_rows(c, c->fp64, r));
                if (diag) {
                    const int nbr = (int)row_blocks(c->fp64, ax->L, ny, 1);
                    CK(launch_reduce_finish(r.red, nbr, r.batch, RS_P, 1, reinterpret_cast<double*>(c->tmp.p), c->st));
                    std::vector<double> h((size_t)r.batch * RS_COUNT);
                    CK(cudaMemcpyAsync(h.data(), c->tmp.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
                    CK(cudaStreamSynchronize(c->st));
                    for (int u = 0; u < r.batch; u++) {
                        const double p = h[(size_t)u * RS_COUNT + RS_P] * dx * dx;
                        if (shared_in) pin_total += p;
                        else pin_unit[k0 + u] += p;
                    }
                }
                if (spec) {  // the shared input's column transform, once for all units
                    ColArgs f = col_defaults(c, dx);
                    f.mode = COL_FFT;
                    f.ncols = nx;
                    fill_axis(f, ay);
                    f.W = W;
                    f.src = S0;
                    f.src_ld = nx;
                    f.in_n = ny;
                    f.dst = S0;
                    f.dst_ld = nx;
                    f.out_n = ny;
                    CK(prof_cols(c, c->fp64, f));
                }
            }
            ColArgs a = col_defaults(c, dx);
            a.mode = COL_FUSED;
            a.ncols = nx;
            fill_axis(a, ay);
            a.W = W;
            a.src = S0;
            a.src_ld = nx;
            a.src_bstride = np;
            a.src_shared = shared_in;
            a.in_n = ny;
            a.dst = S1;
            a.dst_ld = nx;
            a.dst_bstride = np;
            a.out_n = ny;
            a.h = asm_h(c, b.cc, b.z.empty() ? 0.0 : b.z[0], pol, dx, nx, ny);
            a.h.wl = -1;  // per-unit k, k z, k |z| are formed on the device from wl and z
            a.batch_wl = b.wl_dev ? b.wl_dev + k0 : nullptr;
            a.batch_z = b.z_dev ? b.z_dev + k0 : nullptr;
            if (!b.wl_dev) a.h.wl = b.cc.wavelength, a.h.k = 2 * M_PI / b.cc.wavelength;
            a.batch = nb;
            a.src_spectrum = spec;
            if (diag) {
                a.red = red_region(c, 1);
                a.red_bpm = 1;
                a.red_hist = 1;
                a.hist_lx = nx;
                a.hist_ly = ny;
                a.hist_dx = dx;
            }
            CK(prof_cols(c, c->fp64, a));
            if (diag) {
                double* o = reinterpret_cast<double*>(c->tmp.p);
                CK(launch_reduce_finish(a.red, (int)nbc1, nb, RS_SW, 3, o, c->st));
                CK(launch_reduce_finish(a.red, (int)nbc1, nb, RS_HIST, 97, o, c->st));
                std::vector<double> h((size_t)nb * RS_COUNT);
                CK(cudaMemcpyAsync(h.data(), o, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
                CK(cudaStreamSynchronize(c->st));
                for (int u = 0; u < nb; u++)
                    for (int sl = RS_SW; sl < RS_COUNT; sl++)
                        sums[((size_t)(k0 + u) * ncomp + comp) * RS_COUNT + sl] = h[(size_t)u * RS_COUNT + sl];
            }
            RowArgs q = row_defaults(ny, nx, dx);
            q.rows = ny;
            fill_axis(q, ax);
            q.in = S1;
            q.in_ld = nx;
            q.in_bstride = np;
            q.in_n = nx;
            q.out_ld = nx;
            q.out_n = nx;
            if (b.out_int) {
                q.mode = ROW_INV_ACC;
                q.acc_nb = nb;
                q.acc_weight = b.w_dev ? b.w_dev + k0 : nullptr;
                q.acc_add = 1;
                q.out = b.out_int;
                q.out_accum_int = 2;
                q.out_bstride = 0;
                q.batch = 1;
            } else {
                q.mode = ROW_INV;
                q.out = reinterpret_cast<char*>(b.out_planes) + b.out_esz(c) * (((long long)k0 * ncomp + comp) * np);
                q.out_c128 = !b.out_native;
                q.out_bstride = ncomp * np;
                q.batch = nb;
            }
            CK(prof_rows(c, c->fp64, q));
        }
    }
    if (diag) {
        // per unit, in order: asmWrapWarn then asmWarn (optics/propagate.go:325-332)
        for (int u = 0; u < b.units; u++) {
            wos_context cu = b.cc;
            if (!b.wl.empty()) cu.wavelength = b.wl[u];
            const double zu = b.z.empty() ? 0.0 : b.z[u];
            if (zu == 0) continue;
            double sw = 0, s1 = 0, hist[97] = {0};
            for (int comp = 0; comp < ncomp; comp++) {
                const double* rr = &sums[((size_t)u * ncomp + comp) * RS_COUNT];
                sw += rr[RS_SW];
                s1 += rr[RS_SW + 1];
                for (int k = 0; k < 97; k++) hist[k] += rr[RS_HIST + k];
            }
            if (wrap_needed(cu, ny, nx, dx, zu)) wrap_finish(b.diag, cu, ny, nx, dx, zu, hist);
            const double pin = shared_in ? pin_total : pin_unit[u];
            const double frac = sw > 0 ? s1 / sw : 0.0;  // spectral loss fraction of the step
            asm_warn(b.diag, zu, pin, pin - pin * frac, ev_policy(cu, zu));
        }
    }
    return WOS_OK;
}

// Device copy of a small parameter list (wavelengths, distances, weights of
// the device-resident batches): an earlier call's copy holding the same
// values is reused, so a repeated call copies nothing from the host.
int cached_params(wos_ctx c, const std::vector<double>& v, const double** out) {
    for (auto& ps : c->pslot)
        if (ps.buf.p && ps.host == v) {
            if (c->capturing) ps.frozen = true;
            *out = reinterpret_cast<const double*>(ps.buf.p);
            return WOS_OK;
        }
    // the next slot round robin that no captured graph reads, else a new one
    int slot = -1;
    for (size_t i = 0; i < c->pslot.size() && slot < 0; i++) {
        const int j = (int)((c->pslot_next + i) % c->pslot.size());
        if (!c->pslot[j].frozen) slot = j;
    }
    if (slot < 0) {
        c->pslot.emplace_back();
        slot = (int)c->pslot.size() - 1;
    }
    c->pslot_next = (slot + 1) % (int)c->pslot.size();
    wos_ctx_s::ParamSlot& ps = c->pslot[slot];
    ps.frozen = c->capturing;
    ps.host.clear();
    TRY(ensure(ps.buf, sizeof(double) * std::max<size_t>(v.size(), 1)));
    ps.host = v;  // the copy's source: it lives as long as the slot's contents
    if (!v.empty())
        CK(cudaMemcpyAsync(ps.buf.p, ps.host.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice, c->st));
    *out = reinterpret_cast<const double*>(ps.buf.p);
    return WOS_OK;
}

int check_dev_geometry(int ny, int nx, double dx, int ncomp) {
    if (ny < 2 || nx < 2 || ncomp < 1 || ncomp > 2 || !(dx > 0)) return fail(WOS_INVALID_ARG, "invalid field geometry");
    return WOS_OK;
}

// Modes [m0, m0 + count) of an m-mode Gaussian-Schell source (device noise
// [m][n][n] complex128) propagated to z and averaged with weight 1/m into out
// (device FP64 [n][n], overwritten): the whole source when m0 = 0 and count =
// m, one rank's share of a sharded run otherwise.
// The Gaussian-Schell tables of the fused sweeps: sqrt(max(0, Re FFT2(mu)))
// (FP64, [n][n], as GenerateSchellRealizations forms it) and the envelope
// factor of one axis, g(t) = exp(-t^2/w^2) / n (sqrt(I(x, y)) = g(x) g(y) n^2
// with I = exp(-2 (x^2 + y^2) / w^2); the 1/n of each inverse axis folded in).
int schell_tables(wos_ctx c, int n, double dx, double width, double coh, const double** sq, const double** g) {
    const long long nn = (long long)n * n;
    TRY(ensure(c->aux, (size_t)nn * (16 + 8)));
    double2* mu = reinterpret_cast<double2*>(c->aux.p);
    double* sqs = reinterpret_cast<double*>(mu + nn);
    CK(launch_schell_mu(mu, n, dx, coh, c->st));
    TRY(fft2d_fp64(c, n, 1, mu, 0));
    CK(launch_sqrt_re(sqs, mu, nn, c->st));
    std::vector<double> gh(n);
    for (int i = 0; i < n; i++) {
        const double x = ((double)i - (double)n / 2) * dx;
        gh[i] = std::exp(-(x * x) / (width * width)) / (double)n;
    }
    TRY(cached_params(c, gh, g));
    *sq = sqs;
    return WOS_OK;
}

// Realizations count of noise (device complex128 [count][n][n]) synthesised
// inside the propagation sweeps and their weighted intensities added into out
// (device FP64 [n][n]); -1 when the fused sweeps do not cover the case.
int schell_fused(wos_ctx c, int n, double dx, double width, double coh, int m, int count, const double2* noise,
                 double z, const wos_context& cc, double* out) {
    if (c->no_fast || z == 0 || !schell_fast_size(n)) return -1;
    const double *sq, *g, *w_d;
    TRY(schell_tables(c, n, dx, width, coh, &sq, &g));
    TRY(cached_params(c, std::vector<double>(count, 1 / (double)m), &w_d));
    const long long nn = (long long)n * n;
    Batch b{n, n, 1, dx, noise, nn, count, nullptr, nullptr, {}, std::vector<double>(count, z), w_d, out, nullptr, cc,
            nullptr};
    b.schell_sq = sq;
    b.schell_g = g;
    return run_batch_asm(c, b);
}

int schell_dev_range(wos_ctx c, int n, double dx, double width, double coherence, int m, int m0, int count,
                     const void* noise, double z, const wos_context* cci, double* out) {
    if (!c || !noise || !out) return fail(WOS_INVALID_ARG, "null argument");
    TRY(check_dev_geometry(n, n, dx, 1));
    if (!(width > 0) || !(coherence > 0)) return fail(WOS_INVALID_ARG, "schell: width and coherence must be > 0");
    if (m0 < 0 || count < 0 || m0 + count > m) return fail(WOS_INVALID_ARG, "schell: mode range outside the source");
    wos_context cc = cci ? *cci : default_context();
    cc.diagnostics = 0;
    if (z != 0 && !(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long nn = (long long)n * n;
    CK(cudaMemsetAsync(out, 0, sizeof(double) * nn, c->st));
    if (count == 0) return WOS_OK;
    {
        const int rc = schell_fused(c, n, dx, width, coherence, m, count,
                                    reinterpret_cast<const double2*>(noise) + m0 * nn, z, cc, out);
        if (rc != -1) return rc;
    }
    TRY(ensure(c->vol, sizeof(double2) * (size_t)nn * count));
    double2* modes = reinterpret_cast<double2*>(c->vol.p);
    TRY(schell_generate(c, n, dx, width, coherence, count, reinterpret_cast<const double2*>(noise) + m0 * nn, true,
                        modes));
    const double inv = 1 / (double)m;
    if (z == 0) {
        for (int q = 0; q < count; q++) CK(launch_accum_int(1, out, modes + q * nn, 1, nn, inv, c->st));
        return WOS_OK;
    }
    const double* w_d;
    TRY(cached_params(c, std::vector<double>(count, inv), &w_d));
    Batch b{n, n, 1, dx, modes, nn, count, nullptr, nullptr, {}, std::vector<double>(count, z), w_d, out, nullptr, cc,
            nullptr};
    return run_batch_asm(c, b);
}



int upload_params(wos_ctx c, const std::vector<double>& a, const std::vector<double>& b2,
                  const std::vector<double>& c3, double** pa, double** pb, double** pc) {
    const size_t n = a.size() + b2.size() + c3.size();
    TRY(ensure(c->params, sizeof(double) * std::max<size_t>(n, 1)));
    double* p = reinterpret_cast<double*>(c->params.p);
    std::vector<double> all;
    all.insert(all.end(), a.begin(), a.end());
    all.insert(all.end(), b2.begin(), b2.end());
    all.insert(all.end(), c3.begin(), c3.end());
    if (n) CK(cudaMemcpyAsync(p, all.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
    *pa = p;
    *pb = p + a.size();
    *pc = p + a.size() + b2.size();
    return WOS_OK;
}

}  // namespace wapi

extern "C" {

int wos_polychromatic(wos_ctx c, const wos_field* f, double z, const double* wavelengths, const double* weights,
                      int nsamples, int method, const wos_context* base, double* out, wos_diag* diag) {
    if (!c || !wavelengths || !weights || !out) return fail(WOS_INVALID_ARG, "null argument");
    TRY(check_field(f));
    if (nsamples <= 0) return fail(WOS_INVALID_ARG, "polychromatic: no wavelength samples");
    for (int s = 0; s < nsamples; s++)
        if (!(wavelengths[s] > 0)) return fail(WOS_INVALID_ARG, "polychromatic: wavelength must be > 0");
    if (method < WOS_ASM || method > WOS_FRAUNHOFER) return fail(WOS_UNKNOWN_METHOD, "unknown propagation method");
    if (diag) {
        std::memset(diag, 0, sizeof(*diag));
        diag->dx_out = f->dx;
    }
    // a nil base context means Context{Evanescent: "decay", Warnings: &Warnings{}}
    wos_context cc = base ? *base : default_context();
    if (!base) cc.diagnostics = 1;
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int ncomp = f->polarized ? 2 : 1;
    const long long np = (long long)f->ny * f->nx;
    TRY(stage_in(c, const_cast<wos_field*>(f), ncomp));
    TRY(ensure(c->accum, sizeof(double) * np));
    double* acc = reinterpret_cast<double*>(c->accum.p);
    CK(cudaMemsetAsync(acc, 0, sizeof(double) * np, c->st));
    wos_diag* dp = (cc.diagnostics && diag) ? diag : nullptr;
    if (z == 0) {
        for (int s = 0; s < nsamples; s++) CK(launch_accum_int(1, acc, c->stage.p, ncomp, np, weights[s], c->st));
    } else if (method == WOS_ASM) {
        std::vector<double> wl(wavelengths, wavelengths + nsamples), w(weights, weights + nsamples);
        double *wl_d, *w_d, *unused;
        TRY(upload_params(c, wl, w, {}, &wl_d, &w_d, &unused));
        Batch b{f->ny, f->nx, ncomp, f->dx, c->stage.p, 0, nsamples, wl_d, nullptr, wl,
                std::vector<double>(nsamples, z), w_d, acc, nullptr, cc, dp};
        TRY(run_batch_asm(c, b));
    } else {
        TRY(ensure(c->scratch3, (size_t)np * ncomp * c->csz()));
        void* O = c->scratch3.p;
        for (int s = 0; s < nsamples; s++) {
            wos_context cs = cc;
            cs.wavelength = wavelengths[s];
            wos_diag ds;
            Prop p{f->ny, f->nx, f->dx, ncomp, c->stage.p, 1, O, 0, z, method, cs, dp ? &ds : nullptr};
            TRY(run_propagate(c, p));
            if (dp) diag_merge(dp, ds);
            CK(launch_accum_int(c->fp64, acc, O, ncomp, np, weights[s], c->st));
        }
    }
    CK(cudaMemcpyAsync(out, acc, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

int wos_volume(wos_ctx c, const wos_field* f, const double* zs, int nz, int method, const wos_context* cci,
               wos_c128* out, wos_diag* diag) {
    if (!c || (nz > 0 && (!zs || !out)) || nz < 0) return fail(WOS_INVALID_ARG, "null argument");
    TRY(check_field(f));
    if (method < WOS_ASM || method > WOS_FRAUNHOFER) return fail(WOS_UNKNOWN_METHOD, "unknown propagation method");
    if (diag) {
        std::memset(diag, 0, sizeof(*diag));
        diag->dx_out = f->dx;
    }
    if (nz == 0) return WOS_OK;
    const wos_context cc = cci ? *cci : default_context();
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int ncomp = f->polarized ? 2 : 1;
    const long long np = (long long)f->ny * f->nx;
    TRY(stage_in(c, const_cast<wos_field*>(f), ncomp));
    TRY(ensure(c->vol, sizeof(double2) * (size_t)np * ncomp * nz));
    double2* O = reinterpret_cast<double2*>(c->vol.p);
    bool batched = method == WOS_ASM;
    std::vector<double> zb;
    std::vector<int> idx;
    for (int q = 0; q < nz; q++) {
        if (zs[q] != 0) {
            zb.push_back(zs[q]);
            idx.push_back(q);
            if (zs[q] < 0) batched = false;
        }
    }
    wos_diag* dp = diag;
    if (batched && !zb.empty()) {
        // the batch writes its planes compactly, then they move to their slots
        TRY(ensure(c->scratch3, sizeof(double2) * (size_t)np * ncomp * zb.size()));
        double2* Ob = reinterpret_cast<double2*>(c->scratch3.p);
        double *z_d, *u1, *u2;
        TRY(upload_params(c, zb, {}, {}, &z_d, &u1, &u2));
        Batch b{f->ny, f->nx, ncomp, f->dx, c->stage.p, 0, (int)zb.size(), nullptr, z_d, {}, zb, nullptr, nullptr,
                Ob, cc, (cc.diagnostics && dp) ? dp : nullptr};
        TRY(run_batch_asm(c, b));
        for (size_t u = 0; u < zb.size(); u++)
            CK(cudaMemcpyAsync(O + (size_t)idx[u] * ncomp * np, Ob + u * ncomp * np, sizeof(double2) * ncomp * np,
                               cudaMemcpyDeviceToDevice, c->st));
    } else {
        for (size_t u = 0; u < zb.size(); u++) {
            wos_diag ds;
            Prop p{f->ny, f->nx, f->dx, ncomp, c->stage.p, 1, O + (size_t)idx[u] * ncomp * np, 1, zb[u], method, cc,
                   (cc.diagnostics && dp) ? &ds : nullptr};
            TRY(run_propagate(c, p));
            if (cc.diagnostics && dp) diag_merge(dp, ds);
        }
    }
    // z == 0 returns the input unchanged (optics/propagate.go:66-68)
    for (int q = 0; q < nz; q++)
        if (zs[q] == 0)
            CK(cudaMemcpyAsync(O + (size_t)q * ncomp * np, c->stage.p, sizeof(double2) * ncomp * np,
                               cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(out, O, sizeof(double2) * (size_t)np * ncomp * nz, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

int wos_schell_modes(wos_ctx c, int n, double dx, double width, double coherence, int m, const wos_c128* noise,
                     wos_c128* modes_out) {
    if (!c || !noise || !modes_out || n < 2 || !(dx > 0)) return fail(WOS_INVALID_ARG, "null argument");
    if (!(width > 0) || !(coherence > 0)) return fail(WOS_INVALID_ARG, "schell: width and coherence must be > 0");
    if (m <= 0) m = 1;
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long nn = (long long)n * n;
    TRY(ensure(c->vol, sizeof(double2) * (size_t)nn * m));
    double2* modes = reinterpret_cast<double2*>(c->vol.p);
    TRY(schell_generate(c, n, dx, width, coherence, m, noise, false, modes));
    CK(cudaMemcpyAsync(modes_out, modes, sizeof(double2) * (size_t)nn * m, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

int wos_partially_coherent(wos_ctx c, int n, double dx, double width, double coherence, int m,
                           const wos_c128* noise, double z, int method, const wos_context* cci, double* out,
                           wos_diag* diag) {
    if (!c || !noise || !out || n < 2 || !(dx > 0)) return fail(WOS_INVALID_ARG, "null argument");
    if (!(width > 0) || !(coherence > 0)) return fail(WOS_INVALID_ARG, "schell: width and coherence must be > 0");
    if (method < WOS_ASM || method > WOS_FRAUNHOFER) return fail(WOS_UNKNOWN_METHOD, "unknown propagation method");
    if (m <= 0) m = 1;
    if (diag) {
        std::memset(diag, 0, sizeof(*diag));
        diag->dx_out = dx;
    }
    const wos_context cc = cci ? *cci : default_context();
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long nn = (long long)n * n;
    TRY(ensure(c->vol, sizeof(double2) * (size_t)nn * m));
    double2* modes = reinterpret_cast<double2*>(c->vol.p);
    TRY(ensure(c->accum, sizeof(double) * nn));
    double* acc = reinterpret_cast<double*>(c->accum.p);
    CK(cudaMemsetAsync(acc, 0, sizeof(double) * nn, c->st));
    const double inv = 1 / (double)m;
    wos_diag* dp = (cc.diagnostics && diag) ? diag : nullptr;
    if (z != 0 && method == WOS_ASM && !dp && schell_fast_size(n) && !c->no_fast) {
        // the realizations synthesised inside the propagation sweeps
        CK(cudaMemcpyAsync(modes, noise, sizeof(double2) * (size_t)nn * m, cudaMemcpyHostToDevice, c->st));
        const int rc = schell_fused(c, n, dx, width, coherence, m, m, modes, z, cc, acc);
        if (rc != -1) {
            TRY(rc);
            CK(cudaMemcpyAsync(out, acc, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            return WOS_OK;
        }
    }
    TRY(schell_generate(c, n, dx, width, coherence, m, noise, false, modes));
    if (z == 0) {
        for (int q = 0; q < m; q++) CK(launch_accum_int(1, acc, modes + q * nn, 1, nn, inv, c->st));
    } else if (method == WOS_ASM) {
        std::vector<double> w(m, inv);
        double *w_d, *u1, *u2;
        TRY(upload_params(c, w, {}, {}, &w_d, &u1, &u2));
        Batch b{n, n, 1, dx, modes, nn, m, nullptr, nullptr, {}, std::vector<double>(m, z), w_d, acc, nullptr, cc, dp};
        TRY(run_batch_asm(c, b));
    } else {
        TRY(ensure(c->scratch3, (size_t)nn * c->csz()));
        void* O = c->scratch3.p;
        for (int q = 0; q < m; q++) {
            wos_diag ds;
            Prop p{n, n, dx, 1, modes + q * nn, 1, O, 0, z, method, cc, dp ? &ds : nullptr};
            TRY(run_propagate(c, p));
            if (dp) diag_merge(dp, ds);
            CK(launch_accum_int(c->fp64, acc, O, 1, nn, inv, c->st));
        }
    }
    CK(cudaMemcpyAsync(out, acc, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

// ---- device-resident batches
int wos_polychromatic_dev(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* field, double z,
                          const double* wavelengths, const double* weights, int nsamples, const wos_context* base,
                          double* out) {
    if (!c || !field || !out || !wavelengths || !weights) return fail(WOS_INVALID_ARG, "null argument");
    TRY(check_dev_geometry(ny, nx, dx, ncomp));
    if (nsamples <= 0) return fail(WOS_INVALID_ARG, "polychromatic: no wavelength samples");
    for (int s = 0; s < nsamples; s++)
        if (!(wavelengths[s] > 0)) return fail(WOS_INVALID_ARG, "polychromatic: wavelength must be > 0");
    wos_context cc = base ? *base : default_context();
    cc.diagnostics = 0;
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long np = (long long)ny * nx;
    CK(cudaMemsetAsync(out, 0, sizeof(double) * np, c->st));
    if (z == 0) {  // every sample's Propagate returns at once (optics/propagate.go:66-68)
        for (int s = 0; s < nsamples; s++) CK(launch_accum_int(c->fp64, out, field, ncomp, np, weights[s], c->st));
        return WOS_OK;
    }
    std::vector<double> wl(wavelengths, wavelengths + nsamples), w(weights, weights + nsamples);
    const double *wl_d, *w_d;
    TRY(cached_params(c, wl, &wl_d));
    TRY(cached_params(c, w, &w_d));
    Batch b{ny, nx, ncomp, dx, field, 0, nsamples, wl_d, nullptr, wl, std::vector<double>(nsamples, z), w_d, out,
            nullptr, cc, nullptr};
    b.in_native = 1;
    return run_batch_asm(c, b);
}

int wos_volume_dev(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* field, const double* zs, int nz,
                   const wos_context* cci, void* out) {
    if (!c || !field || nz < 0 || (nz > 0 && (!zs || !out))) return fail(WOS_INVALID_ARG, "null argument");
    TRY(check_dev_geometry(ny, nx, dx, ncomp));
    if (nz == 0) return WOS_OK;
    wos_context cc = cci ? *cci : default_context();
    cc.diagnostics = 0;
    if (!(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const size_t plane = (size_t)ny * nx * ncomp * c->csz();
    char* O = reinterpret_cast<char*>(out);
    std::vector<double> zb;
    std::vector<int> idx;
    bool batched = true;
    for (int q = 0; q < nz; q++)
        if (zs[q] != 0) {
            zb.push_back(zs[q]);
            idx.push_back(q);
            if (zs[q] < 0) batched = false;
        }
    if (!zb.empty() && batched) {
        // all planes straight into out, or compactly then moved to their slots
        const bool compact = (int)zb.size() != nz;
        char* dst = O;
        if (compact) {
            TRY(ensure(c->scratch3, plane * zb.size()));
            dst = reinterpret_cast<char*>(c->scratch3.p);
        }
        const double* z_d;
        TRY(cached_params(c, zb, &z_d));
        Batch b{ny, nx, ncomp, dx, field, 0, (int)zb.size(), nullptr, z_d, {}, zb, nullptr, nullptr, dst, cc, nullptr};
        b.in_native = 1;
        b.out_native = 1;
        TRY(run_batch_asm(c, b));
        if (compact)
            for (size_t u = 0; u < zb.size(); u++)
                CK(cudaMemcpyAsync(O + (size_t)idx[u] * plane, dst + u * plane, plane, cudaMemcpyDeviceToDevice, c->st));
    } else {
        for (size_t u = 0; u < zb.size(); u++) {
            Prop p{ny, nx, dx, ncomp, field, 0, O + (size_t)idx[u] * plane, 0, zb[u], WOS_ASM, cc, nullptr};
            TRY(run_propagate(c, p));
        }
    }
    // z == 0 returns the input unchanged (optics/propagate.go:66-68)
    for (int q = 0; q < nz; q++)
        if (zs[q] == 0) CK(cudaMemcpyAsync(O + (size_t)q * plane, field, plane, cudaMemcpyDeviceToDevice, c->st));
    return WOS_OK;
}

int wos_partially_coherent_dev(wos_ctx c, int n, double dx, double width, double coherence, int m, const void* noise,
                               double z, const wos_context* cci, double* out) {
    if (m <= 0) m = 1;
    return schell_dev_range(c, n, dx, width, coherence, m, 0, m, noise, z, cci, out);
}

}  // extern "C"

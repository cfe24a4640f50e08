// wos_bpm.cu -- split-step BPM (PropagateSplitStep, optics/medium.go:22-65)
// on the specialised and the general sweeps, its adjoint, and the
// diffractive stack of phase masks with BPM segments (loss and gradient).
#include "wos_api_internal.cuh"

namespace wapi {

struct ScreenSrc {
    int kind = 1;  // 1 parametric, 2 maps
    wos_index_desc desc{};
    const double* nre = nullptr;
    const double* nim = nullptr;
    int nmaps = 1;
};

void fill_screen(ScreenArgs& s, const ScreenSrc& src, int slice, long long np, double k, double dz, double zc) {
    s = ScreenArgs{};
    s.kind = src.kind;
    s.k = k;
    s.dz = dz;
    s.zc = zc;
    if (src.kind == 1) {
        const wos_index_desc& d = src.desc;
        s.re_bg = d.re_bg;
        s.im_bg = d.im_bg;
        s.core_dn = d.core_dn;
        s.core_x0 = d.core_x0;
        s.core_y0 = d.core_y0;
        s.core_w = d.core_w;
        s.zmod_amp = d.zmod_amp;
        s.zmod_period = d.zmod_period;
        s.zmod_phase = d.zmod_phase;
        s.border_px = d.border_px;
        s.border_order = d.border_order;
        s.border_strength = d.border_strength;
        s.n_layers = d.n_layers < 0 ? 0 : (d.n_layers > 8 ? 8 : d.n_layers);
        for (int i = 0; i < 8; i++) {
            s.layer_z[i] = d.layer_z[i];
            s.layer_re[i] = d.layer_re[i];
            s.layer_im[i] = d.layer_im[i];
        }
    } else {
        const int m = src.nmaps == 1 ? 0 : slice;
        s.nre = src.nre + (long long)m * np;
        s.nim = src.nim + (long long)m * np;
    }
}

// PropagateSplitStep (optics/medium.go:22-45) with merged half steps:
//   rows fwd | cols H(dz/2) | rows inv.M0.fwd | cols H(dz/2)^2 | ... | rows inv.M(S-1).fwd
//   | cols H(dz/2) | rows inv
// The power around every ASM half step (for the evanescent_filtered /
// backward_* warnings of each Propagate(dz/2) call) comes from Parseval sums in
// the column pass, one finished record per pass.
// Split-step BPM on the specialised sweeps: A(dz/2) M A(dz) M ... A(dz/2) with
// the column sweeps of the fused ASM (the merged half steps A(dz/2)^2 are one
// step A(dz): forward steps without an evanescent limit only) and the slice
// screens inside the row sweeps (k_rows_bpm_fast).  The screen of a
// parametric medium factorises as c_s * border(d) * exp(i p_s gx(x) gy(y)):
// the slice constants c_s = exp(-k dz Im n0) exp(i k dz (Re n0 - 1)) are
// multiplied in FP64 on the host and applied once in the last sweep.
// adjoint: the adjoint operator (conj transfer functions and screens, slices
// in reverse order).  Returns -1 when the case is not eligible (the general
// path then runs).
int try_fast_splitstep(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* in, int in_c128, void* out,
                       int out_c128, double z, const ScreenSrc& src, int steps, const wos_context& cc, bool diag,
                       bool adjoint) {
    if (diag || c->no_fast || src.kind != 1 || !is_pow2(nx) || !is_pow2(ny) || !(z > 0)) return -1;
    const double dz = z / (double)steps, hz = dz / 2;
    const double k = 2 * M_PI / cc.wavelength;
    const Policy pol = ev_policy(cc, hz);
    if (pol.limit > 0 || pol.reg) return -1;
    if (!c->fp64 && !(std::fabs(k * dz / (2 * M_PI)) < 268435456.0)) return -1;
    const Tune t = get_tune(c, ny, nx);
    if (!fast_supported(c->fp64, nx, t.rowE) || !fast_supported(c->fp64, ny, t.colE)) return -1;
    const wos_index_desc& d = src.desc;
    Axis *ax, *ay;
    TRY(get_axis(c, nx, c->fp64, &ax));
    TRY(get_axis(c, ny, c->fp64, &ay));
    // complex64: the slice sweeps run the compensated transforms (hi + lo
    // twiddles), whose error does not add up over the slices; their column
    // sweep holds 8 values per thread (16 with the residual twiddles spill)
    const bool comp = !c->fp64 && c->bpm_comp;
    const int colE = (comp && t.colE == 16 && fast_supported(0, ny, 8)) ? 8 : t.colE;
    const void *twx, *twy;
    TRY(fast_tw(c, ax, t.rowE, &twx));
    TRY(fast_tw(c, ay, colE, &twy));
    const void *twx_lo = nullptr, *twy_lo = nullptr;
    if (comp) {
        TRY(fast_tw_lo(c, ax, t.rowE, &twx_lo));
        TRY(fast_tw_lo(c, ay, colE, &twy_lo));
    }
    const long long np = (long long)ny * nx;
    void* S;
    if (!out_c128) {
        S = out;
    } else {
        TRY(ensure(c->scratch, (size_t)np * ncomp * c->csz()));
        S = c->scratch.p;
    }
    // per-run tables: gx of the graded core and the border absorption
    const bool core = d.core_dn != 0;
    const int bpx = (d.border_px > 0 && d.border_strength != 0) ? d.border_px : 0;
    std::vector<double> tab((size_t)nx + (size_t)bpx);
    for (int i = 0; i < nx; i++) {
        const double x = ((double)i - (double)nx / 2) * dx - d.core_x0;
        tab[i] = core ? std::exp(-(x * x) / (d.core_w * d.core_w)) : 0.0;
    }
    for (int q = 0; q < bpx; q++) {
        double p = 1;
        const double tq = (double)(bpx - q) / (double)bpx;
        for (int o = 0; o < d.border_order; o++) p *= tq;
        tab[(size_t)nx + q] = std::exp(-k * d.border_strength * p * dz);
    }
    // uploaded only when they change: a repeated call issues no host copy
    // (and can then be captured in a CUDA graph)
    if (tab != c->bpm_tab_host || !c->bpm_tab.p) {
        TRY(ensure(c->bpm_tab, sizeof(double) * (tab.size() + 1)));
        // (a copy from pageable memory returns once the source has been read)
        CK(cudaMemcpyAsync(c->bpm_tab.p, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, c->st));
        c->bpm_tab_host = tab;
    }
    const double* gx = reinterpret_cast<const double*>(c->bpm_tab.p);
    int nb = 0;
    FastRows r{};
    r.rows = ny;
    r.in = in;
    r.in_c128 = in_c128;
    r.in_ld = nx;
    r.in_bstride = np;
    r.out = S;
    r.out_ld = nx;
    r.out_bstride = np;
    r.tw = twx;
    r.out_scale = 1.0;
    r.batch = ncomp;
    CK(timed_launch(c, 0, [&] { return fast_rows(c->fp64, nx, t.rowE, false, r, c->st, &nb); }));
    FastCols kc{};
    kc.ncols = nx;
    // complex64 with H from the table in registers, on a field that stays in
    // L2 from slice to slice: 4 columns a CTA (cfg3, 1024^2 x 400 slices:
    // 10.64 ms with the table rows in shared memory at 8 columns, 10.87 ms in
    // registers at 8, 10.24 ms in registers at 4).  Larger fields keep the
    // tuned width, whose wider row segments the DRAM traffic needs.
    const bool l2_field = (size_t)np * ncomp * c->csz() <= ((size_t)16 << 20);
    kc.W = (!c->fp64 && c->htab_reg && c->htab_on && l2_field) ? 4 : t.colW;
    kc.data = S;
    kc.ld = nx;
    kc.bstride = np;
    kc.tw = twy;
    kc.batch = ncomp;
    kc.wl = cc.wavelength;
    kc.dx = dx;
    kc.scale = 1.0 / ((double)nx * (double)ny);
    kc.zero_ev = pol.zero;
    kc.precise_phase = 1;
    kc.conj = adjoint;
    kc.tw_lo = twy_lo;
    const double sgn = adjoint ? -1.0 : 1.0;
    FastRows m = r;
    m.in = S;
    m.in_c128 = 0;
    m.bpm_gx = core ? gx : nullptr;
    m.bpm_y0 = d.core_y0;
    m.bpm_w2 = d.core_w * d.core_w;
    m.bpm_dx = dx;
    m.bpm_border = bpx ? gx + nx : nullptr;
    m.bpm_border_px = bpx;
    m.bpm_nx = nx;
    m.tw_lo = twx_lo;
    // Product of the slice constants c_s, each formed as applyMediumPhase forms
    // the screen of a background pixel (t = exp(-k Im n dz) cexpI(k (Re n - 1)
    // dz), optics/medium.go:58-59) and multiplied in FP64 complex arithmetic:
    // the rounding of every factor is then the reference's own.  (Summing the
    // slice phases instead lets the rounding of a running sum near 10^3 rad
    // reach ~1e-11 over 400 slices.)
    double c_re = 1.0, c_im = 0.0;
    for (int s = 0; s <= steps; s++) {
        const double zp = (s == 0 || s == steps) ? hz : dz;
        kc.kz = k * zp;
        kc.kaz = k * zp;
        kc.krev = kc.kz / (2 * M_PI);
        kc.htab = nullptr;
        TRY(attach_htab(c, kc, ny, colE));  // one table for dz, one for the half steps
        CK(timed_launch(c, 4, [&] { return sweep_cols(c, ny, colE, kc, &nb); }));
        if (s < steps) {
            const int sl = adjoint ? steps - 1 - s : s;
            const double zc = z * (double)sl / (double)steps + dz / 2;
            double r0 = d.re_bg, i0 = d.im_bg;
            for (int q = 0; q < d.n_layers && q < 8; q++)
                if (zc < d.layer_z[q]) {
                    r0 = d.layer_re[q];
                    i0 = d.layer_im[q];
                    break;
                }
            double mod = 1;
            if (d.zmod_amp != 0) mod = 1.0 + d.zmod_amp * std::sin(2 * M_PI * zc / d.zmod_period + d.zmod_phase);
            m.bpm_phase = sgn * (k * d.core_dn * mod * dz);
            const double ph = k * (r0 - 1.0) * dz;
            const double am = std::exp(-k * i0 * dz);
            const double tr = am * std::cos(ph), ti = sgn * (am * std::sin(ph));
            const double nr = c_re * tr - c_im * ti, ni = c_re * ti + c_im * tr;
            c_re = nr;
            c_im = ni;
            CK(timed_launch(c, 0, [&] { return fast_rows_bpm(c->fp64, nx, t.rowE, m, c->st, &nb); }));
        }
    }
    FastRows q = r;
    q.in = S;
    q.in_c128 = 0;
    q.out = out;
    q.out_c128 = out_c128;
    q.out_scale = c_re;
    q.out_scale_im = c_im;
    CK(timed_launch(c, 1, [&] { return fast_rows(c->fp64, nx, t.rowE, true, q, c->st, &nb); }));
    return WOS_OK;
}

int run_splitstep(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* in, int in_c128, void* out,
                  int out_c128, double z, const ScreenSrc& src, int steps, const wos_context& cc, wos_diag* d,
                  bool adjoint = false) {
    if (d) {
        std::memset(d, 0, sizeof(*d));
        d->dx_out = dx;
    }
    if (ny < 2 || nx < 2 || ncomp < 1 || ncomp > 2 || !(dx > 0) || !in || !out)
        return fail(WOS_INVALID_ARG, "invalid field geometry");
    if (z == 0) {
        Prop p{ny, nx, dx, ncomp, in, in_c128, out, out_c128, 0.0, WOS_ASM, cc, nullptr};
        return copy_field(c, p);
    }
    if (!(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    if (steps <= 0) steps = 1;
    {
        const int rc = try_fast_splitstep(c, ny, nx, dx, ncomp, in, in_c128, out, out_c128, z, src, steps, cc,
                                          d != nullptr, adjoint);
        if (rc != -1) return rc;
    }
    const double dz = z / (double)steps;
    const double k = 2 * M_PI / cc.wavelength;
    const double hz = dz / 2;
    const Policy pol = ev_policy(cc, hz);
    Axis *ax, *ay;
    TRY(get_axis(c, nx, c->fp64, &ax));
    TRY(get_axis(c, ny, c->fp64, &ay));
    const long long np = (long long)ny * nx;
    void* S;
    if (!out_c128) {
        S = out;
    } else {
        TRY(ensure(c->scratch, (size_t)np * ncomp * c->csz()));
        S = c->scratch.p;
    }
    const int W = auto_colw(c, ay->L);
    const size_t nbr = row_blocks(c->fp64, ax->L, ny, ncomp);
    const size_t nbc = col_blocks(c->fp64, ay->L, W, nx, ncomp);
    TRY(red_prepare(c, std::max(nbr, nbc)));
    const bool diag = d != nullptr;
    const bool wrap = wrap_needed(cc, ny, nx, dx, hz);
    const int npass = steps + 1;
    if (diag) TRY(ensure(c->tmp, sizeof(double) * RS_COUNT * (size_t)npass));
    double* passes = reinterpret_cast<double*>(c->tmp.p);

    RowArgs r = row_defaults(ny, nx, dx);
    r.mode = ROW_FWD;
    r.rows = ny;
    fill_axis(r, ax);
    r.in = in;
    r.in_c128 = in_c128;
    r.in_ld = nx;
    r.in_bstride = np;
    r.in_n = nx;
    r.out = S;
    r.out_ld = nx;
    r.out_bstride = np;
    r.out_n = nx;
    r.batch = ncomp;
    if (diag) {
        r.red = red_region(c, 0);
        r.red_pre = 1;
    }
    CK(prof_rows(c, c->fp64, r));
    if (diag) CK(launch_reduce_finish(r.red, (int)nbr, 1, RS_P, 1, redout_region(c, 0), c->st));

    for (int s = 0; s <= steps; s++) {
        ColArgs a = col_defaults(c, dx);
        a.mode = COL_FUSED;
        a.ncols = nx;
        fill_axis(a, ay);
        a.W = W;
        a.src = S;
        a.src_ld = nx;
        a.src_bstride = np;
        a.in_n = ny;
        a.dst = S;
        a.dst_ld = nx;
        a.dst_bstride = np;
        a.out_n = ny;
        a.h = asm_h(c, cc, hz, pol, dx, nx, ny);
        a.h.kind = (s == 0 || s == steps) ? H_ASM : H_ASM_HALF2;
        a.h.conj = adjoint;
        a.batch = ncomp;
        if (diag) {
            a.red = red_region(c, 1);
            a.red_bpm = 1;
            if (wrap) {
                a.red_hist = 1;
                a.hist_lx = nx;
                a.hist_ly = ny;
                a.hist_dx = dx;
            }
        }
        CK(prof_cols(c, c->fp64, a));
        if (diag) {
            CK(launch_reduce_finish(a.red, (int)nbc, 1, RS_SW, 3, passes + (size_t)s * RS_COUNT, c->st));
            if (wrap) CK(launch_reduce_finish(a.red, (int)nbc, 1, RS_HIST, 97, passes + (size_t)s * RS_COUNT, c->st));
        }
        if (s < steps) {
            RowArgs q = row_defaults(ny, nx, dx);
            q.mode = ROW_INV_FWD;
            q.rows = ny;
            fill_axis(q, ax);
            q.in = S;
            q.in_ld = nx;
            q.in_bstride = np;
            q.in_n = nx;
            q.out = S;
            q.out_ld = nx;
            q.out_bstride = np;
            q.out_n = nx;
            q.batch = ncomp;
            const int sl = adjoint ? steps - 1 - s : s;
            const double zc = z * (double)sl / (double)steps + dz / 2;
            fill_screen(q.scr, src, sl, np, k, dz, zc);
            q.scr.conj = adjoint;
            CK(prof_rows(c, c->fp64, q));
        }
    }
    RowArgs q = row_defaults(ny, nx, dx);
    q.mode = ROW_INV;
    q.rows = ny;
    fill_axis(q, ax);
    q.in = S;
    q.in_ld = nx;
    q.in_bstride = np;
    q.in_n = nx;
    q.out = out;
    q.out_c128 = out_c128;
    q.out_ld = nx;
    q.out_bstride = np;
    q.out_n = nx;
    q.batch = ncomp;
    if (diag) {
        q.red = red_region(c, 2);
        q.red_post = 1;
    }
    CK(prof_rows(c, c->fp64, q));
    if (diag) {
        CK(launch_reduce_finish(q.red, (int)nbr, 1, RS_P, 1, redout_region(c, 2), c->st));
        TRY(fetch_red(c, 3));
        d->p_in = c->hred[RS_P] * dx * dx;
        d->p_out = c->hred[2 * RS_COUNT + RS_P] * dx * dx;
        std::vector<double> h((size_t)npass * RS_COUNT);
        CK(cudaMemcpy(h.data(), passes, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
        for (int s = 0; s <= steps; s++) {
            const double* rr = h.data() + (size_t)s * RS_COUNT;
            const double p0 = rr[RS_SW], l1 = rr[RS_SW + 1], l2 = rr[RS_SW + 2];
            // half step(s) of this pass: P0 -> P0-L1 and, for merged passes, P0-L1 -> P0-L1-L2
            const int nh = (s == 0 || s == steps) ? 1 : 2;
            for (int hh = 0; hh < nh; hh++) {
                if (wrap) wrap_finish(d, cc, ny, nx, dx, hz, rr + RS_HIST);
                if (hh == 0) asm_warn(d, hz, p0, p0 - l1, pol);
                else asm_warn(d, hz, p0 - l1, (p0 - l1) - l2, pol);
            }
        }
    }
    return WOS_OK;
}

// Diffractive stack (no reference counterpart): u = a; for each layer l,
// v_l = u exp(i phi_l) and u = BPM_zseg(v_l); L = sum (|u|^2 - T)^2.  The
// gradient runs the adjoint chain b = BPM^H(r) from r = dL/du* = 4 (|u|^2 - T) u:
// dL/dphi_l = Re(conj(b_l) i v_l), then b <- exp(-i phi_l) b.  The BPM is
// linear in the field, so its adjoint needs no forward state inside a
// segment: the only stored states are the nl fields v_l at the masks.
// a: complex128 when a_c128, else the context's type; phis [nl][ny][nx],
// target, grads: FP64 device arrays (grads null: loss only).
int bpm_stack_impl(wos_ctx c, int ny, int nx, double dx, int nl, const void* a, int a_c128, const double* phis,
                   const double* T, double zseg, int steps, const wos_index_desc& medium, const wos_context& cc,
                   double* loss, double* grads) {
    if (nl < 1 || steps < 1 || ny < 2 || nx < 2 || !(dx > 0) || !a || !phis || !T || !loss)
        return fail(WOS_INVALID_ARG, "bpm stack arguments");
    if (!(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    const long long np = (long long)ny * nx;
    const size_t fb = (size_t)np * c->csz();
    TRY(ensure(c->scratch2, fb));
    TRY(ensure(c->vol, fb * (size_t)nl));
    TRY(red_prepare(c, (size_t)((np + 255) / 256)));
    void* U = c->scratch2.p;
    char* V = reinterpret_cast<char*>(c->vol.p);
    if (a_c128 && !c->fp64) CK(launch_convert(0, a, U, np, c->st));
    else CK(cudaMemcpyAsync(U, a, fb, cudaMemcpyDeviceToDevice, c->st));
    ScreenSrc src;
    src.kind = 1;
    src.desc = medium;
    // (The slices run the compensated complex64 sweeps: with the plain ones
    // the FP32 loss of 2048^2 x 3 masks x 200 slices is 5.3e-4 from the FP64
    // pipeline instead of 6.2e-5, at 69 ms instead of 98 ms.)
    for (int l = 0; l < nl; l++) {
        CK(launch_mask_phase(c->fp64, U, phis + (size_t)l * np, np, 0, c->st));
        CK(cudaMemcpyAsync(V + (size_t)l * fb, U, fb, cudaMemcpyDeviceToDevice, c->st));
        TRY(run_splitstep(c, ny, nx, dx, 1, U, 0, U, 0, zseg, src, steps, cc, nullptr, false));
    }
    int nb = 0;
    CK(launch_residual(c->fp64, U, T, U, np, red_region(c, 0), &nb, c->st));
    CK(launch_reduce_finish(red_region(c, 0), nb, 1, RS_P, 1, redout_region(c, 0), c->st));
    if (grads) {
        for (int l = nl - 1; l >= 0; l--) {
            TRY(run_splitstep(c, ny, nx, dx, 1, U, 0, U, 0, zseg, src, steps, cc, nullptr, true));
            CK(launch_grad_v(c->fp64, U, V + (size_t)l * fb, grads + (size_t)l * np, np, c->st));
            if (l > 0) CK(launch_mask_phase(c->fp64, U, phis + (size_t)l * np, np, 1, c->st));
        }
    }
    CK(cudaMemcpyAsync(c->err_host, c->err_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
    TRY(fetch_red(c, 1));
    *loss = c->hred[RS_P];
    return check_err_word(c);
}

}  // namespace wapi

extern "C" {

int wos_splitstep(wos_ctx c, wos_field* f, double z, const wos_index_desc* n, int steps, const wos_context* cc,
                  wos_diag* diag) {
    if (!c || !n) return fail(WOS_INVALID_ARG, "null argument");
    TRY(check_field(f));
    if (diag) {
        std::memset(diag, 0, sizeof(*diag));
        diag->dx_out = f->dx;
    }
    if (z == 0) return WOS_OK;
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int ncomp = f->polarized ? 2 : 1;
    TRY(stage_in(c, f, ncomp));
    ScreenSrc src;
    src.kind = 1;
    src.desc = *n;
    const wos_context ctx = cc ? *cc : default_context();
    TRY(run_splitstep(c, f->ny, f->nx, f->dx, ncomp, c->stage.p, 1, c->stage.p, 1, z, src, steps, ctx,
                      ctx.diagnostics ? diag : nullptr));
    return stage_out(c, f, ncomp);
}

int wos_splitstep_dev(wos_ctx c, int ny, int nx, double dx, int ncomp, void* field, double z,
                      const wos_index_desc* n, int steps, const wos_context* cc, wos_diag* diag) {
    if (!c || !n) return fail(WOS_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    ScreenSrc src;
    src.kind = 1;
    src.desc = *n;
    const wos_context ctx = cc ? *cc : default_context();
    if (diag && !ctx.diagnostics) {
        std::memset(diag, 0, sizeof(*diag));
        diag->dx_out = dx;
        diag = nullptr;
    }
    return run_splitstep(c, ny, nx, dx, ncomp, field, 0, field, 0, z, src, steps, ctx, diag);
}

int wos_splitstep_maps(wos_ctx c, wos_field* f, double z, const double* n_re, const double* n_im, int nmaps,
                       int steps, const wos_context* cc, wos_diag* diag) {
    if (!c || !n_re || !n_im) return fail(WOS_INVALID_ARG, "null argument");
    TRY(check_field(f));
    if (diag) {
        std::memset(diag, 0, sizeof(*diag));
        diag->dx_out = f->dx;
    }
    if (z == 0) return WOS_OK;
    const int st = steps <= 0 ? 1 : steps;
    if (nmaps != 1 && nmaps != st) return fail(WOS_INVALID_ARG, "nmaps must be 1 or steps");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long np = (long long)f->ny * f->nx;
    TRY(ensure(c->maps, sizeof(double) * 2 * np * nmaps));
    double* re = reinterpret_cast<double*>(c->maps.p);
    double* im = re + np * nmaps;
    CK(cudaMemcpyAsync(re, n_re, sizeof(double) * np * nmaps, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(im, n_im, sizeof(double) * np * nmaps, cudaMemcpyHostToDevice, c->st));
    const int ncomp = f->polarized ? 2 : 1;
    TRY(stage_in(c, f, ncomp));
    ScreenSrc src;
    src.kind = 2;
    src.nre = re;
    src.nim = im;
    src.nmaps = nmaps;
    const wos_context ctx = cc ? *cc : default_context();
    TRY(run_splitstep(c, f->ny, f->nx, f->dx, ncomp, c->stage.p, 1, c->stage.p, 1, z, src, st, ctx,
                      ctx.diagnostics ? diag : nullptr));
    return stage_out(c, f, ncomp);
}

int wos_splitstep_adjoint(wos_ctx c, wos_field* f, double z, const wos_index_desc* n, int steps,
                          const wos_context* cc) {
    if (!c || !n || !cc) return fail(WOS_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    ScreenSrc src;
    src.kind = 1;
    src.desc = *n;
    const int ncomp = f->polarized ? 2 : 1;
    TRY(run_splitstep(c, f->ny, f->nx, f->dx, ncomp, c->stage.p, 1, c->stage.p, 1, z, src, steps, *cc, nullptr,
                      true));
    return stage_out(c, f, ncomp);
}

int wos_splitstep_adjoint_dev(wos_ctx c, int ny, int nx, double dx, int ncomp, void* field, double z,
                              const wos_index_desc* n, int steps, const wos_context* cc) {
    if (!c || !n || !cc) return fail(WOS_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    ScreenSrc src;
    src.kind = 1;
    src.desc = *n;
    return run_splitstep(c, ny, nx, dx, ncomp, field, 0, field, 0, z, src, steps, *cc, nullptr, true);
}

int wos_bpm_stack_loss_grad_dev(wos_ctx c, int ny, int nx, double dx, int nlayers, const void* a, const double* phis,
                                const double* target, double zseg, const wos_index_desc* n, int steps,
                                const wos_context* cc, double* loss, double* grads) {
    if (!c || !n || !cc) return fail(WOS_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    return bpm_stack_impl(c, ny, nx, dx, nlayers, a, 0, phis, target, zseg, steps, *n, *cc, loss, grads);
}

int wos_bpm_stack_loss_grad(wos_ctx c, int ny, int nx, double dx, int nlayers, const wos_c128* a, const double* phis,
                            const double* target, double zseg, const wos_index_desc* n, int steps,
                            const wos_context* cc, double* loss, double* grads) {
    if (!c || !n || !cc || !a || !phis || !target || nlayers < 1 || ny < 2 || nx < 2)
        return fail(WOS_INVALID_ARG, "bpm stack arguments");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long np = (long long)ny * nx;
    TRY(ensure(c->stage, (size_t)np * 16));
    TRY(ensure(c->maps, sizeof(double) * (size_t)np * (2 * (size_t)nlayers + 1)));
    double* phid = reinterpret_cast<double*>(c->maps.p);
    double* Td = phid + (size_t)np * nlayers;
    double* gd = Td + np;
    CK(cudaMemcpyAsync(c->stage.p, a, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(phid, phis, sizeof(double) * (size_t)np * nlayers, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(Td, target, sizeof(double) * (size_t)np, cudaMemcpyHostToDevice, c->st));
    TRY(bpm_stack_impl(c, ny, nx, dx, nlayers, c->stage.p, 1, phid, Td, zseg, steps, *n, *cc, loss,
                       grads ? gd : nullptr));
    if (grads) {
        CK(cudaMemcpyAsync(grads, gd, sizeof(double) * (size_t)np * nlayers, cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    return WOS_OK;
}

}  // extern "C"

// wos_field_ops.cu -- thin elements (optics/elements.go), field operations
// (optics/field.go:109-294), anisotropic media (optics/birefringent.go,
// optics/berreman.go), Propagate1D, vectorial ASM, plane views in the server's
// binary format and the device-resident element train.
#include "wos_api_internal.cuh"

namespace wapi {

int element_begin(wos_ctx c, wos_field* f) {
    TRY(check_field(f));
    TRY(set_device(c));
    return stage_in(c, f, f->polarized ? 2 : 1);
}

double2* stage_ex(wos_ctx c) { return reinterpret_cast<double2*>(c->stage.p); }

double2* stage_ey(wos_ctx c, const wos_field* f) { return stage_ex(c) + (size_t)f->ny * f->nx; }

double2 d2(wos_c128 v) { return make_double2(v.re, v.im); }

// FFT -> multiply by a filter H(fx, fy) -> inverse FFT of `ncomp` complex128
// device planes in place, on the three-sweep propagator (context precision).
int spectral_filter(wos_ctx c, int ny, int nx, double dx, int ncomp, void* planes, int kind, double p0,
                    double p1, double k = 0, double z = 0) {
    Prop p{ny, nx, dx, ncomp, planes, 1, planes, 1, 0.0, 0, default_context(), nullptr};
    Sweep3 s;
    s.h.kind = kind;
    s.h.exact = c->fp64;
    s.h.dx = dx;
    s.h.lfx = nx;
    s.h.lfy = ny;
    s.h.scale = 1.0 / ((double)nx * (double)ny);
    s.h.c_re = 1.0;
    s.h.p0 = p0;
    s.h.p1 = p1;
    s.h.k = k;
    s.h.z = z;
    return run_sweep3(c, p, s);
}

}  // namespace wapi

extern "C" {

int wos_apply_lens(wos_ctx c, wos_field* f, double wavelength, double focal, double aperture, double x0, double y0) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    if (focal == 0) return fail(WOS_INVALID_ARG, "lens: focal length f must be non-zero");
    if (!(wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    const double k = 2 * M_PI / wavelength;
    const double cc = -k / (2 * focal);
    CK(launch_lens(stage_ex(c), stage_ey(c, f), f->polarized, f->ny, f->nx, f->dx, cc, aperture, x0, y0, c->st));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_apply_aperture_circle(wos_ctx c, wos_field* f, double radius, double x0, double y0, double edge_sigma) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    CK(launch_aperture_circle(stage_ex(c), stage_ey(c, f), f->polarized, f->ny, f->nx, f->dx, radius, x0, y0,
                              edge_sigma, c->st));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_apply_grating(wos_ctx c, wos_field* f, int kind, double period, double modulation, double duty,
                      double blaze_depth, double rotation, double offset) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    if (!(period > 0)) return fail(WOS_INVALID_ARG, "grating: period must be > 0");
    if (duty < 0 || duty > 1) return fail(WOS_INVALID_ARG, "grating: duty must be in [0,1]");
    if (kind < 0 || kind > 4) return fail(WOS_INVALID_ARG, "grating: unknown kind");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    CK(launch_grating(stage_ex(c), stage_ey(c, f), f->polarized, f->ny, f->nx, f->dx, kind, period, modulation, duty,
                      blaze_depth, rotation, offset, c->st));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_apply_phase_mask(wos_ctx c, wos_field* f, const double* phi, double amp) {
    if (!c || !phi) return fail(WOS_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    const long long np = (long long)f->ny * f->nx;
    TRY(ensure(c->maps, sizeof(double) * np));
    CK(cudaMemcpyAsync(c->maps.p, phi, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
    CK(launch_phase_mask(stage_ex(c), stage_ey(c, f), f->polarized, np, reinterpret_cast<double*>(c->maps.p), amp,
                         c->st));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_apply_jones(wos_ctx c, wos_field* f, wos_c128 a, wos_c128 b, wos_c128 cc, wos_c128 d) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    int mode = 2;
    if (f && !f->polarized) {
        const bool diag = b.re == 0 && b.im == 0 && cc.re == 0 && cc.im == 0 && d.re == a.re && d.im == a.im;
        mode = diag ? 0 : 1;
        if (mode == 1 && !f->ey) return fail(WOS_INVALID_ARG, "jones: the field needs an Ey buffer");
    }
    TRY(check_field(f));
    TRY(set_device(c));
    TRY(stage_in(c, f, mode == 0 ? 1 : 2));
    const long long np = (long long)f->ny * f->nx;
    CK(launch_jones(stage_ex(c), stage_ey(c, f), np, mode, d2(a), d2(b), d2(cc), d2(d), c->st));
    if (mode == 1) f->polarized = 1;
    return stage_out(c, f, mode == 0 ? 1 : 2);
}

int wos_scale_amplitude(wos_ctx c, wos_field* f, wos_c128 s) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    CK(launch_scale(stage_ex(c), stage_ey(c, f), f->polarized, (long long)f->ny * f->nx, d2(s), c->st));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_apply_tilt(wos_ctx c, wos_field* f, double tx, double ty, double wavelength) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    if (!(wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    const double k = 2 * M_PI / wavelength;
    CK(launch_tilt(stage_ex(c), stage_ey(c, f), f->polarized, f->ny, f->nx, f->dx, k, std::sin(tx), std::sin(ty),
                   c->st));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_apply_bandlimit(wos_ctx c, wos_field* f, double fraction, double sigma) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(check_field(f));
    if (fraction >= 1 || fraction <= 0) return WOS_OK;  // nil or disabled options (field.go:266-268)
    TRY(element_begin(c, f));
    const double fnyq = 1 / (2 * f->dx);
    const double f0 = fraction * fnyq;
    double sig = sigma * fnyq;
    if (sig <= 0) sig = fnyq * 0.01;
    TRY(spectral_filter(c, f->ny, f->nx, f->dx, f->polarized ? 2 : 1, c->stage.p, H_BANDLIMIT, f0, sig));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_shift_field(wos_ctx c, wos_field* f, double du, double dv) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(check_field(f));
    if (du == 0 && dv == 0) return WOS_OK;
    TRY(element_begin(c, f));
    TRY(spectral_filter(c, f->ny, f->nx, f->dx, f->polarized ? 2 : 1, c->stage.p, H_SHIFT, du, dv));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_propagate_anisotropic(wos_ctx c, wos_field* f, double z, const wos_c128* eps, const wos_context* cci) {
    if (!c || !f || !f->ex || !f->ey || !eps || f->ny < 2 || f->nx < 2 || !(f->dx > 0))
        return fail(WOS_INVALID_ARG, "anisotropic: ex, ey, eps and a valid geometry are required");
    const wos_context cc = cci ? *cci : default_context();
    if (!(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int ny = f->ny, nx = f->nx;
    const long long np = (long long)ny * nx;
    TRY(ensure(c->stage, (size_t)np * 16 * 2));
    double2* st = reinterpret_cast<double2*>(c->stage.p);
    CK(cudaMemcpyAsync(st, f->ex, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(st + np, f->ey, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    void* work = st;
    if (!c->fp64) {
        TRY(ensure(c->scratch, (size_t)np * 8 * 2));
        work = c->scratch.p;
        CK(launch_convert(0, st, work, 2 * np, c->st));
    }
    Eps9 e;
    for (int k = 0; k < 9; k++) e.v[k] = make_double2(eps[k].re, eps[k].im);
    TRY(fft2d_impl(c, c->fp64, ny, nx, 2, work, 0));
    CK(launch_aniso(c->fp64, work, ny, nx, f->dx, 2 * M_PI / cc.wavelength, z, e, c->st));
    TRY(fft2d_impl(c, c->fp64, ny, nx, 2, work, 1));
    if (!c->fp64) CK(launch_convert(1, work, st, 2 * np, c->st));
    CK(cudaMemcpyAsync(f->ex, st, (size_t)np * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(f->ey, st + np, (size_t)np * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

int wos_propagate_uniaxial(wos_ctx c, wos_field* f, double z, double no, double ne, const wos_context* cci) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    if (!(no > 0) || !(ne > 0)) return fail(WOS_INVALID_ARG, "uniaxial: n_o and n_e must be > 0");
    const wos_context cc = cci ? *cci : default_context();
    if (!(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    const double k0 = 2 * M_PI / cc.wavelength;
    TRY(spectral_filter(c, f->ny, f->nx, f->dx, 1, stage_ex(c), H_UNIAX_E, no, ne, k0, z));
    if (f->polarized) TRY(spectral_filter(c, f->ny, f->nx, f->dx, 1, stage_ey(c, f), H_UNIAX_O, no, ne, k0, z));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_apply_diffuser(wos_ctx c, wos_field* f, double sigma, double correlation, double amplitude,
                       long long seed, double x0, double y0) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(element_begin(c, f));
    const long long np = (long long)f->ny * f->nx;
    TRY(ensure(c->aux, (size_t)np * sizeof(double2)));
    double2* zp = reinterpret_cast<double2*>(c->aux.p);
    const double cell = f->dx > 0 ? f->dx : 1.0;
    CK(launch_diffuser_noise(zp, f->ny, f->nx, f->dx, cell, x0, y0, seed, c->st));
    if (correlation > 0) {
        const double neg_two_pi_sq = -19.739208802178716;  // -2 pi^2 rounded once, as a Go constant
        TRY(spectral_filter(c, f->ny, f->nx, f->dx, 1, zp, H_GAUSS, neg_two_pi_sq * correlation * correlation, 0));
    }
    const int nb = sum_re2_blocks(np);
    TRY(red_prepare(c, (size_t)nb));
    CK(launch_sum_re2(zp, np, red_region(c, 0), c->st));
    CK(launch_reduce_finish(red_region(c, 0), nb, 1, 0, 2, redout_region(c, 0), c->st));
    CK(launch_diffuser_apply(stage_ex(c), stage_ey(c, f), f->polarized, np, zp, redout_region(c, 0), sigma,
                             amplitude, c->st));
    return stage_out(c, f, f->polarized ? 2 : 1);
}

int wos_propagate1d(wos_ctx c, int n, wos_c128* a, double dx, double z, double wavelength, const wos_context* cci,
                    wos_diag* d) {
    if (!c || !a) return fail(WOS_INVALID_ARG, "null argument");
    if (n < 2 || !(dx > 0)) return fail(WOS_INVALID_ARG, "propagate1d: n >= 2 and dx > 0 required");
    if (!(wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    if (d) {
        std::memset(d, 0, sizeof(*d));
        d->dx_out = dx;
    }
    wos_context cc = cci ? *cci : default_context();
    cc.wavelength = wavelength;  // Propagate1D takes wl apart from the Context
    const Policy pol = ev_policy(cc, z);
    Axis* ax;
    TRY(get_axis(c, n, c->fp64, &ax));
    TRY(ensure(c->stage, (size_t)n * 16));
    TRY(ensure(c->scratch, (size_t)n * c->csz()));
    CK(cudaMemcpyAsync(c->stage.p, a, (size_t)n * 16, cudaMemcpyHostToDevice, c->st));
    TRY(red_prepare(c, 64));
    RowArgs r = row_defaults(1, n, dx);
    r.mode = ROW_FWD;
    r.rows = 1;
    fill_axis(r, ax);
    r.in = c->stage.p;
    r.in_c128 = 1;
    r.in_ld = n;
    r.in_n = n;
    r.out = c->scratch.p;
    r.out_ld = n;
    r.out_n = n;
    r.red = red_region(c, 0);
    r.red_pre = 1;
    CK(prof_rows(c, c->fp64, r));
    CK(launch_reduce_finish(r.red, 1, 1, RS_P, 1, redout_region(c, 0), c->st));
    HArgs h = asm_h(c, cc, z, pol, dx, n, 1);
    h.scale = 1.0 / (double)n;
    int nb = 0;
    CK(launch_asm1d_h(c->fp64, c->scratch.p, n, h, red_region(c, 1), &nb, c->st));
    CK(launch_reduce_finish(red_region(c, 1), nb, 1, RS_SW, 2, redout_region(c, 1), c->st));
    RowArgs q = r;
    q.mode = ROW_INV;
    q.in = c->scratch.p;
    q.in_c128 = 0;
    q.out = c->stage.p;
    q.out_c128 = 1;
    q.red = nullptr;
    q.red_pre = 0;
    CK(prof_rows(c, c->fp64, q));
    CK(cudaMemcpyAsync(a, c->stage.p, (size_t)n * 16, cudaMemcpyDeviceToHost, c->st));
    TRY(fetch_red(c, 2));
    // sum1DSq before and after (no dx factor); the loss fraction comes from
    // the spectral sums, free of the cancellation of pIn - pOut
    const double pin = c->hred[RS_P];
    const double p0 = c->hred[RS_COUNT + RS_SW], l1 = c->hred[RS_COUNT + RS_SW + 1];
    const double pout = pin - pin * (p0 > 0 ? l1 / p0 : 0.0);
    if (d) {
        d->p_in = pin;
        d->p_out = pout;
        if (pin > 0 && pout < pin * (1 - 1e-8) && z > 0)
            warn_add(d, WOS_W_EVANESCENT_FILTERED, (pin - pout) / pin);
    }
    return WOS_OK;
}

int wos_propagate_vectorial(wos_ctx c, wos_field* f, wos_c128* ez, double z, const wos_context* cci) {
    if (!c || !f || !f->ex || !f->ey || !ez || f->ny < 2 || f->nx < 2 || !(f->dx > 0))
        return fail(WOS_INVALID_ARG, "vectorial: ex, ey and ez buffers and a valid geometry are required");
    if (z == 0) return WOS_OK;  // Propagate returns before the vectorial step (propagate.go:66-68)
    const wos_context cc = cci ? *cci : default_context();
    if (!(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int ny = f->ny, nx = f->nx;
    const long long np = (long long)ny * nx;
    TRY(ensure(c->stage, (size_t)np * 16 * 3));
    double2* st = reinterpret_cast<double2*>(c->stage.p);
    CK(cudaMemcpyAsync(st, f->ex, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(st + np, f->ey, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    void* work = st;
    if (!c->fp64) {
        TRY(ensure(c->scratch, (size_t)np * 8 * 3));
        work = c->scratch.p;
        CK(launch_convert(0, st, work, 2 * np, c->st));
    }
    const Policy pol = ev_policy(cc, z);
    HArgs h = asm_h(c, cc, z, pol, f->dx, nx, ny);
    TRY(fft2d_impl(c, c->fp64, ny, nx, 2, work, 0));
    CK(launch_vectorial(c->fp64, work, ny, nx, f->dx, h, c->st));
    TRY(fft2d_impl(c, c->fp64, ny, nx, 3, work, 1));
    if (!c->fp64) CK(launch_convert(1, work, st, 3 * np, c->st));
    CK(cudaMemcpyAsync(f->ex, st, (size_t)np * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(f->ey, st + np, (size_t)np * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(ez, st + 2 * np, (size_t)np * 16, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

int wos_plane_view(wos_ctx c, const wos_field* f, const wos_c128* ez, int view, double mask_cut, float* out) {
    if (!c || !f || !f->ex || !out || f->ny < 1 || f->nx < 1) return fail(WOS_INVALID_ARG, "plane view arguments");
    if (view < WOS_VIEW_TOTAL || view > WOS_VIEW_PHASE_Z) return fail(WOS_INVALID_ARG, "unknown plane view");
    const bool need_ey = view == WOS_VIEW_EY || view == WOS_VIEW_PHASE_Y || (view <= WOS_VIEW_AMPLITUDE && f->polarized);
    const bool need_ez = view == WOS_VIEW_EZ || view == WOS_VIEW_PHASE_Z;
    if ((need_ey && !f->ey) || (need_ez && !ez)) return fail(WOS_INVALID_ARG, "plane view: component missing");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long np = (long long)f->ny * f->nx;
    const bool use_ez = ez && (need_ez || view <= WOS_VIEW_AMPLITUDE);
    TRY(ensure(c->stage, (size_t)np * 16 * 3));
    double2* st = reinterpret_cast<double2*>(c->stage.p);
    CK(cudaMemcpyAsync(st, f->ex, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    if (need_ey) CK(cudaMemcpyAsync(st + np, f->ey, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    if (use_ez) CK(cudaMemcpyAsync(st + 2 * np, ez, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    TRY(ensure(c->accum, sizeof(float) * np));
    TRY(plane_view_dev(c, 1, st, need_ey ? st + np : nullptr, use_ez ? st + 2 * np : nullptr, f->polarized ? 1 : 0,
                       np, view, mask_cut, c->accum.p));
    CK(cudaMemcpyAsync(out, c->accum.p, sizeof(float) * np, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return WOS_OK;
}

int wos_plane_view_dev(wos_ctx c, int ny, int nx, int ncomp, const void* planes, const void* ez, int view,
                       double mask_cut, void* out) {
    if (!c || !planes || !out || ny < 1 || nx < 1 || ncomp < 1 || ncomp > 2)
        return fail(WOS_INVALID_ARG, "plane view arguments");
    if (view < WOS_VIEW_TOTAL || view > WOS_VIEW_PHASE_Z) return fail(WOS_INVALID_ARG, "unknown plane view");
    if ((view == WOS_VIEW_EY || view == WOS_VIEW_PHASE_Y) && ncomp < 2)
        return fail(WOS_INVALID_ARG, "plane view: component missing");
    if ((view == WOS_VIEW_EZ || view == WOS_VIEW_PHASE_Z) && !ez) return fail(WOS_INVALID_ARG, "plane view: no Ez");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const long long np = (long long)ny * nx;
    const char* p = reinterpret_cast<const char*>(planes);
    return plane_view_dev(c, c->fp64, p, ncomp == 2 ? p + (size_t)np * c->csz() : nullptr, ez, ncomp == 2 ? 1 : 0, np,
                          view, mask_cut, out);
}

int wos_train(wos_ctx c, wos_field* f, const wos_op* ops, int nops, const wos_context* cci, double bl_fraction,
              double bl_sigma, wos_diag* diag) {
    if (!c || (nops > 0 && !ops) || nops < 0) return fail(WOS_INVALID_ARG, "train arguments");
    TRY(check_field(f));
    bool need_ey = f->polarized != 0;
    for (int i = 0; i < nops; i++) {
        const wos_op& o = ops[i];
        if (o.kind < WOS_OP_PROPAGATE || o.kind > WOS_OP_VIEW) return fail(WOS_INVALID_ARG, "train: unknown op");
        if (o.kind == WOS_OP_VIEW && (o.method < WOS_VIEW_TOTAL || o.method > WOS_VIEW_PHASE_Y || !o.out))
            return fail(WOS_INVALID_ARG, "train: view kind / output");
        if (o.kind == WOS_OP_VIEW && (o.method == WOS_VIEW_EY || o.method == WOS_VIEW_PHASE_Y)) need_ey = true;
        if (o.kind == WOS_OP_JONES) need_ey = true;
        if (o.kind == WOS_OP_PROPAGATE && (o.method < WOS_ASM || o.method > WOS_FRAUNHOFER))
            return fail(WOS_UNKNOWN_METHOD, "unknown propagation method");
        if ((o.kind == WOS_OP_PHASE_MASK && !o.map) || (o.kind == WOS_OP_INTENSITY && !o.out))
            return fail(WOS_INVALID_ARG, "train: null map / output");
        if (o.kind == WOS_OP_GRATING && (o.method < 0 || o.method > 4 || !(o.a[0] > 0) || o.a[2] < 0 || o.a[2] > 1))
            return fail(WOS_INVALID_ARG, "train: grating parameters");
        if (o.kind == WOS_OP_LENS && (o.a[1] == 0 || !(o.a[0] > 0))) return fail(WOS_INVALID_ARG, "train: lens parameters");
        if (o.kind == WOS_OP_TILT && !(o.a[2] > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    }
    if (need_ey && !f->ey) return fail(WOS_INVALID_ARG, "train: a Jones op or an Ey view needs an Ey buffer");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const wos_context cc = cci ? *cci : default_context();
    if (diag) {
        std::memset(diag, 0, sizeof(*diag));
        diag->dx_out = f->dx;
    }
    const long long np = (long long)f->ny * f->nx;
    int pol = f->polarized ? 1 : 0;
    TRY(ensure(c->stage, (size_t)np * 16 * (need_ey ? 2 : 1)));
    CK(cudaMemcpyAsync(c->stage.p, f->ex, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    // Ey as the reference holds it (zeros for a fresh scalar field) whenever an op can read it
    if (need_ey) CK(cudaMemcpyAsync(stage_ey(c, f), f->ey, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    double2* ex = stage_ex(c);
    double2* ey = stage_ey(c, f);
    double dx = f->dx;
    bool first_prop = true;
    for (int i = 0; i < nops; i++) {
        const wos_op& o = ops[i];
        const double* a = o.a;
        switch (o.kind) {
        case WOS_OP_PROPAGATE: {
            if (a[0] == 0) break;  // Propagate with z == 0 returns at once (propagate.go:66-68)
            wos_diag d{};
            Prop p{f->ny, f->nx, dx, pol ? 2 : 1, c->stage.p, 1, c->stage.p, 1, a[0], o.method, cc, &d};
            if (!diag) p.diag = (o.method == WOS_FRAUNHOFER) ? &d : nullptr;
            TRY(run_propagate(c, p));
            if (o.method == WOS_FRAUNHOFER) dx = d.dx_out;
            if (diag) {
                diag_merge(diag, d);
                if (first_prop) diag->p_in = d.p_in;
                diag->p_out = d.p_out;
                first_prop = false;
            }
            if (bl_fraction > 0 && bl_fraction < 1) {
                const double fnyq = 1 / (2 * dx);
                double sig = bl_sigma * fnyq;
                if (sig <= 0) sig = fnyq * 0.01;
                TRY(spectral_filter(c, f->ny, f->nx, dx, pol ? 2 : 1, c->stage.p, H_BANDLIMIT, bl_fraction * fnyq,
                                    sig));
            }
        } break;
        case WOS_OP_LENS: {
            const double k = 2 * M_PI / a[0];
            CK(launch_lens(ex, ey, pol, f->ny, f->nx, dx, -k / (2 * a[1]), a[2], a[3], a[4], c->st));
        } break;
        case WOS_OP_APERTURE:
            CK(launch_aperture_circle(ex, ey, pol, f->ny, f->nx, dx, a[0], a[1], a[2], a[3], c->st));
            break;
        case WOS_OP_GRATING:
            CK(launch_grating(ex, ey, pol, f->ny, f->nx, dx, o.method, a[0], a[1], a[2], a[3], a[4], a[5], c->st));
            break;
        case WOS_OP_PHASE_MASK: {
            TRY(ensure(c->maps, sizeof(double) * np));
            CK(cudaMemcpyAsync(c->maps.p, o.map, sizeof(double) * np, cudaMemcpyHostToDevice, c->st));
            CK(launch_phase_mask(ex, ey, pol, np, reinterpret_cast<double*>(c->maps.p), a[0], c->st));
        } break;
        case WOS_OP_DIFFUSER: {
            TRY(ensure(c->aux, (size_t)np * sizeof(double2)));
            double2* zp = reinterpret_cast<double2*>(c->aux.p);
            CK(launch_diffuser_noise(zp, f->ny, f->nx, dx, dx > 0 ? dx : 1.0, a[4], a[5], (long long)a[3], c->st));
            if (a[1] > 0) {
                const double neg_two_pi_sq = -19.739208802178716;
                TRY(spectral_filter(c, f->ny, f->nx, dx, 1, zp, H_GAUSS, neg_two_pi_sq * a[1] * a[1], 0));
            }
            const int nb = sum_re2_blocks(np);
            TRY(red_prepare(c, (size_t)nb));
            CK(launch_sum_re2(zp, np, red_region(c, 0), c->st));
            CK(launch_reduce_finish(red_region(c, 0), nb, 1, 0, 2, redout_region(c, 0), c->st));
            CK(launch_diffuser_apply(ex, ey, pol, np, zp, redout_region(c, 0), a[0], a[2], c->st));
        } break;
        case WOS_OP_JONES: {
            int mode = 2;
            if (!pol) {
                const bool dg = o.m[1].re == 0 && o.m[1].im == 0 && o.m[2].re == 0 && o.m[2].im == 0 &&
                                o.m[3].re == o.m[0].re && o.m[3].im == o.m[0].im;
                mode = dg ? 0 : 1;
            }
            CK(launch_jones(ex, ey, np, mode, d2(o.m[0]), d2(o.m[1]), d2(o.m[2]), d2(o.m[3]), c->st));
            if (mode == 1) pol = 1;
        } break;
        case WOS_OP_SCALE:
            CK(launch_scale(ex, ey, pol, np, d2(o.m[0]), c->st));
            break;
        case WOS_OP_TILT:
            CK(launch_tilt(ex, ey, pol, f->ny, f->nx, dx, 2 * M_PI / a[2], std::sin(a[0]), std::sin(a[1]), c->st));
            break;
        case WOS_OP_SHIFT:
            if (a[0] != 0 || a[1] != 0)
                TRY(spectral_filter(c, f->ny, f->nx, dx, pol ? 2 : 1, c->stage.p, H_SHIFT, a[0], a[1]));
            break;
        case WOS_OP_BANDLIMIT:
            if (a[0] > 0 && a[0] < 1) {
                const double fnyq = 1 / (2 * dx);
                double sig = a[1] * fnyq;
                if (sig <= 0) sig = fnyq * 0.01;
                TRY(spectral_filter(c, f->ny, f->nx, dx, pol ? 2 : 1, c->stage.p, H_BANDLIMIT, a[0] * fnyq, sig));
            }
            break;
        case WOS_OP_INTENSITY: {
            TRY(ensure(c->accum, sizeof(double) * np));
            double* acc = reinterpret_cast<double*>(c->accum.p);
            CK(cudaMemsetAsync(acc, 0, sizeof(double) * np, c->st));
            CK(launch_accum_int(1, acc, c->stage.p, pol ? 2 : 1, np, 1.0, c->st));
            CK(cudaMemcpyAsync(o.out, acc, sizeof(double) * np, cudaMemcpyDeviceToHost, c->st));
        } break;
        case WOS_OP_VIEW: {
            TRY(ensure(c->accum, sizeof(double) * np));
            TRY(plane_view_dev(c, 1, ex, ey, nullptr, pol, np, o.method, a[0], c->accum.p));
            CK(cudaMemcpyAsync(o.out, c->accum.p, sizeof(float) * np, cudaMemcpyDeviceToHost, c->st));
        } break;
        }
    }
    f->polarized = pol;
    f->dx = dx;
    if (diag) diag->dx_out = dx;
    return stage_out(c, f, pol ? 2 : 1);
}

}  // extern "C"

// wos_design.cu -- inverse design: the ASM forward / adjoint pair, the loss
// L = sum (|u|^2 - T)^2 and its gradient with respect to a phase mask, and the
// adjoint operator of one ASM step (no counterpart in the reference).
#include "wos_api_internal.cuh"

namespace wapi {

// Inverse design on the specialised sweeps (power-of-two grids): five sweeps,
// forward ASM of a exp(i phi) | residual between the inverse and the forward
// transform of the middle row sweep | adjoint ASM | gradient in the last row
// sweep.  a: complex128 when a_c128, else the context's complex type; phi,
// target, grad: FP64 device arrays (grad null: loss only).  -1: not eligible.
int asm_design_fast(wos_ctx c, int ny, int nx, double dx, double z, const wos_context& cc, const void* a,
                    int a_c128, const double* phi, const double* target, double* loss, double* grad) {
    if (c->no_fast || !is_pow2(nx) || !is_pow2(ny)) return -1;
    const double k = 2 * M_PI / cc.wavelength;
    if (!c->fp64 && !(std::fabs(k * z / (2 * M_PI)) < 268435456.0)) return -1;
    const Tune t = get_tune(c, ny, nx);
    if (!fast_supported(c->fp64, nx, t.rowE) || !fast_supported(c->fp64, ny, t.colE)) return -1;
    Axis *ax, *ay;
    TRY(get_axis(c, nx, c->fp64, &ax));
    TRY(get_axis(c, ny, c->fp64, &ay));
    const void *twx, *twy;
    TRY(fast_tw(c, ax, t.rowE, &twx));
    TRY(fast_tw(c, ay, t.colE, &twy));
    const long long np = (long long)ny * nx;
    TRY(ensure(c->scratch, (size_t)np * c->csz()));
    void* S = c->scratch.p;
    TRY(red_prepare(c, fast_row_blocks(nx, t.rowE, ny, 1)));
    const Policy pol = ev_policy(cc, z);
    const HArgs h = asm_h(c, cc, z, pol, dx, nx, ny);
    FastCols kc{};
    kc.ncols = nx;
    kc.W = t.colW;
    kc.data = S;
    kc.ld = nx;
    kc.bstride = np;
    kc.tw = twy;
    kc.batch = 1;
    kc.wl = h.wl;
    kc.dx = h.dx;
    kc.kz = h.kz;
    kc.kaz = h.kaz;
    kc.krev = h.kz / (2 * M_PI);
    kc.scale = h.scale;
    kc.alpha = h.alpha;
    kc.limit = h.limit;
    kc.zero_ev = h.zero_ev;
    kc.reg = h.reg;
    kc.backward = h.z < 0;
    // H (and conj H for the adjoint) from one table
    if (c->fp64) TRY(attach_htab64(c, kc, ny));
    else TRY(attach_htab_global(c, kc, ny));
    FastRows r{};
    r.rows = ny;
    r.in = S;
    r.in_ld = nx;
    r.in_bstride = np;
    r.out = S;
    r.out_ld = nx;
    r.out_bstride = np;
    r.tw = twx;
    r.out_scale = 1.0;
    r.batch = 1;
    r.red = red_region(c, 0) + RS_P;
    r.red_stride = RS_COUNT;
    DesignArgs dd{phi, target, a, a_c128, grad};
    int nb = 0;
    CK(timed_launch(c, 0, [&] { return fast_rows_design(c->fp64, nx, t.rowE, 0, r, dd, c->st, &nb); }));
    CK(timed_launch(c, 4, [&] { return sweep_cols(c, ny, t.colE, kc, &nb); }));
    CK(timed_launch(c, 1, [&] { return fast_rows_design(c->fp64, nx, t.rowE, 1, r, dd, c->st, &nb); }));
    CK(launch_reduce_finish(red_region(c, 0), nb, 1, RS_P, 1, redout_region(c, 0), c->st));
    if (grad) {
        kc.conj = 1;
        CK(timed_launch(c, 4, [&] { return sweep_cols(c, ny, t.colE, kc, &nb); }));
        CK(timed_launch(c, 1, [&] { return fast_rows_design(c->fp64, nx, t.rowE, 2, r, dd, c->st, &nb); }));
    }
    TRY(fetch_red(c, 1));
    *loss = c->hred[RS_P];
    return WOS_OK;
}

// Inverse design on a host problem: forward (and adjoint) of one ASM step.
int asm_loss_grad_impl(wos_ctx c, int ny, int nx, double dx, double z, const wos_context* cc, const wos_c128* a,
                       const double* phi, const double* target, double* loss, double* grad) {
    if (!cc || !a || !phi || !target || !loss || ny < 2 || nx < 2 || !(dx > 0))
        return fail(WOS_INVALID_ARG, "inverse-design arguments");
    if (!(cc->wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    const long long np = (long long)ny * nx;
    TRY(set_device(c));
    TRY(ensure(c->stage, (size_t)np * 16));
    TRY(ensure(c->maps, (size_t)np * 8 * 3));
    TRY(ensure(c->scratch, (size_t)np * c->csz()));
    TRY(ensure(c->scratch2, (size_t)np * c->csz()));
    double* phid = reinterpret_cast<double*>(c->maps.p);
    double* Td = phid + np;
    double* gd = Td + np;
    CK(cudaMemcpyAsync(c->stage.p, a, (size_t)np * 16, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(phid, phi, (size_t)np * 8, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(Td, target, (size_t)np * 8, cudaMemcpyHostToDevice, c->st));
    {
        const int rc = asm_design_fast(c, ny, nx, dx, z, *cc, c->stage.p, 1, phid, Td, loss, grad ? gd : nullptr);
        if (rc != -1) {
            if (rc == WOS_OK && grad) {
                CK(cudaMemcpyAsync(grad, gd, (size_t)np * 8, cudaMemcpyDeviceToHost, c->st));
                CK(cudaStreamSynchronize(c->st));
            }
            return rc;
        }
    }
    Axis *ax, *ay;
    TRY(get_axis(c, nx, c->fp64, &ax));
    TRY(get_axis(c, ny, c->fp64, &ay));
    const Policy pol = ev_policy(*cc, z);
    const int W = auto_colw(c, ay->L);
    void* S = c->scratch.p;
    void* U = c->scratch2.p;
    const int nres = (int)((np + 255) / 256);
    TRY(red_prepare(c, (size_t)nres));
    auto rows = [&](int mode, const void* in, int in_c128, void* out, const double* pphi) -> int {
        RowArgs r = row_defaults(ny, nx, dx);
        r.mode = mode;
        r.rows = ny;
        fill_axis(r, ax);
        r.in = in;
        r.in_c128 = in_c128;
        r.in_ld = nx;
        r.in_n = nx;
        r.out = out;
        r.out_ld = nx;
        r.out_n = nx;
        r.pre_phi = pphi;
        CK(prof_rows(c, c->fp64, r));
        return WOS_OK;
    };
    auto cols = [&](int conj) -> int {
        ColArgs k = col_defaults(c, dx);
        k.mode = COL_FUSED;
        k.ncols = nx;
        fill_axis(k, ay);
        k.W = W;
        k.src = S;
        k.src_ld = nx;
        k.in_n = ny;
        k.dst = S;
        k.dst_ld = nx;
        k.out_n = ny;
        k.h = asm_h(c, *cc, z, pol, dx, nx, ny);
        k.h.conj = conj;
        CK(prof_cols(c, c->fp64, k));
        return WOS_OK;
    };
    // forward: u = A (a exp(i phi))
    TRY(rows(ROW_FWD, c->stage.p, 1, S, phid));
    TRY(cols(0));
    TRY(rows(ROW_INV, S, 0, U, nullptr));
    // residual r = 4 (|u|^2 - T) u, loss = sum (|u|^2 - T)^2
    int nb = 0;
    CK(launch_residual(c->fp64, U, Td, S, np, red_region(c, 0), &nb, c->st));
    CK(launch_reduce_finish(red_region(c, 0), nb, 1, RS_P, 1, redout_region(c, 0), c->st));
    if (grad) {
        // adjoint: b = A^H r = F^-1 diag(conj H) F r; grad = Re(conj(b) i t a)
        TRY(rows(ROW_FWD, S, 0, S, nullptr));
        TRY(cols(1));
        TRY(rows(ROW_INV, S, 0, S, nullptr));
        CK(launch_grad(c->fp64, S, reinterpret_cast<const double2*>(c->stage.p), phid, gd, np, c->st));
        CK(cudaMemcpyAsync(grad, gd, (size_t)np * 8, cudaMemcpyDeviceToHost, c->st));
    }
    TRY(fetch_red(c, 1));
    *loss = c->hred[RS_P];
    return WOS_OK;
}

}  // namespace wapi

extern "C" {

int wos_asm_forward_loss(wos_ctx c, int ny, int nx, double dx, double z, const wos_context* cc, const wos_c128* a,
                         const double* phi, const double* target, double* loss) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    return asm_loss_grad_impl(c, ny, nx, dx, z, cc, a, phi, target, loss, nullptr);
}

int wos_asm_loss_grad(wos_ctx c, int ny, int nx, double dx, double z, const wos_context* cc, const wos_c128* a,
                      const double* phi, const double* target, double* loss, double* grad) {
    if (!c || !grad) return fail(WOS_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(c->mu);
    return asm_loss_grad_impl(c, ny, nx, dx, z, cc, a, phi, target, loss, grad);
}

int wos_asm_loss_grad_dev(wos_ctx c, int ny, int nx, double dx, double z, const wos_context* cc, const void* a,
                          const double* phi, const double* target, double* loss, double* grad) {
    if (!c || !cc || !a || !phi || !target || !loss || ny < 2 || nx < 2 || !(dx > 0))
        return fail(WOS_INVALID_ARG, "inverse-design arguments");
    if (!(cc->wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int rc = asm_design_fast(c, ny, nx, dx, z, *cc, a, 0, phi, target, loss, grad);
    if (rc == -1)
        return fail(WOS_UNSUPPORTED_SIZE, "device-resident inverse design needs power-of-two ny, nx (256..8192)");
    return rc;
}

int wos_asm_adjoint(wos_ctx c, wos_field* f, double z, const wos_context* cci) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    TRY(check_field(f));
    const wos_context cc = cci ? *cci : default_context();
    if (!(cc.wavelength > 0)) return fail(WOS_INVALID_ARG, "wavelength must be > 0");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const int ncomp = f->polarized ? 2 : 1;
    TRY(stage_in(c, f, ncomp));
    Prop p{f->ny, f->nx, f->dx, ncomp, c->stage.p, 1, c->stage.p, 1, z, WOS_ASM, cc, nullptr};
    Sweep3 s;
    s.h = asm_h(c, cc, z, ev_policy(cc, z), f->dx, f->nx, f->ny);
    s.h.conj = 1;
    TRY(run_sweep3(c, p, s));
    return stage_out(c, f, ncomp);
}

}  // extern "C"

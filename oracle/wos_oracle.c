/*
 * wos_oracle.c -- TEST INFRASTRUCTURE ONLY (parity oracle and CPU baseline).
 *
 * FP64 C restatement of the Tetsuhiro-WOS Go `optics` propagation path.  Each
 * function cites the reference file:line it restates.  It is compiled with
 * -ffp-contract=off so that every a*b+c is two rounded operations, as the Go
 * compiler emits them on amd64, and complex products are written out as
 * (ac-bd, ad+bc) like Go's complex128 multiply.  Nothing in the product
 * library links to or calls this file.
 */
#define _GNU_SOURCE
#include "wos_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------ */
/* complex helpers (Go complex128 semantics for finite values)          */
/* ------------------------------------------------------------------ */
static inline oc128 cmk(double re, double im) { oc128 r = {re, im}; return r; }
static inline oc128 cmul(oc128 a, oc128 b) {
    oc128 r;
    r.re = a.re * b.re - a.im * b.im;
    r.im = a.re * b.im + a.im * b.re;
    return r;
}
static inline oc128 cadd(oc128 a, oc128 b) { return cmk(a.re + b.re, a.im + b.im); }
static inline oc128 csub(oc128 a, oc128 b) { return cmk(a.re - b.re, a.im - b.im); }
static inline double cabs2(oc128 a) { return a.re * a.re + a.im * a.im; }
/* cexpI (field.go:231-234) */
static inline oc128 cexpi(double phi) {
    double s, c;
    sincos(phi, &s, &c);
    return cmk(c, s);
}

/* Go constant expression -2*math.Pi*math.Pi is evaluated exactly and then
 * rounded once: the nearest double to -2*pi^2 (elements.go:750). */
static const double NEG_TWO_PI_SQ = -19.739208802178716;

/* ------------------------------------------------------------------ */
/* parFor (fft.go:91-122)                                               */
/* ------------------------------------------------------------------ */
static int g_threads = 0;

void or_set_threads(int p) { g_threads = p; }
int or_get_threads(void) {
    if (g_threads <= 0) {
        long n = sysconf(_SC_NPROCESSORS_ONLN);
        g_threads = n > 0 ? (int)n : 1;
    }
    return g_threads;
}

typedef void (*par_fn)(int i, void *arg);
typedef struct { int lo, hi; par_fn f; void *arg; } par_chunk;

static void *par_worker(void *p) {
    par_chunk *c = (par_chunk *)p;
    for (int i = c->lo; i < c->hi; i++) c->f(i, c->arg);
    return NULL;
}

static void par_for(int n, par_fn f, void *arg) {
    int P = or_get_threads();
    if (P > n) P = n;
    if (P <= 1 || n < 64) {
        for (int i = 0; i < n; i++) f(i, arg);
        return;
    }
    int chunk = (n + P - 1) / P;
    pthread_t th[256];
    par_chunk ch[256];
    if (P > 256) P = 256;
    int launched = 0;
    for (int c = 0; c < P; c++) {
        int lo = c * chunk, hi = lo + chunk;
        if (hi > n) hi = n;
        if (lo >= hi) break;
        ch[c].lo = lo; ch[c].hi = hi; ch[c].f = f; ch[c].arg = arg;
        if (pthread_create(&th[c], NULL, par_worker, &ch[c]) != 0) {
            par_worker(&ch[c]);
            th[c] = 0;
        }
        launched = c + 1;
    }
    for (int c = 0; c < launched; c++)
        if (th[c]) pthread_join(th[c], NULL);
}

/* ------------------------------------------------------------------ */
/* FFT plan (fft.go:14-51)                                              */
/* ------------------------------------------------------------------ */
typedef struct { int n; int *rev; oc128 *tw; } fft_plan;
#define MAX_PLANS 64
static fft_plan g_plans[MAX_PLANS];
static int g_nplans = 0;
static pthread_mutex_t g_plan_mu = PTHREAD_MUTEX_INITIALIZER;

static const fft_plan *plan_fft(int n) {
    pthread_mutex_lock(&g_plan_mu);
    for (int i = 0; i < g_nplans; i++)
        if (g_plans[i].n == n) { pthread_mutex_unlock(&g_plan_mu); return &g_plans[i]; }
    int bits = 0;
    for (int m = n; m > 1; m >>= 1) bits++;
    int *rev = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) {
        int r = 0, v = i;
        for (int b = 0; b < bits; b++) { r = (r << 1) | (v & 1); v >>= 1; }
        rev[i] = r;
    }
    int half = n / 2;
    oc128 *tw = (oc128 *)malloc(sizeof(oc128) * (size_t)(half + 1));
    for (int k = 0; k <= half; k++) {
        double ang = -2 * M_PI * (double)k / (double)n;
        tw[k] = cmk(cos(ang), sin(ang));
    }
    fft_plan *p;
    if (g_nplans < MAX_PLANS) {
        p = &g_plans[g_nplans++];
    } else { /* evict the oldest (plans are immutable once published; leak the old tables) */
        memmove(&g_plans[0], &g_plans[1], sizeof(fft_plan) * (MAX_PLANS - 1));
        p = &g_plans[MAX_PLANS - 1];
    }
    p->n = n; p->rev = rev; p->tw = tw;
    pthread_mutex_unlock(&g_plan_mu);
    return p;
}

/* fft1D (fft.go:55-87) */
static void fft1d_plan(oc128 *a, const fft_plan *plan, int inverse) {
    int n = plan->n;
    for (int i = 0; i < n; i++) {
        int j = plan->rev[i];
        if (i < j) { oc128 t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (int size = 2; size <= n; size <<= 1) {
        int half = size / 2, step = n / size;
        for (int i = 0; i < n; i += size) {
            for (int j = 0; j < half; j++) {
                oc128 w = plan->tw[j * step];
                if (inverse) w.im = -w.im;
                oc128 u = a[i + j];
                oc128 v = cmul(a[i + j + half], w);
                a[i + j] = cadd(u, v);
                a[i + j + half] = csub(u, v);
            }
        }
    }
    if (inverse) {
        oc128 inv = cmk(1.0 / (double)n, 0); /* 1/complex(n,0) = (1/n, 0) */
        for (int i = 0; i < n; i++) a[i] = cmul(a[i], inv);
    }
}

void or_fft1d_pow2(oc128 *a, int n, int inverse) {
    if (n <= 0) return;
    fft1d_plan(a, plan_fft(n), inverse);
}

/* fft1DBluestein (fft.go:159-204) */
void or_bluestein(oc128 *a, int n, int inverse) {
    if (n <= 1) return;
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    double sign = inverse ? 1.0 : -1.0;
    oc128 *chirp = (oc128 *)malloc(sizeof(oc128) * (size_t)n);
    for (long long k = 0; k < n; k++)
        chirp[k] = cexpi(sign * M_PI * (double)(k * k) / (double)n);
    oc128 *a0 = (oc128 *)calloc((size_t)m, sizeof(oc128));
    oc128 *b0 = (oc128 *)calloc((size_t)m, sizeof(oc128));
    for (int k = 0; k < n; k++) a0[k] = cmul(a[k], chirp[k]);
    b0[0] = cmk(1, 0);
    for (int k = 1; k < n; k++) {
        oc128 ck = cmk(chirp[k].re, -chirp[k].im);
        b0[k] = ck;
        b0[m - k] = ck;
    }
    const fft_plan *plan = plan_fft(m);
    fft1d_plan(a0, plan, 0);
    fft1d_plan(b0, plan, 0);
    for (int k = 0; k < m; k++) a0[k] = cmul(a0[k], b0[k]);
    fft1d_plan(a0, plan, 1);
    for (int k = 0; k < n; k++) a[k] = cmul(a0[k], chirp[k]);
    if (inverse) {
        oc128 inv = cmk(1.0 / (double)n, 0);
        for (int k = 0; k < n; k++) a[k] = cmul(a[k], inv);
    }
    free(chirp); free(a0); free(b0);
}

/* fft1DAnyCPU (fft.go:146-153) */
void or_fft1d(oc128 *a, int n, int inverse) {
    if (n <= 0) return;
    if ((n & (n - 1)) == 0) { fft1d_plan(a, plan_fft(n), inverse); return; }
    or_bluestein(a, n, inverse);
}

/* fft2DCPU (fft.go:219-242): rows, then columns through per-worker scratch */
typedef struct { oc128 *a; int ny, nx, inverse; } fft2_arg;
static void fft2_row(int r, void *p) {
    fft2_arg *g = (fft2_arg *)p;
    or_fft1d(g->a + (size_t)r * g->nx, g->nx, g->inverse);
}
static void fft2_col(int c, void *p) {
    fft2_arg *g = (fft2_arg *)p;
    oc128 *col = (oc128 *)malloc(sizeof(oc128) * (size_t)g->ny);
    for (int r = 0; r < g->ny; r++) col[r] = g->a[(size_t)r * g->nx + c];
    or_fft1d(col, g->ny, g->inverse);
    for (int r = 0; r < g->ny; r++) g->a[(size_t)r * g->nx + c] = col[r];
    free(col);
}
void or_fft2d(oc128 *a, int ny, int nx, int inverse) {
    fft2_arg g = {a, ny, nx, inverse};
    par_for(ny, fft2_row, &g);
    par_for(nx, fft2_col, &g);
}

/* ------------------------------------------------------------------ */
/* Field helpers (field.go)                                             */
/* ------------------------------------------------------------------ */
static inline double fX(const or_field *f, int i) { return ((double)i - (double)f->nx / 2) * f->dx; }
static inline double fY(const or_field *f, int j) { return ((double)j - (double)f->ny / 2) * f->dx; }
/* freq (field.go:297-303), per axis of length n */
static inline double freq_n(int i, int n, double dx) {
    if (i <= n / 2) return (double)i / ((double)n * dx);
    return (double)(i - n) / ((double)n * dx);
}
static inline size_t npix(const or_field *f) { return (size_t)f->ny * (size_t)f->nx; }
/* Intensity (field.go:65-74) */
static inline double intensity(const or_field *f, size_t idx) {
    double p = f->ex[idx].re * f->ex[idx].re + f->ex[idx].im * f->ex[idx].im;
    if (f->polarized) p += f->ey[idx].re * f->ey[idx].re + f->ey[idx].im * f->ey[idx].im;
    return p;
}
/* Power (field.go:77-83) */
double or_power(const or_field *f) {
    double p = 0;
    size_t n = npix(f);
    for (size_t i = 0; i < n; i++) p += intensity(f, i);
    return p * f->dx * f->dx;
}

/* Warnings.Add (field.go:322-338) */
static void warn_add(or_context *ctx, const char *code, double value) {
    if (!ctx || !ctx->has_warnings) return;
    for (int i = 0; i < ctx->n_warn; i++) {
        if (strcmp(ctx->warn[i].code, code) == 0) {
            ctx->warn[i].count++;
            if (value != 0) ctx->warn[i].value = value;
            return;
        }
    }
    if (ctx->n_warn >= 16) return;
    or_warning *w = &ctx->warn[ctx->n_warn++];
    memset(w, 0, sizeof(*w));
    strncpy(w->code, code, sizeof(w->code) - 1);
    w->count = 1;
    w->value = value;
}

/* rmsRadius (propagate.go:105-130) */
double or_rms_radius(const or_field *f) {
    double p = 0, px = 0, py = 0;
    for (int j = 0; j < f->ny; j++) {
        double y = fY(f, j);
        for (int i = 0; i < f->nx; i++) {
            double w = intensity(f, (size_t)j * f->nx + i);
            p += w;
            px += w * fX(f, i);
            py += w * y;
        }
    }
    if (p <= 0) return 0;
    double cx = px / p, cy = py / p;
    double vr = 0;
    for (int j = 0; j < f->ny; j++) {
        double y = fY(f, j);
        for (int i = 0; i < f->nx; i++) {
            double w = intensity(f, (size_t)j * f->nx + i);
            vr += w * ((fX(f, i) - cx) * (fX(f, i) - cx) + (y - cy) * (y - cy));
        }
    }
    return 2 * sqrt(vr / p);
}

/* math.Hypot as the Go amd64 kernel evaluates it: scale by the larger magnitude */
static inline double go_hypot(double p, double q) {
    p = fabs(p); q = fabs(q);
    if (isinf(p) || isinf(q)) return INFINITY;
    if (isnan(p) || isnan(q)) return NAN;
    if (p < q) { double t = p; p = q; q = t; }
    if (p == 0) return 0;
    q = q / p;
    return p * sqrt(1 + q * q);
}

/* spectralRadius (propagate.go:270-320) */
double or_spectral_radius(const or_field *f, double frac) {
    if (frac <= 0 || frac >= 1) frac = 0.99;
    const int bins = 96;
    double fnyq = 1 / (2 * f->dx);
    if (f->nx == 0 || f->ny == 0 || f->dx <= 0) return 0;
    double hist[97];
    memset(hist, 0, sizeof(hist));
    double tot = 0;
    size_t n = npix(f);
    oc128 *a = (oc128 *)malloc(sizeof(oc128) * n);
    for (int comp = 0; comp < (f->polarized ? 2 : 1); comp++) {
        memcpy(a, comp ? f->ey : f->ex, sizeof(oc128) * n);
        or_fft2d(a, f->ny, f->nx, 0);
        for (int j = 0; j < f->ny; j++) {
            double fy = freq_n(j, f->ny, f->dx);
            for (int i = 0; i < f->nx; i++) {
                oc128 v = a[(size_t)j * f->nx + i];
                double w = v.re * v.re + v.im * v.im;
                if (w == 0) continue;
                int b = (int)(go_hypot(freq_n(i, f->nx, f->dx), fy) / fnyq * bins);
                if (b > bins) b = bins;
                hist[b] += w;
                tot += w;
            }
        }
    }
    free(a);
    if (tot <= 0) return 0;
    double run = 0;
    for (int b = 0; b <= bins; b++) {
        run += hist[b];
        if (run >= frac * tot) return (double)b / bins * fnyq;
    }
    return fnyq;
}

/* spectralCentroid (propagate.go:391-416) */
void or_spectral_centroid(const or_field *f, double *fxo, double *fyo) {
    double sx = 0, sy = 0, sw = 0;
    size_t n = npix(f);
    oc128 *a = (oc128 *)malloc(sizeof(oc128) * n);
    for (int comp = 0; comp < (f->polarized ? 2 : 1); comp++) {
        memcpy(a, comp ? f->ey : f->ex, sizeof(oc128) * n);
        or_fft2d(a, f->ny, f->nx, 0);
        for (int j = 0; j < f->ny; j++) {
            double fy = freq_n(j, f->ny, f->dx);
            for (int i = 0; i < f->nx; i++) {
                double fx = freq_n(i, f->nx, f->dx);
                oc128 v = a[(size_t)j * f->nx + i];
                double w = v.re * v.re + v.im * v.im;
                sw += w;
                sx += w * fx;
                sy += w * fy;
            }
        }
    }
    free(a);
    if (sw <= 0) { *fxo = 0; *fyo = 0; return; }
    *fxo = sx / sw;
    *fyo = sy / sw;
}

/* ------------------------------------------------------------------ */
/* transfer functions (propagate.go)                                    */
/* ------------------------------------------------------------------ */
/* asmTF (propagate.go:159-181) */
oc128 or_asm_tf(double wl, double z, int zero_ev, int reg, double alpha, double limit,
                double fx, double fy) {
    double k = 2 * M_PI / wl;
    double az = fabs(z);
    int backward = z < 0;
    double rho = go_hypot(wl * fx, wl * fy);
    if (rho <= 1) return cexpi(k * z * sqrt((1 - rho) * (1 + rho)));
    double decay = k * az * sqrt((rho - 1) * (rho + 1));
    if (zero_ev || (limit > 0 && decay > limit)) return cmk(0, 0);
    if (backward) {
        if (reg) {
            double a = exp(decay);
            return cmk(a / (1 + alpha * alpha * a * a), 0);
        }
        return cmk(exp(decay), 0);
    }
    return cmk(exp(-decay), 0);
}

/* evanescentPolicy (propagate.go:186-199) */
static void ev_policy(const or_context *ctx, double z, int *zero, int *reg, double *alpha,
                      double *limit) {
    *limit = ctx->evanescent_limit;
    *alpha = 0;
    if (z < 0) {
        if (ctx->backward_regularize) {
            *alpha = ctx->tikhonov_alpha;
            if (*alpha <= 0) *alpha = 1e-3;
            *zero = 0; *reg = 1;
            return;
        }
        *zero = 1; *reg = 0;
        return;
    }
    *zero = ctx->evanescent_zero; *reg = 0;
}

/* asmWarn (propagate.go:203-218) */
static void asm_warn(double z, or_context *ctx, double pin, double pout, int zero, int reg) {
    if (pin > 0 && pout < pin * (1 - 1e-8) && z > 0)
        warn_add(ctx, "evanescent_filtered", (pin - pout) / pin);
    if (z < 0) {
        if (reg) warn_add(ctx, "backward_regularized", 0);
        else if (zero) warn_add(ctx, "backward_evanescent", 0);
    }
}

/* asmWrapWarn (propagate.go:247-264); carry generalised to min(nx,ny)*dx */
static void asm_wrap_warn(const or_field *f, double z, or_context *ctx, double carry) {
    if (!ctx || !ctx->has_warnings || z == 0 || carry <= 0) return;
    if (fabs(z) * ctx->wavelength / (2 * f->dx) <= carry) return;
    double fsig = or_spectral_radius(f, 0.90);
    if (fsig <= 0) return;
    double walk = fabs(z) * ctx->wavelength * fsig;
    if (walk > carry) warn_add(ctx, "asm_alias_wrap", walk / carry);
}

static double carry_of(const or_field *f) {
    int n = f->nx < f->ny ? f->nx : f->ny;
    return (double)n * f->dx;
}

typedef struct {
    int kind; /* 0 asm, 1 fresnel_tf */
    double wl, z, alpha, limit;
    int zero, reg;
    double fxoff, fyoff;
} tf_spec;

static inline oc128 tf_eval(const tf_spec *t, double fx, double fy) {
    if (t->kind == 0) return or_asm_tf(t->wl, t->z, t->zero, t->reg, t->alpha, t->limit, fx, fy);
    /* propFresnelTF (propagate.go:511-513) */
    double k = 2 * M_PI / t->wl;
    return cmul(cexpi(k * t->z), cexpi(-M_PI * t->wl * t->z * (fx * fx + fy * fy)));
}

/* Context.transfer (propagate.go:132-148) on an ny x nx array */
static void transfer_arr(oc128 *a, int ny, int nx, double dx, const tf_spec *t) {
    or_fft2d(a, ny, nx, 0);
    for (int j = 0; j < ny; j++) {
        double fy = freq_n(j, ny, dx) + t->fyoff;
        for (int i = 0; i < nx; i++) {
            size_t idx = (size_t)j * nx + i;
            a[idx] = cmul(a[idx], tf_eval(t, freq_n(i, nx, dx) + t->fxoff, fy));
        }
    }
    or_fft2d(a, ny, nx, 1);
}

static void transfer(or_field *f, const tf_spec *t) {
    transfer_arr(f->ex, f->ny, f->nx, f->dx, t);
    if (f->polarized) transfer_arr(f->ey, f->ny, f->nx, f->dx, t);
}

/* propASM (propagate.go:325-332) */
static void prop_asm(or_field *f, double z, or_context *ctx) {
    tf_spec t = {0};
    t.kind = 0; t.wl = ctx->wavelength; t.z = z;
    ev_policy(ctx, z, &t.zero, &t.reg, &t.alpha, &t.limit);
    asm_wrap_warn(f, z, ctx, carry_of(f));
    double pin = or_power(f);
    transfer(f, &t);
    double pout = or_power(f);
    asm_warn(z, ctx, pin, pout, t.zero, t.reg);
}

/* propASMPadCore (propagate.go:346-387), 2x pad per axis */
static void prop_asm_pad_core(or_field *f, double z, or_context *ctx, double fxoff, double fyoff) {
    int ny = f->ny, nx = f->nx, my = 2 * ny, mx = 2 * nx;
    double dx = f->dx;
    tf_spec t = {0};
    t.kind = 0; t.wl = ctx->wavelength; t.z = z;
    ev_policy(ctx, z, &t.zero, &t.reg, &t.alpha, &t.limit);
    asm_wrap_warn(f, z, ctx, carry_of(f));
    double pin = or_power(f);
    oc128 *buf = (oc128 *)malloc(sizeof(oc128) * (size_t)my * mx);
    int offy = ny / 2, offx = nx / 2;
    for (int comp = 0; comp < (f->polarized ? 2 : 1); comp++) {
        oc128 *a = comp ? f->ey : f->ex;
        memset(buf, 0, sizeof(oc128) * (size_t)my * mx);
        for (int j = 0; j < ny; j++)
            memcpy(buf + (size_t)(j + offy) * mx + offx, a + (size_t)j * nx, sizeof(oc128) * nx);
        or_fft2d(buf, my, mx, 0);
        for (int j = 0; j < my; j++) {
            double fy = freq_n(j, my, dx) + fyoff;
            for (int i = 0; i < mx; i++) {
                size_t idx = (size_t)j * mx + i;
                buf[idx] = cmul(buf[idx], tf_eval(&t, freq_n(i, mx, dx) + fxoff, fy));
            }
        }
        or_fft2d(buf, my, mx, 1);
        for (int j = 0; j < ny; j++)
            memcpy(a + (size_t)j * nx, buf + (size_t)(j + offy) * mx + offx, sizeof(oc128) * nx);
    }
    free(buf);
    double pout = or_power(f);
    asm_warn(z, ctx, pin, pout, t.zero, t.reg);
}

/* carrier ramp of propASMShift (propagate.go:437-444) */
static void shift_ramp(or_field *f, oc128 *a, double sgn, double fxc, double fyc) {
    for (int j = 0; j < f->ny; j++) {
        double y = fY(f, j);
        for (int i = 0; i < f->nx; i++) {
            size_t idx = (size_t)j * f->nx + i;
            a[idx] = cmul(a[idx], cexpi(sgn * 2 * M_PI * (fxc * fX(f, i) + fyc * y)));
        }
    }
}

/* propASMShift (propagate.go:426-471) after its spectralCentroid call */
static void prop_asm_shift_at(or_field *f, double z, or_context *ctx, double fxc, double fyc) {
    double fbx = 1 / ((double)f->nx * f->dx), fby = 1 / ((double)f->ny * f->dx);
    if (fabs(fxc) < 0.5 * fbx && fabs(fyc) < 0.5 * fby) { prop_asm(f, z, ctx); return; }
    tf_spec t = {0};
    t.kind = 0; t.wl = ctx->wavelength; t.z = z; t.fxoff = fxc; t.fyoff = fyc;
    ev_policy(ctx, z, &t.zero, &t.reg, &t.alpha, &t.limit);
    asm_wrap_warn(f, z, ctx, carry_of(f));
    double pin = or_power(f);
    shift_ramp(f, f->ex, -1, fxc, fyc);
    if (f->polarized) shift_ramp(f, f->ey, -1, fxc, fyc);
    transfer(f, &t);
    shift_ramp(f, f->ex, +1, fxc, fyc);
    if (f->polarized) shift_ramp(f, f->ey, +1, fxc, fyc);
    double pout = or_power(f);
    asm_warn(z, ctx, pin, pout, t.zero, t.reg);
}

/* propASMShiftPad (propagate.go:479-504) after its spectralCentroid call */
static void prop_asm_shift_pad_at(or_field *f, double z, or_context *ctx, double fxc, double fyc) {
    double fbx = 1 / ((double)f->nx * f->dx), fby = 1 / ((double)f->ny * f->dx);
    if (fabs(fxc) < 0.5 * fbx && fabs(fyc) < 0.5 * fby) { prop_asm_pad_core(f, z, ctx, 0, 0); return; }
    shift_ramp(f, f->ex, -1, fxc, fyc);
    if (f->polarized) shift_ramp(f, f->ey, -1, fxc, fyc);
    prop_asm_pad_core(f, z, ctx, fxc, fyc);
    shift_ramp(f, f->ex, +1, fxc, fyc);
    if (f->polarized) shift_ramp(f, f->ey, +1, fxc, fyc);
}

static void prop_asm_shift(or_field *f, double z, or_context *ctx) {
    double fxc, fyc;
    or_spectral_centroid(f, &fxc, &fyc);
    prop_asm_shift_at(f, z, ctx, fxc, fyc);
}

static void prop_asm_shift_pad(or_field *f, double z, or_context *ctx) {
    double fxc, fyc;
    or_spectral_centroid(f, &fxc, &fyc);
    prop_asm_shift_pad_at(f, z, ctx, fxc, fyc);
}

/* The carrier-shift methods with the centroid supplied by the caller (a test
 * hook: it separates the rounding of the centroid's sequential sums from the
 * rest of the propagation). */
int or_propagate_shift_at(or_field *f, double z, int method, or_context *ctx, double fxc, double fyc) {
    if (z == 0) return 0;
    or_context local;
    if (!ctx) {
        memset(&local, 0, sizeof(local));
        ctx = &local;
    }
    if (method == OR_ASM_SHIFT) prop_asm_shift_at(f, z, ctx, fxc, fyc);
    else if (method == OR_ASM_SHIFT_PAD) prop_asm_shift_pad_at(f, z, ctx, fxc, fyc);
    else return -1;
    return 0;
}

/* propFresnelTF (propagate.go:507-519); alias bound uses min(nx,ny) */
static void prop_fresnel_tf(or_field *f, double z, or_context *ctx) {
    tf_spec t = {0};
    t.kind = 1; t.wl = ctx->wavelength; t.z = z;
    transfer(f, &t);
    int n = f->nx < f->ny ? f->nx : f->ny;
    if (fabs(z) > (double)n * f->dx * f->dx / ctx->wavelength)
        warn_add(ctx, "fresnel_tf_alias", 0);
}

/* impulse-response offset in wrap layout (propagate.go:545-555) */
static inline double wrap_off(int p, int m) {
    double d = (double)p;
    if (p > m / 2) d -= (double)m;
    return d;
}

/* propFresnelIR (propagate.go:533-590); alias bound uses max(nx,ny) */
static void prop_fresnel_ir(or_field *f, double z, or_context *ctx) {
    double wl = ctx->wavelength;
    double k = 2 * M_PI / wl;
    int ny = f->ny, nx = f->nx, my = 2 * ny, mx = 2 * nx;
    double dx = f->dx;
    size_t mm = (size_t)my * mx;
    oc128 *h = (oc128 *)malloc(sizeof(oc128) * mm);
    for (int j = 0; j < my; j++) {
        double y = wrap_off(j, my) * dx;
        for (int i = 0; i < mx; i++) {
            double x = wrap_off(i, mx) * dx;
            h[(size_t)j * mx + i] = cexpi(M_PI * (x * x + y * y) / (wl * z));
        }
    }
    or_fft2d(h, my, mx, 0);
    oc128 pre = cmul(cmul(cmk(0, -1 / (wl * z)), cexpi(k * z)), cmk(dx * dx, 0));
    oc128 *buf = (oc128 *)malloc(sizeof(oc128) * mm);
    int offy = ny / 2, offx = nx / 2;
    for (int comp = 0; comp < (f->polarized ? 2 : 1); comp++) {
        oc128 *a = comp ? f->ey : f->ex;
        memset(buf, 0, sizeof(oc128) * mm);
        for (int j = 0; j < ny; j++)
            memcpy(buf + (size_t)(j + offy) * mx + offx, a + (size_t)j * nx, sizeof(oc128) * nx);
        or_fft2d(buf, my, mx, 0);
        for (size_t i = 0; i < mm; i++) buf[i] = cmul(buf[i], h[i]);
        or_fft2d(buf, my, mx, 1);
        for (size_t i = 0; i < mm; i++) buf[i] = cmul(buf[i], pre);
        for (int j = 0; j < ny; j++)
            memcpy(a + (size_t)j * nx, buf + (size_t)(j + offy) * mx + offx, sizeof(oc128) * nx);
    }
    free(buf); free(h);
    int n = f->nx > f->ny ? f->nx : f->ny;
    if (fabs(z) < (double)n * dx * dx / wl) warn_add(ctx, "fresnel_ir_alias", 0);
}

/* propFraunhofer (propagate.go:603-662); square grids only */
static int prop_fraunhofer(or_field *f, double z, or_context *ctx) {
    if (f->nx != f->ny) return -2;
    double wl = ctx->wavelength;
    double k = 2 * M_PI / wl;
    int n = f->nx;
    double dxout = wl * fabs(z) / ((double)n * f->dx);
    double din = or_rms_radius(f);
    size_t nn = (size_t)n * n;
    oc128 *shift = (oc128 *)malloc(sizeof(oc128) * nn);
    for (int comp = 0; comp < (f->polarized ? 2 : 1); comp++) {
        oc128 *a = comp ? f->ey : f->ex;
        or_fft2d(a, n, n, 0);
        for (size_t i = 0; i < nn; i++) a[i] = cmul(a[i], cmk(f->dx * f->dx, 0));
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++)
                if ((i + j) & 1) {
                    size_t idx = (size_t)j * n + i;
                    a[idx] = cmk(-a[idx].re, -a[idx].im);
                }
        int half = n / 2;
        for (int j = 0; j < n; j++) {
            size_t row = (size_t)j * n;
            memcpy(shift + row, a + row + half, sizeof(oc128) * (size_t)(n - half));
            memcpy(shift + row + half, a + row, sizeof(oc128) * (size_t)half);
        }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < half; j++) {
                oc128 t = shift[(size_t)j * n + i];
                shift[(size_t)j * n + i] = shift[(size_t)(j + half) * n + i];
                shift[(size_t)(j + half) * n + i] = t;
            }
        for (int j = 0; j < n; j++) {
            double y = ((double)j - (double)n / 2) * dxout;
            for (int i = 0; i < n; i++) {
                double x = ((double)i - (double)n / 2) * dxout;
                size_t idx = (size_t)j * n + i;
                oc128 fac = cmul(cmul(cexpi(k * z), cmk(0, -1 / (wl * z))),
                                 cexpi(k * (x * x + y * y) / (2 * z)));
                shift[idx] = cmul(shift[idx], fac);
            }
        }
        memcpy(a, shift, sizeof(oc128) * nn);
    }
    free(shift);
    if (din > 0) {
        double nf = din * din / (wl * fabs(z));
        if (nf > 0.5) warn_add(ctx, "fraunhofer_nearfield", nf);
    }
    f->dx = dxout;
    return 0;
}

/* Propagate (propagate.go:65-102) */
int or_propagate(or_field *f, double z, int method, or_context *ctx) {
    if (z == 0) return 0;
    or_context local;
    if (!ctx) {
        memset(&local, 0, sizeof(local));
        ctx = &local; /* Evanescent "decay", no warnings */
    }
    switch (method) {
    case OR_ASM: prop_asm(f, z, ctx); return 0;
    case OR_ASM_PAD: prop_asm_pad_core(f, z, ctx, 0, 0); return 0;
    case OR_ASM_SHIFT: prop_asm_shift(f, z, ctx); return 0;
    case OR_ASM_SHIFT_PAD: prop_asm_shift_pad(f, z, ctx); return 0;
    case OR_FRESNEL_TF: prop_fresnel_tf(f, z, ctx); return 0;
    case OR_FRESNEL_IR: prop_fresnel_ir(f, z, ctx); return 0;
    case OR_FRAUNHOFER: return prop_fraunhofer(f, z, ctx);
    }
    return -1;
}

/* Propagate1D with asmTF1D (propagate.go:679-738) */
int or_propagate1d(oc128 *a, int n, double dx, double z, double wl, or_context *ctx) {
    or_context local;
    if (!ctx) { memset(&local, 0, sizeof(local)); ctx = &local; }
    int zero, reg; double alpha, limit;
    ev_policy(ctx, z, &zero, &reg, &alpha, &limit);
    double k = 2 * M_PI / wl, az = fabs(z);
    int backward = z < 0;
    double pin = 0;
    for (int i = 0; i < n; i++) pin += a[i].re * a[i].re + a[i].im * a[i].im;
    or_fft1d(a, n, 0);
    for (int i = 0; i < n; i++) {
        double fx = freq_n(i, n, dx);
        double rho = fabs(wl * fx);
        oc128 h;
        if (rho <= 1) {
            h = cexpi(k * z * sqrt((1 - rho) * (1 + rho)));
        } else {
            double decay = k * az * sqrt((rho - 1) * (rho + 1));
            if (zero || (limit > 0 && decay > limit)) h = cmk(0, 0);
            else if (backward) {
                if (reg) { double A = exp(decay); h = cmk(A / (1 + alpha * alpha * A * A), 0); }
                else h = cmk(exp(decay), 0);
            } else h = cmk(exp(-decay), 0);
        }
        a[i] = cmul(a[i], h);
    }
    or_fft1d(a, n, 1);
    double pout = 0;
    for (int i = 0; i < n; i++) pout += a[i].re * a[i].re + a[i].im * a[i].im;
    if (pin > 0 && pout < pin * (1 - 1e-8) && z > 0) warn_add(ctx, "evanescent_filtered", (pin - pout) / pin);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Split-step BPM (medium.go:22-65)                                     */
/* ------------------------------------------------------------------ */
void or_index_eval(const or_index_desc *d, int ny, int nx, double dx, int i, int j,
                   double x, double y, double z, double *re, double *im) {
    (void)dx;
    double r0 = d->re_bg, i0 = d->im_bg;
    for (int k = 0; k < d->n_layers && k < 8; k++) {
        if (z < d->layer_z[k]) { r0 = d->layer_re[k]; i0 = d->layer_im[k]; break; }
    }
    double nr = r0, ni = i0;
    if (d->core_dn != 0) {
        double ddx = x - d->core_x0, ddy = y - d->core_y0;
        double g = exp(-(ddx * ddx + ddy * ddy) / (d->core_w * d->core_w));
        double mod = 1;
        if (d->zmod_amp != 0) mod = 1 + d->zmod_amp * sin(2 * M_PI * z / d->zmod_period + d->zmod_phase);
        nr = r0 + d->core_dn * g * mod;
    }
    if (d->border_px > 0 && d->border_strength != 0) {
        int dd = i;
        if (j < dd) dd = j;
        if (nx - 1 - i < dd) dd = nx - 1 - i;
        if (ny - 1 - j < dd) dd = ny - 1 - j;
        if (dd < d->border_px) {
            double t = (double)(d->border_px - dd) / (double)d->border_px;
            double p = 1;
            for (int q = 0; q < d->border_order; q++) p *= t;
            ni = i0 + d->border_strength * p;
        }
    }
    *re = nr;
    *im = ni;
}

typedef struct { const or_index_desc *d; int ny, nx; double dx; } desc_user;

/* applyMediumPhase (medium.go:50-65) for a sampled index */
static void apply_medium_phase(or_field *f, const double *nre, const double *nim, double k, double dz) {
    for (int j = 0; j < f->ny; j++) {
        for (int i = 0; i < f->nx; i++) {
            size_t idx = (size_t)j * f->nx + i;
            double ph = k * (nre[idx] - 1) * dz;
            oc128 t = cmul(cmk(exp(-k * nim[idx] * dz), 0), cexpi(ph));
            f->ex[idx] = cmul(f->ex[idx], t);
            if (f->polarized) f->ey[idx] = cmul(f->ey[idx], t);
        }
    }
}

static int splitstep_core(or_field *f, double z, or_index_fn fn, void *user, const or_index_desc *d,
                          int steps, or_context *ctx) {
    if (z == 0) return 0;
    if (steps <= 0) steps = 1;
    or_context local;
    if (!ctx) { memset(&local, 0, sizeof(local)); ctx = &local; }
    double dz = z / (double)steps;
    double k = 2 * M_PI / ctx->wavelength;
    size_t n = npix(f);
    double *nre = (double *)malloc(sizeof(double) * n);
    double *nim = (double *)malloc(sizeof(double) * n);
    for (int s = 0; s < steps; s++) {
        double zc = z * (double)s / (double)steps + dz / 2;
        or_propagate(f, dz / 2, OR_ASM, ctx);
        for (int j = 0; j < f->ny; j++) {
            double y = fY(f, j);
            for (int i = 0; i < f->nx; i++) {
                size_t idx = (size_t)j * f->nx + i;
                if (d) or_index_eval(d, f->ny, f->nx, f->dx, i, j, fX(f, i), y, zc, &nre[idx], &nim[idx]);
                else fn(fX(f, i), y, zc, user, &nre[idx], &nim[idx]);
            }
        }
        apply_medium_phase(f, nre, nim, k, dz);
        or_propagate(f, dz / 2, OR_ASM, ctx);
    }
    free(nre); free(nim);
    return 0;
}

int or_splitstep(or_field *f, double z, const or_index_desc *d, int steps, or_context *ctx) {
    return splitstep_core(f, z, NULL, NULL, d, steps, ctx);
}
int or_splitstep_fn(or_field *f, double z, or_index_fn fn, void *user, int steps, or_context *ctx) {
    return splitstep_core(f, z, fn, user, NULL, steps, ctx);
}

/* ------------------------------------------------------------------ */
/* Batches                                                              */
/* ------------------------------------------------------------------ */
static or_field clone_field(const or_field *f) {
    or_field g = *f;
    size_t n = npix(f);
    g.ex = (oc128 *)malloc(sizeof(oc128) * n);
    memcpy(g.ex, f->ex, sizeof(oc128) * n);
    g.ey = (oc128 *)calloc(n, sizeof(oc128));
    if (f->polarized && f->ey) memcpy(g.ey, f->ey, sizeof(oc128) * n);
    return g;
}
static void free_field(or_field *g) { free(g->ex); free(g->ey); }

/* PropagatePolychromatic (polychromatic.go:18-44).  The samples' contexts
 * copy the caller's, whose Warnings is a shared pointer in the reference: what
 * every sample adds ends up in the caller's context (written back here). */
int or_polychromatic(const or_field *f, double z, const double *wl, const double *weight, int ns,
                     int method, or_context *base_io, double *out) {
    if (ns <= 0) return -3;
    or_context base;
    if (base_io) base = *base_io;
    else { memset(&base, 0, sizeof(base)); base.has_warnings = 1; }
    size_t n = npix(f);
    memset(out, 0, sizeof(double) * n);
    int rc = 0;
    for (int s = 0; s < ns && rc == 0; s++) {
        if (wl[s] <= 0) { rc = -4; break; }
        or_field g = clone_field(f);
        or_context c = base;
        c.wavelength = wl[s];
        rc = or_propagate(&g, z, method, &c);
        base.n_warn = c.n_warn;
        memcpy(base.warn, c.warn, sizeof(base.warn));
        if (rc == 0)
            for (size_t i = 0; i < n; i++) out[i] += weight[s] * intensity(&g, i);
        free_field(&g);
    }
    if (base_io) {
        base_io->n_warn = base.n_warn;
        memcpy(base_io->warn, base.warn, sizeof(base.warn));
    }
    return rc;
}

/* Propagate3D (volume.go:8-18) */
int or_propagate3d(const or_field *f, const double *zs, int nz, int method, or_context *ctx_io,
                   oc128 *out) {
    size_t n = npix(f);
    int ncomp = f->polarized ? 2 : 1;
    or_context ctx;
    if (ctx_io) ctx = *ctx_io; else memset(&ctx, 0, sizeof(ctx));
    int rc = 0;
    for (int q = 0; q < nz && rc == 0; q++) {
        or_field g = clone_field(f);
        rc = or_propagate(&g, zs[q], method, &ctx);
        if (rc == 0) {
            memcpy(out + (size_t)q * ncomp * n, g.ex, sizeof(oc128) * n);
            if (ncomp == 2) memcpy(out + ((size_t)q * ncomp + 1) * n, g.ey, sizeof(oc128) * n);
        }
        free_field(&g);
    }
    if (ctx_io) { /* the same Context (and Warnings) for every plane (volume.go:8-18) */
        ctx_io->n_warn = ctx.n_warn;
        memcpy(ctx_io->warn, ctx.warn, sizeof(ctx.warn));
    }
    return rc;
}

/* GenerateSchellRealizations (coherence.go:22-80) with caller noise */
int or_schell_realizations(int n, double dx, double width, double coherence, int m,
                           const oc128 *noise, oc128 *out) {
    if (width <= 0 || coherence <= 0) return -4;
    if (m <= 0) m = 1;
    size_t nn = (size_t)n * n;
    oc128 *sqs = (oc128 *)malloc(sizeof(oc128) * nn);
    for (int j = 0; j < n; j++) {
        double dy = (j <= n / 2) ? (double)j * dx : (double)(j - n) * dx;
        for (int i = 0; i < n; i++) {
            double d = (i <= n / 2) ? (double)i * dx : (double)(i - n) * dx;
            double mu = exp(-(d * d + dy * dy) / (2 * coherence * coherence));
            sqs[(size_t)j * n + i] = cmk(mu, 0);
        }
    }
    or_fft2d(sqs, n, n, 0);
    for (size_t i = 0; i < nn; i++) {
        double s = sqs[i].re;
        if (s < 0) s = 0;
        sqs[i] = cmk(sqrt(s), 0);
    }
    double *I = (double *)malloc(sizeof(double) * nn);
    for (int j = 0; j < n; j++) {
        double y = ((double)j - (double)n / 2) * dx;
        for (int i = 0; i < n; i++) {
            double x = ((double)i - (double)n / 2) * dx;
            I[(size_t)j * n + i] = exp(-2 * (x * x + y * y) / (width * width));
        }
    }
    for (int q = 0; q < m; q++) {
        oc128 *e = out + (size_t)q * nn;
        memcpy(e, noise + (size_t)q * nn, sizeof(oc128) * nn);
        for (size_t i = 0; i < nn; i++) e[i] = cmul(e[i], sqs[i]);
        or_fft2d(e, n, n, 1);
        for (size_t i = 0; i < nn; i++) e[i] = cmul(e[i], cmk(sqrt(I[i]), 0));
    }
    free(sqs); free(I);
    return 0;
}

/* AverageIntensity (coherence.go:85-99) for scalar fields */
void or_average_intensity(const oc128 *fields, int m, int np, double *out) {
    memset(out, 0, sizeof(double) * (size_t)np);
    for (int q = 0; q < m; q++) {
        const oc128 *e = fields + (size_t)q * np;
        for (int i = 0; i < np; i++) out[i] += e[i].re * e[i].re + e[i].im * e[i].im;
    }
    double inv = 1 / (double)m;
    for (int i = 0; i < np; i++) out[i] *= inv;
}

/* ------------------------------------------------------------------ */
/* Field-level helpers (field.go)                                       */
/* ------------------------------------------------------------------ */
/* ApplyJones (field.go:109-131) */
void or_apply_jones(or_field *f, oc128 a, oc128 b, oc128 c, oc128 d) {
    size_t n = npix(f);
    if (!f->polarized) {
        if (b.re == 0 && b.im == 0 && c.re == 0 && c.im == 0 && d.re == a.re && d.im == a.im) {
            for (size_t i = 0; i < n; i++) f->ex[i] = cmul(f->ex[i], a);
            return;
        }
        f->polarized = 1;
        for (size_t i = 0; i < n; i++) {
            oc128 ex = f->ex[i];
            f->ex[i] = cmul(a, ex);
            f->ey[i] = cmul(c, ex);
        }
        return;
    }
    for (size_t i = 0; i < n; i++) {
        oc128 ex = f->ex[i], ey = f->ey[i];
        f->ex[i] = cadd(cmul(a, ex), cmul(b, ey));
        f->ey[i] = cadd(cmul(c, ex), cmul(d, ey));
    }
}

/* ScaleAmplitude (field.go:134-148) */
void or_scale_amplitude(or_field *f, oc128 s) {
    size_t n = npix(f);
    for (size_t i = 0; i < n; i++) f->ex[i] = cmul(f->ex[i], s);
    if (f->polarized)
        for (size_t i = 0; i < n; i++) f->ey[i] = cmul(f->ey[i], s);
}

/* ApplyTilt (field.go:151-168): sequential phase accumulation along each row */
void or_apply_tilt(or_field *f, double tx, double ty, double wl) {
    double k = 2 * M_PI / wl;
    double sx = sin(tx), sy = sin(ty);
    for (int j = 0; j < f->ny; j++) {
        double ph = k * (sx * fX(f, 0) + sy * fY(f, j));
        for (int i = 0; i < f->nx; i++) {
            size_t idx = (size_t)j * f->nx + i;
            f->ex[idx] = cmul(f->ex[idx], cexpi(ph));
            if (f->polarized) f->ey[idx] = cmul(f->ey[idx], cexpi(ph));
            ph += k * sx * f->dx;
        }
    }
}

/* ApplyBandlimit (field.go:264-294) */
void or_apply_bandlimit(or_field *f, double fraction, double sigma) {
    if (fraction >= 1 || fraction <= 0) return;
    double fnyq = 1 / (2 * f->dx);
    double f0 = fraction * fnyq;
    double sig = sigma * fnyq;
    if (sig <= 0) sig = fnyq * 0.01;
    for (int comp = 0; comp < (f->polarized ? 2 : 1); comp++) {
        oc128 *a = comp ? f->ey : f->ex;
        or_fft2d(a, f->ny, f->nx, 0);
        for (int j = 0; j < f->ny; j++) {
            double fy = freq_n(j, f->ny, f->dx);
            for (int i = 0; i < f->nx; i++) {
                double fx = freq_n(i, f->nx, f->dx);
                double fr = go_hypot(fx, fy);
                if (fr > f0) {
                    double d = (fr - f0) / sig;
                    size_t idx = (size_t)j * f->nx + i;
                    a[idx] = cmul(a[idx], cmk(exp(-d * d), 0));
                }
            }
        }
        or_fft2d(a, f->ny, f->nx, 1);
    }
}

/* ShiftField (field.go:199-228) */
void or_shift_field(or_field *f, double du, double dv) {
    if (du == 0 && dv == 0) return;
    for (int comp = 0; comp < (f->polarized ? 2 : 1); comp++) {
        oc128 *a = comp ? f->ey : f->ex;
        or_fft2d(a, f->ny, f->nx, 0);
        for (int j = 0; j < f->ny; j++) {
            double fy = freq_n(j, f->ny, f->dx);
            for (int i = 0; i < f->nx; i++) {
                double fx = freq_n(i, f->nx, f->dx);
                size_t idx = (size_t)j * f->nx + i;
                a[idx] = cmul(a[idx], cexpi(-2 * M_PI * (fx * du + fy * dv)));
            }
        }
        or_fft2d(a, f->ny, f->nx, 1);
    }
}

/* ------------------------------------------------------------------ */
/* Thin elements (elements.go)                                          */
/* ------------------------------------------------------------------ */
/* hashNoise01 (elements.go:710-720) */
double or_hash_noise01(long long x, long long y, long long seed) {
    uint64_t h = (uint64_t)seed * 0x9E3779B97F4A7C15ULL ^ (uint64_t)x * 0xC2B2AE3D27D4EB4FULL ^
                 (uint64_t)y * 0x165667B19E3779F9ULL;
    h ^= h >> 30;
    h *= 0xBF58476D1CE4E5B9ULL;
    h ^= h >> 27;
    h *= 0x94D049BB133111EBULL;
    h ^= h >> 31;
    return (double)(h >> 11) / (double)(1ULL << 53);
}

static inline void mul_both(or_field *f, size_t idx, oc128 t) {
    f->ex[idx] = cmul(f->ex[idx], t);
    if (f->polarized) f->ey[idx] = cmul(f->ey[idx], t);
}

/* lensEl.Apply (elements.go:195-221) */
void or_apply_lens(or_field *f, double wl, double focal, double ap, double x0, double y0) {
    double k = 2 * M_PI / wl;
    double c = -k / (2 * focal);
    for (int j = 0; j < f->ny; j++) {
        double dy = fY(f, j) - y0;
        for (int i = 0; i < f->nx; i++) {
            double dx = fX(f, i) - x0;
            double r2 = dx * dx + dy * dy;
            size_t idx = (size_t)j * f->nx + i;
            if (ap > 0 && r2 > ap * ap) {
                f->ex[idx] = cmk(0, 0);
                if (f->polarized) f->ey[idx] = cmk(0, 0);
                continue;
            }
            mul_both(f, idx, cexpi(c * r2));
        }
    }
}

/* apertureEl.Apply with the circle outline (elements.go:288-313, shape.go:163-169) */
void or_apply_aperture_circle(or_field *f, double radius, double x0, double y0, double sig) {
    for (int j = 0; j < f->ny; j++) {
        double dy = fY(f, j) - y0;
        for (int i = 0; i < f->nx; i++) {
            double dx = fX(f, i) - x0;
            double d = radius - go_hypot(dx, dy);
            oc128 t;
            if (sig > 0) t = cmk(0.5 * (1 + erf(d / (M_SQRT2 * sig))), 0);
            else t = d >= 0 ? cmk(1, 0) : cmk(0, 0);
            mul_both(f, (size_t)j * f->nx + i, t);
        }
    }
}

/* gratingEl.Apply (elements.go:488-532) */
int or_apply_grating(or_field *f, int kind, double period, double modulation, double duty,
                     double blaze_depth, double rotation, double off) {
    if (kind < 0 || kind > 4) return -1;
    double c = cos(rotation), s = sin(rotation);
    for (int j = 0; j < f->ny; j++) {
        for (int i = 0; i < f->nx; i++) {
            double uu = c * fX(f, i) + s * fY(f, j);
            double ph = 2 * M_PI * uu / period;
            oc128 t = cmk(0, 0);
            switch (kind) {
            case 0: t = cmk(0.5 * (1 + modulation * cos(ph + off)), 0); break;
            case 1: if (cos(ph + off) >= cos(M_PI * duty)) t = cmk(1, 0); break;
            case 2: t = cexpi(modulation / 2 * sin(ph + off)); break;
            case 3: t = (cos(ph + off) >= 0) ? cexpi(modulation) : cmk(1, 0); break;
            case 4: {
                double fr = fmod(uu / period, 1);
                if (fr < 0) fr += 1;
                t = cexpi(blaze_depth * fr);
            } break;
            }
            mul_both(f, (size_t)j * f->nx + i, t);
        }
    }
    return 0;
}

/* diffuserEl.Apply (elements.go:722-783) */
void or_apply_diffuser(or_field *f, double sigma, double corr, double amp, long long seed,
                       double x0, double y0) {
    size_t n = npix(f);
    double *phase = (double *)malloc(sizeof(double) * n);
    double dx = f->dx;
    if (dx <= 0) dx = 1;
    for (int j = 0; j < f->ny; j++) {
        long long gy = (long long)round((fY(f, j) + y0) / dx);
        for (int i = 0; i < f->nx; i++) {
            long long gx = (long long)round((fX(f, i) + x0) / dx);
            phase[(size_t)j * f->nx + i] = or_hash_noise01(gx, gy, seed) * 2 * M_PI - M_PI;
        }
    }
    if (corr > 0) {
        oc128 *zz = (oc128 *)malloc(sizeof(oc128) * n);
        for (size_t i = 0; i < n; i++) zz[i] = cmk(phase[i], 0);
        or_fft2d(zz, f->ny, f->nx, 0);
        for (int j = 0; j < f->ny; j++) {
            double fy = freq_n(j, f->ny, f->dx);
            for (int i = 0; i < f->nx; i++) {
                double fx = freq_n(i, f->nx, f->dx);
                double f2 = fx * fx + fy * fy;
                size_t idx = (size_t)j * f->nx + i;
                zz[idx] = cmul(zz[idx], cmk(exp(NEG_TWO_PI_SQ * corr * corr * f2), 0));
            }
        }
        or_fft2d(zz, f->ny, f->nx, 1);
        for (size_t i = 0; i < n; i++) phase[i] = zz[i].re;
        free(zz);
    }
    double m = 0, s2 = 0;
    for (size_t i = 0; i < n; i++) { m += phase[i]; s2 += phase[i] * phase[i]; }
    m /= (double)n;
    s2 = s2 / (double)n - m * m;
    if (s2 > 0) {
        double sc = sigma / sqrt(s2);
        for (size_t i = 0; i < n; i++) phase[i] = (phase[i] - m) * sc;
    }
    for (size_t i = 0; i < n; i++) mul_both(f, i, cmul(cmk(amp, 0), cexpi(phase[i])));
    free(phase);
}

/* applyMask (elements.go:128-141) with a phase-only transmission */
void or_apply_phase_mask(or_field *f, const double *phi, double amp) {
    size_t n = npix(f);
    for (size_t i = 0; i < n; i++) mul_both(f, i, cmul(cmk(amp, 0), cexpi(phi[i])));
}

/* ------------------------------------------------------------------ */
/* Inverse design: FP64 forward + adjoint of the ASM step                */
/* ------------------------------------------------------------------ */
double or_asm_phase_loss_grad(int ny, int nx, double dx, double z, const or_context *ctx,
                              const oc128 *a, const double *phi, const double *target,
                              double *grad) {
    size_t n = (size_t)ny * nx;
    oc128 *u = (oc128 *)malloc(sizeof(oc128) * n);
    oc128 *t = (oc128 *)malloc(sizeof(oc128) * n);
    for (size_t i = 0; i < n; i++) { t[i] = cexpi(phi[i]); u[i] = cmul(a[i], t[i]); }
    tf_spec tf = {0};
    tf.kind = 0; tf.wl = ctx->wavelength; tf.z = z;
    ev_policy(ctx, z, &tf.zero, &tf.reg, &tf.alpha, &tf.limit);
    transfer_arr(u, ny, nx, dx, &tf);
    double loss = 0;
    for (size_t i = 0; i < n; i++) {
        double d = cabs2(u[i]) - target[i];
        loss += d * d;
        u[i] = cmul(cmk(4 * d, 0), u[i]); /* r = dL/du* */
    }
    if (grad) {
        /* A^H = F^-1 diag(conj H) F */
        or_fft2d(u, ny, nx, 0);
        for (int j = 0; j < ny; j++) {
            double fy = freq_n(j, ny, dx);
            for (int i = 0; i < nx; i++) {
                size_t idx = (size_t)j * nx + i;
                oc128 h = tf_eval(&tf, freq_n(i, nx, dx), fy);
                h.im = -h.im;
                u[idx] = cmul(u[idx], h);
            }
        }
        or_fft2d(u, ny, nx, 1);
        for (size_t i = 0; i < n; i++) {
            /* g = Re(conj(b) * i * t * a) */
            oc128 ita = cmul(cmk(0, 1), cmul(t[i], a[i]));
            oc128 cb = cmk(u[i].re, -u[i].im);
            grad[i] = cmul(cb, ita).re;
        }
    }
    free(u); free(t);
    return loss;
}

/* ------------------------------------------------------------------ */
/* Diffractive stack: phase masks with split-step BPM segments between */
/* them (no reference counterpart).                                     */
/* ------------------------------------------------------------------ */
/* Adjoint of one Propagate(z) step of the plain ASM: F^-1 diag(conj H) F. */
static void asm_adjoint_arr(oc128 *a, int ny, int nx, double dx, double z, const or_context *ctx) {
    tf_spec tf = {0};
    tf.kind = 0; tf.wl = ctx->wavelength; tf.z = z;
    ev_policy(ctx, z, &tf.zero, &tf.reg, &tf.alpha, &tf.limit);
    or_fft2d(a, ny, nx, 0);
    for (int j = 0; j < ny; j++) {
        double fy = freq_n(j, ny, dx);
        for (int i = 0; i < nx; i++) {
            size_t idx = (size_t)j * nx + i;
            oc128 h = tf_eval(&tf, freq_n(i, nx, dx), fy);
            h.im = -h.im;
            a[idx] = cmul(a[idx], h);
        }
    }
    or_fft2d(a, ny, nx, 1);
}

/* Adjoint of splitstep_core with a parametric medium: the slices in reverse
 * order, each A(dz/2)^H M_s^H A(dz/2)^H with M_s^H = conj of the screen. */
static void splitstep_adjoint(oc128 *a, int ny, int nx, double dx, double z, const or_index_desc *d, int steps,
                              const or_context *ctx) {
    if (z == 0) return;
    if (steps <= 0) steps = 1;
    double dz = z / (double)steps;
    double k = 2 * M_PI / ctx->wavelength;
    for (int s = steps - 1; s >= 0; s--) {
        double zc = z * (double)s / (double)steps + dz / 2;
        asm_adjoint_arr(a, ny, nx, dx, dz / 2, ctx);
        for (int j = 0; j < ny; j++) {
            double y = ((double)j - (double)ny / 2) * dx;
            for (int i = 0; i < nx; i++) {
                size_t idx = (size_t)j * nx + i;
                double nr, ni;
                or_index_eval(d, ny, nx, dx, i, j, ((double)i - (double)nx / 2) * dx, y, zc, &nr, &ni);
                double ph = k * (nr - 1) * dz;
                oc128 t = cmul(cmk(exp(-k * ni * dz), 0), cexpi(-ph));
                a[idx] = cmul(a[idx], t);
            }
        }
        asm_adjoint_arr(a, ny, nx, dx, dz / 2, ctx);
    }
}

double or_bpm_stack_loss_grad(int ny, int nx, double dx, int nl, const oc128 *a, const double *phis,
                              const double *target, double zseg, int steps, const or_index_desc *d,
                              const or_context *ctx_in, double *grads) {
    size_t n = (size_t)ny * nx;
    or_context ctx = *ctx_in;
    ctx.has_warnings = 0;
    oc128 *u = (oc128 *)malloc(sizeof(oc128) * n);
    oc128 *ey = (oc128 *)calloc(n, sizeof(oc128));
    oc128 *V = (oc128 *)malloc(sizeof(oc128) * n * (size_t)(nl > 0 ? nl : 1));
    memcpy(u, a, sizeof(oc128) * n);
    or_field f = {ny, nx, dx, 0, u, ey};
    for (int l = 0; l < nl; l++) {
        const double *phi = phis + (size_t)l * n;
        for (size_t i = 0; i < n; i++) u[i] = cmul(u[i], cexpi(phi[i]));
        memcpy(V + (size_t)l * n, u, sizeof(oc128) * n);
        or_splitstep(&f, zseg, d, steps, &ctx);
    }
    double loss = 0;
    for (size_t i = 0; i < n; i++) {
        double dd = cabs2(u[i]) - target[i];
        loss += dd * dd;
        u[i] = cmul(cmk(4 * dd, 0), u[i]); /* r = dL/du* */
    }
    if (grads) {
        for (int l = nl - 1; l >= 0; l--) {
            const double *phi = phis + (size_t)l * n;
            const oc128 *v = V + (size_t)l * n;
            double *g = grads + (size_t)l * n;
            splitstep_adjoint(u, ny, nx, dx, zseg, d, steps, &ctx);
            for (size_t i = 0; i < n; i++) {
                /* g = Re(conj(b) * i * v), v = field just after mask l */
                oc128 iv = cmul(cmk(0, 1), v[i]);
                oc128 cb = cmk(u[i].re, -u[i].im);
                g[i] = cmul(cb, iv).re;
                oc128 t = cexpi(phi[i]);
                u[i] = cmul(u[i], cmk(t.re, -t.im));
            }
        }
    }
    free(u); free(ey); free(V);
    return loss;
}

/* ------------------------------------------------------------------ */
/* PropagateVectorial (vectorial.go:14-80)                              */
/* ------------------------------------------------------------------ */
int or_propagate_vectorial(or_field *f, oc128 *ez_out, double z, or_context *ctx) {
    or_context local;
    if (!ctx) { memset(&local, 0, sizeof(local)); ctx = &local; }
    int ny = f->ny, nx = f->nx;
    size_t n = npix(f);
    double wl = ctx->wavelength;
    double k = 2 * M_PI / wl;
    double az = fabs(z);
    int backward = z < 0;
    int zero, reg; double alpha, limit;
    ev_policy(ctx, z, &zero, &reg, &alpha, &limit);
    or_fft2d(f->ex, ny, nx, 0);
    or_fft2d(f->ey, ny, nx, 0);
    oc128 *ez = (oc128 *)calloc(n, sizeof(oc128));
    for (int j = 0; j < ny; j++) {
        double fy = freq_n(j, ny, f->dx);
        double ky = 2 * M_PI * fy;
        for (int i = 0; i < nx; i++) {
            double fx = freq_n(i, nx, f->dx);
            double kx = 2 * M_PI * fx;
            double rho = wl * go_hypot(fx, fy);
            size_t idx = (size_t)j * nx + i;
            oc128 H;
            oc128 ex = f->ex[idx], ey = f->ey[idx];
            /* -(kx Ex + ky Ey), the complex products with a real factor exact */
            double sr = -(kx * ex.re + ky * ey.re), si = -(kx * ex.im + ky * ey.im);
            if (rho <= 1) {
                double kz = k * sqrt((1 - rho) * (1 + rho));
                H = cexpi(kz * z);
                if (kz > 0) ez[idx] = cmk(sr / kz, si / kz);
            } else {
                double decay = k * az * sqrt((rho - 1) * (rho + 1));
                if (zero || (limit > 0 && decay > limit)) H = cmk(0, 0);
                else if (backward && reg) { double a = exp(decay); H = cmk(a / (1 + alpha * alpha * a * a), 0); }
                else if (backward) H = cmk(exp(decay), 0);
                else H = cmk(exp(-decay), 0);
                double kzi = k * sqrt((rho - 1) * (rho + 1));
                if (kzi > 0) ez[idx] = cmk(si / kzi, -sr / kzi); /* s / (i kzi) */
            }
            f->ex[idx] = cmul(f->ex[idx], H);
            f->ey[idx] = cmul(f->ey[idx], H);
            ez[idx] = cmul(ez[idx], H);
        }
    }
    or_fft2d(f->ex, ny, nx, 1);
    or_fft2d(f->ey, ny, nx, 1);
    or_fft2d(ez, ny, nx, 1);
    memcpy(ez_out, ez, sizeof(oc128) * n);
    free(ez);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Uniaxial and anisotropic media (birefringent.go:19-61, berreman.go)  */
/* ------------------------------------------------------------------ */
/* Go's complex128 division: Smith's algorithm (R. L. Smith, Algorithm 116,
 * Commun. ACM 5(8), 1962), as the Go runtime divides. */
static inline oc128 go_cdiv(oc128 n, oc128 m) {
    double e, f;
    if (fabs(m.re) >= fabs(m.im)) {
        double ratio = m.im / m.re;
        double denom = m.re + ratio * m.im;
        e = (n.re + n.im * ratio) / denom;
        f = (n.im - n.re * ratio) / denom;
    } else {
        double ratio = m.re / m.im;
        double denom = m.im + ratio * m.re;
        e = (n.re * ratio + n.im) / denom;
        f = (n.im * ratio - n.re) / denom;
    }
    return cmk(e, f);
}
static inline oc128 cneg(oc128 a) { return cmk(-a.re, -a.im); }

static void uniaxial_arr(oc128 *a, int ny, int nx, double dx, double k0, double z, double no, double ne, int extra) {
    double az = fabs(z);
    or_fft2d(a, ny, nx, 0);
    for (int j = 0; j < ny; j++) {
        double fy = freq_n(j, ny, dx);
        for (int i = 0; i < nx; i++) {
            double fx = freq_n(i, nx, dx);
            double arg;
            if (!extra) {
                arg = k0 * k0 * no * no - (2 * M_PI * fx) * (2 * M_PI * fx) - (2 * M_PI * fy) * (2 * M_PI * fy);
            } else {
                double kx = 2 * M_PI * fx, ky = 2 * M_PI * fy;
                arg = k0 * k0 * ne * ne - (ne * ne / (no * no)) * kx * kx - ky * ky;
            }
            oc128 h = arg < 0 ? cmk(exp(-az * sqrt(-arg)), 0) : cexpi(z * sqrt(arg));
            size_t idx = (size_t)j * nx + i;
            a[idx] = cmul(a[idx], h);
        }
    }
    or_fft2d(a, ny, nx, 1);
}

int or_propagate_uniaxial(or_field *f, double z, double no, double ne, const or_context *ctx) {
    if (no <= 0 || ne <= 0) return -1;
    double k0 = 2 * M_PI / ctx->wavelength;
    uniaxial_arr(f->ex, f->ny, f->nx, f->dx, k0, z, no, ne, 1);
    if (f->polarized) uniaxial_arr(f->ey, f->ny, f->nx, f->dx, k0, z, no, ne, 0);
    return 0;
}

typedef struct { oc128 m[4][4]; } m4;

static m4 berreman_matrix(const oc128 *eps, double xi, double eta) {
#define E(i, j) eps[(i) * 3 + (j)]
    oc128 one = cmk(1, 0);
    oc128 r = go_cdiv(one, E(2, 2));
    oc128 x = cmk(xi, 0), y = cmk(eta, 0);
    m4 D;
    D.m[0][0] = cmul(cmul(cneg(x), r), E(2, 0));
    D.m[0][1] = csub(one, cmul(cmul(x, x), r));
    D.m[0][2] = cmul(cmul(cneg(x), r), E(2, 1));
    D.m[0][3] = cmul(cmul(cneg(x), r), y);
    D.m[1][0] = csub(csub(E(0, 0), cmul(y, y)), cmul(cmul(E(0, 2), r), E(2, 0)));
    D.m[1][1] = cmul(cmul(cneg(E(0, 2)), r), x);
    D.m[1][2] = csub(cadd(E(0, 1), cmul(y, x)), cmul(cmul(E(0, 2), r), E(2, 1)));
    D.m[1][3] = cmul(cmul(cneg(E(0, 2)), r), y);
    D.m[2][0] = cmul(cmul(cneg(y), r), E(2, 0));
    D.m[2][1] = cmul(cmul(cneg(y), r), x);
    D.m[2][2] = cmul(cmul(cneg(y), r), E(2, 1));
    D.m[2][3] = csub(one, cmul(cmul(y, y), r));
    D.m[3][0] = csub(cadd(E(1, 0), cmul(x, y)), cmul(cmul(E(1, 2), r), E(2, 0)));
    D.m[3][1] = cmul(cmul(cneg(E(1, 2)), r), x);
    D.m[3][2] = csub(csub(E(1, 1), cmul(x, x)), cmul(cmul(E(1, 2), r), E(2, 1)));
    D.m[3][3] = cmul(cmul(cneg(E(1, 2)), r), y);
#undef E
    return D;
}

static oc128 trace4m(const m4 *A) {
    return cadd(cadd(cadd(A->m[0][0], A->m[1][1]), A->m[2][2]), A->m[3][3]);
}
/* A (B + c I): the identity scaled by c is complex(0,0)*c off the diagonal */
static m4 mul_shift(const m4 *A, const m4 *B, oc128 c) {
    m4 S, out;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) S.m[i][j] = cadd(B->m[i][j], cmul(cmk(i == j ? 1 : 0, 0), c));
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            oc128 s = cmk(0, 0);
            for (int k = 0; k < 4; k++) s = cadd(s, cmul(A->m[i][k], S.m[k][j]));
            out.m[i][j] = s;
        }
    return out;
}
/* Faddeev-LeVerrier (berreman.go:130-144) */
static void char_poly4(const m4 *A, oc128 *c) {
    m4 B = *A;
    c[3] = cneg(trace4m(&B));
    B = mul_shift(A, &B, c[3]);
    c[2] = go_cdiv(cneg(trace4m(&B)), cmk(2, 0));
    B = mul_shift(A, &B, c[2]);
    c[1] = go_cdiv(cneg(trace4m(&B)), cmk(3, 0));
    B = mul_shift(A, &B, c[1]);
    c[0] = go_cdiv(cneg(trace4m(&B)), cmk(4, 0));
}
static oc128 poly4(oc128 z, const oc128 *c) {
    oc128 z2 = cmul(z, z);
    oc128 t = cmul(cmul(z2, z), z);
    t = cadd(t, cmul(cmul(cmul(c[3], z), z), z));
    t = cadd(t, cmul(cmul(c[2], z), z));
    t = cadd(t, cmul(c[1], z));
    return cadd(t, c[0]);
}
/* Durand-Kerner (berreman.go:186-214) */
static void roots4(const oc128 *c, oc128 *z) {
    z[0] = cmk(0.4, 0.9); z[1] = cmk(0.4, -0.9); z[2] = cmk(-0.4, 0.9); z[3] = cmk(-0.4, -0.9);
    for (int iter = 0; iter < 300; iter++) {
        double maxd = 0;
        for (int i = 0; i < 4; i++) {
            oc128 num = poly4(z[i], c);
            oc128 den = cmk(1, 0);
            for (int j = 0; j < 4; j++)
                if (j != i) den = cmul(den, csub(z[i], z[j]));
            oc128 dz = go_cdiv(num, den);
            z[i] = csub(z[i], dz);
            double d = go_hypot(dz.re, dz.im);
            if (d > maxd) maxd = d;
        }
        if (maxd < 1e-14) break;
    }
}
static int forward_mode(oc128 q) {
    if (q.im > 1e-12) return 1;
    if (q.im < -1e-12) return 0;
    return q.re > 0;
}
static oc128 det3(oc128 m[3][3]) {
    oc128 a = cmul(m[0][0], csub(cmul(m[1][1], m[2][2]), cmul(m[1][2], m[2][1])));
    oc128 b = cmul(m[0][1], csub(cmul(m[1][0], m[2][2]), cmul(m[1][2], m[2][0])));
    oc128 c = cmul(m[0][2], csub(cmul(m[1][0], m[2][1]), cmul(m[1][1], m[2][0])));
    return cadd(csub(a, b), c);
}
/* largest-norm column of adj(A - qI) (berreman.go:228-272) */
static void null_vector4(const m4 *A, oc128 q, oc128 *best) {
    m4 M = *A;
    for (int i = 0; i < 4; i++) M.m[i][i] = csub(M.m[i][i], q);
    double bestn = -1;
    for (int col = 0; col < 4; col++) {
        oc128 v[4];
        for (int row = 0; row < 4; row++) {
            oc128 m[3][3];
            int ri = 0;
            for (int r = 0; r < 4; r++) {
                if (r == row) continue;
                int ci = 0;
                for (int cc = 0; cc < 4; cc++) {
                    if (cc == col) continue;
                    m[ri][ci++] = M.m[r][cc];
                }
                ri++;
            }
            oc128 cof = det3(m);
            if ((row + col) % 2 == 1) cof = cneg(cof);
            v[row] = cof;
        }
        double nn = 0;
        for (int t = 0; t < 4; t++) nn += v[t].re * v[t].re + v[t].im * v[t].im;
        if (nn > bestn) {
            bestn = nn;
            for (int t = 0; t < 4; t++) best[t] = v[t];
        }
    }
}
/* anisoMode (berreman.go:41-92) */
static void aniso_mode(const oc128 *eps, double xi, double eta, double k0, double z, oc128 *ex, oc128 *ey) {
    m4 D = berreman_matrix(eps, xi, eta);
    oc128 c[4], roots[4], qs[2], vs[2][4];
    char_poly4(&D, c);
    roots4(c, roots);
    int cnt = 0, used[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++)
        if (forward_mode(roots[i]) && cnt < 2) {
            qs[cnt] = roots[i];
            null_vector4(&D, roots[i], vs[cnt]);
            used[i] = 1;
            cnt++;
        }
    while (cnt < 2) {
        double best = -1e300;
        int bi = -1;
        for (int i = 0; i < 4; i++)
            if (!used[i] && roots[i].re > best) { best = roots[i].re; bi = i; }
        if (bi < 0) break;
        qs[cnt] = roots[bi];
        null_vector4(&D, roots[bi], vs[cnt]);
        used[bi] = 1;
        cnt++;
    }
    oc128 a = vs[0][0], b = vs[1][0], cc = vs[0][2], d = vs[1][2];
    oc128 det = csub(cmul(a, d), cmul(b, cc));
    oc128 m1 = go_cdiv(csub(cmul(d, *ex), cmul(b, *ey)), det);
    oc128 m2 = go_cdiv(cadd(cmul(cneg(cc), *ex), cmul(a, *ey)), det);
    oc128 p0 = cmul(cexpi(k0 * qs[0].re * z), cmk(exp(-k0 * qs[0].im * z), 0));
    oc128 p1 = cmul(cexpi(k0 * qs[1].re * z), cmk(exp(-k0 * qs[1].im * z), 0));
    *ex = cadd(cmul(cmul(m1, p0), a), cmul(cmul(m2, p1), b));
    *ey = cadd(cmul(cmul(m1, p0), cc), cmul(cmul(m2, p1), d));
}

int or_propagate_anisotropic(or_field *f, double z, const oc128 *eps, const or_context *ctx) {
    int ny = f->ny, nx = f->nx;
    double k0 = 2 * M_PI / ctx->wavelength;
    or_fft2d(f->ex, ny, nx, 0);
    or_fft2d(f->ey, ny, nx, 0);
    for (int j = 0; j < ny; j++) {
        double fy = freq_n(j, ny, f->dx);
        double ky = 2 * M_PI * fy;
        for (int i = 0; i < nx; i++) {
            double fx = freq_n(i, nx, f->dx);
            double kx = 2 * M_PI * fx;
            size_t idx = (size_t)j * nx + i;
            aniso_mode(eps, kx / k0, ky / k0, k0, z, &f->ex[idx], &f->ey[idx]);
        }
    }
    or_fft2d(f->ex, ny, nx, 1);
    or_fft2d(f->ey, ny, nx, 1);
    return 0;
}

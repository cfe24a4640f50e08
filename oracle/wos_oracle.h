/*
 * wos_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the Tetsuhiro-WOS propagation hot path (Go package
 * `optics`), used as the parity oracle by tests/, by __graft_entry__.smoke()
 * and by the CPU-baseline leg of bench.py.  It is never linked into, called by
 * or shipped with the product library (libwosgpu.so).
 *
 * Every function names the reference file:line it restates.  Grids are
 * generalised from the reference's square N x N to ny rows x nx columns by
 * applying each 1-D rule per axis; for ny == nx the arithmetic is the
 * reference's, operation for operation (radix-2 DIT order, twiddle table,
 * Bluestein chirp, complex multiply (ac-bd, ad+bc), no FMA contraction).
 *
 * Parity of this file is pinned by the reference's own known-answer tests
 * (the optics package test files), ported in tests/test_oracle_kat.py.
 */
#ifndef WOS_ORACLE_H
#define WOS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } oc128;

/* Method ids: identical to the product's wos_method enum. */
enum {
    OR_ASM = 1, OR_ASM_PAD = 2, OR_ASM_SHIFT = 3, OR_ASM_SHIFT_PAD = 4,
    OR_FRESNEL_TF = 5, OR_FRESNEL_IR = 6, OR_FRAUNHOFER = 7
};

typedef struct {
    char code[32];
    int count;
    double value;
} or_warning;

/* optics.Context (field.go:237-254) plus its Warnings list. */
typedef struct {
    double wavelength;
    int evanescent_zero;        /* Evanescent == "zero" */
    double evanescent_limit;    /* nepers, 0 = off */
    int backward_regularize;
    double tikhonov_alpha;      /* <= 0 -> 1e-3 */
    int has_warnings;           /* Warnings != nil */
    int n_warn;
    or_warning warn[16];
} or_context;

/* optics.Field (field.go:14-22), generalised to ny x nx. */
typedef struct {
    int ny, nx;
    double dx;
    int polarized;
    oc128 *ex;
    oc128 *ey;
} or_field;

/* Parametric refractive index n(x,y,z), shared with the product ABI
 * (wos_index_desc).  Re n = re0(z) + core_dn*exp(-((x-x0)^2+(y-y0)^2)/w^2)
 *                           * (1 + zmod_amp*sin(2*pi*z/zmod_period + zmod_phase))
 * Im n = im0(z) + border_strength*((border_px - d)/border_px)^border_order
 *        for pixel distance d < border_px from the nearest window edge.
 * re0(z), im0(z): layer k applies for z < layer_z[k] (first match), else
 * (re_bg, im_bg). */
typedef struct {
    double re_bg, im_bg;
    double core_dn, core_x0, core_y0, core_w;
    double zmod_amp, zmod_period, zmod_phase;
    int border_px;
    int border_order;
    double border_strength;
    int n_layers;
    double layer_z[8];
    double layer_re[8];
    double layer_im[8];
} or_index_desc;

/* threads used by parFor (fft.go:91-122); default = online CPUs */
void or_set_threads(int p);
int or_get_threads(void);

/* ---- FFT core (optics/fft.go) ---- */
void or_fft1d(oc128 *a, int n, int inverse);               /* fft1DAnyCPU fft.go:146-153 */
void or_fft1d_pow2(oc128 *a, int n, int inverse);          /* fft1D fft.go:55-87 */
void or_bluestein(oc128 *a, int n, int inverse);           /* fft1DBluestein fft.go:159-204 */
void or_fft2d(oc128 *a, int ny, int nx, int inverse);      /* fft2DCPU fft.go:219-242 */

/* ---- field helpers (optics/field.go) ---- */
double or_power(const or_field *f);                        /* field.go:77-83 */
double or_rms_radius(const or_field *f);                   /* propagate.go:105-130 */
double or_spectral_radius(const or_field *f, double frac); /* propagate.go:270-320 */
void or_spectral_centroid(const or_field *f, double *fx, double *fy); /* propagate.go:391-416 */
void or_apply_jones(or_field *f, oc128 a, oc128 b, oc128 c, oc128 d); /* field.go:109-131 */
void or_scale_amplitude(or_field *f, oc128 s);             /* field.go:134-148 */
void or_apply_tilt(or_field *f, double tx, double ty, double wl); /* field.go:151-168 */
void or_apply_bandlimit(or_field *f, double fraction, double sigma); /* field.go:264-294 */
void or_shift_field(or_field *f, double du, double dv);    /* field.go:199-228 */

/* ---- propagation (optics/propagate.go) ---- */
int or_propagate(or_field *f, double z, int method, or_context *ctx); /* propagate.go:65-102 */
int or_propagate_shift_at(or_field *f, double z, int method, or_context *ctx, double fxc, double fyc);
int or_propagate1d(oc128 *a, int n, double dx, double z, double wl, or_context *ctx); /* :718-738 */
/* PropagateVectorial (vectorial.go:14-80): ex and ey (both used whatever
 * f->polarized, as the reference uses f.Ey) propagate in place, ez_out
 * receives the reconstructed longitudinal component. */
int or_propagate_vectorial(or_field *f, oc128 *ez_out, double z, or_context *ctx);
/* PropagateUniaxial (birefringent.go:19-61): Ex extraordinary, Ey ordinary (if polarized). */
int or_propagate_uniaxial(or_field *f, double z, double no, double ne, const or_context *ctx);
/* PropagateAnisotropic (berreman.go:13-36): eps row-major 3x3; Ex and Ey both used. */
int or_propagate_anisotropic(or_field *f, double z, const oc128 *eps, const or_context *ctx);
/* asmTF (propagate.go:159-181) evaluated at (fx, fy) with the policy of ctx */
oc128 or_asm_tf(double wl, double z, int zero_ev, int reg, double alpha, double limit,
                double fx, double fy);

/* ---- split-step BPM (optics/medium.go) ---- */
void or_index_eval(const or_index_desc *d, int ny, int nx, double dx, int i, int j,
                   double x, double y, double z, double *re, double *im);
int or_splitstep(or_field *f, double z, const or_index_desc *d, int steps, or_context *ctx);
/* generic: n(x,y,z) sampled per slice into caller arrays via callback */
typedef void (*or_index_fn)(double x, double y, double z, void *user, double *re, double *im);
int or_splitstep_fn(or_field *f, double z, or_index_fn fn, void *user, int steps, or_context *ctx);

/* ---- batches ---- */
/* polychromatic.go:18-44; out[ny*nx] */
int or_polychromatic(const or_field *f, double z, const double *wl, const double *weight, int ns,
                     int method, or_context *base, double *out);
/* volume.go:8-18; out = nz * ncomp * ny*nx (ncomp = 1 + polarized) */
int or_propagate3d(const or_field *f, const double *zs, int nz, int method, or_context *ctx,
                   oc128 *out);
/* coherence.go:22-80 with caller-supplied complex noise (m * n*n values that
 * replace complex(rng.NormFloat64()/sqrt2, rng.NormFloat64()/sqrt2)) */
int or_schell_realizations(int n, double dx, double width, double coherence, int m,
                           const oc128 *noise, oc128 *out);
/* coherence.go:85-99 */
void or_average_intensity(const oc128 *fields, int m, int npix, double *out);

/* ---- thin elements (optics/elements.go) ---- */
double or_hash_noise01(long long x, long long y, long long seed);  /* elements.go:710-720 */
void or_apply_lens(or_field *f, double wl, double focal, double aperture, double x0, double y0); /* :195-221 */
void or_apply_aperture_circle(or_field *f, double radius, double x0, double y0, double edge_sigma); /* :288-313 */
/* kind: 0 amplitude_sin, 1 amplitude_binary, 2 phase_sin, 3 phase_binary, 4 blazed (:488-532) */
int or_apply_grating(or_field *f, int kind, double period, double modulation, double duty,
                     double blaze_depth, double rotation, double offset);
void or_apply_diffuser(or_field *f, double sigma, double corr, double amp, long long seed,
                       double x0, double y0);  /* :722-783 */
/* phase-only mask t = amp * exp(i*phi[j*nx+i]) (applyMask, :128-141) */
void or_apply_phase_mask(or_field *f, const double *phi, double amp);

/* ---- inverse design (FP64 forward + adjoint, no reference counterpart) ----
 * u = ASM_z(a * exp(i phi)); L = sum (|u|^2 - T)^2; grad = dL/dphi. */
double or_asm_phase_loss_grad(int ny, int nx, double dx, double z, const or_context *ctx,
                              const oc128 *a, const double *phi, const double *target,
                              double *grad /* may be NULL */);

/* Diffractive stack: u_0 = a; for each layer l: u = BPM_zseg(u * exp(i phi_l))
 * (split-step, `steps` slices, parametric medium d); L = sum (|u|^2 - T)^2;
 * grads[l] = dL/dphi_l by the exact adjoint (conj transfer functions and
 * screens, slices in reverse order). */
double or_bpm_stack_loss_grad(int ny, int nx, double dx, int nl, const oc128 *a, const double *phis,
                              const double *target, double zseg, int steps, const or_index_desc *d,
                              const or_context *ctx, double *grads /* may be NULL */);

#ifdef __cplusplus
}
#endif
#endif

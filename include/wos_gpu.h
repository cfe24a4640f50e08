/*
 * wos_gpu.h -- C ABI of libwosgpu.so, the B200 (sm_100a) propagation backend
 * for the Tetsuhiro-WOS `optics` package.
 *
 * The reference's GPU seam is per FFT: fft2D / fft1DAny call gpuFFT2D /
 * gpuFFT1D (optics/fft.go:135-142,209-216), which copy the whole array to the
 * device and back around one cuFFT Z2Z call (optics/gpu.go:173-207).  This
 * library moves the seam up to the propagation call itself: one entry point
 * per reference function of the hot path, each crossing PCIe once per field.
 *
 * Conventions
 *  - All signatures are plain C: pointers, sizes, doubles, ints.
 *  - A field component is row-major ny x nx (index y*nx + x), exactly the Go
 *    Field.Ex / Field.Ey layout (optics/field.go:14-22) with ny = nx = N.
 *    Host buffers are complex128 (wos_c128 = Go complex128 = C double _Complex).
 *  - Device-resident entry points (suffix _dev) take device pointers whose
 *    element type is the context precision: complex64 (float2) for WOS_FP32,
 *    complex128 (double2) for WOS_FP64.
 *  - Every call returns a wos_status; on failure wos_last_error() returns a
 *    thread-local message.  There is no CPU fallback: an error is reported to
 *    the caller, never hidden.
 *  - A context owns one CUDA stream, its device workspace and its plans.  It
 *    may be used by one host thread at a time (calls serialise on an internal
 *    lock); use one context per concurrent caller.
 */
#ifndef WOS_GPU_H
#define WOS_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WOS_ABI_VERSION 1

#if defined(__GNUC__)
#define WOS_API __attribute__((visibility("default")))
#else
#define WOS_API
#endif

typedef struct { double re, im; } wos_c128;
typedef struct wos_ctx_s* wos_ctx;
typedef struct wos_graph_s* wos_graph;

/* Status codes (replace the cufftResult / cudaError_t strings of optics/gpu.go:51-79). */
enum wos_status {
    WOS_OK = 0,
    WOS_INVALID_ARG = 1,
    WOS_UNSUPPORTED_SIZE = 2,
    WOS_OOM = 3,
    WOS_CUDA_ERROR = 4,
    WOS_TIMEOUT = 5,
    WOS_NOT_INITIALISED = 6,
    WOS_UNKNOWN_METHOD = 7
};

/* Method ids: the Method constants of optics/propagate.go:40-50. */
enum wos_method {
    WOS_ASM = 1,
    WOS_ASM_PAD = 2,
    WOS_ASM_SHIFT = 3,
    WOS_ASM_SHIFT_PAD = 4,
    WOS_FRESNEL_TF = 5,
    WOS_FRESNEL_IR = 6,
    WOS_FRAUNHOFER = 7
};

enum wos_precision { WOS_FP64 = 0, WOS_FP32 = 1 };

/* Warning bits: the Warnings.Add codes of the hot path (optics/propagate.go:203-264,515,586,654). */
enum wos_warn_bit {
    WOS_W_EVANESCENT_FILTERED = 0,
    WOS_W_BACKWARD_REGULARIZED = 1,
    WOS_W_BACKWARD_EVANESCENT = 2,
    WOS_W_ASM_ALIAS_WRAP = 3,
    WOS_W_FRESNEL_TF_ALIAS = 4,
    WOS_W_FRESNEL_IR_ALIAS = 5,
    WOS_W_FRAUNHOFER_NEARFIELD = 6,
    WOS_W_COUNT = 7
};

/* optics.Context (optics/field.go:237-254), the fields the hot path reads. */
typedef struct {
    double wavelength;        /* m */
    int evanescent_zero;      /* Evanescent == "zero" */
    double evanescent_limit;  /* nepers, 0 = off */
    int backward_regularize;  /* BackwardRegularize */
    double tikhonov_alpha;    /* <= 0 -> 1e-3 */
    int diagnostics;          /* 1 when ctx.Warnings != nil: compute what the warnings need */
} wos_context;

/* Scalars behind the reference's warnings, plus the warnings themselves
 * (count and value per code, as Warnings.Add would record them). */
typedef struct {
    double p_in, p_out;           /* Field.Power() before / after (W), compensated FP64 sums */
    double centroid_fx, centroid_fy; /* spectral centroid (asm_shift*), 1/m */
    int carrier_applied;          /* 1 when the carrier shift branch ran */
    int wrap_checked;             /* 1 when spectralRadius ran */
    double spectral_radius;       /* f_sig: 90 % spectral power radius, 1/m */
    double rms_radius_in;         /* fraunhofer input support D, m */
    double dx_out;                /* output pixel pitch (fraunhofer changes it), m */
    int warn_count[WOS_W_COUNT];
    double warn_value[WOS_W_COUNT];
} wos_diag;

/* Host field: optics.Field (optics/field.go:14-22), generalised to ny x nx. */
typedef struct {
    int ny, nx;
    double dx;
    int polarized;       /* 1: ey is propagated too */
    wos_c128* ex;
    wos_c128* ey;
} wos_field;

/* Parametric refractive index n(x,y,z) of a split-step medium (the IndexFunc
 * closure of optics/medium.go:8 cannot cross the ABI; this descriptor covers
 * uniform, stratified, graded-core, z-modulated and absorbing-border media):
 *   Re n = re0(z) + core_dn * exp(-((x-x0)^2+(y-y0)^2)/core_w^2)
 *                 * (1 + zmod_amp * sin(2 pi z / zmod_period + zmod_phase))
 *   Im n = im0(z) + border_strength * ((border_px - d)/border_px)^border_order, d < border_px
 * where d is the pixel distance to the nearest window edge and (re0, im0)(z)
 * is layer k for the first k with z < layer_z[k], else (re_bg, im_bg). */
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
} wos_index_desc;

/* ---- device and context (replaces gpuInit / GPUAvailable / GPUBackendInfo,
 *      optics/gpu.go:106-143) ---- */
WOS_API int wos_device_count(void);
WOS_API int wos_device_name(int device, char* buf, int buflen);
WOS_API int wos_ctx_create(int device, int precision, wos_ctx* out);
WOS_API int wos_ctx_destroy(wos_ctx ctx);
/* Use the caller's CUDA stream (cudaStream_t) instead of the context's own. */
WOS_API int wos_ctx_set_stream(wos_ctx ctx, void* stream);
WOS_API void* wos_ctx_get_stream(wos_ctx ctx);
WOS_API int wos_ctx_precision(wos_ctx ctx);
/* Columns per CTA of the fused column pass (power of two; 0 = automatic). */
WOS_API int wos_ctx_set_col_width(wos_ctx ctx, int w);
WOS_API int wos_ctx_synchronize(wos_ctx ctx);
/* Per-launch CUDA-event profile on the context stream (no counterpart in the
 * reference, whose only timers are Result.ElapsedMS and Go benchmarks).
 * kind: 0 row forward, 1 row inverse, 2 row inverse.screen.forward,
 * 3 row inverse.accumulate, 4 column fused (FFT.H.IFFT), 5 column Fraunhofer,
 * 6 column reduction, 7 column FFT.  Reading synchronises outstanding events. */
WOS_API int wos_ctx_set_profiling(wos_ctx ctx, int on);
WOS_API int wos_ctx_profile(wos_ctx ctx, int kind, double* total_ms, long long* launches);
WOS_API int wos_ctx_profile_reset(wos_ctx ctx);
/* Number of sweep kernels this context has launched since the last reset. */
WOS_API long long wos_ctx_launch_count(wos_ctx ctx);
/* Sweep selection for the power-of-two ASM path, all computing the same
 * transform: 1 (default) the specialised sweeps, the column sweep (and the
 * FP64 row sweep) as persistent TMA-pipelined kernels where the layout and
 * shared memory allow; 3 both row and column sweeps pipelined; 2 the
 * specialised one-shot kernels only; 0 the general sweeps.  The pipelined kernels bound every wait on a copy; a wait
 * that expired is reported as WOS_TIMEOUT by the next call that synchronises
 * (host-buffer entry points, wos_ctx_synchronize). */
WOS_API int wos_ctx_set_fast_path(wos_ctx ctx, int enabled);
/* Autotuner of the specialised sweeps (no counterpart in the reference): times
 * every (row elements/thread, column elements/thread, columns/CTA) launch
 * configuration for an ny x nx grid on this device (best of three rounds of
 * ten propagations each) and keeps the fastest for the context, or the
 * default unless another is more than 2 % faster; *col_w reports the width the
 * ASM column sweep runs with (4 when complex64 uses the tiled intermediate).
 * wos_ctx_set_tune installs a configuration from a cache. */
WOS_API int wos_autotune(wos_ctx ctx, int ny, int nx, int* row_e, int* col_e, int* col_w);
WOS_API int wos_ctx_set_tune(wos_ctx ctx, int ny, int nx, int row_e, int col_e, int col_w);
WOS_API const char* wos_status_string(int status);
WOS_API const char* wos_last_error(void);
WOS_API const char* wos_backend_info(void);

/* ---- FFT users outside the propagators (fft2D / fft1DAny callers,
 *      optics/fft.go:135-142,209-216; gpuFFT2D / gpuFFT1D, optics/gpu.go:275-304).
 *      Host complex128 in place; inverse scales by 1/n per axis like fft1D. ---- */
WOS_API int wos_fft2d(wos_ctx ctx, int ny, int nx, wos_c128* a, int inverse);
WOS_API int wos_fft1d(wos_ctx ctx, int n, wos_c128* a, int inverse);
WOS_API int wos_fft2d_dev(wos_ctx ctx, int ny, int nx, int batch, void* a, int inverse);

/* ---- Propagate (optics/propagate.go:65-102): the host Field in place. ---- */
WOS_API int wos_propagate(wos_ctx ctx, wos_field* f, double z, int method, const wos_context* c,
                  wos_diag* diag /* may be NULL */);
/* A batch of host fields (each as wos_propagate, in place; diags may be NULL,
 * else one per field).  Uploads, sweeps and downloads of consecutive fields
 * overlap (separate copy streams, three device staging slots), so with
 * page-locked host buffers a field costs about one PCIe direction instead of
 * both.  No counterpart in the reference (one field per call). */
WOS_API int wos_propagate_batch(wos_ctx ctx, int nfields, wos_field* fields, double z, int method,
                                const wos_context* c, wos_diag* diags);

/* Device-resident variant: in/out hold ncomp components [ncomp][ny][nx] in the
 * context precision; in == out is allowed.  dx_out returns the output pitch
 * through diag. */
WOS_API int wos_propagate_dev(wos_ctx ctx, int ny, int nx, double dx, int ncomp, const void* in, void* out,
                      double z, int method, const wos_context* c, wos_diag* diag);

/* Device-resident variant with complex128 device I/O in either precision
 * (the FP32 pipeline converts inside its first and last sweep). */
WOS_API int wos_propagate_dev_c128(wos_ctx ctx, int ny, int nx, double dx, int ncomp, const void* in,
                           void* out, double z, int method, const wos_context* c, wos_diag* diag);
/* A batch of independent device fields propagated with the same geometry and
 * settings (in[i] -> out[i], each as wos_propagate_dev without diagnostics).
 * On the power-of-two ASM path the fields run concurrently on streams forked
 * from the context stream and joined back into it, so the kernels of one
 * field fill the SMs that another leaves idle; otherwise they run in order.
 * No counterpart in the reference (which propagates one field per call). */
WOS_API int wos_propagate_batch_dev(wos_ctx ctx, int nfields, int ny, int nx, double dx, int ncomp,
                                    const void* const* in, void* const* out, double z, int method,
                                    const wos_context* c);

/* ---- PropagateSplitStep (optics/medium.go:22-45) with a parametric medium.
 *      diag receives the powers and warnings only when c->diagnostics is set
 *      (a Context with Warnings); otherwise it is zeroed apart from dx_out and
 *      the slices take the specialised power-of-two sweeps where they apply. ---- */
WOS_API int wos_splitstep(wos_ctx ctx, wos_field* f, double z, const wos_index_desc* n, int steps,
                  const wos_context* c, wos_diag* diag);
WOS_API int wos_splitstep_dev(wos_ctx ctx, int ny, int nx, double dx, int ncomp, void* field, double z,
                      const wos_index_desc* n, int steps, const wos_context* c, wos_diag* diag);
/* Sampled medium: n_re / n_im are host FP64 maps [nmaps][ny][nx]; nmaps == 1
 * for a z-independent medium, else nmaps == steps (slice s uses map s). */
WOS_API int wos_splitstep_maps(wos_ctx ctx, wos_field* f, double z, const double* n_re, const double* n_im,
                       int nmaps, int steps, const wos_context* c, wos_diag* diag);

/* ---- PropagatePolychromatic (optics/polychromatic.go:18-44): out[ny*nx] FP64
 *      intensity sum_k weight_k |U_k|^2; the input field is not modified.
 *      The batch entry points accumulate the warnings of every unit into diag
 *      (the reference's shared ctx.Warnings). ---- */
WOS_API int wos_polychromatic(wos_ctx ctx, const wos_field* f, double z, const double* wavelengths,
                      const double* weights, int nsamples, int method, const wos_context* base,
                      double* out, wos_diag* diag /* may be NULL */);

/* ---- Propagate3D (optics/volume.go:8-18): out = nz * ncomp * ny*nx complex128,
 *      plane q is the input propagated to zs[q] (zs[q] == 0 copies the input). ---- */
WOS_API int wos_volume(wos_ctx ctx, const wos_field* f, const double* zs, int nz, int method,
               const wos_context* c, wos_c128* out, wos_diag* diag);

/* ---- GenerateSchellRealizations + PropagatePartiallyCoherent + AverageIntensity
 *      (optics/coherence.go:22-116).  noise holds m*n*n complex values that take
 *      the place of complex(rng.NormFloat64(), rng.NormFloat64())/sqrt2. ---- */
WOS_API int wos_schell_modes(wos_ctx ctx, int n, double dx, double width, double coherence, int m,
                     const wos_c128* noise, wos_c128* modes_out);
WOS_API int wos_partially_coherent(wos_ctx ctx, int n, double dx, double width, double coherence, int m,
                           const wos_c128* noise, double z, int method, const wos_context* c,
                           double* out, wos_diag* diag);

/* ---- device-resident batches: the forms of wos_polychromatic, wos_volume and
 *      wos_partially_coherent for callers that keep fields on the GPU (no
 *      counterpart in the reference, whose loops at optics/polychromatic.go:29-42,
 *      optics/volume.go:10-16 and optics/coherence.go:110-115 they replace).
 *      Method WOS_ASM, no diagnostics; fields of the context's complex type,
 *      intensities FP64.  The wavelength, distance and weight lists are host
 *      arrays, copied to the device only when they differ from an earlier
 *      call's, and nothing synchronises the host: after a first call with the
 *      same geometry and lists, a call can be recorded between
 *      wos_graph_capture_begin and _end.  The units of one call share the row
 *      spectrum of the input and run in one column launch (gridDim.y = units)
 *      and one row launch per chunk of up to 4 GiB of spectra. ---- */
/* out: device FP64 [ny][nx], overwritten with sum_k weights[k] |U_k|^2 over
 * the components of field (device [ncomp][ny][nx]). */
WOS_API int wos_polychromatic_dev(wos_ctx ctx, int ny, int nx, double dx, int ncomp, const void* field, double z,
                                  const double* wavelengths, const double* weights, int nsamples,
                                  const wos_context* base, double* out);
/* out: device [nz][ncomp][ny][nx] of the context's complex type; plane q is the
 * field propagated to zs[q] (zs[q] == 0 copies the field). */
WOS_API int wos_volume_dev(wos_ctx ctx, int ny, int nx, double dx, int ncomp, const void* field, const double* zs,
                           int nz, const wos_context* c, void* out);
/* noise: device complex128 [m][n][n] (the place of Go's math/rand draws, as in
 * wos_partially_coherent); out: device FP64 [n][n], the mean of |U_k|^2. */
WOS_API int wos_partially_coherent_dev(wos_ctx ctx, int n, double dx, double width, double coherence, int m,
                                       const void* noise, double z, const wos_context* c, double* out);

/* ---- batches sharded over GPUs (no counterpart in the reference, whose loops
 *      at optics/polychromatic.go:29-42, optics/coherence.go:110-115 and
 *      optics/volume.go:10-16 run their units in sequence).  One process or
 *      thread per GPU, each with its own context; rank 0 makes an id with
 *      wos_comm_unique_id and hands it to the others out of band, and every
 *      rank calls wos_comm_init with it (NCCL, loaded at the first call; a
 *      collective: all ranks must call it).  The sharded calls are
 *      collectives too: every rank passes the whole unit list and its own
 *      device buffers, runs the contiguous share wos_shard_range gives it,
 *      and receives the whole result (an FP64 all-reduce of the intensity, or
 *      a broadcast of each rank's planes) on the context stream. ---- */
#define WOS_COMM_ID_BYTES 128
WOS_API int wos_comm_unique_id(unsigned char* id /* [WOS_COMM_ID_BYTES] */);
WOS_API int wos_comm_init(wos_ctx ctx, int nranks, int rank, const unsigned char* id);
WOS_API int wos_comm_destroy(wos_ctx ctx);
/* Units [*begin, *end) of rank `rank` among nranks: contiguous, the first
 * units % nranks ranks one unit more (host only, needs no GPU). */
WOS_API int wos_shard_range(int units, int nranks, int rank, int* begin, int* end);
WOS_API int wos_polychromatic_sharded_dev(wos_ctx ctx, int ny, int nx, double dx, int ncomp, const void* field,
                                          double z, const double* wavelengths, const double* weights, int nsamples,
                                          const wos_context* base, double* out);
WOS_API int wos_partially_coherent_sharded_dev(wos_ctx ctx, int n, double dx, double width, double coherence, int m,
                                               const void* noise, double z, const wos_context* c, double* out);
WOS_API int wos_volume_sharded_dev(wos_ctx ctx, int ny, int nx, double dx, int ncomp, const void* field,
                                   const double* zs, int nz, const wos_context* c, void* out);

/* ---- thin-element multiply (optics/elements.go:128-141,195-221,288-313,488-532). ---- */
WOS_API int wos_apply_lens(wos_ctx ctx, wos_field* f, double wavelength, double focal, double aperture,
                   double x0, double y0);
WOS_API int wos_apply_aperture_circle(wos_ctx ctx, wos_field* f, double radius, double x0, double y0,
                              double edge_sigma);
/* kind: 0 amplitude_sin, 1 amplitude_binary, 2 phase_sin, 3 phase_binary, 4 blazed */
WOS_API int wos_apply_grating(wos_ctx ctx, wos_field* f, int kind, double period, double modulation,
                      double duty, double blaze_depth, double rotation, double offset);
WOS_API int wos_apply_phase_mask(wos_ctx ctx, wos_field* f, const double* phi, double amp);

/* ---- field operations (optics/field.go:109-168,199-228,264-294), host Field in
 *      place.  Element arithmetic is FP64 whatever the context precision; the
 *      FFT filters (bandlimit, shift, diffuser correlation) run in it. ---- */
/* Field.ApplyJones (field.go:109-131): [[a b] [c d]] at every pixel.  A scalar
 * field with a non-diagonal or non-uniform matrix becomes polarized (Ey = c Ex;
 * f->ey must hold ny*nx elements and f->polarized is set to 1). */
WOS_API int wos_apply_jones(wos_ctx ctx, wos_field* f, wos_c128 a, wos_c128 b, wos_c128 c, wos_c128 d);
/* Field.ScaleAmplitude (field.go:134-148). */
WOS_API int wos_scale_amplitude(wos_ctx ctx, wos_field* f, wos_c128 s);
/* Field.ApplyTilt (field.go:151-168): exp(i k (sin(tx) x + sin(ty) y)), the
 * row phase accumulated pixel by pixel exactly as the reference sums it. */
WOS_API int wos_apply_tilt(wos_ctx ctx, wos_field* f, double tx, double ty, double wavelength);
/* Field.ApplyBandlimit (field.go:264-294): fraction / sigma of Nyquist;
 * fraction outside (0, 1) leaves the field unchanged. */
WOS_API int wos_apply_bandlimit(wos_ctx ctx, wos_field* f, double fraction, double sigma);
/* Field.ShiftField (field.go:199-228): G(x, y) = F(x - du, y - dv) by a Fourier ramp. */
WOS_API int wos_shift_field(wos_ctx ctx, wos_field* f, double du, double dv);
/* diffuserEl.Apply (elements.go:722-783): hashNoise01 phase screen on the lab
 * lattice, Gaussian correlation filter (correlation > 0), rescaled to standard
 * deviation sigma, transmission amplitude * exp(i phase). */
WOS_API int wos_apply_diffuser(wos_ctx ctx, wos_field* f, double sigma, double correlation, double amplitude,
                               long long seed, double x0, double y0);

/* ---- PropagateVectorial (optics/vectorial.go:14-80; Propagate with method
 *      "vectorial", propagate.go:90-93): Ex and Ey (both used whatever
 *      f->polarized says, as the reference uses f.Ey) propagate in place and
 *      ez [ny][nx] complex128 receives the longitudinal component
 *      Ez = -(kx Ex + ky Ey) / kz propagated with them.  z == 0 leaves
 *      everything untouched (Propagate returns first). ---- */
WOS_API int wos_propagate_vectorial(wos_ctx ctx, wos_field* f, wos_c128* ez, double z, const wos_context* c);

/* ---- anisotropic media.  PropagateUniaxial (optics/birefringent.go:19-61):
 *      optic axis along x, Ex takes the extraordinary transfer function and Ey
 *      (when polarized) the ordinary one; evanescent components decay.
 *      PropagateAnisotropic (optics/berreman.go:13-272): relative permittivity
 *      eps (row-major 3x3 complex), Berreman 4x4 method per spectral component
 *      (two forward eigenmodes, each with its own complex kz); Ex and Ey both
 *      used whatever f->polarized says, as the reference uses f.Ey.  Both need
 *      the Context's wavelength > 0. ---- */
WOS_API int wos_propagate_uniaxial(wos_ctx ctx, wos_field* f, double z, double n_o, double n_e, const wos_context* c);
WOS_API int wos_propagate_anisotropic(wos_ctx ctx, wos_field* f, double z, const wos_c128* eps,
                                      const wos_context* c);

/* ---- plane views in the binary plane format of the reference's server
 *      (fmt=bin, server/server.go:582-634, server/views.go:131-258): float32
 *      little-endian [ny][nx], row-major, no header, computed in FP64 on the
 *      device and rounded once.  Views: TOTAL = Field.Intensity (|Ex|^2, + |Ey|^2
 *      when polarized, + |Ez|^2 when ez is given), AMPLITUDE = sqrt(TOTAL),
 *      EX / EY / EZ = |c|^2 of one component, PHASE_X / _Y / _Z = atan2 of one
 *      component, NaN (0x7fc00000) where its |c|^2 < mask_cut * its peak
 *      (mask_cut <= 0: 2e-3, the server's default) or everywhere when the
 *      component carries no light. ---- */
enum wos_view {
    WOS_VIEW_TOTAL = 0,
    WOS_VIEW_AMPLITUDE = 1,
    WOS_VIEW_EX = 2,
    WOS_VIEW_EY = 3,
    WOS_VIEW_EZ = 4,
    WOS_VIEW_PHASE_X = 5,
    WOS_VIEW_PHASE_Y = 6,
    WOS_VIEW_PHASE_Z = 7
};
/* Host field (ez may be NULL unless an Ez view is asked for; the Ey views read
 * f->ey whatever f->polarized says, as the server reads the part's Ey). */
WOS_API int wos_plane_view(wos_ctx ctx, const wos_field* f, const wos_c128* ez, int view, double mask_cut, float* out);
/* Device planes of the context's complex type: planes = [ncomp][ny][nx]
 * (ncomp 1 or 2; polarized when 2), ez null or one plane; out: device float
 * [ny][nx]. */
WOS_API int wos_plane_view_dev(wos_ctx ctx, int ny, int nx, int ncomp, const void* planes, const void* ez, int view,
                               double mask_cut, void* out);

/* ---- element train on the device (the element loop of trainer.runTrain,
 *      optics/simulator.go:397-500, without beam-splitter arms): the field is
 *      uploaded once, every op runs on the device in order, and the field is
 *      downloaded once at the end.  After every WOS_OP_PROPAGATE the
 *      bandlimit (fraction, sigma of Nyquist) is applied when fraction is in
 *      (0, 1), as runTrain does when ctx.Bandlimit is set.  diag (may be NULL)
 *      accumulates the warnings of every propagation (the shared
 *      ctx.Warnings); dx_out is the final pitch (fraunhofer changes it, and
 *      later ops use the new pitch).  f->polarized is updated when a Jones op
 *      turns a scalar field into a polarized one (f->ey must then hold
 *      ny*nx elements).  Parameters per kind, in the order of the matching
 *      wos_apply_* call:
 *        PROPAGATE   method = wos_method, a[0] = z
 *        LENS        a = {wavelength, focal, aperture, x0, y0}
 *        APERTURE    a = {radius, x0, y0, edge_sigma}
 *        GRATING     method = grating kind, a = {period, modulation, duty, blaze_depth, rotation, offset}
 *        PHASE_MASK  map = host phi [ny][nx], a[0] = amplitude
 *        DIFFUSER    a = {sigma, correlation, amplitude, seed, x0, y0}
 *        JONES       m = {a, b, c, d}
 *        SCALE       m[0] = s
 *        TILT        a = {tx, ty, wavelength}
 *        SHIFT       a = {du, dv}
 *        BANDLIMIT   a = {fraction, sigma}
 *        INTENSITY   out = host [ny][nx] FP64, receives |Ex|^2 (+ |Ey|^2) at this
 *                    point of the train (a sensor plane; only it crosses PCIe)
 *        VIEW        method = wos_view, a[0] = mask cut, out = host float [ny][nx]
 *                    (the binary plane format, see wos_plane_view) ---- */
enum wos_op_kind {
    WOS_OP_PROPAGATE = 1,
    WOS_OP_LENS = 2,
    WOS_OP_APERTURE = 3,
    WOS_OP_GRATING = 4,
    WOS_OP_PHASE_MASK = 5,
    WOS_OP_DIFFUSER = 6,
    WOS_OP_JONES = 7,
    WOS_OP_SCALE = 8,
    WOS_OP_TILT = 9,
    WOS_OP_SHIFT = 10,
    WOS_OP_BANDLIMIT = 11,
    WOS_OP_INTENSITY = 12,
    WOS_OP_VIEW = 13
};
typedef struct {
    int kind;
    int method;
    double a[8];
    wos_c128 m[4];
    const double* map;
    void* out;   /* INTENSITY: double [ny][nx]; VIEW: float [ny][nx] */
} wos_op;
WOS_API int wos_train(wos_ctx ctx, wos_field* f, const wos_op* ops, int nops, const wos_context* c,
                      double bandlimit_fraction, double bandlimit_sigma, wos_diag* diag);

/* ---- Propagate1D (optics/propagate.go:718-738): a[n] complex128 in place,
 *      pixel dx, distance z, wavelength wl (the Context's wavelength is not
 *      used).  diag (may be NULL): p_in / p_out are sum |a|^2 without a dx
 *      factor (sum1DSq) and evanescent_filtered is the only warning. ---- */
WOS_API int wos_propagate1d(wos_ctx ctx, int n, wos_c128* a, double dx, double z, double wavelength,
                            const wos_context* c, wos_diag* diag);

/* ---- inverse design (no counterpart in the reference): ASM forward / adjoint.
 *      u = ASM_z(a * exp(i phi)), L = sum (|u|^2 - T)^2, grad = dL/dphi. ---- */
WOS_API int wos_asm_forward_loss(wos_ctx ctx, int ny, int nx, double dx, double z, const wos_context* c,
                         const wos_c128* a, const double* phi, const double* target, double* loss);
WOS_API int wos_asm_loss_grad(wos_ctx ctx, int ny, int nx, double dx, double z, const wos_context* c,
                      const wos_c128* a, const double* phi, const double* target, double* loss,
                      double* grad);
/* Device-resident form of wos_asm_loss_grad for optimisation loops that keep
 * the design on the GPU: a is a device [ny][nx] array of the context's complex
 * type, phi and target device FP64 arrays, grad a device FP64 array (or NULL
 * for the loss alone); the loss is returned to the host.  Power-of-two ny, nx
 * from 256 to 8192 (else WOS_UNSUPPORTED_SIZE). */
WOS_API int wos_asm_loss_grad_dev(wos_ctx ctx, int ny, int nx, double dx, double z, const wos_context* c,
                                  const void* a, const double* phi, const double* target, double* loss,
                                  double* grad);
/* ---- diffractive stack (no counterpart in the reference): nlayers phase masks,
 *      each followed by a split-step BPM segment of `steps` slices over zseg
 *      through the parametric medium n (PropagateSplitStep, optics/medium.go:22-45):
 *      u = a; for l: u = BPM(u * exp(i phis[l])); L = sum (|u|^2 - T)^2;
 *      grads[l] = dL/dphis[l] by the exact adjoint chain.  Host arrays:
 *      a [ny][nx] complex128, phis / grads [nlayers][ny][nx], target [ny][nx]
 *      FP64; grads may be NULL (loss only). ---- */
WOS_API int wos_bpm_stack_loss_grad(wos_ctx ctx, int ny, int nx, double dx, int nlayers, const wos_c128* a,
                                    const double* phis, const double* target, double zseg,
                                    const wos_index_desc* n, int steps, const wos_context* c, double* loss,
                                    double* grads);
/* Device-resident form: a of the context's complex type, phis / target /
 * grads FP64 device arrays; the loss is returned to the host. */
WOS_API int wos_bpm_stack_loss_grad_dev(wos_ctx ctx, int ny, int nx, double dx, int nlayers, const void* a,
                                        const double* phis, const double* target, double zseg,
                                        const wos_index_desc* n, int steps, const wos_context* c, double* loss,
                                        double* grads);
/* Adjoint of wos_splitstep (conj transfer functions and screens, slices in
 * reverse order): the backward BPM operator, host field in place. */
WOS_API int wos_splitstep_adjoint(wos_ctx ctx, wos_field* f, double z, const wos_index_desc* n, int steps,
                                  const wos_context* c);
/* Adjoint of wos_splitstep_dev (conj transfer functions and screens, slices
 * in reverse order), device field in place, no diagnostics. */
WOS_API int wos_splitstep_adjoint_dev(wos_ctx ctx, int ny, int nx, double dx, int ncomp, void* field, double z,
                                      const wos_index_desc* n, int steps, const wos_context* c);
/* Adjoint operator A^H = F^-1 diag(conj H) F of an ASM step, host field in place. */
WOS_API int wos_asm_adjoint(wos_ctx ctx, wos_field* f, double z, const wos_context* c);

/* ---- CUDA graphs of device-resident calls (no counterpart in the reference).
 *      Between capture_begin and capture_end, the device-resident entry points
 *      called on this context (wos_propagate_dev / _batch_dev / _dev_c128,
 *      wos_splitstep_dev, wos_splitstep_adjoint_dev, wos_fft2d_dev,
 *      wos_asm_loss_grad_dev, wos_bpm_stack_loss_grad_dev, ...) are recorded,
 *      not run; wos_graph_launch replays the whole sequence on the context
 *      stream with one launch, for loops that repeat it on the same device
 *      buffers.  Each call must have run once on the same geometry before the
 *      capture (its work space and tables are then in place: nothing is
 *      allocated or built while capturing) and must not ask for diagnostics
 *      or return values that need a synchronisation (a call that does fails
 *      and the capture with it).  Replays use the buffers and parameters of
 *      the capture: the transfer-function tables and device copies of
 *      parameter lists a capture uses are kept as they are until the context
 *      is destroyed (later calls with other distances or lists take other
 *      entries). ---- */
WOS_API int wos_graph_capture_begin(wos_ctx ctx);
/* Concurrent branches of one capture: after wos_graph_capture_begin(ctx),
 * wos_graph_capture_fork(ctx, other) makes another context (same device, its
 * own stream) a branch of the capture: the device-resident calls made on
 * `other` are recorded into ctx's graph, after what ctx recorded before the
 * fork and concurrently with what ctx records after it.
 * wos_graph_capture_join(ctx, other) closes the branch (ctx's later calls and
 * the end of the graph wait for it); every branch must be joined before
 * wos_graph_capture_end(ctx).  The same rules as for ctx apply to the calls
 * on a branch.  Independent batches (e.g. the wavelengths, modes and planes
 * of three jobs) replay this way as one graph whose jobs share the GPU.
 * Destroying a branch before its join makes ctx's capture fail at its end;
 * destroying ctx mid-capture ends the capture and releases its branches. */
WOS_API int wos_graph_capture_fork(wos_ctx ctx, wos_ctx other);
WOS_API int wos_graph_capture_join(wos_ctx ctx, wos_ctx other);
WOS_API int wos_graph_capture_end(wos_ctx ctx, wos_graph* out);
WOS_API int wos_graph_launch(wos_ctx ctx, wos_graph g);
WOS_API int wos_graph_destroy(wos_graph g);

/* ---- zero-padded ASM that allocates no device memory (no counterpart in the
 *      reference).  For callers that cannot call cudaMalloc: processes that
 *      reserve all device memory up front behind their own allocator, or
 *      pipelines that cannot afford the device-wide synchronisation of
 *      cudaFree.  Same result as wos_propagate_dev(..., WOS_ASM_PAD, ...) on a
 *      WOS_FP32 context, without diagnostics.  in / out: device complex64
 *      [ny][nx] (in == out allowed); ny and nx powers of two, 4..1024, larger
 *      sizes return WOS_UNSUPPORTED_SIZE.  Work space: file-scope device arrays
 *      (a 1024 x 2048 complex64 intermediate, 16 MiB, plus 32 KiB of
 *      twiddles); once a device holds them it keeps them until exit.  The
 *      CUDA runtime places them when it loads their module into the device's
 *      context: under lazy module loading (the default since CUDA 12.2) that
 *      is the first call on the device, so a caller whose allocator reserves
 *      the whole GPU must make the first call before reserving, or run with
 *      CUDA_MODULE_LOADING=EAGER.  The first call on a device (and the first
 *      after the caller re-created the device's context, e.g. by
 *      cudaDeviceReset) resolves their addresses and fills the twiddles (a
 *      kernel and a synchronisation of `stream`): make that first call
 *      before any stream capture.  All calls share the arrays, so calls that
 *      overlap on the GPU (different streams or threads) race; serialise them.
 *      Nothing needs clearing between calls: each call writes every scratch
 *      element it reads.  stream: a cudaStream_t (NULL = legacy default). ---- */
WOS_API int wos_asm_pad_c64_noalloc(const void* in, void* out, int ny, int nx, double dx, double z,
                                    const wos_context* c, void* stream);

#ifdef __cplusplus
}
#endif
#endif

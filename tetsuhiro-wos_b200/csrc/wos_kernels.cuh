// wos_kernels.cuh -- argument blocks and launchers of the propagation kernels.
//
// Data layout in HBM: a field component is a row-major ny x nx array of
// complex (float2 for the FP32 pipeline, double2 for FP64), row stride ld
// elements.  Host I/O (the Go complex128 slices) is double2; the FP32
// pipeline converts inside its first and last sweep, never in a separate pass.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace wos {

// Transfer-function kinds evaluated inside the fused column pass.
enum HKind {
    H_NONE = 0,        // identity (pure FFT round trip / reductions only)
    H_ASM = 1,         // band-limited angular spectrum, evanescent policy
    H_FRESNEL_TF = 2,  // exp(ikz) exp(-i pi lambda z f^2)
    H_TABLE_XY = 3,    // separable product tx[col] * ty[q] (Fresnel impulse response)
    H_ASM_HALF2 = 4,   // (H_asm(z))^2 evaluated as a product: merged BPM half-steps
    H_GAUSS = 5,       // exp(p0 (fx^2+fy^2)): diffuser correlation filter (elements.go:744-754)
    H_BANDLIMIT = 6,   // exp(-((|f|-p0)/p1)^2) for |f| > p0: ApplyBandlimit (field.go:264-294)
    H_SHIFT = 7,       // exp(-2 pi i (fx p0 + fy p1)): ShiftField (field.go:199-228)
    H_UNIAX_O = 8,     // ordinary wave of a uniaxial crystal, n_o = p0 (birefringent.go:38-44)
    H_UNIAX_E = 9,     // extraordinary wave, n_o = p0, n_e = p1 (birefringent.go:45-53)
};

struct HArgs {
    int kind;
    int conj;            // adjoint: multiply by conj(H)
    int exact;           // FP64 mirror of the reference's operation order
    double wl, k;        // wavelength, 2 pi / wl
    double z, kz, kaz;   // z, k*z, k*|z|
    int zero_ev, reg;    // evanescent policy
    double alpha, limit;
    double dx;
    int lfx, lfy;        // frequency grid lengths (padded / logical)
    double fxoff, fyoff; // carrier offsets (asm_shift)
    double scale;        // normalisation folded into H (1/(Lx*Ly) ...)
    double c_re, c_im;   // extra complex constant (Fresnel prefactors)
    const void* tx;      // H_TABLE_XY tables (C type), length lfx / lfy
    const void* ty;
    double p0, p1;       // parameters of the spectral filters (H_GAUSS .. H_SHIFT)
};

// Reduction slots (FP64) written per CTA; finalised by k_reduce_finish.
enum RedSlot {
    RS_P = 0,        // sum |E|^2
    RS_PX = 1,       // sum |E|^2 x        (fraunhofer rms radius)
    RS_PY = 2,       // sum |E|^2 y
    RS_PR2 = 3,      // sum |E|^2 (x^2+y^2)
    RS_SW = 4,       // spectral: sum |F|^2
    RS_SFX = 5,      // spectral: sum |F|^2 fx
    RS_SFY = 6,      // spectral: sum |F|^2 fy
    RS_SH1 = 7,      // spectral: sum |F H|^2 (BPM half step power)
    RS_SH2 = 8,      // spectral: sum |F H H|^2
    RS_HIST = 9,     // 97-bin radial spectral histogram
    RS_SLO = 9 + 97, // low parts of RS_SW, RS_SFX, RS_SFY (compensated centroid sums)
    RS_COUNT = RS_SLO + 3,
};

// ROW_FWD     : load (+pre ops) -> forward transform -> store
// ROW_INV     : load -> inverse transform -> store (+post ops)
// ROW_INV_FWD : load -> inverse -> real-space screen -> forward -> store (BPM slice)
// ROW_INV_ACC : for every batch b: load -> inverse -> acc += weight[b] |E|^2; store acc
enum RowMode { ROW_FWD = 0, ROW_INV = 1, ROW_INV_FWD = 2, ROW_INV_ACC = 3 };
// COL_FUSED      : forward -> H (+spectral sums) -> inverse -> store
// COL_FRAUNHOFER : forward -> far-field epilogue store
// COL_REDUCE     : forward -> spectral sums / histogram, no store
// COL_FFT        : forward or inverse (col_inverse) -> store (fft2D users)
enum ColMode { COL_FUSED = 0, COL_FRAUNHOFER = 1, COL_REDUCE = 2, COL_FFT = 3 };

// Pointwise real-space screen applied between the inverse and forward row
// transforms of a split-step BPM slice, or on load/store of a row pass.
struct ScreenArgs {
    int kind;          // 0 none, 1 parametric index, 2 index maps (re/im FP64 arrays)
    double k, dz;      // k0, slice thickness
    double zc;         // slice centre
    // parametric index (wos_index_desc)
    double re_bg, im_bg, core_dn, core_x0, core_y0, core_w;
    double zmod_amp, zmod_period, zmod_phase;
    int border_px, border_order;
    double border_strength;
    int n_layers;
    double layer_z[8], layer_re[8], layer_im[8];
    const double* nre; const double* nim;   // maps (kind 2)
    int conj;          // adjoint: conj(t)
};

struct RowArgs {
    int mode;
    int rows;                 // lines in this launch
    int L;                    // transform length (power of two, M for Bluestein)
    int blue_n;               // logical Bluestein length (0: plain power-of-two)
    int ny_grid, nx_grid;     // unpadded grid, for coordinates
    double dx;
    int row0;                 // grid row of line 0 (coordinates / padding)
    // input
    const void* in; int in_c128; long long in_ld; long long in_bstride;
    int in_off, in_n;         // input occupies positions [in_off, in_off+in_n)
    // output
    void* out; int out_c128; long long out_ld; long long out_bstride;
    int out_off, out_n;       // positions [out_off, out_off+out_n) are stored
    int out_accum_int;        // 0 store field; 1 accumulate weight*|E|^2 into float; 2 into double
    double weight;
    double out_scale;         // scalar applied on store
    // tables
    const void* tw;           // twiddles for L
    const void* chirp;        // Bluestein chirp (forward sign), length blue_n
    const void* bhat_f;       // FFT_M(b0_forward) / M
    const void* bhat_i;       // FFT_M(b0_inverse) / M
    // carrier ramp exp(sgn 2 pi i (fxc x + fyc y)) on load (pre_shift) / store (post_shift)
    int pre_shift, post_shift;
    double fxc, fyc;
    // phase mask exp(i phi) * amp applied on load (inverse design)
    const double* pre_phi; const float* pre_phi_f; double pre_amp;
    // screen
    ScreenArgs scr;
    // reductions
    double* red;              // [gridDim.x][RS_COUNT] partials, or null
    int red_pre, red_post;    // reduce |E|^2 on load / on store
    int red_moments;          // also x, y, r^2 moments (rms radius)
    int batch;                // gridDim.y batches, strides in/out_bstride
    const double* acc_weight; // ROW_INV_ACC: weight per batch
    int acc_nb;               // ROW_INV_ACC: number of batches read by each CTA
    int acc_add;              // ROW_INV_ACC: add into the existing output
};

struct ColArgs {
    int mode;
    int ncols;                // lines
    int L, blue_n;
    int W;                    // columns per CTA (power of two)
    const void* src; long long src_ld; long long src_bstride;
    int in_off, in_n;
    void* dst; long long dst_ld; long long dst_bstride;
    int out_off, out_n;
    const void* tw;
    const void* chirp; const void* bhat_f; const void* bhat_i;
    HArgs h;
    // per-batch H parameters (batched polychromatic / volume): arrays of gridDim.y
    const double* batch_wl;   // wavelength per batch (null: h.wl)
    const double* batch_z;    // z per batch (null: h.z)
    int src_shared;           // 1: every batch reads batch 0 of src
    double* red;
    int red_spec;             // spectral sums (SW, SFX, SFY), compensated: high parts in RS_SW.., low in RS_SLO..
    int red_hist;             // radial histogram
    int red_bpm;              // SH1 / SH2 sums
    int hist_lx, hist_ly;     // grid for the histogram / centroid frequencies
    double hist_dx;
    // Fraunhofer epilogue
    double fr_c_re, fr_c_im;  // cexpI(kz) * (-i/(wl z)) * dx^2
    double fr_k2z;            // k/(2z)
    double fr_dxout;
    int fr_n;
    int batch;
    int col_inverse;          // COL_FFT direction
    double out_scale;         // COL_FFT scale on store
    int src_spectrum;         // COL_FUSED: src is already column-transformed (shared by a batch's
                              // units), so the first transform is skipped; lines without Bluestein
};

// launchers (wos_kernels.cu)
cudaError_t launch_rows(int fp64, const RowArgs& a, cudaStream_t st);
cudaError_t launch_cols(int fp64, const ColArgs& a, cudaStream_t st);
cudaError_t launch_twiddles(int fp64, void* tw, int L, cudaStream_t st);
// Per-pass tables of a mixed-radix line, written after its L-point table.
cudaError_t launch_mixed_twiddles(int fp64, void* out, int L, cudaStream_t st);
cudaError_t launch_chirp_b0(int fp64, void* chirp, double2* b0f, double2* b0i, int n, int M,
                            cudaStream_t st);
cudaError_t launch_bhat_finish(int fp64, void* dst_f, void* dst_i, const double2* bf,
                               const double2* bi, int M, cudaStream_t st);
// Sums per-CTA partials: nbatch groups of nblocks blocks each, slots [s0, s0+ns),
// out[g*RS_COUNT + slot].
cudaError_t launch_reduce_finish(const double* partials, int nblocks, int nbatch, int s0, int ns,
                                 double* out, cudaStream_t st);
int max_threads_for(int fp64, int E);
cudaError_t launch_convert(int to_c128, const void* src, void* dst, long long n, cudaStream_t st);
cudaError_t launch_fresnel_ir_axis(double2* h, int m, double dx, double wl, double z, cudaStream_t st);
cudaError_t launch_scale_copy(int fp64, const double2* src, void* dst, long long n, double sre,
                              double sim, cudaStream_t st);

// pointwise kernels (wos_elem.cu)
cudaError_t launch_lens(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double c, double ap, double x0,
                        double y0, cudaStream_t st);
cudaError_t launch_aperture_circle(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double radius,
                                   double x0, double y0, double sig, cudaStream_t st);
cudaError_t launch_grating(double2* ex, double2* ey, int pol, int ny, int nx, double dx, int kind, double period,
                           double modulation, double duty, double blaze, double rotation, double off,
                           cudaStream_t st);
cudaError_t launch_phase_mask(double2* ex, double2* ey, int pol, long long n, const double* phi, double amp,
                              cudaStream_t st);
cudaError_t launch_jones(double2* ex, double2* ey, long long n, int mode, double2 a, double2 b, double2 c, double2 d,
                         cudaStream_t st);
cudaError_t launch_scale(double2* ex, double2* ey, int pol, long long n, double2 s, cudaStream_t st);
// k = 2 pi / wl, sx = sin(tx), sy = sin(ty) (the running row phase of ApplyTilt)
cudaError_t launch_tilt(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double k, double sx, double sy,
                        cudaStream_t st);
cudaError_t launch_diffuser_noise(double2* z, int ny, int nx, double dx, double cell, double x0, double y0,
                                  long long seed, cudaStream_t st);
int sum_re2_blocks(long long n);
cudaError_t launch_sum_re2(const double2* z, long long n, double* partials, cudaStream_t st);
cudaError_t launch_diffuser_apply(double2* ex, double2* ey, int pol, long long n, const double2* z,
                                  const double* sums, double sigma, double amp, cudaStream_t st);
// u *= exp(i phi) (exp(-i phi) when conj), u of the context's complex type
cudaError_t launch_mask_phase(int fp64, void* u, const double* phi, long long n, int conj, cudaStream_t st);
// g = Re(conj(b) * i * v)
cudaError_t launch_grad_v(int fp64, const void* b, const void* v, double* g, long long n, cudaStream_t st);
// Peak |c|^2 of a plane (partial: norm2_max_blocks(n) doubles; out: one double).
int norm2_max_blocks(long long n);
cudaError_t launch_norm2_max(int fp64, const void* a, long long n, double* partial, double* out, cudaStream_t st);
// One view of a plane as float32 bits (see k_plane_view); ey / ez may be null
// when not read; peak: device double (phase views).
cudaError_t launch_plane_view(int fp64, const void* ex, const void* ey, const void* ez, int pol, long long n, int view,
                              const double* peak, double cut, void* out, cudaStream_t st);
// Relative permittivity tensor, row-major 3x3 (complex).
struct Eps9 {
    double2 v[9];
};
// Berreman 4x4 propagation on the spectra of [Ex, Ey] planes (wos_aniso.cu).
cudaError_t launch_aniso(int fp64, void* planes, int ny, int nx, double dx, double k0, double z, const Eps9& e,
                         cudaStream_t st);
// Vector angular spectrum step on the spectra of [Ex, Ey, Ez] planes (Ez written).
cudaError_t launch_vectorial(int fp64, void* planes, int ny, int nx, double dx, const HArgs& h, cudaStream_t st);
// 1-D angular spectrum step on a forward-transformed line (asmTF1D,
// optics/propagate.go:668-738): a[i] *= H(fx_i) / n; spectral power sums
// (RS_SW: sum |F|^2, RS_SW+1: sum |F|^2 (1 - |H|^2)) per CTA into partials.
cudaError_t launch_asm1d_h(int fp64, void* a, int n, const HArgs& h, double* partials, int* nblocks,
                           cudaStream_t st);
cudaError_t launch_schell_mu(double2* a, int n, double dx, double coh, cudaStream_t st);
cudaError_t launch_sqrt_re(double* s, const double2* a, long long nn, cudaStream_t st);
cudaError_t launch_mul_map(double2* a, const double* s, long long nn, int batches, cudaStream_t st);
cudaError_t launch_schell_env(double2* a, int n, double dx, double width, int batches, cudaStream_t st);
cudaError_t launch_accum_int(int fp64, double* out, const void* f, int ncomp, long long np, double w,
                             cudaStream_t st);
cudaError_t launch_residual(int fp64, const void* u, const double* T, void* r, long long n, double* partials,
                            int* nblocks, cudaStream_t st);
cudaError_t launch_grad(int fp64, const void* b, const double2* a, const double* phi, double* g, long long n,
                        cudaStream_t st);

int row_threads_per_line(int L, int E);
int pick_E(int fp64, int L);
size_t row_smem_bytes(int fp64, int L, int E, int lines);
size_t col_smem_bytes(int fp64, int L, int W);

}  // namespace wos

// wos_fast.cuh -- argument blocks of the compile-time specialised ASM sweeps.
#pragma once
#include <cuda_runtime.h>

namespace wos {

struct FastRows {
    int rows;
    const void* in; int in_c128; long long in_ld, in_bstride;
    void* out; int out_c128; long long out_ld, out_bstride;
    const void* tw;       // twiddles for L (pipeline precision)
    double out_scale;
    double* red;          // per-CTA sum |E|^2 (record stride red_stride), or null
    long long red_stride;
    int batch;
    unsigned* err;        // device error word of the pipelined kernels (bit 0: a bounded wait expired)
    double out_scale_im;  // imaginary part of the output scale (complex scale when non-zero)
    // split-step slice screen between an inverse and a forward row transform
    // (k_rows_bpm_fast): t = border[d] * exp(i phase gx[x] gy(y)), the
    // constant part of the slice (background index, interior absorption) being
    // applied once per run by the caller
    const double* bpm_gx;     // exp(-(x - x0)^2 / w^2) per column, or null (no graded core)
    double bpm_y0, bpm_w2;    // row factor gy = exp(-(y - y0)^2 / w^2)
    double bpm_dx;            // pixel pitch (y = (r - ny/2) dx)
    double bpm_phase;         // k dz core_dn (1 + zmod_amp sin(2 pi zc / period + phase))
    const double* bpm_border; // exp(-k dz strength ((px - d)/px)^order) for edge distance d < px, or null
    int bpm_border_px;
    int bpm_nx;               // grid width (edge distance)
    // tiled intermediate of the three-sweep ASM: columns grouped in tiles of
    // kTileW, element (r, x) of a batch item at (x / kTileW) * tile_len *
    // kTileW + r * kTileW + x % kTileW, so that a column tile is one
    // contiguous block; out_tiled on the forward sweep's store, in_tiled on
    // the inverse sweep's load (native complex type only)
    int out_tiled, in_tiled;
    long long tile_len;       // rows of the field (the column length)
    // residual twiddle table of the compensated transforms (complex64
    // split-step row sweep): same layout as tw, (float)(W - tw) from FP64; null
    // for the plain transforms
    const void* tw_lo;
    // Gaussian-Schell synthesis fused into the first row sweep
    // (k_rows_schell_fast): the complex128 input (a realization's noise) is
    // multiplied by pre_map[r][x] (FP64, shared by the batch) on load, inverse
    // transformed, multiplied by env_x[x] and forward transformed
    const double* pre_map;
    const double* env_x;
    int out_stream;       // inverse sweep: the output with streaming (evict-first) stores
};
constexpr int kTileW = 4;

struct FastCols {
    int ncols;            // columns = the frequency grid length along x
    int W;                // columns per CTA (power of two)
    void* data;           // in place, row stride ld
    long long ld, bstride;
    const void* tw;
    int batch;
    // band-limited ASM transfer function (optics/propagate.go:159-199)
    double wl, dx, kz, kaz, scale, alpha, limit;
    int zero_ev, reg, backward;
    int conj;             // adjoint: multiply by conj(H)
    double krev;          // kz / (2 pi): the propagating phase in revolutions (FP32: |krev| < 2^28)
    int precise_phase;    // FP32: sin/cos of the phase to ~1 ulp (repeated application, e.g. split-step)
    double* red;          // per-CTA [sum |F|^2, sum |F|^2 (1-|H|^2)], or null
    long long red_stride;
    // radial histogram of |F|^2 for the alias-wrap check (97 bins of
    // hypot(fx, fy) / f_Nyquist, optics/propagate.go:203-245), per CTA at
    // hist + block * red_stride, or null
    double* hist;
    double hist_dx;
    unsigned* err;        // device error word of the pipelined kernels (bit 0: a bounded wait expired)
    // batches of units (polychromatic wavelengths, volume distances): unit b =
    // blockIdx.y reads src + b * src_bstride (src null: in place) and writes
    // data + b * bstride; its wavelength and distance come from batch_wl[b] /
    // batch_z[b] when given (else wl / z)
    const void* src;
    long long src_bstride;
    const double* batch_wl;
    const double* batch_z;
    double z;
    int tiled;            // data (and src) in the tiled layout of FastRows (W == kTileW, ld == kTileW)
    // split tiles (FP32, L = 2048, W = 8): a tile is held by a two-CTA cluster,
    // half of every column per CTA; per-pass twiddles of length L/2 and the
    // table W_L^n for n < L/2 (both null: one CTA per tile)
    const void* tw_half;
    const void* tw_pair;
    // residual twiddle table of the compensated transforms (complex64
    // split-step column sweep), as FastRows::tw_lo; null for the plain ones
    const void* tw_lo;
    // quarter-plane table of the complex64 transfer function (FP64 evaluation
    // in the reference's operation order, scale folded in, rounded once): row
    // c = |fx index| (0 .. ncols/2) holds htab_ld entries, entry q = |fy
    // index| (0 .. L/2; the rest zero).  When set (complex64, no loss sums,
    // one wavelength and distance), a CTA copies the W rows of its columns
    // into shared memory while it transforms and reads H there instead of
    // evaluating it (conj applied on reading).  With tw_lo (compensated
    // sweeps) an entry is the pair (H_hi, H_lo), 16 bytes, H_lo = H - H_hi.
    const float2* htab;
    int htab_ld;
    // 1: the plain complex64 sweep (no loss sums, histogram or compensated
    // transforms) reads its H straight from the table in global memory (L2
    // resident across a batch) into registers, at the positions the forward
    // transform leaves in them, instead of staging the spectrum in shared
    // memory to evaluate H once per (q, L - q) pair
    int htab_global;
    // Gaussian-Schell synthesis fused into the column sweep (instantiations
    // with PRE = 1): each column is inverse transformed, multiplied by
    // env_y[y] and forward transformed before the transfer function
    const double* env_y;
};
// Table rows of the W columns from col0 (W | ncols / 2): contiguous, in order
// below ncols / 2 and reversed above it.
__host__ __device__ inline int htab_row0(int col0, int ncols, int W) {
    return col0 < ncols / 2 ? col0 : ncols - col0 - (W - 1);
}
// Row length of the table for columns of L points (a power of two >= 32):
// L/2 + 8 >= L/2 + 1 entries, so rows are whole 16-byte units and consecutive
// rows start 16 shared-memory banks apart.
inline int htab_ld_for(int L) { return L / 2 + 8; }
// Build the table of a's transfer function for columns of L points (the H
// arguments in a, with conj ignored); hilo 0: float2 entries, 1: (H_hi, H_lo)
// pairs of float2 per entry, for the compensated sweeps (which read them as
// such), 2: double2 entries, for the complex128 pipeline.
cudaError_t fast_build_htab(const FastCols& a, int L, float2* out, int ld, int hilo, cudaStream_t st);
// Shared memory of a complex64 column CTA with the table rows.
size_t fast_col_smem_htab(int L, int E, int W, int ld, int hilo);

cudaError_t fast_rows(int fp64, int L, int E, bool inv, const FastRows& a, cudaStream_t st, int* nblocks);
// Gaussian-Schell sweeps (wos_schell.cu): the first row sweep of a batch of
// realizations (a.pre_map, a.env_x; complex128 input) and the column sweep
// with the column envelope (a.env_y).  cudaErrorNotSupported outside E = 8,
// L = 256 .. 4096.
cudaError_t fast_rows_schell(int fp64, int L, int E, const FastRows& a, cudaStream_t st, int* nblocks);
cudaError_t fast_cols_env(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks);
// The column sweep of a batch whose source (a.src, shared: src_bstride 0) is
// already column-transformed: H and the inverse only.
cudaError_t fast_cols_spec(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks);
cudaError_t fast_cols(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks);
// The column sweep on two-CTA clusters (see FastCols::tw_half); returns
// cudaErrorNotSupported outside its case (FP32, L = 2048, E = 16, W = 8, no
// histogram, tables given).
cudaError_t fast_cols_pair(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks);
bool fast_cols_pair_case(int fp64, int L, int E, int W);
// W_L^n (forward sign) for n < L/2 in the pipeline's precision, generated in FP64.
cudaError_t fast_build_pair_twiddles(int fp64, int L, void* out, cudaStream_t st);
// Inverse design on rows (ASM forward / adjoint of L = sum (|u|^2 - T)^2):
// stage 0 loads a exp(i phi) and transforms forward; stage 1 transforms back
// to u, forms r = 4 (|u|^2 - T) u (loss partial per CTA, slot 0 of a record of
// red_stride) and transforms r forward; stage 2 transforms back to b = A^H r
// and writes g = Re(conj(b) i exp(i phi) a).  Single component, row-major
// ny x nx; a is complex128 when amp_c128, else the pipeline's complex type.
struct DesignArgs {
    const double* phi;
    const double* target;
    const void* amp;
    int amp_c128;
    double* grad;
};
cudaError_t fast_rows_design(int fp64, int L, int E, int stage, const FastRows& a, const DesignArgs& d,
                             cudaStream_t st, int* nblocks);

// Inverse row transforms of the units of a batch, accumulated as weighted
// intensity in one pass: out[r][x] (+)= sum_u w[u] |IFFT(in_u)[r][x]|^2, in_u =
// in + u * in_bstride (nb units), out FP64 [rows][L].
struct AccArgs {
    int nb;
    const double* weight;  // per unit, or null (1)
    double* out;
    int add;               // add to out instead of overwriting it
};
cudaError_t fast_rows_acc(int fp64, int L, int E, const FastRows& a, const AccArgs& acc, cudaStream_t st,
                          int* nblocks);

// One split-step slice on rows: inverse transform, slice screen, forward
// transform (native precision in and out, in place allowed).
cudaError_t fast_rows_bpm(int fp64, int L, int E, const FastRows& a, cudaStream_t st, int* nblocks);
bool fast_supported(int fp64, int L, int E);

}  // namespace wos

namespace wos {
// per-pass twiddle tables of the specialised sweeps (forward passes, then inverse)
int fast_table_len(int L, int E);
cudaError_t fast_build_twiddles(int fp64, int L, int E, void* out, cudaStream_t st);
// Residuals of the complex64 per-pass tables: (float)(W - (float)W) with W in FP64.
cudaError_t fast_build_twiddles_lo(int L, int E, void* out, cudaStream_t st);
// Compensated (hi + lo) complex64 split-step sweeps (wos_fast_cp.cu); the
// plain launchers forward to them when tw_lo is set.
cudaError_t fast_rows_bpm_cp(int L, int E, const FastRows& a, cudaStream_t st, int* nblocks);
cudaError_t fast_cols_cp(int L, int E, const FastCols& a, cudaStream_t st, int* nblocks);
size_t fast_col_smem(int fp64, int L, int E, int W);
int fast_col_width(int fp64, int L, int E, int W);
// lines per CTA of the fast row sweeps (the launchers and the record sizing share it)
int fast_row_lines(int L, int E, int rows);
}  // namespace wos

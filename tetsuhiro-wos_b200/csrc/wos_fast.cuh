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
};

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
    double* red;          // per-CTA [sum |F|^2, sum |F|^2 (1-|H|^2)], or null
    long long red_stride;
    // radial histogram of |F|^2 for the alias-wrap check (97 bins of
    // hypot(fx, fy) / f_Nyquist, optics/propagate.go:203-245), per CTA at
    // hist + block * red_stride, or null
    double* hist;
    double hist_dx;
    unsigned* err;        // device error word of the pipelined kernels (bit 0: a bounded wait expired)
};

cudaError_t fast_rows(int fp64, int L, int E, bool inv, const FastRows& a, cudaStream_t st, int* nblocks);
cudaError_t fast_cols(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks);
bool fast_supported(int fp64, int L, int E);

}  // namespace wos

namespace wos {
// per-pass twiddle tables of the specialised sweeps (forward passes, then inverse)
int fast_table_len(int L, int E);
cudaError_t fast_build_twiddles(int fp64, int L, int E, void* out, cudaStream_t st);
size_t fast_col_smem(int fp64, int L, int E, int W);
int fast_col_width(int fp64, int L, int E, int W);
}  // namespace wos

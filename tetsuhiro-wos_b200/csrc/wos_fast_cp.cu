// wos_fast_cp.cu -- the compensated (hi + lo twiddles and rotation constants)
// complex64 split-step sweeps: the row sweep inverse . screen . forward and the
// fused column sweep, instantiated apart from wos_fast.cu so the two compile
// in parallel.  fast_rows_bpm / fast_cols forward here when the argument
// block carries a residual table (tw_lo).
#include "wos_fast_kern.cuh"

namespace wos {

#define WOS_FAST_L(X) X(256) X(512) X(1024) X(2048) X(4096) X(8192)

cudaError_t fast_rows_bpm_cp(int L, int E, const FastRows& a, cudaStream_t st, int* nblocks) {
#define CASE_B(LL)                                                                \
    case LL:                                                                      \
        if constexpr (LL <= 4096) {                                               \
            if (E == 8) return go_rows_bpm<float, LL, 8, true>(a, st, nblocks);   \
        }                                                                         \
        if (E == 16) return go_rows_bpm<float, LL, 16, true>(a, st, nblocks);     \
        break;
    switch (L) { WOS_FAST_L(CASE_B) }
#undef CASE_B
    return cudaErrorNotSupported;
}

template <int L, int E>
static cudaError_t go_cols_cp(const FastCols& a, cudaStream_t st, int* nblocks) {
    if (a.htab_global) {  // H (hi + lo) from the table, in registers
        switch (fast_col_width(0, L, E, a.W)) {
        case 4: return go_cols_w<float, L, E, 4, true, false, true>(a, st, nblocks);
        case 8: return go_cols_w<float, L, E, 8, true, false, true>(a, st, nblocks);
        default: break;  // other widths: H from the table rows in shared memory
        }
    }
    switch (fast_col_width(0, L, E, a.W)) {
    case 1: return go_cols_w<float, L, E, 1, true>(a, st, nblocks);
    case 2: return go_cols_w<float, L, E, 2, true>(a, st, nblocks);
    case 4: return go_cols_w<float, L, E, 4, true>(a, st, nblocks);
    case 8: return go_cols_w<float, L, E, 8, true>(a, st, nblocks);
    case 16: return go_cols_w<float, L, E, 16, true>(a, st, nblocks);
    default: return cudaErrorInvalidConfiguration;
    }
}

cudaError_t fast_cols_cp(int L, int E, const FastCols& a, cudaStream_t st, int* nblocks) {
#define CASE_C(LL)                                                     \
    case LL:                                                           \
        if constexpr (LL <= 4096) {                                    \
            if (E == 8) return go_cols_cp<LL, 8>(a, st, nblocks);      \
        }                                                              \
        if (E == 16) return go_cols_cp<LL, 16>(a, st, nblocks);        \
        break;
    switch (L) { WOS_FAST_L(CASE_C) }
#undef CASE_C
    return cudaErrorNotSupported;
}

}  // namespace wos

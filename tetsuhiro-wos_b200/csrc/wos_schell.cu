// wos_schell.cu -- the batch-only variants of the specialised sweeps,
// instantiated for E = 8 on 256 .. 4096 points apart from wos_fast.cu so the
// two compile in parallel: the two sweeps that fuse the synthesis of
// Gaussian-Schell realizations (optics/coherence.go:22-80) into their
// propagation (the first row sweep, k_rows_schell_fast, and the column sweep
// with the envelope's y factor, k_cols_fast with PRE = 1), and the column
// sweep that starts from a shared, already column-transformed spectrum
// (PRE = 2: polychromatic wavelengths and volume planes).
#include "wos_fast_kern.cuh"

namespace wos {

#define WOS_SCHELL_L(X) X(256) X(512) X(1024) X(2048) X(4096)

cudaError_t fast_rows_schell(int fp64, int L, int E, const FastRows& a, cudaStream_t st, int* nblocks) {
    if (E != 8) return cudaErrorNotSupported;
#define CASE_S(LL)                                                                             \
    case LL:                                                                                   \
        return fp64 ? go_rows_schell<double, LL, 8>(a, st, nblocks) : go_rows_schell<float, LL, 8>(a, st, nblocks);
    switch (L) { WOS_SCHELL_L(CASE_S) }
#undef CASE_S
    return cudaErrorNotSupported;
}

template <typename Real, int L, int PRE>
static cudaError_t go_cols_pre(const FastCols& a, cudaStream_t st, int* nblocks) {
    switch (fast_col_width(sizeof(Real) == 8, L, 8, a.W)) {
    case 1: return go_cols_w<Real, L, 8, 1, false, PRE>(a, st, nblocks);
    case 2: return go_cols_w<Real, L, 8, 2, false, PRE>(a, st, nblocks);
    case 4: return go_cols_w<Real, L, 8, 4, false, PRE>(a, st, nblocks);
    default: return cudaErrorInvalidConfiguration;
    }
}

cudaError_t fast_cols_env(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks) {
    if (E != 8 || !a.env_y || a.htab || a.tw_lo || a.tiled) return cudaErrorNotSupported;
#define CASE_E(LL)                                                                                      \
    case LL:                                                                                            \
        return fp64 ? go_cols_pre<double, LL, 1>(a, st, nblocks) : go_cols_pre<float, LL, 1>(a, st, nblocks);
    switch (L) { WOS_SCHELL_L(CASE_E) }
#undef CASE_E
    return cudaErrorNotSupported;
}

cudaError_t fast_cols_spec(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks) {
    if (E != 8 || a.htab || a.tw_lo || a.tiled || !a.src) return cudaErrorNotSupported;
#define CASE_P(LL)                                                                                      \
    case LL:                                                                                            \
        return fp64 ? go_cols_pre<double, LL, 2>(a, st, nblocks) : go_cols_pre<float, LL, 2>(a, st, nblocks);
    switch (L) { WOS_SCHELL_L(CASE_P) }
#undef CASE_P
    return cudaErrorNotSupported;
}

}  // namespace wos

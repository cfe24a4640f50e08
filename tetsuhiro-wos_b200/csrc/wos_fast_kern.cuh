// wos_fast_kern.cuh -- kernels of the specialised power-of-two sweeps that two
// translation units instantiate: the fused ASM column sweep (k_cols_fast) and
// the split-step row sweep (k_rows_bpm_fast), each with CP = false (wos_fast.cu)
// and, for complex64, CP = true (wos_fast_cp.cu): the compensated transforms
// of the split-step, whose twiddles and rotation constants are applied as
// hi + lo pairs.  A split-step applies the same forward / inverse transform
// pair to a slowly changing field hundreds of times, so the rounding of a
// single-precision twiddle is a fixed operator error that adds up slice after
// slice (linearly); with the pairs only the data rounding remains, which does
// not correlate between slices.
#pragma once
#include <stdlib.h>

#include "wos_fast_dev.cuh"

namespace wos {

// Sweeps are launched with programmatic stream serialization (the kernels
// call pdl_wait() before touching memory), so a sweep's CTAs are scheduled
// while the previous sweep of the stream drains; WOS_PDL=0 launches them as
// ordinary kernels.
inline bool pdl_enabled() {
    static const bool on = [] {
        const char* e = getenv("WOS_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename A>
inline cudaError_t launch_sweep(void (*k)(A), dim3 grid, int threads, size_t smem, cudaStream_t st, const A& a) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k, a);
    return e != cudaSuccess ? e : cudaGetLastError();
}

// exp(2 pi i t) - 1 as (cos - 1, sin) for |t| < 2^28 revolutions, single
// precision, from the exactly reduced fraction f (cexp_rev): cos - 1 =
// -2 sin^2(pi f) and sin = 2 sin(pi f) cos(pi f), both to ~1 ulp of their own
// size (the direct cos of a small angle would carry an error of half an ulp
// of 1).
__device__ __forceinline__ float2 cexpm1_rev(double t) {
    const double u = t + 805306368.0;  // 1.5 * 2^29
    const int s23 = (int)((unsigned)__double2loint(u) << 9) >> 9;
    const float f = __int_as_float(0x4b400000 + s23) - 12582912.0f;
    float sh, ch;
    sincospif(f * 1.1920928955078125e-07f, &sh, &ch);  // 2^-23: pi f
    return make_float2(-2.0f * sh * sh, 2.0f * sh * ch);
}

// One split-step slice on a row (optics/medium.go:50-65 for the screen): the
// inverse row transform, the screen t(x, y) = border[d] exp(i phase gx gy) at
// the inverse's natural output positions, which are the forward transform's
// natural input positions (radix rs both), and the forward row transform, all
// in registers.  The screen's phase argument and Gaussian factors are FP64 in
// both pipelines; complex64 takes sin/cos of the exactly reduced revolution
// fraction in single precision.  CP (complex64): compensated transforms
// (twiddle residuals from a.tw_lo) and the screen applied as u + u (t - 1)
// with t - 1 formed without cancellation; a phase of at most pi is taken in
// single precision directly (no reduction, so no quantisation of the angle).
template <typename Real, int L, int E, bool CP = false>
__global__ void __launch_bounds__(FMaxT<Real, E>::v) k_rows_bpm_fast(const FastRows a) {
    pdl_wait();
    pdl_trigger();
    using C = typename CT<Real>::t;
    using PL = FPlan<L, E>;
    constexpr int T = PL::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lines = blockDim.x / T;
    const int line = threadIdx.x / T, tt = threadIdx.x - line * T;
    C* smb = reinterpret_cast<C*>(smraw) + line * frow_stride(L, E);
    const int r = blockIdx.x * lines + line;
    const bool act = r < a.rows;
    const C* twp = reinterpret_cast<const C*>(a.tw);
    const C* twl = reinterpret_cast<const C*>(a.tw_lo);
    const long long ib = (long long)blockIdx.y * a.in_bstride + (long long)r * a.in_ld;
    const long long ob = (long long)blockIdx.y * a.out_bstride + (long long)r * a.out_ld;
    C v[E];
    if (act) {
        const C* in = reinterpret_cast<const C*>(a.in) + ib + tt;
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = __ldcs(in + fpos<E, E, L>(s, 0));
    } else {
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
    }
    fpasses<L, E, true, 0, 1, C, CP>(v, smb, tt, twp, twl);
    if (act) {
        const double y = ((double)r - (double)a.rows / 2) * a.bpm_dx;
        const double gy = a.bpm_gx ? exp(-((y - a.bpm_y0) * (y - a.bpm_y0)) / a.bpm_w2) : 0.0;
        const double pg = a.bpm_phase * gy;
        const int dr = min(r, a.rows - 1 - r);
        // complex64: the FP64 phase in revolutions (|gx| <= 1 bounds it by
        // |pg| / 2 pi, uniform over the row), reduced exactly and turned into
        // sin/cos in single precision (cexp_rev); complex128, or a phase too
        // large for the exact reduction: FP64 sincos
        const double prev = pg * (0.5 / M_PI);
        const bool rev = sizeof(Real) == 4 && fabs(prev) < 0x1p27;
        const bool small = CP && fabs(pg) <= M_PI;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = fpos<PL::RS, E, L>(s, tt);
            if constexpr (CP) {
                // t - 1 = b (cos - 1) + (b - 1) + i b sin
                float2 e = make_float2(0.f, 0.f);
                if (a.bpm_gx) {
                    if (small) {
                        float sh, ch;
                        sincosf(0.5f * (float)(pg * __ldg(a.bpm_gx + q)), &sh, &ch);
                        e = make_float2(-2.0f * sh * sh, 2.0f * sh * ch);
                    } else if (rev) {
                        e = cexpm1_rev(prev * __ldg(a.bpm_gx + q));
                    } else {
                        double sd, cd;
                        sincos(pg * __ldg(a.bpm_gx + q), &sd, &cd);
                        e = make_float2((float)(cd - 1.0), (float)sd);
                    }
                }
                float b = 1.f, bm1 = 0.f;
                if (a.bpm_border) {
                    const int d = min(dr, min(q, a.bpm_nx - 1 - q));
                    if (d < a.bpm_border_px) {
                        const double bd = __ldg(a.bpm_border + d);
                        b = (float)bd;
                        bm1 = (float)(bd - 1.0);
                    }
                }
                const C tm1 = mkc<C>(fmaf(b, e.x, bm1), b * e.y);
                v[s] = mkc<C>(fmaf(v[s].x, tm1.x, fmaf(-v[s].y, tm1.y, v[s].x)),
                              fmaf(v[s].x, tm1.y, fmaf(v[s].y, tm1.x, v[s].y)));
            } else {
                Real sn = 0, cs = 1;
                if (a.bpm_gx) {
                    const double g = __ldg(a.bpm_gx + q);
                    if (rev) {
                        const float2 e = cexp_rev(prev * g, true);
                        cs = (Real)e.x;
                        sn = (Real)e.y;
                    } else {
                        double sd, cd;
                        sincos(pg * g, &sd, &cd);
                        cs = (Real)cd;
                        sn = (Real)sd;
                    }
                }
                if (a.bpm_border) {
                    const int d = min(dr, min(q, a.bpm_nx - 1 - q));
                    if (d < a.bpm_border_px) {
                        const Real b = (Real)__ldg(a.bpm_border + d);
                        sn *= b;
                        cs *= b;
                    }
                }
                v[s] = cmul(v[s], mkc<C>(cs, sn));
            }
        }
    }
    fpasses<L, E, false, 0, 1, C, CP>(v, smb, tt, twp, twl);
    if (act) {
        C* out = reinterpret_cast<C*>(a.out) + ob + tt;
#pragma unroll
        for (int s = 0; s < E; s++) out[fpos<E, E, L>(s, 0)] = v[s];
    }
}

// The first row sweep of a batch of Gaussian-Schell realizations
// (GenerateSchellRealizations, optics/coherence.go:22-80, with the
// propagation's forward row transform): realization b = blockIdx.y, row r.
// The noise (complex128) times sqrt(S) (pre_map, FP64) is inverse
// transformed along x, multiplied by the x factor of the separable envelope
// sqrt(I) = exp(-x^2/w^2) exp(-y^2/w^2) (env_x, with the generation's 1/nx
// folded in) and transformed forward again.  The envelope's y factor and the
// column transforms follow in the column sweep (k_cols_fast, PRE = 1):
// operators along different axes commute, so the realization's inverse FFT2,
// its envelope and the propagation's forward FFT2 take one pass over the data
// per axis.
template <typename Real, int L, int E>
__global__ void __launch_bounds__(FMaxT<Real, E>::v) k_rows_schell_fast(const FastRows a) {
    pdl_wait();
    pdl_trigger();
    using C = typename CT<Real>::t;
    using PL = FPlan<L, E>;
    constexpr int T = PL::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int lines = blockDim.x / T;
    const int line = threadIdx.x / T, tt = threadIdx.x - line * T;
    C* smb = reinterpret_cast<C*>(smraw) + line * frow_stride(L, E);
    const int r = blockIdx.x * lines + line;
    const bool act = r < a.rows;
    const C* twp = reinterpret_cast<const C*>(a.tw);
    C v[E];
    if (act) {
        const double2* in = reinterpret_cast<const double2*>(a.in) + (long long)blockIdx.y * a.in_bstride +
                            (long long)r * a.in_ld + tt;
        const double* m = a.pre_map + (long long)r * a.in_ld + tt;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int p = fpos<E, E, L>(s, 0);
            const double2 x = __ldcs(in + p);
            const double g = __ldg(m + p);
            v[s] = mkc<C>((Real)(x.x * g), (Real)(x.y * g));
        }
    } else {
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
    }
    fpasses<L, E, true, 0, 1, C>(v, smb, tt, twp);
#pragma unroll
    for (int s = 0; s < E; s++) {
        const Real g = (Real)__ldg(a.env_x + fpos<PL::RS, E, L>(s, tt));
        v[s] = mkc<C>(v[s].x * g, v[s].y * g);
    }
    fpasses<L, E, false, 0, 1, C>(v, smb, tt, twp);
    if (act) {
        C* out = reinterpret_cast<C*>(a.out) + (long long)blockIdx.y * a.out_bstride + (long long)r * a.out_ld + tt;
#pragma unroll
        for (int s = 0; s < E; s++) out[fpos<E, E, L>(s, 0)] = v[s];
    }
}

// Fused column sweep: W adjacent columns per CTA (strided, or one contiguous
// tile in the tiled layout); forward column transform, H of asmTF
// (optics/propagate.go:159-181) from an FP64 argument or from the table
// (FastCols::htab), optional spectral sums and wrap histogram, inverse column
// transform.  CP: compensated transforms (twiddle residuals from a.tw_lo) and
// hi + lo table entries.  PRE, what precedes H: 0 the forward column
// transform of the loaded columns; 1 (Gaussian-Schell batches after
// k_rows_schell_fast) an inverse transform, the factor env_y and the forward
// transform, so H meets the realization's spectrum; 2 nothing: the source is
// already the column spectrum (a batch's shared input, transformed once), loaded
// where the forward transform would leave it.
// HG (complex64, a.htab_global): H from the table in global memory, applied
// in registers (no shared-memory spectrum stage, no H evaluation).
template <typename Real, int L, int E, int W, bool CP = false, int PRE = 0, bool HG = false>
__global__ void __launch_bounds__(FColB<Real, L, E, W>::threads, FColB<Real, L, E, W>::minb)
    k_cols_fast(const FastCols a) {
    pdl_wait();
    pdl_trigger();
    using C = typename CT<Real>::t;
    using PL = FPlan<L, E>;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    C* smb = reinterpret_cast<C*>(smraw) + w;
    const int col = blockIdx.x * W + w;
    const bool act = col < a.ncols;
    const C* twp = reinterpret_cast<const C*>(a.tw);
    const C* twl = reinterpret_cast<const C*>(a.tw_lo);
    // strided columns, or one contiguous block per tile in the tiled layout (ld == W)
    const long long coff = a.tiled ? (long long)blockIdx.x * L * W + w : (long long)col;
    C* base = reinterpret_cast<C*>(a.data) + (long long)blockIdx.y * a.bstride + coff;
    const C* sbase = a.src ? reinterpret_cast<const C*>(a.src) + (long long)blockIdx.y * a.src_bstride + coff : base;
    __shared__ double hsm[97];
    if (a.hist)
        for (int k = threadIdx.x; k < 97; k += blockDim.x) hsm[k] = 0;
    // transfer-function table rows of this tile, behind the exchange tile
    float2* hs = nullptr;
    if constexpr (sizeof(Real) == 4 && !HG) {
        if (a.htab && !a.htab_global) {
            hs = reinterpret_cast<float2*>(smraw + fcol_htab_off(L, E, W));
            htab_prefetch<W, CP>(hs, a, blockIdx.x * W);
        }
    }
    C v[E];
    if constexpr (PRE == 2) {
        if (act) {  // (shared by the batch's units: cached loads)
            const C* src = sbase + (long long)tt * a.ld;
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = __ldg(src + (long long)(s * (L / E)) * a.ld);
        } else {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
        }
    } else if constexpr (PRE == 1) {
        if (act) {
            const C* src = sbase + (long long)tt * a.ld;
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = __ldcs(src + (long long)fpos<E, E, L>(s, 0) * a.ld);
        } else {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
        }
        fpasses<L, E, true, 0, W, C, CP>(v, smb, tt, twp, twl);
#pragma unroll
        for (int s = 0; s < E; s++) {
            const Real g = (Real)__ldg(a.env_y + fpos<PL::RS, E, L>(s, tt));
            v[s] = mkc<C>(v[s].x * g, v[s].y * g);
        }
    } else {
        constexpr int R1 = PL::RS;
        if (act) {
            // a source shared by the batch's units (src_bstride 0) is read by
            // every unit: cached loads; otherwise streaming
            const C* src = sbase + (long long)tt * a.ld;
            if (a.src && a.src_bstride == 0) {
#pragma unroll
                for (int s = 0; s < E; s++) v[s] = __ldg(src + (long long)fpos<R1, E, L>(s, 0) * a.ld);
            } else {
#pragma unroll
                for (int s = 0; s < E; s++) v[s] = __ldcs(src + (long long)fpos<R1, E, L>(s, 0) * a.ld);
            }
        } else {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
        }
    }
    // interleaved tile: stride W between consecutive positions of a column
    if constexpr (PRE != 2) fpasses<L, E, false, 0, W, C, CP>(v, smb, tt, twp, twl);

    double p0 = 0, l1 = 0;
    if constexpr (HG) {
        // v[s] holds frequency q = tt + s*T, where the inverse transform
        // starts: H(|fx|, |fy|) from the table row of this column (CP: hi + lo
        // entries, applied as x H_hi + x H_lo)
        static_assert(sizeof(Real) == 4, "table in registers: complex64 sweeps");
        if (act) {
            const int cabs = col <= a.ncols / 2 ? col : a.ncols - col;
            const float sg = a.conj ? -1.f : 1.f;
            if constexpr (CP) {
                const float4* hr = reinterpret_cast<const float4*>(a.htab) + (long long)cabs * a.htab_ld;
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int q = tt + s * (L / E);
                    const float4 t = __ldg(hr + (q <= L / 2 ? q : L - q));
                    v[s] = cmul_cp(v[s], mkc<C>(t.x, sg * t.y), mkc<C>(t.z, sg * t.w));
                }
            } else {
                const float2* hr = a.htab + (long long)cabs * a.htab_ld;
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int q = tt + s * (L / E);
                    const float2 t = __ldg(hr + (q <= L / 2 ? q : L - q));
                    v[s] = cmul(v[s], mkc<C>(t.x, sg * t.y));
                }
            }
        }
    } else {
        col_spectral_stage<Real, L, E, W, C, CP>(v, reinterpret_cast<C*>(smraw), hsm, blockIdx.x * W, a,
                                                 h_unit(a, blockIdx.y), p0, l1, hs);
    }
    fpasses<L, E, true, 0, W, C, CP>(v, smb, tt, twp, twl);
    if (act) {
        constexpr int RO = PL::RS;
        C* dst = base + (long long)tt * a.ld;
#pragma unroll
        for (int s = 0; s < E; s++) dst[(long long)fpos<RO, E, L>(s, 0) * a.ld] = v[s];
    }
    col_write_red(a, (long long)blockIdx.y * gridDim.x + blockIdx.x, p0, l1, hsm);
}

// ------------------------------------------------------------------ launch
template <typename Real, int L, int E, bool CP = false>
inline cudaError_t go_rows_bpm(const FastRows& a, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    const int lines = fast_row_lines(L, E, a.rows);
    const size_t smem = (size_t)frow_stride(L, E) * lines * sizeof(typename CT<Real>::t);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows_bpm_fast<Real, L, E, CP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((a.rows + lines - 1) / lines, a.batch > 0 ? a.batch : 1);
    if (nblocks) *nblocks = (int)(grid.x * grid.y);
    return launch_sweep(k_rows_bpm_fast<Real, L, E, CP>, grid, lines * T, smem, st, a);
}

template <typename Real, int L, int E>
inline cudaError_t go_rows_schell(const FastRows& a, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    const int lines = fast_row_lines(L, E, a.rows);
    const size_t smem = (size_t)frow_stride(L, E) * lines * sizeof(typename CT<Real>::t);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows_schell_fast<Real, L, E>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((a.rows + lines - 1) / lines, a.batch > 0 ? a.batch : 1);
    if (nblocks) *nblocks = (int)(grid.x * grid.y);
    return launch_sweep(k_rows_schell_fast<Real, L, E>, grid, lines * T, smem, st, a);
}

template <typename Real, int L, int E, int W, bool CP = false, int PRE = 0, bool HG = false>
inline cudaError_t go_cols_w(const FastCols& a, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    if constexpr (W * T < 32 || W * T > fcol_max_threads(sizeof(Real) == 8, T)) {
        return cudaErrorInvalidConfiguration;
    } else {
        size_t smem = (size_t)fcol_elems(L, E, W) * sizeof(typename CT<Real>::t);
        if (sizeof(Real) == 4 && a.htab && !a.htab_global && !HG)
            smem = fcol_htab_off(L, E, W) + (size_t)W * a.htab_ld * sizeof(float2) * (CP ? 2 : 1);
        if (smem > kSmemNoOptIn) {
            cudaError_t e = cudaFuncSetAttribute(k_cols_fast<Real, L, E, W, CP, PRE, HG>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        dim3 grid((a.ncols + W - 1) / W, a.batch > 0 ? a.batch : 1);
        if (nblocks) *nblocks = (int)(grid.x * grid.y);
        return launch_sweep(k_cols_fast<Real, L, E, W, CP, PRE, HG>, grid, W * T, smem, st, a);
    }
}

}  // namespace wos

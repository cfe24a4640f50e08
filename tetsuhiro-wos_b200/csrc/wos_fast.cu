// wos_fast.cu -- compile-time specialised sweeps of the band-limited ASM hot
// path (power-of-two lines).  The transform length L and the elements per
// thread E are template parameters, so every pass radix, Stockham stride,
// shared-memory offset and twiddle offset is a compile-time constant:
//  * shared memory is padded (one slot per 2^SH positions) so that each
//    exchange is conflict-free and every address is a per-thread base plus an
//    immediate (the padding commutes with the pass strides, see padq below);
//  * twiddles come from per-pass tables W_{NS R}^{r k} laid out [r][k]
//    (generated in FP64, rounded once), so the threads of a warp read
//    consecutive entries and each load is base + immediate.
//
//   k_rows_fast<Real, L, E, INV>: one row per T = L/E threads, coalesced
//       loads straight into registers, optional complex128 conversion and
//       sum |E|^2, coalesced stores.
//   k_cols_fast<Real, L, E>: W adjacent columns per CTA; forward column FFT,
//       H(fx, fy) of asmTF (optics/propagate.go:159-181) generated on the fly
//       from an FP64 argument, inverse column FFT, optional spectral loss sums.
#include <stdlib.h>

#include <cooperative_groups.h>

#include "wos_fast_kern.cuh"

namespace wos {

namespace cg = cooperative_groups;

// ------------------------------------------------------------------- rows
// (Holding the FP32 E = 16 rows to 48 registers for five resident 256-thread
// CTAs per SM instead of four measured slower: 24.8 against 23.7 us per
// 2048^2 sweep.)
template <typename Real, int L, int E, bool INV>
__global__ void __launch_bounds__(FMaxT<Real, E>::v) k_rows_fast(const FastRows a) {
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
    constexpr int R1 = INV ? E : PL::RS;
    constexpr int RO = INV ? PL::RS : E;
    const long long ib = (long long)blockIdx.y * a.in_bstride + (long long)r * a.in_ld;
    const long long ob = (long long)blockIdx.y * a.out_bstride + (long long)r * a.out_ld;
    C v[E];
    double pw = 0;
    if (act) {
        if (a.in_c128) {
            const double2* in = reinterpret_cast<const double2*>(a.in) + ib + tt;
#pragma unroll
            for (int s = 0; s < E; s++) {
                const double2 d = in[fpos<R1, E, L>(s, 0)];
                v[s] = mkc<C>((Real)d.x, (Real)d.y);
            }
        } else if (INV && a.in_tiled) {
            // x = tt + s*T (R1 == E): tile (tt / kTileW) + s * (T / kTileW), lane tt % kTileW
            static_assert(!INV || R1 == E, "tiled loads follow the natural mapping of radix E");
            const long long tstride = a.tile_len * kTileW;
            const C* in = reinterpret_cast<const C*>(a.in) + (long long)blockIdx.y * a.in_bstride +
                          (long long)r * kTileW + (long long)(tt / kTileW) * tstride + (tt % kTileW);
            const long long step = (long long)(T / kTileW) * tstride;
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = __ldcs(in + s * step);
        } else {
            const C* in = reinterpret_cast<const C*>(a.in) + ib + tt;
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = __ldcs(in + fpos<R1, E, L>(s, 0));
        }
        if (a.red && !INV) {
#pragma unroll
            for (int s = 0; s < E; s++) pw += (double)v[s].x * v[s].x + (double)v[s].y * v[s].y;
        }
    } else {
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
    }
    fpasses<L, E, INV, 0, 1>(v, smb, tt, twp);
    if (act) {
        if (a.out_scale_im != 0.0) {
            const C cs = mkc<C>((Real)a.out_scale, (Real)a.out_scale_im);
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = cmul(v[s], cs);
        } else if (a.out_scale != 1.0) {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = cscale(v[s], (Real)a.out_scale);
        }
        if (a.red && INV) {
#pragma unroll
            for (int s = 0; s < E; s++) pw += (double)v[s].x * v[s].x + (double)v[s].y * v[s].y;
        }
        if (a.out_c128) {
            double2* out = reinterpret_cast<double2*>(a.out) + ob + tt;
#pragma unroll
            for (int s = 0; s < E; s++) out[fpos<RO, E, L>(s, 0)] = make_double2(v[s].x, v[s].y);
        } else if (!INV && a.out_tiled) {
            static_assert(INV || RO == E, "tiled stores follow the natural mapping of radix E");
            const long long tstride = a.tile_len * kTileW;
            C* out = reinterpret_cast<C*>(a.out) + (long long)blockIdx.y * a.out_bstride + (long long)r * kTileW +
                     (long long)(tt / kTileW) * tstride + (tt % kTileW);
            const long long step = (long long)(T / kTileW) * tstride;
#pragma unroll
            for (int s = 0; s < E; s++) out[s * step] = v[s];
        } else if (INV && a.out_stream) {
            // the propagation's result: streaming stores leave L2 to the
            // intermediates of the fields still in flight
            C* out = reinterpret_cast<C*>(a.out) + ob + tt;
#pragma unroll
            for (int s = 0; s < E; s++) __stcs(out + fpos<RO, E, L>(s, 0), v[s]);
        } else {
            C* out = reinterpret_cast<C*>(a.out) + ob + tt;
#pragma unroll
            for (int s = 0; s < E; s++) out[fpos<RO, E, L>(s, 0)] = v[s];
        }
    }
    if (a.red) {
        // per-CTA partial of sum |E|^2 (slot 0 of a record of stride red_stride)
        __shared__ double rsm[32];
        for (int o = 16; o > 0; o >>= 1) pw += __shfl_down_sync(0xffffffffu, pw, o);
        if ((threadIdx.x & 31) == 0) rsm[threadIdx.x >> 5] = pw;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += rsm[w];
            a.red[((long long)blockIdx.y * gridDim.x + blockIdx.x) * a.red_stride] = t;
        }
    }
}

// Inverse-design row stages (see DesignArgs).  Positions q of a row follow
// the natural order of radix rs (the forward transform's input order, the
// inverse's output order), so every pointwise step sits between two
// transforms in registers.
template <typename Real, int L, int E, int STAGE>
__global__ void __launch_bounds__(FMaxT<Real, E>::v) k_rows_design(const FastRows a, const DesignArgs d) {
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
    const long long row = (long long)r * L;
    C v[E];
    double loss = 0;
    if (STAGE == 0) {
        if (act) {
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int q = fpos<PL::RS, E, L>(s, tt);
                double sn, cs;
                sincos(__ldg(d.phi + row + q), &sn, &cs);
                double ar, ai;
                if (d.amp_c128) {
                    const double2 x = reinterpret_cast<const double2*>(d.amp)[row + q];
                    ar = x.x;
                    ai = x.y;
                } else {
                    const C x = reinterpret_cast<const C*>(d.amp)[row + q];
                    ar = x.x;
                    ai = x.y;
                }
                v[s] = mkc<C>((Real)(cs * ar - sn * ai), (Real)(cs * ai + sn * ar));
            }
        } else {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
        }
    } else {
        if (act) {
            const C* in = reinterpret_cast<const C*>(a.in) + row + tt;
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = __ldcs(in + fpos<E, E, L>(s, 0));
        } else {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
        }
        fpasses<L, E, true, 0, 1>(v, smb, tt, twp);
    }
    if (STAGE == 1 && act) {
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = fpos<PL::RS, E, L>(s, tt);
            const double ur = v[s].x, ui = v[s].y;
            const double dd = ur * ur + ui * ui - __ldg(d.target + row + q);
            loss += dd * dd;
            v[s] = mkc<C>((Real)(4 * dd * ur), (Real)(4 * dd * ui));
        }
    }
    if (STAGE == 2) {
        if (act) {
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int q = fpos<PL::RS, E, L>(s, tt);
                double sn, cs;
                sincos(__ldg(d.phi + row + q), &sn, &cs);
                double ar, ai;
                if (d.amp_c128) {
                    const double2 x = reinterpret_cast<const double2*>(d.amp)[row + q];
                    ar = x.x;
                    ai = x.y;
                } else {
                    const C x = reinterpret_cast<const C*>(d.amp)[row + q];
                    ar = x.x;
                    ai = x.y;
                }
                // i t a = (-Im(t a), Re(t a))
                const double tr = cs * ar - sn * ai, ti = cs * ai + sn * ar;
                d.grad[row + q] = (double)v[s].x * (-ti) + (double)v[s].y * tr;
            }
        }
    } else {
        fpasses<L, E, false, 0, 1>(v, smb, tt, twp);
        if (act) {
            C* out = reinterpret_cast<C*>(a.out) + row + tt;
#pragma unroll
            for (int s = 0; s < E; s++) out[fpos<E, E, L>(s, 0)] = v[s];
        }
    }
    if (STAGE == 1 && a.red) {
        __shared__ double rsm[32];
        for (int o = 16; o > 0; o >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, o);
        if ((threadIdx.x & 31) == 0) rsm[threadIdx.x >> 5] = loss;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += rsm[w];
            a.red[(long long)blockIdx.x * a.red_stride] = t;
        }
    }
}

// Inverse row transforms of the nb units of a batch with their weighted
// intensity accumulated in registers (PropagatePolychromatic /
// AverageIntensity, optics/polychromatic.go:18-44, coherence.go:82-101); one
// FP64 store per element.
template <typename Real, int L, int E>
__global__ void __launch_bounds__(FMaxT<Real, E>::v) k_rows_acc_fast(const FastRows a, const AccArgs acc) {
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
    Real sum[E];
#pragma unroll
    for (int s = 0; s < E; s++) sum[s] = 0;
    for (int u = 0; u < acc.nb; u++) {
        C v[E];
        if (act) {
            const C* in = reinterpret_cast<const C*>(a.in) + (long long)u * a.in_bstride + (long long)r * a.in_ld + tt;
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = __ldcs(in + fpos<E, E, L>(s, 0));
        } else {
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
        }
        fpasses<L, E, true, 0, 1>(v, smb, tt, twp);
        const double w = acc.weight ? acc.weight[u] : 1.0;
#pragma unroll
        for (int s = 0; s < E; s++) sum[s] += (Real)(w * ((double)v[s].x * v[s].x + (double)v[s].y * v[s].y));
    }
    if (act) {
        double* out = acc.out + (long long)r * L + tt;
#pragma unroll
        for (int s = 0; s < E; s++) {
            double* o = out + fpos<PL::RS, E, L>(s, 0);
            *o = (acc.add ? *o : 0.0) + (double)sum[s];
        }
    }
}

// ------------------------------------------------------------- split tiles
// H on the half spectrum a CTA of a pair holds: local index k of rank r is the
// frequency q = 2k + r.  The partner of q, L - q, is local LH - k (rank 0; k = 0
// and the Nyquist row k = LH/2 pair with themselves) or LH - 1 - k (rank 1), so
// each pair stays in one CTA and H is evaluated once for both.
template <int L, int E, int W>
__device__ __forceinline__ void col_tile_h_pair(float2* tile, int r, int col0, const FastCols& a, const HUnit& hu,
                                                double& p0, double& l1) {
    constexpr int LH = L / 2, T = LH / E;
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    const int col = col0 + w;
    if (col >= a.ncols) return;  // zero columns stay zero
    const bool red = a.red != nullptr;
    auto apply = [&](int k, const float2 h, double m2) {
        float2 x = tile[k * W + w];
        if (red) {
            const double pp = (double)x.x * x.x + (double)x.y * x.y;
            p0 += pp;
            l1 += pp * (1.0 - m2);
        }
        tile[k * W + w] = cmul(x, h);
    };
    const double fx = (col <= a.ncols / 2 ? (double)col : (double)(col - a.ncols)) / ((double)a.ncols * a.dx);
    const double ax = hu.wl * fx;
    const double cx = fma(-ax, ax, 1.0);
    const double g = hu.wl / ((double)L * a.dx);
    const double tg = 2.0 * (double)T * g, ay0 = (2.0 * (double)tt + (double)r) * g;
#pragma unroll
    for (int i = 0; i < E / 2; i++) {
        const int k = tt + i * T;
        double m2;
        const float2 h = h_f32(a, hu, cx, fma((double)i, tg, ay0), m2);
        apply(k, h, m2);
        if (r == 0) {
            if (k != 0) apply(LH - k, h, m2);
        } else {
            apply(LH - 1 - k, h, m2);
        }
    }
    if (r == 0 && tt == 0) {
        double m2;
        const float2 h = h_f32(a, hu, cx, (double)LH * g, m2);
        apply(LH / 2, h, m2);
    }
}

// Fused column sweep with a tile of W columns split over a two-CTA cluster:
// rank r holds rows [r L/2, (r+1) L/2) of the tile, in 512 threads and 80 KB
// of shared memory, so two CTAs are resident per SM and one's global-memory
// phases overlap the other's transforms (a whole-column CTA needs the full
// register file).  Forward: one radix-2 decimation-in-frequency step across
// the pair through distributed shared memory (rank 0 keeps x[n] + x[n+L/2],
// rank 1 (x[n] - x[n+L/2]) W_L^n), then a local L/2 transform gives the even
// (rank 0) or odd (rank 1) frequencies.  After H, the local inverse and the
// mirrored step: x[n] = e[n] + W_L^-n o[n] (rank 0), x[n+L/2] = e[n] -
// W_L^-n o[n] (rank 1).  Every thread of both CTAs reaches the four cluster
// barriers; a CTA's shared memory is read by its partner only between them.
template <int L, int E, int W>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(W * (L / 2 / E), 2) k_cols_pair(const FastCols a) {
    using C = float2;
    constexpr int LH = L / 2;
    using PL = FPlan<LH, E>;
    constexpr int T = PL::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    cg::cluster_group cl = cg::this_cluster();
    const int r = (int)cl.block_rank();
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    C* tile = reinterpret_cast<C*>(smraw);
    C* smb = tile + w;
    const C* ptile = cl.map_shared_rank(tile, r ^ 1);
    const int col0 = (int)(blockIdx.x >> 1) * W;
    const int col = col0 + w;
    const bool act = col < a.ncols;
    const C* twh = reinterpret_cast<const C*>(a.tw_half);
    const C* twl = reinterpret_cast<const C*>(a.tw_pair);
    const long long roff = (long long)r * LH * a.ld;
    C* base = reinterpret_cast<C*>(a.data) + (long long)blockIdx.y * a.bstride + col + roff;
    const C* sbase =
        a.src ? reinterpret_cast<const C*>(a.src) + (long long)blockIdx.y * a.src_bstride + col + roff : base;
    constexpr int R1 = PL::RS;  // first forward pass (natural mapping on load)
    constexpr int RO = PL::RS;  // last inverse pass (natural mapping on store)
    C v[E];
    if (act) {
        const C* src = sbase + (long long)tt * a.ld;
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = __ldcs(src + (long long)fpos<R1, E, LH>(s, 0) * a.ld);
    } else {
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
    }
#pragma unroll
    for (int s = 0; s < E; s++) tile[fpos<R1, E, LH>(s, tt) * W + w] = v[s];
    cl.sync();
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int n = fpos<R1, E, LH>(s, tt);
        const C y = ptile[n * W + w];
        if (r == 0) v[s] = make_float2(v[s].x + y.x, v[s].y + y.y);
        else v[s] = cmul(make_float2(y.x - v[s].x, y.y - v[s].y), ldg_keep(twl + n));
    }
    cl.sync();  // the partner has read this CTA's tile
    fpasses<LH, E, false, 0, W>(v, smb, tt, twh);

    double p0 = 0, l1 = 0;
    __syncthreads();
#pragma unroll
    for (int s = 0; s < E; s++) tile[(tt + s * T) * W + w] = v[s];
    __syncthreads();
    col_tile_h_pair<L, E, W>(tile, r, col0, a, h_unit(a, blockIdx.y), p0, l1);
    __syncthreads();
#pragma unroll
    for (int s = 0; s < E; s++) v[s] = tile[(tt + s * T) * W + w];
    fpasses<LH, E, true, 0, W>(v, smb, tt, twh);

    __syncthreads();
#pragma unroll
    for (int s = 0; s < E; s++) tile[fpos<RO, E, LH>(s, tt) * W + w] = v[s];
    cl.sync();
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int n = fpos<RO, E, LH>(s, tt);
        const C y = ptile[n * W + w];
        C t = ldg_keep(twl + n);
        t.y = -t.y;
        if (r == 0) {
            const C o = cmul(t, y);
            v[s] = make_float2(v[s].x + o.x, v[s].y + o.y);
        } else {
            const C o = cmul(t, v[s]);
            v[s] = make_float2(y.x - o.x, y.y - o.y);
        }
    }
    cl.sync();  // the partner has read this CTA's tile
    if (act) {
        C* dst = base + (long long)tt * a.ld;
#pragma unroll
        for (int s = 0; s < E; s++) dst[(long long)fpos<RO, E, LH>(s, 0) * a.ld] = v[s];
    }
    col_write_red(a, (long long)blockIdx.y * gridDim.x + blockIdx.x, p0, l1, nullptr);
}

bool fast_cols_pair_case(int fp64, int L, int E, int W) { return !fp64 && L == 2048 && E == 16 && W == 8; }

cudaError_t fast_cols_pair(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks) {
    if (!fast_cols_pair_case(fp64, L, E, fast_col_width(fp64, L, E, a.W)) || a.hist || !a.tw_half || !a.tw_pair)
        return cudaErrorNotSupported;
    constexpr int LL = 2048, EE = 16, WW = 8;
    const size_t smem = (size_t)fcol_elems(LL / 2, EE, WW) * sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(k_cols_pair<LL, EE, WW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(2 * ((a.ncols + WW - 1) / WW), a.batch > 0 ? a.batch : 1);
    if (nblocks) *nblocks = (int)(grid.x * grid.y);
    k_cols_pair<LL, EE, WW><<<grid, WW * (LL / 2 / EE), smem, st>>>(a);
    return cudaGetLastError();
}

// W_L^n = exp(-2 pi i n / L), n < L/2
template <typename C>
__global__ void k_pair_twiddles(C* out, int L) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L / 2) return;
    double s, c;
    sincospi(-2.0 * (double)n / (double)L, &s, &c);
    out[n] = mkc<C>((decltype(C::x))c, (decltype(C::x))s);
}
cudaError_t fast_build_pair_twiddles(int fp64, int L, void* out, cudaStream_t st) {
    const int g = (L / 2 + 255) / 256;
    if (fp64) k_pair_twiddles<double2><<<g, 256, 0, st>>>(reinterpret_cast<double2*>(out), L);
    else k_pair_twiddles<float2><<<g, 256, 0, st>>>(reinterpret_cast<float2*>(out), L);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ tables
// Quarter-plane table of the complex64 transfer function: entry [c][q] =
// scale * H(|fx_c|, |fy_q|) of asmTF (optics/propagate.go:159-181) evaluated
// in FP64 in the reference's operation order (h_f64) and rounded once; hilo:
// entries are (H_hi, H_lo) float4 pairs, H_lo = (float)(H - H_hi), for the
// compensated sweeps.
__global__ void k_htab_build(const FastCols a, int L, float2* out, int ld, int hilo) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int cx = blockIdx.y;
    if (q >= ld) return;
    double2 h = make_double2(0.0, 0.0);
    if (q <= L / 2) {
        const HUnit hu{a.wl, a.kz, a.kaz, a.krev};
        const double fxe = __ddiv_rn((double)cx, __dmul_rn((double)a.ncols, a.dx));
        const double px = fabs(__dmul_rn(hu.wl, fxe));
        const double fy = __ddiv_rn((double)q, __dmul_rn((double)L, a.dx));
        double m2;
        h = h_f64(a, hu, px, fy, m2);
    }
    if (hilo == 2) {  // complex128 entries (the FP64 pipeline)
        reinterpret_cast<double2*>(out)[(long long)cx * ld + q] = h;
        return;
    }
    const float hx = (float)h.x, hy = (float)h.y;
    if (hilo) {
        reinterpret_cast<float4*>(out)[(long long)cx * ld + q] =
            make_float4(hx, hy, (float)(h.x - (double)hx), (float)(h.y - (double)hy));
    } else {
        out[(long long)cx * ld + q] = make_float2(hx, hy);
    }
}

cudaError_t fast_build_htab(const FastCols& a, int L, float2* out, int ld, int hilo, cudaStream_t st) {
    FastCols b = a;
    b.conj = 0;
    b.batch_wl = nullptr;
    b.batch_z = nullptr;
    dim3 grid((ld + 255) / 256, a.ncols / 2 + 1);
    k_htab_build<<<grid, 256, 0, st>>>(b, L, out, ld, hilo);
    return cudaGetLastError();
}

size_t fast_col_smem_htab(int L, int E, int W, int ld, int hilo) {
    return fcol_htab_off(L, E, W) + (size_t)W * ld * (hilo ? 16 : 8);
}

// Residuals of the complex64 per-pass table: (float)(W - (double)(float)W).
__global__ void k_pass_twiddles_lo(float2* out, int off, int NS, int R) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NS * (R - 1)) return;
    const int r = i / NS + 1, k = i % NS;
    double s, c;
    sincospi(-2.0 * (double)r * (double)k / ((double)NS * (double)R), &s, &c);
    out[off + i] = make_float2((float)(c - (double)(float)c), (float)(s - (double)(float)s));
}

cudaError_t fast_build_twiddles_lo(int L, int E, void* out, cudaStream_t st) {
    int LG = 0, LE = 0;
    while ((1 << LG) < L) LG++;
    while ((1 << LE) < E) LE++;
    const int P = (LG + LE - 1) / LE;
    const int RS = (LG % LE) ? (1 << (LG % LE)) : E;
    for (int d = 0; d < 2; d++) {
        const bool inv = d == 1;
        for (int p = 1; p < P; p++) {
            const int NS = fp_ns(P, RS, E, inv, p), R = fp_radix(P, RS, E, inv, p);
            const int off = fp_twoff(P, RS, E, inv, p);
            const int n = NS * (R - 1);
            k_pass_twiddles_lo<<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<float2*>(out), off, NS, R);
        }
    }
    return cudaGetLastError();
}
// Per-pass twiddles W_{NS R}^{r k} (forward sign), [r-1][k], FP64 -> pipeline type.
template <typename C>
__global__ void k_pass_twiddles(C* out, int off, int NS, int R) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NS * (R - 1)) return;
    const int r = i / NS + 1, k = i % NS;
    double s, c;
    sincospi(-2.0 * (double)r * (double)k / ((double)NS * (double)R), &s, &c);
    out[off + i] = mkc<C>((decltype(C::x))c, (decltype(C::x))s);
}

int fast_table_len(int L, int E) {
    int LG = 0, LE = 0;
    while ((1 << LG) < L) LG++;
    while ((1 << LE) < E) LE++;
    const int P = (LG + LE - 1) / LE;
    const int RS = (LG % LE) ? (1 << (LG % LE)) : E;
    return fp_twoff(P, RS, E, true, P) + 1;  // past the last inverse pass
}

cudaError_t fast_build_twiddles(int fp64, int L, int E, void* out, cudaStream_t st) {
    int LG = 0, LE = 0;
    while ((1 << LG) < L) LG++;
    while ((1 << LE) < E) LE++;
    const int P = (LG + LE - 1) / LE;
    const int RS = (LG % LE) ? (1 << (LG % LE)) : E;
    for (int d = 0; d < 2; d++) {
        const bool inv = d == 1;
        for (int p = 1; p < P; p++) {
            const int NS = fp_ns(P, RS, E, inv, p), R = fp_radix(P, RS, E, inv, p);
            const int off = fp_twoff(P, RS, E, inv, p);
            const int n = NS * (R - 1);
            if (fp64) k_pass_twiddles<double2><<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<double2*>(out), off, NS, R);
            else k_pass_twiddles<float2><<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<float2*>(out), off, NS, R);
        }
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------ launch
// Threads per row CTA: lines of T threads are grouped up to this size.  Small
// CTAs spread the lines of a sweep evenly over the SMs and let each CTA finish
// on its own (1024^2 split-step slices: 9.99 ms per 400-slice run at 256
// threads, 9.44 ms at 64; 2048^2 rows 22.7 -> 22.1 us); lines of 32 threads or
// fewer go four to a CTA (512^2: 13.3 -> 12.3 us per propagation).
// WOS_ROW_THREADS (64, 128, 256 or 512) overrides the choice.
static int row_cta_target(int T) {
    static const int over = [] {
        const char* e = getenv("WOS_ROW_THREADS");
        const int v = e ? atoi(e) : 0;
        return (v == 64 || v == 128 || v == 256 || v == 512) ? v : 0;
    }();
    if (over) return over;
    return T <= 32 ? 128 : 64;
}

// Lines per CTA of the fast row sweeps: grouped up to row_cta_target
// threads, at least one warp.  The host sizes the per-CTA reduction records
// from this count (fast_row_blocks), so every row launcher takes it from here.
int fast_row_lines(int L, int E, int rows) {
    const int T = L / E;
    int lines = 1;
    while (lines * 2 * T <= row_cta_target(T) && lines * 2 <= rows) lines *= 2;
    while (lines * T < 32) lines *= 2;
    return lines;
}

template <typename Real, int L, int E, bool INV>
static cudaError_t go_rows(const FastRows& a, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    const int lines = fast_row_lines(L, E, a.rows);
    if (lines * T > FMaxT<Real, E>::v) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)frow_stride(L, E) * lines * sizeof(typename CT<Real>::t);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows_fast<Real, L, E, INV>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((a.rows + lines - 1) / lines, a.batch > 0 ? a.batch : 1);
    if (nblocks) *nblocks = (int)(grid.x * grid.y);
    return launch_sweep(k_rows_fast<Real, L, E, INV>, grid, lines * T, smem, st, a);
}

template <typename Real, int L, int E>
static cudaError_t go_rows_acc(const FastRows& a, const AccArgs& acc, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    const int lines = fast_row_lines(L, E, a.rows);
    const size_t smem = (size_t)frow_stride(L, E) * lines * sizeof(typename CT<Real>::t);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows_acc_fast<Real, L, E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((a.rows + lines - 1) / lines, 1);
    if (nblocks) *nblocks = (int)grid.x;
    k_rows_acc_fast<Real, L, E><<<grid, lines * T, smem, st>>>(a, acc);
    return cudaGetLastError();
}

template <typename Real, int L, int E, int STAGE>
static cudaError_t go_rows_design(const FastRows& a, const DesignArgs& d, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    const int lines = fast_row_lines(L, E, a.rows);
    const size_t smem = (size_t)frow_stride(L, E) * lines * sizeof(typename CT<Real>::t);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows_design<Real, L, E, STAGE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((a.rows + lines - 1) / lines, 1);
    if (nblocks) *nblocks = (int)grid.x;
    k_rows_design<Real, L, E, STAGE><<<grid, lines * T, smem, st>>>(a, d);
    return cudaGetLastError();
}

template <typename Real, int L, int E>
static cudaError_t go_rows_design_s(int stage, const FastRows& a, const DesignArgs& d, cudaStream_t st, int* nb) {
    switch (stage) {
    case 0: return go_rows_design<Real, L, E, 0>(a, d, st, nb);
    case 1: return go_rows_design<Real, L, E, 1>(a, d, st, nb);
    default: return go_rows_design<Real, L, E, 2>(a, d, st, nb);
    }
}

template <typename Real, int L, int E>
static cudaError_t go_cols(const FastCols& a, cudaStream_t st, int* nblocks) {
    if constexpr (sizeof(Real) == 4) {  // H from the table, in registers: widths 4 (the tiled layout) and 8
        if (a.htab_global) {
            const int w = fast_col_width(0, L, E, a.W);
            if (w == kTileW) return go_cols_w<float, L, E, kTileW, false, 0, true>(a, st, nblocks);
            if (w == 8) return go_cols_w<float, L, E, 8, false, 0, true>(a, st, nblocks);
        }
    }
    switch (fast_col_width(sizeof(Real) == 8, L, E, a.W)) {
    case 1: return go_cols_w<Real, L, E, 1>(a, st, nblocks);
    case 2: return go_cols_w<Real, L, E, 2>(a, st, nblocks);
    case 4: return go_cols_w<Real, L, E, 4>(a, st, nblocks);
    case 8: return go_cols_w<Real, L, E, 8>(a, st, nblocks);
    case 16: return go_cols_w<Real, L, E, 16>(a, st, nblocks);
    default: return cudaErrorInvalidConfiguration;
    }
}

#define WOS_FAST_L(X) X(256) X(512) X(1024) X(2048) X(4096) X(8192)

cudaError_t fast_rows(int fp64, int L, int E, bool inv, const FastRows& a, cudaStream_t st, int* nblocks) {
#define CASE_R(LL)                                                                                  \
    case LL:                                                                                        \
        if (fp64) {                                                                                 \
            if constexpr (LL <= 4096) {                                                             \
                if (E == 8) return inv ? go_rows<double, LL, 8, true>(a, st, nblocks)               \
                                       : go_rows<double, LL, 8, false>(a, st, nblocks);             \
            } else {                                                                                \
                if (E == 16) return inv ? go_rows<double, LL, 16, true>(a, st, nblocks)             \
                                        : go_rows<double, LL, 16, false>(a, st, nblocks);           \
            }                                                                                       \
        } else {                                                                                    \
            if constexpr (LL <= 4096) {                                                             \
                if (E == 8) return inv ? go_rows<float, LL, 8, true>(a, st, nblocks)                \
                                       : go_rows<float, LL, 8, false>(a, st, nblocks);              \
            }                                                                                       \
            if (E == 16) return inv ? go_rows<float, LL, 16, true>(a, st, nblocks)                  \
                                    : go_rows<float, LL, 16, false>(a, st, nblocks);                \
        }                                                                                           \
        break;
    switch (L) { WOS_FAST_L(CASE_R) }
#undef CASE_R
    return cudaErrorNotSupported;
}

cudaError_t fast_cols(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks) {
    if (!fp64 && a.tw_lo) return fast_cols_cp(L, E, a, st, nblocks);
#define CASE_C(LL)                                                                  \
    case LL:                                                                        \
        if (fp64) {                                                                 \
            if constexpr (LL <= 4096) {                                             \
                if (E == 8) return go_cols<double, LL, 8>(a, st, nblocks);          \
            } else {                                                                \
                if (E == 16) return go_cols<double, LL, 16>(a, st, nblocks);        \
            }                                                                       \
        } else {                                                                    \
            if constexpr (LL <= 4096) {                                             \
                if (E == 8) return go_cols<float, LL, 8>(a, st, nblocks);           \
            }                                                                       \
            if (E == 16) return go_cols<float, LL, 16>(a, st, nblocks);             \
        }                                                                           \
        break;
    switch (L) { WOS_FAST_L(CASE_C) }
#undef CASE_C
    return cudaErrorNotSupported;
}

// Columns per CTA actually launched for a requested width W: raised until a CTA
// holds a full warp, lowered until it fits the kernel's thread bound; 0 if
// no width fits.
int fast_col_width(int fp64, int L, int E, int W) {
    const int T = L / E;
    const int maxt = fcol_max_threads(fp64 != 0, T);
    if (W < 1) W = 1;
    while (W * T < 32) W *= 2;
    while (W > 1 && W * T > maxt) W /= 2;
    if (W > 16 || W * T > maxt || W * T < 32) return 0;
    return W;
}

cudaError_t fast_rows_bpm(int fp64, int L, int E, const FastRows& a, cudaStream_t st, int* nblocks) {
    if (!fp64 && a.tw_lo) return fast_rows_bpm_cp(L, E, a, st, nblocks);
#define CASE_B(LL)                                                                   \
    case LL:                                                                         \
        if (fp64) {                                                                  \
            if constexpr (LL <= 4096) {                                              \
                if (E == 8) return go_rows_bpm<double, LL, 8>(a, st, nblocks);       \
            } else {                                                                 \
                if (E == 16) return go_rows_bpm<double, LL, 16>(a, st, nblocks);     \
            }                                                                        \
        } else {                                                                     \
            if constexpr (LL <= 4096) {                                              \
                if (E == 8) return go_rows_bpm<float, LL, 8>(a, st, nblocks);        \
            }                                                                        \
            if (E == 16) return go_rows_bpm<float, LL, 16>(a, st, nblocks);          \
        }                                                                            \
        break;
    switch (L) { WOS_FAST_L(CASE_B) }
#undef CASE_B
    return cudaErrorNotSupported;
}

cudaError_t fast_rows_acc(int fp64, int L, int E, const FastRows& a, const AccArgs& acc, cudaStream_t st,
                          int* nblocks) {
#define CASE_A(LL)                                                                    \
    case LL:                                                                          \
        if (fp64) {                                                                   \
            if constexpr (LL <= 4096) {                                               \
                if (E == 8) return go_rows_acc<double, LL, 8>(a, acc, st, nblocks);   \
            } else {                                                                  \
                if (E == 16) return go_rows_acc<double, LL, 16>(a, acc, st, nblocks); \
            }                                                                         \
        } else {                                                                      \
            if constexpr (LL <= 4096) {                                               \
                if (E == 8) return go_rows_acc<float, LL, 8>(a, acc, st, nblocks);    \
            }                                                                         \
            if (E == 16) return go_rows_acc<float, LL, 16>(a, acc, st, nblocks);      \
        }                                                                             \
        break;
    switch (L) { WOS_FAST_L(CASE_A) }
#undef CASE_A
    return cudaErrorNotSupported;
}

cudaError_t fast_rows_design(int fp64, int L, int E, int stage, const FastRows& a, const DesignArgs& d,
                             cudaStream_t st, int* nblocks) {
#define CASE_D(LL)                                                                                  \
    case LL:                                                                                        \
        if (fp64) {                                                                                 \
            if constexpr (LL <= 4096) {                                                             \
                if (E == 8) return go_rows_design_s<double, LL, 8>(stage, a, d, st, nblocks);       \
            } else {                                                                                \
                if (E == 16) return go_rows_design_s<double, LL, 16>(stage, a, d, st, nblocks);     \
            }                                                                                       \
        } else {                                                                                    \
            if constexpr (LL <= 4096) {                                                             \
                if (E == 8) return go_rows_design_s<float, LL, 8>(stage, a, d, st, nblocks);        \
            }                                                                                       \
            if (E == 16) return go_rows_design_s<float, LL, 16>(stage, a, d, st, nblocks);          \
        }                                                                                           \
        break;
    switch (L) { WOS_FAST_L(CASE_D) }
#undef CASE_D
    return cudaErrorNotSupported;
}

bool fast_supported(int fp64, int L, int E) {
    if (L < 256 || L > 8192 || (L & (L - 1))) return false;
    if (fp64) return (E == 8 && L <= 4096) || (E == 16 && L >= 8192);
    return E == 16 || (E == 8 && L <= 4096);
}

size_t fast_col_smem(int fp64, int L, int E, int W) { return (size_t)fcol_elems(L, E, W) * (fp64 ? 16 : 8); }

}  // namespace wos

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
#include <cuda_runtime.h>
#include <math.h>

#include "wos_fast.cuh"
#include "wos_fft.cuh"

namespace wos {

template <int N> struct Log2 { static constexpr int v = 1 + Log2<N / 2>::v; };
template <> struct Log2<1> { static constexpr int v = 0; };

template <int L, int E> struct FPlan {
    static constexpr int LG = Log2<L>::v, LE = Log2<E>::v;
    static constexpr int P = (LG + LE - 1) / LE;                 // passes
    static constexpr int RS = (LG % LE) ? (1 << (LG % LE)) : E;  // the odd radix (E if none)
    static constexpr int T = L / E;                              // threads per line
};
// radix and sub-transform length NS of pass p (forward order (RS, E, ..), inverse reversed)
__host__ __device__ constexpr int fp_radix(int P, int RS, int E, bool inv, int p) {
    return inv ? (p == P - 1 ? RS : E) : (p == 0 ? RS : E);
}
__host__ __device__ constexpr int fp_ns(int P, int RS, int E, bool inv, int p) {
    int ns = 1;
    for (int q = 0; q < p; q++) ns *= fp_radix(P, RS, E, inv, q);
    return ns;
}
// offset of pass p's table: forward passes first, then inverse passes;
// pass p holds NS*(R-1) entries (pass 0 has NS = 1 and needs none)
__host__ __device__ constexpr int fp_twoff(int P, int RS, int E, bool inv, int p) {
    int off = 0;
    for (int d = 0; d < 2; d++) {
        const bool dinv = d == 1;
        for (int q = 1; q < P; q++) {
            if (dinv == inv && q == p) return off;
            off += fp_ns(P, RS, E, dinv, q) * (fp_radix(P, RS, E, dinv, q) - 1);
        }
    }
    return off;
}

// padded slot of position q: one pad slot every 2^SH positions
template <int SH> __device__ __forceinline__ int padq(int q) { return q + (q >> SH); }

// One Stockham DIT pass, radix R, sub-transform length NS.
template <int R, int E, int L, int NS, int TWOFF, bool INV, typename C>
__device__ __forceinline__ void fpass(C* v, int tt, const C* __restrict__ twp) {
    constexpr int T = L / E;
#pragma unroll
    for (int b = 0; b < E / R; b++) {
        if constexpr (NS > 1) {
            const int k = (tt + b * T) & (NS - 1);
            const C* tk = twp + TWOFF + k;
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = __ldg(tk + (r - 1) * NS);
                if (INV) w.y = -w.y;
                v[b * R + r] = cmul(v[b * R + r], w);
            }
        }
        dft<R, INV>(v + b * R);
    }
}

// Exchange stores / loads on a line whose element q lives at
// sm[line_base + STR * padq<SH>(q)] (STR = W for interleaved columns).
template <int R, int E, int L, int NS, int SH, int STR, typename C>
__device__ __forceinline__ void fstore(const C* v, C* smb, int tt) {
    constexpr int T = L / E;
    static_assert(NS >= (1 << SH) || NS == 1 || NS * R >= (1 << SH), "padding does not commute with this pass");
#pragma unroll
    for (int b = 0; b < E / R; b++) {
        const int j = tt + b * T;
        const int k = j & (NS - 1);
        const int base = (j - k) * R + k;
        int tb;
        if constexpr (NS >= (1 << SH)) tb = padq<SH>(base);
        else tb = base + ((base - k) >> SH);
        C* p = smb + STR * tb;
#pragma unroll
        for (int r = 0; r < R; r++) p[STR * (r * NS + ((r * NS) >> SH))] = v[b * R + r];
    }
}

template <int R, int E, int L, int SH, int STR, typename C>
__device__ __forceinline__ void fload(C* v, const C* smb, int tt) {
    constexpr int T = L / E;
    constexpr int LR = L / R;
    static_assert(LR % (1 << SH) == 0, "load stride must be a multiple of the pad period");
#pragma unroll
    for (int b = 0; b < E / R; b++) {
        const C* p = smb + STR * padq<SH>(tt + b * T);
#pragma unroll
        for (int r = 0; r < R; r++) v[b * R + r] = p[STR * (r * (LR + (LR >> SH)))];
    }
}

// All passes from p on.  Each exchange has its own padding period, the radix
// of the pass that stores (SH = log2 R): for every power-of-two line stride W
// that makes the store of each pass conflict-free, and the natural-order load
// of the next pass stays a per-thread base plus immediates.
template <int L, int E, bool INV, int p, int STR, typename C>
__device__ __forceinline__ void fpasses(C* v, C* smb, int tt, const C* __restrict__ twp) {
    using PL = FPlan<L, E>;
    if constexpr (p < PL::P) {
        constexpr int R = fp_radix(PL::P, PL::RS, E, INV, p);
        constexpr int NS = fp_ns(PL::P, PL::RS, E, INV, p);
        constexpr int TWOFF = fp_twoff(PL::P, PL::RS, E, INV, p);
        fpass<R, E, L, NS, TWOFF, INV>(v, tt, twp);
        if constexpr (p < PL::P - 1) {
            constexpr int R2 = fp_radix(PL::P, PL::RS, E, INV, p + 1);
            constexpr int SH = Log2<R>::v;
            __syncthreads();
            fstore<R, E, L, NS, SH, STR>(v, smb, tt);
            __syncthreads();
            fload<R2, E, L, SH, STR>(v, smb, tt);
            fpasses<L, E, INV, p + 1, STR>(v, smb, tt, twp);
        }
    }
}

// padded length of a line: the largest padq over the exchanges of both directions
__host__ __device__ constexpr int fp_padded_len(int L, int E) {
    int LG = 0, LE = 0;
    while ((1 << LG) < L) LG++;
    while ((1 << LE) < E) LE++;
    const int P = (LG + LE - 1) / LE;
    const int RS = (LG % LE) ? (1 << (LG % LE)) : E;
    int m = L;
    for (int d = 0; d < 2; d++)
        for (int p = 0; p < P - 1; p++) {
            int R = fp_radix(P, RS, E, d == 1, p), sh = 0;
            while ((1 << sh) < R) sh++;
            const int len = (L - 1) + ((L - 1) >> sh) + 1;
            if (len > m) m = len;
        }
    return m;
}

// position of register slot s under the natural mapping of radix R
template <int R, int E, int L>
__device__ __forceinline__ int fpos(int s, int tt) {
    return tt + (s / R) * (L / E) + (s % R) * (L / R);
}

template <typename Real, int E> struct FMaxT { static constexpr int v = (E >= 16 || sizeof(Real) == 8) ? 512 : 1024; };
// column kernels: 256-thread CTAs for lines of up to 256 threads, three
// resident per SM for FP32 radix-8 lines (<= 85 registers), two otherwise
// (<= 128, which 16 complex64 or 8 complex128 values per thread fit without
// spilling); longer lines keep 512-thread CTAs
template <typename Real, int L, int E> struct FColB {
    static constexpr int maxt = (L / E <= 256) ? 256 : 512;
    static constexpr int minb = (L / E <= 256) ? ((sizeof(Real) == 4 && E == 8) ? 3 : 2) : 1;
};

__host__ __device__ constexpr int frow_stride(int L, int E) { return fp_padded_len(L, E) + 2; }
__host__ __device__ constexpr int fcol_elems(int L, int E, int W) { return W * fp_padded_len(L, E) + 2; }

// ------------------------------------------------------------------- rows
template <typename Real, int L, int E, bool INV>
__global__ void __launch_bounds__(FMaxT<Real, E>::v) k_rows_fast(const FastRows a) {
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
        } else {
            const C* in = reinterpret_cast<const C*>(a.in) + ib + tt;
#pragma unroll
            for (int s = 0; s < E; s++) v[s] = in[fpos<R1, E, L>(s, 0)];
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
        if (a.out_scale != 1.0) {
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

// ------------------------------------------------------------------- cols
__device__ __forceinline__ double fast_reduce_2pi_d(double arg) {
    const double inv2pi = 0.15915494309189533577;
    const double p2hi = 6.283185307179586232;
    const double p2lo = 2.4492935982947064e-16;
    const double n = rint(arg * inv2pi);
    double r = fma(-n, p2hi, arg);
    return fma(-n, p2lo, r);
}

// sqrt of s in (0, 1] to ~1e-14 relative: single-precision reciprocal square
// root seed refined by one Newton step in FP64 (s in FP32 range here).
__device__ __forceinline__ double fast_sqrt_d(double s) {
    const double r0 = (double)rsqrtf((float)s);
    const double y0 = s * r0;
    return fma(0.5 * r0, fma(-y0, y0, s), y0);
}

// sqrt of s in [2^-100, 1] to ~1e-13 relative without FP64<->FP32 conversion
// instructions: the single-precision seed is assembled from the double's bit
// fields (exponent rebias 1023 -> 127, mantissa truncated to 23 bits), its
// reciprocal square root is taken in single precision, widened back by the
// same rebias, and refined by one Newton step in FP64.
__device__ __forceinline__ double fast_sqrt_bits(double s) {
    const int hi = __double2hiint(s), lo = __double2loint(s);
    const float sf = __int_as_float(__funnelshift_l(lo, hi - 0x38000000, 3));
    const int rb = __float_as_int(rsqrtf(sf));
    const double r0 = __hiloint2double((rb >> 3) + 0x38000000, (int)((unsigned)rb << 29));
    const double y0 = s * r0;
    return fma(0.5 * r0, fma(-y0, y0, s), y0);
}

// exp(2 pi i t) for |t| < 2^28 revolutions in single precision.  Adding
// 1.5 * 2^29 rounds t to a multiple of 2^-23 and leaves that multiple, modulo
// 2^23, in the low mantissa bits; sign-extending 23 of them gives the
// fractional part in [-1/2, 1/2) as an integer, converted exactly through the
// 1.5 * 2^23 float pattern, then scaled to radians.
__device__ __forceinline__ float2 cexp_rev(double t) {
    const double u = t + 805306368.0;  // 1.5 * 2^29
    const int s23 = (int)((unsigned)__double2loint(u) << 9) >> 9;
    const float f = __int_as_float(0x4b400000 + s23) - 12582912.0f;
    float sn, cs;
    __sincosf(f * 7.490140565847857e-07f, &sn, &cs);  // 2 pi / 2^23
    return make_float2(cs, sn);
}

template <typename Real, int L, int E, int W>
__global__ void __launch_bounds__(FColB<Real, L, E>::maxt, FColB<Real, L, E>::minb) k_cols_fast(const FastCols a) {
    using C = typename CT<Real>::t;
    using PL = FPlan<L, E>;
    constexpr int T = PL::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    C* smb = reinterpret_cast<C*>(smraw) + w;
    const int col = blockIdx.x * W + w;
    const bool act = col < a.ncols;
    const C* twp = reinterpret_cast<const C*>(a.tw);
    C* base = reinterpret_cast<C*>(a.data) + (long long)blockIdx.y * a.bstride + col;
    C v[E];
    constexpr int R1 = PL::RS;
    if (act) {
        const C* src = base + (long long)tt * a.ld;
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = src[(long long)fpos<R1, E, L>(s, 0) * a.ld];
    } else {
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = mkc<C>(0, 0);
    }
    // interleaved tile: stride W between consecutive positions of a column
    fpasses<L, E, false, 0, W>(v, smb, tt, twp);

    // radial histogram of the spectrum (before H) for the alias-wrap check
    __shared__ double hsm[97];
    if (a.hist) {
        double* P = reinterpret_cast<double*>(smraw);  // [q][w], W*L doubles: inside the tile
        __syncthreads();  // the tile is free once every thread has loaded its last pass
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = tt + s * T;
            P[q * W + w] = act ? (double)v[s].x * v[s].x + (double)v[s].y * v[s].y : 0.0;
        }
        for (int k = threadIdx.x; k < 97; k += blockDim.x) hsm[k] = 0;
        __syncthreads();
        // |q| = j and L - j share a bin; each warp takes 32 consecutive j of one column
        constexpr int NJ = (L / 2 + 1 + 31) / 32 * 32;
        const double fnyq = 1.0 / (2.0 * a.hist_dx);
        const double den = __dmul_rn((double)L, a.hist_dx);
        const double dnx = __dmul_rn((double)a.ncols, a.hist_dx);
        for (int idx = threadIdx.x; idx < W * NJ; idx += blockDim.x) {
            const int wc = idx / NJ, j = idx - wc * NJ;
            const int c2 = blockIdx.x * W + wc;
            double pw = 0;
            int b = 0;
            if (j <= L / 2 && c2 < a.ncols) {
                pw = P[j * W + wc];
                if (j > 0 && j < L / 2) pw += P[(L - j) * W + wc];
                const double hfx = (c2 <= a.ncols / 2) ? __ddiv_rn((double)c2, dnx) : __ddiv_rn((double)(c2 - a.ncols), dnx);
                const double fy = __ddiv_rn((double)j, den);
                double hp = fabs(hfx), hq = fabs(fy);
                if (hp < hq) { const double t = hp; hp = hq; hq = t; }
                double hy = 0;
                if (hp != 0) {
                    const double r = __ddiv_rn(hq, hp);
                    hy = __dmul_rn(hp, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(r, r))));
                }
                b = (int)__dmul_rn(__ddiv_rn(hy, fnyq), 96.0);
                b = b > 96 ? 96 : (b < 0 ? 0 : b);
            }
            const int b0 = __shfl_sync(0xffffffffu, b, 0);
            if (__all_sync(0xffffffffu, b == b0 || pw == 0)) {
                for (int o = 16; o > 0; o >>= 1) pw += __shfl_down_sync(0xffffffffu, pw, o);
                if ((threadIdx.x & 31) == 0 && pw != 0) atomicAdd(&hsm[b0], pw);
            } else if (pw != 0) {
                atomicAdd(&hsm[b], pw);
            }
        }
    }

    // transfer function on the radix-E natural mapping: q = tt + s*T
    const double wl = a.wl;
    double p0 = 0, l1 = 0;
    if constexpr (sizeof(Real) == 4) {
        // FP32 pipeline: FP64 argument kz*sqrt(1 - (wl fx)^2 - (wl fy)^2),
        // reduced modulo one period in FP64, sin/cos in single precision
        const double fx = (col <= a.ncols / 2 ? (double)col : (double)(col - a.ncols)) / ((double)a.ncols * a.dx);
        const double ax = wl * fx;
        const double cx = fma(-ax, ax, 1.0);
        const double g = wl / ((double)L * a.dx);
        const double tg = (double)T * g, ay0 = (double)tt * g;
        const float sc = (float)a.scale;
        const float sgn = a.conj ? -1.f : 1.f;
#pragma unroll
        for (int s = 0; s < E; s++) {
            // signed position of q = tt + s*T is q - L from s = E/2 on (q = L/2
            // itself has the same |fy| either way)
            const double ay = fma((double)(s < E / 2 ? s : s - E), tg, ay0);
            const double sq = fma(-ay, ay, cx);
            float hr, hi;
            double m2 = 1.0;
            if (sq >= 0) {  // rho <= 1: propagating
                if (a.rev_phase) {
                    const double sr = sq > 0x1p-100 ? fast_sqrt_bits(sq) : 0.0;
                    const float2 e = cexp_rev(a.krev * sr);
                    hr = e.x;
                    hi = e.y;
                } else {
                    const double sr = sq > 0 ? fast_sqrt_d(sq) : 0.0;
                    __sincosf((float)fast_reduce_2pi_d(a.kz * sr), &hi, &hr);
                }
            } else {
                const double decay = a.kaz * sqrt(-sq);
                double amp;
                if (a.zero_ev || (a.limit > 0 && decay > a.limit)) amp = 0;
                else if (a.backward) amp = a.reg ? exp(decay) / (1.0 + a.alpha * a.alpha * exp(2 * decay)) : exp(decay);
                else amp = exp(-decay);
                hr = (float)amp;
                hi = 0.f;
                m2 = amp * amp;
            }
            if (a.red) {
                const double pp = (double)v[s].x * v[s].x + (double)v[s].y * v[s].y;
                p0 += pp;
                l1 += pp * (1.0 - m2);
            }
            v[s] = cmul(v[s], make_float2(hr * sc, sgn * hi * sc));
        }
    } else {
        // FP64 pipeline: the reference's operation sequence, uncontracted
        const double fxe = (col <= a.ncols / 2) ? __ddiv_rn((double)col, __dmul_rn((double)a.ncols, a.dx))
                                                : __ddiv_rn((double)(col - a.ncols), __dmul_rn((double)a.ncols, a.dx));
        const double den = __dmul_rn((double)L, a.dx);
        const double px = fabs(__dmul_rn(wl, fxe));
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = tt + s * T;
            const double fy = (q <= L / 2) ? __ddiv_rn((double)q, den) : __ddiv_rn((double)(q - L), den);
            double p = px, qv = fabs(__dmul_rn(wl, fy));
            if (p < qv) { const double t = p; p = qv; qv = t; }
            double rho = 0;
            if (p != 0) {
                const double qq = __ddiv_rn(qv, p);
                rho = __dmul_rn(p, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(qq, qq))));
            }
            double hr, hi, m2 = 1.0;
            if (rho <= 1.0) {
                sincos(__dmul_rn(a.kz, __dsqrt_rn(__dmul_rn(__dsub_rn(1.0, rho), __dadd_rn(1.0, rho)))), &hi, &hr);
            } else {
                const double decay = __dmul_rn(a.kaz, __dsqrt_rn(__dmul_rn(__dsub_rn(rho, 1.0), __dadd_rn(rho, 1.0))));
                double amp;
                if (a.zero_ev || (a.limit > 0 && decay > a.limit)) amp = 0;
                else if (a.backward) {
                    if (a.reg) {
                        const double e = exp(decay);
                        amp = __ddiv_rn(e, __dadd_rn(1.0, __dmul_rn(__dmul_rn(__dmul_rn(a.alpha, a.alpha), e), e)));
                    } else {
                        amp = exp(decay);
                    }
                } else {
                    amp = exp(-decay);
                }
                hr = amp;
                hi = 0;
                m2 = amp * amp;
            }
            if (a.red) {
                const double pp = v[s].x * v[s].x + v[s].y * v[s].y;
                p0 += pp;
                l1 += pp * (1.0 - m2);
            }
            v[s] = cmul(v[s], make_double2(hr * a.scale, (a.conj ? -hi : hi) * a.scale));
        }
    }
    if (!act) {
        p0 = 0;
        l1 = 0;
    }
    fpasses<L, E, true, 0, W>(v, smb, tt, twp);
    if (act) {
        constexpr int RO = PL::RS;
        C* dst = base + (long long)tt * a.ld;
#pragma unroll
        for (int s = 0; s < E; s++) dst[(long long)fpos<RO, E, L>(s, 0) * a.ld] = v[s];
    }
    if (a.red) {
        __shared__ double rsm[32][2];
        for (int o = 16; o > 0; o >>= 1) {
            p0 += __shfl_down_sync(0xffffffffu, p0, o);
            l1 += __shfl_down_sync(0xffffffffu, l1, o);
        }
        if ((threadIdx.x & 31) == 0) {
            rsm[threadIdx.x >> 5][0] = p0;
            rsm[threadIdx.x >> 5][1] = l1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double t0 = 0, t1 = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
                t0 += rsm[k][0];
                t1 += rsm[k][1];
            }
            double* o = a.red + ((long long)blockIdx.y * gridDim.x + blockIdx.x) * a.red_stride;
            o[0] = t0;
            o[1] = t1;
        }
    }
    if (a.hist) {
        __syncthreads();
        double* o = a.hist + ((long long)blockIdx.y * gridDim.x + blockIdx.x) * a.red_stride;
        for (int k = threadIdx.x; k < 97; k += blockDim.x) o[k] = hsm[k];
    }
}

// ------------------------------------------------------------------ tables
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
template <typename Real, int L, int E, bool INV>
static cudaError_t go_rows(const FastRows& a, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    int lines = 1;
    while (lines * 2 * T <= 256 && lines * 2 <= a.rows) lines *= 2;
    while (lines * T < 32) lines *= 2;
    const size_t smem = (size_t)frow_stride(L, E) * lines * sizeof(typename CT<Real>::t);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows_fast<Real, L, E, INV>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((a.rows + lines - 1) / lines, a.batch > 0 ? a.batch : 1);
    if (nblocks) *nblocks = (int)grid.x;
    k_rows_fast<Real, L, E, INV><<<grid, lines * T, smem, st>>>(a);
    return cudaGetLastError();
}

template <typename Real, int L, int E, int W>
static cudaError_t go_cols_w(const FastCols& a, cudaStream_t st, int* nblocks) {
    constexpr int T = L / E;
    if constexpr (W * T < 32 || W * T > FColB<Real, L, E>::maxt) {
        return cudaErrorInvalidConfiguration;
    } else {
        const size_t smem = (size_t)fcol_elems(L, E, W) * sizeof(typename CT<Real>::t);
        if (smem > kSmemNoOptIn) {
            cudaError_t e = cudaFuncSetAttribute(k_cols_fast<Real, L, E, W>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        dim3 grid((a.ncols + W - 1) / W, a.batch > 0 ? a.batch : 1);
        if (nblocks) *nblocks = (int)grid.x;
        k_cols_fast<Real, L, E, W><<<grid, W * T, smem, st>>>(a);
        return cudaGetLastError();
    }
}

template <typename Real, int L, int E>
static cudaError_t go_cols(const FastCols& a, cudaStream_t st, int* nblocks) {
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
    const int maxt = (T <= 256) ? 256 : 512;
    if (W < 1) W = 1;
    while (W * T < 32) W *= 2;
    while (W > 1 && W * T > maxt) W /= 2;
    if (W > 16 || W * T > maxt || W * T < 32) return 0;
    (void)fp64;
    return W;
}

bool fast_supported(int fp64, int L, int E) {
    if (L < 256 || L > 8192 || (L & (L - 1))) return false;
    if (fp64) return (E == 8 && L <= 4096) || (E == 16 && L >= 8192);
    return E == 16 || (E == 8 && L <= 4096);
}

size_t fast_col_smem(int fp64, int L, int E, int W) { return (size_t)fcol_elems(L, E, W) * (fp64 ? 16 : 8); }

}  // namespace wos

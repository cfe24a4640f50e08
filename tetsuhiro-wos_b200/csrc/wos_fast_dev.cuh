// wos_fast_dev.cuh -- device building blocks of the compile-time specialised
// power-of-two sweeps (pass plan, padded exchanges, transfer function,
// histogram and loss sums), shared by the one-shot and the pipelined kernels.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "wos_fast.cuh"
#include "wos_fft.cuh"

namespace wos {

// Programmatic dependent launch.  A sweep launched with the programmatic
// stream-serialization attribute may become resident while the kernel before
// it in the stream is still draining; pdl_wait() blocks (in hardware, not a
// spin loop) until that grid has completed and its writes are visible, and is
// a no-op for an ordinary launch.  Every kernel that a launcher may start with
// the attribute calls it before its first global-memory access.
// pdl_trigger() then lets the next sweep of the stream be scheduled; that
// grid's own pdl_wait() still waits for this one to complete.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

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

// Read-only load that asks L1 to keep the line (twiddle tables are re-read by
// every line of a sweep while the field streams through).
__device__ __forceinline__ float2 ldg_keep(const float2* p) {
    float2 r;
    asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];" : "=f"(r.x), "=f"(r.y) : "l"(p));
    return r;
}
__device__ __forceinline__ double2 ldg_keep(const double2* p) {
    double2 r;
    asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(p));
    return r;
}

// Twiddles of one Stockham DIT pass (radix R, sub-transform length NS) for
// this thread's E/R butterflies, [b][r-1] = W^(r k); none when NS == 1.
// Complex64 passes of radix 8 and 16 load only W^k, W^2k, W^4k (and W^8k);
// ftw_expand forms the others as products once the loads have landed (after
// the exchange barrier), at most three roundings deep: four global loads and
// eleven complex products per radix-16 butterfly instead of fifteen loads.
template <int R, typename C, bool CP = false> struct FtwPow2 {
    static constexpr bool v = !CP && sizeof(C) == 8 && (R == 8 || R == 16);
};
// CP (compensated, complex64): every twiddle is the pair W_hi + W_lo from
// the table and its residual table twl (same layout, (float)(W - W_hi) from
// FP64), all loaded (no products), and applied as x W_hi + x W_lo.
template <int R, int E, int L, int NS, int TWOFF, bool CP, typename C>
__device__ __forceinline__ void ftw_load(C* w, C* wl, int tt, const C* __restrict__ twp, const C* __restrict__ twl) {
    constexpr int T = L / E;
    if constexpr (NS > 1) {
#pragma unroll
        for (int b = 0; b < E / R; b++) {
            const int o = TWOFF + ((tt + b * T) & (NS - 1));
            const C* tk = twp + o;
#pragma unroll
            for (int r = 1; r < R; r++) {
                if (!FtwPow2<R, C, CP>::v || (r & (r - 1)) == 0) w[b * (R - 1) + r - 1] = ldg_keep(tk + (r - 1) * NS);
                if constexpr (CP) wl[b * (R - 1) + r - 1] = ldg_keep(twl + o + (r - 1) * NS);
            }
        }
    }
}
template <int R, int E, int NS, bool CP, typename C>
__device__ __forceinline__ void ftw_expand(C* w) {
    if constexpr (NS > 1 && FtwPow2<R, C, CP>::v) {
#pragma unroll
        for (int b = 0; b < E / R; b++) {
            C* p = w + b * (R - 1);  // p[r - 1] = W^(r k)
            p[2] = cmul(p[0], p[1]);
            p[4] = cmul(p[0], p[3]);
            p[5] = cmul(p[1], p[3]);
            p[6] = cmul(p[2], p[3]);
            if constexpr (R == 16) {
#pragma unroll
                for (int r = 1; r < 8; r++) p[r + 7] = cmul(p[r - 1], p[7]);
            }
        }
    }
}

// x (t + tl) for a twiddle t with its residual tl (complex64): the small
// product x tl first, then the main product folded in by FMAs.
template <typename C>
__device__ __forceinline__ C cmul_cp(C x, C t, C tl) {
    const C c = cmul(x, tl);
    return mkc<C>(fma(x.x, t.x, fma(-x.y, t.y, c.x)), fma(x.x, t.y, fma(x.y, t.x, c.y)));
}

// One Stockham DIT pass on registers, its twiddles already loaded.
template <int R, int E, int NS, bool INV, bool CP, typename C>
__device__ __forceinline__ void fpass_tw(C* v, const C* w, const C* wl) {
#pragma unroll
    for (int b = 0; b < E / R; b++) {
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                C t = w[b * (R - 1) + r - 1];
                if (INV) t.y = -t.y;
                if constexpr (CP) {
                    C tl = wl[b * (R - 1) + r - 1];
                    if (INV) tl.y = -tl.y;
                    v[b * R + r] = cmul_cp(v[b * R + r], t, tl);
                } else {
                    v[b * R + r] = cmul(v[b * R + r], t);
                }
            }
        }
        dft<R, INV, C, CP>(v + b * R);
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

// Padding period 2^SH of the exchange after a radix-R pass.  By default the
// storing radix (SH = log2 R), which keeps every store conflict-free.  Complex64
// rows (STR == 1) take at least 16 positions where the pass strides allow it:
// the next pass's loads are 16 consecutive 64-bit words per half-warp, which a
// pad every 8 positions (radix 8) puts twice on one bank pair; with a pad every
// 16 they land on 16 distinct pairs, and the stores of a radix 2, 4 or 8 pass
// stay conflict-free; a radix-8 pass with 1 < NS < 16 (lines of E = 8) keeps
// 8, where a period of 16 puts two of a half-warp's stores on one bank pair
// (and 8 leaves fewer conflicts on the load side than 16 does on the store
// side).  Complex128 lines take 8 after radix-2 and radix-4
// passes: a wavefront serves 8 threads' 16-byte slots, and a pad every 2 or 4
// put two of the next pass's 8 consecutive loads on one bank group (the
// forward 2048-point row sweep: 524K load conflicts per launch); with 8 the
// stores of those passes stay conflict-free too.  (A period of 16 would
// conflict on the store side of complex128.)
template <int L, int R, int NS, int R2, int STR, typename C>
__host__ __device__ constexpr int fx_shift() {
    constexpr int s = Log2<R>::v;
    if (sizeof(C) == 8 && STR == 1 && s < 4 && (L / R2) % 16 == 0 && (NS >= 16 || NS == 1)) return 4;
    if (sizeof(C) == 16 && STR == 1 && s < 3 && (L / R2) % 8 == 0 && (NS >= 8 || NS == 1 || NS * R >= 8)) return 3;
    return s;
}

// All passes from p on; wcur holds pass p's twiddles.  Each exchange has its
// own padding period (fx_shift: the radix of the pass that stores, or 16 for
// complex64 rows): for every power-of-two line stride W that makes the store
// of each pass conflict-free, and the natural-order load of the next pass
// stays a per-thread base plus immediates.  The next pass's twiddles are requested
// once this thread's stores are issued (the data registers are free then), so
// their latency runs under the barrier.
template <int L, int E, bool INV, int p, int STR, bool CP, typename C>
__device__ __forceinline__ void fpasses_from(C* v, C* smb, int tt, const C* __restrict__ twp, const C* __restrict__ twl,
                                             const C* wcur, const C* wlcur) {
    using PL = FPlan<L, E>;
    if constexpr (p < PL::P) {
        constexpr int R = fp_radix(PL::P, PL::RS, E, INV, p);
        constexpr int NS = fp_ns(PL::P, PL::RS, E, INV, p);
        fpass_tw<R, E, NS, INV, CP>(v, wcur, wlcur);
        if constexpr (p < PL::P - 1) {
            constexpr int R2 = fp_radix(PL::P, PL::RS, E, INV, p + 1);
            constexpr int NS2 = fp_ns(PL::P, PL::RS, E, INV, p + 1);
            constexpr int TWOFF2 = fp_twoff(PL::P, PL::RS, E, INV, p + 1);
            constexpr int SH = fx_shift<L, R, NS, R2, STR, C>();
            C wn[(E / R2) * (R2 - 1)];
            C wln[CP ? (E / R2) * (R2 - 1) : 1];
            __syncthreads();
            fstore<R, E, L, NS, SH, STR>(v, smb, tt);
            ftw_load<R2, E, L, NS2, TWOFF2, CP>(wn, wln, tt, twp, twl);
            __syncthreads();
            fload<R2, E, L, SH, STR>(v, smb, tt);
            ftw_expand<R2, E, NS2, CP>(wn);
            fpasses_from<L, E, INV, p + 1, STR, CP>(v, smb, tt, twp, twl, wn, wln);
        }
    }
}

// A whole line transform (the first pass has NS == 1: no twiddles).  twl: the
// residual table of the compensated transform (CP), else unused.
template <int L, int E, bool INV, int p, int STR, typename C, bool CP = false>
__device__ __forceinline__ void fpasses(C* v, C* smb, int tt, const C* __restrict__ twp,
                                        const C* __restrict__ twl = nullptr) {
    static_assert(p == 0, "a line transform starts at pass 0");
    fpasses_from<L, E, INV, 0, STR, CP>(v, smb, tt, twp, twl, static_cast<const C*>(nullptr),
                                        static_cast<const C*>(nullptr));
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
// Column kernels: a CTA holds W columns of T = L/E threads.  A tile row of W
// complex64 values is one global-memory segment, so wide tiles (W*8 bytes >=
// one 32-byte sector) are what keep the strided column access efficient:
// FP32 CTAs go up to 1024 threads, with three resident per SM at 256 threads
// (<= 84 registers), two at 512 and one at 1024 (<= 64 registers: the line's
// values and the transfer function never share the registers, H is applied
// in shared memory); FP64 CTAs keep 256 threads (two per SM, <= 128 registers) unless a
// line needs more.
__host__ __device__ constexpr int fcol_max_threads(bool fp64, int T) { return fp64 ? (T <= 256 ? 256 : 512) : 1024; }
template <typename Real, int L, int E, int W> struct FColB {
    static constexpr int threads = W * (L / E);
    // resident CTAs per SM: FP32 <= 84 registers per thread up to 256 threads
    // (three 256-thread CTAs), two 512-thread CTAs; FP64 <= 128 registers
    static constexpr int minb = sizeof(Real) == 4 ? (threads <= 256 ? 65536 / (threads * 84) : 65536 / (threads * 64))
                                                  : (threads <= 512 ? 65536 / (threads * 128) : 1);
};

__host__ __device__ constexpr int frow_stride(int L, int E) { return fp_padded_len(L, E) + 2; }
__host__ __device__ constexpr int fcol_elems(int L, int E, int W) { return W * fp_padded_len(L, E) + 2; }
// byte offset of the transfer-function table rows behind a complex64 column tile
__host__ __device__ constexpr size_t fcol_htab_off(int L, int E, int W) {
    return ((size_t)fcol_elems(L, E, W) * 8 + 15) / 16 * 16;
}

// ------------------------------------------------------------------- cols
// Radial histogram of |F|^2 (the spectrum before H) for the alias-wrap check
// (spectralRadius, optics/propagate.go:270-310), added into hsm (97 bins,
// zeroed by the caller) from the W columns held dense in the tile ([q][w]):
// |q| = j and L - j share a bin; each warp takes 32 consecutive j of one
// column.  Out of line: it runs only for the alias-wrap check and keeps the
// unrolled sweep code compact.
template <typename C>
__device__ __noinline__ void col_hist_bin(const C* tile, double* hsm, int col0, int L, int W, int ncols,
                                          double hist_dx) {
    const int NJ = (L / 2 + 1 + 31) / 32 * 32;
    const double fnyq = 1.0 / (2.0 * hist_dx);
    const double den = __dmul_rn((double)L, hist_dx);
    const double dnx = __dmul_rn((double)ncols, hist_dx);
    const float inv_dnx = (float)(1.0 / dnx), inv_den = (float)(1.0 / den), bins_per_f = (float)(96.0 / fnyq);
    for (int idx = threadIdx.x; idx < W * NJ; idx += blockDim.x) {
        const int wc = idx / NJ, j = idx - wc * NJ;
        const int c2 = col0 + wc;
        double pw = 0;
        int b = 0;
        if (j <= L / 2 && c2 < ncols) {
            const C x = tile[j * W + wc];
            pw = (double)x.x * x.x + (double)x.y * x.y;
            if (j > 0 && j < L / 2) {
                const C y = tile[(L - j) * W + wc];
                pw += (double)y.x * y.x + (double)y.y * y.y;
            }
            // bin from a single-precision radius (error < 1e-4 of a bin), the
            // reference's exact FP64 sequence only within 1e-3 of a bin edge
            const int cf = (c2 <= ncols / 2) ? c2 : c2 - ncols;
            const float rf = sqrtf(fmaf((float)cf * inv_dnx, (float)cf * inv_dnx,
                                        ((float)j * inv_den) * ((float)j * inv_den))) * bins_per_f;
            const float fl = floorf(rf);
            if (rf - fl > 1e-3f && rf - fl < 1.0f - 1e-3f) {
                b = (int)fl;
            } else {
                const double hfx = __ddiv_rn((double)cf, dnx);
                const double fy = __ddiv_rn((double)j, den);
                double hp = fabs(hfx), hq = fabs(fy);
                if (hp < hq) { const double t = hp; hp = hq; hq = t; }
                double hy = 0;
                if (hp != 0) {
                    const double r = __ddiv_rn(hq, hp);
                    hy = __dmul_rn(hp, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(r, r))));
                }
                b = (int)__dmul_rn(__ddiv_rn(hy, fnyq), 96.0);
            }
            b = b > 96 ? 96 : (b < 0 ? 0 : b);
        }
        // the warp's 32 consecutive j of one column have non-decreasing bins
        // (|fy| grows with j; lanes past L/2 take the sentinel 97), so runs of
        // equal bins are contiguous: a segmented scan leaves each run's sum in
        // its last lane, and one atomic per run (a few per warp) adds it
        if (!(j <= L / 2 && c2 < ncols)) b = 97;
        const int lane = threadIdx.x & 31;
        for (int o = 1; o < 32; o <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, pw, o);
            const int bt = __shfl_up_sync(0xffffffffu, b, o);
            if (lane >= o && bt == b) pw += t;
        }
        const int bn = __shfl_down_sync(0xffffffffu, b, 1);
        if ((lane == 31 || bn != b) && b < 97 && pw != 0) atomicAdd(&hsm[b], pw);
    }
}

// Evanescent amplitude of asmTF (optics/propagate.go:168-180) for the FP32
// pipeline (sq = 1 - rho^2 < 0); out of line, it is rarely taken.
static __device__ __noinline__ double ev_amp_f(double sq, double kaz, int zero_ev, double limit, int backward, int reg,
                                        double alpha) {
    const double decay = kaz * sqrt(-sq);
    if (zero_ev || (limit > 0 && decay > limit)) return 0;
    if (backward) return reg ? exp(decay) / (1.0 + alpha * alpha * exp(2 * decay)) : exp(decay);
    return exp(-decay);
}

// The same in the reference's operation sequence (FP64 pipeline), rho > 1.
static __device__ __noinline__ double ev_amp_d(double rho, double kaz, int zero_ev, double limit, int backward, int reg,
                                        double alpha) {
    const double decay = __dmul_rn(kaz, __dsqrt_rn(__dmul_rn(__dsub_rn(rho, 1.0), __dadd_rn(rho, 1.0))));
    if (zero_ev || (limit > 0 && decay > limit)) return 0;
    if (backward) {
        if (reg) {
            const double e = exp(decay);
            return __ddiv_rn(e, __dadd_rn(1.0, __dmul_rn(__dmul_rn(__dmul_rn(alpha, alpha), e), e)));
        }
        return exp(decay);
    }
    return exp(-decay);
}

// Wavelength and distance of one unit of a batch (or of the single launch):
// k = 2 pi / wl, kz = k z, k |z|, kz / 2 pi, formed as the host forms them.
struct HUnit {
    double wl, kz, kaz, krev;
};
__device__ __forceinline__ HUnit h_unit(const FastCols& a, int b) {
    if (!a.batch_wl && !a.batch_z) return HUnit{a.wl, a.kz, a.kaz, a.krev};
    const double wl = a.batch_wl ? a.batch_wl[b] : a.wl;
    const double z = a.batch_z ? a.batch_z[b] : a.z;
    const double k = 2 * M_PI / wl;
    const double kz = k * z;
    return HUnit{wl, kz, k * fabs(z), kz / (2 * M_PI)};
}

// H(fx, fy) of asmTF (optics/propagate.go:159-181) times `scale` (conj(H)
// for the adjoint) and |H|^2, FP32 pipeline: cx = 1 - (wl fx)^2 of the
// column, ay = wl fy; the FP64 argument kz sqrt(1 - rho^2) is taken in
// revolutions (|kz / 2 pi| < 2^28, checked by the host) and reduced exactly.
__device__ __forceinline__ float2 h_f32(const FastCols& a, const HUnit& hu, double cx, double ay, double& m2) {
    const double sq = fma(-ay, ay, cx);
    float hr, hi;
    m2 = 1.0;
    if (sq >= 0) {  // rho <= 1: propagating
        const double sr = sq > 0x1p-100 ? fast_sqrt_bits(sq) : 0.0;
        const float2 e = cexp_rev(hu.krev * sr, a.precise_phase != 0);
        hr = e.x;
        hi = e.y;
    } else {
        const double amp = ev_amp_f(sq, hu.kaz, a.zero_ev, a.limit, a.backward, a.reg, a.alpha);
        hr = (float)amp;
        hi = 0.f;
        m2 = amp * amp;
    }
    const float sc = (float)a.scale;
    return make_float2(hr * sc, (a.conj ? -hi : hi) * sc);
}

// The same in the FP64 pipeline, with the reference's operation sequence
// (uncontracted): px = |wl fx| of the column, fy = freq(q).
__device__ __forceinline__ double2 h_f64(const FastCols& a, const HUnit& hu, double px, double fy, double& m2) {
    double p = px, qv = fabs(__dmul_rn(hu.wl, fy));
    if (p < qv) { const double t = p; p = qv; qv = t; }
    double rho = 0;
    if (p != 0) {
        const double qq = __ddiv_rn(qv, p);
        rho = __dmul_rn(p, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(qq, qq))));
    }
    double hr, hi;
    m2 = 1.0;
    if (rho <= 1.0) {
        sincos(__dmul_rn(hu.kz, __dsqrt_rn(__dmul_rn(__dsub_rn(1.0, rho), __dadd_rn(1.0, rho)))), &hi, &hr);
    } else {
        const double amp = ev_amp_d(rho, hu.kaz, a.zero_ev, a.limit, a.backward, a.reg, a.alpha);
        hr = amp;
        hi = 0;
        m2 = amp * amp;
    }
    return make_double2(hr * a.scale, (a.conj ? -hi : hi) * a.scale);
}

// Multiply the spectrum of the W columns held dense in the tile ([q][w],
// W*L values) by H, once per pair (q, L - q): |fy| and so H are the same for
// both.  Thread (tt, w) takes q = tt + i*T for i < E/2, i.e. q < L/2; the
// thread with q = 0 also takes the Nyquist row L/2.  p0 += |F|^2 and
// l1 += |F|^2 (1 - |H|^2) when the loss sums are requested.  Every thread of
// the CTA calls this between two barriers.
template <typename Real, int L, int E, int W, bool HCP, typename C>
__device__ __forceinline__ void col_tile_h(C* tile, int col0, const FastCols& a, const HUnit& hu, double& p0,
                                           double& l1, const float2* hs) {
    constexpr int T = L / E;
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    const int col = col0 + w;
    if (col >= a.ncols) return;  // zero columns stay zero
    const bool red = a.red != nullptr;
    auto apply = [&](int q, const C h, double m2) {
        C x = tile[q * W + w];
        if (red) {
            const double pp = (double)x.x * x.x + (double)x.y * x.y;
            p0 += pp;
            l1 += pp * (1.0 - m2);
        }
        tile[q * W + w] = cmul(x, h);
    };
    if constexpr (sizeof(Real) == 4) {
        if (HCP && hs) {  // hi + lo table rows (compensated sweeps): x H_hi + x H_lo
            const int cabs = col <= a.ncols / 2 ? col : a.ncols - col;
            const float4* hr = reinterpret_cast<const float4*>(hs) + (cabs - htab_row0(col0, a.ncols, W)) * a.htab_ld;
            const float sg = a.conj ? -1.f : 1.f;
            auto apply4 = [&](int q, const float4 t) {
                tile[q * W + w] = cmul_cp(tile[q * W + w], mkc<C>(t.x, sg * t.y), mkc<C>(t.z, sg * t.w));
            };
#pragma unroll
            for (int i = 0; i < E / 2; i++) {
                const int q = tt + i * T;
                const float4 t = hr[q];
                apply4(q, t);
                if (q != 0) apply4(L - q, t);
            }
            if (tt == 0) apply4(L / 2, hr[L / 2]);
            return;
        }
        if (hs) {  // the table rows of this CTA's columns (no loss sums here)
            const int cabs = col <= a.ncols / 2 ? col : a.ncols - col;
            const float2* hr = hs + (cabs - htab_row0(col0, a.ncols, W)) * a.htab_ld;
            const float sg = a.conj ? -1.f : 1.f;
#pragma unroll
            for (int i = 0; i < E / 2; i++) {
                const int q = tt + i * T;
                const float2 t = hr[q];
                const C h = mkc<C>(t.x, sg * t.y);
                apply(q, h, 1.0);
                if (q != 0) apply(L - q, h, 1.0);
            }
            if (tt == 0) {
                const float2 t = hr[L / 2];
                apply(L / 2, mkc<C>(t.x, sg * t.y), 1.0);
            }
            return;
        }
        const double fx = (col <= a.ncols / 2 ? (double)col : (double)(col - a.ncols)) / ((double)a.ncols * a.dx);
        const double ax = hu.wl * fx;
        const double cx = fma(-ax, ax, 1.0);
        const double g = hu.wl / ((double)L * a.dx);
        const double tg = (double)T * g, ay0 = (double)tt * g;
#pragma unroll
        for (int i = 0; i < E / 2; i++) {
            const int q = tt + i * T;
            double m2;
            const float2 h = h_f32(a, hu, cx, fma((double)i, tg, ay0), m2);
            apply(q, h, m2);
            if (q != 0) apply(L - q, h, m2);
        }
        if (tt == 0) {
            double m2;
            const float2 h = h_f32(a, hu, cx, (double)(L / 2) * g, m2);
            apply(L / 2, h, m2);
        }
    } else {
        const double fxe = (col <= a.ncols / 2) ? __ddiv_rn((double)col, __dmul_rn((double)a.ncols, a.dx))
                                                : __ddiv_rn((double)(col - a.ncols), __dmul_rn((double)a.ncols, a.dx));
        const double den = __dmul_rn((double)L, a.dx);
        const double px = fabs(__dmul_rn(hu.wl, fxe));
#pragma unroll
        for (int i = 0; i < E / 2; i++) {
            const int q = tt + i * T;
            double m2;
            const double2 h = h_f64(a, hu, px, __ddiv_rn((double)q, den), m2);
            apply(q, h, m2);
            if (q != 0) apply(L - q, h, m2);
        }
        if (tt == 0) {
            double m2;
            const double2 h = h_f64(a, hu, px, __ddiv_rn((double)(L / 2), den), m2);
            apply(L / 2, h, m2);
        }
    }
}

// The column part of one band-limited ASM step on registers v (the tile's
// forward transform is done, natural order q = tt + s*T): the spectrum goes
// to the tile, the alias-wrap histogram and H are applied there, and v is
// reloaded in the natural order of the inverse transform's first pass.
// cp.async (16 bytes, global -> shared, bypassing L1) and its completion.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Copy the table rows of the W columns from col0 to hs (shared memory); the
// copies complete under the forward transform (col_spectral_stage waits).
// HCP: entries are (H_hi, H_lo) pairs, 16 bytes.
template <int W, bool HCP>
__device__ __forceinline__ void htab_prefetch(float2* hs, const FastCols& a, int col0) {
    constexpr int U = HCP ? 2 : 1;  // float2 units per entry
    const float4* g =
        reinterpret_cast<const float4*>(a.htab + (long long)htab_row0(col0, a.ncols, W) * a.htab_ld * U);
    const int n16 = W * a.htab_ld * U / 2;
    for (int i = threadIdx.x; i < n16; i += blockDim.x) cp_async16(hs + 2 * i, g + i);
    cp_async_commit();
}

template <typename Real, int L, int E, int W, typename C, bool HCP = false>
__device__ __forceinline__ void col_spectral_stage(C* v, C* tile, double* hsm, int col0, const FastCols& a,
                                                   const HUnit& hu, double& p0, double& l1,
                                                   const float2* hs = nullptr) {
    constexpr int T = L / E;
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    if (hs) cp_async_wait_all();  // this thread's table copies (the barriers below publish them)
    __syncthreads();  // every thread has loaded its last forward pass
#pragma unroll
    for (int s = 0; s < E; s++) tile[(tt + s * T) * W + w] = v[s];
    __syncthreads();
    if (a.hist) {
        col_hist_bin(tile, hsm, col0, L, W, a.ncols, a.hist_dx);
        __syncthreads();
    }
    col_tile_h<Real, L, E, W, HCP>(tile, col0, a, hu, p0, l1, hs);
    __syncthreads();
#pragma unroll
    for (int s = 0; s < E; s++) v[s] = tile[(tt + s * T) * W + w];
}

// Per-CTA record blk of the loss sums [sum |F|^2, sum |F|^2 (1 - |H|^2)] and
// of the histogram; every thread of the CTA calls this.
__device__ __forceinline__ void col_write_red(const FastCols& a, long long blk, double p0, double l1,
                                              const double* hsm) {
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
            double* o = a.red + blk * a.red_stride;
            o[0] = t0;
            o[1] = t1;
        }
    }
    if (a.hist) {
        __syncthreads();
        double* o = a.hist + blk * a.red_stride;
        for (int k = threadIdx.x; k < 97; k += blockDim.x) o[k] = hsm[k];
    }
}

}  // namespace wos

// wos_fft.cuh -- CTA-cooperative Stockham line FFT for sm_100a.
//
// A "line" is one row or one column of a field (length L, a power of two; for
// Bluestein lines L is the padded convolution length M).  A group of T = L/E
// threads owns a line; every thread keeps E complex values in registers.  Each
// pass is a radix-R decimation-in-time Stockham butterfly (R = E, plus at most
// one smaller pass), with twiddles from an FP64-generated table, and passes
// exchange data through shared memory.  The forward radix order is
// (rs, E, ..., E) and the inverse order is its reverse, so that the values a
// thread holds after a forward FFT are exactly the inputs of its first inverse
// pass (and vice versa): a fused FFT . pointwise . IFFT never round-trips
// shared memory at the junction.
//
// Register mapping of a radix-R pass (the "natural" mapping):
//   v[b*R + r] = x[j_b + r*(L/R)],  j_b = tt + b*T,  b < E/R
// which, for the first and last pass, is also a coalesced global mapping.
//
// Transforms are unnormalised: forward uses exp(-2 pi i k n / L), inverse uses
// exp(+2 pi i k n / L); 1/L factors are folded into the pointwise stages.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace wos {

// Dynamic shared memory above which a kernel must opt in: the 48 KiB default
// limit covers dynamic plus static shared memory, and the sweeps keep up to
// 2 KiB of static reduction scratch.
constexpr size_t kSmemNoOptIn = 46 * 1024;


template <typename R> struct CT;
template <> struct CT<float> { using t = float2; };
template <> struct CT<double> { using t = double2; };

template <typename C> __device__ __forceinline__ C mkc(decltype(C::x) a, decltype(C::x) b) { C r; r.x = a; r.y = b; return r; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mkc<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mkc<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mkc<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {  // a * conj(b)
    return mkc<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mkc<C>(a.x * s, a.y * s); }
// complex64 sums and differences as one paired-FP32 instruction each (sm_100:
// add/sub.f32x2 on a 64-bit register pair, IEEE round-to-nearest per lane,
// i.e. the same results as two scalar operations); the butterflies of every
// line transform are made of these
#if !defined(WOS_SCALAR_CADD)
__device__ __forceinline__ unsigned long long f2_bits(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 f2_from(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_from(d);
}
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_from(d);
}
#endif
template <typename C> __device__ __forceinline__ C cconj(C a) { return mkc<C>(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C mul_mi(C a) {
    return INV ? mkc<C>(-a.y, a.x) : mkc<C>(a.y, -a.x);
}

template <typename C> __device__ __forceinline__ C ldg_c(const C* p) { return __ldg(p); }

// ---------------------------------------------------------------- small DFTs
template <bool INV, typename C>
__device__ __forceinline__ void dft2(C& a, C& b) {
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

// Butterfly a = e + w x, b = e - w x for w = -i (forward) or +i (inverse):
// four scalar adds with the swap and sign folded into the operands (the
// paired add would first have to build the swapped, negated pair).
template <bool INV, typename C>
__device__ __forceinline__ void bfly_mi(C& a, C& b, C e, C x) {
    if (INV) {
        a = mkc<C>(e.x - x.y, e.y + x.x);
        b = mkc<C>(e.x + x.y, e.y - x.x);
    } else {
        a = mkc<C>(e.x + x.y, e.y - x.x);
        b = mkc<C>(e.x - x.y, e.y + x.x);
    }
}

template <bool INV, typename C>
__device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
    C a0 = cadd(v0, v2), a1 = csub(v0, v2);
    C a2 = cadd(v1, v3), d = csub(v1, v3);
    v0 = cadd(a0, a2);
    v2 = csub(a0, a2);
    bfly_mi<INV>(v1, v3, a1, d);
}

template <typename C> struct K;
template <> struct K<float2> {
    static constexpr float S2 = 0.70710678118654752440f;
    static constexpr float C8 = 0.92387953251128675613f;
    static constexpr float S8 = 0.38268343236508977173f;
    // residuals of the single-precision constants (value - S2 etc., rounded):
    // with them a rotation is exact to ~2^-48 instead of 2^-25, which matters
    // where the same transform pair runs hundreds of times (split-step slices)
    static constexpr float S2L = (float)(0.70710678118654752440 - (double)S2);
    static constexpr float C8L = (float)(0.92387953251128675613 - (double)C8);
    static constexpr float S8L = (float)(0.38268343236508977173 - (double)S8);
};
template <> struct K<double2> {
    static constexpr double S2 = 0.70710678118654752440;
    static constexpr double C8 = 0.92387953251128675613;
    static constexpr double S8 = 0.38268343236508977173;
};

// w8^k * x for k = 1, 3 (forward: w = exp(-i pi/4))
template <bool INV, typename C> __device__ __forceinline__ C w8_1(C x) {
    const auto s = K<C>::S2;
    return INV ? mkc<C>((x.x - x.y) * s, (x.x + x.y) * s) : mkc<C>((x.x + x.y) * s, (x.y - x.x) * s);
}
template <bool INV, typename C> __device__ __forceinline__ C w8_3(C x) {
    const auto s = K<C>::S2;
    return INV ? mkc<C>(-(x.x + x.y) * s, (x.x - x.y) * s) : mkc<C>((x.y - x.x) * s, -(x.x + x.y) * s);
}

// Butterfly for w = w8^k (k = 1, 3): w x = sqrt(1/2) u with u the sums and
// differences of x's parts; complex64 takes e +- sqrt(1/2) u as two paired
// FMAs (fma.rn.f32x2, one rounding per lane), complex128 the products of
// w8_1 / w8_3 and a sum and a difference.
template <int k, bool INV, typename C>
__device__ __forceinline__ void bfly_w8(C& a, C& b, C e, C x) {
    const C t = k == 1 ? w8_1<INV>(x) : w8_3<INV>(x);
    a = cadd(e, t);
    b = csub(e, t);
}
#if !defined(WOS_SCALAR_CADD)
__device__ __forceinline__ float2 f2_fma(float2 s, float2 u, float2 e) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(s)), "l"(f2_bits(u)), "l"(f2_bits(e)));
    return f2_from(d);
}
template <int k, bool INV>
__device__ __forceinline__ void bfly_w8_f2(float2& a, float2& b, float2 e, float2 x) {
    float2 u;
    if (k == 1) u = INV ? make_float2(x.x - x.y, x.x + x.y) : make_float2(x.x + x.y, x.y - x.x);
    else u = INV ? make_float2(-x.x - x.y, x.x - x.y) : make_float2(x.y - x.x, -x.x - x.y);
    const float s = K<float2>::S2;
    a = f2_fma(make_float2(s, s), u, e);
    b = f2_fma(make_float2(-s, -s), u, e);
}
template <> __device__ __forceinline__ void bfly_w8<1, false, float2>(float2& a, float2& b, float2 e, float2 x) {
    bfly_w8_f2<1, false>(a, b, e, x);
}
template <> __device__ __forceinline__ void bfly_w8<1, true, float2>(float2& a, float2& b, float2 e, float2 x) {
    bfly_w8_f2<1, true>(a, b, e, x);
}
template <> __device__ __forceinline__ void bfly_w8<3, false, float2>(float2& a, float2& b, float2 e, float2 x) {
    bfly_w8_f2<3, false>(a, b, e, x);
}
template <> __device__ __forceinline__ void bfly_w8<3, true, float2>(float2& a, float2& b, float2 e, float2 x) {
    bfly_w8_f2<3, true>(a, b, e, x);
}
#endif

// Compensated rotations (CP): the constant c is applied as c_hi + c_lo, the
// small product with c_lo folded in first, so that the rotation's own error
// is that of the data rounding only (complex64).
#if !defined(WOS_SCALAR_CADD)
template <int k, bool INV>
__device__ __forceinline__ void bfly_w8_cp(float2& a, float2& b, float2 e, float2 x) {
    float2 u;
    if (k == 1) u = INV ? make_float2(x.x - x.y, x.x + x.y) : make_float2(x.x + x.y, x.y - x.x);
    else u = INV ? make_float2(-x.x - x.y, x.x - x.y) : make_float2(x.y - x.x, -x.x - x.y);
    const float s = K<float2>::S2, sl = K<float2>::S2L;
    a = f2_fma(make_float2(s, s), u, f2_fma(make_float2(sl, sl), u, e));
    b = f2_fma(make_float2(-s, -s), u, f2_fma(make_float2(-sl, -sl), u, e));
}
#endif
template <int k, bool INV, bool CP, typename C>
__device__ __forceinline__ void bfly_w8x(C& a, C& b, C e, C x) {
#if !defined(WOS_SCALAR_CADD)
    if constexpr (CP && sizeof(C) == 8) {
        bfly_w8_cp<k, INV>(a, b, e, x);
        return;
    }
#endif
    bfly_w8<k, INV>(a, b, e, x);
}

template <bool INV, typename C, bool CP = false>
__device__ __forceinline__ void dft8(C* v) {
    // even / odd radix-4 then combine
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    bfly_w8x<1, INV, CP>(v[1], v[5], e1, o1);
    bfly_mi<INV>(v[2], v[6], e2, o2);
    bfly_w8x<3, INV, CP>(v[3], v[7], e3, o3);
}

// multiply by w16^k (forward w16 = exp(-2 pi i/16)), k = 0..7
template <int k, bool INV, typename C>
__device__ __forceinline__ C w16(C x) {
    using T = decltype(C::x);
    if (k == 0) return x;
    if (k == 4) return mul_mi<INV>(x);
    if (k == 2) return w8_1<INV>(x);
    if (k == 6) return w8_3<INV>(x);
    T c, s;  // w = c - i s (forward)
    if (k == 1) { c = K<C>::C8; s = K<C>::S8; }
    else if (k == 3) { c = K<C>::S8; s = K<C>::C8; }
    else if (k == 5) { c = -K<C>::S8; s = K<C>::C8; }
    else { c = -K<C>::C8; s = K<C>::S8; }  // k == 7
    if (INV) s = -s;
    return mkc<C>(x.x * c + x.y * s, x.y * c - x.x * s);
}

// w16^k x (k odd) with the constants as hi + lo pairs (complex64, CP).
template <int k, bool INV>
__device__ __forceinline__ float2 w16_cp(float2 x) {
    float c, s, cl, sl;  // w = c - i s (forward)
    if (k == 1) { c = K<float2>::C8; s = K<float2>::S8; cl = K<float2>::C8L; sl = K<float2>::S8L; }
    else if (k == 3) { c = K<float2>::S8; s = K<float2>::C8; cl = K<float2>::S8L; sl = K<float2>::C8L; }
    else if (k == 5) { c = -K<float2>::S8; s = K<float2>::C8; cl = -K<float2>::S8L; sl = K<float2>::C8L; }
    else { c = -K<float2>::C8; s = K<float2>::S8; cl = -K<float2>::C8L; sl = K<float2>::S8L; }
    if (INV) { s = -s; sl = -sl; }
    const float tx = fmaf(x.x, cl, x.y * sl), ty = fmaf(x.y, cl, -(x.x * sl));
    return make_float2(fmaf(x.x, c, fmaf(x.y, s, tx)), fmaf(x.y, c, fmaf(-x.x, s, ty)));
}
template <int k, bool INV, bool CP, typename C>
__device__ __forceinline__ C w16x(C x) {
    if constexpr (CP && sizeof(C) == 8) return w16_cp<k, INV>(x);
    else return w16<k, INV>(x);
}

template <bool INV, typename C, bool CP = false>
__device__ __forceinline__ void dft16(C* v) {
    C e[8], o[8];
#pragma unroll
    for (int i = 0; i < 8; i++) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
    dft8<INV, C, CP>(e);
    dft8<INV, C, CP>(o);
    o[1] = w16x<1, INV, CP>(o[1]); o[3] = w16x<3, INV, CP>(o[3]);
    o[5] = w16x<5, INV, CP>(o[5]); o[7] = w16x<7, INV, CP>(o[7]);
#pragma unroll
    for (int i = 0; i < 8; i += 2) { v[i + 1] = cadd(e[i + 1], o[i + 1]); v[i + 9] = csub(e[i + 1], o[i + 1]); }
    v[0] = cadd(e[0], o[0]); v[8] = csub(e[0], o[0]);
    bfly_w8x<1, INV, CP>(v[2], v[10], e[2], o[2]);
    bfly_mi<INV>(v[4], v[12], e[4], o[4]);
    bfly_w8x<3, INV, CP>(v[6], v[14], e[6], o[6]);
}

// Radix 3 and 5 (mixed-radix lines): the DFT sums written with the real and
// imaginary parts of the roots of unity, w = exp(-2 pi i / R) forward.
template <typename C> struct K35;
template <> struct K35<float2> {
    static constexpr float S3 = 0.86602540378443864676f;  // sin(2 pi / 3)
    static constexpr float C51 = 0.30901699437494742410f; // cos(2 pi / 5)
    static constexpr float C52 = -0.80901699437494742410f;
    static constexpr float S51 = 0.95105651629515357212f;
    static constexpr float S52 = 0.58778525229247312917f;
};
template <> struct K35<double2> {
    static constexpr double S3 = 0.86602540378443864676;
    static constexpr double C51 = 0.30901699437494742410;
    static constexpr double C52 = -0.80901699437494742410;
    static constexpr double S51 = 0.95105651629515357212;
    static constexpr double S52 = 0.58778525229247312917;
};

template <bool INV, typename C>
__device__ __forceinline__ void dft3(C* v) {
    using T = decltype(C::x);
    const C s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const C m = mkc<C>(v[0].x - (T)0.5 * s.x, v[0].y - (T)0.5 * s.y);
    const T k = INV ? -K35<C>::S3 : K35<C>::S3;  // forward: -i sin(2pi/3) (v1 - v2)
    v[0] = cadd(v[0], s);
    v[1] = mkc<C>(m.x + k * d.y, m.y - k * d.x);
    v[2] = mkc<C>(m.x - k * d.y, m.y + k * d.x);
}

template <bool INV, typename C>
__device__ __forceinline__ void dft5(C* v) {
    using T = decltype(C::x);
    const C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const T c1 = K35<C>::C51, c2 = K35<C>::C52;
    const T s1 = INV ? -K35<C>::S51 : K35<C>::S51, s2 = INV ? -K35<C>::S52 : K35<C>::S52;
    // y_k = v0 + sum_r v_r w^{rk}: real parts from a, -i sin parts from b
    const C m1 = mkc<C>(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    const C m2 = mkc<C>(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    const C n1 = mkc<C>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);  // y1: -i * n1
    const C n2 = mkc<C>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);  // y2: -i * n2
    v[0] = mkc<C>(v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y);
    v[1] = mkc<C>(m1.x + n1.y, m1.y - n1.x);
    v[4] = mkc<C>(m1.x - n1.y, m1.y + n1.x);
    v[2] = mkc<C>(m2.x + n2.y, m2.y - n2.x);
    v[3] = mkc<C>(m2.x - n2.y, m2.y + n2.x);
}

template <int R, bool INV, typename C, bool CP = false>
__device__ __forceinline__ void dft(C* v) {
    if (R == 2) dft2<INV>(v[0], v[1]);
    else if (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
    else if (R == 8) dft8<INV, C, CP>(v);
    else if (R == 16) dft16<INV, C, CP>(v);
    else if (R == 3) dft3<INV>(v);
    else if (R == 5) dft5<INV>(v);
}

// ------------------------------------------------------------- shared layouts
// Line-contiguous layout (rows): line l at l*S, one pad slot per 16 elements.
struct RowIdx {
    int S;
    __device__ __forceinline__ int operator()(int line, int p) const { return line * S + p + (p >> 4); }
};
__host__ __device__ inline int row_line_stride(int L) { return L + (L >> 4) + 1; }

// Interleaved layout (columns): element (line w, position p) at p*W + w, padded.
struct ColIdx {
    int W;
    __device__ __forceinline__ int operator()(int line, int p) const {
        int i = p * W + line;
        return i + (i >> 4);
    }
};
__host__ __device__ inline int col_tile_elems(int L, int W) { int n = L * W; return n + (n >> 4) + 1; }

// ------------------------------------------------------------- pass pieces
template <int R, int E, bool INV, typename C>
__device__ __forceinline__ void pass_compute(C* v, int tt, int T, int Ns, int L, const C* __restrict__ tw) {
#pragma unroll
    for (int b = 0; b < E / R; b++) {
        if (Ns > 1) {
            const int j = tt + b * T;
            const int k = j & (Ns - 1);
            const int step = L / (Ns * R);
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = ldg_c(tw + r * k * step);
                if (INV) w.y = -w.y;
                v[b * R + r] = cmul(v[b * R + r], w);
            }
        }
        dft<R, INV>(v + b * R);
    }
}

template <int R, int E, typename C, typename IDX>
__device__ __forceinline__ void sm_store(const C* v, C* sm, const IDX& ix, int line, int tt, int T, int Ns) {
#pragma unroll
    for (int b = 0; b < E / R; b++) {
        const int j = tt + b * T;
        const int k = j & (Ns - 1);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) sm[ix(line, base + r * Ns)] = v[b * R + r];
    }
}

template <int R, int E, typename C, typename IDX>
__device__ __forceinline__ void sm_load(C* v, const C* sm, const IDX& ix, int line, int tt, int T, int L) {
    const int LR = L / R;
#pragma unroll
    for (int b = 0; b < E / R; b++) {
        const int j = tt + b * T;
#pragma unroll
        for (int r = 0; r < R; r++) v[b * R + r] = sm[ix(line, j + r * LR)];
    }
}

// Runtime radix dispatch helpers (R <= E, both powers of two).
#define WOS_DISPATCH_R(R_, E_, BODY)                    \
    do {                                                \
        switch (R_) {                                   \
        case 2: { constexpr int RR = 2; BODY; } break;  \
        case 4: { constexpr int RR = 4; BODY; } break;  \
        case 8: { constexpr int RR = 8; BODY; } break;  \
        default: { constexpr int RR = 16; BODY; } break; \
        }                                               \
    } while (0)

// Radix of pass p of a P-pass transform: forward (rs, E, ..., E), inverse reversed.
__device__ __forceinline__ int pass_radix(bool inv, int p, int P, int rs, int E) {
    if (rs > 1) {
        if (!inv && p == 0) return rs;
        if (inv && p == P - 1) return rs;
    }
    return E;
}

// Plan of a line transform: number of passes and the small radix.
struct LinePlan {
    int L;    // length (power of two, or 2^a 3^b 5^c for a mixed-radix line)
    int P;    // passes
    int rs;   // small radix (1 if none)
    int mixed;  // 1: radix 16/8/4/2/3/5 passes through shared memory (mixed_line_fft)
};
__host__ __device__ inline LinePlan make_line_plan(int L, int E) {
    LinePlan p;
    p.L = L;
    p.mixed = (L & (L - 1)) != 0;
    if (p.mixed) {  // registers hold positions tt + s*T on entry and exit
        p.P = 0;
        p.rs = 1;
        return p;
    }
    int lg = 0;
    while ((1 << lg) < L) lg++;
    int le = 0;
    while ((1 << le) < E) le++;
    p.P = lg / le + ((lg % le) ? 1 : 0);
    p.rs = (lg % le) ? (1 << (lg % le)) : 1;
    return p;
}
__host__ __device__ inline int first_radix(const LinePlan& lp, bool inv, int E) {
    return (!inv && lp.rs > 1) ? lp.rs : E;
}
__host__ __device__ inline int last_radix(const LinePlan& lp, bool inv, int E) {
    return (inv && lp.rs > 1) ? lp.rs : E;
}

// Full line transform.  On entry v holds the natural mapping for the first
// pass radix; on exit v holds the natural mapping for the last pass radix.
// Must be called by every thread of the CTA (it synchronises).
template <int E, bool INV, typename C, typename IDX>
__device__ __forceinline__ void line_fft(C* v, C* sm, const IDX& ix, int line, int tt, int T,
                                         const LinePlan& lp, const C* __restrict__ tw) {
    int Ns = 1;
    for (int p = 0; p < lp.P; p++) {
        const int R = pass_radix(INV, p, lp.P, lp.rs, E);
        WOS_DISPATCH_R(R, E, (pass_compute<RR, E, INV>(v, tt, T, Ns, lp.L, tw)));
        if (p < lp.P - 1) {
            const int R2 = pass_radix(INV, p + 1, lp.P, lp.rs, E);
            __syncthreads();
            WOS_DISPATCH_R(R, E, (sm_store<RR, E>(v, sm, ix, line, tt, T, Ns)));
            __syncthreads();
            WOS_DISPATCH_R(R2, E, (sm_load<RR, E>(v, sm, ix, line, tt, T, lp.L)));
        }
        Ns *= R;
    }
}

// Radix of the next pass of a mixed-radix plan with `rem` points left to
// factor: 16, 8, 4, 2 first, then 3, then 5 (host and device agree).
__host__ __device__ inline int mixed_radix_of(int rem) {
    if (rem % 16 == 0) return 16;
    if (rem % 8 == 0) return 8;
    if (rem % 4 == 0) return 4;
    if (rem % 2 == 0) return 2;
    if (rem % 3 == 0) return 3;
    return 5;
}
// Entries of the per-pass twiddle tables of a mixed-radix line of L points:
// pass p (radix R, sub-transform length NS) holds W_{NS R}^{r k} at [r-1][k].
__host__ __device__ inline int mixed_table_len(int L) {
    int rem = L, NS = 1, n = 0;
    while (rem > 1) {
        const int R = mixed_radix_of(rem);
        n += NS * (R - 1);
        NS *= R;
        rem /= R;
    }
    return n;
}

// One Stockham pass of a mixed-radix line from src to dst (shared memory), one
// radix-R butterfly at a time: each thread holds only the R values of its
// current butterfly (a pass in place would have to hold all of them across a
// barrier).  Sub-transform length NS; twiddles from the pass's table ptw
// ([r-1][k], consecutive k for consecutive threads).  k = j mod NS comes from a
// single-precision quotient corrected by one step (exact for j < 2^23).
template <int R, bool INV, typename C, typename IDX>
__device__ __forceinline__ void mixed_pass_pp(const C* src, C* dst, const IDX& ix, int line, int tt, int T, int L,
                                              int NS, const C* __restrict__ ptw) {
    const int LR = L / R;
    const float inv_ns = 1.0f / (float)NS;
    for (int j = tt; j < LR; j += T) {
        C x[R];
#pragma unroll
        for (int r = 0; r < R; r++) x[r] = src[ix(line, j + r * LR)];
        int k = j - (int)((float)j * inv_ns) * NS;
        if (k < 0) k += NS;
        else if (k >= NS) k -= NS;
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = ldg_c(ptw + (r - 1) * NS + k);
                if (INV) w.y = -w.y;
                x[r] = cmul(x[r], w);
            }
        }
        dft<R, INV>(x);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[ix(line, base + r * NS)] = x[r];
    }
}

// Mixed-radix line transform (L = 2^a 3^b 5^c, a >= 1): registers (positions
// tt + s*T) to shared memory, radix 16 / 8 / 4 / 2 then 3 then 5 passes
// alternating between sm and alt (two buffers of the same layout), back to
// the same registers.  tw: the L-point table followed by the per-pass tables
// (mixed_table_len(L) entries).  Must be called by every thread of the CTA
// (it synchronises).
template <int E, bool INV, typename C, typename IDX>
__device__ __forceinline__ void mixed_line_fft(C* v, C* sm, C* alt, const IDX& ix, int line, int tt, int T, int L,
                                               const C* __restrict__ tw) {
    __syncthreads();
#pragma unroll
    for (int s = 0; s < E; s++) sm[ix(line, tt + s * T)] = v[s];
    __syncthreads();
    C* src = sm;
    C* dst = alt;
    const C* ptw = tw + L;
    int rem = L, NS = 1;
    while (rem > 1) {
        const int R = mixed_radix_of(rem);
        switch (R) {
        case 16: mixed_pass_pp<16, INV>(src, dst, ix, line, tt, T, L, NS, ptw); break;
        case 8: mixed_pass_pp<8, INV>(src, dst, ix, line, tt, T, L, NS, ptw); break;
        case 4: mixed_pass_pp<4, INV>(src, dst, ix, line, tt, T, L, NS, ptw); break;
        case 2: mixed_pass_pp<2, INV>(src, dst, ix, line, tt, T, L, NS, ptw); break;
        case 3: mixed_pass_pp<3, INV>(src, dst, ix, line, tt, T, L, NS, ptw); break;
        default: mixed_pass_pp<5, INV>(src, dst, ix, line, tt, T, L, NS, ptw); break;
        }
        __syncthreads();
        C* t = src;
        src = dst;
        dst = t;
        ptw += NS * (R - 1);
        NS *= R;
        rem /= R;
    }
#pragma unroll
    for (int s = 0; s < E; s++) v[s] = src[ix(line, tt + s * T)];
}

// Position held by register slot s (= b*R + r) under the natural mapping of radix R.
__device__ __forceinline__ int nat_pos(int s, int R, int tt, int T, int L) {
    const int b = s / R, r = s % R;
    return tt + b * T + r * (L / R);
}

// FP64 helpers of the complex64 transfer functions (specialised and lean sweeps).
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
// 1.5 * 2^23 float pattern.  `precise` evaluates sin/cos of that exact fraction
// to about 1 ulp (sincospif, for transfer functions applied hundreds of times,
// whose errors add up); otherwise the hardware approximation (absolute error
// about 2^-21) serves a single application.
__device__ __forceinline__ float2 cexp_rev(double t, bool precise) {
    const double u = t + 805306368.0;  // 1.5 * 2^29
    const int s23 = (int)((unsigned)__double2loint(u) << 9) >> 9;
    const float f = __int_as_float(0x4b400000 + s23) - 12582912.0f;
    float sn, cs;
    if (precise) sincospif(f * 2.384185791015625e-07f, &sn, &cs);  // 2^-22: half-revolutions
    else __sincosf(f * 7.490140565847857e-07f, &sn, &cs);            // 2 pi / 2^23
    return make_float2(cs, sn);
}

}  // namespace wos

// wos_kernels_dev.cuh -- device code of the general sweeps (k_rows, k_cols)
// and their helpers, shared by the translation unit of the power-of-two /
// Bluestein instantiations (wos_kernels.cu) and those of the mixed-radix ones
// (wos_kernels_mix*.cu), which compile in parallel.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "wos_fft.cuh"
#include "wos_kernels.cuh"

namespace wos {

// ------------------------------------------------------------------ helpers
template <typename C>
__device__ __forceinline__ C load_elem(const void* base, int is_c128, long long idx) {
    if (is_c128) {
        double2 d = reinterpret_cast<const double2*>(base)[idx];
        return mkc<C>((decltype(C::x))d.x, (decltype(C::x))d.y);
    }
    return reinterpret_cast<const C*>(base)[idx];
}
template <typename C>
__device__ __forceinline__ void store_elem(void* base, int is_c128, long long idx, C v) {
    if (is_c128) {
        double2 d;
        d.x = (double)v.x;
        d.y = (double)v.y;
        reinterpret_cast<double2*>(base)[idx] = d;
    } else {
        reinterpret_cast<C*>(base)[idx] = v;
    }
}

// FP64 operations that are never contracted into FMAs: the argument of every
// transfer function is formed with exactly the reference's rounding sequence.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// math.Hypot as the reference evaluates it (scale by the larger magnitude).
__device__ __forceinline__ double go_hypot(double p, double q) {
    p = fabs(p);
    q = fabs(q);
    if (isinf(p) || isinf(q)) return INFINITY;
    if (p < q) { double t = p; p = q; q = t; }
    if (p == 0) return 0;
    q = ddiv(q, p);
    return dmul(p, __dsqrt_rn(dadd(1.0, dmul(q, q))));
}

// freq (optics/field.go:297-303) on a grid of n points.
__device__ __forceinline__ double freq_n(int i, int n, double dx) {
    const double den = dmul((double)n, dx);
    return (i <= n / 2) ? ddiv((double)i, den) : ddiv((double)(i - n), den);
}

// exp(i*arg) in the pipeline's precision.  FP64: sincos of the full argument.
// FP32: the FP64 argument is reduced to [-pi, pi] in FP64 (Cody-Waite with a
// two-term 2*pi), then evaluated with single-precision sincosf.
template <typename C> __device__ __forceinline__ C cexpi(double arg);
template <> __device__ __forceinline__ double2 cexpi<double2>(double arg) {
    double s, c;
    sincos(arg, &s, &c);
    return make_double2(c, s);
}
__device__ __forceinline__ float reduce_2pi(double arg) {
    const double inv2pi = 0.15915494309189533577;
    const double p2hi = 6.283185307179586232;
    const double p2lo = 2.4492935982947064e-16;
    double n = rint(arg * inv2pi);
    double r = fma(-n, p2hi, arg);
    r = fma(-n, p2lo, r);
    return (float)r;
}
template <> __device__ __forceinline__ float2 cexpi<float2>(double arg) {
    float s, c;
    sincosf(reduce_2pi(arg), &s, &c);
    return make_float2(c, s);
}

// asmTF (optics/propagate.go:159-181) at (fx, fy).  m2 receives |H|^2 in FP64
// (exactly 1 for propagating components), from which the power lost in a step
// is summed without cancellation whatever the pipeline precision.
template <typename C>
__device__ __forceinline__ C asm_tf(const HArgs& h, double wl, double kz, double kaz, bool backward,
                                    double fx, double fy, double& m2) {
    using T = decltype(C::x);
    double decay;
    if (h.exact) {
        const double rho = go_hypot(dmul(wl, fx), dmul(wl, fy));
        if (rho <= 1.0) {
            m2 = 1.0;
            return cexpi<C>(dmul(kz, __dsqrt_rn(dmul(dsub(1.0, rho), dadd(1.0, rho)))));
        }
        decay = dmul(kaz, __dsqrt_rn(dmul(dsub(rho, 1.0), dadd(rho, 1.0))));
    } else {
        // separable form 1 - (wl fx)^2 - (wl fy)^2 = (1-rho)(1+rho), FP64 argument
        const double ax = wl * fx, ay = wl * fy;
        const double s = fma(-ay, ay, fma(-ax, ax, 1.0));
        if (s >= 0) {
            m2 = 1.0;
            return cexpi<C>(kz * sqrt(s));
        }
        decay = kaz * sqrt(-s);
    }
    double a;
    if (h.zero_ev || (h.limit > 0 && decay > h.limit)) a = 0;
    else if (backward) {
        if (h.reg) {
            const double e = exp(decay);
            a = h.exact ? ddiv(e, dadd(1.0, dmul(dmul(dmul(h.alpha, h.alpha), e), e)))
                        : e / (1.0 + h.alpha * h.alpha * e * e);
        } else {
            a = exp(decay);
        }
    } else {
        a = exp(-decay);
    }
    m2 = a * a;
    return mkc<C>((T)a, 0);
}

// Transfer function H(col, q) with normalisation; per-batch wl / z overrides.
// m2 = |H|^2 before normalisation (FP64).
template <typename C>
__device__ __forceinline__ C eval_h(const HArgs& h, double wl, double z, int col, int q, double& m2) {
    using T = decltype(C::x);
    const double fx = h.fxoff != 0 ? dadd(freq_n(col, h.lfx, h.dx), h.fxoff) : freq_n(col, h.lfx, h.dx);
    const double fy = h.fyoff != 0 ? dadd(freq_n(q, h.lfy, h.dx), h.fyoff) : freq_n(q, h.lfy, h.dx);
    C r;
    m2 = 1.0;
    switch (h.kind) {
    case H_ASM: {
        const double k = (wl == h.wl) ? h.k : 2 * M_PI / wl;
        const double kz = (wl == h.wl && z == h.z) ? h.kz : k * z;
        const double kaz = (wl == h.wl && z == h.z) ? h.kaz : k * fabs(z);
        r = asm_tf<C>(h, wl, kz, kaz, z < 0, fx, fy, m2);
    } break;
    case H_ASM_HALF2: {
        C a = asm_tf<C>(h, wl, h.kz, h.kaz, h.z < 0, fx, fy, m2);
        r = cmul(a, a);
        m2 = m2 * m2;
    } break;
    case H_FRESNEL_TF: {
        // cexpI(k z) * cexpI(-pi wl z (fx^2+fy^2))   (propagate.go:511-513)
        const double ph = h.exact ? dmul(dmul(dmul(-M_PI, wl), z), dadd(dmul(fx, fx), dmul(fy, fy)))
                                  : (-M_PI * wl * z) * (fx * fx + fy * fy);
        r = cmul(mkc<C>((T)h.c_re, (T)h.c_im), cexpi<C>(ph));
    } break;
    case H_TABLE_XY: {
        const C* tx = reinterpret_cast<const C*>(h.tx);
        const C* ty = reinterpret_cast<const C*>(h.ty);
        r = cmul(cmul(ldg_c(tx + col), ldg_c(ty + q)), mkc<C>((T)h.c_re, (T)h.c_im));
    } break;
    case H_GAUSS: {
        // exp(c corr^2 f^2) with p0 = c corr^2 formed on the host, c = -2 pi^2
        const double a = h.exact ? dmul(h.p0, dadd(dmul(fx, fx), dmul(fy, fy))) : h.p0 * (fx * fx + fy * fy);
        r = mkc<C>((T)exp(a), 0);
    } break;
    case H_BANDLIMIT: {
        const double fr = go_hypot(fx, fy);
        r = mkc<C>(1, 0);
        if (fr > h.p0) {
            const double d = h.exact ? ddiv(dsub(fr, h.p0), h.p1) : (fr - h.p0) / h.p1;
            r = mkc<C>((T)exp(h.exact ? -dmul(d, d) : -(d * d)), 0);
        }
    } break;
    case H_SHIFT: {
        const double a = h.exact ? dmul(-2 * M_PI, dadd(dmul(fx, h.p0), dmul(fy, h.p1)))
                                 : (-2 * M_PI) * (fx * h.p0 + fy * h.p1);
        r = cexpi<C>(a);
    } break;
    case H_UNIAX_O:
    case H_UNIAX_E: {
        // arg = k0^2 n^2 - (n_e/n_o)^2 kx^2 - ky^2 (extraordinary) or
        // k0^2 n_o^2 - kx^2 - ky^2 (ordinary), in the reference's order;
        // evanescent components decay as exp(-|z| sqrt(-arg))
        const double kx = dmul(2 * M_PI, fx), ky = dmul(2 * M_PI, fy);
        double arg;
        if (h.kind == H_UNIAX_O) {
            arg = dsub(dsub(dmul(dmul(dmul(h.k, h.k), h.p0), h.p0), dmul(kx, kx)), dmul(ky, ky));
        } else {
            const double rr = ddiv(dmul(h.p1, h.p1), dmul(h.p0, h.p0));
            arg = dsub(dsub(dmul(dmul(dmul(h.k, h.k), h.p1), h.p1), dmul(dmul(rr, kx), kx)), dmul(ky, ky));
        }
        if (arg < 0) r = mkc<C>((T)exp(-dmul(fabs(z), __dsqrt_rn(-arg))), 0);
        else r = cexpi<C>(dmul(z, __dsqrt_rn(arg)));
    } break;
    default: r = mkc<C>(1, 0); break;
    }
    if (h.conj) r.y = -r.y;
    return cscale(r, (T)h.scale);
}

// Block-wide FP64 sum of K accumulators, written by thread 0 to out[0..K).
// Compensated (Neumaier) addition: s + c carries the sum of everything added
// with the rounding error of each addition kept in c.
__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

// Compensated block sum of K per-thread pairs (s[k] + c[k]); thread 0 writes
// the high parts to hi[k] and the low parts to lo[k].
template <int K>
__device__ __forceinline__ void block_sum2_write(double (&s)[K], double (&c)[K], double* hi, double* lo) {
    __shared__ double rsm2[32][K][2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // a previous reduction's readers are done with rsm2
#pragma unroll
    for (int k = 0; k < K; k++) {
        double v = s[k], e = c[k];
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_down_sync(0xffffffffu, v, o);
            const double e2 = __shfl_down_sync(0xffffffffu, e, o);
            e += e2;
            neumaier_add(v, e, v2);
        }
        if (lane == 0) {
            rsm2[warp][k][0] = v;
            rsm2[warp][k][1] = e;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < K; k++) {
            double ts = 0, tc = 0;
            for (int w = 0; w < nw; w++) {
                tc += rsm2[w][k][1];
                neumaier_add(ts, tc, rsm2[w][k][0]);
            }
            hi[k] = ts;
            lo[k] = tc;
        }
    }
}

template <int K>
__device__ __forceinline__ void block_sum_write(double (&acc)[K], double* out) {
    __shared__ double rsm[32][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // a previous reduction's readers are done with rsm
#pragma unroll
    for (int k = 0; k < K; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) rsm[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < K; k++) {
            double s = 0;
            for (int w = 0; w < nw; w++) s += rsm[w][k];
            out[k] = s;
        }
    }
}

// Refractive index n(x,y,z) of a parametric medium, then the slice screen
// t = exp(-k Im(n) dz) * exp(i k (Re(n)-1) dz)   (optics/medium.go:50-65).
template <typename C>
__device__ __forceinline__ C screen_eval(const ScreenArgs& s, int i, int j, int ny, int nx, double x,
                                         double y) {
    using T = decltype(C::x);
    double nr, ni;
    if (s.kind == 2) {
        const long long idx = (long long)j * nx + i;
        nr = s.nre[idx];
        ni = s.nim[idx];
    } else {
        double r0 = s.re_bg, i0 = s.im_bg;
        for (int k = 0; k < s.n_layers && k < 8; k++) {
            if (s.zc < s.layer_z[k]) { r0 = s.layer_re[k]; i0 = s.layer_im[k]; break; }
        }
        nr = r0;
        ni = i0;
        if (s.core_dn != 0) {
            const double ddx = dsub(x, s.core_x0), ddy = dsub(y, s.core_y0);
            const double g = exp(ddiv(-dadd(dmul(ddx, ddx), dmul(ddy, ddy)), dmul(s.core_w, s.core_w)));
            double mod = 1;
            if (s.zmod_amp != 0)
                mod = dadd(1.0, dmul(s.zmod_amp,
                                     sin(dadd(ddiv(dmul(2 * M_PI, s.zc), s.zmod_period), s.zmod_phase))));
            nr = dadd(r0, dmul(dmul(s.core_dn, g), mod));
        }
        if (s.border_px > 0 && s.border_strength != 0) {
            int dd = i;
            if (j < dd) dd = j;
            if (nx - 1 - i < dd) dd = nx - 1 - i;
            if (ny - 1 - j < dd) dd = ny - 1 - j;
            if (dd < s.border_px) {
                const double t = ddiv((double)(s.border_px - dd), (double)s.border_px);
                double p = 1;
                for (int q = 0; q < s.border_order; q++) p = dmul(p, t);
                ni = dadd(i0, dmul(s.border_strength, p));
            }
        }
    }
    const double ph = dmul(dmul(s.k, dsub(nr, 1.0)), s.dz);
    const double amp = exp(dmul(dmul(-s.k, ni), s.dz));
    C e = cexpi<C>(ph);
    if (s.conj) e.y = -e.y;
    return mkc<C>((T)(amp * (double)e.x), (T)(amp * (double)e.y));
}

__device__ __forceinline__ double gX(int i, int nx, double dx) { return dmul(dsub((double)i, (double)nx / 2), dx); }

// ------------------------------------------------------------------ transforms
// Line transforms on the register array.  "Conv" is the Bluestein convolution
// M-FFT . B^ . M-IFFT (chirps are applied by the callers, where they can be
// merged with other pointwise factors).
//   radix of the register mapping on entry / exit:
//     plain forward : in first_radix(fwd), out E
//     plain inverse : in E,               out last_radix(inv)
//     Bluestein     : in first_radix(fwd), out last_radix(inv)
__device__ __forceinline__ int in_radix(const LinePlan& lp, bool inv, bool blue, int E) {
    return (blue || !inv) ? first_radix(lp, false, E) : E;
}
__device__ __forceinline__ int out_radix(const LinePlan& lp, bool inv, bool blue, int E) {
    return (blue || inv) ? last_radix(lp, true, E) : E;
}
// alt: the second shared-memory buffer of the mixed-radix kernels (same
// layout as sm, placed after it), null otherwise.
template <int E, bool MIX, typename C, typename IDX>
__device__ __forceinline__ void xform(C* v, C* sm, C* alt, const IDX& ix, int line, int tt, int T,
                                      const LinePlan& lp, const C* __restrict__ tw, bool inv,
                                      const C* __restrict__ bhat) {
    if constexpr (MIX) {  // kernels launched for mixed-radix lines only
        if (inv) mixed_line_fft<E, true>(v, sm, alt, ix, line, tt, T, lp.L, tw);
        else mixed_line_fft<E, false>(v, sm, alt, ix, line, tt, T, lp.L, tw);
        return;
    }
    if (!bhat) {
        if (inv) line_fft<E, true>(v, sm, ix, line, tt, T, lp, tw);
        else line_fft<E, false>(v, sm, ix, line, tt, T, lp, tw);
        return;
    }
    line_fft<E, false>(v, sm, ix, line, tt, T, lp, tw);
    const int Rm = last_radix(lp, false, E);
#pragma unroll
    for (int s = 0; s < E; s++) v[s] = cmul(v[s], ldg_c(bhat + nat_pos(s, Rm, tt, T, lp.L)));
    line_fft<E, true>(v, sm, ix, line, tt, T, lp, tw);
}

template <typename Real, int E> struct MaxT { static constexpr int v = (E >= 16 || sizeof(Real) == 8) ? 512 : 1024; };

// ------------------------------------------------------------------ k_rows
template <typename Real, int E, bool MIX>
__global__ void __launch_bounds__(MaxT<Real, E>::v) k_rows(const RowArgs a) {
    using C = typename CT<Real>::t;
    using T_ = Real;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int L = a.L;
    const int T = L / E;
    const int lines = blockDim.x / T;
    const int line = threadIdx.x / T, tt = threadIdx.x - line * T;
    const int r = blockIdx.x * lines + line;
    const bool act = r < a.rows;
    const int bz = blockIdx.y;
    const int grow = a.row0 + r;  // grid row (coordinates)
    const RowIdx ix{row_line_stride(L)};
    C* const alt = MIX ? sm + (size_t)row_line_stride(L) * lines : nullptr;  // launched with two buffers
    const LinePlan lp = make_line_plan(L, E);
    const C* tw = reinterpret_cast<const C*>(a.tw);
    const bool blue = a.blue_n > 0;
    const int Lq = blue ? a.blue_n : L;
    const C* chirp = reinterpret_cast<const C*>(a.chirp);
    const C* bhf = blue ? reinterpret_cast<const C*>(a.bhat_f) : nullptr;
    const C* bhi = blue ? reinterpret_cast<const C*>(a.bhat_i) : nullptr;
    double acc[4] = {0, 0, 0, 0};
    const double yrow = gX(grow, a.ny_grid, a.dx);
    const bool fwd_first = (a.mode == ROW_FWD);

    C v[E];
    Real iacc[E];
    const int nb = (a.mode == ROW_INV_ACC) ? a.acc_nb : 1;
    int Rout = 0;
    for (int bb = 0; bb < nb; bb++) {
        const long long ibase = (long long)(a.mode == ROW_INV_ACC ? bb : bz) * a.in_bstride + (long long)r * a.in_ld;
        // ---- load (register mapping of the first pass)
        const int R1 = MIX ? E : in_radix(lp, !fwd_first, blue, E);  // mixed lines: natural radix E
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int p = nat_pos(s, R1, tt, T, L);
            C x = mkc<C>(0, 0);
            if (act && p >= a.in_off && p < a.in_off + a.in_n) {
                const int i = p - a.in_off;
                x = load_elem<C>(a.in, a.in_c128, ibase + i);
                if (fwd_first) {
                    if (a.pre_phi || a.pre_phi_f) {
                        const long long gi = (long long)grow * a.nx_grid + i;
                        const double phi = a.pre_phi ? a.pre_phi[gi] : (double)a.pre_phi_f[gi];
                        x = cscale(cmul(x, cexpi<C>(phi)), (T_)a.pre_amp);
                    }
                    if (a.pre_shift) {
                        const double arg = dmul(dmul(-2.0, M_PI), dadd(dmul(a.fxc, gX(i, a.nx_grid, a.dx)), dmul(a.fyc, yrow)));
                        x = cmul(x, cexpi<C>(arg));
                    }
                    if (a.red_pre) {
                        const double w = (double)x.x * x.x + (double)x.y * x.y;
                        acc[0] += w;
                        if (a.red_moments) {
                            const double xx = gX(i, a.nx_grid, a.dx);
                            acc[1] += w * xx;
                            acc[2] += w * yrow;
                            acc[3] += w * (xx * xx + yrow * yrow);
                        }
                    }
                }
                if (blue) {
                    const C c = ldg_c(chirp + p);
                    x = fwd_first ? cmul(x, c) : cmulc(x, c);
                }
            }
            v[s] = x;
        }

        // ---- transform(s)
        xform<E, MIX>(v, sm, alt, ix, line, tt, T, lp, tw, !fwd_first, fwd_first ? bhf : bhi);
        Rout = MIX ? E : out_radix(lp, !fwd_first, blue, E);
        if (a.mode == ROW_INV_FWD) {
            // real-space screen between the inverse and the next forward row
            // transform; for Bluestein lines the conj(chirp) / chirp pair
            // around the screen cancels and is not applied
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int q = nat_pos(s, Rout, tt, T, L);
                if (q < Lq) {
                    if (act) v[s] = cmul(v[s], screen_eval<C>(a.scr, q, grow, a.ny_grid, a.nx_grid, gX(q, a.nx_grid, a.dx), yrow));
                } else {
                    v[s] = mkc<C>(0, 0);
                }
            }
            xform<E, MIX>(v, sm, alt, ix, line, tt, T, lp, tw, false, bhf);
            Rout = MIX ? E : out_radix(lp, false, blue, E);
            if (blue) {
#pragma unroll
                for (int s = 0; s < E; s++) {
                    const int q = nat_pos(s, Rout, tt, T, L);
                    if (q < Lq) v[s] = cmul(v[s], ldg_c(chirp + q));
                }
            }
        } else if (blue) {
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int q = nat_pos(s, Rout, tt, T, L);
                if (q < Lq) {
                    const C c = ldg_c(chirp + q);
                    v[s] = fwd_first ? cmul(v[s], c) : cmulc(v[s], c);
                }
            }
        }
        if (a.mode == ROW_INV_ACC) {
            const double wgt = a.acc_weight ? a.acc_weight[bb] : 1.0;
#pragma unroll
            for (int s = 0; s < E; s++) {
                const C x = cscale(v[s], (T_)a.out_scale);
                const Real pw = (Real)(wgt * ((double)x.x * x.x + (double)x.y * x.y));
                iacc[s] = (bb == 0) ? pw : iacc[s] + pw;
            }
        }
    }

    // ---- store
    const long long obase = (long long)bz * a.out_bstride + (long long)r * a.out_ld;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int q = nat_pos(s, Rout, tt, T, L);
        if (a.red_post && act && q < Lq && (q < a.out_off || q >= a.out_off + a.out_n)) {
            // energy cropped away by the store (zero-padded methods)
            const C x = cscale(v[s], (T_)a.out_scale);
            acc[1] += (double)x.x * x.x + (double)x.y * x.y;
        }
        if (act && q >= a.out_off && q < a.out_off + a.out_n) {
            const int i = q - a.out_off;
            if (a.mode == ROW_INV_ACC) {
                if (a.out_accum_int == 2) {
                    double* o = reinterpret_cast<double*>(a.out);
                    o[obase + i] = (a.acc_add ? o[obase + i] : 0.0) + (double)iacc[s];
                } else {
                    float* o = reinterpret_cast<float*>(a.out);
                    o[obase + i] = (a.acc_add ? o[obase + i] : 0.0f) + iacc[s];
                }
                continue;
            }
            C x = v[s];
            if (a.out_scale != 1.0) x = cscale(x, (T_)a.out_scale);
            if (a.post_shift) {
                const double arg = dmul(dmul(2.0, M_PI), dadd(dmul(a.fxc, gX(i, a.nx_grid, a.dx)), dmul(a.fyc, yrow)));
                x = cmul(x, cexpi<C>(arg));
            }
            if (a.red_post) acc[0] += (double)x.x * x.x + (double)x.y * x.y;
            if (a.out_accum_int == 1) {
                float* o = reinterpret_cast<float*>(a.out);
                o[obase + i] += (float)(a.weight * ((double)x.x * x.x + (double)x.y * x.y));
            } else if (a.out_accum_int == 2) {
                double* o = reinterpret_cast<double*>(a.out);
                o[obase + i] += a.weight * ((double)x.x * x.x + (double)x.y * x.y);
            } else {
                store_elem<C>(a.out, a.out_c128, obase + i, x);
            }
        }
    }
    if (a.red) {
        const long long blk = (long long)blockIdx.y * gridDim.x + blockIdx.x;
        if (a.red_moments) {
            block_sum_write<4>(acc, a.red + blk * RS_COUNT + RS_P);
        } else if (a.red_post) {
            double two[2] = {acc[0], acc[1]};  // kept, cropped
            block_sum_write<2>(two, a.red + blk * RS_COUNT + RS_P);
        } else {
            double one[1] = {acc[0]};
            block_sum_write<1>(one, a.red + blk * RS_COUNT + RS_P);
        }
    }
}

// ------------------------------------------------------------------ k_cols
template <typename Real, int E, bool MIX>
__global__ void __launch_bounds__(MaxT<Real, E>::v) k_cols(const ColArgs a) {
    using C = typename CT<Real>::t;
    using T_ = Real;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    __shared__ double hist[97];
    const int L = a.L;
    const int T = L / E;
    const int W = a.W;
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    const int col = blockIdx.x * W + w;
    const bool act = col < a.ncols;
    const int bz = blockIdx.y;
    const ColIdx ix{W};
    C* const alt = MIX ? sm + (size_t)col_tile_elems(L, W) : nullptr;  // launched with two buffers
    const LinePlan lp = make_line_plan(L, E);
    const C* tw = reinterpret_cast<const C*>(a.tw);
    const bool blue = a.blue_n > 0;
    const C* chirp = reinterpret_cast<const C*>(a.chirp);
    const C* bhf = blue ? reinterpret_cast<const C*>(a.bhat_f) : nullptr;
    const C* bhi = blue ? reinterpret_cast<const C*>(a.bhat_i) : nullptr;
    const int Lq = blue ? a.blue_n : L;
    const double wl = a.batch_wl ? a.batch_wl[bz] : a.h.wl;
    const double zz = a.batch_z ? a.batch_z[bz] : a.h.z;
    const bool inv_first = (a.mode == COL_FFT && a.col_inverse);

    if (a.red_hist) {
        for (int k = threadIdx.x; k < 97; k += blockDim.x) hist[k] = 0;
    }

    C v[E];
    const C* src = reinterpret_cast<const C*>(a.src) + (a.src_shared ? 0 : (long long)bz * a.src_bstride);
    // mixed lines: natural radix E; a loaded spectrum sits where the forward transform leaves it
    const bool spec = a.src_spectrum && !blue;
    const int R1 = MIX ? E : (spec ? out_radix(lp, false, false, E) : in_radix(lp, inv_first, blue, E));
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int p = nat_pos(s, R1, tt, T, L);
        C x = mkc<C>(0, 0);
        if (act && p >= a.in_off && p < a.in_off + a.in_n) {
            x = src[(long long)(p - a.in_off) * a.src_ld + col];
            if (blue) x = inv_first ? cmulc(x, ldg_c(chirp + p)) : cmul(x, ldg_c(chirp + p));
        }
        v[s] = x;
    }

    // first column transform
    if (!spec) xform<E, MIX>(v, sm, alt, ix, w, tt, T, lp, tw, inv_first, inv_first ? bhi : bhf);
    int Rm = MIX ? E : out_radix(lp, inv_first, blue, E);
    if (blue && (a.mode == COL_FRAUNHOFER || a.mode == COL_FFT)) {
        // the chirp of the Bluestein output has unit modulus: applied only
        // where the phase of the spectrum leaves the kernel
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = nat_pos(s, Rm, tt, T, L);
            if (q < Lq) v[s] = inv_first ? cmulc(v[s], ldg_c(chirp + q)) : cmul(v[s], ldg_c(chirp + q));
        }
    }

    if (a.mode == COL_FFT) {
        C* dst = reinterpret_cast<C*>(a.dst) + (long long)bz * a.dst_bstride;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = nat_pos(s, Rm, tt, T, L);
            if (act && q >= a.out_off && q < a.out_off + a.out_n)
                dst[(long long)(q - a.out_off) * a.dst_ld + col] = cscale(v[s], (T_)a.out_scale);
        }
        return;
    }

    if (a.mode == COL_FRAUNHOFER) {
        // propFraunhofer (propagate.go:603-662): dx^2, checkerboard, fftshift, quadratic phase
        const int n = a.fr_n;
        const int io = (col + n / 2) % n;
        const double xo = dmul(dsub((double)io, (double)n / 2), a.fr_dxout);
        C* dst = reinterpret_cast<C*>(a.dst) + (long long)bz * a.dst_bstride;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = nat_pos(s, Rm, tt, T, L);
            if (act && q < Lq) {
                C x = v[s];
                if ((q + col) & 1) x = mkc<C>(-x.x, -x.y);
                const int jo = (q + n / 2) % n;
                const double yo = dmul(dsub((double)jo, (double)n / 2), a.fr_dxout);
                const double arg = ddiv(dmul(a.h.k, dadd(dmul(xo, xo), dmul(yo, yo))), dmul(2.0, zz));
                const C fac = cmul(mkc<C>((T_)a.fr_c_re, (T_)a.fr_c_im), cexpi<C>(arg));
                dst[(long long)jo * a.dst_ld + io] = cmul(x, fac);
            }
        }
        return;
    }

    double acc[5] = {0, 0, 0, 0, 0};
    double spc[3] = {0, 0, 0};  // compensation of the centroid sums
    double drop = 0;
    const double hfx = (a.red_spec || a.red_hist) ? freq_n(col, a.hist_lx, a.hist_dx) : 0.0;
    const double fnyq = 1.0 / (2.0 * a.hist_dx);
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int q = nat_pos(s, Rm, tt, T, L);
        const C x = v[s];
        if (q >= Lq) {
            v[s] = mkc<C>(0, 0);
            continue;
        }
        if (act && (a.red_spec || a.red_hist)) {
            const double pw = (double)x.x * x.x + (double)x.y * x.y;
            const double fy = freq_n(q, a.hist_ly, a.hist_dx);
            if (a.red_spec) {
                neumaier_add(acc[0], spc[0], pw);
                neumaier_add(acc[1], spc[1], pw * hfx);
                neumaier_add(acc[2], spc[2], pw * fy);
            }
            if (a.red_hist && pw != 0) {
                int b = (int)(dmul(ddiv(go_hypot(hfx, fy), fnyq), 96.0));
                if (b > 96) b = 96;
                if (b < 0) b = 0;
                atomicAdd(&hist[b], pw);
            }
        }
        if (a.mode == COL_FUSED && a.h.kind != H_NONE) {
            if (a.red_bpm) {
                // power around each ASM half step, summed in the spectral
                // domain (Parseval) from FP64 |h|^2:  P0 = sum |x|^2,
                // loss of step 1 = sum |x|^2 (1-|h|^2), of step 2 (merged
                // split-step halves) = sum |x|^2 |h|^2 (1-|h|^2)
                HArgs h1 = a.h;
                h1.kind = H_ASM;
                h1.scale = 1.0;
                double m2;
                const C hh = eval_h<C>(h1, wl, zz, col, q, m2);
                const C y1 = cmul(x, hh);
                const C y2 = (a.h.kind == H_ASM_HALF2) ? cmul(y1, hh) : y1;
                if (act) {
                    const double p0 = (double)x.x * x.x + (double)x.y * x.y;
                    acc[0] += p0;
                    if (m2 != 1.0) {
                        acc[3] += p0 * (1.0 - m2);
                        acc[4] += p0 * m2 * (1.0 - m2);
                    }
                }
                v[s] = cscale(y2, (T_)a.h.scale);
            } else {
                double m2;
                v[s] = cmul(x, eval_h<C>(a.h, wl, zz, col, q, m2));
            }
        }
    }

    if (a.mode == COL_FUSED) {
        xform<E, MIX>(v, sm, alt, ix, w, tt, T, lp, tw, true, bhi);
        Rm = MIX ? E : out_radix(lp, true, blue, E);
        if (blue) {
#pragma unroll
            for (int s = 0; s < E; s++) {
                const int q = nat_pos(s, Rm, tt, T, L);
                if (q < Lq) v[s] = cmulc(v[s], ldg_c(chirp + q));
            }
        }
        C* dst = reinterpret_cast<C*>(a.dst) + (long long)bz * a.dst_bstride;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = nat_pos(s, Rm, tt, T, L);
            if (act && q >= a.out_off && q < a.out_off + a.out_n)
                dst[(long long)(q - a.out_off) * a.dst_ld + col] = v[s];
            else if (a.red_bpm && act && q < Lq)  // rows cropped away (zero-padded methods)
                drop += (double)v[s].x * v[s].x + (double)v[s].y * v[s].y;
        }
    }

    if (a.red) {
        const long long blk = (long long)blockIdx.y * gridDim.x + blockIdx.x;
        double* out = a.red + blk * RS_COUNT;
        if (a.red_spec) {
            double s3[3] = {acc[0], acc[1], acc[2]};
            block_sum2_write<3>(s3, spc, out + RS_SW, out + RS_SLO);
        }
        if (a.red_bpm) {
            double s4[4] = {acc[0], acc[3], acc[4], drop};
            block_sum_write<4>(s4, out + RS_SW);
        }
        if (a.red_hist) {
            __syncthreads();
            for (int k = threadIdx.x; k < 97; k += blockDim.x) out[RS_HIST + k] = hist[k];
        }
    }
}


// ------------------------------------------------------------------ lean mixed-radix sweeps
// The general sweeps carry every mode inline (Bluestein, screens, carrier
// ramps, reductions, Fraunhofer, every transfer function): 128 registers a
// thread and code that overflows the instruction cache, which on mixed-radix
// lines (2^a 3^b 5^c) left the batched ASM column sweep stalled on
// instruction fetch.  These two kernels do only what an ASM step on such
// lines needs.  k_rows_mix_lean: load (complex128 conversion, window
// in_off/in_n, carrier ramp on load), one transform, store (window, scale,
// carrier ramp on store) or, for ROW_INV_ACC, the weighted |E|^2 summed over
// the batch into an FP64 map.  k_cols_mix_asm: load the source columns (or
// their spectrum, SPEC), transform, H of asmTF with per-unit wavelength and
// distance (formed once per thread), inverse, store.

// exp(i arg), complex64 from the FP64 argument reduced to revolutions (small
// code, about one ulp); complex128 as the general sweeps (FP64 sincos).
template <typename C> __device__ __forceinline__ C cexpi_lean(double arg);
template <> __device__ __forceinline__ double2 cexpi_lean<double2>(double arg) { return cexpi<double2>(arg); }
template <> __device__ __forceinline__ float2 cexpi_lean<float2>(double arg) {
    const double t = arg * 0.15915494309189533577;  // revolutions
    const float f = (float)(t - rint(t));           // in [-1/2, 1/2]
    float sn, cs;
    sincospif(2.0f * f, &sn, &cs);
    return make_float2(cs, sn);
}

// asmTF, complex64: 1 - (wl fx)^2 - (wl fy)^2 in FP64 from the column's
// cx = 1 - (wl fx)^2, its square root from the single-precision seed plus one
// FP64 Newton step, and the phase k z sqrt(.) taken in revolutions (krev =
// k z / 2 pi, |krev| < 2^27) and reduced exactly before sin/cos in single
// precision; complex128 as asm_tf, in the reference's operation order.
template <typename C>
__device__ __forceinline__ C asm_tf_lean(const HArgs& h, double wl, double kz, double kaz, double krev, double cx,
                                         bool backward, double fx, double fy, double& m2) {
    if constexpr (sizeof(C) == 16) {
        return asm_tf<C>(h, wl, kz, kaz, backward, fx, fy, m2);
    } else {
        const double ay = wl * fy;
        const double s = fma(-ay, ay, cx);
        if (s >= 0) {
            m2 = 1.0;
            if (fabs(krev) < 0x1p27) return cexp_rev(krev * (s > 0x1p-100 ? fast_sqrt_bits(s) : 0.0), true);
            return cexpi_lean<C>(kz * sqrt(s));
        }
        return asm_tf<C>(h, wl, kz, kaz, backward, fx, fy, m2);
    }
}

// MODE: 0 forward, 1 inverse, 2 inverse with the weighted |E|^2 accumulated.
template <typename Real, int E, int MODE>
__global__ void __launch_bounds__(MaxT<Real, E>::v) k_rows_mix_lean(const RowArgs a) {
    constexpr bool INV = MODE != 0;
    using C = typename CT<Real>::t;
    using T_ = Real;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int L = a.L;
    const int T = L / E;
    const int lines = blockDim.x / T;
    const int line = threadIdx.x / T, tt = threadIdx.x - line * T;
    const int r = blockIdx.x * lines + line;
    const bool act = r < a.rows;
    const int bz = blockIdx.y;
    const int grow = a.row0 + r;
    const RowIdx ix{row_line_stride(L)};
    C* const alt = sm + (size_t)row_line_stride(L) * lines;
    const C* tw = reinterpret_cast<const C*>(a.tw);
    const double yrow = gX(grow, a.ny_grid, a.dx);
    constexpr bool acc_mode = MODE == 2;
    const int nb = acc_mode ? a.acc_nb : 1;
    C v[E];
    double iacc[acc_mode ? E : 1];
    for (int bb = 0; bb < nb; bb++) {
        const long long ibase = (long long)(acc_mode ? bb : bz) * a.in_bstride + (long long)r * a.in_ld;
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int p = tt + s * T;
            C x = mkc<C>(0, 0);
            if (act && p >= a.in_off && p < a.in_off + a.in_n) {
                const int i = p - a.in_off;
                x = load_elem<C>(a.in, a.in_c128, ibase + i);
                if (!INV && a.pre_shift) {
                    const double arg =
                        dmul(dmul(-2.0, M_PI), dadd(dmul(a.fxc, gX(i, a.nx_grid, a.dx)), dmul(a.fyc, yrow)));
                    x = cmul(x, cexpi_lean<C>(arg));
                }
            }
            v[s] = x;
        }
        mixed_line_fft<E, INV>(v, sm, alt, ix, line, tt, T, L, tw);
        if constexpr (acc_mode) {
            const double wgt = a.acc_weight ? a.acc_weight[bb] : 1.0;
#pragma unroll
            for (int s = 0; s < E; s++) {
                const C x = cscale(v[s], (T_)a.out_scale);
                const double pw = wgt * ((double)x.x * x.x + (double)x.y * x.y);
                iacc[s] = (bb == 0) ? pw : iacc[s] + pw;
            }
        }
    }
    const long long obase = (long long)bz * a.out_bstride + (long long)r * a.out_ld;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int q = tt + s * T;
        if (!act || q < a.out_off || q >= a.out_off + a.out_n) continue;
        const int i = q - a.out_off;
        if constexpr (acc_mode) {
            double* o = reinterpret_cast<double*>(a.out);
            o[obase + i] = (a.acc_add ? o[obase + i] : 0.0) + iacc[s];
            continue;
        }
        C x = v[s];
        if (a.out_scale != 1.0) x = cscale(x, (T_)a.out_scale);
        if (a.post_shift) {
            const double arg = dmul(dmul(2.0, M_PI), dadd(dmul(a.fxc, gX(i, a.nx_grid, a.dx)), dmul(a.fyc, yrow)));
            x = cmul(x, cexpi_lean<C>(arg));
        }
        store_elem<C>(a.out, a.out_c128, obase + i, x);
    }
}

template <typename Real, int E, bool SPEC>
__global__ void __launch_bounds__(MaxT<Real, E>::v) k_cols_mix_asm(const ColArgs a) {
    using C = typename CT<Real>::t;
    using T_ = Real;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int L = a.L;
    const int T = L / E;
    const int W = a.W;
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    const int col = blockIdx.x * W + w;
    const bool act = col < a.ncols;
    const int bz = blockIdx.y;
    const ColIdx ix{W};
    C* const alt = sm + (size_t)col_tile_elems(L, W);
    const C* tw = reinterpret_cast<const C*>(a.tw);
    C v[E];
    const C* src = reinterpret_cast<const C*>(a.src) + (a.src_shared ? 0 : (long long)bz * a.src_bstride);
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int p = tt + s * T;
        C x = mkc<C>(0, 0);
        if (act && p >= a.in_off && p < a.in_off + a.in_n) x = src[(long long)(p - a.in_off) * a.src_ld + col];
        v[s] = x;
    }
    if (!SPEC) mixed_line_fft<E, false>(v, sm, alt, ix, w, tt, T, L, tw);

    // asmTF (optics/propagate.go:159-181) with this unit's wavelength and distance
    const HArgs& h = a.h;
    const double wl = a.batch_wl ? a.batch_wl[bz] : h.wl;
    const double z = a.batch_z ? a.batch_z[bz] : h.z;
    const double k = (wl == h.wl) ? h.k : 2 * M_PI / wl;
    const double kz = (wl == h.wl && z == h.z) ? h.kz : k * z;
    const double kaz = (wl == h.wl && z == h.z) ? h.kaz : k * fabs(z);
    const double fx = h.fxoff != 0 ? dadd(freq_n(col, h.lfx, h.dx), h.fxoff) : freq_n(col, h.lfx, h.dx);
    const double cx = fma(-(wl * fx), wl * fx, 1.0);
    const double krev = kz * 0.15915494309189533577;
    const double fyu = 1.0 / ((double)h.lfy * h.dx);  // complex64: fy by one multiply
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int q = tt + s * T;
        double fy;
        if constexpr (sizeof(C) == 16) fy = freq_n(q, h.lfy, h.dx);
        else fy = (double)(q <= h.lfy / 2 ? q : q - h.lfy) * fyu;
        if (h.fyoff != 0) fy = dadd(fy, h.fyoff);
        double m2;
        C hh = asm_tf_lean<C>(h, wl, kz, kaz, krev, cx, z < 0, fx, fy, m2);
        if (h.conj) hh.y = -hh.y;
        v[s] = cscale(cmul(v[s], hh), (T_)h.scale);
    }
    mixed_line_fft<E, true>(v, sm, alt, ix, w, tt, T, L, tw);
    C* dst = reinterpret_cast<C*>(a.dst) + (long long)bz * a.dst_bstride;
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int q = tt + s * T;
        if (act && q >= a.out_off && q < a.out_off + a.out_n) dst[(long long)(q - a.out_off) * a.dst_ld + col] = v[s];
    }
}

// The spectral-centroid sums of mixed-radix columns (COL_REDUCE without the
// histogram): forward transform, then |F|^2, |F|^2 fx and |F|^2 fy added with
// compensation, as the general sweep adds them.
template <typename Real, int E>
__global__ void __launch_bounds__(MaxT<Real, E>::v) k_cols_mix_reduce(const ColArgs a) {
    using C = typename CT<Real>::t;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    const int L = a.L;
    const int T = L / E;
    const int W = a.W;
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    const int col = blockIdx.x * W + w;
    const bool act = col < a.ncols;
    const int bz = blockIdx.y;
    const ColIdx ix{W};
    C* const alt = sm + (size_t)col_tile_elems(L, W);
    const C* tw = reinterpret_cast<const C*>(a.tw);
    C v[E];
    const C* src = reinterpret_cast<const C*>(a.src) + (a.src_shared ? 0 : (long long)bz * a.src_bstride);
#pragma unroll
    for (int s = 0; s < E; s++) {
        const int p = tt + s * T;
        C x = mkc<C>(0, 0);
        if (act && p >= a.in_off && p < a.in_off + a.in_n) x = src[(long long)(p - a.in_off) * a.src_ld + col];
        v[s] = x;
    }
    mixed_line_fft<E, false>(v, sm, alt, ix, w, tt, T, L, tw);
    double acc[3] = {0, 0, 0}, spc[3] = {0, 0, 0};
    if (act) {
        const double hfx = freq_n(col, a.hist_lx, a.hist_dx);
#pragma unroll
        for (int s = 0; s < E; s++) {
            const int q = tt + s * T;
            const double pw = (double)v[s].x * v[s].x + (double)v[s].y * v[s].y;
            const double fy = freq_n(q, a.hist_ly, a.hist_dx);
            neumaier_add(acc[0], spc[0], pw);
            neumaier_add(acc[1], spc[1], pw * hfx);
            neumaier_add(acc[2], spc[2], pw * fy);
        }
    }
    double* out = a.red + ((long long)blockIdx.y * gridDim.x + blockIdx.x) * RS_COUNT;
    block_sum2_write<3>(acc, spc, out + RS_SW, out + RS_SLO);
}

// Whether a general launch can take the lean kernels above (mixed lines only).
__host__ inline bool rows_mix_lean_ok(const RowArgs& a) {
    if (a.blue_n || a.red || a.pre_phi || a.pre_phi_f || a.scr.kind) return false;
    if (a.mode == ROW_INV_ACC) return a.out_accum_int == 2;
    return (a.mode == ROW_FWD || a.mode == ROW_INV) && a.out_accum_int == 0 && (a.mode == ROW_FWD || !a.pre_shift) &&
           (a.mode == ROW_INV || !a.post_shift);
}
__host__ inline bool cols_mix_reduce_ok(const ColArgs& a) {
    return a.mode == COL_REDUCE && a.red && a.red_spec && !a.red_hist && !a.red_bpm && !a.blue_n;
}
__host__ inline bool cols_mix_lean_ok(const ColArgs& a) {
    return a.mode == COL_FUSED && a.h.kind == H_ASM && !a.blue_n && !a.red && !a.red_spec && !a.red_hist &&
           !a.red_bpm;
}

// Launchers of the mixed-radix instantiations (wos_kernels_mix*.cu).
template <typename Real, int E>
cudaError_t launch_rows_mix(const RowArgs& a, dim3 grid, int threads, size_t smem, cudaStream_t st);
template <typename Real, int E>
cudaError_t launch_cols_mix(const ColArgs& a, dim3 grid, int threads, size_t smem, cudaStream_t st);

// Definitions, included by the translation units that instantiate them.
#ifdef WOS_DEFINE_MIX_LAUNCHERS
template <typename K>
cudaError_t launch_mix_kernel(K kern, dim3 grid, int threads, size_t smem, cudaStream_t st, const void* args) {
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    void* argv[] = {const_cast<void*>(args)};
    return cudaLaunchKernel(reinterpret_cast<const void*>(kern), grid, dim3(threads), argv, smem, st);
}

template <typename Real, int E>
cudaError_t launch_rows_mix(const RowArgs& a, dim3 grid, int threads, size_t smem, cudaStream_t st) {
    if (rows_mix_lean_ok(a)) {
        if (a.mode == ROW_FWD) return launch_mix_kernel(k_rows_mix_lean<Real, E, 0>, grid, threads, smem, st, &a);
        if (a.mode == ROW_INV) return launch_mix_kernel(k_rows_mix_lean<Real, E, 1>, grid, threads, smem, st, &a);
        return launch_mix_kernel(k_rows_mix_lean<Real, E, 2>, grid, threads, smem, st, &a);
    }
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows<Real, E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_rows<Real, E, true><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

template <typename Real, int E>
cudaError_t launch_cols_mix(const ColArgs& a, dim3 grid, int threads, size_t smem, cudaStream_t st) {
    if (cols_mix_lean_ok(a)) {
        if (a.src_spectrum) return launch_mix_kernel(k_cols_mix_asm<Real, E, true>, grid, threads, smem, st, &a);
        return launch_mix_kernel(k_cols_mix_asm<Real, E, false>, grid, threads, smem, st, &a);
    }
    if (cols_mix_reduce_ok(a)) return launch_mix_kernel(k_cols_mix_reduce<Real, E>, grid, threads, smem, st, &a);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_cols<Real, E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_cols<Real, E, true><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

#define WOS_MIX_INST(R, E)                                                                       \
    template cudaError_t launch_rows_mix<R, E>(const RowArgs&, dim3, int, size_t, cudaStream_t); \
    template cudaError_t launch_cols_mix<R, E>(const ColArgs&, dim3, int, size_t, cudaStream_t);
#endif

}  // namespace wos

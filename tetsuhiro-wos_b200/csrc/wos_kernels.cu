// wos_kernels.cu -- sm_100a propagation kernels.
//
// Two sweep kernels carry every method:
//   k_rows : one CTA owns whole rows (line-contiguous shared layout).  Loads a
//            row with coalesced accesses, applies load-side pointwise work
//            (zero padding, carrier ramp, phase mask, Bluestein chirp), runs the
//            line FFT in registers/shared memory and stores with store-side work
//            (crop, carrier ramp, type conversion, intensity accumulation,
//            power reductions).  ROW_INV_FWD runs inverse . screen . forward on
//            the same row (one sweep per split-step slice).
//   k_cols : one CTA owns W adjacent columns (interleaved layout, 64 B row
//            segments).  Forward column FFT, the transfer function generated on
//            the fly (FP64 argument), inverse column FFT, all on chip: the
//            band-limited ASM costs three HBM sweeps in total.
// Reference path replaced: optics/gpu.go:173-207 (per-FFT cuFFT Z2Z with host
// scaling) and the host loops of optics/propagate.go:132-148,339-387,426-504.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <stdint.h>

#include <algorithm>

#include "wos_kernels_dev.cuh"

namespace wos {

// ------------------------------------------------------------------ tables
template <typename C>
__global__ void k_twiddles(C* tw, int L) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    double s, c;
    sincospi(-2.0 * (double)i / (double)L, &s, &c);
    tw[i] = mkc<C>((decltype(C::x))c, (decltype(C::x))s);
}

// Bluestein chirp exp(-i pi k^2 / n), with k^2 reduced mod 2n in integers
// before any floating-point operation, and the two convolution kernels
// b0 (forward: conj chirp; inverse: chirp), mirrored, zero in the middle
// (optics/fft.go:173-187).
template <typename C>
__global__ void k_chirp(C* chirp, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const long long kk = ((long long)k * k) % (2LL * n);
    double s, c;
    sincospi(-(double)kk / (double)n, &s, &c);
    chirp[k] = mkc<C>((decltype(C::x))c, (decltype(C::x))s);
}
__global__ void k_b0_fill(double2* b0f, double2* b0i, int n, int M) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    double2 f = make_double2(0, 0), iv = make_double2(0, 0);
    int kk = -1;
    if (k < n) kk = k;
    else if (M - k < n) kk = M - k;
    if (kk >= 0) {
        const long long q = ((long long)kk * kk) % (2LL * n);
        double s, c;
        sincospi(-(double)q / (double)n, &s, &c);
        f = make_double2(c, -s);   // conj(chirp)
        iv = make_double2(c, s);   // chirp
    }
    b0f[k] = f;
    b0i[k] = iv;
}

template <typename C>
__global__ void k_bhat_finish(C* df, C* di, const double2* bf, const double2* bi, int M) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const double inv = 1.0 / (double)M;
    df[k] = mkc<C>((decltype(C::x))(bf[k].x * inv), (decltype(C::x))(bf[k].y * inv));
    di[k] = mkc<C>((decltype(C::x))(bi[k].x * inv), (decltype(C::x))(bi[k].y * inv));
}

// Neumaier-compensated sum of the per-CTA partials of slots [s0, s0+ns) for
// batch group blockIdx.x (nblocks partials each), one thread per slot, blocks
// summed in a fixed order (deterministic).
// Compensated sum of slot s0 + blockIdx.y over the nblocks per-CTA records of
// batch blockIdx.x.  Each thread keeps a Neumaier pair (sum, compensation)
// over a fixed stride of records; the pairs are combined in a fixed tree, so
// the result is deterministic and carries the compensation of every term.
__global__ void __launch_bounds__(256) k_reduce_finish(const double* partials, int nblocks, int s0, double* out) {
    const int k = blockIdx.y;
    const double* p = partials + (long long)blockIdx.x * nblocks * RS_COUNT + s0 + k;
    double s = 0, c = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) neumaier_add(s, c, p[(long long)b * RS_COUNT]);
    for (int o = 16; o > 0; o >>= 1) {
        const double s2 = __shfl_down_sync(0xffffffffu, s, o);
        const double c2 = __shfl_down_sync(0xffffffffu, c, o);
        c += c2;
        neumaier_add(s, c, s2);
    }
    __shared__ double ws[8][2];
    if ((threadIdx.x & 31) == 0) {
        ws[threadIdx.x >> 5][0] = s;
        ws[threadIdx.x >> 5][1] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0, tc = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            tc += ws[w][1];
            neumaier_add(ts, tc, ws[w][0]);
        }
        out[(long long)blockIdx.x * RS_COUNT + s0 + k] = ts + tc;
    }
}

// Vector angular spectrum (PropagateVectorial, optics/vectorial.go:14-80) on
// the 2-D spectra of Ex and Ey: Ez = -(kx Ex + ky Ey) / kz (kz = i kzi for
// evanescent bins), then all three times H; rho = wl hypot(fx, fy) and the
// phase (k sqrt(1 - rho^2)) z in the reference's operation order.
template <typename C>
__global__ void k_vectorial(C* ex, C* ey, C* ez, int ny, int nx, double dx, HArgs h) {
    using T = decltype(C::x);
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)ny * nx) return;
    const int j = (int)(idx / nx), i = (int)(idx - (long long)j * nx);
    const double fx = freq_n(i, nx, dx), fy = freq_n(j, ny, dx);
    const double kx = dmul(2 * M_PI, fx), ky = dmul(2 * M_PI, fy);
    const double rho = dmul(h.wl, go_hypot(fx, fy));
    const C x = ex[idx], y = ey[idx];
    const double sr = -dadd(dmul(kx, (double)x.x), dmul(ky, (double)y.x));
    const double si = -dadd(dmul(kx, (double)x.y), dmul(ky, (double)y.y));
    C H = mkc<C>(0, 0), zz = mkc<C>(0, 0);
    if (rho <= 1.0) {
        const double kz = dmul(h.k, __dsqrt_rn(dmul(dsub(1.0, rho), dadd(1.0, rho))));
        H = cexpi<C>(dmul(kz, h.z));
        if (kz > 0) zz = mkc<C>((T)ddiv(sr, kz), (T)ddiv(si, kz));
    } else {
        const double sq = __dsqrt_rn(dmul(dsub(rho, 1.0), dadd(rho, 1.0)));
        const double decay = dmul(h.kaz, sq);
        double a;
        if (h.zero_ev || (h.limit > 0 && decay > h.limit)) a = 0;
        else if (h.z < 0 && h.reg) {
            const double e = exp(decay);
            a = ddiv(e, dadd(1.0, dmul(dmul(dmul(h.alpha, h.alpha), e), e)));
        } else if (h.z < 0) {
            a = exp(decay);
        } else {
            a = exp(-decay);
        }
        H = mkc<C>((T)a, 0);
        const double kzi = dmul(h.k, sq);
        if (kzi > 0) zz = mkc<C>((T)ddiv(si, kzi), (T)(-ddiv(sr, kzi)));
    }
    ex[idx] = cmul(x, H);
    ey[idx] = cmul(y, H);
    ez[idx] = cmul(zz, H);
}

// 1-D angular spectrum step (asmTF1D, optics/propagate.go:680-701): rho =
// |wl fx| is asm_tf's hypot with fy = 0.  Spectral power sums for the
// evanescent_filtered warning, as in the 2-D column pass.
template <typename C>
__global__ void __launch_bounds__(256) k_asm1d_h(C* a, int n, HArgs h, double* partials) {
    using T = decltype(C::x);
    double p0 = 0, l1 = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double m2;
        const C hh = asm_tf<C>(h, h.wl, h.kz, h.kaz, h.z < 0, freq_n(i, h.lfx, h.dx), 0.0, m2);
        const C x = a[i];
        const double pw = (double)x.x * x.x + (double)x.y * x.y;
        p0 += pw;
        if (m2 != 1.0) l1 += pw * (1.0 - m2);
        a[i] = cmul(x, cscale(hh, (T)h.scale));
    }
    __shared__ double sm[2][8];
    for (int o = 16; o > 0; o >>= 1) {
        p0 += __shfl_down_sync(0xffffffffu, p0, o);
        l1 += __shfl_down_sync(0xffffffffu, l1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sm[0][threadIdx.x >> 5] = p0;
        sm[1][threadIdx.x >> 5] = l1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double u = 0, v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            u += sm[0][w];
            v += sm[1][w];
        }
        partials[(long long)blockIdx.x * RS_COUNT + RS_SW] = u;
        partials[(long long)blockIdx.x * RS_COUNT + RS_SW + 1] = v;
    }
}

__global__ void k_convert(int to_c128, const void* src, void* dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (to_c128) {
            float2 a = reinterpret_cast<const float2*>(src)[i];
            reinterpret_cast<double2*>(dst)[i] = make_double2(a.x, a.y);
        } else {
            double2 a = reinterpret_cast<const double2*>(src)[i];
            reinterpret_cast<float2*>(dst)[i] = make_float2((float)a.x, (float)a.y);
        }
    }
}

// One axis of the Fresnel impulse response in wrap layout:
// h[p] = cexpI(pi * x^2 / (wl z)), x = (p or p-m) * dx   (propagate.go:543-558)
__global__ void k_fresnel_ir_axis(double2* h, int m, double dx, double wl, double z) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m) return;
    double d = (double)p;
    if (p > m / 2) d -= (double)m;
    const double x = dmul(d, dx);
    double s, c;
    sincos(ddiv(dmul(M_PI, dmul(x, x)), dmul(wl, z)), &s, &c);
    h[p] = make_double2(c, s);
}

template <typename C>
__global__ void k_scale_copy(const double2* src, C* dst, long long n, double sre, double sim) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 a = src[i];
    dst[i] = mkc<C>((decltype(C::x))(a.x * sre - a.y * sim), (decltype(C::x))(a.x * sim + a.y * sre));
}

// ------------------------------------------------------------------ launchers
// Elements per thread: 16 (FP32 power-of-two lines) / 8 (FP32 mixed-radix
// lines; FP64, 16 for lines of 8192), never more than L; WOS_MIXE (4, 8 or 16)
// sets the start for mixed-radix lines.  (Complex64 mixed lines at 8 rather
// than 16: 128 planes of 768^2 1.90 -> 1.78 ms, cfg2 0.527 -> 0.510 ms.)
static int mix_e_override() {
    static const int v = [] {
        const char* e = getenv("WOS_MIXE");
        const int x = e ? atoi(e) : 0;
        return (x == 4 || x == 8 || x == 16) ? x : 0;
    }();
    return v;
}
int pick_E(int fp64, int L) {
    const bool mixed = (L & (L - 1)) != 0;
    int e = fp64 ? (L >= 8192 ? 16 : 8) : (mixed ? 8 : 16);
    if (mixed && mix_e_override()) e = mix_e_override();
    while (e > L) e >>= 1;
    while (e > 2 && L % e != 0) e >>= 1;  // a mixed-radix line: E divides L
    // a long line whose threads would not fit one CTA takes more values per thread
    while (e < 16 && L / e > max_threads_for(fp64, e) && L % (2 * e) == 0) e <<= 1;
    return e;
}
int max_threads_for(int fp64, int E) { return (E >= 16 || fp64) ? 512 : 1024; }
int row_threads_per_line(int L, int E) { return L / E; }
size_t row_smem_bytes(int fp64, int L, int E, int lines) {
    (void)E;
    return (size_t)row_line_stride(L) * lines * (fp64 ? 16 : 8);
}
size_t col_smem_bytes(int fp64, int L, int W) { return (size_t)col_tile_elems(L, W) * (fp64 ? 16 : 8); }

template <typename Real, int E>
static cudaError_t launch_rows_t(const RowArgs& a, cudaStream_t st) {
    const int T = a.L / E;
    const int maxt = MaxT<Real, E>::v;
    if (T > maxt) return cudaErrorInvalidConfiguration;
    int lines = 1;
    while (lines * 2 * T <= 256 && lines * 2 <= a.rows) lines *= 2;
    while (lines * T < 32) lines *= 2;  // whole warps (idle lines are inactive)
    const size_t smem = (size_t)row_line_stride(a.L) * lines * sizeof(typename CT<Real>::t);
    const int nbat = (a.mode == ROW_INV_ACC) ? 1 : (a.batch > 0 ? a.batch : 1);
    dim3 grid((a.rows + lines - 1) / lines, nbat);
    // mixed-radix lines alternate between two shared-memory buffers
    if ((a.L & (a.L - 1)) != 0) return launch_rows_mix<Real, E>(a, grid, lines * T, 2 * smem, st);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_rows<Real, E, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_rows<Real, E, false><<<grid, lines * T, smem, st>>>(a);
    return cudaGetLastError();
}

template <typename Real, int E>
static cudaError_t launch_cols_t(const ColArgs& a, cudaStream_t st) {
    const int T = a.L / E;
    const int maxt = MaxT<Real, E>::v;
    ColArgs b = a;
    while (b.W * T < 32) b.W *= 2;  // whole warps (idle columns are inactive)
    while (b.W > 1 && b.W * T > maxt) b.W /= 2;
    if (b.W * T > maxt) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)col_tile_elems(b.L, b.W) * sizeof(typename CT<Real>::t);
    dim3 grid((b.ncols + b.W - 1) / b.W, b.batch > 0 ? b.batch : 1);
    if ((b.L & (b.L - 1)) != 0) return launch_cols_mix<Real, E>(b, grid, b.W * T, 2 * smem, st);
    if (smem > kSmemNoOptIn) {
        cudaError_t e = cudaFuncSetAttribute(k_cols<Real, E, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_cols<Real, E, false><<<grid, b.W * T, smem, st>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_rows(int fp64, const RowArgs& a, cudaStream_t st) {
    const int E = pick_E(fp64, a.L);
    if (fp64) {
        switch (E) {
        case 2: return launch_rows_t<double, 2>(a, st);
        case 4: return launch_rows_t<double, 4>(a, st);
        case 8: return launch_rows_t<double, 8>(a, st);
        default: return launch_rows_t<double, 16>(a, st);
        }
    }
    switch (E) {
    case 2: return launch_rows_t<float, 2>(a, st);
    case 4: return launch_rows_t<float, 4>(a, st);
    case 8: return launch_rows_t<float, 8>(a, st);
    default: return launch_rows_t<float, 16>(a, st);
    }
}

cudaError_t launch_cols(int fp64, const ColArgs& a, cudaStream_t st) {
    const int E = pick_E(fp64, a.L);
    if (fp64) {
        switch (E) {
        case 2: return launch_cols_t<double, 2>(a, st);
        case 4: return launch_cols_t<double, 4>(a, st);
        case 8: return launch_cols_t<double, 8>(a, st);
        default: return launch_cols_t<double, 16>(a, st);
        }
    }
    switch (E) {
    case 2: return launch_cols_t<float, 2>(a, st);
    case 4: return launch_cols_t<float, 4>(a, st);
    case 8: return launch_cols_t<float, 8>(a, st);
    default: return launch_cols_t<float, 16>(a, st);
    }
}

cudaError_t launch_vectorial(int fp64, void* planes, int ny, int nx, double dx, const HArgs& h, cudaStream_t st) {
    const long long np = (long long)ny * nx;
    const unsigned g = (unsigned)((np + 255) / 256);
    if (fp64) {
        double2* p = reinterpret_cast<double2*>(planes);
        k_vectorial<double2><<<g, 256, 0, st>>>(p, p + np, p + 2 * np, ny, nx, dx, h);
    } else {
        float2* p = reinterpret_cast<float2*>(planes);
        k_vectorial<float2><<<g, 256, 0, st>>>(p, p + np, p + 2 * np, ny, nx, dx, h);
    }
    return cudaGetLastError();
}

cudaError_t launch_asm1d_h(int fp64, void* a, int n, const HArgs& h, double* partials, int* nblocks,
                           cudaStream_t st) {
    const int g = std::min((n + 255) / 256, 64);
    *nblocks = g;
    if (fp64) k_asm1d_h<double2><<<g, 256, 0, st>>>(reinterpret_cast<double2*>(a), n, h, partials);
    else k_asm1d_h<float2><<<g, 256, 0, st>>>(reinterpret_cast<float2*>(a), n, h, partials);
    return cudaGetLastError();
}

// Per-pass twiddle tables of a mixed-radix line (see mixed_table_len):
// W_{NS R}^{r k} generated in FP64, entry [off_p + (r-1) NS + k].
template <typename C>
__global__ void k_mixed_twiddles(C* out, int L, int total) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int rem = L, NS = 1, off = 0;
    while (rem > 1) {
        const int R = mixed_radix_of(rem);
        const int n = NS * (R - 1);
        if (idx < off + n) {
            const int t = idx - off, r = t / NS + 1, k = t % NS;
            double s, c;
            sincospi(-2.0 * (double)r * (double)k / ((double)NS * (double)R), &s, &c);
            out[idx] = mkc<C>((decltype(C::x))c, (decltype(C::x))s);
            return;
        }
        off += n;
        NS *= R;
        rem /= R;
    }
}
cudaError_t launch_mixed_twiddles(int fp64, void* out, int L, cudaStream_t st) {
    const int total = mixed_table_len(L);
    const int b = 256, g = (total + b - 1) / b;
    if (total == 0) return cudaSuccess;
    if (fp64) k_mixed_twiddles<double2><<<g, b, 0, st>>>(reinterpret_cast<double2*>(out), L, total);
    else k_mixed_twiddles<float2><<<g, b, 0, st>>>(reinterpret_cast<float2*>(out), L, total);
    return cudaGetLastError();
}

cudaError_t launch_twiddles(int fp64, void* tw, int L, cudaStream_t st) {
    const int b = 256, g = (L + b - 1) / b;
    if (fp64) k_twiddles<double2><<<g, b, 0, st>>>(reinterpret_cast<double2*>(tw), L);
    else k_twiddles<float2><<<g, b, 0, st>>>(reinterpret_cast<float2*>(tw), L);
    return cudaGetLastError();
}

cudaError_t launch_chirp_b0(int fp64, void* chirp, double2* b0f, double2* b0i, int n, int M,
                            cudaStream_t st) {
    const int b = 256;
    if (fp64) k_chirp<double2><<<(n + b - 1) / b, b, 0, st>>>(reinterpret_cast<double2*>(chirp), n);
    else k_chirp<float2><<<(n + b - 1) / b, b, 0, st>>>(reinterpret_cast<float2*>(chirp), n);
    k_b0_fill<<<(M + b - 1) / b, b, 0, st>>>(b0f, b0i, n, M);
    return cudaGetLastError();
}

cudaError_t launch_bhat_finish(int fp64, void* df, void* di, const double2* bf, const double2* bi, int M,
                               cudaStream_t st) {
    const int b = 256, g = (M + b - 1) / b;
    if (fp64) k_bhat_finish<double2><<<g, b, 0, st>>>(reinterpret_cast<double2*>(df), reinterpret_cast<double2*>(di), bf, bi, M);
    else k_bhat_finish<float2><<<g, b, 0, st>>>(reinterpret_cast<float2*>(df), reinterpret_cast<float2*>(di), bf, bi, M);
    return cudaGetLastError();
}

cudaError_t launch_reduce_finish(const double* partials, int nblocks, int nbatch, int s0, int ns,
                                 double* out, cudaStream_t st) {
    if (ns <= 0 || nbatch <= 0) return cudaSuccess;
    k_reduce_finish<<<dim3(nbatch, ns), 256, 0, st>>>(partials, nblocks, s0, out);
    return cudaGetLastError();
}

cudaError_t launch_convert(int to_c128, const void* src, void* dst, long long n, cudaStream_t st) {
    k_convert<<<148 * 8, 256, 0, st>>>(to_c128, src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_fresnel_ir_axis(double2* h, int m, double dx, double wl, double z, cudaStream_t st) {
    k_fresnel_ir_axis<<<(m + 255) / 256, 256, 0, st>>>(h, m, dx, wl, z);
    return cudaGetLastError();
}

cudaError_t launch_scale_copy(int fp64, const double2* src, void* dst, long long n, double sre, double sim,
                              cudaStream_t st) {
    const int b = 256;
    const long long g = (n + b - 1) / b;
    if (fp64) k_scale_copy<double2><<<(unsigned)g, b, 0, st>>>(src, reinterpret_cast<double2*>(dst), n, sre, sim);
    else k_scale_copy<float2><<<(unsigned)g, b, 0, st>>>(src, reinterpret_cast<float2*>(dst), n, sre, sim);
    return cudaGetLastError();
}

}  // namespace wos

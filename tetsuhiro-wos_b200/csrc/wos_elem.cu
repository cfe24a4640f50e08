// wos_elem.cu -- pointwise kernels: thin-element transmissions, Gaussian
// Schell-model mode synthesis, intensity accumulation and the inverse-design
// residual / gradient.  All element arithmetic is FP64 on complex128 fields,
// formed in the reference's operation order (no FMA contraction) so that the
// FP64 path reproduces optics/elements.go and optics/coherence.go.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "wos_fft.cuh"
#include "wos_kernels.cuh"

namespace wos {

namespace {
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }
// Go complex128 product (ac - bd, ad + bc) without contraction
__device__ __forceinline__ double2 gmul(double2 a, double2 b) {
    return make_double2(ds(dm(a.x, b.x), dm(a.y, b.y)), da(dm(a.x, b.y), dm(a.y, b.x)));
}
__device__ __forceinline__ double2 gexpi(double phi) {
    double s, c;
    sincos(phi, &s, &c);
    return make_double2(c, s);
}
__device__ __forceinline__ double coord(int i, int n, double dx) { return dm(ds((double)i, (double)n / 2), dx); }
__device__ __forceinline__ double ghypot(double p, double q) {
    p = fabs(p);
    q = fabs(q);
    if (p < q) { double t = p; p = q; q = t; }
    if (p == 0) return 0;
    q = dd(q, p);
    return dm(p, __dsqrt_rn(da(1.0, dm(q, q))));
}
__device__ __forceinline__ void apply2(double2* ex, double2* ey, int pol, long long idx, double2 t) {
    ex[idx] = gmul(ex[idx], t);
    if (pol) ey[idx] = gmul(ey[idx], t);
}
}  // namespace

// lensEl.Apply (optics/elements.go:195-221); c = -k/(2f) formed by the caller
__global__ void k_lens(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double c, double ap,
                       double x0, double y0) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)ny * nx) return;
    const int j = (int)(idx / nx), i = (int)(idx % nx);
    const double dy = ds(coord(j, ny, dx), y0);
    const double dxx = ds(coord(i, nx, dx), x0);
    const double r2 = da(dm(dxx, dxx), dm(dy, dy));
    if (ap > 0 && r2 > dm(ap, ap)) {
        ex[idx] = make_double2(0, 0);
        if (pol) ey[idx] = make_double2(0, 0);
        return;
    }
    apply2(ex, ey, pol, idx, gexpi(dm(c, r2)));
}

// apertureEl.Apply with the circle outline (elements.go:288-313, shape.go:163-169)
__global__ void k_aperture_circle(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double radius,
                                  double x0, double y0, double sig) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)ny * nx) return;
    const int j = (int)(idx / nx), i = (int)(idx % nx);
    const double dy = ds(coord(j, ny, dx), y0);
    const double dxx = ds(coord(i, nx, dx), x0);
    const double d = ds(radius, ghypot(dxx, dy));
    double t;
    if (sig > 0) t = dm(0.5, da(1.0, erf(dd(d, dm(M_SQRT2, sig)))));
    else t = d >= 0 ? 1.0 : 0.0;
    apply2(ex, ey, pol, idx, make_double2(t, 0));
}

// gratingEl.Apply (elements.go:488-532)
__global__ void k_grating(double2* ex, double2* ey, int pol, int ny, int nx, double dx, int kind, double period,
                          double modulation, double duty, double blaze, double rotation, double off) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)ny * nx) return;
    const int j = (int)(idx / nx), i = (int)(idx % nx);
    const double c = cos(rotation), s = sin(rotation);
    const double uu = da(dm(c, coord(i, nx, dx)), dm(s, coord(j, ny, dx)));
    const double ph = dd(dm(2 * M_PI, uu), period);
    double2 t = make_double2(0, 0);
    switch (kind) {
    case 0: t = make_double2(dm(0.5, da(1.0, dm(modulation, cos(da(ph, off))))), 0); break;
    case 1: if (cos(da(ph, off)) >= cos(dm(M_PI, duty))) t = make_double2(1, 0); break;
    case 2: t = gexpi(dm(dd(modulation, 2.0), sin(da(ph, off)))); break;
    case 3: t = (cos(da(ph, off)) >= 0) ? gexpi(modulation) : make_double2(1, 0); break;
    default: {
        double fr = fmod(dd(uu, period), 1.0);
        if (fr < 0) fr = da(fr, 1.0);
        t = gexpi(dm(blaze, fr));
    } break;
    }
    apply2(ex, ey, pol, idx, t);
}

// applyMask with t = amp * exp(i phi) (elements.go:128-141)
__global__ void k_phase_mask(double2* ex, double2* ey, int pol, long long n, const double* phi, double amp) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    apply2(ex, ey, pol, idx, gmul(make_double2(amp, 0), gexpi(phi[idx])));
}

// ---- Field operations (optics/field.go:109-168)
// ApplyJones: mode 0 scalar field, diagonal matrix a*I (Ex *= a); mode 1
// scalar -> polarized transition (Ex = a Ex, Ey = c Ex); mode 2 full 2x2.
__global__ void k_jones(double2* ex, double2* ey, long long n, int mode, double2 a, double2 b, double2 c,
                        double2 d) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double2 x = ex[idx];
    if (mode == 0) {
        ex[idx] = gmul(x, a);
    } else if (mode == 1) {
        ex[idx] = gmul(a, x);
        ey[idx] = gmul(c, x);
    } else {
        const double2 y = ey[idx];
        const double2 p = gmul(a, x), q = gmul(b, y), r = gmul(c, x), t = gmul(d, y);
        ex[idx] = make_double2(da(p.x, q.x), da(p.y, q.y));
        ey[idx] = make_double2(da(r.x, t.x), da(r.y, t.y));
    }
}

// ScaleAmplitude
__global__ void k_scale(double2* ex, double2* ey, int pol, long long n, double2 s) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    apply2(ex, ey, pol, idx, s);
}

// ApplyTilt: the phase along a row is accumulated sequentially from its
// first pixel (ph += k sx dx), so every pixel carries exactly the rounding of
// the reference's running sum.  One CTA per row: thread 0 runs the sum for a
// chunk of pixels into shared memory, then all threads apply exp(i ph).
constexpr int kTiltChunk = 1024;
__global__ void k_tilt(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double k, double sx,
                       double sy) {
    __shared__ double ph_s[kTiltChunk];
    __shared__ double carry;
    const int j = blockIdx.x;
    const double step = dm(dm(k, sx), dx);
    if (threadIdx.x == 0) carry = dm(k, da(dm(sx, coord(0, nx, dx)), dm(sy, coord(j, ny, dx))));
    for (int i0 = 0; i0 < nx; i0 += kTiltChunk) {
        const int m = min(kTiltChunk, nx - i0);
        __syncthreads();  // the previous chunk has been applied
        if (threadIdx.x == 0) {
            double ph = carry;
            for (int i = 0; i < m; i++) {
                ph_s[i] = ph;
                ph = da(ph, step);
            }
            carry = ph;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const long long idx = (long long)j * nx + i0 + i;
            const double2 t = gexpi(ph_s[i]);
            ex[idx] = gmul(ex[idx], t);
            if (pol) ey[idx] = gmul(ey[idx], t);
        }
    }
}

// ---- Diffuser (optics/elements.go:710-783)
// hashNoise01: splitmix-style finaliser of the lab cell and the seed.
__device__ __forceinline__ double hash_noise01(long long x, long long y, long long seed) {
    unsigned long long h = (unsigned long long)seed * 0x9E3779B97F4A7C15ULL ^
                           (unsigned long long)x * 0xC2B2AE3D27D4EB4FULL ^
                           (unsigned long long)y * 0x165667B19E3779F9ULL;
    h ^= h >> 30;
    h *= 0xBF58476D1CE4E5B9ULL;
    h ^= h >> 27;
    h *= 0x94D049BB133111EBULL;
    h ^= h >> 31;
    return (double)(h >> 11) / 9007199254740992.0;  // / 2^53
}
// White phase noise on the lab lattice, as a complex128 plane (phase, 0).
__global__ void k_diffuser_noise(double2* z, int ny, int nx, double dx, double cell, double x0, double y0,
                                 long long seed) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)ny * nx) return;
    const int j = (int)(idx / nx), i = (int)(idx % nx);
    const long long gy = (long long)round(dd(da(coord(j, ny, dx), y0), cell));
    const long long gx = (long long)round(dd(da(coord(i, nx, dx), x0), cell));
    z[idx] = make_double2(ds(dm(dm(hash_noise01(gx, gy, seed), 2.0), M_PI), M_PI), 0);
}
// Per-CTA sums of Re z and (Re z)^2 into partials[block * RS_COUNT + {0, 1}].
__global__ void k_sum_re2(const double2* z, long long n, double* partials) {
    __shared__ double sm[2][32];
    double s1 = 0, s2 = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double v = z[i].x;
        s1 += v;
        s2 += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sm[0][threadIdx.x >> 5] = s1;
        sm[1][threadIdx.x >> 5] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            a += sm[0][w];
            b += sm[1][w];
        }
        partials[(long long)blockIdx.x * RS_COUNT + 0] = a;
        partials[(long long)blockIdx.x * RS_COUNT + 1] = b;
    }
}
// Rescale the phase to standard deviation sigma (sums = {sum v, sum v^2},
// on the device) and multiply by amp exp(i phase).
__global__ void k_diffuser_apply(double2* ex, double2* ey, int pol, long long n, const double2* z,
                                 const double* sums, double sigma, double amp) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double m = dd(sums[0], (double)n);
    const double s2 = ds(dd(sums[1], (double)n), dm(m, m));
    double ph = z[idx].x;
    if (s2 > 0) ph = dm(ds(ph, m), dd(sigma, __dsqrt_rn(s2)));
    apply2(ex, ey, pol, idx, gmul(make_double2(amp, 0), gexpi(ph)));
}

// ---- Gaussian Schell-model synthesis (optics/coherence.go:32-77)
__global__ void k_schell_mu(double2* a, int n, double dx, double coh) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)n * n) return;
    const int j = (int)(idx / n), i = (int)(idx % n);
    const double dy = (j <= n / 2) ? dm((double)j, dx) : dm((double)(j - n), dx);
    const double d = (i <= n / 2) ? dm((double)i, dx) : dm((double)(i - n), dx);
    const double mu = exp(dd(-da(dm(d, d), dm(dy, dy)), dm(dm(2.0, coh), coh)));
    a[idx] = make_double2(mu, 0);
}
__global__ void k_sqrt_re(double* s, const double2* a, long long nn) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= nn) return;
    double v = a[idx].x;
    if (v < 0) v = 0;
    s[idx] = sqrt(v);
}
__global__ void k_mul_map(double2* a, const double* s, long long nn, int batches) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= nn * batches) return;
    a[idx] = gmul(a[idx], make_double2(s[idx % nn], 0));
}
__global__ void k_schell_env(double2* a, int n, double dx, double width, int batches) {
    const long long nn = (long long)n * n;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= nn * batches) return;
    const long long p = idx % nn;
    const int j = (int)(p / n), i = (int)(p % n);
    const double x = coord(i, n, dx), y = coord(j, n, dx);
    const double I = exp(dd(dm(-2.0, da(dm(x, x), dm(y, y))), dm(width, width)));
    a[idx] = gmul(a[idx], make_double2(sqrt(I), 0));
}

// out[i] += w * sum_c |f[c][i]|^2  (PropagatePolychromatic / AverageIntensity)
template <typename C>
__global__ void k_accum_int(double* out, const C* f, int ncomp, long long np, double w) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= np) return;
    double p = 0;
    for (int c = 0; c < ncomp; c++) {
        const C v = f[c * np + idx];
        p += (double)v.x * v.x + (double)v.y * v.y;
    }
    out[idx] += w * p;
}

// r = 4 (|u|^2 - T) u and per-CTA partial sums of (|u|^2 - T)^2
template <typename C>
__global__ void k_residual(const C* u, const double* T, C* r, long long n, double* partials) {
    __shared__ double sm[32];
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double l = 0;
    if (idx < n) {
        const C v = u[idx];
        const double d = (double)v.x * v.x + (double)v.y * v.y - T[idx];
        l = d * d;
        r[idx] = mkc<C>((decltype(C::x))(4 * d * (double)v.x), (decltype(C::x))(4 * d * (double)v.y));
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sm[w];
        partials[(long long)blockIdx.x * RS_COUNT + RS_P] = s;
    }
}

// g = Re(conj(b) * i * t * a), t = exp(i phi)
template <typename C>
__global__ void k_grad(const C* b, const double2* a, const double* phi, double* g, long long n) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    double s, c;
    sincos(phi[idx], &s, &c);
    const double2 av = a[idx];
    const double tar = c * av.x - s * av.y, tai = c * av.y + s * av.x;  // t*a
    const double ir = -tai, ii = tar;                                  // i*t*a
    const C bv = b[idx];
    g[idx] = (double)bv.x * ir + (double)bv.y * ii;
}

// u *= exp(+-i phi) in the context precision (stack masks and their adjoint)
template <typename C>
__global__ void k_mask_phase(C* u, const double* phi, long long n, int conj) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    double s, c;
    sincos(phi[idx], &s, &c);
    if (conj) s = -s;
    const C v = u[idx];
    u[idx] = mkc<C>((decltype(C::x))(c * (double)v.x - s * (double)v.y),
                    (decltype(C::x))(c * (double)v.y + s * (double)v.x));
}

// g = Re(conj(b) * i * v), v = the field just after a mask
template <typename C>
__global__ void k_grad_v(const C* b, const C* v, double* g, long long n) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const C bv = b[idx], vv = v[idx];
    g[idx] = (double)bv.y * vv.x - (double)bv.x * vv.y;
}

// ---- Plane views for the binary plane format (server/views.go:131-258,
// server/server.go:582-634): float32 little-endian [ny][nx].
// Per-CTA maxima of |c|^2 over a plane (peak of a component for the phase mask).
template <typename C>
__global__ void k_norm2_max(const C* a, long long n, double* partial) {
    __shared__ double sm[32];
    double m = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const C v = a[i];
        const double p = da(dm((double)v.x, (double)v.x), dm((double)v.y, (double)v.y));
        m = fmax(m, p);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = fmax(r, sm[w]);
        partial[blockIdx.x] = r;
    }
}
__global__ void k_max_finish(const double* partial, int nb, double* out) {
    __shared__ double sm[32];
    double m = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) m = fmax(m, partial[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = fmax(r, sm[w]);
        *out = r;
    }
}
// view: 0 total (|Ex|^2 [+ |Ey|^2 when polarized] [+ |Ez|^2 when given], as
// Field.Intensity), 1 amplitude (sqrt of total), 2/3/4 |Ex|^2 / |Ey|^2 / |Ez|^2,
// 5/6/7 phase of Ex / Ey / Ez (atan2, NaN where the component's |c|^2 is below
// cut * its peak, or everywhere when the peak is 0).  Written as float32 bits;
// NaN as 0x7fc00000 (the quiet NaN a float32 conversion of math.NaN() gives).
template <typename C>
__global__ void k_plane_view(const C* ex, const C* ey, const C* ez, int pol, long long n, int view,
                             const double* peak, double cut, unsigned* out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    auto n2 = [](C v) { return da(dm((double)v.x, (double)v.x), dm((double)v.y, (double)v.y)); };
    double val;
    bool nan = false;
    if (view <= 1) {
        val = n2(ex[i]);
        if (pol) val = da(val, n2(ey[i]));
        if (ez) val = da(val, n2(ez[i]));
        if (view == 1) val = __dsqrt_rn(val);
    } else if (view <= 4) {
        val = n2(view == 2 ? ex[i] : (view == 3 ? ey[i] : ez[i]));
    } else {
        const C v = view == 5 ? ex[i] : (view == 6 ? ey[i] : ez[i]);
        const double pk = *peak;
        if (pk <= 0 || n2(v) < dm(cut, pk)) {
            nan = true;
            val = 0;
        } else {
            val = atan2((double)v.y, (double)v.x);
        }
    }
    out[i] = nan ? 0x7fc00000u : __float_as_uint(__double2float_rn(val));
}

// ---------------------------------------------------------------- launchers
static inline unsigned nblk(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

cudaError_t launch_lens(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double c, double ap, double x0,
                        double y0, cudaStream_t st) {
    k_lens<<<nblk((long long)ny * nx), 256, 0, st>>>(ex, ey, pol, ny, nx, dx, c, ap, x0, y0);
    return cudaGetLastError();
}
cudaError_t launch_aperture_circle(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double radius,
                                   double x0, double y0, double sig, cudaStream_t st) {
    k_aperture_circle<<<nblk((long long)ny * nx), 256, 0, st>>>(ex, ey, pol, ny, nx, dx, radius, x0, y0, sig);
    return cudaGetLastError();
}
cudaError_t launch_grating(double2* ex, double2* ey, int pol, int ny, int nx, double dx, int kind, double period,
                           double modulation, double duty, double blaze, double rotation, double off,
                           cudaStream_t st) {
    k_grating<<<nblk((long long)ny * nx), 256, 0, st>>>(ex, ey, pol, ny, nx, dx, kind, period, modulation, duty, blaze,
                                                       rotation, off);
    return cudaGetLastError();
}
cudaError_t launch_phase_mask(double2* ex, double2* ey, int pol, long long n, const double* phi, double amp,
                              cudaStream_t st) {
    k_phase_mask<<<nblk(n), 256, 0, st>>>(ex, ey, pol, n, phi, amp);
    return cudaGetLastError();
}
cudaError_t launch_jones(double2* ex, double2* ey, long long n, int mode, double2 a, double2 b, double2 c, double2 d,
                         cudaStream_t st) {
    k_jones<<<nblk(n), 256, 0, st>>>(ex, ey, n, mode, a, b, c, d);
    return cudaGetLastError();
}
cudaError_t launch_scale(double2* ex, double2* ey, int pol, long long n, double2 s, cudaStream_t st) {
    k_scale<<<nblk(n), 256, 0, st>>>(ex, ey, pol, n, s);
    return cudaGetLastError();
}
cudaError_t launch_tilt(double2* ex, double2* ey, int pol, int ny, int nx, double dx, double k, double sx, double sy,
                        cudaStream_t st) {
    k_tilt<<<ny, 256, 0, st>>>(ex, ey, pol, ny, nx, dx, k, sx, sy);
    return cudaGetLastError();
}
cudaError_t launch_diffuser_noise(double2* z, int ny, int nx, double dx, double cell, double x0, double y0,
                                  long long seed, cudaStream_t st) {
    k_diffuser_noise<<<nblk((long long)ny * nx), 256, 0, st>>>(z, ny, nx, dx, cell, x0, y0, seed);
    return cudaGetLastError();
}
int sum_re2_blocks(long long n) { return (int)std::min<long long>(nblk(n), 1184); }
cudaError_t launch_sum_re2(const double2* z, long long n, double* partials, cudaStream_t st) {
    k_sum_re2<<<sum_re2_blocks(n), 256, 0, st>>>(z, n, partials);
    return cudaGetLastError();
}
cudaError_t launch_diffuser_apply(double2* ex, double2* ey, int pol, long long n, const double2* z,
                                  const double* sums, double sigma, double amp, cudaStream_t st) {
    k_diffuser_apply<<<nblk(n), 256, 0, st>>>(ex, ey, pol, n, z, sums, sigma, amp);
    return cudaGetLastError();
}
cudaError_t launch_schell_mu(double2* a, int n, double dx, double coh, cudaStream_t st) {
    k_schell_mu<<<nblk((long long)n * n), 256, 0, st>>>(a, n, dx, coh);
    return cudaGetLastError();
}
cudaError_t launch_sqrt_re(double* s, const double2* a, long long nn, cudaStream_t st) {
    k_sqrt_re<<<nblk(nn), 256, 0, st>>>(s, a, nn);
    return cudaGetLastError();
}
cudaError_t launch_mul_map(double2* a, const double* s, long long nn, int batches, cudaStream_t st) {
    k_mul_map<<<nblk(nn * batches), 256, 0, st>>>(a, s, nn, batches);
    return cudaGetLastError();
}
cudaError_t launch_schell_env(double2* a, int n, double dx, double width, int batches, cudaStream_t st) {
    k_schell_env<<<nblk((long long)n * n * batches), 256, 0, st>>>(a, n, dx, width, batches);
    return cudaGetLastError();
}
cudaError_t launch_accum_int(int fp64, double* out, const void* f, int ncomp, long long np, double w,
                             cudaStream_t st) {
    if (fp64) k_accum_int<double2><<<nblk(np), 256, 0, st>>>(out, reinterpret_cast<const double2*>(f), ncomp, np, w);
    else k_accum_int<float2><<<nblk(np), 256, 0, st>>>(out, reinterpret_cast<const float2*>(f), ncomp, np, w);
    return cudaGetLastError();
}
cudaError_t launch_residual(int fp64, const void* u, const double* T, void* r, long long n, double* partials,
                            int* nblocks, cudaStream_t st) {
    *nblocks = (int)nblk(n);
    if (fp64)
        k_residual<double2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const double2*>(u), T, reinterpret_cast<double2*>(r), n, partials);
    else
        k_residual<float2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const float2*>(u), T, reinterpret_cast<float2*>(r), n, partials);
    return cudaGetLastError();
}
cudaError_t launch_grad(int fp64, const void* b, const double2* a, const double* phi, double* g, long long n,
                        cudaStream_t st) {
    if (fp64) k_grad<double2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const double2*>(b), a, phi, g, n);
    else k_grad<float2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const float2*>(b), a, phi, g, n);
    return cudaGetLastError();
}

cudaError_t launch_mask_phase(int fp64, void* u, const double* phi, long long n, int conj, cudaStream_t st) {
    if (fp64) k_mask_phase<double2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<double2*>(u), phi, n, conj);
    else k_mask_phase<float2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<float2*>(u), phi, n, conj);
    return cudaGetLastError();
}
cudaError_t launch_grad_v(int fp64, const void* b, const void* v, double* g, long long n, cudaStream_t st) {
    if (fp64)
        k_grad_v<double2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const double2*>(b), reinterpret_cast<const double2*>(v), g, n);
    else
        k_grad_v<float2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const float2*>(b), reinterpret_cast<const float2*>(v), g, n);
    return cudaGetLastError();
}

int norm2_max_blocks(long long n) { return (int)std::min<long long>(nblk(n), 1024); }
cudaError_t launch_norm2_max(int fp64, const void* a, long long n, double* partial, double* out, cudaStream_t st) {
    const int nb = norm2_max_blocks(n);
    if (fp64) k_norm2_max<double2><<<nb, 256, 0, st>>>(reinterpret_cast<const double2*>(a), n, partial);
    else k_norm2_max<float2><<<nb, 256, 0, st>>>(reinterpret_cast<const float2*>(a), n, partial);
    k_max_finish<<<1, 1024, 0, st>>>(partial, nb, out);
    return cudaGetLastError();
}
cudaError_t launch_plane_view(int fp64, const void* ex, const void* ey, const void* ez, int pol, long long n, int view,
                              const double* peak, double cut, void* out, cudaStream_t st) {
    unsigned* o = reinterpret_cast<unsigned*>(out);
    if (fp64)
        k_plane_view<double2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const double2*>(ex),
                                                       reinterpret_cast<const double2*>(ey),
                                                       reinterpret_cast<const double2*>(ez), pol, n, view, peak, cut, o);
    else
        k_plane_view<float2><<<nblk(n), 256, 0, st>>>(reinterpret_cast<const float2*>(ex),
                                                      reinterpret_cast<const float2*>(ey),
                                                      reinterpret_cast<const float2*>(ez), pol, n, view, peak, cut, o);
    return cudaGetLastError();
}

}  // namespace wos

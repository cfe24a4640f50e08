// wos_aniso.cu -- anisotropic (possibly biaxial, absorbing) propagation by the
// Berreman 4x4 method, one spectral component per thread (PropagateAnisotropic,
// optics/berreman.go:13-272): the Berreman matrix of the component's
// normalised transverse wavevector, its characteristic polynomial
// (Faddeev-LeVerrier), the four roots (Durand-Kerner), the two forward modes
// with their null vectors (largest adjugate column), the 2x2 decomposition of
// (Ex, Ey) on them and the propagation of each mode.  FP64 throughout, each
// complex operation in the reference's order without contraction; FP64
// compute-bound, between the 2-D FFTs of the context precision.
#include <cuda_runtime.h>
#include <math.h>

#include "wos_fft.cuh"
#include "wos_kernels.cuh"

namespace wos {

namespace {
struct Z {
    double re, im;
};
__device__ __forceinline__ Z zk(double r, double i) { return Z{r, i}; }
__device__ __forceinline__ Z zmul(Z a, Z b) {
    return Z{__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
             __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ Z zadd(Z a, Z b) { return Z{__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)}; }
__device__ __forceinline__ Z zsub(Z a, Z b) { return Z{__dsub_rn(a.re, b.re), __dsub_rn(a.im, b.im)}; }
__device__ __forceinline__ Z zneg(Z a) { return Z{-a.re, -a.im}; }
// complex division as the Go runtime divides: Smith's algorithm
// (R. L. Smith, Algorithm 116, Commun. ACM 5(8), 1962)
__device__ __forceinline__ Z zdiv(Z n, Z m) {
    double e, f;
    if (fabs(m.re) >= fabs(m.im)) {
        const double ratio = __ddiv_rn(m.im, m.re);
        const double denom = __dadd_rn(m.re, __dmul_rn(ratio, m.im));
        e = __ddiv_rn(__dadd_rn(n.re, __dmul_rn(n.im, ratio)), denom);
        f = __ddiv_rn(__dsub_rn(n.im, __dmul_rn(n.re, ratio)), denom);
    } else {
        const double ratio = __ddiv_rn(m.re, m.im);
        const double denom = __dadd_rn(m.im, __dmul_rn(ratio, m.re));
        e = __ddiv_rn(__dadd_rn(__dmul_rn(n.re, ratio), n.im), denom);
        f = __ddiv_rn(__dsub_rn(__dmul_rn(n.im, ratio), n.re), denom);
    }
    return Z{e, f};
}
__device__ __forceinline__ double hyp(double p, double q) {  // math.Hypot's scaling form
    p = fabs(p);
    q = fabs(q);
    if (p < q) {
        const double t = p;
        p = q;
        q = t;
    }
    if (p == 0) return 0;
    q = __ddiv_rn(q, p);
    return __dmul_rn(p, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(q, q))));
}
__device__ __forceinline__ double freq_of(int i, int n, double dx) {
    return (i <= n / 2) ? __ddiv_rn((double)i, __dmul_rn((double)n, dx))
                        : __ddiv_rn((double)(i - n), __dmul_rn((double)n, dx));
}

struct M4 {
    Z m[4][4];
};

// buildBerreman (berreman.go:94-118), psi = (Ex, Hy, Ey, -Hx)
__device__ void berreman(const Eps9& e, double xi, double eta, M4& D) {
    auto E = [&](int i, int j) { return Z{e.v[i * 3 + j].x, e.v[i * 3 + j].y}; };
    const Z one = zk(1, 0);
    const Z r = zdiv(one, E(2, 2));
    const Z x = zk(xi, 0), y = zk(eta, 0);
    D.m[0][0] = zmul(zmul(zneg(x), r), E(2, 0));
    D.m[0][1] = zsub(one, zmul(zmul(x, x), r));
    D.m[0][2] = zmul(zmul(zneg(x), r), E(2, 1));
    D.m[0][3] = zmul(zmul(zneg(x), r), y);
    D.m[1][0] = zsub(zsub(E(0, 0), zmul(y, y)), zmul(zmul(E(0, 2), r), E(2, 0)));
    D.m[1][1] = zmul(zmul(zneg(E(0, 2)), r), x);
    D.m[1][2] = zsub(zadd(E(0, 1), zmul(y, x)), zmul(zmul(E(0, 2), r), E(2, 1)));
    D.m[1][3] = zmul(zmul(zneg(E(0, 2)), r), y);
    D.m[2][0] = zmul(zmul(zneg(y), r), E(2, 0));
    D.m[2][1] = zmul(zmul(zneg(y), r), x);
    D.m[2][2] = zmul(zmul(zneg(y), r), E(2, 1));
    D.m[2][3] = zsub(one, zmul(zmul(y, y), r));
    D.m[3][0] = zsub(zadd(E(1, 0), zmul(x, y)), zmul(zmul(E(1, 2), r), E(2, 0)));
    D.m[3][1] = zmul(zmul(zneg(E(1, 2)), r), x);
    D.m[3][2] = zsub(zsub(E(1, 1), zmul(x, x)), zmul(zmul(E(1, 2), r), E(2, 1)));
    D.m[3][3] = zmul(zmul(zneg(E(1, 2)), r), y);
}

__device__ __forceinline__ Z trace(const M4& A) {
    return zadd(zadd(zadd(A.m[0][0], A.m[1][1]), A.m[2][2]), A.m[3][3]);
}
// B <- A (B + c I), the identity scaled as complex(0|1, 0) * c
__device__ void mul_shift(const M4& A, M4& B, Z c) {
    M4 S;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) S.m[i][j] = zadd(B.m[i][j], zmul(zk(i == j ? 1.0 : 0.0, 0), c));
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            Z s = zk(0, 0);
            for (int k = 0; k < 4; k++) s = zadd(s, zmul(A.m[i][k], S.m[k][j]));
            B.m[i][j] = s;
        }
}
// Faddeev-LeVerrier (berreman.go:130-144): c[0..3] of q^4 + c3 q^3 + c2 q^2 + c1 q + c0
__device__ void char_poly(const M4& A, Z* c) {
    M4 B = A;
    c[3] = zneg(trace(B));
    mul_shift(A, B, c[3]);
    c[2] = zdiv(zneg(trace(B)), zk(2, 0));
    mul_shift(A, B, c[2]);
    c[1] = zdiv(zneg(trace(B)), zk(3, 0));
    mul_shift(A, B, c[1]);
    c[0] = zdiv(zneg(trace(B)), zk(4, 0));
}
__device__ __forceinline__ Z poly(Z z, const Z* c) {
    Z t = zmul(zmul(zmul(z, z), z), z);
    t = zadd(t, zmul(zmul(zmul(c[3], z), z), z));
    t = zadd(t, zmul(zmul(c[2], z), z));
    t = zadd(t, zmul(c[1], z));
    return zadd(t, c[0]);
}
// Durand-Kerner (berreman.go:186-214), at most 300 sweeps
__device__ void roots(const Z* c, Z* z) {
    z[0] = zk(0.4, 0.9);
    z[1] = zk(0.4, -0.9);
    z[2] = zk(-0.4, 0.9);
    z[3] = zk(-0.4, -0.9);
    for (int iter = 0; iter < 300; iter++) {
        double maxd = 0;
        for (int i = 0; i < 4; i++) {
            const Z num = poly(z[i], c);
            Z den = zk(1, 0);
            for (int j = 0; j < 4; j++)
                if (j != i) den = zmul(den, zsub(z[i], z[j]));
            const Z dz = zdiv(num, den);
            z[i] = zsub(z[i], dz);
            const double d = hyp(dz.re, dz.im);
            if (d > maxd) maxd = d;
        }
        if (maxd < 1e-14) break;
    }
}
__device__ __forceinline__ bool forward_mode(Z q) {
    if (q.im > 1e-12) return true;
    if (q.im < -1e-12) return false;
    return q.re > 0;
}
__device__ __forceinline__ Z det3(const Z m[3][3]) {
    const Z a = zmul(m[0][0], zsub(zmul(m[1][1], m[2][2]), zmul(m[1][2], m[2][1])));
    const Z b = zmul(m[0][1], zsub(zmul(m[1][0], m[2][2]), zmul(m[1][2], m[2][0])));
    const Z c = zmul(m[0][2], zsub(zmul(m[1][0], m[2][1]), zmul(m[1][1], m[2][0])));
    return zadd(zsub(a, b), c);
}
// largest-norm column of adj(A - qI) (berreman.go:228-272)
__device__ void null_vector(const M4& A, Z q, Z* best) {
    M4 M = A;
    for (int i = 0; i < 4; i++) M.m[i][i] = zsub(M.m[i][i], q);
    double bestn = -1;
    for (int col = 0; col < 4; col++) {
        Z v[4];
        for (int row = 0; row < 4; row++) {
            Z m[3][3];
            int ri = 0;
            for (int r = 0; r < 4; r++) {
                if (r == row) continue;
                int ci = 0;
                for (int cc = 0; cc < 4; cc++) {
                    if (cc == col) continue;
                    m[ri][ci++] = M.m[r][cc];
                }
                ri++;
            }
            Z cof = det3(m);
            if ((row + col) % 2 == 1) cof = zneg(cof);
            v[row] = cof;
        }
        double nn = 0;
        for (int t = 0; t < 4; t++) nn = __dadd_rn(nn, __dadd_rn(__dmul_rn(v[t].re, v[t].re), __dmul_rn(v[t].im, v[t].im)));
        if (nn > bestn) {
            bestn = nn;
            for (int t = 0; t < 4; t++) best[t] = v[t];
        }
    }
}
__device__ __forceinline__ Z zexpi(double a) {
    double s, c;
    sincos(a, &s, &c);
    return Z{c, s};
}
// anisoMode (berreman.go:41-92)
__device__ void aniso_mode(const Eps9& e, double xi, double eta, double k0, double z, Z& ex, Z& ey) {
    M4 D;
    berreman(e, xi, eta, D);
    Z c[4], rts[4], qs[2], vs[2][4];
    char_poly(D, c);
    roots(c, rts);
    int cnt = 0;
    bool used[4] = {false, false, false, false};
    for (int i = 0; i < 4; i++)
        if (forward_mode(rts[i]) && cnt < 2) {
            qs[cnt] = rts[i];
            null_vector(D, rts[i], vs[cnt]);
            used[i] = true;
            cnt++;
        }
    while (cnt < 2) {
        double best = -1e300;
        int bi = -1;
        for (int i = 0; i < 4; i++)
            if (!used[i] && rts[i].re > best) {
                best = rts[i].re;
                bi = i;
            }
        if (bi < 0) break;
        qs[cnt] = rts[bi];
        null_vector(D, rts[bi], vs[cnt]);
        used[bi] = true;
        cnt++;
    }
    const Z a = vs[0][0], b = vs[1][0], cc = vs[0][2], d = vs[1][2];
    const Z det = zsub(zmul(a, d), zmul(b, cc));
    const Z m1 = zdiv(zsub(zmul(d, ex), zmul(b, ey)), det);
    const Z m2 = zdiv(zadd(zmul(zneg(cc), ex), zmul(a, ey)), det);
    const Z p0 = zmul(zexpi(__dmul_rn(__dmul_rn(k0, qs[0].re), z)), zk(exp(__dmul_rn(__dmul_rn(-k0, qs[0].im), z)), 0));
    const Z p1 = zmul(zexpi(__dmul_rn(__dmul_rn(k0, qs[1].re), z)), zk(exp(__dmul_rn(__dmul_rn(-k0, qs[1].im), z)), 0));
    ex = zadd(zmul(zmul(m1, p0), a), zmul(zmul(m2, p1), b));
    ey = zadd(zmul(zmul(m1, p0), cc), zmul(zmul(m2, p1), d));
}
}  // namespace

template <typename C>
__global__ void __launch_bounds__(128) k_aniso(C* ex, C* ey, int ny, int nx, double dx, double k0, double z,
                                               Eps9 e) {
    using T = decltype(C::x);
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)ny * nx) return;
    const int j = (int)(idx / nx), i = (int)(idx - (long long)j * nx);
    const double kx = __dmul_rn(2 * M_PI, freq_of(i, nx, dx));
    const double ky = __dmul_rn(2 * M_PI, freq_of(j, ny, dx));
    Z a = Z{(double)ex[idx].x, (double)ex[idx].y}, b = Z{(double)ey[idx].x, (double)ey[idx].y};
    aniso_mode(e, __ddiv_rn(kx, k0), __ddiv_rn(ky, k0), k0, z, a, b);
    ex[idx] = mkc<C>((T)a.re, (T)a.im);
    ey[idx] = mkc<C>((T)b.re, (T)b.im);
}

cudaError_t launch_aniso(int fp64, void* planes, int ny, int nx, double dx, double k0, double z, const Eps9& e,
                         cudaStream_t st) {
    const long long np = (long long)ny * nx;
    const unsigned g = (unsigned)((np + 127) / 128);
    if (fp64) {
        double2* p = reinterpret_cast<double2*>(planes);
        k_aniso<double2><<<g, 128, 0, st>>>(p, p + np, ny, nx, dx, k0, z, e);
    } else {
        float2* p = reinterpret_cast<float2*>(planes);
        k_aniso<float2><<<g, 128, 0, st>>>(p, p + np, ny, nx, dx, k0, z, e);
    }
    return cudaGetLastError();
}

}  // namespace wos

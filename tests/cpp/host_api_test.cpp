// Exercises the C++ host interface (include/wos_optics.hpp) on a GPU and
// checks it against the FP64 oracle: Propagate for every method, the nil
// context and z == 0 rules, ParseMethod errors, split-step, polychromatic,
// volume, and the inverse-design Forward / Backward pairs (adjoint identity).
// Prints "ok" and returns 0 on success.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/wos_optics.hpp"
#include "../../oracle/wos_oracle.h"

using namespace wos::optics;

static double rel_l2(const std::vector<cplx>& a, const oc128* b) {
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); i++) {
        const double dr = a[i].real() - b[i].re, di = a[i].imag() - b[i].im;
        num += dr * dr + di * di;
        den += b[i].re * b[i].re + b[i].im * b[i].im;
    }
    return std::sqrt(num / den);
}

#define REQUIRE(c)                                                         \
    do {                                                                   \
        if (!(c)) {                                                        \
            std::fprintf(stderr, "FAILED %s at line %d\n", #c, __LINE__); \
            return 1;                                                      \
        }                                                                  \
    } while (0)

int main() {
    const int n = 128;
    const double dx = 2e-6, wl = 632.8e-9, z = 4e-3;
    Field f(n, dx, true);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            const double x = f.X(i), y = f.Y(j);
            const double g = std::exp(-(x * x + y * y) / (40e-6 * 40e-6));
            f.Ex[(size_t)j * n + i] = cplx(g * std::cos(3e4 * x), g * std::sin(3e4 * x));
            f.Ey[(size_t)j * n + i] = 0.5 * f.Ex[(size_t)j * n + i] * cplx(0, 1);
        }
    Backend b(WOS_FP64);
    REQUIRE(GPUAvailable());
    const char* methods[] = {"asm", "asm_pad", "asm_shift", "asm_shift_pad", "fresnel_tf", "fresnel_ir", "fraunhofer"};
    for (const char* ms : methods) {
        Method m = ParseMethod(ms);
        Field g = f.Clone();
        Warnings w;
        Context c;
        c.Wavelength = wl;
        c.W = &w;
        Propagate(b, g, z, m, &c);
        std::vector<oc128> ex(f.Ex.size()), ey(f.Ey.size());
        std::memcpy(ex.data(), f.Ex.data(), ex.size() * sizeof(oc128));
        std::memcpy(ey.data(), f.Ey.data(), ey.size() * sizeof(oc128));
        or_field of{n, n, dx, 1, ex.data(), ey.data()};
        or_context oc{};
        oc.wavelength = wl;
        oc.has_warnings = 1;
        REQUIRE(or_propagate(&of, z, method_id(m), &oc) == 0);
        const double e = rel_l2(g.Ex, ex.data());
        std::printf("%-14s rel_l2 %.3e  warnings %zu/%d  dx %.6g\n", ms, e, w.List().size(), oc.n_warn, g.DX);
        // carrier-shift methods: two correct FP64 implementations of the
        // reference algorithm differ by up to 3.2e-11 on tilted fields
        const bool shifted = m == Method::ASMShift || m == Method::ASMShiftPad;
        const double tol = shifted ? 5e-11 : 1e-12;
        REQUIRE(e <= tol);
        REQUIRE(rel_l2(g.Ey, ey.data()) <= tol);
        REQUIRE((int)w.List().size() == oc.n_warn);
        REQUIRE(std::fabs(g.DX - of.dx) <= 1e-15 * of.dx);
    }
    // nil context -> Evanescent "decay", no warnings; z == 0 is a no-op
    {
        Field g = f.Clone();
        Propagate(b, g, 0.0, Method::ASM, nullptr);
        REQUIRE(g.Ex == f.Ex);
        bool threw = false;
        try {
            ParseMethod("vectorial_x");
        } catch (const Error& e) {
            threw = e.status == WOS_UNKNOWN_METHOD;
        }
        REQUIRE(threw);
    }
    // PropagateSplitStep through a uniform medium: plane-wave phase k0 n z
    {
        Field g(n, 1e-5, false);
        for (auto& v : g.Ex) v = cplx(1, 0);
        wos_index_desc d{};
        d.re_bg = 1.5;
        Context c;
        c.Wavelength = wl;
        PropagateSplitStep(b, g, 0.1, d, 20, &c);
        const cplx v = g.Ex[(size_t)(n / 2) * n + n / 2];
        const double got = std::remainder(std::atan2(v.imag(), v.real()) - 2 * M_PI / wl * 1.5 * 0.1, 2 * M_PI);
        REQUIRE(std::fabs(got) <= 1e-6);
    }
    // PropagatePolychromatic and Propagate3D
    {
        Context c;
        c.Wavelength = wl;
        Field s = f.Clone();
        s.Polarized = false;
        auto I = PropagatePolychromatic(b, s, z, {{wl, 1.0}, {532e-9, 0.5}}, Method::ASM, &c);
        REQUIRE(I.size() == (size_t)n * n);
        auto vol = Propagate3D(b, s, {0.0, z}, Method::ASM, &c);
        REQUIRE(vol.size() == 2 && vol[0].Ex == s.Ex);
        double ip = 0;
        for (double v : I) ip += v;
        REQUIRE(ip > 0);
    }
    // Inverse-design pair: BackwardBPM is the adjoint of ForwardBPM, BackwardASM of ForwardASM
    {
        const int m = 64;
        Field x(m, 1e-6, false), y(m, 1e-6, false);
        for (int i = 0; i < m * m; i++) {
            x.Ex[i] = cplx(std::sin(0.37 * i), std::cos(0.11 * i));
            y.Ex[i] = cplx(std::cos(0.23 * i), std::sin(0.71 * i));
        }
        wos_index_desc d{};
        d.re_bg = 1.5;
        d.core_dn = 0.01;
        d.core_w = 15e-6;
        d.border_px = 4;
        d.border_order = 2;
        d.border_strength = 3e-3;
        Context c;
        c.Wavelength = wl;
        for (int op = 0; op < 2; op++) {
            Field ax = x.Clone(), ahy = y.Clone();
            if (op == 0) {
                ForwardBPM(b, ax, 20e-6, d, 4, &c);
                BackwardBPM(b, ahy, 20e-6, d, 4, c);
            } else {
                ForwardASM(b, ax, 30e-6, &c);
                BackwardASM(b, ahy, 30e-6, c);
            }
            cplx lhs = 0, rhs = 0;
            double nax = 0, ny = 0;
            for (int i = 0; i < m * m; i++) {
                lhs += std::conj(y.Ex[i]) * ax.Ex[i];
                rhs += std::conj(ahy.Ex[i]) * x.Ex[i];
                nax += std::norm(ax.Ex[i]);
                ny += std::norm(y.Ex[i]);
            }
            REQUIRE(std::abs(lhs - rhs) <= 1e-11 * std::sqrt(nax * ny));
        }
    }
    std::printf("ok\n");
    return 0;
}

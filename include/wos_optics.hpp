// wos_optics.hpp -- C++17 host interface over libwosgpu.so with the names and
// semantics of the reference's Go `optics` package for the propagation path:
//
//   Method / ParseMethod        optics/propagate.go:38-61
//   Context, Warnings           optics/field.go:237-254, 305-346
//   Field                       optics/field.go:14-83
//   Propagate                   optics/propagate.go:65-102
//   PropagateSplitStep          optics/medium.go:22-45 (parametric medium)
//   PropagatePolychromatic      optics/polychromatic.go:18-44
//   Propagate3D                 optics/volume.go:8-18
//   GenerateSchellRealizations, PropagatePartiallyCoherent
//                               optics/coherence.go:22-116
//   Propagate1D                 optics/propagate.go:718-738
//   ForwardASM / BackwardASM, ForwardBPM / BackwardBPM   (inverse design; no reference counterpart)
//   Field.ApplyJones / ScaleAmplitude / ApplyTilt / ShiftField / ApplyBandlimit
//                               optics/field.go:109-168,199-228,264-294
//   ApplyDiffuser               optics/elements.go:722-783 (diffuserEl.Apply)
//   SetGPU / GPUEnabled / GPUAvailable / GPUBackendInfo
//                               optics/gpu.go:106-143 (WOS_GPU=1 enables)
//
// Every numeric step runs on the GPU through the C ABI; errors come back as
// Error exceptions carrying the wos_status and message.  There is no CPU
// path: without a device the calls fail.
#pragma once

#include <complex>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "wos_gpu.h"

namespace wos {
namespace optics {

using cplx = std::complex<double>;

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(int st) {
    if (st != WOS_OK) throw Error(st, std::string(wos_status_string(st)) + ": " + wos_last_error());
}

enum class Method { Auto, ASM, ASMPad, ASMShift, ASMShiftPad, FresnelTF, FresnelIR, Fraunhofer };

// ParseMethod: unknown names are errors; "" means auto.
inline Method ParseMethod(const std::string& s) {
    if (s == "" || s == "auto") return Method::Auto;
    if (s == "asm") return Method::ASM;
    if (s == "asm_pad") return Method::ASMPad;
    if (s == "asm_shift") return Method::ASMShift;
    if (s == "asm_shift_pad") return Method::ASMShiftPad;
    if (s == "fresnel_tf") return Method::FresnelTF;
    if (s == "fresnel_ir") return Method::FresnelIR;
    if (s == "fraunhofer") return Method::Fraunhofer;
    throw Error(WOS_UNKNOWN_METHOD, "unknown propagation method \"" + s + "\"");
}

inline int method_id(Method m) {
    switch (m) {
    case Method::Auto:
    case Method::ASM: return WOS_ASM;
    case Method::ASMPad: return WOS_ASM_PAD;
    case Method::ASMShift: return WOS_ASM_SHIFT;
    case Method::ASMShiftPad: return WOS_ASM_SHIFT_PAD;
    case Method::FresnelTF: return WOS_FRESNEL_TF;
    case Method::FresnelIR: return WOS_FRESNEL_IR;
    case Method::Fraunhofer: return WOS_FRAUNHOFER;
    }
    return WOS_ASM;
}

struct Warning {
    std::string code;
    int count = 0;
    double value = 0;
};

// Warnings: identical codes accumulate a count; a non-zero value replaces the
// stored one (Warnings.Add semantics).
class Warnings {
  public:
    void Add(const std::string& code, double value) {
        for (auto& w : items_)
            if (w.code == code) {
                w.count++;
                if (value != 0) w.value = value;
                return;
            }
        items_.push_back({code, 1, value});
    }
    const std::vector<Warning>& List() const { return items_; }

  private:
    std::vector<Warning> items_;
};

struct Context {
    double Wavelength = 0;
    std::string Evanescent = "decay";
    double EvanescentLimit = 0;
    bool BackwardRegularize = false;
    double TikhonovAlpha = 0;
    Warnings* W = nullptr;  // nil Warnings: diagnostics are not computed

    wos_context c() const {
        wos_context r{};
        r.wavelength = Wavelength;
        r.evanescent_zero = Evanescent == "zero";
        r.evanescent_limit = EvanescentLimit;
        r.backward_regularize = BackwardRegularize;
        r.tikhonov_alpha = TikhonovAlpha;
        r.diagnostics = W != nullptr;
        return r;
    }
    // Warnings.Add for every warning code a call raised
    void absorb(const wos_diag& d) {
        static const char* codes[WOS_W_COUNT] = {"evanescent_filtered", "backward_regularized",
                                                 "backward_evanescent", "asm_alias_wrap", "fresnel_tf_alias",
                                                 "fresnel_ir_alias", "fraunhofer_nearfield"};
        if (!W) return;
        for (int b = 0; b < WOS_W_COUNT; b++)
            for (int k = 0; k < d.warn_count[b]; k++) W->Add(codes[b], k + 1 == d.warn_count[b] ? d.warn_value[b] : 0);
    }
};

// Field: Ex / Ey row-major ny x nx complex128 (ny == nx == N for the reference).
struct Field {
    int NY = 0, NX = 0;
    double DX = 0;
    bool Polarized = false;
    std::vector<cplx> Ex, Ey;

    Field() = default;
    Field(int n, double dx, bool polarized) : Field(n, n, dx, polarized) {}
    Field(int ny, int nx, double dx, bool polarized)
        : NY(ny), NX(nx), DX(dx), Polarized(polarized), Ex((size_t)ny * nx), Ey((size_t)ny * nx) {}
    double X(int i) const { return ((double)i - (double)NX / 2) * DX; }
    double Y(int j) const { return ((double)j - (double)NY / 2) * DX; }
    double Intensity(size_t i) const {
        double p = std::norm(Ex[i]);
        if (Polarized) p += std::norm(Ey[i]);
        return p;
    }
    double Power() const {
        double p = 0;
        for (size_t i = 0; i < Ex.size(); i++) p += Intensity(i);
        return p * DX * DX;
    }
    Field Clone() const { return *this; }
    wos_field c() {
        wos_field f{};
        f.ny = NY;
        f.nx = NX;
        f.dx = DX;
        f.polarized = Polarized;
        f.ex = reinterpret_cast<wos_c128*>(Ex.data());
        f.ey = reinterpret_cast<wos_c128*>(Ey.data());
        return f;
    }
};

// One device context; Backend::Default() follows SetGPU / WOS_GPU.
class Backend {
  public:
    explicit Backend(int precision = WOS_FP64, int device = 0) { check(wos_ctx_create(device, precision, &ctx_)); }
    ~Backend() {
        if (ctx_) wos_ctx_destroy(ctx_);
    }
    Backend(const Backend&) = delete;
    Backend& operator=(const Backend&) = delete;
    wos_ctx handle() const { return ctx_; }

  private:
    wos_ctx ctx_ = nullptr;
};

inline bool& gpu_enabled_flag() {
    static bool on = [] {
        const char* v = std::getenv("WOS_GPU");
        return v && std::string(v) == "1";
    }();
    return on;
}
inline bool GPUAvailable() { return wos_device_count() > 0; }
inline bool GPUEnabled() { return gpu_enabled_flag() && GPUAvailable(); }
inline bool SetGPU(bool on) {
    gpu_enabled_flag() = on && GPUAvailable();
    return gpu_enabled_flag();
}
inline std::string GPUBackendInfo() { return wos_backend_info(); }

// Propagate: z == 0 is a no-op, auto means asm, a nil context means
// Context{Evanescent: "decay"}; the field is updated in place (DX changes
// for fraunhofer).
inline void Propagate(Backend& b, Field& f, double z, Method m, Context* ctx) {
    if (z == 0) return;
    Context local;
    if (!ctx) ctx = &local;
    wos_field cf = f.c();
    wos_diag d{};
    wos_context cc = ctx->c();
    check(wos_propagate(b.handle(), &cf, z, method_id(m), &cc, &d));
    f.DX = cf.dx;
    ctx->absorb(d);
}

// PropagateSplitStep with a parametric medium (wos_index_desc).
inline void PropagateSplitStep(Backend& b, Field& f, double z, const wos_index_desc& n, int steps, Context* ctx) {
    if (z == 0) return;
    Context local;
    if (!ctx) ctx = &local;
    wos_field cf = f.c();
    wos_diag d{};
    wos_context cc = ctx->c();
    check(wos_splitstep(b.handle(), &cf, z, &n, steps, &cc, &d));
    ctx->absorb(d);
}

struct WavelengthSample {
    double Wavelength = 0, Weight = 0;
};

inline std::vector<double> PropagatePolychromatic(Backend& b, Field& f, double z,
                                                  const std::vector<WavelengthSample>& samples, Method m,
                                                  Context* ctx) {
    std::vector<double> wl, w, out((size_t)f.NY * f.NX);
    for (auto& s : samples) {
        wl.push_back(s.Wavelength);
        w.push_back(s.Weight);
    }
    wos_field cf = f.c();
    wos_diag d{};
    wos_context cc = ctx ? ctx->c() : wos_context{};
    check(wos_polychromatic(b.handle(), &cf, z, wl.data(), w.data(), (int)samples.size(), method_id(m),
                            ctx ? &cc : nullptr, out.data(), &d));
    if (ctx) ctx->absorb(d);
    return out;
}

inline std::vector<Field> Propagate3D(Backend& b, Field& f, const std::vector<double>& zs, Method m, Context* ctx) {
    const int ncomp = f.Polarized ? 2 : 1;
    const size_t np = (size_t)f.NY * f.NX;
    std::vector<cplx> out(np * ncomp * zs.size());
    wos_field cf = f.c();
    wos_diag d{};
    Context local;
    if (!ctx) ctx = &local;
    wos_context cc = ctx->c();
    check(wos_volume(b.handle(), &cf, zs.data(), (int)zs.size(), method_id(m), &cc,
                     reinterpret_cast<wos_c128*>(out.data()), &d));
    ctx->absorb(d);
    std::vector<Field> res;
    for (size_t q = 0; q < zs.size(); q++) {
        Field g(f.NY, f.NX, f.DX, f.Polarized);
        std::copy(out.begin() + q * ncomp * np, out.begin() + (q * ncomp + 1) * np, g.Ex.begin());
        if (ncomp == 2) std::copy(out.begin() + (q * ncomp + 1) * np, out.begin() + (q * ncomp + 2) * np, g.Ey.begin());
        res.push_back(std::move(g));
    }
    return res;
}

struct SchellSourceParams {
    double Width = 0, Coherence = 0;
};

// noise: m * n * n values in place of complex(NormFloat64(), NormFloat64())/sqrt2
inline std::vector<Field> GenerateSchellRealizations(Backend& b, int n, double dx, const SchellSourceParams& p,
                                                     int m, const std::vector<cplx>& noise) {
    if (m <= 0) m = 1;
    std::vector<cplx> out((size_t)n * n * m);
    check(wos_schell_modes(b.handle(), n, dx, p.Width, p.Coherence, m,
                           reinterpret_cast<const wos_c128*>(noise.data()), reinterpret_cast<wos_c128*>(out.data())));
    std::vector<Field> res;
    for (int q = 0; q < m; q++) {
        Field g(n, dx, false);
        std::copy(out.begin() + (size_t)q * n * n, out.begin() + (size_t)(q + 1) * n * n, g.Ex.begin());
        res.push_back(std::move(g));
    }
    return res;
}

inline std::vector<double> PropagatePartiallyCoherent(Backend& b, int n, double dx, const SchellSourceParams& src,
                                                      int m, const std::vector<cplx>& noise, double z, Method meth,
                                                      Context* ctx) {
    std::vector<double> out((size_t)n * n);
    wos_diag d{};
    Context local;
    if (!ctx) ctx = &local;
    wos_context cc = ctx->c();
    check(wos_partially_coherent(b.handle(), n, dx, src.Width, src.Coherence, m,
                                 reinterpret_cast<const wos_c128*>(noise.data()), z, method_id(meth), &cc, out.data(),
                                 &d));
    ctx->absorb(d);
    return out;
}

// Inverse design: the forward operators and their adjoints (conj transfer
// functions, conj screens, BPM slices in reverse order), host fields in place.
inline void ForwardASM(Backend& b, Field& f, double z, Context* ctx) { Propagate(b, f, z, Method::ASM, ctx); }
inline void BackwardASM(Backend& b, Field& f, double z, const Context& ctx) {
    wos_field cf = f.c();
    wos_context cc = ctx.c();
    check(wos_asm_adjoint(b.handle(), &cf, z, &cc));
}
inline void ForwardBPM(Backend& b, Field& f, double z, const wos_index_desc& n, int steps, Context* ctx) {
    PropagateSplitStep(b, f, z, n, steps, ctx);
}
inline void BackwardBPM(Backend& b, Field& f, double z, const wos_index_desc& n, int steps, const Context& ctx) {
    wos_field cf = f.c();
    wos_context cc = ctx.c();
    check(wos_splitstep_adjoint(b.handle(), &cf, z, &n, steps, &cc));
}

// Propagate1D: a line of n = a.size() samples in place (wl apart from ctx).
inline void Propagate1D(Backend& b, std::vector<cplx>& a, double dx, double z, double wl, Context* ctx) {
    Context local;
    if (!ctx) ctx = &local;
    wos_diag d{};
    wos_context cc = ctx->c();
    check(wos_propagate1d(b.handle(), (int)a.size(), reinterpret_cast<wos_c128*>(a.data()), dx, z, wl, &cc, &d));
    ctx->absorb(d);
}

inline wos_c128 c128(cplx v) { return wos_c128{v.real(), v.imag()}; }

// Field methods of the reference, as free functions over a Backend.
inline void ApplyJones(Backend& b, Field& f, cplx a, cplx bb, cplx c, cplx d) {
    wos_field cf = f.c();
    check(wos_apply_jones(b.handle(), &cf, c128(a), c128(bb), c128(c), c128(d)));
    f.Polarized = cf.polarized != 0;
}
inline void ScaleAmplitude(Backend& b, Field& f, cplx s) {
    wos_field cf = f.c();
    check(wos_scale_amplitude(b.handle(), &cf, c128(s)));
}
inline void ApplyTilt(Backend& b, Field& f, double tx, double ty, double wl) {
    wos_field cf = f.c();
    check(wos_apply_tilt(b.handle(), &cf, tx, ty, wl));
}
inline void ShiftField(Backend& b, Field& f, double du, double dv) {
    wos_field cf = f.c();
    check(wos_shift_field(b.handle(), &cf, du, dv));
}
struct BandlimitOpts {
    double Fraction = 0, Sigma = 0;
};
inline void ApplyBandlimit(Backend& b, Field& f, const BandlimitOpts* bl) {
    if (!bl) return;
    wos_field cf = f.c();
    check(wos_apply_bandlimit(b.handle(), &cf, bl->Fraction, bl->Sigma));
}
inline void ApplyDiffuser(Backend& b, Field& f, double sigma, double correlation, double amplitude, long long seed,
                          double x0, double y0) {
    wos_field cf = f.c();
    check(wos_apply_diffuser(b.handle(), &cf, sigma, correlation, amplitude, seed, x0, y0));
}

}  // namespace optics
}  // namespace wos

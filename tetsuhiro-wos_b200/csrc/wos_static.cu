// wos_static.cu -- zero-padded angular-spectrum propagation that allocates no
// device memory, for callers that cannot call cudaMalloc.
//
// Who needs it: applications that reserve all of a GPU's memory up front and
// hand it out through their own allocator (a serving process with a fixed
// memory budget, a framework's caching allocator), and pipelines that cannot
// tolerate the device-wide synchronisation cudaFree implies.  The regular
// entry points grow a per-context workspace with cudaMalloc on first use; this
// one keeps its workspace in file-scope __device__ arrays instead, so calling
// it never allocates.
//
// The price: the arrays below bound the problem size, every call shares them,
// and once placed on a device they stay there until the process exits (16 MiB
// + 32 KiB per device).  They are placed when the CUDA runtime loads this
// file's device code into the device's context: under lazy module loading
// (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2) that is the first
// call of this entry point on the device, so a caller whose allocator takes
// the whole GPU must make that first call before reserving its memory, or run
// with CUDA_MODULE_LOADING=EAGER (the arrays are then placed when the context
// is created).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/wos_gpu.h"
#include "wos_kernels.cuh"

namespace wos {
void set_last_error(const char* msg);
}

using namespace wos;

namespace {

constexpr int kNoAllocMaxN = 1024;                 // largest nx and ny (powers of two)
constexpr int kNoAllocMaxL = 2 * kNoAllocMaxN;     // padded line length
constexpr int kNoAllocMaxDev = 64;

// Intermediate of the padded propagation: ny rows x 2nx complex64.
__device__ __align__(256) float2 g_noalloc_scratch[(size_t)kNoAllocMaxN * kNoAllocMaxL];
// Twiddles exp(-2 pi i k / L) of every power-of-two L <= kNoAllocMaxL, table
// of L at offset L - 2 (2 + 4 + ... + 2048 < 2 * 2048 entries).
__device__ __align__(256) float2 g_noalloc_twiddles[2 * kNoAllocMaxL];

struct DeviceState {
    bool ready = false;
    unsigned long long ctx_id = 0;  // the context the addresses and tables belong to
    float2* scratch = nullptr;      // device address of g_noalloc_scratch on this device
    float2* tw = nullptr;           // device address of g_noalloc_twiddles
};
DeviceState g_state[kNoAllocMaxDev];
std::mutex g_state_mu;

int err(int status, const char* msg) {
    set_last_error(msg);
    return status;
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// The unique id of the current CUDA context (cuCtxGetId, through the
// runtime's driver entry points, so nothing links libcuda).  A context that
// the caller destroyed and re-created (cudaDeviceReset) has a new id, and its
// copy of the arrays starts uninitialised.
int current_ctx_id(unsigned long long* id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
            return err(WOS_CUDA_ERROR, "no-alloc asm_pad: cuCtxGetCurrent / cuCtxGetId not available");
        get_current = reinterpret_cast<GetCurrent>(f1);
        get_id = reinterpret_cast<GetId>(f2);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS)
        return err(WOS_CUDA_ERROR, "no-alloc asm_pad: no current CUDA context");
    return WOS_OK;
}

// Once per device context, with that device current: resolve the arrays'
// device addresses and fill the twiddle tables (a kernel on the caller's
// stream, then a stream synchronisation so later calls on any stream see
// them).  Done again when the device's context has been re-created.
int setup(int dev, cudaStream_t st, DeviceState** out) {
    std::lock_guard<std::mutex> lk(g_state_mu);
    DeviceState& s = g_state[dev];
    unsigned long long id = 0;
    const int rc = current_ctx_id(&id);
    if (rc != WOS_OK) return rc;
    if (s.ready && s.ctx_id != id) s.ready = false;
    if (!s.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));
        s.scratch = static_cast<float2*>(p);
        e = cudaGetSymbolAddress(&p, g_noalloc_twiddles);
        if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));
        s.tw = static_cast<float2*>(p);
        for (int L = 2; L <= kNoAllocMaxL; L <<= 1) {
            e = launch_twiddles(0, s.tw + (L - 2), L, st);
            if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));
        }
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));
        s.ctx_id = id;
        s.ready = true;
    }
    *out = &s;
    return WOS_OK;
}

}  // namespace

extern "C" WOS_API int wos_asm_pad_c64_noalloc(const void* in, void* out, int ny, int nx, double dx, double z,
                                               const wos_context* c, void* stream) {
    if (!in || !out) return err(WOS_INVALID_ARG, "null field pointer");
    if (!pow2(ny) || !pow2(nx) || ny < 4 || nx < 4)
        return err(WOS_UNSUPPORTED_SIZE, "no-alloc asm_pad: ny and nx must be powers of two >= 4");
    if (ny > kNoAllocMaxN || nx > kNoAllocMaxN)
        return err(WOS_UNSUPPORTED_SIZE, "no-alloc asm_pad: ny and nx must not exceed 1024 "
                                         "(the static workspace holds a 1024 x 2048 complex64 intermediate)");
    if (!(dx > 0)) return err(WOS_INVALID_ARG, "dx must be > 0");
    wos_context cc{};
    if (c) cc = *c;
    if (!(cc.wavelength > 0)) return err(WOS_INVALID_ARG, "wavelength must be > 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDev) return err(WOS_INVALID_ARG, "device index out of range");
    const long long np = (long long)ny * nx;
    if (z == 0) {  // Propagate returns the field unchanged (optics/propagate.go:66-68)
        if (in == out) return WOS_OK;
        e = cudaMemcpyAsync(out, in, (size_t)np * sizeof(float2), cudaMemcpyDeviceToDevice, st);
        return e == cudaSuccess ? WOS_OK : err(WOS_CUDA_ERROR, cudaGetErrorString(e));
    }
    DeviceState* s = nullptr;
    const int rc = setup(dev, st, &s);
    if (rc != WOS_OK) return rc;

    const int mx = 2 * nx, my = 2 * ny, offx = nx / 2, offy = ny / 2;
    // evanescent policy (optics/propagate.go:186-199)
    int zero = 0, reg = 0;
    double alpha = 0;
    if (z < 0) {
        if (cc.backward_regularize) {
            reg = 1;
            alpha = cc.tikhonov_alpha > 0 ? cc.tikhonov_alpha : 1e-3;
        } else {
            zero = 1;
        }
    } else {
        zero = cc.evanescent_zero;
    }

    // rows: input into the middle of 2nx-point lines -> scratch (every
    // position of every scratch row is written here before it is read below,
    // so nothing has to be cleared between calls)
    RowArgs r{};
    r.mode = ROW_FWD;
    r.rows = ny;
    r.L = mx;
    r.ny_grid = ny;
    r.nx_grid = nx;
    r.dx = dx;
    r.in = in;
    r.in_ld = nx;
    r.in_off = offx;
    r.in_n = nx;
    r.out = s->scratch;
    r.out_ld = mx;
    r.out_n = mx;
    r.out_scale = 1.0;
    r.pre_amp = 1.0;
    r.weight = 1.0;
    r.tw = s->tw + (mx - 2);
    r.batch = 1;
    e = launch_rows(0, r, st);
    if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));

    // columns: zero-padded 2ny-point FFT, band-limited H, inverse, keep ny rows
    ColArgs a{};
    a.mode = COL_FUSED;
    a.ncols = mx;
    a.L = my;
    int W = 8;
    {
        const int E = pick_E(0, my), T = my / E, maxt = max_threads_for(0, E);
        while (W > 1 && (W * T > maxt || col_smem_bytes(0, my, W) > 200 * 1024)) W >>= 1;
    }
    a.W = W;
    a.src = s->scratch;
    a.src_ld = mx;
    a.in_off = offy;
    a.in_n = ny;
    a.dst = s->scratch;
    a.dst_ld = mx;
    a.out_off = offy;
    a.out_n = ny;
    a.tw = s->tw + (my - 2);
    a.h.kind = H_ASM;
    a.h.exact = 0;
    a.h.wl = cc.wavelength;
    a.h.k = 2 * M_PI / cc.wavelength;
    a.h.z = z;
    a.h.kz = a.h.k * z;
    a.h.kaz = a.h.k * (z < 0 ? -z : z);
    a.h.zero_ev = zero;
    a.h.reg = reg;
    a.h.alpha = alpha;
    a.h.limit = cc.evanescent_limit;
    a.h.dx = dx;
    a.h.lfx = mx;
    a.h.lfy = my;
    a.h.scale = 1.0 / ((double)mx * (double)my);
    a.h.c_re = 1.0;
    a.hist_dx = dx;
    a.out_scale = 1.0;
    a.batch = 1;
    e = launch_cols(0, a, st);
    if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));

    // rows: inverse over 2nx points, keep the nx central columns -> out
    RowArgs q{};
    q.mode = ROW_INV;
    q.rows = ny;
    q.L = mx;
    q.ny_grid = ny;
    q.nx_grid = nx;
    q.dx = dx;
    q.in = s->scratch;
    q.in_ld = mx;
    q.in_n = mx;
    q.out = out;
    q.out_ld = nx;
    q.out_off = offx;
    q.out_n = nx;
    q.out_scale = 1.0;
    q.pre_amp = 1.0;
    q.weight = 1.0;
    q.tw = s->tw + (mx - 2);
    q.batch = 1;
    e = launch_rows(0, q, st);
    if (e != cudaSuccess) return err(WOS_CUDA_ERROR, cudaGetErrorString(e));
    return WOS_OK;
}

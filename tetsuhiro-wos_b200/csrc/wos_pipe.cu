// wos_pipe.cu -- persistent, double-buffered sweeps of the band-limited ASM
// hot path (power-of-two lines, native precision in and out).
//
// Both kernels run one CTA per resident slot and walk the work units
// u = blockIdx.x, blockIdx.x + gridDim.x, ...  Shared memory holds two stages;
// the k-th unit of a CTA lands in stage k & 1, signalled by that stage's
// mbarrier (phase parity (k >> 1) & 1).  When a unit is done with its stage
// (its input read into registers and the stage used as the exchange buffer of
// its passes), one thread hands the stage to the unit after next.
//
//   k_rows_pipe: a unit is LINES consecutive rows of one batch element,
//       fetched by one-dimensional bulk copies (cp.async.bulk);
//   k_cols_pipe: a unit is a tile of W adjacent columns, fetched as L/BR
//       boxes of BR rows x W columns by tiled tensor copies
//       (cp.async.bulk.tensor.3d over a {columns, rows, batch} map).
//
// Every wait is bounded (kWaitCycles SM clocks).  A wait that expires sets
// kPipeErrWait in the device error word, waits (bounded again) for the copies
// it still has in flight and ends the CTA; the host reports it as a timeout.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <unordered_map>

#include "wos_fast_dev.cuh"
#include "wos_pipe.cuh"

namespace wos {
namespace {

constexpr long long kWaitCycles = 4000000000LL;  // about two seconds of SM clock

__device__ __forceinline__ unsigned saddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of parity `parity` to complete; false after kWaitCycles.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(b, parity))
        if (clock64() - t0 > kWaitCycles) return false;
    return true;
}
// Order this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes to the same stage.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     saddr(dst)),
                 "l"(src), "r"(bytes), "r"(saddr(b))
                 : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* b) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(saddr(b))
        : "memory");
}

// A failed wait: record it, drain (bounded) the copies this CTA still has in
// flight, and let the caller return.  Called by every thread of the CTA.
__device__ void pipe_fail(unsigned* err, unsigned long long* bar, int k, bool next_issued) {
    if (threadIdx.x == 0) {
        mbar_wait(&bar[k & 1], (unsigned)((k >> 1) & 1));
        if (next_issued) mbar_wait(&bar[(k + 1) & 1], (unsigned)(((k + 1) >> 1) & 1));
        if (err) atomicOr(err, kPipeErrWait);
    }
}

constexpr size_t round128(size_t b) { return (b + 127) / 128 * 128; }
constexpr size_t kMaxSmem = 227 * 1024;  // opt-in shared memory per CTA

// ------------------------------------------------------------------- rows
template <typename Real, int L, int E> struct RowPipe {
    using C = typename CT<Real>::t;
    static constexpr int T = L / E;
    static constexpr int LINES = T >= 256 ? 1 : 256 / T;
    static constexpr int THREADS = LINES * T;
    static constexpr size_t STAGE = round128((size_t)LINES * frow_stride(L, E) * sizeof(C));
    static constexpr size_t SMEM = 2 * STAGE + 16;
    // two resident CTAs (<= 128 registers a thread at 256 threads): the
    // complex128 forward sweep of 2048 points otherwise takes 134 and runs one
    // CTA per SM
    static constexpr int MINB = THREADS <= 256 ? 2 : 1;
};

template <typename Real, int L, int E, bool INV>
__global__ void __launch_bounds__(RowPipe<Real, L, E>::THREADS, RowPipe<Real, L, E>::MINB) k_rows_pipe(const FastRows a) {
    using C = typename CT<Real>::t;
    using PL = FPlan<L, E>;
    using RP = RowPipe<Real, L, E>;
    constexpr int T = RP::T, LINES = RP::LINES;
    constexpr unsigned ESZ = sizeof(C);
    constexpr int R1 = INV ? E : PL::RS;
    constexpr int RO = INV ? PL::RS : E;
    extern __shared__ __align__(128) unsigned char smraw[];
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw + 2 * RP::STAGE);
    const int line = threadIdx.x / T, tt = threadIdx.x - line * T;
    const int groups = (a.rows + LINES - 1) / LINES;
    const long long units = (long long)groups * (a.batch > 0 ? a.batch : 1);
    const C* twp = reinterpret_cast<const C*>(a.tw);

    // unit u -> rows [g*LINES, g*LINES + nr) of batch element b, landing dense
    // (line i at i*L) in its stage
    auto issue = [&](long long u, int stage) {
        const int b = (int)(u / groups), g = (int)(u - (long long)b * groups);
        const int r0 = g * LINES, nr = min(LINES, a.rows - r0);
        unsigned char* dst = smraw + stage * RP::STAGE;
        const C* src = reinterpret_cast<const C*>(a.in) + (long long)b * a.in_bstride + (long long)r0 * a.in_ld;
        mbar_expect_tx(&bar[stage], (unsigned)nr * L * ESZ);
        if (a.in_ld == L) {
            bulk_g2s(dst, src, (unsigned)nr * L * ESZ, &bar[stage]);
        } else {
            for (int i = 0; i < nr; i++)
                bulk_g2s(dst + (size_t)i * L * ESZ, src + (long long)i * a.in_ld, L * ESZ, &bar[stage]);
        }
    };

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (blockIdx.x < units) issue(blockIdx.x, 0);
        if (blockIdx.x + gridDim.x < units) issue(blockIdx.x + gridDim.x, 1);
    }
    double pw = 0;
    int k = 0;
    for (long long u = blockIdx.x; u < units; u += gridDim.x, k++) {
        const int stage = k & 1;
        if (!__syncthreads_and(mbar_wait(&bar[stage], (unsigned)((k >> 1) & 1)))) {
            pipe_fail(a.err, bar, k, u + gridDim.x < units);
            return;
        }
        const int b = (int)(u / groups), g = (int)(u - (long long)b * groups);
        const int r = g * LINES + line;
        const bool act = r < a.rows;
        C* stg = reinterpret_cast<C*>(smraw + stage * RP::STAGE);
        C v[E];
        const C* in = stg + line * L + tt;
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = in[fpos<R1, E, L>(s, 0)];
        if (a.red && !INV && act) {
#pragma unroll
            for (int s = 0; s < E; s++) pw += (double)v[s].x * v[s].x + (double)v[s].y * v[s].y;
        }
        fpasses<L, E, INV, 0, 1>(v, stg + line * frow_stride(L, E), tt, twp);
        if (act) {
            if (a.out_scale != 1.0) {
#pragma unroll
                for (int s = 0; s < E; s++) v[s] = cscale(v[s], (Real)a.out_scale);
            }
            if (a.red && INV) {
#pragma unroll
                for (int s = 0; s < E; s++) pw += (double)v[s].x * v[s].x + (double)v[s].y * v[s].y;
            }
            if (!INV && a.out_tiled) {
                // the tiled intermediate (FastRows::out_tiled): x = tt + s*T
                // (RO == E) lies in tile x / kTileW, lane x % kTileW
                static_assert(INV || RO == E, "tiled stores follow the natural mapping of radix E");
                const long long tstride = a.tile_len * kTileW;
                C* out = reinterpret_cast<C*>(a.out) + (long long)b * a.out_bstride + (long long)r * kTileW +
                         (long long)(tt / kTileW) * tstride + (tt % kTileW);
                const long long step = (long long)(T / kTileW) * tstride;
#pragma unroll
                for (int s = 0; s < E; s++) out[s * step] = v[s];
            } else {
                C* out = reinterpret_cast<C*>(a.out) + (long long)b * a.out_bstride + (long long)r * a.out_ld + tt;
#pragma unroll
                for (int s = 0; s < E; s++) out[fpos<RO, E, L>(s, 0)] = v[s];
            }
        }
        __syncthreads();  // every thread is done with the stage
        if (threadIdx.x == 0 && u + 2 * (long long)gridDim.x < units) {
            fence_proxy_async();
            issue(u + 2 * (long long)gridDim.x, stage);
        }
    }
    if (a.red) {
        __shared__ double rsm[32];
        for (int o = 16; o > 0; o >>= 1) pw += __shfl_down_sync(0xffffffffu, pw, o);
        if ((threadIdx.x & 31) == 0) rsm[threadIdx.x >> 5] = pw;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += rsm[w];
            a.red[(long long)blockIdx.x * a.red_stride] = t;
        }
    }
}

// ------------------------------------------------------------------- cols
template <typename Real, int L, int E, int W> struct ColPipe {
    using C = typename CT<Real>::t;
    static constexpr int T = L / E;
    static constexpr int THREADS = W * T;
    static constexpr int BR = L < 256 ? L : 256;  // rows per tensor-copy box (box extents <= 256)
    static constexpr size_t STAGE = round128((size_t)fcol_elems(L, E, W) * sizeof(C));
    static constexpr size_t SMEM = 2 * STAGE + 16;
};

template <typename Real, int L, int E, int W>
__global__ void __launch_bounds__(FColB<Real, L, E, W>::threads, FColB<Real, L, E, W>::minb)
    k_cols_pipe(const FastCols a, const __grid_constant__ CUtensorMap map) {
    using C = typename CT<Real>::t;
    using PL = FPlan<L, E>;
    using CP = ColPipe<Real, L, E, W>;
    constexpr unsigned ESZ = sizeof(C);
    constexpr int K8 = ESZ / 8;  // 8-byte map elements per complex value
    constexpr int R1 = PL::RS;
    extern __shared__ __align__(128) unsigned char smraw[];
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw + 2 * CP::STAGE);
    const int w = threadIdx.x & (W - 1);
    const int tt = threadIdx.x / W;
    const int tiles = (a.ncols + W - 1) / W;
    const long long units = (long long)tiles * (a.batch > 0 ? a.batch : 1);
    const C* twp = reinterpret_cast<const C*>(a.tw);

    auto issue = [&](long long u, int stage) {
        const int b = (int)(u / tiles), c0 = (int)(u - (long long)b * tiles) * W;
        unsigned char* dst = smraw + stage * CP::STAGE;
        mbar_expect_tx(&bar[stage], (unsigned)L * W * ESZ);
#pragma unroll 1
        for (int i = 0; i < L / CP::BR; i++)
            tma_load_3d(dst + (size_t)i * CP::BR * W * ESZ, &map, c0 * K8, i * CP::BR, b, &bar[stage]);
    };

    __shared__ double hsm[97];
    if (a.hist)
        for (int i = threadIdx.x; i < 97; i += blockDim.x) hsm[i] = 0;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (blockIdx.x < units) issue(blockIdx.x, 0);
        if (blockIdx.x + gridDim.x < units) issue(blockIdx.x + gridDim.x, 1);
    }
    double p0 = 0, l1 = 0;
    int k = 0;
    for (long long u = blockIdx.x; u < units; u += gridDim.x, k++) {
        const int stage = k & 1;
        if (!__syncthreads_and(mbar_wait(&bar[stage], (unsigned)((k >> 1) & 1)))) {
            pipe_fail(a.err, bar, k, u + gridDim.x < units);
            return;
        }
        const int b = (int)(u / tiles), c0 = (int)(u - (long long)b * tiles) * W;
        const int col = c0 + w;
        const bool act = col < a.ncols;
        C* stg = reinterpret_cast<C*>(smraw + stage * CP::STAGE);
        C v[E];
        // the stage holds the tile dense, [q][w]
#pragma unroll
        for (int s = 0; s < E; s++) v[s] = stg[fpos<R1, E, L>(s, tt) * W + w];
        fpasses<L, E, false, 0, W>(v, stg + w, tt, twp);
        bool h_done = false;
        if constexpr (sizeof(Real) == 8) {
            if (a.htab_global) {
                // complex128 H from the table (the same FP64 values the stage
                // would evaluate), at the frequencies q = tt + s*T the forward
                // transform leaves in v
                if (act) {
                    const int cabs = col <= a.ncols / 2 ? col : a.ncols - col;
                    const double2* hr = reinterpret_cast<const double2*>(a.htab) + (long long)cabs * a.htab_ld;
                    const double sg = a.conj ? -1.0 : 1.0;
#pragma unroll
                    for (int s = 0; s < E; s++) {
                        const int q = tt + s * (L / E);
                        const double2 t = __ldg(hr + (q <= L / 2 ? q : L - q));
                        v[s] = cmul(v[s], make_double2(t.x, sg * t.y));
                    }
                }
                h_done = true;
            }
        }
        if (!h_done) col_spectral_stage<Real, L, E, W>(v, stg, hsm, c0, a, h_unit(a, b), p0, l1);
        fpasses<L, E, true, 0, W>(v, stg + w, tt, twp);
        if (act) {
            constexpr int RO = PL::RS;
            C* dst = reinterpret_cast<C*>(a.data) + (long long)b * a.bstride + col + (long long)tt * a.ld;
#pragma unroll
            for (int s = 0; s < E; s++) dst[(long long)fpos<RO, E, L>(s, 0) * a.ld] = v[s];
        }
        __syncthreads();  // every thread is done with the stage
        if (threadIdx.x == 0 && u + 2 * (long long)gridDim.x < units) {
            fence_proxy_async();
            issue(u + 2 * (long long)gridDim.x, stage);
        }
    }
    col_write_red(a, blockIdx.x, p0, l1, hsm);
}

// ------------------------------------------------------------------ host
int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    static std::mutex mu;
    static std::unordered_map<int, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = n;
    return n;
}

// Resident CTAs per SM of a kernel at its shared-memory size (once per kernel).
template <typename K>
cudaError_t resident(K kernel, int threads, size_t smem, int* out) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(reinterpret_cast<const void*>(kernel));
    if (it != cache.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    if (n < 1) return cudaErrorInvalidConfiguration;
    cache[reinterpret_cast<const void*>(kernel)] = n;
    *out = n;
    return cudaSuccess;
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

bool aligned16(const void* p, long long ld_bytes, long long bstride_bytes) {
    return (reinterpret_cast<uintptr_t>(p) & 15) == 0 && ld_bytes % 16 == 0 && bstride_bytes % 16 == 0;
}

template <typename Real, int L, int E, bool INV>
cudaError_t go_rows_pipe(const FastRows& a, cudaStream_t st, int* nblocks) {
    using RP = RowPipe<Real, L, E>;
    constexpr long long esz = sizeof(typename CT<Real>::t);
    if constexpr (RP::SMEM > kMaxSmem) {
        return cudaErrorNotSupported;
    } else {
        if (a.in_c128 || a.out_c128 || !aligned16(a.in, a.in_ld * esz, a.in_bstride * esz))
            return cudaErrorNotSupported;
        int occ = 0;
        cudaError_t e = resident(k_rows_pipe<Real, L, E, INV>, RP::THREADS, RP::SMEM, &occ);
        if (e != cudaSuccess) return e;
        const long long units = (long long)((a.rows + RP::LINES - 1) / RP::LINES) * (a.batch > 0 ? a.batch : 1);
        const int grid = (int)std::min<long long>(units, (long long)occ * sm_count());
        if (nblocks) *nblocks = grid;
        k_rows_pipe<Real, L, E, INV><<<grid, RP::THREADS, RP::SMEM, st>>>(a);
        return cudaGetLastError();
    }
}

template <typename Real, int L, int E, int W>
cudaError_t go_cols_pipe_w(const FastCols& a, cudaStream_t st, int* nblocks) {
    using CP = ColPipe<Real, L, E, W>;
    constexpr int K8 = sizeof(typename CT<Real>::t) / 8;
    constexpr long long esz = sizeof(typename CT<Real>::t);
    if constexpr (W * K8 < 2 || CP::THREADS > fcol_max_threads(K8 == 2, CP::T) || CP::THREADS < 32 ||
                  CP::SMEM > kMaxSmem) {
        return cudaErrorNotSupported;
    } else {
        if (a.src) return cudaErrorNotSupported;  // the tensor map covers the in-place plane only
        const int nb = a.batch > 0 ? a.batch : 1;
        const long long bstride = nb > 1 ? a.bstride : a.ld * L;
        if (!aligned16(a.data, a.ld * esz, bstride * esz)) return cudaErrorNotSupported;
        EncodeTiled enc = encode_tiled();
        if (!enc) return cudaErrorNotSupported;
        CUtensorMap map;
        const cuuint64_t dims[3] = {(cuuint64_t)a.ncols * K8, (cuuint64_t)L, (cuuint64_t)nb};
        const cuuint64_t strides[2] = {(cuuint64_t)(a.ld * esz), (cuuint64_t)(bstride * esz)};
        const cuuint32_t box[3] = {(cuuint32_t)(W * K8), (cuuint32_t)CP::BR, 1};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, a.data, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorNotSupported;
        int occ = 0;
        cudaError_t e = resident(k_cols_pipe<Real, L, E, W>, CP::THREADS, CP::SMEM, &occ);
        if (e != cudaSuccess) return e;
        const long long units = (long long)((a.ncols + W - 1) / W) * nb;
        const int grid = (int)std::min<long long>(units, (long long)occ * sm_count());
        if (nblocks) *nblocks = grid;
        k_cols_pipe<Real, L, E, W><<<grid, CP::THREADS, CP::SMEM, st>>>(a, map);
        return cudaGetLastError();
    }
}

template <typename Real, int L, int E>
cudaError_t go_cols_pipe(const FastCols& a, cudaStream_t st, int* nblocks) {
    switch (fast_col_width(sizeof(Real) == 8, L, E, a.W)) {
    case 1: return go_cols_pipe_w<Real, L, E, 1>(a, st, nblocks);
    case 2: return go_cols_pipe_w<Real, L, E, 2>(a, st, nblocks);
    case 4: return go_cols_pipe_w<Real, L, E, 4>(a, st, nblocks);
    case 8: return go_cols_pipe_w<Real, L, E, 8>(a, st, nblocks);
    case 16: return go_cols_pipe_w<Real, L, E, 16>(a, st, nblocks);
    default: return cudaErrorNotSupported;
    }
}

}  // namespace

#define WOS_PIPE_L(X) X(256) X(512) X(1024) X(2048) X(4096) X(8192)

cudaError_t pipe_rows(int fp64, int L, int E, bool inv, const FastRows& a, cudaStream_t st, int* nblocks) {
#define CASE_R(LL)                                                                                \
    case LL:                                                                                      \
        if (fp64) {                                                                               \
            if constexpr (LL <= 4096) {                                                           \
                if (E == 8) return inv ? go_rows_pipe<double, LL, 8, true>(a, st, nblocks)        \
                                       : go_rows_pipe<double, LL, 8, false>(a, st, nblocks);      \
            } else {                                                                              \
                if (E == 16) return inv ? go_rows_pipe<double, LL, 16, true>(a, st, nblocks)      \
                                        : go_rows_pipe<double, LL, 16, false>(a, st, nblocks);    \
            }                                                                                     \
        } else {                                                                                  \
            if constexpr (LL <= 4096) {                                                           \
                if (E == 8) return inv ? go_rows_pipe<float, LL, 8, true>(a, st, nblocks)         \
                                       : go_rows_pipe<float, LL, 8, false>(a, st, nblocks);       \
            }                                                                                     \
            if (E == 16) return inv ? go_rows_pipe<float, LL, 16, true>(a, st, nblocks)           \
                                    : go_rows_pipe<float, LL, 16, false>(a, st, nblocks);         \
        }                                                                                         \
        break;
    switch (L) { WOS_PIPE_L(CASE_R) }
#undef CASE_R
    return cudaErrorNotSupported;
}

cudaError_t pipe_cols(int fp64, int L, int E, const FastCols& a, cudaStream_t st, int* nblocks) {
#define CASE_C(LL)                                                                \
    case LL:                                                                      \
        if (fp64) {                                                               \
            if constexpr (LL <= 4096) {                                           \
                if (E == 8) return go_cols_pipe<double, LL, 8>(a, st, nblocks);   \
            } else {                                                              \
                if (E == 16) return go_cols_pipe<double, LL, 16>(a, st, nblocks); \
            }                                                                     \
        } else {                                                                  \
            if constexpr (LL <= 4096) {                                           \
                if (E == 8) return go_cols_pipe<float, LL, 8>(a, st, nblocks);    \
            }                                                                     \
            if (E == 16) return go_cols_pipe<float, LL, 16>(a, st, nblocks);      \
        }                                                                         \
        break;
    switch (L) { WOS_PIPE_L(CASE_C) }
#undef CASE_C
    return cudaErrorNotSupported;
}

}  // namespace wos

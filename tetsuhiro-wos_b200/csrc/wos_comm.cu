// wos_comm.cu -- batches sharded over GPUs (no counterpart in the reference,
// whose polychromatic, coherence and volume loops run their units in
// sequence: optics/polychromatic.go:29-42, optics/coherence.go:110-115,
// optics/volume.go:10-16).  One process (or thread) per GPU, each with its own
// context; the contexts join one NCCL communicator.  Every rank passes the
// whole unit list, runs its contiguous share on its own GPU and takes part in
// the one exchange step: an in-place all-reduce of the FP64 intensity map
// (wavelengths, modes) or a broadcast of each rank's planes (volume), on the
// context stream, between device buffers.  NCCL is loaded with dlopen at the
// first wos_comm_init, so the library does not depend on it otherwise.
#include <dlfcn.h>
#include <nccl.h>

#include "wos_api_internal.cuh"

namespace wapi {

// The NCCL entry points the sharded batches use.
struct Nccl {
    bool ok = false;
    std::string why;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    ncclResult_t (*broadcast)(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

const Nccl& nccl() {
    static Nccl n;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            n.why = std::string("cannot load libnccl.so.2: ") + dlerror();
            return;
        }
        auto sym = [&](const char* s) { return dlsym(h, s); };
        n.get_unique_id = reinterpret_cast<decltype(n.get_unique_id)>(sym("ncclGetUniqueId"));
        n.comm_init_rank = reinterpret_cast<decltype(n.comm_init_rank)>(sym("ncclCommInitRank"));
        n.comm_destroy = reinterpret_cast<decltype(n.comm_destroy)>(sym("ncclCommDestroy"));
        n.all_reduce = reinterpret_cast<decltype(n.all_reduce)>(sym("ncclAllReduce"));
        n.broadcast = reinterpret_cast<decltype(n.broadcast)>(sym("ncclBroadcast"));
        n.group_start = reinterpret_cast<decltype(n.group_start)>(sym("ncclGroupStart"));
        n.group_end = reinterpret_cast<decltype(n.group_end)>(sym("ncclGroupEnd"));
        n.error_string = reinterpret_cast<decltype(n.error_string)>(sym("ncclGetErrorString"));
        n.ok = n.get_unique_id && n.comm_init_rank && n.comm_destroy && n.all_reduce && n.broadcast &&
               n.group_start && n.group_end && n.error_string;
        if (!n.ok) n.why = "libnccl.so.2 lacks an entry point the sharded batches use";
    });
    return n;
}

int nccl_fail(ncclResult_t r, const char* what) {
    return fail(WOS_CUDA_ERROR, std::string(what) + ": " + nccl().error_string(r));
}

void comm_release(wos_ctx c) {
    if (c && c->comm && nccl().ok) nccl().comm_destroy(static_cast<ncclComm_t>(c->comm));
    if (c) {
        c->comm = nullptr;
        c->comm_size = 1;
        c->comm_rank = 0;
    }
}

// Contiguous range of rank r among n ranks over `units` units: the first
// units % n ranks take one unit more.
void shard(int units, int n, int r, int* b, int* e) {
    const int q = units / n, rem = units % n;
    *b = r * q + std::min(r, rem);
    *e = *b + q + (r < rem ? 1 : 0);
}

int need_comm(wos_ctx c) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    if (!c->comm) return fail(WOS_NOT_INITIALISED, "sharded batch: wos_comm_init has not been called on this context");
    return WOS_OK;
}

}  // namespace wapi

extern "C" {

int wos_shard_range(int units, int nranks, int rank, int* begin, int* end) {
    if (units < 0 || nranks < 1 || rank < 0 || rank >= nranks || !begin || !end)
        return fail(WOS_INVALID_ARG, "shard range: need units >= 0 and 0 <= rank < nranks");
    shard(units, nranks, rank, begin, end);
    return WOS_OK;
}

int wos_comm_unique_id(unsigned char* id) {
    if (!id) return fail(WOS_INVALID_ARG, "null id");
    const Nccl& n = nccl();
    if (!n.ok) return fail(WOS_NOT_INITIALISED, n.why);
    static_assert(sizeof(ncclUniqueId) == WOS_COMM_ID_BYTES, "NCCL unique id size");
    ncclUniqueId u;
    const ncclResult_t r = n.get_unique_id(&u);
    if (r != ncclSuccess) return nccl_fail(r, "ncclGetUniqueId");
    std::memcpy(id, &u, sizeof u);
    return WOS_OK;
}

int wos_comm_init(wos_ctx c, int nranks, int rank, const unsigned char* id) {
    if (!c || !id || nranks < 1 || rank < 0 || rank >= nranks)
        return fail(WOS_INVALID_ARG, "comm init: need 0 <= rank < nranks and an id");
    const Nccl& n = nccl();
    if (!n.ok) return fail(WOS_NOT_INITIALISED, n.why);
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    comm_release(c);
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof u);
    ncclComm_t comm = nullptr;
    const ncclResult_t r = n.comm_init_rank(&comm, nranks, u, rank);
    if (r != ncclSuccess) return nccl_fail(r, "ncclCommInitRank");
    c->comm = comm;
    c->comm_size = nranks;
    c->comm_rank = rank;
    return WOS_OK;
}

int wos_comm_destroy(wos_ctx c) {
    if (!c) return fail(WOS_INVALID_ARG, "null ctx");
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    comm_release(c);
    return WOS_OK;
}

int wos_polychromatic_sharded_dev(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* field, double z,
                                  const double* wavelengths, const double* weights, int nsamples,
                                  const wos_context* base, double* out) {
    TRY(need_comm(c));
    if (!out || nsamples <= 0 || !wavelengths || !weights) return fail(WOS_INVALID_ARG, "null argument");
    int b, e;
    shard(nsamples, c->comm_size, c->comm_rank, &b, &e);
    if (e > b) {
        TRY(wos_polychromatic_dev(c, ny, nx, dx, ncomp, field, z, wavelengths + b, weights + b, e - b, base, out));
    } else {
        std::lock_guard<std::mutex> lk(c->mu);
        TRY(set_device(c));
        CK(cudaMemsetAsync(out, 0, sizeof(double) * ny * nx, c->st));
    }
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const ncclResult_t r = nccl().all_reduce(out, out, (size_t)ny * nx, ncclFloat64, ncclSum,
                                             static_cast<ncclComm_t>(c->comm), c->st);
    return r == ncclSuccess ? WOS_OK : nccl_fail(r, "ncclAllReduce");
}

int wos_partially_coherent_sharded_dev(wos_ctx c, int n, double dx, double width, double coherence, int m,
                                       const void* noise, double z, const wos_context* cc, double* out) {
    TRY(need_comm(c));
    if (m <= 0) m = 1;
    int b, e;
    shard(m, c->comm_size, c->comm_rank, &b, &e);
    TRY(schell_dev_range(c, n, dx, width, coherence, m, b, e - b, noise, z, cc, out));
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const ncclResult_t r = nccl().all_reduce(out, out, (size_t)n * n, ncclFloat64, ncclSum,
                                             static_cast<ncclComm_t>(c->comm), c->st);
    return r == ncclSuccess ? WOS_OK : nccl_fail(r, "ncclAllReduce");
}

int wos_volume_sharded_dev(wos_ctx c, int ny, int nx, double dx, int ncomp, const void* field, const double* zs,
                           int nz, const wos_context* cc, void* out) {
    TRY(need_comm(c));
    if (nz < 0 || (nz > 0 && (!zs || !out))) return fail(WOS_INVALID_ARG, "null argument");
    if (nz == 0) return WOS_OK;
    const size_t plane = (size_t)ny * nx * ncomp * c->csz();
    int b, e;
    shard(nz, c->comm_size, c->comm_rank, &b, &e);
    if (e > b) TRY(wos_volume_dev(c, ny, nx, dx, ncomp, field, zs + b, e - b, cc, static_cast<char*>(out) + b * plane));
    std::lock_guard<std::mutex> lk(c->mu);
    TRY(set_device(c));
    const Nccl& nc = nccl();
    ncclResult_t r = nc.group_start();
    for (int q = 0; q < c->comm_size && r == ncclSuccess; q++) {
        int qb, qe;
        shard(nz, c->comm_size, q, &qb, &qe);
        if (qe > qb) {
            char* p = static_cast<char*>(out) + qb * plane;
            r = nc.broadcast(p, p, (qe - qb) * plane, ncclUint8, q, static_cast<ncclComm_t>(c->comm), c->st);
        }
    }
    const ncclResult_t r2 = nc.group_end();
    if (r != ncclSuccess) return nccl_fail(r, "ncclBroadcast");
    return r2 == ncclSuccess ? WOS_OK : nccl_fail(r2, "ncclGroupEnd");
}

}  // extern "C"

// wos_api_internal.cuh -- types and helpers shared by the host-side
// translation units of the C ABI: wos_api.cu (contexts, axes, reductions, the
// three-sweep propagator and the core entry points), wos_bpm.cu (split-step
// BPM and the diffractive stack), wos_batch.cu (polychromatic, volume and
// Gaussian-Schell batches), wos_design.cu (inverse design) and
// wos_field_ops.cu (thin elements, field operations, anisotropic media, plane
// views, the element train).  Host code only, not part of the public ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wos_gpu.h"
#include "wos_fast.cuh"
#include "wos_pipe.cuh"
#include "wos_fft.cuh"
#include "wos_kernels.cuh"

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? WOS_OOM : WOS_CUDA_ERROR,           \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                 \
        }                                                                                     \
    } while (0)

#define TRY(x)                  \
    do {                        \
        int rc_ = (x);          \
        if (rc_ != WOS_OK) return rc_; \
    } while (0)

namespace wapi {

using namespace wos;

// thread-local message of the last failed call (wos_last_error)
extern thread_local std::string g_err;
int fail(int st, const std::string& msg);

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
};
// Everything needed to transform a line of logical length n in one precision.
struct Axis {
    int n = 0, L = 0, blue = 0;
    void* tw = nullptr;
    void* chirp = nullptr;
    void* bf = nullptr;
    void* bi = nullptr;
    void* ftw[2] = {nullptr, nullptr};  // per-pass twiddles of the specialised sweeps (E = 8, 16)
    void* ftw_lo[2] = {nullptr, nullptr};  // their complex64 residuals (compensated split-step sweeps)
    void* ptw = nullptr;                // W_L^n, n < L/2: split column tiles
};
constexpr int kMaxL32 = 8192;  // largest line held on chip (threads x elements)
constexpr int kMaxL64 = 8192;
// Launch configuration of the specialised sweeps for one grid: elements per
// thread of the row and column passes, columns per CTA.
struct Tune {
    int rowE, colE, colW;
};

int ensure(DevBuf& b, size_t bytes);
inline bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
int next_pow2(int n);
inline long long tune_key(int fp64, int ny, int nx) { return ((long long)fp64 << 62) | ((long long)ny << 31) | nx; }

}  // namespace wapi

using wapi::Axis;
using wapi::DevBuf;
using wapi::Tune;

struct wos_ctx_s {
    int device = 0;
    int fp64 = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    std::mutex mu;
    std::map<int, Axis> axes[2];  // [fp64][n]
    DevBuf stage, scratch, scratch2, scratch3, red, redout, tmp, maps, params, vol, accum, aux;
    double* hred = nullptr;  // pinned mirror of redout
    size_t hred_n = 0;
    int colw = 0;
    bool no_fast = false;               // force the general sweeps (tests compare both)
    int sweep_mode = 1;                 // wos_ctx_set_fast_path: 1, 2 or 3 (0 is no_fast)
    int col_pair = 0;                   // column tiles split over two-CTA clusters where supported
    DevBuf bpm_tab;                     // split-step tables (core profile, border absorption) on the device
    std::vector<double> bpm_tab_host;   // ... and their host copy, to skip identical uploads
    int tiled = 0;                      // three-sweep ASM through the tiled intermediate (FastRows::out_tiled)
    int bpm_comp = 1;                   // complex64 split-step slices on the compensated transforms (WOS_BPM_COMP=0: off)
    // transfer-function tables of the complex64 column sweep (FastCols::htab),
    // keyed by grid and H parameters; a few slots, reused round robin (a
    // slot is rebuilt on the context stream, after the work that read it)
    struct HTab {
        bool valid = false;
        bool frozen = false;  // read by a captured graph: never rebuilt
        int L = 0, ncols = 0;
        double key[9] = {};
        DevBuf buf;
    };
    static constexpr int kHTabs = 4;    // tables kept round robin (more while graphs pin some)
    std::vector<HTab> htab = std::vector<HTab>(kHTabs);
    int htab_next = 0;
    int htab_on = 1;                    // WOS_HTAB=0: evaluate H in the split-step sweeps
    int htab_reg = 1;                   // WOS_HTAB_REG=0: evaluate H in the plain ASM column sweep
    int out_stream = 1;                 // WOS_OUT_STREAM=0: the last row sweep stores without evict-first hints
    // device copies of the small parameter lists (wavelengths, distances,
    // weights) of the device-resident batches, keyed by content and reused
    // round robin: a repeated call copies nothing from the host
    struct ParamSlot {
        std::vector<double> host;
        bool frozen = false;  // read by a captured graph: never rewritten
        DevBuf buf;
    };
    static constexpr int kParamSlots = 8;
    std::vector<ParamSlot> pslot = std::vector<ParamSlot>(kParamSlots);
    int pslot_next = 0;
    bool capturing = false;             // between wos_graph_capture_begin and _end
    wos_ctx cap_owner = nullptr;        // the capturing context this one is a branch of (wos_graph_capture_fork)
    std::vector<wos_ctx> cap_open;      // open branches of this context's capture
    cudaEvent_t cap_ev = nullptr;       // fork / join point of a capture branch
    // communicator of the sharded batches (wos_comm_init): NCCL's ncclComm_t
    void* comm = nullptr;
    int comm_size = 1, comm_rank = 0;
    unsigned* err_dev = nullptr;        // error word of the pipelined kernels (device)
    unsigned* err_host = nullptr;       // pinned mirror, read where the host synchronises
    // streams for independent fields of a batch (wos_propagate_batch_dev),
    // forked from and joined back into st
    static constexpr int kMaxAux = 4;
    cudaStream_t side[kMaxAux] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kMaxAux] = {};
    int naux = 0;
    DevBuf tsc[kMaxAux + 1];            // tiled intermediates: [0] context stream, [1 + k] side stream k
    int cur_slot = 0;                   // which of them the current stream uses
    // copy pipeline of wos_propagate_batch: host-to-device and device-to-host
    // streams, staging slots and their events
    static constexpr int kSlots = 3;
    cudaStream_t h2d = nullptr, d2h = nullptr;
    DevBuf slot[kSlots];
    // page-locked host staging of the batch slots for pageable fields, and
    // the host threads that convert into and out of it (wos_host.cu)
    void* hst[kSlots] = {};
    size_t hst_n[kSlots] = {};
    void* host_pool = nullptr;
    cudaEvent_t in_ev[kSlots] = {}, done_ev[kSlots] = {}, free_ev[kSlots] = {};
    bool pipe_made = false;
    std::map<long long, Tune> tune;     // autotuned launch configurations
    size_t csz() const { return fp64 ? 16 : 8; }
    // per-launch CUDA-event profile (wos_ctx_set_profiling): a ring of event
    // pairs; a slot's elapsed time is folded into its kind when it is reused
    // or read, by which time the pair has long completed.
    static constexpr int kRing = 1024;
    bool prof_on = false, prof_made = false;
    cudaEvent_t ev0[kRing], ev1[kRing];
    int ev_kind[kRing];
    bool ev_used[kRing];
    int ev_head = 0;
    double prof_ms[8] = {0};
    long long prof_n[8] = {0};
    long long launches = 0;
};

namespace wapi {

// ---- reductions: partial region r, finished into redout[r]
constexpr int kRegions = 8;

struct Red {
    wos_ctx c;
    size_t per_region = 0;  // doubles per region
};

// ---- evanescent policy (optics/propagate.go:186-199)
struct Policy {
    int zero = 0, reg = 0;
    double alpha = 0, limit = 0;
};

// ---------------------------------------------------------------- pipeline
struct Prop {
    int ny, nx;
    double dx;
    int ncomp;
    const void* in;
    int in_c128;
    void* out;
    int out_c128;
    double z;
    int method;
    wos_context c;
    wos_diag* diag;
};

// The three-sweep propagator shared by asm / asm_shift / asm_pad /
// asm_shift_pad / fresnel_tf / fresnel_ir:
//   rows:  in (ny x nx) -> scratch rows, forward transform over mx points
//   cols:  forward over my points, H, inverse, keep rows [offy, offy+ny)
//   rows:  inverse over mx points, keep columns [offx, offx+nx) -> out
// pad = 1 doubles both axes (zero-padded linear convolution,
// optics/propagate.go:346-387); the padding is folded into addressing.
struct Sweep3 {
    int pad = 0;
    int shift = 0;
    double fxc = 0, fyc = 0;
    HArgs h{};
    bool red_pin = false, red_pout = false, hist = false;
    bool red_loss = false;  // spectral power-loss sums of the H_ASM step (region 1)
    bool fast = false;      // set when the specialised sweeps ran (no crop sums)
};

int set_device(wos_ctx c);
int check_err_word(wos_ctx c);
void prof_fold(wos_ctx c, int slot);
cudaError_t prof_rows(wos_ctx c, int fp64, const RowArgs& a);
cudaError_t prof_cols(wos_ctx c, int fp64, const ColArgs& a);
bool mixed_radix_ok(int n);
int build_axis(wos_ctx c, int n, int fp64, Axis& ax);
int get_axis(wos_ctx c, int n, int fp64, Axis** out);
void fill_axis(RowArgs& r, const Axis* a);
void fill_axis(ColArgs& r, const Axis* a);
RowArgs row_defaults(int ny, int nx, double dx);
ColArgs col_defaults(wos_ctx c, double dx);
int auto_colw_p(wos_ctx c, int fp64, int L);
int auto_colw(wos_ctx c, int L);
int red_prepare(wos_ctx c, size_t max_blocks);
double* red_region(wos_ctx c, int r);
size_t red_region_blocks(wos_ctx c);
double* redout_region(wos_ctx c, int r);
size_t row_blocks(int fp64, int L, int rows, int batch);
size_t col_blocks(int fp64, int L, int W, int ncols, int batch);
Policy ev_policy(const wos_context& c, double z);
void warn_add(wos_diag* d, int bit, double value);
void asm_warn(wos_diag* d, double z, double pin, double pout, const Policy& p);
double spectral_radius_from_hist(const double* hist, double dx, double frac);
bool wrap_needed(const wos_context& c, int ny, int nx, double dx, double z);
void wrap_finish(wos_diag* d, const wos_context& c, int ny, int nx, double dx, double z, const double* hist);
int fetch_red(wos_ctx c, int nreg);
HArgs asm_h(wos_ctx c, const wos_context& cc, double z, const Policy& p, double dx, int lfx, int lfy);
int spectrum_stats(wos_ctx c, const Prop& p, void* dst, bool centroid, bool hist, int shift, double fxc,
                   double fyc, int region, int* blocks_out);
int env_int(const char* name, int def);
Tune get_tune(wos_ctx c, int ny, int nx);
size_t fast_row_blocks(int L, int E, int rows, int batch);
size_t fast_col_blocks(int fp64, int L, int E, int W, int ncols, int batch);
int fast_tw(wos_ctx c, Axis* a, int E, const void** out);
int fast_tw_lo(wos_ctx c, Axis* a, int E, const void** out);
int attach_htab(wos_ctx c, FastCols& k, int L, int E);
int attach_htab_global(wos_ctx c, FastCols& k, int L);
int attach_htab64(wos_ctx c, FastCols& k, int L);
cudaError_t sweep_rows(wos_ctx c, int L, int E, bool inv, const FastRows& a, int* nb);
bool pair_tables(wos_ctx c, int L, int E, const void** twh, const void** twp);
bool pair_eligible(wos_ctx c, int L, int E, const FastCols& a);
cudaError_t sweep_cols(wos_ctx c, int L, int E, const FastCols& a, int* nb);
void fill_asm_h(FastCols& k, const HArgs& h);
bool asm_tiled(wos_ctx c, int ny, int nx, const Tune& t);
int try_fast_sweep3(wos_ctx c, const Prop& p, Sweep3& s);
int run_sweep3(wos_ctx c, const Prop& p, Sweep3& s);
int copy_field(wos_ctx c, const Prop& p);
int run_propagate(wos_ctx c, const Prop& p0);
int stage_in(wos_ctx c, const wos_field* f, int ncomp);
int stage_out(wos_ctx c, wos_field* f, int ncomp);
int check_field(const wos_field* f);
wos_context default_context();
int fft2d_impl(wos_ctx c, int fp64, int ny, int nx, int batch, void* a, int inverse);
int plane_view_dev(wos_ctx c, int fp64, const void* ex, const void* ey, const void* ez, int pol, long long np,
                   int view, double mask_cut, void* out);
void diag_merge(wos_diag* into, const wos_diag& d);

// Kinds: 0..3 row modes (fwd, inv, inv.screen.fwd, inv.accumulate), 4..7 column
// modes (fused, fraunhofer, reduce, fft).
template <typename F>
cudaError_t timed_launch(wos_ctx c, int kind, F&& launch) {
    c->launches++;
    if (!c->prof_on) return launch();
    const int slot = c->ev_head;
    prof_fold(c, slot);
    cudaEventRecord(c->ev0[slot], c->st);
    cudaError_t e = launch();
    cudaEventRecord(c->ev1[slot], c->st);
    c->ev_kind[slot] = kind;
    c->ev_used[slot] = true;
    c->ev_head = (slot + 1) % wos_ctx_s::kRing;
    return e;
}

// defined in wos_batch.cu
int fft2d_fp64(wos_ctx c, int n, int batch, double2* a, int inverse);
int upload_params(wos_ctx c, const std::vector<double>& a, const std::vector<double>& b2,
                  const std::vector<double>& c3, double** pa, double** pb, double** pc);
int schell_dev_range(wos_ctx c, int n, double dx, double width, double coherence, int m, int m0, int count,
                     const void* noise, double z, const wos_context* cci, double* out);
// defined in wos_comm.cu: releases the context's communicator, if any
void comm_release(wos_ctx c);
// defined in wos_host.cu: staging of pageable host fields
bool host_pageable(const void* p);
int host_stage(wos_ctx c, int slot, size_t bytes);
void host_convert(wos_ctx c, wos_field& f, void* dst, bool to_host);
void host_release(wos_ctx c);
// defined in wos_field_ops.cu
int element_begin(wos_ctx c, wos_field* f);
double2* stage_ex(wos_ctx c);
double2* stage_ey(wos_ctx c, const wos_field* f);

}  // namespace wapi

using namespace wapi;

// pd_env_impl.h -- host-side environment object and helpers shared by the
// host translation units (pd_env.cu, pd_solver.cu, pd_contact.cu,
// pd_fast.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "pd_internal.h"

namespace pd {
pd_status fail(pd_status s, const char *fmt, ...);
pd_status cuda_fail(cudaError_t e, const char *what, const char *file, int line);
}  // namespace pd

#define PD_TRY(expr)                       \
    do {                                   \
        pd_status s_ = (expr);             \
        if (s_ != PD_OK) return s_;        \
    } while (0)

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return pd::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

namespace pd {

// Owning device buffer.
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DBuf &operator=(DBuf &&o) noexcept {
        reset();
        p = o.p;
        n = o.n;
        o.p = nullptr;
        o.n = 0;
        return *this;
    }
    ~DBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    pd_status alloc(size_t count) {
        reset();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return fail(PD_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T),
                        cudaGetErrorString(e));
        }
        n = count;
        return PD_OK;
    }
};

// Device buffer allocated and freed in stream order (cudaMallocAsync /
// cudaFreeAsync on one stream): for temporaries of a call that may run
// while other streams of the device are busy (a server admitting a job),
// since cudaMalloc / cudaFree wait for the whole device.
template <class T>
struct SBuf {
    T *p = nullptr;
    cudaStream_t st = nullptr;
    SBuf() = default;
    SBuf(const SBuf &) = delete;
    SBuf &operator=(const SBuf &) = delete;
    ~SBuf() { reset(); }
    void reset() {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
    }
    pd_status alloc(size_t count, cudaStream_t stream) {
        reset();
        st = stream;
        if (count == 0) count = 1;
        cudaError_t e = cudaMallocAsync((void **)&p, count * sizeof(T), stream);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return fail(PD_ERR_OOM, "cudaMallocAsync of %zu bytes failed: %s", count * sizeof(T),
                        cudaGetErrorString(e));
        }
        return PD_OK;
    }
};

struct HostBlock {
    int64_t n = 0;
    int32_t kind = 0, nt = 1;
    int64_t type_start = 1;
    double horizon = 0, particle_size = 0;
    int64_t max_neigh = 100;
    std::vector<double> x, y, v, vol;
    std::vector<int64_t> type;
    std::vector<double> c, K, G, cs, dens, psi;
    bool host_family = false;
    int64_t rows = 0;  // reference family rows M'
    std::vector<int64_t> family;
    std::vector<uint8_t> intact;
    int64_t first_env = 0, first_int = 0;
    int64_t cell_part_off = 0;
};

struct HostBC {
    int32_t kind = 0, dims = 7, onlyatstart = 0;
    double rate[3] = {0, 0, 0};
    double freq = 0;
    int64_t applyafter = 0;
    int dir = 1;
    std::vector<int64_t> env_idx;
    double scale[3] = {0, 0, 0}, fix[3] = {0, 0, 0};  // DeltaScale / ScaleFixWait
    int64_t wait = 1;                                   // ScaleFixWait
    std::vector<int64_t> scale_idx;                     // ScaleFixWait scalebool
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};        // Container
    int32_t has_limits = 0;
    // check! (ScaleFixWaitBC.jl:63) at this time_step
    bool scales_at(int64_t ts) const { return kind == PD_BC_SCALE_FIX_WAIT && wait != 0 && ts % wait == 0; }
};

struct DevBC {
    DBuf<int32_t> idx;
    DBuf<double4> last;
    int64_t n = 0;
    DBuf<int32_t> sidx;
    int64_t sn = 0;
};

struct HostContact {
    int32_t kind = 0;
    int64_t b1 = 0, b2 = 0;
    double exponent = 1, stiffness = 0, equi_dist = 0, distance = 0;
    int64_t max_neighs = 50;
    int64_t rows = 0;  // neighbour rows of the reference layout
};

// Device state of one contact model.
struct DevContact {
    int64_t n1 = 0, n2 = 0;       // particles of pair[1] / pair[2] (block sizes)
    int64_t first1 = 0, first2 = 0;  // internal first index of the two blocks
    int64_t rows = 0;
    int64_t nbrows = 0;     // rows stored in nb (1 for the reference contact-11 search)
    DBuf<int32_t> nb;       // nbrows x n1 (row r of particle i at r*n1+i), internal indices, -1 pad
    DBuf<int32_t> rev_off;  // n2+1 reverse-list offsets
    DBuf<int32_t> rev;      // reverse lists (internal indices of set-1 particles, ascending)
    DBuf<int32_t> rev_cnt;  // n2 scratch
    int64_t rev_cap = 0;
    bool has_neighs = false;
    // particles with contact work, built with the neighbour lists: set-1
    // particles with a neighbour (self contact: or a reverse entry), set-2
    // particles with a reverse entry (two-block contact); -1 = not built
    DBuf<int32_t> act1, act2, act_n;
    int64_t nact1 = -1, nact2 = -1;
    // neighbour-search scratch, kept between updates (grown, never shrunk)
    DBuf<int32_t> s_cell_of, s_ccount, s_cstart, s_cursor, s_clist, s_tmp, s_c1cnt, s_c1off, s_cand, s_rtmp;
};

// Reallocates b only when it holds fewer than n elements.
template <class T>
inline pd_status grow(DBuf<T> &b, int64_t n) {
    if ((int64_t)b.n >= n && b.p) return PD_OK;
    return b.alloc((size_t)std::max<int64_t>(n, 1));
}

}  // namespace pd

struct pd_env {
    int device = 0, precision = 0;
    int sm_count = 0;  // multiprocessors of the device (read once)
    double dt = 0;
    int64_t ts = 0;
    cudaStream_t st = nullptr;
    bool finalized = false;

    std::vector<pd::HostBlock> hb;
    std::vector<pd::HostBC> hbc;
    std::vector<pd::HostContact> hc;
    int64_t N_env = 0;  // particles in environment order
    int64_t N = 0;      // internal (padded) particles
    std::vector<int64_t> map_h;
    std::vector<pd::DevBlock> blocks_h;
    std::vector<int> deformed_h;
    // runtime bond layout: S+1 slice descriptors (the last one only marks
    // the end of nbr[] and of the bit arrays)
    std::vector<pd::SliceInfo> sinfo_h;
    std::vector<int32_t> cnt_h;
    int64_t nnz = 0;       // bond slots (bits per bit array)
    int64_t walked = 0;    // slots the walks visit: per slice 32 x its largest slot count
    int64_t nbr_len = 0;   // entries of nbr[]
    int64_t stencil_slices = 0;
    // Record staging plans of stencil slices (throughput path): the
    // 32-record windows [p0 + o, p0 + o + 32) of a slice's offsets o merged
    // into ranges of consecutive records.  splan_off[s] = start of slice s's
    // plan in splan (-1: not staged); a plan is {ranges, records, then
    // (first record, count) per range}.  spos[i] = staged position of lane
    // 0's record of the stencil slot stored at nbr[i].
    int64_t splan_slices = 0, splan_max = 0;

    pd::DBuf<int64_t> map;
    pd::DBuf<double4> x4, y, v, f, p;
    pd::DBuf<double> mass, dens, tdens;
    pd::DBuf<int32_t> tinfo, cnt, intact0, deformed;
    pd::DBuf<pd::SliceInfo> sinfo;
    pd::DBuf<int32_t> nbr;
    pd::DBuf<int32_t> splan_off, splan, spos;
    pd::DBuf<uint32_t> words[2], words0, fam;
    // elasto-plastic state: td_norm2 per particle, edp per bond slot
    // (double-buffered by force evaluation, edp[ecur] current)
    pd::DBuf<double> td2, edp[2];
    int ecur = 0;
    int cur = 0;
    pd::DBuf<double2> mth;
    pd::DBuf<pd::DevBlock> blocks_d;
    pd::DBuf<pd::PairParam> pairs;
    pd::DBuf<double> partials, out3, stage;
    pd::DBuf<pd::GateItem> gate_items;  // undeformed blocks for the gate kernels
    pd::DBuf<double> gate_part;
    std::vector<pd::GateItem> gate_items_h;
    std::vector<int> deformed0;  // gate flags right after finalize
    pd::DBuf<int32_t> flag;
    std::vector<pd::DevBC> bcs;
    std::vector<pd::DevContact> contacts;
    int64_t contact_epoch = 0;  // incremented whenever the contact lists change

    // scratch for the device-pointer entry point and solvers
    pd::DBuf<double4> tmp_y, tmp_f, opt;
    pd::DBuf<double> scr_d;    // per-particle result scratch (damage), kept between calls
    pd::DBuf<int32_t> scr_i;   // per-particle count scratch (bond counts)
    pd::DBuf<int32_t> free_mask;
    pd::DBuf<double> red;

    // optional CUDA-event timing of the bond-force kernel launches
    bool prof = false;
    std::vector<cudaEvent_t> prof_ev;  // start/stop pairs
    std::vector<int32_t> prof_w;       // steps covered by each pair
    size_t prof_used = 0;
    double prof_ms = 0.0;
    int64_t prof_launches = 0;

    // output staging (pd_env_stage_state): device pack buffers, pinned host
    // copies, completion events, one copy stream
    struct StageSlot {
        pd::DBuf<double> dev;
        double *host = nullptr;
        cudaEvent_t packed = nullptr, done = nullptr;
        bool pending = false;
        int64_t ts = 0;
    } slots[2];
    cudaStream_t copy_st = nullptr;

    // fast (FP64 / FP32C) state; see pd_fast.cu
    bool fast_valid = false;
    void *fast = nullptr;
    int shape = 0;  // fixed kernel shape 10 * warps_per_slice + unroll, 0 = autotune
    bool gate_hold = false;  // pd_env_set_deformed(..., hold): the library does not evaluate the gate
    int staging = 0;  // record staging: 0 = none, 1 = staged shapes, 2 = the autotuner decides

    pd::Geo geo() const;
    void release_device();
};

namespace pd {
// Bracket the bond kernels of one step, or one graph replay of `steps`
// steps, with timing events (no-op unless profiling is enabled on the
// environment).
void prof_begin(pd_env *env, cudaStream_t st);
void prof_end(pd_env *env, cudaStream_t st, int32_t steps = 1);
pd_status contacts_finalize(pd_env *env);
pd_status contacts_update_neighs(pd_env *env, int64_t max_part);
pd_status contacts_force(pd_env *env);
// Bring the FP64 arrays up to date with the throughput-mode state; with
// invalidate the throughput state is rebuilt from them on its next use
// (for callers that modify y, v, f or the dilatation).
pd_status sync_state_to_fp64(pd_env *env, bool invalidate = true);
void fast_release(pd_env *env);
pd_status fast_vv_steps(pd_env *env, int64_t nsteps);
pd_status fast_vv_enqueue(pd_env *env, int64_t nsteps);
// Serving batches: whether an environment may be advanced in shared
// launches with others, and nsteps of a batch of them (one precision) on
// stream st.
bool fast_batchable(pd_env *env);
pd_status fast_batch_steps(pd_env *const *envs, int n_envs, int64_t nsteps, cudaStream_t st);
pd_status fast_land_flags(pd_env *env);
// Device bytes an assembled environment will hold once finalized (upper
// estimate from particle counts and family rows; for admission control).
int64_t footprint_estimate(const pd_env *env);
pd_status fast_update_acc(pd_env *env);
pd_status update_acc_serial(pd_env *env);
}  // namespace pd

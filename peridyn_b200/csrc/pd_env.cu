// pd_env.cu -- the C ABI (include/peridyn_b200.h): environment assembly,
// device memory ownership, family construction and the solver sequencing of
// src/solvers/*.jl on one CUDA stream.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <iterator>
#include <thread>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "pd_env_impl.h"
#include "pd_stage_plan.h"

using namespace pd;

#include <atomic>

namespace {
thread_local std::string g_err;
std::atomic<int64_t> g_launches{0};
}  // namespace

namespace pd {

pd_status fail(pd_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void add_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

void prof_begin(pd_env *env, cudaStream_t st) {
    if (!env->prof) return;
    if (env->prof_used + 2 > env->prof_ev.size()) {
        if (env->prof_ev.size() >= 16384) return;
        for (int k = 0; k < 256; ++k) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return;
            env->prof_ev.push_back(e);
        }
    }
    cudaEventRecord(env->prof_ev[env->prof_used], st);
}

void prof_end(pd_env *env, cudaStream_t st, int32_t steps) {
    if (!env->prof || env->prof_used + 2 > env->prof_ev.size()) return;
    cudaEventRecord(env->prof_ev[env->prof_used + 1], st);
    if (env->prof_w.size() < env->prof_ev.size() / 2) env->prof_w.resize(env->prof_ev.size() / 2);
    env->prof_w[env->prof_used / 2] = steps;
    env->prof_used += 2;
}

pd_status cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    pd_status s = e == cudaErrorMemoryAllocation ? PD_ERR_OOM : PD_ERR_CUDA;
    return fail(s, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

}  // namespace pd

pd::Geo pd_env::geo() const {
    pd::Geo g;
    g.N = N;
    g.x4 = x4.p;
    g.tinfo = tinfo.p;
    g.blocks = blocks_d.p;
    g.pairs = pairs.p;
    g.tdens = tdens.p;
    g.si = sinfo.p;
    g.cnt = cnt.p;
    g.nbr = nbr.p;
    g.fam = fam.p;
    g.deformed = deformed.p;
    g.td2 = td2.p;
    g.edp_in = edp[ecur].p;
    g.edp_out = edp[1 - ecur].p;
    return g;
}


// ---------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------
namespace {

inline int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

// fn(begin, end) over [0, n) split across the host's cores.
template <class F>
void parallel_for(int64_t n, F fn) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw ? hw : 1, 32));
    if (n < 256 || nt == 1) {
        fn((int64_t)0, n);
        return;
    }
    const int64_t per = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t a = t * per, b = std::min(n, a + per);
        if (a >= b) break;
        th.emplace_back(fn, a, b);
    }
    for (auto &x : th) x.join();
}

bool symmetric(const std::vector<double> &m, int nt) {
    for (int i = 0; i < nt; ++i)
        for (int j = 0; j < nt; ++j)
            if (!(m[i + j * nt] == m[j + i * nt]) && !(std::isnan(m[i + j * nt]) && std::isnan(m[j + i * nt])))
                return false;
    return true;
}

pd_status check_env(const pd_env *env) {
    if (!env) return fail(PD_ERR_ARG, "environment handle is NULL");
    return PD_OK;
}

pd_status need_final(const pd_env *env) {
    PD_TRY(check_env(env));
    if (!env->finalized) return fail(PD_ERR_STATE, "environment is not finalized (call pd_env_finalize)");
    return PD_OK;
}

// Cell grid of a block for the family search: cubic cells one horizon
// (times 1+1e-9) wide over the block's bounding box, at most 1024 per axis
// (wider domains fold into the edge cells).  Any binning whose cells are at
// least a horizon wide yields the same family sets; the order is fixed
// afterwards by sorting.  The particles are binned on the device
// (k_cell_ids / k_cell_scatter).
struct CellGrid {
    double3 lo;
    double cell;
    int3 dims;
};

CellGrid block_grid(const HostBlock &b) {
    CellGrid g;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < b.n; ++i)
        for (int d = 0; d < 3; ++d) {
            mn[d] = std::min(mn[d], b.x[3 * i + d]);
            mx[d] = std::max(mx[d], b.x[3 * i + d]);
        }
    g.cell = b.horizon * (1.0 + 1e-9);
    int dims[3];
    for (int d = 0; d < 3; ++d) {
        double span = b.n > 0 ? (mx[d] - mn[d]) / g.cell : 0.0;
        double nd = std::floor(span) + 1.0;
        if (!(nd >= 1.0)) nd = 1.0;
        if (nd > 1024.0) nd = 1024.0;
        dims[d] = (int)nd;
    }
    g.lo = make_double3(b.n > 0 ? mn[0] : 0.0, b.n > 0 ? mn[1] : 0.0, b.n > 0 ? mn[2] : 0.0);
    g.dims = make_int3(dims[0], dims[1], dims[2]);
    return g;
}

}  // namespace

// ---------------------------------------------------------------------
// ABI: library
// ---------------------------------------------------------------------
extern "C" int pd_abi_version(void) { return PD_ABI_VERSION; }

extern "C" const char *pd_status_string(pd_status s) {
    switch (s) {
        case PD_OK: return "ok";
        case PD_ERR_ARG: return "invalid argument";
        case PD_ERR_OOM: return "out of memory";
        case PD_ERR_FAMILY_OVERFLOW: return "family exceeds max_neigh";
        case PD_ERR_NAN: return "non-finite value";
        case PD_ERR_CUDA: return "CUDA error";
        case PD_ERR_TIMEOUT: return "device wait timed out";
        case PD_ERR_STATE: return "invalid state";
        case PD_ERR_NO_DEVICE: return "no CUDA device";
        case PD_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

extern "C" const char *pd_last_error(void) { return g_err.c_str(); }

extern "C" pd_status pd_device_count(int32_t *count) {
    if (!count) return fail(PD_ERR_ARG, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return PD_OK;
}

// ---------------------------------------------------------------------
// ABI: environment assembly
// ---------------------------------------------------------------------
extern "C" pd_status pd_env_create(pd_env **out, int32_t device, int32_t precision, double dt) {
    if (!out) return fail(PD_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (precision < PD_PREC_FP64_SERIAL || precision > PD_PREC_FP32C)
        return fail(PD_ERR_ARG, "unknown precision mode %d", precision);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(PD_ERR_NO_DEVICE, "no CUDA device is visible; libperidyn_b200 has no CPU path");
    }
    if (device < 0 || device >= n) return fail(PD_ERR_ARG, "device %d out of range (%d visible)", device, n);
    std::unique_ptr<pd_env> env(new (std::nothrow) pd_env());
    if (!env) return fail(PD_ERR_OOM, "host allocation failed");
    env->device = device;
    env->precision = precision;
    env->dt = dt;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&env->st, cudaStreamNonBlocking));
    *out = env.release();
    return PD_OK;
}

extern "C" pd_status pd_env_destroy(pd_env *env) {
    if (!env) return PD_OK;
    cudaSetDevice(env->device);
    if (env->st) cudaStreamSynchronize(env->st);
    if (env->copy_st) {
        cudaStreamSynchronize(env->copy_st);
        cudaStreamDestroy(env->copy_st);
    }
    for (auto &s : env->slots) {
        if (s.host) cudaFreeHost(s.host);
        if (s.packed) cudaEventDestroy(s.packed);
        if (s.done) cudaEventDestroy(s.done);
    }
    env->release_device();
    for (cudaEvent_t e : env->prof_ev) cudaEventDestroy(e);
    if (env->st) cudaStreamDestroy(env->st);
    delete env;
    return PD_OK;
}

extern "C" pd_status pd_env_add_block(pd_env *env, int64_t n, const double *x, const double *y,
                                      const double *v, const double *volume,
                                      const int64_t *type, const pd_material_desc *mat,
                                      int64_t *out_block) {
    PD_TRY(check_env(env));
    if (env->finalized) return fail(PD_ERR_STATE, "environment already finalized");
    if (!env->hbc.empty()) return fail(PD_ERR_STATE, "blocks must be added before boundary conditions");
    if (n <= 0 || !x || !y || !v || !volume || !type || !mat)
        return fail(PD_ERR_ARG, "pd_env_add_block: NULL array or n <= 0");
    if (n > (int64_t)1 << 30) return fail(PD_ERR_ARG, "block too large (%lld)", (long long)n);
    if (mat->kind < PD_MAT_BOND_BASED || mat->kind > PD_MAT_ELASTO_PLASTIC)
        return fail(PD_ERR_ARG, "unknown material kind %d", mat->kind);
    if (mat->ntypes < 1 || mat->ntypes > 255) return fail(PD_ERR_ARG, "ntypes must be 1..255");
    if (!mat->density) return fail(PD_ERR_ARG, "density is NULL");
    if (!(mat->horizon > 0.0) && mat->kind != PD_MAT_SKIP) return fail(PD_ERR_ARG, "horizon must be > 0");
    const int nt = mat->ntypes;
    const size_t nt2 = (size_t)nt * nt;
    HostBlock b;
    b.n = n;
    b.kind = mat->kind;
    b.nt = nt;
    b.type_start = mat->type_start;
    b.horizon = mat->horizon;
    b.particle_size = mat->particle_size;
    b.max_neigh = mat->max_neigh;
    b.x.assign(x, x + 3 * n);
    b.y.assign(y, y + 3 * n);
    b.v.assign(v, v + 3 * n);
    b.vol.assign(volume, volume + n);
    b.type.assign(type, type + n);
    for (int64_t i = 0; i < n; ++i)
        if (type[i] < mat->type_start || type[i] >= mat->type_start + nt)
            return fail(PD_ERR_ARG, "particle %lld has type %lld outside the block's type range", (long long)i,
                        (long long)type[i]);
    b.dens.assign(mat->density, mat->density + nt);
    b.cs.assign(nt2, INFINITY);
    b.c.assign(nt2, 0.0);
    b.K.assign(nt2, 0.0);
    b.G.assign(nt2, 0.0);
    if (mat->kind != PD_MAT_SKIP) {
        if (!mat->critical_stretch) return fail(PD_ERR_ARG, "critical_stretch is NULL");
        b.cs.assign(mat->critical_stretch, mat->critical_stretch + nt2);
        if (!symmetric(b.cs, nt)) return fail(PD_ERR_ARG, "critical_stretch must be symmetric");
        if (mat->max_neigh < 1) return fail(PD_ERR_ARG, "max_neigh must be >= 1");
    }
    if (mat->kind == PD_MAT_BOND_BASED) {
        if (!mat->bond_stiffness) return fail(PD_ERR_ARG, "bond_stiffness is NULL");
        b.c.assign(mat->bond_stiffness, mat->bond_stiffness + nt2);
    }
    if (mat->kind == PD_MAT_ELASTO_PLASTIC) {
        if (!mat->plastic_psi) return fail(PD_ERR_ARG, "plastic_psi is NULL");
        b.psi.assign(mat->plastic_psi, mat->plastic_psi + nt2);
        if (!symmetric(b.psi, nt)) return fail(PD_ERR_ARG, "plastic_psi must be symmetric");
    }
    if (mat->kind == PD_MAT_ORDINARY_STATE_BASED || mat->kind == PD_MAT_ELASTO_PLASTIC) {
        if (!mat->bulk_modulus || !mat->shear_modulus) return fail(PD_ERR_ARG, "bulk/shear modulus is NULL");
        b.K.assign(mat->bulk_modulus, mat->bulk_modulus + nt2);
        b.G.assign(mat->shear_modulus, mat->shear_modulus + nt2);
        if (!symmetric(b.K, nt) || !symmetric(b.G, nt))
            return fail(PD_ERR_ARG, "bulk_modulus/shear_modulus must be symmetric");
    }
    b.first_env = env->N_env;
    env->N_env += n;
    env->hb.push_back(std::move(b));
    if (out_block) *out_block = (int64_t)env->hb.size() - 1;
    return PD_OK;
}

extern "C" pd_status pd_env_set_family(pd_env *env, int64_t block, int64_t rows,
                                       const int64_t *family, const uint8_t *intact) {
    PD_TRY(check_env(env));
    if (env->finalized) return fail(PD_ERR_STATE, "environment already finalized");
    if (block < 0 || block >= (int64_t)env->hb.size()) return fail(PD_ERR_ARG, "no block %lld", (long long)block);
    HostBlock &b = env->hb[block];
    if (rows < 1 || !family) return fail(PD_ERR_ARG, "family is NULL or rows < 1");
    size_t tot = (size_t)rows * (size_t)b.n;
    for (int64_t i = 0; i < b.n; ++i) {
        int64_t prev = INT64_MAX;
        bool zero_seen = false;
        for (int64_t r = 0; r < rows; ++r) {
            int64_t j = family[(size_t)i * rows + r];
            if (j < 0 || j > b.n) return fail(PD_ERR_ARG, "family entry out of range");
            if (j == 0) {
                zero_seen = true;
                continue;
            }
            if (zero_seen) return fail(PD_ERR_ARG, "family column %lld has an entry after padding", (long long)i);
            if (j >= prev) return fail(PD_ERR_ARG, "family column %lld is not in descending order", (long long)i);
            if (j == i + 1) return fail(PD_ERR_ARG, "family column %lld contains the particle itself", (long long)i);
            prev = j;
            if (intact && intact[(size_t)i * rows + r] > 1) return fail(PD_ERR_ARG, "intact must be 0/1");
        }
    }
    b.host_family = true;
    b.rows = rows;
    b.family.assign(family, family + tot);
    b.intact.resize(tot);
    for (size_t e = 0; e < tot; ++e) b.intact[e] = intact ? (uint8_t)(intact[e] && family[e] > 0) : (uint8_t)(family[e] > 0);
    return PD_OK;
}

extern "C" pd_status pd_env_add_bc(pd_env *env, int32_t kind, const uint8_t *mask,
                                   const uint8_t *dims, const double *rate, double freq,
                                   int64_t applyafter, int32_t onlyatstart, int64_t *out_bc) {
    PD_TRY(check_env(env));
    if (env->finalized) return fail(PD_ERR_STATE, "environment already finalized");
    if (kind != PD_BC_FIX && kind != PD_BC_TOFRO) return fail(PD_ERR_ARG, "unknown BC kind %d", kind);
    if (!mask || !dims) return fail(PD_ERR_ARG, "mask/dims is NULL");
    if (kind == PD_BC_TOFRO && !rate) return fail(PD_ERR_ARG, "rate is NULL");
    if (env->hbc.size() >= 64) return fail(PD_ERR_UNSUPPORTED, "at most 64 boundary conditions");
    HostBC bc;
    bc.kind = kind;
    bc.dims = (dims[0] ? 1 : 0) | (dims[1] ? 2 : 0) | (dims[2] ? 4 : 0);
    for (int d = 0; d < 3; ++d) bc.rate[d] = kind == PD_BC_TOFRO ? rate[d] : 0.0;
    bc.freq = freq;
    bc.applyafter = applyafter;
    bc.onlyatstart = onlyatstart;
    bc.dir = 1;
    for (int64_t e = 0; e < env->N_env; ++e)
        if (mask[e]) bc.env_idx.push_back(e);
    env->hbc.push_back(std::move(bc));
    if (out_bc) *out_bc = (int64_t)env->hbc.size() - 1;
    return PD_OK;
}

static pd_status new_bc(pd_env *env, int32_t kind, const uint8_t *mask, const uint8_t *dims, int32_t onlyatstart,
                        HostBC &bc) {
    PD_TRY(check_env(env));
    if (env->finalized) return fail(PD_ERR_STATE, "environment already finalized");
    if (!mask || !dims) return fail(PD_ERR_ARG, "mask/dims is NULL");
    if (env->hbc.size() >= 64) return fail(PD_ERR_UNSUPPORTED, "at most 64 boundary conditions");
    bc.kind = kind;
    bc.dims = (dims[0] ? 1 : 0) | (dims[1] ? 2 : 0) | (dims[2] ? 4 : 0);
    bc.freq = INFINITY;
    bc.onlyatstart = onlyatstart;
    for (int64_t e = 0; e < env->N_env; ++e)
        if (mask[e]) bc.env_idx.push_back(e);
    return PD_OK;
}

extern "C" pd_status pd_env_add_scaled_bc(pd_env *env, int32_t kind, const uint8_t *mask, const uint8_t *dims,
                                          const double *scale, const double *fixpoint, int64_t wait,
                                          const uint8_t *scalemask, int32_t onlyatstart, int64_t *out_bc) {
    if (kind != PD_BC_DELTA_SCALE && kind != PD_BC_SCALE_FIX_WAIT)
        return fail(PD_ERR_ARG, "kind must be PD_BC_DELTA_SCALE or PD_BC_SCALE_FIX_WAIT");
    if (!scale || !fixpoint) return fail(PD_ERR_ARG, "scale/fixpoint is NULL");
    if (kind == PD_BC_SCALE_FIX_WAIT && (!scalemask || wait == 0))
        return fail(PD_ERR_ARG, "ScaleFixWaitBC needs scalebool and a nonzero wait");
    HostBC bc;
    PD_TRY(new_bc(env, kind, mask, dims, onlyatstart, bc));
    for (int d = 0; d < 3; ++d) {
        bc.scale[d] = scale[d];
        bc.fix[d] = fixpoint[d];
    }
    if (kind == PD_BC_SCALE_FIX_WAIT) {
        bc.wait = wait;
        for (int64_t e = 0; e < env->N_env; ++e)
            if (scalemask[e]) bc.scale_idx.push_back(e);
    }
    env->hbc.push_back(std::move(bc));
    if (out_bc) *out_bc = (int64_t)env->hbc.size() - 1;
    return PD_OK;
}

extern "C" pd_status pd_env_add_container_bc(pd_env *env, const uint8_t *mask, const uint8_t *dims,
                                             const double *limits, int32_t onlyatstart, int64_t *out_bc) {
    HostBC bc;
    PD_TRY(new_bc(env, PD_BC_CONTAINER, mask, dims, onlyatstart, bc));
    if (limits) {
        bc.has_limits = 1;
        for (int d = 0; d < 3; ++d) {
            bc.lo[d] = limits[d];
            bc.hi[d] = limits[3 + d];
        }
    }
    env->hbc.push_back(std::move(bc));
    if (out_bc) *out_bc = (int64_t)env->hbc.size() - 1;
    return PD_OK;
}

extern "C" pd_status pd_env_add_contact(pd_env *env, int32_t kind, int64_t block1, int64_t block2,
                                        double exponent, double stiffness, double equi_dist,
                                        double distance, int64_t max_neighs, int64_t *out_contact) {
    PD_TRY(check_env(env));
    if (env->finalized) return fail(PD_ERR_STATE, "environment already finalized");
    if (kind != PD_CONTACT_12 && kind != PD_CONTACT_11 && kind != PD_CONTACT_11_ORDERED)
        return fail(PD_ERR_ARG, "unknown contact kind %d", kind);
    int64_t nb = (int64_t)env->hb.size();
    if (block1 < 0 || block1 >= nb) return fail(PD_ERR_ARG, "no block %lld", (long long)block1);
    if (kind == PD_CONTACT_12 && (block2 < 0 || block2 >= nb || block2 == block1))
        return fail(PD_ERR_ARG, "contact-12 needs two distinct blocks");
    if (max_neighs < 1) return fail(PD_ERR_ARG, "max_neighs must be >= 1");
    if (!(equi_dist > 0.0) || !(distance > 0.0)) return fail(PD_ERR_ARG, "equi_dist/distance must be > 0");
    HostContact c;
    c.kind = kind;
    c.b1 = block1;
    c.b2 = kind == PD_CONTACT_12 ? block2 : block1;
    c.exponent = exponent;
    c.stiffness = stiffness;
    c.equi_dist = equi_dist;
    c.distance = distance;
    c.max_neighs = max_neighs;
    env->hc.push_back(std::move(c));
    if (out_contact) *out_contact = (int64_t)env->hc.size() - 1;
    return PD_OK;
}

namespace {
// Wall-clock phases of pd_env_finalize (and of the device layout
// conversion), printed to stderr when the process environment has
// PD_SETUP_TIMES=1 (a diagnostic for setup cost).
struct SetupClock {
    bool on = false;
    std::chrono::steady_clock::time_point t0, t;
    SetupClock() {
        const char *e = std::getenv("PD_SETUP_TIMES");
        on = e && std::strcmp(e, "1") == 0;
        t0 = t = std::chrono::steady_clock::now();
    }
    void mark(const char *phase, cudaStream_t st) {
        if (!on) return;
        cudaStreamSynchronize(st);
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "pd_env_finalize %-32s %8.1f ms (total %8.1f ms)\n", phase,
                     std::chrono::duration<double, std::milli>(now - t).count(),
                     std::chrono::duration<double, std::milli>(now - t0).count());
        t = now;
    }
};
}  // namespace

// Record staging plans of the stencil slices (opt-in staged kernels), from
// each slice's union of offsets, built on the host and uploaded: per plan
// {ranges, records, (first record, count) per range}, and per stencil slot
// the staged position of lane 0's record.  nbr_size: entries of the
// runtime neighbour array (spos has one per entry).
// Slots the step kernels walk: a slice's warps together visit the slots up
// to the largest slot count of its 32 particles (whatever the kernel shape),
// 32 lanes each.
static int64_t walked_slots(const std::vector<int32_t> &cnt) {
    int64_t w = 0;
    for (size_t s0 = 0; s0 < cnt.size(); s0 += kSlice) {
        int32_t m = 0;
        for (size_t l = s0; l < s0 + kSlice && l < cnt.size(); ++l) m = std::max(m, cnt[l]);
        w += (int64_t)kSlice * m;
    }
    return w;
}

static pd_status upload_stage_plans(pd_env *env, const std::vector<SliceInfo> &si,
                                    const std::vector<std::vector<int32_t>> &uni, size_t nbr_size) {
    const int64_t N = env->N, S = N / kSlice;
    std::vector<std::vector<int32_t>> plans(S);
    std::vector<int32_t> spos(nbr_size, 0);
    parallel_for(S, [&](int64_t s0, int64_t s1) {
        std::vector<int32_t> rs, pos;
        for (int64_t s = s0; s < s1; ++s) {
            const SliceInfo &d = si[s];
            if (d.mode != kStencil) continue;
            const int64_t T = stage_plan(s * kSlice, N, uni[s], rs, pos);
            if (T == 0 || T > kStageMaxRecords) continue;
            std::copy(pos.begin(), pos.end(), spos.begin() + d.nbr);
            std::vector<int32_t> &pl = plans[s];
            pl.reserve(2 + rs.size());
            pl.push_back((int32_t)(rs.size() / 2));
            pl.push_back((int32_t)T);
            pl.insert(pl.end(), rs.begin(), rs.end());
        }
    });
    std::vector<int32_t> splan_off(S + 1, -1), splan;
    int64_t nplan = 0, pmax = 0;
    for (int64_t s = 0; s < S; ++s) {
        if (plans[s].empty()) continue;
        splan_off[s] = (int32_t)splan.size();
        splan.insert(splan.end(), plans[s].begin(), plans[s].end());
        pmax = std::max<int64_t>(pmax, plans[s][1]);
        ++nplan;
    }
    if (splan.empty()) splan.push_back(0);
    env->splan_slices = nplan;
    env->splan_max = pmax;
    cudaStream_t st = env->st;
    PD_TRY(env->splan_off.alloc(S + 1));
    PD_TRY(env->splan.alloc((int64_t)splan.size()));
    PD_TRY(env->spos.alloc((int64_t)spos.size()));
    CK(cudaMemcpyAsync(env->splan_off.p, splan_off.data(), (S + 1) * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->splan.p, splan.data(), splan.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->spos.p, spos.data(), spos.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return PD_OK;
}

// ---------------------------------------------------------------------
// Runtime bond layout.  Input: the build layout (SELL-32, bond k of lane l
// of slice s at nbr_b[slice_ptr[s] + 32k + l], intact bit k%32 of word
// slice_ptr[s]/32 + 32(k/32) + l, cnt[p] members in descending index order).
// Output: one SliceInfo per slice.  A slice whose lanes' neighbour offsets
// q - p form a small union (a lattice, where every particle sees the same
// stencil) stores one offset per slot and reads no per-bond index; the
// others keep the explicit indices.  cnt becomes the number of slots to scan.
// ---------------------------------------------------------------------
static pd_status build_runtime_layout(pd_env *env, const std::vector<int64_t> &slice_ptr, std::vector<int32_t> &cnt,
                                      const std::vector<int32_t> &nbr_b, const std::vector<uint32_t> &w_b) {
    const int64_t N = env->N, S = N / kSlice;
    const char *lay = std::getenv("PD_FAMILY_LAYOUT");
    const bool force_explicit = lay && std::strcmp(lay, "explicit") == 0;
    std::vector<SliceInfo> si(S + 1);
    std::vector<std::vector<int32_t>> uni(S);
    // pass 1 (per slice): the union of the lanes' offsets q - p, merged from
    // the lanes' descending lists; stencil form when it stays small
    parallel_for(S, [&](int64_t s0, int64_t s1) {
        std::vector<int32_t> cur, lane, tmp;
        for (int64_t s = s0; s < s1; ++s) {
            int32_t maxc = 0;
            for (int l = 0; l < kSlice; ++l) maxc = std::max(maxc, cnt[s * kSlice + l]);
            const int64_t limit = (int64_t)maxc + maxc / 4 + 32;
            bool stencil = !force_explicit && maxc > 0;
            cur.clear();
            for (int l = 0; stencil && l < kSlice; ++l) {
                const int64_t p = s * kSlice + l;
                const int64_t base = slice_ptr[s] + l;
                lane.resize(cnt[p]);
                for (int32_t k = 0; k < cnt[p]; ++k) lane[k] = nbr_b[base + 32 * (int64_t)k] - (int32_t)p;
                tmp.clear();
                std::set_union(cur.begin(), cur.end(), lane.begin(), lane.end(), std::back_inserter(tmp),
                               std::greater<int32_t>());
                cur.swap(tmp);
                if ((int64_t)cur.size() > limit) stencil = false;
            }
            // every slot a lane scans must name an in-range record
            for (int l = 0; stencil && l < kSlice; ++l) {
                const int64_t p = s * kSlice + l;
                if (cnt[p] == 0) continue;
                stencil = p + cur.front() < N && p + cur.back() >= 0;
            }
            SliceInfo &d = si[s];
            if (stencil) {
                d.mode = kStencil;
                d.len = (int32_t)round_up((int64_t)cur.size(), 32);
                uni[s] = cur;
            } else {
                d.mode = kExplicit;
                d.len = (int32_t)round_up(maxc, 32);
            }
        }
    });
    int64_t nbr_len = 0, nwords = 0, nst = 0;
    for (int64_t s = 0; s < S; ++s) {
        SliceInfo &d = si[s];
        d.nbr = nbr_len;
        d.word = nwords;
        nbr_len += d.mode == kStencil ? d.len : (int64_t)kSlice * d.len;
        nwords += d.len;
        nst += d.mode == kStencil;
    }
    si[S].nbr = nbr_len;
    si[S].word = nwords;
    si[S].len = 0;
    si[S].mode = kExplicit;
    std::vector<int32_t> nbr(std::max<int64_t>(nbr_len, 32), 0);
    std::vector<uint32_t> words(std::max<int64_t>(nwords, 1), 0), fam(std::max<int64_t>(nwords, 1), 0);
    std::vector<int32_t> cnt_rt(N, 0);
    // pass 2 (per slice, disjoint outputs): slots, bits and slot counts
    parallel_for(S, [&](int64_t s0, int64_t s1) {
        for (int64_t s = s0; s < s1; ++s) {
            const SliceInfo &d = si[s];
            const std::vector<int32_t> &u = uni[s];
            if (d.mode == kStencil)
                for (size_t j = 0; j < u.size(); ++j) nbr[d.nbr + j] = u[j];
            for (int l = 0; l < kSlice; ++l) {
                const int64_t p = s * kSlice + l;
                const int64_t base = slice_ptr[s] + l, wb = slice_ptr[s] / 32 + l, ow = d.word + l;
                int32_t j = 0, last = -1;
                for (int32_t k = 0; k < cnt[p]; ++k) {
                    const int32_t q = nbr_b[base + 32 * (int64_t)k];
                    int32_t slot = k;
                    if (d.mode == kStencil) {
                        // both lists descend: advance to this offset
                        while (u[j] != q - (int32_t)p) ++j;
                        slot = j;
                    } else {
                        nbr[d.nbr + 32 * (int64_t)k + l] = q;
                    }
                    const uint32_t bit = 1u << (slot & 31);
                    fam[ow + 32 * (int64_t)(slot >> 5)] |= bit;
                    if ((w_b[wb + 32 * (int64_t)(k >> 5)] >> (k & 31)) & 1u)
                        words[ow + 32 * (int64_t)(slot >> 5)] |= bit;
                    last = slot;
                }
                cnt_rt[p] = last + 1;
            }
        }
    });
    cnt.swap(cnt_rt);
    // pass 3 (per stencil slice): record staging plans
    PD_TRY(upload_stage_plans(env, si, uni, nbr.size()));
    env->sinfo_h = si;
    env->cnt_h = cnt;
    env->nnz = (int64_t)kSlice * nwords;
    env->walked = walked_slots(env->cnt_h);
    env->nbr_len = nbr_len;
    env->stencil_slices = nst;
    cudaStream_t st = env->st;
    const int64_t nw = std::max<int64_t>(nwords, 1);
    // zero entries past the end: the stencil walks load the offsets of the
    // next slots ahead of use and may read up to kNbrPad entries beyond a
    // slice's own (those values are never used)
    nbr.resize(nbr.size() + kNbrPad, 0);
    PD_TRY(env->sinfo.alloc(S + 1));
    PD_TRY(env->nbr.alloc((int64_t)nbr.size()));
    PD_TRY(env->words[0].alloc(nw));
    PD_TRY(env->words[1].alloc(nw));
    PD_TRY(env->words0.alloc(nw));
    PD_TRY(env->fam.alloc(nw));
    CK(cudaMemcpyAsync(env->sinfo.p, si.data(), (S + 1) * sizeof(SliceInfo), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->nbr.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->words[0].p, words.data(), nw * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->words[1].p, words.data(), nw * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->words0.p, words.data(), nw * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->fam.p, fam.data(), nw * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->cnt.p, cnt.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return PD_OK;
}

// The runtime layout of build_runtime_layout, converted on the device from
// the build layout already there (d_nbr, d_words; cnt_b = the build family
// sizes, also in env->cnt): the per-slice unions and stencil decisions
// (k_layout_union), the slice offsets on the host from the slices' modes
// and lengths, then the runtime arrays (k_layout_fill).  Only per-slice
// values, the slot counts and the runtime neighbour array (one entry per
// stencil slot) come back to the host, instead of the whole build layout.
static pd_status build_runtime_layout_device(pd_env *env, const std::vector<int64_t> &slice_ptr,
                                             std::vector<int32_t> &cnt_b, const int64_t *d_slice_ptr,
                                             const int32_t *d_nbr, const uint32_t *d_words) {
    const int64_t N = env->N, S = N / kSlice;
    cudaStream_t st = env->st;
    SetupClock clk;
    const char *lay = std::getenv("PD_FAMILY_LAYOUT");
    const bool force_explicit = lay && std::strcmp(lay, "explicit") == 0;
    int32_t maxc_all = 0;
    for (int64_t p = 0; p < N; ++p) maxc_all = std::max(maxc_all, cnt_b[p]);
    const int64_t ustride = round_up((int64_t)maxc_all + maxc_all / 4 + 33, 32);
    SBuf<int32_t> d_mode, d_len, d_uni, d_cnt_rt;
    PD_TRY(d_mode.alloc(std::max<int64_t>(S, 1), st));
    PD_TRY(d_len.alloc(std::max<int64_t>(S, 1), st));
    PD_TRY(d_uni.alloc(std::max<int64_t>(S * ustride, 1), st));
    PD_TRY(d_cnt_rt.alloc(std::max<int64_t>(N, 1), st));
    launch_layout_union(st, S, N, d_slice_ptr, env->cnt.p, d_nbr, force_explicit ? 1 : 0, ustride, d_mode.p,
                        d_len.p, d_uni.p);
    CK(cudaGetLastError());
    std::vector<int32_t> mode(S), ulen(S);
    if (S > 0) {
        CK(cudaMemcpyAsync(mode.data(), d_mode.p, S * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(ulen.data(), d_len.p, S * 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    clk.mark("  layout: unions", st);
    std::vector<SliceInfo> si(S + 1);
    int64_t nbr_len = 0, nwords = 0, nst = 0;
    for (int64_t s = 0; s < S; ++s) {
        SliceInfo &d = si[s];
        d.mode = mode[s];
        d.len = (int32_t)round_up((int64_t)ulen[s], 32);
        d.nbr = nbr_len;
        d.word = nwords;
        nbr_len += d.mode == kStencil ? d.len : (int64_t)kSlice * d.len;
        nwords += d.len;
        nst += d.mode == kStencil;
    }
    si[S].nbr = nbr_len;
    si[S].word = nwords;
    si[S].len = 0;
    si[S].mode = kExplicit;
    const int64_t nw = std::max<int64_t>(nwords, 1);
    const int64_t nb = std::max<int64_t>(nbr_len, 32) + kNbrPad;  // zero read-ahead margin past the end
    PD_TRY(env->sinfo.alloc(S + 1));
    PD_TRY(env->nbr.alloc(nb));
    PD_TRY(env->words[0].alloc(nw));
    PD_TRY(env->words[1].alloc(nw));
    PD_TRY(env->words0.alloc(nw));
    PD_TRY(env->fam.alloc(nw));
    CK(cudaMemcpyAsync(env->sinfo.p, si.data(), (S + 1) * sizeof(SliceInfo), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(env->nbr.p, 0, nb * 4, st));
    CK(cudaMemsetAsync(env->words[0].p, 0, nw * 4, st));
    CK(cudaMemsetAsync(env->fam.p, 0, nw * 4, st));
    launch_layout_fill(st, N, d_slice_ptr, env->cnt.p, d_nbr, d_words, env->sinfo.p, d_len.p, ustride, d_uni.p,
                       env->nbr.p, env->words[0].p, env->fam.p, d_cnt_rt.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(env->words[1].p, env->words[0].p, nw * 4, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(env->words0.p, env->words[0].p, nw * 4, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(env->cnt.p, d_cnt_rt.p, N * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    std::vector<int32_t> cnt_rt(N), nbr(std::max<int64_t>(nbr_len, 32));
    CK(cudaMemcpyAsync(cnt_rt.data(), d_cnt_rt.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(nbr.data(), env->nbr.p, nbr.size() * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    clk.mark("  layout: fill, slot counts back", st);
    // staging plans from the stencil slices' unions
    std::vector<std::vector<int32_t>> uni(S);
    for (int64_t s = 0; s < S; ++s)
        if (si[s].mode == kStencil) uni[s].assign(nbr.begin() + si[s].nbr, nbr.begin() + si[s].nbr + ulen[s]);
    PD_TRY(upload_stage_plans(env, si, uni, nbr.size()));
    clk.mark("  layout: staging plans", st);
    cnt_b.swap(cnt_rt);
    env->sinfo_h = si;
    env->cnt_h = cnt_b;
    env->nnz = (int64_t)kSlice * nwords;
    env->walked = walked_slots(env->cnt_h);
    env->nbr_len = nbr_len;
    env->stencil_slices = nst;
    return PD_OK;
}

// ---------------------------------------------------------------------
// finalize: layout, upload, families, weighted volume, intact0
// ---------------------------------------------------------------------

extern "C" pd_status pd_env_finalize(pd_env *env) {
    PD_TRY(check_env(env));
    if (env->finalized) return fail(PD_ERR_STATE, "environment already finalized");
    if (env->hb.empty()) return fail(PD_ERR_STATE, "environment has no material blocks");
    CK(cudaSetDevice(env->device));
    cudaStream_t st = env->st;
    SetupClock clk;

    // --- internal layout ---
    int64_t N = 0;
    for (auto &b : env->hb) {
        b.first_int = N;
        N += round_up(b.n, kSlice);
    }
    env->N = N;
    const int64_t NE = env->N_env;
    env->map_h.resize(NE);
    for (auto &b : env->hb)
        for (int64_t i = 0; i < b.n; ++i) env->map_h[b.first_env + i] = b.first_int + i;

    std::vector<double4> x4(N, make_double4(0, 0, 0, 0)), y4(N, make_double4(0, 0, 0, 0)),
        v4(N, make_double4(0, 0, 0, 0));
    std::vector<int32_t> tinfo(N, -1);
    std::vector<double> mass(N, 0.0), dens(N, 0.0);
    std::vector<DevBlock> blocks;
    std::vector<PairParam> pairs;
    std::vector<double> tdens;
    env->deformed_h.assign(env->hb.size(), 0);
    for (size_t bi = 0; bi < env->hb.size(); ++bi) {
        HostBlock &b = env->hb[bi];
        DevBlock d{};
        d.kind = b.kind;
        d.nt = b.nt;
        d.pair_base = (int32_t)pairs.size();
        d.type_base = (int32_t)tdens.size();
        d.first = b.first_int;
        d.n = b.n;
        d.c11 = b.c[0];
        d.c11f = (float)b.c[0];
        double cen[3] = {0, 0, 0};
        for (int64_t i = 0; i < b.n; ++i)
            for (int k = 0; k < 3; ++k) cen[k] += b.x[3 * i + k];
        d.center = make_double3(cen[0] / b.n, cen[1] / b.n, cen[2] / b.n);
        for (int j = 0; j < b.nt; ++j)
            for (int i = 0; i < b.nt; ++i) {
                size_t e = (size_t)i + (size_t)j * b.nt;
                PairParam pp;
                pp.cs = b.cs[e];
                // ordinary_state_based.jl:183 (3K - 5G); elasto_plastic.jl:239 (3K)
                pp.k35 = b.kind == PD_MAT_ELASTO_PLASTIC ? 3 * b.K[e] : 3 * b.K[e] - 5 * b.G[e];
                pp.g15 = 15 * b.G[e];
                pp.psi2 = b.kind == PD_MAT_ELASTO_PLASTIC ? 2 * b.psi[e] : 0.0;
                pairs.push_back(pp);
            }
        for (int t = 0; t < b.nt; ++t) tdens.push_back(b.dens[t]);
        blocks.push_back(d);
        bool deformed = false;
        for (int64_t i = 0; i < b.n; ++i) {
            int64_t p = b.first_int + i;
            x4[p] = make_double4(b.x[3 * i], b.x[3 * i + 1], b.x[3 * i + 2], b.vol[i]);
            y4[p] = make_double4(b.y[3 * i], b.y[3 * i + 1], b.y[3 * i + 2], 0.0);
            v4[p] = make_double4(b.v[3 * i], b.v[3 * i + 1], b.v[3 * i + 2], 0.0);
            int t = (int)(b.type[i] - b.type_start);
            tinfo[p] = ((int32_t)bi << 8) | t;
            // environment.jl:173-180,214: mass = volume * rho[t]; density = mass / volume
            mass[p] = b.vol[i] * b.dens[t];
            dens[p] = mass[p] / b.vol[i];
            for (int k = 0; k < 3; ++k) deformed |= !(b.y[3 * i + k] == b.x[3 * i + k]);
        }
        // general_material.jl:92-96: deformed = (y0 != x)
        env->deformed_h[bi] = deformed ? 1 : 0;
    }
    env->deformed0 = env->deformed_h;
    env->blocks_h = blocks;

    PD_TRY(env->x4.alloc(N));
    PD_TRY(env->y.alloc(N));
    PD_TRY(env->v.alloc(N));
    PD_TRY(env->f.alloc(N));
    PD_TRY(env->p.alloc(N));
    PD_TRY(env->tinfo.alloc(N));
    PD_TRY(env->mass.alloc(N));
    PD_TRY(env->dens.alloc(N));
    PD_TRY(env->mth.alloc(N));
    PD_TRY(env->cnt.alloc(N));
    PD_TRY(env->intact0.alloc(N));
    PD_TRY(env->map.alloc(NE));
    PD_TRY(env->blocks_d.alloc(blocks.size()));
    PD_TRY(env->pairs.alloc(pairs.size()));
    PD_TRY(env->tdens.alloc(tdens.size()));
    PD_TRY(env->deformed.alloc(blocks.size()));
    PD_TRY(env->partials.alloc(3 * 256));
    PD_TRY(env->out3.alloc(8));
    PD_TRY(env->flag.alloc(4));
    PD_TRY(env->stage.alloc(3 * (size_t)std::max<int64_t>(NE, 1)));
    CK(cudaMemcpyAsync(env->x4.p, x4.data(), N * sizeof(double4), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->y.p, y4.data(), N * sizeof(double4), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->v.p, v4.data(), N * sizeof(double4), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(env->f.p, 0, N * sizeof(double4), st));
    CK(cudaMemsetAsync(env->p.p, 0, N * sizeof(double4), st));
    CK(cudaMemsetAsync(env->mth.p, 0, N * sizeof(double2), st));
    CK(cudaMemcpyAsync(env->tinfo.p, tinfo.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->mass.p, mass.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->dens.p, dens.data(), N * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->map.p, env->map_h.data(), NE * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->blocks_d.p, blocks.data(), blocks.size() * sizeof(DevBlock),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(env->pairs.p, pairs.data(), pairs.size() * sizeof(PairParam), cudaMemcpyHostToDevice,
                       st));
    CK(cudaMemcpyAsync(env->tdens.p, tdens.data(), tdens.size() * sizeof(double), cudaMemcpyHostToDevice,
                       st));
    {
        std::vector<int32_t> df(env->deformed_h.begin(), env->deformed_h.end());
        CK(cudaMemcpyAsync(env->deformed.p, df.data(), df.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                           st));
        CK(cudaStreamSynchronize(st));
    }

    clk.mark("assembly and upload", st);
    // --- family sizes: GPU neighbour count per GPU-built block ---
    std::vector<int32_t> cnt(N, 0);
    std::vector<CellGrid> cells(env->hb.size());
    std::vector<int64_t> cell_base(env->hb.size(), 0);
    SBuf<int32_t> d_cell_of, d_cell_start, d_cell_list;
    {
        int64_t tot_cells = 0, tot_part = 0;
        std::vector<int64_t> part_off(env->hb.size(), 0);
        for (size_t bi = 0; bi < env->hb.size(); ++bi) {
            HostBlock &b = env->hb[bi];
            if (b.kind == PD_MAT_SKIP || b.host_family) continue;
            cells[bi] = block_grid(b);
            cell_base[bi] = tot_cells;
            part_off[bi] = tot_part;
            b.cell_part_off = tot_part;
            tot_cells += (int64_t)cells[bi].dims.x * cells[bi].dims.y * cells[bi].dims.z;
            tot_part += b.n;
        }
        if (tot_cells >= ((int64_t)1 << 31) || tot_part >= ((int64_t)1 << 31))
            return fail(PD_ERR_UNSUPPORTED, "family search grid too large (%lld cells)", (long long)tot_cells);
        if (tot_part > 0) {
            // counting sort by cell on the device: ids and counts, starts
            // (scanned on the host: one entry per cell), lists
            PD_TRY(d_cell_of.alloc(tot_part, st));
            PD_TRY(d_cell_start.alloc(tot_cells + 1, st));
            PD_TRY(d_cell_list.alloc(tot_part, st));
            SBuf<int32_t> d_count;
            PD_TRY(d_count.alloc(tot_cells + 1, st));
            CK(cudaMemsetAsync(d_count.p, 0, (tot_cells + 1) * sizeof(int32_t), st));
            for (size_t bi = 0; bi < env->hb.size(); ++bi) {
                HostBlock &b = env->hb[bi];
                if (b.kind == PD_MAT_SKIP || b.host_family) continue;
                launch_cell_ids(st, b.n, b.first_int, env->x4.p, cells[bi].lo, cells[bi].cell, cells[bi].dims,
                                cell_base[bi], d_cell_of.p + part_off[bi], d_count.p);
            }
            CK(cudaGetLastError());
            std::vector<int32_t> start(tot_cells + 1, 0);
            CK(cudaMemcpyAsync(start.data(), d_count.p, tot_cells * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            int32_t run = 0;
            for (int64_t c = 0; c < tot_cells; ++c) {
                const int32_t k = start[c];
                start[c] = run;
                run += k;
            }
            start[tot_cells] = run;
            CK(cudaMemcpyAsync(d_cell_start.p, start.data(), (tot_cells + 1) * sizeof(int32_t),
                               cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_count.p, start.data(), (tot_cells + 1) * sizeof(int32_t), cudaMemcpyHostToDevice,
                               st));  // scatter cursors
            for (size_t bi = 0; bi < env->hb.size(); ++bi) {
                HostBlock &b = env->hb[bi];
                if (b.kind == PD_MAT_SKIP || b.host_family) continue;
                launch_cell_scatter(st, b.n, b.first_int, d_cell_of.p + part_off[bi], d_count.p, d_cell_list.p);
            }
            CK(cudaGetLastError());
            CK(cudaMemsetAsync(env->cnt.p, 0, N * sizeof(int32_t), st));
            for (size_t bi = 0; bi < env->hb.size(); ++bi) {
                HostBlock &b = env->hb[bi];
                if (b.kind == PD_MAT_SKIP || b.host_family) continue;
                launch_count_neighbors(st, b.n, b.first_int, env->x4.p, d_cell_of.p + part_off[bi],
                                       d_cell_start.p, d_cell_list.p, cell_base[bi], cells[bi].dims,
                                       b.horizon, env->cnt.p);
            }
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(cnt.data(), env->cnt.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
    }
    // host-provided families
    for (auto &b : env->hb) {
        if (!b.host_family) continue;
        for (int64_t i = 0; i < b.n; ++i) {
            int32_t c = 0;
            for (int64_t r = 0; r < b.rows; ++r) c += b.family[(size_t)i * b.rows + r] > 0;
            cnt[b.first_int + i] = c;
        }
    }
    // overflow check and reference row counts (general_material.jl:88)
    for (auto &b : env->hb) {
        int64_t maxc = 0;
        for (int64_t i = 0; i < b.n; ++i) maxc = std::max<int64_t>(maxc, cnt[b.first_int + i]);
        if (b.kind == PD_MAT_SKIP && !b.host_family) {
            b.rows = 1;
            continue;
        }
        if (!b.host_family) {
            int64_t mn = std::min<int64_t>(b.max_neigh, b.n);
            if (maxc >= mn)
                return fail(PD_ERR_FAMILY_OVERFLOW,
                            "a family has %lld members but max_neigh allows at most %lld (reference: BoundsError)",
                            (long long)maxc, (long long)(mn - 1));
            b.rows = maxc + 1;
        }
    }
    clk.mark("binning and family counts", st);
    // Build layout: SELL-32 with one explicit index per (slot, lane), filled
    // and sorted on the device.
    const int64_t S = N / kSlice;
    std::vector<int64_t> slice_ptr(S + 1, 0);
    for (int64_t s = 0; s < S; ++s) {
        int32_t m = 0;
        for (int l = 0; l < kSlice; ++l) m = std::max(m, cnt[s * kSlice + l]);
        slice_ptr[s + 1] = slice_ptr[s] + (int64_t)kSlice * round_up(m, 32);
    }
    const int64_t bnnz = slice_ptr[S];
    std::vector<int32_t> nbr_b;
    std::vector<uint32_t> w_b;
    bool any_host = false;
    for (auto &b : env->hb) any_host |= b.host_family;
    // The runtime layout is converted on the device unless a block's family
    // came from the host (then the build layout is patched on the host) or
    // PD_LAYOUT_HOST=1 asks for the host conversion.
    const char *lh = std::getenv("PD_LAYOUT_HOST");
    const bool layout_on_device = !any_host && !(lh && std::strcmp(lh, "1") == 0);
    SBuf<int64_t> d_slice_ptr;
    SBuf<int32_t> d_nbr;
    SBuf<uint32_t> d_words;
    {
        PD_TRY(d_slice_ptr.alloc(S + 1, st));
        PD_TRY(d_nbr.alloc(std::max<int64_t>(bnnz, 32), st));
        PD_TRY(d_words.alloc(std::max<int64_t>(bnnz / 32, 1), st));
        CK(cudaMemcpyAsync(d_slice_ptr.p, slice_ptr.data(), (S + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(env->cnt.p, cnt.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(d_nbr.p, 0, std::max<int64_t>(bnnz, 32) * sizeof(int32_t), st));
        CK(cudaMemsetAsync(d_words.p, 0, std::max<int64_t>(bnnz / 32, 1) * 4, st));
        for (size_t bi = 0; bi < env->hb.size(); ++bi) {
            HostBlock &b = env->hb[bi];
            if (b.kind == PD_MAT_SKIP || b.host_family) continue;
            launch_fill_neighbors(st, b.n, b.first_int, env->x4.p, d_cell_of.p + b.cell_part_off, d_cell_start.p,
                                  d_cell_list.p, cell_base[bi], cells[bi].dims, b.horizon, d_slice_ptr.p, d_nbr.p);
        }
        launch_sort_neighbors(st, N, d_slice_ptr.p, env->cnt.p, d_nbr.p);
        launch_init_intact(st, N, d_slice_ptr.p, env->cnt.p, d_words.p);
        CK(cudaGetLastError());
        if (!layout_on_device) {
            nbr_b.assign(bnnz, 0);
            w_b.assign(bnnz / 32, 0);
            if (bnnz > 0) {
                CK(cudaMemcpyAsync(nbr_b.data(), d_nbr.p, bnnz * 4, cudaMemcpyDeviceToHost, st));
                CK(cudaMemcpyAsync(w_b.data(), d_words.p, (bnnz / 32) * 4, cudaMemcpyDeviceToHost, st));
            }
        }
        CK(cudaStreamSynchronize(st));
    }
    // host-provided families (already descending): write entries and bits
    if (any_host) {
        for (auto &b : env->hb) {
            if (!b.host_family) continue;
            for (int64_t i = 0; i < b.n; ++i) {
                int64_t p = b.first_int + i;
                int64_t base = slice_ptr[p / 32] + (p % 32), wb = slice_ptr[p / 32] / 32 + (p % 32);
                int64_t k = 0;
                for (int64_t r = 0; r < b.rows; ++r) {
                    int64_t j = b.family[(size_t)i * b.rows + r];
                    if (j <= 0) continue;
                    nbr_b[base + 32 * k] = (int32_t)(b.first_int + j - 1);
                    uint32_t bit = 1u << (k % 32);
                    uint32_t &w = w_b[wb + 32 * (k / 32)];
                    if (b.intact[(size_t)i * b.rows + r]) w |= bit;
                    else w &= ~bit;
                    ++k;
                }
            }
        }
        // symmetry of the bond set (the serial-order gather relies on it)
        if (env->precision == PD_PREC_FP64_SERIAL) {
            for (auto &b : env->hb) {
                if (!b.host_family) continue;
                for (int64_t i = 0; i < b.n; ++i) {
                    int64_t p = b.first_int + i;
                    int64_t base = slice_ptr[p / 32] + (p % 32), wb = slice_ptr[p / 32] / 32 + (p % 32);
                    for (int64_t k = 0; k < cnt[p]; ++k) {
                        int64_t q = nbr_b[base + 32 * k];
                        bool bit = (w_b[wb + 32 * (k / 32)] >> (k % 32)) & 1u;
                        int64_t qb = slice_ptr[q / 32] + (q % 32), qwb = slice_ptr[q / 32] / 32 + (q % 32);
                        bool found = false;
                        for (int64_t kk = 0; kk < cnt[q]; ++kk)
                            if (nbr_b[qb + 32 * kk] == p) {
                                found = ((w_b[qwb + 32 * (kk / 32)] >> (kk % 32)) & 1u) == bit;
                                break;
                            }
                        if (!found)
                            return fail(PD_ERR_ARG,
                                        "family/intact are not symmetric (bond %lld-%lld); the serial-order "
                                        "mode requires symmetric bonds",
                                        (long long)i + 1, (long long)(q - b.first_int + 1));
                    }
                }
            }
        }
    }
    clk.mark("family fill, sort, download", st);
    // Runtime layout (stencil or explicit per slice).
    if (layout_on_device) {
        PD_TRY(build_runtime_layout_device(env, slice_ptr, cnt, d_slice_ptr.p, d_nbr.p, d_words.p));
    } else {
        PD_TRY(build_runtime_layout(env, slice_ptr, cnt, nbr_b, w_b));
    }
    d_nbr.reset();
    d_words.reset();
    d_slice_ptr.reset();
    nbr_b.clear();
    nbr_b.shrink_to_fit();
    w_b.clear();
    w_b.shrink_to_fit();
    env->cur = 0;
    // elasto-plastic state (elasto_plastic.jl:60-68): td_norm2, edp = 0
    bool any_ep = false;
    for (auto &b : env->hb) any_ep |= b.kind == PD_MAT_ELASTO_PLASTIC;
    if (any_ep) {
        PD_TRY(env->td2.alloc(N));
        CK(cudaMemsetAsync(env->td2.p, 0, N * sizeof(double), st));
        for (auto &e : env->edp) {
            PD_TRY(e.alloc(std::max<int64_t>(env->nnz, 32)));
            CK(cudaMemsetAsync(e.p, 0, std::max<int64_t>(env->nnz, 32) * sizeof(double), st));
        }
    }
    clk.mark("runtime layout", st);
    // weighted volume (peri.jl:342-354) and intact0 (environment.jl:169)
    launch_weighted_volume(st, env->geo(), env->mth.p);
    launch_popcount(st, N, env->sinfo.p, env->cnt.p, env->words[0].p, env->intact0.p);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));

    clk.mark("weighted volume, intact0", st);
    // --- boundary conditions ---
    for (auto &hb : env->hbc) {
        DevBC d;
        std::vector<int32_t> idx(hb.env_idx.size());
        for (size_t j = 0; j < idx.size(); ++j) idx[j] = (int32_t)env->map_h[hb.env_idx[j]];
        PD_TRY(d.idx.alloc(std::max<size_t>(idx.size(), 1)));
        PD_TRY(d.last.alloc(std::max<size_t>(idx.size(), 1)));
        if (!idx.empty()) {
            CK(cudaMemcpyAsync(d.idx.p, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, st));
            CK(cudaMemsetAsync(d.last.p, 0, idx.size() * sizeof(double4), st));
        }
        d.n = (int64_t)idx.size();
        if (!hb.scale_idx.empty()) {
            std::vector<int32_t> sidx(hb.scale_idx.size());
            for (size_t j = 0; j < sidx.size(); ++j) sidx[j] = (int32_t)env->map_h[hb.scale_idx[j]];
            PD_TRY(d.sidx.alloc(sidx.size()));
            CK(cudaMemcpyAsync(d.sidx.p, sidx.data(), sidx.size() * 4, cudaMemcpyHostToDevice, st));
            d.sn = (int64_t)sidx.size();
        }
        env->bcs.push_back(std::move(d));
    }
    PD_TRY(pd::contacts_finalize(env));
    CK(cudaStreamSynchronize(st));
    clk.mark("boundary conditions, contacts", st);
    env->finalized = true;
    // release host copies of the big per-particle inputs
    for (auto &b : env->hb) {
        b.y.clear();
        b.y.shrink_to_fit();
        b.v.clear();
        b.v.shrink_to_fit();
        b.family.clear();
        b.family.shrink_to_fit();
        b.intact.clear();
        b.intact.shrink_to_fit();
    }
    return PD_OK;
}

// ---------------------------------------------------------------------
// sizes / families
// ---------------------------------------------------------------------
extern "C" pd_status pd_env_num_particles(const pd_env *env, int64_t *n) {
    PD_TRY(check_env(env));
    if (!n) return fail(PD_ERR_ARG, "n is NULL");
    *n = env->N_env;
    return PD_OK;
}

extern "C" pd_status pd_env_num_bonds(pd_env *env, int64_t *intact_bonds) {
    PD_TRY(need_final(env));
    if (!intact_bonds) return fail(PD_ERR_ARG, "intact_bonds is NULL");
    CK(cudaSetDevice(env->device));
    PD_TRY(grow(env->scr_i, env->N));
    launch_popcount(env->st, env->N, env->sinfo.p, env->cnt.p, env->words[env->cur].p, env->scr_i.p);
    std::vector<int32_t> h(env->N);
    CK(cudaMemcpyAsync(h.data(), env->scr_i.p, env->N * 4, cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    int64_t s = 0;
    for (int32_t c : h) s += c;
    *intact_bonds = s;
    return PD_OK;
}

extern "C" pd_status pd_env_family_rows(const pd_env *env, int64_t block, int64_t *rows) {
    PD_TRY(need_final(env));
    if (block < 0 || block >= (int64_t)env->hb.size() || !rows) return fail(PD_ERR_ARG, "bad block or NULL rows");
    *rows = env->hb[block].rows;
    return PD_OK;
}

extern "C" pd_status pd_env_get_family(pd_env *env, int64_t block, int64_t *family, uint8_t *intact) {
    PD_TRY(need_final(env));
    if (block < 0 || block >= (int64_t)env->hb.size()) return fail(PD_ERR_ARG, "no block %lld", (long long)block);
    CK(cudaSetDevice(env->device));
    const HostBlock &b = env->hb[block];
    const int64_t s0 = b.first_int / 32, s1 = (b.first_int + round_up(b.n, 32)) / 32;
    const SliceInfo *si = env->sinfo_h.data();
    const int64_t e0 = si[s0].nbr, e1 = si[s1].nbr, w0 = si[s0].word, w1 = si[s1].word;
    std::vector<int32_t> nb(e1 - e0);
    std::vector<uint32_t> w(w1 - w0), fm(w1 - w0);
    if (e1 > e0)
        CK(cudaMemcpyAsync(nb.data(), env->nbr.p + e0, (e1 - e0) * 4, cudaMemcpyDeviceToHost, env->st));
    if (w1 > w0) {
        CK(cudaMemcpyAsync(w.data(), env->words[env->cur].p + w0, (w1 - w0) * 4, cudaMemcpyDeviceToHost, env->st));
        CK(cudaMemcpyAsync(fm.data(), env->fam.p + w0, (w1 - w0) * 4, cudaMemcpyDeviceToHost, env->st));
    }
    CK(cudaStreamSynchronize(env->st));
    const int64_t R = b.rows;
    if (family) std::fill(family, family + (size_t)R * b.n, 0);
    if (intact) std::fill(intact, intact + (size_t)R * b.n, 0);
    for (int64_t i = 0; i < b.n; ++i) {
        const int64_t p = b.first_int + i;
        const SliceInfo &d = si[p / 32];
        const int64_t wb = d.word - w0 + (p % 32);
        int64_t r = 0;
        for (int32_t k = 0; k < env->cnt_h[p] && r < R; ++k) {
            const uint32_t bit = 1u << (k % 32);
            if (!(fm[wb + 32 * (k / 32)] & bit)) continue;
            const int64_t q = d.mode == kStencil ? p + nb[d.nbr - e0 + k] : nb[d.nbr - e0 + 32 * (int64_t)k + (p % 32)];
            if (family) family[(size_t)i * R + r] = q - b.first_int + 1;
            if (intact) intact[(size_t)i * R + r] = (w[wb + 32 * (k / 32)] & bit) != 0;
            ++r;
        }
    }
    return PD_OK;
}

static pd_status get_block_scalar(pd_env *env, int64_t block, double *out, int comp) {
    PD_TRY(need_final(env));
    if (block < 0 || block >= (int64_t)env->hb.size() || !out) return fail(PD_ERR_ARG, "bad block or NULL output");
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::sync_state_to_fp64(env, false));
    const HostBlock &b = env->hb[block];
    std::vector<double2> h(b.n);
    CK(cudaMemcpyAsync(h.data(), env->mth.p + b.first_int, b.n * sizeof(double2), cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    for (int64_t i = 0; i < b.n; ++i) out[i] = comp == 0 ? h[i].x : h[i].y;
    return PD_OK;
}

extern "C" pd_status pd_env_get_weighted_volume(pd_env *env, int64_t block, double *m) {
    return get_block_scalar(env, block, m, 0);
}

extern "C" pd_status pd_env_get_theta(pd_env *env, int64_t block, double *theta) {
    return get_block_scalar(env, block, theta, 1);
}

// ---------------------------------------------------------------------
// state
// ---------------------------------------------------------------------
static pd_status download3(pd_env *env, const double4 *src, double *dst) {
    if (!dst) return PD_OK;
    launch_pack3(env->st, env->N_env, src, env->map.p, env->stage.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, env->stage.p, 3 * env->N_env * sizeof(double), cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

static pd_status upload3(pd_env *env, const double *src, double4 *dst) {
    if (!src) return PD_OK;
    CK(cudaMemcpyAsync(env->stage.p, src, 3 * env->N_env * sizeof(double), cudaMemcpyHostToDevice, env->st));
    launch_unpack3(env->st, env->N_env, env->stage.p, env->map.p, dst);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

extern "C" pd_status pd_env_get_state(pd_env *env, double *y, double *v, double *f, double *p) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::sync_state_to_fp64(env, false));
    PD_TRY(download3(env, env->y.p, y));
    PD_TRY(download3(env, env->v.p, v));
    PD_TRY(download3(env, env->f.p, f));
    PD_TRY(download3(env, env->p.p, p));
    return PD_OK;
}

extern "C" pd_status pd_env_set_state(pd_env *env, const double *y, const double *v, const double *f) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::sync_state_to_fp64(env));
    PD_TRY(upload3(env, y, env->y.p));
    PD_TRY(upload3(env, v, env->v.p));
    PD_TRY(upload3(env, f, env->f.p));
    env->fast_valid = false;
    return PD_OK;
}

extern "C" pd_status pd_env_get_mass(pd_env *env, double *mass, double *volume, double *density) {
    PD_TRY(need_final(env));
    for (const auto &b : env->hb)
        for (int64_t i = 0; i < b.n; ++i) {
            double m = b.vol[i] * b.dens[b.type[i] - b.type_start];
            if (mass) mass[b.first_env + i] = m;
            if (volume) volume[b.first_env + i] = b.vol[i];
            if (density) density[b.first_env + i] = m / b.vol[i];
        }
    return PD_OK;
}

extern "C" pd_status pd_env_get_time_step(const pd_env *env, int64_t *ts) {
    PD_TRY(check_env(env));
    if (!ts) return fail(PD_ERR_ARG, "time_step is NULL");
    *ts = env->ts;
    return PD_OK;
}

extern "C" pd_status pd_env_set_time_step(pd_env *env, int64_t ts) {
    PD_TRY(check_env(env));
    env->ts = ts;
    return PD_OK;
}

extern "C" pd_status pd_env_reset_deformed(pd_env *env) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::fast_land_flags(env));
    std::vector<int32_t> h(env->deformed0.begin(), env->deformed0.end());
    CK(cudaMemcpyAsync(env->deformed.p, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice, env->st));
    CK(cudaStreamSynchronize(env->st));
    env->deformed_h = env->deformed0;
    return PD_OK;
}

extern "C" pd_status pd_env_set_deformed(pd_env *env, const uint8_t *flags, int32_t hold) {
    PD_TRY(need_final(env));
    if (!flags) return fail(PD_ERR_ARG, "flags is NULL");
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::fast_land_flags(env));
    std::vector<int32_t> h(env->hb.size());
    for (size_t b = 0; b < h.size(); ++b) h[b] = flags[b] ? 1 : 0;
    CK(cudaMemcpyAsync(env->deformed.p, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice, env->st));
    CK(cudaStreamSynchronize(env->st));
    env->deformed_h.assign(h.begin(), h.end());
    env->gate_hold = hold != 0;
    return PD_OK;
}

extern "C" pd_status pd_env_reset_bonds(pd_env *env) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    size_t nw = std::max<int64_t>(env->nnz / 32, 1) * 4;
    CK(cudaMemcpyAsync(env->words[0].p, env->words0.p, nw, cudaMemcpyDeviceToDevice, env->st));
    CK(cudaMemcpyAsync(env->words[1].p, env->words0.p, nw, cudaMemcpyDeviceToDevice, env->st));
    env->cur = 0;
    for (auto &e : env->edp)  // elasto-plastic bond state starts over with the bonds
        if (e.p) CK(cudaMemsetAsync(e.p, 0, std::max<int64_t>(env->nnz, 32) * sizeof(double), env->st));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

// ---------------------------------------------------------------------
// diagnostics
// ---------------------------------------------------------------------
static pd_status damage_internal(pd_env *env, std::vector<double> &dint) {
    PD_TRY(grow(env->scr_d, env->N));
    launch_damage(env->st, env->N, env->sinfo.p, env->cnt.p, env->words[env->cur].p, env->intact0.p,
                  env->tinfo.p, env->scr_d.p);
    CK(cudaGetLastError());
    dint.resize(env->N);
    CK(cudaMemcpyAsync(dint.data(), env->scr_d.p, env->N * sizeof(double), cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

extern "C" pd_status pd_env_intact0(pd_env *env, int64_t *intact0) {
    PD_TRY(need_final(env));
    if (!intact0) return fail(PD_ERR_ARG, "intact0 is NULL");
    CK(cudaSetDevice(env->device));
    std::vector<int32_t> h(env->N);
    CK(cudaMemcpyAsync(h.data(), env->intact0.p, env->N * sizeof(int32_t), cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    for (int64_t e = 0; e < env->N_env; ++e) intact0[e] = h[env->map_h[e]];
    return PD_OK;
}

extern "C" pd_status pd_env_damage(pd_env *env, double *damage) {
    PD_TRY(need_final(env));
    if (!damage) return fail(PD_ERR_ARG, "damage is NULL");
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::sync_state_to_fp64(env, false));
    std::vector<double> dint;
    PD_TRY(damage_internal(env, dint));
    for (int64_t e = 0; e < env->N_env; ++e) damage[e] = dint[env->map_h[e]];
    return PD_OK;
}

extern "C" pd_status pd_env_diagnostics(pd_env *env, double *out8) {
    PD_TRY(need_final(env));
    if (!out8) return fail(PD_ERR_ARG, "out is NULL");
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::sync_state_to_fp64(env, false));
    double h[3];
    launch_sum4(env->st, env->N, env->p.p, env->partials.p, env->out3.p);
    CK(cudaMemcpyAsync(h, env->out3.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    out8[0] = h[0];
    out8[1] = h[1];
    out8[2] = h[2];
    launch_sum4(env->st, env->N, env->f.p, env->partials.p, env->out3.p);
    CK(cudaMemcpyAsync(h, env->out3.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    out8[3] = h[0];
    out8[4] = h[1];
    out8[5] = h[2];
    std::vector<double> dint;
    PD_TRY(damage_internal(env, dint));
    double s = 0.0;
    for (int64_t e = 0; e < env->N_env; ++e) s += dint[env->map_h[e]];
    out8[6] = env->N_env > 0 ? s / (double)env->N_env : 0.0;
    int64_t nb = 0;
    PD_TRY(pd_env_num_bonds(env, &nb));
    out8[7] = (double)nb;
    return PD_OK;
}

extern "C" pd_status pd_env_deformed(pd_env *env, uint8_t *flags) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    std::vector<int32_t> h(env->hb.size());
    CK(cudaMemcpyAsync(h.data(), env->deformed.p, h.size() * 4, cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    bool all = true;
    for (size_t b = 0; b < h.size(); ++b) {
        env->deformed_h[b] = h[b];
        if (flags) flags[b] = (uint8_t)(h[b] != 0);
        if (env->hb[b].kind != PD_MAT_SKIP) all &= h[b] != 0;
    }
    (void)all;
    return PD_OK;
}

extern "C" pd_status pd_env_check_finite(pd_env *env) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(pd::sync_state_to_fp64(env, false));
    CK(cudaMemsetAsync(env->flag.p, 0, 4, env->st));
    launch_nonfinite(env->st, env->N, env->y.p, env->flag.p);
    launch_nonfinite(env->st, env->N, env->v.p, env->flag.p);
    launch_nonfinite(env->st, env->N, env->f.p, env->flag.p);
    int32_t h = 0;
    CK(cudaMemcpyAsync(&h, env->flag.p, 4, cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    if (h) return fail(PD_ERR_NAN, "NaN or Inf in y, v or f");
    return PD_OK;
}

extern "C" pd_status pd_env_layout(const pd_env *env, int64_t *out4) {
    PD_TRY(need_final(env));
    if (!out4) return fail(PD_ERR_ARG, "out4 is NULL");
    out4[0] = env->N / kSlice;
    out4[1] = env->stencil_slices;
    out4[2] = env->nnz;
    out4[3] = env->nbr_len;
    return PD_OK;
}

extern "C" pd_status pd_env_layout_stats(const pd_env *env, int64_t *out, int64_t n) {
    PD_TRY(need_final(env));
    if (!out || n < 0) return fail(PD_ERR_ARG, "out is NULL or n < 0");
    const int64_t v[6] = {env->N / kSlice, env->stencil_slices, env->nnz, env->nbr_len, env->splan_slices,
                          env->walked};
    for (int64_t i = 0; i < n && i < 6; ++i) out[i] = v[i];
    return PD_OK;
}

// ---------------------------------------------------------------------
// instrumentation
// ---------------------------------------------------------------------
extern "C" pd_status pd_env_stream(pd_env *env, void **stream) {
    PD_TRY(check_env(env));
    if (!stream) return fail(PD_ERR_ARG, "stream is NULL");
    *stream = (void *)env->st;
    return PD_OK;
}

extern "C" pd_status pd_kernel_launches(int64_t *count) {
    if (!count) return fail(PD_ERR_ARG, "count is NULL");
    *count = g_launches.load(std::memory_order_relaxed);
    return PD_OK;
}

static pd_status prof_collect(pd_env *env) {
    if (env->prof_used == 0) return PD_OK;
    CK(cudaStreamSynchronize(env->st));
    for (size_t k = 0; k + 1 < env->prof_used; k += 2) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, env->prof_ev[k], env->prof_ev[k + 1]));
        env->prof_ms += ms;
        env->prof_launches += env->prof_w[k / 2];
    }
    env->prof_used = 0;
    return PD_OK;
}

extern "C" pd_status pd_env_profile(pd_env *env, int32_t enable) {
    PD_TRY(check_env(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(prof_collect(env));
    env->prof = enable != 0;
    env->prof_ms = 0.0;
    env->prof_launches = 0;
    return PD_OK;
}

extern "C" pd_status pd_env_profile_read(pd_env *env, double *total_ms, int64_t *launches) {
    PD_TRY(check_env(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(prof_collect(env));
    if (total_ms) *total_ms = env->prof_ms;
    if (launches) *launches = env->prof_launches;
    return PD_OK;
}

namespace pd {
int64_t footprint_estimate(const pd_env *env) {
    // per particle: FP64 state and tables (~300 B), throughput-mode records
    // (~250 B); per bond slot: build-layout index + bits (4.2 B, transient)
    // and runtime bits (4 arrays) + explicit index (4.5 B)
    int64_t bytes = 64ll << 20;  // stream, scratch, reductions
    for (const auto &b : env->hb) {
        const int64_t np = (b.n + 31) / 32 * 32;
        const int64_t rows = b.host_family ? std::max<int64_t>(b.rows, 1) : std::min<int64_t>(b.max_neigh, b.n);
        bytes += np * 560 + np * rows * 9;
    }
    for (const auto &c : env->hc) {
        const int64_t n1 = env->hb[c.b1].n;
        bytes += n1 * std::max<int64_t>(c.max_neighs, 1) * 8 + (64ll << 10);
    }
    return bytes;
}
}  // namespace pd

// ---------------------------------------------------------------------
// output staging
// ---------------------------------------------------------------------
extern "C" pd_status pd_env_stage_state(pd_env *env, int32_t slot) {
    PD_TRY(need_final(env));
    if (slot < 0 || slot > 1) return fail(PD_ERR_ARG, "slot must be 0 or 1");
    CK(cudaSetDevice(env->device));
    auto &S = env->slots[slot];
    const int64_t NE = env->N_env, N = env->N;
    const size_t count = (size_t)(9 * NE + N);  // y, v, f packed (3 x NE each) + damage (internal order)
    if (!S.host) {
        if (!env->copy_st) CK(cudaStreamCreateWithFlags(&env->copy_st, cudaStreamNonBlocking));
        PD_TRY(S.dev.alloc(count));
        CK(cudaMallocHost(&S.host, count * sizeof(double)));
        CK(cudaEventCreateWithFlags(&S.packed, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming));
    }
    if (S.pending) CK(cudaEventSynchronize(S.done));  // the slot's previous copy is still in flight
    PD_TRY(pd::sync_state_to_fp64(env, false));
    launch_pack3(env->st, NE, env->y.p, env->map.p, S.dev.p);
    launch_pack3(env->st, NE, env->v.p, env->map.p, S.dev.p + 3 * NE);
    launch_pack3(env->st, NE, env->f.p, env->map.p, S.dev.p + 6 * NE);
    launch_damage(env->st, N, env->sinfo.p, env->cnt.p, env->words[env->cur].p, env->intact0.p, env->tinfo.p,
                  S.dev.p + 9 * NE);
    CK(cudaGetLastError());
    CK(cudaEventRecord(S.packed, env->st));
    CK(cudaStreamWaitEvent(env->copy_st, S.packed, 0));
    CK(cudaMemcpyAsync(S.host, S.dev.p, count * sizeof(double), cudaMemcpyDeviceToHost, env->copy_st));
    CK(cudaEventRecord(S.done, env->copy_st));
    S.pending = true;
    S.ts = env->ts;
    return PD_OK;
}

extern "C" pd_status pd_env_stage_read(pd_env *env, int32_t slot, double *y, double *v, double *f, double *damage,
                                       int64_t *time_step) {
    PD_TRY(need_final(env));
    if (slot < 0 || slot > 1) return fail(PD_ERR_ARG, "slot must be 0 or 1");
    auto &S = env->slots[slot];
    if (!S.pending) return fail(PD_ERR_STATE, "nothing staged in slot %d", slot);
    CK(cudaSetDevice(env->device));
    CK(cudaEventSynchronize(S.done));
    const int64_t NE = env->N_env;
    if (y) std::memcpy(y, S.host, 3 * NE * sizeof(double));
    if (v) std::memcpy(v, S.host + 3 * NE, 3 * NE * sizeof(double));
    if (f) std::memcpy(f, S.host + 6 * NE, 3 * NE * sizeof(double));
    if (damage)
        for (int64_t e = 0; e < NE; ++e) damage[e] = S.host[9 * NE + env->map_h[e]];
    if (time_step) *time_step = S.ts;
    S.pending = false;
    return PD_OK;
}

extern "C" pd_status pd_env_get_plastic_strain(pd_env *env, int64_t block, double *edp) {
    PD_TRY(need_final(env));
    if (block < 0 || block >= (int64_t)env->hb.size() || !edp) return fail(PD_ERR_ARG, "bad block or NULL edp");
    const HostBlock &b = env->hb[block];
    if (b.kind != PD_MAT_ELASTO_PLASTIC) return fail(PD_ERR_ARG, "block %lld is not elasto-plastic", (long long)block);
    CK(cudaSetDevice(env->device));
    const int64_t s0 = b.first_int / 32, s1 = (b.first_int + round_up(b.n, 32)) / 32;
    const SliceInfo *si = env->sinfo_h.data();
    const int64_t w0 = si[s0].word, w1 = si[s1].word;
    std::vector<uint32_t> fm(w1 - w0);
    std::vector<double> e(32 * (w1 - w0));
    if (w1 > w0) {
        CK(cudaMemcpyAsync(fm.data(), env->fam.p + w0, (w1 - w0) * 4, cudaMemcpyDeviceToHost, env->st));
        CK(cudaMemcpyAsync(e.data(), env->edp[env->ecur].p + 32 * w0, 32 * (w1 - w0) * sizeof(double),
                           cudaMemcpyDeviceToHost, env->st));
    }
    CK(cudaStreamSynchronize(env->st));
    const int64_t R = b.rows;
    std::fill(edp, edp + (size_t)R * b.n, 0.0);
    for (int64_t i = 0; i < b.n; ++i) {
        const int64_t p = b.first_int + i;
        const int64_t wb = si[p / 32].word - w0 + (p % 32);
        int64_t r = 0;
        for (int32_t k = 0; k < env->cnt_h[p] && r < R; ++k) {
            const int64_t w = wb + 32 * (k / 32);
            if (!((fm[w] >> (k % 32)) & 1u)) continue;
            edp[(size_t)i * R + r] = e[32 * w + (k % 32)];
            ++r;
        }
    }
    return PD_OK;
}

// pd_solver.cu -- solver sequencing of src/solvers/*.jl on the device:
// update_acc!, velocity_verlet_step!, minimize! (QSDrag), apply_bc_at0,
// and the block-level device-pointer entry point.  Compiled with
// -fmad=false (the QSDrag update below must round like the reference).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pd_env_impl.h"

using namespace pd;

void pd_env::release_device() {
    fast_release(this);
    map.reset();
    x4.reset();
    y.reset();
    v.reset();
    f.reset();
    p.reset();
    mass.reset();
    dens.reset();
    tdens.reset();
    tinfo.reset();
    cnt.reset();
    intact0.reset();
    deformed.reset();
    sinfo.reset();
    fam.reset();
    nbr.reset();
    words[0].reset();
    words[1].reset();
    words0.reset();
    mth.reset();
    blocks_d.reset();
    pairs.reset();
    partials.reset();
    out3.reset();
    stage.reset();
    flag.reset();
    bcs.clear();
    contacts.clear();
    tmp_y.reset();
    scr_d.reset();
    scr_i.reset();
    splan_off.reset();
    splan.reset();
    spos.reset();
    tmp_f.reset();
    opt.reset();
    free_mask.reset();
    red.reset();
}

namespace {

pd_status need_final(const pd_env *env) {
    if (!env) return fail(PD_ERR_ARG, "environment handle is NULL");
    if (!env->finalized) return fail(PD_ERR_STATE, "environment is not finalized (call pd_env_finalize)");
    return PD_OK;
}

pd::BCDev bc_view(pd_env *env, size_t k) {
    const HostBC &h = env->hbc[k];
    DevBC &d = env->bcs[k];
    BCDev b;
    b.kind = h.kind;
    b.dims = h.dims;
    for (int i = 0; i < 3; ++i) b.rate[i] = h.rate[i];
    for (int i = 0; i < 3; ++i) {
        b.scale[i] = h.scale[i];
        b.fix[i] = h.fix[i];
        b.lo[i] = h.lo[i];
        b.hi[i] = h.hi[i];
    }
    b.has_limits = h.has_limits;
    b.pad = 0;
    b.n = d.n;
    b.idx = d.idx.p;
    b.last = d.last.p;
    b.sn = d.sn;
    b.sidx = d.sidx.p;
    return b;
}

// ToFroBC.jl:101-105 check!: flip when time_step > applyafter and
// time_step % freq == 0 (Int % Float64 is rem).
// ScaleFixWaitBC.jl:63-68 check!: at time_step % wait == 0 scale the
// scalebool particles about the fix point and re-read last.
void bc_check(pd_env *env) {
    for (size_t k = 0; k < env->hbc.size(); ++k) {
        auto &h = env->hbc[k];
        if (h.scales_at(env->ts)) launch_bc_scale(env->st, bc_view(env, k), env->dt, env->y.p);
        if (h.kind != PD_BC_TOFRO) continue;
        double r = std::fmod((double)env->ts, h.freq);
        if ((env->ts > h.applyafter) && (r == 0.0)) h.dir = -h.dir;
    }
}

__device__ __forceinline__ double jl_min(double x, double y) {
    if (x != x || y != y) return x + y;  // NaN propagates
    if (x < y) return x;
    if (y < x) return y;
    return signbit(x) ? x : y;
}
__device__ __forceinline__ double jl_max(double x, double y) {
    if (x != x || y != y) return x + y;
    if (x > y) return x;
    if (y > x) return y;
    return signbit(x) ? y : x;
}

__device__ __forceinline__ double nanmax(double a, double b) {
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000LL);
    return a > b ? a : b;
}

// Fixed partial-reduction width, independent of the device's SM count so
// that the reduction order is the same on every GPU.
constexpr int kRedBlocks = 148;
// Largest number of CTAs sharing one block in the gate's partial norms
// (fixed for the same reason).
constexpr int kGateWidth = 148;

// minimize.jl:149-155 apply_! and :202 y[:, mask] .+= dy, fused with the
// max|f| / max|dy| reductions of :204.
__global__ void __launch_bounds__(256)
    k_qs_apply(int64_t N, const int32_t *__restrict__ freem, const double4 *__restrict__ f,
               double4 *__restrict__ opt, double4 *__restrict__ y, double lambda, double kk,
               double ss, double a, double *__restrict__ partial) {
    __shared__ double sf[256], sy[256];
    double mf = 0.0, my = 0.0;
    for (int64_t i = blockIdx.x * 256 + threadIdx.x; i < N; i += (int64_t)kRedBlocks * 256) {
        if (!freem[i]) continue;
        double4 fi = f[i], oi = opt[i], yi = y[i];
        double fo[3] = {fi.x, fi.y, fi.z}, o[3] = {oi.x, oi.y, oi.z}, yy[3] = {yi.x, yi.y, yi.z};
        for (int d = 0; d < 3; ++d) {
            double force = fo[d] - lambda * o[d] * (1.0 + kk * fabs(o[d]));
            double dy = 0.5 * force * (ss * ss) + o[d] * ss;
            o[d] = o[d] + ss * force;
            dy = jl_max(jl_min(dy, a), -a);
            yy[d] = yy[d] + dy;
            mf = nanmax(mf, fabs(fo[d]));
            my = nanmax(my, fabs(dy));
        }
        opt[i] = make_double4(o[0], o[1], o[2], 0.0);
        y[i] = make_double4(yy[0], yy[1], yy[2], yi.w);
    }
    sf[threadIdx.x] = mf;
    sy[threadIdx.x] = my;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sf[threadIdx.x] = nanmax(sf[threadIdx.x], sf[threadIdx.x + s]);
            sy[threadIdx.x] = nanmax(sy[threadIdx.x], sy[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = sf[0];
        partial[2 * blockIdx.x + 1] = sy[0];
    }
}

__global__ void k_qs_final(const double *__restrict__ partial, double *__restrict__ out2) {
    double mf = 0.0, my = 0.0;
    for (int b = 0; b < kRedBlocks; ++b) {
        mf = nanmax(mf, partial[2 * b]);
        my = nanmax(my, partial[2 * b + 1]);
    }
    out2[0] = mf;
    out2[1] = my;
}

__global__ void k_set_free(int64_t N, const int32_t *__restrict__ tinfo, int32_t *__restrict__ freem) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    freem[i] = tinfo[i] >= 0 ? 1 : 0;
}

__global__ void k_clear_idx(int64_t n, const int32_t *__restrict__ idx, int32_t *__restrict__ freem) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    freem[idx[j]] = 0;
}

}  // namespace

namespace pd {

// update_acc! (solvers.jl:320-336) in serial-order FP64.
pd_status update_acc_serial(pd_env *env) {
    cudaStream_t st = env->st;
    Geo g = env->geo();
    // force_density! gate for blocks still undeformed
    std::vector<GateItem> items;
    for (size_t b = 0; b < env->hb.size() && !env->gate_hold; ++b) {
        const HostBlock &hb = env->hb[b];
        if (hb.kind == PD_MAT_SKIP || env->deformed_h[b]) continue;
        items.push_back(GateItem{hb.first_int, hb.n, (int32_t)b, 0});
    }
    if (!items.empty()) {
        const int ni = (int)items.size();
        const int gx = std::max(1, std::min(kGateWidth, (kGateWidth * 8) / ni));
        if (env->gate_items_h.size() != items.size() ||
            std::memcmp(env->gate_items_h.data(), items.data(), items.size() * sizeof(GateItem)) != 0) {
            PD_TRY(grow(env->gate_items, (int64_t)items.size()));
            PD_TRY(grow(env->gate_part, 3 * (int64_t)ni * gx));
            CK(cudaMemcpyAsync(env->gate_items.p, items.data(), items.size() * sizeof(GateItem),
                               cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
            env->gate_items_h = items;
        }
        launch_gate_multi(st, env->gate_items.p, ni, gx, env->x4.p, env->y.p, env->gate_part.p, env->deformed.p);
    }
    // out_of_loop!: dilatation for state-based blocks
    bool any_lps = false, any_ep = false;
    for (const auto &hb : env->hb) {
        any_lps |= hb.kind == PD_MAT_ORDINARY_STATE_BASED || hb.kind == PD_MAT_ELASTO_PLASTIC;
        any_ep |= hb.kind == PD_MAT_ELASTO_PLASTIC;
    }
    if (any_lps) launch_theta_serial(st, g, env->y.p, env->words[env->cur].p, env->mth.p, 0, env->N);
    if (any_ep) {
        // elasto_plastic.jl:170-171: td_norm2 pass (breaks bonds), then the
        // bond loop on its flags, back into words[cur]; edp is double-buffered
        launch_td_serial(st, g, env->y.p, env->mth.p, env->words[env->cur].p, env->words[1 - env->cur].p, 0,
                         env->N);
        prof_begin(env, st);
        launch_force_serial(st, g, env->y.p, env->mth.p, env->words[1 - env->cur].p, env->words[env->cur].p,
                            env->f.p, 0, 0, env->N);
        prof_end(env, st);
        env->ecur = 1 - env->ecur;
    } else {
        // fill!(f, 0) + force_density_T! for every block
        prof_begin(env, st);
        launch_force_serial(st, g, env->y.p, env->mth.p, env->words[env->cur].p, env->words[1 - env->cur].p,
                            env->f.p, 0, 0, env->N);
        prof_end(env, st);
        env->cur = 1 - env->cur;
    }
    CK(cudaGetLastError());
    // short_range_contact!
    PD_TRY(contacts_force(env));
    // update_misc!
    launch_momentum(st, env->N, env->mass.p, env->v.p, env->p.p);
    CK(cudaGetLastError());
    return PD_OK;
}

pd_status refresh_deformed(pd_env *env) {
    bool all = true;
    for (size_t b = 0; b < env->hb.size(); ++b)
        if (env->hb[b].kind != PD_MAT_SKIP && !env->deformed_h[b]) all = false;
    if (all) return PD_OK;
    std::vector<int32_t> h(env->hb.size());
    CK(cudaMemcpyAsync(h.data(), env->deformed.p, h.size() * 4, cudaMemcpyDeviceToHost, env->st));
    CK(cudaStreamSynchronize(env->st));
    for (size_t b = 0; b < h.size(); ++b) env->deformed_h[b] = h[b];
    return PD_OK;
}

}  // namespace pd

extern "C" pd_status pd_env_update_acc(pd_env *env) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    if (env->precision != PD_PREC_FP64_SERIAL) return fast_update_acc(env);
    PD_TRY(sync_state_to_fp64(env));
    PD_TRY(update_acc_serial(env));
    PD_TRY(refresh_deformed(env));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

extern "C" pd_status pd_env_apply_bc_at0(pd_env *env) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(sync_state_to_fp64(env, false));
    for (size_t k = 0; k < env->hbc.size(); ++k)
        if (env->hbc[k].kind != PD_BC_CONTAINER)  // ContainerBC.jl:84 does nothing
            launch_bc_snapshot(env->st, bc_view(env, k), env->y.p);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

// velocity_verlet.jl:57-89, nsteps times, in the serial mode, enqueued on
// the environment's stream.
static pd_status serial_steps(pd_env *env, int64_t nsteps) {
    const double c = env->dt / 2;
    const double dt = env->dt;
    for (int64_t s = 0; s < nsteps; ++s) {
        launch_kick_drift(env->st, env->N, c, dt, env->f.p, env->v.p, env->y.p);
        for (size_t k = 0; k < env->hbc.size(); ++k)
            launch_bc_pos(env->st, bc_view(env, k), dt, env->hbc[k].dir, env->ts, env->y.p);
        PD_TRY(update_acc_serial(env));
        launch_kick(env->st, env->N, c, env->f.p, env->v.p);
        for (size_t k = 0; k < env->hbc.size(); ++k)
            launch_bc_vel(env->st, bc_view(env, k), env->hbc[k].dir, env->y.p, env->v.p);
        bc_check(env);
        env->ts += 1;
        if ((s & 63) == 63) CK(cudaGetLastError());
    }
    CK(cudaGetLastError());
    return PD_OK;
}

extern "C" pd_status pd_env_vv_steps(pd_env *env, int64_t nsteps) {
    PD_TRY(need_final(env));
    if (nsteps < 0) return fail(PD_ERR_ARG, "nsteps < 0");
    CK(cudaSetDevice(env->device));
    if (env->precision != PD_PREC_FP64_SERIAL) return fast_vv_steps(env, nsteps);
    PD_TRY(serial_steps(env, nsteps));
    PD_TRY(refresh_deformed(env));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

// pd_env_vv_steps without the final wait: the steps are enqueued on the
// environment's stream.  Only an environment whose deformed flags the host
// already knows (every block deformed, or the gate held) can skip the
// read-back; others wait as pd_env_vv_steps does.
extern "C" pd_status pd_env_vv_steps_async(pd_env *env, int64_t nsteps) {
    PD_TRY(need_final(env));
    if (nsteps < 0) return fail(PD_ERR_ARG, "nsteps < 0");
    bool known = env->gate_hold;
    if (!known) {
        known = true;
        for (size_t b = 0; b < env->hb.size(); ++b)
            if (env->hb[b].kind != PD_MAT_SKIP && !env->deformed_h[b]) known = false;
    }
    if (!known) return pd_env_vv_steps(env, nsteps);
    CK(cudaSetDevice(env->device));
    if (env->precision != PD_PREC_FP64_SERIAL) return fast_vv_enqueue(env, nsteps);
    return serial_steps(env, nsteps);
}

// minimize.jl:105-231 (one QSDrag solver step).
extern "C" pd_status pd_env_qsdrag(pd_env *env, double step_size, double drag, int64_t max_iter,
                                   double x_tol, double f_tol, int64_t *iters) {
    PD_TRY(need_final(env));
    if (max_iter < 1) return fail(PD_ERR_ARG, "max_iter must be >= 1");
    CK(cudaSetDevice(env->device));
    PD_TRY(sync_state_to_fp64(env));
    cudaStream_t st = env->st;
    const int64_t N = env->N;
    // :112-115 apply BCs (position then velocity, per BC)
    for (size_t k = 0; k < env->hbc.size(); ++k) {
        launch_bc_pos(st, bc_view(env, k), env->dt, env->hbc[k].dir, env->ts, env->y.p);
        launch_bc_vel(st, bc_view(env, k), env->hbc[k].dir, env->y.p, env->v.p);
    }
    const double dt = step_size;
    const double ps = env->hb[0].particle_size;
    // :138-145 free particles: not in any BC that acts beyond the start
    if (!env->free_mask.p) PD_TRY(env->free_mask.alloc(N));
    if (!env->opt.p) PD_TRY(env->opt.alloc(N));
    if (!env->red.p) PD_TRY(env->red.alloc(2 * kRedBlocks + 2));
    k_set_free<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(N, env->tinfo.p, env->free_mask.p); pd::note_launch();
    for (size_t k = 0; k < env->hbc.size(); ++k)
        if (!env->hbc[k].onlyatstart && env->bcs[k].n > 0)
            k_clear_idx<<<(unsigned)((env->bcs[k].n + 255) / 256), 256, 0, st>>>(env->bcs[k].n, env->bcs[k].idx.p,
                                                                                  env->free_mask.p); pd::note_launch();
    // :146 opt = zero(f[:, mask]); :147 k = lambda/10
    CK(cudaMemsetAsync(env->opt.p, 0, N * sizeof(double4), st));
    const double lambda = drag;
    const double kk = lambda / 10;
    const double a = ps / 10;
    int64_t it = 0;
    for (int64_t i = 1; i <= max_iter; ++i) {
        it = i;
        PD_TRY(update_acc_serial(env));
        k_qs_apply<<<kRedBlocks, 256, 0, st>>>(N, env->free_mask.p, env->f.p, env->opt.p, env->y.p, lambda, kk,
                                               step_size, a, env->red.p); pd::note_launch();
        k_qs_final<<<1, 1, 0, st>>>(env->red.p, env->red.p + 2 * kRedBlocks); pd::note_launch();
        CK(cudaGetLastError());
        double h[2];
        CK(cudaMemcpyAsync(h, env->red.p + 2 * kRedBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if ((h[0] < f_tol) && (h[1] < x_tol)) break;
    }
    (void)dt;
    bc_check(env);
    env->ts += 1;
    PD_TRY(refresh_deformed(env));
    CK(cudaStreamSynchronize(st));
    if (iters) *iters = it;
    return PD_OK;
}

extern "C" pd_status pd_env_update_neighs(pd_env *env, int64_t max_part) {
    PD_TRY(need_final(env));
    CK(cudaSetDevice(env->device));
    PD_TRY(sync_state_to_fp64(env, false));
    PD_TRY(contacts_update_neighs(env, max_part));
    CK(cudaStreamSynchronize(env->st));
    return PD_OK;
}

// force_density_T!(f, y, limits, mat, Val{:cuda}) on caller-owned device
// arrays (3 x N_env column-major).
extern "C" pd_status pd_force_density_device(pd_env *env, int64_t block, double *f_dev,
                                             const double *y_dev, void *stream) {
    PD_TRY(need_final(env));
    if (block < 0 || block >= (int64_t)env->hb.size()) return fail(PD_ERR_ARG, "no block %lld", (long long)block);
    if (!f_dev || !y_dev) return fail(PD_ERR_ARG, "f/y device pointer is NULL");
    if (env->precision != PD_PREC_FP64_SERIAL)
        return fail(PD_ERR_UNSUPPORTED, "pd_force_density_device requires PD_PREC_FP64_SERIAL");
    CK(cudaSetDevice(env->device));
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, f_dev) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
        at.device != env->device || cudaPointerGetAttributes(&at, y_dev) != cudaSuccess ||
        at.type != cudaMemoryTypeDevice || at.device != env->device) {
        cudaGetLastError();
        return fail(PD_ERR_ARG, "f/y must be device pointers on the environment's device %d", env->device);
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : env->st;
    const HostBlock &hb = env->hb[block];
    if (hb.kind == PD_MAT_ELASTO_PLASTIC)
        return fail(PD_ERR_UNSUPPORTED, "the device-pointer entry point does not evaluate elasto-plastic blocks");
    if (!env->tmp_y.p) PD_TRY(env->tmp_y.alloc(env->N));
    if (!env->tmp_f.p) PD_TRY(env->tmp_f.alloc(env->N));
    const int64_t *map = env->map.p + hb.first_env;
    launch_unpack3(st, hb.n, y_dev + 3 * hb.first_env, map, env->tmp_y.p);
    launch_unpack3(st, hb.n, f_dev + 3 * hb.first_env, map, env->tmp_f.p);
    Geo g = env->geo();
    int64_t p0 = hb.first_int, p1 = hb.first_int + ((hb.n + 31) / 32) * 32;
    if (hb.kind == PD_MAT_ORDINARY_STATE_BASED)
        launch_theta_serial(st, g, env->tmp_y.p, env->words[env->cur].p, env->mth.p, p0, p1);
    // force_density_T! itself has no gate: compute unconditionally
    std::vector<int32_t> one(1, 1);
    CK(cudaMemcpyAsync(env->deformed.p + block, one.data(), 4, cudaMemcpyHostToDevice, st));
    launch_force_serial(st, g, env->tmp_y.p, env->mth.p, env->words[env->cur].p, env->words[1 - env->cur].p,
                        env->tmp_f.p, 1, p0, p1);
    int64_t w0 = env->sinfo_h[p0 / 32].word, w1 = env->sinfo_h[p1 / 32].word;
    if (w1 > w0)
        CK(cudaMemcpyAsync(env->words[env->cur].p + w0, env->words[1 - env->cur].p + w0, (w1 - w0) * 4,
                           cudaMemcpyDeviceToDevice, st));
    launch_pack3(st, hb.n, env->tmp_f.p, map, f_dev + 3 * hb.first_env);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    env->deformed_h[block] = 1;
    return PD_OK;
}

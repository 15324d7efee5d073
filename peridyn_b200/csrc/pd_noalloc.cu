// pd_noalloc.cu -- pd_force_density_device_static: the block force
// evaluation of pd_force_density_device with its scratch in a fixed,
// file-scope device array, so that the call itself allocates nothing.
//
// Who needs it: a host whose device memory is owned by another allocator
// (for example a Julia session in which CUDA.jl's memory pool holds the
// GPU and foreign cudaMalloc calls would fragment or exceed it), and code
// that must not pay the implicit device synchronisation cudaMalloc/cudaFree
// can cause in the middle of a time step.  pd_force_density_device
// allocates two staging buffers on its first call; this variant uses the
// static array below instead.
//
// Limits and sharing:
//  * one block of at most kStaticMaxParticles particles (after padding the
//    block to a multiple of 32); larger blocks are rejected with
//    PD_ERR_UNSUPPORTED before anything is launched;
//  * the array exists once per GPU that loads the library and stays
//    allocated until the process exits (2 x 65536 x 32 B = 4 MiB);
//  * every call on a GPU uses the same array: calls whose work overlaps on
//    that GPU (different streams, host threads or environments) race and
//    must be serialised by the caller;
//  * the array keeps the last call's contents; every element a call reads
//    is written by the same call first, so nothing needs clearing;
//  * the first call on each device looks the array's address up with
//    cudaGetSymbolAddress (with that device current); make that first call
//    before any stream capture on the device;
//  * the address is kept for the life of the process, so the device must
//    not be reset (cudaDeviceReset) while the library is loaded, and calls
//    must come from the device's primary context (the runtime API's
//    default, which CUDA.jl also uses).
#include <mutex>

#include "pd_env_impl.h"

using namespace pd;

namespace {

constexpr int64_t kStaticMaxParticles = 65536;
constexpr int kMaxDevices = 64;

// [0, kStaticMaxParticles): unpacked positions; [kStaticMaxParticles, 2x):
// the force accumulator of the block.
static __device__ __align__(256) double4 g_static_scratch[2 * kStaticMaxParticles];

std::mutex g_setup_mutex;
double4 *g_scratch_addr[kMaxDevices] = {};

// Device address of g_static_scratch on `device` (looked up once, with the
// device current).  Host code must not pass g_static_scratch itself to a
// kernel: on the host that name is a stand-in, not a device address.
pd_status scratch_for(int device, double4 **out) {
    if (device < 0 || device >= kMaxDevices) return fail(PD_ERR_UNSUPPORTED, "device index %d too large", device);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(PD_ERR_CUDA, "cudaGetSymbolAddress(g_static_scratch) failed: %s", cudaGetErrorString(e));
        }
        g_scratch_addr[device] = (double4 *)p;
    }
    *out = g_scratch_addr[device];
    return PD_OK;
}

const int32_t kOne = 1;

}  // namespace

extern "C" pd_status pd_force_density_device_static(pd_env *env, int64_t block, double *f_dev,
                                                    const double *y_dev, void *stream) {
    if (!env) return fail(PD_ERR_ARG, "environment handle is NULL");
    if (!env->finalized) return fail(PD_ERR_STATE, "environment is not finalized (call pd_env_finalize)");
    if (block < 0 || block >= (int64_t)env->hb.size()) return fail(PD_ERR_ARG, "no block %lld", (long long)block);
    if (!f_dev || !y_dev) return fail(PD_ERR_ARG, "f/y device pointer is NULL");
    if (env->precision != PD_PREC_FP64_SERIAL)
        return fail(PD_ERR_UNSUPPORTED, "pd_force_density_device_static requires PD_PREC_FP64_SERIAL");
    const HostBlock &hb = env->hb[block];
    const int64_t n_pad = ((hb.n + 31) / 32) * 32;
    if (n_pad > kStaticMaxParticles)
        return fail(PD_ERR_UNSUPPORTED,
                    "block has %lld particles (%lld padded); the static scratch holds at most %lld",
                    (long long)hb.n, (long long)n_pad, (long long)kStaticMaxParticles);
    CK(cudaSetDevice(env->device));
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, f_dev) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
        at.device != env->device || cudaPointerGetAttributes(&at, y_dev) != cudaSuccess ||
        at.type != cudaMemoryTypeDevice || at.device != env->device) {
        cudaGetLastError();
        return fail(PD_ERR_ARG, "f/y must be device pointers on the environment's device %d", env->device);
    }
    if (hb.kind == PD_MAT_ELASTO_PLASTIC)
        return fail(PD_ERR_UNSUPPORTED, "the device-pointer entry point does not evaluate elasto-plastic blocks");
    double4 *scratch = nullptr;
    PD_TRY(scratch_for(env->device, &scratch));
    cudaStream_t st = stream ? (cudaStream_t)stream : env->st;
    // The kernels index particles by internal index; shift the scratch so
    // that internal index first_int lands on its first element.
    double4 *ys = scratch - hb.first_int;
    double4 *fs = scratch + kStaticMaxParticles - hb.first_int;
    const int64_t *map = env->map.p + hb.first_env;
    launch_unpack3(st, hb.n, y_dev + 3 * hb.first_env, map, ys);
    launch_unpack3(st, hb.n, f_dev + 3 * hb.first_env, map, fs);
    Geo g = env->geo();
    const int64_t p0 = hb.first_int, p1 = hb.first_int + n_pad;
    if (hb.kind == PD_MAT_ORDINARY_STATE_BASED)
        launch_theta_serial(st, g, ys, env->words[env->cur].p, env->mth.p, p0, p1);
    // force_density_T! has no deformed gate: mark the block active
    CK(cudaMemcpyAsync(env->deformed.p + block, &kOne, sizeof(int32_t), cudaMemcpyHostToDevice, st));
    launch_force_serial(st, g, ys, env->mth.p, env->words[env->cur].p, env->words[1 - env->cur].p, fs, 1, p0, p1);
    const int64_t w0 = env->sinfo_h[p0 / 32].word, w1 = env->sinfo_h[p1 / 32].word;
    if (w1 > w0)
        CK(cudaMemcpyAsync(env->words[env->cur].p + w0, env->words[1 - env->cur].p + w0, (w1 - w0) * sizeof(uint32_t),
                           cudaMemcpyDeviceToDevice, st));
    launch_pack3(st, hb.n, fs, map, f_dev + 3 * hb.first_env);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    env->deformed_h[block] = 1;
    return PD_OK;
}

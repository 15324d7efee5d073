// pd_peaks.cu -- pd_pipe_peaks: measured issue and pipe rates of the GPU for
// the instruction classes the FP32C bond walk is made of, the compute-side
// denominators of its roofline (the HBM one is a measured copy bandwidth).
//
// Each kernel runs C independent dependency chains per thread over a full
// grid (every SM, 64 warps each), so the pipe under test, not latency,
// sets the rate:
//   0  FFMA           FP32 fused multiply-add, lane operations per second
//   1  FFMA2          packed f32x2 multiply-add, lane FMAs per second (two
//                     per lane per instruction)
//   2  sqrt.approx    MUFU square root, lane operations per second
//   3  rcp.approx     MUFU reciprocal, lane operations per second
//                     (each followed by an FP32 add, which its pipe hides)
//   4  FFMA + LOP3    one FP32 multiply-add and one integer logic op per
//                     chain step, warp instructions per second (both pipes
//                     busy: the rate at which one SM sub-partition issues)
// Every rate is the best of three timed launches after one untimed launch,
// each ~10 ms at B200 speeds.  No kernel waits on anything.
#include "pd_env_impl.h"

using namespace pd;

namespace {

constexpr int kChains = 16;
constexpr int kThreads = 256;
constexpr int kBlocksPerSM = 8;

__global__ void __launch_bounds__(kThreads) k_peak_ffma(float *out, int iters, float a, float b) {
    float acc[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) acc[i] = 1e-3f * (float)(threadIdx.x + i);
#pragma unroll 4
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < kChains; ++i) acc[i] = fmaf(acc[i], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += acc[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_peak_ffma2(float *out, int iters, float a, float b) {
    float2 acc[kChains / 2];
#pragma unroll
    for (int i = 0; i < kChains / 2; ++i) acc[i] = make_float2(1e-3f * (float)(threadIdx.x + i), (float)i);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll 4
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < kChains / 2; ++i) acc[i] = __ffma2_rn(acc[i], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < kChains / 2; ++i) s += acc[i].x + acc[i].y;
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <int OP>
__global__ void __launch_bounds__(kThreads) k_peak_mufu(float *out, int iters) {
    float acc[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i) acc[i] = 1.5f + 1e-3f * (float)(threadIdx.x + i);
#pragma unroll 4
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < kChains; ++i) {
            // each MUFU result feeds an add (FP32 pipe, 8x the MUFU rate),
            // so no chain of MUFU operations collapses to the identity
            float r;
            if (OP == 0)
                asm volatile("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(acc[i]));
            else
                asm volatile("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(acc[i]));
            acc[i] = r + 1.0f;
        }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < kChains; ++i) s += acc[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_peak_mix(float *out, int iters, float a, float b, uint32_t m,
                                                       uint32_t c) {
    float acc[kChains / 2];
    uint32_t k[kChains / 2];
#pragma unroll
    for (int i = 0; i < kChains / 2; ++i) {
        acc[i] = 1e-3f * (float)(threadIdx.x + i);
        k[i] = threadIdx.x * 2654435761u + i;
    }
#pragma unroll 4
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < kChains / 2; ++i) {
            acc[i] = fmaf(acc[i], a, b);
            uint32_t r;
            asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(k[i]), "r"(m), "r"(c));
            k[i] = r;
        }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < kChains / 2; ++i) s += acc[i] + (float)(k[i] & 1u);
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" pd_status pd_pipe_peaks(int32_t device, double *out5) {
    if (!out5) return fail(PD_ERR_ARG, "out is NULL");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(PD_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
    int prev = 0;
    CK(cudaGetDevice(&prev));
    CK(cudaSetDevice(device));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * kBlocksPerSM;
    const double threads = (double)blocks * kThreads;
    float *buf = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaMalloc(&buf, (size_t)blocks * kThreads * sizeof(float));
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    // iterations per launch (~10 ms each at B200 rates)
    const int it_fma = 65536, it_mufu = 8192, it_mix = 65536;
    // lane operations (or warp instructions, test 4) per launch
    const double work[5] = {threads * it_fma * kChains, threads * it_fma * kChains, threads * it_mufu * kChains,
                            threads * it_mufu * kChains, threads / 32.0 * it_mix * kChains};
    for (int t = 0; t < 5 && err == cudaSuccess; ++t) {
        float best = 0.f;
        for (int rep = 0; rep < 4 && err == cudaSuccess; ++rep) {
            err = cudaEventRecord(e0, st);
            if (err != cudaSuccess) break;
            switch (t) {
                case 0: k_peak_ffma<<<blocks, kThreads, 0, st>>>(buf, it_fma, 0.9999999f, 1e-7f); break;
                case 1: k_peak_ffma2<<<blocks, kThreads, 0, st>>>(buf, it_fma, 0.9999999f, 1e-7f); break;
                case 2: k_peak_mufu<0><<<blocks, kThreads, 0, st>>>(buf, it_mufu); break;
                case 3: k_peak_mufu<1><<<blocks, kThreads, 0, st>>>(buf, it_mufu); break;
                default: k_peak_mix<<<blocks, kThreads, 0, st>>>(buf, it_mix, 0.9999999f, 1e-7f, 0x5bd1e995u, 0x27d4eb2fu);
                    break;
            }
            note_launch();
            err = cudaGetLastError();
            if (err == cudaSuccess) err = cudaEventRecord(e1, st);
            if (err == cudaSuccess) err = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
            if (err == cudaSuccess && rep > 0 && (best == 0.f || ms < best)) best = ms;
        }
        if (err == cudaSuccess) out5[t] = best > 0.f ? work[t] / (best * 1e-3) : 0.0;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (buf) cudaFree(buf);
    cudaSetDevice(prev);
    if (err != cudaSuccess) return cuda_fail(err, "pd_pipe_peaks", __FILE__, __LINE__);
    return PD_OK;
}

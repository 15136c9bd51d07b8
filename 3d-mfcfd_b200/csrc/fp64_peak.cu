/*
 * fp64_peak.cu - the FP64 denominator of the roofline: the device's fused
 * multiply-add rate, measured with a loop kernel timed by CUDA events.
 *
 * Built into its own library (mfcfd/libmfcfd_peak.so) for the benchmark;
 * the solver does not use it.  Every thread runs eight independent FMA
 * chains (a = a*b + c with b just below 1, so the values stay finite and
 * normal), enough in flight on a full grid to keep the FP64 pipes busy.
 */
#include <cuda_runtime.h>

namespace {

constexpr int CHAINS = 8;
constexpr int THREADS = 256;

__global__ void __launch_bounds__(THREADS) k_fma_loop(double *out, int iters, double b, double c) {
    double a[CHAINS];
#pragma unroll
    for (int j = 0; j < CHAINS; ++j) a[j] = 1.0 + 1e-3 * (double)(threadIdx.x + j);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < CHAINS; ++j) a[j] = __fma_rn(a[j], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < CHAINS; ++j) s += a[j];
    if (s == -1.0) out[blockIdx.x] = s;   // never true; keeps the chains live
}

}  // namespace

extern "C" {

/* Best of `reps` timed launches after one untimed: *tflops = FP64 TFLOP/s
 * (an FMA is two operations), *ms = the best launch's milliseconds.
 * Returns 0, or the CUDA error code. */
int mfcfd_fp64_fma_peak(int device, int reps, double *tflops, double *ms) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return (int)e;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * (2048 / THREADS);
    const int iters = 1 << 14;
    double *out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(double) * blocks)) != cudaSuccess) return (int)e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 0.0f;
    for (int r = 0; r <= reps; ++r) {
        cudaEventRecord(e0);
        k_fma_loop<<<blocks, THREADS>>>(out, iters, 0.9999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (r > 0 && (best == 0.0f || t < best)) best = t;
    }
    e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return (int)e;
    const double flops = 2.0 * CHAINS * (double)iters * (double)blocks * THREADS;
    if (ms) *ms = best;
    if (tflops) *tflops = flops / (best * 1e-3) / 1e12;
    return 0;
}

}  // extern "C"

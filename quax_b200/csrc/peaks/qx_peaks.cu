// qx_peaks.cu -- FP64 / FP32 FMA throughput probe (libqx_peaks.so).
//
// The roofline denominator for the FP64 integral kernels: the measured peaks the
// machine provides cover HBM bandwidth and bf16 tensor throughput only,
// so the FP64 and FP32 FMA peaks are measured here.  Every thread runs 8
// independent FMA chains (enough to cover the pipe latency), the grid covers every
// SM many times, and time comes from CUDA events around the launch.
#include <cuda_runtime.h>

template <class T>
__global__ void k_fma(T* out, int iters, T a, T b) {
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)123.456) out[blockIdx.x] = s;  // keeps the chains live
}

// Returns TFLOP/s (2 flops per FMA) of `reps` launches; fp64 != 0 selects double.
extern "C" double qx_fma_peak_tflops(int fp64, int iters, int reps) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int bs = 256, nb = sms * 16;
    void* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * nb) != cudaSuccess) return -1.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto launch = [&]() {
        if (fp64) k_fma<double><<<nb, bs>>>((double*)out, iters, 0.999999, 1e-7);
        else k_fma<float><<<nb, bs>>>((float*)out, iters, 0.9999f, 1e-4f);
    };
    launch();
    cudaEventRecord(e0);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    const double flops = 2.0 * 8.0 * (double)iters * (double)bs * (double)nb * (double)reps;
    return flops / (ms * 1e-3) / 1e12;
}

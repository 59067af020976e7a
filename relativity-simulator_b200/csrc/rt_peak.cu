// rt_peak.cu -- FMA-pipe throughput of this device (the roofline denominator
// for the tracer, which is bound by the FP64 pipe in FP64 mode and by the FP32
// pipe in the far-field stages of mixed mode).
//
// Each thread runs 8 independent FMA chains entirely in registers; the result
// is stored only when it is impossible (keeps the chains alive).  FLOP count =
// 2 per FMA.
#include <cuda_runtime.h>

namespace relsim {

template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T seed, int iters, T* sink) {
    T a0 = seed + T(threadIdx.x), a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
    T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
    const T m = T(0.999999), c = T(1e-7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, m, c);
            a1 = fma(a1, m, c);
            a2 = fma(a2, m, c);
            a3 = fma(a3, m, c);
            a4 = fma(a4, m, c);
            a5 = fma(a5, m, c);
            a6 = fma(a6, m, c);
            a7 = fma(a7, m, c);
        }
    }
    const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == T(-12345.678)) sink[threadIdx.x] = s;
}

// Returns TFLOP/s; best of three timed launches after a warm-up.
double measure_fma_peak(bool fp64, int sm_count, cudaStream_t stream, float* ms_out) {
    const int block = 256;
    const int grid = sm_count * 8;
    const int iters = fp64 ? 2048 : 4096;
    void* sink = nullptr;
    if (cudaMalloc(&sink, block * sizeof(double)) != cudaSuccess) return 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0, stream);
        if (fp64)
            fma_chain_kernel<double><<<grid, block, 0, stream>>>(1.0, iters, static_cast<double*>(sink));
        else
            fma_chain_kernel<float><<<grid, block, 0, stream>>>(1.0f, iters, static_cast<float*>(sink));
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (ms_out) *ms_out = best;
    const double flops = 2.0 * 8.0 * 16.0 * static_cast<double>(iters) * grid * block;
    return flops / (static_cast<double>(best) * 1e-3) / 1e12;
}

}  // namespace relsim

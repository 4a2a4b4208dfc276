// FP32 fused multiply-add throughput probe: the SIMT roofline of the plain correlation form.
// Each thread runs 16 independent FMA chains; nothing is read from memory; the result is
// stored only when it takes an impossible value so the chains cannot be removed.
#include <cuda_runtime.h>

__global__ void fma_probe(float* sink, int iters, float seed)
{
    float a[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = seed + threadIdx.x * 1e-7f + k;
    const float b = 0.9999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int k = 0; k < 16; ++k) a[k] = fmaf(a[k], b, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; ++k) s += a[k];
    if (s == -1.0f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// returns the best of `reps` timed launches in TFLOP/s (2 flops per FMA), or a negative value
extern "C" double fp32_fma_tflops(int device, int reps)
{
    if (cudaSetDevice(device) != cudaSuccess) return -1.0;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int threads = 256, blocks = sms * 8, iters = 4096;
    float* sink = nullptr;
    if (cudaMalloc(&sink, (size_t)blocks * threads * sizeof(float)) != cudaSuccess) return -2.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_probe<<<blocks, threads>>>(sink, iters, 1.0f);
    double best = 0.0;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0);
        fma_probe<<<blocks, threads>>>(sink, iters, 1.0f + r);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 16 * 8 * (double)iters * threads * blocks;
        const double tf = flops / (ms * 1e-3) / 1e12;
        if (tf > best) best = tf;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return cudaGetLastError() == cudaSuccess ? best : -3.0;
}

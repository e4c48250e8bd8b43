// nz_diag.cu -- peak probes used as roofline denominators.
//
// The flash is bound by the FP64 (or FP32) CUDA-core pipes, whose peaks are
// not in the driver-measured peaks file, so they are measured here with a
// dependency-chain-free FMA kernel: 8 independent FMA chains per thread,
// a grid of 8 x 148 x 1024 threads, timed with CUDA events.
#include "common.cuh"

namespace nz
{

template <class T>
__global__ void __launch_bounds__(256) fmaPeakKernel(T *out, int iters, T a, T b)
{
    T r[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        r[k] = T(threadIdx.x + k);
#pragma unroll 1
    for (int i = 0; i < iters; ++i)
    {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k)
                r[k] = fma(r[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        s += r[k];
    if (s == T(-1.2345))   // practically never; keeps the chains alive
        out[blockIdx.x] = s;
}

template <class T>
static double measure(int device, int iters)
{
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    const int blocks = prop.multiProcessorCount * 8;
    T *out = nullptr;
    cudaMalloc(&out, sizeof(T) * blocks);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fmaPeakKernel<T><<<blocks, 256>>>(out, iters / 10, T(0.999999), T(1e-7));
    cudaEventRecord(e0);
    fmaPeakKernel<T><<<blocks, 256>>>(out, iters, T(0.999999), T(1e-7));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * 16.0 * double(iters) * double(blocks) * 256.0;
    return flops / (double(ms) * 1e-3) / 1e12;
}

} // namespace nz

extern "C" int nz_diag_fma_peak(int32_t device, double *fp64_tflops, double *fp32_tflops)
{
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess)
        return nz::cudaFail(e, "nz_diag_fma_peak");
    if (fp64_tflops)
        *fp64_tflops = nz::measure<double>(device, 4000);
    if (fp32_tflops)
        *fp32_tflops = nz::measure<float>(device, 8000);
    e = cudaGetLastError();
    return e == cudaSuccess ? NZ_OK : nz::cudaFail(e, "nz_diag_fma_peak");
}

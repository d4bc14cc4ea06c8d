// Measurement helpers for bench.py (not part of the SPH boundary):
//   sphx_fp32_fma_tflops  — the FP32 FMA-pipe peak of this GPU, measured live;
//   sphx_launch_count     — kernels this library has launched so far.
//
// The pair kernels are bound by the FP32 (or FP64) FMA pipes, not by tensor
// cores or HBM, so their roofline denominator is the FMA throughput.  The
// microbenchmark runs 8 independent FMA chains per thread on every SM
// (148 SMs x 8 blocks x 256 threads) so the pipes, not latency, limit it.
#include "sph_launch.hpp"

#include <atomic>

namespace sph
{
    namespace
    {
        std::atomic<unsigned long long> g_launches{0};

        template<typename T>
        __global__ void __launch_bounds__(256) kFmaChains(T* out, int iters, T a, T b)
        {
            T x0 = T(threadIdx.x), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
            T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
            for(int i = 0; i < iters; ++i)
            {
#pragma unroll
                for(int k = 0; k < 16; ++k)
                {
                    x0 = fma(x0, a, b);
                    x1 = fma(x1, a, b);
                    x2 = fma(x2, a, b);
                    x3 = fma(x3, a, b);
                    x4 = fma(x4, a, b);
                    x5 = fma(x5, a, b);
                    x6 = fma(x6, a, b);
                    x7 = fma(x7, a, b);
                }
            }
            T const s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
            if(s == T(-1.2345))
                out[blockIdx.x * blockDim.x + threadIdx.x] = s;
        }
    } // namespace

    void countLaunches(unsigned k)
    {
        g_launches.fetch_add(k, std::memory_order_relaxed);
    }

    unsigned long long launchesSoFar()
    {
        return g_launches.load(std::memory_order_relaxed);
    }

    void uncountLaunches(unsigned long long k)
    {
        g_launches.fetch_sub(k, std::memory_order_relaxed);
    }
} // namespace sph

extern "C" {

//! Measured dense FMA throughput (TFLOP/s, FMA = 2 flops) in FP32 (fp64 = 0) or FP64.
int sphx_fma_tflops(int device, int fp64, double* out)
{
    if(!out)
        return SPH_ERR_INVALID;
    if(cudaSetDevice(device) != cudaSuccess)
        return SPH_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int const blocks = sms * 8, threads = 256, iters = fp64 ? 1024 : 4096;
    void* buf = nullptr;
    if(cudaMalloc(&buf, size_t(blocks) * threads * 8) != cudaSuccess)
        return SPH_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for(int rep = 0; rep < 4; ++rep)
    {
        cudaEventRecord(e0);
        if(fp64)
            sph::kFmaChains<double><<<blocks, threads>>>(static_cast<double*>(buf), iters, 0.999999, 1e-7);
        else
            sph::kFmaChains<float><<<blocks, threads>>>(static_cast<float*>(buf), iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if(rep > 0 && ms < best)
            best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    if(cudaGetLastError() != cudaSuccess)
        return SPH_ERR_CUDA;
    double const flops = 2.0 * 8.0 * 16.0 * double(iters) * double(blocks) * double(threads);
    *out = flops / (double(best) * 1e-3) / 1e12;
    return SPH_OK;
}

//! Kernels launched by this library since it was loaded.
unsigned long long sphx_launch_count(void)
{
    return sph::g_launches.load();
}
}

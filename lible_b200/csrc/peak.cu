// FP64 throughput probes used as roofline denominators: a dependent-chain-free DFMA loop on the
// vector pipe and a DMMA (mma.sync m8n8k4 f64) loop on the tensor pipe, both register-resident.
#include "engine_api.hpp"

#include <cuda_runtime.h>

namespace lible_b200
{
    constexpr int kPeakIters = 4096;

    __global__ void __launch_bounds__(256) dfmaPeakKernel(double *out, double a, double b)
    {
        double x[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            x[k] = threadIdx.x * 1e-9 + k;
        for (int i = 0; i < kPeakIters; i++)
        {
#pragma unroll
            for (int k = 0; k < 8; k++)
                x[k] = fma(x[k], a, b);
        }
        double s = 0;
#pragma unroll
        for (int k = 0; k < 8; k++)
            s += x[k];
        if (s == 12345.678)
            out[0] = s;
    }

    __global__ void __launch_bounds__(256) dmmaPeakKernel(double *out, double a, double b)
    {
        double A = a + threadIdx.x * 1e-9, B = b;
        double c[4][2];
#pragma unroll
        for (int k = 0; k < 4; k++)
            c[k][0] = c[k][1] = 0.0;
        for (int i = 0; i < kPeakIters; i++)
        {
#pragma unroll
            for (int k = 0; k < 4; k++)
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                             : "+d"(c[k][0]), "+d"(c[k][1])
                             : "d"(A), "d"(B));
        }
        double s = 0;
#pragma unroll
        for (int k = 0; k < 4; k++)
            s += c[k][0] + c[k][1];
        if (s == 12345.678)
            out[0] = s;
    }

    // Returns {DFMA TFLOP/s, DMMA TFLOP/s}, best of 5 timed launches each.
    std::pair<double, double> measureFp64Peak(int device, cudaStream_t s)
    {
        cudaDeviceProp prop;
        cudaCheck(cudaGetDeviceProperties(&prop, device), "props");
        double *out;
        cudaCheck(cudaMalloc(&out, sizeof(double)), "malloc");
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        const int blocks = prop.multiProcessorCount * 8, threads = 256;
        double best[2] = {0, 0};
        for (int kind = 0; kind < 2; kind++)
            for (int rep = 0; rep < 6; rep++)
            {
                cudaEventRecord(e0, s);
                if (kind == 0)
                    dfmaPeakKernel<<<blocks, threads, 0, s>>>(out, 0.999999, 1e-7);
                else
                    dmmaPeakKernel<<<blocks, threads, 0, s>>>(out, 0.999999, 1e-7);
                cudaEventRecord(e1, s);
                cudaCheck(cudaEventSynchronize(e1), "peak");
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                double flops = kind == 0 ? 2.0 * 8 * kPeakIters * (double)blocks * threads
                                         // one m8n8k4 per warp: 8*8*4 FMAs
                                         : 2.0 * 256 * 4 * kPeakIters * (double)blocks * (threads / 32);
                if (rep > 0)
                    best[kind] = std::max(best[kind], flops / (ms * 1e-3) / 1e12);
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(out);
        return {best[0], best[1]};
    }
}

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

    // FP32 probes: scalar FFMA chains, and packed pairs (fma.rn.f32x2, two FP32 FMAs per instruction
    // on sm_100).
    __global__ void __launch_bounds__(256) ffmaPeakKernel(float *out, float a, float b)
    {
        float x[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            x[k] = threadIdx.x * 1e-6f + k;
        for (int i = 0; i < kPeakIters; i++)
        {
#pragma unroll
            for (int k = 0; k < 8; k++)
                x[k] = fmaf(x[k], a, b);
        }
        float s = 0;
#pragma unroll
        for (int k = 0; k < 8; k++)
            s += x[k];
        if (s == 12345.678f)
            out[0] = s;
    }

    __global__ void __launch_bounds__(256) ffma2PeakKernel(float *out, float a, float b)
    {
        const unsigned long long A = ((unsigned long long)__float_as_uint(a) << 32) | __float_as_uint(a);
        const unsigned long long B = ((unsigned long long)__float_as_uint(b) << 32) | __float_as_uint(b);
        unsigned long long x[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
        {
            const float v = threadIdx.x * 1e-6f + k;
            x[k] = ((unsigned long long)__float_as_uint(v) << 32) | __float_as_uint(v + 0.5f);
        }
        for (int i = 0; i < kPeakIters; i++)
        {
#pragma unroll
            for (int k = 0; k < 8; k++)
                asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[k]) : "l"(A), "l"(B));
        }
        float s = 0;
#pragma unroll
        for (int k = 0; k < 8; k++)
            s += __uint_as_float((unsigned)x[k]) + __uint_as_float((unsigned)(x[k] >> 32));
        if (s == 12345.678f)
            out[0] = s;
    }

    // Returns {FFMA TFLOP/s, packed FFMA2 TFLOP/s}, best of 5 timed launches each.
    std::pair<double, double> measureFp32Peak(int device, cudaStream_t s)
    {
        cudaDeviceProp prop;
        cudaCheck(cudaGetDeviceProperties(&prop, device), "props");
        float *out;
        cudaCheck(cudaMalloc(&out, sizeof(float)), "malloc");
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
                    ffmaPeakKernel<<<blocks, threads, 0, s>>>(out, 0.999999f, 1e-7f);
                else
                    ffma2PeakKernel<<<blocks, threads, 0, s>>>(out, 0.999999f, 1e-7f);
                cudaEventRecord(e1, s);
                cudaCheck(cudaEventSynchronize(e1), "peak");
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                const double flops = 2.0 * 8 * kPeakIters * (double)blocks * threads * (kind == 0 ? 1 : 2);
                if (rep > 0)
                    best[kind] = std::max(best[kind], flops / (ms * 1e-3) / 1e12);
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(out);
        return {best[0], best[1]};
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

// Direct evaluation of the device special functions the class kernels use, for their tests: e^{-x}
// (expNeg), the FP64 Boys function F_0..F_N (boysF, table staged in shared memory as the register
// path does) and its FP32 form (boysF32).
#include "device_common.cuh"

namespace lible_b200
{
    template <int N>
    __device__ void boysEvalOne(int which, double x, const double *tab, const float *tabf, double *out)
    {
        if (which == 1)
        {
            double F[N + 1];
            boysF<N, true>(x, tab, F);
            for (int k = 0; k <= N; k++)
                out[k] = F[k];
        }
        else
        {
            float F[N + 1];
            boysF32<N>((float)x, tabf, F);
            for (int k = 0; k <= N; k++)
                out[k] = F[k];
        }
    }

    template <int N>
    __global__ void __launch_bounds__(128) specialEvalKernel(int which, long long n, const double *x, double *out,
                                                             const double *boys, const float *boys_f)
    {
        __shared__ double tab[kBoysTerms * kBoysPitch];
        __shared__ float tabf[(kBoysMaxN + kBoysTermsF) * kBoysPitch];
        stageBoys(boys, N, tab);
        stageBoys(boys_f, N, tabf);
        __syncthreads();
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
            if (which == 0)
                out[i] = expNeg(x[i]);
            else
                boysEvalOne<N>(which, x[i], tab, tabf, out + i * (N + 1));
        }
    }

    template <int N>
    static void launchSpecial(int which, int order, long long n, const double *x, double *out, const double *boys,
                              const float *boys_f, int sms, cudaStream_t s)
    {
        if constexpr (N <= kBoysMaxN)
        {
            if (order != N)
                return launchSpecial<N + 1>(which, order, n, x, out, boys, boys_f, sms, s);
            specialEvalKernel<N><<<sms * 4, 128, 0, s>>>(which, n, x, out, boys, boys_f);
        }
    }

    void Engine::evalSpecial(int which, int order, long long n, const double *x_dev, double *out_dev)
    {
        if (which < 0 || which > 2 || n < 0 || (which > 0 && (order < 0 || order > kBoysMaxN)))
            throw EngineError(kStatusInvalid, "special-function evaluation: bad arguments");
        if (n == 0)
            return;
        launchSpecial<0>(which, which == 0 ? 0 : order, n, x_dev, out_dev, boys_, boys_f_, num_sms_, stream_);
        cudaCheck(cudaGetLastError(), "specialEvalKernel");
        cudaCheck(cudaStreamSynchronize(stream_), "special");
    }
}

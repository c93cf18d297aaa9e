// Launch wrapper of the first-derivative class kernels (eri_d1_kernel.cuh).
#pragma once

#include "eri_d1_kernel.cuh"
#include "eri_launch.cuh"

#include <algorithm>

namespace lible_b200
{
    template <int LA, int LB, int LC, int LD>
    cudaError_t launchD1(const QuartetArgs &a, cudaStream_t s, int num_sms)
    {
        using S = ShapeD1<LA, LB, LC, LD>;
        if (a.n_tasks <= 0)
            return cudaSuccess;
        if constexpr (d1RegisterClass(LA, LB, LC, LD))
        {
            // J/K gradient of the smallest classes: one quartet per thread, the block's gradient in
            // shared memory (up to 2,048 atoms)
            const size_t sg = sizeof(double) * 3 * (size_t)std::max(a.n_atoms, 1);
            if ((a.mode == kD1Grad || a.mode == kD1GradRI) && a.n_atoms > 0 && sg <= 48 * 1024)
            {
                auto rk = eriD1RegKernel<LA, LB, LC, LD>;
                int occ = 0;
                cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, rk, 128, sg);
                if (e != cudaSuccess)
                    return e;
                long long grid = a.chunks ? (a.n_chunks + 3) / 4 : (a.n_tasks + 8LL * 128 - 1) / (8LL * 128);
                grid = std::max<long long>(1, std::min<long long>(grid, (long long)num_sms * std::max(occ, 1)));
                rk<<<(unsigned)grid, 128, sg, s>>>(a);
                return cudaGetLastError();
            }
        }
        if constexpr (ShapeD1M<LA, LB, LC, LD>::USE)
        {
            // gradient epilogues of the larger classes: both contractions on the DMMA pipe
            if (a.mode == kD1Grad || a.mode == kD1GradRI)
            {
                using SM = ShapeD1M<LA, LB, LC, LD>;
                auto mk = eriD1MmaKernel<LA, LB, LC, LD>;
                if (SM::smem > 48 * 1024)
                {
                    cudaError_t e = cudaFuncSetAttribute(mk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::smem);
                    if (e != cudaSuccess)
                        return e;
                }
                int occ = 0;
                cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mk, SM::G, SM::smem);
                if (e != cudaSuccess)
                    return e;
                long long grid = a.chunks ? std::min<long long>(a.n_chunks, (long long)num_sms * std::max(occ, 1))
                                          : std::min<long long>(a.n_tasks, (long long)num_sms * std::max(occ, 1) * 4);
                grid = std::max<long long>(grid, 1);
                mk<<<(unsigned)grid, SM::G, SM::smem, s>>>(a);
                return cudaGetLastError();
            }
        }
        auto kern = eriD1Kernel<LA, LB, LC, LD>;
        if (S::smem > 48 * 1024)
        {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem);
            if (e != cudaSuccess)
                return e;
        }
        int occ = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, S::G, S::smem);
        if (e != cudaSuccess)
            return e;
        long long grid = a.chunks ? std::min<long long>(a.n_chunks, (long long)num_sms * std::max(occ, 1))
                                  : std::min<long long>(a.n_tasks, (long long)num_sms * std::max(occ, 1) * 4);
        grid = std::max<long long>(grid, 1);
        kern<<<(unsigned)grid, S::G, S::smem, s>>>(a);
        return cudaGetLastError();
    }

}

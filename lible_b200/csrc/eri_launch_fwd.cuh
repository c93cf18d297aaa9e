// Launch wrapper of the forward class kernels (eri_kernel.cuh).
#pragma once

#include "eri_kernel.cuh"
#include "eri_launch.cuh"

#include <algorithm>

namespace lible_b200
{
    // Quartets a worker processes side by side: QPW per warp on the register path, one per block on
    // the group path.  Work-queue chunks are cut so that each holds at least one unit of the most
    // expensive quartets.
    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    constexpr int workUnit()
    {
        using S = Shape<LA, LB, LC, LD, T, SV>;
        return S::W == 0 ? S::QPW : 1;
    }

    template <int LA, int LB, int LC, int LD, typename T, int SV = 0>
    cudaError_t launchFwd(const QuartetArgs &a, cudaStream_t s, int num_sms)
    {
        using S = Shape<LA, LB, LC, LD, T, SV>;
        if (a.n_tasks <= 0)
            return cudaSuccess;
        auto kern = eriKernelFor<LA, LB, LC, LD, T, SV>();
        long long grid;
        if (a.chunks)
        {
            // persistent grid: every resident block pulls chunks from the work queue
            if (S::smem > 48 * 1024)
            {
                cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem);
                if (e != cudaSuccess)
                    return e;
            }
            int occ = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, S::block, S::smem);
            if (e != cudaSuccess)
                return e;
            const long long workers_per_block = S::W == 0 ? S::block / 32 : 1;
            grid = std::min<long long>((a.n_chunks + workers_per_block - 1) / workers_per_block,
                                       (long long)num_sms * std::max(occ / std::max(a.grid_div, 1), 1));
            grid = std::max<long long>(grid, 1);
        }
        else if constexpr (S::W == 0)
        {
            // one chunk of 8 warp-iterations per warp, at most 32 blocks per SM in flight
            const long long chunks = (a.n_tasks + 8LL * S::QPW - 1) / (8LL * S::QPW);
            grid = std::min<long long>((chunks + S::block / 32 - 1) / (S::block / 32), (long long)num_sms * 32);
            if (S::smem > 48 * 1024)
            {
                cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem);
                if (e != cudaSuccess)
                    return e;
            }
        }
        else
        {
            if (S::smem > 48 * 1024)
            {
                cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem);
                if (e != cudaSuccess)
                    return e;
            }
            int occ = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, S::block, S::smem);
            if (e != cudaSuccess)
                return e;
            grid = std::min<long long>((a.n_tasks + 7) / 8, (long long)num_sms * std::max(occ, 1) * 4);
        }
        kern<<<(unsigned)grid, S::block, S::smem, s>>>(a);
        return cudaGetLastError();
    }

}

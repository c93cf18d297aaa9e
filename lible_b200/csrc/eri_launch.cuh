// Launch wrappers and the dispatch table that maps a quartet class to its kernel instantiation.
#pragma once

#include "eri_kernel.cuh"
#include "eri_d1_kernel.cuh"

#include <algorithm>

namespace lible_b200
{
    using LaunchFn = cudaError_t (*)(const QuartetArgs &, cudaStream_t, int num_sms);

    // Pair types in canonical order; a quartet class is instantiated with the larger type in the
    // bra.  Index: la*(la+1)/2 + lb for la <= 3, then (4,0) -> 10, (5,0) -> 11.
    constexpr int kNumPairTypes = 12;
    inline int pairType(int la, int lb)
    {
        if (la <= 3)
            return la * (la + 1) / 2 + lb;
        return la == 4 ? 10 : 11;
    }

    // Quartets a worker processes side by side: QPW per warp on the register path, one per block on
    // the group path.  Work-queue chunks are cut so that each holds at least one unit of the most
    // expensive quartets.
    template <int LA, int LB, int LC, int LD, typename T>
    constexpr int workUnit()
    {
        using S = Shape<LA, LB, LC, LD, T>;
        return S::W == 0 ? S::QPW : 1;
    }

    template <int LA, int LB, int LC, int LD, typename T>
    cudaError_t launchFwd(const QuartetArgs &a, cudaStream_t s, int num_sms)
    {
        using S = Shape<LA, LB, LC, LD, T>;
        if (a.n_tasks <= 0)
            return cudaSuccess;
        auto kern = eriKernelFor<LA, LB, LC, LD, T>();
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

    // Implemented by the generated instantiation files.
    LaunchFn lookupFwd64(int bra_type, int ket_type);
    LaunchFn lookupFwd32(int bra_type, int ket_type);
    LaunchFn lookupD1(int bra_type, int ket_type);
    int unitFwd(int bra_type, int ket_type, bool fp32);
}

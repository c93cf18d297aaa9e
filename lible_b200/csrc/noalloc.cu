// Allocation-free variant of the batched ERI4Kernel call.
//
// The regular lible_gpu_eri4_batch stages the caller's (ipair_ab, ipair_cd) list in a device buffer
// it allocates and frees on every call.  Some callers cannot allow that: a host program that has
// handed all free device memory to its own pool allocator, or one that overlaps work on other
// streams and cannot afford the implicit device-wide synchronisation of cudaFree.  For them the
// list is staged instead in a fixed buffer that lives in this library's device image, so the call
// performs no cudaMalloc / cudaFree and no allocating library routine.
//
// Limits and sharing: the buffer holds kNoAllocMaxPairs index pairs (8 MiB of device memory,
// reserved on every GPU that loads the library until the process exits).  All calls share it: two
// calls whose work overlaps on the GPU (different streams or contexts on one device) race on it.
// Each call overwrites the part it uses before reading it, so nothing needs clearing.
#include "../../include/lible_b200.h"
#include "engine_api.hpp"
#include "eri_launch.cuh"

#include <vector>

namespace lible_b200
{
    constexpr long long kNoAllocMaxPairs = 1LL << 20;

    // The staging buffer.  In host code this name is only a host-side stand-in; its device address
    // comes from cudaGetSymbolAddress below.
    static __device__ __align__(256) uint32_t g_pair_list_scratch[2 * kNoAllocMaxPairs];

    // Device address of the buffer on the current device.  It is looked up on every call (a cheap
    // host call) rather than cached, so a new primary context, which may load the module at another
    // address, is always seen.
    static uint32_t *scratchAddress()
    {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_pair_list_scratch);
        if (e != cudaSuccess)
            throw EngineError(kStatusCuda, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return static_cast<uint32_t *>(p);
    }

    void Engine::eri4BatchNoAlloc(bool use_symm, int cab, int ccd, long long n, const uint32_t *pairs_host,
                                  double *out_dev, uint32_t *scratch, long long max_pairs)
    {
        const int inject = wait_inject_;
        wait_inject_ = 0;
        requireSingle();
        if (n < 0 || n > max_pairs)
            throw EngineError(kStatusInvalid, "eri4 batch without allocation: n = " + std::to_string(n) +
                                                  " exceeds the maximum of " + std::to_string(max_pairs) + " pairs");
        ClassSet &cs = use_symm ? symm_ : nosymm_;
        if (!cs.built)
            throw EngineError(kStatusInvalid, "eri4 batch without allocation: the shell-pair classes are not on the "
                                              "device yet; call lible_gpu_pair_classes with this use_symm first");
        if (cab < 0 || ccd < 0 || cab >= (int)cs.dev.size() || ccd >= (int)cs.dev.size())
            throw EngineError(kStatusInvalid, "class index out of range");
        const DevPairClass &bra = cs.dev[cab], &ket = cs.dev[ccd];
        for (long long i = 0; i < n; i++)
            if (pairs_host[2 * i] >= bra.n_pairs || pairs_host[2 * i + 1] >= ket.n_pairs)
                throw EngineError(kStatusInvalid, "pair index out of range");
        if (n == 0)
            return;
        // the kernel is instantiated with the larger pair type in the bra; swap the two index columns
        // while staging when the caller's orientation is the other one
        const int tb = pairType(bra.la, bra.lb), tk = pairType(ket.la, ket.lb);
        const bool swap = tb < tk;
        if (!swap)
            cudaCheck(cudaMemcpyAsync(scratch, pairs_host, (size_t)n * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                      stream_),
                      "stage");
        else
        {
            // swapped columns in host memory (the no-allocation rule is about device memory), staged
            // with one contiguous copy
            std::vector<uint32_t> h(2 * (size_t)n);
            for (long long i = 0; i < n; i++)
            {
                h[2 * i] = pairs_host[2 * i + 1];
                h[2 * i + 1] = pairs_host[2 * i];
            }
            cudaCheck(cudaMemcpyAsync(scratch, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_),
                      "stage");
            cudaCheck(cudaStreamSynchronize(stream_), "stage");
        }
        const bool bs = cs.swapped[cab], ks = cs.swapped[ccd];
        QuartetArgs a{};
        a.bra = view(swap ? ket : bra);
        a.ket = view(swap ? bra : ket);
        a.ket_EtP = (swap ? bra : ket).EtP;
        a.boys = boys_;
        a.boys_f = boys_f_;
        a.status = d_status_;  // allocated with the context: a bounded wait that gives up is reported
        a.wait_inject = inject;
        cudaCheck(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_), "memset");
        a.list = scratch;
        a.n_tasks = n;
        a.same_class = (use_symm && cab == ccd) ? 1 : 0;
        a.flags = swap ? ((ks ? 1 : 0) | (bs ? 2 : 0) | 4) : ((bs ? 1 : 0) | (ks ? 2 : 0));
        a.mode = kStore;
        a.out = out_dev;
        LaunchFn fn = lookupFwd64(swap ? tk : tb, swap ? tb : tk);
        if (!fn)
            throw EngineError(kStatusUnsupported, "quartet class not instantiated");
        cudaCheck(fn(a, stream_, num_sms_), "eri kernel");
        checkStatus();  // synchronises
    }

    uint32_t *noAllocScratch(long long *max_pairs)
    {
        *max_pairs = kNoAllocMaxPairs;
        return scratchAddress();
    }
}

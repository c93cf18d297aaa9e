// The engine object behind the C ABI.
#pragma once

#include "engine.hpp"

#include <cuda_runtime.h>

#include <map>
#include <stdexcept>
#include <string>

namespace lible_b200
{
    struct PairView;
    struct QuartetArgs;
    using LaunchFn = cudaError_t (*)(const QuartetArgs &, cudaStream_t, int num_sms);

    // Status codes returned through the C ABI (mirrors include/lible_b200.h).
    enum Status : int
    {
        kStatusOk = 0,
        kStatusInvalid = 1,
        kStatusCuda = 2,
        kStatusNoStructure = 3,
        kStatusNoAux = 4,
        kStatusUnsupported = 5,
        kStatusTimeout = 6,
        kStatusInternal = 7,
    };

    struct EngineError : std::runtime_error
    {
        int code;
        EngineError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
    };

    void cudaCheck(cudaError_t e, const char *what);

    struct JKOptions
    {
        double schwarz = 1e-12;
        double fp32_threshold = 1e-4;
        int precision = 0;  // 0 FP64, 1 mixed (FP32 where Q_ab Q_cd < fp32_threshold)
        int use_graph = 0;  // replay the launch sequence from a captured CUDA graph
    };

    struct JKStats
    {
        long long n_quartets = 0;
        long long n_fp32 = 0;
        long long n_launches = 0;
    };

    // Size of a J/K plan: unique contracted quartets, primitive quartets and algorithmic FLOPs
    // (dense-equivalent count per primitive quartet: Boys (20 + 4L), R recursion 3 C(L+4,4) plus
    // the signed matrix H_ab H_cd, ket contraction 2 H_ab H_cd S_cd, and per bra primitive pair the
    // bra contraction 2 S_ab H_ab S_cd).
    struct JKPlanInfo
    {
        long long n_quartets = 0, n_fp32 = 0, n_prim_quartets = 0, n_launches = 0;
        double flops_fp64 = 0, flops_fp32 = 0;
    };

    std::pair<double, double> measureFp64Peak(int device, cudaStream_t s);

    class Engine
    {
    public:
        explicit Engine(int device);
        ~Engine();
        Engine(const Engine &) = delete;
        Engine &operator=(const Engine &) = delete;

        void setStructure(const std::vector<BasisAtom> &main, const std::vector<BasisAtom> *aux,
                          const std::vector<std::array<double, 3>> &xyz_bohr);
        size_t nao() const { return nao_; }
        size_t naux() const { return naux_; }
        int nAtoms() const { return n_atoms_; }
        int maxL() const { return max_l_; }
        bool hasAux() const { return has_aux_; }
        cudaStream_t stream() const { return stream_; }
        int device() const { return device_; }

        // Full tensors (device output pointers) and diagonals (host output).
        void eri4(double *out_dev);
        void eri4Diagonal(double *out_host);
        void eri3(double *out_dev);
        void eri2(double *out_dev);
        void eri2Diagonal(double *out_host);

        // Kernel-API batches; classes in the reference's shellPairData / shellDataAux order.
        struct ClassInfo
        {
            int la, lb;
            long long n_pairs, n_ppairs;
        };
        std::vector<ClassInfo> pairClasses(bool use_symm)
        {
            auto &cs = mainSet(use_symm);
            std::vector<ClassInfo> v;
            for (size_t c = 0; c < cs.host.size(); c++)
                v.push_back({cs.req_l[c].first, cs.req_l[c].second, (long long)cs.host[c].n_pairs,
                             (long long)cs.host[c].n_ppairs});
            return v;
        }
        std::vector<ClassInfo> auxClasses()
        {
            auto &cs = auxSet();
            std::vector<ClassInfo> v;
            for (size_t c = 0; c < cs.host.size(); c++)
                v.push_back({cs.req_l[c].first, 0, (long long)cs.host[c].n_pairs, (long long)cs.host[c].n_ppairs});
            return v;
        }
        void eri4Batch(bool use_symm, int cab, int ccd, long long n, const uint32_t *pairs_host, double *out_dev,
                       bool d1);
        void eri3Batch(bool use_symm, int cab, int cx, long long n, const uint32_t *idx_host, double *out_dev, bool d1);
        void eri2Batch(int ca, int cb, long long n, const uint32_t *idx_host, double *out_dev, bool d1);
        // ERI4SOCKernel (kind 0, main x main), ERI3SOCKernel (1, main x aux), ERI2D2Kernel (2, aux x
        // aux) batches: out [n][3][block] (SOC) or [n][6][6][Sa][Sb] (D2), device memory.
        void specialBatch(int kind, bool use_symm, int c_ab, int c_cd, long long n, const uint32_t *pairs_host,
                          double *out_dev);
        // eri4Batch without any device allocation: the pair list is staged in `scratch` (device
        // memory the caller owns, room for 2 * max_pairs indices); `out_dev` must be device memory.
        // The class set must already exist on the device (built by an earlier pairClasses call).
        void eri4BatchNoAlloc(bool use_symm, int cab, int ccd, long long n, const uint32_t *pairs_host,
                              double *out_dev, uint32_t *scratch, long long max_pairs);

        // A batch of molecules whose J/K are built together: every class pair of every molecule goes
        // through one launch per quartet class.  D, J and K are packed: molecule m's N_m x N_m
        // matrix starts at element molBase()[m].  Only the J/K calls accept a batch.
        void setBatch(const std::vector<std::vector<BasisAtom>> &mols,
                      const std::vector<std::vector<std::array<double, 3>>> &xyz_bohr);
        bool isBatch() const { return batch_; }
        // Autotune cache read when J/K plans are built (empty: none).
        void setTuneCache(const std::string &path) { tune_cache_ = path; }
        const std::vector<long long> &molNao() const { return mol_nao_; }
        const std::vector<long long> &molBase() const { return mol_base_; }
        long long packedSize() const { return packed_; }

        // Direct J/K (device pointers).  J, K symmetric on return.  With opt.use_graph the launch
        // sequence is captured once per (plan, D, J, K) into a CUDA graph and replayed.
        void jk(const double *D_dev, double *J_dev, double *K_dev, const JKOptions &opt, JKStats *stats);
        // One J/K build with every class launch serialised on the context stream and timed with CUDA
        // events: (la, lb, lc, ld), FP32 flag, milliseconds, algorithmic FLOPs, tasks per launch.
        struct LaunchTime
        {
            int l[4];
            int fp32;
            double ms, flops;
            long long tasks;
        };
        std::vector<LaunchTime> jkProfile(const double *D_dev, double *J_dev, double *K_dev, const JKOptions &opt);
        // Times the candidate launch parameters of every class pair of the plan for `opt` on the
        // given buffers, keeps the fastest and appends them to `cache` (if non-empty).  Returns a
        // one-line summary per class pair.
        std::string jkAutotune(const double *D_dev, double *J_dev, double *K_dev, const JKOptions &opt,
                               const std::string &cache);
        long long jkLaunchCount(const JKOptions &opt);
        JKPlanInfo jkPlanInfo(const JKOptions &opt);
        struct JKClassInfo
        {
            int l[4];
            long long n64, n32;
            double prim, flops;
        };
        std::vector<JKClassInfo> jkPlanClasses(const JKOptions &opt);
        // Gradient of 1/2 Tr(DJ) - 1/4 Tr(DK) with respect to nuclear coordinates, [n_atoms][3].
        void jkGradient(const double *D_dev, double *grad_dev, double schwarz);
        // RI-J contractions (either output may be null).
        void riContract(const double *D_dev, const double *dcoef_dev, double *gamma_dev, double *J_dev,
                        double schwarz);
        // Dense block of three-centre integrals: T[P - P_lo][m][n] = (mn|P) for the auxiliary
        // functions P in [P_lo, P_hi) (block ends on shell boundaries, see auxShellStarts), with the
        // Schwarz test of the RI plan; enqueued on the context stream.  packed: rows of the lower
        // triangle only, T[P - P_lo][i (i + 1) / 2 + j] = (ij|P) for j <= i (nao (nao + 1) / 2 each).
        void riStore(int P_lo, int P_hi, double *T_dev, double schwarz, bool packed = false);
        // Gradient of the RI-J energy 1/2 gamma^T (P|Q)^{-1} gamma given d = (P|Q)^{-1} gamma (device
        // vector): sum_P d_P sum_mn D_mn d(mn|P)/dR - 1/2 sum_PQ d_P d_Q d(P|Q)/dR, [n_atoms][3].
        void riGradient(const double *D_dev, const double *dcoef_dev, double *grad_dev, double schwarz);
        // First auxiliary function of every auxiliary shell, ascending, followed by naux.
        std::vector<int> auxShellStarts();
        // One-electron integrals (device outputs, any may be null): overlap, kinetic energy and the
        // attraction of point charges ([n][4] x, y, z in bohr, q; with `nuclei` the atoms' nuclei).
        void oneElectron(const double *charges_host, int n_charges, bool nuclei, double *S_dev, double *T_dev,
                         double *V_dev);
        // Per-pair one-electron blocks of class `cls` of shellPairData(use_symm) for the listed pairs:
        // op 0..2 = S, T, V ([S_a][S_b] each), 3..5 = their first derivatives ([6][S_a][S_b]: A_xyz,
        // B_xyz; V orbital part), 6 = dipole, 7 = momentum, 8 = angular momentum ([3][S_a][S_b],
        // x, y, z; `origin` for 6 and 8), 9 = erf-attenuated V (`omegas`, one per charge).  Charges as
        // above, null = the nuclei.  out_dev: device memory.
        void oneElectronBatch(bool use_symm, int cls, int op, long long n_tasks, const uint32_t *pairs_host,
                              const double *charges_host, int n_charges, double *out_dev,
                              const double *omegas_host = nullptr, const double *origin = nullptr);
        // Whole-matrix form of ops 6..9 over every shell pair: out_dev [blocks][nao][nao], the lower
        // triangle mirrored (negated for the antisymmetric momentum and angular momentum).
        void oneElectronOperator(int op, const double *charges_host, int n_charges, const double *omegas_host,
                                 const double *origin, double *out_dev);
        // grad[atom][xyz] = d/dR ( sum_mn D_mn (T + V)_mn - sum_mn W_mn S_mn ), the nuclei as the
        // charges of V (orbital and operator parts); D, W symmetric device matrices, either may be null.
        void oneElectronGrad(const double *D_dev, const double *W_dev, double *grad_dev);
        std::vector<double> nucleiCharges() const;

        void sync();
        // Throws kStatusTimeout when a kernel reported a bounded wait that gave up (synchronises);
        // the status word is cleared first, so the context stays usable.
        void checkStatus();
        // Runs one bounded wait that cannot complete (a barrier that nothing arrives on, no copy in
        // flight) with `polls` polls, then checkStatus(): exercises the give-up path end to end.
        void checkBoundedWait(int polls);
        // The next kernel-API store call (eri4/eri3/eri2 batches, their no-allocation form) runs its
        // bulk-copy classes without issuing the copies, so their waits give up after `polls` polls
        // (1 .. 2^20) and the call returns kStatusTimeout; one call only, 0 cancels.
        void injectWaitTimeout(int polls);
        // Evaluates the device special functions for tests: which 0 = e^{-x} (out[i]), 1 = FP64 Boys
        // F_0..F_order (out[i * (order + 1) + k]), 2 = the FP32 Boys form; x in [0, 700] resp. x >= 0.
        void evalSpecial(int which, int order, long long n, const double *x_dev, double *out_dev);
        // Cached device staging buffer `slot` (0..3) of at least n doubles (grow-only).
        double *staging(int slot, size_t n);

    private:
        // Schwarz order of one class: pairs grouped by primitive-pair count K, decreasing Q inside
        // a group (see jkPlan).
        struct ClassOrder
        {
            struct Group
            {
                uint32_t k, start, end;
                int32_t mol;  // packed-matrix base of the group's molecule (batches)
                int bucket;   // floor(log4 Q) of its pairs
                double qmax, qmin;
            };
            std::vector<uint32_t> order;
            std::vector<double> q;   // Q per position
            std::vector<double> qs;  // per group, its Q values in decreasing order (same index range)
            std::vector<Group> groups;
            uint32_t *d_order = nullptr;
            double *d_q = nullptr;   // Q per position (device)
        };
        struct ClassSet
        {
            bool built = false;
            bool schwarz_done = false;
            std::vector<PairClass> host;
            std::vector<DevPairClass> dev;
            std::vector<bool> swapped;
            std::vector<std::pair<int, int>> req_l;
            std::vector<ClassOrder> orders;
        };
        struct JKClassPair
        {
            int cb = 0, ck = 0, n_bra = 0;
            bool swap = false;  // RI plans: bra is the auxiliary class
            long long n64 = 0, n32 = 0;  // surviving quartets
            long long t64 = 0, t32 = 0;  // launched tasks (whole bra groups; the kernels test each)
            bool all64 = false;          // mixed plan, but every quartet of this pair in FP64
            double prim64 = 0, prim32 = 0, flops64 = 0, flops32 = 0;
            unsigned long long *prefix64 = nullptr, *prefix32 = nullptr;
            uint32_t *begin64 = nullptr, *begin32 = nullptr, *majors = nullptr;
            // work-queue chunks (task boundaries) and the runs they are cut from
            unsigned long long *chunks64 = nullptr, *chunks32 = nullptr;
            long long n_chunks64 = 0, n_chunks32 = 0;
            std::vector<unsigned long long> run64, run32;
            std::vector<double> cost;
            // launch parameters (autotuned): resident blocks per SM divided by grid_div, chunks of
            // at most chunk_mult work units
            int grid_div64 = 1, grid_div32 = 1, chunk_mult64 = 8, chunk_mult32 = 8;
            // tile-shape variant of the class kernel (0 default, 1 the alternative), autotuned
            int shape64 = 0, shape32 = 0;
            unsigned long long *chunksD1 = nullptr;  // gradient launches: chunks of one-quartet units
            long long n_chunksD1 = 0;
            int branch = 0;  // stream branch of the fork/join launch sequence
            int tb = 0, tk = 0;  // pair types of the launched (bra, ket) classes
        };
        struct JKPlan
        {
            double thr = 0, thr32 = 0;
            long long n_quartets = 0, n_fp32 = 0;
            double n_prim = 0, flops64 = 0, flops32 = 0;
            std::vector<JKClassPair> pairs;
            unsigned long long *counters = nullptr;  // two work-queue counters per class pair
            std::string key;
            bool tuned = false;
        };
        // One class pair of a plan: bra class cb of set bs, ket class ck of set ks; `triangle`
        // keeps only unique pairs when both are the same class of the same set.
        JKClassPair buildClassPair(const ClassSet &bs, int cb, const ClassSet &ks, int ck, bool triangle,
                                   double thr, double thr32, bool mixed);
        JKPlan &riPlan(double thr);
        JKPlan &ri2Plan(double thr);
        QuartetArgs riArgs(const JKPlan &plan, size_t ip);
        LaunchFn riLaunchFn(const JKPlan &plan, size_t ip);

        void rebuildChunks(JKClassPair &cp, bool fp32, int mult);
        void assignBranches(JKPlan &plan);
        struct LaunchTimer;
        void enqueueJK(JKPlan &plan, const double *D, double *J, double *K, bool mixed, LaunchTimer *timer = nullptr);
        void gatherDab(const double *D);
        void applyTuneCache(JKPlan &plan);
        void requireSingle() const;
        void releaseGraph();
        void clearStructure();
        void freeSet(ClassSet &cs);
        void freePlan(JKPlan &p);
        void requireStructure() const;
        static std::vector<Shell> shellsL(const std::vector<Shell> &all, int l);
        void uploadClass(const PairClass &pc, bool with_d1, bool with_f32, DevPairClass &d);
        ClassSet &mainSet(bool use_symm);
        ClassSet &auxSet();
        static PairView view(const DevPairClass &d);
        void runStore(const DevPairClass &bra, bool bra_swapped, const DevPairClass &ket, bool ket_swapped,
                      const uint32_t *d_list, long long n, bool d1, double *d_out, bool same_class);
        std::vector<std::vector<double>> diagonalBatches(ClassSet &cs);
        void ensureSchwarz(ClassSet &cs);
        JKPlan &jkPlan(double thr, double thr32, bool mixed);

        int device_ = 0;
        int num_sms_ = 0;
        cudaStream_t stream_ = nullptr;
        double *boys_ = nullptr;
        float *boys_f_ = nullptr;
        int *sph_rc_ = nullptr;
        double *sph_val_ = nullptr;
        std::vector<int> sph_ofs_;
        std::vector<void *> persistent_;

        int *d_status_ = nullptr;
        int wait_inject_ = 0;  // see injectWaitTimeout
        double *staging_[4] = {};
        size_t staging_n_[4] = {};
        static constexpr int kBranches = 4;
        cudaStream_t branch_[kBranches] = {};
        cudaEvent_t fork_ = nullptr, join_[kBranches] = {};
        cudaGraphExec_t graph_exec_ = nullptr;
        std::string graph_key_;
        std::string tune_cache_;
        std::string gpu_name_;

        bool batch_ = false;
        std::vector<std::vector<Shell>> mol_shells_;
        std::vector<long long> mol_nao_, mol_base_;
        long long packed_ = 0;
        long long *d_blocks_ = nullptr;  // [n_mol][2] packed base, N_m

        bool has_structure_ = false, has_aux_ = false;
        std::vector<Shell> shells_, aux_shells_;
        size_t nao_ = 0, naux_ = 0;
        int n_atoms_ = 0, max_l_ = 0, max_l_aux_ = 0;
        ClassSet symm_, nosymm_, aux_;
        std::map<std::string, JKPlan> plans_, ri_plans_;
    };
}

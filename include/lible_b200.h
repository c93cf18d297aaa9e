/*
 * lible_b200: C ABI of the B200 electron-repulsion-integral engine.
 *
 * A drop-in for the `lible::ints` calls of MihkuU/Lible that produce 2-, 3- and 4-centre ERIs and
 * their first nuclear derivatives, plus Schwarz-screened direct J/K, RI-J and the J/K energy
 * gradient.  Every entry point returns a lible_gpu_status; a human-readable message for the last
 * failure on a context is available from lible_gpu_last_error().  No C++ exception crosses this
 * boundary.
 *
 * Pointers: every array argument may be a host pointer or a device pointer of the context's GPU;
 * the library detects which (cudaPointerGetAttributes) and stages host arrays through device memory.
 * Layouts are row-major, matching the reference's VectorMD (src/lible/vectormd.hpp:24-27).
 *
 * Conventions (identical to the reference): coordinates in bohr internally; `units` = 0 means the
 * caller passes Angstrom, converted with 1/0.5291772083 (src/lible/ints/defs.hpp:9-12); AO order is
 * atom -> shell (basis-file order) -> m = 0, +1, -1, +2, -2, ...
 *
 * Threading: a context owns one CUDA stream.  Calls on one context may come from several threads
 * (the reference calls its kernel functors concurrently from OpenMP threads, src/lible/ints/twoel/
 * eri4.cpp:55-63): each call holds the context's lock, so they run one after another.  Different
 * contexts run independently.  lible_gpu_last_error reports the calling thread's last failure on
 * the context.
 */
#ifndef LIBLE_B200_H
#define LIBLE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lible_gpu_ctx lible_gpu_ctx;

typedef enum lible_gpu_status {
    LIBLE_GPU_OK = 0,
    LIBLE_GPU_EINVAL = 1,        /* invalid argument (index out of range, bad size, null pointer) */
    LIBLE_GPU_ECUDA = 2,         /* CUDA runtime error */
    LIBLE_GPU_ENOSTRUCT = 3,     /* no structure set on the context */
    LIBLE_GPU_ENORI = 4,         /* RI call without an auxiliary basis; reference: eri2.cpp:29-30, eri3.cpp:9-10 */
    LIBLE_GPU_EUNSUPPORTED = 5,  /* angular momentum / class outside the instantiated range */
    LIBLE_GPU_ETIMEOUT = 6,      /* a bounded device wait gave up */
    LIBLE_GPU_EINTERNAL = 7
} lible_gpu_status;

/* ---- context ------------------------------------------------------------------------------ */
int lible_gpu_create(int device, lible_gpu_ctx **ctx);
int lible_gpu_destroy(lible_gpu_ctx *ctx);
const char *lible_gpu_last_error(const lible_gpu_ctx *ctx);

/* ---- structure ------------------------------------------------------------------------------
 * Replaces lible::ints::Structure(basis_set, [basis_set_aux,] atomic_nrs, coords_angstrom)
 * (src/lible/ints/structure.hpp:18-27).  Basis files are read from <root>/<family>/<name>.txt in
 * the reference's text format (src/lible/ints/basis_sets.cpp:214-277).  aux_basis may be NULL. */
int lible_gpu_set_structure_named(lible_gpu_ctx *ctx, const char *basis_root, const char *basis,
                                  const char *aux_root, const char *aux_basis, int n_atoms,
                                  const int *atomic_nrs, const double *xyz, int units);

/* Replaces Structure(basis_atoms_t, [basis_atoms_t,] atomic_nrs, coords) (structure.hpp:29-35):
 * per-atom shell counts, then per shell l and primitive count, then exponents / coefficients
 * concatenated.  The aux_* arrays may all be NULL. */
int lible_gpu_set_structure(lible_gpu_ctx *ctx, int n_atoms, const int *atomic_nrs, const double *xyz,
                            int units, const int *shells_per_atom, const int *shell_l,
                            const int *shell_nprim, const double *exps, const double *coeffs,
                            const int *aux_shells_per_atom, const int *aux_shell_l,
                            const int *aux_shell_nprim, const double *aux_exps, const double *aux_coeffs);

/* Structure::getDimAO / getDimAOAux / getNAtoms / getMaxL (structure.hpp:70-92). */
int lible_gpu_dims(lible_gpu_ctx *ctx, long long *nao, long long *naux, int *n_atoms, int *max_l);

/* ---- full tensors ----------------------------------------------------------------------------
 * vec4d eri4(const Structure&)            (src/lible/ints/ints.hpp:165; twoel/eri4.cpp:38-95)   out[N^4]
 * vec2d eri4Diagonal(const Structure&)    (ints.hpp:168; eri4.cpp:152-174)                    out[N^2]
 * vec3d eri3(const Structure&)            (ints.hpp:171; eri3.cpp:7-48)                        out[N*N*Naux]
 * vec2d eri2(const Structure&)            (ints.hpp:174; eri2.cpp:27-72)                       out[Naux^2]
 * std::vector<double> eri2Diagonal(...)   (ints.hpp:177; eri2.cpp:74-96)                       out[Naux]   */
int lible_gpu_eri4(lible_gpu_ctx *ctx, double *out);
int lible_gpu_eri4_diagonal(lible_gpu_ctx *ctx, double *out);
int lible_gpu_eri3(lible_gpu_ctx *ctx, double *out);
int lible_gpu_eri2(lible_gpu_ctx *ctx, double *out);
int lible_gpu_eri2_diagonal(lible_gpu_ctx *ctx, double *out);

/* ---- kernel API (shell-pair classes) -----------------------------------------------------------
 * Classes are those of shellPairData(use_symm, structure) (src/lible/ints/shell_pair_data.cpp:294-309)
 * and shellDataAux(structure) (:280-292), in the same order, with the same pair lists and primitive
 * screening.  ls[2*i], ls[2*i+1] = (la, lb) of class i. */
int lible_gpu_pair_classes(lible_gpu_ctx *ctx, int use_symm, int *n_classes, int *ls,
                           long long *n_pairs, long long *n_ppairs);
int lible_gpu_aux_classes(lible_gpu_ctx *ctx, int *n_classes, int *ls, long long *n_shells);

/* Batched ERI4Kernel::operator()(ipair_ab, ipair_cd, sp_ab, sp_cd) (twoel/eri_kernels.hpp:60-76):
 * pairs[2*i], pairs[2*i+1] = (ipair_ab, ipair_cd); out[i] = the vec4d batch [Sa][Sb][Sc][Sd]. */
int lible_gpu_eri4_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                         const unsigned *pairs, double *out);
/* ERI4D1Kernel (eri_kernels.hpp:114-132): out[i] = 12 blocks [A,B,C,D] x [x,y,z], each [Sa][Sb][Sc][Sd]. */
int lible_gpu_eri4d1_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                           const unsigned *pairs, double *out);
/* lible_gpu_eri4_batch for callers that cannot allocate device memory (no counterpart in the
 * reference).  A host program that has handed all free device memory to its own pool allocator, or
 * that overlaps work on other streams and cannot accept the device-wide synchronisation cudaFree
 * implies, can call this instead: it performs no cudaMalloc, cudaFree or other allocating call.
 * The pair list is staged in a fixed 8 MiB buffer inside the library's device image (held on every
 * GPU that loads the library until the process exits), so n may be at most 1048576 pairs; larger n
 * returns LIBLE_GPU_EINVAL.  pairs must be host memory, out device memory of the context's GPU.
 * The context must hold a single structure (a batch context returns LIBLE_GPU_EUNSUPPORTED), and
 * its shell-pair classes must already be on the device: call lible_gpu_pair_classes(ctx, use_symm,
 * ...) once first.  Every call looks up the buffer's device address (cudaGetSymbolAddress); the
 * first call on a device may load the module, so make it before any stream capture.  A bounded
 * device wait that gives up returns LIBLE_GPU_ETIMEOUT, as for lible_gpu_eri4_batch.  All calls
 * share the buffer: calls whose GPU work overlaps (other streams or contexts on the same device)
 * race. */
int lible_gpu_eri4_batch_noalloc(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                                 const unsigned *pairs, double *out);
/* ERI3Kernel (eri_kernels.hpp:78-94): idx[2*i] = ipair_ab, idx[2*i+1] = ishell_c; out[i] = [Sa][Sb][Sc]. */
int lible_gpu_eri3_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int aux_class, long long n,
                         const unsigned *idx, double *out);
/* ERI3D1Kernel (eri_kernels.hpp:134-151): out[i] = 9 blocks [A,B,C] x [x,y,z]. */
int lible_gpu_eri3d1_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int aux_class, long long n,
                           const unsigned *idx, double *out);
/* ERI2Kernel (eri_kernels.hpp:96-112) and ERI2D1Kernel (:153-169, 6 blocks [A,B] x [x,y,z]). */
int lible_gpu_eri2_batch(lible_gpu_ctx *ctx, int aux_class_a, int aux_class_b, long long n,
                         const unsigned *idx, double *out);
int lible_gpu_eri2d1_batch(lible_gpu_ctx *ctx, int aux_class_a, int aux_class_b, long long n,
                           const unsigned *idx, double *out);
/* ERI4SOCKernel / ERI3SOCKernel (twoel/eri_kernels.hpp:187-223): the three Cartesian components of the
 * two-electron spin-orbit integrals, out[i] = [3][Sa][Sb][Sc][Sd] (resp. [3][Sa][Sb][Sc]).
 * ERI2D2Kernel (eri_kernels.hpp:171-185): second derivatives of (P|Q), out[i] = [6][6][Sa][Sb]
 * (A_xyz, B_xyz twice).  Pairs as for the batches above. */
int lible_gpu_eri4soc_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int class_cd, long long n,
                            const unsigned *pairs, double *out);
int lible_gpu_eri3soc_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int aux_class, long long n,
                            const unsigned *pairs, double *out);
int lible_gpu_eri2d2_batch(lible_gpu_ctx *ctx, int aux_class_a, int aux_class_b, long long n, const unsigned *pairs,
                           double *out);

/* ---- direct Coulomb / exchange (no reference counterpart; built on the eri4 kernels) ----------
 * J_mn = sum_ls (mn|ls) D_ls,  K_mn = sum_ls (ml|ns) D_ls over Schwarz-surviving unique quartets
 * (Q_ab Q_cd >= schwarz_threshold, Q_ab = max sqrt|(mn|mn)| over the pair).  precision 0 = FP64;
 * 1 = quartets with Q_ab Q_cd < fp32_threshold evaluated in FP32 (Boys function and J/K
 * accumulation stay FP64).  D must be symmetric, N x N. */
typedef struct lible_gpu_jk_opts {
    double schwarz_threshold;  /* default 1e-12 */
    double fp32_threshold;     /* default 1e-4 */
    int precision;             /* 0 FP64, 1 mixed */
    int use_graph;             /* 1: capture the launch sequence once per (plan, D, J, K) in a CUDA graph
                                  and replay it; the first call per buffer set must not be inside a
                                  caller's stream capture */
} lible_gpu_jk_opts;

typedef struct lible_gpu_jk_stats {
    long long n_quartets;      /* unique contracted shell quartets evaluated */
    long long n_fp32;          /* of which in FP32 */
    long long n_launches;      /* kernels launched by the call */
} lible_gpu_jk_stats;

int lible_gpu_jk(lible_gpu_ctx *ctx, const double *D, double *J, double *K, const lible_gpu_jk_opts *opts,
                 lible_gpu_jk_stats *stats);

/* ---- batches of molecules (no reference counterpart) -------------------------------------------
 * A context can hold a batch of molecules instead of one structure: their J/K are built together,
 * every quartet class of every molecule going through one persistent work-queue launch per class,
 * and lible_gpu_jk with use_graph replays the whole sequence as one CUDA graph.  Molecule m has
 * n_atoms[m] atoms (atomic_nrs and xyz concatenated over molecules, xyz as 3 per atom) and the basis
 * basis[m], read from basis_root like lible_gpu_set_structure_named.  D, J and K are then packed:
 * molecule m's N_m x N_m row-major matrix starts at element base[m] (lible_gpu_batch_layout), and
 * lible_gpu_jk / lible_gpu_jk_energy_forward / lible_gpu_jk_plan* / lible_gpu_jk_autotune take
 * packed arrays of *packed elements.  Other calls return LIBLE_GPU_EUNSUPPORTED for a batch. */
int lible_gpu_set_batch(lible_gpu_ctx *ctx, int n_mol, const char *basis_root, const char *const *basis,
                        const int *n_atoms, const int *atomic_nrs, const double *xyz, int units);
int lible_gpu_batch_layout(lible_gpu_ctx *ctx, int *n_mol, long long *nao, long long *base, long long *packed);

/* Autotuner of the J/K class launches: for every class pair of the plan for opts, times each
 * candidate on D/J/K with CUDA events and keeps the fastest.  Candidates: the kernel's tile shape
 * (the default, and where it differs the alternative: twice the warps per quartet on the group
 * paths, the next larger thread group per quartet on the register path, or the default register
 * bound for classes compiled with a raised occupancy bound), the class in the other orientation
 * ((cd|ab) for (ab|cd), where that orientation takes the register path), resident blocks per SM
 * (all or half) and work-queue chunks of 2, 8 or 32 work units.  J and K are overwritten with
 * meaningless values.  When cache_path is non-empty the choices are appended to that text file;
 * lible_gpu_set_tune_cache(ctx, path) makes later plans start from a cache.  summary (may be NULL)
 * receives one line per class pair. */
int lible_gpu_jk_autotune(lible_gpu_ctx *ctx, const double *D, double *J, double *K, const lible_gpu_jk_opts *opts,
                          const char *cache_path, char *summary, int summary_len);
int lible_gpu_set_tune_cache(lible_gpu_ctx *ctx, const char *path);

/* Per-launch timing of one J/K build (no reference counterpart; the reference's only timing hook
 * is eri4Benchmark, src/lible/ints/twoel/eri4.cpp:97-150): every class launch runs serialised on
 * the context stream between two CUDA events.  On entry *n is the capacity of the arrays (any of
 * which may be NULL); on return *n is the number of launches.  Per launch: ls[4i..4i+3] = (la, lb,
 * lc, ld), fp32[i] (bit 0: FP32 arithmetic; bits 1-2: the shape the autotuner chose, 1 = the
 * alternative tile shape, 2 = the other orientation), ms[i], algorithmic FLOPs flops[i] and
 * quartets tasks[i].  J, K receive the
 * build's result. */
int lible_gpu_jk_profile(lible_gpu_ctx *ctx, const double *D, double *J, double *K, const lible_gpu_jk_opts *opts,
                         int *n, int *ls, int *fp32, double *ms, double *flops, long long *tasks);

/* Size of the (cached) screening plan for these options: quartets, primitive quartets and the
 * algorithmic FP64 / FP32 FLOPs one lible_gpu_jk call performs (dense-equivalent count). */
typedef struct lible_gpu_jk_plan_info {
    long long n_quartets;
    long long n_fp32;
    long long n_prim_quartets;
    long long n_launches;
    double flops_fp64;
    double flops_fp32;
} lible_gpu_jk_plan_info;

int lible_gpu_jk_plan(lible_gpu_ctx *ctx, const lible_gpu_jk_opts *opts, lible_gpu_jk_plan_info *info);

/* Per class pair of that plan, in launch order: ls[4*i..4*i+3] = (la, lb, lc, ld), quartets in
 * FP64 / FP32, primitive quartets, algorithmic FLOPs.  Call with ls == NULL to get *n only. */
int lible_gpu_jk_plan_classes(lible_gpu_ctx *ctx, const lible_gpu_jk_opts *opts, int *n, int *ls,
                              long long *n64, long long *n32, double *n_prim, double *flops);

/* The context's CUDA stream (cudaStream_t), for callers that time or order work around the calls. */
int lible_gpu_stream(lible_gpu_ctx *ctx, void **stream);

/* Measured FP64 throughput of this GPU (TFLOP/s): a register-resident DFMA loop and a DMMA
 * (mma.sync m8n8k4 f64) loop; the roofline denominators of the engine's kernels. */
int lible_gpu_fp64_peak(lible_gpu_ctx *ctx, double *dfma_tflops, double *dmma_tflops);
/* Measured FP32 throughput (TFLOP/s): a scalar FFMA loop and a packed fma.rn.f32x2 loop; the
 * roofline denominators of the FP32 quartet kernels. */
int lible_gpu_fp32_peak(lible_gpu_ctx *ctx, double *ffma_tflops, double *ffma2_tflops);

/* Diagnostic of the failure path of the kernels' bounded waits: one wait on a barrier that nothing
 * completes gives up after `polls` polls (1 .. 2^20) and the call returns LIBLE_GPU_ETIMEOUT, the
 * status a stalled bulk copy produces.  No copy is in flight and the context stays usable.  It has
 * no counterpart in the reference, whose CPU code has no device waits. */
int lible_gpu_check_bounded_wait(lible_gpu_ctx *ctx, int polls);

/* The same failure path in the real class kernels: the next kernel-API store launch on the context
 * (lible_gpu_eri4_batch, lible_gpu_eri4_batch_noalloc, ...) runs its bulk-copy (DMMA) classes
 * without issuing the ket-tile copies, so their first wait gives up after `polls` polls (1 .. 2^20);
 * the block stops without using the tile and the call returns LIBLE_GPU_ETIMEOUT.  Applies to one
 * launch; 0 cancels.  No copy is in flight and the context stays usable.  No reference counterpart. */
int lible_gpu_inject_wait_timeout(lible_gpu_ctx *ctx, int polls);

/* The device special functions of the class kernels, evaluated directly (for their tests; no
 * reference counterpart as a call, the reference's are BoysF2 / calcBoysF, boys_function.hpp:68-109):
 * which = 0: out[i] = e^{-x[i]}, x in [0, 700]; which = 1: FP64 Boys F_0..F_order(x[i]) into
 * out[i*(order+1) + k], order <= 14; which = 2: the FP32 Boys form used by FP32 quartets. */
int lible_gpu_eval_special(lible_gpu_ctx *ctx, int which, int order, long long n, const double *x, double *out);

/* ---- J/K energy and its nuclear gradient (forward / backward pair) ----------------------------
 * forward:  E = 1/2 Tr(D J) - 1/4 Tr(D K)  (J, K from lible_gpu_jk with opts; J/K may be NULL).
 * backward: grad[3*atom + x] = dE/dR_{atom,x}, contracting the first-derivative integrals
 *           (ERI4D1Kernel semantics) with the two-particle density of E on the device, over the
 *           same Schwarz-surviving quartets as the FP64 forward pass with opts->schwarz_threshold
 *           (opts->precision is ignored: the gradient is FP64). */
int lible_gpu_jk_energy_forward(lible_gpu_ctx *ctx, const double *D, const lible_gpu_jk_opts *opts,
                                double *energy, double *J, double *K);
int lible_gpu_jk_energy_backward(lible_gpu_ctx *ctx, const double *D, const lible_gpu_jk_opts *opts,
                                 double *grad);

/* ---- RI-J ------------------------------------------------------------------------------------
 * gamma_P = sum_mn (mn|P) D_mn; (P|Q) d = gamma (Cholesky, FP64); J_mn = sum_P (mn|P) d_P.
 * Three-centre quartets with Q_mn Q_P < schwarz_threshold are skipped (Q_P = sqrt (P|P)).
 * gamma / dcoef outputs may be NULL.  The first call builds the tensor (mn|P), its lower
 * triangle in m, n (naux * nao (nao + 1) / 2 doubles), in device memory when it takes at most 60%
 * of the free memory and keeps it while the structure and the threshold stay the same; later calls
 * then contract that tensor instead of evaluating the integrals twice.  The metric factor is kept
 * the same way. */
int lible_gpu_rij(lible_gpu_ctx *ctx, const double *D, double schwarz_threshold, double *J, double *gamma,
                  double *dcoef);
/* mode 1 (default): lible_gpu_rij keeps the three-centre tensor when it fits; 0: never build it
 * (frees a cached one) and evaluate the integrals on every call. */
int lible_gpu_rij_set_cached(lible_gpu_ctx *ctx, int mode);
/* How the last lible_gpu_rij solved (P|Q) d = gamma: method 0 = Cholesky (lo, hi = smallest and
 * largest squared diagonal of the factor, a lower bound of the condition number hi/lo); 2 = the
 * metric was not numerically positive definite and Cholesky of (P|Q) + shift I succeeded (shift =
 * 1e-11 of the largest diagonal element); 1 = eigendecomposition (when that also failed: lo, hi =
 * smallest kept and largest eigenvalue, `dropped` eigenpairs below 1e-12 of the largest left out);
 * -1 = none yet.  Any output may be NULL. */
int lible_gpu_rij_last_solve(lible_gpu_ctx *ctx, int *method, double *lo, double *hi, int *dropped, double *shift);
/* Gradient of the RI-J energy E = 1/2 gamma^T (P|Q)^{-1} gamma (= 1/2 Tr(D J_RI)) with respect to
 * the nuclear coordinates, grad[n_atoms][3]:
 *   sum_P d_P sum_mn D_mn d(mn|P)/dR - 1/2 sum_PQ d_P d_Q d(P|Q)/dR,   d = (P|Q)^{-1} gamma,
 * the derivative integrals (ERI3D1 / ERI2D1 semantics, src/lible/ints/twoel/eri_kernels.hpp:134-169)
 * contracted inside the class kernels.  D symmetric; `energy` (may be NULL) receives E. */
int lible_gpu_rij_grad(lible_gpu_ctx *ctx, const double *D, double schwarz_threshold, double *grad, double *energy);
/* The two contractions separately (either output may be NULL). */
int lible_gpu_ri_contract(lible_gpu_ctx *ctx, const double *D, const double *dcoef, double schwarz_threshold,
                          double *gamma, double *J);

/* ---- one-electron integrals ------------------------------------------------------------------
 * lible::ints::overlap, kineticEnergy, nuclearAttraction and externalCharges
 * (src/lible/ints/ints.hpp:29-61, oneelints.cpp:169-197, 348-376, 1087-1120, 1703-1744): full
 * nao x nao matrices, AO order as eri4.  Point charges are [n_charges][4] = x, y, z (bohr), q; the
 * potential is that of the charges acting on an electron (negative for positive q), as in the
 * reference.  lible_gpu_one_electron computes any subset in one pass (NULL outputs are skipped;
 * charges NULL = the nuclei).  Main-basis shells up to l = 3; charges in host memory, outputs host
 * or device. */
int lible_gpu_overlap(lible_gpu_ctx *ctx, double *out);
int lible_gpu_kinetic_energy(lible_gpu_ctx *ctx, double *out);
int lible_gpu_nuclear_attraction(lible_gpu_ctx *ctx, double *out);
int lible_gpu_external_charges(lible_gpu_ctx *ctx, const double *charges, int n_charges, double *out);
int lible_gpu_one_electron(lible_gpu_ctx *ctx, const double *charges, int n_charges, double *S, double *T,
                           double *V);
/* The per-pair kernels of the reference: overlapKernel, kineticEnergyKernel, externalChargesKernel
 * (op 0, 1, 2; blocks [S_a][S_b]) and overlapD1Kernel, kineticEnergyD1Kernel,
 * externalChargesD1Kernel (op 3, 4, 5; [6][S_a][S_b] = d/dA x, y, z, d/dB x, y, z; for op 5 the
 * orbital part, as the reference) for `n` pair indices of class `class_ab` of
 * lible_gpu_pair_classes(use_symm) (src/lible/ints/ints.hpp:33-93, oneelints.cpp:57-164, 199-346,
 * 508-789).  charges as above (NULL = the nuclei); out: n consecutive blocks, host or device. */
int lible_gpu_one_electron_batch(lible_gpu_ctx *ctx, int use_symm, int class_ab, int op, long long n,
                                 const unsigned *pairs, const double *charges, int n_charges, double *out);
/* The same with the remaining per-pair kernels: op 6 dipoleMomentKernel, 7 momentumKernel, 8
 * angularMomentumKernel ([3][S_a][S_b] = x, y, z; `origin` [3] for 6 and 8, bohr), op 9
 * externalChargesErfKernel ([S_a][S_b]), op 10 externalChargesErfD1Kernel ([6][S_a][S_b], orbital
 * part), op 11 / 12 the operator part d/dC_xyz of externalChargesKernel / externalChargesErfKernel
 * summed over the given charges ([3][S_a][S_b]; one charge per call gives the reference's
 * externalChargesOperator(Erf)D1Kernel entry for that charge), op 13 spinOrbitCoupling1ElKernel
 * ([3][S_a][S_b], the given charges; ints.hpp:135-137, oneelints.cpp:1209-1316), op 14 pVpKernel
 * ([3][3][S_a][S_b] = <d_i a| V |d_j b> for the given charges; ints.hpp:159-161; see pVpIntegrals).  `omegas`: one range parameter per
 * charge for 9, 10, 12 (NULL charges = the nuclei, one omega per atom; 9 scales a charge by
 * w / sqrt(w^2 + p), 10 and 12 by sqrt(w^2 / (w^2 + p)), as the reference's kernels do) (ints.hpp:66-148;
 * oneelints.cpp:379-473, 587-680, 791-889, 1513-1577, 1617-1701, 1844-2060).  Unused pointers may be
 * NULL. */
int lible_gpu_one_electron_batch_ex(lible_gpu_ctx *ctx, int use_symm, int class_ab, int op, long long n,
                                    const unsigned *pairs, const double *charges, const double *omegas, int n_charges,
                                    const double *origin, double *out);
/* Whole-matrix forms, out [3][nao][nao] (x, y, z) or [nao][nao], host or device:
 *   dipoleMoment (ints.hpp:123-125): <m| r - origin |n>, symmetric;
 *   momentum (ints.hpp:139): -<m| d/dr |n>, antisymmetric, every element filled (the reference's
 *     driver, oneelints.cpp:1477-1511, writes only the (a, b) blocks of its unique pairs, negated);
 *   angularMomentum (ints.hpp:146-147): -<m| (r - origin) x d/dr |n>, antisymmetric;
 *   nuclearAttractionErf (ints.hpp:52): the nuclei's erf(w r)/r attraction, `omegas` one per atom;
 *   externalChargesErf (ints.hpp:60-62): the same for point charges [n][4], one omega each;
 *   spinOrbitCoupling1El (ints.hpp:131): the one-electron SOC integrals of the nuclei, antisymmetric;
 *   pVpIntegrals (ints.hpp:154): out [3][3][nao][nao], <d_i m| V |d_j n> for the nuclei (charges
 *     NULL) or the point charges [n][4], with out[i][j] = out[j][i]^T.  These are the integrals themselves: the reference's pVpKernel leaves
 *     out the E factor of its first term and the R factor of its last and builds its x second-
 *     derivative coefficients from the y first derivatives (oneelints.cpp:1392-1460, ecoeffs.cpp:
 *     205), and its driver mirrors each component without exchanging i and j, so its values differ. */
int lible_gpu_dipole_moment(lible_gpu_ctx *ctx, const double *origin, double *out);
int lible_gpu_momentum(lible_gpu_ctx *ctx, double *out);
int lible_gpu_angular_momentum(lible_gpu_ctx *ctx, const double *origin, double *out);
int lible_gpu_spin_orbit_coupling_1el(lible_gpu_ctx *ctx, double *out);
int lible_gpu_pvp_integrals(lible_gpu_ctx *ctx, const double *charges, int n_charges, double *out);
int lible_gpu_nuclear_attraction_erf(lible_gpu_ctx *ctx, const double *omegas, double *out);
int lible_gpu_external_charges_erf(lible_gpu_ctx *ctx, const double *charges, const double *omegas, int n_charges,
                                   double *out);
/* Nuclear gradient of the one-electron energy terms, grad[atom][xyz] = d/dR (sum D (T + V) -
 * sum W S), V the nuclear attraction (orbital and operator parts).  D and W symmetric nao x nao,
 * either may be NULL (the term is skipped). */
int lible_gpu_one_electron_grad(lible_gpu_ctx *ctx, const double *D, const double *W, double *grad);

/* ---- RI-K ------------------------------------------------------------------------------------
 * K_mn = sum_{PQ} (ml|P) [(P|Q)^{-1}]_{PQ} (Q|ns) D_ls, the exchange half of RI-JK (no reference
 * driver; built on the reference's ERI3Kernel / eri2 semantics, src/lible/ints/twoel/
 * eri_kernels.cpp:1122-1162, and Schwarz-screened like lible_gpu_rij).  The density is given either
 * as its factor C ([nao][n_occ] row-major, D = C C^T; D may then be NULL) or, with C NULL, as the
 * symmetric D itself, which is factorised by its eigendecomposition (D = C+ C+^T - C- C-^T over the
 * eigenpairs with |w| > 1e-12 max|w|).  (P|Q) is factorised as for lible_gpu_rij
 * (lible_gpu_rij_last_solve reports it).  The first call on a structure (and Schwarz threshold)
 * builds the fitted three-centre tensor B_R = sum_P F_PR (mn|P) with the metric's factor F
 * (naux * nao^2 doubles) and keeps it on the context when it takes at most 60% of the free device
 * memory; later calls are then one batched DGEMM and one DSYRK.  Without the room every call
 * streams blocks of integrals and solves with the factor.  `info` (may be NULL) receives the
 * factor ranks, the number of auxiliary blocks, per-stage device times (t_ints includes the
 * tensor build on the call that made it) and FLOP counts, and whether the tensor was used.
 * D, C, K: host or device. */
typedef struct lible_gpu_rik_info
{
    long long n_pos, n_neg;  /* columns of C+ and C- (n_occ and 0 when C is given) */
    int n_blocks;            /* blocks of auxiliary functions the three-centre integrals were built in */
    double t_ints, t_gemm, t_solve, t_syrk;               /* seconds */
    double flops_gemm, flops_solve, flops_syrk;           /* algorithmic FLOPs of the three stages */
    int fitted;              /* 1: the cached fitted tensor served the call */
} lible_gpu_rik_info;
int lible_gpu_rik(lible_gpu_ctx *ctx, const double *D, const double *C, long long n_occ, double schwarz_threshold,
                  double *K, lible_gpu_rik_info *info);
/* mode 1 (default): RI-K keeps the fitted tensor when it fits; 0: never build it (frees a cached one)
 * and stream the integrals on every call. */
int lible_gpu_rik_set_fitted(lible_gpu_ctx *ctx, int mode);

/* ---- host-only helpers (no GPU needed) --------------------------------------------------------
 * The host set-up the kernels consume, exposed for checking against the reference:
 *  - sphericalTrafo(l) (src/lible/ints/spherical_trafo.cpp:9-690): up to *n (row, cart, value) terms;
 *  - shell AO norms from the spherical self-overlap (src/lible/ints/shell.cpp:11-46);
 *  - shell-pair class sizes of shellPairData(use_symm, structure) (shell_pair_data.cpp:73-309);
 *  - the Boys function F_0..F_n(x) by the engine's grid method (boys_function.cpp:71-118). */
int lible_host_spherical_trafo(int l, int *n, int *rows, int *carts, double *vals);
int lible_host_shell_norms(int l, int n_prim, const double *exps, const double *coeffs, double *norms);
int lible_host_pair_classes(const char *basis_root, const char *basis, int n_atoms, const int *atomic_nrs,
                            const double *xyz, int units, int use_symm, int *n_classes, int *ls,
                            long long *n_pairs, long long *n_ppairs);
int lible_host_boys(int n, double x, double *F);

#ifdef __cplusplus
}
#endif

#endif /* LIBLE_B200_H */

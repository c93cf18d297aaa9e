#!/usr/bin/env python
"""Direct J+K build benchmark: (H2O)_32 / cc-pVDZ (768 basis functions), Schwarz 1e-12.

One step = one J+K build from a device-resident density D to device-resident J and K (unique
Schwarz-surviving quartets, all quartet classes).  The reported `value` is unique contracted shell
quartets per second of the whole job (N GPUs run independent replicas: the path has no collective).
The default path is the mixed-precision build (quartets with Q_ab Q_cd < 1e-4 in FP32) when it
meets |dE| <= 1e-8 Eh against the FP64 build of the same run; the FP64 build is always timed and
reported beside it.  Set-up (basis, E coefficients, Schwarz factors, screening plan) is excluded
and reported separately.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import math
import os
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "J+K build s and quartets/s, (H2O)_32 DZ: mixed/batched vs FP64 GPU, |ΔE|≤1e-8 Eh"
N_WATERS, SEED, OCC = 32, 2024, 160
SCHWARZ, FP32_THR = 1e-12, 1e-4
# DRAM bytes (read + write) per launch of the dominant class kernels at this workload, from one ncu
# capture each (dram__bytes_read.sum + dram__bytes_write.sum); the working set stays in L2
DOMINANT_TRAFFIC = {((1, 0, 0, 0), False): 34.29e6, ((2, 1, 1, 0), False): 24.16e6, ((1, 0, 0, 0), True): 28.35e6}
# L2 atomic (RED) bytes per launch of the dominant kernels, lts__t_sectors_op_red.sum x 32 from one
# ncu capture each of this workload (profiles/)
L2_ATOMIC_BYTES = {"eriKernelOcc<1,0,0,0,double,0>": 1222249650 * 32, "eriKernel<1,0,0,0,float,0>": 1107513230 * 32}
# classes whose default tile shape is compiled with a raised occupancy bound (eriKernelOcc,
# minBlocksPerSM in lible_b200/csrc/eri_kernel.cuh): (class, fp32)
OCC_KERNELS = {(c, f) for c, f in [((2, 1, 1, 0), False), ((2, 0, 1, 0), False), ((2, 1, 0, 0), False),
                                                  ((1, 0, 0, 0), False), ((2, 1, 1, 0), True), ((2, 0, 1, 1), True),
                                                  ((1, 1, 1, 0), True), ((1, 0, 1, 0), True), ((2, 0, 0, 0), True)]}
WORKLOAD = {"workload": "direct J+K build, (H2O)_32 water cluster, cc-pVDZ", "n_waters": N_WATERS, "nao": 768,
            "seed": SEED, "occupied": OCC, "schwarz": SCHWARZ, "fp32_threshold": FP32_THR,
            "geometry": "5.7 bohr cubic lattice, random rotations, +-0.6 bohr jitter",
            "l2": "256 MiB buffer rewritten between timed steps"}


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def max_over_ranks(x, dist=None, device="cpu"):
    """The largest value of x over all ranks (timings of a multi-GPU job are its slowest rank's)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def emit(obj):
    print(json.dumps(obj), flush=True)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def digestion_bytes(classes):
    """Algorithmic bytes of the J/K digestion of one build: per unique quartet (ab|cd), 8 bytes per
    D-block element read and 16 per J/K-block element read-modify-written, over the six blocks
    (ab), (cd), (ac), (ad), (bc), (bd) of spherical sizes n_x n_y."""
    total = 0.0
    for (la, lb, lc, ld), n64, n32, _, _ in classes:
        na, nb, nc, nd = (2 * l + 1 for l in (la, lb, lc, ld))
        blocks = na * nb + nc * nd + na * nc + na * nd + nb * nc + nb * nd
        total += (n64 + n32) * 24.0 * blocks
    return total


def clocks_start(gpu_index):
    # nvidia-smi samples of the timed region, in the temporary directory (summarised into the JSON line)
    path = os.path.join(tempfile.gettempdir(), f"lible_b200_clocks_{os.getpid()}_{gpu_index}.csv")
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        fh = open(path, "w")
        p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                              "-lms", "200"], stdout=fh, stderr=subprocess.DEVNULL)
        return p, fh, path
    except Exception:
        return None, None, path


def clocks_stop(handle):
    p, fh, path = handle
    if p is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    p.terminate()
    p.wait()
    fh.close()
    sm, smax, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            smax = float(f[2])
        except ValueError:
            continue
        for n, v in zip(names, f[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
            "samples": len(sm)}


def cpu_reference(steps, warmup, Z, xyz, D, target_s=12.0):
    """The reference's own ERI4Kernel batches digested into J/K on every host core (oracle/_ref),
    timed on a bounded, class-balanced sample: every `stride`-th bra shell pair of every class pair."""
    from oracle import ref as R
    cores = os.cpu_count() or 1
    R.set_threads(cores)
    r = R.RefStructure("cc-pvdz", Z, xyz)
    _, _, nq, sec = r.jk(D, SCHWARZ, 256)
    stride = max(1, int(math.ceil(256 * sec / target_s)))
    for _ in range(max(0, warmup)):
        r.jk(D, SCHWARZ, stride)
    rates = []
    for _ in range(max(1, steps)):
        _, _, nq, sec = r.jk(D, SCHWARZ, stride)
        rates.append(nq / sec)
    return float(np.mean(rates)), cores, stride, nq, sec


def oracle_jk_full(Z, xyz, D):
    """The reference's ERI4Kernel batches digested into J/K on every host core, unsampled: the CPU
    baseline of the whole workload and the oracle the GPU builds are checked against."""
    from oracle import ref as R
    cores = os.cpu_count() or 1
    R.set_threads(cores)
    r = R.RefStructure("cc-pvdz", Z, xyz)
    J, K, nq, sec = r.jk(D, SCHWARZ, 1)
    return J, K, nq, sec, cores


def run_reference(args):
    rank, local, world = env_rank()
    if rank != 0:
        return
    from lible_b200.workloads import random_density, water_cluster
    from oracle import ref as R
    if not R.available():
        emit({"impl": "reference", "unavailable": "oracle/_ref/liblible_ref.so not built (needs the reference sources)"})
        return
    Z, xyz, rng = water_cluster(N_WATERS, SEED)
    D = random_density(768, OCC, rng)
    qps, cores, stride, nq, sec = cpu_reference(args.steps, args.warmup, Z, xyz, D)
    sample = f"every {stride}-th bra shell pair of every class pair ({nq} quartets, {sec:.2f} s per step)"
    emit({"impl": "reference", "metric": METRIC, "value": qps, "unit": "quartets/s", "n_gpus": args.gpus,
          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
          "config": WORKLOAD,
          "cpu_baseline": {"value": qps, "unit": "quartets/s", "cores": cores, "kind": "reference", "sample": sample,
                           "cpu_model": cpu_model()},
          "e2e": {"value": qps, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})


def run_batch(steps, warmup, dev):
    """The heterogeneous batch: 64 water clusters (1..12 waters, half cc-pVDZ, half cc-pVTZ), FP64,
    Schwarz 1e-12.  Times the batched build (one work-queue launch per quartet class for all
    molecules, replayed from a CUDA graph, class launches autotuned once in the set-up) against the
    same molecules built one after another through the single-structure path, and the mixed
    precision batch with its largest per-molecule energy error against FP64."""
    import torch

    from lible_b200 import ints as L
    from lible_b200.workloads import batch_clusters

    specs = batch_clusters()
    t0 = time.perf_counter()
    b = L.Batch([(bs, Z, xyz) for bs, Z, xyz, _ in specs], device=dev.index or 0)
    Ds = [f(int(b.nao[m])) for m, (_, _, _, f) in enumerate(specs)]
    Dp = torch.tensor(b.pack(Ds), device=dev)
    J, K = torch.empty_like(Dp), torch.empty_like(Dp)
    plan = L.jk_plan(b, SCHWARZ, "fp64")
    setup_s = time.perf_counter() - t0
    # one-time autotuning of the batch's class launches (tile shapes, occupancy, queue granularity)
    t0 = time.perf_counter()
    L.jk_autotune(b, Dp, SCHWARZ, "fp64", J=J, K=K)
    L.jk_autotune(b, Dp, SCHWARZ, "mixed", FP32_THR, J=J, K=K)
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(L.stream_handle(b), device=dev)

    def time_batch(use_graph, precision="fp64"):
        for _ in range(warmup):
            L.jk(b, Dp, SCHWARZ, precision, FP32_THR, J=J, K=K, use_graph=use_graph)
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            L.jk(b, Dp, SCHWARZ, precision, FP32_THR, J=J, K=K, use_graph=use_graph)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.mean(ms))

    # the mixed-precision batch (FP32 for every class up to (ff|ff)): time and largest per-molecule
    # energy error against the FP64 batch
    t_mixed = time_batch(True, "mixed")
    Jx, Kx = J.cpu().numpy(), K.cpu().numpy()
    L.jk(b, Dp, SCHWARZ, "fp64", J=J, K=K)
    J64, K64 = J.cpu().numpy(), K.cpu().numpy()
    Dh = Dp.cpu().numpy()
    dE_mixed = max(abs(float(np.sum(d * (0.5 * (jx - j) - 0.25 * (kx - k)))))
                   for d, j, k, jx, kx in zip(b.unpack(Dh), b.unpack(J64), b.unpack(K64), b.unpack(Jx), b.unpack(Kx)))
    t_direct = time_batch(False)
    t_graph = time_batch(True)
    flops = plan["flops_fp64"]
    Jb = J.cpu().numpy()
    # the same molecules one by one through the single-structure path
    singles = [L.Structure(bs, Z, xyz, units="bohr", device=dev.index or 0) for bs, Z, xyz, _ in specs]
    Dd = [torch.tensor(D, device=dev) for D in Ds]
    Jm = [torch.empty_like(x) for x in Dd]
    Km = [torch.empty_like(x) for x in Dd]
    for s, D_, J_, K_ in zip(singles, Dd, Jm, Km):
        L.jk(s, D_, SCHWARZ, "fp64", J=J_, K=K_)
    torch.cuda.synchronize()
    err = max(float(np.abs(b.unpack(Jb)[m] - Jm[m].cpu().numpy()).max()) for m in range(len(specs)))
    seq = []
    for _ in range(steps):
        torch.cuda.synchronize()
        a = time.perf_counter()
        for s, D_, J_, K_ in zip(singles, Dd, Jm, Km):
            L.jk(s, D_, SCHWARZ, "fp64", J=J_, K=K_)
        torch.cuda.synchronize()
        seq.append(time.perf_counter() - a)
    t_seq = 1e3 * float(np.mean(seq))
    nq = plan["n_quartets"]
    return {"workload": "64 water clusters, 1..12 waters, half cc-pVDZ / half cc-pVTZ, FP64, Schwarz 1e-12",
            "n_molecules": len(specs), "n_quartets": nq, "n_prim_quartets": plan["n_prim_quartets"],
            "packed_elements": int(b.packed), "setup_s": setup_s, "autotune_s": tune_s,
            "batched_graph_ms": t_graph, "batched_direct_ms": t_direct, "sequential_single_ms": t_seq,
            "mixed_batched_graph_ms": t_mixed, "mixed_max_abs_dE_Eh_per_molecule": dE_mixed,
            "quartets_per_s": nq / (t_graph * 1e-3), "speedup_vs_sequential": t_seq / t_graph,
            "algorithmic_fp64_tflops": flops / (t_graph * 1e-3) / 1e12,
            "max_abs_dJ_vs_single": err}


def run_rij(Z, xyz, D, J64, steps):
    """RI-J of the (H2O)_32 workload with the even-tempered s-f auxiliary basis (0.1 * 2.5^k,
    k = 0..11 per l and atom): wall time of one lible_gpu_rij call from host D to host J (both
    contractions over the kept three-centre tensor (its packed lower triangle), and the solve with
    the cached metric factor;
    the first call, which builds both, is timed separately; the median of at least five calls, all
    listed), the rate at which a call reads the tensor (two passes, whole-call time), and the RI
    error against the direct FP64 J of the same run."""
    from lible_b200 import ints as L
    from lible_b200.workloads import even_tempered_aux

    t0 = time.perf_counter()
    s = L.Structure("cc-pvdz", Z, xyz, even_tempered_aux(Z), units="bohr")
    setup = time.perf_counter() - t0
    # first call: plans, Schwarz factors of the auxiliary classes, the metric factor and the kept
    # three-centre tensor
    t0 = time.perf_counter()
    Jri, _, _ = L.rij(s, D, SCHWARZ)
    first = time.perf_counter() - t0
    ts = []
    for _ in range(max(5, steps)):
        t = time.perf_counter()
        Jri, _, _ = L.rij(s, D, SCHWARZ)
        ts.append(time.perf_counter() - t)
    tensor_bytes = 8.0 * s.naux * s.nao * (s.nao + 1) / 2  # the packed lower triangle of (mn|P)
    return {"workload": "RI-J, (H2O)_32 cc-pVDZ, even-tempered s-f auxiliary basis, FP64", "naux": s.naux,
            "setup_s": setup, "first_call_s": first, "rij_s": float(np.median(ts)), "rij_samples_s": ts,
            "tensor_bytes": tensor_bytes,
            "tensor_read_gbs": 2 * tensor_bytes / float(np.median(ts)) / 1e9,
            "solve": L.rij_last_solve(s),
            "dEJ_Eh_vs_direct": float(0.5 * np.sum(D * (Jri - J64))),
            "dJ_fro_vs_direct": float(np.linalg.norm(Jri - J64))}


def run_rijk(Z, xyz, D, J64, K64, occ, steps):
    """RI-JK of the (H2O)_32 workload with def2-universal-jkfit (3,616 auxiliary functions): wall
    time of lible_gpu_rij (host D -> host J), of the RI-J nuclear gradient, and of lible_gpu_rik from
    the occupied factor C
    (host C -> host K; D = C C^T, C from the eigenvectors of D), with the per-stage device times
    and rates of the exchange build, and the RI errors against the direct FP64 J and K of the same
    run.  The first call of each builds and factorises (P|Q), which later calls reuse; the RI-J and
    RI-K times are medians of at least five alternating calls, all listed."""
    from lible_b200 import ints as L

    w, V = np.linalg.eigh(D)
    C = np.ascontiguousarray(V[:, -occ:] * np.sqrt(np.clip(w[-occ:], 0, None)))
    t0 = time.perf_counter()
    s = L.Structure("cc-pvdz", Z, xyz, "def2-universal-jkfit", units="bohr")
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    Jri, _, _ = L.rij(s, D, SCHWARZ)
    Kri = L.rik(s, C=C, schwarz=SCHWARZ)
    first = time.perf_counter() - t0
    tj, tk = [], []
    for _ in range(max(5, steps)):
        t = time.perf_counter()
        Jri, _, _ = L.rij(s, D, SCHWARZ)
        tj.append(time.perf_counter() - t)
        t = time.perf_counter()
        Kri, info = L.rik(s, C=C, schwarz=SCHWARZ, info=True)
        tk.append(time.perf_counter() - t)
    t = time.perf_counter()
    Kd = L.rik(s, D=D, schwarz=SCHWARZ)
    t_dpath = time.perf_counter() - t
    L.rij_grad(s, D, SCHWARZ)
    t = time.perf_counter()
    gJ, _ = L.rij_grad(s, D, SCHWARZ)
    t_grad = time.perf_counter() - t
    rates = {k: info["flops_" + k] / max(info["t_" + k], 1e-12) / 1e12 for k in ("gemm", "solve", "syrk")}
    return {"workload": "RI-JK, (H2O)_32 cc-pVDZ / def2-universal-jkfit, FP64, occupied factor C (160)",
            "naux": s.naux, "setup_s": setup, "first_call_s": first, "rij_s": float(np.median(tj)),
            "rik_s": float(np.median(tk)), "rij_samples_s": tj, "rik_samples_s": tk, "rik_from_D_s": t_dpath,
            "rij_gradient_s": t_grad,
            "rij_gradient_translational_residual": float(np.abs(gJ.sum(axis=0)).max()),
            "solve": L.rij_last_solve(s),
            "rik_stages_s": {k: info["t_" + k] for k in ("ints", "gemm", "solve", "syrk")},
            "rik_stage_tflops": rates, "rik_aux_blocks": info["n_blocks"],
            "dEJ_Eh_vs_direct": float(0.5 * np.sum(D * (Jri - J64))),
            "dEK_Eh_vs_direct": float(-0.25 * np.sum(D * (Kri - K64))),
            "dK_fro_vs_direct": float(np.linalg.norm(Kri - K64)),
            "dK_fro_C_vs_D_path": float(np.linalg.norm(Kri - Kd))}


def run_one_electron(Z, xyz, steps, cpu=True):
    """Overlap, kinetic energy and nuclear attraction of the (H2O)_32 cc-pVDZ workload in one pass
    (lible_gpu_one_electron, host outputs), beside the reference's own overlap / kineticEnergy /
    nuclearAttraction on every host core (oracle/_ref), with the largest element difference."""
    from lible_b200 import ints as L

    s = L.Structure("cc-pvdz", Z, xyz, units="bohr")
    S, T, V = L.one_electron(s)
    ts = []
    for _ in range(max(1, steps)):
        t = time.perf_counter()
        S, T, V = L.one_electron(s)
        ts.append(time.perf_counter() - t)
    out = {"workload": "overlap + kinetic + nuclear attraction, (H2O)_32 cc-pVDZ, FP64", "nao": s.nao,
           "gpu_s": float(np.mean(ts))}
    from oracle import ref as R
    if cpu and R.available():
        R.set_threads(os.cpu_count() or 1)
        r = R.RefStructure("cc-pvdz", Z, xyz)
        t = time.perf_counter()
        ref = [r.one_electron(k) for k in range(3)]
        out["reference_cpu_s"] = time.perf_counter() - t
        out["reference_cores"] = os.cpu_count() or 1
        out["max_abs_diff"] = float(max(np.abs(a - b).max() for a, b in zip((S, T, V), ref)))
    return out


def run_gradient(steps, seed=2024, cpu=True):
    """J/K energy gradient of (H2O)_8 cc-pVTZ (464 AOs, occupation 40): wall time of the backward
    pass (derivative integrals contracted with the two-particle density on the device) and its
    agreement with central finite differences (step 1e-4 bohr) of the forward energy on two
    coordinates."""
    from lible_b200 import ints as L
    from lible_b200.workloads import random_density, water_cluster

    Z, xyz, rng = water_cluster(8, seed)
    s = L.Structure("cc-pvtz", Z, xyz, units="bohr")
    D = random_density(s.nao, 40, rng)
    g = L.jk_energy_backward(s, D, SCHWARZ)
    ts = []
    for _ in range(max(1, steps)):
        t = time.perf_counter()
        g = L.jk_energy_backward(s, D, SCHWARZ)
        ts.append(time.perf_counter() - t)
    L.jk_energy_forward(s, D, SCHWARZ)  # builds the forward plan
    t = time.perf_counter()
    L.jk_energy_forward(s, D, SCHWARZ)
    t_fwd = time.perf_counter() - t
    h, worst = 1e-4, 0.0
    for atom, x in [(0, 0), (13, 2)]:
        e = []
        for sgn in (1, -1):
            c = xyz.copy()
            c[atom, x] += sgn * h
            e.append(L.jk_energy_forward(L.Structure("cc-pvtz", Z, c, units="bohr"), D, SCHWARZ))
        worst = max(worst, abs((e[0] - e[1]) / (2 * h) - g[atom, x]))
    out = {"workload": "J/K energy gradient, (H2O)_8 cc-pVTZ, occupation 40, FP64", "nao": s.nao,
           "backward_s": float(np.mean(ts)), "forward_energy_s": t_fwd,
           "max_abs_fd_minus_analytic_Eh_per_bohr": worst, "fd_step_bohr": h}
    from oracle import ref as R
    if cpu and R.available():
        # the reference's ERI4D1Kernel batches contracted with the same two-particle density on every
        # host core, over the same Schwarz-surviving quartets of every stride-th bra pair (~10 s)
        cores = os.cpu_count() or 1
        R.set_threads(cores)
        r = R.RefStructure("cc-pvtz", Z, xyz)
        _, nq, sec = r.jk_grad_sample(D, SCHWARZ, 512)
        stride = max(1, int(math.ceil(512 * sec / 10.0)))
        _, nq, sec = r.jk_grad_sample(D, SCHWARZ, stride)
        n_full = L.jk_plan(s, SCHWARZ, "fp64")["n_quartets"]
        est = sec * n_full / max(nq, 1)
        out["reference_cpu"] = {"cores": cores, "cpu_model": cpu_model(), "quartets": nq, "seconds": sec,
                                "quartets_per_s": nq / sec, "estimated_full_s": est,
                                "gpu_speedup_estimate": est / out["backward_s"],
                                "sample": f"every {stride}-th bra shell pair, Schwarz 1e-12 ({nq} of {n_full} quartets)"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-molecule batched measurement")
    ap.add_argument("--no-autotune", action="store_true", help="skip the one-time launch-shape autotuning")
    ap.add_argument("--no-extras", action="store_true", help="skip the RI-J, RI-JK, one-electron and gradient measurements")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    from lible_b200 import ints as L
    from lible_b200.workloads import random_density, water_cluster

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    Z, xyz, rng = water_cluster(N_WATERS, SEED)
    t0 = time.perf_counter()
    s = L.Structure("cc-pvdz", Z, xyz, units="bohr", device=local)
    D = random_density(s.nao, OCC, rng)
    dev = torch.device("cuda", local)
    Dd = torch.tensor(D, device=dev)
    J = torch.empty_like(Dd)
    K = torch.empty_like(Dd)
    plan64 = L.jk_plan(s, SCHWARZ, "fp64")
    planmx = L.jk_plan(s, SCHWARZ, "mixed", FP32_THR)
    plan_s = time.perf_counter() - t0
    # one-time launch-shape autotuning of both plans on this workload (part of the set-up, as a
    # user would do once per structure or load from a tune cache)
    if not args.no_autotune:
        L.jk_autotune(s, Dd, SCHWARZ, "fp64", J=J, K=K)
        L.jk_autotune(s, Dd, SCHWARZ, "mixed", FP32_THR, J=J, K=K)
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(L.stream_handle(s), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    dfma, dmma = L.fp64_peak(s)

    def timed(precision, steps, warmup):
        for _ in range(warmup):
            L.jk(s, Dd, SCHWARZ, precision, FP32_THR, J=J, K=K)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            L.jk(s, Dd, SCHWARZ, precision, FP32_THR, J=J, K=K)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return ms

    # accuracy of the mixed path against FP64 (same run)
    L.jk(s, Dd, SCHWARZ, "fp64", J=J, K=K)
    J64, K64 = J.double().cpu().numpy(), K.double().cpu().numpy()
    L.jk(s, Dd, SCHWARZ, "mixed", FP32_THR, J=J, K=K)
    Jmx, Kmx = J.double().cpu().numpy(), K.double().cpu().numpy()
    E64 = float(np.sum(D * (0.5 * J64 - 0.25 * K64)))
    Emx = float(np.sum(D * (0.5 * Jmx - 0.25 * Kmx)))
    dE = abs(Emx - E64)
    mixed_ok = dE <= 1e-8

    clk = clocks_start(local)
    ms64 = timed("fp64", args.steps, args.warmup)
    msmx = timed("mixed", args.steps, args.warmup)
    clocks = clocks_stop(clk)

    def agg(ms):
        return max_over_ranks(float(np.mean(ms)), dist, dev)

    t64, tmx = agg(ms64), agg(msmx)
    head = "mixed" if mixed_ok else "fp64"
    th = tmx if mixed_ok else t64
    plan = planmx if mixed_ok else plan64
    value = world * plan["n_quartets"] / (th * 1e-3)

    # end to end through the public API with host (pinned) buffers: H2D of D, D2H of J and K per step
    Dh = torch.tensor(D).pin_memory()
    Jh = torch.empty_like(Dh).pin_memory()
    Kh = torch.empty_like(Dh).pin_memory()
    for _ in range(max(1, args.warmup)):
        L.jk(s, Dh, SCHWARZ, head, FP32_THR, J=Jh, K=Kh)
    e2e_s = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a = time.perf_counter()
        L.jk(s, Dh, SCHWARZ, head, FP32_THR, J=Jh, K=Kh)
        e2e_s.append(time.perf_counter() - a)
    e2e_t = max_over_ranks(float(np.mean(e2e_s)), dist, dev)

    # the batch is seconds per build: two timed steps after one warm-up keep the run short
    batch = None if args.no_batch else run_batch(min(args.steps, 2), 1, dev)
    rij = rijk = one_el = gradient = None
    if not args.no_extras and rank == 0:
        rij = run_rij(Z, xyz, D, J64, min(args.steps, 2))
        rijk = run_rijk(Z, xyz, D, J64, K64, OCC, min(args.steps, 2))
        one_el = run_one_electron(Z, xyz, min(args.steps, 2), cpu=not args.no_cpu_baseline)
        gradient = run_gradient(min(args.steps, 2), cpu=not args.no_cpu_baseline)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    # CPU leg (rank 0, one GPU): the reference's ERI4Kernel batches digested into J/K on every host
    # core, unsampled -- the CPU baseline of the whole workload and the oracle of both GPU builds
    cpu = oracle = None
    if world == 1 and not args.no_cpu_baseline:
        from oracle import ref as R
        if R.available():
            Jr, Kr, nq_ref, sec_ref, cores = oracle_jk_full(Z, xyz, D)
            Er = float(np.sum(D * (0.5 * Jr - 0.25 * Kr)))
            cpu = {"value": nq_ref / sec_ref, "unit": "quartets/s", "cores": cores, "kind": "reference",
                   "cpu_model": cpu_model(),
                   "sample": f"whole workload, unsampled: reference ERI4Kernel batches + J/K digestion (OpenMP), "
                             f"{nq_ref} quartets in {sec_ref:.2f} s"}
            oracle = {"n_quartets_match": int(nq_ref) == int(plan64["n_quartets"]),
                      "fp64_max_abs_dJ": float(np.abs(J64 - Jr).max()), "fp64_max_abs_dK": float(np.abs(K64 - Kr).max()),
                      "fp64_abs_dE_Eh": abs(E64 - Er),
                      "mixed_max_abs_dJ": float(np.abs(Jmx - Jr).max()), "mixed_max_abs_dK": float(np.abs(Kmx - Kr).max()),
                      "mixed_abs_dE_Eh": abs(Emx - Er),
                      "mixed_dJ_fro": float(np.linalg.norm(Jmx - Jr)), "mixed_dK_fro": float(np.linalg.norm(Kmx - Kr))}

    flops64 = plan64["flops_fp64"]
    achieved64 = flops64 / (t64 * 1e-3) / 1e12
    ffma, ffma2 = L.fp32_peak(s)
    fp64_peak, fp32_peak = max(dfma, dmma), max(ffma, ffma2)

    # every class launch timed by CUDA events (launches serialised on the structure's stream), mean
    # of three profiled builds after the timed region; the dominant launch of a build is its roofline
    def dominant(precision):
        prof = {}
        for _ in range(3):
            for r in L.jk_profile(s, Dd, SCHWARZ, precision, FP32_THR, J=J, K=K):
                key = (r["classes"], r["fp32"])
                e = prof.setdefault(key, {"ms": [], "flops": r["flops"], "tasks": r["tasks"], "shape": r["shape"]})
                e["ms"].append(r["ms"])
        key, d = max(prof.items(), key=lambda kv: np.mean(kv[1]["ms"]))
        ms = float(np.mean(d["ms"]))
        tf = d["flops"] / (ms * 1e-3) / 1e12
        fp32 = bool(key[1])
        peak = fp32_peak if fp32 else fp64_peak
        occ = d["shape"] == 0 and (tuple(key[0]), fp32) in OCC_KERNELS
        name = "%s<%d,%d,%d,%d,%s,%d>" % (("eriKernelOcc" if occ else "eriKernel",) + tuple(key[0]) +
                                          ("float" if fp32 else "double", d["shape"]))
        return {"bound": "fp32" if fp32 else "fp64", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                "frac": tf / peak if peak else None, "traffic": DOMINANT_TRAFFIC.get((tuple(key[0]), fp32)),
                "kernel": name, "kernel_ms": ms, "kernel_quartets": d["tasks"],
                "scope": f"dominant class kernel of the {precision} build: algorithmic FLOPs per launch / CUDA-event "
                         "launch time (serialised profile builds after the timed region); the limiter ncu shows is "
                         "issue / L1 latency, not the HBM (the working set stays in L2)",
                "peak_source": ("FP32 peak measured in this run (lible_gpu_fp32_peak: scalar FFMA and packed "
                                "fma.rn.f32x2 loops, the larger)" if fp32 else
                                "FP64 peak measured in this run (lible_gpu_fp64_peak: DFMA and DMMA m8n8k4 loops, the "
                                "larger)") + "; the measured-peaks file has no FP64 or FP32 entry"}

    roof_head = dominant(head)
    roof64 = roof_head if head == "fp64" else dominant("fp64")
    roof64 = dict(roof64, build_fp64_tflops=achieved64, dfma_peak=dfma, dmma_peak=dmma)
    roof_head = dict(roof_head, ffma_peak=ffma, ffma2_peak=ffma2) if head == "mixed" else roof64

    # J/K digestion: algorithmic bytes of one build over the build time, against the measured HBM copy
    # bandwidth (the accumulators stay in L2, so this is an L2-side rate)
    hbm, hbm_src = 6650.0, "fallback"
    try:
        hbm, hbm_src = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        pass
    dig_b = digestion_bytes(L.jk_plan_classes(s, SCHWARZ, "fp64", FP32_THR))
    digestion = {"bytes_per_build": dig_b, "fp64_gbs": dig_b / (t64 * 1e-3) / 1e9,
                 "mixed_gbs": dig_b / (tmx * 1e-3) / 1e9, "hbm_gbs": hbm, "hbm_source": hbm_src,
                 "fp64_frac_of_hbm": dig_b / (t64 * 1e-3) / 1e9 / hbm,
                 "l2_atomic_bytes_fp64_dominant_launch": L2_ATOMIC_BYTES.get(roof64["kernel"]),
                 "l2_atomic_bytes_headline_dominant_launch": L2_ATOMIC_BYTES.get(roof_head["kernel"]),
                 "l2_atomic_source": "ncu lts__t_sectors_op_red.sum x 32 B, one launch "
                                     "(profiles/jk_digestion_atomics_h2o32_dz.md)",
                 "definition": "per unique quartet 8 B per D-block element read + 16 B per J/K-block element updated, "
                               "blocks ab, cd, ac, ad, bc, bd"}
    out = {
        "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": th, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32 (mixed)" if mixed_ok else "f64", "data": "synthetic",
        "config": WORKLOAD,
        "batch": batch,
        "rij": rij,
        "rijk": rijk,
        "one_electron": one_el,
        "gradient": gradient,
        "setup_s": setup_s, "plan_setup_s": plan_s, "autotuned": not args.no_autotune,
        "parallelism": f"replicas x{world}",
        "roofline_fp64": roof64,
        "cpu_baseline": cpu,
        "e2e": {"value": world * plan["n_quartets"] / e2e_t, "unit": "quartets/s",
                "h2d_bytes_per_step": int(D.nbytes), "d2h_bytes_per_step": int(2 * D.nbytes),
                "path": "lible_b200.jk -> lible_gpu_jk with pinned host D/J/K"},
        "clocks": clocks,
        "gpu_launches": int(plan["n_launches"]) * args.steps,
        "roofline": roof_head,
        "digestion": digestion,
        "oracle_check": oracle,
        "fp64": {"jk_build_s": t64 * 1e-3, "quartets_per_s": world * plan64["n_quartets"] / (t64 * 1e-3),
                 "n_quartets": plan64["n_quartets"], "n_prim_quartets": plan64["n_prim_quartets"]},
        "mixed": {"jk_build_s": tmx * 1e-3, "quartets_per_s": world * planmx["n_quartets"] / (tmx * 1e-3),
                  "n_fp32_quartets": planmx["n_fp32"], "abs_dE_Eh_vs_fp64": dE,
                  "dJ_fro": float(np.linalg.norm(Jmx - J64)), "dK_fro": float(np.linalg.norm(Kmx - K64)),
                  "meets_1e-8": mixed_ok, "speedup_vs_fp64": t64 / tmx},
        "path": head,
        "jk_build_s": th * 1e-3,
    }
    emit(out)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

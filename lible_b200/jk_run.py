"""Runs direct J/K builds of a seeded water cluster and prints the screening plan and timings.

    python -m lible_b200.jk_run --waters 8 --basis cc-pvdz --precision fp64 --repeat 2
    python -m lible_b200.jk_run --waters 2 --basis cc-pvtz --gradient --repeat 2
    python -m lible_b200.jk_run --waters 8 --rik def2-universal-jkfit --occ 40 --repeat 2
    python -m lible_b200.jk_run --waters 8 --basis cc-pvtz --autotune --repeat 2

The cluster and density follow lible_b200.workloads (5.7 bohr lattice, random rotations, +-0.6 bohr
jitter, D = C C^T with occupation 5 per water unless --occ is given).  Every build is a separate
lible_gpu_jk call on the structure's stream; the first one also builds the Schwarz factors and the
screening plan.  --gradient runs the J/K energy gradient (lible_gpu_jk_energy_backward) instead;
--rik AUX runs RI-K with that auxiliary basis from an orthonormal occupied factor C (the first call
builds and keeps the fitted three-centre tensor); --autotune runs the launch autotuner once on the
J/K plan before the timed builds (the choices apply to this structure's plan).
Small cases of this command are what kernel profiles are taken on.
"""
import argparse
import json
import sys
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--waters", type=int, default=8)
    ap.add_argument("--basis", default="cc-pvdz")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--schwarz", type=float, default=1e-12)
    ap.add_argument("--fp32-threshold", type=float, default=1e-4)
    ap.add_argument("--occ", type=int, default=None)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--gradient", action="store_true")
    ap.add_argument("--rik", default=None, metavar="AUX")
    ap.add_argument("--autotune", action="store_true")
    args = ap.parse_args(argv)

    import torch

    from . import ints as L
    from .workloads import random_density, water_cluster

    Z, xyz, rng = water_cluster(args.waters, args.seed)
    if args.rik:
        import numpy as np

        s = L.Structure(args.basis, Z, xyz, args.rik, units="bohr")
        C = np.linalg.qr(rng.standard_normal((s.nao, args.occ or 5 * args.waters)))[0]
        times, info = [], None
        for _ in range(args.repeat):
            t = time.perf_counter()
            _, info = L.rik(s, C=C, schwarz=args.schwarz, info=True)
            times.append(time.perf_counter() - t)
        print(json.dumps({"waters": args.waters, "basis": args.basis, "aux": args.rik, "nao": s.nao,
                          "naux": s.naux, "rik": info, "wall_s": times}))
        return 0
    s = L.Structure(args.basis, Z, xyz, units="bohr")
    D = random_density(s.nao, args.occ or 5 * args.waters, rng)
    Dd = torch.tensor(D, device="cuda")
    J, K = torch.empty_like(Dd), torch.empty_like(Dd)
    if args.autotune and not args.gradient:
        L.jk_autotune(s, D, args.schwarz, args.precision, args.fp32_threshold)
    times = []
    for _ in range(args.repeat):
        torch.cuda.synchronize()
        t = time.perf_counter()
        if args.gradient:
            L.jk_energy_backward(s, D, args.schwarz)
        else:
            L.jk(s, Dd, args.schwarz, args.precision, args.fp32_threshold, J=J, K=K)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
    plan = L.jk_plan(s, args.schwarz, args.precision, args.fp32_threshold)
    print(json.dumps({"waters": args.waters, "basis": args.basis, "nao": s.nao, "precision": args.precision,
                      "gradient": args.gradient, "plan": plan, "wall_s": times}))
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Python mirror of the `lible::ints` calls this engine replaces (src/lible/ints/ints.hpp of the
reference), running on the B200 through the C ABI of include/lible_b200.h.

    s = Structure("cc-pvdz", [8, 1, 1], coords_angstrom)
    V = eri4(s)                       # lible::ints::eri4          -> (N, N, N, N)
    d = eri4Diagonal(s)               # lible::ints::eri4Diagonal  -> (N, N)
    sp = shellPairData(True, s)       # lible::ints::shellPairData
    k = ERI4Kernel(sp[1], sp[0]); b = k(0, 0, sp[1], sp[0])
    J, K, st = jk(s, D)               # direct Coulomb / exchange (new)

Array arguments may be numpy arrays (host) or CUDA torch tensors (device); outputs are numpy
unless `out=` device tensors are given.  Errors raise LibleGpuError with the library's message.
"""
import ctypes
import os

import numpy as np

from ._lib import JKOpts, JKPlanInfo, JKStats, LibleGpuError, RIKInfo, check, load

BASIS_ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis", "main")
AUX_BASIS_ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis", "aux")
ANG_TO_BOHR = 1.0 / 0.5291772083


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)


def _i32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


def _f64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def basis_atoms(name, atomic_nrs, root=None):
    """Per-atom shells [(l, exps, coeffs), ...] of a named basis, read from <root>/<family>/<name>.txt
    in the reference's text format (element=Z, blocks "l=L n=K" of K exponent/coefficient lines,
    end=Z; src/lible/ints/basis_sets.cpp:214-277)."""
    root = root or BASIS_ROOT
    path = None
    for fam in sorted(os.listdir(root)):
        cand = os.path.join(root, fam, name.lower() + ".txt")
        if os.path.exists(cand):
            path = cand
    if path is None:
        raise LibleGpuError(1, f"basis set {name} not found under {root}")
    elements, cur, z = {}, None, None
    lines = iter(open(path).read().split("\n"))
    for line in lines:
        line = line.strip()
        if line.startswith("element="):
            z, cur = int(line.split("=")[1]), []
        elif line.startswith("end="):
            elements[z] = cur
        elif line.startswith("l="):
            parts = dict(p.split("=") for p in line.split())
            l, n = int(parts["l"]), int(parts["n"])
            rows = [next(lines).split() for _ in range(n)]
            cur.append((l, [float(r[0]) for r in rows], [float(r[1]) for r in rows]))
    try:
        return [list(elements[int(zz)]) for zz in atomic_nrs]
    except KeyError as e:
        raise LibleGpuError(1, f"element {e.args[0]} missing from basis set {name}") from None


class Structure:
    """lible::ints::Structure (src/lible/ints/structure.hpp:18-62).

    `basis_set` is a basis name (read from `basis_root`, default the shipped subset) or a
    basis_atoms list: one list per atom of (l, exps, coeffs) shells.  Coordinates are Angstrom
    unless units="bohr"."""

    def __init__(self, basis_set, atomic_nrs, coords, basis_set_aux=None, *, units="angstrom",
                 basis_root=None, aux_root=None, device=0):
        self._lib = load()
        ctx = ctypes.c_void_p()
        check(None, self._lib.lible_gpu_create(device, ctypes.byref(ctx)))
        self._ctx = ctx
        Z = _i32(atomic_nrs)
        xyz = _f64(coords).reshape(-1, 3)
        if len(Z) != len(xyz):
            raise ValueError("number of atomic numbers does not match the number of coordinates")
        u = 0 if units == "angstrom" else 1
        if isinstance(basis_set, str) and basis_set_aux is not None and not isinstance(basis_set_aux, str):
            basis_set = basis_atoms(basis_set, Z, basis_root)
        if isinstance(basis_set, str):
            rc = self._lib.lible_gpu_set_structure_named(
                ctx, (basis_root or BASIS_ROOT).encode(), basis_set.encode(),
                (aux_root or AUX_BASIS_ROOT).encode(), basis_set_aux.encode() if basis_set_aux else None,
                len(Z), _ptr(Z), _ptr(xyz), u)
        else:
            main = self._flatten(basis_set)
            aux = self._flatten(basis_set_aux) if basis_set_aux is not None else (None,) * 5
            self._keep = (main, aux)
            rc = self._lib.lible_gpu_set_structure(ctx, len(Z), _ptr(Z), _ptr(xyz), u, *[_ptr(x) for x in main],
                                                   *[_ptr(x) for x in aux])
        check(ctx, rc)
        nao, naux, nat, maxl = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        check(ctx, self._lib.lible_gpu_dims(ctx, ctypes.byref(nao), ctypes.byref(naux), ctypes.byref(nat),
                                            ctypes.byref(maxl)))
        self.nao, self.naux, self.n_atoms, self.max_l = nao.value, naux.value, nat.value, maxl.value
        self.use_ri = basis_set_aux is not None

    @staticmethod
    def _flatten(basis_atoms):
        nsh, ls, nps, ex, co = [], [], [], [], []
        for atom in basis_atoms:
            nsh.append(len(atom))
            for (l, exps, coeffs) in atom:
                ls.append(l)
                nps.append(len(exps))
                ex.extend(exps)
                co.extend(coeffs)
        return _i32(nsh), _i32(ls), _i32(nps), _f64(ex), _f64(co)

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            self._lib.lible_gpu_destroy(ctx)
            self._ctx = None

    @property
    def ctx(self):
        return self._ctx

    def getDimAO(self):
        return self.nao

    def getDimAOAux(self):
        return self.naux

    def getNAtoms(self):
        return self.n_atoms

    def getMaxL(self):
        return self.max_l

    def getUseRI(self):
        return self.use_ri


def _call(s, name, *args):
    check(s.ctx, getattr(load(), name)(s.ctx, *args))


def eri4(structure, out=None):
    n = structure.nao
    out = np.empty((n, n, n, n)) if out is None else out
    _call(structure, "lible_gpu_eri4", _ptr(out))
    return out


def eri4Diagonal(structure):
    n = structure.nao
    out = np.empty((n, n))
    _call(structure, "lible_gpu_eri4_diagonal", _ptr(out))
    return out


def eri3(structure, out=None):
    out = np.empty((structure.nao, structure.nao, structure.naux)) if out is None else out
    _call(structure, "lible_gpu_eri3", _ptr(out))
    return out


def eri2(structure, out=None):
    out = np.empty((structure.naux, structure.naux)) if out is None else out
    _call(structure, "lible_gpu_eri2", _ptr(out))
    return out


def eri2Diagonal(structure):
    out = np.empty(structure.naux)
    _call(structure, "lible_gpu_eri2_diagonal", _ptr(out))
    return out


class ShellPairData:
    """Handle of one shell-pair class of shellPairData(use_symm, structure): (la, lb), number of
    pairs and primitive pairs (src/lible/ints/shell_pair_data.hpp:50-120)."""

    def __init__(self, structure, use_symm, index, la, lb, n_pairs, n_ppairs):
        self.structure, self.uses_symm, self.index = structure, use_symm, index
        self.la_, self.lb_, self.n_pairs_, self.n_ppairs_ = la, lb, n_pairs, n_ppairs

    def getLPair(self):
        return self.la_, self.lb_


class ShellData:
    """Handle of one auxiliary shell class of shellDataAux(structure) (shell_pair_data.hpp:8-45)."""

    def __init__(self, structure, index, l, n_shells):
        self.structure, self.index, self.l_, self.n_shells_ = structure, index, l, n_shells


def shellPairData(use_symm, structure):
    n = ctypes.c_int()
    _call(structure, "lible_gpu_pair_classes", int(bool(use_symm)), ctypes.byref(n), None, None, None)
    ls = np.zeros(2 * n.value, np.int32)
    npairs = np.zeros(n.value, np.int64)
    nppairs = np.zeros(n.value, np.int64)
    _call(structure, "lible_gpu_pair_classes", int(bool(use_symm)), ctypes.byref(n), _ptr(ls), _ptr(npairs),
          _ptr(nppairs))
    return [ShellPairData(structure, bool(use_symm), i, int(ls[2 * i]), int(ls[2 * i + 1]), int(npairs[i]),
                          int(nppairs[i])) for i in range(n.value)]


def shellDataAux(structure):
    if not structure.use_ri:
        raise LibleGpuError(4, "shellDataAux(): RI approximation is not enabled!")
    n = ctypes.c_int()
    _call(structure, "lible_gpu_aux_classes", ctypes.byref(n), None, None)
    ls = np.zeros(n.value, np.int32)
    nsh = np.zeros(n.value, np.int64)
    _call(structure, "lible_gpu_aux_classes", ctypes.byref(n), _ptr(ls), _ptr(nsh))
    return [ShellData(structure, i, int(ls[i]), int(nsh[i])) for i in range(n.value)]


def _nsph(l):
    return 2 * l + 1


class _Kernel:
    _fn = None
    _nblk = 1

    def _dims(self):
        raise NotImplementedError

    def batch(self, idx):
        """Evaluates many (i, j) index pairs at once: idx is (n, 2); returns (n, *block_shape)."""
        idx = np.ascontiguousarray(np.asarray(idx, dtype=np.uint32).reshape(-1, 2))
        shape = self._dims()
        out = np.empty((len(idx), self._nblk) + shape) if self._nblk > 1 else np.empty((len(idx),) + shape)
        self._run(len(idx), idx, out)
        return out

    def __call__(self, i, j, *_):
        r = self.batch([[i, j]])[0]
        return list(r) if self._nblk > 1 else r


class ERI4Kernel(_Kernel):
    """lible::ints::ERI4Kernel (src/lible/ints/twoel/eri_kernels.hpp:60-76)."""
    _fn, _nblk = "lible_gpu_eri4_batch", 1

    def __init__(self, sp_ab, sp_cd):
        self.ab, self.cd, self.s = sp_ab, sp_cd, sp_ab.structure

    def _dims(self):
        return (_nsph(self.ab.la_), _nsph(self.ab.lb_), _nsph(self.cd.la_), _nsph(self.cd.lb_))

    def _run(self, n, idx, out):
        _call(self.s, self._fn, int(self.ab.uses_symm), self.ab.index, self.cd.index, n, _ptr(idx), _ptr(out))


class ERI4D1Kernel(ERI4Kernel):
    """lible::ints::ERI4D1Kernel (eri_kernels.hpp:114-132): 12 blocks [A, B, C, D] x [x, y, z]."""
    _fn, _nblk = "lible_gpu_eri4d1_batch", 12


class ERI3Kernel(_Kernel):
    """lible::ints::ERI3Kernel (eri_kernels.hpp:78-94)."""
    _fn, _nblk = "lible_gpu_eri3_batch", 1

    def __init__(self, sp_ab, sh_c):
        self.ab, self.c, self.s = sp_ab, sh_c, sp_ab.structure

    def _dims(self):
        return (_nsph(self.ab.la_), _nsph(self.ab.lb_), _nsph(self.c.l_))

    def _run(self, n, idx, out):
        _call(self.s, self._fn, int(self.ab.uses_symm), self.ab.index, self.c.index, n, _ptr(idx), _ptr(out))


class ERI3D1Kernel(ERI3Kernel):
    """lible::ints::ERI3D1Kernel (eri_kernels.hpp:134-151): 9 blocks [A, B, C] x [x, y, z]."""
    _fn, _nblk = "lible_gpu_eri3d1_batch", 9


class ERI2Kernel(_Kernel):
    """lible::ints::ERI2Kernel (eri_kernels.hpp:96-112)."""
    _fn, _nblk = "lible_gpu_eri2_batch", 1

    def __init__(self, sh_a, sh_b):
        self.a, self.b, self.s = sh_a, sh_b, sh_a.structure

    def _dims(self):
        return (_nsph(self.a.l_), _nsph(self.b.l_))

    def _run(self, n, idx, out):
        _call(self.s, self._fn, self.a.index, self.b.index, n, _ptr(idx), _ptr(out))


class ERI2D1Kernel(ERI2Kernel):
    """lible::ints::ERI2D1Kernel (eri_kernels.hpp:153-169): 6 blocks [A, B] x [x, y, z]."""
    _fn, _nblk = "lible_gpu_eri2d1_batch", 6


class ERI2D2Kernel(ERI2Kernel):
    """lible::ints::ERI2D2Kernel (eri_kernels.hpp:171-185): 6 x 6 blocks [A, B] x [x, y, z]."""
    _fn, _nblk = "lible_gpu_eri2d2_batch", 36

    def batch(self, idx):
        return super().batch(idx).reshape(-1, 6, 6, *self._dims())

    def __call__(self, i, j, *_):
        return self.batch([[i, j]])[0]


class ERI4SOCKernel(ERI4Kernel):
    """lible::ints::ERI4SOCKernel (eri_kernels.hpp:187-203): the three spin-orbit components."""
    _fn, _nblk = "lible_gpu_eri4soc_batch", 3


class ERI3SOCKernel(ERI3Kernel):
    """lible::ints::ERI3SOCKernel (eri_kernels.hpp:205-221)."""
    _fn, _nblk = "lible_gpu_eri3soc_batch", 3


class Batch:
    """A batch of molecules whose J/K are built together (no reference counterpart).

    `molecules` is a list of (basis name, atomic numbers, coordinates).  D, J and K are packed 1-D
    arrays of `packed` elements: molecule m's N_m x N_m matrix starts at `base[m]` (see pack() and
    unpack()).  Every quartet class of every molecule goes through one work-queue launch per class;
    jk(batch, D, use_graph=True) replays the whole build as one CUDA graph."""

    def __init__(self, molecules, *, units="bohr", basis_root=None, device=0):
        self._lib = load()
        ctx = ctypes.c_void_p()
        check(None, self._lib.lible_gpu_create(device, ctypes.byref(ctx)))
        self._ctx = ctx
        names = [m[0].encode() for m in molecules]
        arr = (ctypes.c_char_p * len(names))(*names)
        n_atoms = _i32([len(m[1]) for m in molecules])
        Z = _i32(np.concatenate([np.asarray(m[1], dtype=np.int32) for m in molecules]))
        xyz = _f64(np.vstack([np.asarray(m[2], dtype=float).reshape(-1, 3) for m in molecules]))
        u = 0 if units == "angstrom" else 1
        check(ctx, self._lib.lible_gpu_set_batch(ctx, len(molecules), (basis_root or BASIS_ROOT).encode(),
                                                 ctypes.cast(arr, ctypes.c_void_p), _ptr(n_atoms), _ptr(Z),
                                                 _ptr(xyz), u))
        nm = ctypes.c_int()
        nao = np.zeros(len(molecules), np.int64)
        base = np.zeros(len(molecules), np.int64)
        packed = ctypes.c_longlong()
        check(ctx, self._lib.lible_gpu_batch_layout(ctx, ctypes.byref(nm), _ptr(nao), _ptr(base), ctypes.byref(packed)))
        self.nao, self.base, self.packed = nao, base, packed.value
        self.n_molecules = nm.value

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            self._lib.lible_gpu_destroy(ctx)
            self._ctx = None

    @property
    def ctx(self):
        return self._ctx

    def pack(self, mats):
        """Packs per-molecule N_m x N_m matrices into one array."""
        out = np.empty(self.packed)
        for m, M in enumerate(mats):
            n = self.nao[m]
            out[self.base[m]:self.base[m] + n * n] = np.asarray(M, dtype=float).reshape(-1)
        return out

    def unpack(self, arr):
        """Splits a packed array (numpy or torch) into per-molecule N_m x N_m views."""
        return [arr[self.base[m]:self.base[m] + self.nao[m] ** 2].reshape(int(self.nao[m]), int(self.nao[m]))
                for m in range(self.n_molecules)]


def _opts(schwarz, precision, fp32_threshold, use_graph=False):
    return JKOpts(float(schwarz), float(fp32_threshold), 1 if precision in (1, "mixed") else 0, 1 if use_graph else 0)


def _jk_shape(structure):
    return (structure.packed,) if isinstance(structure, Batch) else (structure.nao, structure.nao)


def jk(structure, D, schwarz=1e-12, precision="fp64", fp32_threshold=1e-4, J=None, K=None, use_graph=False):
    """Direct Coulomb and exchange matrices for a symmetric density D (N x N, or packed for a Batch).
    With use_graph the launch sequence is captured once per (plan, D, J, K) and replayed."""
    Dh = D if hasattr(D, "data_ptr") else _f64(D)
    J = np.empty(_jk_shape(structure)) if J is None else J
    K = np.empty(_jk_shape(structure)) if K is None else K
    st = JKStats()
    opts = _opts(schwarz, precision, fp32_threshold, use_graph)
    _call(structure, "lible_gpu_jk", _ptr(Dh), _ptr(J), _ptr(K), ctypes.byref(opts), ctypes.byref(st))
    return J, K, {"n_quartets": st.n_quartets, "n_fp32": st.n_fp32, "n_launches": st.n_launches}


def jk_autotune(structure, D, schwarz=1e-12, precision="fp64", fp32_threshold=1e-4, cache=None, J=None, K=None):
    """Autotunes the class launches of the J/K plan on D (J and K are overwritten); returns the
    per-class summary.  With `cache`, the choices are appended to that file."""
    Dh = D if hasattr(D, "data_ptr") else _f64(D)
    J = np.empty(_jk_shape(structure)) if J is None else J
    K = np.empty(_jk_shape(structure)) if K is None else K
    buf = ctypes.create_string_buffer(1 << 16)
    opts = _opts(schwarz, precision, fp32_threshold)
    _call(structure, "lible_gpu_jk_autotune", _ptr(Dh), _ptr(J), _ptr(K), ctypes.byref(opts),
          cache.encode() if cache else None, buf, len(buf))
    return buf.value.decode()


def jk_profile(structure, D, schwarz=1e-12, precision="fp64", fp32_threshold=1e-4, J=None, K=None):
    """One J/K build with every class launch serialised and timed by CUDA events.  Returns a list of
    dicts (classes, fp32, shape = the launch's shape: 0 default, 1 alternative tile shape, 2 the class
    in the other orientation; ms, flops, tasks) in launch order."""
    Dh = D if hasattr(D, "data_ptr") else _f64(D)
    J = np.empty(_jk_shape(structure)) if J is None else J
    K = np.empty(_jk_shape(structure)) if K is None else K
    cap = 4096
    n = ctypes.c_int(cap)
    ls, f32 = np.zeros(4 * cap, np.int32), np.zeros(cap, np.int32)
    ms, fl, tk = np.zeros(cap), np.zeros(cap), np.zeros(cap, np.int64)
    opts = _opts(schwarz, precision, fp32_threshold)
    _call(structure, "lible_gpu_jk_profile", _ptr(Dh), _ptr(J), _ptr(K), ctypes.byref(opts), ctypes.byref(n),
          _ptr(ls), _ptr(f32), _ptr(ms), _ptr(fl), _ptr(tk))
    return [{"classes": tuple(int(x) for x in ls[4 * i:4 * i + 4]), "fp32": bool(f32[i] & 1),
             "shape": int(f32[i] >> 1), "ms": float(ms[i]), "flops": float(fl[i]), "tasks": int(tk[i])}
            for i in range(min(n.value, cap))]


def set_tune_cache(structure, path):
    """Later J/K plans of this structure start from the autotune cache at `path`."""
    _call(structure, "lible_gpu_set_tune_cache", path.encode() if path else None)


def jk_energy_forward(structure, D, schwarz=1e-12, precision="fp64", fp32_threshold=1e-4):
    """E = 1/2 Tr(DJ) - 1/4 Tr(DK)."""
    e = ctypes.c_double()
    opts = _opts(schwarz, precision, fp32_threshold)
    Dh = D if hasattr(D, "data_ptr") else _f64(D)  # N x N, or packed for a Batch
    _call(structure, "lible_gpu_jk_energy_forward", _ptr(Dh), ctypes.byref(opts), ctypes.byref(e), None, None)
    return e.value


def jk_energy_backward(structure, D, schwarz=1e-12):
    """dE/dR of E = 1/2 Tr(DJ) - 1/4 Tr(DK), shape (n_atoms, 3), in Eh/bohr, over the quartets the
    FP64 forward pass keeps with the same Schwarz threshold."""
    g = np.empty((structure.n_atoms, 3))
    opts = _opts(schwarz, "fp64", 1e-4)
    _call(structure, "lible_gpu_jk_energy_backward", _ptr(_f64(D)), ctypes.byref(opts), _ptr(g))
    return g


def rij(structure, D, schwarz=1e-12):
    """RI-J: returns J, gamma, d with (P|Q) d = gamma."""
    n, na = structure.nao, structure.naux
    J, g, d = np.empty((n, n)), np.empty(na), np.empty(na)
    _call(structure, "lible_gpu_rij", _ptr(_f64(D)), float(schwarz), _ptr(J), _ptr(g), _ptr(d))
    return J, g, d


def rij_grad(structure, D, schwarz=1e-12):
    """Gradient [n_atoms][3] of the RI-J energy 1/2 gamma^T (P|Q)^-1 gamma, and that energy."""
    g = np.empty((structure.n_atoms, 3))
    e = ctypes.c_double()
    _call(structure, "lible_gpu_rij_grad", _ptr(_f64(D)), float(schwarz), _ptr(g), ctypes.byref(e))
    return g, e.value


def rij_last_solve(structure):
    """How the last rij() solved the metric equations:
    {'method': 'cholesky'|'cholesky+shift'|'eigen', 'lo', 'hi', 'dropped', 'shift'}."""
    m, lo, hi, dr, sh = ctypes.c_int(), ctypes.c_double(), ctypes.c_double(), ctypes.c_int(), ctypes.c_double()
    _call(structure, "lible_gpu_rij_last_solve", ctypes.byref(m), ctypes.byref(lo), ctypes.byref(hi), ctypes.byref(dr),
          ctypes.byref(sh))
    return {"method": {0: "cholesky", 1: "eigen", 2: "cholesky+shift"}.get(m.value, None), "lo": lo.value,
            "hi": hi.value, "dropped": dr.value, "shift": sh.value}


def _square(structure, fn, *args):
    n = structure.nao
    out = np.empty((n, n))
    _call(structure, fn, *args, _ptr(out))
    return out


def overlap(structure):
    """lible::ints::overlap (src/lible/ints/ints.hpp:30): the nao x nao overlap matrix."""
    return _square(structure, "lible_gpu_overlap")


def kineticEnergy(structure):
    """lible::ints::kineticEnergy (ints.hpp:39)."""
    return _square(structure, "lible_gpu_kinetic_energy")


def nuclearAttraction(structure):
    """lible::ints::nuclearAttraction (ints.hpp:48): the nuclei's attraction on an electron."""
    return _square(structure, "lible_gpu_nuclear_attraction")


def externalCharges(point_charges, structure):
    """lible::ints::externalCharges (ints.hpp:55): point charges [[x, y, z, q], ...] in bohr."""
    q = _f64(point_charges).reshape(-1, 4)
    return _square(structure, "lible_gpu_external_charges", _ptr(q), int(len(q)))


def one_electron(structure, point_charges=None):
    """(S, T, V) in one pass; V from the nuclei, or from `point_charges` ([n][4], bohr) if given."""
    n = structure.nao
    S, T, V = np.empty((n, n)), np.empty((n, n)), np.empty((n, n))
    if point_charges is None:
        _call(structure, "lible_gpu_one_electron", None, 0, _ptr(S), _ptr(T), _ptr(V))
    else:
        q = _f64(point_charges).reshape(-1, 4)
        _call(structure, "lible_gpu_one_electron", _ptr(q), int(len(q)), _ptr(S), _ptr(T), _ptr(V))
    return S, T, V


def _one_batch(op, ipair, sp, charges=None, omegas=None, origin=None):
    """Per-pair one-electron blocks through lible_gpu_one_electron_batch_ex; `ipair` an index (returns
    the block, or the list of 6 derivative / 3 Cartesian blocks) or a sequence of indices (returns an
    array)."""
    single = np.ndim(ipair) == 0
    idx = np.ascontiguousarray(np.atleast_1d(np.asarray(ipair, dtype=np.uint32)))
    nb = 9 if op == 14 else 6 if (3 <= op <= 5 or op == 10) else 3 if (6 <= op <= 8 or op >= 11) else 1
    out = np.empty((len(idx), nb, _nsph(sp.la_), _nsph(sp.lb_)))
    if charges is None:
        q, nq = None, 0
    else:
        q = _f64(charges).reshape(-1, 4)
        nq = len(q)
    w = None if omegas is None else _f64(omegas)
    o = None if origin is None else _f64(origin)
    _call(sp.structure, "lible_gpu_one_electron_batch_ex", int(sp.uses_symm), int(sp.index), int(op), int(len(idx)),
          _ptr(idx), _ptr(q), _ptr(w), nq, _ptr(o), _ptr(out))
    if nb == 1:
        out = out[:, 0]
    if single:
        return list(out[0]) if nb > 1 else out[0]
    return out


def overlapKernel(ipair, sp_data):
    """lible::ints::overlapKernel (ints.hpp:33)."""
    return _one_batch(0, ipair, sp_data)


def kineticEnergyKernel(ipair, sp_data):
    """lible::ints::kineticEnergyKernel (ints.hpp:42)."""
    return _one_batch(1, ipair, sp_data)


def externalChargesKernel(ipair, charges, sp_data):
    """lible::ints::externalChargesKernel (ints.hpp:66); the Boys grid argument is not needed."""
    return _one_batch(2, ipair, sp_data, charges)


def overlapD1Kernel(ipair, sp_data):
    """lible::ints::overlapD1Kernel (ints.hpp:36): [d/dA x, y, z, d/dB x, y, z]."""
    return _one_batch(3, ipair, sp_data)


def kineticEnergyD1Kernel(ipair, sp_data):
    """lible::ints::kineticEnergyD1Kernel (ints.hpp:45)."""
    return _one_batch(4, ipair, sp_data)


def externalChargesD1Kernel(ipair, charges, sp_data):
    """lible::ints::externalChargesD1Kernel (ints.hpp:79): the orbital part."""
    return _one_batch(5, ipair, sp_data, charges)


def dipoleMomentKernel(ipair, origin, sp_data):
    """lible::ints::dipoleMomentKernel (ints.hpp:127-129): [x, y, z] blocks of <a| r - origin |b>."""
    return _one_batch(6, ipair, sp_data, origin=origin)


def momentumKernel(ipair, sp_data):
    """lible::ints::momentumKernel (ints.hpp:141): [x, y, z] blocks of -<a| d/dr |b>."""
    return _one_batch(7, ipair, sp_data)


def angularMomentumKernel(ipair, origin, sp_data):
    """lible::ints::angularMomentumKernel (ints.hpp:149-151): [x, y, z] blocks of
    -<a| (r - origin) x d/dr |b>."""
    return _one_batch(8, ipair, sp_data, origin=origin)


def externalChargesErfKernel(ipair, charges, omegas, sp_data):
    """lible::ints::externalChargesErfKernel (ints.hpp:71-75): erf(w r)/r attraction of the charges
    [x, y, z, q], one omega per charge; the Boys grid argument is not needed."""
    return _one_batch(9, ipair, sp_data, charges, omegas=omegas)


def externalChargesErfD1Kernel(ipair, charges, omegas, sp_data):
    """lible::ints::externalChargesErfD1Kernel (ints.hpp:86-89): the orbital part, six blocks."""
    return _one_batch(10, ipair, sp_data, charges, omegas=omegas)


def _per_charge(op, ipair, charges, sp_data, omegas=None):
    q = _f64(charges).reshape(-1, 4)
    w = None if omegas is None else _f64(omegas).ravel()
    if w is not None and w.size != len(q):
        raise ValueError("one omega per charge")
    parts = [np.asarray(_one_batch(op, ipair, sp_data, q[c:c + 1], omegas=None if w is None else w[c:c + 1]))
             for c in range(len(q))]
    if np.ndim(ipair) == 0:
        return [list(p) if op >= 11 else p for p in parts]
    return np.stack(parts, axis=1)


def externalChargesOperatorD1Kernel(ipair, charges, sp_data):
    """lible::ints::externalChargesOperatorD1Kernel (ints.hpp:93-96): per charge, the derivatives
    with respect to its position [x, y, z]."""
    return _per_charge(11, ipair, charges, sp_data)


def externalChargesOperatorErfD1Kernel(ipair, charges, omegas, sp_data):
    """lible::ints::externalChargesOperatorErfD1Kernel (ints.hpp:101-105)."""
    return _per_charge(12, ipair, charges, sp_data, omegas)


def potentialAtExternalChargesKernel(ipair, charges, sp_data):
    """lible::ints::potentialAtExternalChargesKernel (ints.hpp:109-112): one block per charge."""
    return _per_charge(2, ipair, charges, sp_data)


def potentialAtExternalChargesErfKernel(ipair, charges, omegas, sp_data):
    """lible::ints::potentialAtExternalChargesErfKernel (ints.hpp:116-120)."""
    return _per_charge(9, ipair, charges, sp_data, omegas)


def spinOrbitCoupling1ElKernel(ipair, charges, sp_data):
    """lible::ints::spinOrbitCoupling1ElKernel (ints.hpp:135-137): [x, y, z] blocks for the point
    charges [x, y, z, q]; the Boys grid argument is not needed."""
    return _one_batch(13, ipair, sp_data, charges)


def _one_operator(structure, fn, nblk, *args):
    n = structure.nao
    out = np.empty((nblk, n, n) if nblk > 1 else (n, n))
    _call(structure, fn, *args, _ptr(out))
    return out


def dipoleMoment(origin, structure):
    """lible::ints::dipoleMoment (ints.hpp:123-125): [3][nao][nao], symmetric."""
    return _one_operator(structure, "lible_gpu_dipole_moment", 3, _ptr(_f64(origin)))


def momentum(structure):
    """lible::ints::momentum (ints.hpp:139): [3][nao][nao] of -<m| d/dr |n>, the full antisymmetric
    matrices (the reference's driver leaves the lower blocks of its unique pairs unwritten and negates
    the upper ones)."""
    return _one_operator(structure, "lible_gpu_momentum", 3)


def angularMomentum(origin, structure):
    """lible::ints::angularMomentum (ints.hpp:146-147): [3][nao][nao], antisymmetric."""
    return _one_operator(structure, "lible_gpu_angular_momentum", 3, _ptr(_f64(origin)))


def pVpKernel(ipair, charges, sp_data):
    """lible::ints::pVpKernel (ints.hpp:159-161): <d_i a| V |d_j b> for the point charges
    [x, y, z, q], as [3][3] blocks (an index) or an array [n][3][3][S_a][S_b] (a sequence).  The
    integrals themselves; the reference's kernel differs (include/lible_b200.h, pVpIntegrals)."""
    single = np.ndim(ipair) == 0
    out = np.asarray(_one_batch(14, np.atleast_1d(ipair), sp_data, charges))
    out = out.reshape(out.shape[0], 3, 3, out.shape[-2], out.shape[-1])
    if single:
        return [[out[0, i, j] for j in range(3)] for i in range(3)]
    return out


def pVpIntegrals(structure, point_charges=None):
    """lible::ints::pVpIntegrals (ints.hpp:154): [3][3][nao][nao] of <d_i m| V |d_j n> for the
    nuclei (or the given point charges [n][4], bohr), out[i][j] = out[j][i]^T."""
    n = structure.nao
    if point_charges is None:
        q, nq = None, 0
    else:
        q = _f64(point_charges).reshape(-1, 4)
        nq = len(q)
    return _one_operator(structure, "lible_gpu_pvp_integrals", 9, _ptr(q), nq).reshape(3, 3, n, n)


def spinOrbitCoupling1El(structure):
    """lible::ints::spinOrbitCoupling1El (ints.hpp:131): [3][nao][nao] for the nuclei, antisymmetric."""
    return _one_operator(structure, "lible_gpu_spin_orbit_coupling_1el", 3)


def nuclearAttractionErf(structure, omegas):
    """lible::ints::nuclearAttractionErf (ints.hpp:52): one omega per atom."""
    w = _f64(omegas)
    if w.size != structure.n_atoms:
        raise ValueError("one omega per atom")
    return _one_operator(structure, "lible_gpu_nuclear_attraction_erf", 1, _ptr(w))


def externalChargesErf(point_charges, omegas, structure):
    """lible::ints::externalChargesErf (ints.hpp:60-62): charges [n][4] (x, y, z bohr, q), one omega
    per charge."""
    q = _f64(point_charges).reshape(-1, 4)
    w = _f64(omegas)
    if w.size != len(q):
        raise ValueError("one omega per charge")
    return _one_operator(structure, "lible_gpu_external_charges_erf", 1, _ptr(q), _ptr(w), len(q))


def one_electron_grad(structure, D=None, W=None):
    """[n_atoms][3] gradient of sum D (T + V) - sum W S with respect to the nuclear coordinates."""
    g = np.empty((structure.n_atoms, 3))
    _call(structure, "lible_gpu_one_electron_grad", _ptr(_f64(D)) if D is not None else None,
          _ptr(_f64(W)) if W is not None else None, _ptr(g))
    return g


def rik(structure, D=None, C=None, schwarz=1e-12, info=False):
    """RI-K: K_mn = sum_PQ (ml|P) [(P|Q)^-1]_PQ (Q|ns) D_ls.  Give the density factor C ([nao][occ],
    D = C C^T) or the symmetric D itself (factorised on the device by its eigendecomposition).
    With info=True also returns the stage times / FLOPs of the build."""
    n = structure.nao
    if C is None and D is None:
        raise ValueError("rik needs D or C")
    K = np.empty((n, n))
    st = RIKInfo()
    if C is not None:
        C = C if hasattr(C, "data_ptr") else _f64(C)
        if len(C.shape) != 2 or C.shape[0] != n:
            raise ValueError(f"C must be [{n}][occ]")
        _call(structure, "lible_gpu_rik", None, _ptr(C), int(C.shape[1]), float(schwarz), _ptr(K),
              ctypes.byref(st))
    else:
        D = D if hasattr(D, "data_ptr") else _f64(D)
        _call(structure, "lible_gpu_rik", _ptr(D), None, 0, float(schwarz), _ptr(K), ctypes.byref(st))
    if info:
        return K, {k: getattr(st, k) for k, _ in RIKInfo._fields_}
    return K


def rik_set_fitted(structure, mode):
    """1 (default): RI-K keeps the fitted three-centre tensor on the context when it fits; 0: stream
    the integrals on every call (and drop a cached tensor)."""
    _call(structure, "lible_gpu_rik_set_fitted", int(mode))


def rij_set_cached(structure, mode):
    """1 (default): rij() keeps the three-centre tensor (mn|P) on the context when it fits; 0:
    evaluate the integrals on every call (and drop a cached tensor)."""
    _call(structure, "lible_gpu_rij_set_cached", int(mode))


def ri_contract(structure, D=None, dcoef=None, schwarz=1e-12):
    """gamma_P = sum (mn|P) D_mn (if D is given) and J_mn = sum_P (mn|P) d_P (if dcoef is given)."""
    n, na = structure.nao, structure.naux
    g = np.empty(na) if D is not None else None
    J = np.empty((n, n)) if dcoef is not None else None
    _call(structure, "lible_gpu_ri_contract", _ptr(_f64(D)) if D is not None else None,
          _ptr(_f64(dcoef)) if dcoef is not None else None, float(schwarz), _ptr(g), _ptr(J))
    return g, J


def jk_plan(structure, schwarz=1e-12, precision="fp64", fp32_threshold=1e-4):
    """Quartet / primitive-quartet counts and algorithmic FLOPs of one J/K build with these options."""
    info = JKPlanInfo()
    opts = _opts(schwarz, precision, fp32_threshold)
    _call(structure, "lible_gpu_jk_plan", ctypes.byref(opts), ctypes.byref(info))
    return {k: getattr(info, k) for k, _ in JKPlanInfo._fields_}


def stream_handle(structure):
    """The cudaStream_t the structure's calls run on (integer handle)."""
    p = ctypes.c_void_p()
    _call(structure, "lible_gpu_stream", ctypes.byref(p))
    return p.value or 0


def fp64_peak(structure):
    """Measured (DFMA, DMMA) FP64 TFLOP/s of the structure's GPU."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _call(structure, "lible_gpu_fp64_peak", ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def fp32_peak(structure):
    """Measured (scalar FFMA, packed FFMA2) FP32 TFLOP/s of the structure's GPU."""
    a, b = ctypes.c_double(), ctypes.c_double()
    _call(structure, "lible_gpu_fp32_peak", ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def check_bounded_wait(structure, polls=4096):
    """Runs one device wait that cannot complete and lets it give up after `polls` polls: raises
    LibleGpuError with code 6 (ETIMEOUT), the error a stalled bulk copy produces."""
    _call(structure, "lible_gpu_check_bounded_wait", int(polls))


def eval_special(structure, which, x, order=0):
    """Device special functions for tests: which "exp" -> e^{-x}; "boys" / "boys32" -> F_0..F_order(x)
    in FP64 / in the FP32 form of FP32 quartets (rows per x)."""
    w = {"exp": 0, "boys": 1, "boys32": 2}[which]
    x = _f64(x).ravel()
    out = np.empty(len(x) if w == 0 else (len(x), order + 1))
    _call(structure, "lible_gpu_eval_special", w, int(order), len(x), _ptr(x), _ptr(out))
    return out


def inject_wait_timeout(structure, polls=4096):
    """Makes the next kernel-API store launch on the structure's context run its bulk-copy classes
    without issuing the copies, so their waits give up after `polls` polls and that call raises
    LibleGpuError with code 6 (ETIMEOUT); nothing is in flight and the context stays usable."""
    _call(structure, "lible_gpu_inject_wait_timeout", int(polls))


def jk_plan_classes(structure, schwarz=1e-12, precision="fp64", fp32_threshold=1e-4):
    """Per class pair of the J/K plan (launch order): (la, lb, lc, ld), n_fp64, n_fp32, primitive
    quartets, algorithmic FLOPs."""
    opts = _opts(schwarz, precision, fp32_threshold)
    n = ctypes.c_int()
    _call(structure, "lible_gpu_jk_plan_classes", ctypes.byref(opts), ctypes.byref(n), None, None, None, None, None)
    k = n.value
    ls, n64, n32 = np.zeros(4 * k, np.int32), np.zeros(k, np.int64), np.zeros(k, np.int64)
    prim, fl = np.zeros(k), np.zeros(k)
    _call(structure, "lible_gpu_jk_plan_classes", ctypes.byref(opts), ctypes.byref(n), _ptr(ls), _ptr(n64), _ptr(n32),
          _ptr(prim), _ptr(fl))
    return [(tuple(int(x) for x in ls[4 * i:4 * i + 4]), int(n64[i]), int(n32[i]), float(prim[i]), float(fl[i]))
            for i in range(k)]

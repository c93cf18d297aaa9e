"""Test infrastructure only: Python access to the C restatement (oracle/eri_port.c, built into
oracle/_ref/liberi_port.so).  Reads basis sets from the engine's shipped basis directory in the
reference's text format with its own small parser."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_ref", "liberi_port.so")
BASIS_MAIN = os.path.join(os.path.dirname(HERE), "lible_b200", "basis", "main")

_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(PORT_LIB)
        P = ctypes.c_void_p
        L.port_new.restype = P
        L.port_new.argtypes = [ctypes.c_int] + [P] * 7
        L.port_free.argtypes = [P]
        L.port_nao.argtypes = [P]
        L.port_nao.restype = ctypes.c_int
        L.port_boys.argtypes = [ctypes.c_int, ctypes.c_double, P]
        L.port_eri4.argtypes = [P, P]
        L.port_jk.argtypes = [P, P, P, P, ctypes.c_double, ctypes.c_int]
        L.port_jk.restype = ctypes.c_longlong
        L.port_jk_grad.argtypes = [P, P, P]
        _lib = L
    return _lib


def read_basis(name, Z, root=BASIS_MAIN):
    """Per-atom shells [(l, exps, coeffs), ...] from <root>/<family>/<name>.txt."""
    path = None
    for fam in sorted(os.listdir(root)):
        cand = os.path.join(root, fam, name.lower() + ".txt")
        if os.path.exists(cand):
            path = cand
    if path is None:
        raise FileNotFoundError(name)
    lines = open(path).read().splitlines()
    out = []
    for z in Z:
        i = lines.index(f"element={z}") + 1
        shells = []
        while lines[i] != f"end={z}":
            if "l=" in lines[i]:
                shells.append((int(lines[i].split("l=")[1][0]), [], []))
            elif lines[i].strip():
                e, c = lines[i].split()[:2]
                shells[-1][1].append(float(e))
                shells[-1][2].append(float(c))
            i += 1
        out.append(shells)
    return out


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class PortMolecule:
    def __init__(self, basis, Z, xyz_bohr):
        atoms = read_basis(basis, Z) if isinstance(basis, str) else basis
        nsh = np.array([len(a) for a in atoms], np.int32)
        ls = np.array([s[0] for a in atoms for s in a], np.int32)
        nps = np.array([len(s[1]) for a in atoms for s in a], np.int32)
        ex = np.array([e for a in atoms for s in a for e in s[1]], np.float64)
        co = np.array([c for a in atoms for s in a for c in s[2]], np.float64)
        Zs = np.asarray(Z, np.int32)
        xyz = np.ascontiguousarray(xyz_bohr, np.float64).reshape(-1, 3)
        self.n_atoms = len(Zs)
        self.h = ctypes.c_void_p(lib().port_new(len(Zs), _p(Zs), _p(xyz), _p(nsh), _p(ls), _p(nps), _p(ex), _p(co)))
        self.nao = lib().port_nao(self.h)

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.port_free(self.h)
            self.h = None

    def eri4(self):
        out = np.empty((self.nao,) * 4)
        lib().port_eri4(self.h, _p(out))
        return out

    def jk(self, D, schwarz=0.0, bra_stride=1):
        D = np.ascontiguousarray(D, np.float64)
        J, K = np.empty_like(D), np.empty_like(D)
        nq = lib().port_jk(self.h, _p(D), _p(J), _p(K), schwarz, bra_stride)
        return J, K, nq

    def jk_grad(self, D):
        D = np.ascontiguousarray(D, np.float64)
        g = np.empty((self.n_atoms, 3))
        lib().port_jk_grad(self.h, _p(D), _p(g))
        return g


def boys(n, x):
    F = np.empty(n + 1)
    lib().port_boys(n, float(x), _p(F))
    return F


def jk(basis, Z, xyz_bohr, D, schwarz=0.0):
    J, K, _ = PortMolecule(basis, Z, xyz_bohr).jk(D, schwarz)
    return J, K

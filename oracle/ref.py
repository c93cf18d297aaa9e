"""Test infrastructure only: ctypes access to the reference's own ERI code built by oracle/Makefile
(oracle/_ref/liblible_ref.so, see oracle/ref_capi.cpp).  Used by tests/ and by the CPU-baseline
and reference arms of bench.py; never by the product."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "liblible_ref.so")
BASIS = os.path.join(os.path.dirname(HERE), "lible_b200", "basis")
BOHR_TO_ANG = 0.5291772083

_lib = None


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(REF_LIB)
        P = ctypes.c_void_p
        L.ref_structure_named.restype = P
        L.ref_structure_named.argtypes = [ctypes.c_char_p] * 4 + [ctypes.c_int, P, P]
        L.ref_structure_custom.restype = P
        L.ref_structure_custom.argtypes = [ctypes.c_int] + [P] * 12
        L.ref_structure_free.argtypes = [P]
        for f in ("ref_dim_ao", "ref_dim_ao_aux", "ref_n_atoms"):
            getattr(L, f).restype = ctypes.c_long
            getattr(L, f).argtypes = [P]
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_deploy_sum.restype = ctypes.c_double
        L.ref_deploy_sum.argtypes = [P, ctypes.c_int]
        L.ref_jk.argtypes = [P, P, P, P, ctypes.c_double, ctypes.c_int, P, P]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        for f in ("ref_eri4", "ref_eri4_diagonal", "ref_eri3", "ref_eri2", "ref_eri2_diagonal"):
            getattr(L, f).argtypes = [P, P]
        L.ref_eri4_class.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.ref_eri4d1_class.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.ref_eri3_class.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.ref_eri3d1_class.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.ref_eri2d1_class.argtypes = [P, ctypes.c_int, ctypes.c_int, P]
        L.ref_pair_classes.argtypes = [P, ctypes.c_int, P, P, P, P]
        L.ref_aux_classes.argtypes = [P, P, P, P]
        L.ref_jk_grad.argtypes = [P, P, P]
        L.ref_jk_grad_sample.argtypes = [P, P, P, ctypes.c_double, ctypes.c_int, P, P]
        L.ref_rij_gamma.argtypes = [P, P, P]
        L.ref_rij_j.argtypes = [P, P, P]
        L.ref_one_electron.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P]
        L.ref_eri4soc_class.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.ref_eri3soc_class.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.ref_eri2d2_class.argtypes = [P, ctypes.c_int, ctypes.c_int, P]
        L.ref_one_electron_class.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int, P]
        L.ref_one_electron_class_ex.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int, P, P]
        L.ref_one_electron_ex.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int, P, P]
        _lib = L
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class RefStructure:
    """The reference's lible::ints::Structure.  coords in bohr unless units='angstrom'."""

    def __init__(self, basis, Z, coords, aux=None, units="bohr"):
        L = lib()
        Z = np.ascontiguousarray(Z, dtype=np.int32)
        xyz = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        if units == "bohr":
            xyz = xyz * BOHR_TO_ANG
        if isinstance(basis, str):
            h = L.ref_structure_named(os.path.join(BASIS, "main").encode(), os.path.join(BASIS, "aux").encode(),
                                      basis.encode(), aux.encode() if aux else None, len(Z), _p(Z), _p(xyz))
        else:
            m = _flatten(basis)
            a = _flatten(aux) if aux is not None else [None] * 5
            self._keep = (m, a)
            h = L.ref_structure_custom(len(Z), _p(Z), _p(xyz), *[_p(x) for x in m],
                                       *[(_p(x) if x is not None else None) for x in a])
        if not h:
            raise RuntimeError(L.ref_last_error().decode())
        self.h = ctypes.c_void_p(h)
        self.nao = L.ref_dim_ao(self.h)
        self.naux = L.ref_dim_ao_aux(self.h)
        self.n_atoms = L.ref_n_atoms(self.h)

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.ref_structure_free(self.h)
            self.h = None

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(lib().ref_last_error().decode())

    def eri4(self):
        out = np.empty((self.nao,) * 4)
        self._chk(lib().ref_eri4(self.h, _p(out)))
        return out

    def eri4_diagonal(self):
        out = np.empty((self.nao,) * 2)
        self._chk(lib().ref_eri4_diagonal(self.h, _p(out)))
        return out

    def eri3(self):
        out = np.empty((self.nao, self.nao, self.naux))
        self._chk(lib().ref_eri3(self.h, _p(out)))
        return out

    def eri2(self):
        out = np.empty((self.naux, self.naux))
        self._chk(lib().ref_eri2(self.h, _p(out)))
        return out

    def one_electron(self, which, charges=None):
        """The reference's overlap / kineticEnergy / nuclearAttraction / externalCharges
        (which = 0..3; charges [n][4] = x, y, z in bohr, q)."""
        out = np.empty((self.nao, self.nao))
        q = np.ascontiguousarray(charges if charges is not None else np.zeros((0, 4)), dtype=np.float64)
        self._chk(lib().ref_one_electron(self.h, which, _p(q), len(q), _p(out)))
        return out

    def one_electron_ex(self, which, charges=None, omegas=None, origin=None):
        """The reference's dipoleMoment / momentum / angularMomentum ([3][nao][nao], which = 4, 5, 6)
        and nuclearAttractionErf / externalChargesErf (which = 7, 8)."""
        out = np.empty((3, self.nao, self.nao) if (which <= 6 or which == 9) else (self.nao, self.nao))
        q = np.ascontiguousarray(charges if charges is not None else np.zeros((0, 4)), dtype=np.float64)
        w = None if omegas is None else np.ascontiguousarray(omegas, dtype=np.float64)
        o = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
        self._chk(lib().ref_one_electron_ex(self.h, which, _p(q), _p(w) if w is not None else None, len(q),
                                            _p(o) if o is not None else None, _p(out)))
        return out

    def eri4soc_class(self, use_symm, iab, icd):
        cls = self.pair_classes(use_symm)
        (la, lb, na, _), (lc, ld, nc, _) = cls[iab], cls[icd]
        out = np.empty((na, nc, 3, 2 * la + 1, 2 * lb + 1, 2 * lc + 1, 2 * ld + 1))
        self._chk(lib().ref_eri4soc_class(self.h, int(use_symm), iab, icd, _p(out)))
        return out

    def eri3soc_class(self, use_symm, iab, ic):
        (la, lb, na, _), (lc, nc) = self.pair_classes(use_symm)[iab], self.aux_classes()[ic]
        out = np.empty((na, nc, 3, 2 * la + 1, 2 * lb + 1, 2 * lc + 1))
        self._chk(lib().ref_eri3soc_class(self.h, int(use_symm), iab, ic, _p(out)))
        return out

    def eri2d2_class(self, ia, ib):
        acls = self.aux_classes()
        (la, na), (lb, nb) = acls[ia], acls[ib]
        out = np.empty((na, nb, 6, 6, 2 * la + 1, 2 * lb + 1))
        self._chk(lib().ref_eri2d2_class(self.h, ia, ib, _p(out)))
        return out

    def one_electron_class(self, use_symm, iab, op, charges=None):
        la, lb, na, _ = self.pair_classes(use_symm)[iab]
        nb = 6 if op >= 3 else 1
        out = np.empty((na, nb, 2 * la + 1, 2 * lb + 1))
        q = np.ascontiguousarray(charges if charges is not None else np.zeros((0, 4)), dtype=np.float64)
        self._chk(lib().ref_one_electron_class(self.h, int(use_symm), iab, op, _p(q), len(q), _p(out)))
        return out if nb > 1 else out[:, 0]

    def one_electron_class_ex(self, use_symm, iab, op, charges=None, omegas=None, origin=None):
        """op 6 dipoleMomentKernel, 7 momentumKernel, 8 angularMomentumKernel ([n][3][Sa][Sb]),
        9 externalChargesErfKernel ([n][Sa][Sb]), 10 externalChargesErfD1Kernel ([n][6][Sa][Sb]),
        11 / 12 externalChargesOperator(Erf)D1Kernel ([n][n_charges * 3][Sa][Sb]), 13 / 14
        potentialAtExternalCharges(Erf)Kernel ([n][n_charges][Sa][Sb]) for every pair of one class."""
        la, lb, na, _ = self.pair_classes(use_symm)[iab]
        q = np.ascontiguousarray(charges if charges is not None else np.zeros((0, 4)), dtype=np.float64)
        nq = len(q)
        nb = 1 if op == 9 else 6 if op == 10 else 9 if op == 16 else 3 * nq if op in (11, 12) else nq if op in (13, 14) else 3
        out = np.empty((na, nb, 2 * la + 1, 2 * lb + 1))
        w = None if omegas is None else np.ascontiguousarray(omegas, dtype=np.float64)
        o = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
        self._chk(lib().ref_one_electron_class_ex(self.h, int(use_symm), iab, op, _p(q),
                                                  _p(w) if w is not None else None, len(q),
                                                  _p(o) if o is not None else None, _p(out)))
        return out if nb > 1 else out[:, 0]

    def eri2_diagonal(self):
        out = np.empty(self.naux)
        self._chk(lib().ref_eri2_diagonal(self.h, _p(out)))
        return out

    def deploy_sum(self, which):
        return lib().ref_deploy_sum(self.h, which)

    def pair_classes(self, use_symm):
        n = ctypes.c_int()
        self._chk(lib().ref_pair_classes(self.h, int(use_symm), ctypes.byref(n), None, None, None))
        ls = np.zeros(2 * n.value, np.int32)
        npairs = np.zeros(n.value, np.int64)
        nppairs = np.zeros(n.value, np.int64)
        self._chk(lib().ref_pair_classes(self.h, int(use_symm), ctypes.byref(n), _p(ls), _p(npairs), _p(nppairs)))
        return [(int(ls[2 * i]), int(ls[2 * i + 1]), int(npairs[i]), int(nppairs[i])) for i in range(n.value)]

    def aux_classes(self):
        n = ctypes.c_int()
        self._chk(lib().ref_aux_classes(self.h, ctypes.byref(n), None, None))
        ls = np.zeros(n.value, np.int32)
        nsh = np.zeros(n.value, np.int64)
        self._chk(lib().ref_aux_classes(self.h, ctypes.byref(n), _p(ls), _p(nsh)))
        return [(int(ls[i]), int(nsh[i])) for i in range(n.value)]

    def eri4_class(self, use_symm, iab, icd, d1=False):
        cl = self.pair_classes(use_symm)
        (la, lb, na, _), (lc, ld, nc, _) = cl[iab], cl[icd]
        shape = (na, nc) + ((12,) if d1 else ()) + (2 * la + 1, 2 * lb + 1, 2 * lc + 1, 2 * ld + 1)
        out = np.empty(shape)
        f = lib().ref_eri4d1_class if d1 else lib().ref_eri4_class
        self._chk(f(self.h, int(use_symm), iab, icd, _p(out)))
        return out

    def eri3_class(self, use_symm, iab, ic, d1=False):
        la, lb, na, _ = self.pair_classes(use_symm)[iab]
        lc, nc = self.aux_classes()[ic]
        shape = (na, nc) + ((9,) if d1 else ()) + (2 * la + 1, 2 * lb + 1, 2 * lc + 1)
        out = np.empty(shape)
        f = lib().ref_eri3d1_class if d1 else lib().ref_eri3_class
        self._chk(f(self.h, int(use_symm), iab, ic, _p(out)))
        return out

    def eri2d1_class(self, ia, ib):
        la, na = self.aux_classes()[ia]
        lb, nb = self.aux_classes()[ib]
        out = np.empty((na, nb, 6, 2 * la + 1, 2 * lb + 1))
        self._chk(lib().ref_eri2d1_class(self.h, ia, ib, _p(out)))
        return out

    def jk(self, D, schwarz=1e-12, bra_stride=1):
        D = np.ascontiguousarray(D, dtype=np.float64)
        J, K = np.empty_like(D), np.empty_like(D)
        nq, sec = ctypes.c_longlong(), ctypes.c_double()
        self._chk(lib().ref_jk(self.h, _p(D), _p(J), _p(K), schwarz, bra_stride, ctypes.byref(nq), ctypes.byref(sec)))
        return J, K, nq.value, sec.value

    def jk_grad(self, D):
        D = np.ascontiguousarray(D, dtype=np.float64)
        g = np.empty((self.n_atoms, 3))
        self._chk(lib().ref_jk_grad(self.h, _p(D), _p(g)))
        return g

    def jk_grad_sample(self, D, schwarz=1e-12, bra_stride=1):
        """The gradient over the Schwarz-surviving quartets of every bra_stride-th bra pair (a timing
        sample); returns (grad, quartets processed, seconds)."""
        D = np.ascontiguousarray(D, dtype=np.float64)
        g = np.empty((self.n_atoms, 3))
        nq, sec = ctypes.c_longlong(), ctypes.c_double()
        self._chk(lib().ref_jk_grad_sample(self.h, _p(D), _p(g), schwarz, bra_stride, ctypes.byref(nq),
                                           ctypes.byref(sec)))
        return g, nq.value, sec.value

    def rij_gamma(self, D):
        D = np.ascontiguousarray(D, dtype=np.float64)
        g = np.empty(self.naux)
        self._chk(lib().ref_rij_gamma(self.h, _p(D), _p(g)))
        return g

    def rij_j(self, d):
        d = np.ascontiguousarray(d, dtype=np.float64)
        J = np.empty((self.nao, self.nao))
        self._chk(lib().ref_rij_j(self.h, _p(d), _p(J)))
        return J


def _flatten(basis_atoms):
    nsh, ls, nps, ex, co = [], [], [], [], []
    for atom in basis_atoms:
        nsh.append(len(atom))
        for (l, exps, coeffs) in atom:
            ls.append(l)
            nps.append(len(exps))
            ex.extend(exps)
            co.extend(coeffs)
    return (np.asarray(nsh, np.int32), np.asarray(ls, np.int32), np.asarray(nps, np.int32),
            np.asarray(ex, np.float64), np.asarray(co, np.float64))


def set_threads(n):
    lib().ref_set_threads(int(n))


def max_threads():
    return lib().ref_max_threads()

"""Maintenance recipe: regenerates the basis-set text files shipped in lible_b200/basis/.

The engine reads basis sets in the reference's plain-text format
(``element=Z`` / ``l=L n=K`` / ``exponent coefficient`` lines / ``end=Z``; parser at
src/lible/ints/basis_sets.cpp:214-277 of the reference) and in its directory layout
(``<root>/<family>/<name>.txt``, src/lible/ints/basis_sets.cpp:318-360).  Only the elements and
basis sets the tests and benchmarks use are kept: H, C and O, in the main sets
cc-pVDZ, cc-pVTZ, def2-SVP, def2-TZVP, 6-31+G and the auxiliary sets def2-QZVP-RIFIT,
def2-universal-JKFIT and cc-pVDZ-RIFIT.  The numbers are the published basis-set data, copied
verbatim so that integrals agree with the reference to the last bit.

Usage (needs a checkout of the reference project, given explicitly):
    python oracle/extract_basis.py <reference checkout>
"""
import os
import sys

ELEMENTS = (1, 6, 8)
MAIN = {"dunning": ("cc-pvdz", "cc-pvtz"), "ahlrichs": ("def2-svp", "def2-tzvp"), "pople": ("6-31+g",)}
AUX = {"ahlrichs": ("def2-qzvp-rifit", "def2-universal-jkfit"), "dunning": ("cc-pvdz-rifit",)}


def extract(src_path, dst_path):
    keep, out = False, []
    with open(src_path) as fh:
        for line in fh:
            s = line.rstrip("\n")
            if s.startswith("element="):
                keep = int(s.split("=")[1]) in ELEMENTS
            if keep:
                out.append(s)
            if s.startswith("end="):
                keep = False
    os.makedirs(os.path.dirname(dst_path), exist_ok=True)
    with open(dst_path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def main(ref_root):
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lible_b200", "basis")
    src = os.path.join(ref_root, "src", "lible", "ints")
    for kind, table, sub in (("main", MAIN, "lible_basis"), ("aux", AUX, "lible_aux_basis")):
        for family, names in table.items():
            for name in names:
                extract(os.path.join(src, sub, family, name + ".txt"),
                        os.path.join(here, kind, family, name + ".txt"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python oracle/extract_basis.py <reference checkout>")
    main(sys.argv[1])

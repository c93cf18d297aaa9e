"""B200-native electron-repulsion-integral engine: a drop-in for the lible::ints ERI calls of
MihkuU/Lible (2-, 3- and 4-centre integrals and their first derivatives) with direct J/K, RI-J and
the J/K energy gradient.  The compute path is the sm_100a CUDA library liblible_b200.so behind the
C ABI of include/lible_b200.h; this package is its Python host mirror."""
from ._lib import LibleGpuError, LIB_PATH  # noqa: F401
from .ints import (Structure, eri4, eri4Diagonal, eri3, eri2, eri2Diagonal, shellPairData,  # noqa: F401
                   shellDataAux, ERI4Kernel, ERI3Kernel, ERI2Kernel, ERI4D1Kernel, ERI3D1Kernel,
                   ERI2D1Kernel, jk, jk_energy_forward, jk_energy_backward, rij)

"""gradscf_b200 -- B200-native direct-SCF J/K (Coulomb/exchange) build.

Drop-in for GradSCF's direct J/K path: the C ABI in include/b200jk.h
(libb200jk.so, hand-written sm_100a CUDA) with Python mirrors of the
reference's ``direct_jk`` / ``IntegralPlan.get_jk`` / ``NativeDirectBasis``.
"""
from .basis import (BasisParameters, BasisTopology, Molecule, build_tables, load_basis, pack,
                    parse_molecule, prepare_basis)

__all__ = ["BasisParameters", "BasisTopology", "Molecule", "build_tables", "load_basis", "pack",
           "parse_molecule", "prepare_basis"]

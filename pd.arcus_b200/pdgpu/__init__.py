"""pdgpu: PD's GB/SA energy-force hot path on B200 (sm_100a).

Importable as ``pdgpu`` with ``pd.arcus_b200`` on sys.path.  All evaluation
runs in libpdgpu.so (hand-written CUDA behind a C ABI, include/pdgpu.h);
there is no CPU fallback.
"""
from ._abi import (PdgpuError, UnstableError, lib, last_error, ff_params_default,  # noqa: F401
                   md_params_default, min_params_default, FFParams, MDParams, MinParams)
from .core import (Context, SystemSpec, WorkSpace, NeighbourList, Hamiltonian,  # noqa: F401
                   ForcefieldBase, Forcefield, FF_Bonded, FF_NonBonded, FF_GeneralizedBorn_Still, FF_SASA_LCPO,
                   ProtocolBase, Energy, Minimisation, MolecularDynamics, MonteCarlo, J2KCAL_NA)
from .batch import Batch  # noqa: F401
from .serve import Server  # noqa: F401

# the reference's pre-rename aliases used by its example scripts (src/RENAME.log)
GB_Still = FF_GeneralizedBorn_Still
BondedForcefield = FF_Bonded
NonBondedForcefield = FF_NonBonded

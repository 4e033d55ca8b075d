"""B200-native implementation of the DASH (dreid1991/md_engine) per-timestep
force hot path: cell-binned neighbour list, LJ/WCA + Ewald real-space pair
forces, P3M reciprocal space, E3B three-body water, SETTLE rigid water and the
velocity-Verlet / Nose-Hoover update, as hand-written sm_100a CUDA behind the
C ABI of include/mdx.h (libmdx.so)."""
from .dash import (Bounds, FixChargeEwald, FixChargePairDSF, FixE3B, FixLJCHARMM, FixLJCut,  # noqa: F401
                   FixLJCutFS, FixNoseHoover, FixPressureBerendsen, FixRigid, FixTICG, FixWCA, BatchReplicas,
                   IntegratorVerlet, State, Vector, WriteConfig, kernel_launches)
from ._lib import LIB_PATH, MdxError, lib  # noqa: F401

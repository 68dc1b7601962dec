"""susy_b200: B200-native RHMC fermion path of SUSY LATTICE (4d_Q16).

The compute path is ``libsusy_b200.so`` (hand-written sm_100a CUDA behind
the C ABI in include/susy_b200.h).  This package holds the Python mirror of
the reference interface (:class:`Lattice`) and seeded synthetic inputs.
"""
from .lattice import (Lattice, DeviceTF, SusyError, RHMC, load_library, LIB_PATH,  # noqa: F401
                      SOLVER_FP64, SOLVER_MIXED, HMC, SMD, update_batch, dsq_batch,
                      congrad_multi_batch)

from . import learned  # noqa: F401,E402

__all__ = ["learned", "Lattice", "DeviceTF", "SusyError", "RHMC", "load_library", "LIB_PATH",
           "SOLVER_FP64", "SOLVER_MIXED", "HMC", "SMD", "update_batch", "dsq_batch",
           "congrad_multi_batch"]

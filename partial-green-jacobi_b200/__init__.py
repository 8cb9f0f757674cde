"""B200-native periodic HEX8 homogenization with the partial Green-Jacobi preconditioned PCG.

Host package over libpgj.so (hand-written sm_100a CUDA behind a C ABI, include/pgj.h). Import it as
``pgj_b200`` via ``load_package()`` in ``__graft_entry__`` (the directory name is not a Python
identifier).
"""
from . import _lib
from .resident import (Backend, Operator, PaperBackend, PaperResident, Resident, SelectorResident, ETA_ANCHORS,
                       PAPER_MEDIUM, STUDY1_MEDIUM)
from .outer import PaperOuter, ResidentOuter, cone_stencil, gaussian_weights
from .designs import baseline_density, baseline_design, simp, study1_initial, study1_state0
from .batch import Batch, BatchedOperator, Request, Result
from . import alpha_selectors, replay_state, serve, shear_design

__all__ = ["Backend", "Operator", "PaperBackend", "PaperResident", "Resident", "SelectorResident", "PaperOuter",
           "ResidentOuter", "cone_stencil", "gaussian_weights", "baseline_density", "baseline_design", "simp",
           "study1_initial", "study1_state0", "Batch", "BatchedOperator", "Request", "Result", "alpha_selectors", "replay_state",
           "serve", "shear_design", "ETA_ANCHORS", "PAPER_MEDIUM", "STUDY1_MEDIUM", "_lib"]

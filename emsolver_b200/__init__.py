"""emsolver_b200 -- B200-native SCN TLM time step with EMSolver's TlmSolver interface,
and the reference's Yee FDTD solver behind the same interface (FdtdSolver).

The compute path is the in-tree CUDA library ``libtlm_b200.so`` (C ABI in
``include/tlm_b200.h``); this package is its Python host side.
"""
from .batch import Batch, BatchTuning
from .emsim import Project, load_project
from .fdtd import FdtdSolver
from .server import Server
from .solver import (FieldProbe, MAT_AIR, MAT_DIEL0, MAT_PEC, MatProps, Storage, TlmConfig,
                     TlmPort, TlmSolver, VoxelGridSpec, WaveformType, s11_from_dft)

__all__ = ["Batch", "BatchTuning", "Project", "load_project", "FdtdSolver", "Server", "TlmSolver", "TlmConfig", "VoxelGridSpec", "MatProps", "TlmPort", "FieldProbe",
           "WaveformType", "Storage", "MAT_AIR", "MAT_PEC", "MAT_DIEL0", "s11_from_dft"]

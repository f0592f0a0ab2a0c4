"""cuda_fsp_b200 -- B200-native (sm_100a, FP64) Finite State Projection engine.

The product is the CUDA library behind include/cufsp.h (cuda_fsp_b200/lib/libcufsp.so); this
package is its Python mirror of the reference's API (FSPMat, KryExpvFSP, FSPSolver, Likelihood,
the BDF integrator that replaces its CVODE path) plus the workload definitions in `models`.
"""
from . import models
from ._lib import CufspError
from .batch import BatchKrylov
from .fsp import FSPMat, KryExpvFSP, MatrixFormat, expm, get_states, num_states
from .likelihood import AdaptiveFSP, FSPSolver, Likelihood, generate_data, histograms
from .ode import BDFIntegrator

__all__ = ["models", "CufspError", "BatchKrylov", "FSPMat", "KryExpvFSP", "MatrixFormat", "expm", "get_states", "num_states",
           "FSPSolver", "AdaptiveFSP", "Likelihood", "generate_data", "histograms", "BDFIntegrator"]

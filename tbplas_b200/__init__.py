"""tbplas_b200: the TBPM core of TBPLaS rebuilt for NVIDIA B200 (sm_100a).

The package keeps the reference's TBPM API (`Config`, `Solver`, `Analyzer`,
and an f2py-compatible `fortran.f2py` module) and runs the Chebyshev
propagation and correlation loops as CUDA kernels in libtbpm_b200.so.
"""
from .base import EPSILON0, H_BAR_EV, KB
from .builder import LatticeSample, PackedSamples, make_graphene_sample, pack_samples
from .parallel import MPIEnv
from .supercell import DeviceSample, make_graphene_device_sample
from .tbpm import (Analyzer, Config, Solver, read_config, window_exp, window_exp_ten,
                   window_hanning)

__all__ = ["Config", "read_config", "Solver", "Analyzer", "window_hanning", "window_exp",
           "window_exp_ten", "LatticeSample", "make_graphene_sample", "pack_samples",
           "PackedSamples", "MPIEnv", "KB", "H_BAR_EV", "EPSILON0", "DeviceSample",
           "make_graphene_device_sample"]

"""B200-native flat-panel circular cone-beam FDK and Joseph projector pair.

A from-scratch sm_100a implementation of one hot path of YKCBCT
(YuuKozlx/fdk_cuda_impl): FDK (cosine preweight, ramp filter, voxel-driven
weighted backprojection) and the Joseph forward projector with its exact
matched backprojector.  Compute lives in libykb.so (include/ykb.h); this
package is the torch-facing host layer over that C-ABI.
"""
from . import _lib
from .geometry import CircularScan, RampFilter, VolumeGrid

__all__ = ["CircularScan", "RampFilter", "VolumeGrid", "FdkPlan", "JosephPlan",
           "JosephProjector", "library_path", "load_library"]


def library_path() -> str:
    return _lib.LIB_PATH


def load_library():
    return _lib.load()


def __getattr__(name):
    # torch-dependent parts load lazily so that geometry helpers work without CUDA
    if name in ("FdkPlan", "JosephPlan"):
        from . import projectors
        return getattr(projectors, name)
    if name == "JosephProjector":
        from .autograd import JosephProjector
        return JosephProjector
    raise AttributeError(name)

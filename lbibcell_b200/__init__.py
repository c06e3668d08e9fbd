"""lbibcell_b200: LBIBCell's lattice hot path on one NVIDIA B200.

The compute path is liblbibcuda.so (hand-written sm_100a CUDA kernels behind
the C ABI of include/lbibcell.h); this package is the host-side mirror of the
reference's simulation interface (``runner.Simulation``) and the seeded
synthetic configurations in the reference's file formats (``configs``).
"""
from . import configs  # noqa: F401
from ._lib import LIB_PATH, LbibError, load  # noqa: F401

__all__ = ["configs", "load", "LbibError", "LIB_PATH", "Simulation", "FP64", "FP32_SHIFTED"]


def __getattr__(name):
    if name in ("Simulation", "FP64", "FP32_SHIFTED"):
        from . import runner
        return getattr(runner, name)
    raise AttributeError(name)

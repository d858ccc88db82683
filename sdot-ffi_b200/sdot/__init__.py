"""sdot (B200 build): the semi-discrete optimal transport path of hleclerc/sdot-ffi -- power diagrams and the
damped-Newton SDOT solve -- on hand-written sm_100a CUDA kernels behind a C ABI (include/sdot_b200.h).

The names are the reference's (src/sdot/__init__.py:25-60) for the parts of its API this path covers.
"""
from .PowerDiagram import PowerDiagram, Voronoi, box_half_spaces, axis_aligned_box
from .OtProblem import OtProblem, Iterative, Tuning, OtNotConverged, ot_solve
from .SdotPlanNd import SdotPlanNd, exact_duplicates
from .distributions import SumOfDiracs, Image, SumOfGaussians, Box
from ._lib import KernelFailure
from .quantization import quantization

_KERNEL_DTYPE = "FP64"


def set_kernel_dtype(dtype):
    """the float the cells are cut in: FP64 only in this build"""
    global _KERNEL_DTYPE
    if dtype not in ("FP64", "fp64"):
        raise NotImplementedError("set_kernel_dtype: FP64 only in this build")
    _KERNEL_DTYPE = "FP64"


def kernel_dtype():
    return _KERNEL_DTYPE


def plan(f, g):
    return OtProblem(f, g).solve()


def w2(f, g):
    return plan(f, g).cost


__all__ = ["PowerDiagram", "Voronoi", "box_half_spaces", "axis_aligned_box", "OtProblem", "Iterative", "Tuning", "OtNotConverged", "ot_solve",
           "SdotPlanNd", "exact_duplicates", "SumOfDiracs", "Image", "SumOfGaussians", "Box", "KernelFailure", "set_kernel_dtype",
           "kernel_dtype", "plan", "w2", "quantization"]

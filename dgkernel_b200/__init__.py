"""B200 (sm_100a) backend for DGKernel's partition-parallel tet-DG right-hand side.

The compute path is libdgk.so (hand-written CUDA + C++ behind the C ABI in include/dgk.h); this package
is the Python mirror of the reference's runner API over it.  Importing it loads the library; there is no
CPU fallback.
"""
from ._lib import DGKError, lib, LIB_PATH
from .runner import (Config, Copy, CopyBack, CopyTo, Float32, Float64, INT32, INT64, InOut, Input, NewRunner,
                     NoAction, Output, ParamBuilder, Runner, Scalar, Temp, CacheLineAlign, NoAlignment, PageAlign,
                     WarpAlign)
from .element import Element
from . import mesh

__all__ = ["DGKError", "lib", "LIB_PATH", "Config", "Runner", "NewRunner", "Input", "Output", "InOut", "Scalar", "Temp",
           "ParamBuilder", "Float32", "Float64", "INT32", "INT64", "Copy", "CopyTo", "CopyBack", "NoAction",
           "NoAlignment", "CacheLineAlign", "WarpAlign", "PageAlign", "Element", "mesh"]

"""bempp_cuda: B200-native dense Galerkin assembly and potential evaluation.

A ``cuda`` device interface for bempp-cl's dense assembly path.  Host code is
Python; the kernels are hand-written CUDA for sm_100a in libbemppcuda.so,
called through a flat C ABI (include/bemppcuda.h) with ctypes.  torch
provides device buffers and streams only.

* ``bempp_cuda.plugin.install()`` routes bempp_cl's dispatcher to this
  package for ``device_interface="cuda"`` / ``"cuda_mixed"``.
* ``bempp_cuda.grid``, ``space``, ``shapes``, ``operators`` give the same
  path without bempp_cl installed.
"""

from . import _lib  # noqa: F401
from .grid import Grid  # noqa: F401
from .shapes import regular_sphere, ellipsoid, perturbed_sphere, read_gmsh  # noqa: F401
from .space import function_space  # noqa: F401
from .operators import (  # noqa: F401
    OperatorDescriptor,
    Parameters,
    boundary,
    potential,
    far_field,
    DenseDeviceOperator,
)

__version__ = "0.1.0"

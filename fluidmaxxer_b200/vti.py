"""VTK ImageData (.vti) geometry I/O through ``fm_vti_*`` (``include/fm.h``).

:func:`read_vti` mirrors ``readVTI`` (``include/vti/VTIReader.hpp:35-160``):
dimensions from WholeExtent/Extent, the first DataArray thresholded into a
0/1 mask (vector data by magnitude).  It also returns the per-cell values
(a continuous solid fraction, for instance) and reads the binary (base64)
and appended (raw / base64) encodings the reference cannot.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _abi
from ._abi import check


@dataclasses.dataclass
class VTIResult:
    Nx: int
    Ny: int
    Nz: int
    mask: np.ndarray      # uint8 [Nx*Ny*Nz], x fastest
    values: np.ndarray    # float64 [Nx*Ny*Nz]: the scalar, or the vector magnitude


def vti_info(path):
    nx, ny, nz, nv = C.c_int(), C.c_int(), C.c_int(), C.c_longlong()
    check(_abi.lib().fm_vti_info(str(path).encode(), C.byref(nx), C.byref(ny), C.byref(nz), C.byref(nv)))
    return nx.value, ny.value, nz.value, nv.value


def read_vti(path, threshold=0.5) -> VTIResult:
    nx, ny, nz, _ = vti_info(path)
    n = nx * ny * nz
    mask = np.empty(n, np.uint8)
    vals = np.empty(n, np.float64)
    check(_abi.lib().fm_vti_read(str(path).encode(), float(threshold), mask.ctypes.data, vals.ctypes.data, n))
    return VTIResult(nx, ny, nz, mask, vals)


def write_vti(path, nx, ny, nz, values, name="field", binary=True):
    """Write Nx*Ny*Nz scalars (or Nx*Ny*Nz*3 components) as CellData, Float64."""
    v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    n = nx * ny * nz
    comps = v.size // n
    if comps * n != v.size or comps not in (1, 3):
        raise ValueError("write_vti: values must hold 1 or 3 components per cell")
    check(_abi.lib().fm_vti_write(str(path).encode(), nx, ny, nz, v.ctypes.data, comps, name.encode(), int(binary)))

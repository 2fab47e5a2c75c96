"""srf_b200 — B200-native listmode PET projector pair (drop-in for SRF's native ops).

Layers, bottom to top:

* ``libsrf_b200.so`` (``csrc/``, C ABI in ``include/srf_b200.h``): the CUDA kernels —
  TOR and Siddon projection / back-projection / map / adjoint, LOR preprocessing and
  the image algebra of the MLEM/OSEM update.
* ``ops``: tensor-level functions with the reference TF ops' argument lists.
* ``data`` / ``physics``: ``Image``, ``ListModeData*``, ``SplitLoRsModel`` (TOR) and
  ``CompleteLoRsModel`` (Siddon) with ``projection`` / ``backprojection`` dispatch.
* ``preprocess``: ``recon_process`` / ``map_process`` on the device, effmap merge.
* ``recon``: MLEM / OSEM and the efficiency-map pass.

The CUDA library is loaded on first use; there is no CPU compute path.
"""

from . import data, ops, physics, preprocess  # noqa: F401
from .data import (Image, ListModeData, ListModeDataSplit, ListModeDataSplitWithoutTOF,  # noqa
                   ListModeDataWithoutTOF)
from .physics import (CompleteLoRsModel, SplitLoRsModel, backproject_adjoint,  # noqa: F401
                      backprojection, map_lors, projection, projection_backprojection)
from .preprocess import map_process, recon_process  # noqa: F401

__version__ = "0.1.0"


def library():
    """Load (building if needed) and return the CUDA library handle."""
    from . import _lib
    return _lib.load()

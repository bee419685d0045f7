"""gregpackagescpp_b200: the force-and-step hot path of the gtd:: N-body library
(GregW10/GregPackagesCPP) on NVIDIA B200, behind a C ABI (include/gtd_b200.h).

* libgtd_b200.so         - CUDA kernels for sm_100a + the C ABI (built in-tree by ``build``)
* ``System`` / ``Body``  - Python mirror of gtd::system / gtd::body over that ABI
* ``ics``                - seeded synthetic initial conditions (Plummer spheres, ensembles)
"""
from . import ics  # noqa: F401
from ._lib import GtdError, NbodyError, OverlappingBodiesError, TwoBodyError, BarnesHutError  # noqa: F401
from ._lib import InvalidBodyPlacement, IndistinguishableBodies, NsysLoadError, NsysFormatError  # noqa: F401
from ._lib import CallbackError  # noqa: F401
from .system import System, Body, parse_units, RestFromCom, WhileRestBelow, DeviceHook  # noqa: F401

__all__ = ["System", "Body", "parse_units", "ics", "GtdError", "NbodyError", "OverlappingBodiesError",
           "TwoBodyError", "BarnesHutError", "InvalidBodyPlacement", "IndistinguishableBodies", "NsysLoadError",
           "NsysFormatError", "CallbackError", "RestFromCom", "WhileRestBelow", "DeviceHook"]

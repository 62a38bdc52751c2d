"""PF-FLIP uniform-grid time step on B200 (sm_100a).

Drop-in for the reference package's uniform path: ``from pfflip import Config,
Simulator, scenes`` and ``from pfflip.poisson import MGPCG, apply_A`` keep their
names, arguments and results.  The compute runs in libpfflip.so (hand-written
CUDA for sm_100a, C ABI in include/pfflip.h) over torch-owned device memory.
"""

from . import scenes  # noqa: F401
from ._arrays import DeviceArray, copy  # noqa: F401
from .config import Config  # noqa: F401
from .kernels import launch  # noqa: F401


def __getattr__(name):
    # Simulator pulls in torch CUDA state; import it lazily
    if name == "Simulator":
        from .sim import Simulator

        return Simulator
    raise AttributeError(name)


__all__ = ["Config", "Simulator", "scenes", "copy", "launch", "DeviceArray"]

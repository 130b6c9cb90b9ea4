"""B200-native Harmony batch integration, a drop-in for
``rapids_singlecell.pp.harmony_integrate``.

``pp.harmony_integrate`` (AnnData surface) and ``harmonize`` (tensor surface)
call hand-written sm_100a kernels in ``_lib/libharmony_b200.so`` through a C ABI
(``include/harmony_b200.h``).
"""

from . import pp
from .harmony import HarmonyInfo, harmonize

__all__ = ["pp", "harmonize", "HarmonyInfo"]
__version__ = "0.1.0"

"""B200-native Harmony batch integration, a drop-in for
``rapids_singlecell.pp.harmony_integrate``.

``pp.harmony_integrate`` (AnnData surface) and ``harmonize`` (tensor surface), and
``pp.pca`` / ``pca_arrays`` (the PCA that produces the embedding Harmony corrects) and
``pp.neighbors`` / ``knn_arrays`` (the kNN graph built on the corrected embedding),
call hand-written sm_100a kernels in ``_lib/libharmony_b200.so`` through a C ABI
(``include/harmony_b200.h``).
"""

from . import pp
from .harmony import HarmonyInfo, harmonize
from .neighbors import knn_arrays
from .pca import PcaOutput, pca_arrays

__all__ = ["pp", "harmonize", "HarmonyInfo", "pca_arrays", "PcaOutput", "knn_arrays"]
__version__ = "0.1.0"

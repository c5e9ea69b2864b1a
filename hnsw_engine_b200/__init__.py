"""B200-native HNSW query engine: the search half of anamankev/hnsw-engine on sm_100a kernels.

Graphs are built by the reference's host build and saved with ``save_native``; this package opens
them (``HNSWIndex.load_native``) and searches them on the GPU through the C ABI of
``libhnsw_b200.so`` with the reference's exact results.
"""

from .index import HNSWIndex, IndexStats
from .quantization import QuantizedIndex, ScalarQuantizer

__all__ = ["HNSWIndex", "IndexStats", "QuantizedIndex", "ScalarQuantizer"]

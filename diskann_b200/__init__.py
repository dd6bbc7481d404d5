"""B200-native batched greedy graph search (Vamana beam search) behind a C ABI.

The compute path is ``_lib/libdiskann_b200.so`` (hand-written sm_100a CUDA kernels; see
include/diskann_b200.h).  This package is the host-side mirror of the reference's search
surface (``Knn``, ``Metric``, strategies, ``DiskANNIndex.search``) plus the data tooling on
either side of the path (synthetic inputs, graph construction, file formats).
"""

from .index import (  # noqa: F401
    ANNError,
    BF16,
    DiskANNIndex,
    FP8,
    FullPrecision,
    GpuProvider,
    Hybrid,
    Knn,
    KnnSearchError,
    Metric,
    PQData,
    Quantized,
    InmemProvider,
    PagedSearch,
    Range,
    STATS_DTYPE,
    SearchServer,
    Status,
)

__all__ = [
    "ANNError", "BF16", "DiskANNIndex", "FP8", "FullPrecision", "GpuProvider", "Hybrid", "Knn",
    "KnnSearchError", "Metric", "InmemProvider", "PQData", "PagedSearch", "Quantized", "Range", "STATS_DTYPE", "SearchServer", "Status",
]

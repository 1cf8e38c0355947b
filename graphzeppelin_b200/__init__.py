"""graphzeppelin_b200: B200-native (sm_100a) sketch ingest and Boruvka connected-components
query for dynamic graph streams, with the reference GraphZeppelin's CCSketchAlg /
GraphSketchDriver surface.

The compute path is libgz_b200.so (CUDA kernels + the C ABI of include/gz_b200.h); this package
is the host-side mirror of the reference interface over that ABI, plus stream I/O.
"""
from .cc import (CACHETREE, CONNECTIVITY, END_OF_STREAM, GUTTERTREE, KSPANNINGFORESTS, STANDALONE,
                 BadVertexError, BinaryFileStream, CCAlgConfiguration, CCSketchAlg,
                 ConnectedComponents, DriverConfiguration, DriverException, Edge, GraphSketchDriver,
                 GraphUpdate, GutterSystem, GZError, OutOfSamplesException, QueryCode,
                 SampleResult, SpanningForest, UpdateLockedException, UpdateType,
                 concat_pairing_fn, inv_concat_pairing_fn)
from .batch import BatchResult, CCSketchBatch
from .streams import RECORD_DTYPE, Stream, read_stream

__all__ = [n for n in dir() if not n.startswith("_")]
__version__ = "0.1.0"

"""ffdas_b200: B200-native delay-and-sum (das / das_sparse) behind the ffdas C-ABI.

Drop-in for the delay-and-sum call of BrainEchoLab/ffdas: same C entry points
(include/ffdas.h, libffdas_b200.so) and the same Python signatures
(`das(x, srcpos, dstpos, offsets, weights, *, srcdir, wavenum, algorithm,
use_fp16, channels_trailing, out)`, and the rank filter that follows it,
`truncate_rank(x, start, stop=None, *, out=None)`), with torch tensors or any DLPack CUDA
array.  The compute path is hand-written sm_100a CUDA; importing this package
loads the compiled library and fails if it is missing.
"""
from . import _lib
from ._lib import Algorithm, ComputeType, DataType, DasConfig, FFDASError
from .library import get_cuda_device, set_cuda_device, get_library_handle
from .das import das, das_from_host, das_sparse, sparse_select, DowncastWarning
from .timing import Timer
from .truncate_rank import truncate_rank

_lib.load()

__version__ = "0.1.0"

__all__ = [
    "das", "das_from_host", "das_sparse", "sparse_select", "truncate_rank", "Algorithm", "ComputeType", "DataType", "DasConfig", "FFDASError",
    "DowncastWarning", "get_cuda_device", "set_cuda_device", "get_library_handle", "Timer",
]

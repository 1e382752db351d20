"""LATEC on NVIDIA B200: error-bounded progressive compression with CUDA kernels.

Drop-in for the reference package's public API (``latec/__init__.py``):
``compress``, ``decompress``, ``InterpPredictor`` and the learned
``GNNCodec``, plus ``compress_many`` / ``decompress_many`` for lists of
tensors. The compute runs in ``liblatec_b200.so`` (sm_100a); there is no CPU
fallback.
"""

from .batch import autotune_many, compress_many, decompress_many
from .codec import compress, decompress
from .gnn_codec import GNNCodec, GNNCompressorCodec
from .predictor import InterpPredictor

__all__ = ["compress", "decompress", "compress_many", "decompress_many", "autotune_many",
           "InterpPredictor",
           "GNNCodec", "GNNCompressorCodec"]
__version__ = "0.1.0"

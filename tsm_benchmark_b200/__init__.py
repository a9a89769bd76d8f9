"""B200-native TSMTTSM library: C = A^T * B for tall-skinny row-major A, B.

The compute path is hand-written sm_100a CUDA in ``csrc/`` behind the C ABI
of ``include/tsm.h`` (built into ``libtsm_b200.so``); this package is its host
side: ctypes bindings, torch-tensor entry points, the variant generator and
the autotuner.
"""
from ._capi import TsmError, TsmLibraryError, variants  # noqa: F401
from .api import (block_orthogonalize, default_variant, fill_uniform, gram, tsmm, tsmttsm, tsmttsm_backward,  # noqa: F401
                  tsmttsm_split, workspace_status)
from .autograd import TSMTTSMFunction, gram_tn  # noqa: F401
from .batched import BatchedTSMTTSM  # noqa: F401

__version__ = "0.1.0"

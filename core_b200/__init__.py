"""B200-native (sm_100a) DCT+IRLS L1 2-D phase unwrapper.

Drop-in for insardev's `utils_unwrap2d.irls_unwrap_2d`
(insardev/insardev/utils_unwrap2d.py:1082).  The compute runs in
libunwrap_b200.so (hand-written CUDA kernels behind the C ABI in
include/unwrap_b200.h); PyTorch supplies device memory and the stream.
"""
from .irls import irls_unwrap_2d, irls_unwrap_2d_batch, resolve_device  # noqa: F401
from .adapters import unwrap2d_chunk  # noqa: F401
from .autodiff import irls_adjoint, irls_adjoint_batch, irls_unwrap_2d_diff  # noqa: F401
from .goldstein import goldstein  # noqa: F401
from .link import link_components, unwrap2d, unwrap2d_link  # noqa: F401

__all__ = ["irls_unwrap_2d", "irls_unwrap_2d_batch", "unwrap2d_chunk", "irls_unwrap_2d_diff", "irls_adjoint",
           "irls_adjoint_batch",
           "goldstein", "link_components", "unwrap2d", "unwrap2d_link"]

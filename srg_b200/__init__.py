"""srg_b200 -- B200 (sm_100a) time-domain backprojection for ASFHyP3/SRG.

The product is libsrg_bp.so (CUDA kernels + the C ABI of include/srg_bp.h);
this package builds it (``build``), binds it (``_lib``, ``api``) and makes
synthetic bursts for it (``scene``).
"""
from . import scene  # noqa: F401

__all__ = ["scene", "api", "build"]

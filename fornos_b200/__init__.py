"""B200-native (sm_100a) implementation of the Fornos texture-baking path.

The product is libfornos_b200.so (C ABI in include/fornos_gpu.h); this
package is its Python front-end.  See fornos_b200.api for the solver API.
"""
from . import workloads  # noqa: F401

__all__ = ["api", "workloads", "build"]

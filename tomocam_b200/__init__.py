"""tomocam_b200 -- B200 implementation of tomoCAM's MBIR path.

Drop-in for the reference package ``tomocam`` on its MBIR path
(``tomocam/__init__.py:4-7``): ``import tomocam_b200 as tomocam`` gives
``radon``, ``radon_adj`` and ``MBIR`` with the same signatures, backed by the
``cTomocam`` module (same names as ``src/pyTomocam.cpp``) and the CUDA
library ``libtomocam_b200.so``.
"""
from ._version import __version__
from .transform import radon, radon_adj
from .modeling import MBIR

__all__ = ["radon", "radon_adj", "MBIR", "__version__"]

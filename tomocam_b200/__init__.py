"""tomocam_b200 -- B200 implementation of tomoCAM's MBIR path.

Drop-in for the reference package ``tomocam`` on its MBIR path
(``tomocam/__init__.py:4-7``): ``import tomocam_b200 as tomocam`` gives
``radon``, ``radon_adj`` and ``MBIR`` with the same signatures, backed by the
``cTomocam`` module (same names as ``src/pyTomocam.cpp``) and the CUDA
library ``libtomocam_b200.so``.

The three names are resolved on first use, so that ``tomocam_b200.build``
can be imported (and run) before the compiled modules exist; using them in
an unbuilt tree raises ImportError.
"""
from ._version import __version__

__all__ = ["radon", "radon_adj", "MBIR", "__version__"]


def __getattr__(name):
    if name in ("radon", "radon_adj"):
        from . import transform
        return getattr(transform, name)
    if name == "MBIR":
        from .modeling import MBIR
        return MBIR
    raise AttributeError(f"module 'tomocam_b200' has no attribute {name!r}")

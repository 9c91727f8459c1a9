"""tomocam -- the reference package's import name, served by tomocam_b200.

Existing code that does ``import tomocam`` (``tomocam/__init__.py:4-7`` of the
reference: ``radon``, ``radon_adj``, ``MBIR``, and the submodules ``recon``,
``modeling``, ``transform``, ``gradients`` and the binding ``cTomocam``) runs
unchanged on the B200 implementation.  ``tomocam.autograd`` adds the
differentiable forms.
"""
import sys as _sys

from tomocam_b200 import __version__  # noqa: F401
from tomocam_b200._ext import cTomocam  # noqa: F401
from tomocam_b200.modeling import MBIR  # noqa: F401
from tomocam_b200.transform import radon, radon_adj  # noqa: F401

_sys.modules[__name__ + ".cTomocam"] = cTomocam

__all__ = ["radon", "radon_adj", "MBIR", "cTomocam", "__version__"]

"""tomocam.recon.MBIR (reference tomocam/recon.py:5-40)."""
from .modeling import MBIR  # noqa: F401

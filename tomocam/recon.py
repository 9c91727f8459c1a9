"""tomocam.recon, served by tomocam_b200.recon."""
from tomocam_b200.recon import *  # noqa: F401,F403

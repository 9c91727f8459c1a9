"""tomocam.transform, served by tomocam_b200.transform."""
from tomocam_b200.transform import *  # noqa: F401,F403

"""tomocam.modeling, served by tomocam_b200.modeling."""
from tomocam_b200.modeling import *  # noqa: F401,F403

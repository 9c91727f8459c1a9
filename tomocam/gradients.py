"""tomocam.gradients, served by tomocam_b200.gradients."""
from tomocam_b200.gradients import *  # noqa: F401,F403

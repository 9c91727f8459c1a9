"""tomocam.autograd, served by tomocam_b200.autograd."""
from tomocam_b200.autograd import *  # noqa: F401,F403

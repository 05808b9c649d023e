"""`import nricp_dp` for callers of the reference's extension module: the
B200 implementation of its route B / route C surface (nricp_b200.nricp_dp)."""

from nricp_b200 import nricp_dp as _impl
from nricp_b200.nricp_dp import *  # noqa: F401,F403
from nricp_b200.nricp_dp import __version__  # noqa: F401

__getattr__ = _impl.__getattr__  # names the reference has and this module does not, with the reason

"""nricp_b200: the non-rigid ICP wrapping path of PDE26jjk/nricp on B200.

``nricp_b200.nricp_dp`` is the drop-in for the reference's ``nricp_dp``
extension module (route B / route C); ``nricp_b200.synthetic`` generates the
seeded benchmark wraps; ``nricp_b200.serving`` runs the continuous-batching
request loop.  The CUDA library (libnricp_b200.so, sm_100a) does the work.
"""

__version__ = "0.1.0"

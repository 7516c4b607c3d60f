"""Field Engine on B200: the host side of the sm_100a law backend (libfe_b200.so, include/fe.h)."""
from ._lib import FeError, lib, last_error  # noqa: F401

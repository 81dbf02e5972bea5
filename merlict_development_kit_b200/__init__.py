"""B200-native photon propagation behind merlict's propagation entry point."""
from . import abi  # noqa: F401

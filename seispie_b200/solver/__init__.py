"""Solver plugins.  ``b200`` is the drop-in for seispie's ``fd2d``."""
from .b200 import b200, DeviceArray

__all__ = ["b200", "DeviceArray"]

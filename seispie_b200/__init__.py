"""seispie_b200: B200-native (sm_100a) FWI hot path of icui/seispie.

The package holds the host side of the drop-in solver plugin
(``seispie_b200.solver.b200``), the torch-owned device state
(``seispie_b200.engine``) and the C-ABI CUDA library that does all the
numerical work (``seispie_b200/csrc``, declared in include/seispie_b200.h).
"""
__version__ = "0.1.0"

"""lucky_droplets_b200: the forced pseudospectral DNS step with droplets of
Rajarshi-prime/lucky-droplets (forced-dns-sm.py + particles.py), rebuilt for one B200.

Host code in Python; every device operation is a hand-written sm_100a kernel in
liblucky_droplets.so, reached through the C ABI of include/ld.h (ctypes, see ``_lib``).
"""
from ._lib import LDError, LIB_PATH  # noqa: F401


def __getattr__(name):
    # lazy imports keep `import lucky_droplets_b200` free of torch/CUDA initialisation
    if name in ("Plan",):
        from .spectral import Plan
        return Plan
    if name in ("ForcedDNS", "Droplets", "BlowUpError"):
        from . import dns
        return getattr(dns, name)
    raise AttributeError(name)

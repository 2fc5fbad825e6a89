"""ldsc_b200 -- B200-native engine for the ldsc `l2` LD-score path.

The compute lives in ``libldsc_b200.so`` (CUDA for sm_100a, C ABI in
``include/ldsc_b200.h``); this package is its Python binding plus host-side
helpers (PLINK I/O, synthetic panels, output writers).
"""
from .plink import BimTable, parse_bim, parse_bim_text, count_fam, read_bed, write_plink  # noqa: F401

__all__ = ["api", "plink", "synth"]


def __getattr__(name):
    # the compute API loads the shared library lazily, and fails loudly if it is missing
    if name in ("api",):
        from . import api
        return api
    raise AttributeError(name)

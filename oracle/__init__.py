"""CPU oracle for the ldsc `l2` path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this package, and only as the checker or as the timed
CPU baseline.  The product (``ldsc_b200``) never imports it.
"""
from .oracle import (  # noqa: F401
    OracleL2Args,
    oracle_l2,
    block_lefts,
    countsketch_hash,
    wyrand_stream,
    scatter_column_f32,
    max_threads,
    oracle_snp_stats,
)

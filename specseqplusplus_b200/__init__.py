"""B200-native persistent-homology reduction engine with SpecSeq++ semantics.

The reduction runs in ``libsspp.so`` (hand-written CUDA for sm_100a behind the
C ABI of ``include/sspp.h``).  ``engine`` is the Python host mirror of that ABI
and of the reference's ``SpecSeqPlusPlus`` class; ``gen`` builds synthetic
filtered complexes.
"""
from .engine import (ASCII, BINARY, Engine, Params, SpecSeqPlusPlus, SsppError,  # noqa: F401
                     compute_persistence_pairs, load_library)

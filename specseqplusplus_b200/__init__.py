"""B200-native persistent-homology reduction engine with SpecSeq++ semantics.

The reduction runs in ``libsspp.so`` (hand-written CUDA for sm_100a behind the
C ABI of ``include/sspp.h``).  ``engine`` is the Python host mirror of that ABI
and of the reference's ``SpecSeqPlusPlus`` class, plus ``Server`` (the resident
request loop with continuous batching); ``gen`` builds synthetic filtered
complexes and ``workloads`` the batched and served request mixes.
"""
from .engine import (ASCII, BINARY, Engine, Params, Server, SpecSeqPlusPlus, SsppError,  # noqa: F401
                     compute_persistence_pairs, load_library)

"""B200-native persistent-homology reduction engine with SpecSeq++ semantics.

The reduction runs in ``libsspp.so`` (hand-written CUDA for sm_100a behind the
C ABI of ``include/sspp.h``).  ``engine`` is the Python host mirror of that ABI
and of the reference's ``SpecSeqPlusPlus`` class, plus ``Server`` (the resident
request loop with continuous batching); ``gen`` builds synthetic filtered
complexes and ``workloads`` the batched and served request mixes.
"""
import os

# CTA-tier launches of successive spectral-sequence steps run on separate
# streams; the driver maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware
# queues (8 by default) and launches on streams that share a queue wait for
# each other.  Ask for the maximum, 32, unless the caller chose a value; it
# applies to a CUDA context created after this import.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from .engine import (ASCII, BINARY, Engine, Params, Server, SpecSeqPlusPlus, SsppError,  # noqa: F401
                     compute_persistence_pairs, load_library)

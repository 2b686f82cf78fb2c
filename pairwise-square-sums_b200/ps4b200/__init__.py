"""B200 (sm_100a) search for sets of positive integers whose pairwise sums are all squares.

Host-side mirror of the reference census engine's interface (exhaustive/s4.c) over the C-ABI
of lib/libps4.so.  See ``search.Search``.
"""
from . import _abi
from .search import Ps4Error, RangeResult, Search

__all__ = ["Search", "RangeResult", "Ps4Error", "_abi"]

"""seticore-b200: a B200-native (sm_100a) dedoppler search with seticore's API.

The search runs in hand-written CUDA kernels (seticore_b200/csrc) behind a C ABI
(include/seticore_b200.h); this package is the Python host side of that ABI.
"""
from ._capi import NO_BEAM, DedopplerError  # noqa: F401
from .pool import SearchPool, SearchRequest  # noqa: F401
from .serving import SearchServer, run_load  # noqa: F401
from .dedoppler import (  # noqa: F401
    DedopplerHit,
    Dedopplerer,
    FilterbankBuffer,
    FilterbankMetadata,
    HitList,
    driftStepsLessThan,
    makeNoisyBuffer,
    roundUpToPowerOfTwo,
)

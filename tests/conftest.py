import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def rmb():
    import rmetis_b200
    rmetis_b200._lib.load()
    return rmetis_b200


def greedy_options(seed=1, ncuts=1, niter=10, ufactor=30, ctype=1, iptype=0):
    import numpy as np
    a = np.full(40, -1, dtype=np.int32)
    a[0] = 0            # PTYPE != -1: use the array
    a[1] = 0            # OBJTYPE cut
    a[2] = ctype        # CTYPE
    a[3] = iptype       # IPTYPE
    a[4] = 1            # RTYPE greedy
    a[5] = 0
    a[6] = niter
    a[7] = ncuts
    a[8] = seed
    a[9] = 0
    a[10] = 0
    a[11] = 0
    a[16] = ufactor
    a[17] = 0
    return a


def fm_options(seed=1, ncuts=1, niter=10, ufactor=30, ctype=1, iptype=0):
    """The option array of greedy_options with RTYPE = 0 (k-way FM)."""
    a = greedy_options(seed, ncuts, niter, ufactor, ctype, iptype)
    a[4] = 0
    return a

"""mochii_launch_records_noalloc: the launch-record hook for callers that
cannot allocate device memory at call time (their device memory belongs to
another allocator, or a memory limit makes cudaMalloc fail).  It stages the
records in the library's static device array instead of a cudaMallocAsync
buffer, so its output must equal the allocating entry point's, call after
call, while the array keeps the previous call's contents.

This file is named to be collected last: it must pass alone in a fresh
process and after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from mochii_b200 import MochiiError, Nebula, configs, parse_namelist
from mochii_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_RECORDS = 65536


def noalloc_records(neb, ip0, n):
    out = np.full((n, 8), np.nan)
    rc = neb.lib.mochii_launch_records_noalloc(neb.ctx, int(ip0), int(n), out.ctypes.data)
    if rc != _lib.OK:
        raise MochiiError(rc, (neb.lib.mochii_last_error(neb.ctx) or b"").decode())
    return out


def test_noalloc_records_equal_allocating_entry_point_on_consecutive_calls():
    nl = configs.stromgren64(nphotons=200000, n=32)
    neb = Nebula(parse_namelist(nl))
    # two calls in a row; the second is smaller and starts elsewhere, so
    # slots the first call filled and the second does not read stay stale
    for ip0, n in ((0, MAX_RECORDS), (123457, 5000)):
        got = noalloc_records(neb, ip0, n)
        ref = neb.launch_records(ip0, n)
        # same kernel, same inputs: identical records (the launch tolerance of
        # the parity tests is bit-exact energies and bins, 4e-16 on directions)
        assert np.array_equal(got, ref), (ip0, n)
    neb.close()


def test_noalloc_records_reject_sizes_beyond_the_static_array():
    neb = Nebula(parse_namelist(configs.stromgren64(nphotons=1000, n=8)))
    out = np.zeros((MAX_RECORDS + 1, 8))
    rc = neb.lib.mochii_launch_records_noalloc(neb.ctx, 0, MAX_RECORDS + 1, out.ctypes.data)
    assert rc == 1   # MOCHII_ERR_BAD_PARAM, refused on the host before any launch
    assert b"65536" in neb.lib.mochii_last_error(neb.ctx)
    neb.close()

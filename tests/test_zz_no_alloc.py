"""ppt_moments_noalloc (the bunch-moments entry point that allocates nothing)
against ppt_moments (the allocating one), called through the C ABI.

The no-alloc entry point is for callers that may not allocate device memory
while they run -- an application whose GPU memory is all owned by another
allocator's pool, or an analysis hook inside a latency-bound tracking loop
that must not let cudaMalloc/cudaFree synchronise the device.  Its scratch is
a static device array shared by every call, so the test makes two calls in a
row of different sizes and checks each against the allocating entry point.
This file is named to be collected last and passes alone or after the rest.
"""
import ctypes

import numpy as np
import pytest

from pypatools_b200 import _lib
from pypatools_b200.species import IonSpecies

pytestmark = pytest.mark.gpu


def _bunch(seed, n):
    rng = np.random.default_rng(seed)
    r = rng.normal(0.0, 1e-3, (n, 3))
    v = np.column_stack([rng.normal(0.0, 3e4, n), rng.normal(0.0, 3e4, n), rng.normal(1.38e7, 1e5, n)])
    return r, v


def test_noalloc_moments_match_allocating_entry_point(cuda):
    torch = cuda
    lib = _lib.load()
    stream = _lib.stream_handle()
    mass = IonSpecies("proton").mass_mev
    for seed, n in ((1, 100_000), (2, 4_097)):
        r, v = _bunch(seed, n)
        dr = torch.from_numpy(r).cuda()
        dv = torch.from_numpy(v).cuda()
        ref = torch.empty(_lib.MOMENTS_LEN, dtype=torch.float64, device="cuda")
        scratch = torch.empty(lib.ppt_moments_scratch_bytes(n), dtype=torch.uint8, device="cuda")
        _lib.check(lib.ppt_moments(n, dr.data_ptr(), dv.data_ptr(), mass, ref.data_ptr(), scratch.data_ptr(), stream))
        out = torch.empty(_lib.MOMENTS_LEN, dtype=torch.float64, device="cuda")
        _lib.check(lib.ppt_moments_noalloc(n, dr.data_ptr(), dv.data_ptr(), mass, out.data_ptr(), stream))
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=0.0)


def test_noalloc_moments_rejects_bad_sizes(cuda):
    lib = _lib.load()
    out = cuda.empty(_lib.MOMENTS_LEN, dtype=cuda.float64, device="cuda")
    assert lib.ppt_moments_noalloc(0, None, None, 1.0, out.data_ptr(), None) == -1
    assert b"n >= 1" in lib.ppt_last_error()
    assert lib.ppt_moments_noalloc((1 << 53) + 1, 1, 1, 1.0, out.data_ptr(), None) == -1
    assert b"2^53" in lib.ppt_last_error()

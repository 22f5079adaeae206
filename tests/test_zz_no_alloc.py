"""amg_restrict_raw_noalloc: the level-0 restriction for callers that may not allocate device
memory while they run (an application that hands out all device memory from its own pool, or
code running where an allocation would synchronise the device or fail).  It keeps its partial
sums in a fixed 4 MiB array that the library owns on every device, so the caller passes only
the test vectors, the sources and the output.

Checked through the C ABI against the context's restriction (amg_restrict, level 0) on two
calls in a row with different sources and source counts, so the second call runs over the
partial sums the first one left in the shared array, and then on a source count large enough
that the entry point takes fewer chunks per aggregate to fit its array.  Bar: 1e-13
relative, the bar of the other FP64 stencil-level parity tests.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _sources(nrhs, N, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((nrhs, N, 2)) + 1j * rng.standard_normal((nrhs, N, 2))).astype(np.complex128)


def test_restrict_noalloc_matches_context_restriction():
    import torch

    from amg_schwingermodel_b200 import AMGContext, _lib
    from amg_schwingermodel_b200.inputs import gauge_field

    # 128x128 lattice, 4x4 aggregates of 32x32 sites, 8 test vectors: 8 chunks per aggregate
    nx = nt = 128
    N = nx * nt
    with AMGContext(nx, nt, [[0, 4, 4, 8, 4, 4]], -0.1) as ctx:
        ctx.set_gauge(gauge_field(nx, nt, 4.0, 31))
        ctx.setup()
        W = ctx.test_vectors(0)
        c1 = ctx.info[1]
        bx, bt, ntest = c1["nx"], c1["nt"], ctx.info[0]["ntest"]
        # 3 and 2 sources, then 160: 160 x 16 aggregates x 16 values x 8 chunks exceeds the
        # 4 MiB array, so that call sums over fewer chunks
        cases = [_sources(nrhs, N, seed) for nrhs, seed in ((3, 41), (2, 42), (160, 43))]
        wants = [np.stack([ctx.restrict(0, v) for v in vs]) for vs in cases]

    lib = _lib.lib()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    Wd = torch.from_numpy(W).to(dev)
    for v, want in zip(cases, wants):
        nrhs = v.shape[0]
        vd = torch.from_numpy(v).to(dev)
        out = torch.full((nrhs, bx * bt, 2 * ntest), complex("nan"), dtype=torch.complex128, device=dev)
        torch.cuda.synchronize(dev)
        rc = lib.amg_restrict_raw_noalloc(C.c_void_p(Wd.data_ptr()), C.c_void_p(vd.data_ptr()),
                                          C.c_void_p(out.data_ptr()), nx, nt, bx, bt, ntest, nrhs,
                                          C.c_void_p(stream.cuda_stream))
        assert rc == _lib.AMG_OK, lib.amg_last_error()
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel(got, want.reshape(got.shape)) < TOL

    # a request whose partial sums cannot fit the 4 MiB array is refused before any launch
    big = (4 << 20) // (16 * bx * bt * 2 * ntest) + 1
    rc = lib.amg_restrict_raw_noalloc(C.c_void_p(Wd.data_ptr()), C.c_void_p(Wd.data_ptr()),
                                      C.c_void_p(Wd.data_ptr()), nx, nt, bx, bt, ntest, big,
                                      C.c_void_p(stream.cuda_stream))
    assert rc == _lib.AMG_ERR_INVALID
    assert b"4 MiB" in lib.amg_last_error()


def test_restrict_noalloc_few_test_vectors_many_sources():
    """2 test vectors and 128 sources: the tiled kernel's staging (268 KB) exceeds what one
    block may hold, so the call takes the untiled kernel and still equals the context's
    one-source restrictions."""
    import torch

    from amg_schwingermodel_b200 import AMGContext, _lib
    from amg_schwingermodel_b200.inputs import gauge_field

    nx = nt = 64
    N = nx * nt
    with AMGContext(nx, nt, [[0, 4, 4, 2, 4, 4]], -0.1) as ctx:
        ctx.set_gauge(gauge_field(nx, nt, 3.0, 33))
        ctx.setup()
        W = ctx.test_vectors(0)
        bx, bt, ntest = ctx.info[1]["nx"], ctx.info[1]["nt"], ctx.info[0]["ntest"]
        assert ntest == 2
        v = _sources(128, N, 44)
        want = np.stack([ctx.restrict(0, vi) for vi in v])

    lib = _lib.lib()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    Wd = torch.from_numpy(W).to(dev)
    vd = torch.from_numpy(v).to(dev)
    for _ in range(2):
        out = torch.full((128, bx * bt, 2 * ntest), complex("nan"), dtype=torch.complex128, device=dev)
        torch.cuda.synchronize(dev)
        rc = lib.amg_restrict_raw_noalloc(C.c_void_p(Wd.data_ptr()), C.c_void_p(vd.data_ptr()),
                                          C.c_void_p(out.data_ptr()), nx, nt, bx, bt, ntest, 128,
                                          C.c_void_p(stream.cuda_stream))
        assert rc == _lib.AMG_OK, lib.amg_last_error()
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel(got, want.reshape(got.shape)) < TOL

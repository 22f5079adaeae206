"""The bounded device waits report instead of hanging: amg_debug_dirac_wait_test runs the
bulk-copy D apply (k_dirac_tma) without issuing its copies, so the first mbarrier wait of
every CTA runs out after its poll limit with nothing in flight.  The call must return
AMG_ERR_DEVICE_WAIT, and the device must stay usable: the same buffers then go through the
normal D apply, which must match the restated D_phi (src/dirac_operator.cpp:3-54) to 1e-13,
and a second self-test reports again (the flag is cleared after each report)."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel
from oracle import restatement as R

pytestmark = pytest.mark.gpu


def test_bulk_copy_wait_timeout_is_reported_and_device_stays_usable():
    import torch

    from amg_schwingermodel_b200 import _lib, dirac_apply_raw
    from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor

    nx, nt, nrhs, m0 = 8, 256, 3, -0.1
    U = gauge_field(nx, nt, 3.0, 81)
    psi = gaussian_spinor(nx * nt, 2, 82, nrhs=nrhs)
    dev = torch.device("cuda:0")
    Ud = torch.from_numpy(U.view(np.float64).copy()).to(dev)
    a = torch.from_numpy(psi.view(np.float64).copy()).to(dev)
    b = torch.zeros_like(a)
    lib = _lib.lib()

    for _ in range(2):
        rc = lib.amg_debug_dirac_wait_test(C.c_void_p(Ud.data_ptr()), C.c_void_p(a.data_ptr()),
                                           C.c_void_p(b.data_ptr()), nx, nt, nrhs)
        assert rc == _lib.AMG_ERR_DEVICE_WAIT, (rc, lib.amg_last_error())
        assert b"self-test" in lib.amg_last_error()

    torch.cuda.synchronize(dev)
    dirac_apply_raw(Ud.data_ptr(), a.data_ptr(), b.data_ptr(), nx, nt, nrhs, m0)
    torch.cuda.synchronize(dev)
    got = b.cpu().numpy().view(np.complex128).reshape(nrhs, nx * nt, 2)
    want = np.stack([R.d_phi(U, psi[r], m0, nx, nt) for r in range(nrhs)])
    assert rel(got, want) < 1e-13

    # a lattice the kernel does not take is refused before any launch
    rc = lib.amg_debug_dirac_wait_test(C.c_void_p(Ud.data_ptr()), C.c_void_p(a.data_ptr()),
                                       C.c_void_p(b.data_ptr()), nx, 128, nrhs)
    assert rc == _lib.AMG_ERR_INVALID

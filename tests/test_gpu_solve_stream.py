"""amg_solve_stream: batches of host-resident sources solved one after another, their copies
on a second stream through two device slots.  Every batch's solution and solve record must
equal amg_solve's on the same sources (the same kernels on the same data: bit for bit), for
one, two and five batches, from page-locked and from pageable host arrays, in the FP64 and
the mixed form; bad arguments are rejected."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROWS = [[0, 4, 4, 8, 4, 4], [1, 2, 2, 8, 2, 2]]


def make(prec):
    from amg_schwingermodel_b200 import AMGContext
    from amg_schwingermodel_b200.inputs import gauge_field
    ctx = AMGContext(64, 64, ROWS, -0.1, precision=prec, max_rhs=3)
    ctx.set_gauge(gauge_field(64, 64, 3.0, 17))
    ctx.setup()
    return ctx


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("nbatch", [1, 2, 5])
@pytest.mark.parametrize("pinned", [True, False])
def test_stream_batches_equal_single_solves(prec, nbatch, pinned):
    import torch
    from amg_schwingermodel_b200.inputs import gaussian_spinor
    R, N = 3, 64 * 64
    with make(prec) as ctx:
        bs = [gaussian_spinor(N, 2, 100 + i, nrhs=R) for i in range(nbatch)]
        want = [ctx.solve(b) for b in bs]
        bt = [torch.from_numpy(b.view(np.float64).copy()) for b in bs]
        xt = [torch.zeros_like(t) for t in bt]
        if pinned:
            bt = [t.pin_memory() for t in bt]
            xt = [t.pin_memory() for t in xt]
        infos = ctx.solve_stream_ptrs([t.data_ptr() for t in bt], [t.data_ptr() for t in xt], R)
        for i in range(nbatch):
            x = xt[i].numpy().view(np.complex128).reshape(R, N, 2)
            np.testing.assert_array_equal(x, want[i][0])
            assert [d["iterations"] for d in infos[i]] == [d["iterations"] for d in want[i][1]]
            assert all(d["converged"] and d["rel_residual"] < 1e-10 for d in infos[i])


def test_stream_rejects_bad_arguments():
    from amg_schwingermodel_b200._lib import AmgError
    with make(1) as ctx:
        with pytest.raises(ValueError):
            ctx.solve_stream_ptrs([], [], 1)
        with pytest.raises(AmgError):
            ctx.solve_stream_ptrs([0], [0], 1)

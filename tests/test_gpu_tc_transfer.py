"""The mixed form's level-0 transfers (amg_restrict0_mixed_dev / amg_prolong0_mixed_dev): the
tensor-core kernels (tcgen05, TF32 inputs, FP32 accumulation; csrc/tc_transfer.cuh) and the
CUDA-core kernels they replace (AMG_TC_TRANSFER=0), against numpy restrictions and
prolongations (Level::Pt_v / P_v, src/level.cpp:182-237) built from the same BF16 test
vectors and FP32 sources.

Bars: the CUDA-core kernels multiply in FP32, 1e-5 relative; the tensor cores read their
inputs as TF32 (10 mantissa bits), 2e-3 relative.  Shapes: 12 and 20 test vectors (64- and
128-row accumulators), 1 to 40 sources (the source count padded inside), aggregation
blocks of 32x32 and 16x32 sites, and 8x8-site blocks, whose 8-site rows the tensor-core
kernels do not tile (the CUDA-core kernels run).  Each configuration runs in its own process (the kernel
choice is read from the environment once per process).
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import ctypes as C, json, sys
sys.path.insert(0, {root!r})
import numpy as np, torch
from amg_schwingermodel_b200 import AMGContext, _lib
from amg_schwingermodel_b200.inputs import gauge_field

def bf16(x):
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    b = (b + np.uint32(0x7FFF) + ((b >> 16) & 1)) & np.uint32(0xFFFF0000)
    return b.view(np.float32)

out = []
dev = torch.device("cuda:0")
for nx, nt, rows, nrhs in {cases!r}:
    with AMGContext(nx, nt, rows, -0.05, precision=1, max_rhs=max(nrhs, 1)) as ctx:
        ctx.set_gauge(gauge_field(nx, nt, 3.0, 5))
        ctx.setup()
        W = ctx.test_vectors(0)                       # FP64 master copy [ntest][N][2]
        ntest = W.shape[0]
        Wb = bf16(W.view(np.float64).astype(np.float32)).astype(np.float64).view(np.complex128)
        bx, bt = rows[0][1], rows[0][2]
        xe, te, N, nblk = nx // bx, nt // bt, nx * nt, bx * bt
        blk = ((np.arange(N) // nt) // xe) * bt + (np.arange(N) % nt) // te
        rng = np.random.default_rng(nrhs)
        v = (rng.standard_normal((nrhs, N, 2)) + 1j * rng.standard_normal((nrhs, N, 2))).astype(np.complex64)
        vc = (rng.standard_normal((nrhs, nblk, 2 * ntest)) + 1j * rng.standard_normal((nrhs, nblk, 2 * ntest))).astype(np.complex64)
        psi0 = (rng.standard_normal((nrhs, N, 2)) + 1j * rng.standard_normal((nrhs, N, 2))).astype(np.complex64)
        # numpy: out[r][b][2k+s] = sum over n in b of conj(W[k][n][s]) v[r][n][s];
        # psi[r][n][s] += sum over k of W[k][n][s] vc[r][b(n)][2k+s]
        want_r = np.zeros((nrhs, nblk, 2 * ntest), np.complex128)
        for k in range(ntest):
            for s in range(2):
                prod = np.conj(Wb[k, :, s])[None, :] * v[:, :, s].astype(np.complex128)
                for b in range(nblk):
                    want_r[:, b, 2 * k + s] = prod[:, blk == b].sum(axis=1)
        want_p = psi0.astype(np.complex128).copy()
        for k in range(ntest):
            for s in range(2):
                want_p[:, :, s] += Wb[k, :, s][None, :] * vc[:, blk, 2 * k + s].astype(np.complex128)
        lib = _lib.lib()
        vd = torch.from_numpy(v).to(dev)
        rd = torch.full((nrhs, nblk, 2 * ntest), complex("nan"), dtype=torch.complex64, device=dev)
        torch.cuda.synchronize()
        rc = lib.amg_restrict0_mixed_dev(ctx._h, C.c_void_p(vd.data_ptr()), C.c_void_p(rd.data_ptr()), nrhs)
        assert rc == 0, lib.amg_last_error()
        got_r = rd.cpu().numpy()
        vcd = torch.from_numpy(vc).to(dev)
        pd = torch.from_numpy(psi0).to(dev)
        rc = lib.amg_prolong0_mixed_dev(ctx._h, C.c_void_p(vcd.data_ptr()), C.c_void_p(pd.data_ptr()), nrhs)
        assert rc == 0, lib.amg_last_error()
        got_p = pd.cpu().numpy()
        err_r = float(np.linalg.norm(got_r - want_r) / np.linalg.norm(want_r))
        err_p = float(np.linalg.norm(got_p - want_p) / np.linalg.norm(want_p - psi0))
        out.append(dict(nx=nx, rows=rows, nrhs=nrhs, err_r=err_r, err_p=err_p,
                        finite=bool(np.isfinite(got_r).all() and np.isfinite(got_p).all())))
print("RESULT" + json.dumps(out))
"""

CASES = [(128, 128, [[0, 4, 4, 12, 4, 4]], 32), (128, 128, [[0, 4, 4, 12, 4, 4]], 1),
         (128, 128, [[0, 4, 4, 20, 4, 4]], 5), (64, 128, [[0, 4, 4, 12, 2, 4], [1, 2, 2, 8, 2, 2]], 40),
         (64, 64, [[0, 2, 2, 16, 2, 2]], 17), (64, 64, [[0, 8, 8, 12, 2, 2]], 9)]


@pytest.mark.parametrize("tc", [1, 0])
def test_mixed_transfers_match_numpy(tc):
    env = dict(os.environ, AMG_TC_TRANSFER=str(tc))
    code = SCRIPT.format(root=str(ROOT), cases=CASES)
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    res = json.loads(p.stdout.split("RESULT", 1)[1])
    bar = 2e-3 if tc else 1e-5
    for r in res:
        assert r["finite"], r
        assert r["err_r"] < bar, r
        assert r["err_p"] < bar, r

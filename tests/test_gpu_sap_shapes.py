"""The FP32 fine SAP kernels on block shapes the golden fixtures do not have: blocks that
span the whole lattice in t or in x (so the block operator wraps around periodically inside
the block), 128- and 256-site blocks (one and two warps, four sites per thread), and blocks
whose t extent is not a multiple of the sites a thread owns (the dispatcher falls back to
the lean kernel).  Each shape is solved in mixed precision (FP32 cycle inside the FP64 outer
FGMRES) with the paired MGS kernel, the paired classical Gram-Schmidt kernel and the
16-bit-basis kernel with an FP16 and a BF16 basis (which takes the 256- and 512-site
blocks, the wrap-around ones included, and hands the others to the paired kernel), and
compared with the FP64 solve on the same context, whose parity with the reference the
fixture tests pin.
Bars: FP64 true residual <= 1e-10 for both, mixed x within 1e-8 of the FP64 x, and at most
one outer iteration more than the FP64 solve."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

# (lattice, rows): fine SAP blocks of 16x32 sites on a 32x32 lattice (t wrap inside the
# block), 32x16 (x wrap), 8x16 (128 sites), 16x16 (256 sites) and 64x2 (t extent 2: lean
# fallback)
SHAPES = {
    "t_wrap_16x32": (32, [[0, 4, 4, 8, 2, 1], [1, 2, 2, 8, 2, 2]]),
    "x_wrap_32x16": (32, [[0, 4, 4, 8, 1, 2], [1, 2, 2, 8, 2, 2]]),
    "blk_8x16": (64, [[0, 8, 8, 8, 8, 4], [1, 4, 4, 8, 2, 2]]),
    "blk_16x16": (64, [[0, 8, 8, 8, 4, 4], [1, 4, 4, 8, 2, 2]]),
    "blk_64x2": (64, [[0, 8, 8, 8, 1, 32], [1, 4, 4, 8, 2, 2]]),
}

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
from conftest import rel
from oracle import restatement as R
from amg_schwingermodel_b200 import AMGContext
from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
shapes = {shapes!r}
out = {{}}
for name, (ns, rows) in shapes.items():
    U = gauge_field(ns, ns, 3.0, 41)
    b = gaussian_spinor(ns * ns, 2, 42)
    res = {{}}
    for prec in (0, 1):
        ctx = AMGContext(ns, ns, rows, -0.1, precision=prec, autotune=0)
        ctx.set_gauge(U)
        ctx.setup()
        x, info = ctx.solve(b)
        res[prec] = (x, info[0]["iterations"], info[0]["rel_residual"])
        ctx.close()
    true_res = R.true_residual(U, res[1][0], b, -0.1, ns, ns)
    out[name] = dict(it64=res[0][1], it32=res[1][1], res64=res[0][2], res32=res[1][2], true32=true_res,
                     err=rel(res[1][0], res[0][0]))
print("RESULT" + json.dumps(out))
"""


@pytest.mark.parametrize("sap", ["paired", "cgs", "half", "bf16"])
def test_fp32_sap_block_shapes(sap):
    env = dict(os.environ, AMG_SAP_KERNEL=sap)
    code = SCRIPT.format(root=str(ROOT), tests=str(ROOT / "tests"), shapes=SHAPES)
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    res = json.loads(p.stdout.split("RESULT", 1)[1])
    assert set(res) == set(SHAPES)
    for name, r in res.items():
        assert r["res64"] <= 1e-10 and r["res32"] <= 1e-10, (name, r)
        assert r["true32"] <= 1e-10, (name, r)
        assert r["it32"] <= r["it64"] + 1, (name, r)
        assert r["err"] < 1e-8, (name, r)

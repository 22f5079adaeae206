"""The 16-bit-basis fine SAP kernel (k_sap0_h, csrc/sap_h.cuh; AMG_SAP_KERNEL=half for the
FP16 basis, =bf16 for the BF16 basis) inside the mixed-precision solve, against complete
solves of the reference (tests/golden/solve*.npz) on the workloads whose SAP blocks are
32x32 sites: 128^2 (beta 2), 256^2 (beta 3), 512^2 (beta 4) and the 1024^2 benchmark rows.

The kernel runs the reference's block GMRES(5) x 5 restarts (src/sap.cpp:44-62,
include/sap.h:27-47) in FP32 with the Krylov basis stored in 16 bits, so the smoother's output
moves by about that rounding and the outer FGMRES sees a slightly different
preconditioner.  Bars, as for every mixed solve: at most one outer iteration more than the
reference, x within 1e-8 of the reference on the fixture's sample, FP64 true residual
<= 1e-10.  The same solves with the FP32-basis kernel (AMG_SAP_KERNEL=paired) run beside
them: their outer residual histories must differ after the first preconditioner application
(the 16-bit kernel ran) by less than 10 % (it is the same smoother).  Each kernel choice runs in
its own process (the choice is read from the environment once per process).
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

NAMES = ["solve128_l3_b2", "solve256_l3_b3", "solve512_l3_b4", "solve1024_l4"]

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
import numpy as np
from conftest import load_golden, rel
from amg_schwingermodel_b200 import AMGContext
from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor

out = {{}}
for name in {names!r}:
    g = load_golden(name)
    m, idx = g["meta"], g["sites"]
    job = m["job"]
    U = gauge_field(m["ns"], m["nt"], m["beta"], m["seed"])
    b = gaussian_spinor(m["ns"] * m["nt"], 2, m["seed"] + 1000)
    with AMGContext(m["ns"], m["nt"], m["rows"], m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"],
                    nit=job["nit"], sap_tv_iters=job["sap_tv_iters"], precision=1) as ctx:
        ctx.set_gauge(U)
        ctx.setup()
        x, info = ctx.solve(b)
        hist = ctx.residual_history()
    out[name] = dict(iterations=info[0]["iterations"], ref_iterations=int(m["iterations"]),
                     converged=bool(info[0]["converged"]), resid=float(info[0]["rel_residual"]),
                     err=float(rel(x[idx], g["x_sample"])), hist=[float(h) for h in hist])
print("RESULT" + json.dumps(out))
"""


def run(kernel):
    env = dict(os.environ, AMG_SAP_KERNEL=kernel)
    code = SCRIPT.format(root=str(ROOT), tests=str(ROOT / "tests"), names=NAMES)
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.split("RESULT", 1)[1])


@pytest.fixture(scope="module")
def paired():
    return run("paired")


@pytest.mark.parametrize("kernel", ["half", "bf16"])
def test_sap_16bit_basis_solves_match_reference(kernel, paired):
    half = run(kernel)
    for name in NAMES:
        h, p = half[name], paired[name]
        print(f"{name}: {kernel} basis {h['iterations']} iterations, FP32 basis {p['iterations']}, reference "
              f"{h['ref_iterations']}; |x - x_ref|/|x_ref| {h['err']:.2e}; residual {h['resid']:.2e}")
        assert h["iterations"] <= h["ref_iterations"] + 1, h
        assert h["converged"] and h["resid"] < 1e-10, h
        assert h["err"] < 1e-8, h
        d = abs(h["hist"][1] / p["hist"][1] - 1)
        assert 0 < d < 0.1, (name, h["hist"][:3], p["hist"][:3])

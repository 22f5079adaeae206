"""The alternative kernel paths give the reference's results too: the generic and the lean
fine-level SAP block solvers, and the coarse engine on one CTA or on thread-block clusters
of 4 and 16 CTAs, in FP64; and in the mixed form (FP32 cycle inside the FP64 outer
FGMRES) the paired-FP32 MGS SAP kernel (default) with four or two sites per thread, with
its residual as a launch of its own (default) or formed inside the block solves
(AMG_SAP_FUSE=1), the paired kernel with classical Gram-Schmidt, the
communication-avoiding FP32 kernel, the lean kernel, and the 16-bit-basis kernel with an
FP16 and a BF16 basis (on the 512- and 1024-site blocks of c64_l2_sap512 and
c64_l3_sap1024; the other fixtures' blocks go to the paired kernel).
Each variant runs in its own process (the choice is read from the environment once per
process).  Mixed-precision bars: FP64 true residual <= 1e-10, x within 1e-8 of the
reference's, at most one outer iteration more than the reference."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
from conftest import load_golden, rel
from oracle import restatement as R
from amg_schwingermodel_b200 import AMGContext
out = {{}}
for name in ("c32_l3_k", "c64_l4_k", "c64_l2_k", "c64_l3_sap1024", "c64_l2_sap512"):
    g = load_golden(name); m = g["meta"]; job = m["job"]
    ctx = AMGContext(m["ns"], m["nt"], m["rows"], m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"],
                     nit=job["nit"], sap_tv_iters=job["sap_tv_iters"], max_rhs=3, precision={prec})
    ctx.set_gauge(g["gauge"])
    for l, W in enumerate(R.reference_initial_test_vectors(R.read_parameters(m["ns"], m["nt"], m["rows"]))):
        ctx.set_initial_test_vectors(l, W)
    ctx.setup()
    x, info = ctx.solve(g["rhs"])
    # three sources at once: each must equal its single-source solve
    b3 = np.stack([g["rhs"], g["probe_l0"], g["rhs"] * (1 + 2j)])
    x3, info3 = ctx.solve(b3)
    xs = [ctx.solve(b3[i])[0] for i in range(3)]
    out[name] = dict(it=info[0]["iterations"], ref_it=m["iterations"], err=rel(x, g["x"]),
                     batch_err=max(rel(x3[i], xs[i]) for i in range(3)),
                     batch_it=[i["iterations"] for i in info3], res=max(i["rel_residual"] for i in info3))
    ctx.close()
print("RESULT" + json.dumps(out))
"""


@pytest.mark.parametrize("sap,cluster,prec", [
    ("generic", "1", 0), ("lean", "1", 0), ("lean", "4", 0), ("lean", "16", 0),
    ("ca", "16", 1), ("ca", "1", 1), ("paired", "16", 1), ("paired2", "16", 1), ("lean", "16", 1),
    ("paired", "4", 1), ("cgs", "16", 1), ("cgs", "1", 1), ("paired_fuse", "16", 1), ("half", "16", 1),
    ("bf16", "4", 1)])
def test_variant_matches_reference(sap, cluster, prec):
    env = dict(os.environ, AMG_SAP_KERNEL=sap, AMG_ENGINE_CLUSTER=cluster)
    if sap == "paired2":
        env["AMG_SAP_SPT"] = "2"
    if sap == "paired_fuse":
        env.update(AMG_SAP_KERNEL="paired", AMG_SAP_FUSE="1")
    code = SCRIPT.format(root=str(ROOT), tests=str(ROOT / "tests"), prec=prec)
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    res = json.loads(p.stdout.split("RESULT", 1)[1])
    for name, r in res.items():
        if prec == 0:
            assert r["it"] == r["ref_it"], (name, r)
            assert r["batch_err"] < 1e-12, (name, r)
        else:
            assert r["it"] <= r["ref_it"] + 1, (name, r)
            assert r["batch_err"] < 1e-10, (name, r)
        assert r["err"] < 1e-8, (name, r)
        assert r["res"] < 1e-10, (name, r)

"""The preconditioner replayed from CUDA graphs gives the eager launches' results.

The cycle from the fine level is captured into a graph on a key's second use (mixed
precision: one graph per source count; FP64: one per Krylov slot) and replayed afterwards.
Three solves in a row run the eager, captured and replayed paths; each must equal the run
with graphs disabled (AMG_GRAPHS=0) exactly, in FP64 and in the mixed form, and the library
must report the same number of kernel launches either way."""
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
from conftest import load_golden
from amg_schwingermodel_b200 import AMGContext, launch_count
out = {{}}
for name in ("c32_l3_k", "c64_l3_sap1024"):
    g = load_golden(name); m = g["meta"]
    for prec in (0, 1):
        ctx = AMGContext(m["ns"], m["nt"], m["rows"], m["m0"], precision=prec, max_rhs=2, autotune=0)
        ctx.set_gauge(g["gauge"])
        ctx.setup()
        b = np.stack([g["rhs"], g["probe_l0"]])
        xs, its = [], []
        l0 = launch_count()
        for _ in range(3):
            x, info = ctx.solve(b)
            xs.append(np.asarray(x).view(np.float64).tolist())
            its.append([i["iterations"] for i in info])
        out[name + str(prec)] = dict(x=xs, it=its, launches=launch_count() - l0)
        ctx.close()
print("RESULT" + json.dumps(out))
"""


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    code = SCRIPT.format(root=str(ROOT), tests=str(ROOT / "tests"))
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.split("RESULT", 1)[1])


def test_graph_replay_equals_eager():
    eager = _run({"AMG_GRAPHS": "0"})
    graph = _run({})
    for key in eager:
        assert graph[key]["it"] == eager[key]["it"], key
        assert graph[key]["x"] == eager[key]["x"], key
        assert graph[key]["launches"] == eager[key]["launches"], key

"""The many-configuration solve's grouped SAP (amg_solve_many with AMG_SAP_GROUP on, the
default): contexts of different lattice sizes whose fine SAP takes the 16-bit-basis kernel
go through their cycles in lock step, and each colour's block solves of all of them are one
launch (k_sap0_h_group over a table of (lattice, block) columns).

Three configurations of the uneven batch (128^2 beta 2, 256^2 beta 3, 512^2 beta 4; fixtures
from the compiled reference, tests/golden/solve*.npz), 8 sources each with the fixture's
source first, solved once grouped and once with one SAP launch per lattice
(AMG_SAP_GROUP=0), each in its own process (the switch is read once per process).  Bars:
the reference's iteration count (at most one more, the mixed bar) and x within 1e-8 of
the reference on the fixture's sample in both runs, every source to FP64 residual <= 1e-10,
the two runs' solutions within 1e-8 of each other, and the grouped run issuing fewer
launches (its SAP launches serve all three lattices)."""
import json
import os
import subprocess
import sys

from conftest import ROOT

import pytest

pytestmark = pytest.mark.gpu

NAMES = ["solve128_l3_b2", "solve256_l3_b3", "solve512_l3_b4"]

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r})
sys.path.insert(0, {tests!r})
import numpy as np
from conftest import load_golden, rel
from amg_schwingermodel_b200 import AMGContext, solve_many, launch_count
from amg_schwingermodel_b200.inputs import gauge_field, gaussian_spinor
ctxs, bs, gs = [], [], []
for name in {names!r}:
    g = load_golden(name)
    m = g["meta"]; job = m["job"]
    N = m["ns"] * m["nt"]
    ctx = AMGContext(m["ns"], m["nt"], m["rows"], m["m0"], cycle=job["cycle"], nu1=job["nu1"], nu2=job["nu2"],
                     nit=job["nit"], sap_tv_iters=job["sap_tv_iters"], precision=1, max_rhs=8)
    ctx.set_gauge(gauge_field(m["ns"], m["nt"], m["beta"], m["seed"]))
    ctx.setup()
    b = gaussian_spinor(N, 2, m["seed"] + 1000)
    bs.append(np.concatenate([b[None], gaussian_spinor(N, 2, m["seed"] + 5000, nrhs=7)]))
    ctxs.append(ctx); gs.append(g)
solve_many(ctxs, bs)          # autotuning and first-use allocations
l0 = launch_count()
xs, infos = solve_many(ctxs, bs)
launches = launch_count() - l0
out = dict(launches=launches, runs=[])
for g, x, info in zip(gs, xs, infos):
    m = g["meta"]
    out["runs"].append(dict(it=info[0]["iterations"], ref_it=int(m["iterations"]), err=rel(x[0][g["sites"]], g["x_sample"]),
                            res=max(i["rel_residual"] for i in info), conv=all(i["converged"] for i in info)))
np.save({xfile!r}, np.concatenate([x.reshape(-1) for x in xs]))
for c in ctxs:
    c.close()
print("RESULT" + json.dumps(out))
"""


def run(group, tmp_path):
    env = dict(os.environ, AMG_SAP_GROUP="1" if group else "0")
    xfile = str(tmp_path / f"x{int(group)}.npy")
    code = SCRIPT.format(root=str(ROOT), tests=str(ROOT / "tests"), names=NAMES, xfile=xfile)
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    import numpy as np
    return json.loads(p.stdout.split("RESULT", 1)[1]), np.load(xfile)


def test_grouped_sap_matches_reference_and_per_lattice_launches(tmp_path):
    import numpy as np
    grouped, xg = run(True, tmp_path)
    single, xs = run(False, tmp_path)
    print(f"launches: grouped {grouped['launches']}, per lattice {single['launches']}")
    for name, rg, rs in zip(NAMES, grouped["runs"], single["runs"]):
        print(f"{name}: grouped {rg['it']} iterations, per lattice {rs['it']}, reference {rg['ref_it']}; "
              f"|x - x_ref|/|x_ref| {rg['err']:.2e} / {rs['err']:.2e}")
        for r in (rg, rs):
            assert r["it"] <= r["ref_it"] + 1, (name, r)
            assert r["err"] < 1e-8, (name, r)
            assert r["conv"] and r["res"] < 1e-10, (name, r)
    assert np.linalg.norm(xg - xs) <= 1e-8 * np.linalg.norm(xs)
    assert grouped["launches"] < single["launches"]

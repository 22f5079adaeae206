"""The C++ drop-in (include/amg_b200/amg_b200.hpp): a reference-style driver
(tests/cpp/dropin_main.cpp) written against the reference's class and function names --
readParameters, GaugeConf::read_conf, read_rhs, FGMRES_AMG::fgmres, D_phi, D_dagger_phi,
AlgebraicMG::setUpPhase / k_cycle / applyMultilevel, Level::D_operator / Pt_v / P_v,
SAP_level_l::SAP, GMRES_level_l::fgmres, FGMRES_SAP::fgmres, FGMRES_fine_level::fgmres,
conjugate_gradient, bi_cgstab -- built with g++ against libschwinger_amg.so.

CPU: the driver compiles and links for two lattice configurations.
GPU: it reproduces the golden fixtures (outputs of the reference itself on the same
inputs, passed in the reference's text formats): iteration count equal, x within 1e-8,
D and D^dagger within 1e-13, level operations within 1e-8; FGMRES_SAP and the
unpreconditioned FGMRES_fine_level within one iteration and 1e-8 of the restatement;
conjugate_gradient within two iterations and 1e-8, bi_cgstab within 1e-8 of the restatement
(itself equal to the reference's runs on the Krylov fixture).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import load_golden, rel
from oracle import restatement as R

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "amg_schwingermodel_b200"
CASES = ["c16_l2_k", "c32_l3_k"]


def build_driver(ns, nt, levels, out: Path) -> Path:
    exe = out / f"dropin_{ns}x{nt}_l{levels}"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-DNS={ns}", f"-DNT={nt}",
           f"-DLEVELS={levels}", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "dropin_main.cpp"),
           "-L", str(PKG), "-lschwinger_amg", f"-Wl,-rpath,{PKG}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def write_inputs(g, wd: Path):
    m = g["meta"]
    ns, nt = m["ns"], m["nt"]
    (wd / "parameters.dat").write_text("".join(" ".join(map(str, r)) + "\n" for r in m["rows"]))
    (wd / "m0.txt").write_text(repr(float(m["m0"])))

    def text(a, path):
        with open(path, "w") as f:
            for n in range(ns * nt):
                x, t = divmod(n, nt)
                for mu in range(2):
                    f.write(f"{x} {t} {mu} {a[n, mu].real:.17e} {a[n, mu].imag:.17e}\n")

    text(g["gauge"], wd / "gauge.ctxt")
    text(g["rhs"], wd / "rhs.rhs")
    for k in g:
        if k.startswith("probe_l"):
            np.ascontiguousarray(g[k], dtype=np.complex128).tofile(wd / f"{k}.bin")


@pytest.mark.parametrize("name", CASES)
def test_driver_compiles_and_links(name, tmp_path):
    m = load_golden(name)["meta"]
    assert build_driver(m["ns"], m["nt"], len(m["rows"]) + 1, tmp_path).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_driver_reproduces_reference(name, tmp_path):
    g = load_golden(name)
    m = g["meta"]
    L = len(m["rows"]) + 1
    exe = build_driver(m["ns"], m["nt"], L, tmp_path)
    write_inputs(g, tmp_path)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    res = dict(l.split() for l in (tmp_path / "results.txt").read_text().splitlines())

    def out(key, like):
        return np.fromfile(tmp_path / f"{key}.bin", dtype=np.complex128).reshape(np.shape(like))

    assert int(res["iterations"]) == m["iterations"]
    assert rel(out("x", g["x"]), g["x"]) < 1e-8
    # FGMRES_SAP (include/sap.h:194-225) on the reference's 4 x 4 SAP blocks, against the
    # restatement (itself equal to the reference's own FGMRES_SAP runs): within one outer iteration
    rows4 = [list(r) for r in m["rows"]]
    rows4[0][4] = rows4[0][5] = 4
    x_ref, it_ref = R.AMG(g["gauge"], m["ns"], m["nt"], rows4, R.SolverParams(m0=m["m0"])).solve_sap(g["rhs"])
    assert abs(int(res["sap_solver_iterations"]) - it_ref) <= 1, (res["sap_solver_iterations"], it_ref)
    assert rel(out("x_sap", x_ref), x_ref) < 1e-8
    ns, nt, m0 = m["ns"], m["nt"], m["m0"]
    x_g, it_g = R.gmres_fine(g["gauge"], g["rhs"], np.zeros_like(g["rhs"]), m0, ns, nt)
    assert abs(int(res["gmres_iterations"]) - it_g) <= 1, (res["gmres_iterations"], it_g)
    assert rel(out("x_gmres", x_g), x_g) < 1e-8
    x_c, it_c, _ = R.cg_normal(g["gauge"], g["rhs"], m0, ns, nt)
    assert abs(int(res["cg_iterations"]) - it_c) <= 2, (res["cg_iterations"], it_c)
    assert rel(out("x_cg", x_c), x_c) < 1e-8
    x_b, _, _ = R.bicgstab(g["gauge"], g["rhs"], np.zeros_like(g["rhs"]), m0, ns, nt)
    assert rel(out("x_bicg", x_b), x_b) < 1e-8
    assert rel(out("dphi", g["dphi"]), g["dphi"]) < 1e-13
    assert rel(out("ddagphi", g["ddagphi"]), g["ddagphi"]) < 1e-13
    assert rel(out("dop_l0", g["dop_l0"]), g["dop_l0"]) < 1e-13
    for k in ("dop_l1", "pt_l0", "ppt_l0", "sap_l0", f"gmres_l{L - 1}", "cycle0_rhs"):
        assert rel(out(k, g[k]), g[k]) < 1e-8, k
    assert int(res["sap_ret_l0"]) == m["sap_ret"]["0"]
    assert float(res["multilevel_rel_residual"]) < 1e-10
    # the residual file the reference writes with save_res (src/fgmres.cpp:70-79)
    hist = np.loadtxt(tmp_path / f"Residuals_FGMRES_{m['ns']}x{m['nt']}_Levels{L}_Kcycle.res")
    assert rel(hist[:, 1], g["residual_history"]) < 1e-6

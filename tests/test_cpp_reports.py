"""The reference's text outputs and experiment reports in the C++ adapter
(include/amg_b200/amg_b200.hpp): printParameters, save_vec, save_rhs, random_rhs and
saveParameters (src/variables.cpp:101-290), which the reference's main and script.sh workflow
write (metadata_*.dat, results_*.out).

tests/cpp/reports_main.cpp is built against the adapter and run; random_rhs must draw the
reference's mt19937 stream (the restatement's ReferenceUniform, itself pinned to the
reference's draws), save_rhs must round-trip, and the reports must carry the values given.
Where the reference's sources and the oracle's objects for 16x16 / 2 levels are present, the
same program is also built against the reference's own headers and objects, and every file
and the banner must be byte-identical.  No GPU is used.
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import ref_runner
from oracle import restatement as R

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "amg_schwingermodel_b200"
SRC = ROOT / "tests" / "cpp" / "reports_main.cpp"
NS = NT = 16
ROWS = "0 4 4 4 2 2\n"
FILES = ["vec.txt", "rhs1.txt", "rhs2.txt", "metadata_16x16_Levels2_Kcycle.dat", "results_16x16_Levels2_Kcycle.out"]


def run(exe: Path, wd: Path) -> str:
    wd.mkdir(parents=True, exist_ok=True)
    (wd / "parameters.dat").write_text(ROWS)
    p = subprocess.run([str(exe), str(wd)], cwd=str(wd), capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    return p.stdout.replace(str(wd), "<wd>")


@pytest.fixture(scope="module")
def adapter_run(tmp_path_factory):
    if not (PKG / "libschwinger_amg.so").exists():
        pytest.skip("libschwinger_amg.so not built")
    d = tmp_path_factory.mktemp("reports")
    exe = d / "reports_adapter"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-DNS={NS}", f"-DNT={NT}", "-DLEVELS=2",
           "-I", str(ROOT / "include"), str(SRC), "-L", str(PKG), "-lschwinger_amg", f"-Wl,-rpath,{PKG}", "-o",
           str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    wd = d / "out"
    return run(exe, wd), wd


def read_rhs_text(path: Path) -> np.ndarray:
    a = np.loadtxt(path)
    v = np.zeros((NS * NT, 2), dtype=np.complex128)
    n = (a[:, 0] * NT + a[:, 1]).astype(int)
    v[n, a[:, 2].astype(int)] = a[:, 3] + 1j * a[:, 4]
    return v


def test_adapter_reports(adapter_run):
    out, wd = adapter_run
    assert "| Nx = 16 Nt = 16" in out and "| Bare mass parameter m0 = -0.25" in out
    assert "Each block has 128 variables" in out
    # random_rhs: one generator seeded on the first call, uniform(-1, 1) parts
    u = R.ReferenceUniform(7).complex(4 * NS * NT).reshape(2, NS * NT, 2)
    np.testing.assert_array_equal(read_rhs_text(wd / "rhs1.txt"), u[0])
    np.testing.assert_array_equal(read_rhs_text(wd / "rhs2.txt"), u[1])
    vec = np.loadtxt(wd / "vec.txt")
    np.testing.assert_array_equal(vec[:, 1], [1.0, -2.5e-11, 3.0e7])
    meta = (wd / "metadata_16x16_Levels2_Kcycle.dat").read_text().split("\n")
    assert meta[0] == "#level, blocks_x, blocks_t, Ntest, SAP_blocks_x, SAP_blocks_t"
    assert meta[1].split() == ["0", "4", "4", "4", "2", "2"]
    assert meta[-2] == "17"
    res = np.loadtxt(wd / "results_16x16_Levels2_Kcycle.out")
    np.testing.assert_array_equal(res, [[0, 5.0, 0.5, 1.5, 0.1], [2, 6.5, 0.25, 2.5e-3, 0.2],
                                        [4, 7.25, 0.125, 3.0, 0.3]])


def test_adapter_reports_equal_reference_bytes(adapter_run, tmp_path):
    refdir = Path(ref_runner.DEFAULT_REFDIR)
    obj = ref_runner.REF_DIR / "obj_16x16_l2"
    if not (refdir / "src" / "variables.cpp").exists():
        pytest.skip("reference sources not present")
    ref_runner.build(NS, NT, 2)
    objs = sorted(str(p) for p in obj.glob("*.o") if p.name != "ref_harness.o")
    exe = tmp_path / "reports_reference"
    cmd = ["g++", "-std=c++20", "-O2", "-w", "-DAMG_REFERENCE_BUILD", "-include", str(obj / "oracle_config.h"),
           "-I", str(ROOT / "oracle" / "mpi_shim"), "-I", str(refdir / "include"), str(SRC), *objs, "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    ref_out = run(exe, tmp_path / "out")
    out, wd = adapter_run
    assert out == ref_out
    for f in FILES:
        assert (wd / f).read_bytes() == (tmp_path / "out" / f).read_bytes(), f

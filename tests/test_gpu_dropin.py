"""The reference's own driver programs on this library (drop-in check).

tests/dropin/Makefile compiles TESTS/Lap/LapPLanN.c and
TESTS0/Matvec/test1.c of the reference, unchanged, against include/pevsl.h
and links them to libpevsl_b200.so.  Running them must reproduce what the
reference prints for the same arguments: the README configuration's slices
and per-slice eigenvalue counts (equal to the analytic counts), and a
parallel-vs-sequential SpMV difference of 0.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import HERE, golden

pytestmark = pytest.mark.gpu
BUILD = os.path.join(HERE, "dropin", "_build")


def binary(name):
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        from checkers import REFERENCE_TREE
        if os.path.isdir(REFERENCE_TREE):
            subprocess.run(["make", "-s", "-C", os.path.join(HERE, "dropin"),
                            f"REFDIR={REFERENCE_TREE}"], check=True)
        else:
            pytest.fail(f"{path} missing: build tests/dropin where the reference tree exists")
    return path


def test_reference_laplacian_driver(gpu, tmp_path):
    exe = binary("LapPLanN")
    os.makedirs(tmp_path / "OUT")
    r = subprocess.run([exe, "-nx", "20", "-ny", "20", "-nz", "20", "-a", "0.6", "-b", "1.2",
                        "-nslices", "5", "-ngroups", "1"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = (tmp_path / "OUT" / "LapPLanN_G0.out").read_text()
    found = [(int(a), int(b)) for a, b in
             re.findall(r"\[Group 0\]: number of eigenvalues: (\d+), found: (\d+)", out)]
    assert found == [(21, 21), (24, 24), (27, 27), (19, 19), (27, 27)], found
    # slices: the reference's run with the same (glibc, srand(0)) stream
    block = out.split("SLICES FOUND")[1].split("=====\n")[1]
    sl = [tuple(float(x) for x in m) for m in
          re.findall(r"\s*\d+: \[\s*([-\d.e+]+)\s*,\s*([-\d.e+]+)\]", block)]
    assert len(sl) == 5
    g = golden("lap20_kpm.json")["cases"]["glibc"]["sli"]
    assert np.max(np.abs(np.array([s[0] for s in sl] + [sl[-1][1]]) - g)) <= 1e-12 * 1.2
    degs = [int(x) for x in re.findall(r"polynomial \[type \d\] deg (\d+)", out)]
    assert degs == [59, 73, 92, 96, 113]
    assert "KPMDOS: estimated eig count in interval: 118.37" in r.stdout


def test_reference_matvec_driver(gpu):
    """TESTS0/Matvec/test1.c writes x.data[i] from the host (managed memory)
    and compares pEVSL_ParcsrMatvec with the sequential pEVSL_Matvec."""
    exe = binary("MatvecTest1")
    r = subprocess.run([exe, "-nx", "16", "-ny", "16", "-nz", "16", "-ngroups", "1"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"Matvec \|\|SEQ-PARA\|\| = ([-\d.e+]+)", r.stdout)
    assert m, r.stdout
    assert float(m.group(1)) == 0.0


def _driver_report(out):
    """Slices, filter degrees, per-slice counts and listed eigenvalues of an
    OUT/LapPLanN_G0.out written by the reference's drivers."""
    sl = [tuple(float(x) for x in m) for m in
          re.findall(r"^\s*\d+: \[\s*([-\d.e+]+)\s*,\s*([-\d.e+]+)\]", out, re.M)]
    degs = [int(x) for x in re.findall(r"polynomial \[type \d\] deg (\d+)", out)]
    counts = [int(x) for x in re.findall(r"number of eigenvalues found: (\d+)", out)]
    lams = [float(x) for x in re.findall(r"^\s*(-?\d\.\d{15}e[-+]\d+)\s+\d\.\de[-+]\d+\s*$", out, re.M)]
    return sl, degs, counts, lams


def test_reference_matrix_market_driver(gpu, tmp_path):
    """TESTS/MM/MMPLanN.c with the reference's Matrix Market reader
    (TESTS/COMMON/parmm.c, mmio.c), unchanged, on this library: the
    reference's stiff1 matrix (MATRICES/A.mtx, n = 5795) and the first two
    intervals of TESTS/MM/matfile give the reference driver's slices,
    degrees and per-slice counts, and its listed eigenvalues to 1e-10
    (fixture: tests/golden/mm_stiff1.npz, from the reference build)."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import write_matfile, write_mm
    exe = binary("MMPLanN")
    g = np.load(os.path.join(HERE, "golden", "mm_stiff1.npz"))
    write_mm(tmp_path / "stiff1.mtx", int(g["n"]), g["i"], g["j"], g["v"])
    write_matfile(tmp_path / "matfile", "stiff1.mtx",
                  [(float(a), float(b), int(c)) for a, b, c in g["intervals"]])
    os.makedirs(tmp_path / "OUT")
    r = subprocess.run([exe, "-matfile", "matfile", "-ngroups", "1"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    got = _driver_report((tmp_path / "OUT" / "LapPLanN_G0.out").read_text())
    ref = _driver_report(str(g["output"]))
    assert got[2] == ref[2] == [45, 55, 61, 85, 66]
    assert got[1] == ref[1]
    assert len(got[0]) == len(ref[0]) == 5
    assert np.max(np.abs(np.array(got[0]) - np.array(ref[0]))) <= 1e-12 * 0.14
    assert len(got[3]) == len(ref[3]) > 0
    assert np.max(np.abs(np.array(got[3]) - ref[3]) / np.abs(ref[3])) <= 1e-10

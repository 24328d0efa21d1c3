"""The command-line driver (xmatch_b200/bin/xmatch, options and flow of
BoostXmatch.x): argument handling on the CPU, pair files against the oracle on
the GPU, whole and in segments (A segments resident in device memory, or held
in host memory and paged in per job, x rounds of B segments)."""
import os
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "xmatch_b200", "bin", "xmatch")
GOLD = os.path.join(ROOT, "tests", "golden")
ARCSEC = 1.0 / 3600.0


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=300)


def test_help_and_argument_errors(tmp_path):
    assert run("--help").returncode == 0
    assert run().returncode == 1                                   # two input files needed
    assert run("--bogus", "a", "b").returncode == 1
    assert run("-r", "-1", "a", "b").returncode == 1
    r = run(os.path.join(GOLD, "missing.idradec"), os.path.join(GOLD, "test.idradec"))
    assert r.returncode == 1 and "missing.idradec" in r.stderr
    d = tmp_path / "out"
    d.mkdir()
    r = run("-o", str(d), os.path.join(GOLD, "test.idradec"), os.path.join(GOLD, "test2.idradec"))
    assert r.returncode == 1 and "exists" in r.stderr


def read_pairs(outdir, rec):
    parts = []
    for f in sorted(os.listdir(outdir), key=int):
        b = np.fromfile(os.path.join(outdir, f), np.uint8)
        if rec == 16:
            parts.append(b.view(np.int64).reshape(-1, 2))
        else:
            parts.append(b.view(np.dtype([("a", "<i8"), ("b", "<i8"), ("d", "<f8")])))
    return parts


@pytest.mark.gpu
@pytest.mark.parametrize("numobj", [None, "300"])
def test_pairs_equal_the_oracle(tmp_path, numobj):
    # fileA = the 1,000-record fixture (resident), fileB = the 10,000-record one (looped)
    fa, fb = os.path.join(GOLD, "test2.idradec"), os.path.join(GOLD, "test.idradec")
    A, B = np.fromfile(fa, oracle.OBJ_DTYPE), np.fromfile(fb, oracle.OBJ_DTYPE)
    po, do, _ = oracle.xmatch(A, B, 5 * ARCSEC)
    order = np.lexsort((po[:, 1], po[:, 0]))
    po, do = po[order], do[order]
    extra = ["-n", numobj] if numobj else []
    out = tmp_path / "o16"
    r = run("-r", "5", "-o", str(out), *extra, fa, fb)
    assert r.returncode == 0, r.stderr
    p = np.concatenate(read_pairs(out, 16))
    p = p[np.lexsort((p[:, 1], p[:, 0]))]
    assert np.array_equal(p, po)
    out = tmp_path / "o24"
    r = run("-r", "5", "--dist", "-o", str(out), *extra, fa, fb)
    assert r.returncode == 0, r.stderr
    q = np.concatenate(read_pairs(out, 24))
    q = q[np.lexsort((q["b"], q["a"]))]
    assert np.array_equal(np.stack([q["a"], q["b"]], 1), po)
    assert np.max(np.abs(q["d"] - do), initial=0) <= 1e-12
    if numobj:
        assert len(os.listdir(out)) == (len(B) + 299) // 300       # one file per worker per round


@pytest.mark.gpu
def test_fileA_larger_than_the_device_budget(tmp_path):
    """fileA's segments exceed --resident-mb: they are held in pinned host memory
    and paged in one job at a time (the reference's host-resident segments,
    BoostXmatch.cpp:247-274); the pair files equal the oracle's."""
    fa, fb = os.path.join(GOLD, "test.idradec"), os.path.join(GOLD, "test2.idradec")
    A, B = np.fromfile(fa, oracle.OBJ_DTYPE), np.fromfile(fb, oracle.OBJ_DTYPE)
    for r_arcsec in (5, 30):
        po, do, _ = oracle.xmatch(A, B, r_arcsec * ARCSEC)
        po = po[np.lexsort((po[:, 1], po[:, 0]))]
        out = tmp_path / ("paged%d" % r_arcsec)
        # 10,000 A records in 34 segments of 300 (each with its zone offsets, about 0.5 MB at zh = 5")
        # against a 0.1 MiB budget; B (1,000 records) in 4 rounds of 300, which alternate the order of
        # the A segments
        r = run("-r", str(r_arcsec), "-n", "300", "--resident-mb", "0.1", "-v", "1", "-o", str(out), fa, fb)
        assert r.returncode == 0, r.stderr
        assert "paged in per job" in r.stderr
        p = np.concatenate(read_pairs(out, 16))
        p = p[np.lexsort((p[:, 1], p[:, 0]))]
        assert np.array_equal(p, po)

"""CPU tests of the C ABI: the library loads, exports every declared entry
point, and its host-only functions (formats, RA half-width) behave.  No
compute call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "xmatch.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(xm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import xmatch_b200._capi as capi
    lib = ctypes.CDLL(capi.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares each of them too
    assert sorted(capi.SIGNATURES) == names


def test_no_device_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import xmatch_b200 as xm
    with pytest.raises(xm.XmatchError) as e:
        xm.Context(0)
    assert e.value.status == 6   # XM_ERR_NODEVICE


def test_status_strings():
    import xmatch_b200 as xm
    for s in range(10):
        assert xm._lib.xm_status_str(s)


def test_idradec_roundtrip(tmp_path, fixtures):
    import xmatch_b200 as xm
    a, _ = fixtures
    f = str(tmp_path / "a.idradec")
    xm.write_idradec(f, a)
    assert os.path.getsize(f) == 24 * len(a)
    b = xm.read_idradec(f)
    assert b.tobytes() == a.tobytes()
    c = xm.read_idradec(f, 100, 50)
    assert c.tobytes() == a[100:150].tobytes()
    with pytest.raises(xm.XmatchError):
        xm.read_idradec(str(tmp_path / "missing.idradec"))
    with pytest.raises(xm.XmatchError):   # records beyond the end of the file
        xm.read_idradec(f, len(a) - 10, 20)


def test_idradec_read_in_parallel_pieces(tmp_path):
    # 200 MB: the reader splits it into 64 MB pieces read by several threads
    import xmatch_b200 as xm
    n = 200 * 2 ** 20 // 24 + 5
    a = np.empty(n, xm.OBJ_DTYPE)
    a["id"] = np.arange(n, dtype=np.int64) * 7 + 1
    a["ra"] = np.arange(n, dtype=np.float64) * 1e-5
    a["dec"] = -np.arange(n, dtype=np.float64) * 1e-6
    f = str(tmp_path / "big.idradec")
    a.tofile(f)
    b = xm.read_idradec(f)
    assert b.tobytes() == a.tobytes()
    c = xm.read_idradec(f, 3, n - 4)
    assert c.tobytes() == a[3 : n - 1].tobytes()


def test_pairs_writer_formats(tmp_path):
    import xmatch_b200 as xm
    p = np.array([[1, 2], [3, 4], [5, 6]], np.int64)
    d = np.array([0.5, 1e-6, 2.0])
    f16, f24, fa = (str(tmp_path / n) for n in ("p16", "p24", "ptxt"))
    xm.write_pairs(f16, p, mode=16)
    xm.write_pairs(f16, p[:1], mode=16, append=True)
    raw = np.fromfile(f16, np.int64).reshape(-1, 2)
    assert np.array_equal(raw, np.concatenate([p, p[:1]]))   # reference records {idA, idB}
    xm.write_pairs(f24, p, d, mode=24)
    rec = np.fromfile(f24, np.dtype([("a", "<i8"), ("b", "<i8"), ("d", "<f8")]))
    assert np.array_equal(rec["a"], p[:, 0]) and np.array_equal(rec["d"], d)
    xm.write_pairs(fa, p, d, mode=0)
    lines = open(fa).read().split("\n")
    assert lines[1].split()[:2] == ["3", "4"] and float(lines[1].split()[2]) == 1e-6
    with pytest.raises(xm.XmatchError):
        xm.write_pairs(f24, p, None, mode=24)


@pytest.mark.parametrize("r_arcsec,zh_arcsec", [(1, 1), (3, 3), (5, 2.5), (0.1, 0.1), (60, 60)])
def test_alpha_table_matches_oracle(r_arcsec, zh_arcsec):
    import xmatch_b200 as xm
    a = xm.alpha_table(r_arcsec / 3600, zh_arcsec / 3600)
    b = oracle.alpha_table(r_arcsec / 3600, zh_arcsec / 3600)
    assert a.tobytes() == b.tobytes()   # bit-identical host libm evaluation

"""Golden vectors from the REFERENCE's own pair kernel, run on a B200.

    python tests/golden/make_ref_golden.py OUTDIR

Runs BoostXmatch's xmatch_kernel (Worker.cu, compiled unmodified for sm_100a
into oracle/_ref/libref_kernel.so by oracle/ref_kernel.mk) over the reference
zone loop on the cases below and writes, per case, the sorted (idA, idB)
pairs it finds (ref_<case>.npz) and a summary (ref_summary.json).  The CPU
tests compare the oracle with these files.  Inputs: the reference fixture
Data/test.idradec (tests/golden/test.idradec, test2.idradec) and seeded
synthetic catalogs.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import OBJ_DTYPE, ref_kernel  # noqa: E402
from xmatch_b200 import synth  # noqa: E402

ARCSEC = 1.0 / 3600.0


def wrap_case(seed=21, n=4000):
    """Dense sources within 20" of ra = 0 on the equator: pairs across ra = 0."""
    rng = np.random.default_rng(seed)
    ra = rng.uniform(-20 * ARCSEC, 20 * ARCSEC, n) % 360.0
    dec = rng.uniform(-20 * ARCSEC, 20 * ARCSEC, n)
    A = np.empty(n, OBJ_DTYPE)
    A["id"], A["ra"], A["dec"] = np.arange(n), ra, dec
    B = np.empty(n, OBJ_DTYPE)
    B["id"] = np.arange(n) + 10 ** 9
    B["ra"] = (ra + rng.normal(0, 2 * ARCSEC, n)) % 360.0
    B["dec"] = dec + rng.normal(0, 2 * ARCSEC, n)
    return A, B


def cases():
    t = np.fromfile(os.path.join(HERE, "test.idradec"), OBJ_DTYPE)
    t2 = np.fromfile(os.path.join(HERE, "test2.idradec"), OBJ_DTYPE)
    for r in (1, 5, 30):
        yield "test_x_test_r%d" % r, t, t, r
    yield "test2_x_test_r5", t2, t, 5
    a, b = synth.config0(n_a=50_000, n_b=50_000, seed=5)
    yield "config0_50k_r3", a, b, 3
    a, b = wrap_case()
    np.savez_compressed(os.path.join(HERE, "wrap_case_inputs.npz"), A=a, B=b)
    yield "wrap_r5", a, b, 5


def srt(p):
    return p[np.lexsort((p[:, 1], p[:, 0]))] if len(p) else p.reshape(0, 2)


def save_case(out, name, pr, po):
    """Full pair list for small cases; for large ones only the pairs the
    oracle does not have plus the total (the pin test checks the rest)."""
    f = os.path.join(out, "ref_%s.npz" % name)
    if len(pr) <= 100_000:
        np.savez_compressed(f, pairs=pr)
    else:
        so = set(map(tuple, po.tolist()))
        only = np.array([p for p in pr.tolist() if tuple(p) not in so], np.int64).reshape(-1, 2)
        np.savez_compressed(f, ref_only=srt(only), n_pairs=np.int64(len(pr)))


def main(out):
    os.makedirs(out, exist_ok=True)
    summary = {}
    for name, A, B, r in cases():
        # the reference launch geometry as is: its compaction loses / invents pairs
        pu, outside_u, _ = ref_kernel.xmatch(A, B, r * ARCSEC, pad=False)
        su = set(map(tuple, pu.tolist()))
        # whole blocks only: the reference predicate by its own kernel
        pr, outside, launches = ref_kernel.xmatch(A, B, r * ARCSEC, pad=True)
        pr = srt(pr)
        po, _, _ = oracle.xmatch(A, B, r * ARCSEC)
        po = srt(po)
        sr = set(map(tuple, pr.tolist()))
        so = set(map(tuple, po.tolist()))
        summary[name] = {"reference_pairs": len(pr), "reference_unique": len(sr), "oracle_pairs": len(po),
                         "reference_only": len(sr - so), "oracle_only": len(so - sr),
                         "padded_pairs_outside_zone_ranges": outside, "launches": launches,
                         "unpadded": {"pairs": len(pu), "unique": len(su), "outside_launch_ranges": outside_u,
                                      "missing_vs_oracle": len(so - su), "extra_vs_oracle": len(su - so)}}
        save_case(out, name, pr, po)
        print(name, summary[name], flush=True)
    with open(os.path.join(out, "ref_summary.json"), "w") as f:
        json.dump(summary, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)

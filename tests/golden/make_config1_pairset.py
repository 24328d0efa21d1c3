"""Digest of the oracle's pair set for the full-scale 50M x 50M crossmatch.

    python tests/golden/make_config1_pairset.py [N]

Generates the seeded config-1 catalogs (xmatch_b200/synth.py config1: A and
B of N = 50M sources, 80 % uniform + 20 % in 500 clusters, B = 70 % perturbed
copies of A + 30 % random, wrap and polar sources), runs the oracle
(oracle/xm_oracle.c, windowed mode, all host threads) at r = zh = 1", and
writes tests/golden/config1_pairset.json: match and candidate counts, the
order-independent digest of the (idA, idB) set (xmatch_b200/pairhash.py) and
a fingerprint of the inputs.  bench.py compares the GPU pair set of its
headline step with this digest.  Takes a few minutes on 8 cores.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from xmatch_b200 import pairhash, synth  # noqa: E402

ARCSEC = 1.0 / 3600.0


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 50_000_000
    t0 = time.time()
    A, B = synth.config1(n=n)
    t1 = time.time()
    p, _, st = oracle.xmatch(A, B, ARCSEC, ARCSEC, with_dist=False)
    t2 = time.time()
    rec = {"workload": "config1 %d x %d, seed 1001, r = zh = 1 arcsec" % (n, n), "n": n, "seed": 1001,
           "r_arcsec": 1.0, "zh_arcsec": 1.0, "matches": int(st.n_match), "candidates": int(st.n_cand),
           "digest": pairhash.pairset_digest(p),
           "inputs": {"A": pairhash.inputs_fingerprint(A), "B": pairhash.inputs_fingerprint(B)},
           "oracle_seconds": round(t2 - t1, 1), "generate_seconds": round(t1 - t0, 1),
           "oracle_threads": os.cpu_count()}
    out = os.path.join(HERE, "config1_pairset.json" if n == 50_000_000 else "config1_pairset_%d.json" % n)
    with open(out, "w") as f:
        json.dump(rec, f, indent=1)
        f.write("\n")
    print(json.dumps(rec))


if __name__ == "__main__":
    main()

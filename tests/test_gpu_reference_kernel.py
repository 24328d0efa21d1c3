"""The reference's own pair kernel (BoostXmatch/Worker.cu compiled for
sm_100a, oracle/_ref) against the oracle and the CUDA path, live on the GPU.
Skipped when the harness library was not built (it needs the reference tree
at build time)."""
import numpy as np
import pytest

import oracle
from oracle import ref_kernel

pytestmark = pytest.mark.gpu

ARCSEC = 1.0 / 3600.0


def srt(p):
    return p[np.lexsort((p[:, 1], p[:, 0]))]


@pytest.mark.skipif(not ref_kernel.available(), reason="oracle/_ref/libref_kernel.so not built")
@pytest.mark.parametrize("seed,r", [(9, 3.0), (10, 10.0)])
def test_reference_kernel_agrees(ctx, seed, r):
    from xmatch_b200 import synth
    A, B = synth.config0(n_a=20_000, n_b=20_000, seed=seed)
    pr, outside, _ = ref_kernel.xmatch(A, B, r * ARCSEC, pad=True)
    po, _, _ = oracle.xmatch(A, B, r * ARCSEC)
    sa = ctx.build(A, r * ARCSEC)
    sb = ctx.build(B, r * ARCSEC)
    pg, _, _ = ctx.match(sa, sb, r * ARCSEC)
    sa.free()
    sb.free()
    # no RA wraparound pairs and no pair near the threshold in these catalogs:
    # the three must agree exactly (the reference kernel launched on whole
    # 16x16 blocks, where its compaction of Worker.cu:157-233 is sound)
    assert np.array_equal(srt(pr), srt(po))
    assert np.array_equal(srt(pg), srt(po))


@pytest.mark.skipif(not ref_kernel.available(), reason="oracle/_ref/libref_kernel.so not built")
def test_reference_launch_geometry_loses_pairs():
    """Evidence for the compaction defect: with the reference's own launch
    geometry (partial blocks) the kernel appends pairs outside the launched
    ranges and misses matches that whole-block launches find."""
    from xmatch_b200 import synth
    A, B = synth.config0(n_a=20_000, n_b=20_000, seed=9)
    pu, outside_u, _ = ref_kernel.xmatch(A, B, 3 * ARCSEC, pad=False)
    pp, _, _ = ref_kernel.xmatch(A, B, 3 * ARCSEC, pad=True)
    assert outside_u > 0
    assert len(set(map(tuple, pp.tolist())) - set(map(tuple, pu.tolist()))) > 0

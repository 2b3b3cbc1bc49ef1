"""The seeded benchmark inputs restated in the oracle (oracle/isg_inputs.c)
equal the library's generators bit for bit, so that bench.py's reference arm
builds the same inputs without loading the product library.  Host code only."""
import numpy as np
import pytest

import isg
from _oracle import Reference, seeded_ellipses, seeded_plane_waves


@pytest.mark.parametrize("level,count,eps,tand,seed", [(5, 3, (1.1, 1.5), 0.0, 1001), (6, 20, (1.1, 2.0), 0.1, 2000)])
def test_oracle_ellipses_equal_the_library(level, count, eps, tand, seed):
    s = isg.Solver(level)
    want = s.phantom(seed=seed, count=count, axis=(1.0, 3.0), eps=eps, tand_max=tand)
    got = seeded_ellipses(s.side, seed, count, (1.0, 3.0), eps, tand)
    assert np.count_nonzero(want) > 0
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("level", [4, 6])
def test_oracle_plane_waves_equal_the_library(level):
    s = isg.Solver(level)
    um = s.host_table("unkmap")
    for order, m in ((isg.ORDER_TREE, um), (isg.ORDER_RASTER, None)):
        want = s.plane_waves(16, first=3, count=5, order=order)
        got = seeded_plane_waves(s.side, 16, 3, 5, m)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), order


def test_reference_unkmap_is_the_library_unkmap():
    """The reference arm maps raster inputs to tree order with the reference's
    own unkmap (setup_mlfma.cpp:177-185); it is the library's."""
    if not Reference.available():
        pytest.skip("oracle/_ref not built")
    s = isg.Solver(5)
    ref = Reference(5)
    assert np.array_equal(ref.table("unkmap", 0, s.numunk, "i"), s.host_table("unkmap"))

"""The library's FP64 host tables (csrc/isg_tables.cpp) against the oracle.

These run without a GPU: isg_create builds every table on the host.
"""
import numpy as np
import pytest

import isg
from _oracle import Oracle, rel


@pytest.mark.parametrize("level", [3, 4, 5, 6])
def test_tables_match_oracle(level):
    nrx = 48
    s = isg.Solver(level, numrx=nrx)
    o = Oracle(level, numrx=nrx)
    L = level
    ns = [s.numsamp(i) for i in range(L)]
    assert ns == o.ns
    assert (s.host_table("numsamp") == np.array(ns)).all()
    items = [("near", 0, 9 * 4096, "c"), ("coeff_multi", 0, ns[-1] * 64, "c"), ("basis_local", 0, ns[-1] * 64, "c"),
             ("unkmap", 0, s.numunk, "i"), ("pos", 0, s.numunk, "c"), ("interph", 0, nrx * 30, "d"),
             ("intindh", 0, nrx * 30, "i"), ("anterph", 0, ns[0] * 60, "d"), ("antindh", 0, ns[0] * 60, "i")]
    items += [("trans", i, 49 * ns[i], "c") for i in range(2, L)]
    items += [("interp", i, ns[i] * 30, "d") for i in range(L - 1)]
    items += [("intind", i, ns[i] * 30, "i") for i in range(L - 1)]
    items += [("anterp", i, ns[i] * 60, "d") for i in range(1, L)]
    items += [("antind", i, ns[i] * 60, "i") for i in range(1, L)]
    items += [(n, i, 4 * ns[i], "c") for i in range(L - 1) for n in ("shiftmul", "shiftloc")]
    for name, lv, n, kind in items:
        a = o.table(name, lv, n, kind)
        b = s.host_table(name, lv)
        assert b.shape == a.shape, name
        if kind == "i":
            assert (a == b).all(), name
        else:
            assert rel(b, a) < 1e-13, (name, lv)


def test_orderings_are_permutations():
    s = isg.Solver(5)
    U = s.numunk
    for name in ("unkmap", "tree_of_blocked", "raster_of_blocked"):
        p = s.host_table(name)
        assert np.array_equal(np.sort(p), np.arange(U)), name
    # blocked -> tree must equal raster -> tree composed with blocked -> raster
    assert np.array_equal(s.host_table("tree_of_blocked"), s.host_table("unkmap")[s.host_table("raster_of_blocked")])


def test_phantom_and_sources_are_seeded():
    s = isg.Solver(5)
    a = s.phantom(seed=3, count=3, axis=(1, 3), eps=(1.1, 1.5))
    b = s.phantom(seed=3, count=3, axis=(1, 3), eps=(1.1, 1.5))
    c = s.phantom(seed=4, count=3, axis=(1, 3), eps=(1.1, 1.5))
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.real.max() <= 0.5 + 1e-12 and a.real.min() >= 0.0 and (a.real > 0).any()
    pw = s.plane_waves(8, order=isg.ORDER_TREE)
    pos = s.host_table("pos")
    ang = 2 * np.pi * 3 / 8
    assert rel(pw[3], np.exp(1j * 2 * np.pi * (np.cos(ang) * pos.real + np.sin(ang) * pos.imag))) < 1e-12
    grf = s.phantom(seed=5, kind=1, eps=(1.0, 1.6), corr_len=2.0)
    assert abs(grf.real.min()) < 1e-12 and abs(grf.real.max() - 0.6) < 1e-12

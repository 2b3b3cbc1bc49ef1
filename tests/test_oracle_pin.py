"""Pins the restated FP64 oracle (oracle/isg_oracle.c) to the reference.

The reference has no tests or vectors of its own; the fixtures in
tests/golden/ were produced by its own CPU path (oracle/_ref, see
tests/golden/make_golden.py).  When the compiled reference is present the
oracle is also compared with it live, table by table.
"""
import os

import numpy as np
import pytest

from _oracle import Oracle, Reference, rel

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@pytest.fixture(scope="module", params=["golden_l4.npz", "golden_l5.npz"])
def case(request):
    d = load(request.param)
    o = Oracle(int(d["level"]), float(d["k0"]), numrx=int(d["numrx"]))
    return d, o


def test_sample_counts(case):
    d, o = case
    assert o.ns == list(d["numsamp"])


def test_operator_matches_golden(case):
    d, o = case
    assert rel(o.mlfma(d["x"]), d["mlfma"]) < 1e-11
    assert rel(o.mlfmah(d["x"]), d["mlfmah"]) < 1e-11
    assert rel(o.aggregate(d["x"]), d["aggregate"]) < 1e-11
    assert rel(o.aggregateh(d["rx"]), d["aggregateh"]) < 1e-11


def test_mlfma_against_dense_mom(case):
    """MLFMA reproduces the dense MoM operator (integrate.cpp) to ~1e-6."""
    d, o = case
    r = o.mlfma(d["x"])
    rows = d["dense_rows"]
    assert rel(r[rows], d["dense"]) < 5e-6


def test_bicgs_matches_golden(case):
    d, o = case
    xf, itf, _ = o.bicgs(d["g"], d["b"], False, 1e-5, 300)
    xa, ita, _ = o.bicgs(d["g"], d["b"], True, 1e-5, 300)
    assert itf == int(d["bicgs_fwd_iters"]) and ita == int(d["bicgs_adj_iters"])
    assert rel(xf, d["bicgs_fwd"]) < 1e-9
    assert rel(xa, d["bicgs_adj"]) < 1e-9


def test_small_tables_match_golden(case):
    d, o = case
    ns = o.ns
    assert np.abs(o.table("near", 0, 9 * 4096, "c")[4 * 4096:4 * 4096 + 64] - d["near_slot4_row0"]).max() < 1e-15
    t = o.table("trans", 2, 49 * ns[2], "c")
    m = np.abs(d["trans2"]) > 0
    assert rel(t[m], d["trans2"][m]) < 1e-12
    assert rel(o.table("interp", 0, ns[0] * 30, "d"), d["interp0"]) < 1e-12
    assert (o.table("intind", 0, ns[0] * 30, "i") == d["intind0"]).all()


def test_matvec_definitions(case):
    """bicgs.cpp:62-87: forward y = x - G(g x); adjoint y = x - conj(g G(conj x))."""
    d, o = case
    x, g = d["x"], d["g"]
    assert rel(o.matvec(x, g, False), x - o.mlfma(g * x)) < 1e-14
    assert rel(o.matvec(x, g, True), x - np.conj(g * o.mlfma(np.conj(x)))) < 1e-14


@pytest.mark.skipif(not Reference.available(), reason="compiled reference (oracle/_ref) not built")
# The reference's setup_mlfma prints recvmap/sendmap rows 0..4 (setup_mlfma.cpp:379-383,
# 400-404), which reads past its level+1 rows below level 4, so it runs from level 4 up.
@pytest.mark.parametrize("level", [4, 5])
def test_oracle_tables_match_reference_live(level):
    ref = Reference(level, 2 * np.pi, 40)
    o = Oracle(level, 2 * np.pi, numrx=40)
    ns = o.ns
    assert ref.ns == ns
    L = level
    checks = [("near", 0, 9 * 4096, "c"), ("coeff_multi", 0, ns[-1] * 64, "c"), ("basis_local", 0, ns[-1] * 64, "c"),
              ("interph", 0, 40 * 30, "d"), ("anterph", 0, ns[0] * 60, "d"), ("intindh", 0, 40 * 30, "i"),
              ("antindh", 0, ns[0] * 60, "i"), ("unkmap", 0, o.U, "i"), ("clusnear", L - 1, 9 * 4 ** (L - 1), "i")]
    checks += [("trans", i, 49 * ns[i], "c") for i in range(2, L)]
    checks += [("clusfar", i, 27 * 4 ** i, "i") for i in range(2, L)]
    checks += [("interp", i, ns[i] * 30, "d") for i in range(L - 1)]
    checks += [("intind", i, ns[i] * 30, "i") for i in range(L - 1)]
    checks += [("anterp", i, ns[i] * 60, "d") for i in range(1, L)]
    checks += [("antind", i, ns[i] * 60, "i") for i in range(1, L)]
    checks += [(n, i, 4 * ns[i], "c") for i in range(L - 1) for n in ("shiftmul", "shiftloc")]
    for name, lv, n, kind in checks:
        a, b = ref.table(name, lv, n, kind), o.table(name, lv, n, kind)
        if kind == "i":
            assert (a == b).all(), name
        else:
            assert rel(b, a) < 1e-12, name
    # traid is only defined where the far list has an entry (setup_mlfma.cpp:515-525).
    for i in range(2, L):
        far = o.table("clusfar", i, 27 * 4 ** i, "i")
        m = far != -1
        assert (ref.table("traid", i, 27 * 4 ** i, "i")[m] == o.table("traid", i, 27 * 4 ** i, "i")[m]).all()


@pytest.mark.skipif(not Reference.available(), reason="compiled reference (oracle/_ref) not built")
def test_oracle_solves_match_reference_live():
    ref = Reference(4, 2 * np.pi, 32)
    o = Oracle(4, numrx=32)
    pos = o.pos()
    rng = np.random.default_rng(7)
    g = (2 * np.pi) ** 2 * (0.2 + 0.05j) * (np.abs(pos - (0.5 + 0.3j)) < 1.7)
    b = rng.standard_normal(o.U) + 1j * rng.standard_normal(o.U)
    for h in (False, True):
        xr, itr = ref.bicgs(g, b, h, 1e-6, 300)
        xo, ito, _ = o.bicgs(g, b, h, 1e-6, 300)
        assert itr == ito
        assert rel(xo, xr) < 1e-9

"""The restated inversion loop (orc_dbim) against the reference's own driver
run (tests/golden/golden_dbim_l7.npz, made by tests/golden/make_golden_dbim.py):
4 plane waves, 32 far-field receivers, 512 x 512 pixels, 3 Polak-Ribiere
iterations, inner BiCGSTAB to 1e-4.  About half a minute on 8 cores."""
import os

import numpy as np

import isg
from _oracle import Oracle, oracle_dbim, rel

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_dbim_l7.npz")


def test_oracle_inversion_matches_reference_driver():
    d = dict(np.load(GOLDEN))
    s = isg.Solver(int(d["level"]), numrx=int(d["numrx"]))
    o = Oracle(int(d["level"]), numrx=int(d["numrx"]))
    chi_true = s.raster_to_tree(d["phantom"].astype(np.float64) * 0.1 + 0j)
    inc = s.plane_waves(int(d["ntx"]), order=isg.ORDER_TREE)
    chi, hist, alpha, beta = oracle_dbim(o, inc, chi_true, 3, 0.0, float(d["tol"]))
    ref_hist = d["hist"]
    # hist.txt columns: misfit, object error, reg cost, gradient norm, object norm (printed to 7 digits)
    for col in (0, 1, 3, 4):
        m = np.abs(ref_hist[:, col]) > 0
        assert np.max(np.abs(hist[m, col] - ref_hist[m, col]) / np.abs(ref_hist[m, col])) < 1e-4, col
    assert np.max(np.abs(alpha - d["alpha"]) / np.abs(d["alpha"])) < 1e-4
    assert np.max(np.abs(beta - d["beta"]) / np.abs(d["beta"])) < 1e-3
    um = s.host_table("unkmap")
    assert rel(chi[um], d["cg2"]) < 1e-3

"""The drop-in boundary end to end: the reference's own driver sources
(mom.cpp and setup_born.cpp, unmodified) linked against libisg_ref.so instead of
the reference's solver (oracle/_ref/mom_isg, built by oracle/Makefile) run the
reference's inversion on the GPU.  Its hist.txt and final contrast must match
the reference's own CPU run of the same inputs (tests/golden/golden_dbim_l7.npz)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from _oracle import rel

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOM_ISG = os.path.join(ROOT, "oracle", "_ref", "mom_isg")
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_dbim_l7.npz")


@pytest.mark.skipif(not os.path.exists(MOM_ISG), reason="reference driver linked to libisg_ref.so not built")
@pytest.mark.parametrize("engine", ["0", "1"])
def test_reference_driver_on_libisg_ref(engine):
    d = dict(np.load(GOLDEN))
    with tempfile.TemporaryDirectory() as tmp:
        run = os.path.join(tmp, "run")
        os.makedirs(run)
        os.makedirs(os.path.join(tmp, "phantoms"))
        with open(os.path.join(tmp, "phantoms", "phantom_256.txt"), "w") as f:
            f.write("\n".join(repr(float(v)) for v in d["phantom"]) + "\n")
        env = dict(os.environ, NUMFREQ="1", NUMTX=str(int(d["ntx"])), TXPROC=str(int(d["ntx"])),
                   NUMRX=str(int(d["numrx"])), MLFMA="1", MINFREQ="1", MAXFREQ="1", ISG_ENGINE=engine)
        out = subprocess.run([MOM_ISG], cwd=run, env=env, capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr[-2000:]
        hist = np.loadtxt(os.path.join(run, "hist.txt"))
        cg2 = np.fromfile(os.path.join(run, "cg_2.bin"), dtype=np.complex128)
    ref = d["hist"]
    for col in (0, 1, 3, 4):
        m = np.abs(ref[:, col]) > 0
        assert np.max(np.abs(hist[m, col] - ref[m, col]) / np.abs(ref[m, col])) < 1e-3, (col, hist, ref)
    assert rel(cg2, d["cg2"]) < 2e-3
    assert "NOT CONVERGED" not in out.stdout

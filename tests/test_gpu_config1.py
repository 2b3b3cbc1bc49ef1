"""The reference's own small case end to end on the GPU: 128 x 128 pixels
(12.8 wavelengths at lambda/10), 4 MLFMA levels with 8 x 8-pixel leaves, three
random ellipses with real eps_r in [1.1, 1.5], 32 line-source transmitters and
32 receivers on a 20-wavelength circle (the near-field forms of
setup_born.cpp:52-72), one BiCGSTAB solve per transmitter to relative residual
1e-5 (mom.cpp:21), all transmitters as one batch.

Against the FP64 oracle (`tests/_oracle.py`, whose MLFMA matches the
reference's compiled operator to 5e-14 and the dense MoM rows of integrate.cpp
to 5e-6): every total field within 1e-4 of the oracle's solve converged to
1e-10, every receiver sample within 1e-4 of the oracle's near-field
receivers applied to that field, and the iteration count of each solve within
2 of the oracle's own BiCGSTAB at the same tolerance (the reference's
algorithm in FP64), on both engines."""
import numpy as np
import pytest

import isg
from _oracle import Oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


@pytest.mark.parametrize("engine", [isg.ENGINE_SIMT, isg.ENGINE_TENSOR])
def test_config1_fields_and_receivers_match_the_fp64_oracle(engine):
    import torch
    level, ntx, nrx, radius, tol = 5, 32, 32, 20.0, 1e-5
    s = isg.Solver(level, numrx=nrx, max_rhs=ntx, device=0)
    s.set_nearfield_receivers(radius)
    o = Oracle(level, numrx=nrx)
    o.set_nearfield(radius)
    chi = s.raster_to_tree(s.phantom(seed=101, count=3, axis=(1.0, 3.0), eps=(1.1, 1.5)))
    g = (2 * np.pi) ** 2 * chi
    inc = s.line_sources(ntx, radius)
    gd = torch.from_numpy(g.astype(np.complex64)).cuda()
    bd = torch.from_numpy(inc.astype(np.complex64)).cuda()
    x = torch.zeros_like(bd)
    info = s.bicgs(x, gd, bd, tol=tol, engine=engine)
    assert all(i["status"] == 0 and 0 <= i["true_residual"] <= tol for i in info), info
    rx = s.receive(gd * x).cpu().numpy()
    X = x.cpu().numpy()
    # the oracle computes in FP64 from the same complex64-rounded inputs
    g64 = g.astype(np.complex64).astype(np.complex128)
    errs, rx_errs, dits = [], [], []
    for j in range(ntx):
        b64 = inc[j].astype(np.complex64).astype(np.complex128)
        want = o.bicgs(g64, b64, False, 1e-10, 1000)[0]
        errs.append(rel(X[j], want))
        rx_errs.append(rel(rx[j], o.receive(g64 * want)))
        dits.append(info[j]["iterations"] - o.bicgs(g64, b64, False, tol, 1000)[1])
    print("config 1 engine", engine, "max field error", max(errs), "max receiver error", max(rx_errs),
          "iterations - oracle's", sorted(set(dits)))
    assert max(errs) <= 1e-4
    assert max(rx_errs) <= 1e-4
    assert max(abs(d) for d in dits) <= 2

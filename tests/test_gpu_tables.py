"""The Green's-function tables built on the device at set-up (near-field blocks
and translation operators: csrc/isg_tables_gpu.cu, Bessel J_p by Miller's
backward recurrence and Y_p by forward recurrence) against the same tables
built on the host with glibc's jn, yn, j0 and y0, as the reference builds them
(setup_mlfma.cpp:492-543, integrate.cpp:15-41).  Bar: 1e-10 relative per
table (both FP64; the translation series sums up to ~1000 terms whose cosines
of arguments up to ~6000 rad carry ~1e-13 of rounding)."""
import time

import numpy as np
import pytest

import isg
from _oracle import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level", [3, 5, 8, 10])
def test_device_green_tables_match_glibc(level):
    t0 = time.perf_counter()
    dev = isg.Solver(level, numrx=32, max_rhs=1, device=0)
    dev.setup_gpu()                      # near and trans computed on the device
    t_dev = time.perf_counter() - t0
    host = isg.Solver(level, numrx=32)   # queried before any set-up: host (glibc) tables
    t0 = time.perf_counter()
    want_near = host.host_table("near")
    t_host = time.perf_counter() - t0
    err = {"near": rel(dev.host_table("near"), want_near)}
    for i in range(2, level):
        a, b = dev.host_table("trans", i), host.host_table("trans", i)
        assert np.count_nonzero(b) == 40 * host.numsamp(i)  # the 40 far offsets of the 7 x 7 stencil
        err[f"trans{i}"] = rel(a, b)
    print("level", level, "device set-up", round(t_dev, 3), "s; host Green's tables", round(t_host, 3), "s;",
          {k: f"{v:.1e}" for k, v in err.items()})
    assert max(err.values()) < 1e-10, err


def test_device_tables_drive_the_same_operator():
    """A matvec on device-built tables equals one on host-built tables (the
    host tables are forced by a query before set-up) to FP32 rounding."""
    import torch
    a = isg.Solver(6, numrx=32, max_rhs=2, device=0)
    b = isg.Solver(6, numrx=32, max_rhs=2, device=0)
    b.host_table("trans", 2)             # host path for b
    rng = np.random.default_rng(4)
    X = torch.from_numpy((rng.standard_normal((2, a.numunk)) + 1j * rng.standard_normal((2, a.numunk)))
                         .astype(np.complex64)).cuda()
    ya = a.mlfma(X, engine=isg.ENGINE_SIMT).cpu().numpy()
    yb = b.mlfma(X, engine=isg.ENGINE_SIMT).cpu().numpy()
    assert rel(ya, yb) < 1e-6

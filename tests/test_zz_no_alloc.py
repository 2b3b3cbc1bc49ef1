"""isg_aggregate_noalloc (the receiver projection working in libisg.so's
static device array) against isg_aggregate, called through the C ABI twice in
a row.  Both run the same complex64 kernels; the tolerance written here is
1e-6 relative.  Named to be collected last, after every other GPU test."""
import ctypes

import numpy as np
import pytest

import isg

pytestmark = pytest.mark.gpu
TOL = 1e-6
SCRATCH_BYTES = 64 << 20


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def noalloc(s, x, rx, nrhs, order):
    import torch
    st = torch.cuda.current_stream().cuda_stream or None
    return isg.lib().isg_aggregate_noalloc(s._h, x.data_ptr(), rx.data_ptr(), nrhs, order, st)


@pytest.mark.parametrize("level,nrhs,order", [(6, 3, isg.ORDER_TREE), (7, 2, isg.ORDER_RASTER),
                                              (8, 2, isg.ORDER_TREE), (8, 4, isg.ORDER_BLOCKED)])
def test_noalloc_matches_aggregate_twice(level, nrhs, order):
    import torch
    s = isg.Solver(level, numrx=128, max_rhs=nrhs, device=0)
    s.setup_gpu()
    gen = torch.Generator(device="cuda").manual_seed(7 + level)
    for call in range(2):
        x = torch.randn((nrhs, s.numunk), dtype=torch.complex64, device="cuda", generator=gen)
        want = s.aggregate(x, order=order)
        got = torch.full_like(want, complex(float("nan"), float("nan")))
        assert noalloc(s, x, got, nrhs, order) == 0, isg.lib().isg_last_error(s._h).decode()
        torch.cuda.synchronize()
        g, w = got.cpu().numpy(), want.cpu().numpy()
        assert np.isfinite(g).all()
        assert rel(g, w) < TOL, (call, rel(g, w))


def test_noalloc_rejects_batches_beyond_the_static_array():
    import torch
    s = isg.Solver(8, numrx=64, max_rhs=1, device=0)
    s.setup_gpu()
    mp = sum(4 ** i * s.numsamp(i) for i in range(8))
    fit = SCRATCH_BYTES // ((mp + s.numunk) * 8)
    assert fit == 2
    x = torch.zeros((fit + 1, s.numunk), dtype=torch.complex64, device="cuda")
    rx = torch.zeros((fit + 1, s.numrx), dtype=torch.complex64, device="cuda")
    assert noalloc(s, x, rx, fit + 1, isg.ORDER_TREE) == 5
    msg = isg.lib().isg_last_error(s._h).decode()
    assert "static array" in msg and "at most 2 RHS" in msg, msg
    assert noalloc(s, x, rx, 0, isg.ORDER_TREE) == 5


def test_noalloc_needs_setup_gpu():
    s = isg.Solver(5, numrx=32, max_rhs=1, device=0)
    buf = ctypes.create_string_buffer(16)
    assert isg.lib().isg_aggregate_noalloc(s._h, ctypes.addressof(buf), ctypes.addressof(buf), 1, 0, None) == 5
    assert "isg_setup_gpu" in isg.lib().isg_last_error(s._h).decode()


FULL_HBM_SCRIPT = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import isg

s = isg.Solver(6, numrx=64, max_rhs=2, device=0)
s.setup_gpu()
x = torch.randn((2, s.numunk), dtype=torch.complex64, device="cuda")
got = torch.zeros((2, s.numrx), dtype=torch.complex64, device="cuda")
want = torch.zeros_like(got)
torch.cuda.synchronize()
# Leave less free device memory than the static array's size, so that a
# first call which still had to load it would fail.
margin = 24 << 20
hold = []
for _ in range(64):
    free, _ = torch.cuda.mem_get_info()
    if free <= margin + (8 << 20):
        break
    hold.append(torch.empty(free - margin, dtype=torch.uint8, device="cuda"))
free, _ = torch.cuda.mem_get_info()
assert free < (64 << 20), free
st = torch.cuda.current_stream().cuda_stream or None
rc = isg.lib().isg_aggregate_noalloc(s._h, x.data_ptr(), got.data_ptr(), 2, isg.ORDER_TREE, st)
assert rc == 0, (rc, isg.lib().isg_last_error(s._h).decode())
assert isg.lib().isg_aggregate(s._h, x.data_ptr(), want.data_ptr(), 2, isg.ORDER_TREE, st) == 0
torch.cuda.synchronize()
free_after, _ = torch.cuda.mem_get_info()
del hold
g, w = got.cpu().numpy(), want.cpu().numpy()
err = float(np.linalg.norm(g - w) / np.linalg.norm(w))
print("free before", free, "after", free_after, "rel", err)
assert err < 1e-6, err
"""


def test_first_call_succeeds_with_device_memory_full():
    """The array is resolved by isg_setup_gpu, so the process's first call
    needs no device memory: after set-up the test fills the device to within
    24 MiB of full and only then makes that first call (a fresh process, so
    no earlier call loaded anything)."""
    import os
    import subprocess
    import sys
    pkg = os.path.dirname(os.path.dirname(isg.__file__))
    r = subprocess.run([sys.executable, "-c", FULL_HBM_SCRIPT, pkg], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

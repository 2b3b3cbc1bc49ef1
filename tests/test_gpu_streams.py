"""Stream ordering of the Python binding: inputs that torch has just produced
on its current stream (an index, a copy) are complete before the library reads
them on a caller's side stream.  The current stream is held back by a bounded
spin (`torch.cuda._sleep`, about 30 ms) before the gather that builds the
inputs, so a solve that started without waiting would read unwritten memory."""
import numpy as np
import pytest

import isg

pytestmark = pytest.mark.gpu


def test_side_stream_call_waits_for_inputs_built_on_the_current_stream():
    import torch
    s = isg.Solver(4, numrx=16, max_rhs=8, device=0)  # 64 x 64 pixels
    s.setup_gpu()
    U = s.numunk
    G = torch.from_numpy(np.stack([(2 * np.pi) ** 2 * s.raster_to_tree(s.phantom(seed=500 + j, count=2,
                                                                               eps=(1.1, 1.4)))
                                   for j in range(4)]).astype(np.complex64)).cuda()
    B = torch.from_numpy(s.plane_waves(16).astype(np.complex64)).cuda()
    gi = torch.tensor([0, 1, 2, 3, 0, 1, 2, 3], device="cuda")
    bi = torch.tensor([0, 2, 4, 6, 8, 10, 12, 14], device="cuda")
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    torch.cuda._sleep(60_000_000)  # the current stream spins; the gathers below queue behind it
    g, b = G[gi], B[bi]
    x = torch.zeros((8, U), dtype=torch.complex64, device="cuda")
    info = s.bicgs(x, g, b, tol=1e-6, engine=isg.ENGINE_TENSOR, stream=side)
    torch.cuda.synchronize()
    ref = torch.zeros_like(x)
    want = s.bicgs(ref, G[gi], B[bi], tol=1e-6, engine=isg.ENGINE_TENSOR)
    torch.cuda.synchronize()
    assert [i["iterations"] for i in info] == [i["iterations"] for i in want]
    assert torch.equal(x, ref)

"""ffs_lbm_step inside a CUDA graph.

After one eager step (which picks the dense-kernel variant and sizes the link
table), the step records only stream work: kernel launches and the events that
fork link detection onto the grid's side stream and join it back.  A graph
captured on the caller's stream then replays like eager steps.  The grid's
buffer parity flips on the host once per step, so a graph holds an even number
of steps; each captured step keeps the surface buffers it was given, whose
contents the caller refreshes before every replay.
"""
import numpy as np
import pytest

from freeflow_b200 import workloads as W

from helpers import make_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [2, 3])
def test_two_step_graph_replays_like_eager_steps(cuda, dim):
    import torch

    from freeflow_b200 import DeviceSurface

    if dim == 2:
        wl = W.swimmer_2d(nx=300, ny=120, body_frac=0.5, n_boundary=120, seed=2)
    else:
        wl = W.swimmer_3d(nx=64, ny=32, nz=32, body_frac=0.4, nlat=16, nlon=24, seed=4)
    ge, se = make_gpu(wl)                          # eager
    gg, _ = make_gpu(wl)                           # graph
    v0, u0 = wl.surface_at(0)
    sa = DeviceSurface(v0, u0, wl.elements, with_forces64=True)
    sb = DeviceSurface(v0, u0, wl.elements, with_forces64=True)
    ge.step(se)
    gg.step(sa)
    torch.cuda.synchronize()

    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        gg.step(sa, stream=stream)
        gg.step(sb, stream=stream)

    for k in range(1, 11, 2):
        for j in (k, k + 1):
            se.update(*wl.surface_at(j))
            ge.step(se)
        sa.update(*wl.surface_at(k))
        sb.update(*wl.surface_at(k + 1))
        graph.replay()
    torch.cuda.synchronize()

    assert ge.status() == 0 and gg.status() == 0
    assert np.array_equal(ge.get_moments(), gg.get_moments())
    fe = se.forces64.cpu().numpy()
    fg = sa.forces64.cpu().numpy() + sb.forces64.cpu().numpy()
    assert np.abs(fe).max() > 0
    assert np.abs(fg - fe).max() <= 1e-9 * np.abs(fe).max()
    del graph
    ge.close()
    gg.close()

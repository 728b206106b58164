"""A warm time-step solve captured into a CUDA graph and replayed.

A hydro code that calls the solver once per step on fixed density/potential
buffers can record the call once (stream capture: the side-stream ADI forks
and joins through events, programmatic launches become graph edges) and replay
it each step.  Every replay must equal the same call made directly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRID = (130, 98, 256, 1.0 / 126.0, 2, 30)


def test_captured_warm_solve_replays_like_direct_calls(bph):
    import torch

    from bipoly_hydro_b200 import fields

    base = fields.bipolytrope_pair()
    seq = [np.ascontiguousarray(fields.rotate(base, t).ravel(order="F")) for t in range(5)]

    direct = bph.PotentialSolver(*GRID)
    d_rho0 = torch.from_numpy(seq[0]).cuda()
    d_pot0 = torch.empty_like(d_rho0)
    direct.set_stream(torch.cuda.current_stream())
    direct.potential_solver_device(d_rho0, d_pot0, 0)
    want = []
    for t in range(1, 5):
        d_rho0.copy_(torch.from_numpy(seq[t]))
        direct.potential_solver_device(d_rho0, d_pot0, t + 1)
        want.append(d_pot0.clone())
    torch.cuda.synchronize()

    g = bph.PotentialSolver(*GRID)
    d_rho = torch.from_numpy(seq[0]).cuda()
    d_pot = torch.empty_like(d_rho)
    g.set_stream(torch.cuda.current_stream())
    g.potential_solver_device(d_rho, d_pot, 0)  # cold start, outside the graph
    g.synchronize()
    graph = torch.cuda.CUDAGraph()
    d_rho.copy_(torch.from_numpy(seq[1]))
    torch.cuda.synchronize()
    capture_stream = torch.cuda.Stream()
    with torch.cuda.graph(graph, stream=capture_stream):
        g.set_stream(torch.cuda.current_stream())
        g.potential_solver_device(d_rho, d_pot, 2)
    g.set_stream(torch.cuda.current_stream())
    # capture records the work without running it: replay step 1, then 2..4
    got = []
    for t in range(1, 5):
        d_rho.copy_(torch.from_numpy(seq[t]))
        graph.replay()
        got.append(d_pot.clone())
    torch.cuda.synchronize()
    g.synchronize()
    for t in range(4):
        assert torch.equal(got[t], want[t]), t
    del graph
    g.close()
    direct.close()

"""dem_wall_reactions_noalloc: the allocation-free entry point.

Callers that cannot call cudaMalloc (code running during CUDA graph capture,
hosts that hand over memory from their own pool, real-time loops that forbid
allocation) get per-wall reaction forces from a fixed device scratch array
instead of allocated memory.  This test feeds it the particle state from just
before a dem_step and checks its output against what the step itself reports
for the walls (dem_get_wall), within the parity tests' force tolerance (1e-8
of the largest reaction), on two calls in a row so that reuse of the shared
scratch is exercised.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu

WALLS = [("xlo", (0, 0, 0), (1, 0, 0)), ("xhi", (6, 0, 0), (-1, 0, 0)), ("ylo", (0, 0, 0), (0, 1, 0)),
         ("yhi", (0, 6, 0), (0, -1, 0)), ("zlo", (0, 0, 0), (0, 0, 1)), ("zhi", (0, 0, 12), (0, 0, -1))]


def test_noalloc_wall_reactions_match_step(dem_lib):
    import torch

    from esys.lsm import _capi

    sim = S.gravity_box(lambda *a: _capi.DemSim(*a), 6)
    sim.step(120)
    # radii by id, as drawn by the scenario builder (seeded)
    rng = np.random.default_rng(1)
    g = np.stack(np.meshgrid(np.arange(6), np.arange(6), np.arange(6), indexing="ij"), -1).reshape(-1, 3)
    rng.uniform(-0.05, 0.05, size=g.shape)
    rad = rng.uniform(0.4, 0.5, size=len(g))
    before = sim.particles()
    sim.step(1)  # the wall reactions of this step are computed from `before`
    expected = np.stack([sim.wall(name)[1] for name, _, _ in WALLS])
    assert np.abs(expected).max() > 0.0

    dev = torch.device("cuda:0")
    parts = torch.tensor(np.column_stack([before["pos"], rad[before["id"]]]), dtype=torch.float64, device=dev)
    walls = torch.tensor([list(o) + list(n) + [1000.0] for _, o, n in WALLS], dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    fn = dem_lib.dem_wall_reactions_noalloc
    for call in range(2):
        out = torch.full((len(WALLS), 3), float("nan"), dtype=torch.float64, device=dev)
        rc = fn(parts.shape[0], ctypes.c_void_p(parts.data_ptr()), len(WALLS), ctypes.c_void_p(walls.data_ptr()),
                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, (call, rc)
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert np.abs(got - expected).max() <= 1e-8 * np.abs(expected).max(), (call, got, expected)


def test_noalloc_rejects_sizes_beyond_the_limit(dem_lib):
    import torch

    fn = dem_lib.dem_wall_reactions_noalloc
    buf = torch.zeros(64, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(buf.data_ptr())
    odd = ctypes.c_void_p(buf.data_ptr() + 4)
    assert fn(1, p, 9, p, p, None) == -1            # more than 8 walls
    assert fn(1 << 25, p, 1, p, p, None) == -1      # more than 16777216 particles
    assert fn(-1, p, 1, p, p, None) == -1
    assert fn(1, p, 1, odd, p, None) == -1           # walls not 8-byte aligned
    assert fn(1, p, 1, p, odd, None) == -1           # reactions not 8-byte aligned


def test_noalloc_counts_every_given_particle(dem_lib):
    """Unlike the step's reaction, which counts only a wall's candidates, every particle passed in
    counts: one far behind a wall plane gets the elastic wall force of its overlap,
    k pi r (r - d) along the normal (CElasticWallInteraction, pi = 3.141592654)."""
    import torch

    dev = torch.device("cuda:0")
    r, d, k = 0.5, -3.0, 1000.0
    parts = torch.tensor([[1.0, d, 2.0, r]], dtype=torch.float64, device=dev)
    walls = torch.tensor([[0, 0, 0, 0, 1, 0, k]], dtype=torch.float64, device=dev)
    out = torch.full((1, 3), float("nan"), dtype=torch.float64, device=dev)
    rc = dem_lib.dem_wall_reactions_noalloc(1, ctypes.c_void_p(parts.data_ptr()), 1, ctypes.c_void_p(walls.data_ptr()),
                                            ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize(dev)
    expect = k * 3.141592654 * r * (r - d)
    assert np.allclose(out.cpu().numpy(), [[0.0, expect, 0.0]], rtol=1e-12, atol=0.0)

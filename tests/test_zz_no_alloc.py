"""gdf_lh_noalloc: the Lh residual for callers that cannot allocate device
memory (their memory is planned at start-up, or a framework pool forbids
allocations outside it). It runs on caller-owned device buffers with the
face-flux scratch in a fixed array inside the library. Checked through the
C ABI against the existing entry point gdf_lh on three calls in a row. The
first call fills the scratch; the second and third use grids whose face
planes sit at other offsets, so both read scratch that an earlier call left
non-zero, and a face point a call failed to write would show up there.
This file sorts last so that a run stopping at the first failure has run
every other test before it."""
import numpy as np
import pytest

import gdf
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _state(problem, nx, ny):
    cfg, _ = gdf.problem_config(problem, nx, ny)
    o = Oracle(cfg)
    uh, bx, by = o.init_data(problem)
    o.prepare(uh, bx, by)
    o.set_bc(uh)
    return cfg, uh


def test_lh_noalloc_matches_gdf_lh_on_consecutive_calls():
    import torch
    stream = torch.cuda.current_stream()
    grids = ((gdf.PROB_ROTOR, 40, 36), (gdf.PROB_ORSZAG_TANG, 24, 16), (gdf.PROB_BLAST, 18, 30))
    for problem, nx, ny in grids:
        cfg, uh = _state(problem, nx, ny)
        ref = gdf.Solver(cfg).lh(uh)                 # existing entry point (product build)
        d_uh = torch.from_numpy(uh).to("cuda")
        d_du = torch.full_like(d_uh, float("nan"))  # every entry must be written
        torch.cuda.synchronize()
        gdf.lh_noalloc(cfg, d_uh.data_ptr(), d_du.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        du = d_du.cpu().numpy()
        # the product build's tolerance: value for value
        assert np.array_equal(du, ref), f"grid {nx}x{ny}"


def test_lh_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    cfg, _ = gdf.problem_config(gdf.PROB_ORSZAG_TANG, 200, 100)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(gdf.GdfError) as e:
        gdf.lh_noalloc(cfg, d.data_ptr(), d.data_ptr(), 0)
    assert e.value.code == gdf._abi.GDF_ERR_ARG
    assert "16640" in str(e.value)

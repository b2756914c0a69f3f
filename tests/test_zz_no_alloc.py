"""The render entry point that allocates no device memory.

Some callers cannot call cudaMalloc while rendering: a host application whose
device memory belongs to its own allocator or is held to a fixed budget, or a
plugin that may not grow the process's footprint after start-up.  For them
hk_render_image_static keeps its scratch (work counter, counters, film
accumulator) in a static device array and writes into an image the caller
supplies.  This test checks, through the C ABI, that two calls in a row give
the image of the allocating entry point (hk_render_image) within the
tolerance of the other GPU tests -- the same sample streams, summed in a
different atomic order -- and that a film beyond the array's limit is
rejected.  The file sorts last so a stop-at-first-failure run has already run
every other test."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from tests.gpu_helpers import rel_close  # noqa: E402

RTOL = 1e-5


@pytest.mark.gpu
def test_static_scratch_render_matches_allocating_entry_point():
    sd = scenes.cornell_box(width=64, height=48)
    gs = hk.Scene.from_desc(sd)
    ref, ref_ctr = gs.render_image(256, sd.depth, seed=11)
    for call in range(2):
        out = torch.full((48, 64, 3), -1.0, dtype=torch.float32, device="cuda")
        ctr = torch.zeros(5, dtype=torch.int64, device="cuda")
        gs.render_image_static(out, 256, sd.depth, seed=11, counters=ctr)
        torch.cuda.synchronize()
        img = out.cpu().numpy()
        ok = rel_close(img, ref, RTOL, atol=1e-6 * float(np.abs(ref).max()))
        assert ok.all(), f"call {call}: {np.sum(~ok)} pixels differ beyond {RTOL}"
        c = ctr.cpu().numpy()
        assert c[0] == ref_ctr[0] and c[1] == ref_ctr[1], (call, c, ref_ctr)


@pytest.mark.gpu
def test_static_scratch_rejects_films_beyond_its_size():
    sd = scenes.cornell_box(width=600, height=600)
    gs = hk.Scene.from_desc(sd)
    out = torch.empty((600, 600, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(hk.HikariError, match="static scratch"):
        gs.render_image_static(out, 1, sd.depth)

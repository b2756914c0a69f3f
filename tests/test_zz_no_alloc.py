"""The render entry point that allocates no device memory.

Some callers cannot call cudaMalloc while rendering: a host application whose
device memory belongs to its own allocator or is held to a fixed budget, or a
plugin that may not grow the process's footprint after start-up.  For them
hk_render_image_static keeps its scratch (work counter, counters, film
accumulator) in a static device array and writes into an image the caller
supplies.  This test checks, through the C ABI, that two calls in a row give
the image of the allocating entry point (hk_render_image) within the
tolerance of the other GPU tests -- the same sample streams, summed in a
different atomic order -- that the second call still succeeds with the
device's free memory taken up (where the allocating entry point then fails),
and that a film beyond the array's limit is rejected.  The file sorts last so
a stop-at-first-failure run has already run every other test."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hikari_b200 as hk  # noqa: E402
from hikari_b200 import scenes  # noqa: E402
from tests.gpu_helpers import rel_close  # noqa: E402

RTOL = 1e-5


def _take_free_memory(keep_bytes: int):
    """Hold device memory in shrinking chunks until less than 2 * keep_bytes
    is free: an allocation of more than that cannot succeed then."""
    torch.cuda.empty_cache()
    held = []
    for chunk in (8 << 30, 1 << 30, 128 << 20, 16 << 20, 2 << 20):
        while torch.cuda.mem_get_info()[0] - chunk >= keep_bytes:
            try:
                held.append(torch.empty(chunk, dtype=torch.uint8, device="cuda"))
            except torch.OutOfMemoryError:
                break
    return held


@pytest.mark.gpu
def test_static_scratch_render_matches_allocating_entry_point():
    w, h = 256, 192
    sd = scenes.cornell_box(width=w, height=h)
    gs = hk.Scene.from_desc(sd)
    gs.set_image_form(hk.FORM_MEGAKERNEL)   # the same kernel as the static entry point
    ref, ref_ctr = gs.render_image(64, sd.depth, seed=11)
    # a second scene, 2048 x 2048, that has not rendered yet: its first
    # render_image must allocate a 67 MB film (built here, before the device
    # memory is taken)
    big = scenes.cornell_box(width=2048, height=2048)
    fresh = hk.Scene.from_desc(big)
    fresh.set_image_form(hk.FORM_MEGAKERNEL)
    for call in range(2):
        out = torch.full((h, w, 3), -1.0, dtype=torch.float32, device="cuda")
        ctr = torch.zeros(5, dtype=torch.int64, device="cuda")
        held = []
        try:
            if call == 1:
                # the second call runs with the device's free memory taken (less
                # than 32 MB left): the allocating path fails there
                held = _take_free_memory(4 << 20)
                assert torch.cuda.mem_get_info()[0] < (32 << 20)
                with pytest.raises(hk.HikariError):
                    fresh.render_image(1, big.depth, seed=11)
            gs.render_image_static(out, 64, sd.depth, seed=11, counters=ctr)
            torch.cuda.synchronize()
        finally:
            del held
            torch.cuda.empty_cache()
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


@pytest.mark.gpu
def test_static_scratch_checks_its_buffers():
    sd = scenes.cornell_box(width=32, height=32)
    gs = hk.Scene.from_desc(sd)
    with pytest.raises(TypeError):
        gs.render_image_static(np.zeros((32, 32, 3), np.float32), 1, sd.depth)
    with pytest.raises(ValueError):
        gs.render_image_static(torch.zeros((32, 32, 3), dtype=torch.float64, device="cuda"), 1, sd.depth)
    with pytest.raises(ValueError):
        gs.render_image_static(torch.zeros((16, 32, 3), dtype=torch.float32, device="cuda"), 1, sd.depth)
    with pytest.raises(ValueError):
        gs.render_image_static(torch.zeros((32, 3, 32), dtype=torch.float32, device="cuda").transpose(1, 2), 1,
                               sd.depth)
    with pytest.raises(ValueError):
        gs.render_image_static(torch.zeros((32, 32, 3), dtype=torch.float32, device="cuda"), 1, sd.depth,
                               counters=torch.zeros(4, dtype=torch.int64, device="cuda"))

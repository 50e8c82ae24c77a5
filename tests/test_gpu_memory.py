"""Device memory across uploads: a context's buffers only grow, and a scene
uploaded again (every frame, as a caller streaming frames does) allocates
nothing and frees nothing, so device memory in use stays flat. The pass
buffers (bins, tile records, PTCL, glyph lists) are handed from each upload
to the next."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk

pytestmark = pytest.mark.gpu


def free_bytes() -> int:
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def test_gpu_reupload_allocates_nothing():
    r = tk.NativeRenderer(0)
    try:
        big = tk.generate(2, 6, width=1536, height=1024, paths=3000, device_flatten=True)
        small = tk.generate(2, 7, width=512, height=384, paths=300)
        first = r.render_to_image(big)
        records = r.stats()["ptcl_records"]
        r.render_to_image(small)
        r.render_to_image(big)
        before = free_bytes()
        for _ in range(6):
            img = r.render_to_image(big)
            r.render_to_image(small)
        after = free_bytes()
        assert np.array_equal(img, first)
        # every buffer was sized by the first frames; nothing grows or leaks
        assert before - after < (8 << 20), (before, after)
        assert records > 100000
    finally:
        r.close()

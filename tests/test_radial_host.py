"""Host logic of the radial eps model (pipeline.c:445-456) against the FP64 oracle: the
per-tile eps is plan-time scalar work, so it runs on the host and needs no device."""
import ctypes as C

import numpy as np
import pytest

from oracle import o64, p


@pytest.mark.parametrize("have,a,b,med,geps", [
    (1, 0.01, 2e-5, 0.015, 4e-3),        # inside the clamp
    (1, 0.01, 2e-3, 0.015, 4e-3),        # far rim: clamped at 8
    (1, 1e-4, 0.0, 0.015, 4e-3),         # small fn: clamped at 0.4
    (0, 0.01, 2e-5, 0.015, 4e-3),        # model off -> 0 (use the global eps)
    (1, 0.01, 2e-5, 0.0, 4e-3),          # no median -> 0
    (1, 0.01, 2e-5, 0.015, 0.0),         # no global eps -> 0
])
def test_tile_eps_matches_oracle(fy, have, a, b, med, geps):
    lib = fy.load()
    fit = fy.RadialEps(a=a, b=b, corr=0.9, median=med, guided_eps=geps, have=have, n=64)
    rng = np.random.default_rng(1)
    for _ in range(20):
        cy, cx = rng.uniform(0, 4000, 2)
        y0, x0 = (int(v) for v in rng.integers(0, 8000, 2))
        ty, tx = (int(v) for v in rng.integers(1, 1024, 2))
        got = lib.fy_radial_tile_eps(C.byref(fit), geps, cy, cx, y0, x0, ty, tx)
        want = o64().o64_radial_tile_eps(have, a, b, med, geps, cy, cx, y0, x0, ty, tx)
        assert got == pytest.approx(want, rel=1e-15, abs=0.0)


def test_median_floor_oracle():
    v = np.array([0.3, 0.1, 0.2, 0.4])
    assert o64().o64_median_floor(p(v), 4) == pytest.approx(0.25)
    assert o64().o64_median_floor(p(v), 3) == 0.2
    assert o64().o64_median_floor(p(v), 0) == 0.015

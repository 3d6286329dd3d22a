"""GPU test of the allocation-free dot product (hyb_fn_dot_noalloc) against hyb_fn_dot.

Collected last on purpose: it must pass both alone in a fresh process and after every other test
has run on the same device."""

import numpy as np
import pytest

import hyteg_b200 as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("L", [3, 6])
def test_noalloc_dot_matches_dot(ctx, dtype, L):
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    a = H.P1Function("a", pm, L, L, ctx, dtype)
    b = H.P1Function("b", pm, L, L, ctx, dtype)
    a.fill_random(L, 31)
    b.fill_random(L, 32)
    for flag in (H.Inner, H.All):
        ref = a.dotGlobal(b, L, flag)
        got1 = a.dotGlobalNoAlloc(b, L, flag)
        got2 = a.dotGlobalNoAlloc(b, L, flag)
        assert got1 == got2
        assert abs(got1 - ref) <= 1e-14 * max(1.0, abs(ref))
    np.testing.assert_allclose(a.dotGlobalNoAlloc(a, L, H.All), a.dotGlobal(a, L, H.All), rtol=1e-14)


def test_noalloc_dot_rejects_oversized_and_unprepared_levels(ctx):
    shell = H.PrimitiveStorage.spherical_shell(5, 3, 0.55, 1.0, ctx=ctx)  # 1920 macro-cells
    L = 5  # about 105,000 block partials, above the 65,536 of the fixed scratch
    f = H.P1Function("f", shell, L, L, ctx)
    f.fill_random(L, 1)
    with pytest.raises(H.HybError, match="block partials"):
        f.dotGlobalNoAlloc(f, L, H.All)
    cube = H.PrimitiveStorage.cuboid(ctx=ctx)
    g = H.P1Function("g", cube, 4, 4, ctx)  # no operation has run on level 4 of this mesh yet
    with pytest.raises(H.HybError, match="not on the device"):
        g.dotGlobalNoAlloc(g, 4, H.All)

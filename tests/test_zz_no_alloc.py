"""GPU test of the allocation-free dot product (hyb_fn_dot_noalloc) against hyb_fn_dot.

Some callers cannot let a library call allocate device memory, for example a host runtime that
reserves the device memory up front and hands it out through its own allocator.  The entry point
under test keeps its partial sums in a fixed device array instead of the context's growable buffer.
These tests check that it gives exactly the bits of hyb_fn_dot, on two calls in a row, and that the
context's scratch does not grow while it runs.

Collected last on purpose: it must pass both alone in a fresh process and after every other test
has run on the same device."""

import pytest

import hyteg_b200 as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("L", [3, 6])
def test_noalloc_dot_matches_dot_without_allocating(dtype, L):
    ctx = H.Context(0)  # a fresh context: nothing allocated for reductions yet
    pm = H.PrimitiveStorage.cuboid(ctx=ctx)
    A = H.P1ConstantLaplaceOperator(pm, L, L, ctx)
    a = H.P1Function("a", pm, L, L, ctx, dtype)
    b = H.P1Function("b", pm, L, L, ctx, dtype)
    a.fill_random(L, 31)
    b.fill_random(L, 32)
    A.apply(a, b, L, H.Inner)  # puts the level's tables on the device; no reduction
    ctx.synchronize()
    before = ctx.scratch_bytes
    got = {}
    for flag in (H.Inner, H.All):
        got1 = a.dotGlobalNoAlloc(b, L, flag)
        got2 = a.dotGlobalNoAlloc(b, L, flag)
        assert got1 == got2
        got[flag] = got1
    assert ctx.scratch_bytes == before, "the allocation-free dot grew the context's scratch"
    for flag in (H.Inner, H.All):
        assert a.dotGlobal(b, L, flag) == got[flag]  # same kernels, same order: the same bits
    assert ctx.scratch_bytes > before  # the plain dot did allocate its partials
    ctx.close()


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

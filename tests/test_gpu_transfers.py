"""Host transfers: the synchronous and the asynchronous (double-buffered) paths give the packed
vectors bit for bit, for every value type, and refresh the copies of owned DoFs."""

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["float64", "float32", "float16"])
def test_async_transfers_match_sync(ctx, dtype):
    coords, tets = M.octahedron_8()
    om = O.MacroMesh(coords, tets)
    pm = H.PrimitiveStorage.from_tets(coords, tets, ctx)
    L = 3
    lev = O.Level(om, L)
    rng = np.random.default_rng(5)
    x = np.zeros(lev.size)
    m = lev.owned_mask(O.ALL)
    x[m] = rng.uniform(-1, 1, m.sum())
    x = lev.sync(x)
    c2 = H.Context(0)
    f = H.P1Function("f", pm, L, L, c2, dtype)
    g = H.P1Function("g", pm, L, L, ctx, dtype)
    f.upload_async(L, x)
    out = np.zeros(f.packed_size(L))
    f.download_async(L, out)
    c2.synchronize()
    g.upload(L, x)
    ref = g.download(L)
    keep = m.copy()
    keep[lev.copy_map()[0]] = True
    np.testing.assert_array_equal(out[keep], ref[keep])
    if dtype == "float64":
        np.testing.assert_array_equal(out[keep], x[keep])

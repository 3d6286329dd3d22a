"""CPU tests of the C ABI boundary: the library loads, exports every declared entry point, and its
host-side logic (mesh topology, HyTeG layout, argument checks) matches the oracle.  No device work."""

import os
import re

import numpy as np
import pytest

import hyteg_b200 as H
from oracle import hyteg_oracle as O
from tests import meshes as M

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "hyteg_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hyb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = H.lib()
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binds_every_declared_symbol():
    assert set(declared_symbols()) <= set(H._SIGS)


@pytest.mark.parametrize("name", sorted(M.ALL))
def test_topology_matches_reference_ordering(name):
    coords, tets = M.ALL[name]()
    om = O.MacroMesh(coords, tets)
    pm = H.PrimitiveStorage.from_tets(coords, tets)
    assert pm.counts() == (om.nV, om.nE, om.nF, om.nC)
    for kind, lst in ((1, om.edges), (2, om.faces), (3, om.cells)):
        for i, v in enumerate(lst):
            assert pm.primitive_vertices(kind, i) == list(v)
    for kind, flags in ((0, om.flag_v), (1, om.flag_e), (2, om.flag_f), (3, om.flag_c)):
        assert [pm.primitive_flag(kind, i) for i in range(len(flags))] == list(flags)


@pytest.mark.parametrize("name", ["cube_6", "octahedron_8", "cube_2x1x1"])
@pytest.mark.parametrize("L", [0, 1, 2, 5])
def test_layout_matches_vertexdof_memory(name, L):
    coords, tets = M.ALL[name]()
    om = O.MacroMesh(coords, tets)
    pm = H.PrimitiveStorage.from_tets(coords, tets)
    lev = O.Level(om, L)
    off, sz = pm.primitive_offsets(L)
    assert np.array_equal(sz, np.array(lev.sizes["v"] + lev.sizes["e"] + lev.sizes["f"] + lev.sizes["c"]))
    assert np.array_equal(off, np.concatenate([lev.off_v, lev.off_e, lev.off_f, lev.off_c]))
    assert pm.packed_size(L) == lev.size


def test_index_functions():
    """VertexDoFMacroCellIndexingTest / MacroFaceIndexing: exact integer layouts."""
    lib = H.lib()
    for L in (0, 2, 4):
        n = 1 << L
        for z in range(n + 1):
            for y in range(n + 1 - z):
                for x in range(n + 1 - y - z):
                    assert lib.hyb_layout_cell_index(L, x, y, z) == O.cell_index(n, x, y, z)
        # linear in memory order without gaps
        seq = [lib.hyb_layout_cell_index(L, *p) for p in O.tet_points(n + 1)]
        assert seq == list(range(O.tet_size(n + 1)))
        fseq = [lib.hyb_layout_face_index(L, i, j) for j in range(n + 1) for i in range(n + 1 - j)]
        assert fseq == list(range(O.tri_size(n + 1)))


def test_cuboid_generator_matches_oracle():
    pm = H.PrimitiveStorage.cuboid()
    coords, tets = O.mesh_cuboid()
    om = O.MacroMesh(coords, tets)
    for i, v in enumerate(om.cells):
        assert pm.primitive_vertices(3, i) == list(v)


def test_invalid_meshes_are_rejected():
    with pytest.raises(H.HybError):
        H.PrimitiveStorage.from_tets(np.zeros((3, 3)), [(0, 1, 2, 5)])
    with pytest.raises(H.HybError):
        H.PrimitiveStorage.from_tets(np.zeros((4, 3)), [(0, 1, 2, 2)])
    with pytest.raises(H.HybError):
        H.PrimitiveStorage.cuboid(lo=(1, 0, 0), hi=(0, 1, 1))
    with pytest.raises(H.HybError):
        H.PrimitiveStorage.from_gmsh("/nonexistent/mesh.msh")
    assert "cannot open" in H.lib().hyb_last_error().decode()


def test_gmsh_reader(tmp_path):
    p = tmp_path / "two.msh"
    p.write_text(
        "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n5\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n5 1 1 1\n$EndNodes\n"
        "$Elements\n2\n1 4 2 0 0 1 2 3 4\n2 4 2 0 0 2 3 4 5\n$EndElements\n")
    pm = H.PrimitiveStorage.from_gmsh(str(p))
    assert pm.counts() == (5, 9, 7, 2)
    assert pm.primitive_vertices(3, 0) == [0, 1, 2, 3]


@pytest.mark.parametrize("ntan", [2, 3, 5])
def test_spherical_shell_matches_reference_generator(ntan):
    """MeshGenTest.cpp:120-122 counts for (5, 3): 486 vertices, 2724 edges, 4160 faces, 1920 cells."""
    coords, tets = O.mesh_spherical_shell(ntan, 3, 0.55, 1.0)
    om = O.MacroMesh(coords, tets)
    pm = H.PrimitiveStorage.spherical_shell(ntan, 3, 0.55, 1.0)
    assert pm.counts() == (om.nV, om.nE, om.nF, om.nC)
    if ntan == 5:
        assert pm.counts() == (486, 2724, 4160, 1920)
    for i, v in enumerate(om.cells):
        assert pm.primitive_vertices(3, i) == list(v)
    np.testing.assert_allclose(pm.vertex_coords(), coords, rtol=0, atol=1e-15)
    r = np.linalg.norm(coords, axis=1)
    assert np.allclose(np.sort(np.unique(np.round(r, 12))), [0.55, 0.775, 1.0])
    with pytest.raises(H.HybError):
        H.PrimitiveStorage.spherical_shell(4, 3, 0.55, 1.0)  # ntan-1 not a power of two (SHELLMESH_CLASSIC)


def test_python_rejects_unknown_solver_options():
    """Option names are checked before any device work: unknown smoothers and velocity blocks raise."""
    with pytest.raises(ValueError):
        H.GeometricMultigridSolver(None, None, 0, 1, smoother="ilu")
    with pytest.raises(ValueError):
        H.StokesUzawaMultigrid(None, None, 0, 1, velocity_block="stress")


def test_sor_and_viscous_entry_points_validate_arguments():
    """NULL handles are refused with an error code (no device needed)."""
    import ctypes as C
    assert H.lib().hyb_op_smooth_sor(None, None, None, C.c_double(1.0), 1, 1, 0) != 0
    assert H.lib().hyb_p2_full_viscous_apply(None, None, None, 1, 1, 0) != 0
    assert H.lib().hyb_p2_full_viscous_inverse_diagonal(None, None, 1) != 0

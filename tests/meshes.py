"""Small macro meshes used by the tests (defined here by coordinates and tetrahedra)."""

import numpy as np

from oracle import hyteg_oracle as O


def unit_tet():
    return np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float), [(0, 1, 2, 3)]


def tilted_tet():
    return np.array([[0.1, 0.0, 0.2], [1.3, 0.1, 0.0], [0.2, 0.9, 0.3], [0.4, 0.3, 1.1]], float), [(0, 2, 1, 3)]


def pyramid_2():
    # square pyramid split along a base diagonal
    c = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 1.0]], float)
    return c, [(0, 1, 2, 4), (0, 2, 3, 4)]


def pyramid_4():
    # square pyramid with a centre vertex on the base
    c = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 0.0], [0.5, 0.5, 1.0]], float)
    return c, [(0, 1, 4, 5), (1, 2, 4, 5), (2, 3, 4, 5), (3, 0, 4, 5)]


def octahedron_8():
    c = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], float)
    tets = []
    for a in (1, 2):
        for b in (3, 4):
            for d in (5, 6):
                tets.append((0, a, b, d))
    return c, tets


def cube_6():
    return O.mesh_cuboid()


def cube_2x1x1():
    return O.mesh_cuboid(hi=(2.0, 1.0, 1.0), nx=2)


ALL = {
    "unit_tet": unit_tet,
    "tilted_tet": tilted_tet,
    "pyramid_2": pyramid_2,
    "pyramid_4": pyramid_4,
    "octahedron_8": octahedron_8,
    "cube_6": cube_6,
    "cube_2x1x1": cube_2x1x1,
}

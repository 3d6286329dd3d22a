"""Generate tests/golden/ref_p1_kernels.npz from the reference's own kernels.

Runs the reference's generated P1 cell apply, restriction and prolongation kernels and its FEniCS
P1 diffusion form (compiled into oracle/_ref/libhyteg_ref.so by oracle/Makefile) on seeded inputs,
and stores inputs and outputs.  Re-run after `make -C oracle`:

    python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import hyteg_oracle as O  # noqa: E402
from oracle import ref as R  # noqa: E402


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    # element matrices of seeded tetrahedra
    X = rng.uniform(-1.0, 1.0, (6, 4, 3))
    out["elem_X"] = X
    out["elem_A"] = np.stack([R.p1_diffusion_element(x) for x in X])
    # cell apply at level 3 with a seeded stencil and input
    L = 3
    n = 1 << L
    size = O.tet_size(n + 1)
    out["apply_level"] = np.array(L)
    out["apply_stencil"] = rng.uniform(-1.0, 1.0, 15)
    out["apply_src"] = rng.uniform(-1.0, 1.0, size)
    out["apply_dst"] = R.cell_apply(out["apply_src"], L, out["apply_stencil"])
    # restriction level 3 -> 2 and prolongation 2 -> 3 on one cell with neighbour counts
    nc14 = np.array([3, 4, 5, 2, 6, 1, 2, 1, 2, 1, 8, 4, 6, 2], dtype=float)
    out["nc14"] = nc14
    out["restrict_fine"] = rng.uniform(-1.0, 1.0, size)
    out["restrict_coarse"] = R.restrict(out["restrict_fine"], L - 1, nc14)
    out["prolong_coarse"] = rng.uniform(-1.0, 1.0, O.tet_size((n // 2) + 1))
    out["prolong_fine"] = R.prolongate(out["prolong_coarse"], L - 1, nc14)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_p1_kernels.npz"), **out)


if __name__ == "__main__":
    main()

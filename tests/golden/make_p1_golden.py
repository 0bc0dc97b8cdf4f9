"""Write golden fixtures for dense P1 simplex assembly by running PyMHM's own CPU
operators, the ones the reference's GPU test compares ``assemble_p1_batch`` with
(``tests/test_gpu_batch.py``): ``p1_operators`` on ``TriangleMesh.unit_square(3)``
and ``tetra_operators`` (degree 1) on ``TetraMesh.unit_cube(1).submesh(0, 2)`` and on
``submesh(0, 8)`` (165 nodes, the local mesh of the 3-D configuration).

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_p1_golden.py

Basix is replaced by ``_basix_shim`` (degree-one simplex basis).
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if not os.environ.get("PYMHM_SRC"):
    sys.exit("set PYMHM_SRC to the src/ directory of a PyMHM 1.3.2 checkout")
sys.path.insert(0, os.environ["PYMHM_SRC"])
sys.path.insert(0, str(HERE))

import _basix_shim  # noqa: E402

_basix_shim.install()

from pymhm.fem.scalar.operators import p1_operators  # noqa: E402
from pymhm.fem.scalar.tetrahedron import tetra_operators  # noqa: E402
from pymhm.meshes.tetrahedron import TetraMesh  # noqa: E402
from pymhm.meshes.triangle import TriangleMesh  # noqa: E402


def main():
    out = {}
    mesh = TriangleMesh.unit_square(3)
    tensor = np.array([[2.0, 0.2], [0.2, 1.0]])
    a, m, f = p1_operators(mesh, diffusion=tensor, source=3.0)
    out.update(tri_points=mesh.points, tri_cells=mesh.cells, tri_tensor=tensor, tri_source=3.0,
               tri_A=a.toarray(), tri_M=m.toarray(), tri_f=f)
    tetra = TetraMesh.unit_cube(1).submesh(0, 2)
    tensor = np.array([[2.0, 0.2, 0.0], [0.2, 1.0, 0.1], [0.0, 0.1, 3.0]])
    a, m, f = tetra_operators(tetra, degree=1, diffusion=tensor, source=2.5)
    out.update(tet_points=tetra.points, tet_cells=tetra.cells, tet_tensor=tensor, tet_source=2.5,
               tet_A=a.toarray(), tet_M=m.toarray(), tet_f=f)
    # config-4 size: one macro tetrahedron of the unit cube refined with submesh(cell, 8)
    big = TetraMesh.unit_cube(1).submesh(0, 8)
    a, m, f = tetra_operators(big, degree=1, diffusion=tensor, source=2.5)
    out.update(tet8_points=big.points, tet8_cells=big.cells, tet8_A=a.toarray(), tet8_M=m.toarray(), tet8_f=f)
    np.savez_compressed(HERE / "p1_operators.npz", **out)
    print("tri", mesh.points.shape, mesh.cells.shape, "tet", tetra.points.shape, tetra.cells.shape)


if __name__ == "__main__":
    main()

"""NumPy restatement of PyMHM's dense batched P1 simplex assembly (the oracle).

Test infrastructure only: imported by ``tests/``; the library never calls it.
``assemble_p1_batch`` follows ``execution/cuda.py:27-105`` step by step (affine
Jacobians, barycentric gradients, ``vol G K G^T`` element stiffness, the consistent
mass ``vol (1 + delta) / ((d+1)(d+2))`` and the load ``vol f / (d+1)``, scattered
with ``add.at``), with CuPy replaced by NumPy.  It is pinned against the
reference's own CPU operators ``p1_operators`` / ``tetra_operators`` through the
fixtures of ``tests/golden/make_p1_golden.py`` and against the closed-form simplex
moments of the reference's test ``test_resident_p1_assembly_moments``.
"""

from __future__ import annotations

from math import factorial

import numpy as np


def assemble_p1_batch(points, cells, *, diffusion=1.0, source=0.0):
    """``assemble_p1_batch`` (``execution/cuda.py:27-105``) on the host."""
    coordinates = np.asarray(points, dtype=float)
    connectivity = np.asarray(cells)
    count, size, dimension = coordinates.shape
    vertices = coordinates[:, connectivity]
    jacobian = (vertices[:, :, 1:] - vertices[:, :, :1]).swapaxes(-1, -2)
    determinant = np.linalg.det(jacobian)
    bound = np.prod(np.linalg.norm(jacobian, axis=-2), axis=-1)
    if np.any(np.abs(determinant) <= np.finfo(float).eps * bound):
        raise ValueError("degenerate simplex in resident geometry")
    volume = np.abs(determinant) / factorial(dimension)
    reference = np.concatenate((-np.ones((1, dimension)), np.eye(dimension)))
    gradients = np.einsum("ij,btjk->btik", reference, np.linalg.inv(jacobian))
    raw = np.asarray(diffusion, dtype=float)
    if raw.ndim == 0:
        raw = raw * np.eye(dimension)
    tensor = np.broadcast_to(raw, (count, len(connectivity), dimension, dimension))
    forcing = np.broadcast_to(np.asarray(source, dtype=float), (count, len(connectivity)))
    local_stiffness = np.einsum("et,etia,etab,etjb->etij", volume, gradients, tensor, gradients)
    local_mass = (volume[:, :, None, None] * (np.ones((dimension + 1, dimension + 1)) + np.eye(dimension + 1))
                  / ((dimension + 1) * (dimension + 2)))
    stiffness, mass = np.zeros((count, size, size)), np.zeros((count, size, size))
    load = np.zeros((count, size))
    batch_indices = np.arange(count)[:, None, None, None]
    rows = connectivity[None, :, :, None]
    columns = connectivity[None, :, None, :]
    np.add.at(stiffness, (batch_indices, rows, columns), local_stiffness)
    np.add.at(mass, (batch_indices, rows, columns), local_mass)
    np.add.at(load, (np.arange(count)[:, None, None], connectivity[None]),
              (volume * forcing)[:, :, None] / (dimension + 1))
    return stiffness, mass, load

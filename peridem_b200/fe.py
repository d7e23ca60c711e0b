"""Finite-element quadrature data for the strain/stress output
(pdgpu_strain_stress_tri).

The reference computes quadrature-point strain and stress on each
particle's finite-element mesh (DEMModel::output with the Strain_Stress
tag, src/model/dem/demModel.cpp:2026-2072, through fe::getCurrentQuadPoints
and fe::getStrainStress, src/fe/meshUtil.cpp:170-420).  For linear
triangles it places the quadrature points of the reference triangle
(0,0)-(1,0)-(0,1) from fe::TriElem::init (src/fe/triElem.cpp:195-417) and
stores three entries per element: fe::BaseElem::getNumQuadPoints returns
the element's node count (baseElem.cpp:17), whatever the rule.  So with
the one-point rule (order 1, the centroid) entries 1 and 2 of each element
keep the arrays' zero, with the three-point rule (order 2) all three are
written, and the rules of orders 3-5 (4, 6 and 7 points) write past their
element's entries and past the end of the arrays in the reference; only
orders 1 and 2 are supported here.  The device kernel takes the points
from the host and evaluates the shape functions N = (1 - xi - eta, xi, eta)
at them itself.
"""
from typing import Dict, List, Tuple

import numpy as np

# vtk cell types of a linear triangle and tetrahedron (util::vtk_type_*)
VTK_TRIANGLE = 5
VTK_TETRA = 10

# reference-triangle quadrature points per order, in the reference's order
TRI_POINTS: Dict[int, List[Tuple[float, float]]] = {
    1: [(1. / 3., 1. / 3.)],
    2: [(1. / 6., 1. / 6.), (2. / 3., 1. / 6.), (1. / 6., 2. / 3.)],
}
ENTRIES_PER_TRIANGLE = 3  # quadrature entries the reference stores per element


def tri_points(order: int) -> np.ndarray:
    """[nq, 2] reference-triangle points of a quadrature order (1 or 2)."""
    if order not in TRI_POINTS:
        raise ValueError(f"triangle quadrature order {order}: 1 and 2 are supported (the reference's "
                         f"rules of order 3-5 write past its arrays)")
    return np.array(TRI_POINTS[order], dtype=np.float64)


def grid_triangles(x: np.ndarray, h: float) -> np.ndarray:
    """Linear triangles over a square grid of spacing h (nodes x [n, 2|3]):
    every grid square whose four corners are nodes becomes two triangles
    (counter-clockwise, split along alternating diagonals).  Returns
    connectivity [m, 3] (node ids)."""
    ij = np.round(np.asarray(x)[:, :2] / h).astype(np.int64)
    index = {(int(a), int(b)): k for k, (a, b) in enumerate(ij)}
    tris = []
    for (a, b), k0 in sorted(index.items()):
        k1, k2, k3 = index.get((a + 1, b)), index.get((a + 1, b + 1)), index.get((a, b + 1))
        if k1 is None or k2 is None or k3 is None:
            continue
        if (a + b) % 2 == 0:
            tris += [(k0, k1, k2), (k0, k2, k3)]
        else:
            tris += [(k0, k1, k3), (k1, k2, k3)]
    return np.array(tris, dtype=np.int64).reshape(-1, 3)


def grid_tetrahedra(x: np.ndarray, h: float) -> np.ndarray:
    """Linear tetrahedra over a cubic grid of spacing h (nodes x [n, 3]):
    every grid cube whose eight corners are nodes becomes six tetrahedra
    around its main diagonal (one per order of the three axis steps).
    Returns connectivity [m, 4] (node ids)."""
    ijk = np.round(np.asarray(x)[:, :3] / h).astype(np.int64)
    index = {tuple(int(v) for v in p): k for k, p in enumerate(ijk)}
    steps = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
    tets = []
    for p0, k0 in sorted(index.items()):
        corners = [(p0[0] + a, p0[1] + b, p0[2] + c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
        if any(q not in index for q in corners):
            continue
        for order in steps:
            path, cur = [k0], list(p0)
            for ax in order:
                cur[ax] += 1
                path.append(index[tuple(cur)])
            tets.append(path)
    return np.array(tets, dtype=np.int64).reshape(-1, 4)

"""VTK output from the device (pmg_write_vtk) against the reference's
TOutput3D::WriteVtk (src/FE/Output3D.C:1773-2140).

The drop-in driver (oracle/ref/dropin_driver.C, vtk=1) solves the same system
with the reference's TSystemCD3D and with TPmgSystemCD3D, then writes the
reference's solution through TOutput3D::WriteVtk and ours through
pmg_write_vtk from the device-resident solution.  The reference numbers the
vertices by memory address, so the files are compared through coordinates:
the same points, the same cells (corner order included), the same cell types,
and point values equal to the 7 printed digits (the solutions agree to
1e-10, both solved to |r| <= 1e-14 |r0|).  A second test checks the written
values against the solution vector on this library's own hierarchy."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "oracle", "_ref", "pmg_dropin")


def parse_vtk(path):
    with open(path) as f:
        tok = f.read().split()
    out, i, section = {}, 0, None
    while i < len(tok):
        t = tok[i]
        if t == "POINTS":
            n = int(tok[i + 1])
            out["points"] = np.array(tok[i + 3:i + 3 + 3 * n], dtype=float).reshape(n, 3)
            i += 3 + 3 * n
        elif t == "CELLS":
            n, size = int(tok[i + 1]), int(tok[i + 2])
            flat = np.array(tok[i + 3:i + 3 + size], dtype=int)
            cells, k = [], 0
            for _ in range(n):
                m = flat[k]
                cells.append(tuple(flat[k + 1:k + 1 + m]))
                k += 1 + m
            out["cells"] = cells
            i += 3 + size
        elif t == "CELL_TYPES":
            n = int(tok[i + 1])
            out["types"] = np.array(tok[i + 2:i + 2 + n], dtype=int)
            i += 2 + n
        elif t in ("POINT_DATA", "CELL_DATA"):
            section = t
            i += 2
        elif t == "SCALARS":  # SCALARS name type [components] LOOKUP_TABLE default values
            j = i + 3 if tok[i + 3] == "LOOKUP_TABLE" else i + 4
            n = len(out["points"]) if section == "POINT_DATA" else len(out["cells"])
            vals = np.array(tok[j + 2:j + 2 + n], dtype=float)
            if section == "POINT_DATA":
                out["name"], out["values"] = tok[i + 1], vals
            else:
                out["cell_" + tok[i + 1]] = vals
            i = j + 2 + n
        else:
            i += 1
    return out


def key(p):
    return tuple(np.round(p, 9))


def by_coordinates(v):
    pts = [key(p) for p in v["points"]]
    vals = dict(zip(pts, v["values"]))
    cells = sorted(tuple(pts[j] for j in c) for c in v["cells"])
    return vals, cells


@pytest.mark.parametrize("order,geo,problem", [(1, "Wuerfel", "laplace"), (2, "Wuerfel", "cd"),
                                               (2, "SixTetras", "laplace"), (1, "SixTetras", "cd")])
def test_vtk_matches_reference_writer(tmp_path, order, geo, problem):
    if not os.path.exists(EXE):
        pytest.fail("oracle/_ref/pmg_dropin missing: build the checker (make -C oracle/ref dropin)")
    args = [EXE, str(tmp_path), f"order={order}", f"geo={geo}", f"problem={problem}", "levels=3", "coarse_steps=1",
            "red=1e-14", "vtk=1"]
    p = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0 and "vtk status=0" in p.stdout, p.stdout[-2000:] + p.stderr[-2000:]
    ref, ours = parse_vtk(tmp_path / "ref.vtk"), parse_vtk(tmp_path / "pmg.vtk")
    assert len(ref["points"]) == len(ours["points"]) and len(ref["cells"]) == len(ours["cells"])
    assert np.array_equal(ref["types"], ours["types"])
    rv, rc = by_coordinates(ref)
    ov, oc = by_coordinates(ours)
    assert rc == oc
    assert np.array_equal(ref["cell_RegionID"], ours["cell_RegionID"])  # both in the collection's cell order
    assert rv.keys() == ov.keys()
    scale = max(abs(v) for v in rv.values())
    for k, v in rv.items():
        assert abs(ov[k] - v) <= 1e-6 * max(abs(v), 1e-3 * scale), (k, v, ov[k])


def test_vtk_values_are_the_solution(pmg, tmp_path):
    levels = pmg.struct_hierarchy(pmg.Q2_HEX, 8, 2)
    h = pmg.Handle(2)
    h.set_coefficients(pmg.coeff(kind=pmg.COEF_CONST, eps=1e-2, b=(1.0, 0.5, 0.25), f=1.0))
    pmg.load_hierarchy(h, levels, dirichlet=lambda x, y, z: x + y * z)
    h.assemble(-1, pmg.FORM_SUPG, copy_out=False)
    h.solve()
    x = h.get_solution()
    F = levels[-1]
    h.write_vtk(tmp_path / "u.vtk", name="u")
    v = parse_vtk(tmp_path / "u.vtk")
    assert v["name"] == "u" and len(v["cells"]) == F["elem_dof"].size // 27 and set(v["types"]) == {12}
    assert not v["cell_RegionID"].any()
    # the Q2 vertices are the lattice nodes with even indices: 9^3 of the 17^3 dofs
    assert len(v["points"]) == 9 ** 3
    dof_at = {key(p): d for d, p in enumerate(F["dof_xyz"].reshape(-1, 3))}
    for p, val in zip(v["points"], v["values"]):
        d = dof_at[key(p)]
        assert abs(val - x[d]) <= 5e-7 * max(abs(x[d]), 1e-12)
    # a host vector instead of the device solution
    h.write_vtk(tmp_path / "w.vtk", name="w", values=2.0 * x)
    w = parse_vtk(tmp_path / "w.vtk")
    assert np.allclose(w["values"], 2.0 * v["values"], rtol=1e-6, atol=0)
    h.close()

"""Boundary parity: Problem/YAML parsing, mesh indexing and Ke.

Golden values come from the reference's own modules (tests/golden/boundary.npz,
made by tests/golden/make_golden.py); the structural checks restate the
reference's tests (tests/test_material.py, test_mesh.py, test_problem.py).
Everything here must be bit-exact.
"""

import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO, golden
from toptimization_b200 import material, mesh
from toptimization_b200.problem import Problem, load_problem, problem_from_dict

B = golden("boundary")


def make_problem(nelx=4, nely=3, **kw):
    args = dict(name="t", dim=2, nelx=nelx, nely=nely, nelz=1, E=1.0, nu=0.3, E_min=1e-9,
                fixed_dofs=np.array([0, 1]),
                force_dofs=np.array([2 * (nelx + 1) * (nely + 1) - 1]),
                force_values=np.array([-1.0]), volfrac=0.5, penalty=3.0, rmin=1.5,
                filter_type="density", max_iter=100, tol=0.01, move_limit=0.2,
                max_cg_iter=500, cg_tol=1e-8, preconditioner="jacobi",
                output_dir=Path("results"), save_interval=10, output_format="png")
    args.update(kw)
    return Problem(**args)


# ---------------------------------------------------------------- Ke
def test_ke_bit_exact_vs_reference():
    assert np.array_equal(material.compute_Ke_2d(1.0, 0.3), B["Ke2d"])
    assert np.array_equal(material.compute_Ke_3d(1.0, 0.3), B["Ke3d"])
    assert np.array_equal(material.compute_Ke_2d(2.0, 0.25), B["Ke2d_E2_nu025"])


def test_ke_known_entry():
    # k(0,0) of the unit Q4 plane-stress element, E=1, nu=0.3: 0.4945054945...
    assert material.compute_Ke_2d()[0, 0] == pytest.approx(0.49450549450549447, abs=1e-15)


def test_ke_structure():
    Ke = material.compute_Ke_2d()
    np.testing.assert_allclose(Ke, Ke.T, atol=1e-12)
    assert np.linalg.eigvalsh(Ke).min() > -1e-10
    assert np.linalg.matrix_rank(Ke, tol=1e-10) == 5          # 3 rigid-body modes
    np.testing.assert_allclose(material.compute_Ke_2d(2.0), 2 * Ke, rtol=1e-10)
    Ke3 = material.compute_Ke_3d()
    assert Ke3.shape == (24, 24)
    assert np.linalg.matrix_rank(Ke3, tol=1e-8) == 18


def test_regularized_inverse_matches_reference():
    inv, alpha = material.regularized_inverse(B["Ke2d"])
    assert alpha == float(B["Ke2d_alpha"])
    np.testing.assert_array_equal(inv, B["Ke2d_inv"])


# ---------------------------------------------------------------- mesh
def test_edof_bit_exact():
    p = make_problem(4, 3)
    e = mesh.build_edof_2d(p)
    assert e.dtype == np.int32 and e.shape == (12, 8)
    np.testing.assert_array_equal(e, B["edof_4x3"])
    np.testing.assert_array_equal(mesh.element_centers_2d(p), B["centers_4x3"])


def test_edof_element_zero_and_sharing():
    p = make_problem(4, 3)
    e = mesh.build_edof_2d(p)
    n1, n2, n3, n4 = 0, 4, 5, 1
    np.testing.assert_array_equal(e[0], [2 * n1, 2 * n1 + 1, 2 * n2, 2 * n2 + 1,
                                         2 * n3, 2 * n3 + 1, 2 * n4, 2 * n4 + 1])
    assert all(len(set(row)) == 8 for row in e)
    assert len(set(e[0]) & set(e[3])) == 4      # horizontal neighbours share 2 nodes
    assert e.min() >= 0 and e.max() < 2 * 5 * 4


def test_edof_3d_layout():
    p = make_problem(3, 2, dim=3, nelz=2)
    e = mesh.build_edof_3d(p)
    assert e.shape == (12, 24)
    # element 0 corner 6 = node (1,1,1)
    n = (1 * 3 + 1) * 3 + 1
    assert list(e[0, 18:21]) == [3 * n, 3 * n + 1, 3 * n + 2]


def test_fixed_node_mask_and_force_vector():
    p = make_problem(4, 3, fixed_dofs=np.array([0, 1, 3, 38]),
                     force_dofs=np.array([5, 5, 3]), force_values=np.array([1.0, 2.0, 7.0]))
    m = mesh.fixed_node_mask(p)
    assert m.dtype == np.uint8 and m.shape == (20,)
    assert m[0] == 3 and m[1] == 2 and m[19] == 1 and m[2:19].sum() == 0
    f = mesh.force_vector(p)
    assert f[5] == 3.0 and f[3] == 0.0         # duplicates add, fixed DOFs zeroed
    assert f.sum() == 3.0


# ---------------------------------------------------------------- YAML
@pytest.mark.parametrize("name", ["specs_mix", "edges_right_left", "region_default"])
def test_parser_coverage_bit_exact(name):
    """Files exercising every 2D node-spec kind, parsed by the reference's
    load_problem when the fixtures were made."""
    pr = load_problem(REPO / "tests" / "golden" / "yaml" / f"{name}.yaml")
    tag = f"yaml_{name}"
    np.testing.assert_array_equal(pr.fixed_dofs, B[f"{tag}__fixed"])
    np.testing.assert_array_equal(pr.force_dofs, B[f"{tag}__fdofs"])
    np.testing.assert_array_equal(pr.force_values, B[f"{tag}__fvals"])
    assert [pr.nelx, pr.nely, pr.n_nodes, pr.n_dofs, pr.n_elem] == list(B[f"{tag}__sizes"])


@pytest.mark.parametrize("name", ["mbb_60x20", "cantilever_400x200", "bridge_2048x1024"])
def test_config_examples_bit_exact(name):
    pr = load_problem(REPO / "examples" / f"{name}.yaml")
    tag = f"ex_{name}"
    np.testing.assert_array_equal(pr.fixed_dofs, B[f"{tag}__fixed"])
    np.testing.assert_array_equal(pr.force_dofs, B[f"{tag}__fdofs"])
    np.testing.assert_array_equal(pr.force_values, B[f"{tag}__fvals"])


def test_config_boundary_conditions():
    mbb = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    assert len(mbb.fixed_dofs) == 22 and 2521 in mbb.fixed_dofs
    assert list(mbb.force_dofs) == [41] and list(mbb.force_values) == [-1.0]
    cant = load_problem(REPO / "examples" / "cantilever_400x200.yaml")
    assert len(cant.fixed_dofs) == 402 and list(cant.force_dofs) == [161001]
    br = load_problem(REPO / "examples" / "bridge_2048x1024.yaml")
    assert list(br.fixed_dofs) == [0, 1, 4198400, 4198401]
    assert len(br.force_dofs) == 2049 and br.force_values.sum() == pytest.approx(-1.0, abs=1e-12)
    assert br.n_dofs == 4200450 and br.n_elem == 2097152


CANTILEVER_YAML = """\
problem: {name: "Test Cantilever", dimension: 2}
domain: {nelx: 10, nely: 5}
material: {E: 1.0, nu: 0.3, E_min: 1.0e-9}
boundary_conditions:
  fixed:
    - nodes: {type: "edge", edge: "left"}
      dofs: ["x", "y"]
loads:
  - nodes: {type: "point", location: [10, 2]}
    force: [0.0, -1.0]
optimization: {volume_fraction: 0.5, penalty: 3.0, filter_radius: 1.5,
               filter_type: "density", max_iterations: 100, tolerance: 0.01,
               move_limit: 0.2}
solver: {max_cg_iterations: 500, cg_tolerance: 1.0e-8, preconditioner: "jacobi"}
output: {directory: "results/test", save_interval: 5, format: "png"}
"""


def _write(text):
    fh = tempfile.NamedTemporaryFile("w", suffix=".yaml", delete=False)
    fh.write(text)
    fh.close()
    return Path(fh.name)


def test_load_problem_cantilever():
    p = load_problem(_write(CANTILEVER_YAML))
    assert p.name == "Test Cantilever" and p.dim == 2
    assert (p.nelx, p.nely, p.n_nodes, p.n_dofs, p.n_elem) == (10, 5, 66, 132, 50)
    assert len(p.fixed_dofs) == 12
    assert p.fixed_dofs.min() >= 0 and p.fixed_dofs.max() < p.n_dofs
    np.testing.assert_array_equal(np.union1d(p.free_dofs, p.fixed_dofs), np.arange(132))
    assert np.intersect1d(p.free_dofs, p.fixed_dofs).size == 0
    assert p.volfrac == pytest.approx(0.5) and p.precision == "fp64"


def test_defaults_and_extensions():
    raw = {"domain": {"nelx": 4, "nely": 2},
           "loads": [{"nodes": {"type": "point", "corner": "top-right"}, "force": [1, 0]}],
           "solver": {"preconditioner": "nodal_block_jacobi", "precision": "mixed",
                      "inner_tolerance": 1e-3}}
    p = problem_from_dict(raw)
    assert p.cg_tol == 1e-6 and p.max_cg_iter == 2000 and p.rmin == 1.5
    assert p.move_limit == 0.2 and p.penalty == 3.0 and p.E_min == 1e-9
    assert p.preconditioner == "nodal_block_jacobi" and p.precision == "mixed"
    assert p.inner_tol == 1e-3
    assert list(p.force_dofs) == [2 * (4 * 3 + 2)]


@pytest.mark.parametrize("bad, msg", [
    ({"problem": {"dimension": 4}}, "dimension"),
    ({"optimization": {"filter_type": "x"}}, "filter_type"),
    ({"solver": {"preconditioner": "ilu"}}, "preconditioner"),
    ({"solver": {"precision": "fp16"}}, "precision"),
    ({"output": {"format": "gif"}}, "format"),
    ({"loads": [{"nodes": {"type": "point", "location": [0, 0]}, "force": [0.0, 0.0]}]},
     "No nonzero forces"),
    ({"loads": [{"nodes": {"type": "edge", "edge": "middle"}, "force": [0.0, 1.0]}]},
     "Unknown edge"),
    ({"loads": [{"nodes": {"type": "point", "corner": "nowhere"}, "force": [0.0, 1.0]}]},
     "corner"),
    ({"loads": [{"nodes": {"type": "point", "corner": "top-left"}, "force": [1.0]}]},
     "force vector length"),
    ({"boundary_conditions": {"fixed": [{"nodes": {"type": "edge", "edge": "left"},
                                         "dofs": ["z"]}]}}, "not valid for 2D"),
])
def test_validation_errors(bad, msg):
    raw = {"domain": {"nelx": 4, "nely": 2},
           "loads": [{"nodes": {"type": "point", "corner": "top-right"}, "force": [0, -1]}]}
    raw.update(bad)
    with pytest.raises(ValueError, match=msg):
        problem_from_dict(raw)


def test_point_location_clamped_and_region():
    raw = {"domain": {"nelx": 4, "nely": 2},
           "boundary_conditions": {"fixed": [{"nodes": {"type": "region", "x": [1, 2],
                                                        "y": [0, 1]}, "dofs": ["y"]}]},
           "loads": [{"nodes": {"type": "point", "location": [99, 99]}, "force": [0, -1]}]}
    p = problem_from_dict(raw)
    assert list(p.force_dofs) == [2 * (4 * 3 + 2) + 1]
    assert list(p.fixed_dofs) == sorted(2 * n + 1 for n in (3, 4, 6, 7))


@pytest.mark.parametrize("bad, msg", [
    ({"loads": [{"nodes": {"type": "edge", "edge": "left"}, "force": [0.0, 1.0, 0.0]}]},
     "Unknown node spec type 'edge' for dim=3"),
    ({"loads": [{"nodes": {"type": "face", "face": "middle"}, "force": [0.0, 1.0, 0.0]}]},
     "Unknown face"),
    ({"loads": [{"nodes": {"type": "point", "corner": "top-right"}, "force": [0.0, 1.0, 0.0]}]},
     "Unknown 3D corner"),
    ({"loads": [{"nodes": {"type": "face", "face": "top"}, "force": [0.0, 1.0]}]},
     "force vector length 2 != dim 3"),
    ({"boundary_conditions": {"fixed": [{"nodes": {"type": "face", "face": "left"},
                                         "dofs": ["w"]}]}}, "Unknown DOF label"),
])
def test_validation_errors_3d(bad, msg):
    """The reference's 3D parser rules (problem.py:231-263,281-367): faces only
    in 3D, edges only in 2D, the four named 3D corners, force length = dim."""
    raw = {"problem": {"dimension": 3}, "domain": {"nelx": 4, "nely": 2, "nelz": 3},
           "loads": [{"nodes": {"type": "point", "corner": "back-bottom-right"},
                      "force": [0, -1, 0]}]}
    raw.update(bad)
    with pytest.raises(ValueError, match=msg):
        problem_from_dict(raw)


def test_face_in_2d_rejected_and_3d_defaults():
    raw = {"domain": {"nelx": 4, "nely": 2},
           "loads": [{"nodes": {"type": "face", "face": "top"}, "force": [0, -1]}]}
    with pytest.raises(ValueError, match="Unknown node spec type 'face' for dim=2"):
        problem_from_dict(raw)
    # 3D: nelz defaults to 1, fixed DOFs default to x and y only, the 3D
    # location is not clamped, z ranges default to the whole depth
    raw = {"problem": {"dimension": 3}, "domain": {"nelx": 2, "nely": 1},
           "boundary_conditions": {"fixed": [{"nodes": {"type": "region", "x": [0, 0],
                                                        "y": [0, 0]}}]},
           "loads": [{"nodes": {"type": "point", "location": [2, 1, 1]}, "force": [0, 0, 1]}]}
    p = problem_from_dict(raw)
    assert p.nelz == 1 and p.n_nodes == 3 * 2 * 2 and p.n_dofs == 36
    assert list(p.fixed_dofs) == [0, 1, 3, 4]          # nodes (0,0,0), (0,0,1): x, y
    assert list(p.force_dofs) == [3 * ((2 * 2 + 1) * 2 + 1) + 2]

"""Host-side checks of the batched-design engine: the seeded workload
generator and the workspace-size queries of the C ABI (no GPU needed)."""

import numpy as np
import pytest

from toptimization_b200 import _lib
from toptimization_b200.batch import design_struct, footprint_bytes, random_designs


@pytest.fixture(scope="module")
def lib(tpo_built):
    return _lib.load()


def test_random_designs_are_seeded_and_in_range():
    a = random_designs(64, seed=7)
    b = random_designs(64, seed=7)
    assert [p.name for p in a] == [p.name for p in b]
    assert [list(p.force_dofs) for p in a] == [list(p.force_dofs) for p in b]
    assert [p.name for p in random_designs(64, seed=8)] != [p.name for p in a]
    for p in a:
        assert 64 <= p.nelx <= 512
        assert p.nely in {max(1, round(p.nelx / k)) for k in (1, 2, 3)}
        assert 0.3 <= p.volfrac <= 0.6 and 1.5 <= p.rmin <= 4.0
        assert p.precision == "mixed" and p.max_iter == 50
        assert p.E_min == 1e-9 and p.penalty == 3.0 and p.nu == 0.3
    fams = {p.name.split()[0] for p in a}
    assert fams == {"mbb", "cantilever", "bridge"}


def test_boundary_conditions_and_load_position():
    for p in random_designs(60, seed=1, nelx_range=(64, 200)):
        fam = p.name.split()[0]
        nx, ny = p.nelx, p.nely
        (dof,) = p.force_dofs
        node, axis = divmod(int(dof), 2)
        ix, iy = divmod(node, ny + 1)
        assert axis == 1 and p.force_values[0] == -1.0
        if fam == "cantilever":
            assert ix == nx and round(0.1 * ny) <= iy <= round(0.9 * ny)
            assert len(p.fixed_dofs) == 2 * (ny + 1)
        else:
            assert iy == ny and round(0.1 * nx) <= ix <= round(0.9 * nx)
            if fam == "mbb":
                fixed = set(int(d) for d in p.fixed_dofs)
                assert len(fixed) == (ny + 1) + 1
                assert 2 * (nx * (ny + 1)) + 1 in fixed      # bottom-right y
                assert all(2 * iy0 in fixed for iy0 in range(ny + 1))  # left edge x
            else:
                assert sorted(int(d) for d in p.fixed_dofs) == [
                    0, 1, 2 * nx * (ny + 1), 2 * nx * (ny + 1) + 1]


def test_workspace_queries(lib):
    assert lib.tpo_batch_workspace_bytes(0) == 0
    assert lib.tpo_batch_workspace_bytes(64) > lib.tpo_batch_workspace_bytes(1) > 0
    small, big = random_designs(2, seed=3, nelx_range=(64, 64))[0], None
    p = random_designs(1, seed=4, nelx_range=(400, 400))[0]
    assert footprint_bytes(p) > footprint_bytes(small)
    layout = _lib.TpoBatchLayout()
    n = lib.tpo_batch_design_workspace_bytes(design_struct(p), layout)
    assert n == footprint_bytes(p)
    offs = [layout.rho, layout.rho_phys, layout.u, layout.hist]
    assert all(o % 256 == 0 for o in offs) and offs == sorted(offs)
    assert layout.rho_phys - layout.rho >= 8 * p.n_elem
    assert layout.hist - layout.u >= 8 * p.n_dofs
    # footprint ~ 84 N + 40 E bytes in the estimate used for admission; the
    # padded layout adds the pad rows
    assert n < 200 * p.n_dofs + 80 * p.n_elem
    bad = design_struct(p)
    bad.rmin = 17.0
    assert lib.tpo_batch_design_workspace_bytes(bad, None) == 0


def test_poisson_stream_is_seeded():
    from toptimization_b200.serve import poisson_stream
    a = poisson_stream(400, rate=50.0, seed=5)
    b = poisson_stream(400, rate=50.0, seed=5)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    t = np.array([r.arrival for r in a])
    assert np.all(np.diff(t) > 0)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 50.0) < 0.2 / 50.0
    assert all(64 <= r.problem.nelx <= 1024 for r in a)

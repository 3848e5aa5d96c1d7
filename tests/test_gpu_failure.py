"""Failure detection without a GPU fault: a stencil launch is made to withhold
the bulk copies of one column group (tpo_test_withhold_stage), so that the
bounded mbarrier waits for it run out. The kernel then flags the timeout,
lets the copies it did start land, and returns; the blocking solve reports
TPO_ERR_TIMEOUT, the asynchronous one TPO_SOLVE_TIMEOUT in its device
record, and the device still answers: the next solves on the same workspace
give the same bits as on a fresh one.
"""

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from toptimization_b200 import _lib  # noqa: E402
from toptimization_b200.fem.solver import PCGSolver  # noqa: E402
from toptimization_b200.material import compute_Ke_2d, regularized_inverse  # noqa: E402
from toptimization_b200.mesh import fixed_node_mask, force_vector  # noqa: E402
from toptimization_b200.problem import load_problem  # noqa: E402

TPO_ERR_TIMEOUT = 6


def _setup(pre, prec):
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    Ke = compute_Ke_2d(pr.E, pr.nu)
    inv, alpha = regularized_inverse(Ke)
    _lib.ensure_stiffness(Ke, inv, alpha)
    dev = torch.device("cuda", 0)
    f_np = force_vector(pr)
    f = torch.from_numpy(f_np).to(dev)
    fixed = torch.from_numpy(fixed_node_mask(pr)).to(dev)
    rho = torch.full((pr.n_elem,), 0.5, dtype=torch.float64, device=dev)

    def solver():
        return PCGSolver(pr.nelx, pr.nely, pr.E_min, pr.penalty, float(f_np @ f_np),
                         preconditioner=pre, precision=prec, max_iter=3000, tol=1e-8,
                         device=dev)
    return pr, dev, f, fixed, rho, solver


@pytest.mark.parametrize("pre,prec", [("jacobi", "fp64"), ("nodal_block_jacobi", "mixed")])
def test_withheld_copies_time_out_and_the_device_recovers(tpo_built, pre, prec):
    pr, dev, f, fixed, rho, solver = _setup(pre, prec)
    s = solver()
    u = torch.zeros(pr.n_dofs, dtype=torch.float64, device=dev)
    _lib.check(_lib.load().tpo_test_withhold_stage(1))
    with pytest.raises(_lib.TpoError) as e:
        s.solve(rho, f, fixed, u, warm_start=False)
    assert e.value.code == TPO_ERR_TIMEOUT
    # the device answers, and the same workspace solves as a fresh one does
    u.zero_()
    info = s.solve(rho, f, fixed, u, warm_start=False)
    u_ref = torch.zeros_like(u)
    info_ref = solver().solve(rho, f, fixed, u_ref, warm_start=False)
    assert info.status == info_ref.status == "converged"
    assert info.iters == info_ref.iters and torch.equal(u, u_ref)


def test_withheld_copies_in_the_asynchronous_solve(tpo_built):
    pr, dev, f, fixed, rho, solver = _setup("jacobi", "fp64")
    s = solver()
    u = torch.zeros(pr.n_dofs, dtype=torch.float64, device=dev)
    res = s.result_buffer()
    _lib.check(_lib.load().tpo_test_withhold_stage(1))
    s.solve_async(rho, f, fixed, u, res, warm_start=False)
    torch.cuda.synchronize()
    assert PCGSolver.decode(res).status == "timeout"
    u.zero_()
    s.solve_async(rho, f, fixed, u, res, warm_start=False)
    torch.cuda.synchronize()
    assert PCGSolver.decode(res).status == "converged"

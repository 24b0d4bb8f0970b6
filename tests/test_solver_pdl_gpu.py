"""Launch forms of the solve against one another; the arithmetic is the same, so the solves must agree
bit for bit:
- the V-cycle's and the CG iteration's kernels launched as programmatic dependents of their
  predecessors (each reads what the kernel before it wrote only after griddepcontrol.wait) against
  plain stream-ordered launches, inside and outside the V-cycle's CUDA graph;
- the mixed-precision CG iterations run by a graph with a device-side while loop against the
  host-driven loop;
- the V-cycle's uniform tail (restriction into the small uniform levels, their V-cycle,
  prolongation back) as one single-CTA launch against one launch per step."""
import os

import pytest

torch = pytest.importorskip("torch")

import anitowave_adaptive_b200 as aw  # noqa: E402

pytestmark = pytest.mark.gpu


def _solve(prob, precision, tol, no_pdl, no_graph=False, no_devloop=False, no_tail=False):
    env = {"AW_NO_PDL": no_pdl, "AW_NO_GRAPH": no_graph, "AW_NO_DEVLOOP": no_devloop, "AW_NO_DENSE_TAIL": no_tail}
    for k, v in env.items():
        if v:
            os.environ[k] = "1"
    try:
        sv = aw.Solver(prob.grid, precision=precision, tolerance=tol, max_cycles=60)
    finally:
        for k in env:
            os.environ.pop(k, None)
    sv.setup(prob.fluid)
    dt = torch.float64 if precision == aw.PRECISION_MIXED else torch.float32
    p = torch.zeros(prob.b.numel(), dtype=dt, device="cuda")
    cyc, rel, st = sv.solve(prob.b, p, raise_on_error=False)
    torch.cuda.synchronize()
    sv.close()
    return cyc, rel, p.cpu()


@pytest.mark.parametrize("N,levels", [(128, 4), (64, 3)])
@pytest.mark.parametrize("precision,tol", [(aw.PRECISION_MIXED, 1e-6), (aw.PRECISION_FP32, 1e-5),
                                           (aw.PRECISION_FP32_PCG, 1e-5)])
def test_dependent_launches_match_plain_launches(N, levels, precision, tol):
    from anitowave_adaptive_b200 import poisson as pz
    prob = pz.build_problem(N, levels=levels)
    c1, r1, p1 = _solve(prob, precision, tol, no_pdl=False)
    c0, r0, p0 = _solve(prob, precision, tol, no_pdl=True)
    assert c1 == c0 and r1 == r0, (c1, r1, c0, r0)
    assert torch.equal(p1, p0)
    # outside a CUDA graph too (stream launches)
    c2, r2, p2 = _solve(prob, precision, tol, no_pdl=False, no_graph=True)
    assert c2 == c0 and r2 == r0 and torch.equal(p2, p0)
    prob.grid.close()


@pytest.mark.parametrize("N,levels,tol", [(128, 4, 1e-6), (128, 4, 1e-9), (64, 3, 1e-8)])
def test_device_loop_matches_host_loop(N, levels, tol):
    from anitowave_adaptive_b200 import poisson as pz
    prob = pz.build_problem(N, levels=levels)
    c1, r1, p1 = _solve(prob, aw.PRECISION_MIXED, tol, no_pdl=False)
    c0, r0, p0 = _solve(prob, aw.PRECISION_MIXED, tol, no_pdl=False, no_devloop=True)
    assert c1 == c0 and r1 == r0, (c1, r1, c0, r0)
    assert torch.equal(p1, p0)
    prob.grid.close()


@pytest.mark.parametrize("N,levels", [(128, 4), (64, 3), (256, 4)])
@pytest.mark.parametrize("precision,tol", [(aw.PRECISION_MIXED, 1e-6), (aw.PRECISION_FP32, 1e-5)])
def test_dense_tail_matches_level_launches(N, levels, precision, tol):
    from anitowave_adaptive_b200 import poisson as pz
    prob = pz.build_problem(N, levels=levels)
    c1, r1, p1 = _solve(prob, precision, tol, no_pdl=False)
    c0, r0, p0 = _solve(prob, precision, tol, no_pdl=False, no_tail=True)
    assert c1 == c0 and r1 == r0, (c1, r1, c0, r0)
    assert torch.equal(p1, p0)
    prob.grid.close()

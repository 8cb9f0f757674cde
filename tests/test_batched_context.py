"""A batched context (several designs, every launch carrying all of them) gives each design exactly
the result of solving it alone: same solution bits, same iteration counts, same C_H, in both
precisions, at a small grid and at the benchmark grid n = 64. A design that fails inside a batch
(a non-finite density never certifies and takes the restarts the reference would) stops alone; its
batch-mates are left untouched by its later attempts and keep their stand-alone results.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes, skipped
    pytest.skip("CUDA device required", allow_module_level=True)


def dev(x):
    return torch.tensor(np.ascontiguousarray(x), device="cuda", dtype=torch.float64)


def alone(pkg, n, a, alpha, precision):
    op = pkg.Operator(n, 6, *pkg.PAPER_MEDIUM, precision=precision)
    op.set_material(dev(a))
    op.set_alpha(alpha)
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos, st = op.solve(np.eye(6), 1e-8, u)
    C = op.effective_tensor(u)
    torch.cuda.synchronize()
    return u.cpu(), [i["iterations"] for i in infos], C.cpu(), st


def batched(pkg, n, designs, precision):
    D = len(designs)
    s = torch.cuda.current_stream()
    op = pkg.BatchedOperator(n, D, 6, *pkg.PAPER_MEDIUM, precision=precision)
    for d, (a, alpha) in enumerate(designs):
        op.set_material(d, dev(a), s)
        op.set_alpha(d, alpha, s)
    u = torch.zeros((6 * D, 3 * n ** 3), dtype=torch.float64, device="cuda")
    op.solve_async(D, np.eye(6), 1e-8, u, s)
    infos, st = op.wait(D, s)
    Cs = torch.empty((D, 6, 6), dtype=torch.float64, device="cuda")
    for d in range(D):
        op.effective_tensor(d, u[6 * d:6 * d + 6], Cs[d], s)
    torch.cuda.synchronize()
    return u.cpu(), infos, Cs.cpu(), st


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n,emins", [(16, (1e-4, 1e-6, 1e-9)), (64, (1e-6, 1e-4))])
def test_batched_designs_are_bitwise_their_single_solves(pkg, precision, n, emins):
    designs = [(pkg.baseline_design(n, 40 + k, emin), alpha)
               for k, (emin, alpha) in enumerate(zip(emins, (0.5, 0.75, 0.875)))]
    ub, infos, Cb, st = batched(pkg, n, designs, precision)
    for d, (a, alpha) in enumerate(designs):
        u1, its1, C1, st1 = alone(pkg, n, a, alpha, precision)
        mine = infos[6 * d:6 * d + 6]
        assert st1 == 0, (d, precision, its1)
        assert all(i["converged"] for i in mine), (d, precision, mine)
        assert [i["iterations"] for i in mine] == its1, (d, precision)
        assert torch.equal(ub[6 * d:6 * d + 6], u1), (d, precision)
        assert torch.equal(Cb[d], C1), (d, precision)
    assert st == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_failing_design_stops_alone(pkg, precision):
    n = 12
    good = pkg.baseline_design(n, 5, 1e-6)
    broken = good.copy()
    broken[3, 4, 5] = np.nan
    ub, infos, Cb, st = batched(pkg, n, [(good, 0.5), (broken, 0.5), (good, 0.25)], precision)
    assert st == pkg._lib.PGJ_ERR_CERTIFICATION
    assert all(i["converged"] for i in infos[:6]) and all(i["converged"] for i in infos[12:])
    assert not any(i["converged"] for i in infos[6:12])
    # the broken design may restart (its certificate is not finite), its batch-mates never do
    assert all(i["restarts"] == 0 for i in infos[:6] + infos[12:])
    for d, alpha in ((0, 0.5), (2, 0.25)):
        u1, its1, C1, _ = alone(pkg, n, good, alpha, precision)
        assert [i["iterations"] for i in infos[6 * d:6 * d + 6]] == its1
        assert torch.equal(ub[6 * d:6 * d + 6], u1)
        assert torch.equal(Cb[d], C1)


def test_batch_collects_in_completion_order(pkg):
    """Batch returns every request once, with results equal to stand-alone solves, when groups of
    different grids and sizes finish in an order other than their launch order."""
    reqs = [pkg.Request(torch.tensor(pkg.baseline_design(n, s, 1e-4)), 0.5, tag=(n, s))
            for n, s in [(24, 1), (12, 2), (12, 3), (24, 4), (12, 5)]]
    res = pkg.Batch(slots=2, designs=2, precision="fp64").run(reqs)
    assert sorted(r.tag for r in res) == sorted(r.tag for r in reqs)
    for r in res:
        n, s = r.tag
        _, its, C1, st = alone(pkg, n, pkg.baseline_design(n, s, 1e-4), 0.5, "fp64")
        assert r.status == 0 and [i["iterations"] for i in r.infos] == its
        assert np.array_equal(r.C, C1.numpy())

"""Failure detection without a GPU fault: failures are made on the host (bad inputs, an unsolvable
configuration) or by a bounded device wait that nothing completes; the device stays usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)


def test_nonfinite_density_is_reported_not_certified(pkg):
    n = 8
    op = pkg.Operator(n, 6, *pkg.PAPER_MEDIUM)
    a = torch.ones((n, n, n), dtype=torch.float64, device="cuda")
    a[1, 2, 3] = float("nan")
    op.set_material(a)
    op.set_alpha(0.5)
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos, st = op.solve(np.eye(6), 1e-8, u)
    assert st == pkg._lib.PGJ_ERR_CERTIFICATION
    assert not any(i["converged"] for i in infos)
    # the context recovers with a valid design
    op.set_material(torch.ones((n, n, n), dtype=torch.float64, device="cuda"))
    op.set_alpha(0.5)
    u.zero_()
    infos, st = op.solve(np.eye(6), 1e-8, u)
    assert st == 0


def test_nonfinite_macro_rejected_on_host(pkg):
    n = 8
    op = pkg.Operator(n, 6, *pkg.PAPER_MEDIUM)
    op.set_material(torch.ones((n, n, n), dtype=torch.float64, device="cuda"))
    m = np.eye(6)
    m[2, 2] = np.inf
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    with pytest.raises(RuntimeError, match="non-finite"):
        op.solve(m, 1e-8, u)


def test_bounded_device_wait_times_out_and_context_survives(pkg):
    n = 8
    op = pkg.Operator(n, 6, *pkg.PAPER_MEDIUM)
    st = pkg._lib.lib().pgj_selftest_wait_timeout(op._ctx, 1000, torch.cuda.current_stream().cuda_stream)
    assert st == pkg._lib.PGJ_ERR_TIMEOUT
    op.set_material(torch.ones((n, n, n), dtype=torch.float64, device="cuda"))
    op.set_alpha(0.5)
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    _, st = op.solve(np.eye(6), 1e-8, u)
    assert st == 0


def test_argument_errors_raise(pkg):
    op = pkg.Operator(8, 6, *pkg.PAPER_MEDIUM)
    with pytest.raises(ValueError):
        op.apply(torch.zeros((6, 10), dtype=torch.float64, device="cuda"))
    with pytest.raises(RuntimeError, match="unsupported grid size"):
        pkg.Operator(17, 6, *pkg.PAPER_MEDIUM)

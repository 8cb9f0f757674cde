"""The allocation-free C_H entry point gives the same tensor as the context entry point.

pgj_effective_tensor_noalloc exists for callers that cannot allocate device memory (a host that
owns the whole device pool and forbids third-party allocations). It keeps its scratch in a
fixed device array inside the library, so this test calls it through the C ABI twice in a row on
different inputs (the second call reuses the scratch the first one left behind) and compares each
result with pgj_effective_tensor run on a regular context. This file is collected last so that a
stop-at-first-failure run has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes, skipped
    pytest.skip("CUDA device required", allow_module_level=True)


def test_noalloc_matches_context_entry_point_twice(pkg):
    lib = pkg._lib.lib()
    lam, mu = pkg.PAPER_MEDIUM
    rng = np.random.default_rng(77)
    stream = torch.cuda.current_stream().cuda_stream
    for call, n in enumerate((12, 16)):
        a = torch.tensor(pkg.baseline_design(n, seed=20 + call, emin=1e-6), device="cuda")
        u = torch.tensor(rng.standard_normal((6, 3 * n ** 3)) * 1e-2, device="cuda")
        op = pkg.Operator(n, 6, lam, mu)
        op.set_material(a)
        expected = op.effective_tensor(u)
        got = torch.full((6, 6), float("nan"), dtype=torch.float64, device="cuda")
        pkg._lib.check(lib.pgj_effective_tensor_noalloc(n, lam, mu, a.data_ptr(), u.data_ptr(), got.data_ptr(),
                                                        stream), "pgj_effective_tensor_noalloc")
        torch.cuda.synchronize()
        e, g = expected.cpu().numpy(), got.cpu().numpy()
        assert np.isfinite(g).all()
        assert np.abs(g - e).max() <= 1e-12 * np.abs(e).max(), (call, g, e)


def test_noalloc_rejects_sizes_beyond_its_scratch(pkg):
    lib = pkg._lib.lib()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = lib.pgj_effective_tensor_noalloc(512, 1.0, 1.0, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream)
    assert st == pkg._lib.PGJ_ERR_ARGUMENT

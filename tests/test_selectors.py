"""Global alpha selectors (contrast, gray, compact8, compact8q) of the density-selector study.

The compact-law features and law8 values are pinned to the reference's own ``law.py`` through
``tests/golden/selector_law.npz`` (written by ``make_selector_golden.py``); the selector formulas
of ``exp/asg_density_selector_20261105/run.py:27-43,53-67`` are restated in the oracle. Features
are FP32 like the reference, so they are compared at 1e-5 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def golden(golden_dir):
    d = np.load(golden_dir / "selector_law.npz")
    names = sorted({k.split("/")[0] for k in d.files})
    return {k: dict(a=d[f"{k}/a"], features=d[f"{k}/features"], law8=float(d[f"{k}/law8"])) for k in names}


def test_oracle_law_features_match_reference(oracle, golden):
    for name, g in golden.items():
        f = oracle.law_features(g["a"])
        assert np.allclose(f, g["features"], rtol=1e-5, atol=1e-7), name
        expect = 0.0 if g["law8"] < 0.375 else g["law8"]
        assert oracle.compact8_alpha(g["a"]) == pytest.approx(expect, abs=1e-5), name


def test_selectors_match_reference_and_oracle_on_cpu(pkg, oracle, golden):
    sel = pkg.alpha_selectors
    for name, g in golden.items():
        a = torch.tensor(g["a"], dtype=torch.float64)
        assert np.allclose(sel.law_features(a).numpy(), g["features"], rtol=1e-5, atol=1e-7), name
        value = float(sel.compact8_alpha(a))
        assert value == pytest.approx(0.0 if g["law8"] < 0.375 else g["law8"], abs=1e-5), name
        assert float(sel.compact8_alpha(a, quantize=True)) == oracle.compact8_alpha(g["a"], quantize=True), name
        assert float(sel.contrast_alpha(a)) == oracle.contrast_alpha(g["a"]), name
        rho = np.clip(np.cbrt(g["a"]), 0.0, 1.0)
        assert float(sel.gray_alpha(a, torch.tensor(rho))) == oracle.gray_alpha(g["a"], rho), name


def test_selector_edge_cases(pkg, golden):
    sel = pkg.alpha_selectors
    flat = torch.tensor(golden["homogeneous"]["a"])
    # a homogeneous field: no contrast, every selector gives the plain Green preconditioner
    for value in (sel.compact8_alpha(flat), sel.compact8_alpha(flat, quantize=True), sel.contrast_alpha(flat),
                  sel.gray_alpha(flat, flat)):
        assert float(value) == 0.0
    # simp0 lies just below the 0.375 cut-off of the compact law: alpha falls back to 0
    assert 0.37 < golden["simp0"]["law8"] < 0.375
    assert float(sel.compact8_alpha(torch.tensor(golden["simp0"]["a"]))) == 0.0
    # quantization rounds to sixteenths
    q = float(sel.compact8_alpha(torch.tensor(golden["simp2"]["a"]), quantize=True))
    assert q * 16 == int(q * 16) and abs(q - golden["simp2"]["law8"]) <= 1 / 32


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["contrast", "gray", "compact8", "compact8q", "eta"])
def test_selector_resident_choose_on_device(pkg, oracle, golden, method):
    if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes
        pytest.skip("CUDA device required")
    a = golden["simp2"]["a"]
    n = a.shape[0]
    r = pkg.SelectorResident(None, n, "shear", 0.2, rmin=2.1, emin=1e-9)
    r.material(torch.tensor(a, device="cuda"))
    r.outer.set_initial(np.full((n, n, n), 0.3))
    r.outer.evaluate()
    r.select(method)
    got = float(r.alpha)
    rho = r.outer.ph.cpu().numpy()
    expect = {"contrast": oracle.contrast_alpha(a), "gray": oracle.gray_alpha(a, rho),
              "compact8": oracle.compact8_alpha(a), "compact8q": oracle.compact8_alpha(a, quantize=True),
              "eta": 13 / 16}[method]
    assert got == pytest.approx(expect, abs=1e-5)
    assert 0.0 < got <= 1.0


@pytest.mark.gpu
def test_resident_select_asg_on_device(pkg, oracle, golden_dir):
    """Resident.select('asg') on the device density gives the reference network's alpha (the golden
    prediction of tests/golden/make_asg_golden.py, thresholded at 0.2), and builds that scale."""
    if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes
        pytest.skip("CUDA device required")
    g = np.load(golden_dir / "asg_selector.npz")
    for (n, seed, emin), pred in zip(g["cases"], g["predictions"]):
        n = int(n)
        r = pkg.Resident(None, n)
        a = oracle.simp(oracle.baseline_density(n, int(seed)), float(emin))
        r.material(torch.tensor(a, device="cuda"))
        r.select("asg")
        expect = 0.0 if pred < float(g["threshold"]) else pred
        # FP32 feature means over n^3 values sum in another order on the device than in the
        # reference's CPU evaluation; the network turns that into differences of a few 1e-5
        assert float(r.alpha) == pytest.approx(expect, abs=2e-4), (n, seed)
        ref_scale = oracle.scale_field(a, float(r.alpha), *pkg.STUDY1_MEDIUM)
        assert np.abs(r.op.scale.cpu().numpy() - ref_scale).max() <= 1e-12 * np.abs(ref_scale).max()

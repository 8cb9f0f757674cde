"""ASG alpha selector (features + frozen MLP) against the reference's own extractor and network,
evaluated by tests/golden/make_asg_golden.py. The selector is plain torch and runs where its input
lives, so this check runs on CPU tensors; the GPU test runs the same code on the device."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def golden(golden_dir):
    return np.load(golden_dir / "asg_selector.npz")


def test_weights_are_the_frozen_model(pkg):
    from importlib import import_module

    w = import_module("pgj_b200.asg_weights").load()
    assert w["w0"].shape == (64, 92) and w["w1"].shape == (32, 64) and w["w2"].shape == (1, 32)
    assert w["threshold"] == 0.2


def test_features_and_prediction_match_reference(pkg, oracle, golden):
    sel = pkg.alpha_selectors
    for (n, seed, emin), f_ref, p_ref in zip(golden["cases"], golden["features"], golden["predictions"]):
        a = torch.tensor(oracle.simp(oracle.baseline_density(int(n), int(seed)), float(emin)))
        f = sel.asg_features(a).numpy()
        assert np.allclose(f, f_ref, rtol=2e-5, atol=1e-6), (n, seed, np.abs(f - f_ref).max())
        p = float(sel.asg_prediction(a))
        assert abs(p - p_ref) <= 1e-5, (n, seed, p, p_ref)
        alpha = float(sel.asg_alpha(a))
        assert alpha == (0.0 if p < float(golden["threshold"]) else pytest.approx(p))


def test_features_reject_unsupported_grids(pkg):
    with pytest.raises(ValueError):
        pkg.alpha_selectors.asg_features(torch.ones((24, 24, 24), dtype=torch.float64))

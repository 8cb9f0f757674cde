"""The package's design generators (host side) against the oracle's, on CPU."""
import numpy as np


def test_baseline_design_is_the_oracle_generator(pkg, oracle):
    # the config-2 parity cases regenerate their fields through the package generator
    for n, seed, emin in ((32, 0, 1e-4), (32, 4, 1e-9), (64, 0, 1e-6)):
        a = pkg.baseline_design(n, seed, emin)
        b = oracle.simp(oracle.baseline_density(n, seed), emin)
        assert np.array_equal(a, b)


def test_uneven_designs_are_seeded_and_in_range(pkg):
    specs = [pkg.designs.uneven_spec(s) for s in range(64)]
    assert specs == [pkg.designs.uneven_spec(s) for s in range(64)]
    assert {n for n, _, _ in specs} == {24, 32, 48, 64}
    assert all(0.2 <= vf <= 0.5 and 0.0 <= alpha <= 1.0 for _, vf, alpha in specs)
    seed, n, vf, alpha, a = pkg.designs.uneven_designs(2, 1e-6)[1]
    assert a.shape == (n, n, n) and abs(((a - 1e-6) / (1 - 1e-6)) ** (1 / 3)).mean() > 0

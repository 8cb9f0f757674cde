"""Pin the CPU oracle to the reference's own fixtures (tests/golden/, made by make_golden.py)."""
import hashlib
import json

import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref(golden_dir):
    return np.load(golden_dir / "reference_cpu.npz")


@pytest.fixture(scope="module")
def meta(golden_dir):
    return json.loads((golden_dir / "reference_meta.json").read_text())


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_element_stiffness_matches_reference(oracle, ref):
    assert rel(oracle.element_stiffness(4, *oracle.STUDY1), ref["ke_study1_n4"]) < 1e-15
    assert rel(oracle.element_stiffness(4, *oracle.PAPER), ref["ke_paper_n4"]) < 1e-15


@pytest.mark.parametrize("name,medium", [("study1", "STUDY1"), ("paper", "PAPER")])
@pytest.mark.parametrize("n", [4, 64])
def test_element_action_matches_reference_fi_modal(oracle, ref, name, medium, n):
    ke = oracle.element_stiffness(n, *getattr(oracle, medium))
    assert rel(ref["fi_dofs"] @ ke, ref[f"fi_{name}_n{n}"]) < 1e-14


def test_dense_fe_reference(oracle, ref):
    a = ref["dense_a"]
    loads = np.vstack([np.eye(6), [1, 1, 1, 0, 0, 0]])
    lam, mu = oracle.PAPER
    f = oracle.rhs(a, loads, lam, mu)
    assert rel(f, ref["dense_rhs"]) < 1e-14
    assert rel(oracle.apply_operator(a, ref["dense_u"], lam, mu), f) < 1e-12
    e = oracle.energies(ref["dense_u"], oracle.affine(4, loads), 4, lam, mu)
    assert rel(e, ref["dense_energies"]) < 1e-14
    assert rel((e * a.reshape(1, -1)).mean(1), ref["dense_moduli"]) < 1e-14


def test_oracle_solve_matches_dense_solution(oracle, ref):
    a = ref["dense_a"]
    lam, mu = oracle.PAPER
    loads = np.vstack([np.eye(6), [1, 1, 1, 0, 0, 0]])
    out = oracle.homogenize(a, lam, mu, 0.5, rtol=1e-12, macros=loads)
    assert not out["raised"]
    assert rel(out["u"], ref["dense_u"]) < 1e-9


def test_study1_chain_matches_reference(oracle, ref):
    ph, dp = oracle.study1_physical(ref["s1_x"], 2.0)
    assert rel(ph, ref["s1_ph"]) < 1e-15 and rel(dp, ref["s1_dp"]) < 1e-15
    g = oracle.study1_filter(dp * 3 * (1 - 1e-4) * ph ** 2 * ref["s1_energy"])
    dv = oracle.study1_filter(dp)
    assert rel(g, ref["s1_g"]) < 1e-15 and rel(dv, ref["s1_dv"]) < 1e-15
    assert rel(oracle.study1_oc(ref["s1_x"], g, dv, 2.0), ref["s1_new"]) < 1e-15


def test_cone_stencil_and_paper_initial(oracle, ref):
    offs, ws = oracle.cone_stencil(3.2)
    assert np.array_equal(offs, ref["cone_offsets"]) and np.allclose(ws, ref["cone_weights"], rtol=0, atol=0)


@pytest.mark.parametrize("n", [16, 32])
def test_study1_state0_regenerates_bitwise(oracle, meta, n):
    a = oracle.study1_state0(n)
    assert hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() == meta["study1_state0"][str(n)]["sha256"]


def test_package_generator_equals_oracle(pkg, oracle):
    for n, seed in ((8, 0), (16, 3)):
        assert np.array_equal(pkg.baseline_density(n, seed), oracle.baseline_density(n, seed))
    assert np.array_equal(pkg.study1_state0(16), oracle.study1_state0(16))


def test_green_symbol_inverts_homogeneous_operator(oracle):
    """G(k) = K0(k)^-1 on the zero-mean range: K0 G P r = P r (fft_precision.py:61-91)."""
    n = 6
    lam, mu = oracle.PAPER
    rng = np.random.default_rng(1)
    r = oracle.project(rng.standard_normal((2, 3 * n ** 3)))
    z = oracle.green_unscaled(r, oracle.green_symbol(n, lam, mu))
    back = oracle.apply_operator(np.ones((n, n, n)), z, lam, mu)
    assert rel(back, r) < 1e-11


def test_preconditioner_matches_dense_pinv(oracle):
    """M_alpha^-1 = P S pinv(K0) S P at n=4 (adaptive_green_scaling/study.py:205-248)."""
    n = 4
    lam, mu = oracle.STUDY1
    rng = np.random.default_rng(20261028)
    a = np.exp(rng.uniform(-np.log(100), 0, (n, n, n)))
    N3 = 3 * n ** 3
    eye = np.eye(N3)
    K0 = oracle.apply_operator(np.ones((n, n, n)), eye, lam, mu).T
    G = np.linalg.pinv(K0, rcond=1e-13)
    T = np.tile(np.eye(3), (n ** 3, 1))
    P = np.eye(N3) - T @ T.T / n ** 3
    v = P @ rng.standard_normal(N3)
    for alpha in (0.0, 0.5, 1.0):
        prob = oracle.Problem(a, lam, mu, alpha)
        s = prob.scale.ravel()
        B = P @ (s[:, None] * G * s[None, :]) @ P
        assert rel(prob.B(v[None])[0], B @ v) < 1e-11


def test_oracle_reproduces_archived_iterations_n32(oracle, golden_dir):
    """Study I state 0, n=32, alpha=0.5: the archived per-load counts [57, 57, 58] and J."""
    g = json.loads((golden_dir / "replay_k000.json").read_text())["32"]
    a = oracle.study1_state0(32)
    f = oracle.rhs(a, np.eye(6)[3:], *oracle.STUDY1)
    assert rel(np.sqrt((f * f).sum(1)), g["rows"]["0.5/serial"][0]["rhs_norm"]) < 1e-14
    prob = oracle.Problem(a, *oracle.STUDY1, 0.5)
    u, infos, raised = oracle.solve_batch(prob, f)
    assert not raised and [i.iterations for i in infos] == [57, 57, 58]
    e = oracle.energies(u, oracle.affine(32, np.eye(6)[3:]), 32, *oracle.STUDY1)
    J = (e * a.reshape(1, -1)).mean(1).mean()
    assert abs(J - g["reference_J"]) / g["reference_J"] < 1e-12

"""Design sensitivities of the Study II objectives against central finite differences.

Follows the reference's per-objective check (``exp/asg_sctop_reproduction_20261105/verify.py:39-96``):
n=4, clipped cone filter rmin=2.1, tanh(4, 0.5) projection, Emin=1e-9, x ~ U[0.15, 0.7] from
``default_rng(51)``, iteration 7 of the auxetic weight schedule, one unit random direction and a
central difference of step 1e-5. Bars, as there: objective sensitivity < 1e-5 relative, volume
sensitivity < 1e-7 absolute.

The CPU test pins the oracle's sensitivity formula. The GPU test runs the whole chain through the
C ABI: device filter / projection, certified solve, device energies and objective, and the filtered
sensitivities the device OC update forms.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

N, RMIN, EMIN, ITERATION, STEP = 4, 2.1, 1e-9, 7, 1e-5
OBJECTIVES = {"shear": 0.2, "bulk": 0.3, "auxetic": 0.2}  # objective -> volume fraction


def start_and_direction():
    rng = np.random.default_rng(51)
    x = rng.uniform(0.15, 0.7, size=(N, N, N))
    d = rng.normal(size=x.shape)
    return x, d / np.linalg.norm(d)


def oracle_objective(oracle, x, objective):
    """(J, local, ph, dp, hs, u) of the Study II chain on the CPU."""
    lam, mu = oracle.PAPER
    hs = oracle.cone_filter(np.ones_like(x), RMIN)
    ph, dp, a = oracle.paper_physical(oracle.cone_filter(x, RMIN), hs, emin=EMIN)
    u = oracle.homogenize(a, lam, mu, 0.5, rtol=1e-12)["u"]
    local, _ = oracle.paper_local_energy(u, N, lam, mu, objective, ITERATION)
    return float((local * a.ravel()).mean()), local.reshape(x.shape), ph, dp, hs, u


@pytest.mark.parametrize("objective", list(OBJECTIVES))
def test_oracle_sensitivity_matches_finite_difference(oracle, objective):
    x, d = start_and_direction()
    _, local, ph, dp, hs, _ = oracle_objective(oracle, x, objective)
    g, dv = oracle.paper_sensitivity(local, ph, dp, hs, RMIN, EMIN)
    values, volumes = [], []
    for sign in (-1, 1):
        j, _, p, _, _, _ = oracle_objective(oracle, x + sign * STEP * d, objective)
        values.append(j)
        volumes.append(p.sum())
    fd = (values[1] - values[0]) / (2 * STEP)
    analytic = float((g * d).sum())
    assert abs(fd - analytic) / max(abs(fd), abs(analytic), 1e-12) < 1e-5
    assert abs((volumes[1] - volumes[0]) / (2 * STEP) - float((dv * d).sum())) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("objective", list(OBJECTIVES))
def test_device_sensitivity_matches_finite_difference(pkg, oracle, objective):
    if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes
        pytest.skip("CUDA device required")
    x, d = start_and_direction()
    r = pkg.PaperResident(None, N, objective, OBJECTIVES[objective], rmin=RMIN, emin=EMIN)
    r.capture()

    def evaluate(xv):
        r.outer.set_initial(xv)
        r.outer.evaluate()
        r.material(r.outer.a)
        r.select("0.5")
        r.solutions.zero_()
        r.solve(1e-11)
        f, local, _ = r.energy(ITERATION)
        return float(f), local, float(r.outer.ph.sum())

    f, local, _ = evaluate(x)
    j_ref, local_ref, ph, dp, hs, u_ref = oracle_objective(oracle, x, objective)
    assert abs(f - j_ref) < 1e-11
    assert np.linalg.norm(local.cpu().numpy() - local_ref) / np.linalg.norm(local_ref) < 1e-8
    u = r.solutions.cpu().numpy()
    assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) < 1e-7

    # the device OC update leaves ratio = -g/dv in scratch[0:N] and dv in scratch[N:2N]
    r.outer.step(local)
    n3 = N ** 3
    scratch = r.outer.scratch.cpu().numpy()
    dv = scratch[n3:2 * n3].reshape(x.shape)
    g = -scratch[:n3].reshape(x.shape) * dv
    g_ref, dv_ref = oracle.paper_sensitivity(local_ref, ph, dp, hs, RMIN, EMIN)
    assert np.abs(g - g_ref).max() <= 1e-8 * np.abs(g_ref).max()
    assert np.abs(dv - dv_ref).max() <= 1e-13 * np.abs(dv_ref).max()
    new, steps, _ = oracle.paper_oc(x, local_ref, ph, dp, hs, RMIN, OBJECTIVES[objective], emin=EMIN)
    assert r.outer.steps == steps
    assert np.abs(r.outer.new.cpu().numpy() - new).max() < 1e-9

    values, volumes = [], []
    for sign in (-1, 1):
        fj, _, vol = evaluate(x + sign * STEP * d)
        values.append(fj)
        volumes.append(vol)
    fd = (values[1] - values[0]) / (2 * STEP)
    analytic = float((g * d).sum())
    assert abs(fd - analytic) / max(abs(fd), abs(analytic), 1e-12) < 1e-5
    assert abs((volumes[1] - volumes[0]) / (2 * STEP) - float((dv * d).sum())) < 1e-7

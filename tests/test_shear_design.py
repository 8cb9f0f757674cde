"""Study I design driver (``examples/shear_design.py:14-74``): beta schedule, stop rule, rows.

CPU: the loop control with a scripted fake resident. GPU: the first design steps on the device,
whose step 0 is Study I state 0 (J as archived by the reference).
"""
import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")


class FakeOuter:
    def __init__(self, n, change):
        self.change_script = change
        self.betas, self.advanced, self.steps = [], 0, 0
        self.a = torch.ones((n, n, n), dtype=torch.float64)
        self.ph = torch.full((n, n, n), 0.3, dtype=torch.float64)
        self.x = torch.zeros((n, n, n), dtype=torch.float64)
        self.change = 1.0

    def set_initial(self, x):
        self.x.copy_(torch.as_tensor(x))

    def evaluate(self, beta):
        self.betas.append(beta)

    def step(self, energy):
        self.change = self.change_script(self.steps)
        self.steps += 1

    def advance(self):
        self.advanced += 1


class FakeResident:
    def __init__(self, n=4, change=lambda k: 0.001, objective=lambda k: 0.02):
        self.outer = FakeOuter(n, change)
        self.objective = objective
        self.solutions = torch.ones((3, 3 * n ** 3), dtype=torch.float64)
        self.alpha = torch.zeros((), dtype=torch.float64)
        self.n = n

    def material(self, a):
        pass

    def select(self, method):
        self.alpha.fill_(float(method))

    def solve(self, rtol=1e-8):
        return [dict(iterations=5, converged=True)] * 3, 1

    def energy(self):
        J = self.objective(self.outer.steps)
        return torch.full((3,), J, dtype=torch.float64), torch.zeros((self.n,) * 3, dtype=torch.float64)


def test_beta_schedule(pkg):
    sd = pkg.shear_design
    assert [sd.beta_at(k) for k in (0, 24, 25, 49, 50, 74, 75, 179)] == [1, 1, 2, 2, 4, 4, 8, 8]


def test_stop_rule_after_five_stable_steps(pkg):
    sd = pkg.shear_design
    r = FakeResident()
    rows, converged = sd.run(r, np.full((4, 4, 4), 0.3), "0.5", 180)
    # stable from k = 95 (beta 8, change < 0.005, objective unchanged): five stable steps end at k = 99
    assert converged and len(rows) == 100 and rows[-1]["step"] == 99
    assert r.outer.advanced == 99
    assert [row["beta"] for row in rows[:1]] == [1.0] and rows[80]["beta"] == 8.0
    assert all(row["volume"] == pytest.approx(0.3) and row["alpha"] == 0.5 for row in rows)
    json.dumps(rows)  # records are plain JSON


def test_step_limit_and_unstable_objective(pkg):
    sd = pkg.shear_design
    r = FakeResident(objective=lambda k: 0.02 * (1 + 0.01 * (k % 2)))  # relative change 1e-2 every step
    rows, converged = sd.run(r, np.full((4, 4, 4), 0.3), "0.5", 120)
    assert not converged and len(rows) == 120 and r.outer.advanced == 119
    r = FakeResident()
    rows, converged = sd.run(r, np.full((4, 4, 4), 0.3), "0.5", 3)
    assert not converged and len(rows) == 3 and r.outer.advanced == 2 and r.outer.betas == [1.0] * 3


def test_argument_checks(pkg, tmp_path):
    sd = pkg.shear_design
    sd.check_args(16, 10, ["0.5", "gj", "green", "compact8", "0.69"])
    sd.check_args(32, 10, ["asg"])  # the ASG features need n >= 32, a multiple of 16
    for n, steps, methods in ((5, 10, ["0.5"]), (2, 10, ["0.5"]), (16, 0, ["0.5"]), (16, 181, ["0.5"]),
                              (16, 10, ["asg"])):
        with pytest.raises(ValueError):
            sd.check_args(n, steps, methods)
    with pytest.raises(SystemExit):
        sd.main(["--n", "7", "--output", str(tmp_path / "o")])


@pytest.mark.gpu
def test_first_design_steps_on_device(pkg, oracle, golden_dir):
    if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes
        pytest.skip("CUDA device required")
    n = 32
    reference_J = json.loads((golden_dir / "replay_k000.json").read_text())[str(n)]["reference_J"]
    r = pkg.Resident(None, n, load_mode="parallel")
    r.capture()
    rows, converged = pkg.shear_design.run(r, pkg.study1_initial(n), "0.5", 2, torch.cuda.synchronize)
    assert len(rows) == 2 and not converged
    # step 0 evaluates the initial design at beta = 1: Study I state 0
    assert abs(rows[0]["objective"] - reference_J) / reference_J < 1e-9
    assert rows[0]["volume"] == pytest.approx(0.3, abs=1e-9)
    assert all(l["converged"] for row in rows for l in row["loads"])
    assert all(abs(i - j) <= 1 for i, j in zip([l["iterations"] for l in rows[0]["loads"]], [57, 57, 58]))
    # the compact law on the device density equals the oracle's
    rows, _ = pkg.shear_design.run(r, pkg.study1_initial(n), "compact8", 1, torch.cuda.synchronize)
    assert rows[0]["alpha"] == pytest.approx(oracle.compact8_alpha(r.outer.a.cpu().numpy()), abs=1e-5)

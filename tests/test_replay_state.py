"""Study II state files and the preconditioner replay of ``examples/replay_state.py:14-64``.

CPU: the .npz layout (``docs/DATA.md`` array conventions), its checks, the reference CLI's method
and eta checks, and the replay sequence with a recording fake resident. GPU: the replay of a
synthetic state through ``SelectorResident`` with a certified warm start.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def make_state(n=6, loads=6, seed=0):
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.0, 1.0, (n, n, n))
    return dict(a=1e-6 + rho ** 3 * (1 - 1e-6), rho=rho, u0=rng.standard_normal((loads, 3 * n ** 3)))


def test_state_round_trip(pkg, tmp_path):
    rs = pkg.replay_state
    s = make_state()
    path = tmp_path / "state.npz"
    rs.save_state(path, s["a"], s["rho"], s["u0"], x=s["rho"])
    back = rs.load_state(path)
    assert set(back) == {"a", "rho", "u0", "x"}
    for k in ("a", "rho", "u0"):
        assert back[k].dtype == np.float64 and np.array_equal(back[k], s[k])


def test_state_checks(pkg, tmp_path):
    rs = pkg.replay_state
    s = make_state()
    with pytest.raises(ValueError, match="'a' must be an"):
        rs.check_state(dict(a=np.ones((4, 4, 5))))
    with pytest.raises(ValueError, match="finite and positive"):
        rs.check_state(dict(a=-np.ones((4, 4, 4))))
    with pytest.raises(ValueError, match="'rho' must have the shape"):
        rs.check_state(dict(a=s["a"], rho=np.ones((5, 5, 5))))
    with pytest.raises(ValueError, match="load-major"):
        rs.check_state(dict(a=s["a"], u0=s["u0"].reshape(6, -1, 3)))
    with pytest.raises(ValueError, match="load-major"):
        rs.check_state(dict(a=s["a"], u0=s["u0"][:4]))
    with pytest.raises(ValueError, match="no 'a'"):
        rs.check_state(dict(rho=s["rho"]))
    # object arrays are never unpickled
    path = tmp_path / "pickled.npz"
    np.savez(path, a=s["a"], extra=np.array([{"k": 1}], dtype=object))
    with pytest.raises(ValueError):
        rs.load_state(path)


def test_method_checks_follow_reference_cli(pkg, tmp_path):
    rs = pkg.replay_state
    rs.check_methods(["gj", "eta", "compact8", "compact8q", "gray", "contrast", "green", "0.25"], 1e-6)
    for bad, msg in ((["nope"], "Unknown method"), (["1.5"], "Unknown method"), (["asg"], "Study I")):
        with pytest.raises(ValueError, match=msg):
            rs.check_methods(bad, 1e-6)
    with pytest.raises(ValueError, match="eta table"):
        rs.check_methods(["gj"], 1e-5)
    out = tmp_path / "out.json"
    out.write_text("{}")
    with pytest.raises(SystemExit):
        rs.main([str(tmp_path / "missing.npz"), "--eta", "1e-6", "--output", str(out)])


class FakeResident:
    """Records the replay's calls; same attribute surface as SelectorResident."""

    def __init__(self, n):
        self.log = []
        self.alpha = torch.zeros((), dtype=torch.float64)
        self.solutions = torch.zeros((6, 3 * n ** 3), dtype=torch.float64)
        self.outer = type("Outer", (), {})()
        self.outer.ph = torch.zeros((n, n, n), dtype=torch.float64)

    def material(self, a):
        self.log.append(("material", float(a.sum())))

    def select(self, method):
        self.alpha.fill_({"gj": 1.0, "eta": 11 / 16}.get(method, 0.5))
        self.log.append(("select", method))

    def solve(self, rtol=1e-8):
        self.log.append(("solve", float(self.solutions.abs().sum())))
        self.solutions.mul_(0.5)  # a solve changes the solutions; the replay must reset them
        return [dict(iterations=3)] * 6, 1

    def effective_tensor(self):
        return torch.eye(6, dtype=torch.float64)


def test_replay_sequence_with_fake_resident(pkg):
    rs = pkg.replay_state
    s = make_state()
    fake = FakeResident(6)
    records = rs.replay(s, 1e-6, methods=["gj", "eta"], resident=(fake, torch.as_tensor, lambda: None))
    u0_sum = float(np.abs(s["u0"]).sum())
    assert [r["method"] for r in records] == ["gj", "eta"]
    assert [r["alpha"] for r in records] == [1.0, 11 / 16]
    assert np.array_equal(fake.outer.ph.numpy(), s["rho"])
    # every solve (warm-up and timed) starts from the archived u0
    solves = [v for k, v in fake.log if k == "solve"]
    assert len(solves) == 4 and all(v == pytest.approx(u0_sum) for v in solves)
    assert [k for k, _ in fake.log].count("select") == 4
    assert records[0]["C"] == np.eye(6).tolist() and records[0]["host_checks"] == 1
    with pytest.raises(ValueError, match="'rho' and 'u0'"):
        rs.replay(dict(a=s["a"]), 1e-6, resident=(fake, torch.as_tensor, lambda: None))


@pytest.mark.gpu
def test_replay_with_certified_warm_start(pkg, tmp_path):
    if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes
        pytest.skip("CUDA device required")
    n, eta = 12, 1e-6
    rho = pkg.baseline_density(n, seed=7)
    a = pkg.simp(rho, eta)
    r = pkg.PaperResident(None, n, "shear", 0.2, emin=eta)
    r.material(torch.tensor(a, device="cuda"))
    r.select("0.5")
    r.solve(1e-10)
    path = tmp_path / "state.npz"
    pkg.replay_state.save_state(path, a, rho, r.solutions.cpu().numpy())
    records = pkg.replay_state.replay(pkg.replay_state.load_state(path), eta, methods=["gj", "eta", "compact8", "0.25"])
    C0 = np.array(records[0]["C"])
    for rec in records:
        # the archived u0 is certified already: every method certifies it without an iteration
        assert all(l["iterations"] == 0 and l["converged"] for l in rec["loads"]), rec["method"]
        assert np.abs(np.array(rec["C"]) - C0).max() <= 1e-12 * np.abs(C0).max()
    assert records[1]["alpha"] == 11 / 16

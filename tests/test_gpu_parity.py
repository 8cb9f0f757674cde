"""GPU parity of the libpgj kernels against the CPU oracle (pgj_oracle), through the C ABI.

Tolerances: operator / RHS / symbol / preconditioner actions are FP64 reformulations of the same
exact products, compared at <= 1e-12 relative (the reference's own specialised-vs-general operator
check uses 2e-14 on identical arithmetic; ours sums in a different order). Solves are compared by
iteration counts and by responses (J, C_H) at <= 1e-10 relative. Iteration counts of a
well-conditioned problem match exactly (Study I golden records); at weak-material ratios 1e-6 and
1e-9 (hundreds to a thousand iterations) rounding-order differences move counts by up to 2%, the
spread the reference itself shows between its serial and parallel schedules (e.g. 582 vs 592).
"""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected on CPU boxes, skipped
    pytest.skip("CUDA device required", allow_module_level=True)


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def dev(x):
    return torch.tensor(np.ascontiguousarray(x), device="cuda", dtype=torch.float64)


@pytest.fixture(scope="module")
def rng():
    return np.random.default_rng(20261203)


@pytest.mark.parametrize("n", [4, 8, 16, 32])
@pytest.mark.parametrize("contrast", [1.0, 1e4])
@pytest.mark.parametrize("medium", ["study1", "paper"])
def test_operator_matches_oracle(pkg, oracle, rng, n, contrast, medium):
    lam, mu = pkg.STUDY1_MEDIUM if medium == "study1" else pkg.PAPER_MEDIUM
    a = np.exp(-np.log(contrast) * rng.random((n, n, n)))
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(dev(a))
    u = rng.standard_normal((6, 3 * n ** 3))
    q = op.apply(dev(u)).cpu().numpy()
    ref = oracle.apply_operator(a, u, lam, mu)
    assert rel(q, ref) < 1e-12
    # symmetry and translation invariance of the device operator
    v = rng.standard_normal((6, 3 * n ** 3))
    qv = op.apply(dev(v)).cpu().numpy()
    sym = abs((u * qv).sum() - (v * q).sum()) / np.sqrt((u * q).sum() * (v * qv).sum())
    assert sym < 1e-13
    shifted = (u.reshape(6, -1, 3) + np.array([1.0, -2.0, 0.5])).reshape(6, -1)
    qs = op.apply(dev(shifted)).cpu().numpy()
    assert rel(qs, q) < 1e-11


def test_operator_masked_loads_and_fp32(pkg, oracle, rng):
    n = 16
    lam, mu = pkg.PAPER_MEDIUM
    a = np.exp(-np.log(1e3) * rng.random((n, n, n)))
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(dev(a))
    u = rng.standard_normal((6, 3 * n ** 3))
    full = op.apply(dev(u)).cpu().numpy()
    active = np.array([1, 0, 1, 1, 0, 1], dtype=np.int32)
    masked = op.apply(dev(u), active=torch.tensor(active, device="cuda")).cpu().numpy()
    assert np.all(masked[active == 0] == 0)
    assert np.array_equal(masked[active == 1], full[active == 1])
    q32 = op.apply(torch.tensor(u, device="cuda", dtype=torch.float32)).double().cpu().numpy()
    assert rel(q32, full) < 2e-5


def test_operator_deterministic(pkg, rng):
    n = 32
    op = pkg.Operator(n, 3, *pkg.STUDY1_MEDIUM)
    op.set_material(dev(rng.random((n, n, n)) + 0.01))
    u = dev(rng.standard_normal((3, 3 * n ** 3)))
    q1 = op.apply(u)
    q2 = op.apply(u)
    assert torch.equal(q1, q2)


@pytest.mark.parametrize("n", [4, 12, 16])
def test_rhs_matches_oracle(pkg, oracle, rng, n):
    lam, mu = pkg.PAPER_MEDIUM
    a = rng.random((n, n, n)) + 1e-3
    op = pkg.Operator(n, 7, lam, mu)
    op.set_material(dev(a))
    macros = np.vstack([np.eye(6), [1, 1, 1, 0, 0, 0]])
    f = op.compute_rhs(macros).cpu().numpy()
    assert rel(f, oracle.rhs(a, macros, lam, mu)) < 1e-13


@pytest.mark.parametrize("n", [8, 12, 30, 64])
def test_symbol_matches_oracle(pkg, oracle, n):
    lam, mu = pkg.PAPER_MEDIUM
    sym = torch.empty((6, n, n, n // 2 + 1), dtype=torch.float64, device="cuda")
    L = pkg._lib.lib()
    pkg._lib.check(L.pgj_green_symbol(n, lam, mu, sym.data_ptr(), torch.cuda.current_stream().cuda_stream), "sym")
    got = sym.cpu().numpy()
    ref = oracle.green_symbol(n, lam, mu)
    assert rel(got, ref) < 1e-13


@pytest.mark.parametrize("n", [8, 12, 16, 32])
@pytest.mark.parametrize("alpha", [0.0, 0.5, 1.0])
def test_preconditioner_matches_oracle(pkg, oracle, rng, n, alpha):
    lam, mu = pkg.PAPER_MEDIUM
    a = pkg.baseline_design(n, seed=n, emin=1e-6)
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(dev(a))
    op.set_alpha(alpha)
    scale = op.scale.cpu().numpy()
    assert rel(scale, oracle.scale_field(a, alpha, lam, mu)) < 1e-13
    r = rng.standard_normal((6, 3 * n ** 3))
    z = op.apply_precond(dev(r)).cpu().numpy()
    prob = oracle.Problem(a, lam, mu, alpha)
    assert rel(z, prob.B(r)) < 1e-12


def test_green_inverts_homogeneous_operator(pkg, rng):
    """G = K0^-1 on the zero-mean range (dense inverse of the FE symbol, fft_precision.py:61-91)."""
    n = 12
    op = pkg.Operator(n, 3, *pkg.PAPER_MEDIUM)
    op.set_material(torch.ones((n, n, n), dtype=torch.float64, device="cuda"))
    op.set_alpha(0.0)
    r = rng.standard_normal((3, 3 * n ** 3))
    r = (r.reshape(3, -1, 3) - r.reshape(3, -1, 3).mean(1, keepdims=True)).reshape(3, -1)
    z = op.apply_precond(dev(r))
    back = op.apply(z).cpu().numpy()
    assert rel(back, r) < 1e-11


def _golden(golden_dir):
    return json.loads((golden_dir / "replay_k000.json").read_text())


@pytest.mark.parametrize("alpha,method", [(0.5, "0.5"), (1.0, "gj"), (0.0, "green")])
def test_study1_state0_matches_golden(pkg, oracle, golden_dir, alpha, method):
    """Study I state 0, n=32, zero start, 3 shear loads: iterations and J as archived by the reference."""
    n = 32
    g = _golden(golden_dir)[str(n)]
    a = pkg.study1_state0(n)
    r = pkg.Resident(None, n, load_mode="parallel")
    r.capture()
    r.material(dev(a))
    r.select(method)
    infos, _ = r.solve(1e-8)
    moduli, _ = r.energy()
    J = float(moduli.mean())
    its = [i["iterations"] for i in infos]
    archived = [row["iterations"] for key, rows in g["rows"].items() if key.startswith(method + "/") for row in rows]
    lo = np.min(archived, axis=0)
    hi = np.max(archived, axis=0)
    # the archived range of the reference's own schedules, widened by the parity bar max(1, 2%):
    # the autotuned tile shapes set the block-partial order of the p.q and r.z sums, which moves
    # ill-conditioned counts (alpha = 0: ~360 iterations) by one or two between runs
    slack_lo = np.maximum(1, np.ceil(0.02 * lo))
    slack_hi = np.maximum(1, np.ceil(0.02 * hi))
    assert np.all(np.array(its) >= lo - slack_lo) and np.all(np.array(its) <= hi + slack_hi), (its, archived)
    if method == "0.5":
        assert its == [57, 57, 58]
    assert abs(J - g["reference_J"]) / g["reference_J"] < 1e-10
    norms = [i["rhs_norm"] for i in infos]
    ref_norms = g["rows"][method + "/parallel"][0]["rhs_norm"] if method + "/parallel" in g["rows"] else None
    if ref_norms:
        assert rel(norms, ref_norms) < 1e-13
    assert all(i["converged"] and i["relative_residual"] <= 1e-8 for i in infos)


@pytest.mark.parametrize("n,emin,alpha", [(16, 1e-6, 0.5), (16, 1e-4, 0.0), (12, 1e-9, 1.0)])
def test_six_load_homogenization_matches_oracle(pkg, oracle, n, emin, alpha):
    lam, mu = pkg.PAPER_MEDIUM
    a = pkg.baseline_design(n, seed=7, emin=emin)
    ref = oracle.homogenize(a, lam, mu, alpha)
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(dev(a))
    op.set_alpha(alpha)
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos, st = op.solve(np.eye(6), 1e-8, u)
    assert st == 0
    its = np.array([i["iterations"] for i in infos])
    its_ref = np.array([i.iterations for i in ref["infos"]])
    assert np.all(np.abs(its - its_ref) <= np.maximum(1, np.ceil(0.02 * its_ref))), (its, its_ref)
    C = op.effective_tensor(u).cpu().numpy()
    assert rel(C, ref["C"]) < 1e-10
    assert all(i["relative_residual"] <= 1e-8 for i in infos)


@pytest.mark.parametrize("value,alpha", [(1.0, 0.5), (0.13, 1.0)])
def test_homogeneous_gives_c0_and_zero_iterations(pkg, value, alpha):
    """Compatible zero RHS: a constant field certifies at the zero start (verify.py:47-49, study.py:294-301)."""
    n = 8
    lam, mu = pkg.PAPER_MEDIUM
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(torch.full((n, n, n), value, dtype=torch.float64, device="cuda"))
    op.set_alpha(alpha)
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos, st = op.solve(np.eye(6), 1e-8, u)
    assert st == 0
    assert all(i["iterations"] == 0 for i in infos)
    C = op.effective_tensor(u).cpu().numpy()
    c0 = np.zeros((6, 6)); c0[:3, :3] = lam; c0[np.arange(3), np.arange(3)] += 2 * mu
    c0[np.arange(3, 6), np.arange(3, 6)] = mu
    assert all(i["converged"] for i in infos)
    assert np.abs(C - value * c0).max() < 1e-11


def test_serial_equals_parallel(pkg):
    n = 12
    a = pkg.baseline_design(n, seed=11, emin=1e-4)
    out = {}
    for mode in ("serial", "parallel"):
        r = pkg.PaperResident(None, n, "shear", 0.2, load_mode=mode)
        r.material(dev(a))
        r.select("0.5")
        infos, _ = r.solve(1e-10)
        out[mode] = (r.effective_tensor().cpu().numpy(), [i["iterations"] for i in infos])
    assert rel(out["serial"][0], out["parallel"][0]) < 1e-12
    assert out["serial"][1] == out["parallel"][1]


def test_energies_match_oracle(pkg, oracle, rng):
    n = 8
    lam, mu = pkg.PAPER_MEDIUM
    a = rng.random((n, n, n)) + 0.01
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(dev(a))
    u = rng.standard_normal((6, 3 * n ** 3)) * 1e-2
    e = op.energies(dev(u), np.eye(6)).cpu().numpy()
    ref = oracle.energies(u, oracle.affine(n, np.eye(6)), n, lam, mu)
    assert rel(e, ref) < 1e-12
    C = op.effective_tensor(dev(u)).cpu().numpy()
    assert rel(C, oracle.effective_tensor(a, u, lam, mu)) < 1e-11


def test_warm_start_and_restart_free(pkg):
    n = 16
    a = pkg.baseline_design(n, seed=5, emin=1e-6)
    r = pkg.PaperResident(None, n, "shear", 0.2)
    r.material(dev(a))
    r.select("0.5")
    infos, _ = r.solve()
    first = [i["iterations"] for i in infos]
    infos2, _ = r.solve()
    # a certified warm start needs no iterations
    assert all(i["iterations"] == 0 and i["converged"] for i in infos2), (first, infos2)


def test_dense_fe_reference(pkg, golden_dir):
    """Dense assembled FE at n=4 (reference dense_reference): solutions and energies."""
    d = np.load(golden_dir / "reference_cpu.npz")
    a = d["dense_a"]
    n = 4
    lam, mu = pkg.PAPER_MEDIUM
    op = pkg.Operator(n, 7, lam, mu)
    op.set_material(dev(a))
    op.set_alpha(0.5)
    loads = np.vstack([np.eye(6), [1, 1, 1, 0, 0, 0]])
    u = torch.zeros((7, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos, st = op.solve(loads, 1e-12, u)
    assert st == 0
    assert rel(u.cpu().numpy(), d["dense_u"]) < 1e-9
    e = op.energies(u, loads).cpu().numpy()
    assert rel(e, d["dense_energies"]) < 1e-9
    moduli = (e * a.reshape(1, -1)).mean(1)
    assert rel(moduli, d["dense_moduli"]) < 1e-9


@pytest.mark.parametrize("n,emin", [(16, 1e-6), (24, 1e-9), (32, 1e-4)])
def test_mixed_reliable_updates_certify_and_match_fp64(pkg, oracle, n, emin):
    """FP32 inner PCG inside FP64 refinement: FP64 certificate, C_H within 1e-7 of the FP64 oracle."""
    lam, mu = pkg.PAPER_MEDIUM
    a = pkg.baseline_design(n, seed=13, emin=emin)
    ref = oracle.homogenize(a, lam, mu, 0.5) if n <= 24 else None
    out = {}
    for prec in ("fp64", "mixed"):
        op = pkg.Operator(n, 6, lam, mu, precision=prec)
        op.set_material(dev(a))
        op.set_alpha(0.5)
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        infos, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0, (prec, infos)
        assert all(i["converged"] and i["relative_residual"] <= 1e-8 for i in infos)
        out[prec] = (op.effective_tensor(u).cpu().numpy(), op.last_refinements(),
                     max(i["iterations"] for i in infos))
    C64, Cmx = out["fp64"][0], out["mixed"][0]
    # one FP32 recurrence with true-residual replacements needs about the FP64 iteration count
    assert out["mixed"][2] <= 1.5 * out["fp64"][2] + 20, (out["mixed"][2], out["fp64"][2])
    assert rel(Cmx, C64) < 1e-7, rel(Cmx, C64)
    if ref is not None:
        assert rel(Cmx, ref["C"]) < 1e-7
        assert rel(C64, ref["C"]) < 1e-10
    assert out["mixed"][1] >= 1


def test_mixed_inner_tolerance_changes_sweeps(pkg):
    n = 16
    lam, mu = pkg.PAPER_MEDIUM
    a = pkg.baseline_design(n, seed=2, emin=1e-6)
    sweeps = []
    for rtol_in in (1e-3, 1e-5):
        op = pkg.Operator(n, 6, lam, mu, precision="mixed")
        op.set_mixed_mode("sweeps")
        op.set_inner_rtol(rtol_in)
        op.set_material(dev(a))
        op.set_alpha(0.5)
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        infos, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0
        sweeps.append(op.last_refinements())
    assert sweeps[0] >= sweeps[1]


def test_profile_iteration_reports_all_kernels(pkg):
    n = 16
    for prec in ("fp64", "mixed"):
        op = pkg.Operator(n, 6, *pkg.PAPER_MEDIUM, precision=prec)
        op.set_material(dev(pkg.baseline_design(n, seed=1, emin=1e-6)))
        op.set_alpha(0.5)
        for fused in (True, False):
            op.set_fused_iteration(fused)
            prof = op.profile_iteration(np.eye(6), reps=3)
            assert len(prof) == (4 if fused else 8)
            assert all(v["ms"] > 0 and v["bytes"] > 0 for v in prof.values()), prof


@pytest.mark.parametrize("n,prec,emin", [(12, "fp64", 1e-6), (30, "fp64", 1e-4), (16, "mixed", 1e-6),
                                         (20, "mixed", 1e-9)])
def test_fused_iteration_matches_unfused(pkg, n, prec, emin):
    """Four-kernel iteration (updates fused with the slab transforms, projection means by Parseval)
    against the step-by-step kernels: same iteration counts, same C_H."""
    lam, mu = pkg.PAPER_MEDIUM
    a = dev(pkg.baseline_design(n, seed=21, emin=emin))
    out = {}
    for fused in (False, True):
        op = pkg.Operator(n, 6, lam, mu, precision=prec)
        op.set_fused_iteration(fused)
        assert op.fused_iteration == fused
        op.set_material(a)
        op.set_alpha(0.5)
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        infos, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0, (fused, infos)
        out[fused] = (op.effective_tensor(u).cpu().numpy(), np.array([i["iterations"] for i in infos]))
    (C0, i0), (C1, i1) = out[False], out[True]
    assert np.all(np.abs(i1 - i0) <= np.maximum(1, np.ceil(0.02 * i0))), (i0, i1)
    assert rel(C1, C0) < (1e-10 if prec == "fp64" else 1e-7), rel(C1, C0)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_register_z_pass_matches_generic_z_pass(pkg, prec, monkeypatch):
    """n = 64: the z pass and the slab transforms with the line transforms in registers against the
    generic shared-memory passes (both in the four-kernel iteration)."""
    n = 64
    lam, mu = pkg.PAPER_MEDIUM
    a = dev(pkg.baseline_design(n, seed=5, emin=1e-4))
    out = {}
    for flag in ("0", "1"):
        # "0": generic shared-memory passes; "1": register line transforms in the z pass and slabs
        monkeypatch.setenv("PGJ_FZ64", flag)
        monkeypatch.setenv("PGJ_SLAB64", flag)
        op = pkg.Operator(n, 6, lam, mu, precision=prec)
        op.set_material(a)
        op.set_alpha(0.5)
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        infos, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0, (flag, infos)
        out[flag] = (op.effective_tensor(u).cpu().numpy(), np.array([i["iterations"] for i in infos]))
    (C0, i0), (C1, i1) = out["0"], out["1"]
    assert np.all(np.abs(i1 - i0) <= np.maximum(1, np.ceil(0.02 * i0))), (i0, i1)
    assert rel(C1, C0) < (1e-10 if prec == "fp64" else 1e-7), rel(C1, C0)


def test_fused_iteration_falls_back_when_the_slab_does_not_fit(pkg):
    op = pkg.Operator(128, 1, *pkg.PAPER_MEDIUM)
    assert not op.fused_iteration
    with pytest.raises(RuntimeError, match="unsupported"):
        op.set_fused_iteration(True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_concurrent_designs_match_single_solves(pkg, precision):
    """Designs of uneven n in flight on separate streams give the single-design results."""
    lam, mu = pkg.PAPER_MEDIUM
    designs = [(12, 3, 1e-4, 0.5), (16, 4, 1e-6, 0.25), (12, 5, 1e-9, 1.0), (16, 6, 1e-4, 0.0), (16, 7, 1e-4, 0.75)]
    reqs = [pkg.Request(torch.tensor(pkg.baseline_design(n, seed, emin)), alpha, tag=i)
            for i, (n, seed, emin, alpha) in enumerate(designs)]
    batch = pkg.Batch(slots=2, precision=precision)
    results = sorted(batch.run(reqs), key=lambda r: r.tag)
    assert [r.tag for r in results] == list(range(len(designs)))
    for r, (n, seed, emin, alpha) in zip(results, designs):
        assert r.status == 0 and all(i["converged"] for i in r.infos)
        op = pkg.Operator(n, 6, lam, mu)
        op.set_material(dev(pkg.baseline_design(n, seed, emin)))
        op.set_alpha(alpha)
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        _, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0
        C64 = op.effective_tensor(u).cpu().numpy()
        assert rel(r.C, C64) < (1e-12 if precision == "fp64" else 1e-7), (precision, n, rel(r.C, C64))
        assert r.latency_ms > 0


def test_async_solve_equals_blocking_solve(pkg):
    n = 16
    lam, mu = pkg.PAPER_MEDIUM
    a = dev(pkg.baseline_design(n, 9, 1e-6))
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(a)
    op.set_alpha(0.5)
    u1 = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos1, st1 = op.solve(np.eye(6), 1e-8, u1)
    L = pkg._lib.lib()
    m = np.ascontiguousarray(np.eye(6))
    u2 = torch.zeros_like(u1)
    s = torch.cuda.current_stream().cuda_stream
    pkg._lib.check(L.pgj_solve_async(op._ctx, 6, m.ctypes.data, 1e-8, u2.data_ptr(), s), "async")
    info = (pkg._lib.LoadInfo * 6)()
    assert L.pgj_solve_wait(op._ctx, info, s) == 0
    assert st1 == 0 and [i.iterations for i in info] == [i["iterations"] for i in infos1]
    assert torch.equal(u1, u2)


def test_green_alpha0_fails_certification_like_the_oracle(pkg, oracle):
    """alpha=0 (pure Green) at Emin=1e-6 does not certify within 4000 iterations (the reference records
    141 such failures in data/study2/replay_parallel_summary.csv:7); the device path must report the
    same failure instead of a result."""
    n = 16
    lam, mu = pkg.PAPER_MEDIUM
    a = pkg.baseline_design(n, 6, 1e-6)
    ref = oracle.homogenize(a, lam, mu, 0.0)
    assert ref["raised"] and all(i.iterations == 4000 for i in ref["infos"])
    op = pkg.Operator(n, 6, lam, mu)
    op.set_material(dev(a))
    op.set_alpha(0.0)
    u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
    infos, st = op.solve(np.eye(6), 1e-8, u)
    assert st == pkg._lib.PGJ_ERR_CERTIFICATION
    assert all(i["iterations"] == 4000 and not i["converged"] for i in infos)
    r = pkg.PaperResident(None, n, "shear", 0.2, emin=1e-6)
    r.material(dev(a))
    r.select("green")
    with pytest.raises(RuntimeError, match="true residual certification failed"):
        r.solve()


# ------------------------------------------------------------------------------ design updates (OC)
def test_study1_chain_matches_reference_fixture(pkg, golden_dir):
    """Study I Gaussian filter, projection and 45-step OC vs the reference study.py functions (n=8)."""
    d = np.load(golden_dir / "reference_cpu.npz")
    n = 8
    out = pkg.ResidentOuter(n)
    out.set_initial(d["s1_x"])
    out.evaluate(2.0)
    assert rel(out.ph.cpu().numpy(), d["s1_ph"]) < 1e-13
    assert rel(out.dp.cpu().numpy(), d["s1_dp"]) < 1e-13
    out.step(torch.tensor(d["s1_energy"], device="cuda"))
    # 45 fixed bisections can take an adjacent final branch (check_outer.py:38-40): 2e-8
    assert rel(out.new.cpu().numpy(), d["s1_new"]) < 2e-8


def test_paper_chain_matches_oracle(pkg, oracle):
    """Study II clipped cone filter, tanh(beta,eta) projection and damped OC with the MATLAB stop."""
    n, rmin, volume = 10, 2.1, 0.3
    rng = np.random.default_rng(51)
    x = rng.uniform(0.15, 0.7, (n, n, n))
    energy = -rng.uniform(0.5, 1.5, (n, n, n))
    po = pkg.PaperOuter(n, volume, rmin=rmin, beta=4.0, eta=0.5, emin=1e-9)
    po.set_initial(x)
    po.evaluate()
    hs = oracle.cone_filter(np.ones((n, n, n)), rmin)
    assert rel(po.hs.cpu().numpy(), hs) < 1e-13
    ph, dp, a = oracle.paper_physical(oracle.cone_filter(x, rmin), hs)
    assert rel(po.ph.cpu().numpy(), ph) < 1e-13 and rel(po.a.cpu().numpy(), a) < 1e-13
    po.step(torch.tensor(energy, device="cuda"))
    new, steps, change = oracle.paper_oc(x, energy, ph, dp, hs, rmin, volume)
    assert po.steps == steps
    assert rel(po.new.cpu().numpy(), new) < 1e-9
    assert abs(float(po.change) - change) < 1e-12
    # the device record keeps the reference's layout (verify.py:84): bisections in bounds[3], flag off
    assert po.change.shape == (1,) and int(po.bounds[3]) == steps and not bool(po.bounds[2])


@pytest.mark.parametrize("n,rmin", [(37, 2.1), (64, 3.0), (13, 5.5), (20, 7.0)])
def test_cone_filter_matches_oracle(pkg, oracle, n, rmin):
    """The clipped cone filter against the oracle: grids that end inside a 32 x 8 column tile, and
    tap tables longer than one shared-memory chunk of 512 (rmin 5.5: 739 taps, 7.0: 1365)."""
    rng = np.random.default_rng(n)
    x = rng.uniform(0.0, 1.0, (n, n, n))
    po = pkg.PaperOuter(n, 0.3, rmin=rmin)
    out = torch.empty((n, n, n), device="cuda", dtype=torch.float64)
    po.raw_filter(torch.tensor(x, device="cuda"), out)
    assert rel(out.cpu().numpy(), oracle.cone_filter(x, rmin)) < 1e-13
    again = torch.empty_like(out)
    po.raw_filter(torch.tensor(x, device="cuda"), again)
    assert torch.equal(out, again)


def test_design_step_objective_and_sensitivity(pkg, oracle):
    """One Study II design step: solve, shear objective / local energy, OC update (verify.py:39-96)."""
    n = 8
    lam, mu = pkg.PAPER_MEDIUM
    r = pkg.PaperResident(None, n, "shear", 0.2, rmin=2.1)
    rng = np.random.default_rng(3)
    x = rng.uniform(0.15, 0.7, (n, n, n))
    r.outer.set_initial(x)
    r.outer.evaluate()
    r.material(r.outer.a)
    r.select("0.5")
    r.solve(1e-11)
    f, local, diag = r.energy(7)
    a = r.outer.a.cpu().numpy()
    out = oracle.homogenize(a, lam, mu, 0.5, rtol=1e-11)
    e = oracle.energies(out["u"], oracle.affine(n, np.eye(6)), n, lam, mu)
    local_ref = -e[3:].sum(0)
    assert rel(local.cpu().numpy().ravel(), local_ref) < 1e-8
    assert abs(float(f) - (local_ref * a.ravel()).mean()) < 1e-11
    assert rel(diag.cpu().numpy(), (e * a.reshape(1, -1)).mean(1)) < 1e-8


def test_serving_design_steps_same_alone_and_in_mix(pkg):
    """Continuous batching: a lineage's design steps give the same results alone and among other
    lineages and homogenizations of other grid sizes that overlap it on the device."""
    sv = pkg.serve
    lin = sv.Lineage(n=16, seed=3, emin=1e-4, steps=3, tag="L")
    hom = sv.Homogenize(pkg.baseline_design(16, 5, 1e-6), 0.5, tag="H")
    alone = sv.Server(precision="mixed").run([sv.Arrival(0.0, lin), sv.Arrival(0.0, hom)], realtime=False)
    mix = [sv.Arrival(0.0, lin), sv.Arrival(0.0, hom)]
    mix += [sv.Arrival(0.0, sv.Lineage(n=m, seed=10 + k, emin=1e-6, steps=2, tag=k)) for k, m in enumerate((12, 20, 24))]
    server = sv.Server(precision="mixed", max_workers_per_n=2)
    got = server.run(mix, realtime=False)
    assert server.max_inflight >= 2
    assert all(r.status == 0 for r in got + alone)
    assert len([r for r in got if r.kind == "design_step"]) == 3 + 3 * 2
    for tag, steps in (("L", 3), ("H", 1)):
        for step in range(steps):
            a = [r for r in alone if r.tag == tag and r.step == step][0]
            b = [r for r in got if r.tag == tag and r.step == step][0]
            assert rel(b.C, a.C) <= 1e-12, (tag, step, rel(b.C, a.C))
            if tag == "L":
                assert b.objective == pytest.approx(a.objective, rel=1e-12)
                assert b.oc_steps == a.oc_steps and b.oc_steps > 0
    # the homogenization request equals a direct certified solve of the same field
    lam, mu = pkg.PAPER_MEDIUM
    op = pkg.Operator(16, 6, lam, mu, precision="mixed")
    op.set_material(dev(pkg.baseline_design(16, 5, 1e-6)))
    op.set_alpha(0.5)
    u = torch.zeros((6, 3 * 16 ** 3), dtype=torch.float64, device="cuda")
    _, st = op.solve(np.eye(6), 1e-8, u)
    assert st == 0
    C = op.effective_tensor(u).cpu().numpy()
    h = [r for r in got if r.tag == "H"][0]
    assert rel(h.C, C) <= 1e-12


def test_serving_design_step_matches_oracle_chain(pkg, oracle):
    """First design step of a lineage: filter/projection, certified solve, shear objective and OC
    update against the CPU restatement."""
    sv = pkg.serve
    n = 10
    lin = sv.Lineage(n=n, seed=4, emin=1e-4, steps=1, volume=0.3, alpha=0.5, rmin=1.5, move=0.2, tag=0)
    res = sv.Server(precision="fp64").run([sv.Arrival(0.0, lin)], realtime=False)
    assert len(res) == 1 and res[0].status == 0
    lam, mu = pkg.PAPER_MEDIUM
    x0 = pkg.baseline_density(n, 4, 0.3)
    t = oracle.cone_filter(x0, 1.5)
    hs = oracle.cone_filter(np.ones_like(x0), 1.5)
    ph, dp, a = oracle.paper_physical(t, hs, 4.0, 0.5, 1e-4)
    ref = oracle.homogenize(a, lam, mu, 0.5)
    assert rel(res[0].C, ref["C"]) < 1e-10
    e = oracle.energies(ref["u"], oracle.affine(n, np.eye(6)), n, lam, mu)
    local = -e[3:].sum(0)
    assert res[0].objective == pytest.approx((local * a.reshape(-1)).mean(), rel=1e-9)
    _, steps, change = oracle.paper_oc(x0, local.reshape(x0.shape), ph, dp, hs, 1.5, 0.3, 4.0, 0.5, 1e-4, move=0.2)
    assert res[0].oc_steps == steps
    assert res[0].change == pytest.approx(change, rel=1e-6, abs=1e-9)


def test_serving_mixed_falls_back_to_fp64_and_certifies(pkg):
    """With an FP64 policy below Emin 1e-7, high-contrast lineages run FP64; a mixed request that
    fails certification is redone in FP64 from the mixed iterate, and the result is certified."""
    sv = pkg.serve
    lin = sv.Lineage(n=24, seed=8, emin=1e-9, steps=2, tag="hi")
    res = sv.Server(precision="mixed", fp64_below_emin=1e-7).run([sv.Arrival(0.0, lin)], realtime=False)
    assert [r.precision for r in res] == ["fp64", "fp64"] and all(r.status == 0 for r in res)
    # on the mixed path with alpha 0.5, this n=54, Emin=1e-9 design reaches the iteration cap near
    # 2e-8; the FP64 redo certifies
    server = sv.Server(precision="mixed", fp64_below_emin=0.0)
    lin = sv.Lineage(n=54, seed=1004, emin=1e-9, steps=1, alpha=0.5, tag="forced")
    out = server.run([sv.Arrival(0.0, lin)], realtime=False)
    assert len(out) == 1 and server.fallbacks == 1
    assert out[0].precision == "fp64-fallback" and out[0].status == 0


def test_n96_mixed_and_fp64_certify_and_agree(pkg):
    """n = 96 (the mixed-refinement grid size): the mixed solve runs the generic fused kernels, the
    FP64 solve the step-by-step kernels (its slab does not fit in shared memory); both certify and
    C_H agrees to the mixed tolerance."""
    n = 96
    lam, mu = pkg.PAPER_MEDIUM
    a = dev(pkg.baseline_design(n, seed=3, emin=1e-6))
    out = {}
    for prec in ("fp64", "mixed"):
        op = pkg.Operator(n, 6, lam, mu, precision=prec)
        op.set_material(a)
        op.set_alpha(0.5)
        assert op.fused_iteration == (prec == "mixed")
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        infos, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0 and all(i["relative_residual"] <= 1e-8 for i in infos), (prec, infos)
        out[prec] = op.effective_tensor(u).cpu().numpy()
    assert rel(out["mixed"], out["fp64"]) < 1e-7, rel(out["mixed"], out["fp64"])


def test_serving_eta_alpha_runs_high_contrast_lineages_mixed(pkg):
    """By default a mixed server runs every lineage mixed, with the eta-lookup alpha of its Emin
    (13/16 at 1e-9), and its steps certify without an FP64 redo; the first step's C_H agrees with an
    FP64 server's within the mixed tolerance."""
    sv = pkg.serve
    assert sv.eta_alpha(1e-9) == 13 / 16 and sv.eta_alpha(1e-4) == 9 / 16
    lin = sv.Lineage(n=24, seed=8, emin=1e-9, steps=2, tag="hi")
    server = sv.Server(precision="mixed")
    res = server.run([sv.Arrival(0.0, lin)], realtime=False)
    assert [r.precision for r in res] == ["mixed", "mixed"] and all(r.status == 0 for r in res)
    assert server.fallbacks == 0
    ref = sv.Server(precision="fp64").run([sv.Arrival(0.0, sv.Lineage(n=24, seed=8, emin=1e-9, steps=1, tag="f"))],
                                         realtime=False)
    assert rel(res[0].C, ref[0].C) < 1e-7


@pytest.mark.parametrize("n,emin,alpha,fused", [(16, 1e-6, 0.5, True), (32, 1e-9, 0.8125, True), (64, 1e-6, 0.5, True),
                                                (16, 1e-6, 0.5, False), (24, 1e-9, 0.5, False)])
def test_mixed_flexible_beta_certifies_and_agrees(pkg, n, emin, alpha, fused):
    """The flexible (Polak-Ribiere) direction update of the FP32 recurrences, in the slab-fused and
    in the step-by-step iteration, certifies to 1e-8 and gives C_H within the mixed tolerance of the
    FP64 solve; the step-by-step form takes the fused form's iteration counts (within 3%: the sums
    run in another order) and, at Emin 1e-9, other counts than the plain direction update (the
    option takes effect); FP64 contexts refuse it."""
    lam, mu = pkg.PAPER_MEDIUM
    a = dev(pkg.baseline_design(n, 2, emin))
    out, its = {}, {}
    runs = [("fp64", False, True), ("mixed", True, fused)]
    if not fused:
        runs += [("mixed", True, True), ("mixed", False, False)]
    for prec, flex, fz in runs:
        op = pkg.Operator(n, 6, lam, mu, precision=prec)
        if prec == "mixed":
            op.set_fused_iteration(fz)
            assert op.fused_iteration == fz
            op.set_flexible_beta(flex)
        op.set_material(a)
        op.set_alpha(alpha)
        u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        infos, st = op.solve(np.eye(6), 1e-8, u)
        assert st == 0 and all(i["relative_residual"] <= 1e-8 for i in infos), (prec, infos)
        out[(prec, flex, fz)] = op.effective_tensor(u).cpu().numpy()
        its[(prec, flex, fz)] = [i["iterations"] for i in infos]
    assert rel(out[("mixed", True, fused)], out[("fp64", False, True)]) < 1e-7
    if not fused:
        for d, f in zip(its[("mixed", True, False)], its[("mixed", True, True)]):
            assert abs(d - f) <= max(2, 0.03 * f), its
        if emin < 1e-8:
            assert its[("mixed", True, False)] != its[("mixed", False, False)], its
    with pytest.raises(RuntimeError, match="unsupported"):
        pkg.Operator(8, 6, lam, mu).set_flexible_beta(True)


@pytest.mark.parametrize("n,emin,designs", [(64, 1e-9, 1), (64, 1e-6, 2)])
def test_halo_free_operator_matches_halo_form(pkg, monkeypatch, n, emin, designs):
    """The halo-free FP32 recurrence operator of n = 64 mixed contexts (each element once per launch,
    the tiles' first rows completed by the slab update from the boundary array) against the halo form
    (PGJ_HF=0): both certify, C_H agrees within the mixed tolerance and the iteration counts within 2%
    (only the rounding of the first tile rows differs); the halo-free results are bitwise
    reproducible, alone and in a batched context."""
    lam, mu = pkg.PAPER_MEDIUM
    a = [pkg.baseline_design(n, 30 + d, emin) for d in range(designs)]
    out = {}
    for hf in ("1", "0", "1"):
        monkeypatch.setenv("PGJ_HF", hf)
        res = []
        for d in range(designs):
            op = pkg.Operator(n, 6, lam, mu, precision="mixed")
            op.set_material(dev(a[d]))
            op.set_alpha(0.8125 if emin < 1e-8 else 0.5)
            u = torch.zeros((6, 3 * n ** 3), dtype=torch.float64, device="cuda")
            infos, st = op.solve(np.eye(6), 1e-8, u)
            assert st == 0 and all(i["relative_residual"] <= 1e-8 for i in infos), (hf, infos)
            res.append((op.effective_tensor(u).cpu().numpy(), [i["iterations"] for i in infos]))
        out.setdefault(hf, []).append(res)
    (hf1, hf1b), (halo,) = out["1"], out["0"]
    for d in range(designs):
        assert np.array_equal(hf1[d][0], hf1b[d][0]) and hf1[d][1] == hf1b[d][1]
        assert rel(hf1[d][0], halo[d][0]) < 1e-7
        for x, y in zip(hf1[d][1], halo[d][1]):
            assert abs(x - y) <= max(2, 0.02 * y), (hf1[d][1], halo[d][1])
    if designs > 1:
        monkeypatch.setenv("PGJ_HF", "1")
        bop = pkg.BatchedOperator(n, designs, 6, lam, mu, "mixed")
        s = torch.cuda.current_stream()
        for d in range(designs):
            bop.set_material(d, dev(a[d]), s)
            bop.set_alpha(d, 0.8125 if emin < 1e-8 else 0.5, s)
        u = torch.zeros((designs * 6, 3 * n ** 3), dtype=torch.float64, device="cuda")
        bop.solve_async(designs, np.eye(6), 1e-8, u, s)
        infos, st = bop.wait(designs, s)
        assert st == 0
        for d in range(designs):
            C = torch.empty((6, 6), dtype=torch.float64, device="cuda")
            bop.effective_tensor(d, u[6 * d:6 * (d + 1)], C, s)
            assert np.array_equal(C.cpu().numpy(), hf1[d][0])
            assert [i["iterations"] for i in infos[6 * d:6 * (d + 1)]] == hf1[d][1]

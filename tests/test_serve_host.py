"""Host logic of the serving loop (no GPU): grid-size snapping, Poisson lineage arrivals, HBM
accounting, and the request loop itself (admission under the budget, FP64 redo of failed mixed
requests, design updates committed only after certified steps, the precision policy) driven with
fake workers whose device work completes after a few polls."""
import numpy as np
import pytest


def test_supported_and_snapped_grid_sizes(pkg):
    sv = pkg.serve
    assert [n for n in range(4, 40) if sv.supported_n(n)] == [4, 6, 8, 10, 12, 16, 18, 20, 24, 30, 32, 36]
    assert sv.snap_n(17) == 16 and sv.snap_n(23) == 24 and sv.snap_n(61) == 60 and sv.snap_n(96) == 96
    assert all(sv.supported_n(sv.snap_n(x)) for x in np.linspace(16, 96, 41))


def test_poisson_lineages_are_seeded_and_in_range(pkg):
    sv = pkg.serve
    a = sv.poisson_lineages(40, rate=3.0, seed=7, steps=30)
    b = sv.poisson_lineages(40, rate=3.0, seed=7, steps=30)
    assert [(x.t, x.req.n, x.req.emin) for x in a] == [(x.t, x.req.n, x.req.emin) for x in b]
    ts = [x.t for x in a]
    assert all(t2 > t1 for t1, t2 in zip(ts, ts[1:]))
    assert all(16 <= x.req.n <= 96 and sv.supported_n(x.req.n) for x in a)
    assert {x.req.emin for x in a} <= {1e-4, 1e-6, 1e-9}
    assert all(x.req.steps == 30 and x.req.move == 0.2 and x.req.rmin == 1.5 for x in a)
    # mean inter-arrival close to 1 / rate
    assert abs(np.mean(np.diff([0.0] + ts)) - 1 / 3.0) < 0.15


def test_hbm_accounting_grows_with_grid_size(pkg):
    sv = pkg.serve
    wb = [sv.worker_bytes(n, "mixed") for n in (16, 32, 64)]
    lb = [sv.lineage_bytes(n) for n in (16, 32, 64)]
    assert wb[0] < wb[1] < wb[2] and lb[0] < lb[1] < lb[2]
    assert sv.worker_bytes(64, "fp64") > sv.worker_bytes(64, "mixed")
    # a 120 GB budget holds many n=96 workers and lineages
    assert 120e9 // (sv.worker_bytes(96, "mixed") + sv.lineage_bytes(96)) > 50


# ------------------------------------------------------------------ the request loop with fake workers
class _Event:
    def __init__(self, polls):
        self.polls = polls

    def query(self):
        self.polls -= 1
        return self.polls <= 0


class _FakeLineage:
    def __init__(self, bytes_):
        self.step, self.bytes, self.pending_advance, self.advanced = 0, bytes_, False, 0


def _fake_server(pkg, fail=lambda job: False, **kw):
    sv = pkg.serve

    class FakeWorker:
        def __init__(self, n, prec):
            self.n, self.precision, self.job, self.last_used = n, prec, None, 0.0
            self.bytes = sv.worker_bytes(n, prec)
            self.u0 = None

    class FakeServer(sv.Server):
        def _new_worker(self, n, prec):
            return FakeWorker(n, prec)

        def _snapshot_iterate(self, w):
            return "iterate"

        def _drain(self):
            pass

        def _launch(self, w, job):
            w.job = job
            job.admitted = 0.0
            if isinstance(job.req, sv.Lineage):
                if job.lineage is None:
                    job.lineage = _FakeLineage(sv.lineage_bytes(job.req.n))
                    self.used += job.lineage.bytes
                if job.lineage.pending_advance:
                    job.lineage.advanced += 1
                    job.lineage.pending_advance = False
            job.end = _Event(2)
            self.log.append((job.req.tag, job.step, job.precision, job.fallback))

        def _finish(self, w, now):
            job = w.job
            w.job = None
            st = 6 if fail(job) else 0
            return sv.StepResult(tag=job.req.tag, kind="x", step=job.step, n=w.n, C=np.zeros((6, 6)), objective=0.0,
                                 status=st, iterations=1, queued_ms=0.0, latency_ms=0.0, device_ms=0.0,
                                 precision="fp64-fallback" if job.fallback else w.precision)

    s = FakeServer(**kw)
    s.log = []
    return s


def test_request_loop_respects_the_hbm_budget(pkg):
    sv = pkg.serve
    budget = 2 * sv.worker_bytes(16, "mixed") + 1024
    s = _fake_server(pkg, precision="mixed", hbm_budget=budget)
    reqs = [sv.Arrival(0.0, sv.Homogenize(np.zeros((16, 16, 16)), 0.5, tag=k)) for k in range(5)]
    out = s.run(reqs, realtime=False)
    assert sorted(r.tag for r in out) == list(range(5))
    assert s.max_inflight == 2 and s.peak_used <= budget


def test_failed_mixed_request_is_redone_in_fp64(pkg):
    sv = pkg.serve
    s = _fake_server(pkg, fail=lambda job: job.req.tag == "bad" and job.precision == "mixed", precision="mixed")
    out = s.run([sv.Arrival(0.0, sv.Homogenize(np.zeros((16, 16, 16)), 0.5, tag="bad")),
                 sv.Arrival(0.0, sv.Homogenize(np.zeros((16, 16, 16)), 0.5, tag="ok"))], realtime=False)
    by = {r.tag: r for r in out}
    assert len(out) == 2 and s.fallbacks == 1
    assert by["bad"].precision == "fp64-fallback" and by["bad"].status == 0 and by["ok"].precision == "mixed"
    assert ("bad", 0, "fp64", True) in s.log


def test_design_updates_commit_only_after_certified_steps(pkg):
    sv = pkg.serve
    # FP64 server, no fallback: step 1 fails, so only step 0's update is committed (at step 1's launch)
    s = _fake_server(pkg, fail=lambda job: job.step == 1, precision="fp64")
    lin = sv.Lineage(n=16, seed=0, emin=1e-4, steps=3, tag="L")
    out = s.run([sv.Arrival(0.0, lin)], realtime=False)
    assert [r.status for r in sorted(out, key=lambda r: r.step)] == [0, 6, 0]
    jobs = [e for e in s.log if e[0] == "L"]
    assert [j[1] for j in jobs] == [0, 1, 2]
    # a mixed failure is redone in FP64 without advancing the design a second time
    s2 = _fake_server(pkg, fail=lambda job: job.step == 1 and job.precision == "mixed", precision="mixed")
    out2 = s2.run([sv.Arrival(0.0, sv.Lineage(n=16, seed=0, emin=1e-4, steps=3, tag="M"))], realtime=False)
    assert [r.precision for r in sorted(out2, key=lambda r: r.step)] == ["mixed", "fp64-fallback", "fp64"]
    assert s2.fallbacks == 1 and all(r.status == 0 for r in out2)


def test_policy_and_oversized_requests(pkg):
    sv = pkg.serve
    s = _fake_server(pkg, precision="mixed", fp64_below_emin=1e-7)
    out = s.run([sv.Arrival(0.0, sv.Lineage(n=16, seed=0, emin=1e-9, steps=1, tag="hi"))], realtime=False)
    assert out[0].precision == "fp64"  # Emin below the threshold runs in FP64
    s = _fake_server(pkg, precision="mixed")
    out = s.run([sv.Arrival(0.0, sv.Lineage(n=16, seed=0, emin=1e-9, steps=1, tag="hi"))], realtime=False)
    assert out[0].precision == "mixed"  # by default every lineage runs mixed
    tiny = _fake_server(pkg, precision="mixed", hbm_budget=1024)
    with pytest.raises(RuntimeError, match="HBM budget"):
        tiny.run([sv.Arrival(0.0, sv.Homogenize(np.zeros((16, 16, 16)), 0.5, tag=0))], realtime=False)

"""Host logic of the serving loop (no GPU): grid-size snapping, Poisson lineage arrivals, HBM
accounting."""
import numpy as np


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

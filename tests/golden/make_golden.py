"""Generate the golden fixtures under tests/golden/ from the reference checkout.

Run in a container that has the reference tree (default /root/reference) and a CPU torch:

    python tests/golden/make_golden.py [--ref /root/reference]

It imports the reference's own CPU-runnable Python (the Study I generator, the exact Q1
element stiffness, the Study II stencil / initial fields, the dense FE reference) and the
reference element action built by ``oracle/Makefile`` (``oracle/_ref/libref_fi_modal.so``),
and writes small fixtures. It also extracts the per-load golden records (iterations, rhs
norms, J) from the reference's archived replay JSONs. Nothing here runs on the GPU, and
nothing at test time reads the reference tree: the tests only read the files written here.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ref = Path(ap.parse_args().ref)
    sys.path.insert(0, str(ref / "exp/asg_topopt_20261103"))
    sys.path.insert(0, str(ref / "exp/asg_candidates_20261103"))
    import study as pilot  # reference Study I generator / OC (CPU)
    from candidates import element_geometry, stiffness  # reference exact Q1 stiffness (CPU)

    out = {}
    # 1. Archived per-load records for Study I state 0 (zero start, 3 shear loads).
    replay = {}
    for n in (32, 64):
        d = json.loads((ref / f"exp/asg_mutopopt_20261104/results/replay_n{n}_k000.json").read_text())
        rows = {}
        for r in d["rows"]:
            if r["method"].startswith("mutopopt"):
                continue
            key = f"{r['method']}/{r['load_mode']}"
            rows.setdefault(key, []).append(dict(iterations=[l["iterations"] for l in r["loads"]],
                                                 rhs_norm=[l["rhs_norm"] for l in r["loads"]], J=r["J"]))
        replay[str(n)] = dict(reference_J=d["reference_J"], rows=rows,
                              source=f"exp/asg_mutopopt_20261104/results/replay_n{n}_k000.json")
    (HERE / "replay_k000.json").write_text(json.dumps(replay, indent=1) + "\n")

    # 2. Study I state 0 regenerated by the reference generator: hash + summary per n.
    states = {}
    for n in (16, 32, 64):
        a = pilot.material(pilot.physical(pilot.initial(n, 20261104), 1.0)[0])
        states[str(n)] = dict(sha256=hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest(),
                              sum=float(a.sum()), min=float(a.min()), max=float(a.max()))
    out["study1_state0"] = states

    # 3. Exact element stiffness (reference CPU helper) for both media, n=4.
    c1 = np.zeros((6, 6)); c1[:3, :3] = 4 / 3; c1[np.arange(3), np.arange(3)] += 2; c1[np.arange(3, 6), np.arange(3, 6)] = 1
    lam, mu = 15 / 26, 5 / 13
    c2 = np.zeros((6, 6)); c2[:3, :3] = lam; c2[np.arange(3), np.arange(3)] += 2 * mu; c2[np.arange(3, 6), np.arange(3, 6)] = mu
    _, grad = element_geometry(4)
    ke1 = stiffness(grad, c1, 1 / 4 ** 3)
    ke2 = stiffness(grad, c2, 1 / 4 ** 3)

    # 4. Reference element action (fi_modal built from the reference header) on random DOFs.
    lib_path = REPO / "oracle/_ref/libref_fi_modal.so"
    lib = ctypes.CDLL(str(lib_path))
    rng = np.random.default_rng(20261203)
    U = rng.standard_normal((64, 24))
    fi = {}
    for name, c in (("study1", c1), ("paper", c2)):
        c21 = np.array([c[i, j] for i in range(6) for j in range(i, 6)])
        for n in (4, 64):
            h = 1.0 / n
            g = np.array([1 / (4 * h)] * 3 + [h ** 3])
            F = np.zeros_like(U)
            lib.ref_fi_modal_batch(U.ctypes.data_as(ctypes.c_void_p), c21.ctypes.data_as(ctypes.c_void_p),
                                   g.ctypes.data_as(ctypes.c_void_p), F.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.c_long(U.shape[0]))
            fi[f"{name}_n{n}"] = F

    # 5. Study I physical / OC chain at n=8 (reference functions).
    x = rng.uniform(0.1, 0.9, (8, 8, 8))
    ph, dp = pilot.physical(x, 2.0)
    energy = rng.uniform(0.5, 1.5, (8, 8, 8))
    g = pilot.filt(dp * 3 * (1 - 1e-4) * ph ** 2 * energy)
    dv = pilot.filt(dp)
    new = pilot.oc(x, g, dv, 2.0)

    # 6. Study II stencil, initial fields and the dense FE reference at n=4.
    sys.path.insert(0, str(ref / "exp/asg_gpu_resident_20261103"))
    sys.path.insert(0, str(ref / "exp/asg_scenarios_20261105"))
    sys.path.insert(0, str(ref / "exp/asg_sctop_reproduction_20261105"))
    import reproduction as rp
    import verify as sv  # scenarios' dense FE reference (dense_reference)
    offs, ws = rp.stencil(3.2)
    init = {f"initial_f{k}_n12": rp.initial(12, k) for k in (1, 2, 3, 4)}
    a4 = np.exp(rng.uniform(-4, 0, (4, 4, 4)))
    loads = np.vstack([np.eye(6), [1, 1, 1, 0, 0, 0]])
    ur, rr, qr, er = sv.dense_reference(SimpleNamespace(C0=c2), 4, a4, loads)

    np.savez_compressed(HERE / "reference_cpu.npz", ke_study1_n4=ke1, ke_paper_n4=ke2, fi_dofs=U,
                        **{f"fi_{k}": v for k, v in fi.items()},
                        s1_x=x, s1_ph=ph, s1_dp=dp, s1_energy=energy, s1_g=g, s1_dv=dv, s1_new=new,
                        cone_offsets=offs, cone_weights=ws, **init,
                        dense_a=a4, dense_u=ur, dense_rhs=rr, dense_moduli=qr, dense_energies=er)
    (HERE / "reference_meta.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", sorted(p.name for p in HERE.iterdir()))


if __name__ == "__main__":
    main()

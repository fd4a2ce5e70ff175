"""Regenerate tests/golden/oracle_small.npz: a small em2 case run through the
oracle (three full steps and the separate move / curnt / fields pieces),
used to catch any change in the oracle's arithmetic.  The reference em2 is
Fortran + MPI and cannot be built in this environment, so the oracle itself
is pinned by tests/golden/em2_initial_state.json (the reference's published
initial-state numbers) and these vectors freeze the pinned oracle.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def small_case(seed=7, nx=16, ny=12, n=300):
    rng = np.random.default_rng(seed)
    p = oracle.Params(nx=nx, ny=ny, dx=0.5, dy=0.5, dt=0.05,
                      qm=[-1.0, 1 / 25.0], q=[-0.02, 0.02], dn=[1.0, 1.0],
                      am=[0.02, 0.5], isav=2)
    fld = np.zeros((13, ny + 3, nx + 3))
    fld[:6] = rng.normal(scale=0.05, size=(6, ny + 3, nx + 3))
    parts = []
    for s in range(2):
        x = rng.random(n) * nx
        y = rng.random(n) * ny
        u = rng.normal(scale=0.1 if s == 0 else 0.02, size=(3, n))
        g = np.sqrt(1 + (u * u).sum(0))
        parts.append(np.vstack([x, y, u / g, g]))
    return p, fld, parts


def run(p, fld, parts):
    st = oracle.State(p, fld, parts)
    out = {}
    ake = st.move()
    out["move_ake"] = np.array(ake)
    out["move_part0"] = st.parts[0].copy()
    st.curnt()
    out["curnt_fld"] = st.fld.copy()
    out["curnt_part1"] = st.parts[1].copy()
    n, e6 = st.fields(2)
    out["fields_fld"] = st.fld.copy()
    out["fields_cg"] = np.array([n])
    out["fields_e6"] = e6
    st.it = 2
    for k in range(3):
        r = st.step()
    out["step3_fld"] = st.fld.copy()
    out["step3_part0"] = st.parts[0].copy()
    out["step3_ake"] = r["ake"]
    return out


if __name__ == "__main__":
    p, fld, parts = small_case()
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **run(p, fld, parts))
    print("wrote", os.path.join(HERE, "oracle_small.npz"))

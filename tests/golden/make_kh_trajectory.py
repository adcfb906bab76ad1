"""Generate the Kelvin-Helmholtz trajectory fixture from the CPU oracle.

The case: BASELINE config 3's flow (KelvinHelmholtzInstability.hpp:17-22) on
a 128^2 periodic quad mesh on [-1,1]^2, N=3, modal indicator with
alpha_max 0.5 and subcell FV blending (reference mode), SSP-RK3 at the fixed
dt = 0.4 hmin / (lambda_max(u0) (N+1)^2), 8000 steps (t ~ 1.38; the indicator
first blends elements near step 7000).  The oracle (oracle/liboracle.so, the
restatement of the reference's operator) advances it; the fixture keeps the
state at steps 4000, 7000 and 8000 on a fixed sample of 8192 DOFs, the
per-field L2 norms of the full states and the number of blended elements at
step 8000.  About 30 minutes on 8 cores.

    python tests/golden/make_kh_trajectory.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from prandtl_b200 import cases  # noqa: E402
from prandtl_b200.ensemble import fixed_dt  # noqa: E402

N_EL, ORDER, STEPS = 128, 3, (4000, 7000, 8000)


def sample_index(size, count=8192, seed=20261205):
    return np.sort(np.random.default_rng(seed).choice(size, count, replace=False))


def main():
    import pyoracle
    mesh, u, _ = cases.make_case("kh", N_EL, ORDER)
    dt = fixed_dt(mesh, u, 0.4)
    op = pyoracle.Oracle(mesh, blending=1, alpha_max=0.5, quirks=0)
    idx = sample_index(u.size)
    out = {"dt": np.array(dt), "index": idx}
    done = 0
    for s in STEPS:
        u = op.step(u, dt, scheme=0, nsteps=s - done)
        done = s
        out[f"u{s}"] = u[idx]
        out[f"norm{s}"] = np.linalg.norm(u.reshape(4, -1), axis=1)
    out["blended8000"] = np.array(int((op.rhs(u, want_alpha=True)["alpha"] > 0).sum()))
    np.savez_compressed(os.path.join(HERE, "kh128_trajectory.npz"), **out)
    print("blended elements at step 8000:", int(out["blended8000"]))


if __name__ == "__main__":
    main()

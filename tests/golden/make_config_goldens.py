"""Oracle fixtures for the large parity cases: tests/golden/config_goldens.json.

The oracle (oracle/ueg_oracle.c, the reference's Fortran restated loop for loop and
pinned bitwise to the reference's own outputs by tests/test_oracle_golden.py) needs
minutes of one host core per converged N=54 solve (about 3 s per CCD iteration).
This script runs those solves once, on every core of the machine it runs on, and
stores what the GPU tests compare against:

  c2_rs1, c2_rs5   N=54, 'Momentum Cutoff: 24' (485 plane waves), Gamma point, rs 1 and 5:
                   the reference's own iteration (1/2-damped Jacobi, inert DIIS, TolMax
                   1e-8; DrvCCD, CCD.f90:53-124) run to its stopping point.
  c4_twK           the 100-twist N=54 rs=1 batch workload (twists from numpy
                   default_rng(2024) in [-0.5,0.5)^3, |n|^2 <= 30 pool, fcut 6.857 -> 485
                   orbitals), twists K = 0, 1, 2: the same replay run, and a tight run of
                   the same iteration to max|dT| < 1e-12 (the fixed point, against which
                   a Pulay-DIIS solve on the GPU is compared).

Each case keeps the Input keys it was built from, NOcc and NAO, E(2), the iteration
count, every iteration's energy and max|dT|, Ec, MaxRes and the fail flag.

    python tests/golden/make_config_goldens.py            # about 10 minutes on 8 cores
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "config_goldens.json")

# the batched-twist workload: N=54, rs=1, |n|^2 <= 30 candidate pool, fcut 6.857 (485 orbitals)
TWIST_SEED = 2024
TWIST_COUNT = 100
TWIST_IDS = (0, 1, 2)


def batch_twists():
    import numpy as np

    return np.random.default_rng(TWIST_SEED).random((TWIST_COUNT, 3)) - 0.5


def case_keys():
    cases = {}
    for rs in ("1.0", "5.0"):
        name = "c2_rs" + rs[0]
        cases[name] = ({"# Electrons": "54", "Momentum Cutoff": "24", "rSMin": rs, "rSMax": rs}, 0.0)
    tw = batch_twists()
    for k in TWIST_IDS:
        keys = {"# Electrons": "54", "Momentum Cutoff": "30", "rSMin": "1.0", "rSMax": "1.0", "fcut": "6.857",
                "NTwist": " ".join(repr(float(x)) for x in tw[k])}
        cases[f"c4_tw{k}"] = (keys, 0.0)
        cases[f"c4_tw{k}_tight"] = (keys, 1e-12)
    return cases


def run_case(item):
    name, (keys, tol) = item
    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle, parse_input_text

    vals = parse_input_text("")
    vals.update(keys)
    o = Oracle(vals)
    t0 = time.time()
    e2, ta, tb, tc, _ = o.mp2()
    st, en, dts = o.ccd(ta, tb, tc, max_rec=1100, tol=tol)
    return name, {
        "keys": keys, "tol_override": tol, "nocc": o.nocc, "nao": o.nao, "e2": e2,
        "niter": st.niter, "ecorr": st.ecorr, "max_res": st.max_res, "last_dt": st.last_dt, "fail": st.fail,
        "energies": [float(x) for x in en], "dts": [float(x) for x in dts],
        "oracle_seconds": round(time.time() - t0, 1),
    }


def main():
    cases = case_keys()
    only = set(sys.argv[1:])
    items = [(k, v) for k, v in cases.items() if not only or k in only]
    out = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            out = json.load(f)
    # the longest runs first, one process per case
    items.sort(key=lambda kv: (kv[1][1] == 0.0, kv[0] != "c2_rs5"))
    with mp.get_context("spawn").Pool(min(len(items), os.cpu_count() or 1)) as pool:
        for name, rec in pool.imap_unordered(run_case, items):
            out[name] = rec
            print(f"{name}: niter {rec['niter']} Ec {rec['ecorr']:.12f} ({rec['oracle_seconds']} s)", flush=True)
    out["source"] = ("oracle/ueg_oracle.c (the reference restated; pinned by tests/test_oracle_golden.py), "
                     "written by tests/golden/make_config_goldens.py")
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

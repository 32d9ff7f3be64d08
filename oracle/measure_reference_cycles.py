"""Record how many GMRES(12) restart cycles the reference algorithm needs.

Runs the oracle's FP64 restatement of CSLASolverGMRES (SparseLinearAlgebra/
CSolverGMRES.cpp:111-358: MGS Arnoldi, Givens, restart) on the even-odd Wilson
system of a bench workload until the true relative residual of the full system
is <= 1e-10, and writes the cycle count to oracle/reference_cycles.json.  The
reference arm of bench.py times a bounded number of cycles on the box's host
cores and converts with this count.

  python oracle/measure_reference_cycles.py wilson_eo_32x32x32x16
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from bench import WORKLOADS  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main(name):
    W = WORKLOADS[name]
    L, kappa = W["dims"], W["kappa"]
    V = int(np.prod(L))
    U = O.gauge_expH(L, W["seed"], W["eps"])
    b = O.gauss(V, 12, W["seed"], 2).reshape(V, 4, 3)
    pm = O.parity_mask(L)
    be, bo = b.copy(), b.copy()
    be[pm == 1] = 0
    bo[pm == 0] = 0
    bt = be + kappa * O.wilson_hop(L, U, bo, 0)
    op = O.Operator("WILSON_MEE", L, U, kappa)
    full = O.Operator("WILSON_D", L, U, kappa)
    x = None
    cycles = 0
    t0 = time.time()
    chunk = 10
    res = 1.0
    while cycles < 20000:
        x, info = O.gmres(op, bt, x0=x, maxdim=12, restart=chunk, accuracy=0.0)
        cycles += chunk
        xo = bo + kappa * O.wilson_hop(L, U, x, 1)
        xf = x.copy()
        xf[pm == 1] = xo[pm == 1]
        res = full.true_residual(b, xf)
        print(f"cycles {cycles} true residual {res:.3e} ({time.time() - t0:.0f} s)", flush=True)
        if res <= 1e-10:
            break
    # refine to the exact cycle within the last chunk
    path = os.path.join(HERE, "reference_cycles.json")
    d = json.load(open(path)) if os.path.exists(path) else {}
    d[name] = {"cycles": cycles, "granularity": chunk, "true_rel_residual": res, "maxdim": 12,
               "seconds_here": round(time.time() - t0, 1)}
    json.dump(d, open(path, "w"), indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "wilson_eo_32x32x32x16")

"""Golden outputs of the reference's own CUDA implementation of the path.

Runs CLGLib itself (FP64, sm_100a; built from the reference's sources by
``oracle/ref/Makefile`` into ``oracle/_ref/clg_ref_driver``) on seeded inputs
made by the oracle's generator, and writes what it returns as compact fixtures
``ref_<case>.npz``:

* ``<op>.proj``  : 8 inner products <r_k, y> of the output y with fixed probe
  fields r_k (oracle Gaussian generator, seed 0x5EED0000, field ids 200..207);
* ``<op>.sites`` / ``<op>.vals`` : the output at 67 sampled sites (every V/64-th
  site plus the lattice's last site and the two sites next to the t boundary);
* ``<op>.norm2`` : |y|^2;
* ``<op>.ms``    : the device time of the call;
* ``<op>.true_res``: for solves, |b - (A + c) x| / |b| of the reference's
  solution x, recomputed by the oracle's FP64 operator when the fixture was made.

The inputs are not stored: the oracle's generator reproduces them bit for bit
from the recorded seeds, and ``input_sha256`` records the bytes the reference
was given.  Needs a GPU (the driver is CUDA code).  Usage:

    python tests/golden/make_ref_golden.py --driver oracle/_ref/clg_ref_driver \
        --work /tmp/refwork --out tests/golden [--timing TIMING.json]

``--timing`` adds the reference's timings on the 32^3x16 exp(i eps H) lattice
(Wilson D applications and one full GMRES(12) solve of D x = b) and writes them
as JSON; no fixture is made from those.
"""
import argparse
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

KAPPA = 0.1355
MASS_2AM = 0.02
PROBE_SEED = 0x5EED0000
NPROBE = 8
# the complex shifts of the reference's multi-shift test (Tests/TestMultiShiftSolver.cpp:22-28)
WILSON_SHIFTS = [2.0, 1.0, 0.5, 1j, 0.5 + 0.5j, 1.0 - 1.0j]
KS_SHIFTS = [float(s) for s in np.logspace(-2, 1, 6)]


def sample_sites(L):
    V = O.volume(L)
    step = V // 64
    s = list(range(0, V, step))[:64]
    Lt = L[3]
    s += [V - 1, Lt - 1, Lt]          # last site; t = Lt-1 and t = 0 of the next column
    return np.array(sorted(set(s)), np.int64)


def probes(V, ncomp):
    return [O.gauss(V, ncomp, PROBE_SEED, 200 + k).reshape(-1) for k in range(NPROBE)]


def summarize(y, pr, sites):
    V = y.shape[0]
    flat = y.reshape(V, -1)
    return {
        "proj": np.array([np.vdot(p, flat.reshape(-1)) for p in pr]),
        "sites": sites,
        "vals": flat[sites],
        "norm2": float(np.vdot(flat, flat).real),
    }


def yaml_job(path, L, gauge_file, fermion, src_file, out_prefix, ops, solver=None, ms_solver=None,
             shifts=None, repeat=20, pool=40):
    """A CLGLib parameter file (the keys of Bin/Debug/TestSuit_Solver.yaml) plus the RefJob block."""
    lines = [
        "Job:", "",
        "    Dim : 4", "    Dir : 4",
        "    LatticeLength : [%d, %d, %d, %d]" % tuple(L),
        "    LatticeIndex : CIndexSquare",
        "    LatticeBoundary : CBoundaryConditionTorusSquare",
        "    ThreadAutoDecompose : 1",
        "    RandomType : ER_Schrage", "    RandomSeed : 1234567",
        "    ExponentialPrecision : 4",
        "    FermionFieldCount : 1", "",
        "    Gauge:", "",
        "        FieldName : CFieldGaugeSU3",
        "        FieldInitialType : EFIT_ReadFromFile",
        "        GaugeFileType : EFFT_CLGBinDouble",
        "        GaugeFileName : %s" % gauge_file,
        "        Period : [1, 1, 1, 1]", "",
        "    FermionField1:", "",
    ]
    if fermion == "wilson":
        lines += ["        FieldName : CFieldFermionWilsonSquareSU3",
                  "        Hopping : %r" % KAPPA]
    else:
        lines += ["        FieldName : CFieldFermionKSSU3",
                  "        Mass : %r" % MASS_2AM,
                  "        MC : [1.0]", "        MD : [1.0]"]
    lines += ["        FieldInitialType : EFIT_ReadFromFile",
              "        FieldId : 2", "        PoolNumber : %d" % pool,
              "        Period : [1, 1, 1, -1]", ""]
    for name, block in (("Solver", solver), ("MSSolver", ms_solver)):
        if block:
            lines += ["    %s:" % name, ""] + ["        %s : %s" % kv for kv in block.items()] + [""]
    job = ["    RefJob:", "",
           "        SourceFile : %s" % src_file,
           "        OutPrefix : %s" % out_prefix,
           "        Ops : [%s]" % ", ".join(ops),
           "        Repeat : %d" % repeat]
    if shifts:
        job += ["        ShiftRe : [%s]" % ", ".join(repr(complex(c).real) for c in shifts),
                "        ShiftIm : [%s]" % ", ".join(repr(complex(c).imag) for c in shifts)]
    with open(path, "w") as f:
        f.write("\n".join(lines + job) + "\n")


def run_driver(driver, yaml_path, timeout):
    p = subprocess.run([driver, yaml_path], capture_output=True, text=True, timeout=timeout)
    results = {}
    for line in p.stdout.splitlines():
        if line.startswith("REFRESULT "):
            r = json.loads(line[len("REFRESULT "):])
            results[r["op"]] = r
    if p.returncode != 0:
        sys.stderr.write(p.stdout[-4000:] + p.stderr[-4000:])
        raise RuntimeError("reference driver exited %d on %s" % (p.returncode, yaml_path))
    return results


def read_field(path, V, ncomp):
    raw = np.fromfile(path, np.float64)
    assert raw.size == V * 2 * ncomp, (path, raw.size)
    return raw.view(np.complex128).reshape(V, ncomp)


def make_inputs(case):
    L = case["L"]
    V = O.volume(L)
    if case["links"] == "haar":
        U = O.gauge_haar(L, case["seed"], 1)
    else:
        U = O.gauge_expH(L, case["seed"], 0.25)
    ncomp = 12 if case["fermion"] == "wilson" else 3
    b = O.gauss(V, ncomp, case["seed"], 2)
    return L, V, U, b, ncomp


def oracle_op(case, L, U):
    if case["fermion"] == "wilson":
        return lambda op, x: {
            "D": lambda v: O.wilson_D(L, U, v, KAPPA),
            "Ddagger": lambda v: O.wilson_D(L, U, v, KAPPA, dagger=True),
        }[op](x)
    return lambda op, x: {
        "D": lambda v: O.ks_D(L, U, v, MASS_2AM),
        "Ddagger": lambda v: O.ks_D(L, U, v, MASS_2AM, dagger=True),
    }[op](x)


def residual(case, L, U, b, x, base, shift=0j):
    A = oracle_op(case, L, U)
    shp = b.shape
    xs = x.reshape(shp)
    if base == "D":
        Ax = A("D", xs)
    elif base == "Ddagger":
        Ax = A("Ddagger", xs)
    else:  # DDdagger
        Ax = A("D", A("Ddagger", xs))
    r = b - Ax - shift * xs
    return float(np.linalg.norm(r) / np.linalg.norm(b))


CASES = [
    # the small 8^4 workload: Haar links, one Gaussian source; D, D^+, products,
    # GMRES(12), BiCGStab and the multi-shift FOM on the reference test's shifts
    {"name": "wilson_haar_8x8x8x8", "L": (8, 8, 8, 8), "links": "haar", "seed": 0xC1A60000,
     "fermion": "wilson",
     "jobs": [
         {"ops": ["D", "Ddagger", "DD", "DDdagger", "InverseD", "InverseDdagger"],
          "solver": "gmres"},
         {"ops": ["InverseD"], "solver": "bicgstab", "tag": "bicgstab"},
         {"ops": ["MultiShiftD"], "ms_solver": "fom", "shifts": WILSON_SHIFTS},
         {"ops": ["MultiShiftD"], "ms_solver": "gmres_ms", "shifts": WILSON_SHIFTS, "tag": "gmres"},
         {"ops": ["MultiShiftD"], "ms_solver": "bicgstab_ms", "shifts": WILSON_SHIFTS, "tag": "bicgstab"},
     ]},
    # the near-ordered exp(i eps H) links of configs 2-4 on 8^3x16
    {"name": "wilson_expH_8x8x8x16", "L": (8, 8, 8, 16), "links": "expH", "seed": 0xC1A60001,
     "fermion": "wilson",
     "jobs": [
         # restarted GMRES(12) stagnates on this field: a budget of 100 cycles
         {"ops": ["D", "Ddagger", "InverseD"], "solver": "gmres", "restart": 100},
     ]},
    # staggered (DD^+)_ee, the multi-shift workload's operator, on 8^3x16, 2am = 0.02
    {"name": "ks_expH_8x8x8x16", "L": (8, 8, 8, 16), "links": "expH", "seed": 0xC1A60005,
     "fermion": "ks",
     "jobs": [
         {"ops": ["D", "Ddagger", "DDdagger"]},
         {"ops": ["MultiShiftDDdagger"], "ms_solver": "fom", "shifts": KS_SHIFTS},
     ]},
]


def solver_block(kind, bnorm):
    if kind == "gmres":
        # stop when |g_m|^2 < Accuracy (absolute): relative estimate 1e-12
        return {"SolverName": "CSLASolverGMRES", "SolverForFieldId": 2, "UseCudaForSmallMatrix": 0,
                "MaxDim": 12, "Restart": 2000, "AbsoluteAccuracy": 1,
                "Accuracy": repr((1e-12 * bnorm) ** 2)}
    if kind == "bicgstab":
        # stop when |s|^2 < Accuracy, checked every DiviationStep iterations
        return {"SolverName": "CSLASolverBiCGStab", "SolverForFieldId": 2, "DiviationStep": 1,
                "MaxStep": 500, "Restart": 5, "AbsoluteAccuracy": 1,
                "Accuracy": repr((1e-12 * bnorm) ** 2)}
    if kind == "fom":
        # stop when every |beta_n| < Accuracy
        return {"SolverName": "CMultiShiftFOM", "SolverForFieldId": 2, "UseCudaForSmallMatrix": 0,
                "MaxDim": 30, "Restart": 2000, "AbsoluteAccuracy": 1,
                "Accuracy": repr(1e-12 * bnorm)}
    if kind == "gmres_ms":
        # stop when every collinearity factor |beta0_n| < Accuracy (absolute)
        return {"SolverName": "CMultiShiftGMRES", "SolverForFieldId": 2, "MaxDim": 10, "Restart": 2000,
                "AbsoluteAccuracy": 1, "Accuracy": repr(1e-12)}
    if kind == "bicgstab_ms":
        # stop when |s| and every |s_n| < Accuracy, checked every DiviationStep iterations
        return {"SolverName": "CMultiShiftBiCGStab", "SolverForFieldId": 2, "DiviationStep": 10, "MaxStep": 500,
                "AbsoluteAccuracy": 1, "Accuracy": repr(1e-12 * bnorm)}
    raise ValueError(kind)


def make_case(case, driver, work, out):
    L, V, U, b, ncomp = make_inputs(case)
    gauge_file = os.path.join(work, case["name"] + ".gauge.bin")
    src_file = os.path.join(work, case["name"] + ".src.bin")
    U.astype(np.complex128).tofile(gauge_file)
    b.astype(np.complex128).tofile(src_file)
    bnorm = float(np.linalg.norm(b))
    pr = probes(V, ncomp)
    sites = sample_sites(L)
    rec = {"dims": np.array(L), "kappa": KAPPA, "mass_2am": MASS_2AM, "seed": case["seed"],
           "links": case["links"], "fermion": case["fermion"],
           "input_sha256": hashlib.sha256(U.tobytes() + b.tobytes()).hexdigest()}
    for j, job in enumerate(case["jobs"]):
        prefix = os.path.join(work, "%s.job%d" % (case["name"], j))
        yml = prefix + ".yaml"
        sblock = solver_block(job["solver"], bnorm) if job.get("solver") else None
        if sblock and "restart" in job:
            sblock["Restart"] = job["restart"]
        yaml_job(yml, L, gauge_file, case["fermion"], src_file, prefix, job["ops"],
                 solver=sblock,
                 ms_solver=solver_block(job["ms_solver"], bnorm) if job.get("ms_solver") else None,
                 shifts=job.get("shifts"))
        res = run_driver(driver, yml, timeout=600)
        for op in job["ops"]:
            r = res[op]
            key = op if "tag" not in job else "%s_%s" % (op, job["tag"])
            if op.startswith("MultiShift"):
                base = op[len("MultiShift"):]
                for k, c in enumerate(job["shifts"]):
                    x = read_field("%s.%s.%d.bin" % (prefix, op, k), V, ncomp)
                    s = summarize(x, pr, sites)
                    for f, v in s.items():
                        rec["%s.%d.%s" % (key, k, f)] = v
                    rec["%s.%d.true_res" % (key, k)] = residual(case, L, U, b, x, base, c)
                rec[key + ".shifts"] = np.array(job["shifts"], np.complex128)
            else:
                y = read_field("%s.%s.bin" % (prefix, op), V, ncomp)
                for f, v in summarize(y, pr, sites).items():
                    rec["%s.%s" % (key, f)] = v
                if op.startswith("Inverse"):
                    rec[key + ".true_res"] = residual(case, L, U, b, y, op[len("Inverse"):])
            rec[key + ".ms"] = r["ms"]
            rec[key + ".ok"] = r["ok"]
            if sblock and op.startswith("Inverse"):
                rec[key + ".restart"] = int(sblock["Restart"])
    path = os.path.join(out, "ref_%s.npz" % case["name"])
    np.savez_compressed(path, **rec)
    print("wrote", path)


def timing(driver, work, path):
    """The reference on the 32^3x16 exp(i eps H) lattice: D / D^+ applications
    and one GMRES(12) solve of the full D to relative residual 1e-10."""
    case = {"name": "timing_32x32x32x16", "L": (32, 32, 32, 16), "links": "expH", "seed": 0xC1A60001,
            "fermion": "wilson"}
    L, V, U, b, ncomp = make_inputs(case)
    gauge_file = os.path.join(work, "timing.gauge.bin")
    src_file = os.path.join(work, "timing.src.bin")
    U.tofile(gauge_file)
    b.tofile(src_file)
    bnorm = float(np.linalg.norm(b))
    prefix = os.path.join(work, "timing")
    solver = solver_block("gmres", bnorm)
    solver["Accuracy"] = repr((1e-10 * bnorm) ** 2)
    solver["Restart"] = 2000
    yml = prefix + ".yaml"
    yaml_job(yml, L, gauge_file, "wilson", src_file, prefix, ["TimeD", "TimeDdagger", "InverseD"],
             solver=solver, repeat=50)
    res = run_driver(driver, yml, timeout=1800)
    x = read_field(prefix + ".InverseD.bin", V, ncomp)
    out = {"lattice": list(L), "links": "exp(i 0.25 H), seed 0xC1A60001", "kappa": KAPPA,
           "build": "CLGLib FP64 (_CLG_DOUBLEFLOAT=1), -gencode arch=compute_100a,code=sm_100a, -O3",
           "D_ms": res["TimeD"]["ms_per_apply"], "Ddagger_ms": res["TimeDdagger"]["ms_per_apply"],
           "gmres12_solve_ms": res["InverseD"]["ms"], "gmres12_ok": res["InverseD"]["ok"],
           "gmres12_true_rel_residual": residual(case, L, U, b, x, "D")}
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--driver", required=True)
    ap.add_argument("--work", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--timing", default=None)
    ap.add_argument("--cases", default=None, help="comma-separated case names (default: all)")
    a = ap.parse_args()
    os.makedirs(a.work, exist_ok=True)
    os.makedirs(a.out, exist_ok=True)
    O.build()
    want = set(a.cases.split(",")) if a.cases else None
    for case in CASES:
        if want is None or case["name"] in want:
            make_case(case, a.driver, a.work, a.out)
    if a.timing:
        timing(a.driver, a.work, a.timing)


if __name__ == "__main__":
    main()

"""Generate the committed golden fixtures from the reference source tree.

Run in a container where the CudaLatticeGauge sources are mounted (default
path below, or pass it as the first argument).  Outputs, next to this script:

  bridgepp_4x4x4x8.npz   the reference's Bridge++ 4^3x8 configuration
                         (Bin/Debug/bridgepp_conf_text.dat) as float64, Bridge++
                         order; known plaquette 0.625129946974942
                         (Code/CLGTest/Tests/TestConfigurationFileIO.cpp:12-38)
  fileio.json            MD5 digests of the reference's configuration files
                         Bin/Release/bridgepp_conf_binary.dat (the same 4^3x8
                         configuration as big-endian doubles; checked here to
                         hold exactly the text file's values) and
                         Bin/Debug/testGaugeDouble.con_ / testGaugeSingle.con_
                         (8^4 CLGBin double / float), with the sum of |U|^2 that
                         TestConfigurationFileIO.cpp expects of the latter (49152)
  gamma_chiral.json      the chiral gamma-matrix table parsed from
                         Code/CLGLib/Tools/Math/GammaMatrix.h (the `else` branch of
                         gammaMatrixSet::CreateGammaMatrix): for GAMMA1..GAMMA5, per
                         row the non-zero column and the power b of i^b
"""
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    txt = os.path.join(ref, "Bin", "Debug", "bridgepp_conf_text.dat")
    vals = np.loadtxt(txt, dtype=np.float64)
    assert vals.size == 4 * 4 * 4 * 8 * 4 * 18
    np.savez_compressed(os.path.join(HERE, "bridgepp_4x4x4x8.npz"), links=vals,
                        dims=np.array([4, 4, 4, 8]), plaquette=np.array(0.625129946974942))

    binf = os.path.join(ref, "Bin", "Release", "bridgepp_conf_binary.dat")
    raw = open(binf, "rb").read()
    assert np.array_equal(np.frombuffer(raw, dtype=">f8").astype(np.float64), vals)
    info = {"bridgepp_conf_binary.dat": {"md5": hashlib.md5(raw).hexdigest(), "bytes": len(raw),
                                         "dims": [4, 4, 4, 8], "equals": "bridgepp_4x4x4x8.npz links, big-endian"}}
    for name, dt in (("testGaugeDouble.con_", "<f8"), ("testGaugeSingle.con_", "<f4")):
        raw = open(os.path.join(ref, "Bin", "Debug", name), "rb").read()
        u = np.frombuffer(raw, dtype=dt).astype(np.float64)
        info[name] = {"md5": hashlib.md5(raw).hexdigest(), "bytes": len(raw), "dims": [8, 8, 8, 8],
                      "sum_abs2": float(np.dot(u, u)), "expected_sum_abs2": 49152.0}
    with open(os.path.join(HERE, "fileio.json"), "w") as f:
        json.dump(info, f, indent=1)

    src = open(os.path.join(ref, "Code", "CLGLib", "Tools", "Math", "GammaMatrix.h")).read()
    start = src.index("CreateGammaMatrix(EGammaMatrixSet eSet")
    body = src[start:]
    chiral = body[body.index("else"):]  # the chiral branch follows the EGMS_Dirac branch
    table = {}
    for name in ("GAMMA1", "GAMMA2", "GAMMA3", "GAMMA4", "GAMMA5"):
        rows = {}
        for line in chiral.splitlines():
            s = line.strip()
            if s.startswith("//"):
                continue
            m = re.match(r"gmarray\[%s\]\.Set\((\d), (\d), (\d)\);" % name, s)
            if m:
                r, c, b = map(int, m.groups())
                rows.setdefault(r, [c, b])
        table[name] = [rows[r] for r in range(4)]
    with open(os.path.join(HERE, "gamma_chiral.json"), "w") as f:
        json.dump({"source": "Code/CLGLib/Tools/Math/GammaMatrix.h chiral set", "rows": table}, f, indent=1)


if __name__ == "__main__":
    # the CudaLatticeGauge source tree: first argument, else $CLG_REFERENCE
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CLG_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <CudaLatticeGauge tree>  (or set CLG_REFERENCE)")
    main(ref)

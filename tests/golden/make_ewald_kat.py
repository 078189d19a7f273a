"""Pin the Ewald reciprocal-space oracle against the reference's only numeric
known answer: cpu_gse.cpp:324-330 (ap-hynninen/GSE) hard-codes the Ewald-recip
energy 1733.61 for data/xyzq_48k.txt (48,191 charges), sigma=2.12132034355964,
box 80, kcut 64.

Runs in the container that holds the reference sources (it reads the data file
there) and writes tests/golden/ewald_kat_48k.json with the oracle's energy.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

REF_DATA = os.path.join(os.environ.get("GSE_REFERENCE_DIR", "/root/reference"), "data",
                        "xyzq_48k.txt")


def main():
    xyzq = np.loadtxt(REF_DATA, dtype=np.float64).reshape(-1, 4)
    t = time.time()
    e, _ = oracle.ewald_recip(2.12132034355964, 64, (80.0, 80.0, 80.0), xyzq, forces=False)
    out = {
        "source": "cpu_gse.cpp:324-330 (energy_ew = 1733.61)",
        "n": int(xyzq.shape[0]),
        "sigma": 2.12132034355964,
        "box": 80.0,
        "kcut": 64,
        "reference_energy": 1733.61,
        "oracle_energy": e,
        "oracle_seconds": time.time() - t,
    }
    with open(os.path.join(HERE, "ewald_kat_48k.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()

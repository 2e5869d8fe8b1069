"""Pack the reference's own full-run benchmark curves into reference_curves.npz.
Run in a container where the reference sources are present:

    python tests/golden/make_reference_curves.py [reference root]

Arrays:
  marshak_wave_<k>   (512, 3) x [cm], T_gas [K], T_rad [K]: the diffusion reference
                     profiles examples/marshak_wave_<k>/reference.txt, k = 1..4, read
                     as LoadReference reads them (MarshakCommon.hpp:176-191)
  densmore2012       (n, 2) x [cm], T_gas [keV]: the digitised Milagro curve
                     examples/densmore2012/data/densmore2012_fig4_mc.csv, read as
                     LoadCSV reads it (main.cpp:86-110: '#' lines skipped)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(root):
    out = {}
    for k in range(1, 5):
        path = os.path.join(root, "examples", f"marshak_wave_{k}", "reference.txt")
        out[f"marshak_wave_{k}"] = np.loadtxt(path, dtype=np.float64).reshape(-1, 3)
    rows = []
    with open(os.path.join(root, "examples", "densmore2012", "data", "densmore2012_fig4_mc.csv")) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            x, t = line.split(",")[:2]
            rows.append((float(x), float(t)))
    out["densmore2012"] = np.array(rows, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "reference_curves.npz"), **out)
    for k, v in out.items():
        print(k, v.shape)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("STORM_REFERENCE_SRC", "")
    if not src:
        sys.exit("usage: make_reference_curves.py <reference source tree> (or set STORM_REFERENCE_SRC)")
    main(src)

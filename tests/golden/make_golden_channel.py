"""Writes tests/golden/channel.json: the reference's own closed-form answers for the straight-duct
A + B -> C check, evaluated on the lattice the GPU test uses.

The reference checks a finished duct run with ABC_sweep_package/tools/analytic_channel.py: the
three reaction-free combinations A - B, A + C and B + C of a run with every x face held (Dirichlet
A = A0, B = 0 at x = 0; A = 0, B = B0 at x = nx - 1; C = 0 at both) are conservative tracers whose
steady cross-section means follow its ade_1d(x/L, s0, sL, Pe): exactly linear at Pe = 0, the 1-D
exponential profile at Pe > 0 (approximate in a duct). This script imports that module from the
reference checkout and records ade_1d at the duct's x-planes for each combination and Peclet
number, so the GPU test compares with the reference's function itself and not a restatement.

    python tests/golden/make_golden_channel.py <CompLaB3D-GEMS checkout>
"""
import json
import os
import sys

import numpy as np

NX = 34                       # lattice x-planes, the two Dirichlet planes included
PECLETS = [0.0, 0.5, 2.0]     # U (nx - 1) / D
A0, B0 = 1.0, 1.0             # the reference campaign's feeds (make_campaign.py A0, B0)


def main(ref):
    sys.path.insert(0, os.path.join(ref, "ABC_sweep_package", "tools"))
    import analytic_channel as ac

    x = np.arange(NX) / (NX - 1.0)  # as analytic_channel.main builds it
    cases = []
    for pe in PECLETS:
        for name, s0, sL in (("A - B", A0, -B0), ("A + C", A0, 0.0), ("B + C", 0.0, B0)):
            cases.append({"combination": name, "peclet": pe, "s0": s0, "sL": sL,
                          "profile": [float(v) for v in ac.ade_1d(x, s0, sL, pe)]})
    out = {"source": "ABC_sweep_package/tools/analytic_channel.py ade_1d", "nx": NX, "A0": A0, "B0": B0,
           "cases": cases}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "channel.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, len(cases), "profiles")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])

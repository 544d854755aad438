"""Generates the golden fixtures from the reference's own kernels.

Runs the reference's ConvexCell.cl / knearests.cl, compiled for the CPU by
oracle/build_ref.sh into oracle/_ref/libref_kernels.so, through the oracle's
restatement of the reference host flow (binning, passes, retries), on small
seeded inputs, and stores inputs and outputs in tests/golden/*.npz.  Needs
the reference sources at build time only; the fixtures are committed.

  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "gpu-restricted-power-diagrams_b200")):
    sys.path.insert(0, p)

import oracle  # noqa: E402
import rpd  # noqa: E402
from rpd import synth  # noqa: E402

CASES = {
    # no domain: unit box, weighted jittered lattice
    "lattice_w_nogrid": dict(seeds=lambda: synth.jittered_lattice(14, seed=11, weights=True), grid=None,
                             K=30, P=30, V=40, T=100),
    # ellipsoid blob domain, uniform seeds, small caps (retry passes)
    "uniform_blob24": dict(seeds=lambda: synth.uniform(3000, seed=12), grid=(24, 5, 2), K=20, P=25, V=30, T=60),
    # weighted lattice in a blob at a finer grid
    "lattice_w_blob32": dict(seeds=lambda: synth.jittered_lattice(16, seed=13, weights=True), grid=(32, 3, 7),
                             K=50, P=30, V=40, T=100),
}


def main():
    if not oracle.has_reference_kernels():
        sys.exit("reference kernels not built (oracle/build_ref.sh needs the reference sources)")
    for name, c in CASES.items():
        x = c["seeds"]().astype(np.float64)
        out = {"xyzw": x.astype(np.float32), "caps": np.array([c["K"], c["P"], c["V"], c["T"]], np.int32)}
        ga = None
        if c["grid"] is not None:
            g = rpd.Grid.blob(*c["grid"])
            a = g.arrays()
            for k, v in a.items():
                out["grid_" + k] = np.asarray(v)
            ga = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"],
                                   a["offsets"])
        out["knn_ref"] = oracle.knn(x, c["K"], kernels=1, knn_mode=0)
        for tag, dbl in (("f32", False), ("f64", True)):
            b, s, st = oracle.solve(x, grid=ga, K=c["K"], P=c["P"], V=c["V"], T=c["T"], vhs0=2, vhs1=2,
                                    use_double=dbl, kernels=1, knn_mode=0, return_stats=True)
            out[f"bary_{tag}"] = b
            out[f"status_{tag}"] = s
            out[f"passes_{tag}"] = np.array(st["pass_cells"], np.int32)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, len(x), "passes", out["passes_f64"].tolist())


if __name__ == "__main__":
    main()

"""Regenerate tests/golden/oracle_fixtures.json from the checker (oracle/).

The fixtures pin outcomes that take the checker long to recompute, so that the
GPU tests can compare against them directly:
  * LAS2 on the 5000 x 2000 Poisson(20) workload (seed 42, dimensions 10) for
    lanczos::svd_las2 as written and for legacy::svdLAS2;
  * start-vector draws (bit patterns) for a few seeds;
  * as-written lanczos::svd_las2 results on the small golden matrices.

Usage: python tests/golden/make_fixtures.py   (about 90 s, single-threaded)
"""
import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

import matrices as M  # noqa: E402
import oracle as O  # noqa: E402


def hexd(x):
    return struct.pack("<d", float(x)).hex()


def main():
    O.set_threads(1)
    out = {"_source": "generated by tests/golden/make_fixtures.py from oracle/svd_oracle.cpp"}
    out["start_vector"] = {str(seed): [hexd(v) for v in O.start_vector(seed, 37)] for seed in (1, 42, 3141, 4294967295)}

    A = M.poisson_rows(5000, 2000, 20, 42)
    cfg = {"nnz": int(len(A["data"])), "sparsity": 1 - len(A["data"]) / (5000 * 2000)}
    r = O.las2("csr", A, 10, 0, seed=42, legacy=True)
    cfg["legacy"] = {"d": r["d"], "s": r["s"].tolist(), "lanczos_steps": r["diagnostics"]["lanczos_steps"],
                     "ritz_values_stabilized": r["diagnostics"]["ritz_values_stabilized"],
                     "singular_values": r["diagnostics"]["singular_values"]}
    try:
        O.las2("csr", A, 10, 0, seed=42, legacy=False)
        cfg["lanczos"] = {"error": None}
    except O.OracleError as e:
        cfg["lanczos"] = {"error": e.kind, "message": str(e), "lanczos_steps": e.steps + 1}
    out["poisson_5000x2000_seed42_dim10"] = cfg

    small = {}
    for name, Mx, fmt, seed in [("basic_2x2", [[4, 0], [3, -5]], "csr", 42),
                                ("squares_3x3", [[1, 16, 49], [4, 25, 64], [9, 36, 81]], "csc", 3141)]:
        A = M.dense(Mx)
        if fmt == "csc":
            A = M.to_csc(A)
        r = O.las2(fmt, A, 0, 0, seed=seed, legacy=False)
        small[name] = {"seed": seed, "format": fmt, "d": r["d"], "s": r["s"].tolist(),
                       "lanczos_steps": r["diagnostics"]["lanczos_steps"]}
    out["lanczos_as_written"] = small
    with open(os.path.join(HERE, "oracle_fixtures.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "oracle_fixtures.json"))


if __name__ == "__main__":
    main()

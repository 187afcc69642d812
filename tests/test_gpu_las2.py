"""LAS2 on the GPU against the checker: lanczos::svd_las2 as written and
legacy::svdLAS2, through the C ABI (libsvdb200.so).

Tolerances: singular values 1e-10 relative to the largest; alpha/beta of the
first steps 1e-10 relative; converged singular vectors parallel to 1e-8.  The
GPU sums dot products in a different order than the crate, so exact bits are
not expected, but the decisions (steps, stabilised Ritz values, significant
values) must agree.
"""
import json
import os
import struct

import numpy as np
import pytest

import matrices as M
import oracle as O
from gpu_util import assert_rows_parallel, oracle_args, upload
from single_svdlib import Imtql2Error, Las2Error, StartvError, lanczos, legacy

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.json")))
FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_fixtures.json")))

CASES = {
    "dense_30x20": lambda: M.uniform(30, 20, 1.0, 1),
    "sparse_200x120": lambda: M.uniform(200, 120, 0.05, 2),
    "wide_60x150": lambda: M.uniform(60, 150, 0.1, 3),
    "poisson_800x300": lambda: M.poisson_rows(800, 300, 8, 4),
    "lowrank_150x90": lambda: M.lowrank_plus_noise(150, 90, 5, 1e-6, 5),
}


def run_pair(kind, A, dims, seed, algorithm, iterations=0):
    ref, ref_err = None, None
    try:
        ref = O.las2(kind if kind != "masked" else "masked", oracle_args(kind, A), dims, iterations, seed=seed,
                     legacy=(algorithm == "legacy"))
    except O.OracleError as e:
        ref_err = e
    got = lanczos.las2_traced(upload(kind, A), dims, iterations, random_seed=seed, algorithm=algorithm)
    return ref, ref_err, got


def check_same(ref, got, s_tol=1e-10, vec_tol=1e-8, check_vectors=True):
    rec = got["rec"]
    assert got["error"] is None, got["error"]
    dg = rec.diagnostics
    assert rec.d == ref["d"]
    assert dg.lanczos_steps == ref["diagnostics"]["lanczos_steps"]
    assert dg.ritz_values_stabilized == ref["diagnostics"]["ritz_values_stabilized"]
    assert dg.singular_values == ref["diagnostics"]["singular_values"]
    assert dg.transposed == ref["diagnostics"]["transposed"]
    assert rec.u.shape == ref["ut"].shape and rec.vt.shape == ref["vt"].shape
    k = min(20, ref["steps"] + 1)
    scale = max(np.max(np.abs(ref["alf"][:k])), 1e-300)
    np.testing.assert_allclose(got["alf"][:k], ref["alf"][:k], rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(got["bet"][:k], ref["bet"][:k], rtol=0, atol=1e-10 * scale)
    if rec.d and s_tol is not None:
        smax = np.max(np.abs(ref["s"]))
        np.testing.assert_allclose(rec.s, ref["s"], rtol=0, atol=s_tol * smax)
        if check_vectors:
            assert_rows_parallel(rec.vt, ref["vt"], vec_tol)
            assert_rows_parallel(rec.u, ref["ut"], vec_tol)


@pytest.mark.parametrize("case", sorted(CASES))
def test_legacy_parity(case):
    A = CASES[case]()
    ref, err, got = run_pair("csr", A, 6, 4242, "legacy")
    assert err is None, err
    check_same(ref, got)


def ulp_spread(A, dims, seed, trials=6):
    """Largest change of the checker's singular values when A's values move by one ulp.

    lanczos::svd_las2 as written applies non-orthogonal QL rotations
    (svd_pythag mod.rs:372, imtqlb mod.rs:452-453), so on long runs its output
    is not a continuous function of the input bits; this measures by how much.
    """
    base = O.las2("csr", A, dims, 0, seed=seed, legacy=False)
    rng = np.random.default_rng(0)
    spread = 0.0
    for _ in range(trials):
        B = dict(A)
        B["data"] = A["data"] * (1 + rng.choice([-1.0, 1.0], len(A["data"])) * 2.0 ** -52)
        r = O.las2("csr", B, dims, 0, seed=seed, legacy=False)
        if r["d"] == base["d"]:
            spread = max(spread, float(np.max(np.abs(r["s"] - base["s"]))))
    return spread


@pytest.mark.parametrize("case", sorted(CASES))
def test_lanczos_as_written_parity(case):
    """Discrete outputs and alpha/beta as for legacy; singular values within 1e-10,
    or within twice the spread the crate itself shows under one-ulp input changes."""
    A = CASES[case]()
    ref, err, got = run_pair("csr", A, 6, 4242, "lanczos")
    if err is not None:
        assert got["error"] is not None and type(got["error"]).__name__ == err.kind, (err, got["error"])
        return
    try:
        check_same(ref, got, check_vectors=False)
    except AssertionError:
        check_same(ref, got, s_tol=None, check_vectors=False)  # everything but sigma
        dev = float(np.max(np.abs(got["rec"].s - ref["s"])))
        spread = ulp_spread(A, 6, 4242)
        assert dev <= 2.0 * spread + 1e-10 * np.max(ref["s"]), (dev, spread)


@pytest.mark.parametrize("kind", ["csc", "coo", "masked"])
@pytest.mark.parametrize("algorithm", ["legacy", "lanczos"])
def test_formats(kind, algorithm):
    A = M.uniform(120, 70, 0.08, 12)
    if kind == "masked":
        mask = (np.random.default_rng(1).random(70) < 0.6).astype(np.uint8)
        ref = None
        try:
            ref = O.las2("masked", A, 5, 0, seed=99, legacy=(algorithm == "legacy"), mask=mask)
        except O.OracleError as e:
            err = e
        got = lanczos.las2_traced(upload("masked", A, mask), 5, 0, random_seed=99, algorithm=algorithm)
        if ref is None:
            assert type(got["error"]).__name__ == err.kind
            return
        check_same(ref, got, check_vectors=(algorithm == "legacy"))
        return
    ref, err, got = run_pair(kind, A, 5, 99, algorithm)
    if err is not None:
        assert type(got["error"]).__name__ == err.kind
        return
    check_same(ref, got, check_vectors=(algorithm == "legacy"))


def test_start_vector_bit_exact():
    for seed, hexes in FIX["start_vector"].items():
        got = lanczos.start_vector(int(seed), len(hexes))
        assert [struct.pack("<d", v).hex() for v in got] == hexes
    big = lanczos.start_vector(42, 100003)
    np.testing.assert_array_equal(big, O.start_vector(42, 100003))


def test_golden_legacy_doc_example():  # src/legacy.rs:172-283
    g = GOLD["squares_3x3_seed3141"]
    A = M.dense(g["dense"])
    r = legacy.svd_dim_seed(upload("csc", A), 0, 3141)
    assert r.d == 3
    np.testing.assert_allclose(r.s, g["s"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(r.ut, g["ut"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(r.vt, g["vt"], atol=1e-12, rtol=0)
    for k, v in g["diagnostics"].items():
        assert getattr(r.diagnostics, k) == v, k
    np.testing.assert_allclose(r.recompose(), g["dense"], atol=1e-12)


def test_golden_legacy_2x2_and_identity():  # src/legacy.rs:2182-2235
    g = GOLD["basic_2x2"]
    r = legacy.svd(upload("coo", M.dense([[4, 0], [3, -5]])))
    assert r.d == 2
    np.testing.assert_allclose(r.s, g["s"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(r.recompose(), [[4, 0], [3, -5]], atol=1e-12)
    r = legacy.svd(upload("csc", M.dense(np.eye(3))))
    assert r.d == 1 and abs(r.s[0] - 1.0) < 1e-12


def test_lanczos_as_written_small_fixture():
    for name, f in FIX["lanczos_as_written"].items():
        g = {"basic_2x2": [[4, 0], [3, -5]], "squares_3x3": [[1, 16, 49], [4, 25, 64], [9, 36, 81]]}[name]
        r = lanczos.svd_dim_seed(upload(f["format"], M.dense(g)), 0, f["seed"])
        assert r.d == f["d"] and r.diagnostics.lanczos_steps == f["lanczos_steps"]
        np.testing.assert_allclose(r.s, f["s"], rtol=1e-10)


def test_errors():
    with pytest.raises(Las2Error, match="insufficient dimensions"):
        lanczos.svd(upload("csr", M.dense([[1.0, 2.0, 3.0]])))
    Z = {"nrows": 6, "ncols": 5, "indptr": np.array([0, 1, 2, 2, 2, 2, 2]), "indices": np.array([0, 1]),
         "data": np.array([0.0, 0.0])}
    with pytest.raises(StartvError):
        lanczos.svd_dim_seed(upload("csr", Z), 3, 5)


@pytest.mark.slow
def test_poisson_5000x2000_legacy():
    f = FIX["poisson_5000x2000_seed42_dim10"]
    A = M.poisson_rows(5000, 2000, 20, 42)
    r = legacy.svd_dim_seed(upload("csr", A), 10, 42)
    assert r.d == f["legacy"]["d"]
    assert r.diagnostics.lanczos_steps == f["legacy"]["lanczos_steps"]
    assert r.diagnostics.ritz_values_stabilized == f["legacy"]["ritz_values_stabilized"]
    assert r.diagnostics.singular_values == f["legacy"]["singular_values"]
    np.testing.assert_allclose(r.s, f["legacy"]["s"], rtol=1e-10)


@pytest.mark.slow
def test_poisson_5000x2000_legacy_vectors_with_pieced_rotations():
    """192 steps give lanso's last imtqlb about 38,000 rotations: Z is built in
    five pieces of at most 8,192 while the host recurrence runs, after a first
    analysis pass on T of order 20 (Z reallocated as T grows).  u and vt
    against the oracle's sequential imtql2."""
    A = M.poisson_rows(5000, 2000, 20, 42)
    ref, err, got = run_pair("csr", A, 10, 42, "legacy")
    assert err is None
    assert ref["steps"] + 1 > 128  # js^2 / 2 well above one piece
    check_same(ref, got, s_tol=1e-11, vec_tol=1e-9)


@pytest.mark.slow
def test_poisson_5000x2000_lanczos_as_written_fails_like_the_crate():
    f = FIX["poisson_5000x2000_seed42_dim10"]["lanczos"]
    A = M.poisson_rows(5000, 2000, 20, 42)
    got = lanczos.las2_traced(upload("csr", A), 10, 0, random_seed=42, algorithm="lanczos")
    assert isinstance(got["error"], Imtql2Error)
    assert str(got["error"]).endswith(f["message"].split(": ", 1)[1])
    assert got["steps"] + 1 == f["lanczos_steps"]


@pytest.mark.parametrize("algorithm", ["lanczos", "legacy"])
def test_cluster_and_grid_lanczos_blocks_agree(algorithm, monkeypatch):
    """Small operators run the Lanczos blocks as one thread-block cluster (hardware
    barrier, partials in shared memory) of 16 or 8 blocks; larger ones as a
    cooperative grid.  Both
    follow the same steps: decisions equal, sigma within 1e-12."""
    A = M.poisson_rows(3000, 1200, 10, 21)
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("SVDB_LZ_CLUSTER", mode)
        out[mode] = lanczos.las2_traced(upload("csr", A), 8, 0, random_seed=5, algorithm=algorithm)
    g, c = out["0"], out["1"]
    assert c["lanczos_blocks"] in (8, 16)  # 16 where the device allows the non-portable cluster size
    # the as-written path may end in the crate's Imtql2Error: then both modes must
    assert type(g["error"]) is type(c["error"]), (g["error"], c["error"])
    assert g["steps"] == c["steps"] and g["purges"] == c["purges"]
    np.testing.assert_allclose(c["alf"], g["alf"], rtol=0, atol=1e-12 * np.abs(g["alf"]).max())
    np.testing.assert_allclose(c["bet"], g["bet"], rtol=0, atol=1e-12 * np.abs(g["bet"]).max())
    if g["error"] is None:
        assert g["rec"].d == c["rec"].d
        np.testing.assert_allclose(c["rec"].s, g["rec"].s, rtol=0, atol=1e-12 * g["rec"].s.max())

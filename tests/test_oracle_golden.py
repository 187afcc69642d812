"""The checker (oracle/) against the crate's own known answers and dense truth.

These pin the CPU restatement before it is trusted as the parity reference for
the GPU path.  No GPU needed.
"""
import json
import os
import struct

import numpy as np
import pytest

import matrices as M
import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.json")))
FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_fixtures.json")))


def test_chacha20_rfc8439_block():
    words = O.chacha_block(bytes(32), 0, 0, 20)
    assert words.astype("<u4").tobytes().hex() == GOLD["chacha20_rfc8439_a1_1"]["keystream_hex"]


def test_start_vector_matches_chacha12_stream():
    # value i uses keystream words (2i, 2i+1) of ChaCha12 keyed by the seed bytes
    seed, n = 3141, 21
    key = seed.to_bytes(4, "little") + bytes(28)
    words = np.concatenate([O.chacha_block(key, b, 0, 12) for b in range(3)])
    u = words[0::2].astype(np.uint64) | (words[1::2].astype(np.uint64) << np.uint64(32))
    expect = (2.0 * ((u >> np.uint64(12)).astype(np.float64)) - 2.0 ** 52) / 2.0 ** 52
    assert np.array_equal(O.start_vector(seed, n), expect[:n])


def test_start_vector_fixture():
    for seed, hexes in FIX["start_vector"].items():
        got = O.start_vector(int(seed), len(hexes))
        assert [struct.pack("<d", v).hex() for v in got] == hexes


def _las2_gold(case, legacy=True):
    g = GOLD[case]
    if "coo" in g:
        return O.las2("coo", g["coo"], 0, 0, seed=g.get("seed", 42), legacy=legacy)
    A = M.dense(g["dense"])
    if g["format"] == "csc":
        A = M.to_csc(A)
    return O.las2(g["format"], A, 0, 0, seed=g.get("seed", 42), legacy=legacy)


def test_legacy_basic_2x2():  # src/legacy.rs:2182-2213
    g = GOLD["basic_2x2"]
    r = _las2_gold("basic_2x2")
    assert r["d"] == g["d"]
    np.testing.assert_allclose(r["s"], g["s"], atol=g["tol"])
    rec = r["ut"].T @ np.diag(r["s"]) @ r["vt"]
    np.testing.assert_allclose(rec, [[4, 0], [3, -5]], atol=1e-12)


def test_legacy_identity_3x3():  # src/legacy.rs:2215-2235
    r = _las2_gold("identity_3x3")
    assert r["d"] == 1
    assert abs(r["s"][0] - 1.0) < 1e-12


def test_legacy_doc_example_seed_3141():  # src/legacy.rs:172-283
    g = GOLD["squares_3x3_seed3141"]
    r = _las2_gold("squares_3x3_seed3141")
    assert r["d"] == g["d"]
    np.testing.assert_allclose(r["s"], g["s"], atol=g["tol"], rtol=0)
    # the printed vectors, signs included: the signs follow from the start vector
    np.testing.assert_allclose(r["ut"], g["ut"], atol=g["tol"], rtol=0)
    np.testing.assert_allclose(r["vt"], g["vt"], atol=g["tol"], rtol=0)
    for k, v in g["diagnostics"].items():
        assert r["diagnostics"][k] == v, k


def test_legacy_coo_csc_csr_agree():  # src/legacy.rs:2158-2165
    g = GOLD["coo_csc_csr"]
    coo = {"nrows": 4, "ncols": 4, "row": g["row"], "col": g["col"], "data": g["data"]}
    csr = M.from_scipy(M.to_scipy({"nrows": 4, "ncols": 4, "indptr": [0, 0, 1, 2, 2], "indices": [0, 1],
                                   "data": [3.0, 4.0]}))
    res = [O.las2("coo", coo, 3, 0, seed=g["seed"], legacy=True), O.las2("csc", M.to_csc(csr), 3, 0,
                                                                        seed=g["seed"], legacy=True),
           O.las2("csr", csr, 3, 0, seed=g["seed"], legacy=True)]
    for r in res[1:]:
        assert r["d"] == res[0]["d"]
        np.testing.assert_array_equal(r["s"], res[0]["s"])
        np.testing.assert_array_equal(r["vt"], res[0]["vt"])


def test_masked_3x5_maps_and_nnz():  # src/lanczos/masked.rs:885-907
    g = GOLD["masked_3x5"]
    A = M.from_scipy(M.to_scipy(M.dense(np.zeros((3, 5)))))
    import scipy.sparse as sp
    A = M.from_scipy(sp.csr_matrix((g["data"], (g["row"], g["col"])), shape=(3, 5)))
    mask = np.zeros(5, np.uint8)
    mask[g["columns"]] = 1
    m2o, o2m, mnnz = O.masked_maps(A, mask)
    assert list(m2o) == g["columns"]
    assert list(o2m) == [0, -1, 1, -1, 2]
    assert mnnz == g["masked_nnz"]


@pytest.mark.parametrize("legacy", [True, False])
def test_masked_equals_physical_subset(legacy):  # src/lanczos/masked.rs:914-1000
    rng = np.random.default_rng(42)
    import scipy.sparse as sp
    r = rng.integers(0, 14, 40)
    c = rng.integers(0, 10, 40)
    v = rng.uniform(0.1, 10.0, 40)
    full = sp.csr_matrix((v, (r, c)), shape=(14, 10))
    full.sum_duplicates()
    A = M.from_scipy(full)
    cols = [1, 3, 5, 7]
    mask = np.zeros(10, np.uint8)
    mask[cols] = 1
    phys = M.from_scipy(full[:, cols])
    rm = O.las2("masked", A, 0, 0, seed=7, legacy=legacy, mask=mask)
    rp = O.las2("csr", phys, 0, 0, seed=7, legacy=legacy)
    assert rm["d"] == rp["d"]
    np.testing.assert_allclose(np.sort(rm["s"]), np.sort(rp["s"]), atol=1e-10, rtol=0)
    assert rm["masked_would_panic"]  # the crate's small-matrix delegate asserts here (masked.rs:133-143)


@pytest.mark.parametrize("shape,density,seed", [((60, 30), 0.3, 1), ((200, 120), 0.05, 2), ((50, 130), 0.2, 3)])
def test_legacy_matches_dense_svd(shape, density, seed):
    A = M.uniform(shape[0], shape[1], density, seed)
    r = O.las2("csr", A, 8, 0, seed=1234, legacy=True)
    truth = np.linalg.svd(M.to_scipy(A).toarray(), compute_uv=False)
    assert r["d"] >= 1
    np.testing.assert_allclose(r["s"], truth[: r["d"]], rtol=1e-10)
    # singular vectors: |u_i . u_true_i| = 1
    U, S, Vt = np.linalg.svd(M.to_scipy(A).toarray())
    for i in range(r["d"]):
        assert abs(abs(r["vt"][i] @ Vt[i]) - 1) < 1e-8


def test_lanczos_as_written_fixture():
    for name, f in FIX["lanczos_as_written"].items():
        g = {"basic_2x2": [[4, 0], [3, -5]], "squares_3x3": [[1, 16, 49], [4, 25, 64], [9, 36, 81]]}[name]
        A = M.dense(g)
        if f["format"] == "csc":
            A = M.to_csc(A)
        r = O.las2(f["format"], A, 0, 0, seed=f["seed"], legacy=False)
        assert r["d"] == f["d"] and r["diagnostics"]["lanczos_steps"] == f["lanczos_steps"]
        np.testing.assert_array_equal(r["s"], f["s"])


def test_lanczos_as_written_pythag_and_imtqlb():
    # svd_pythag as written (mod.rs:361-380) overestimates hypot for comparable arguments
    assert abs(O.pythag(3.0, 4.0, legacy=True) - 5.0) < 1e-15
    assert O.pythag(3.0, 4.0, legacy=False) > 5.0 + 1e-3
    assert abs(O.pythag(1e-9, 1.0, legacy=False) - np.hypot(1e-9, 1.0)) < 1e-15
    # legacy imtqlb returns the eigenvalues of T; the as-written one does not
    rng = np.random.default_rng(5)
    d, e = rng.standard_normal(12), rng.standard_normal(12)
    T = np.diag(d) + np.diag(e[1:], 1) + np.diag(e[1:], -1)
    vals, _ = O.imtqlb(d, e, legacy=True)
    np.testing.assert_allclose(np.sort(vals), np.linalg.eigvalsh(T), atol=1e-12)


def test_randomized_checker_recovers_spectrum():
    A = M.lowrank_plus_noise(300, 80, 10, 1e-3, 11)
    om = M.omega(80, 15, 3)
    r = O.randomized(A, 10, 5, 3, "QR", omega=om)
    truth = np.linalg.svd(M.to_scipy(A).toarray(), compute_uv=False)[:10]
    np.testing.assert_allclose(r["s"], truth, rtol=1e-8)
    assert r["u"].shape == (300, 10) and r["vt"].shape == (10, 80)


def test_randomized_checker_power_iterations_and_d3():
    # flat (noise-like) spectrum: power iterations help (randomized/mod.rs:693-777), and the
    # masked A^T Y indexing of masked.rs:388-393 cancels most of that gain
    A = M.uniform(400, 120, 0.1, 9)
    om = M.omega(120, 15, 3)
    truth = np.linalg.svd(M.to_scipy(A).toarray(), compute_uv=False)[:10]
    err = lambda r: np.max(np.abs(r["s"] - truth) / truth)  # noqa: E731
    e0 = err(O.randomized(A, 10, 5, 0, "QR", omega=om))
    e3 = err(O.randomized(A, 10, 5, 3, "QR", omega=om))
    e3_d3 = err(O.randomized(A, 10, 5, 3, "QR", omega=om, compat_d3=True))
    assert e3 < 0.9 * e0
    assert e3_d3 > 2 * e3


@pytest.mark.parametrize("masked", [False, True])
def test_randomized_checker_mean_center_is_the_centred_svd(masked):
    # mean_center (randomized/mod.rs:46-53, column means masked.rs:240-263): with a
    # sketch as wide as the matrix the result is the exact SVD of A - 1 mu^T
    A = M.uniform(120, 40, 0.3, 17, low=0.5, high=3.0)
    mask = (np.arange(40) % 4 != 1).astype(np.uint8) if masked else None
    Ad = M.to_scipy(A).toarray()
    if masked:
        Ad = Ad[:, mask.astype(bool)]
    nc = Ad.shape[1]
    U, s, Vt = np.linalg.svd(Ad - Ad.mean(0), full_matrices=False)
    r = O.randomized(A, 8, nc - 8, 1, "QR", omega=M.omega(nc, nc, 4), mask=mask, mean_center=True)
    np.testing.assert_allclose(r["s"], s[:8], rtol=1e-12)
    np.testing.assert_allclose(np.abs(np.sum(r["u"] * U[:, :8], 0)), 1.0, atol=1e-12)
    # uncentred, the column means dominate the leading singular value
    r0 = O.randomized(A, 8, nc - 8, 1, "QR", omega=M.omega(nc, nc, 4), mask=mask)
    assert r0["s"][0] > 2 * r["s"][0]


def test_f32_checker_is_the_crate_at_t_f32():
    # the same restatement built with T = f32 (impl SvdFloat for f32, src/utils.rs:87-99):
    # start vector = the f64 draws rounded to f32 (mod.rs:604-606), kappa clamped to f32 eps34
    sv = O.start_vector(11, 1000, scalar="f32")
    np.testing.assert_array_equal(sv, O.start_vector(11, 1000).astype(np.float32).astype(np.float64))
    U, _ = np.linalg.qr(np.random.default_rng(1).standard_normal((120, 6)))
    V, _ = np.linalg.qr(np.random.default_rng(2).standard_normal((80, 6)))
    D = ((U * np.geomspace(100, 1, 6)) @ V.T).astype(np.float32)
    A = M.dense(D)
    r = O.las2("csr", A, 3, 0, seed=3, scalar="f32")
    assert r["diagnostics"]["kappa"] == float(np.float32(np.finfo(np.float32).eps) ** np.float32(0.75))
    assert r["d"] == 3
    # randomized at T = f32 against the dense spectrum
    truth = np.linalg.svd(D.astype(np.float64), compute_uv=False)
    om = M.omega(80, 12, 3)
    rr = O.randomized(A, 6, 6, 1, "QR", omega=om, scalar="f32")
    np.testing.assert_allclose(rr["s"], truth[:6], rtol=2e-6)
    with pytest.raises(ValueError):
        O.las2("csr", A, 3, 0, legacy=True, scalar="f32")


def test_poisson_workload_fixture_shape():
    f = FIX["poisson_5000x2000_seed42_dim10"]
    A = M.poisson_rows(5000, 2000, 20, 42)
    assert len(A["data"]) == f["nnz"]
    assert f["sparsity"] > 0.99  # takes the >0.99 branch (adaptive eps 100 eps, 300 QL iterations)
    assert f["lanczos"]["error"] == "Imtql2Error"

"""Dense exact tier on the GPU against the numpy oracle: GrmBuilder::compute
(libCosmicCore/src/grm_builder.cpp:140-394), EigenVce::prepare / runNullModel
(libCosmicCore/src/eigen_vce.cpp:19-153, vce.cpp:3073-3175) and LmmEngine::scan's exact branch
(src/lmm_engine.cpp:1363-1474).

Tolerances: G 1e-12 relative to its largest entry, the valid-SNP count and the float-rounded
2pq sum exact; eigenvalues 1e-10 of the largest; Uty^2 summed over each eigenvalue (the basis
of a repeated eigenvalue is arbitrary) 1e-8; variance components 1e-6 relative, SEs and the
REML log-likelihood 1e-6; the scan's BETA/SE 1e-8 relative (FP64) / 1e-5 (mixed), -log10 P
1e-6 / 1e-3 absolute, FREQ and the tested set exact."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


@pytest.fixture(scope="module")
def data():
    d = synth.cohort(420, 2600, 19, missing=0.03, n_causal=30, h2=0.5)
    bed = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    return d, bed, g


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("algorithm", [1, 0, 2, 4, 5])
def test_grm_matches_oracle(data, algorithm):
    d, bed, g = data
    variants = None if algorithm != 2 else np.arange(100, 2600, 3, dtype=np.int32)
    G_o, nv_o, s_o = oracle.grm_dense(bed, algorithm=algorithm, variants=variants)
    b = cs.GrmBuilder(algorithm=algorithm).compute(g, variants)
    assert b.getTotalSnps() == nv_o
    assert b.getSum2pq() == s_o
    G = b.getGrm()
    assert rel(G, G_o) < 1e-12
    assert np.array_equal(G, G.T)
    keep = np.arange(3, d["n"], 2, dtype=np.int32)
    assert np.array_equal(b.getGrm(keep), G[np.ix_(keep, keep)])
    b.close()


def grouped(D, v, tol=1e-9):
    """Sums of v^2 over groups of equal eigenvalues (the invariant part of U^T y)."""
    out, i = [], 0
    while i < len(D):
        j = i + 1
        while j < len(D) and abs(D[j] - D[i]) <= tol * max(1.0, abs(D[i])):
            j += 1
        out.append((v[i:j] ** 2).sum())
        i = j
    return np.array(out)


@pytest.mark.parametrize("projection", [True, False])
def test_eigen_vce_matches_oracle(data, projection):
    d, bed, g = data
    n = d["n"]
    keep = np.sort(np.random.default_rng(4).choice(n, 380, replace=False)).astype(np.int32)
    y = d["y"][keep]
    X = d["X"][keep].astype(np.float32).astype(np.float64)
    G_o, _, _ = oracle.grm_dense(bed)
    Gk = G_o[np.ix_(keep, keep)]
    D_o, W_o, Uty_o, UtX_o = oracle.eigen_vce_prepare(Gk, y, X, projection)
    b = cs.GrmBuilder().compute(g)
    v = cs.EigenVce(projection).prepare(y, X, b, keep)
    D = v.getEigenvalues()
    assert v.n_eig == len(D_o) and v.p == UtX_o.shape[1]
    assert np.abs(D - D_o).max() < 1e-10 * D_o.max()
    Uty = v.getUty()
    assert rel(grouped(D_o, Uty), grouped(D_o, Uty_o)) < 1e-8
    W = v.getProjectedW()
    # same projected operator: W diag(D) W^T
    assert rel(W @ (D[:, None] * W.T), W_o @ (D_o[:, None] * W_o.T)) < 1e-9
    if projection:
        assert np.abs(W.T @ X).max() < 1e-10  # W spans the complement of X
    r = v.runNullModel()
    o = oracle.solve_diagonal(D_o, Uty_o, UtX_o)
    for key in ("sigma2_g", "sigma2_e", "delta"):
        assert abs(r[key] - o[key]) <= 1e-6 * abs(o[key]), key
    diag = oracle.reml_diagnostics(D_o, Uty_o, UtX_o, r["sigma2_g"], r["sigma2_e"])
    for key in ("sigma2_g_se", "sigma2_e_se", "log_likelihood"):
        assert abs(r[key] - diag[key]) <= 1e-6 * abs(diag[key]), key
    assert r["max_score"] < 1e-2 and r["converged"] == 1
    v.close()
    b.close()


@pytest.mark.parametrize("precision,tol_b,tol_p", [("fp64", 1e-8, 1e-6), ("mixed", 1e-5, 1e-3)])
@pytest.mark.parametrize("projection,residuals", [(True, False), (False, False), (False, True)])
def test_exact_scan_matches_oracle(data, precision, tol_b, tol_p, projection, residuals):
    d, bed, g = data
    n = d["n"]
    keep = np.arange(n, dtype=np.int32) if projection else \
        np.sort(np.random.default_rng(6).choice(n, 400, replace=False)).astype(np.int32)
    y = d["y"][keep]
    X = d["X"][keep].astype(np.float32).astype(np.float64)
    b = cs.GrmBuilder().compute(g)
    v = cs.EigenVce(projection).prepare(y, X, b, keep)
    v.runNullModel()
    eng = cs.LmmEngine()
    eng.prepareFromVce(v, use_residuals=residuals)
    out = eng.scan(g, keep, precision=precision)
    D, W, Uty, UtX = v.getEigenvalues(), v.getProjectedW(), v.getUty(), v.getUtX()
    exp = oracle.scan_exact(bed, keep, W, D, Uty, UtX, v.getSigma2g(), v.getSigma2e(),
                            use_residuals=residuals)
    t = exp["tested"]
    assert np.array_equal(out["tested"], t) and t.sum() > 0.9 * d["m"]
    assert np.array_equal(out["freq"][t], exp["freq"][t])
    assert rel(out["beta"][t], exp["beta"][t]) < tol_b
    assert rel(out["se"][t], exp["se"][t]) < tol_b
    assert np.abs(out["log10p"][t] - exp["log10p"][t]).max() < tol_p
    # a window gives the same rows
    w = eng.scan_window(g, keep, 700, 1900, precision=precision)
    assert np.array_equal(w["tested"], out["tested"][700:1900])
    tw = w["tested"]
    assert rel(w["beta"][tw], out["beta"][700:1900][tw]) < 1e-12
    eng.close()
    v.close()
    b.close()


def test_exact_scan_reference_basis(data):
    """The scan from the oracle's own basis (a caller's GRM through from_matrix): the
    statistics do not depend on which eigenvector basis of a repeated eigenvalue is used."""
    d, bed, g = data
    n = d["n"]
    keep = np.arange(n, dtype=np.int32)
    y, X = d["y"], d["X"].astype(np.float32).astype(np.float64)
    G_o, _, _ = oracle.grm_dense(bed)
    b = cs.GrmBuilder.from_matrix(G_o)
    assert b.getNumSamples() == n and b.getTotalSnps() == 0
    v = cs.EigenVce().prepare(y, X, b)
    r = v.runNullModel()
    D_o, W_o, Uty_o, UtX_o = oracle.eigen_vce_prepare(G_o, y, X)
    o = oracle.solve_diagonal(D_o, Uty_o, UtX_o)
    assert abs(r["sigma2_g"] - o["sigma2_g"]) <= 1e-6 * o["sigma2_g"]
    eng = cs.LmmEngine()
    eng.prepareFromVce(v)
    out = eng.scan(g, keep, precision="fp64")
    exp = oracle.scan_exact(bed, keep, W_o, D_o, Uty_o, UtX_o, o["sigma2_g"], o["sigma2_e"])
    t = exp["tested"]
    assert np.array_equal(out["tested"], t)
    assert np.abs(out["log10p"][t] - exp["log10p"][t]).max() < 1e-5


def test_dense_errors(data):
    d, bed, g = data
    with pytest.raises(cs.CosmicError):
        cs.GrmBuilder(algorithm=7).compute(g)
    with pytest.raises(cs.CosmicError):
        cs.GrmBuilder().compute(g, np.array([5, 3], dtype=np.int32))  # not increasing
    b = cs.GrmBuilder().compute(g)
    X = np.ones((d["n"], 2))  # two identical columns: rank deficient
    with pytest.raises(cs.CosmicError, match="rank deficient"):
        cs.EigenVce().prepare(d["y"], X, b)
    v = cs.EigenVce().prepare(d["y"], X[:, :1], b)
    eng = cs.LmmEngine()
    with pytest.raises(cs.CosmicError, match="null model has not been run"):
        eng.prepareFromVce(v)


@pytest.mark.parametrize("algorithm", [1, 0])
def test_grm_loco_matches_oracle(data, algorithm):
    d, bed, g = data
    G, nv, s2 = oracle.grm_dense(bed, algorithm=algorithm)
    chr_snps = np.arange(1500, 2600, dtype=np.int32)
    raw, nc, sc = oracle.grm_dense(bed, algorithm=algorithm, variants=chr_snps, raw=True)
    exp = oracle.grm_loco(G, nv, s2, raw, nc, sc, algorithm)
    glob = cs.GrmBuilder(algorithm=algorithm).compute(g)
    ch = cs.GrmBuilder(algorithm=algorithm).compute(g, chr_snps)
    assert ch.getTotalSnps() == nc
    loco = cs.GrmBuilder.loco(glob, ch)
    assert loco.getTotalSnps() == nv - nc
    assert rel(loco.getGrm(), exp) < 1e-12


def test_exact_route_from_files(tmp_path, data):
    """`gwas --model lmm` (dense route) end to end from files with LOCO over two chromosomes:
    per chromosome the LOCO GRM, its Brent null model and the exact scan of its SNPs, against
    the oracle's dense restatement."""
    d, bed, g = data
    n, m = d["n"], d["m"]
    prefix = str(tmp_path / "c")
    open(prefix + ".bed", "wb").write(d["bed"].tobytes())
    chrom = np.array(["1"] * 1400 + ["2"] * (m - 1400))
    with open(prefix + ".bim", "w") as f:
        for j in range(m):
            f.write(f"{chrom[j]}\trs{j}\t0\t{100 + j}\tA\tG\n")
    with open(prefix + ".fam", "w") as f:
        for i in range(n):
            f.write(f"F{i} I{i} 0 0 1 {float(d['y'][i])!r}\n")
    with open(str(tmp_path / "q.txt"), "w") as f:
        for i in range(n):
            f.write(f"F{i} I{i} {'-9' if i % 50 == 7 else round(float(d['X'][i, 1]), 4)}\n")
    out = str(tmp_path / "res")
    res, diags, inputs = cs.run_gwas_lmm(prefix, out, qcovar=str(tmp_path / "q.txt"),
                                         precision="fp64", exact=True)
    keep, y, X = inputs["keep"], inputs["y"], inputs["X"]
    assert len(keep) == n - len([i for i in range(n) if i % 50 == 7])
    G, nv, s2 = oracle.grm_dense(bed)
    for c, lo, hi in (("1", 0, 1400), ("2", 1400, m)):
        raw, nc, sc = oracle.grm_dense(bed, variants=np.arange(lo, hi), raw=True)
        Gl = oracle.grm_loco(G, nv, s2, raw, nc, sc)
        D, W, Uty, UtX = oracle.eigen_vce_prepare(Gl[np.ix_(keep, keep)], y, X)
        o = oracle.solve_diagonal(D, Uty, UtX)
        assert abs(diags[c]["sigma2_g"] - o["sigma2_g"]) <= 1e-6 * o["sigma2_g"]
        sub = oracle.Bed(bed.rows[lo:hi], n)
        e = oracle.scan_exact(sub, keep, W, D, Uty, UtX, o["sigma2_g"], o["sigma2_e"])
        t = e["tested"]
        assert np.array_equal(res["tested"][lo:hi], t)
        assert np.abs(res["log10p"][lo:hi][t] - e["log10p"][t]).max() < 1e-5
    meta = open(out + ".scan.meta.txt").read()
    assert "matrix_approximation\tfull_eigen" in meta and "RANK_SELECTION\tFULL" in meta
    assert "LOCO\ttrue" in meta
    import os
    assert not os.path.exists(out + ".low_rank.meta.tsv")
    lines = open(out + ".assoc.txt").read().splitlines()
    assert len(lines) == 1 + int(res["tested"].sum())

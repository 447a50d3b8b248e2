"""Multi-right-hand-side PCG and the matrix-free AI-REML (STCG_VCE) on the GPU against the
CPU oracle.

The oracle restates libCosmicCore/src/matrix_free_pcg.h and stcg_vce.cpp one vector at a
time; the GPU solves every right-hand side of a covariance matrix as one block.  Both draw
the same trace probes (one mt19937_64 stream through uniform_int_distribution<int>(0, 1))
and the same SLQ probes, so the FP64 runs agree to CG tolerance: variance components and
the log-likelihood within 1e-7 relative, beta and BLUPs within 1e-6.  The mixed-precision
kinship applies keep the variance components within 1e-5 relative of the FP64 run.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def single():
    d = synth.cohort(400, 1500, 21, missing=0.02, n_causal=40, h2=0.5)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.createKinshipOperator(g, None, None)
    return d, ref, g, op


@pytest.fixture(scope="module")
def records():
    d = synth.repeatability_cohort(250, 1200, 33, max_records=3)
    ref = oracle.Bed(d["bed"][3:].reshape(d["m"], -1), d["n"])
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.createKinshipOperator(g, None, None)
    return d, ref, g, op


def test_pcg_block_matches_single_vector_oracle(single):
    d, ref, g, op = single
    n = d["n"]
    rng = np.random.default_rng(3)
    B = np.asfortranarray(rng.standard_normal((n, 7)))
    B[:, 3] = 0.0  # solved by x = 0 before any iteration
    sg2, se2 = 0.6, 0.4
    pcg = cs.MatrixFreePCG(op, sg2, se2)
    X = pcg.solve(B, tol=1e-10, max_iter=500)
    for c in range(B.shape[1]):
        xo, it = ref.pcg_solve(B[:, c], sg2, se2, 1e-10, 500)
        if c == 3:
            assert pcg.iterations[c] == 0 and np.all(X[:, c] == 0.0)
            continue
        assert abs(int(pcg.iterations[c]) - it) <= 1
        assert rel(X[:, c], xo) < 1e-9
    # the solution solves the system
    KX = op.apply(X)
    assert rel(sg2 * KX + se2 * X, B) < 1e-9


def test_pcg_relative_stopping_and_max_iter(single):
    d, ref, g, op = single
    b = np.random.default_rng(4).standard_normal(d["n"])
    pcg = cs.MatrixFreePCG(op, 0.5, 0.5)
    x = pcg.solve(b, tol=1e-6, max_iter=500, relative=True)
    r = b - (0.5 * op.apply(x) + 0.5 * x)
    assert np.linalg.norm(r) < 1e-6 * np.linalg.norm(b) * 1.01
    x2 = pcg.solve(b, tol=1e-30, max_iter=3)
    assert pcg.iterations[0] == 3


@pytest.mark.parametrize("slq", [0, 4])
def test_stcg_single_record_matches_oracle(single, slq):
    d, ref, g, op = single
    kw = dict(max_iter=6, mc_samples=6, slq_probes=slq, slq_steps=6)
    ro, beta_o, a_o, pe_o = oracle.stcg_vce(ref, d["y"], d["X"], **kw)
    vce = cs.StcgVce()
    r = vce.solve(op, d["y"], d["X"], kinship_divisor=d["m"], **kw)
    assert r["iterations"] == ro["iterations"]
    assert abs(r["sigma2_g"] - ro["sigma2_g"]) <= 1e-7 * ro["sigma2_g"]
    assert abs(r["sigma2_e"] - ro["sigma2_e"]) <= 1e-7 * ro["sigma2_e"]
    assert r["sigma2_pe"] == 0.0
    if slq:
        assert abs(r["logl"] - ro["logl"]) <= 1e-7 * abs(ro["logl"])
    else:
        assert np.isnan(r["logl"])
    beta, a, pe = vce.solution()
    assert rel(beta, beta_o) < 1e-6
    assert rel(a, a_o) < 1e-6
    assert np.all(pe == 0.0)
    h = vce.history()
    assert h.shape == (r["iterations"], 5)
    assert list(h[:4, 4]) == [0, 0, 0, 0] and np.all(h[4:, 4] == 1)


def test_stcg_repeatability_records_match_oracle(records):
    d, ref, g, op = records
    kw = dict(max_iter=6, mc_samples=6, slq_probes=3, slq_steps=5)
    ro, beta_o, a_o, pe_o = oracle.stcg_vce(ref, d["y"], d["X"], rec_to_row=d["rec_to_row"],
                                            with_pe=True, **kw)
    vce = cs.StcgVce()
    r = vce.solve(op, d["y"], d["X"], rec_to_row=d["rec_to_row"], with_pe=True,
                  kinship_divisor=d["m"], **kw)
    for key in ("sigma2_g", "sigma2_pe", "sigma2_e"):
        assert abs(r[key] - ro[key]) <= 1e-7 * ro[key], key
    assert abs(r["logl"] - ro["logl"]) <= 1e-7 * abs(ro["logl"])
    beta, a, pe = vce.solution()
    assert rel(beta, beta_o) < 1e-6
    assert rel(a, a_o) < 1e-6
    assert rel(pe, pe_o) < 1e-6


def test_stcg_mixed_precision_within_tolerance(single):
    d, ref, g, op = single
    kw = dict(max_iter=8, mc_samples=8, slq_probes=0)
    r64 = cs.StcgVce().solve(op, d["y"], d["X"], kinship_divisor=d["m"], **kw)
    rmx = cs.StcgVce().solve(op, d["y"], d["X"], kinship_divisor=d["m"], precision="mixed", **kw)
    for key in ("sigma2_g", "sigma2_e"):
        assert abs(rmx[key] - r64[key]) <= 1e-5 * r64[key], (key, rmx[key], r64[key])


def test_stcg_rejects_bad_input(single):
    d, ref, g, op = single
    vce = cs.StcgVce()
    with pytest.raises(cs.InvalidArgument):
        vce.solve(op, d["y"][:-1], d["X"][:-1])  # records != rows without a record map
    with pytest.raises(cs.InvalidArgument):
        vce.solve(op, d["y"], d["X"], rec_to_row=np.full(d["n"], d["n"], np.int32))
    with pytest.raises(cs.InvalidArgument):
        vce.solution()


@pytest.fixture(scope="module")
def structured():
    d = synth.cohort(700, 2500, 27, n_pops=2, fst=0.05, missing=0.02, n_causal=40, h2=0.5)
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.createKinshipOperator(g, None, None)
    return d, g, op


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stcg_deflation_preconditioner(structured, precision):
    """The low-rank deflation preconditioner (precond_rank > 0) solves the same CG systems as
    the reference's scalar one to the same tolerance, so the variance components agree to CG
    accuracy, in fewer CG iterations (15-20 % fewer here: CG already absorbs the few large
    eigenvalues population structure gives K in a handful of iterations; deflating the top 32
    also narrows the bulk)."""
    d, g, op = structured
    kw = dict(max_iter=6, mc_samples=8, slq_probes=0, precision=precision)
    r0 = cs.StcgVce().solve(op, d["y"], d["X"], kinship_divisor=d["m"], **kw)
    r1 = cs.StcgVce().solve(op, d["y"], d["X"], kinship_divisor=d["m"], precond_rank=32, **kw)
    for key in ("sigma2_g", "sigma2_e"):
        assert abs(r1[key] - r0[key]) <= 1e-7 * r0[key], (key, r1[key], r0[key])
    assert r1["pcg_iterations"] < 0.92 * r0["pcg_iterations"], (r1["pcg_iterations"],
                                                                r0["pcg_iterations"])

"""The association path end to end from files, as `cosmicscanner gwas --model lmm --fastlmm
--fastlmm-matrix-free` runs it: .bed/.bim/.fam, a phenotype file with missing values, a
quantitative and a categorical covariate file, the keep list of complete samples
(src/models/univariate_model.cpp:389-426), leave-one-chromosome-out over the .bim's two
chromosomes (src/gwas_scanner.cpp:299-314, 464-472) and OUT.assoc.txt
(src/gwas_output.cpp:123-183).  Compared with the oracle's low-rank null model and scan on
the same analysed samples; tolerances as the single-null path (mixed form)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

cs = pytest.importorskip("cosmicscanner_b200")
synth = pytest.importorskip("cosmicscanner_b200.synth")


def test_gwas_lmm_from_files(tmp_path):
    n, m = 640, 2000
    d = synth.cohort(n, m, 31, missing=0.02, n_causal=40, h2=0.5)
    prefix = str(tmp_path / "cohort")
    open(prefix + ".bed", "wb").write(d["bed"].tobytes())
    chrom = np.array(["1"] * 1100 + ["2"] * 900)
    with open(prefix + ".bim", "w") as f:
        for j in range(m):
            f.write(f"{chrom[j]}\trs{j}\t0\t{1000 + 10 * j}\tA\tG\n")
    with open(prefix + ".fam", "w") as f:
        for i in range(n):
            f.write(f"FAM{i} IND{i} 0 0 1 -9\n")
    rng = np.random.default_rng(3)
    y = d["y"]
    drop_y = set(rng.choice(n, 12, replace=False).tolist())
    drop_q = set(rng.choice(n, 5, replace=False).tolist())
    age = np.round(rng.normal(50, 10, n), 3)
    site = rng.choice(["north", "east", "west"], n)
    with open(str(tmp_path / "y.txt"), "w") as f:
        f.write("FID IID trait\n")
        for i in range(n):
            v = ("-9" if i % 2 else "NA") if i in drop_y else repr(float(y[i]))
            f.write(f"FAM{i} IND{i} {v}\n")
    with open(str(tmp_path / "q.txt"), "w") as f:
        for i in range(n):
            f.write(f"FAM{i} IND{i} {'-9' if i in drop_q else age[i]}\n")
    with open(str(tmp_path / "c.txt"), "w") as f:
        for i in range(n):
            f.write(f"FAM{i} IND{i} {site[i]}\n")
    out = str(tmp_path / "res")
    res, diags, inputs = cs.run_gwas_lmm(prefix, out, pheno=str(tmp_path / "y.txt"),
                                         qcovar=str(tmp_path / "q.txt"),
                                         covar=str(tmp_path / "c.txt"), rank=30,
                                         precision="mixed")
    keep = np.array([i for i in range(n) if i not in drop_y and i not in drop_q], dtype=np.int32)
    assert np.array_equal(inputs["keep"], keep)
    X = np.column_stack([np.ones(len(keep)), age[keep].astype(np.float32),
                         (site[keep] == "north"), (site[keep] == "west")]).astype(np.float64)
    # east is the reference level; the covariate file's decimals are read as float (direct
    # decimal -> float rounding may differ in the last bit from float64 -> float32)
    assert np.array_equal(inputs["X"][:, [0, 2, 3]], X[:, [0, 2, 3]])
    assert np.allclose(inputs["X"][:, 1], X[:, 1], rtol=1e-6, atol=0)
    X = inputs["X"]
    assert np.array_equal(inputs["y"], y[keep])
    assert list(diags) == ["1", "2"]
    rows = d["bed"][3:].reshape(m, -1)
    ref = oracle.Bed(rows, n)
    variants = cs.grm_variant_selection(cs.Genotypes.from_bed_bytes(d["bed"], n, m).stats(), 0.01)
    for c in ["1", "2"]:
        loco = variants[chrom[variants] != c]
        U, lam, r = ref.lowrank_prepare(y[keep], X, 30, keep=keep, variants=loco, n_threads=8)
        assert abs(diags[c]["sigma2_g"] - r.sigma2_g) <= 1e-5 * r.sigma2_g
        assert abs(diags[c]["sigma2_e"] - r.sigma2_e) <= 1e-5 * r.sigma2_e
        idx = np.flatnonzero(chrom == c)
        sub = oracle.Bed(rows[idx[0]:idx[-1] + 1], n)
        o = sub.scan_lowrank(keep, U, lam, r.residual_eigenvalue, r.sigma2_g, r.sigma2_e,
                             y[keep], X)
        t = res["tested"][idx]
        assert np.array_equal(t, o["tested"])
        assert np.array_equal(res["freq"][idx][t], o["freq"][t])
        assert np.abs(res["log10p"][idx][t] - o["log10p"][t]).max() < 1e-3
        assert np.abs(res["beta"][idx][t] - o["beta"][t]).max() <= 1e-5 * np.abs(o["beta"][t]).max()
    # the result file: the reference's header, one row per tested SNP, N = kept samples
    lines = open(out + ".assoc.txt").read().splitlines()
    assert lines[0].split("\t")[:7] == ["CHR", "SNP", "BP", "A1", "A2", "FREQ", "N"]
    body = [l.split("\t") for l in lines[1:]]
    assert len(body) == int(res["tested"].sum())
    assert all(r[6] == str(len(keep)) for r in body)
    first = int(np.flatnonzero(res["tested"])[0])
    assert body[0][1] == f"rs{first}" and body[0][0] == chrom[first]
    # run metadata: one low-rank row per LOCO null model
    meta = [l.split("\t") for l in open(out + ".low_rank.meta.tsv").read().splitlines()]
    assert [r[0] for r in meta[1:]] == ["1", "2"]
    assert all(r[12] == str(len(keep)) and r[-1] == "none" for r in meta[1:])
    assert [r[3] for r in meta[1:]] == [str(diags[c]["effective_rank"]) for c in ["1", "2"]]
    meta_txt = open(out + ".scan.meta.txt").read().splitlines()
    assert "requested_rank\t30" in meta_txt
    assert meta_txt[-7:-4] == ["MODEL\tadditive", f"N\t{len(keep)}",
                               "N_SEMANTICS\tanalysis_samples_after_phenotype_and_covariate_"
                               "filtering;per-SNP_missing_genotypes_mean-imputed"]
    assert meta_txt[-3] == "LOCO\ttrue"
    # canonical sumstats: one block per chromosome, BETA at 10 significant digits
    ss = open(out + ".cosmic.sumstats").read().splitlines()
    assert ss[0] == "# CosmicScanner Summary Statistics v1.0" and ss[2] == "# Model: LMM"
    rows = [l.split("\t") for l in ss[5:]]
    assert len(rows) == int(res["tested"].sum())
    tj = np.flatnonzero(res["tested"])
    assert [r[1] for r in rows] == [f"rs{j}" for j in tj]
    assert all(r[5] == "%.10g" % res["beta"][j] for r, j in zip(rows[:50], tj[:50]))
    # the same run with --out-gz --out-ssf: gzip members of the same text, SSF rows
    import gzip
    out2 = str(tmp_path / "res_gz")
    res2, _, _ = cs.run_gwas_lmm(prefix, out2, pheno=str(tmp_path / "y.txt"),
                                 qcovar=str(tmp_path / "q.txt"), covar=str(tmp_path / "c.txt"),
                                 rank=30, precision="mixed", out_gz=True, out_ssf=True,
                                 created=ss[1][len("# Created: "):])
    assert np.array_equal(res2["tested"], res["tested"])
    ss2 = gzip.decompress(open(out2 + ".cosmic.sumstats", "rb").read()).decode().splitlines()
    assert ss2[:5] == ss[:5]
    rows2 = [l.split("\t") for l in ss2[5:]]
    assert [r[1] for r in rows2] == [r[1] for r in rows]
    assert all(r[5] == "%.10g" % res2["beta"][j] for r, j in zip(rows2[:50], tj[:50]))
    ssf = gzip.decompress(open(out2 + ".assoc.txt", "rb").read()).decode().splitlines()
    assert ssf[0].startswith("chromosome\tbase_pair_location") and len(ssf) == len(lines)
    assert ssf[1].split("\t")[-1] == body[0][1]


def test_low_rank_fallback_labels():
    """The fall-back decision of src/gwas_scanner.cpp:347-383: with --fastlmm-no-fallback the
    sketch that misses the trace threshold is kept ("none"); without it the run falls back to
    the fixed-rank MatrixFreeVce sketch ("trace_threshold"), which at the same requested rank
    and seed gives the same null and scan; an error above --lmm-low-rank-error-tol falls back
    with "error_tolerance"."""
    n, m = 500, 1500
    d = synth.cohort(n, m, 13, missing=0.02, n_causal=20, h2=0.5)
    y, X = d["y"], d["X"].astype(np.float32).astype(np.float64)
    a, da = cs.run_lmm_matrix_free(d["bed"], n, m, y, X, rank=20, precision="mixed")
    assert not da["trace_threshold_met"] and da["fallback"] == "none"
    b, db = cs.run_lmm_matrix_free(d["bed"], n, m, y, X, rank=20, precision="mixed",
                                   no_fallback=False)
    assert db["fallback"] == "trace_threshold"
    assert abs(db["sigma2_g"] - da["sigma2_g"]) <= 1e-12 * da["sigma2_g"]
    t = a["tested"]
    assert np.array_equal(b["tested"], t)
    assert np.abs(b["log10p"][t] - a["log10p"][t]).max() <= 1e-9
    c, dc = cs.run_lmm_matrix_free(d["bed"], n, m, y, X, rank=20, precision="mixed",
                                   trace_threshold=0.0, error_tol=0.0)
    assert dc["fallback"] == "error_tolerance"
    assert abs(dc["sigma2_g"] - da["sigma2_g"]) <= 1e-9 * da["sigma2_g"]


def test_cpp_job_writes_the_same_files(tmp_path):
    """cs_run_gwas_lmm (inputs, LOCO null models, scan and result files orchestrated in the
    library's C++) writes byte-identical files to the same run assembled from the individual
    entry points."""
    n, m = 500, 1600
    d = synth.cohort(n, m, 37, missing=0.02, n_causal=30, h2=0.5)
    prefix = str(tmp_path / "c")
    open(prefix + ".bed", "wb").write(d["bed"].tobytes())
    chrom = np.array(["2"] * 700 + ["10"] * 500 + ["X"] * 400)
    with open(prefix + ".bim", "w") as f:
        for j in range(m):
            f.write(f"{chrom[j]}\trs{j}\t0\t{1000 + 10 * j}\tA\tG\n")
    rng = np.random.default_rng(8)
    with open(prefix + ".fam", "w") as f:
        for i in range(n):
            v = "-9" if i % 37 == 5 else repr(float(d["y"][i]))
            f.write(f"F{i} I{i} 0 0 1 {v}\n")
    with open(str(tmp_path / "q.txt"), "w") as f:
        for i in range(n):
            f.write(f"F{i} I{i} {rng.normal():.4f}\n")
    created = "2026-01-01 00:00:00 UTC"
    a = str(tmp_path / "py")
    res, diags, inputs = cs.run_gwas_lmm(prefix, a, qcovar=str(tmp_path / "q.txt"), rank=25,
                                         precision="mixed", created=created)
    b = str(tmp_path / "cpp")
    n_kept, n_scopes = cs.gwas_lmm_files(prefix, b, qcovar=str(tmp_path / "q.txt"), rank=25,
                                         precision="mixed", created=created)
    assert n_kept == len(inputs["keep"]) and n_scopes == 3 == len(diags)
    for ext in (".assoc.txt", ".cosmic.sumstats", ".scan.meta.txt"):
        assert open(a + ext, "rb").read() == open(b + ext, "rb").read(), ext
    # .low_rank.meta.tsv: equal but for DECOMPOSITION_SECONDS (a wall-clock time)
    ra, rb = ([l.split("\t") for l in open(p + ".low_rank.meta.tsv").read().splitlines()]
              for p in (a, b))
    col = ra[0].index("DECOMPOSITION_SECONDS")
    assert [r[:col] + r[col + 1:] for r in ra] == [r[:col] + r[col + 1:] for r in rb]
    assert [r[0] for r in rb[1:]] == ["2", "10", "X"]

"""`.assoc.txt` writer: the reference's header, row layout and default 6-digit formatting
(src/gwas_output_schema.h:14-37, src/gwas_output.cpp:123-183).  Host-only: no GPU."""
import numpy as np
import pytest

import cosmicscanner_b200 as cs

HEADER = ("CHR\tSNP\tBP\tA1\tA2\tFREQ\tN\tBETA_A\tSE_A\tP_A\tLOG10P_A\tBETA_D\tSE_D\tP_D"
          "\tLOG10P_D\tP_JOINT\tLOG10P_JOINT")


def fmt(x):
    # std::ostream's default floating-point output: %g with precision 6
    return "%g" % x


def test_assoc_txt_rows_and_formatting(tmp_path):
    bim = tmp_path / "c.bim"
    bim.write_text("1\trs1\t0\t1000\tA\tG\n1\trs2\t0\t2000\tC\tT\n\n2\trs3\t0.5\t123456789\tG\tA\n")
    res = {
        "freq": np.array([0.123456789, 0.5, 0.0123]),
        "beta": np.array([1.23456789e-5, -2.0, 3.3]),
        "se": np.array([0.000123456789, 1.0 / 3.0, 12345678.9]),
        "p": np.array([1e-300, np.nan, 0.999999999]),
        "log10p": np.array([300.0, np.nan, 4.34e-10]),
        "tested": np.array([1, 1, 1], dtype=np.int32),
    }
    out = tmp_path / "r.assoc.txt"
    cs.write_assoc_txt(str(out), str(bim), res, 4321)
    lines = out.read_text().split("\n")
    assert lines[0] == HEADER
    assert lines[-1] == ""
    rows = lines[1:-1]
    assert len(rows) == 2  # the NaN-P row is skipped
    want0 = ["1", "rs1", "1000", "A", "G", fmt(0.123456789), "4321", fmt(1.23456789e-5),
             fmt(0.000123456789), fmt(1e-300), fmt(300.0)] + ["NA"] * 6
    assert rows[0].split("\t") == want0
    f = rows[1].split("\t")
    assert f[:5] == ["2", "rs3", "123456789", "G", "A"]
    assert f[7] == fmt(3.3) and f[8] == fmt(12345678.9) == "1.23457e+07"
    assert f[9] == "1" and f[10] == fmt(4.34e-10)


def test_stcg_layout_and_untested_rows(tmp_path):
    bim = tmp_path / "c.bim"
    bim.write_text("1 a 0 10 A C\n1 b 0 20 G T\n")
    res = {k: np.array([0.25, 0.5]) for k in ("freq", "beta", "se", "p", "log10p")}
    res["tested"] = np.array([0, 1], dtype=np.int32)
    out = tmp_path / "r.stcg.assoc.txt"
    cs.write_assoc_txt(str(out), str(bim), res, 10, stcg_columns=True)
    lines = out.read_text().strip().split("\n")
    assert lines[0] == "CHR\tSNP\tBP\tA1\tA2\tFREQ\tN\tBETA\tSE\tP\tLOG10P"
    assert lines[1].split("\t") == ["1", "b", "20", "G", "T", "0.5", "10", "0.5", "0.5", "0.5", "0.5"]
    assert len(lines) == 2


def test_writer_errors(tmp_path):
    res = {k: np.zeros(1) for k in ("freq", "beta", "se", "p", "log10p")}
    with pytest.raises(cs.CosmicError):
        cs.write_assoc_txt(str(tmp_path / "x"), str(tmp_path / "missing.bim"), res, 1)
    bim = tmp_path / "c.bim"
    bim.write_text("1 a 0 10 A C\n1 b 0 20 G T\n")
    with pytest.raises(cs.InvalidArgument):
        cs.write_assoc_txt(str(tmp_path / "x"), str(bim), res, 1)


def test_chromosome_order_and_bim_reader(tmp_path):
    """LOCO chromosome order (src/gwas_scanner.cpp:62-72: std::stoi comparison, else string)
    and the .bim columns of PlinkReader::readBim."""
    assert cs.sort_chrom_labels(["10", "2", "X", "1", "MT", "2", "22", "Y"]) == \
        ["1", "2", "10", "22", "MT", "X", "Y"]
    bim = tmp_path / "x.bim"
    bim.write_text("1 rs1 0.0 100 A G\n\n2 rs2 0.5 200 C T\n")
    b = cs.read_bim(str(bim))
    assert list(b["chrom"]) == ["1", "2"] and list(b["bp"]) == [100, 200]
    assert b["a1"] == ["A", "C"] and b["a2"] == ["G", "T"]


def test_assoc_mv_txt(tmp_path):
    """`.assoc.mv.txt` columns (src/models/multivariate_model.cpp:943-951, multivariate_output.cpp:
    40-70): WALD_STAT, P, then BETA_t / SE_t with SE = sqrt(Var diagonal); NaN-P rows skipped."""
    bim = tmp_path / "c.bim"
    bim.write_text("1 a 0 10 A C\n1 b 0 20 G T\n")
    res = {"freq": np.array([0.25, 0.5]), "wald": np.array([3.5, np.nan]),
           "p": np.array([0.17, np.nan]), "beta": np.array([[0.1, -0.2], [0, 0]]),
           "cov": np.array([[[0.04, 0.01], [0.01, 0.09]], [[1, 0], [0, 1]]])}
    out = tmp_path / "r.assoc.mv.txt"
    cs.write_assoc_mv_txt(str(out), str(bim), res)
    lines = out.read_text().strip().split("\n")
    assert lines[0] == "CHR\tSNP\tBP\tA1\tA2\tFREQ\tWALD_STAT\tP\tBETA_1\tSE_1\tBETA_2\tSE_2"
    assert lines[1].split("\t") == ["1", "a", "10", "A", "C", "0.25", "3.5", "0.17", "0.1", "0.2",
                                    "-0.2", "0.3"]
    assert len(lines) == 2
    res["cov"][0, 1, 1] = -1.0
    with pytest.raises(cs.CosmicError):
        cs.write_assoc_mv_txt(str(out), str(bim), res)


def test_scan_and_low_rank_meta(tmp_path):
    """OUT.scan.meta.txt (src/gwas_scanner.cpp:93-108) and OUT.low_rank.meta.tsv (:109-115,
    409-428): the reference's items, columns and number formatting (default 6 significant
    digits; 12 from RESIDUAL_EIGENVALUE on, kept for the following rows)."""
    out = str(tmp_path / "run")
    cs.write_scan_meta(out, 256, 0.95)
    lines = open(out + ".scan.meta.txt").read().splitlines()
    assert lines[0] == "Item\tValue"
    items = dict(l.split("\t") for l in lines[1:])
    assert items["analysis_model"] == "univariate_lmm"
    assert items["resolved_scan_tier"] == "approx" and items["snp_vc_strategy"] == "fixed_null"
    assert items["matrix_approximation"] == "fastlmm_auto_trace"
    assert items["requested_rank"] == "256" and items["trace_threshold"] == "0.95"
    assert items["RANK_SELECTION"] == "AUTO_TRACE" and items["HWE_APPLIED"] == "false"
    base = dict(requested_rank=256, effective_rank=30, sketch_size=40, trace_threshold_met=1,
                residual_eigenvalue=0.123456789012345, relative_frobenius_error=0.0123456789,
                trace=1.0, trace_fraction=0.987654321, sigma2_g=0.5, sigma2_e=0.5, delta=1.0,
                log_eta=0.0, reml_objective=0.0, seconds=1.5)
    other = dict(base, effective_rank=28, residual_eigenvalue=0.2, seconds=2.25)
    cs.write_low_rank_meta(out, [("1", base), ("2", other)], n=600)
    rows = [l.split("\t") for l in open(out + ".low_rank.meta.tsv").read().splitlines()]
    assert rows[0][:3] == ["SCOPE", "ALGORITHM", "REQUESTED_RANK"] and rows[0][-1] == "FALLBACK"
    assert len(rows[0]) == 16
    n = 600
    for r, scope, d in ((rows[1], "1", base), (rows[2], "2", other)):
        k, sk = d["effective_rank"], d["sketch_size"]
        assert r == [scope, "randomized_subspace_iteration_tail_mean_woodbury", str(k), str(k),
                     str(sk), "%.12g" % d["residual_eigenvalue"],
                     "%.12g" % d["relative_frobenius_error"], "1", "%.12g" % d["seconds"],
                     str(8 * (2 * n * sk + n * k + sk * sk)), str(24 * n * n), str(k), str(n),
                     "%.12g" % d["trace_fraction"], "MATRIX_FREE_AUTO_TRACE", "none"]


def _results():
    return {
        "freq": np.array([0.123456789, 0.5, 0.0123, 0.3]),
        "beta": np.array([1.23456789012e-5, -2.0, 3.3, 0.25]),
        "se": np.array([0.000123456789, 1.0 / 3.0, 0.0, 0.5]),
        "p": np.array([1e-300, np.nan, 0.999999999, 0.5]),
        "log10p": np.array([300.0, np.nan, 4.34e-10, 0.30103]),
        "tested": np.array([1, 1, 1, 0], dtype=np.int32),
    }


BIM4 = "1\trs1\t0\t1000\tA\tG\n1\trs2\t0\t2000\tC\tT\n2\trs3\t0\t3000\tG\tA\n2\trs4\t0\t4000\tT\tC\n"


def test_ssf_layout_and_row_order(tmp_path):
    """`--out-ssf` (src/gwas_output.cpp:81-82, 149-153) and rows in a given SNP order."""
    bim = tmp_path / "c.bim"
    bim.write_text(BIM4)
    out = tmp_path / "r.assoc.txt"
    cs.write_assoc_txt(str(out), str(bim), _results(), 77, layout="ssf", order=[2, 0, 1, 3])
    lines = out.read_text().splitlines()
    assert lines[0] == ("chromosome\tbase_pair_location\teffect_allele\tother_allele"
                        "\teffect_allele_frequency\tsample_size\tbeta\tstandard_error\tp_value"
                        "\tvariant_id")
    assert [l.split("\t")[-1] for l in lines[1:]] == ["rs3", "rs1"]  # NaN P and untested skipped
    assert lines[2].split("\t") == ["1", "1000", "A", "G", fmt(0.123456789), "77",
                                    fmt(1.23456789012e-5), fmt(0.000123456789), fmt(1e-300), "rs1"]
    with pytest.raises(cs.InvalidArgument):
        cs.write_assoc_txt(str(out), str(bim), _results(), 77, order=[0, 0])
    with pytest.raises(cs.InvalidArgument):
        cs.write_assoc_txt(str(out), str(bim), _results(), 77, order=[4])


def _zlib_matches_python():
    import ctypes
    import ctypes.util
    import zlib
    try:
        lib = ctypes.CDLL(ctypes.util.find_library("z") or "libz.so.1")
    except OSError:
        return False
    lib.zlibVersion.restype = ctypes.c_char_p
    return lib.zlibVersion().decode() == zlib.ZLIB_RUNTIME_VERSION


def test_gzip_output(tmp_path):
    """`--out-gz` (src/gzip_writer.cpp:12-55): the same text as a gzip member; the mode string
    "wb-1" puts zlib at level 1, which the header's XFL byte records (4).  Where this
    process's zlib is the library's, the bytes equal a level-1 gzip stream of the text."""
    import gzip
    import zlib
    bim = tmp_path / "c.bim"
    bim.write_text(BIM4)
    res = _results()
    plain, packed = tmp_path / "a.assoc.txt", tmp_path / "b.assoc.txt"
    cs.write_assoc_txt(str(plain), str(bim), res, 10)
    cs.write_assoc_txt(str(packed), str(bim), res, 10, gzip=True)
    raw = packed.read_bytes()
    assert raw[:4] == b"\x1f\x8b\x08\x00" and raw[4:8] == b"\x00\x00\x00\x00"
    assert raw[8] == 4  # XFL: fastest (level 1)
    assert gzip.decompress(raw) == plain.read_bytes()
    if _zlib_matches_python():
        c = zlib.compressobj(1, zlib.DEFLATED, 31, 8)
        assert raw == c.compress(plain.read_bytes()) + c.flush()
    # a large file crosses the 8 KiB buffer many times
    m = 5000
    big = tmp_path / "big.bim"
    big.write_text("".join(f"1\trs{j}\t0\t{j}\tA\tG\n" for j in range(m)))
    rng = np.random.default_rng(0)
    r2 = {k: rng.random(m) for k in ("freq", "beta", "se", "p", "log10p")}
    cs.write_assoc_txt(str(plain), str(big), r2, 10)
    cs.write_assoc_txt(str(packed), str(big), r2, 10, gzip=True)
    assert gzip.decompress(packed.read_bytes()) == plain.read_bytes()


def test_cosmic_sumstats(tmp_path):
    """`.cosmic.sumstats` (src/gwas_output.cpp:186-234): header on the first call, rows of
    later chromosomes appended; BETA/SE/P at 10 significant digits, AF/LOG10P/Z/WEIGHT at 6,
    INFO 1; gzip appends concatenate members."""
    import gzip
    bim = tmp_path / "c.bim"
    bim.write_text(BIM4)
    res = _results()
    res["tested"] = np.array([1, 1, 0, 0], dtype=np.int32)
    second = dict(res, tested=np.array([0, 0, 1, 1], dtype=np.int32))
    second["tested"][3] = 1
    second["p"] = res["p"].copy()
    for gz in (False, True):
        path = str(tmp_path / ("s.cosmic.sumstats" + (".gz" if gz else "")))
        cs.append_cosmic_sumstats(path, str(bim), res, 900, created="2025-01-02 03:04:05 UTC",
                                  gzip=gz)
        cs.append_cosmic_sumstats(path, str(bim), second, 900, append=True, gzip=gz)
        text = (gzip.decompress(open(path, "rb").read()) if gz else open(path, "rb").read())
        lines = text.decode().splitlines()
        assert lines[:4] == ["# CosmicScanner Summary Statistics v1.0",
                             "# Created: 2025-01-02 03:04:05 UTC", "# Model: LMM", "#"]
        assert lines[4] == ("CHR\tSNP\tPOS\tA1\tA2\tBETA\tSE\tP\tN\tAF\tLOG10P\tMODEL\tZ\tWEIGHT"
                            "\tINFO\tWARNING")
        body = [l.split("\t") for l in lines[5:]]
        assert [b[1] for b in body] == ["rs1", "rs3", "rs4"]
        b, s, p = res["beta"][0], res["se"][0], res["p"][0]
        assert body[0] == ["1", "rs1", "1000", "A", "G", "%.10g" % b, "%.10g" % s, "%.10g" % p,
                           "900", "%.6g" % res["freq"][0], "%.6g" % res["log10p"][0], "LMM",
                           "%.6g" % (b / s), "%.6g" % (1 / (s * s)), "1", "."]
        # SE = 0: Z and WEIGHT are 0
        assert body[1][12:14] == ["0", "0"] and body[1][5] == "3.3"
        if gz:
            assert open(path, "rb").read().count(b"\x1f\x8b\x08") >= 2
    # no fixed time: the current UTC time in the reference's format
    path = str(tmp_path / "t.cosmic.sumstats")
    cs.append_cosmic_sumstats(path, str(bim), res, 900, model="")
    lines = open(path).read().splitlines()
    import re
    assert re.fullmatch(r"# Created: \d{4}-\d\d-\d\d \d\d:\d\d:\d\d UTC", lines[1])
    assert lines[2] == "#"  # an empty model name writes no "# Model:" line


def test_scan_common_meta(tmp_path):
    """The lines appended to OUT.scan.meta.txt after the scan (src/gwas_output_schema.h:57-73)."""
    out = str(tmp_path / "run")
    cs.write_scan_meta(out, 256, 0.95)
    cs.append_scan_common_meta(out, 4321, loco=True)
    lines = open(out + ".scan.meta.txt").read().splitlines()
    assert lines[-7:] == [
        "MODEL\tadditive", "N\t4321",
        "N_SEMANTICS\tanalysis_samples_after_phenotype_and_covariate_filtering;"
        "per-SNP_missing_genotypes_mean-imputed",
        "FREQ_SEMANTICS\tA1_allele_frequency_(not_MAF)", "LOCO\ttrue",
        "COVARIATE_PROJECTION\ttrue", "VCE_CONVERGED\ttrue"]

"""Input side of the association path: .fam samples, phenotype / covariate tables and the
keep list, against the reference's parsing rules (PlinkReader::readFam
libCosmicCore/src/plink_reader.cpp:34-48; PhenoReader::load / align / loadMatrix /
alignMatrix libCosmicCore/src/pheno_reader.cpp:13-215; CovarReader::load / loadCategorical /
align libCosmicCore/src/covar_reader.cpp:19-176, 468-500; DataLoader::loadCovariates
src/data_loader.h:219-261; DataFilter::filterSamples libCosmicCore/src/data_filter.h:21-41).
The expected values are written out from those rules for small synthetic files.  Host code
only: these run without a GPU."""
import math

import numpy as np
import pytest

cs = pytest.importorskip("cosmicscanner_b200")

FAM = """F1 S1 0 0 1 1.5
F1 S2 0 0 2 -9

F2 S3 0 0 1 2.25
F2 S4 0 0 NA 7
F3 S5 0 0 2 0.5
"""


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


@pytest.fixture
def samples(tmp_path):
    return cs.Samples(write(tmp_path, "d.fam", FAM))


def test_fam(samples):
    assert len(samples) == 5  # the empty line is skipped
    assert samples.ids() == [("F1", "S1"), ("F1", "S2"), ("F2", "S3"), ("F2", "S4"), ("F3", "S5")]
    y = samples.fam_phenotype()
    # -9 is not converted here (the .fam column is used as is); a non-numeric sex field
    # leaves the stream failed, so S4's phenotype is never read: the reference leaves it
    # unset, this library gives 0
    assert y.tolist() == [1.5, -9.0, 2.25, 0.0, 0.5]


def test_fam_errors(tmp_path):
    with pytest.raises(cs.CosmicError, match="Cannot open .fam file"):
        cs.Samples(str(tmp_path / "missing.fam"))
    with pytest.raises(cs.CosmicError, match="No samples found"):
        cs.Samples(write(tmp_path, "empty.fam", "\n\n"))


def test_pheno_single_trait(tmp_path, samples):
    path = write(tmp_path, "p.txt", """FID IID height weight
F1 S1 1.5x 10
F1 S2 NA 11
F2 S3 -9.0000001 12
F2 S4 abc 13
F3 S5 3.5
F3 S5 4.5 14
""")
    pr = cs.PhenoReader()
    pr.load(path, 1)
    y, matched = pr.align(samples)
    # "1.5x" -> 1.5 (leading number); NA -> NaN; within 1e-6 of -9 -> missing; "abc" -> NaN;
    # the later S5 row wins
    assert y[0] == 1.5 and math.isnan(y[1]) and math.isnan(y[2]) and math.isnan(y[3])
    assert y[4] == 4.5 and matched == 2
    pr.load(path, 2)
    y2, m2 = pr.align(samples)
    # column 2: every row but the short first S5 row has it; the later S5 row wins
    assert y2.tolist() == [10.0, 11.0, 12.0, 13.0, 14.0] and m2 == 5


def test_pheno_constant_trait(tmp_path, samples):
    path = write(tmp_path, "c.txt", "F1 S1 2\nF1 S2 2\nF2 S3 2\n")
    pr = cs.PhenoReader()
    pr.load(path, 1)
    with pytest.raises(cs.CosmicError, match="zero variance across 3 finite matched samples"):
        pr.align(samples)
    # a single finite value is not refused
    pr.load(write(tmp_path, "one.txt", "F1 S1 2\n"), 1)
    y, m = pr.align(samples)
    assert m == 1 and y[0] == 2.0


def test_pheno_matrix(tmp_path, samples):
    path = write(tmp_path, "m.txt", """F1 S1 1 2 3
F1 S2 4 -9 6
F2 S3 7 8
F2 S4 10 11 12
""")
    pr = cs.PhenoReader()
    pr.loadMatrix(path, [3, 1, 5])
    assert pr.num_traits() == 3
    Y, matched = pr.alignMatrix(samples)
    # the row of S3 has 2 values: column 3 is absent -> NaN (selection keeps the row);
    # column 5 never exists -> NaN everywhere, so no row is complete
    assert Y.shape == (5, 3)
    assert Y[0, :2].tolist() == [3.0, 1.0] and math.isnan(Y[0, 2])
    assert Y[1, :2].tolist() == [6.0, 4.0]
    assert math.isnan(Y[2, 0]) and Y[2, 1] == 7.0
    assert np.isnan(Y[4]).all() and matched == 0
    pr.loadMatrix(path, [])
    assert pr.num_traits() == 3
    Y, matched = pr.alignMatrix(samples)
    # all columns: the first row fixes 3 traits, S3's 2-value row is skipped
    assert Y[0].tolist() == [1.0, 2.0, 3.0] and math.isnan(Y[1, 1]) and np.isnan(Y[2]).all()
    assert Y[3].tolist() == [10.0, 11.0, 12.0] and matched == 2


def test_covar_quantitative(tmp_path, samples):
    path = write(tmp_path, "q.txt", """FID IID age bmi
F1 S1 0.1 20
F1 S2 -9 21
F2 S3 1.0 x 2.0
F2 S4 3 4
""")
    cr = cs.CovarReader()
    cr.load(path)
    assert cr.num_covars() == 2  # the header row has no numbers; the first data row fixes p
    X, matched = cr.align(samples)
    assert X.dtype == np.float32 and X.shape == (5, 2)
    assert X[0, 0] == np.float32(0.1) and X[0, 1] == 20.0  # float32 values
    assert math.isnan(X[1, 0]) and X[1, 1] == 21.0
    assert np.isnan(X[2]).all()  # "1.0 x 2.0" reads 1 value: a short row, skipped
    assert X[3].tolist() == [3.0, 4.0] and np.isnan(X[4]).all()
    assert matched == 2


def test_covar_categorical(tmp_path, samples):
    path = write(tmp_path, "c.txt", """F1 S1 b x 1
F1 S2 a x -9
F2 S3 c x 2
F2 S4 -9 x 1
F3 S5 b x 3
""")
    cr = cs.CovarReader()
    cr.loadCategorical(path)
    # column 1: levels a < b < c -> reference a, dummies b, c; column 2: one level -> none;
    # column 3: levels 1 < 2 < 3 (the missing token excluded) -> dummies 2, 3
    assert cr.num_covars() == 4
    X, matched = cr.align(samples)
    assert X[0].tolist() == [1.0, 0.0, 0.0, 0.0]
    assert X[1, :2].tolist() == [0.0, 0.0] and np.isnan(X[1, 2:]).all()
    assert X[2].tolist() == [0.0, 1.0, 1.0, 0.0]
    assert np.isnan(X[3, :2]).all() and X[3, 2:].tolist() == [0.0, 0.0]
    assert X[4].tolist() == [1.0, 0.0, 0.0, 1.0]
    assert matched == 3


def test_data_filter():
    y = np.array([1.0, np.nan, 3.0, np.inf, 5.0])
    X = np.array([[1, 0], [1, 1], [1, np.nan], [1, 2], [1, 3]], dtype=np.float32)
    # NaN in y or in any covariate drops the sample; inf is kept (only NaN is tested)
    assert cs.DataFilter.filterSamples(y, X).tolist() == [0, 3, 4]
    assert cs.DataFilter.filterSamples(y, np.ones((5, 0), np.float32)).tolist() == [0, 2, 3, 4]
    with pytest.raises(cs.CosmicError, match="dimension mismatch"):
        cs.DataFilter.filterSamples(y, np.ones((4, 1), np.float32))


def test_load_association_inputs(tmp_path):
    n = 14
    fam = "".join(f"F{i} S{i} 0 0 1 {i * 0.5}\n" for i in range(n))
    pheno = "".join(f"F{i} S{i} {'-9' if i == 3 else i * 1.25}\n" for i in range(n))
    qcov = "".join(f"F{i} S{i} {i * 0.1} {'-9' if i == 5 else 1.0}\n" for i in range(n))
    cov = "".join(f"F{i} S{i} {'m' if i % 2 else 'f'}\n" for i in range(n))
    prefix = str(tmp_path / "d")
    open(prefix + ".fam", "w").write(fam)
    d = cs.load_association_inputs(prefix, pheno=write(tmp_path, "p.txt", pheno),
                                   qcovar=write(tmp_path, "q.txt", qcov),
                                   covar=write(tmp_path, "c.txt", cov))
    keep = [i for i in range(n) if i not in (3, 5)]
    assert d["keep"].tolist() == keep
    assert d["y"].tolist() == [i * 1.25 for i in keep]
    X = d["X"]
    assert X.shape == (len(keep), 4)
    assert (X[:, 0] == 1).all()
    assert X[:, 1].tolist() == [float(np.float32(i * 0.1)) for i in keep]
    assert (X[:, 2] == 1).all()
    assert X[:, 3].tolist() == [float(i % 2) for i in keep]  # f is the reference level
    # no phenotype file: the .fam column
    d2 = cs.load_association_inputs(prefix)
    assert d2["y"].tolist() == [i * 0.5 for i in range(n)]
    # fewer than 10 complete samples
    few = "".join(f"F{i} S{i} {'-9' if i > 5 else i}\n" for i in range(n))
    with pytest.raises(cs.CosmicError, match="Too few valid samples"):
        cs.load_association_inputs(prefix, pheno=write(tmp_path, "few.txt", few))

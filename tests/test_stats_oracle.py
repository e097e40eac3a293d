"""The statistics oracle (oracle/stats_oracle.py) pinned against the
reference's own known answers, plus the host parts of the statistics entry
points that need no GPU: the grouping TSV reader (src/tsv.cpp:118-180) and
the HDF5 dataset reader on the reference's output files.

Known answers: src/test_ska.cpp test_center_mat, test_pcoa (crawford 9 x 9:
centred matrix, eigenpairs, coordinates, proportions), test_pcoa_big (57 x 57
from src/test_ska_pcoa_big.dat), test_permanova_{ties,noties,unequal}
(scikit-bio's F), and the scikit-bio PERMANOVA values and PCoA files that
src/testdata/validation_tests.sh compares against (test500.*)."""
import os

import numpy as np
import pytest

import stats_oracle as so
from conftest import ROOT

FIX = os.path.join(ROOT, "tests", "golden", "fixtures")
H5_UNW = os.path.join(FIX, "test500.unweighted_fp32.f.h5")
H5_WU = os.path.join(FIX, "test500.weighted_unnormalized_fp32.h5")
TSV = os.path.join(FIX, "test500.tsv")


def ska(golden, name):
    return golden["test_ska"][name]


def arr(entry, key, shape=None):
    a = np.array(entry["arrays"][key][0], dtype=np.float64)
    return a.reshape(shape) if shape else a


def read_pcoa_big():
    """src/test_ska.cpp:263-300 reads it: '# unifrac n', n*n values, '# pcoa k',
    k eigenvalues, n*k coordinates, k proportions."""
    lines = [ln.strip() for ln in open(os.path.join(FIX, "test_ska_pcoa_big.dat")) if ln.strip()]
    assert lines[0].startswith("# unifrac")
    n = int(lines[0].split()[-1])
    mat = np.array([float(x) for x in lines[1:1 + n * n]]).reshape(n, n)
    rest = lines[1 + n * n:]
    assert rest[0].startswith("# pcoa")
    k = int(rest[0].split()[-1])
    vals = np.array([float(x) for x in rest[1:]])
    return mat, k, vals[:k], vals[k:k + n * k].reshape(n, k), vals[k + n * k:k + n * k + k]


def test_center_matches_reference(golden):
    e = ska(golden, "test_center_mat")
    np.testing.assert_allclose(so.center(arr(e, "matrix", (6, 6))), arr(e, "exp", (6, 6)), atol=1e-6)
    e = ska(golden, "test_pcoa")
    np.testing.assert_allclose(so.center(arr(e, "matrix", (9, 9))), arr(e, "exp2", (9, 9)), atol=1e-5)


def test_pcoa_matches_reference(golden):
    e = ska(golden, "test_pcoa")
    m = arr(e, "matrix", (9, 9))
    w, v = so.eigens(so.center(m), 5)
    np.testing.assert_allclose(w, arr(e, "exp3a"), atol=1e-5)
    np.testing.assert_allclose(np.abs(v), np.abs(arr(e, "exp3b", (9, 5))), atol=1e-5)  # signs may flip
    ev, samples, prop = so.pcoa(m, 5)
    np.testing.assert_allclose(ev, arr(e, "exp3a"), atol=1e-5)
    np.testing.assert_allclose(np.abs(samples), np.abs(arr(e, "exp4b", (9, 5))), atol=1e-5)
    np.testing.assert_allclose(prop, arr(e, "exp4c"), atol=1e-5)


def test_pcoa_big_matches_reference():
    mat, k, ev_exp, samples_exp, prop_exp = read_pcoa_big()
    ev, samples, prop = so.pcoa(mat, k)
    # src/test_ska.cpp:305-330: the last three eigenvalues are close together
    np.testing.assert_allclose(ev[:4], ev_exp[:4], atol=0.01)
    np.testing.assert_allclose(ev[4:], ev_exp[4:], atol=0.1)
    np.testing.assert_allclose(np.abs(samples[:, :4]), np.abs(samples_exp[:, :4]), atol=0.05)
    np.testing.assert_allclose(prop[:4], prop_exp[:4], atol=0.001)
    np.testing.assert_allclose(prop[4:], prop_exp[4:], atol=0.01)


@pytest.mark.parametrize("name", ["test_permanova_ties", "test_permanova_noties", "test_permanova_unequal"])
def test_permanova_f_matches_reference(golden, name):
    e = ska(golden, name)
    n = len(e["arrays"]["grouping_equal"][0])
    for mkey in ("matrix_fp64", "matrix_fp32"):
        m = arr(e, mkey, (n, n))
        for gkey in ("grouping_equal", "grouping_equal_swapped"):
            f = so.permanova_f(m, e["arrays"][gkey][0])
            assert abs(f - e["scalars"]["exp_stat"]) < 1e-5, (mkey, gkey, f)
    # the reference's p-values come from its own random permutations, within 0.05
    p = so.permanova_p_exact(arr(e, "matrix_fp64", (n, n)), e["arrays"]["grouping_equal"][0])
    assert abs(p - e["scalars"]["exp_pvalue"]) < 0.05, p


def test_pcoa_of_reference_outputs(ssu):
    """The 4-axis PCoA stored in the reference's output files against the
    exact one of their own matrices.  validation_tests.sh compares 3 axes at
    relative 0.1; the stored values are randomized-fsvd approximations, within
    0.7 % of the exact eigenvalues and never above them (Ritz values)."""
    for path in (H5_UNW, H5_WU):
        m = ssu.read_h5(path, "matrix")
        ev_exp = ssu.read_h5(path, "pcoa_eigvals")
        samples_exp = ssu.read_h5(path, "pcoa_samples")
        prop_exp = ssu.read_h5(path, "pcoa_proportion_explained")
        ev, samples, prop = so.pcoa(m, len(ev_exp))
        assert np.max(np.abs(ev[:3] - ev_exp[:3]) / ev_exp[:3]) < 0.1
        assert np.max(np.abs(ev - ev_exp) / ev_exp) < 1e-2
        assert np.all(ev_exp <= ev * (1 + 1e-6))
        assert np.max(np.abs(prop - prop_exp) / prop_exp) < 1e-2
        assert np.max(np.abs(np.abs(samples[:, :2]) - np.abs(samples_exp[:, :2]))) < 1e-2
        assert np.max(np.abs(np.abs(samples[:, 2]) - np.abs(samples_exp[:, 2]))) < 0.1


def validation_stats(golden):
    """(check, stored matrix file, same matrix?) per PERMANOVA check.  The
    weighted_unnormalized_fp32 check runs on the matrix stored in
    test500.weighted_unnormalized_fp32.h5; the unweighted checks run without
    -f (bypass_tips, src/su.cpp:634) while test500.unweighted_fp32.f.h5 holds
    the -f matrix, whose distances differ slightly."""
    files = {"unweighted": (H5_UNW, False), "weighted_unnormalized_fp32": (H5_WU, True)}
    return [(c,) + files[c["method"]] for c in golden["validation"]["permanova"]]


def test_permanova_f_of_reference_checks(ssu, golden):
    """scikit-bio's F on the reference's matrices and metadata
    (compare_unifrac_stats.py: relative precision of the value)."""
    checks = validation_stats(golden)
    assert any(same for _, _, same in checks)
    for c, path, same in checks:
        m = ssu.read_h5(path, "matrix")
        ids = ssu.read_h5(path, "order", strings=True)
        st, g, ng = ssu.read_grouping(TSV, c["column"], ids)
        assert st == 0 and ng == c["n_groups"]
        f = so.permanova_f(m, g)
        tol = c["prec_value"] if same else 0.01  # bypass-tips matrix: within 1 %
        assert abs(f - c["value"]) / c["value"] < tol, (c, f)


def test_h5_reader_on_reference_outputs(ssu):
    m = ssu.read_h5(H5_UNW, "matrix")
    assert m.shape == (500, 500)
    np.testing.assert_array_equal(np.diag(m), 0.0)
    np.testing.assert_array_equal(m, m.T)
    ids = ssu.read_h5(H5_UNW, "order", strings=True)
    assert len(ids) == 500 and len(set(ids)) == 500
    assert ssu.read_h5(H5_UNW, "pcoa_samples").shape == (500, 4)
    with pytest.raises(RuntimeError):
        ssu.read_h5(H5_UNW, "no_such_dataset")
    with pytest.raises(RuntimeError):
        ssu.read_h5(H5_UNW, "order")  # strings asked for as numbers


def test_grouping_reader(ssu, tmp_path):
    ids = ["s1", "s2", "s3", "s4"]
    p = tmp_path / "g.tsv"
    p.write_text("#SampleID\tcolA\tcolB\n"
                 "s3\tx\tq\n"
                 "other\ty\tq\n"
                 "s1\ty\t\n"
                 "s2\tx\tq\n"
                 "s4\tz\tq\n")
    st, g, ng = ssu.read_grouping(p, "colA", ids)
    assert st == 0 and ng == 3
    assert list(g) == [1, 0, 0, 2]  # numbered by first appearance among the samples' lines
    st, g, ng = ssu.read_grouping(p, "colB", ids)
    assert st == 0 and ng == 2 and list(g) == [1, 0, 0, 0]  # empty value is a group
    st, _, _ = ssu.read_grouping(p, "#SampleID", ids)
    assert st == 8  # the index column is not a grouping column: grouping_missing
    st, _, _ = ssu.read_grouping(p, "colC", ids)
    assert st == 8
    st, _, _ = ssu.read_grouping(p, "colA", ids + ["s5"])
    assert st == 8  # every sample must have a line
    st, _, _ = ssu.read_grouping(p, "colA", ["s1", "s5"])
    assert st == 8  # the first sample is checked too
    st, _, _ = ssu.read_grouping(tmp_path / "missing.tsv", "colA", ids)
    assert st == 8
    short = tmp_path / "short.tsv"
    short.write_text("#SampleID\tcolA\tcolB\ns1\tx\n")
    st, _, _ = ssu.read_grouping(short, "colB", ["s1"])
    assert st == 8  # a matched line without the field
    dup = tmp_path / "dup.tsv"
    dup.write_text("#SampleID\tc\ns1\ta\ns2\tb\ns1\tc\n")
    st, g, ng = ssu.read_grouping(dup, "c", ["s1", "s2"])
    assert st == 0 and list(g) == [2, 1] and ng == 3  # a later line overrides, its value still numbered


def test_grouping_reader_on_reference_metadata(ssu):
    ids = ssu.read_h5(H5_UNW, "order", strings=True)
    for column, groups in (("empo_2", 5), ("empo_3", 17)):
        st, g, ng = ssu.read_grouping(TSV, column, ids)
        assert st == 0 and ng == groups and g.max() == groups - 1


def test_compute_permanova_status_paths(ssu, tmp_path):
    """grouping_missing before any device work (src/api.cpp:949-975)."""
    m = np.zeros((3, 3))
    ids = ["a", "b", "c"]
    st, _, _ = ssu.compute_permanova(tmp_path / "missing.tsv", ["c1"], m, ids, 9)
    assert st == 8
    p = tmp_path / "g.tsv"
    p.write_text("#SampleID\tc1\na\tx\nb\ty\n")
    st, _, _ = ssu.compute_permanova(p, ["c1"], m, ids, 9)
    assert st == 8  # sample c has no line
    st, _, _ = ssu.compute_permanova(p, ["nope"], m[:2, :2], ids[:2], 9)
    assert st == 8

"""The file-based entry points on the GPU against the reference's own expected
outputs (tests/golden/fixtures, copied from the reference by
tests/golden/make_golden.py): the crawford table with ci/test.ssu.exp,
ci/test.ssu_vaw.exp and ci/test.faith.exp (ci/crawford_test.sh), and the
absquant table with its weighted-normalized matrices
(src/testdata/validation_tests.sh:135-146).  Every one_off_matrix* form
(src/api.hpp:348-436), one_off_v3 and partial_v3 agree with one another."""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_err
from test_biom_files import read_dm, read_faith

pytestmark = pytest.mark.gpu

FIX = os.path.join(ROOT, "tests", "golden", "fixtures")
BIOM = os.path.join(FIX, "crawford.biom")
TRE = os.path.join(FIX, "crawford.tre")


def test_one_off_matrix_v3_reproduces_the_crawford_expected_matrices(ssu):
    for vaw, expected in ((False, "test.ssu.exp"), (True, "test.ssu_vaw.exp")):
        got, ids = ssu.file_matrix("one_off_matrix_v3", BIOM, TRE, "unweighted_fp64", variance_adjust=vaw)
        want_ids, want = read_dm(os.path.join(FIX, expected))
        assert ids == want_ids
        r, z = rel_err(got, want)
        assert r <= 1e-12 and z == 0.0, (expected, r, z)


def test_every_one_off_matrix_form_agrees(ssu):
    ref, ids = ssu.file_matrix("one_off_matrix_v3", BIOM, TRE, "weighted_normalized_fp64")
    opaque = ssu.OpaqueTree(path=TRE)
    for entry in ("one_off_matrix_v3t", "one_off_matrix_v2", "one_off_matrix_v2t", "one_off_matrix"):
        got, got_ids = ssu.file_matrix(entry, BIOM, opaque if entry.endswith("t") else TRE, "weighted_normalized_fp64")
        assert got_ids == ids
        np.testing.assert_array_equal(got, ref)
    ref32, _ = ssu.file_matrix("one_off_matrix_fp32_v3", BIOM, TRE, "weighted_normalized")
    assert ref32.dtype == np.float32
    assert rel_err(ref32, ref)[0] < 1e-5
    for entry in ("one_off_matrix_fp32_v3t", "one_off_matrix_fp32_v2", "one_off_matrix_fp32_v2t",
                  "one_off_matrix_fp32"):
        got, _ = ssu.file_matrix(entry, BIOM, opaque if entry.endswith("t") else TRE, "weighted_normalized")
        np.testing.assert_array_equal(got, ref32)
    opaque.close()


def test_result_precision_follows_the_entry_point_and_arithmetic_the_method(ssu):
    """one_off_matrix_T computes in the method's precision and writes the
    result type's (src/api.cpp:639-696)."""
    f32_in_64, _ = ssu.file_matrix("one_off_matrix_v3", BIOM, TRE, "weighted_normalized")
    f32, _ = ssu.file_matrix("one_off_matrix_fp32_v3", BIOM, TRE, "weighted_normalized")
    assert f32_in_64.dtype == np.float64
    np.testing.assert_array_equal(f32_in_64, f32.astype(np.float64))
    f64_in_32, _ = ssu.file_matrix("one_off_matrix_fp32_v3", BIOM, TRE, "weighted_normalized_fp64")
    f64, _ = ssu.file_matrix("one_off_matrix_v3", BIOM, TRE, "weighted_normalized_fp64")
    np.testing.assert_array_equal(f64_in_32, f64.astype(np.float32))


def test_one_off_v3_and_partial_v3_agree_with_the_matrix(ssu):
    full, ids = ssu.file_matrix("one_off_matrix_v3", BIOM, TRE, "unweighted_fp64")
    cf, cf_ids = ssu.file_one_off(BIOM, TRE, "unweighted_fp64")
    assert cf_ids == ids
    np.testing.assert_array_equal(cf, full[np.triu_indices(len(ids), 1)])
    n = len(ids)
    for start, stop in ((0, 3), (3, 5), (0, 5)):
        stripes, p_ids = ssu.file_partial(BIOM, TRE, "unweighted_fp64", start, stop)
        assert p_ids == ids
        k = np.arange(n)
        want = np.stack([full[k, (k + s + 1) % n] for s in range(start, stop)])
        np.testing.assert_array_equal(stripes, want)


def test_faith_pd_one_off_reproduces_the_crawford_expected_values(ssu):
    vals, ids = ssu.file_faith_pd(BIOM, TRE)
    want_ids, want = read_faith(os.path.join(FIX, "test.faith.exp"))
    assert ids == want_ids
    np.testing.assert_allclose(vals, want, rtol=1e-12)


@pytest.mark.parametrize("method", ["weighted_normalized", "weighted_normalized_fp64"])
@pytest.mark.parametrize("normalize,expected", [(False, "test.absquant.wn.dm"), (True, "test.absquant_not.wn.dm")])
def test_absquant_matrices_with_and_without_sample_normalisation(ssu, method, normalize, expected):
    biom = os.path.join(FIX, "absquant.biom")
    tre = os.path.join(FIX, "absquant.tree")
    got, ids = ssu.file_matrix("one_off_matrix_v3", biom, tre, method, normalize=normalize)
    want_ids, want = read_dm(os.path.join(FIX, expected))
    assert ids == want_ids
    np.testing.assert_allclose(got, want, atol=1.01e-6)  # six decimals in the expected files


def test_subsampled_file_matrix_keeps_the_deep_samples(ssu):
    table = ssu.read_biom(BIOM)
    totals = table.dense().sum(axis=0)
    depth = int(np.sort(totals)[3])
    ssu.lib().ssu_set_random_seed(11)
    m, ids = ssu.file_matrix("one_off_matrix_v3", BIOM, TRE, "unweighted_fp64", subsample_depth=depth)
    assert ids == [table.sample_ids[j] for j in range(table.n_samples) if totals[j] >= depth]
    assert np.all(np.isfinite(m)) and np.all(np.diag(m) == 0)

"""PCoA and PERMANOVA on the GPU (pcoa, pcoa_fp32, pcoa_mixed,
find_eigens_fast(_fp32), compute_permanova_fp64/_fp32,
ssu_b200_permanova_*) against the reference's known answers
(src/test_ska.cpp:7-637, src/testdata/validation_tests.sh) and the numpy
oracle (exact eigendecomposition, exact pseudo-F, exact permutation
p-values for small n)."""
import os

import numpy as np
import pytest

import stats_oracle as so
from conftest import ROOT

pytestmark = pytest.mark.gpu

FIX = os.path.join(ROOT, "tests", "golden", "fixtures")
H5_UNW = os.path.join(FIX, "test500.unweighted_fp32.f.h5")
H5_WU = os.path.join(FIX, "test500.weighted_unnormalized_fp32.h5")
TSV = os.path.join(FIX, "test500.tsv")


def arr(golden, test, key, shape=None):
    a = np.array(golden["test_ska"][test]["arrays"][key][0], dtype=np.float64)
    return a.reshape(shape) if shape else a


def same_up_to_sign(a, b):
    """max |a - s b| over columns, s the better sign per column."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return max(min(np.max(np.abs(a[:, k] - b[:, k])), np.max(np.abs(a[:, k] + b[:, k]))) for k in range(a.shape[1]))


def test_pcoa_reference_known_answers(ssu, golden):
    """src/test_ska.cpp:64-260 (crawford 9 x 9, 5 axes), all three forms."""
    m = arr(golden, "test_pcoa", "matrix", (9, 9))
    exp_ev = arr(golden, "test_pcoa", "exp3a")
    exp_samples = arr(golden, "test_pcoa", "exp4b", (9, 5))
    exp_prop = arr(golden, "test_pcoa", "exp4c")
    o_ev, o_samples, o_prop = so.pcoa(m, 5)
    for entry in ("pcoa", "pcoa_fp32", "pcoa_mixed"):
        ev, samples, prop = ssu.pcoa(m, 5, entry)
        np.testing.assert_allclose(ev, exp_ev, atol=1e-5)
        np.testing.assert_allclose(np.abs(samples), np.abs(exp_samples), atol=1e-5)
        np.testing.assert_allclose(prop, exp_prop, atol=1e-5)
        tol = 1e-11 if entry == "pcoa" else 1e-6
        np.testing.assert_allclose(ev, o_ev, rtol=tol)
        np.testing.assert_allclose(prop, o_prop, rtol=tol)
        assert same_up_to_sign(samples, o_samples) < tol
        # the sign convention: each axis's largest-magnitude coordinate is positive
        big = np.argmax(np.abs(samples), axis=0)
        assert np.all(samples[big, np.arange(5)] > 0)


def test_find_eigens_fast_reference_known_answers(ssu, golden):
    """src/test_ska.cpp:122-156: eigenpairs of the centred crawford matrix."""
    centred = arr(golden, "test_pcoa", "exp2", (9, 9))
    keep = centred.copy()
    for fp32 in (False, True):
        ev, vec = ssu.find_eigens_fast(centred, 5, fp32=fp32)
        np.testing.assert_allclose(ev, arr(golden, "test_pcoa", "exp3a"), atol=1e-5)
        np.testing.assert_allclose(np.abs(vec), np.abs(arr(golden, "test_pcoa", "exp3b", (9, 5))), atol=1e-5)
        np.testing.assert_allclose(np.linalg.norm(vec, axis=0), 1.0, rtol=1e-6)
    np.testing.assert_array_equal(centred, keep)  # input not modified


def read_pcoa_big():
    lines = [ln.strip() for ln in open(os.path.join(FIX, "test_ska_pcoa_big.dat")) if ln.strip()]
    n = int(lines[0].split()[-1])
    mat = np.array([float(x) for x in lines[1:1 + n * n]]).reshape(n, n)
    rest = lines[1 + n * n:]
    k = int(rest[0].split()[-1])
    vals = np.array([float(x) for x in rest[1:]])
    return mat, k, vals[:k], vals[k:k + n * k].reshape(n, k), vals[k + n * k:k + n * k + k]


@pytest.mark.parametrize("entry", ["pcoa", "pcoa_fp32", "pcoa_mixed"])
def test_pcoa_big_reference_known_answers(ssu, entry):
    """src/test_ska.cpp:263-464 with its tolerances, and the exact oracle."""
    mat, k, ev_exp, samples_exp, prop_exp = read_pcoa_big()
    ev, samples, prop = ssu.pcoa(mat, k, entry)
    np.testing.assert_allclose(ev[:4], ev_exp[:4], atol=0.01)
    np.testing.assert_allclose(ev[4:], ev_exp[4:], atol=0.1)
    np.testing.assert_allclose(np.abs(samples[:, :4]), np.abs(samples_exp[:, :4]), atol=0.1)
    np.testing.assert_allclose(prop[:4], prop_exp[:4], atol=0.001)
    np.testing.assert_allclose(prop[4:], prop_exp[4:], atol=0.01)
    o_ev, o_samples, o_prop = so.pcoa(mat, k)
    tol = 1e-8 if entry == "pcoa" else 1e-5
    np.testing.assert_allclose(ev, o_ev, rtol=tol)
    np.testing.assert_allclose(prop, o_prop, rtol=tol)


@pytest.mark.parametrize("path", [H5_UNW, H5_WU])
def test_pcoa_of_reference_outputs(ssu, path):
    """The reference's 500-sample outputs: the stored 4-axis fsvd PCoA at the
    reference's precision (3 axes, relative 0.1), the exact oracle tightly."""
    m = ssu.read_h5(path, "matrix")
    ev_exp = ssu.read_h5(path, "pcoa_eigvals")
    for entry, mm in (("pcoa", m), ("pcoa_fp32", m.astype(np.float32))):
        ev, samples, prop = ssu.pcoa(mm, 4, entry)
        assert np.max(np.abs(ev[:3] - ev_exp[:3]) / ev_exp[:3]) < 0.1
        o_ev, o_samples, o_prop = so.pcoa(m, 4)
        np.testing.assert_allclose(ev, o_ev, rtol=1e-7)
        np.testing.assert_allclose(prop, o_prop, rtol=1e-7)
        assert same_up_to_sign(samples[:, :2], o_samples[:, :2]) < 1e-5


def euclidean_matrix(n, dims, seed, decay=0.7):
    """Distances between n points whose coordinates have geometrically
    decaying spread: a PSD centred matrix with a clear spectrum."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, dims)) * decay ** np.arange(dims)
    sq = (x * x).sum(axis=1)
    d2 = np.maximum(sq[:, None] + sq[None, :] - 2 * x @ x.T, 0.0)
    d = np.sqrt(d2)
    np.fill_diagonal(d, 0.0)
    return d


def test_pcoa_large_against_exact(ssu):
    m = euclidean_matrix(3000, 40, 1)
    ev, samples, prop = ssu.pcoa(m, 10)
    o_ev, o_samples, o_prop = so.pcoa(m, 10)
    np.testing.assert_allclose(ev, o_ev, rtol=1e-9)
    np.testing.assert_allclose(prop, o_prop, rtol=1e-9)
    assert same_up_to_sign(samples, o_samples) < 1e-6 * np.abs(o_samples).max()


def test_pcoa_device_resident_matrix(ssu):
    """A device pointer is read in place and gives the host call's result."""
    import torch
    m = euclidean_matrix(700, 20, 2)
    host = ssu.pcoa(m, 6)
    dev = torch.from_numpy(m).cuda()
    torch.cuda.synchronize()
    out = ssu.pcoa_device(dev.data_ptr(), 700, 6)
    for a, b in zip(host, out):
        np.testing.assert_array_equal(a, b)


def test_pcoa_edge_sizes(ssu):
    ev, samples, prop = ssu.pcoa(np.zeros((1, 1)), 3)
    assert np.all(ev == 0) and samples.shape == (1, 3) and np.all(samples == 0)
    m = np.array([[0.0, 2.0], [2.0, 0.0]])
    ev, samples, prop = ssu.pcoa(m, 3)  # rank 1: one axis, the others zero
    np.testing.assert_allclose(ev, [2.0, 0.0, 0.0], atol=1e-12)
    np.testing.assert_allclose(np.abs(samples[:, 0]), [1.0, 1.0], rtol=1e-12)
    np.testing.assert_allclose(prop, [1.0, 0.0, 0.0], atol=1e-12)
    m = euclidean_matrix(12, 3, 3)  # more axes asked than the rank
    ev, samples, prop = ssu.pcoa(m, 8)
    o_ev, _, _ = so.pcoa(m, 3)
    np.testing.assert_allclose(ev[:3], o_ev, rtol=1e-10)
    assert np.all(np.abs(ev[3:]) < 1e-10 * o_ev[0])
    ev, samples, prop = ssu.pcoa(euclidean_matrix(9, 3, 4), 0)
    assert ev.shape == (0,) and samples.shape == (9, 0)


@pytest.mark.parametrize("name", ["test_permanova_ties", "test_permanova_noties", "test_permanova_unequal"])
def test_permanova_reference_known_answers(ssu, golden, name):
    """src/test_ska.cpp:467-637: F to 1e-5 for both matrices and both
    labelings; p within 0.05 of the reference's and of the exact p."""
    e = golden["test_ska"][name]
    n = len(e["arrays"]["grouping_equal"][0])
    exact_p = so.permanova_p_exact(arr(golden, name, "matrix_fp64", (n, n)), e["arrays"]["grouping_equal"][0])
    for mkey, fp32 in (("matrix_fp64", False), ("matrix_fp32", True)):
        m = arr(golden, name, mkey, (n, n))
        for gkey in ("grouping_equal", "grouping_equal_swapped"):
            g = e["arrays"][gkey][0]
            f, p = ssu.permanova(m, g, 999, fp32=fp32)
            assert abs(f - e["scalars"]["exp_stat"]) < 1e-5
            assert abs(f - so.permanova_f(m.astype(np.float32) if fp32 else m, g)) < 1e-6 * abs(f)
            assert abs(p - e["scalars"]["exp_pvalue"]) < 0.05
            assert abs(p - exact_p) < 0.05


def test_permanova_f_exact_and_p_properties(ssu):
    rng = np.random.default_rng(5)
    n = 2000
    m = euclidean_matrix(n, 30, 6)
    g = rng.integers(0, 4, n)
    f, p = ssu.permanova(m, g, 99)
    assert abs(f - so.permanova_f(m, g)) < 1e-10 * f
    assert 0.01 <= p <= 1.0 and abs(p * 100 - round(p * 100)) < 1e-9  # (1 + k) / 100
    # a strong group effect: no permutation reaches the observed F
    shifted = euclidean_matrix(n, 30, 6) + 5.0 * (g[:, None] != g[None, :])
    np.fill_diagonal(shifted, 0.0)
    f2, p2 = ssu.permanova(shifted, g, 99)
    assert abs(f2 - so.permanova_f(shifted, g)) < 1e-10 * f2
    assert p2 == pytest.approx(0.01)
    # labels are any values: renumbering them changes nothing
    f3, p3 = ssu.permanova(m, g * 7 + 3, 99)
    assert f3 == f and p3 == p


def test_permanova_seed_and_degenerate(ssu):
    L = ssu.lib()
    m = euclidean_matrix(60, 5, 7)
    g = np.arange(60) % 3
    L.ssu_set_random_seed(11)
    a = ssu.permanova(m, g, 199)
    b = ssu.permanova(m, g, 199)
    assert a == b  # same seed, same permutations
    L.ssu_set_random_seed(5489)
    f, p = ssu.permanova(m, g, 0)
    assert np.isfinite(f) and np.isnan(p)  # no permutations: no p-value
    f, p = ssu.permanova(m, np.zeros(60), 99)
    assert np.isnan(f) and np.isnan(p)  # one group
    f, p = ssu.permanova(m, np.arange(60), 99)
    assert np.isnan(f) and np.isnan(p)  # every sample its own group


def test_compute_permanova_on_reference_outputs(ssu, golden):
    """validation_tests.sh's checks through compute_permanova_fp64/_fp32 and
    the metadata file.  The weighted_unnormalized_fp32 check runs on the
    stored matrix: F within its relative 1e-3, p within its relative 0.1.
    The unweighted checks ran without bypass_tips while the stored matrix is
    the bypass_tips one: F is held to the oracle on that matrix instead."""
    for c in golden["validation"]["permanova"]:
        path = H5_WU if c["method"] == "weighted_unnormalized_fp32" else H5_UNW
        m = ssu.read_h5(path, "matrix")
        ids = ssu.read_h5(path, "order", strings=True)
        _, g, _ = ssu.read_grouping(TSV, c["column"], ids)
        for fp32 in (False, True):
            st, fs, ps = ssu.compute_permanova(TSV, [c["column"]], m, ids, c["n_perms"], fp32=fp32)
            assert st == 0
            f, p = fs[0], ps[0]
            assert abs(f - so.permanova_f(m, g)) < (1e-6 if fp32 else 1e-10) * f
            if path == H5_WU:
                assert abs(f - c["value"]) / c["value"] < c["prec_value"]
                assert abs(p - c["pvalue"]) / c["pvalue"] < c["prec_pvalue"], p
    # several columns in one call, each with its own permutations
    m = ssu.read_h5(H5_WU, "matrix")
    ids = ssu.read_h5(H5_WU, "order", strings=True)
    st, fs, ps = ssu.compute_permanova(TSV, ["empo_2", "empo_3"], m, ids, 99)
    assert st == 0 and len(fs) == 2 and fs[0] != fs[1]


def test_permanova_chunked_labels_change_nothing(ssu, monkeypatch):
    """Permutations evaluated in chunks of columns (a label budget far below
    one pass) give the same F and p, bit for bit, as one chunk."""
    L = ssu.lib()
    m = euclidean_matrix(500, 8, 9)
    g = np.arange(500) % 4
    L.ssu_set_random_seed(21)
    whole = ssu.permanova(m, g, 999)
    monkeypatch.setenv("UNIFRAC_B200_PERMANOVA_LABEL_BYTES", str(500 * 2 * 64))  # 64 groupings per chunk
    L.ssu_set_random_seed(21)
    chunked = ssu.permanova(m, g, 999)
    L.ssu_set_random_seed(5489)
    assert chunked == whole

"""Pin the C restatement against the reference's own CPU code, compiled from
its sources into oracle/_ref (oracle/Makefile).  Skipped where the reference
could not be built (it needs the reference checkout)."""
import numpy as np
import pytest

import ssu_synth
from conftest import rel_err

METHODS = ["unweighted", "unweighted_unnormalized", "weighted_normalized", "weighted_unnormalized", "generalized"]


@pytest.fixture(scope="module")
def ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    return oracle_mod


def _small_case(seed, n_tips=60, n_samples=37, density=0.15):
    tree = ssu_synth.random_binary_tree(n_tips, 0.1, seed)
    table = ssu_synth.geometric_table(tree.tip_names()[: n_tips - 5], n_samples, density, 8.0, seed + 7)
    return tree, table


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("vaw", [False, True])
@pytest.mark.parametrize("bypass", [False, True])
def test_oracle_fp64_equals_reference(ref, method, vaw, bypass):
    tree, table = _small_case(11)
    kw = dict(variance_adjust=vaw, bypass_tips=bypass, alpha=0.5)
    a = ref.ref_one_off(tree, table, method + "_fp64", **kw)
    b = ref.oracle_one_off(tree, table, method + "_fp64", **kw)
    assert a["n_embedded"] == b["n_embedded"]
    r, z = rel_err(b["matrix"], a["matrix"])
    assert r <= 1e-13 and z <= 1e-13


@pytest.mark.parametrize("method", METHODS)
def test_oracle_fp32_within_reference_fp32_error(ref, method):
    tree, table = _small_case(12)
    a32 = ref.ref_one_off(tree, table, method + "_fp32", alpha=0.5)["matrix"]
    a64 = ref.ref_one_off(tree, table, method + "_fp64", alpha=0.5)["matrix"]
    b32 = ref.oracle_one_off(tree, table, method + "_fp32", alpha=0.5)["matrix"]
    ref_err, _ = rel_err(a32, a64)
    ours, _ = rel_err(b32, a64)
    assert ours <= 4 * ref_err + 1e-7


def test_oracle_partial_and_generalized_alpha(ref):
    tree, table = _small_case(13, n_samples=24)
    for alpha in (0.0, 0.25, 1.0, 1.7):
        a = ref.ref_one_off(tree, table, "generalized_fp64", alpha=alpha, stripe_start=3, stripe_stop=9)
        b = ref.oracle_one_off(tree, table, "generalized_fp64", alpha=alpha, stripe_start=3, stripe_stop=9)
        r, z = rel_err(b["stripes"], a["stripes"])
        assert r <= 1e-13 and z <= 1e-13


def test_oracle_faith_equals_reference(ref):
    tree, table = _small_case(14)
    # a sample with zero counts is filtered out by both
    dense = table.dense()
    dense[:, 3] = 0
    flat = np.flatnonzero(dense.ravel() > 0)
    t2 = ssu_synth.make_table(table.obs_ids, table.n_samples, flat, dense.ravel()[flat])
    a = ref.ref_faith_pd(tree, t2)
    b = ref.oracle_faith_pd(tree, t2)
    assert list(a["kept"]) == list(b["kept"])
    assert 3 not in list(a["kept"])
    np.testing.assert_allclose(b["values"], a["values"], rtol=1e-14, atol=0)


def test_oracle_unnormalized_counts(ref):
    tree, table = _small_case(15)
    for m in ("weighted_unnormalized_fp64", "weighted_normalized_fp64"):
        a = ref.ref_one_off(tree, table, m, normalize=False)["matrix"]
        b = ref.oracle_one_off(tree, table, m, normalize=False)["matrix"]
        r, _ = rel_err(b, a)
        assert r <= 1e-13


def _negative_case(seed):
    """A table with about 5% of its entries negated (every sample keeps a
    positive total)."""
    tree, table = _small_case(seed)
    rng = np.random.default_rng(seed + 99)
    data = table.data.copy()
    flip = rng.random(data.size) < 0.05
    data[flip] = -0.5 * data[flip]
    return tree, ssu_synth.Table(table.obs_ids, table.sample_ids, table.indptr, table.indices, data)


@pytest.mark.parametrize("method,alpha", [("unweighted", 1.0), ("weighted_normalized", 1.0),
                                          ("weighted_unnormalized", 1.0), ("generalized", 1.0)])
def test_oracle_with_negative_counts_equals_reference(ref, method, alpha):
    tree, table = _negative_case(15)
    a = ref.ref_one_off(tree, table, method + "_fp64", alpha=alpha)["matrix"]
    b = ref.oracle_one_off(tree, table, method + "_fp64", alpha=alpha)["matrix"]
    assert np.array_equal(np.isnan(a), np.isnan(b))
    r, z = rel_err(b, a)
    assert r <= 1e-13 and z <= 1e-13

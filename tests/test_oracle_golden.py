"""The oracle (C restatement, oracle/unifrac_oracle.c) against the reference's
own golden vectors (src/test_su.cpp), read from tests/golden/reference_golden.json.

Tolerances are those of the reference tests (1e-6 absolute,
src/test_helper.hpp) except where the golden is an exact small rational."""
import numpy as np
import pytest

import ssu_synth
from conftest import matrix_from_stripes, stripes_from_golden

CASES = [
    # (test function, golden prefix, method, kwargs)
    ("test_unweighted_unifrac", "", "unweighted_fp64", {}),
    ("test_unweighted_unifrac", "", "unweighted", {}),
    ("test_unweighted_unifrac_fast", "", "unweighted_fp64", {"bypass_tips": True}),
    ("test_unnormalized_unweighted_unifrac", "", "unweighted_unnormalized_fp64", {}),
    ("test_unnormalized_weighted_unifrac", "", "weighted_unnormalized_fp64", {}),
    ("test_normalized_weighted_unifrac", "", "weighted_normalized_fp64", {}),
    ("test_normalized_weighted_unifrac", "", "weighted_normalized", {}),
    ("test_generalized_unifrac", "w_", "generalized_fp64", {"alpha": 1.0}),
    ("test_generalized_unifrac", "d0_", "generalized_fp64", {"alpha": 0.0}),
    ("test_generalized_unifrac", "d05_", "generalized_fp64", {"alpha": 0.5}),
    ("test_vaw_unifrac_weighted_normalized", "w_", "weighted_normalized_fp64", {"variance_adjust": True}),
]


@pytest.mark.parametrize("func,prefix,method,kw", CASES)
def test_oracle_matches_reference_goldens(oracle_mod, golden, test_tree, test_table, func, prefix, method, kw):
    exp = stripes_from_golden(golden["test_su"][func], prefix)
    assert exp.shape == (3, 6)
    r = oracle_mod.oracle_one_off(test_tree, test_table, method, **kw)
    np.testing.assert_allclose(r["stripes"], exp, atol=1e-6, rtol=0)
    np.testing.assert_allclose(r["matrix"], matrix_from_stripes(exp, 6), atol=1e-6, rtol=0)


def test_oracle_faith_golden(oracle_mod, golden, test_table):
    exp = golden["test_su"]["test_faith_pd"]["arrays"]["exp"][0]
    for tre in ("test_faith.tre", "test_faith_shear.tre"):
        import ssu_synth
        tree = ssu_synth.parse_newick(golden["trees"][tre])
        r = oracle_mod.oracle_faith_pd(tree, test_table)
        np.testing.assert_allclose(r["values"], exp, atol=1e-6, rtol=0)
        assert list(r["kept"]) == list(range(6))


def test_oracle_partial_stripes(oracle_mod, golden, test_tree, test_table):
    exp = stripes_from_golden(golden["test_su"]["test_unweighted_unifrac"])
    for start, stop in [(0, 1), (1, 3), (2, 3)]:
        r = oracle_mod.oracle_one_off(test_tree, test_table, "unweighted_fp64", stripe_start=start, stripe_stop=stop)
        np.testing.assert_allclose(r["stripes"], exp[start:stop], atol=1e-6, rtol=0)


def test_oracle_status_codes(oracle_mod, test_tree, test_table):
    with pytest.raises(oracle_mod.OracleError, match="status 4"):
        oracle_mod.oracle_one_off(test_tree, test_table, "not_a_method")
    import ssu_synth
    other = ssu_synth.parse_newick("(a:1,b:2)r;")
    with pytest.raises(oracle_mod.OracleError, match="status 5"):
        oracle_mod.oracle_one_off(other, test_table, "unweighted_fp64")


def test_golden_sample_totals(golden, test_table):
    exp = golden["test_su"]["test_unifrac_sample_counts"]["arrays"]["exp"][0]
    dense = test_table.dense()
    np.testing.assert_array_equal(dense.sum(axis=0), exp)


def test_rarefaction_generator_properties():
    """The host rarefaction that feeds the batched-replicate workload: every
    kept sample sums to the depth, no count grows, lighter samples and
    emptied features are dropped (src/biom_subsampled.cpp:287-353)."""
    import numpy as np
    tree = ssu_synth.random_binary_tree(300, 0.1, 1)
    base = ssu_synth.negbin_table(tree.tip_names(), 80, 0.2, 50.0, 0.5, 2)
    depth = 150
    r = ssu_synth.rarefy(base, depth, 3)
    bd = base.dense()
    keep = np.flatnonzero(bd.sum(axis=0) >= depth)
    assert r.sample_ids == [base.sample_ids[j] for j in keep]
    d = r.dense()
    rows = [base.obs_ids.index(o) for o in r.obs_ids]
    assert np.all(d <= bd[rows][:, keep])
    assert np.all(d.sum(axis=0) == depth)
    assert np.all(d.sum(axis=1) > 0)
    again = ssu_synth.rarefy(base, depth, 3)
    np.testing.assert_array_equal(again.dense(), d)

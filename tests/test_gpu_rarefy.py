"""Rarefied replicates drawn on the GPU (ssu_b200_rarefy_batch), held to the
properties the reference's subsampling tests check (src/test_ska.cpp:639-917:
which samples survive a depth, every kept column summing to the depth, the
n = total - 1 limit, more than 10 distinct draws over 1000 replicates with
replacement) plus: no count grows without replacement, replicate r does not
depend on how many replicates are drawn with it, the seed changes the draws,
the expected counts match the sampling design, and the replicate-batch entry
point computes exactly what one call per drawn table computes."""
import numpy as np
import pytest

import ssu_synth
from conftest import rel_err

pytestmark = pytest.mark.gpu


def column_sums(t):
    return t.dense().sum(axis=0)


@pytest.mark.parametrize("with_replacement", [False, True])
def test_reference_unit_table_depths(ssu, test_table, with_replacement):
    """src/test_ska.cpp:639-700 and 765-830 on test.biom."""
    for t in ssu.rarefy_batch(test_table, 5, 5, with_replacement):
        assert t.sample_ids == ["Sample1", "Sample4"]
        assert t.n_obs <= 3 and set(t.obs_ids) <= {"GG_OTU_2", "GG_OTU_3", "GG_OTU_4"}
        np.testing.assert_array_equal(column_sums(t), [5.0, 5.0])
    empty = ssu.rarefy_batch(test_table, 2, 8, with_replacement)
    assert all(t.n_samples == 0 and t.n_obs == 0 for t in empty)


def limit_table():
    """src/test_ska.cpp:702-712: one sample of 35 counts over ten observations."""
    ids = [f"OTU{i}" for i in range(10)]
    data = np.array([2., 1., 2., 1., 7., 6., 3., 3., 5., 5.])
    return ssu_synth.Table(ids, ["S1"], np.arange(11, dtype=np.uint32), np.zeros(10, np.uint32), data)


@pytest.mark.parametrize("with_replacement", [False, True])
def test_depth_one_below_the_total(ssu, with_replacement):
    base = limit_table()
    reps = ssu.rarefy_batch(base, 1000, 34, with_replacement)
    orig = dict(zip(base.obs_ids, base.data))
    patterns = set()
    for t in reps:
        assert t.n_samples == 1 and t.n_obs <= 10
        assert column_sums(t)[0] == 34.0
        got = dict(zip(t.obs_ids, t.dense()[:, 0]))
        if not with_replacement:
            assert all(v <= orig[k] for k, v in got.items())
            assert sum(orig[k] - got.get(k, 0.0) for k in orig) == 1.0  # exactly one unit left out
        patterns.add(tuple(got.get(k, 0.0) for k in base.obs_ids))
    # src/test_ska.cpp:742-760 asks for more than 10 distinct outcomes with replacement;
    # without replacement there are exactly 10 (which observation loses its unit)
    assert len(patterns) > 10 if with_replacement else len(patterns) == 10


def test_counts_follow_the_sampling_design(ssu):
    """Without replacement the expected count of an observation is
    depth * count / total; with replacement the same, from the weights."""
    tree = ssu_synth.random_binary_tree(300, 0.1, 3)
    base = ssu_synth.negbin_table(tree.tip_names(), 40, 0.2, 30.0, 0.5, 4)
    depth = int(np.percentile(column_sums(base), 30))
    dense = base.dense()
    keep = np.where(column_sums(base) >= depth)[0]
    for with_replacement in (False, True):
        reps = ssu.rarefy_batch(base, 400, depth, with_replacement)
        acc = np.zeros((base.n_obs, len(keep)))
        pos = {o: i for i, o in enumerate(base.obs_ids)}
        for t in reps:
            assert t.sample_ids == [base.sample_ids[j] for j in keep]
            np.testing.assert_array_equal(column_sums(t), np.full(len(keep), float(depth)))
            d = t.dense()
            if not with_replacement:
                rows = [pos[o] for o in t.obs_ids]
                assert np.all(d <= dense[rows][:, keep])
            for i, o in enumerate(t.obs_ids):
                acc[pos[o]] += d[i]
        mean = acc / len(reps)
        expect = dense[:, keep] * depth / dense[:, keep].sum(axis=0)
        big = expect > 5
        # standard error of a mean over 400 draws of a count of mean <= depth
        assert np.all(np.abs(mean[big] - expect[big]) <= 5 * np.sqrt(expect[big] / len(reps)) + 0.05)


def test_replicates_are_reproducible_and_seeded(ssu):
    tree = ssu_synth.random_binary_tree(200, 0.1, 8)
    base = ssu_synth.negbin_table(tree.tip_names(), 30, 0.2, 20.0, 0.5, 9)
    depth = int(np.median(column_sums(base)))
    ssu.lib().ssu_set_random_seed(123)
    a = ssu.rarefy_batch(base, 6, depth)
    b = ssu.rarefy_batch(base, 2, depth)
    for x, y in zip(a[:2], b):  # replicate r is the same whatever the batch size
        assert x.obs_ids == y.obs_ids
        np.testing.assert_array_equal(x.dense(), y.dense())
    ssu.lib().ssu_set_random_seed(124)
    c = ssu.rarefy_batch(base, 1, depth)
    assert not np.array_equal(a[0].dense(), c[0].dense())
    assert not np.array_equal(a[0].dense(), a[1].dense())
    # replicate r of seed s is replicate 0 of seed s + r
    assert c[0].obs_ids == a[1].obs_ids
    np.testing.assert_array_equal(c[0].dense(), a[1].dense())
    ssu.lib().ssu_set_random_seed(5489)


@pytest.mark.parametrize("method", ["unweighted_fp32", "weighted_normalized_fp32", "unweighted_fp64"])
def test_replicate_batch_equals_one_call_per_drawn_table(ssu, method):
    """ssu_b200_subsample_batch_*: the same draws as ssu_b200_rarefy_batch
    (same seed), each replicate's matrix equal to one_off_matrix on it."""
    tree = ssu_synth.random_binary_tree(500, 0.1, 11)
    base = ssu_synth.negbin_table(tree.tip_names(), 120, 0.05, 30.0, 0.5, 12)
    depth = int(np.percentile(column_sums(base), 25))
    ssu.lib().ssu_set_random_seed(77)
    drawn = ssu.rarefy_batch(base, 5, depth)
    ssu.lib().ssu_set_random_seed(77)
    mats = ssu.subsample_batch(tree, base, method, 5, depth)
    for (m, ids), t in zip(mats, drawn):
        assert ids == t.sample_ids
        single, _ = ssu.one_off_matrix(tree, t, method)
        r, z = rel_err(m, single)
        assert r <= (1e-12 if method.endswith("fp64") else 1e-6) and z <= 1e-6, (r, z)

"""Batches of tables sharing one tree (one device plan, one persistent pair
launch per group of tables): every table's result must equal the oracle's
one-table result on that table, whatever the grouping, tile shape or
graph mode.

Bars as the one-table tests: fp64 within 1e-12 relative of the oracle (1e-13
absolute at zeros); fp32 within 4x the reference fp32 build's own error,
floored at 1e-6."""
import numpy as np
import pytest

import ssu_synth
from conftest import rel_err

pytestmark = pytest.mark.gpu

METHODS = ["unweighted", "unweighted_unnormalized", "weighted_normalized", "weighted_unnormalized", "generalized"]
FP64_REL = 1e-12
FP64_ABS = 1e-13


def _uneven_batch(seed, n_tips=120, sizes=(5, 130, 37, 3, 64, 200, 2), density=0.15):
    """Tables of uneven sample counts over different subsets of the tree's
    tips (so each table's own sheared tree differs from the shared one)."""
    tree = ssu_synth.random_binary_tree(n_tips, 0.1, seed)
    tips = tree.tip_names()
    rng = np.random.default_rng(seed + 7)
    tables = []
    for i, n in enumerate(sizes):
        lo = int(rng.integers(0, n_tips // 3))
        hi = int(rng.integers(2 * n_tips // 3, n_tips + 1))
        t = ssu_synth.geometric_table(tips[lo:hi], n, density, 8.0, seed + 100 + i)
        # every sample keeps at least one count
        dense = t.dense()
        empty = np.flatnonzero(dense.sum(axis=0) == 0)
        dense[0, empty] = 3.0
        flat = np.flatnonzero(dense.ravel() > 0)
        t = ssu_synth.make_table(t.obs_ids, n, flat, dense.ravel()[flat], sample_prefix=f"B{i}_")
        tables.append(t)
    return tree, tables


def check_fp64(gpu, ref):
    r, z = rel_err(gpu, ref)
    assert r <= FP64_REL, f"max rel err {r:.3e}"
    assert z <= FP64_ABS, f"max abs err at zeros {z:.3e}"


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("vaw", [False, True])
@pytest.mark.parametrize("bypass", [False, True])
def test_batch_fp64_matches_oracle_per_table(ssu, oracle_mod, method, vaw, bypass):
    tree, tables = _uneven_batch(11)
    kw = dict(variance_adjust=vaw, bypass_tips=bypass, alpha=0.5)
    out = ssu.one_off_batch(tree, tables, method + "_fp64", **kw)
    assert len(out) == len(tables)
    for (gpu, ids), t in zip(out, tables):
        assert ids == t.sample_ids
        ref = oracle_mod.oracle_one_off(tree, t, method + "_fp64", **kw)["matrix"]
        assert np.array_equal(np.isnan(gpu), np.isnan(ref))
        check_fp64(gpu, ref)
        assert np.all(np.diag(gpu) == 0)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("bypass", [False, True])
def test_batch_fp32_within_reference_fp32_error(ssu, oracle_mod, method, bypass):
    """fp32 unweighted batches run on the tensor cores (with bypassed tips,
    on the presence-word stripe kernel)."""
    tree, tables = _uneven_batch(12)
    out = ssu.one_off_batch(tree, tables, method + "_fp32", alpha=0.5, bypass_tips=bypass)
    for (gpu, _), t in zip(out, tables):
        assert gpu.dtype == np.float32
        o64 = oracle_mod.oracle_one_off(tree, t, method + "_fp64", alpha=0.5, bypass_tips=bypass)["matrix"]
        o32 = oracle_mod.oracle_one_off(tree, t, method + "_fp32", alpha=0.5, bypass_tips=bypass)["matrix"]
        ref_err, ref_zero = rel_err(o32, o64)
        ours, ours_zero = rel_err(gpu, o64)
        assert ours <= max(4 * ref_err, 1e-6), (ours, ref_err)
        assert ours_zero <= max(4 * ref_zero, 1e-6)


@pytest.mark.parametrize("alpha", [0.0, 0.25, 1.0])
def test_batch_generalized_alphas(ssu, oracle_mod, alpha):
    tree, tables = _uneven_batch(13, sizes=(40, 3, 129))
    for vaw in (False, True):
        out = ssu.one_off_batch(tree, tables, "generalized_fp64", variance_adjust=vaw, alpha=alpha)
        for (gpu, _), t in zip(out, tables):
            check_fp64(gpu, oracle_mod.oracle_one_off(tree, t, "generalized_fp64", variance_adjust=vaw,
                                                      alpha=alpha)["matrix"])


@pytest.mark.parametrize("bypass", [False, True])
def test_batch_embedded_counts_match_each_tables_own_tree(ssu, oracle_mod, bypass):
    tree, tables = _uneven_batch(14)
    plan = ssu.BatchPlan(tree, tables, "weighted_normalized_fp64", bypass_tips=bypass)
    units = 0
    for i, t in enumerate(tables):
        e = oracle_mod.oracle_one_off(tree, t, "weighted_normalized_fp64", bypass_tips=bypass)["n_embedded"]
        assert plan.table_embedded(i) == e
        units += t.n_samples * (t.n_samples - 1) // 2 * e
    assert plan.work_units() == units
    plan.close()


@pytest.mark.parametrize("method", ["weighted_normalized_fp64", "unweighted_fp32", "generalized_fp64"])
def test_groups_tiles_and_graph_do_not_change_results(ssu, method):
    tree, tables = _uneven_batch(15)
    one = ssu.BatchPlan(tree, tables, method, alpha=0.5, autotune=0)
    one.execute()
    ref = one.results()
    assert one.n_groups() == 1
    one.close()
    # a one-byte budget puts every table in a group of its own
    many = ssu.BatchPlan(tree, tables, method, alpha=0.5, group_bytes=1, autotune=1)
    assert many.n_groups() == len(tables)
    many.set_graph(True)
    for _ in range(2):
        many.execute()
        got = many.results()
        for a, b in zip(got, ref):
            if method.endswith("fp64"):
                check_fp64(a, b)
            else:
                np.testing.assert_allclose(a, b, rtol=2e-6, atol=1e-7)
    assert many.tuning()
    many.close()


def test_subsample_batch_replicates_match_single_calls(ssu):
    tree = ssu_synth.random_binary_tree(150, 0.1, 16)
    base = ssu_synth.negbin_table(tree.tip_names(), 60, 0.2, 30.0, 0.5, 17)
    lib = ssu.lib()
    lib.ssu_set_random_seed(1234)
    reps = ssu.subsample_batch(tree, base, "weighted_normalized_fp64", 4, 200)
    for r, (m, ids) in enumerate(reps):
        lib.ssu_set_random_seed(1234 + r)
        single, sids = ssu.one_off_matrix(tree, base, "weighted_normalized_fp64", subsample_depth=200)
        assert ids == sids
        check_fp64(m, single)
    lib.ssu_set_random_seed(5489)


def test_unweighted_fp32_defaults_to_tensor_cores(ssu, monkeypatch):
    tree, tables = _uneven_batch(19, sizes=(70, 150))
    plan = ssu.BatchPlan(tree, tables, "unweighted_fp32")
    assert plan.pair_kernel() == "unweighted_tc_kernel"
    plan.close()
    single = ssu.Plan(tree, tables[0], "unweighted_fp32")
    assert single.pair_kernel() == "unweighted_tc_kernel"
    single.close()
    monkeypatch.setenv("UNIFRAC_B200_UNWEIGHTED_MODE", "stripe")
    single = ssu.Plan(tree, tables[0], "unweighted_fp32")
    assert single.pair_kernel().startswith("pair_bits")
    single.close()
    plan = ssu.BatchPlan(tree, tables, "unweighted_fp32", bypass_tips=True)
    monkeypatch.delenv("UNIFRAC_B200_UNWEIGHTED_MODE")
    assert plan.pair_kernel().startswith("pair_bits")
    plan.close()


def test_batch_fp32_subsample_and_status_codes(ssu):
    tree, tables = _uneven_batch(18, sizes=(20, 30))
    reps = ssu.subsample_batch(tree, tables[0], "unweighted", 3, 5)
    assert len(reps) == 3 and all(m.dtype == np.float32 for m, _ in reps)
    with pytest.raises(ssu.SSUError) as e:
        ssu.one_off_batch(tree, tables, "weighted_normalized_fp32_typo")
    assert e.value.status == 4  # unknown_method
    bad = ssu_synth.make_table(["nope"], 2, np.array([0, 1]), np.array([1.0, 2.0]))
    with pytest.raises(ssu.SSUError) as e:
        ssu.one_off_batch(tree, [tables[0], bad], "weighted_normalized_fp64")
    assert e.value.status == 5  # table_and_tree_do_not_overlap

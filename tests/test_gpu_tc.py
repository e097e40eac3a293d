"""The tensor-core (tcgen05) unweighted contraction, selected with
UNIFRAC_B200_UNWEIGHTED_MODE=gemm, against the fp64 oracle.  Bar: max
relative error 1e-6 on every pair (the contraction's stated bound; lengths
carried as 23-bit fixed point per chunk of lengths within a factor of two,
each written as 256 u v + s t with 8-bit digits, exact int32 sums of the
two products, fp64 across chunks and in the final ratio)."""
import os

import numpy as np
import pytest

import ssu_synth
from conftest import rel_err

pytestmark = pytest.mark.gpu
TC_REL = 1e-6


@pytest.fixture
def gemm_mode():
    old = os.environ.get("UNIFRAC_B200_UNWEIGHTED_MODE")
    os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"] = "gemm"
    yield
    if old is None:
        del os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"]
    else:
        os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"] = old


def _case(seed, n_tips, n_samples, density=0.1):
    tree = ssu_synth.random_binary_tree(n_tips, 0.05, seed)
    table = ssu_synth.geometric_table(tree.tip_names()[: n_tips - 3], n_samples, density, 6.0, seed + 9)
    return tree, table


@pytest.mark.parametrize("n_samples,n_tips", [(5, 40), (37, 200), (130, 700), (300, 1500)])
@pytest.mark.parametrize("method", ["unweighted_fp64", "unweighted_unnormalized_fp64", "unweighted"])
def test_tc_matches_oracle(ssu, oracle_mod, gemm_mode, n_samples, n_tips, method):
    tree, table = _case(n_samples + n_tips, n_tips, n_samples)
    plan = ssu.Plan(tree, table, method)
    assert plan.pair_kernel() == "unweighted_tc_kernel"
    plan.close()
    gpu, _ = ssu.one_off_matrix(tree, table, method)
    ref = oracle_mod.oracle_one_off(tree, table, method.replace("_fp64", "") + "_fp64")["matrix"]
    r, z = rel_err(gpu, ref)
    assert r <= TC_REL and z <= 1e-9, (r, z)
    assert np.all(np.diag(gpu) == 0)


def test_tc_bypass_and_windows(ssu, oracle_mod, gemm_mode):
    tree, table = _case(7, 900, 200)
    gpu, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64", bypass_tips=True)
    ref = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64", bypass_tips=True)["matrix"]
    assert rel_err(gpu, ref)[0] <= TC_REL
    stripes, _ = ssu.partial(tree, table, "unweighted_fp64", 20, 60)
    ref = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64", stripe_start=20, stripe_stop=60)["stripes"]
    assert rel_err(stripes, ref)[0] <= TC_REL
    cf, _, _ = ssu.one_off(tree, table, "unweighted_fp64")
    full = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64")["matrix"]
    assert rel_err(cf, full[np.triu_indices(200, 1)])[0] <= TC_REL


def test_tc_wide_length_range(ssu, oracle_mod, gemm_mode):
    """Branch lengths over 12 orders of magnitude exercise the per-chunk scales."""
    tree, table = _case(8, 600, 90, density=0.2)
    rng = np.random.default_rng(3)
    tree.lengths = np.where(tree.structure, 10.0 ** rng.uniform(-9, 3, size=tree.lengths.shape), 0.0)
    gpu, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64")
    ref = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64")["matrix"]
    assert rel_err(gpu, ref)[0] <= TC_REL


def test_tc_chunk_closes_at_its_block_limit(ssu, oracle_mod, gemm_mode):
    """80,000 embedded nodes whose lengths lie within a factor of two fill one
    chunk past its limit of 512 blocks of 128 nodes (the int32 product sums'
    bound), so the contraction runs over two chunks of the same scale."""
    tree, table = _case(12, 40000, 48, density=0.3)
    rng = np.random.default_rng(12)
    tree.lengths = np.where(tree.structure, rng.uniform(1.0, 1.9, size=tree.lengths.shape), 0.0)
    gpu, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64")
    ref = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64")["matrix"]
    assert rel_err(gpu, ref)[0] <= TC_REL


def test_tc_plan_agrees_with_stripe_form(ssu, gemm_mode):
    tree, table = _case(9, 2000, 400)
    plan = ssu.Plan(tree, table, "unweighted_fp64")
    plan.execute()
    tc = plan.result()
    plan.close()
    os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"] = "stripe"
    stripe, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64")
    assert rel_err(tc, stripe)[0] <= TC_REL


@pytest.mark.parametrize("n_samples", [2, 63, 64, 65, 127, 128, 129, 255, 256, 257, 319, 383, 385, 511, 513])
@pytest.mark.parametrize("method", ["unweighted_fp64", "unweighted_unnormalized_fp64"])
def test_tc_sample_counts_at_work_unit_edges(ssu, oracle_mod, gemm_mode, n_samples, method):
    """A work unit covers 256 rows x 128 columns: counts around those edges,
    where units straddle the diagonal or hold a single row or column."""
    tree, table = _case(n_samples, 300, n_samples, density=0.08)
    gpu, _ = ssu.one_off_matrix(tree, table, method)
    ref = oracle_mod.oracle_one_off(tree, table, method)["matrix"]
    r, z = rel_err(gpu, ref)
    assert r <= TC_REL and z <= 1e-9, (r, z)


def test_tc_close_and_identical_samples(ssu, oracle_mod, gemm_mode):
    """Samples equal to another one, or differing from it by one short tip:
    the xor sum is small next to the samples' own lengths, where a contraction
    of the shared length (r_k + r_l - 2 X L X^T) would cancel."""
    tree, table = _case(21, 800, 60, density=0.15)
    dense = table.dense()
    lengths = dict(zip(tree.tip_names(), tree.tip_lengths()))
    obs = list(table.obs_ids)
    shortest = min(range(len(obs)), key=lambda i: lengths.get(obs[i], 1e9))
    for j in range(0, 30, 2):
        dense[:, j + 1] = dense[:, j]
        if j % 4 == 0:
            dense[shortest, j + 1] = 0.0 if dense[shortest, j] > 0 else 3.0
    table = ssu_synth.Table.from_dense(dense, obs, table.sample_ids)
    for method in ("unweighted_fp64", "unweighted_unnormalized_fp64"):
        gpu, _ = ssu.one_off_matrix(tree, table, method)
        ref = oracle_mod.oracle_one_off(tree, table, method)["matrix"]
        r, z = rel_err(gpu, ref)
        assert r <= TC_REL and z <= 1e-12, (method, r, z)


def test_tc_wait_that_runs_out_is_an_error_and_the_device_stays_usable(ssu, oracle_mod, gemm_mode, monkeypatch):
    """Failure injection without a fault: with UNIFRAC_B200_TEST_STALL the
    tensor-core kernel's producers issue no copy, so the MMA issuer's and the
    epilogues' bounded waits (here ~1 ms) run out; the call returns
    output_error instead of hanging, and the next call is correct."""
    tree, table = _case(31, 300, 300)
    monkeypatch.setenv("UNIFRAC_B200_TEST_STALL", "1")
    monkeypatch.setenv("UNIFRAC_B200_WAIT_CYCLES", "2000000")
    with pytest.raises(ssu.SSUError) as e:
        ssu.one_off_matrix(tree, table, "unweighted_fp64")
    assert e.value.status == 6  # output_error
    monkeypatch.delenv("UNIFRAC_B200_TEST_STALL")
    monkeypatch.delenv("UNIFRAC_B200_WAIT_CYCLES")
    gpu, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64")
    ref = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64")["matrix"]
    assert rel_err(gpu, ref)[0] <= TC_REL


def test_tc_negative_lengths_keep_the_stripe_form(ssu, oracle_mod, gemm_mode):
    """Lengths are fixed-point magnitudes on the tensor cores: a tree with a
    negative branch length runs on the stripe form instead, and still
    matches the oracle."""
    tree, table = _case(31, 400, 70, density=0.15)
    lengths = tree.lengths.copy()
    lengths[np.flatnonzero(tree.structure)[5]] = -0.01
    tree.lengths = lengths
    gpu, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64")
    ref = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64")["matrix"]
    r, z = rel_err(gpu, ref)
    assert r <= 1e-12 and z <= 1e-13, (r, z)


def test_tc_band_tuning_changes_no_result(ssu):
    """Batch plans time the band height of the unit order (2, 4 or 8 row
    blocks) and keep the fastest; the order changes no result, bit for bit."""
    tree = ssu_synth.random_binary_tree(900, 0.05, 41)
    tables = [ssu_synth.geometric_table(tree.tip_names()[:850], n, 0.08, 6.0, 42 + n) for n in (700, 1100)]
    method = "unweighted"  # fp32 results: the tensor-core form by default
    fixed = ssu.BatchPlan(tree, tables, method, autotune=0)
    fixed.execute()
    ref = fixed.results()
    assert "band 4" in fixed.tuning()
    fixed.close()
    tuned = ssu.BatchPlan(tree, tables, method, autotune=1)
    assert "band" in tuned.tuning() and ("measured" in tuned.tuning() or "cache" in tuned.tuning())
    tuned.execute()
    for a, b in zip(tuned.results(), ref):
        np.testing.assert_array_equal(a, b)
    tuned.close()


@pytest.mark.parametrize("band", ["1", "4"])
def test_tc_copy_out_alongside_computation_covers_the_matrix(ssu, gemm_mode, monkeypatch, band):
    """A full result of one table in page-locked memory is copied out band by
    band of rows while later bands compute.  Bands of 256 and 1,024 rows over
    2,300 samples, the last band short: the copied matrix is the plan's own
    result bit for bit, diagonal included."""
    monkeypatch.setenv("UNIFRAC_B200_TC_BAND", band)
    tree, table = _case(14, 1200, 2300, density=0.05)
    full, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64")
    plan = ssu.Plan(tree, table, "unweighted_fp64")
    plan.execute()
    ref = plan.result()
    plan.close()
    np.testing.assert_array_equal(full, ref)
    assert np.all(np.diag(full) == 0.0)

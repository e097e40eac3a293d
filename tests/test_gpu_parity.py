"""Parity of the CUDA path (through the C ABI of libssu_b200.so) with the
oracle, on seeded inputs.

Bars: fp64 methods within 1e-12 relative of the oracle (1e-13 absolute where
the oracle value is 0); fp32 methods within 4x the reference fp32 build's own
error against fp64 on the same input (measured with the oracle's fp32 mode),
floored at 1e-6; NaN patterns identical."""
import numpy as np
import pytest

import ssu_synth
from conftest import matrix_from_stripes, rel_err, stripes_from_golden

pytestmark = pytest.mark.gpu

METHODS = ["unweighted", "unweighted_unnormalized", "weighted_normalized", "weighted_unnormalized", "generalized"]
FP64_REL = 1e-12
FP64_ABS = 1e-13


def _case(seed, n_tips=90, n_samples=37, density=0.12, drop=7):
    tree = ssu_synth.random_binary_tree(n_tips, 0.1, seed)
    table = ssu_synth.geometric_table(tree.tip_names()[: n_tips - drop], n_samples, density, 10.0, seed + 3)
    return tree, table


def check_fp64(gpu, ref):
    r, z = rel_err(gpu, ref)
    assert r <= FP64_REL, f"max rel err {r:.3e}"
    assert z <= FP64_ABS, f"max abs err at zeros {z:.3e}"


def check_fp32(gpu32, oracle, tree, table, method, **kw):
    o64 = oracle.oracle_one_off(tree, table, method + "_fp64", **kw)["matrix"]
    o32 = oracle.oracle_one_off(tree, table, method + "_fp32", **kw)["matrix"]
    ref_err, ref_zero = rel_err(o32, o64)
    ours, ours_zero = rel_err(gpu32, o64)
    assert ours <= max(4 * ref_err, 1e-6), (ours, ref_err)
    assert ours_zero <= max(4 * ref_zero, 1e-6)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("vaw", [False, True])
@pytest.mark.parametrize("bypass", [False, True])
def test_fp64_matches_oracle(ssu, oracle_mod, method, vaw, bypass):
    tree, table = _case(21)
    kw = dict(variance_adjust=vaw, bypass_tips=bypass, alpha=0.5)
    gpu, ids = ssu.one_off_matrix(tree, table, method + "_fp64", **kw)
    assert ids == table.sample_ids
    check_fp64(gpu, oracle_mod.oracle_one_off(tree, table, method + "_fp64", **kw)["matrix"])


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("vaw", [False, True])
def test_fp32_within_reference_fp32_error(ssu, oracle_mod, method, vaw):
    tree, table = _case(22)
    kw = dict(variance_adjust=vaw, alpha=0.5)
    gpu, _ = ssu.one_off_matrix(tree, table, method + "_fp32", **kw)
    assert gpu.dtype == np.float32
    check_fp32(gpu, oracle_mod, tree, table, method, **kw)


@pytest.mark.parametrize("alpha", [0.0, 0.25, 0.5, 1.0, 1.5])
def test_generalized_alphas(ssu, oracle_mod, alpha):
    tree, table = _case(23)
    for vaw in (False, True):
        gpu, _ = ssu.one_off_matrix(tree, table, "generalized_fp64", variance_adjust=vaw, alpha=alpha)
        check_fp64(gpu, oracle_mod.oracle_one_off(tree, table, "generalized_fp64", variance_adjust=vaw,
                                                  alpha=alpha)["matrix"])


@pytest.mark.parametrize("n", [2, 3, 5, 63, 64, 65, 127, 128, 129, 200, 255, 256, 257])
@pytest.mark.parametrize("method", ["unweighted_fp64", "weighted_normalized_fp64", "generalized_fp64"])
def test_tile_boundaries(ssu, oracle_mod, n, method):
    tree, table = _case(100 + n, n_tips=70, n_samples=n, density=0.2, drop=0)
    gpu, _ = ssu.one_off_matrix(tree, table, method, alpha=0.5)
    check_fp64(gpu, oracle_mod.oracle_one_off(tree, table, method, alpha=0.5)["matrix"])
    assert np.all(np.diag(gpu) == 0)
    np.testing.assert_array_equal(gpu, gpu.T)


GOLDEN_CASES = [
    ("test_unweighted_unifrac", "", "unweighted_fp64", {}),
    ("test_unweighted_unifrac", "", "unweighted_fp32", {}),
    ("test_unweighted_unifrac_fast", "", "unweighted_fp64", {"bypass_tips": True}),
    ("test_unnormalized_unweighted_unifrac", "", "unweighted_unnormalized_fp64", {}),
    ("test_unnormalized_weighted_unifrac", "", "weighted_unnormalized_fp64", {}),
    ("test_normalized_weighted_unifrac", "", "weighted_normalized_fp64", {}),
    ("test_normalized_weighted_unifrac", "", "weighted_normalized_fp32", {}),
    ("test_generalized_unifrac", "w_", "generalized_fp64", {"alpha": 1.0}),
    ("test_generalized_unifrac", "d0_", "generalized_fp64", {"alpha": 0.0}),
    ("test_generalized_unifrac", "d05_", "generalized_fp64", {"alpha": 0.5}),
    ("test_vaw_unifrac_weighted_normalized", "w_", "weighted_normalized_fp64", {"variance_adjust": True}),
]


@pytest.mark.parametrize("func,prefix,method,kw", GOLDEN_CASES)
def test_reference_goldens_through_c_abi(ssu, golden, test_tree, test_table, func, prefix, method, kw):
    exp = stripes_from_golden(golden["test_su"][func], prefix)
    gpu, _ = ssu.one_off_matrix(test_tree, test_table, method, **kw)
    np.testing.assert_allclose(gpu, matrix_from_stripes(exp, 6), atol=1e-6, rtol=0)
    stripes, meta = ssu.partial(test_tree, test_table, method, 0, 3, **kw)
    np.testing.assert_allclose(stripes, exp, atol=1e-6, rtol=0)
    assert meta["total"] == 3 and meta["upper"]


def test_faith_goldens_through_c_abi(ssu, golden, test_table):
    exp = golden["test_su"]["test_faith_pd"]["arrays"]["exp"][0]
    for tre in ("test_faith.tre", "test_faith_shear.tre"):
        tree = ssu_synth.parse_newick(golden["trees"][tre])
        vals, ids = ssu.faith_pd(tree, test_table)
        np.testing.assert_allclose(vals, exp, atol=1e-6, rtol=0)
        assert ids == test_table.sample_ids


@pytest.mark.parametrize("n", [6, 7, 40, 41, 300])
def test_partial_windows_and_condensed(ssu, oracle_mod, n):
    tree, table = _case(40 + n, n_tips=80, n_samples=n, density=0.2, drop=0)
    method = "weighted_normalized_fp64"
    s_total = (n + 1) // 2
    windows = [(0, s_total), (0, 1), (s_total - 1, s_total), (s_total // 3, max(s_total // 3 + 1, 2 * s_total // 3))]
    for start, stop in windows:
        gpu, meta = ssu.partial(tree, table, method, start, stop)
        ref = oracle_mod.oracle_one_off(tree, table, method, stripe_start=start, stripe_stop=stop)["stripes"]
        check_fp64(gpu, ref)
        assert (meta["start"], meta["stop"], meta["total"]) == (start, stop, s_total)
    cf, ids, upper = ssu.one_off(tree, table, method)
    full = oracle_mod.oracle_one_off(tree, table, method)["matrix"]
    iu = np.triu_indices(n, 1)
    check_fp64(cf, full[iu])
    assert upper and len(cf) == n * (n - 1) // 2


def test_partial_out_of_range_is_an_error_not_an_exit(ssu, test_tree, test_table):
    with pytest.raises(ssu.SSUError) as e:
        ssu.partial(test_tree, test_table, "unweighted_fp64", 0, 4)
    assert e.value.status == 6


def test_faith_filters_empty_samples(ssu, oracle_mod):
    tree, table = _case(51, n_samples=30)
    dense = table.dense()
    dense[:, [0, 7]] = 0
    flat = np.flatnonzero(dense.ravel() > 0)
    t2 = ssu_synth.make_table(table.obs_ids, table.n_samples, flat, dense.ravel()[flat])
    vals, ids = ssu.faith_pd(tree, t2)
    ref = oracle_mod.oracle_faith_pd(tree, t2)
    assert ids == [t2.sample_ids[i] for i in ref["kept"]]
    np.testing.assert_allclose(vals, ref["values"], rtol=1e-12, atol=0)


def test_empty_samples_give_reference_nan_pattern(ssu, oracle_mod):
    tree, table = _case(52, n_samples=20)
    dense = table.dense()
    dense[:, [3, 4]] = 0
    flat = np.flatnonzero(dense.ravel() > 0)
    t2 = ssu_synth.make_table(table.obs_ids, table.n_samples, flat, dense.ravel()[flat])
    for m in METHODS:
        gpu, _ = ssu.one_off_matrix(tree, t2, m + "_fp64", alpha=0.5)
        ref = oracle_mod.oracle_one_off(tree, t2, m + "_fp64", alpha=0.5)["matrix"]
        assert np.array_equal(np.isnan(gpu), np.isnan(ref)), m
        check_fp64(gpu, ref)


def test_dense_pair(ssu, golden, oracle_mod):
    tree = ssu_synth.parse_newick(golden["trees"]["test.tre"])
    obs = ["GG_OTU_1", "GG_OTU_2", "GG_OTU_3", "GG_OTU_4", "GG_OTU_5"]
    s1, s3 = [0, 5, 0, 2, 0], [1, 0, 1, 1, 1]
    d = ssu.dense_pair(tree, obs, s1, s3, "unweighted_fp64")
    flat = [i * 2 + j for i in range(5) for j, v in enumerate((s1[i], s3[i])) if v > 0]
    vals = [(s1, s3)[f % 2][f // 2] for f in flat]
    t = ssu_synth.make_table(obs, 2, np.array(flat), np.array(vals, dtype=float))
    exp = oracle_mod.oracle_one_off(tree, t, "unweighted_fp64")["matrix"][0, 1]
    assert abs(d - exp) <= 1e-12 * abs(exp)
    d32 = ssu.dense_pair(tree, obs, s1, s3, "unweighted")
    assert abs(d32 - 0.57142857) < 1e-6  # test/capi_inmem_test.c exp13


def test_unnormalized_sample_counts(ssu, oracle_mod):
    tree, table = _case(53)
    for m in ("weighted_unnormalized_fp64", "weighted_normalized_fp64", "generalized_fp64"):
        gpu, _ = ssu.one_off_matrix(tree, table, m, normalize=False, alpha=0.5)
        check_fp64(gpu, oracle_mod.oracle_one_off(tree, table, m, normalize=False, alpha=0.5)["matrix"])


def test_plan_api_matches_one_off(ssu):
    tree, table = _case(54, n_samples=150)
    for m in ("weighted_normalized_fp64", "unweighted_fp32"):
        plan = ssu.Plan(tree, table, m)
        plan.set_timing(True)
        plan.execute()
        out = plan.result()
        e, p, f = plan.stage_ms()
        assert p > 0 and e >= 0
        ref, _ = ssu.one_off_matrix(tree, table, m)
        np.testing.assert_array_equal(out, ref)
        assert plan.work_units() == 150 * 149 // 2 * plan.n_embedded()
        assert plan.launches() >= 2
        plan.close()


def test_mmap_backed_result(ssu, tmp_path):
    tree, table = _case(55)
    a, _ = ssu.one_off_matrix(tree, table, "weighted_unnormalized_fp64", mmap_dir=str(tmp_path))
    b, _ = ssu.one_off_matrix(tree, table, "weighted_unnormalized_fp64")
    np.testing.assert_array_equal(a, b)


def test_rarefaction_keeps_deep_samples(ssu):
    tree, table = _case(56, n_samples=25, density=0.5)
    totals = table.dense().sum(axis=0)
    depth = int(np.percentile(totals, 40))
    ssu.lib().ssu_set_random_seed(7)
    m, ids = ssu.one_off_matrix(tree, table, "unweighted_fp64", subsample_depth=depth)
    keep = [table.sample_ids[j] for j in range(table.n_samples) if totals[j] >= depth]
    assert ids == keep
    assert m.shape == (len(keep), len(keep))
    assert np.all(np.isfinite(m))


def test_20k_tips_2048_samples_full_size_stripe_windows(ssu, oracle_mod):
    """Full 20,000-tip x 2,048-sample input: the GPU matrix against
    the oracle on the first and last stripes, plus matrix properties."""
    tree, table = ssu_synth.lognormal_20k_tips_2048_samples()
    n = table.n_samples
    s_total = (n + 1) // 2
    for m in ("weighted_normalized_fp64", "weighted_unnormalized_fp64"):
        gpu, _ = ssu.one_off_matrix(tree, table, m)
        assert np.all(np.diag(gpu) == 0)
        np.testing.assert_array_equal(gpu, gpu.T)
        assert np.all(np.isfinite(gpu))
        for start, stop in [(0, 2), (s_total - 2, s_total)]:
            ref = oracle_mod.oracle_one_off(tree, table, m, stripe_start=start, stripe_stop=stop)["stripes"]
            got = np.array([[gpu[k, (k + s + 1) % n] for k in range(n)] for s in range(start, stop)])
            check_fp64(got, ref)
    gpu32, _ = ssu.one_off_matrix(tree, table, "weighted_normalized_fp32")
    ref = oracle_mod.oracle_one_off(tree, table, "weighted_normalized_fp64", stripe_start=0, stripe_stop=1)["stripes"]
    got = np.array([gpu32[k, (k + 1) % n] for k in range(n)], dtype=np.float64)
    r, _ = rel_err(got, ref[0])
    assert r < 1e-4


def test_zero_copy_result_view_outlives_its_parent(ssu):
    import gc
    tree, table = _case(57, n_samples=64)
    ref, _ = ssu.one_off_matrix(tree, table, "weighted_normalized_fp64")
    view, _ = ssu.one_off_matrix(tree, table, "weighted_normalized_fp64", copy=False)
    row = view[3]
    del view
    gc.collect()
    np.testing.assert_array_equal(row, ref[3])
    v32, _ = ssu.one_off_matrix(tree, table, "weighted_normalized_fp32", copy=False)
    assert v32.dtype == np.float32 and v32.shape == (64, 64)


def test_marshalled_inputs_follow_replaced_arrays(ssu):
    tree, table = _case(58, n_samples=40)
    other = ssu_synth.geometric_table(table.obs_ids, 40, 0.12, 10.0, 991)
    first, _ = ssu.one_off_matrix(tree, table, "weighted_unnormalized_fp64")
    again, _ = ssu.one_off_matrix(tree, table, "weighted_unnormalized_fp64")
    np.testing.assert_array_equal(first, again)
    table.indptr, table.indices, table.data = other.indptr, other.indices, other.data
    swapped, _ = ssu.one_off_matrix(tree, table, "weighted_unnormalized_fp64")
    ref, _ = ssu.one_off_matrix(tree, other, "weighted_unnormalized_fp64")
    np.testing.assert_array_equal(swapped, ref)
    table.data = other.data.copy()
    plain, _ = ssu.one_off_matrix(tree, table, "weighted_unnormalized_fp64", normalize=False)
    table.data *= 3.0  # in place: the marshalled view shares the array
    tripled, _ = ssu.one_off_matrix(tree, table, "weighted_unnormalized_fp64", normalize=False)
    np.testing.assert_allclose(tripled, 3.0 * plain, rtol=1e-12)


def _near_duplicates(seed, n_tips=150, n_base=12, copies=4):
    """Samples in clusters of near-duplicates: copies of a base sample with
    one count nudged by a relative 1e-7 (or not at all), so the weighted
    distances inside a cluster are tiny or exactly zero."""
    tree = ssu_synth.random_binary_tree(n_tips, 0.1, seed)
    base = ssu_synth.geometric_table(tree.tip_names(), n_base, 0.1, 10.0, seed + 1).dense()
    base[0, :] += 1.0  # no empty sample
    rng = np.random.default_rng(seed + 2)
    cols = []
    for j in range(n_base):
        for c in range(copies):
            col = base[:, j].copy()
            if c:
                nz = np.flatnonzero(col)
                col[nz[rng.integers(0, nz.size)]] *= 1.0 + 1e-7 * c
            cols.append(col)
    dense = np.stack(cols, axis=1)
    flat = np.flatnonzero(dense.ravel() > 0)
    table = ssu_synth.make_table(tree.tip_names(), dense.shape[1], flat, dense.ravel()[flat])
    return tree, table


@pytest.mark.parametrize("method", ["weighted_normalized_fp64", "weighted_unnormalized_fp64"])
def test_weighted_close_pairs_are_exact(ssu, oracle_mod, method):
    """Pairs whose sparse-form subtraction could lose digits are recomputed
    in the exact |u - v| form: near-duplicate samples still meet 1e-12."""
    tree, table = _near_duplicates(61)
    gpu, _ = ssu.one_off_matrix(tree, table, method)
    ref = oracle_mod.oracle_one_off(tree, table, method)["matrix"]
    check_fp64(gpu, ref)
    small = (ref > 0) & (ref < 1e-5)
    assert small.any()


@pytest.mark.parametrize("method", ["weighted_normalized", "weighted_unnormalized"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_weighted_sparse_and_dense_forms_agree(ssu, monkeypatch, method, prec):
    tree, table = _case(62, n_tips=300, n_samples=300, density=0.03)
    hybrid, _ = ssu.one_off_matrix(tree, table, f"{method}_{prec}")
    monkeypatch.setenv("UNIFRAC_B200_WEIGHTED_MODE", "dense")
    dense, _ = ssu.one_off_matrix(tree, table, f"{method}_{prec}")
    if prec == "fp64":
        check_fp64(hybrid, dense)
    else:
        np.testing.assert_allclose(hybrid, dense, rtol=5e-6, atol=1e-7)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("method", ["weighted_normalized", "weighted_unnormalized"])
def test_weighted_pair_scatter_and_tile_walk_agree(ssu, monkeypatch, method, prec):
    """The sparse rows as per-pair fixed-point sums (the default) against the
    tile kernel's own walk: the same to fp64 rounding, and the integer sums
    make repeated calls agree bit for bit in both precisions."""
    tree, table = _case(65, n_tips=500, n_samples=700, density=0.02)
    scatter = [ssu.one_off_matrix(tree, table, f"{method}_{prec}")[0] for _ in range(2)]
    np.testing.assert_array_equal(scatter[0], scatter[1])
    monkeypatch.setenv("UNIFRAC_B200_HYBRID_SCATTER", "0")
    monkeypatch.setenv("UNIFRAC_B200_DETERMINISTIC", "1")
    walk, _ = ssu.one_off_matrix(tree, table, f"{method}_{prec}")
    if prec == "fp64":
        check_fp64(scatter[0], walk)
    else:
        np.testing.assert_allclose(scatter[0], walk, rtol=2e-6, atol=1e-7)
    # raw counts (no sample normalisation): the fixed-point unit follows the largest total
    monkeypatch.delenv("UNIFRAC_B200_HYBRID_SCATTER")
    big = ssu_synth.geometric_table(table.obs_ids, 300, 0.02, 5000.0, 66)
    raw_scatter, _ = ssu.one_off_matrix(tree, big, f"{method}_{prec}", normalize=False)
    monkeypatch.setenv("UNIFRAC_B200_HYBRID_SCATTER", "0")
    raw_walk, _ = ssu.one_off_matrix(tree, big, f"{method}_{prec}", normalize=False)
    if prec == "fp64":
        check_fp64(raw_scatter, raw_walk)
    else:
        np.testing.assert_allclose(raw_scatter, raw_walk, rtol=2e-6, atol=1e-4)


@pytest.mark.parametrize("method", ["weighted_normalized", "weighted_unnormalized"])
def test_weighted_fp32_deterministic_mode_repeats_bit_for_bit(ssu, monkeypatch, method):
    """UNIFRAC_B200_DETERMINISTIC=1 gives fp32 plans the owner-per-element
    walk of the sparse rows (no atomics): repeated calls agree bit for bit,
    and with the default (atomic) form to fp32 rounding."""
    tree, table = _case(64, n_tips=400, n_samples=600, density=0.02)
    default, _ = ssu.one_off_matrix(tree, table, f"{method}_fp32")
    monkeypatch.setenv("UNIFRAC_B200_DETERMINISTIC", "1")
    runs = [ssu.one_off_matrix(tree, table, f"{method}_fp32")[0] for _ in range(3)]
    for r in runs[1:]:
        np.testing.assert_array_equal(r, runs[0])
    np.testing.assert_allclose(runs[0], default, rtol=2e-6, atol=1e-7)


UNION_RUNS = [("generalized", False, 0.5), ("generalized", False, 0.0), ("generalized", False, 1.0),
              ("generalized", False, 0.25), ("unweighted", True, 1.0), ("unweighted_unnormalized", True, 1.0),
              ("weighted_normalized", True, 1.0), ("weighted_unnormalized", True, 1.0),
              ("generalized", True, 0.5), ("generalized", True, 0.25)]


@pytest.mark.parametrize("method,vaw,alpha", UNION_RUNS)
def test_union_and_dense_forms_agree(ssu, oracle_mod, monkeypatch, method, vaw, alpha):
    """Generalized and variance-adjusted fp64 pairs summed over the union of
    the two supports (sparse rows) equal the dense form and the oracle; the
    small table splits the node range (split partials + finalize)."""
    tree, table = _case(63, n_tips=400, n_samples=260, density=0.03)
    kw = dict(variance_adjust=vaw, alpha=alpha)
    plan = ssu.Plan(tree, table, method + "_fp64", **kw)
    assert plan.pair_kernel().startswith("pair_union")
    plan.close()
    union, _ = ssu.one_off_matrix(tree, table, method + "_fp64", **kw)
    monkeypatch.setenv("UNIFRAC_B200_UNION_MODE", "dense")
    plan = ssu.Plan(tree, table, method + "_fp64", **kw)
    assert plan.pair_kernel().startswith("pair_values")
    plan.close()
    dense, _ = ssu.one_off_matrix(tree, table, method + "_fp64", **kw)
    check_fp64(union, dense)
    check_fp64(union, oracle_mod.oracle_one_off(tree, table, method + "_fp64", **kw)["matrix"])


@pytest.mark.parametrize("n_tips", [5, 9, 40, 301])
def test_union_rows_stream_in_whole_and_partial_stages(ssu, oracle_mod, n_tips):
    """The union kernel streams the embedded rows 16 at a time: trees whose
    row count is below one stage or not a multiple of 16 (the last stage
    partly past the rows, read as zero) give the oracle's matrix; stripe
    windows go through the same kernel."""
    tree, table = _case(64, n_tips=n_tips, n_samples=150, density=0.3 if n_tips < 40 else 0.05, drop=1)
    kw = dict(variance_adjust=True, alpha=0.5)
    plan = ssu.Plan(tree, table, "generalized_fp64", **kw)
    assert plan.pair_kernel().startswith("pair_union")
    plan.close()
    ref = oracle_mod.oracle_one_off(tree, table, "generalized_fp64", **kw)["matrix"]
    gpu, _ = ssu.one_off_matrix(tree, table, "generalized_fp64", **kw)
    check_fp64(gpu, ref)
    stripes, _ = ssu.partial(tree, table, "generalized_fp64", 10, 40, **kw)
    check_fp64(stripes, oracle_mod.oracle_one_off(tree, table, "generalized_fp64", stripe_start=10, stripe_stop=40,
                                                  **kw)["stripes"])


@pytest.mark.parametrize("method,vaw", [("generalized", False), ("generalized", True), ("weighted_normalized", True),
                                        ("unweighted", True)])
def test_union_fp32_within_reference_fp32_error(ssu, oracle_mod, method, vaw):
    """fp32 inputs through the union kernel (terms in fp64, fp32 output)."""
    tree, table = _case(65, n_tips=400, n_samples=200, density=0.03)
    kw = dict(variance_adjust=vaw, alpha=0.5)
    plan = ssu.Plan(tree, table, method + "_fp32", **kw)
    assert plan.pair_kernel().startswith("pair_union")
    plan.close()
    gpu, _ = ssu.one_off_matrix(tree, table, method + "_fp32", **kw)
    assert gpu.dtype == np.float32
    check_fp32(gpu, oracle_mod, tree, table, method, **kw)


@pytest.mark.parametrize("method", ["unweighted", "weighted_normalized", "weighted_unnormalized", "generalized"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_negative_counts_take_the_dense_kernels(ssu, oracle_mod, method, prec):
    """Negative entries (the reference accepts them): presence is u > 0, the
    sparse forms need u >= 0, so weighted and generalized plans run the dense
    kernels; results match the oracle (which matches the reference on this
    input)."""
    tree, base = _case(66, n_tips=120, n_samples=70, density=0.15)
    rng = np.random.default_rng(166)
    data = base.data.copy()
    flip = rng.random(data.size) < 0.05
    data[flip] = -0.5 * data[flip]
    table = ssu_synth.Table(base.obs_ids, base.sample_ids, base.indptr, base.indices, data)
    plan = ssu.Plan(tree, table, f"{method}_{prec}", alpha=1.0)
    kernel = plan.pair_kernel()
    plan.close()
    assert "hybrid" not in kernel and "union" not in kernel and "tc" not in kernel
    gpu, _ = ssu.one_off_matrix(tree, table, f"{method}_{prec}", alpha=1.0)
    if prec == "fp64":
        ref = oracle_mod.oracle_one_off(tree, table, method + "_fp64", alpha=1.0)["matrix"]
        assert np.array_equal(np.isnan(gpu), np.isnan(ref))
        check_fp64(gpu, ref)
    else:
        check_fp32(gpu, oracle_mod, tree, table, method, alpha=1.0)


def test_union_wait_that_runs_out_is_an_error_and_the_device_stays_usable(ssu, oracle_mod, monkeypatch):
    """Failure injection without a fault: with UNIFRAC_B200_TEST_STALL the
    union kernel's producer issues no copy, so every consumer's bounded wait
    (here ~1 ms) runs out; the call returns output_error instead of hanging,
    and the next call in the same process is correct."""
    tree, table = _case(67, n_tips=200, n_samples=80, density=0.05)
    kw = dict(variance_adjust=True, alpha=0.5)
    monkeypatch.setenv("UNIFRAC_B200_TEST_STALL", "1")
    monkeypatch.setenv("UNIFRAC_B200_WAIT_CYCLES", "2000000")
    plan = ssu.Plan(tree, table, "generalized_fp64", **kw)
    assert plan.pair_kernel().startswith("pair_union")
    plan.close()
    with pytest.raises(ssu.SSUError) as e:
        ssu.one_off_matrix(tree, table, "generalized_fp64", **kw)
    assert e.value.status == 6  # output_error
    monkeypatch.delenv("UNIFRAC_B200_TEST_STALL")
    monkeypatch.delenv("UNIFRAC_B200_WAIT_CYCLES")
    gpu, _ = ssu.one_off_matrix(tree, table, "generalized_fp64", **kw)
    check_fp64(gpu, oracle_mod.oracle_one_off(tree, table, "generalized_fp64", **kw)["matrix"])


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_hybrid_with_every_row_sparse_matches_dense_form(ssu, monkeypatch, prec):
    """UNIFRAC_B200_HYBRID_DIV=1 sends every row, however dense, through the
    sparse-row path: rows with more than 32 present columns in a 128-column
    block take its chunked branch (fp32) or long walks (fp64)."""
    tree, table = _case(68, n_tips=200, n_samples=300, density=0.3)
    monkeypatch.setenv("UNIFRAC_B200_WEIGHTED_MODE", "dense")
    dense, _ = ssu.one_off_matrix(tree, table, f"weighted_normalized_{prec}")
    monkeypatch.delenv("UNIFRAC_B200_WEIGHTED_MODE")
    monkeypatch.setenv("UNIFRAC_B200_HYBRID_DIV", "1")
    plan = ssu.Plan(tree, table, f"weighted_normalized_{prec}")
    assert plan.pair_kernel().startswith("pair_hybrid")
    plan.close()
    sparse, _ = ssu.one_off_matrix(tree, table, f"weighted_normalized_{prec}")
    if prec == "fp64":
        check_fp64(sparse, dense)
    else:
        np.testing.assert_allclose(sparse, dense, rtol=5e-6, atol=1e-7)


def test_page_locked_results_are_recycled(ssu):
    """Full results of 2 MiB or more come from the page-locked pool, and a
    result released through destroy_mat_full_fp64 goes back to it: after many
    large results, large and smaller ones are still page-locked (flag
    0x2000), so no call falls back to registering pageable memory."""
    import ctypes
    L = ssu.lib()
    tree, table = _case(67, n_tips=300, n_samples=700, density=0.05)
    small_tree, small = _case(68, n_tips=300, n_samples=520, density=0.05)
    for t, tb in [(tree, table)] * 4 + [(small_tree, small)] * 2 + [(tree, table)]:
        x = ssu.Inputs(t, tb)
        res = ctypes.POINTER(ssu.MatFull64)()
        st = L.one_off_matrix_inmem_v3(ctypes.byref(x.biom), ctypes.byref(x.tree), b"weighted_normalized_fp64",
                                       False, 1.0, False, True, 1, 0, False, None, ctypes.byref(res))
        assert st == 0
        assert res.contents.flags & 0x2000, "result not page-locked"
        L.destroy_mat_full_fp64(ctypes.byref(res))

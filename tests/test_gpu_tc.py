"""The tensor-core (tcgen05) unweighted contraction, selected with
UNIFRAC_B200_UNWEIGHTED_MODE=gemm, against the fp64 oracle.  Bar: max
relative error 1e-6 on every pair (the contraction's stated bound; lengths
carried as fp16 hi+lo per 256-node chunk, fp32 accumulation per chunk, fp64
across chunks and in the final ratio)."""
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


def test_tc_plan_agrees_with_stripe_form(ssu, gemm_mode):
    tree, table = _case(9, 2000, 400)
    plan = ssu.Plan(tree, table, "unweighted_fp64")
    plan.execute()
    tc = plan.result()
    plan.close()
    os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"] = "stripe"
    stripe, _ = ssu.one_off_matrix(tree, table, "unweighted_fp64")
    assert rel_err(tc, stripe)[0] <= TC_REL

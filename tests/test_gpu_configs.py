"""Parity at the benchmark configurations' full sizes, against the reference's
own CPU build (oracle/_ref/libssu_ref.so: the reference's tree, table,
embedding, task and stripe code compiled from its sources, run through
process_stripes as src/unifrac_cmp.cpp:29-152 does).

* 20,000 tips x 2,048 samples: the whole matrix, weighted normalized and
  unnormalized, fp64 at 1e-12; fp32 within 4x the reference fp32 build's own
  error; Faith PD.
* 100,000 tips x 25,000 presence samples: the tensor-core contraction and
  the plain stripe form on 16 windows of 4 stripes spread over all 12,500
  stripes, against the reference fp64 (1e-6 and 1e-12).
* 100 rarefied replicates of 10,000 x 5,000 on 10,000 tips: replicates 0, 49
  and 99 of one batch, unweighted and weighted normalized fp32, within the
  reference fp32 build's error (measured on replicate 0, floor 1e-6).
* 64 uneven tables on 50,000 tips: the 4 smallest tables whole and the first
  and last three stripes of the 4 largest, generalized (alpha 0.5) and the four
  variance-adjusted methods, fp64 at 1e-12.

Each needs the compiled reference (built by __graft_entry__.build() where the
reference checkout is present); without it the tests are skipped."""
import ctypes

import numpy as np
import pytest

import ssu_synth
from conftest import rel_err

pytestmark = pytest.mark.gpu

FP64_REL = 1e-12
FP64_ABS = 1e-13
TC_REL = 1e-6


@pytest.fixture(scope="module")
def ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libssu_ref.so (the compiled reference) is not built")
    return oracle_mod


def check(got, want, rel=FP64_REL, absz=FP64_ABS, what=""):
    r, z = rel_err(got, want)
    assert r <= rel and z <= absz, (what, r, z)


def stripes_of(matrix, start, stop):
    """Stripe s holds d(k, (k + s + 1) mod n) at position k (src/unifrac_cmp.cpp:54-96)."""
    n = matrix.shape[0]
    k = np.arange(n)
    return np.stack([matrix[k, (k + s + 1) % n] for s in range(start, stop)])


def test_20k_tips_2048_samples_whole_matrix_against_reference(ssu, ref):
    tree, table = ssu_synth.lognormal_20k_tips_2048_samples()
    for m in ("weighted_normalized", "weighted_unnormalized"):
        want64 = ref.ref_one_off(tree, table, m + "_fp64")["matrix"]
        got64, _ = ssu.one_off_matrix(tree, table, m + "_fp64")
        check(got64, want64, what=m + "_fp64")
        want32 = ref.ref_one_off(tree, table, m + "_fp32")["matrix"]
        got32, _ = ssu.one_off_matrix(tree, table, m + "_fp32")
        bar, bar_z = rel_err(want32, want64)
        check(got32, want64, rel=max(4 * bar, 1e-6), absz=max(4 * bar_z, 1e-6), what=m + "_fp32")
    vals, ids = ssu.faith_pd(tree, table)
    fref = ref.ref_faith_pd(tree, table)
    check(np.asarray(vals), np.asarray(fref["values"]), what="faith_pd")
    assert list(ids) == [table.sample_ids[j] for j in fref["kept"]]


def _device_matrix(torch, plan, n):
    out = torch.empty((n, n), dtype=torch.float64, device="cuda")
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    assert rt.cudaMemcpy(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(plan.device_result()),
                         out.numel() * 8, 3) == 0
    return out


def _device_stripes(torch, dev, windows):
    n = dev.shape[0]
    k = torch.arange(n, device="cuda")
    return [torch.stack([dev[k, (k + s + 1) % n] for s in range(a, b)]).cpu().numpy() for a, b in windows]


def test_100k_tips_25k_presence_tensor_core_and_stripe_forms_against_reference(ssu, ref, monkeypatch):
    import torch
    tree, table = ssu_synth.presence_100k_tips_25k_samples()
    n = table.n_samples
    s_total = (n + 1) // 2
    starts = np.linspace(0, s_total - 4, 16).astype(int)
    windows = [(int(a), int(a) + 4) for a in starts]
    want = [ref.ref_one_off(tree, table, "unweighted_fp64", stripe_start=a, stripe_stop=b,
                            want_matrix=False)["stripes"] for a, b in windows]
    for mode, bar in (("gemm", TC_REL), ("stripe", FP64_REL)):
        monkeypatch.setenv("UNIFRAC_B200_UNWEIGHTED_MODE", mode)
        plan = ssu.Plan(tree, table, "unweighted_fp64")
        assert (plan.pair_kernel() == "unweighted_tc_kernel") == (mode == "gemm")
        plan.execute()
        torch.cuda.synchronize()  # the plan runs on its own stream
        dev = _device_matrix(torch, plan, n)
        plan.close()
        got = _device_stripes(torch, dev, windows)
        del dev
        torch.cuda.empty_cache()
        for (a, b), g, w in zip(windows, got, want):
            check(g, w, rel=bar, absz=1e-9 if mode == "gemm" else FP64_ABS, what=f"{mode} stripes [{a},{b})")


def test_100_rarefied_replicates_first_middle_last_against_reference(ssu, ref):
    tree, _, reps = ssu_synth.rarefied_replicates_10k_tips_5k_samples()
    picks = (0, 49, 99)
    for m in ("unweighted", "weighted_normalized"):
        plan = ssu.BatchPlan(tree, reps, m + "_fp32")
        plan.execute()
        res = {r: plan.result_of(r) for r in picks}
        plan.close()
        w64 = {r: ref.ref_one_off(tree, reps[r], m + "_fp64")["matrix"] for r in picks}
        w32 = ref.ref_one_off(tree, reps[0], m + "_fp32")["matrix"]
        bar, bar_z = rel_err(w32, w64[0])
        for r in picks:
            check(res[r], w64[r], rel=max(4 * bar, 1e-6), absz=max(4 * bar_z, 1e-6), what=f"{m} replicate {r}")


@pytest.fixture(scope="module")
def uneven_tables():
    return ssu_synth.uneven_tables_50k_tips()


@pytest.mark.parametrize("method,vaw", [("generalized_fp64", False), ("unweighted_fp64", True),
                                        ("weighted_normalized_fp64", True), ("weighted_unnormalized_fp64", True),
                                        ("generalized_fp64", True)])
def test_64_uneven_tables_smallest_and_largest_against_reference(ssu, ref, uneven_tables, method, vaw):
    tree, tables = uneven_tables
    order = sorted(range(len(tables)), key=lambda t: tables[t].n_samples)
    small, large = order[:4], order[-4:]
    plan = ssu.BatchPlan(tree, tables, method, variance_adjust=vaw, alpha=0.5)
    plan.execute()
    res = {t: plan.result_of(t) for t in small + large}
    plan.close()
    for t in small:
        want = ref.ref_one_off(tree, tables[t], method, variance_adjust=vaw, alpha=0.5)["matrix"]
        check(res[t], want, what=f"table {t} ({tables[t].n_samples} samples)")
    for t in large:
        n = tables[t].n_samples
        s_total = (n + 1) // 2
        for a, b in ((0, 3), (s_total - 3, s_total)):
            want = ref.ref_one_off(tree, tables[t], method, variance_adjust=vaw, alpha=0.5, stripe_start=a,
                                   stripe_stop=b, want_matrix=False)["stripes"]
            check(stripes_of(res[t], a, b), want, what=f"table {t} ({n} samples) stripes [{a},{b})")

"""Benchmark: pair-branch updates/s of the B200 Strided State UniFrac engine.

Default line (one step): the full 25,000 x 25,000 unweighted UniFrac matrix
(fp64 ratios) of a 25,000-sample presence table on a 100,000-tip random
binary tree (branch lengths Exponential(mean 0.02), per-sample richness
log-uniform in [50, 2000] distinct tips, seed 3), computed as a tcgen05
tensor-core contraction: presence rows, the contraction with the distances
formed in its epilogue, the matrix written to HBM.  The same plan on the
plain stripe (presence-word) form is timed beside it, and the two are
compared pair by pair.  Units: U = n(n-1)/2 x E pair-branch updates, E the
embedded branches of the sheared tree.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload NAME]

value: U*K / (sum of per-step device times), inputs resident in HBM, L2
flushed between steps, max over ranks.  e2e: the same metric through the C
API (one_off_matrix_inmem_v3, unweighted_fp64 with
UNIFRAC_B200_UNWEIGHTED_MODE=gemm) from host buffers: host tree and table
work, upload, compute and the 5 GB copy-out inside the timed region.  Under
torchrun each rank runs its own table (seed + rank): weak scaling, no
data-path collective.  --impl reference times the reference's own CPU build
(oracle/_ref) on a stripe window of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "unifrac-binaries_b200"))

METRIC = "pair-branch updates/s"
UNIT = "updates/s"
PRESENCE_WORKLOAD = ("unweighted_fp64 UniFrac, 100,000-tip tree (Exponential(0.02) lengths), 25,000 presence "
                     "samples (log-uniform richness 50-2,000), full 25,000 x 25,000 matrix")
WEIGHTED_WORKLOAD = "weighted_normalized_fp64 UniFrac, 20k-tip tree, 20k features x 2048 samples, full matrix"
METHOD = "weighted_normalized_fp64"
# --workload choices: each names the data it runs
WORKLOADS = {
    "100k-tips-25k-presence": "unweighted fp64, 100,000-tip tree, 25,000 presence samples: tensor-core contraction "
                              "vs the plain stripe form (the default line)",
    "20k-tips-2048-samples": "weighted_normalized_fp64, 20,000-tip tree, 20,000 x 2,048 table",
    "1k-tips-128-samples": "unweighted + weighted_normalized fp64, 1,000-tip tree, 1,000 x 128 table, condensed form",
    "100-replicates-5k-samples": "unweighted + weighted_normalized fp32, 100 rarefied replicates of a 10,000 x 5,000 "
                                 "table, 10,000-tip tree",
    "64-uneven-tables": "generalized + four VAW methods fp64, 64 tables of 64-4,096 samples, 50,000-tip tree",
}
# reference-form algorithmic bytes per pair-branch update of the weighted
# normalized fp64 method (accumulator read-modify-write of two fp64 stripes
# per 112-node batch: 2 * 2 * 8 / 112)
ALGO_BYTES_PER_UPDATE = 2 * 2 * 8 / 112.0
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "pair_hybrid_weighted_normalized_fp64_20k_tips_2048_samples.md")
PROFILE_TC = os.path.join(ROOT, "profiles", "unweighted_tc_kernel_100k_tips_25k_presence.md")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--samples", type=int, default=2048)
    p.add_argument("--tips", type=int, default=20000)
    p.add_argument("--method", default=METHOD)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--replicates", type=int, default=100)
    p.add_argument("--uneven-tables", type=int, default=64)
    p.add_argument("--uneven-tips", type=int, default=50000)
    p.add_argument("--workload", default="100k-tips-25k-presence", choices=list(WORKLOADS),
                   help="; ".join(f"{k}: {v}" for k, v in WORKLOADS.items()))
    p.add_argument("--presence-samples", type=int, default=25000)
    p.add_argument("--presence-tips", type=int, default=100000)
    p.add_argument("--no-secondary", action="store_true", help="skip the weighted (20k-tips-2048-samples) keys "
                   "of the default line")
    p.add_argument("--no-stripe-form", action="store_true", help="skip the stripe-form comparison of the default line")
    return p.parse_args()


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def stripe_window(n_samples, rank, world):
    """Balanced split of the (n+1)/2 stripes over ranks, as the reference's
    set_tasks splits them over substeps (src/api.cpp:447-491)."""
    total = (n_samples + 1) // 2
    big, small = -(-total // world), total // world
    n_big = total % world or world
    start = sum(big if r < n_big else small for r in range(rank))
    return start, start + (big if rank < n_big else small)


def combine_ranks(values, world, device):
    """[step_ms, e2e_ms, units, pair_ms] -> max-over-ranks times and summed units."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world == 1:
        return values[0], values[1], values[2], values[3]
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return tmax[0].item(), tmax[1].item(), tsum[2].item(), tmax[3].item()


def make_workload(seed, args):
    import ssu_synth
    return ssu_synth.lognormal_20k_tips_2048_samples(seed=seed, n_samples=args.samples, n_tips=args.tips)


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region.

    Two read-only sources over the same window: `nvidia-smi -lms 200` (the
    CSV query of clocks and event reasons) and an NVML poll every 10 ms in a
    thread, so a timed region of a few tens of milliseconds still holds
    samples.  The GPU is named by its UUID, so the right device is read under
    CUDA_VISIBLE_DEVICES.  start() returns once the poll has its first
    sample."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.uuid = None
        try:
            import torch
            self.uuid = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
        except Exception:
            self.uuid = None
        self.proc = None
        self.thread = None
        self.polled = []
        self.first = None
        self.done = None

    def _poll(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
        except Exception:
            self.first.set()
            return
        try:
            h = nv.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid else nv.nvmlDeviceGetHandleByIndex(self.gpu)
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            while True:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.polled.append((float(sm), float(mx), [n for n, b in zip(self.NAMES, bits) if mask & b]))
                self.first.set()
                if self.done.wait(0.01):
                    break
        except Exception:
            pass
        finally:
            self.first.set()
            try:
                nv.nvmlShutdown()
            except Exception:
                pass

    def start(self):
        import threading
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.uuid or str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        self.polled = []
        self.first, self.done = threading.Event(), threading.Event()
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()
        self.first.wait(2.0)

    def stop(self):
        sm, mx, reasons = [], [], set()
        smi = 0
        if self.thread:
            self.done.set()
            self.thread.join(5.0)
            for s, m, r in self.polled:
                sm.append(s)
                mx.append(m)
                reasons.update(r)
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            for s, m, r in self.parse_smi(out):
                sm.append(s)
                mx.append(m)
                smi += 1
                reasons.update(r)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "sm_min_mhz": min(sm),
                "reasons": sorted(reasons), "samples": len(sm), "nvidia_smi_samples": smi}

    @classmethod
    def parse_smi(cls, text):
        """(sm MHz, max sm MHz, active throttle reasons) per line of the
        FIELDS query in csv,noheader,nounits form; other lines are skipped."""
        rows = []
        for line in text.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                s, m = float(f[1]), float(f[2])
            except ValueError:
                continue
            rows.append((s, m, [name for name, val in zip(cls.NAMES, f[5:9]) if val.lower() == "active"]))
        return rows


def read_profile_value(path, key):
    """A `key: value ...` figure from a committed ncu summary (first token)."""
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1].split()[0])
    except (OSError, ValueError):
        pass
    return None


def read_traffic():
    """dram bytes per hybrid pair-kernel launch from the committed ncu summary."""
    return read_profile_value(PROFILE_TRAFFIC, "dram_bytes_per_launch_full_size")


def peaks():
    """Measured peaks of this pool's B200s (MEASURED_PEAKS.json), else the
    fallback figures: (HBM GB/s, bf16 TFLOP/s burst, sustained, kind)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), float(d.get("bf16_tflops_sustained", 1400.0)), "measured"
    except Exception:
        return 6650.0, 1590.0, 1400.0, "fallback"


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    return oracle_py


def cpu_baseline(tree, table, method, target_s=8.0):
    """The reference's own CPU path (oracle/_ref) on a stripe sub-range of the
    same workload, all host threads; grown until it runs ~target_s."""
    oracle_py = _oracle()
    n = table.n_samples
    s_total = (n + 1) // 2
    kind = "reference"
    if not oracle_py.ref_available():
        kind = "port"
    stripes = 8
    while True:
        stop = min(s_total, stripes)
        if kind == "reference":
            r = oracle_py.ref_one_off(tree, table, method, stripe_start=0, stripe_stop=stop,
                                      want_matrix=(stop == s_total), with_timing=True)
            secs = r["seconds"][0] + r["seconds"][1]
            e = r["n_embedded"]
        else:
            t0 = time.perf_counter()
            r = oracle_py.oracle_one_off(tree, table, method, stripe_start=0, stripe_stop=stop)
            secs = time.perf_counter() - t0
            e = r["n_embedded"]
        if secs >= target_s / 4 or stop == s_total:
            break
        stripes = int(stripes * max(2.0, min(8.0, target_s / max(secs, 1e-3))))
    units = stop * n * e
    what = ("all stripes, process_stripes + stripes_to_matrix_T" if stop == s_total else
            f"stripes [0,{stop}) of {s_total}, process_stripes")
    return {"value": units / secs, "unit": UNIT, "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())),
            "cpu_model": cpu_model(), "kind": kind, "n_embedded": e,
            "sample": f"{what} ({stop * n} pairs x {e} branches), {secs:.2f} s"}


def presence_reference_sample(tree, table, method="unweighted_fp64", target_s=6.0, fixed_s=None):
    """The reference's CPU build (oracle/_ref, all host threads) on a stripe
    window [0, S) of the presence workload.  Each call embeds every node
    for every sample before its stripes (~2 s here whatever S), so the rate
    is the marginal one: (S x n x E) / (t(S) - t(1)), t(1) the time of a
    one-stripe window - the reference's best case, extrapolated linearly to
    all stripes.  Returns (rate, sample dict, fixed seconds)."""
    oracle_py = _oracle()
    kind = "reference" if oracle_py.ref_available() else "port"

    def run(a, b):
        if kind == "reference":
            return oracle_py.ref_one_off(tree, table, method, stripe_start=a, stripe_stop=b, want_matrix=False,
                                         with_timing=True)["seconds"][0]
        t0 = time.perf_counter()
        oracle_py.oracle_one_off(tree, table, method, stripe_start=a, stripe_stop=b)
        return time.perf_counter() - t0

    n = table.n_samples
    s_total = (n + 1) // 2
    if fixed_s is None:
        fixed_s = run(0, 1)
    stripes = 16
    while True:
        secs = run(0, stripes)
        if secs - fixed_s >= target_s / 2 or stripes >= s_total:
            break
        stripes = min(s_total, int(stripes * max(2.0, min(8.0, target_s / max(secs - fixed_s, 1e-3)))))
    e = (oracle_py.ref_one_off if kind == "reference" else oracle_py.oracle_one_off)(
        tree, table, method, stripe_start=0, stripe_stop=1)["n_embedded"]
    marginal = max(secs - fixed_s, 1e-9)
    rate = stripes * n * e / marginal
    full_s = fixed_s + marginal * s_total / stripes
    sample = {"kind": kind, "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())), "cpu_model": cpu_model(),
              "full_matrix_s": full_s,
              "sample": f"stripes [0,{stripes}) of {s_total} ({stripes * n} pairs x {e} branches): {secs:.2f} s, of "
                        f"which {fixed_s:.2f} s is the per-call embedding (timed on a one-stripe window); rate = "
                        f"marginal stripes / (t - t_embed), full matrix extrapolated to {full_s:.0f} s "
                        f"(process_stripes only)"}
    return rate, sample, fixed_s


def run_reference(args):
    """--impl reference: the reference's own CPU build on the box's host
    cores, same workload string, metric and unit as this arm's line."""
    world, rank, _ = dist_init()
    if rank != 0:
        return
    if args.workload == "100k-tips-25k-presence":
        import ssu_synth
        tree, table = ssu_synth.presence_100k_tips_25k_samples(seed=3, n_samples=args.presence_samples,
                                                               n_tips=args.presence_tips)
        fixed = None
        fixed_runs, rates = [], []
        sample = None
        for i in range(args.warmup + args.steps):
            rate, sample, f = presence_reference_sample(tree, table, fixed_s=None if i < max(args.warmup, 1) else
                                                        statistics.median(fixed_runs))
            if i < max(args.warmup, 1):
                fixed_runs.append(f)
            if i >= args.warmup:
                rates.append(rate)
        value = statistics.median(rates)
        cb = dict(sample)
        cb.update({"value": value, "unit": UNIT})
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": sample["full_matrix_s"] * 1e3,
                "ms_per_step_basis": "the whole 25,000 x 25,000 matrix, extrapolated from the sample (cpu_baseline)",
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator presence_100k_tips_25k_samples)",
                "config": {"workload": PRESENCE_WORKLOAD, "method": "unweighted_fp64"},
                "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    tree, table = make_workload(2, args)
    samples = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(tree, table, args.method, target_s=4.0)
        if i >= args.warmup:
            samples.append(cb)
    value = statistics.median(c["value"] for c in samples)
    cb = dict(samples[-1])
    cb["value"] = value
    n = table.n_samples
    full_units = n * (n - 1) / 2 * samples[-1]["n_embedded"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": full_units / value * 1e3,
            "ms_per_step_basis": "the whole matrix at the sample's rate (cpu_baseline)",
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator lognormal_20k_tips_2048_samples)",
            "config": {"workload": WEIGHTED_WORKLOAD, "method": args.method,
                       "n_samples": args.samples, "n_tips": args.tips},
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _device_copy(torch, src_ptr, n, dtype):
    """Device-to-device copy of a plan's n x n result into a torch tensor."""
    import ctypes
    out = torch.empty((n, n), dtype=dtype, device="cuda")
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    rc = rt.cudaMemcpy(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(src_ptr), out.numel() * out.element_size(), 3)
    if rc != 0:
        raise RuntimeError(f"cudaMemcpy failed ({rc})")
    return out


def _step_loop(torch, plan, stream, steps, barrier, flush):
    """K timed executes: per-step CUDA-event time on the plan's stream (L2
    flushed before each, outside the events) and the pair stage's time."""
    plan.set_timing(True)
    step_ms, pair_ms = [], []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute(stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        pair_ms.append(plan.stage_ms()[1])
    barrier()
    plan.set_timing(False)
    return step_ms, pair_ms


def tc_work_units(n):
    """Work units of the tensor-core kernel for one table of n samples: the
    (256-row, 128-column) blocks holding a pair k < l."""
    nkb, nlb = (n + 255) // 256, (n + 127) // 128
    return sum(1 for kb in range(nkb) for lb in range(nlb) if kb * 256 < min(n, (lb + 1) * 128) - 1)


def run_presence(args):
    """The default line: unweighted fp64 on the 100,000-tip / 25,000-sample
    presence table through the tcgen05 contraction, with the plain stripe
    (presence-word) form timed beside it on the same plan inputs."""
    import torch
    import torch.distributed as dist
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    import ssu_b200
    import ssu_synth
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # the 5 GB result comes back into page-locked memory recycled between calls
    os.environ.setdefault("UNIFRAC_B200_PINNED_BYTES", str(8 << 30))
    t0 = time.perf_counter()
    tree, table = ssu_synth.presence_100k_tips_25k_samples(seed=3 + rank, n_samples=args.presence_samples,
                                                           n_tips=args.presence_tips)
    gen_s = time.perf_counter() - t0
    method = "unweighted_fp64"
    os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"] = "gemm"
    gp = ssu_b200.Plan(tree, table, method)
    assert gp.pair_kernel() == "unweighted_tc_kernel", gp.pair_kernel()
    units = gp.work_units()
    flops_issued = gp.tensor_flops()
    n = table.n_samples
    for _ in range(args.warmup):
        gp.execute(stream.cuda_stream)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    step_ms, tc_ms = _step_loop(torch, gp, stream, args.steps, barrier, flush)
    clk = clocks.stop()
    launches_per_step = gp.launches()
    total_ms, _, all_units, mean_tc_ms = combine_ranks([sum(step_ms), 0.0, float(units), sum(tc_ms) / len(tc_ms)],
                                                       world, "cuda")

    extra = {}
    if world == 1 and not args.no_stripe_form:
        # the plain stripe form on the same inputs, and every pair compared
        g_res = _device_copy(torch, gp.device_result(), n, torch.float64)
        gp.close()
        gp = None
        os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"] = "stripe"
        sp = ssu_b200.Plan(tree, table, method)
        sp.execute(stream.cuda_stream)
        torch.cuda.synchronize()
        s_step, s_pair = _step_loop(torch, sp, stream, 1, barrier, flush)
        s_res = _device_copy(torch, sp.device_result(), n, torch.float64)
        s_name = sp.pair_kernel()
        sp.close()
        worst, q999 = 0.0, []
        gen = torch.Generator(device="cuda")
        gen.manual_seed(0)
        for r0 in range(0, n, 2048):
            a = g_res[r0:r0 + 2048]
            b = s_res[r0:r0 + 2048]
            rows = torch.arange(r0, min(n, r0 + 2048), device="cuda").unsqueeze(1)
            cols = torch.arange(n, device="cuda").unsqueeze(0)
            mask = (cols > rows) & (b != 0)
            rel = ((a - b).abs() / b.abs())[mask]
            if rel.numel():
                worst = max(worst, rel.max().item())
                pick = torch.randint(0, rel.numel(), (200000,), device="cuda", generator=gen)
                q999.append(torch.quantile(rel[pick], 0.999).item())
        del g_res, s_res
        extra["stripe_form"] = {"kernel": s_name, "ms_per_step": s_step[0], "kernel_ms": s_pair[0],
                                "value": units / (s_step[0] / 1e3)}
        extra["tc_vs_stripe"] = s_step[0] / (sum(step_ms) / len(step_ms))
        extra["rel_err_vs_fp64_stripe"] = {"max": worst, "p99.9": max(q999) if q999 else None,
                                           "pairs": n * (n - 1) // 2,
                                           "bar": 1e-6}
    if gp is not None:
        gp.close()

    # end to end through the C API: host buffers in, the host matrix out
    os.environ["UNIFRAC_B200_UNWEIGHTED_MODE"] = "gemm"
    e2e_ms = []
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        barrier()
        t0 = time.perf_counter()
        m, _ = ssu_b200.one_off_matrix(tree, table, method, copy=False)
        dt = (time.perf_counter() - t0) * 1e3
        del m  # the caller is done with the result: destroy_mat_full_fp64
        if i > 0:
            e2e_ms.append(dt)
    h2d = int(table.indptr.nbytes + table.indices.nbytes + table.data.nbytes + tree.structure.nbytes +
              tree.lengths.nbytes)
    d2h = n * n * 8
    _, e2e_total, _, _ = combine_ranks([0.0, sum(e2e_ms), 0.0, 0.0], world, "cuda")

    if rank == 0:
        value = all_units * args.steps / (total_ms / 1e3)
        _, peak_burst, peak_sus, peak_kind = peaks()
        algo_flops = 2.0 * units
        achieved = algo_flops / (mean_tc_ms / 1e3) / 1e12
        issued = flops_issued / (mean_tc_ms / 1e3) / 1e12  # int8 tensor ops
        traffic_per_unit = read_profile_value(PROFILE_TC, "dram_bytes_per_work_unit")
        n_units = tc_work_units(n)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "u8 operands (presence times 8-bit digits of 23-bit fixed-point lengths, q = 256 u v + s t), "
                     "exact s32 accumulate per chunk, f64 across chunks and ratios",
            "data": "synthetic (seeded generator presence_100k_tips_25k_samples)",
            "config": {"workload": PRESENCE_WORKLOAD, "method": method, "pair_kernel": "unweighted_tc_kernel",
                       "n_samples": n, "embedded_branches": gp_units_e(units, n), "per_gpu_units": units,
                       "l2": "flushed between steps (256 MiB write outside the step events); operands 30 GB > L2",
                       "generation_s": gen_s},
            "tc_kernel_ms": mean_tc_ms,
            **extra,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak_sus, "unit": "TFLOP/s",
                         "frac": achieved / peak_sus, "traffic": traffic_per_unit * n_units if traffic_per_unit else None,
                         "peak_kind": f"{peak_kind} bf16 sustained (the kernel runs ~0.2 s per launch, back to back)",
                         "frac_of_burst": achieved / peak_burst,
                         "algorithmic_flops_per_launch": algo_flops, "issued_int8_ops_per_launch": flops_issued,
                         "issued_int8_tops": issued, "issued_frac": issued / (2.0 * peak_sus),
                         "issued_peak": f"2 x {peak_kind} bf16 sustained (dense int8 : bf16 = 2 : 1 on B200)",
                         "note": "algorithmic flops = 2 x pair-branch updates (one multiply-add per pair and "
                                 "branch), against the bf16 peak; the kernel issues ~2x that in int8 ops (two "
                                 "digit products per length, padding of the length chunks and of 256 x 128 work "
                                 "units on the diagonal) at twice the bf16 rate; traffic = ncu DRAM bytes per work unit x work "
                                 "units"},
            "e2e": {"value": all_units * len(e2e_ms) / (e2e_total / 1e3) if e2e_ms else None, "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_total / len(e2e_ms) if e2e_ms else None,
                    "path": "one_off_matrix_inmem_v3 (unweighted_fp64, UNIFRAC_B200_UNWEIGHTED_MODE=gemm), host CSR "
                            "and tree arrays in, 25,000 x 25,000 fp64 matrix out (UNIFRAC_B200_PINNED_BYTES="
                            + os.environ.get("UNIFRAC_B200_PINNED_BYTES", "") + ")"},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu_baseline:
            try:
                rate, sample, _ = presence_reference_sample(tree, table, target_s=8.0)
                line["cpu_baseline"] = dict(sample, value=rate, unit=UNIT)
            except Exception as exc:  # the reported baseline never blocks the bench line
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(exc)[:200]}
        if world == 1 and not args.no_secondary:
            try:
                w = measure_weighted(args, 1, 0, local, stream=stream, flush=flush, cpu=not args.no_cpu_baseline)
                line["secondary_weighted_20k_tips_2048_samples"] = {
                    k: w.get(k) for k in ("value", "ms_per_step", "pair_kernel_ms", "e2e", "roofline",
                                          "cpu_baseline", "config", "gpu_launches")}
            except Exception as exc:
                line["secondary_weighted_20k_tips_2048_samples"] = {"error": str(exc)[:300]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _time_batch(torch, plan, stream, steps, warmup, flush):
    """Per-step device time (ms) of a batch plan replayed as a CUDA graph."""
    plan.set_graph(True)
    for _ in range(max(warmup, 1)):
        plan.execute(stream.cuda_stream)
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute(stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return sum(ms) / len(ms)


def _unbatched_ms(torch, ssu_b200, tree, tables, method, stream, **kw):
    """Device time of the same tables run one plan per table (no batching)."""
    total = 0.0
    for t in tables:
        p = ssu_b200.Plan(tree, t, method, **kw)
        p.execute(stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        p.execute(stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
        p.close()
    return total


def _rel_err(a, b):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nz = b != 0
    r = float(np.max(np.abs(a[nz] - b[nz]) / np.abs(b[nz]))) if nz.any() else 0.0
    z = float(np.max(np.abs(a[~nz]))) if (~nz).any() else 0.0
    return r, z


def _batch_setup():
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    return torch, stream, flush


def run_small(args):
    """1,000-tip tree, 1,000 x 128 table: unweighted and weighted-normalized
    fp64, condensed 128 x 128 form through the C API.  Too small for a
    roofline (launch- and latency-bound): times only, next to the reference's
    CPU build on the same input."""
    torch, stream, flush = _batch_setup()
    import ssu_b200
    import ssu_synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    tree, table = ssu_synth.geometric_1k_tips_128_samples()
    out = {}
    total_units, total_e2e, total_dev = 0, 0.0, 0.0
    for m in ("unweighted_fp64", "weighted_normalized_fp64"):
        plan = ssu_b200.Plan(tree, table, m)
        units = plan.work_units()
        for _ in range(args.warmup):
            plan.execute(stream.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            plan.execute(stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        dev_ms = e0.elapsed_time(e1) / args.steps
        kernel = plan.pair_kernel()
        plan.close()
        for _ in range(args.warmup):
            ssu_b200.one_off(tree, table, m)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            cf, _, _ = ssu_b200.one_off(tree, table, m)
        e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
        entry = {"device_ms": dev_ms, "e2e_ms": e2e_ms, "units": units, "kernel": kernel}
        if oracle_py.ref_available():
            ref = oracle_py.ref_one_off(tree, table, m, with_timing=True)
            n = table.n_samples
            iu = __import__("numpy").triu_indices(n, 1)
            entry["reference_cpu_ms"] = 1e3 * sum(ref["seconds"])
            entry["max_rel_vs_reference"] = _rel_err(cf, ref["matrix"][iu])[0]
        out[m] = entry
        total_units += units
        total_e2e += e2e_ms
        total_dev += dev_ms
    line = {"metric": METRIC, "value": total_units / (total_dev / 1e3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_dev, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator geometric_1k_tips_128_samples)",
            "config": {"workload": "unweighted_fp64 + weighted_normalized_fp64, 1k-tip tree, 1k features x 128 "
                                   "samples, condensed form"},
            "methods": out,
            "e2e": {"value": total_units / (total_e2e / 1e3), "unit": UNIT, "ms_per_step": total_e2e}}
    print(json.dumps(line), flush=True)


def _batch_e2e(torch, ssu_b200, tree, tables, method, units, steps, **kw):
    """The batch C API end to end (host tables in, host matrices out): one
    untimed call (first-use costs: memory pools, page-locked results, tuning),
    then `steps` timed calls; seconds per call."""
    times = []
    for i in range(steps + 1):
        t0 = time.perf_counter()
        out = ssu_b200.one_off_batch(tree, tables, method, copy=False, **kw)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        del out
        if i > 0:
            times.append(dt)
    sec = sum(times) / len(times)
    return {"seconds": sec, "value": units / sec}


def run_replicates(args):
    """100 rarefied replicates (depth 1,000) of a 10,000-feature x 5,000-sample
    table on a 10,000-tip tree, unweighted and weighted-normalized fp32, every
    replicate of a method in one batch plan replayed as one CUDA graph."""
    torch, stream, flush = _batch_setup()
    import ssu_b200
    import ssu_synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    t0 = time.perf_counter()
    tree, base, reps = ssu_synth.rarefied_replicates_10k_tips_5k_samples(n_replicates=args.replicates)
    gen_s = time.perf_counter() - t0
    methods = ["unweighted_fp32", "weighted_normalized_fp32"]
    per, total_units, total_ms, launches, e2e = {}, 0, 0.0, 0, {}
    clocks = ClockSampler(0)
    for m in methods:
        t0 = time.perf_counter()
        plan = ssu_b200.BatchPlan(tree, reps, m)
        create_s = time.perf_counter() - t0
        units = plan.work_units()
        clocks.start()
        ms = _time_batch(torch, plan, stream, args.steps, args.warmup, flush)
        clk = clocks.stop()
        launches += plan.launches()
        total_units += units
        total_ms += ms
        r0 = plan.results()[0]
        info = {"groups": plan.n_groups(), "tuning": plan.tuning(), "kernel": plan.pair_kernel(),
                "launches_per_step": plan.launches()}
        plan.close()
        # end to end through the batch C API: host tables in, host matrices out
        if args.e2e_steps > 0:
            e2e[m] = _batch_e2e(torch, ssu_b200, tree, reps, m, units, args.e2e_steps)
        per_table_ms = _unbatched_ms(torch, ssu_b200, tree, reps, m, stream)
        single = ssu_b200.Plan(tree, reps[0], m)
        single.execute()
        s0 = single.result()
        single.close()
        per[m] = {"ms_per_step": ms, "value": units / (ms / 1e3), "units": units, **info,
                  "plan_create_s": create_s, "clocks": clk, "one_plan_per_replicate_ms": per_table_ms,
                  "batched_speedup": per_table_ms / ms,
                  "replicate0_vs_one_table_plan_max_rel": _rel_err(r0, s0)[0]}
        # parity of replicate 0 with the reference's own CPU build (fp32 and fp64)
        if oracle_py.ref_available():
            ref64 = oracle_py.ref_one_off(tree, reps[0], m.replace("_fp32", "_fp64"), with_timing=True)
            ref32 = oracle_py.ref_one_off(tree, reps[0], m, with_timing=True)
            per[m]["replicate0_parity"] = {"ours_vs_ref_fp64_max_rel": _rel_err(r0, ref64["matrix"])[0],
                                           "ref_fp32_vs_ref_fp64_max_rel": _rel_err(ref32["matrix"],
                                                                                    ref64["matrix"])[0]}
            e = ref32["n_embedded"]
            n0 = reps[0].n_samples
            per[m]["cpu_reference_replicate0"] = {"seconds": ref32["seconds"][0],
                                                  "value": n0 * (n0 - 1) / 2 * e / ref32["seconds"][0],
                                                  "cores": os.cpu_count()}
    h2d = sum(int(t.indptr.nbytes + t.indices.nbytes + t.data.nbytes) for t in reps)
    d2h = sum(4 * t.n_samples ** 2 for t in reps)
    line = {
        "metric": METRIC, "value": total_units / (total_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator rarefied_replicates_10k_tips_5k_samples; replicates rarefied "
                                                    "on the host, the same tables fed to both engines)",
        "config": {"workload": f"{args.replicates} rarefied replicates (depth 1000) of 10k features x 5000 samples, "
                               "10k-tip tree; unweighted_fp32 + weighted_normalized_fp32; full matrices",
                   "l2": "flushed between steps; embedding > L2", "generation_s": gen_s},
        "methods": per,
        "e2e": {"value": (sum(e["value"] * e["seconds"] for e in e2e.values()) / sum(e["seconds"] for e in e2e.values()))
                if e2e else None, "unit": UNIT, "per_method": e2e, "h2d_bytes_per_step": h2d * len(methods),
                "d2h_bytes_per_step": d2h * len(methods)},
        "gpu_launches": launches * args.steps,
    }
    print(json.dumps(line), flush=True)


def run_uneven_tables(args):
    """64 tables of log-uniform sample counts in [64, 4096] on one 50,000-tip
    tree, generalized (alpha 0.5) and the four variance-adjusted methods in
    fp64, each method one batch plan replayed as one CUDA graph; per-table
    parity with the reference's CPU build on the smaller tables."""
    torch, stream, flush = _batch_setup()
    import ssu_b200
    import ssu_synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    t0 = time.perf_counter()
    tree, tables = ssu_synth.uneven_tables_50k_tips(n_tables=args.uneven_tables, n_tips=args.uneven_tips)
    gen_s = time.perf_counter() - t0
    runs = [("generalized_fp64", False), ("unweighted_fp64", True), ("weighted_normalized_fp64", True),
            ("weighted_unnormalized_fp64", True), ("generalized_fp64", True)]
    small = sorted(range(len(tables)), key=lambda t: tables[t].n_samples)[:6]
    per, total_units, total_ms, launches = [], 0, 0.0, 0
    clocks = ClockSampler(0)
    for m, vaw in runs:
        t0 = time.perf_counter()
        plan = ssu_b200.BatchPlan(tree, tables, m, variance_adjust=vaw, alpha=0.5)
        create_s = time.perf_counter() - t0
        units = plan.work_units()
        clocks.start()
        ms = _time_batch(torch, plan, stream, args.steps, args.warmup, flush)
        clk = clocks.stop()
        launches += plan.launches()
        total_units += units
        total_ms += ms
        res = plan.results()
        info = {"groups": plan.n_groups(), "tuning": plan.tuning(), "kernel": plan.pair_kernel(),
                "launches_per_step": plan.launches()}
        plan.close()
        per_table_ms = _unbatched_ms(torch, ssu_b200, tree, tables, m, stream, variance_adjust=vaw, alpha=0.5)
        entry = {"method": m, "variance_adjust": vaw, "ms_per_step": ms, "value": units / (ms / 1e3),
                 "one_plan_per_table_ms": per_table_ms, "batched_speedup": per_table_ms / ms,
                 "units": units, **info, "plan_create_s": create_s, "clocks": clk}
        if args.e2e_steps > 0:
            entry["e2e"] = _batch_e2e(torch, ssu_b200, tree, tables, m, units, 1, variance_adjust=vaw, alpha=0.5)
        if oracle_py.ref_available():
            worst = 0.0
            for t in small:
                ref = oracle_py.ref_one_off(tree, tables[t], m, variance_adjust=vaw, alpha=0.5)["matrix"]
                worst = max(worst, _rel_err(res[t], ref)[0])
            entry["parity_vs_reference_fp64"] = {"tables": [int(tables[t].n_samples) for t in small],
                                                 "max_rel": worst}
        per.append(entry)
        del res
    e2e_s = sum(e["e2e"]["seconds"] for e in per if "e2e" in e)
    line = {
        "metric": METRIC, "value": total_units / (total_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator uneven_tables_50k_tips)",
        "config": {"workload": f"{len(tables)} tables, sample counts log-uniform in [64, 4096] "
                               f"(total {sum(t.n_samples for t in tables)}), {args.uneven_tips}-tip tree, 1% non-zero; "
                               "generalized a=0.5 and VAW unweighted / weighted_normalized / "
                               "weighted_unnormalized / generalized a=0.5, fp64, full matrices",
                   "l2": "flushed between steps; embedding > L2", "generation_s": gen_s},
        "methods": per,
        "e2e": {"value": total_units / e2e_s if e2e_s else None, "unit": UNIT,
                "ms_per_step": e2e_s * 1e3 if e2e_s else None,
                "h2d_bytes_per_step": sum(int(t.indptr.nbytes + t.indices.nbytes + t.data.nbytes) for t in tables)
                * len(per),
                "d2h_bytes_per_step": sum(8 * t.n_samples ** 2 for t in tables) * len(per),
                "path": "ssu_b200_one_off_batch_inmem_v3 per method, one untimed call first"},
        "gpu_launches": launches * args.steps,
    }
    print(json.dumps(line), flush=True)


def gp_units_e(units, n):
    return int(units // (n * (n - 1) // 2)) if n > 1 else 0


def measure_weighted(args, world, rank, local, stream=None, flush=None, cpu=True):
    """Weighted normalized fp64 on the 20,000-tip / 2,048-sample table: the
    line's dict (rank 0) with an HBM roofline in reference-form bytes."""
    import torch
    import torch.distributed as dist
    import ssu_b200
    tree, table = make_workload(2 + rank, args)
    plan = ssu_b200.Plan(tree, table, args.method)
    units = plan.work_units()
    if stream is None:
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
    if flush is None:
        flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        plan.execute(stream.cuda_stream)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    step_ms, pair_ms = _step_loop(torch, plan, stream, args.steps, barrier, flush)
    clk = clocks.stop()
    launches_per_step = plan.launches()
    n_emb, kernel = plan.n_embedded(), plan.pair_kernel()
    plan.close()

    # end to end through the C API, host buffers in and out
    e2e_ms = []
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        barrier()
        t0 = time.perf_counter()
        m, _ = ssu_b200.one_off_matrix(tree, table, args.method, copy=False)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) * 1e3
        del m  # the caller is done with the result: destroy_mat_full_fp64
        if i > 0:
            e2e_ms.append(dt)
    h2d = int(table.indptr.nbytes + table.indices.nbytes + table.data.nbytes + tree.structure.nbytes +
              tree.lengths.nbytes)
    d2h = int(args.samples) ** 2 * 8
    total_ms, e2e_total, all_units, mean_pair_ms = combine_ranks(
        [sum(step_ms), sum(e2e_ms), float(units), sum(pair_ms) / len(pair_ms)], world, "cuda")
    if rank != 0:
        return None
    value = all_units * args.steps / (total_ms / 1e3)
    peak, _, _, peak_kind = peaks()
    algo_bytes = ALGO_BYTES_PER_UPDATE * units
    achieved = algo_bytes / (mean_pair_ms / 1e3) / 1e9
    sm_mhz = clk["sm_mhz"] if clk else 1965.0
    fp64_peak = 148 * 64 * 2 * sm_mhz * 1e6 / 1e12  # TFLOP/s at the sampled clock
    # dense-form arithmetic the stage stands in for: sub + mul + add per update
    fp64_achieved = 3.0 * units / (mean_pair_ms / 1e3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator lognormal_20k_tips_2048_samples)",
        "config": {"workload": WEIGHTED_WORKLOAD, "method": args.method, "n_samples": args.samples,
                   "n_tips": args.tips, "embedded_branches": n_emb, "pair_kernel": kernel,
                   "l2": "flushed between steps (256 MiB write outside the step events); embedding 655 MB > L2",
                   "per_gpu_units": units},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": read_traffic(), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": algo_bytes,
                     "note": "reference-form bytes (2 fp64 accumulators RMW per 112-node batch) over the "
                             "pair stage; the hybrid kernel keeps its accumulators on chip (traffic = its "
                             "measured DRAM bytes per launch), so the binding bound is instruction issue: "
                             "see fp64_dense_equivalent and the profile summary",
                     "fp64_dense_equivalent": {"achieved_tflops": fp64_achieved,
                                               "peak_tflops_at_clock": fp64_peak,
                                               "frac": fp64_achieved / fp64_peak}},
        "pair_kernel_ms": mean_pair_ms,
        "e2e": {"value": all_units * len(e2e_ms) / (e2e_total / 1e3) if e2e_ms else None, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_total / len(e2e_ms) if e2e_ms else None},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    if world == 1 and cpu:
        try:
            line["cpu_baseline"] = cpu_baseline(tree, table, args.method)
        except Exception as exc:  # the reported baseline never blocks the bench line
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(exc)[:200]}
    return line


def run_weighted(args):
    import torch
    import torch.distributed as dist
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    line = measure_weighted(args, world, rank, local, cpu=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    runners = {"100k-tips-25k-presence": run_presence, "20k-tips-2048-samples": run_weighted,
               "1k-tips-128-samples": run_small, "100-replicates-5k-samples": run_replicates,
               "64-uneven-tables": run_uneven_tables}
    return runners[args.workload](args)


if __name__ == "__main__":
    main()

"""Benchmark of the polygenic-score hot path on B200.

Workload (the reference's bandwidth configuration): 50,000 samples x
1,000,000 variants of SNP-major 2-bit PLINK rows (12.5 GB packed, resident in
HBM), HWE genotypes with p ~ U(0.01, 0.5) and 0.5% missing calls, one FP32
score over all variants with weights ~ N(0, 0.005^2) and 10% of variants
effect-allele-flipped.  Data are synthetic (seeded counter-based generator).

A step is one full scoring pass: reset + accumulate over all rows + finalize
(baseline added, output rows gathered).  ``value`` is genotype*score pairs/s
of the device-timed steps; ``e2e`` is the same metric through the public C ABI
(``gnm_score_run_ex``) from pinned host buffers, host->device copy of the rows
and device->host copy of the results inside the timed region.

``--impl reference`` times the reference's CPU scoring engine (the C
restatement under oracle/, all host threads) on a bounded sample of the same
workload.  Multi-GPU (torchrun): person sharding — every rank scores its own
50,000-person shard of an N x 50,000 cohort with no collective (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "bandwidth_50k_x_1m"
METRIC = "genotype*score pairs/s"
# B200 dense 8-bit integer tensor throughput, NVIDIA's nominal figure (the
# 2:4-sparse figure halved); the pool measures no int8 peak, and twice its
# measured BF16 GEMM understates what the 8-bit kernels reach
INT8_NOMINAL_TOPS = 4500.0
PROFILE = ROOT / "profiles" / "plain_accumulate_bandwidth_50k_x_1m.md"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def peaks_tc():
    """Sustained dense bf16 tensor-core peak (TFLOP/s) and its source."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["bf16_tflops_sustained"]), "measured"
    return 1400.0, "fallback"


def traffic_from_profile(path=PROFILE, key="traffic_bytes_per_launch"):
    """A DRAM-bytes figure recorded from an ncu capture (profiles/), else None."""
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clock, power and clock-event reasons sampled through NVML every 2 ms
    during the timed region (read-only queries; nothing is set)."""

    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown"}

    def __init__(self, index: int, period_s: float = 0.002):
        self.index, self.period = index, period_s
        self.samples = []          # (sm_mhz, power_w, reasons_mask)
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self._nv = None
        self._h = None

    def _handle(self):
        import pynvml as nv
        nv.nvmlInit()
        self._nv = nv
        try:   # match the CUDA device by PCI bus id (CUDA and NVML orders may differ)
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:  # noqa: BLE001 - fall back to the ordinal
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _reasons(self, h):
        nv = self._nv
        f = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        return int(f(h))

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetPowerUsage(h) / 1000.0, self._reasons(h)))
            except Exception:  # noqa: BLE001
                break
            self._stop.wait(self.period)

    def __enter__(self):
        try:
            self._h = self._handle()
            self.max_mhz = self._nv.nvmlDeviceGetMaxClockInfo(self._h, self._nv.NVML_CLOCK_SM)
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:  # noqa: BLE001 - no NVML: report no samples
            self._t = None
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0,
                    "source": "nvml"}
        mask = 0
        for _, _, r in self.samples:
            mask |= r
        return {"sm_mhz": statistics.median(x[0] for x in self.samples),
                "sm_max_mhz": self.max_mhz,
                "power_w": statistics.median(x[1] for x in self.samples),
                "reasons": sorted(n for bit, n in self.REASONS.items() if mask & bit),
                "samples": len(self.samples), "source": "nvml, 2 ms"}


class CpuReferenceSample:
    """The restated reference CPU engine on a bounded sample of the workload:
    all people, a prefix of the variants sized so one pass takes ~target_s."""

    def __init__(self, w, target_s: float, threads: int, prep=None):
        self.w, self.threads, self.full_prep = w, threads, prep
        nv = 512
        while True:  # grow the prefix until one pass is long enough to extrapolate
            self._make(nv)
            t = min(self.time_once() for _ in range(2))
            if t >= min(0.25, target_s) or nv >= w.variants:
                break
            nv = min(w.variants, nv * 4)
        nv = int(min(w.variants, max(nv, nv * target_s / max(t, 1e-4))))
        if nv != self.nv:
            self._make(nv)

    def _make(self, nv):
        from oracle import oracle
        from gnomon_b200 import synth
        from gnomon_b200.prepare import PreparationResult
        w = self.w
        thr = synth.variant_thresholds(w.seed, 0, nv, w.p_lo, w.p_hi, w.missing_rate)
        self.rows = oracle.synth_rows(w.seed, 0, nv, w.people, thr, w.bytes_per_variant)
        self.nv = nv
        if self.full_prep is not None:   # prefix of the workload's own cells
            fp = self.full_prep
            e = int(fp.sparse_row_offsets[nv])
            self.prep = PreparationResult(fp.sparse_weights[:e], fp.sparse_missing_corrections[:e],
                                          fp.sparse_score_columns[:e],
                                          fp.sparse_row_offsets[:nv + 1], fp.score_names,
                                          w.people)
            self.cells = e
            return
        rng = np.random.default_rng(w.seed)
        wt = (rng.standard_normal(nv) * w.sigma).astype(np.float32)
        fl = rng.random(nv) < w.flip_frac
        self.prep = PreparationResult(
            np.where(fl, -wt, wt).astype(np.float32),
            np.where(fl, np.float32(2) * wt, np.float32(0)).astype(np.float32),
            np.zeros(nv, np.uint32), np.arange(nv + 1, dtype=np.uint64), ["S000"], w.people)
        self.nv = nv

    def time_once(self):
        from oracle import oracle
        t0 = time.perf_counter()
        oracle.score_reference(self.rows, self.prep, threads=self.threads)
        return time.perf_counter() - t0

    @property
    def pairs(self):
        """Useful genotype*score pairs of one pass: people x the prefix's cells."""
        return self.w.people * int(self.prep.sparse_row_offsets[-1])

    def describe(self, seconds):
        return (f"{self.w.people} people x {self.nv} variants (prefix of {self.w.variants}), "
                f"K={self.w.scores}, restated reference CPU engine (decide.rs routing, person-major f32 "
                f"mini-batches, variant-major f64) on {self.threads} threads, {seconds:.2f} s/pass")


def sampled_parity(w, prep, person_begin, sums, counts, people_per_window=8):
    """Checker for the bench's own output at full length: the extended-precision
    oracle (oracle/) on four windows of people (first, a third in, two thirds
    in, last) over every variant and score, against the GPU result rows of
    those people.  Runs in the CPU-baseline leg only."""
    from oracle import oracle
    from gnomon_b200 import synth
    from gnomon_b200.prepare import PreparationResult
    P, K, V = prep.num_people_to_score, prep.num_scores, prep.num_reconciled_variants
    n = min(people_per_window, P)
    starts = sorted({0, P // 3, 2 * P // 3, P - n})
    sums = np.asarray(sums).reshape(P, K)
    counts = np.asarray(counts).reshape(P, K)
    worst, exact = 0.0, True
    t0 = time.perf_counter()
    for a in starts:
        rows = np.zeros((V, (n + 3) // 4), np.uint8)
        for v0 in range(0, V, 100_000):
            v1 = min(V, v0 + 100_000)
            thr = synth.variant_thresholds(w.seed, v0, v1 - v0, w.p_lo, w.p_hi, w.missing_rate)
            rows[v0:v1] = synth.synth_rows(w.seed, v0, v1 - v0, n, thr,
                                           person_begin=person_begin + a)
        sub = PreparationResult(prep.sparse_weights, prep.sparse_missing_corrections,
                                prep.sparse_score_columns, prep.sparse_row_offsets,
                                prep.score_names, n, baseline=prep.baseline)
        es, ec = oracle.score_extended(rows, sub)
        got_s, got_c = sums[a:a + n].reshape(-1), counts[a:a + n].reshape(-1)
        exact &= bool(np.array_equal(got_c.astype(np.uint32), ec))
        worst = max(worst, float(oracle.rel_err(got_s, es).max()))
    return {"people": len(starts) * n, "windows": starts, "variants": V, "scores": K,
            "counts_exact": exact, "max_rel_err_vs_extended_oracle": worst,
            "seconds": round(time.perf_counter() - t0, 2),
            "metric": "|a-b| / max(|a|, |b|, 1) (score/tests/gpu_tests.rs:135-147)"}


def reference_arm(args, rank, world):
    from gnomon_b200 import synth
    if rank != 0:
        return
    w = synth.WORKLOADS[WORKLOAD]
    threads = os.cpu_count() or 1
    sample = CpuReferenceSample(w, args.ref_step_s, threads)
    times = []
    for i in range(args.warmup + args.steps):
        t = sample.time_once()
        if i >= args.warmup:
            times.append(t)
    t_used = statistics.median(times)
    value = sample.pairs / t_used
    sample = sample.describe(t_used)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_used * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "samples": w.people, "variants": w.variants,
                       "scores": w.scores, "engine": "cpu reference restatement"},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _engine(args, K):
    from gnomon_b200 import _lib
    if args.engine == "plain":
        return _lib.ENGINE_PLAIN
    if args.engine == "tensor":
        return _lib.ENGINE_TENSOR
    return _lib.ENGINE_PLAIN if K < 8 else _lib.ENGINE_TENSOR   # the library's AUTO rule


def gpu_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from gnomon_b200 import _lib, sharding, synth
    from gnomon_b200.device import DevicePlan, row_pitch, synth_fill
    from gnomon_b200.pipeline import BedSource, PipelineContext, try_run_cuda
    from gnomon_b200.prepare import from_workload

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = synth.WORKLOADS[args.workload]
    if args.variants:
        w = synth.scaled(w, w.people, args.variants)
    # person sharding (weak scaling): the cohort has world x w.people people and
    # rank r owns .fam range [r * w.people, (r + 1) * w.people), generated as
    # that column slice of the cohort; weights are shared, no collective runs
    # in the scoring pass.
    cohort = synth.Workload(w.name, w.people * world, w.variants, w.scores, w.p_lo, w.p_hi,
                            w.missing_rate, w.sigma, w.flip_frac, w.size_lo, w.size_hi,
                            w.config_id)
    shard = sharding.make_shard(from_workload(cohort), rank, world)
    person_begin = shard.start
    P, V, K = shard.num_people, w.variants, w.scores
    bpv = shard.prep.bytes_per_variant
    pitch = row_pitch(bpv)
    prep = shard.prep
    nnz = int(prep.sparse_row_offsets[-1])
    engine = _engine(args, K)
    tensor = engine == _lib.ENGINE_TENSOR
    stream = torch.cuda.Stream(dev)

    # synthetic rows generated on the device, in blocks of 100k variants
    rows = torch.empty((V, pitch), dtype=torch.uint8, device=dev)
    with torch.cuda.stream(stream):
        for v0 in range(0, V, 100_000):
            n = min(100_000, V - v0)
            thr = synth.variant_thresholds(w.seed, v0, n, w.p_lo, w.p_hi, w.missing_rate)
            synth_fill(rows[v0:v0 + n], pitch, v0, n, P, thr, w.seed, stream=stream,
                       person_begin=person_begin)
    stream.synchronize()

    plan = DevicePlan(prep, engine=engine, device=local_rank)
    tuned = None
    def tensor_shape(shape):
        return {"shape": shape, "raster": shape & 1, "narrow": bool(shape & 2),
                "int8_limbs": bool(shape & 4), "sm_pairs": bool(shape & 8)}
    if args.shape:
        # a pinned launch shape, as profiling runs use: kernel:splits (plain,
        # e.g. 512:94) or the tensor engine's shape bits (e.g. 4)
        if ":" in args.shape:
            kern, splits = (int(x) for x in args.shape.split(":"))
            plan.set_shape((kern << 16) | splits)
            tuned = {"kernel": kern, "splits_per_full_tile": splits, "pinned": True}
        else:
            plan.set_shape(int(args.shape))
            tuned = dict(tensor_shape(int(args.shape)), pinned=True)
    elif not args.no_autotune:
        # the library's autotuner picks the launch shape on these resident rows
        # (outside the timed region; the plan is left reset)
        shape = plan.autotune(rows, pitch, stream=stream)
        tuned = ({"kernel": shape >> 16, "splits_per_full_tile": shape & 0xFFFF}
                 if not tensor else tensor_shape(shape))
    tshape = plan.shape if tensor else 0
    sums, counts = plan.outputs()
    grad_s = None
    if args.backward:
        g = torch.Generator(device=dev).manual_seed(w.seed)
        grad_s = torch.randn(P, K, generator=g, device=dev, dtype=torch.float32)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    k_ev = [(ev(), ev()) for _ in range(args.steps)]
    b_ev = [(ev(), ev()) for _ in range(args.steps)]
    s_ev = [(ev(), ev()) for _ in range(args.steps)]
    # Rows smaller than twice the L2 would be served from L2 by the next step:
    # then a buffer of twice the L2 size is written between timed steps, outside
    # each step's events, and the step time is the mean of the per-step events.
    l2_bytes = int(getattr(torch.cuda.get_device_properties(dev), "L2_cache_size", 0) or (126 << 20))
    flush = None
    if V * bpv < 2 * l2_bytes:
        flush = torch.empty(2 * l2_bytes, dtype=torch.uint8, device=dev)

    def step(i=None):
        plan.reset(stream)
        if i is not None:
            k_ev[i][0].record(stream)
        plan.accumulate(rows, pitch, 0, V, stream)
        if i is not None:
            k_ev[i][1].record(stream)
        plan.finalize(sums, counts, stream)
        if grad_s is not None:
            if i is not None:
                b_ev[i][0].record(stream)
            plan.backward(rows, pitch, grad_s, grad_corr=True, stream=stream)
            if i is not None:
                b_ev[i][1].record(stream)

    for _ in range(args.warmup):
        step()
    plan.sync(stream)
    launches_last_step = plan.launches   # the library's own count (reset each step)
    graphs = None
    if args.graph and grad_s is None:
        # the scoring step (reset + accumulate + finalize) and the accumulate
        # alone, each recorded once into a CUDA graph through the library's
        # capture: replays launch the same kernels with no per-launch host work
        step_graph, _, _ = plan.capture(rows, pitch, sums, counts)
        acc_graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(acc_graph, stream=side):
            plan.accumulate(rows, pitch, 0, V, torch.cuda.current_stream())
        graphs = (step_graph, acc_graph)
        for _ in range(args.warmup):
            with torch.cuda.stream(stream):
                step_graph.replay()
        plan.sync(stream)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        start.record(stream)
        for i in range(args.steps):
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.fill_(i & 0xFF)
            s_ev[i][0].record(stream)
            if graphs is None:
                step(i)
            else:
                with torch.cuda.stream(stream):
                    graphs[0].replay()
            s_ev[i][1].record(stream)
        stop.record(stream)
        stop.synchronize()
    plan.sync(stream)
    if graphs is not None:
        # the accumulate's own time: its graph replayed between events
        for i in range(args.steps):
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.fill_(i & 0xFF)
            k_ev[i][0].record(stream)
            with torch.cuda.stream(stream):
                graphs[1].replay()
            k_ev[i][1].record(stream)
        stream.synchronize()
        plan.sync(stream)
    if flush is None:
        ms = start.elapsed_time(stop) / args.steps
    else:
        ms = statistics.mean(a.elapsed_time(b) for a, b in s_ev)
    kernel_ms = statistics.mean(a.elapsed_time(b) for a, b in k_ev)
    bwd_ms = statistics.mean(a.elapsed_time(b) for a, b in b_ev) if grad_s is not None else None
    # tensor: dosage pass + missing pass + finalize; plain: accumulate + finalize
    # per score column; + the backward kernel when requested
    launches_per_step = launches_last_step
    if world > 1:
        t = torch.tensor([ms, kernel_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, kernel_ms = t.tolist()
        dist.barrier()

    # useful genotype*score pairs: people x cells (a score's own variants only;
    # P * V * K when every score covers every variant)
    pairs = P * nnz
    value = world * pairs / (ms / 1e3)
    peak_hbm, peak_kind = peaks()
    if tensor and tshape & 2:
        # narrow engine: M = 128 people, N = limb planes x 16 scores, two MMAs
        # (dosage, missing) per slice; one launch per block.  BF16: 4 + 4
        # planes (the missing operand's padded to four); 8-bit: 4 + 5 planes
        i8 = bool(tshape & 4)
        ptiles, k16 = -(-P // 128), -(-K // 16) * 16
        vpad = -(-V // 128) * 128 if i8 else -(-V // 64) * 64
        executed = 2.0 * ptiles * 128 * vpad * k16 * (9 if i8 else 8)
        # algorithmic: three BF16 weight limbs (hi/mid/lo) x the useful cells
        flops = 2.0 * P * nnz * 3
        achieved = flops / (kernel_ms / 1e3) / 1e12
        pk = peaks_tc()[0]
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                "frac": achieved / pk, "traffic": None,
                "peak_kind": peak_kind + " (bf16 sustained)",
                "kernel": ("gnm_t8_narrow (8-bit limbs; " if i8 else "gnm_tc_narrow (")
                + "dosage + missing MMAs, one pass)",
                "kernel_ms": kernel_ms, "algorithmic_flops_per_launch": flops,
                "algorithmic": "2 x people x cells x 3 weight limbs",
                ("executed_int_ops_per_launch" if i8 else "executed_flops_per_launch"): executed,
                ("executed_tops" if i8 else "executed_tflops"):
                    executed / (kernel_ms / 1e3) / 1e12,
                "row_bytes_gbs": V * bpv * (k16 // 16) / (kernel_ms / 1e3) / 1e9,
                "row_bytes_frac_of_hbm": V * bpv * (k16 // 16) / (kernel_ms / 1e3) / 1e9
                / peak_hbm}
    elif tensor and tshape & 4:
        # 8-bit limbs: 9 integer MMA planes (4 dosage, 4 correction, 1 count)
        # over 256-person x 128-score tiles (256-score tiles on SM pairs) and
        # 128-variant stages; the integer peak is taken as twice the BF16 one
        # (the nominal dense ratio, 4.5 / 2.25)
        mt = 256 if tshape & 8 else 128
        ptiles, kpad, vpad = -(-P // 256), -(-K // mt) * mt, -(-V // 128) * 128
        executed = 2.0 * ptiles * 256 * vpad * kpad * 9
        flops = 2.0 * P * nnz * 3
        achieved = flops / (kernel_ms / 1e3) / 1e12
        pk = peaks_tc()[0]
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                "frac": achieved / pk, "traffic": None,
                "peak_kind": peak_kind + " (bf16 sustained)",
                "kernel": ("gnm_t8_pair (8-bit limbs on SM pairs, cta_group::2; "
                           if tshape & 8 else "gnm_t8_accumulate (8-bit limbs, ")
                + "dosage + missing + count passes)",
                "kernel_ms": kernel_ms, "algorithmic_flops_per_launch": flops,
                "algorithmic": "2 x people x cells x 3 weight limbs",
                "executed_int_ops_per_launch": executed,
                "executed_tops": executed / (kernel_ms / 1e3) / 1e12,
                "executed_frac_of_int8_nominal": executed / (kernel_ms / 1e3) / 1e12
                / INT8_NOMINAL_TOPS,
                "int8_peak": f"{INT8_NOMINAL_TOPS:.0f} TOPS, B200 nominal dense (no measured "
                             "int8 figure on this pool)"}
    elif tensor:
        # executed tensor-core work: 8 limb MMAs (4 dosage, 3 correction, 1 count)
        # over 256-person x 128-score tiles and 64-variant stages
        ptiles, kpad, vpad = -(-P // 256), -(-K // 128) * 128, -(-V // 64) * 64
        executed = 2.0 * ptiles * 256 * vpad * kpad * 8
        flops = 2.0 * P * nnz * 3
        achieved = flops / (kernel_ms / 1e3) / 1e12
        pk = peaks_tc()[0]
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                "frac": achieved / pk, "traffic": None,
                "peak_kind": peak_kind + " (bf16 sustained)",
                "kernel": "gnm_tc_accumulate (dosage + missing passes)", "kernel_ms": kernel_ms,
                "algorithmic_flops_per_launch": flops,
                "algorithmic": "2 x people x cells x 3 weight limbs",
                "executed_flops_per_launch": executed,
                "executed_tflops": executed / (kernel_ms / 1e3) / 1e12,
                "executed_frac": executed / (kernel_ms / 1e3) / 1e12 / pk}
    else:
        # one launch per score column; algorithmic bytes of a launch = packed rows
        # once + one weight record (4 B + flip bit) per cell of that score
        alg_bytes = V * bpv + nnz / K * 4.125
        launch_ms = kernel_ms / K
        achieved = alg_bytes / (launch_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak_hbm, "unit": "GB/s",
                "frac": achieved / peak_hbm,
                "traffic": traffic_from_profile() if args.workload == WORKLOAD and not args.variants
                else None,
                "peak_kind": peak_kind, "kernel": "gnm_plain_accumulate", "kernel_ms": launch_ms,
                "launches_per_step": K, "algorithmic_bytes_per_launch": alg_bytes}

    s_host = sums.cpu().numpy()
    assert np.isfinite(s_host).all()

    # end-to-end through the public C ABI from pinned host memory; every rank
    # runs its shard in lockstep and a step takes the slowest rank's time
    e2e = None
    host, pin_error = None, None
    if not args.no_e2e:
        try:
            host = torch.empty((V, bpv), dtype=torch.uint8, pin_memory=True)
        except RuntimeError as exc:   # pinned host memory exhausted on this rank
            pin_error = str(exc).splitlines()[0][:160]
        if world > 1:   # every rank takes the e2e leg's collectives, or none does
            ok = torch.tensor([0 if host is None else 1], dtype=torch.int32, device=dev)
            dist.all_reduce(ok, op=dist.ReduceOp.MIN)
            if int(ok.item()) == 0:
                host = None
                pin_error = pin_error or "pinned host allocation failed on another rank"
        if host is None:
            e2e = {"unavailable": f"pinned host rows ({V * bpv / 1e9:.1f} GB per rank): {pin_error}"}
    if host is not None:
        host.copy_(rows[:, :bpv])
        src = BedSource(host.numpy().reshape(-1))
        ctx = PipelineContext(prep)
        for _ in range(min(args.warmup, 1)):
            try_run_cuda(ctx, src, engine=engine, device=local_rank)
        times = []
        for _ in range(args.e2e_steps):
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = try_run_cuda(ctx, src, engine=engine, device=local_rank)
            times.append(time.perf_counter() - t0)
        e_s, e_c = out
        assert np.array_equal(e_c.astype(np.int64), counts.cpu().numpy().astype(np.int64))
        rel = np.abs(e_s - s_host).max() / max(1.0, np.abs(s_host).max())
        assert rel < 1e-9, rel
        if world > 1:
            t = torch.tensor(times, dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            times = t.tolist()
        h2d = V * bpv + (K * (V + 64) * 16 if not tensor else nnz * 12 + (V + 1) * 8) + K * 16 + 4
        d2h = P * K * 12 + 4
        e2e = {"value": world * pairs / statistics.median(times), "unit": "pairs/s",
               "h2d_bytes_per_step": world * h2d, "d2h_bytes_per_step": world * d2h,
               "seconds_per_step": statistics.median(times),
               "timing": "wall clock around gnm_score_run_ex (synchronous), pinned host rows"
                         + (", max over ranks" if world > 1 else "")}
        del host

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            smp = CpuReferenceSample(w, args.cpu_s / 3, threads, prep=prep)
            t = statistics.median(smp.time_once() for _ in range(3))
            cpu = {"value": smp.pairs / t, "unit": "pairs/s", "cores": threads, "kind": "port",
                   "sample": smp.describe(t) + ", median of 3"}
            # the oracle as the checker of this run's own output (full length)
            parity = sampled_parity(w, prep, person_begin, s_host, counts.cpu().numpy())
            cpu["parity_of_the_timed_output"] = parity
            assert parity["counts_exact"], parity
            assert parity["max_rel_err_vs_extended_oracle"] <= 1e-6, parity
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("f32" if not tensor else
                      "s8 limbs x u8 genotypes, s32 accumulate" if tshape & 4 else
                      "bf16 limbs, f32 accumulate"), "data": "synthetic",
            "config": {"workload": w.name, "samples": P, "variants": V, "scores": K,
                       "cells": nnz, "useful_pairs_per_step": P * nnz,
                       "dense_pairs_per_step": P * V * K,
                       "packed_bytes": V * bpv,
                       "engine": ("plain (int32 stage-table LUT on CUDA cores, FP64 reduce)"
                                  if not tensor else
                                  "tcgen05 kind::i8" + (" on SM pairs (cta_group::2)"
                                                        if tshape & 8 else "")
                                  + ", 8-bit limbs (4 dosage + 4 correction + count), "
                                  "FP64 block reduce" if tshape & 4 else
                                  "split-BF16 tcgen05 (4+3 limbs), FP64 block reduce"),
                       "parallelism": f"person-shard x{world}" if world > 1 else "single GPU",
                       "launch_shape": tuned if tuned is not None else "default (not autotuned)",
                       "timing": ("each step one replay of a CUDA graph of reset + accumulate + "
                                  "finalize (DevicePlan.capture)" if graphs is not None else
                                  "each step reset + accumulate + finalize launched from Python"),
                       "l2": (f"inputs ({V * bpv / 1e9:.1f} GB) larger than L2 "
                              f"({l2_bytes >> 20} MB); no flush" if flush is None else
                              f"inputs ({V * bpv / 1e6:.1f} MB) fit in L2 ({l2_bytes >> 20} MB): "
                              f"a {2 * l2_bytes >> 20} MB buffer is written between timed steps, "
                              "outside each step's CUDA events (mean of per-step events)")},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks.summary(),
        }
        if bwd_ms is not None:
            # tcgen05 GEMM: M = variants (tiles of 128), N = 4 limbs x 16 scores per
            # score tile, K = people (stages of 128 on 8-bit limbs, the default);
            # executed work and packed-row bytes
            v_pad = -(-V // 128) * 128
            p_pad = -(-w.people // 128) * 128
            k_pad = -(-K // 16) * 16
            bw_flops = 2.0 * v_pad * p_pad * 4 * k_pad
            bw_tflops = bw_flops / (bwd_ms / 1e3) / 1e12
            line["backward"] = {
                "ms": bwd_ms, "pairs_per_s": P * V * K / (bwd_ms / 1e3),
                "kernel": "gnm_t8_backward (8-bit dS limbs, + limb build)",
                "executed_tops": bw_tflops,
                "executed_frac_of_int8_nominal": bw_tflops / INT8_NOMINAL_TOPS,
                "row_bytes_gbs": V * bpv * (k_pad // 16) / (bwd_ms / 1e3) / 1e9}
        print(json.dumps(line), flush=True)
    plan.close()


def stream_arm(args, rank, world, local_rank):
    """Biobank-style streaming: rows live in pinned host memory and are copied
    block by block (double-buffered, copy stream overlapped with the compute
    stream) into HBM while the previous block is scored.  The full packed matrix
    does not fit host RAM, so two pre-generated blocks are cycled; every block
    is scored against the real weights of its variant range."""
    import torch
    from gnomon_b200 import _lib, synth
    from gnomon_b200.device import DevicePlan, row_pitch, synth_fill
    from gnomon_b200.prepare import from_workload

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = synth.WORKLOADS[args.workload]
    if args.variants:
        w = synth.scaled(w, w.people, args.variants)
    P, V, K = w.people, w.variants, w.scores
    bpv, B = w.bytes_per_variant, args.stream_block
    pitch = row_pitch(bpv)
    prep = from_workload(w)
    engine = _engine(args, K)
    plan = DevicePlan(prep, engine=engine, device=local_rank)
    comp, copy = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    dbuf = [torch.empty((B, pitch), dtype=torch.uint8, device=dev) for _ in range(2)]
    pool = []
    for i in range(2):   # two distinct blocks of synthetic rows, kept in pinned memory
        thr = synth.variant_thresholds(w.seed, i * B, B, w.p_lo, w.p_hi, w.missing_rate)
        synth_fill(dbuf[i], pitch, i * B, B, P, thr, w.seed, stream=comp)
        h = torch.empty((B, pitch), dtype=torch.uint8, pin_memory=True)
        comp.synchronize()
        h.copy_(dbuf[i])
        pool.append(h)
    sums, counts = plan.outputs()
    nblk = -(-V // B)
    copied = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]

    def one_pass():
        plan.reset(comp)
        for b in range(nblk):
            s = b % 2
            n = min(B, V - b * B)
            copy.wait_event(consumed[s])   # the block that last used buffer s is scored
            with torch.cuda.stream(copy):
                dbuf[s][:n].copy_(pool[b % 2][:n], non_blocking=True)
                copied[s].record(copy)
            comp.wait_event(copied[s])
            plan.accumulate(dbuf[s], pitch, b * B, n, comp)
            consumed[s].record(comp)
        plan.finalize(sums, counts, comp)

    for _ in range(args.warmup):
        one_pass()
    plan.sync(comp)
    # pinned host -> device copy rate on its own (the link this mode is bound by)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(copy):
        t0.record(copy)
        for r in range(3):
            dbuf[r % 2].copy_(pool[r % 2], non_blocking=True)
        t1.record(copy)
    t1.synchronize()
    h2d_peak = 3 * B * pitch / (t0.elapsed_time(t1) / 1e3) / 1e9
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record(comp)
        for _ in range(args.steps):
            one_pass()
        stop.record(comp)
        stop.synchronize()
    plan.sync(comp)
    ms = start.elapsed_time(stop) / args.steps
    h2d_bytes = V * pitch
    cells = int(prep.sparse_row_offsets[-1])
    line = {"metric": METRIC, "value": P * cells / (ms / 1e3), "unit": "pairs/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if engine == _lib.ENGINE_PLAIN else "bf16 limbs, f32 accumulate",
            "data": "synthetic (two pinned host blocks cycled through all variant blocks)",
            "config": {"workload": w.name, "samples": P, "variants": V, "scores": K,
                       "cells": cells, "useful_pairs_per_step": P * cells,
                       "dense_pairs_per_step": P * V * K, "block_variants": B,
                       "blocks": nblk, "packed_bytes": V * bpv,
                       "engine": "tensor" if engine == _lib.ENGINE_TENSOR else "plain"},
            "stream": {"h2d_bytes_per_pass": h2d_bytes,
                       "h2d_gbs_achieved": h2d_bytes / (ms / 1e3) / 1e9,
                       "h2d_gbs_copy_alone": h2d_peak},
            "gpu_launches": plan.launches * args.steps,
            "clocks": clocks.summary()}
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        smp = CpuReferenceSample(w, args.cpu_s / 3, threads, prep=prep)
        t = statistics.median(smp.time_once() for _ in range(3))
        line["cpu_baseline"] = {"value": smp.pairs / t, "unit": "pairs/s", "cores": threads,
                                "kind": "port", "sample": smp.describe(t) + ", median of 3"}
    print(json.dumps(line), flush=True)
    plan.close()


def pgen_arm(args, rank, world, local_rank):
    """PLINK 2 .pgen -> .bed rows on the device (gnm_pgen_*): a synthetic
    50,000-sample .pgen of ``--pgen`` variants with linkage (runs of 17
    variants, 2% of calls redrawn per step, REF/ALT swaps), so the file mixes
    2-bit, 1-bit, fill and LD-compressed records as real cohorts do.  2048
    distinct variants are encoded and repeated (each repeat keeps its LD
    anchors).  ``value``: variants/s of device-timed decodes with the file
    resident in HBM; ``e2e``: the one-shot ``gnm_pgen_decode_device`` from host
    bytes, upload of the file included."""
    import torch
    from gnomon_b200 import synth
    from gnomon_b200.device import row_pitch
    from gnomon_b200.pgen import PgenFile, pgen_dims
    from gnomon_b200 import _lib
    import ctypes as C

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = synth.WORKLOADS[args.workload]
    distinct = 2048
    reps = max(1, args.pgen // distinct)
    cats = synth.pgen_ld_categories(w.seed, distinct, w.people)
    types, recs = synth._pgen_records(cats)      # record types and bodies, for the accounting
    data = np.frombuffer(synth._pgen_file(w.people, types * reps, recs * reps), np.uint8)
    V, n = pgen_dims(data)
    bpv = (n + 3) // 4
    pitch = row_pitch(bpv)
    rows = torch.empty(V * pitch, dtype=torch.uint8, device=dev)
    kinds = np.bincount(np.asarray(types * reps) & 7, minlength=8)
    record_bytes = reps * sum(len(r) for r in recs)
    n_ld = int(kinds[2] + kinds[3])
    algo_bytes = record_bytes + V * bpv                   # records read + rows written
    s = torch.cuda.Stream(dev)
    pg = PgenFile(data, device=local_rank)
    for _ in range(args.warmup):
        pg.decode(rows, pitch, stream=s)
    pg.check(s)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        for a, b in ev:
            a.record(s)
            pg.decode(rows, pitch, stream=s)
            b.record(s)
        s.synchronize()
    pg.check(s)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms = statistics.mean(step_ms)
    # end to end: host bytes (pinned, as the e2e inputs are) -> rows through
    # the one-shot C ABI call
    lib = _lib.load()
    pinned = torch.empty(data.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = data
    e2e_s = []
    for i in range(max(1, args.e2e_steps) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e = _lib.gnm_error()
        _lib.check(lib.gnm_pgen_decode_device(pinned.data_ptr(), data.nbytes, local_rank,
                                              rows.data_ptr(), pitch, s.cuda_stream, C.byref(e)), e)
        if i:
            e2e_s.append(time.perf_counter() - t0)
    e2e = statistics.median(e2e_s)
    hbm, src = peaks()
    achieved = algo_bytes / (ms / 1e3) / 1e9
    traffic_pv = traffic_from_profile(ROOT / "profiles" / "pgen_decode_50k_x_16k.md",
                                      "traffic_bytes_per_variant")
    line = {"metric": "pgen variants decoded/s", "value": V / (ms / 1e3), "unit": "variants/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded HWE categories with linkage, 2048 distinct variants "
                    "repeated)",
            "config": {"workload": f"pgen_decode_{n}_x_{V}", "samples": n, "variants": V,
                       "file_bytes": int(data.nbytes), "record_bytes": record_bytes,
                       "rows_bytes": V * bpv, "ld_records": n_ld,
                       "record_types": {str(k): int(c) for k, c in enumerate(kinds) if c},
                       "l2": "rows written per step exceed L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_source": src,
                         "algorithmic_bytes_per_step": algo_bytes,
                         "kernels": "gnm_pgen_direct + gnm_pgen_ld (one decode = both)",
                         "traffic": traffic_pv * V if traffic_pv else None,
                         "traffic_source": "ncu DRAM bytes per variant of the 16,384-variant "
                                           "case, times this case's variants"},
            "e2e": {"value": V / e2e, "unit": "variants/s", "h2d_bytes_per_step": int(data.nbytes),
                    "d2h_bytes_per_step": 8, "seconds": e2e},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks.summary()}
    if rank == 0 and not args.no_cpu:
        from oracle import pgen_oracle
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        pgen_oracle.decode_to_bed_c(data, threads=threads)
        t = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": V / t, "unit": "variants/s", "cores": threads,
                                "kind": "port",
                                "sample": f"C restatement of the decode (oracle/pgen_oracle.c) on "
                                          f"the whole file, {V} variants x {n} samples, {t:.2f} s"}
    pg.close()
    print(json.dumps(line), flush=True)


def project_arm(args, rank, world, local_rank):
    """HWE-PCA projection blocks (gnm_project_*): 50,000 samples onto 20 axes,
    ``--project`` variants in blocks of 32,768 (rows, coefficients and
    loadings staged from host memory per block, as the reference stages
    them; the rows from pinned host memory).  ``value`` is genotype x
    component pairs/s through the host call; the per-block host->device copy
    of the rows is inside the timed region."""
    import torch
    from gnomon_b200 import synth
    from gnomon_b200.device import row_pitch, synth_fill
    from gnomon_b200.project import Projector, hwe_coefficients

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = synth.WORKLOADS[args.workload]
    n, k, B = w.people, 20, 32768
    nblk = max(1, args.project // B)
    bpv = (n + 3) // 4
    pitch = row_pitch(bpv)
    thr = synth.variant_thresholds(w.seed, 0, B, w.p_lo, w.p_hi, w.missing_rate)
    d = torch.empty(B * pitch, dtype=torch.uint8, device=dev)
    synth_fill(d, pitch, 0, B, n, thr, w.seed)
    pinned = torch.empty((B, bpv), dtype=torch.uint8, pin_memory=True)   # e2e inputs: pinned
    pinned.copy_(d.view(B, pitch)[:, :bpv])
    rows = pinned.numpy()
    rng = np.random.default_rng(w.seed)
    freqs = rng.uniform(w.p_lo, w.p_hi, B)
    coeffs = hwe_coefficients(freqs, np.sqrt(2 * freqs * (1 - freqs)))
    loadings = (rng.standard_normal((B, k)) / np.sqrt(B * nblk)).astype(np.float32)
    with Projector(n, k, device=local_rank) as pj:
        for _ in range(max(1, args.warmup)):
            pj.block(rows, coeffs, loadings)
    secs = []
    with ClockSampler(local_rank) as clocks:
        for _ in range(args.steps):
            with Projector(n, k, device=local_rank) as pj:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                for _ in range(nblk):
                    pj.block(rows, coeffs, loadings)
                out = pj.scores()
                secs.append(time.perf_counter() - t0)
    s = statistics.median(secs)
    pairs = n * B * nblk * k
    line = {"metric": "projection genotype*component pairs/s", "value": pairs / s,
            "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 tables, f64 sums",
            "data": "synthetic HWE genotypes (one 32,768-variant block in pinned host "
                    "memory, repeated)",
            "config": {"workload": f"project_{n}_x_{B * nblk}_k{k}", "samples": n,
                       "variants": B * nblk, "components": k, "block_variants": B,
                       "blocks": nblk},
            "e2e": {"value": pairs / s, "unit": "pairs/s",
                    "h2d_bytes_per_step": nblk * B * (bpv + 4 * (3 + k)),
                    "d2h_bytes_per_step": nblk * n * k * 8, "seconds": s},
            "gpu_launches": nblk * (3 * k + 1),   # per block: repitch; per axis: tables, accumulate, finalize
            "clocks": clocks.summary()}
    if rank == 0 and not args.no_cpu:
        from oracle import project_oracle
        m = 512
        t0 = time.perf_counter()
        project_oracle.project_block(rows[:m], n, coeffs[:m], loadings[:m])
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n * m * k / tc, "unit": "pairs/s",
                                "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"numpy float64 oracle (unpack + matmul) on the first {m} "
                                          f"variants x {n} samples x {k} axes, {tc:.2f} s"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gnomon_b200", choices=["gnomon_b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-s", type=float, default=12.0, help="CPU baseline sample seconds")
    ap.add_argument("--ref-step-s", type=float, default=4.0)
    ap.add_argument("--workload", default=WORKLOAD, help="synthetic workload name")
    ap.add_argument("--engine", default="auto", choices=["auto", "plain", "tensor"])
    ap.add_argument("--backward", action="store_true", help="add dW = G^T dS to each step")
    ap.add_argument("--stream-block", type=int, default=0,
                    help="stream rows from pinned host memory in blocks of this many variants")
    ap.add_argument("--graph", action="store_true",
                    help="time steps as replays of one CUDA graph of the step (plan capture)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the plan's default launch shape instead of autotuning it")
    ap.add_argument("--shape", default="",
                    help="pin the plain engine's launch shape, kernel:splits (e.g. 512:94)")
    ap.add_argument("--variants", type=int, default=0,
                    help="override the variant count (small cases for profiler captures)")
    ap.add_argument("--pgen", type=int, default=0,
                    help="time .pgen -> .bed decoding of this many variants instead")
    ap.add_argument("--project", type=int, default=0,
                    help="time HWE-PCA projection blocks over this many variants instead")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.stream_block:
        stream_arm(args, rank, world, local_rank)
        return
    if args.pgen:
        # a one-GPU measurement of the decoder: under torchrun only rank 0 runs it
        if rank == 0:
            pgen_arm(args, rank, 1, local_rank)
        return
    if args.project:
        if rank == 0:
            project_arm(args, rank, 1, local_rank)
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=None)
    try:
        gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

#!/usr/bin/env python3
"""Benchmark: LDE + Merkle commit throughput on B200 (elements/s).

Workload (one step = one commit on each GPU): 256 columns of 2^15 Goldilocks
coefficients, rate_bits 3 -> coset LDE of 2^18 points per column, bit-reversed
into 2^18 leaf rows of 256 elements, Poseidon2 Merkle forest with cap height 4.
Unit of work: one committed LDE element (2^18 * 256 = 67,108,864 per step).
Synthetic seeded field data (splitmix64, values in [0, p)).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 run under torchrun; every rank commits its own job (weak scaling,
no data-path collective).  Rank 0 prints one JSON line.

At N = 1 the same line also carries the uneven batch (64 jobs, one CUDA graph
per memory wave vs one plain C-ABI call per stage per job: batched_over_plain,
batched_elems_per_s, plain_elems_per_s, and the batch's Poseidon permutation
floor), the alternative-hash forests (Poseidon2, Monolith and Keccak over 2^20
leaves x 135, in one batch and alone: alt_hash_forests) and the serving stream
(Poisson requests at 0.7 of the serial capacity: serve_p50_ms, serve_p99_ms,
delivered and offered elements/s); --no-extras skips them.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P = 0xFFFFFFFF00000001
METRIC = "LDE+Merkle commit elems/s"
LG_N, RATE, COLS, CAP, HASH = 15, 3, 256, 4, 3  # Poseidon2
HBM_FALLBACK_GBS = 6650.0
P2_MULS_PER_PERM = 736  # full-width multiplies per Poseidon2 permutation


def field_data(seed, n):
    """Seeded field elements in [0, p) (splitmix64 counters, values >= p folded)."""
    k = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64((seed << 32) & 0xFFFFFFFFFFFFFFFF) + (k + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return np.where(z >= np.uint64(P), z - np.uint64(P), z)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []  # (monotonic time, csv line)
        self.window = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a while to start sampling: wait for its first
            # line so the timed region that follows is covered
            t_end = time.monotonic() + 5.0
            while not self.lines and time.monotonic() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark(self, t0, t1):
        """The timed region, in time.monotonic() seconds: only samples taken
        inside it count (all samples when none fell inside)."""
        self.window = (t0, t1)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [ln for t, ln in self.lines]
        if self.window:
            inside = [ln for t, ln in self.lines if self.window[0] <= t <= self.window[1]]
            lines = inside or lines
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_commit_sample(lg_n, cols, threads):
    """One commit of the workload's shape at 2^lg_n coefficients on the host:
    LDE by the oracle's CPU restatement (the reference has no CPU NTT), bit
    reversal, then the reference's own fill_digests_buf_linear_cpu when built
    (oracle/_ref), else the oracle Merkle.  Returns (seconds, elements, kind)."""
    from oracle import oracle as O
    os.environ["OMP_NUM_THREADS"] = str(threads)
    O.set_threads(threads)
    c = field_data(99, cols << lg_n)
    t0 = time.perf_counter()
    rows = O.lde_rows(c, lg_n, RATE, cols)
    if O.ref_available():
        O.ref_merkle(rows, cols, CAP, HASH)
        kind = "reference"
    else:
        O.merkle(rows, cols, CAP, HASH)
        kind = "port"
    return time.perf_counter() - t0, (cols << (lg_n + RATE)), kind


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    lg = args.cpu_lg
    for _ in range(args.warmup):
        cpu_commit_sample(lg, COLS, threads)
    times, elems, kind = [], 0, "port"
    for _ in range(args.steps):
        t, e, kind = cpu_commit_sample(lg, COLS, threads)
        times.append(t)
        elems = e
    total = sum(times)
    value = elems * len(times) / total
    sample = ("%d cols x 2^%d coeffs, rate_bits %d (2^%d leaves x %d), Poseidon2 cap %d per step; LDE: CPU restatement "
              "(the reference has no CPU NTT), Merkle: %s" % (COLS, lg, RATE, lg + RATE, COLS, CAP,
                                                              "reference fill_digests_buf_linear_cpu" if kind ==
                                                              "reference" else "oracle port"))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "elems/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": config_dict(), "cpu_baseline": {"value": value, "unit": "elems/s", "cores": threads, "kind": kind,
                                                  "sample": sample},
        "e2e": {"value": value, "unit": "elems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict():
    return {"workload": "lde_poseidon2_commit: 256 cols x 2^15 coeffs, rate_bits 3 -> 2^18 leaves x 256, "
                        "Poseidon2 Merkle cap_height 4",
            "cols": COLS, "lg_n": LG_N, "rate_bits": RATE, "leaves": 1 << (LG_N + RATE), "cap_height": CAP,
            "hash": "poseidon2", "parallelism": "replicas", "l2": "flushed between steps (256 MiB write)"}


def run_ours(args, rank, world):
    import torch
    import zeknox_b200 as zk

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)  # every torch op below is ordered with the commits
    sptr = stream.cuda_stream
    n, N = 1 << LG_N, 1 << (LG_N + RATE)
    elems = N * COLS
    host = torch.from_numpy(field_data(1000 + rank, COLS * n).view(np.int64).copy())
    inp = host.to("cuda")
    host_pinned = host.pin_memory()
    leaves = torch.empty(N * COLS, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, CAP)
    dig = torch.empty(n_dig * 4, dtype=torch.int64, device="cuda")
    caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
    caps_host = torch.empty(n_cap * 4, dtype=torch.int64).pin_memory()
    job = zk.commit_job(LG_N, RATE, COLS, CAP, HASH, inp, leaves, dig, caps)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        zk.commit(dev, job, stream=sptr)
    torch.cuda.synchronize()

    # ---- headline: device-resident inputs, one commit per step
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches0 = zk.launch_count()
    t_timed0 = time.monotonic()
    for s in range(args.steps):
        flush.fill_(s & 0xFF)  # evict the previous step's data from L2 (untimed)
        ev[s][0].record(stream)
        zk.commit(dev, job, stream=sptr)
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    sampler.mark(t_timed0, time.monotonic())
    launches = zk.launch_count() - launches0
    barrier()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = elems * world * args.steps / (total_ms * 1e-3)

    # ---- end to end through the public API: pinned host input -> commit -> caps to host
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    # the public API reads the coefficients straight from pinned host memory
    # (copied in column chunks that overlap the LDE of the previous chunk)
    job_host = zk.commit_job(LG_N, RATE, COLS, CAP, HASH, host_pinned, leaves, dig, caps)
    zk.commit(dev, job_host, stream=sptr)
    torch.cuda.synchronize()
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        ev2[s][0].record(stream)
        zk.commit(dev, job_host, stream=sptr)
        caps_host.copy_(caps, non_blocking=True)
        ev2[s][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in ev2)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = elems * world * args.steps / (e2e_ms * 1e-3)

    # ---- per-stage timing for the rooflines (same stream, same buffers)
    reps = max(3, args.steps)
    lde_ms, mk_ms = [], []
    dstream = torch.cuda.default_stream()
    for s in range(reps):
        flush.fill_(s & 0xFF)
        a, b, c, d = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        a.record(stream)
        zk.lde_rows(dev, leaves, inp, LG_N, RATE, COLS, 7, stream=sptr)
        b.record(stream)
        torch.cuda.synchronize()
        # the Merkle entry point queues on the legacy default stream, like the reference
        c.record(dstream)
        zk.load().fill_digests_buf_linear_gpu_with_gpu_ptr(zk._ptr(dig), zk._ptr(caps), zk._ptr(leaves), n_dig, n_cap,
                                                            N, COLS, CAP, HASH, dev)
        d.record(dstream)
        torch.cuda.synchronize()
        lde_ms.append(a.elapsed_time(b))
        mk_ms.append(c.elapsed_time(d))
    lde_t = statistics.median(lde_ms) * 1e-3
    mk_t = statistics.median(mk_ms) * 1e-3
    hbm, hbm_src = peaks()
    lde_bytes = 8 * (n + N) * COLS
    traffic, prof = None, {}
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            prof = json.load(f)
        traffic = prof.get("lde_rows_config2_bytes_per_call")
    except Exception:
        pass
    roofline = {"bound": "hbm", "kernel": "ntt_pass_kernel x2 (fused coset LDE -> leaf rows)",
                "achieved": lde_bytes / lde_t / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": lde_bytes / lde_t / 1e9 / hbm, "traffic": traffic, "peak_source": hbm_src + " hbm_gbs",
                "algorithmic_bytes": lde_bytes, "ms": lde_t * 1e3}
    # the fused LDE's integer roofline: its executed instructions per output
    # element (ncu, profiles/) against the instruction floor of its
    # arithmetic (the primitives' measured costs times their counts per
    # element), and the ALU pipe's utilisation in that capture
    roofline_lde_int = None
    if prof.get("lde_rows_config2_inst_per_elem"):
        inst, floor = prof["lde_rows_config2_inst_per_elem"], prof["lde_rows_inst_floor_per_elem"]
        roofline_lde_int = {"bound": "int issue (ALU pipe)", "achieved_inst_per_elem": inst,
                            "floor_inst_per_elem": floor, "frac": floor / inst,
                            "alu_pipe_pct": prof.get("lde_rows_config2_alu_pipe_pct"),
                            "source": "ncu capture of one call (profiles/lde_rows_lg15_rate3.md)"}
    # compute_transpose_rev of the workload's evaluations (column-major 256 x
    # 2^18 -> bit-reversed leaf-major), the HBM-bound kernel of the unfused path
    ev_cols = torch.empty(N * COLS, dtype=torch.int64, device="cuda")
    tr_bytes = 16 * N * COLS

    def time_transpose(form):
        zk.tune_set("transpose_bulk", form)
        ms = []
        for s in range(reps + 1):
            flush.fill_(s & 0xFF)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            zk.transpose_rev(dev, leaves, ev_cols, LG_N + RATE, COLS, stream=sptr)
            b.record(stream)
            torch.cuda.synchronize()
            if s:
                ms.append(a.elapsed_time(b))
        return statistics.median(ms) * 1e-3

    try:
        tr_16 = time_transpose(0)  # 16-byte loads through registers
        tr_t = time_transpose(zk.TRANSPOSE_AUTO)  # bulk-async copies into shared-memory stages (the default)
    finally:
        zk.tune_set("transpose_bulk", zk.TRANSPOSE_AUTO)
    roofline_transpose = {"bound": "hbm", "kernel": "transpose_rev_bulk_kernel (compute_transpose_rev, 256 x 2^18)",
                          "achieved": tr_bytes / tr_t / 1e9, "peak": hbm, "unit": "GB/s",
                          "frac": tr_bytes / tr_t / 1e9 / hbm, "algorithmic_bytes": tr_bytes, "ms": tr_t * 1e3,
                          "peak_source": hbm_src + " hbm_gbs",
                          "v2_16byte_form": {"ms": tr_16 * 1e3, "frac": tr_bytes / tr_16 / 1e9 / hbm}}
    perms = N * ((COLS + 7) // 8) + (N - 1)
    mul_rate = zk.measure_mul_rate(dev)
    achieved_mul = perms * P2_MULS_PER_PERM / mk_t
    roofline_hash = {"bound": "int", "kernel": "merkle_leaf_levels_kernel<Poseidon2> + fold + tail", "achieved": achieved_mul / 1e9,
                     "peak": mul_rate / 1e9, "unit": "Gmul/s", "frac": achieved_mul / mul_rate if mul_rate > 0 else None,
                     "perms_per_s": perms / mk_t, "leaves_per_s": N / mk_t, "ms": mk_t * 1e3,
                     "peak_source": "measured register-loop Goldilocks multiply (zeknox_measure_mul_rate)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        t, e, kind = cpu_commit_sample(args.cpu_lg, COLS, threads)
        cpu = {"value": e / t, "unit": "elems/s", "cores": threads, "kind": kind,
               "sample": "one commit of %d cols x 2^%d coeffs (rate 3, Poseidon2 cap 4): LDE by the CPU restatement, "
                         "Merkle by %s" % (COLS, args.cpu_lg, "the reference's fill_digests_buf_linear_cpu"
                                           if kind == "reference" else "the oracle port")}
    # the uneven batch (batched graph vs plain per-call) and the serving
    # stream, on this GPU after the headline (one GPU only: they are
    # single-GPU workloads)
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        del ev_cols
        torch.cuda.empty_cache()
        batch = measure_batch(args.batch_steps, args.budget_gb)
        forests = measure_hashes(3)
        serve = measure_serve(args.requests)
        extras = {"batched_over_plain": batch["batched_over_plain"],
                  "batched_elems_per_s": batch["batched_elems_per_s"],
                  "plain_elems_per_s": batch["plain_elems_per_s"],
                  "serve_p50_ms": serve["p50_ms"], "serve_p99_ms": serve["p99_ms"],
                  "serve_delivered_elems_per_s": serve["delivered_elems_per_s"],
                  "serve_offered_elems_per_s": serve["offered_elems_per_s"],
                  "serve_device_loop_p50_ms": serve["device_loop"]["p50_ms"],
                  "serve_device_loop_p99_ms": serve["device_loop"]["p99_ms"],
                  "forests_batched_leaves_per_s": forests["batched_leaves_per_s"],
                  "uneven_batch": batch, "alt_hash_forests": forests, "serving": serve}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "elems/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded splitmix64 field elements)",
            "config": config_dict(), "roofline": roofline, "roofline_lde_int": roofline_lde_int,
            "roofline_hash": roofline_hash,
            "roofline_transpose": roofline_transpose, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "elems/s", "h2d_bytes_per_step": COLS * n * 8,
                    "d2h_bytes_per_step": n_cap * 32},
            "gpu_launches": launches, "clocks": clocks,
            "stage_ms": {"lde_rows": lde_t * 1e3, "merkle": mk_t * 1e3},
            **extras,
        }
        print(json.dumps(line), flush=True)


def run_stage(args):
    """One stage of the workload at 2^lg_n coefficients per column, for ncu captures."""
    import torch
    import zeknox_b200 as zk
    lg = args.lg_n
    if args.only == "ntt":
        # compute_batched_ntt of COLS natural-order columns of 2^lg_n, in place
        x = dev_field(COLS << lg, 5)
        for _ in range(args.warmup + args.steps):
            zk.ntt_batch(0, x, lg, COLS)
        torch.cuda.synchronize()
        print("stage ntt lg_n %d done, %d launches" % (lg, zk.launch_count()))
        return
    n, N = 1 << lg, 1 << (lg + RATE)
    inp = torch.from_numpy(field_data(5, COLS * n).view(np.int64).copy()).cuda()
    leaves = torch.empty(N * COLS, dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(N, CAP)
    dig = torch.empty(n_dig * 4, dtype=torch.int64, device="cuda")
    caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
    zk.lde_rows(0, leaves, inp, lg, RATE, COLS)
    ev_cols = torch.empty(N * COLS, dtype=torch.int64, device="cuda") if args.only == "transpose" else None
    for _ in range(args.warmup + args.steps):
        if args.only == "lde":
            zk.lde_rows(0, leaves, inp, lg, RATE, COLS)
        elif args.only == "transpose":
            zk.transpose_rev(0, leaves, ev_cols, lg + RATE, COLS)
        else:
            zk.fill_digests_buf_linear_gpu(dig, caps, leaves, N, COLS, CAP, args.hash)
    torch.cuda.synchronize()
    print("stage %s lg_n %d done, %d launches" % (args.only, lg, zk.launch_count()))


def dev_field(numel, seed):
    """Seeded uniform field elements generated on the GPU (int64 bit patterns)."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    x = torch.randint(-(1 << 63), (1 << 63) - 1, (numel,), dtype=torch.int64, device="cuda", generator=g)
    # u64 values >= p are the int64 values in [-(2^32 - 1), -1]: subtract p (= add 2^32 - 1)
    big = (x < 0) & (x >= -((1 << 32) - 1))
    return torch.where(big, x + ((1 << 32) - 1), x)


def uneven_jobs(count=64, seed=3):
    """The uneven-batch workload: log2 size U{10..20}, columns U{8..400},
    rate_bits U{1,2,3}, Poseidon, cap_height min(4, log2 leaves)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(count):
        lg = int(rng.integers(10, 21))
        cols = int(rng.integers(8, 401))
        rate = int(rng.integers(1, 4))
        jobs.append({"lg_n": lg, "cols": cols, "rate": rate, "cap": min(4, lg + rate), "hash": 0, "seed": 3000 + j})
    return jobs


def perms_of(n_leaves, leaf_size, cap_height):
    """Permutations of a width-12 sponge forest: ceil(leaf_size / 8) per leaf
    (none for leaves of <= 4 elements), one per internal node."""
    leaf = n_leaves * ((leaf_size + 7) // 8) if leaf_size > 4 else 0
    return leaf + n_leaves - (1 << cap_height)


def poseidon_perm_rate(steps=3):
    """Poseidon permutations/s of one 2^20 x 135 forest, cap height 4 (CUDA
    events, L2 flushed): the throughput the uneven batch's floor is taken at."""
    import torch
    import zeknox_b200 as zk
    nl, ls, ch = 1 << 20, 135, 4
    leaves = dev_field(nl * ls, 77)
    n_dig, n_cap = zk.merkle_sizes(nl, ch)
    dig = torch.empty(n_dig * 4, dtype=torch.int64, device="cuda")
    caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # the Merkle entry point queues on the legacy default stream: time it there
    legacy = torch.cuda.default_stream()
    zk.fill_digests_buf_linear_gpu(dig, caps, leaves, nl, ls, ch, 0)
    torch.cuda.synchronize()
    ts = []
    for s in range(steps):
        with torch.cuda.stream(legacy):
            flush.fill_(s & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(legacy)
        zk.fill_digests_buf_linear_gpu(dig, caps, leaves, nl, ls, ch, 0)
        b.record(legacy)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    del leaves, dig, caps, flush
    torch.cuda.empty_cache()
    return perms_of(nl, ls, ch) / (statistics.median(ts) * 1e-3)


def measure_batch(steps, budget_gb):
    """Uneven batch: one graph per memory wave (batched) vs one synchronous C-ABI
    call per stage per job (plain: compute_batched_lde -> compute_transpose_rev ->
    fill_digests_buf_linear_gpu_with_gpu_ptr), same jobs, same buffers, caps
    compared.  Also the batch's Poseidon permutation count at the measured
    forest rate: no schedule of these jobs on these kernels beats that time;
    and the sum of the batch's own stages (each job's fused LDE and forest)
    run one at a time: the graph's time against it shows how much idle time
    and overlap the schedule has."""
    import torch
    import zeknox_b200 as zk
    jobs = uneven_jobs()
    budget = int(budget_gb * (1 << 30))
    waves, cur, used = [], [], 0
    for jb in jobs:
        n, N = 1 << jb["lg_n"], 1 << (jb["lg_n"] + jb["rate"])
        need = 8 * (n * jb["cols"] + N * jb["cols"] + 2 * N * 4)
        if cur and used + need > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(jb)
        used += need
    waves.append(cur)
    total_elems = sum((1 << (j["lg_n"] + j["rate"])) * j["cols"] for j in jobs)
    total_perms = sum(perms_of(1 << (j["lg_n"] + j["rate"]), j["cols"], j["cap"]) for j in jobs)
    t_batch, t_plain = 0.0, 0.0
    t_stages = {"lde": 0.0, "forest": 0.0}
    all_caps = []
    for wave in waves:
        bufs, cjobs = [], []
        for jb in wave:
            n, N = 1 << jb["lg_n"], 1 << (jb["lg_n"] + jb["rate"])
            inp = dev_field(n * jb["cols"], jb["seed"])
            leaves = torch.empty(N * jb["cols"], dtype=torch.int64, device="cuda")
            n_dig, n_cap = zk.merkle_sizes(N, jb["cap"])
            dig = torch.empty(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
            caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
            bufs.append((inp, leaves, dig, caps, n_dig, n_cap))
            cjobs.append(zk.commit_job(jb["lg_n"], jb["rate"], jb["cols"], jb["cap"], jb["hash"], inp, leaves, dig, caps))
        zk.commit_batch(0, cjobs)  # capture
        torch.cuda.synchronize()
        caps_b = [b[3].clone() for b in bufs]
        all_caps.extend(cb.cpu() for cb in caps_b)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(steps):
            a.record()
            zk.commit_batch(0, cjobs)
            b.record()
            torch.cuda.synchronize()
            t_batch += a.elapsed_time(b) / steps
        # plain path, same jobs and buffers; the caller's evaluation buffer
        # (the LDE output the transpose reads) is allocated once, outside the
        # timed region, at the wave's largest job
        ev_all = torch.empty(max((1 << (jb["lg_n"] + jb["rate"])) * jb["cols"] for jb in wave), dtype=torch.int64,
                             device="cuda")
        for it in range(steps + 1):  # the first pass is untimed: tables, pool growth
            a.record()
            for jb, (inp, leaves, dig, caps, n_dig, n_cap) in zip(wave, bufs):
                N = 1 << (jb["lg_n"] + jb["rate"])
                ev = ev_all[:N * jb["cols"]]
                zk.lde_batch(0, ev, inp, jb["lg_n"], jb["cols"], jb["rate"], with_coset=True)
                zk.transpose_rev_batch(0, leaves, ev, jb["lg_n"] + jb["rate"], jb["cols"])
                zk.fill_digests_buf_linear_gpu(dig, caps, leaves, N, jb["cols"], jb["cap"], jb["hash"])
                torch.cuda.synchronize()
            b.record()
            torch.cuda.synchronize()
            if it:
                t_plain += a.elapsed_time(b) / steps
        for cb, bb in zip(caps_b, bufs):
            assert torch.equal(cb, bb[3]), "batched and plain commitments differ"
        # the batch's own stages one at a time: each job's fused LDE and its
        # forest, each call alone and waited for (what the graph would take
        # if nothing overlapped and nothing were left idle)
        # (events on the legacy stream: the forest call queues there and
        # returns at once; the LDE call waits for its blocking stream)
        legacy = torch.cuda.default_stream()
        for jb, (inp, leaves, dig, caps, n_dig, n_cap) in zip(wave, bufs):
            N = 1 << (jb["lg_n"] + jb["rate"])
            for stage in ("lde", "forest"):
                a.record(legacy)
                if stage == "lde":
                    zk.lde_rows(0, leaves, inp, jb["lg_n"], jb["rate"], jb["cols"])
                else:
                    zk.fill_digests_buf_linear_gpu(dig, caps, leaves, N, jb["cols"], jb["cap"], jb["hash"])
                b.record(legacy)
                torch.cuda.synchronize()
                t_stages[stage] += a.elapsed_time(b)
        del bufs, cjobs, caps_b, ev_all
        torch.cuda.empty_cache()
    # the whole batch through the device-resident loop: every job submitted at
    # once to a server whose persistent kernel runs them (one launch while the
    # stream lasts); results released as they complete; wall clock, submit of
    # the first job -> completion of the last
    inputs = [dev_field((1 << jb["lg_n"]) * jb["cols"], jb["seed"]) for jb in jobs]
    caps_loop = [torch.zeros((1 << jb["cap"]) * 4, dtype=torch.int64).pin_memory() for jb in jobs]
    with zk.Server(0, 100 << 30, 16, device_loop=True) as srv:
        for r in (1, 2, 3):
            srv.prepare(10, 20, r)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pending = {srv.submit(jb["lg_n"], jb["rate"], jb["cols"], jb["cap"], jb["hash"], inp, caps_host=ch): i
                   for i, (jb, inp, ch) in enumerate(zip(jobs, inputs, caps_loop))}
        while pending:
            for t in list(pending):
                res = srv.wait(t, timeout_ms=0.0)
                if res.status == 2:
                    srv.release(t)
                    del pending[t]
                elif res.status < 0:
                    raise RuntimeError("device-loop job failed: %d" % res.status)
            time.sleep(0.0002)
        t_loop = (time.perf_counter() - t0) * 1e3
    for cl, cb in zip(caps_loop, all_caps):
        assert torch.equal(cl, cb), "device-loop and batched commitments differ"
    del inputs, caps_loop
    torch.cuda.empty_cache()
    rate = poseidon_perm_rate()
    floor_ms = total_perms / rate * 1e3
    return {"batched_elems_per_s": total_elems / (t_batch * 1e-3), "plain_elems_per_s": total_elems / (t_plain * 1e-3),
            "batched_over_plain": t_plain / t_batch, "batched_ms": t_batch, "plain_ms": t_plain,
            "poseidon_perms": total_perms, "poseidon_perms_per_s": rate, "perm_floor_ms": floor_ms,
            "batched_frac_of_perm_floor": floor_ms / t_batch, "plain_bound_over_floor": t_plain / floor_ms,
            "device_loop_ms": t_loop, "device_loop_elems_per_s": total_elems / (t_loop * 1e-3),
            "device_loop_over_plain": t_plain / t_loop,
            "stage_sum_ms": t_stages["lde"] + t_stages["forest"], "stage_lde_ms": t_stages["lde"],
            "stage_forest_ms": t_stages["forest"], "batched_over_stage_sum": t_batch / (t_stages["lde"] + t_stages["forest"]),
            "jobs": len(jobs), "waves": len(waves), "elements": total_elems, "steps": steps,
            "workload": "64 jobs: lg_n U{10..20}, cols U{8..400}, rate_bits U{1,2,3}, Poseidon, cap_height min(4, lg N), "
                        "seed 3; waves of <= %g GiB" % budget_gb}


def run_batch(args):
    import torch
    torch.cuda.set_device(0)
    d = measure_batch(args.steps, args.budget_gb)
    line = {"metric": "uneven batch LDE+Merkle commit elems/s (batched graph vs plain per-call)", "unit": "elems/s",
            "dtype": "u64", **d}
    print(json.dumps(line), flush=True)


def measure_hashes(steps):
    """Alternative hashes at scale: 2^20 leaves x 135 elements, cap_height 4,
    Poseidon2 + Monolith + Keccak forests built as one batch (one graph), and
    each forest alone through fill_digests_buf_linear_gpu_with_gpu_ptr (CUDA
    events on the legacy stream the Merkle call queues on)."""
    import torch
    import zeknox_b200 as zk
    nl, ls, ch = 1 << 20, 135, 4
    trees = []
    for k, h in enumerate((3, 4, 1)):
        leaves = dev_field(nl * ls, 40 + k)
        n_dig, n_cap = zk.merkle_sizes(nl, ch)
        dig = torch.empty(n_dig * 4, dtype=torch.int64, device="cuda")
        caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
        trees.append((h, leaves, dig, caps))
    jobs = [zk.merkle_job(l, d, c, nl, ls, ch, h) for h, l, d, c in trees]
    zk.merkle_batch(0, jobs)
    torch.cuda.synchronize()
    legacy = torch.cuda.default_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(legacy)
    for _ in range(steps):
        zk.merkle_batch(0, jobs)
    b.record(legacy)
    torch.cuda.synchronize()
    batch_ms = a.elapsed_time(b) / steps
    per = {}
    # Poseidon-BN128 (hash type 2) alone on the same shape, outside the batch
    leaves_bn = dev_field(nl * ls, 43)
    n_dig, n_cap = zk.merkle_sizes(nl, ch)
    trees.append((2, leaves_bn, torch.empty(n_dig * 4, dtype=torch.int64, device="cuda"),
                  torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")))
    for h, l, d, c in trees:
        zk.fill_digests_buf_linear_gpu(d, c, l, nl, ls, ch, h)
        torch.cuda.synchronize()
        a.record(legacy)
        for _ in range(steps):
            zk.fill_digests_buf_linear_gpu(d, c, l, nl, ls, ch, h)
        b.record(legacy)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / steps
        name = {3: "poseidon2", 4: "monolith", 1: "keccak", 2: "poseidon_bn128"}[h]
        perms = perms_of(nl, ls, ch) if h != 1 else nl * ((ls * 8) // 136 + 1) + (nl - (1 << ch))
        per[name] = {"ms": ms, "leaves_per_s": nl / (ms * 1e-3), "perms_per_s": perms / (ms * 1e-3)}
    del trees, jobs
    torch.cuda.empty_cache()
    return {"batched_leaves_per_s": 3 * nl / (batch_ms * 1e-3), "batched_ms": batch_ms, "per_hash": per,
            "steps": steps, "workload": "Poseidon2 + Monolith + Keccak forests, 2^20 leaves x 135, cap 4, one batch; "
                                        "each alone, and Poseidon-BN128 alone"}


def run_hashes(args):
    import torch
    torch.cuda.set_device(0)
    d = measure_hashes(args.steps)
    line = {"metric": "Merkle forests (2^20 leaves x 135, cap 4) leaves/s", "unit": "leaves/s", "dtype": "u64", **d}
    print(json.dumps(line), flush=True)


def serve_stream(srv, reqs, gaps, caps_host):
    """Submit reqs[i] at the cumulative times gaps[:i+1] (all at once when gaps
    is None) while a client thread takes every result as soon as it is ready,
    in completion order, and releases it.  Returns per-request latency and
    queue time (ms), the completion times and the start time (perf_counter)."""
    import threading as th
    n = len(reqs)
    tickets, submitted, lock, failed = [None] * n, [], th.Lock(), []
    lat, queue, done_t = [None] * n, [None] * n, [None] * n

    def reaper():
        outstanding, seen, n_done = set(), 0, 0
        while n_done < n:
            with lock:
                outstanding.update(submitted[seen:])
                seen = len(submitted)
            finished = []
            for i in outstanding:
                r = srv.wait(tickets[i], 0.0)
                if r.status == 2 or r.status < 0:
                    if r.status < 0:
                        failed.append((i, r.status))  # reported after the stream (the thread must not stop early)
                    lat[i], queue[i], done_t[i] = r.latency_ms, r.queue_ms, time.perf_counter()
                    srv.release(tickets[i])
                    finished.append(i)
            outstanding.difference_update(finished)
            n_done += len(finished)
            if not finished:
                time.sleep(0.0002)

    rt = th.Thread(target=reaper)
    rt.start()
    t0 = time.perf_counter()
    when = t0
    for i, (lg, r, c, cap, h, inp) in enumerate(reqs):
        if gaps is not None:
            when += gaps[i]
            delay = when - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
        tickets[i] = srv.submit(lg, r, c, cap, h, inp, caps_host=caps_host[i])
        with lock:
            submitted.append(i)
    rt.join()
    if failed:
        raise RuntimeError("serving requests failed (index, status): %s" % failed[:8])
    return lat, queue, done_t, t0


def measure_serve(requests, serial_sample=24):
    """Serving: a Poisson stream of LDE + Poseidon commit requests (log2 size
    U{12..22}, columns U{16..256}, rate_bits 3, cap height 4) admitted by
    zeknox_server against a 120 GB budget with 8 slots; arrival rate 0.7x the
    capacity of serial plain calls (one synchronous zeknox_commit per request,
    timed on the first `serial_sample` requests).  Reports p50/p99 latency
    (submit -> caps on host), delivered throughput (elements / first arrival
    -> last completion), offered throughput (elements / arrival span), and
    the server's capacity with every request submitted at once.  Requests read
    their coefficients from one shared seeded pool (the stream can then be
    long without holding every input)."""
    import torch
    import zeknox_b200 as zk
    rng = np.random.default_rng(5)
    shapes = [(int(rng.integers(12, 23)), 3, int(rng.integers(16, 257)), 4, 0) for _ in range(requests)]
    pool = dev_field(256 << 22, 5000)
    reqs = [(lg, r, c, cap, h, pool[:c << lg]) for lg, r, c, cap, h in shapes]
    elems = [(1 << (lg + r)) * c for lg, r, c, _, _ in shapes]
    serial = []
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for lg, r, c, cap, h, inp in reqs[:serial_sample]:
        N = 1 << (lg + r)
        leaves = torch.empty(N * c, dtype=torch.int64, device="cuda")
        n_dig, n_cap = zk.merkle_sizes(N, cap)
        dig = torch.empty(n_dig * 4, dtype=torch.int64, device="cuda")
        caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
        job = zk.commit_job(lg, r, c, cap, h, inp, leaves, dig, caps)
        zk.commit(0, job)  # tables, pool
        a.record()
        zk.commit(0, job)
        b.record()
        torch.cuda.synchronize()
        serial.append(a.elapsed_time(b))
        del leaves, dig, caps
        torch.cuda.empty_cache()
    capacity = sum(elems[:serial_sample]) / (sum(serial) * 1e-3)
    rate = 0.7 / (np.mean(serial) * 1e-3)  # requests per second
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    caps_host = [torch.zeros((1 << cap) * 4, dtype=torch.int64).pin_memory() for _, _, _, cap, _ in shapes]
    with zk.Server(0, 120 << 30, 8) as srv:
        # twiddles and coset tables of the stream's sizes resident before it starts
        srv.prepare(12, 22, 3)
        lat, queue, done_t, t0 = serve_stream(srv, reqs, gaps, caps_host)
        peak = srv.stats()["peak"]
        _, _, done_s, t0s = serve_stream(srv, reqs, None, caps_host)
    span = max(done_t) - t0
    arrivals = float(np.sum(gaps))
    saturated = sum(elems) / (max(done_s) - t0s)
    # the same stream through the device-resident request loop
    with zk.Server(0, 120 << 30, 8, device_loop=True) as srv:
        srv.prepare(12, 22, 3)
        lat_d, queue_d, done_d, t0d = serve_stream(srv, reqs, gaps, caps_host)
        _, _, done_ds, t0ds = serve_stream(srv, reqs, None, caps_host)
    span_d = max(done_d) - t0d
    saturated_d = sum(elems) / (max(done_ds) - t0ds)
    device_loop = {"p50_ms": float(np.percentile(lat_d, 50)), "p99_ms": float(np.percentile(lat_d, 99)),
                   "mean_queue_ms": float(np.mean(queue_d)), "delivered_elems_per_s": sum(elems) / span_d,
                   "delivered_over_offered": arrivals / span_d, "saturated_elems_per_s": saturated_d,
                   "saturated_over_serial": saturated_d / capacity,
                   "form": "one persistent cooperative kernel runs the admitted requests' stages, the active "
                           "request with the least work left first at every stage boundary; the host admits and "
                           "posts plans to a ring in mapped memory"}
    del reqs, pool
    torch.cuda.empty_cache()
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_queue_ms": float(np.mean(queue)), "delivered_elems_per_s": sum(elems) / span,
            "offered_elems_per_s": sum(elems) / arrivals, "delivered_over_offered": arrivals / span,
            "saturated_elems_per_s": saturated, "serial_plain_elems_per_s": capacity,
            "saturated_over_serial": saturated / capacity, "offered_load": 0.7, "requests": len(elems),
            "arrival_rate_per_s": rate, "arrival_span_s": arrivals, "completion_span_s": span,
            "peak_budget_bytes": peak, "budget_bytes": 120 << 30, "slots": 8, "serial_sample": serial_sample,
            "device_loop": device_loop,
            "workload": "Poisson stream: lg_n U{12..22}, cols U{16..256}, rate_bits 3, Poseidon, cap 4, 120 GB budget, "
                        "8 slots, seed 5; latency = submit -> caps on host"}


def run_loop_trace(args):
    """Per-stage device time of the device-resident loop (zeknox_server_trace)
    against the same work through the standalone calls (zeknox_lde_rows and
    fill_digests_buf_linear_gpu_with_gpu_ptr, CUDA events), for single
    Poseidon requests of 2^12 x 16, 2^16 x 128 and 2^20 x 256 (rate 3, cap 4)."""
    import torch
    import zeknox_b200 as zk
    torch.cuda.set_device(0)
    pool = dev_field(256 << 20, 77)
    legacy = torch.cuda.default_stream()
    names = {2: "leaf", 3: "leaf_coop", 4: "level", 5: "fold", 6: "tail"}
    out = []
    for lg, c in [(12, 16), (16, 128), (20, 256)]:
        N = 1 << (lg + 3)
        inp = pool[: c << lg]
        leaves = torch.empty(N * c, dtype=torch.int64, device="cuda")
        n_dig, n_cap = zk.merkle_sizes(N, 4)
        dig = torch.empty(n_dig * 4, dtype=torch.int64, device="cuda")
        caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_lde, t_forest = [], []
        for _ in range(4):
            a.record(legacy)
            zk.lde_rows(0, leaves, inp, lg, 3, c)
            b.record(legacy)
            torch.cuda.synchronize()
            t_lde.append(a.elapsed_time(b))
            a.record(legacy)
            zk.fill_digests_buf_linear_gpu(dig, caps, leaves, N, c, 4, 0)
            b.record(legacy)
            torch.cuda.synchronize()
            t_forest.append(a.elapsed_time(b))
        del leaves, dig, caps
        torch.cuda.empty_cache()
        with zk.Server(0, 40 << 30, 8, device_loop=True) as srv:
            srv.prepare(lg, lg, 3)
            ch = torch.zeros(n_cap * 4, dtype=torch.int64).pin_memory()
            for _ in range(3):
                t = srv.submit(lg, 3, c, 4, 0, inp, caps_host=ch)
                r = srv.wait(t)
                assert r.status == 2, r.status
                tr = srv.trace(t)
                srv.release(t)
        stages = {}
        for kind, ns in tr:
            key = "lde_pass_radix_2^%d" % (kind - 16) if kind >= 16 else names[kind]
            stages[key] = stages.get(key, 0.0) + ns / 1e6
        out.append({"request": [lg, 3, c, 4, 0], "loop_latency_ms": r.latency_ms, "loop_stages_ms": stages,
                    "loop_lde_ms": sum(ns for k, ns in tr if k >= 16) / 1e6,
                    "loop_forest_ms": sum(ns for k, ns in tr if k < 16) / 1e6,
                    "standalone_lde_ms": statistics.median(t_lde[1:]),
                    "standalone_forest_ms": statistics.median(t_forest[1:])})
    print(json.dumps({"metric": "device loop per-stage device time against standalone calls", "unit": "ms",
                      "requests": out}), flush=True)


def run_serve(args):
    import torch
    torch.cuda.set_device(0)
    d = measure_serve(args.requests)
    line = {"metric": "serving LDE+Poseidon commit: p50/p99 latency and throughput", "unit": "ms", "dtype": "u64",
            **d}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-lg", type=int, default=15, help="log2 coefficients per column of the CPU sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--lg-n", type=int, default=LG_N, help="log2 coefficients per column (profiling cases)")
    ap.add_argument("--only", default=None, choices=["lde", "merkle", "transpose", "ntt"],
                    help="profiling: run only this stage for warmup+steps iterations and exit")
    ap.add_argument("--hash", type=int, default=HASH, help="--only merkle: hash type (0 Poseidon, 1 Keccak, "
                    "2 Poseidon-BN128, 3 Poseidon2, 4 Monolith)")
    ap.add_argument("--requests", type=int, default=96, help="serve workload: number of requests")
    ap.add_argument("--batch-steps", type=int, default=1, help="uneven batch: timed passes per wave")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: skip the uneven-batch and serving measurements of the default run")
    ap.add_argument("--workload", default="commit", choices=["commit", "batch", "hashes", "serve", "loop-trace"],
                    help="commit: the headline line; batch: uneven 64-job batch vs plain calls; hashes: 2^20 x 135 "
                         "forests with Poseidon2, Monolith and Keccak")
    ap.add_argument("--budget-gb", type=float, default=48.0, help="batch workload: device memory per wave")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.only:
        return run_stage(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "hashes":
        return run_hashes(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "loop-trace":
        return run_loop_trace(args)
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

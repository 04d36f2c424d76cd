"""Autotuner: times the library's launch-shape knobs on the GPU and writes the
tuning table that ``zeknox_b200.load()`` reads.

    python -m zeknox_b200.autotune [--device 0] [--out zeknox_b200/tuning_b200.txt] [--quick]

Knobs (all shape choices only; results are bit-identical for every value, and
the tuner checks that for each candidate against the default's output):

* ``lde_last_logr`` (per log2 n): radix exponent 6..8 of the fused LDE's last
  pass, the one that writes bit-reversed leaf rows;
* ``lde_chunk_mib`` (per log2 N = log2 n + rate_bits): column-chunk budget of
  the fused LDE (its scratch: the inter-pass intermediate of one chunk);
* ``leaf_threads.<hash>`` (per log2 leaves): CTA size of the Merkle leaf kernel
  (one thread per leaf, a CTA of 64 / 128 / 256 leaves);
* ``wide_level_nodes.<hash>`` (per log2 leaves): Merkle levels with at least this
  many nodes run one launch per level (one thread per node) before the
  in-CTA fold takes over;
* ``coop_leaves.<hash>`` (per log2 leaves; Poseidon and Poseidon2): forests of at
  most this many leaves hash their leaves with four threads per permutation;
* ``ntt_split_logr`` (per log2 n): the largest pass, 2^7..2^10 points, of a
  column-output transform (compute_batched_ntt / compute_batched_lde); 0 keeps
  the built-in split;
* ``transpose_bulk`` (per log2 n): the transpose's form, 0 the 16-byte
  register form, 1..8 a tile shape of the bulk-copy form, 9 the built-in
  choice by column count.

Each candidate is timed with CUDA events on the launching stream, median of
several repetitions after warm-up, with the L2 flushed (a 256 MiB write)
before every repetition.  Knobs are searched one at a time (coordinate
descent) in the order above; a value replaces the built-in default only when
it is faster by more than ``--margin`` (default 2 %).  The table lists every
measured shape with its times as comments.

The reference library has no tuner (its launch shapes are fixed constants in
native/ntt/kernels.cu and native/merkle/merkle.cu); this is the B200 side's
own.
"""
import argparse
import os
import statistics
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

DEFAULTS = {"lde_last_logr": 8, "lde_chunk_mib": 512, "leaf_threads": 256, "wide_level_nodes": 1 << 15,
            "coop_leaves": 1 << 13, "ntt_split_logr": 0, "transpose_bulk": 9}
CANDIDATES = {
    "lde_last_logr": [8, 7, 6],
    "lde_chunk_mib": [512, 96, 128, 256, 2048],
    "leaf_threads": [256, 128, 64],
    "wide_level_nodes": [1 << 15, 1 << 13, 1 << 17, 1 << 40],
    "coop_leaves": [1 << 13, 0, 1 << 40],
    "ntt_split_logr": [0, 10, 9, 8, 7],
    "transpose_bulk": [9, 0, 1, 3, 5],
}
SEARCHES = ("lde", "merkle", "ntt", "transpose")
COOP_HASHES = (0, 3)  # hashes with the cooperative (four threads per permutation) kernels
HASH_NAMES = {0: "poseidon", 1: "keccak", 3: "poseidon2", 4: "monolith"}
RATE = 3


def lde_shapes(quick):
    """(lg_n, cols) of the fused-LDE shapes: rows at most 2^27 words (1 GiB)."""
    lgs = [15, 16] if quick else [12, 13, 14, 15, 16, 17, 18, 19, 20]
    return [(lg, min(256, 1 << (27 - lg - RATE))) for lg in lgs]


def ntt_shapes(quick):
    """(lg n, columns) of the column-output transforms: 2^27 words (1 GiB)."""
    lgs = [19, 20] if quick else [14, 16, 18, 19, 20, 21, 22, 24]
    return [(lg, 1 << (27 - lg)) for lg in lgs]


def transpose_shapes(quick):
    """(lg n, columns) of the transposes: 2^26 words (512 MiB) each way."""
    shapes = [(18, 256), (22, 16)] if quick else [(16, 1024), (18, 256), (20, 64), (22, 16)]
    return shapes


def merkle_shapes(quick):
    """(hash, lg leaves, leaf size): the commit's Poseidon2 forest and the
    alternative-hash forests of 2^20 leaves x 135."""
    out = [(3, 18, 256)]
    if not quick:
        out += [(3, 20, 135), (0, 20, 135), (4, 20, 135), (1, 20, 135), (0, 13, 84), (3, 16, 256)]
        out += [(h, lg, 135) for h in COOP_HASHES for lg in (12, 14, 15, 16)]
    return out


class Timer:
    """CUDA-event timing on one stream, L2 flushed before every repetition."""

    def __init__(self, torch, stream, warmup, reps):
        self.torch, self.stream, self.warmup, self.reps = torch, stream, warmup, reps
        self.flush = torch.empty(32 << 20, dtype=torch.int64, device="cuda")  # 256 MiB > L2

    def on(self, stream):
        """The same timer on another stream (the Merkle calls run on the
        legacy default stream, which torch's own streams do not wait for)."""
        other = Timer.__new__(Timer)
        other.__dict__.update(self.__dict__)
        other.stream = stream
        return other

    def __call__(self, fn):
        t = self.torch
        with t.cuda.stream(self.stream):
            for _ in range(self.warmup):
                fn()
            times = []
            for _ in range(self.reps):
                self.flush.fill_(len(times))
                e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
                e0.record(self.stream)
                fn()
                e1.record(self.stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
        return statistics.median(times)


def search(zk, timer, knob, lg, candidates, default, run, check, margin, log):
    """Time `run` under each candidate value of `knob` at log2 size `lg`;
    `check` compares the output with the default's (raises on a mismatch).
    Leaves the chosen value set and returns (value, {value: ms})."""
    times = {}
    for v in candidates:
        zk.tune_set(knob, v, lg=lg)
        run()
        check(knob, v)
        times[v] = timer(run)
    best = min(times, key=times.get)
    if times[best] >= times[default] * (1.0 - margin):
        best = default  # not clearly faster: keep the built-in value
    zk.tune_set(knob, best, lg=lg)
    log.append((knob, lg, best, times))
    print("  %-22s lg %2d -> %-8d %s" % (knob, lg, best, " ".join("%d=%.3f" % kv for kv in times.items())),
          flush=True)
    return best, times


def tune_lde(zk, torch, timer, dev, stream, lg, cols, margin, log):
    n, N = 1 << lg, 1 << (lg + RATE)
    coeffs = torch.randint(0, 1 << 62, (cols * n,), dtype=torch.int64, device="cuda")
    rows = torch.empty(cols * N, dtype=torch.int64, device="cuda")

    def run():
        zk.lde_rows(dev, rows, coeffs, lg, RATE, cols, stream=stream.cuda_stream)

    run()
    stream.synchronize()
    ref = rows.clone()

    def check(knob, v):
        stream.synchronize()
        if not torch.equal(rows, ref):
            raise RuntimeError("LDE 2^%d x %d differs from the default with %s = %d" % (lg, cols, knob, v))

    print("LDE lg_n %d rate %d cols %d" % (lg, RATE, cols), flush=True)
    search(zk, timer, "lde_last_logr", lg, CANDIDATES["lde_last_logr"], DEFAULTS["lde_last_logr"], run, check,
           margin, log)
    search(zk, timer, "lde_chunk_mib", lg + RATE, CANDIDATES["lde_chunk_mib"], DEFAULTS["lde_chunk_mib"], run,
           check, margin, log)
    del coeffs, rows, ref


def tune_merkle(zk, torch, timer, h, lg, leaf_size, margin, log):
    n = 1 << lg
    cap = 4
    leaves = torch.randint(0, 1 << 62, (n * leaf_size,), dtype=torch.int64, device="cuda")
    n_dig, n_cap = zk.merkle_sizes(n, cap)
    dig = torch.empty(max(n_dig, 1) * 4, dtype=torch.int64, device="cuda")
    caps = torch.empty(n_cap * 4, dtype=torch.int64, device="cuda")

    def run():
        zk.fill_digests_buf_linear_gpu(dig, caps, leaves, n, leaf_size, cap, h)

    run()
    torch.cuda.synchronize()
    ref_d, ref_c = dig.clone(), caps.clone()

    def check(knob, v):
        torch.cuda.synchronize()
        if not (torch.equal(dig, ref_d) and torch.equal(caps, ref_c)):
            raise RuntimeError("%s forest 2^%d x %d differs with %s = %d" % (HASH_NAMES[h], lg, leaf_size, knob, v))

    print("Merkle %s 2^%d leaves x %d" % (HASH_NAMES[h], lg, leaf_size), flush=True)
    search(zk, timer, "leaf_threads.%d" % h, lg, CANDIDATES["leaf_threads"], DEFAULTS["leaf_threads"], run, check,
           margin, log)
    search(zk, timer, "wide_level_nodes.%d" % h, lg, CANDIDATES["wide_level_nodes"], DEFAULTS["wide_level_nodes"],
           run, check, margin, log)
    if h in COOP_HASHES:
        search(zk, timer, "coop_leaves.%d" % h, lg, CANDIDATES["coop_leaves"], DEFAULTS["coop_leaves"], run, check,
               margin, log)
    del leaves, dig, caps, ref_d, ref_c


def tune_ntt(zk, torch, timer, dev, lg, cols, margin, log):
    n = 1 << lg
    x0 = torch.randint(0, 1 << 62, (cols * n,), dtype=torch.int64, device="cuda")
    x = x0.clone()
    ref = x0.clone()
    zk.ntt_batch(dev, ref, lg, cols)

    def run():
        zk.ntt_batch(dev, x, lg, cols)

    def check(knob, v):
        y = x0.clone()
        zk.ntt_batch(dev, y, lg, cols)
        if not torch.equal(y, ref):
            raise RuntimeError("NTT 2^%d x %d differs from the default with %s = %d" % (lg, cols, knob, v))

    print("NTT lg_n %d cols %d" % (lg, cols), flush=True)
    search(zk, timer, "ntt_split_logr", lg, CANDIDATES["ntt_split_logr"], DEFAULTS["ntt_split_logr"], run, check,
           margin, log)
    del x0, x, ref


def tune_transpose(zk, torch, timer, dev, stream, lg, cols, margin, log):
    n = 1 << lg
    src = torch.randint(0, 1 << 62, (cols * n,), dtype=torch.int64, device="cuda")
    out = torch.empty_like(src)

    def run():
        zk.transpose_rev(dev, out, src, lg, cols, stream=stream.cuda_stream)

    run()
    stream.synchronize()
    ref = out.clone()

    def check(knob, v):
        stream.synchronize()
        if not torch.equal(out, ref):
            raise RuntimeError("transpose 2^%d x %d differs with %s = %d" % (lg, cols, knob, v))

    print("transpose lg_n %d cols %d" % (lg, cols), flush=True)
    search(zk, timer, "transpose_bulk", lg, CANDIDATES["transpose_bulk"], DEFAULTS["transpose_bulk"], run, check,
           margin, log)
    del src, out, ref


def kept_table_lines(path, retuned):
    """The lines of an existing table whose knobs are not searched again (a
    run of some searches only keeps the others' measured entries)."""
    keep = []
    if not os.path.exists(path):
        return keep
    for line in open(path):
        if line.startswith("#") or not line.strip():
            continue
        if line.split()[0].split(".")[0] not in retuned:
            keep.append(line.rstrip("\n"))
    return keep


def write_table(path, log, device_name, keep=()):
    lines = ["# zeknox_b200 tuning table: <knob> <log2 size | *> <value>",
             "# measured on %s by python -m zeknox_b200.autotune (CUDA events, median, L2 flushed)" % device_name,
             "# comment after each line: milliseconds per call for every candidate"]
    lines += list(keep)
    for knob, lg, best, times in log:
        lines.append("%-22s %2d %-14d # %s" % (knob, lg, best, " ".join("%d=%.3f" % kv for kv in times.items())))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=os.path.join(HERE, "tuning_b200.txt"))
    ap.add_argument("--quick", action="store_true", help="the headline shapes only")
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--reps", type=int, default=7)
    ap.add_argument("--margin", type=float, default=0.02)
    ap.add_argument("--only", default=",".join(SEARCHES),
                    help="comma-separated searches to run (%s); the other knobs' lines of the existing table are "
                         "kept" % ", ".join(SEARCHES))
    args = ap.parse_args(argv)
    only = [w for w in args.only.split(",") if w]
    for w in only:
        if w not in SEARCHES:
            raise SystemExit("unknown search %r" % w)
    knobs_of = {"lde": ("lde_last_logr", "lde_chunk_mib"), "merkle": ("leaf_threads", "wide_level_nodes", "coop_leaves"),
                "ntt": ("ntt_split_logr",), "transpose": ("transpose_bulk",)}
    retuned = {k for w in only for k in knobs_of[w]}
    keep = kept_table_lines(args.out, retuned) if set(only) != set(SEARCHES) else []
    os.environ["ZEKNOX_TUNE_FILE"] = "none"  # start from the built-in defaults
    import torch
    import zeknox_b200 as zk
    if not torch.cuda.is_available():
        raise SystemExit("autotune needs a GPU")
    torch.cuda.set_device(args.device)
    zk.load()
    zk.tune_clear()
    stream = torch.cuda.Stream()
    timer = Timer(torch, stream, args.warmup, args.reps)
    log = []
    if "lde" in only:
        for lg, cols in lde_shapes(args.quick):
            tune_lde(zk, torch, timer, args.device, stream, lg, cols, args.margin, log)
            torch.cuda.empty_cache()
    if "merkle" in only:
        for h, lg, leaf_size in merkle_shapes(args.quick):
            tune_merkle(zk, torch, timer.on(torch.cuda.default_stream()), h, lg, leaf_size, args.margin, log)
            torch.cuda.empty_cache()
    if "ntt" in only:
        for lg, cols in ntt_shapes(args.quick):
            tune_ntt(zk, torch, timer, args.device, lg, cols, args.margin, log)
            torch.cuda.empty_cache()
    if "transpose" in only:
        for lg, cols in transpose_shapes(args.quick):
            tune_transpose(zk, torch, timer, args.device, stream, lg, cols, args.margin, log)
            torch.cuda.empty_cache()
    write_table(args.out, log, torch.cuda.get_device_name(args.device), keep)
    changed = sum(1 for knob, _, best, _ in log if best != DEFAULTS[knob.split(".")[0]])
    print("wrote %s: %d entries, %d differ from the built-in defaults" % (args.out, len(log), changed))


if __name__ == "__main__":
    main()

"""zeknox_b200 -- B200-native Goldilocks commit path behind zeknox's C ABI.

The computation lives in ``libzeknox.so`` (CUDA, sm_100a; built by
``make -C zeknox_b200`` or ``__graft_entry__.build()``).  This module is the
Python host side: it loads the library, declares the C entry points with
ctypes, and offers the same operations as zeknox's Rust wrapper
(wrappers/rust/src/lib.rs: ``lde_batch``, ``ntt_batch``, ``intt_batch``,
``transpose_rev_batch``, ``init_*``) plus the Merkle builders of
native/merkle/merkle.h and this library's fused commit extension.

Buffers are torch tensors of dtype int64 (bit patterns of u64 field
elements) or uint64; CUDA tensors are passed as device pointers, CPU tensors as
host pointers.  There is no CPU fallback: every GPU entry point fails loudly
(``ZeknoxError`` / ``OSError``) when the CUDA library or a GPU is missing.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# ZEKNOX_LIB selects another build of the library, e.g. libzeknox_checked.so
# (range checks on every kernel's global accesses, zeknox_bounds_report)
LIB_PATH = os.environ.get("ZEKNOX_LIB") or os.path.join(HERE, "libzeknox.so")

P = 0xFFFFFFFF00000001
HASH_POSEIDON, HASH_KECCAK, HASH_POSEIDON_BN128, HASH_POSEIDON2, HASH_MONOLITH = 0, 1, 2, 3, 4
FORWARD, INVERSE = 0, 1
SELFTEST_OPS = 34  # ZK_SELFTEST_OPS of include/zeknox_b200.h
SERVE_CANCELLED = -10000  # ZK_SERVE_CANCELLED
SERVE_FAIL_ALLOC, SERVE_FAIL_SHAPE, SERVE_FAIL_LAUNCH, SERVE_FAIL_GATE = 1, 2, 3, 4  # ZK_SERVE_FAIL_*
SERVE_DEVICE_LOOP = 1  # ZK_SERVE_DEVICE_LOOP

# Exported C symbols (include/lib.h, include/merkle/merkle.h, include/zeknox_b200.h).
ABI_SYMBOLS = [
    "get_number_of_gpus", "list_devices_info", "init_cuda", "init_cuda_degree", "init_cuda_degree_and_generator",
    "init_twiddle_factors", "init_coset", "compute_batched_ntt", "compute_batched_lde",
    "compute_batched_lde_multi_gpu", "compute_transpose_rev", "compute_naive_transpose_rev",
    "fill_digests_buf_linear_gpu_with_gpu_ptr", "fill_digests_buf_linear_multigpu_with_gpu_ptr",
    "fill_digests_buf_linear_cpu", "cuda_available", "fill_digests_buf_linear_cpu_avx",
    "fill_digests_buf_linear_cpu_avx512",
]
EXT_SYMBOLS = ["zeknox_last_error", "zeknox_commit", "zeknox_commit_batch", "zeknox_commit_scratch_words",
               "zeknox_lde_rows", "zeknox_launch_count", "zeknox_measure_mul_rate", "zeknox_merkle_batch",
               "zeknox_lde_rows_noalloc", "zeknox_server_create", "zeknox_server_create_ex", "zeknox_server_submit", "zeknox_server_wait",
               "zeknox_server_release", "zeknox_server_stats", "zeknox_server_destroy", "zeknox_server_prepare",
               "zeknox_server_cancel", "zeknox_server_inject_failure", "zeknox_server_trace", "zeknox_tune_set",
               "zeknox_tune_get", "zeknox_tune_clear", "zeknox_tune_load", "zeknox_transpose_rev",
               "zeknox_lde_rows_scatter", "zeknox_field_selftest", "zeknox_permute", "zeknox_bounds_report",
               "zeknox_inject_wait_timeout"]

# Tuning table measured on B200 by ``python -m zeknox_b200.autotune``; loaded
# by load() unless ZEKNOX_TUNE_FILE names another table ("" or "none": no table).
TUNE_TABLE = os.path.join(HERE, "tuning_b200.txt")


class RustError(ctypes.Structure):
    """native/utils/rusterror.h: {int code; char *message} returned by value."""
    _fields_ = [("code", ctypes.c_int), ("message", ctypes.c_void_p)]


class NTTConfig(ctypes.Structure):
    """native/ntt/ntt.h NTT_Config (24 bytes)."""
    _fields_ = [
        ("batches", ctypes.c_uint32),
        ("order", ctypes.c_int),
        ("ntt_type", ctypes.c_int),
        ("extension_rate_bits", ctypes.c_uint32),
        ("are_inputs_on_device", ctypes.c_bool),
        ("are_outputs_on_device", ctypes.c_bool),
        ("with_coset", ctypes.c_bool),
        ("is_multi_gpu", ctypes.c_bool),
        ("salt_size", ctypes.c_uint32),
    ]


class TransposeConfig(ctypes.Structure):
    """native/ntt/ntt.h NTT_TransposeConfig (8 bytes)."""
    _fields_ = [
        ("batches", ctypes.c_uint32),
        ("are_inputs_on_device", ctypes.c_bool),
        ("are_outputs_on_device", ctypes.c_bool),
    ]


class CommitJob(ctypes.Structure):
    """include/zeknox_b200.h zk_commit_job."""
    _fields_ = [
        ("lg_n", ctypes.c_uint32),
        ("rate_bits", ctypes.c_uint32),
        ("cols", ctypes.c_uint32),
        ("cap_height", ctypes.c_uint32),
        ("hash_type", ctypes.c_uint32),
        ("input_is_values", ctypes.c_uint32),
        ("coset_gen", ctypes.c_uint64),
        ("input", ctypes.c_void_p),
        ("leaves", ctypes.c_void_p),
        ("digests", ctypes.c_void_p),
        ("caps", ctypes.c_void_p),
    ]


class MerkleJob(ctypes.Structure):
    """include/zeknox_b200.h zk_merkle_job."""
    _fields_ = [
        ("leaves", ctypes.c_void_p),
        ("digests", ctypes.c_void_p),
        ("caps", ctypes.c_void_p),
        ("n_leaves", ctypes.c_uint64),
        ("leaf_size", ctypes.c_uint64),
        ("cap_height", ctypes.c_uint32),
        ("hash_type", ctypes.c_uint32),
    ]


class ServeRequest(ctypes.Structure):
    """include/zeknox_b200.h zk_serve_request."""
    _fields_ = [("lg_n", ctypes.c_uint32), ("rate_bits", ctypes.c_uint32), ("cols", ctypes.c_uint32),
                ("cap_height", ctypes.c_uint32), ("hash_type", ctypes.c_uint32), ("input_is_values", ctypes.c_uint32),
                ("coset_gen", ctypes.c_uint64), ("input", ctypes.c_void_p), ("caps_host", ctypes.c_void_p)]


class ServeResult(ctypes.Structure):
    """include/zeknox_b200.h zk_serve_result."""
    _fields_ = [("status", ctypes.c_int), ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("leaves", ctypes.c_void_p), ("digests", ctypes.c_void_p), ("caps", ctypes.c_void_p)]


class ZeknoxError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("zeknox error %d: %s" % (code, message))
        self.code = code


_lib = None
_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def load():
    """Load libzeknox.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("libzeknox.so not built: run `make -C %s` (or __graft_entry__.build())" % HERE)
    L = ctypes.CDLL(LIB_PATH)
    sz, u32, u64, vp = ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
    L.get_number_of_gpus.restype = RustError
    L.get_number_of_gpus.argtypes = [ctypes.POINTER(sz)]
    L.list_devices_info.restype = RustError
    L.init_cuda.restype = None
    L.init_cuda_degree.argtypes = [u32]
    L.init_cuda_degree.restype = None
    L.init_cuda_degree_and_generator.argtypes = [u32, u64]
    L.init_cuda_degree_and_generator.restype = None
    L.init_twiddle_factors.restype = RustError
    L.init_twiddle_factors.argtypes = [sz, sz]
    L.init_coset.restype = RustError
    L.init_coset.argtypes = [sz, sz, u64]
    L.compute_batched_ntt.restype = RustError
    L.compute_batched_ntt.argtypes = [sz, vp, u32, ctypes.c_int, NTTConfig]
    L.compute_batched_lde.restype = RustError
    L.compute_batched_lde.argtypes = [sz, vp, vp, u32, ctypes.c_int, NTTConfig]
    L.compute_batched_lde_multi_gpu.restype = RustError
    L.compute_batched_lde_multi_gpu.argtypes = [vp, vp, u32, ctypes.c_int, NTTConfig, u32, sz, sz]
    for f in (L.compute_transpose_rev, L.compute_naive_transpose_rev):
        f.restype = RustError
        f.argtypes = [sz, vp, vp, u32, TransposeConfig]
    L.fill_digests_buf_linear_gpu_with_gpu_ptr.restype = None
    L.fill_digests_buf_linear_gpu_with_gpu_ptr.argtypes = [vp, vp, vp] + [u64] * 7
    L.fill_digests_buf_linear_multigpu_with_gpu_ptr.restype = None
    L.fill_digests_buf_linear_multigpu_with_gpu_ptr.argtypes = [vp, vp, vp] + [u64] * 6
    for f in (L.fill_digests_buf_linear_cpu, L.fill_digests_buf_linear_cpu_avx, L.fill_digests_buf_linear_cpu_avx512):
        f.restype = None
        f.argtypes = [vp, vp, vp] + [u64] * 6
    L.cuda_available.restype = ctypes.c_bool
    L.zeknox_last_error.restype = ctypes.c_char_p
    L.zeknox_commit.restype = RustError
    L.zeknox_commit.argtypes = [sz, ctypes.POINTER(CommitJob), vp]
    L.zeknox_commit_batch.restype = RustError
    L.zeknox_commit_batch.argtypes = [sz, ctypes.POINTER(CommitJob), u32]
    L.zeknox_commit_scratch_words.restype = u64
    L.zeknox_commit_scratch_words.argtypes = [ctypes.POINTER(CommitJob)]
    L.zeknox_lde_rows.restype = RustError
    L.zeknox_lde_rows.argtypes = [sz, vp, vp, u32, u32, u32, u64, vp]
    L.zeknox_launch_count.restype = u64
    L.zeknox_measure_mul_rate.restype = ctypes.c_double
    L.zeknox_measure_mul_rate.argtypes = [sz]
    L.zeknox_lde_rows_noalloc.restype = RustError
    L.zeknox_lde_rows_noalloc.argtypes = [sz, vp, vp, u32, u32, u32, u64, vp]
    L.zeknox_server_create.restype = RustError
    L.zeknox_server_create.argtypes = [sz, u64, u32, ctypes.POINTER(ctypes.c_void_p)]
    L.zeknox_server_trace.restype = RustError
    L.zeknox_server_trace.argtypes = [vp, u64, ctypes.POINTER(u32), ctypes.POINTER(u64), u32, ctypes.POINTER(u32)]
    L.zeknox_server_create_ex.restype = RustError
    L.zeknox_server_create_ex.argtypes = [sz, u64, u32, u32, ctypes.POINTER(ctypes.c_void_p)]
    L.zeknox_server_submit.restype = RustError
    L.zeknox_server_submit.argtypes = [vp, ctypes.POINTER(ServeRequest), ctypes.POINTER(u64)]
    L.zeknox_server_wait.restype = RustError
    L.zeknox_server_wait.argtypes = [vp, u64, ctypes.c_double, ctypes.POINTER(ServeResult)]
    L.zeknox_server_release.restype = RustError
    L.zeknox_server_release.argtypes = [vp, u64]
    L.zeknox_server_stats.restype = RustError
    L.zeknox_server_stats.argtypes = [vp, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.zeknox_server_destroy.restype = RustError
    L.zeknox_server_destroy.argtypes = [vp]
    L.zeknox_server_prepare.restype = RustError
    L.zeknox_server_prepare.argtypes = [vp, u32, u32, u32, u64]
    L.zeknox_server_cancel.restype = RustError
    L.zeknox_server_cancel.argtypes = [vp, u64]
    L.zeknox_server_inject_failure.restype = RustError
    L.zeknox_server_inject_failure.argtypes = [vp, ctypes.c_int]
    L.zeknox_merkle_batch.restype = RustError
    L.zeknox_merkle_batch.argtypes = [sz, ctypes.POINTER(MerkleJob), u32]
    L.zeknox_lde_rows_scatter.restype = RustError
    L.zeknox_field_selftest.restype = RustError
    L.zeknox_field_selftest.argtypes = [sz, vp, vp, vp, u64, vp, vp]
    L.zeknox_bounds_report.restype = RustError
    L.zeknox_bounds_report.argtypes = [sz, ctypes.POINTER(ctypes.c_uint64)]
    L.zeknox_inject_wait_timeout.restype = RustError
    L.zeknox_inject_wait_timeout.argtypes = [sz, u32]
    L.zeknox_permute.restype = RustError
    L.zeknox_permute.argtypes = [sz, vp, u64, u32, u32, vp]
    L.zeknox_lde_rows_scatter.argtypes = [sz, ctypes.POINTER(ctypes.c_void_p), u32, vp, u32, u32, u32, u32, u32, u64, vp]
    L.zeknox_transpose_rev.restype = RustError
    L.zeknox_transpose_rev.argtypes = [sz, vp, vp, u32, u32, vp]
    L.zeknox_tune_set.restype = RustError
    L.zeknox_tune_set.argtypes = [ctypes.c_char_p, u32, u64]
    L.zeknox_tune_get.restype = u64
    L.zeknox_tune_get.argtypes = [ctypes.c_char_p, u32, u64]
    L.zeknox_tune_clear.restype = RustError
    L.zeknox_tune_clear.argtypes = []
    L.zeknox_tune_load.restype = RustError
    L.zeknox_tune_load.argtypes = [ctypes.c_char_p]
    _lib = L
    table = os.environ.get("ZEKNOX_TUNE_FILE", TUNE_TABLE)
    if table and table != "none" and os.path.exists(table):
        _check(L.zeknox_tune_load(table.encode()))
    return L


def _check(err):
    if err.code != 0:
        msg = ctypes.string_at(err.message).decode() if err.message else ""
        if err.message:
            _libc.free(err.message)
        raise ZeknoxError(err.code, msg)


def last_error():
    m = load().zeknox_last_error()
    return m.decode() if m else None


def _ptr(t):
    if t is None:
        return None
    assert t.is_contiguous(), "buffers must be contiguous"
    return ctypes.c_void_p(t.data_ptr())


# ---------------------------------------------------------------- device info

def get_number_of_gpus():
    n = ctypes.c_size_t(0)
    _check(load().get_number_of_gpus(ctypes.byref(n)))
    return n.value


def cuda_available():
    return bool(load().cuda_available())


def list_devices_info():
    _check(load().list_devices_info())


def init_twiddle_factors(device_id, lg_n):
    _check(load().init_twiddle_factors(device_id, lg_n))


def init_coset(device_id, lg_n, coset_gen=7):
    _check(load().init_coset(device_id, lg_n, coset_gen))


def init_cuda():
    load().init_cuda()


def init_cuda_degree(max_degree):
    load().init_cuda_degree(max_degree)


# ---------------------------------------------------------------- transforms

def ntt_config(batches=1, rate_bits=0, inputs_on_device=False, outputs_on_device=False, with_coset=False,
               salt_size=0):
    c = NTTConfig()
    c.batches = batches
    c.order = 0
    c.ntt_type = 0
    c.extension_rate_bits = rate_bits
    c.are_inputs_on_device = inputs_on_device
    c.are_outputs_on_device = outputs_on_device
    c.with_coset = with_coset
    c.is_multi_gpu = False
    c.salt_size = salt_size
    return c


def ntt_batch(device_id, inout, lg_n, batches, with_coset=False, inverse=False):
    """compute_batched_ntt on a (batches, 2^lg_n) tensor, in place (host or device)."""
    on_dev = inout.is_cuda
    cfg = ntt_config(batches, 0, on_dev, on_dev, with_coset)
    _check(load().compute_batched_ntt(device_id, _ptr(inout), lg_n, INVERSE if inverse else FORWARD, cfg))
    return inout


def intt_batch(device_id, inout, lg_n, batches, with_coset=False):
    return ntt_batch(device_id, inout, lg_n, batches, with_coset, inverse=True)


def lde_batch(device_id, output, inp, lg_n, batches, rate_bits, with_coset=True, inverse=False, salt_size=0):
    """compute_batched_lde: (batches, 2^lg_n) coefficients -> (batches+salt, 2^(lg_n+rate)) evaluations."""
    cfg = ntt_config(batches, rate_bits, inp.is_cuda, output.is_cuda, with_coset, salt_size)
    _check(load().compute_batched_lde(device_id, _ptr(output), _ptr(inp), lg_n, INVERSE if inverse else FORWARD, cfg))
    return output


def lde_batch_multi_gpu(output, inp, num_gpu, lg_n, batches, rate_bits, with_coset=True):
    cfg = ntt_config(batches, rate_bits, False, True, with_coset)
    n_in = batches << lg_n
    n_out = batches << (lg_n + rate_bits)
    _check(load().compute_batched_lde_multi_gpu(_ptr(output), _ptr(inp), num_gpu, FORWARD, cfg, lg_n, n_in, n_out))
    return output


def transpose_rev_batch(device_id, output, inp, lg_n, batches, naive=False):
    cfg = TransposeConfig()
    cfg.batches = batches
    cfg.are_inputs_on_device = inp.is_cuda
    cfg.are_outputs_on_device = output.is_cuda
    f = load().compute_naive_transpose_rev if naive else load().compute_transpose_rev
    _check(f(device_id, _ptr(output), _ptr(inp), lg_n, cfg))
    return output


# -------------------------------------------------------------------- Merkle

def merkle_sizes(n_leaves, cap_height):
    n_caps = 1 << cap_height
    return 2 * (n_leaves - n_caps), n_caps


def fill_digests_buf_linear_gpu(digests, caps, leaves, n_leaves, leaf_size, cap_height, hash_type, gpu_id=0):
    """fill_digests_buf_linear_gpu_with_gpu_ptr; raises ZeknoxError on a rejected call."""
    n_dig, n_caps = merkle_sizes(n_leaves, cap_height)
    L = load()
    L.zeknox_last_error  # noqa: B018  (symbol presence)
    before = last_error()
    L.fill_digests_buf_linear_gpu_with_gpu_ptr(_ptr(digests), _ptr(caps), _ptr(leaves), n_dig, n_caps, n_leaves,
                                               leaf_size, cap_height, hash_type, gpu_id)
    after = last_error()
    if after is not None and after != before:
        raise ZeknoxError(1, after)


def fill_digests_buf_linear_multigpu(digests, caps, leaves, n_leaves, leaf_size, cap_height, hash_type):
    n_dig, n_caps = merkle_sizes(n_leaves, cap_height)
    before = last_error()
    load().fill_digests_buf_linear_multigpu_with_gpu_ptr(_ptr(digests), _ptr(caps), _ptr(leaves), n_dig, n_caps,
                                                         n_leaves, leaf_size, cap_height, hash_type)
    after = last_error()
    if after is not None and after != before:
        raise ZeknoxError(1, after)


def fill_digests_buf_linear_cpu(digests, caps, leaves, n_leaves, leaf_size, cap_height, hash_type, vector=None):
    """Host forest builder.  vector: None (fill_digests_buf_linear_cpu), "avx" or
    "avx512" (the vector builders, Poseidon only)."""
    n_dig, n_caps = merkle_sizes(n_leaves, cap_height)
    L = load()
    fn = {None: L.fill_digests_buf_linear_cpu, "avx": L.fill_digests_buf_linear_cpu_avx,
          "avx512": L.fill_digests_buf_linear_cpu_avx512}[vector]
    before = last_error()
    fn(_ptr(digests), _ptr(caps), _ptr(leaves), n_dig, n_caps, n_leaves, leaf_size, cap_height, hash_type)
    after = last_error()
    if after is not None and after != before:
        raise ZeknoxError(1, after)


# ------------------------------------------------------------------- commits

def commit_job(lg_n, rate_bits, cols, cap_height, hash_type, inp, leaves, digests, caps, input_is_values=False,
               coset_gen=7):
    j = CommitJob()
    j.lg_n, j.rate_bits, j.cols, j.cap_height, j.hash_type = lg_n, rate_bits, cols, cap_height, hash_type
    j.input_is_values = int(bool(input_is_values))
    j.coset_gen = coset_gen
    j.input, j.leaves = inp.data_ptr(), leaves.data_ptr()
    j.digests = digests.data_ptr() if digests is not None and digests.numel() else None
    j.caps = caps.data_ptr()
    return j


def commit(device_id, job, stream=None):
    """zeknox_commit: LDE -> bit-reversed leaf rows -> Merkle forest for one job."""
    _check(load().zeknox_commit(device_id, ctypes.byref(job), ctypes.c_void_p(stream) if stream else None))


def commit_batch(device_id, jobs):
    arr = (CommitJob * len(jobs))(*jobs)
    _check(load().zeknox_commit_batch(device_id, arr, len(jobs)))


def commit_scratch_words(job):
    return load().zeknox_commit_scratch_words(ctypes.byref(job))


def lde_rows(device_id, rows, coeffs, lg_n, rate_bits, cols, coset_gen=7, stream=None):
    """zeknox_lde_rows: coefficient columns -> bit-reversed leaf-major LDE matrix."""
    _check(load().zeknox_lde_rows(device_id, _ptr(rows), _ptr(coeffs), lg_n, rate_bits, cols, coset_gen,
                                  ctypes.c_void_p(stream) if stream else None))
    return rows


def lde_rows_noalloc(device_id, rows, coeffs, lg_n, rate_bits, cols, coset_gen=7, stream=None):
    """zeknox_lde_rows_noalloc: the same result as lde_rows without allocating
    device memory (static 32 MiB scratch; lg_n + rate_bits <= 18), for callers
    whose device memory belongs to another allocator or whose thread must not
    enter the driver's allocator."""
    _check(load().zeknox_lde_rows_noalloc(device_id, _ptr(rows), _ptr(coeffs), lg_n, rate_bits, cols, coset_gen,
                                          ctypes.c_void_p(stream) if stream else None))
    return rows


def lde_rows_scatter(device_id, dst, coeffs, lg_n, rate_bits, cols, col_offset, row_stride, coset_gen=7, stream=None):
    """zeknox_lde_rows_scatter: the fused LDE of `cols` columns with its leaf
    rows spread over the destination buffers `dst` (tensors or device
    addresses; a power of two of them, rows split evenly), written at columns
    [col_offset, col_offset + cols) of rows of `row_stride` words."""
    ptrs = [d if isinstance(d, int) else d.data_ptr() for d in dst]
    arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
    _check(load().zeknox_lde_rows_scatter(device_id, arr, len(ptrs), _ptr(coeffs), lg_n, rate_bits, cols, col_offset,
                                          row_stride, coset_gen, ctypes.c_void_p(stream) if stream else None))


def field_selftest(device_id, a, b, c, out, stream=None):
    """zeknox_field_selftest: the device field primitives on operand arrays
    a, b, c (n words each); out holds SELFTEST_OPS * n words, op-major."""
    n = a.numel()
    assert b.numel() == n and c.numel() == n and out.numel() >= SELFTEST_OPS * n
    _check(load().zeknox_field_selftest(device_id, _ptr(a), _ptr(b), _ptr(c), n, _ptr(out),
                                        ctypes.c_void_p(stream) if stream else None))
    return out


def bounds_report(device_id=0):
    """zeknox_bounds_report: (checked, [count, site, index, extent]) -- the
    out-of-range accesses the checked build's kernels skipped since the last
    report (checked is False for the normal build, whose record is zero)."""
    rec = (ctypes.c_uint64 * 4)()
    err = load().zeknox_bounds_report(device_id, rec)
    if err.message:
        _libc.free(err.message)
    if err.code not in (0, 801):  # 801: cudaErrorNotSupported, the normal build
        raise ZeknoxError(err.code, "zeknox_bounds_report")
    return err.code == 0, [int(v) for v in rec]


# Values of the "transpose_bulk" knob: 0 the 16-byte transpose, 1..8 a tile
# shape of the bulk-copy transpose, TRANSPOSE_AUTO (the default) by column count.
TRANSPOSE_AUTO = 9


def inject_wait_timeout(device_id=0, count=1):
    """zeknox_inject_wait_timeout: the next `count` bulk-copy transposes on the
    device declare more bytes than they copy, so a bounded wait runs out."""
    _check(load().zeknox_inject_wait_timeout(device_id, count))


def permute(device_id, states, hash_type, cooperative=False, stream=None):
    """zeknox_permute: one permutation of every state in place (12 words per
    state; 25 for Keccak-f)."""
    width = 25 if hash_type == HASH_KECCAK else 12
    assert states.numel() % width == 0
    _check(load().zeknox_permute(device_id, _ptr(states), states.numel() // width, hash_type, int(bool(cooperative)),
                                 ctypes.c_void_p(stream) if stream else None))
    return states


def transpose_rev(device_id, output, inp, lg_n, cols, stream=None):
    """zeknox_transpose_rev: bit-reversed transpose of device columns, queued on
    `stream` (an int cudaStream_t handle; None waits on the device's stream)."""
    _check(load().zeknox_transpose_rev(device_id, _ptr(output), _ptr(inp), lg_n, cols,
                                       ctypes.c_void_p(stream) if stream else None))
    return output


def launch_count():
    return load().zeknox_launch_count()


def measure_mul_rate(device_id=0):
    return load().zeknox_measure_mul_rate(device_id)


# ------------------------------------------------------------------ tuning

TUNE_ANY = 0xFFFFFFFF


def tune_set(name, value, lg=None):
    """Set a knob ("leaf_threads.<hash>", "lde_chunk_mib", "lde_last_logr",
    "wide_level_nodes.<hash>"), for log2 size `lg` or for every size (lg None)."""
    _check(load().zeknox_tune_set(name.encode(), TUNE_ANY if lg is None else lg, value))


def tune_get(name, lg=None, default=0):
    """Value of a knob for log2 size `lg` (falls back to the size-free entry,
    then to `default`)."""
    return load().zeknox_tune_get(name.encode(), TUNE_ANY if lg is None else lg, default)


def tune_clear():
    """Forget every knob (built-in defaults again)."""
    _check(load().zeknox_tune_clear())


def tune_load(path):
    """Load a table of "<name> <lg|*> <value>" lines."""
    _check(load().zeknox_tune_load(os.fspath(path).encode()))


def merkle_job(leaves, digests, caps, n_leaves, leaf_size, cap_height, hash_type):
    j = MerkleJob()
    j.leaves, j.caps = leaves.data_ptr(), caps.data_ptr()
    j.digests = digests.data_ptr() if digests is not None and digests.numel() else None
    j.n_leaves, j.leaf_size, j.cap_height, j.hash_type = n_leaves, leaf_size, cap_height, hash_type
    return j


def merkle_batch(device_id, jobs):
    """zeknox_merkle_batch: several forests as one cached CUDA graph."""
    arr = (MerkleJob * len(jobs))(*jobs)
    _check(load().zeknox_merkle_batch(device_id, arr, len(jobs)))


class Server:
    """Continuous-batching commit server (zeknox_server_*): requests are admitted
    in arrival order as slots and the device-memory budget allow, and overlap on
    the GPU.  device_loop=True: a persistent device-resident loop runs the
    admitted requests (zeknox_server_create_ex with ZK_SERVE_DEVICE_LOOP)."""

    def __init__(self, device_id=0, budget_bytes=120 << 30, slots=8, device_loop=False):
        h = ctypes.c_void_p()
        _check(load().zeknox_server_create_ex(device_id, budget_bytes, slots,
                                              SERVE_DEVICE_LOOP if device_loop else 0, ctypes.byref(h)))
        self._h = h

    def submit(self, lg_n, rate_bits, cols, cap_height, hash_type, inp, caps_host=None, input_is_values=False,
               coset_gen=7):
        r = ServeRequest(lg_n, rate_bits, cols, cap_height, hash_type, int(bool(input_is_values)), coset_gen,
                         inp.data_ptr(), caps_host.data_ptr() if caps_host is not None else None)
        t = ctypes.c_uint64()
        _check(load().zeknox_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=-1.0):
        res = ServeResult()
        _check(load().zeknox_server_wait(self._h, ticket, timeout_ms, ctypes.byref(res)))
        return res

    def release(self, ticket):
        _check(load().zeknox_server_release(self._h, ticket))

    def prepare(self, lg_n_min, lg_n_max, rate_bits, coset_gen=7):
        """Build every table requests of these sizes read, ahead of them."""
        _check(load().zeknox_server_prepare(self._h, lg_n_min, lg_n_max, rate_bits, coset_gen))

    def cancel(self, ticket):
        _check(load().zeknox_server_cancel(self._h, ticket))

    def inject_failure(self, stage):
        """Test hook: the next request started fails at `stage` (SERVE_FAIL_*)."""
        _check(load().zeknox_server_inject_failure(self._h, stage))

    def trace(self, ticket):
        """zeknox_server_trace: [(stage kind, device ns)] of a finished
        device-loop request (16 + log2 radix: transform pass; 2/3 leaves; 4
        level; 5/6 cooperative fold/tail; 7/8 fold/tail; 9 copy; 10 reorder)."""
        n = ctypes.c_uint32()
        _check(load().zeknox_server_trace(self._h, ticket, None, None, 0, ctypes.byref(n)))
        kinds, ns = (ctypes.c_uint32 * max(n.value, 1))(), (ctypes.c_uint64 * max(n.value, 1))()
        _check(load().zeknox_server_trace(self._h, ticket, kinds, ns, n.value, ctypes.byref(n)))
        return [(int(kinds[q]), int(ns[q])) for q in range(n.value)]

    def stats(self):
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(load().zeknox_server_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"in_use": a.value, "peak": b.value, "completed": c.value}

    def close(self):
        if self._h:
            _check(load().zeknox_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

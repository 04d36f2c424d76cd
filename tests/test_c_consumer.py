"""A plain C program linked against the static archive exactly as the Rust
wrapper links the reference (libzeknox.a + cudart + libstdc++ + libgomp):
it must build on CPU, and on a GPU its commit through the reference's entry
points must give the oracle's caps."""
import os
import subprocess

import numpy as np
import pytest


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_consumer(tmp_path):
    exe = tmp_path / "consumer"
    cmd = ["gcc", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "c", "consumer.c"), "-o", str(exe),
           os.path.join(ROOT, "zeknox_b200", "libzeknox.a"), "-L", os.path.join(CUDA, "lib64"),
           "-lcudart_static", "-lstdc++", "-lgomp", "-lpthread", "-ldl", "-lrt", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def test_static_archive_links_into_a_c_program(tmp_path):
    assert os.path.exists(build_consumer(tmp_path))


@pytest.mark.gpu
@pytest.mark.parametrize("lg,rate,cols,cap,h", [(10, 2, 12, 3, 3), (12, 1, 9, 2, 0), (9, 3, 20, 4, 4)])
def test_c_consumer_commit_matches_oracle(tmp_path, lg, rate, cols, cap, h):
    from oracle import oracle as O
    exe = build_consumer(tmp_path)
    seed = 1000 + lg
    out = subprocess.run([str(exe), str(lg), str(rate), str(cols), str(cap), str(h), str(seed)], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    caps = np.array([[int(w, 16) for w in line.split()] for line in out.stdout.split("\n") if line.strip()],
                    dtype=np.uint64)
    # the same splitmix64 stream (state += golden ratio, then the finaliser), folded below p
    s = np.uint64(seed)
    k = np.arange(1, cols * (1 << lg) + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = s + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    coeffs = np.where(z >= np.uint64(O.P), z - np.uint64(O.P), z)
    rows = O.lde_rows(coeffs, lg, rate, cols)
    _, cp = O.merkle(rows, cols, cap, h)
    assert np.array_equal(caps, cp)

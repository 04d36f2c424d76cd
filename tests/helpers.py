"""Shared helpers for the parity tests (numpy <-> torch, case tables)."""
import hashlib

import numpy as np

from oracle import oracle as O
from tests.golden.make_golden import MERKLE_CASES, FULL_DIGESTS_MAX, merkle_seed  # noqa: F401

HASHES = {"poseidon": 0, "keccak": 1, "poseidon2": 3, "monolith": 4, "poseidon_bn128": 2}


def to_dev(arr, device="cuda"):
    import torch
    a = np.ascontiguousarray(arr, dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64).copy()).to(device)


def to_np(t):
    return t.detach().cpu().numpy().view(np.uint64)


def empty_dev(n, device="cuda"):
    import torch
    return torch.zeros(max(int(n), 1), dtype=torch.int64, device=device)


def sha256(arr):
    return hashlib.sha256(np.ascontiguousarray(arr, dtype=np.uint64).tobytes()).digest()

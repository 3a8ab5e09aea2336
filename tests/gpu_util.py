"""Helpers for the GPU parity tests: numpy <-> device columns."""
import numpy as np


def dev(torch, a: np.ndarray):
    """Copy an int32 numpy column to a fresh (256-byte aligned) device tensor."""
    return torch.from_numpy(np.ascontiguousarray(a, np.int32)).to("cuda")


def host(t) -> np.ndarray:
    return t.cpu().numpy()


def i32(x: int) -> int:
    return ((x + (1 << 31)) % (1 << 32)) - (1 << 31)


def sorted_rows(cols) -> np.ndarray:
    """Rows of equal-length columns, sorted lexicographically (multiset view)."""
    m = np.stack([np.asarray(c, np.int64) for c in cols], axis=1) if cols else np.zeros((0, 0), np.int64)
    if m.size == 0:
        return m
    return m[np.lexsort(tuple(m[:, k] for k in range(m.shape[1] - 1, -1, -1)))]

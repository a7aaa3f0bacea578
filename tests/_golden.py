"""Loads the golden fixtures (outputs of the reference's own GPU EM, written by
tests/golden/make_golden.py) and compares a result with them."""
from __future__ import annotations

import hashlib
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["tiny", "small", "c1", "hard"]
ITERS = (1, 20)


def input_digest(f) -> str:
    h = hashlib.sha256()
    for a in (f.query, f.img, f.centroids, f.label_ptr):
        h.update(np.ascontiguousarray(a).tobytes())
    for name in f.gauss.dtype.names:
        h.update(np.ascontiguousarray(f.gauss[name]).tobytes())
    return h.hexdigest()


def load(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def rnk_by_pair(ind, rnk, S):
    """{(s, k): rnk} -- compares responsibilities independent of the slot order."""
    ind = ind.reshape(5, S)
    rnk = rnk.reshape(5, S)
    return {(s, int(ind[j, s])): float(rnk[j, s]) for j in range(5) for s in range(S)}


def compare_with_reference(z: dict, it: int, got: dict, S: int, rnk_tol: float, m_tol: float, w_rtol: float,
                           same_slot_order: bool):
    """got: dict(gauss, rnk, ind).  Returns the measured errors (after asserting them)."""
    ri, rr, rg = z[f"em{it}_ind"], z[f"em{it}_rnk"], z[f"em{it}_gauss"]
    if same_slot_order:
        np.testing.assert_array_equal(got["ind"], ri)
    np.testing.assert_array_equal(np.sort(got["ind"].reshape(5, S), 0), np.sort(ri.reshape(5, S), 0))
    a, b = rnk_by_pair(ri, rr, S), rnk_by_pair(got["ind"], got["rnk"], S)
    d_rnk = max(abs(a[k] - b[k]) for k in a)
    gg = got["gauss"]
    alive = rg["m_o"][:, 0] > -1e31
    np.testing.assert_array_equal(gg["m_o"][:, 0] > -1e31, alive)
    np.testing.assert_array_equal(gg["supervoxelNum"], rg["supervoxelNum"])
    for k in range(rg.shape[0]):
        n = rg["supervoxelNum"][k]
        if same_slot_order:
            np.testing.assert_array_equal(gg["supervoxelIdx"][k][:n], rg["supervoxelIdx"][k][:n])
        else:  # appended in slot order: the same set, maybe another order
            np.testing.assert_array_equal(np.sort(gg["supervoxelIdx"][k][:n]), np.sort(rg["supervoxelIdx"][k][:n]))
    d_m = float(np.max(np.abs(gg["m_k"][alive] - rg["m_k"][alive])))
    ws = np.max(np.abs(rg["W_k"][alive]), axis=1, keepdims=True)
    d_w = float(np.max(np.abs(gg["W_k"][alive] - rg["W_k"][alive]) / ws))
    assert d_rnk <= rnk_tol, d_rnk
    assert d_m <= m_tol, d_m
    assert d_w <= w_rtol, d_w
    return d_rnk, d_m, d_w

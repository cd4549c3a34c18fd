"""Test infrastructure: a plain-Python statement of the device breadth-first level
order (swe_dev_rcm_mapping, csrc/device_order.cu), small grids only.

From node 0, level by level: every node of the current level offers itself to its
unmapped stencil neighbours (slots 1..n-1); a neighbour keeps the smallest key
(parent position in the order, slot); the next level is its nodes sorted by key.
The whole order is reversed at the end.  Keys are unique, so the result is exact.
"""
import numpy as np


def levelset_mapping(idx: np.ndarray) -> np.ndarray:
    idx = np.asarray(idx)
    n, nn = idx.shape
    order = [0]
    mapped = np.zeros(n, dtype=bool)
    mapped[0] = True
    lv0, lv1 = 0, 1
    while lv1 < n:
        key = {}
        for p in range(lv0, lv1):
            v = order[p]
            for j in range(1, nn):
                w = int(idx[v, j])
                if mapped[w]:
                    continue
                k = (p << 8) | j
                if w not in key or k < key[w]:
                    key[w] = k
        if not key:
            raise ValueError("stencil graph is not connected")
        nxt = sorted(key, key=key.__getitem__)
        mapped[nxt] = True
        order += nxt
        lv0, lv1 = lv1, lv1 + len(nxt)
    return np.array(order[::-1], dtype=np.int32)

"""Independent restatement of the product's host index construction (TEST INFRASTRUCTURE ONLY).

The SELL-C-sigma layout and the reverse Cuthill-McKee ordering have no counterpart in the
reference (its packer, host/cuper_control_matrix.hpp:130-207, deals rows to 128 FPGA
PEs instead); these pure-Python/numpy restatements of the rules written in
project_xplus_b200/csrc/sell.cpp and rcm.cpp are what the product's builders must match
bit for bit.  Written for clarity, not speed: use on systems of up to ~1e5 rows.
"""
from __future__ import annotations

from collections import deque

import numpy as np


def sell_build(row_ptr, col_idx, values, C=32, sigma=256, chunk=1, diag_split=False):
    row_ptr = np.asarray(row_ptr)
    col_idx = np.asarray(col_idx)
    values = np.asarray(values, np.float64)
    n = len(row_ptr) - 1
    rows = []
    for i in range(n):
        ent = [(int(col_idx[k]), float(values[k])) for k in range(row_ptr[i], row_ptr[i + 1])]
        d = None
        if diag_split:
            for q, (c, v) in enumerate(ent):
                if c == i:
                    d = v
                    del ent[q]
                    break
        rows.append((ent, d))
    lengths = [len(e) for e, _ in rows]
    perm = list(range(n))
    if sigma > 1:
        for w0 in range(0, n, sigma):
            win = perm[w0:w0 + sigma]
            win.sort(key=lambda r: -lengths[r])  # Python sort is stable
            perm[w0:w0 + sigma] = win
    perm = np.array(perm, np.int32)
    iperm = np.empty(n, np.int64)
    iperm[perm] = np.arange(n)
    n_slices = (n + C - 1) // C
    widths = np.zeros(n_slices, np.int32)
    for s in range(n_slices):
        w = max((lengths[perm[i]] for i in range(s * C, min(n, s * C + C))), default=0)
        widths[s] = -(-w // chunk) * chunk
    slice_ptr = np.zeros(n_slices + 1, np.int64)
    slice_ptr[1:] = np.cumsum(widths.astype(np.int64) * C)
    slots = int(slice_ptr[-1])
    col = np.zeros(slots, np.int32)
    val = np.zeros(slots, np.float64)
    diag = np.zeros(n, np.float64) if diag_split else None
    for s in range(n_slices):
        base = slice_ptr[s]
        for lane in range(C):
            i = s * C + lane
            ent = []
            if i < n:
                ent, d = rows[perm[i]]
                if diag_split:
                    diag[i] = d if d is not None else 0.0
            for j in range(widths[s]):
                pos = base + (j // chunk) * C * chunk + lane * chunk + (j % chunk)
                if j < len(ent):
                    col[pos] = iperm[ent[j][0]]
                    val[pos] = ent[j][1]
                else:
                    col[pos] = i
                    val[pos] = 0.0
    return dict(n_slices=n_slices, slots=slots, perm=perm, slice_ptr=slice_ptr, slice_width=widths,
                col=col, val=val, diag=diag)


def rcm(row_ptr, col_idx):
    row_ptr = np.asarray(row_ptr)
    col_idx = np.asarray(col_idx)
    n = len(row_ptr) - 1
    adj = [[int(c) for c in col_idx[row_ptr[i]:row_ptr[i + 1]] if c != i] for i in range(n)]
    deg = [len(a) for a in adj]
    key = lambda v: (deg[v], v)  # noqa: E731
    placed = [False] * n

    def levels(root):
        seen = {root}
        level = [root]
        order = [root]
        nlev = 0
        last = [root]
        while level:
            nlev += 1
            last = level
            nxt = []
            for v in level:
                for u in adj[v]:
                    if not placed[u] and u not in seen:
                        seen.add(u)
                        nxt.append(u)
            order.extend(nxt)
            level = nxt
        return nlev, last, order

    result = []
    for seed in range(n):
        if placed[seed]:
            continue
        _, _, comp = levels(seed)
        v = min(comp, key=key)
        ecc, last, _ = levels(v)
        while True:
            u = min(last, key=key)
            ecc_u, last_u, _ = levels(u)
            if ecc_u > ecc:
                v, ecc, last = u, ecc_u, last_u
            else:
                break
        q = deque([v])
        placed[v] = True
        result.append(v)
        while q:
            x = q.popleft()
            nb = sorted((u for u in adj[x] if not placed[u]), key=key)
            for u in nb:
                placed[u] = True
                result.append(u)
                q.append(u)
    return np.array(result[::-1], np.int32)


def permute_symmetric(row_ptr, col_idx, values, perm):
    row_ptr = np.asarray(row_ptr)
    n = len(row_ptr) - 1
    iperm = np.empty(n, np.int64)
    iperm[np.asarray(perm)] = np.arange(n)
    orp = [0]
    oci, ov = [], []
    for i in range(n):
        old = perm[i]
        ent = sorted(((int(iperm[col_idx[k]]), float(values[k])) for k in range(row_ptr[old], row_ptr[old + 1])),
                     key=lambda e: e[0])
        oci += [c for c, _ in ent]
        ov += [v for _, v in ent]
        orp.append(len(oci))
    return np.array(orp, np.int32), np.array(oci, np.int32), np.array(ov)


def cuper_global_row(channel, lane, packed_row):
    """Inverse of cuper_physical_pe_for_row (host/cuper_control_matrix.hpp:48-54)."""
    packet = (packed_row >> 1) * 128 + (channel >> 1) + (channel & 1) * 8 + lane * 16
    return packet * 2 + (packed_row & 1)

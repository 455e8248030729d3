"""The completeness argument of the cell-list broad phase (melody2d_b200/csrc/mel_prox.cu, cl_*),
checked on the CPU with the kernel's arithmetic restated in Python floats (IEEE doubles, like the
device): a border box is binned by its lower corner into a hashed grid whose columns wrap over the
period; a query gathers the buckets of the cells that a box of the run's largest width and height
overlapping it (with some period shift) can have its corner in, one cell wider on every side, plus
the big boxes kept out of the grid.  For random boxes, periods from tiny to huge, negative
coordinates and shifted copies, every border that the all-pairs pass accepts for a query must be
among the gathered ones (hash collisions only add borders, which the exact tests reject)."""
import math

import numpy as np
import pytest

U32 = 0xFFFFFFFF


def bucket(x, y, xmin, hx, h, ncx, T):
    cx = math.floor((x - xmin) / hx)
    cw = cx % ncx                                   # the kernel adds ncx to a negative remainder
    cy = math.floor(y / h)
    k = ((cw * 73856093) & U32) ^ (((cy & U32) * 19349663) & U32)
    return k & (T - 1)


def shifts(xmin, xmax, pxmin, period):
    inv = 1.0 / period
    return math.floor((xmin - pxmin) * inv), math.floor((xmax - pxmin) * inv)


def overlaps(b1, b2, s1, s2, period):
    """The all-pairs acceptance: y overlap and an x overlap for some shift in the reference's range."""
    (x0a, x1a, y0a, y1a), (x0b, x1b, y0b, y1b) = b1, b2
    if y1b < y0a or y1a < y0b:
        return False
    for s in range(s1[0] - s2[1], s1[1] - s2[0] + 1):
        if x1b + s * period > x0a and x0b + s * period < x1a:
            return True
    return False


def cell_query(b1, boxes, big, grid, W, H, pxmin, hx, h, ncx, T, max_cells=4096):
    """The borders the kernel gathers for box b1 (None: it takes the all-pairs pass)."""
    x0, x1, y0, y1 = b1
    cx0 = math.floor((x0 - W - pxmin) / hx) - 1
    cx1 = math.floor((x1 - pxmin) / hx) + 1
    cy0 = math.floor((y0 - H) / h) - 1
    cy1 = math.floor(y1 / h) + 1
    if cx1 - cx0 + 1 > ncx:
        cx1 = cx0 + ncx - 1
    if cx1 - cx0 + 1 > max_cells or cy1 - cy0 + 1 > max_cells or (cx1 - cx0 + 1) * (cy1 - cy0 + 1) > max_cells:
        return None
    got = set(big)
    for cy in range(cy0, cy1 + 1):
        for cx in range(cx0, cx1 + 1):
            xc = pxmin + (cx + 0.5) * hx
            yc = (cy + 0.5) * h
            got |= grid.get(bucket(xc, yc, pxmin, hx, h, ncx, T), set())
    return got


@pytest.mark.parametrize("seed", range(40))
def test_cell_query_covers_all_pairs(seed):
    rng = np.random.default_rng(seed)
    ext = float(rng.uniform(0.5e-3, 3e-3))             # the largest initial box
    h = 1.5 * ext
    kind = seed % 4
    period = [0.7 * h, 5.3 * h, 40.0 * h, 2.0][kind]  # fewer columns than one box, a few, many, huge
    pxmin = float(rng.uniform(-1.0, 1.0)) * period
    ncx = int(max(1.0, min(1e6, math.floor(period / h))))
    hx = period / ncx
    n = 300
    boxes = []
    for _ in range(n):
        w = float(rng.uniform(0.05, 1.0)) * ext * (1.6 if rng.random() < 0.05 else 1.0)   # a few above a cell
        ht = float(rng.uniform(0.05, 1.0)) * ext
        span = 15 * h if kind == 3 else 3 * period        # a huge period: a dense patch of it
        x0 = pxmin + float(rng.uniform(-span, span))
        y0 = float(rng.uniform(-20 * h, 20 * h))
        boxes.append((x0, x0 + w, y0, y0 + ht))
    for _ in range(3):                                 # walls and plates: far larger than a cell
        x0 = pxmin + float(rng.uniform(-period, period))
        y0 = float(rng.uniform(-20 * h, 20 * h))
        if rng.random() < 0.5:
            boxes.append((x0, x0 + 0.2 * h, y0, y0 + 30 * h))
        else:
            boxes.append((x0, x0 + min(30 * h, 0.9 * period), y0, y0 + 0.2 * h))
    T = 64
    while T < 2 * len(boxes):
        T *= 2
    sh = [shifts(b[0], b[1], pxmin, period) for b in boxes]
    is_big = [(b[1] - b[0] > h or b[3] - b[2] > h) for b in boxes]
    W = max((b[1] - b[0]) for b, bg in zip(boxes, is_big) if not bg)
    H = max((b[3] - b[2]) for b, bg in zip(boxes, is_big) if not bg)
    grid = {}
    for i, (b, bg) in enumerate(zip(boxes, is_big)):
        if not bg:
            grid.setdefault(bucket(b[0], b[2], pxmin, hx, h, ncx, T), set()).add(i)
    big = {i for i, bg in enumerate(is_big) if bg}
    queried = pairs = 0
    for i, b1 in enumerate(boxes):
        got = cell_query(b1, boxes, big, grid, W, H, pxmin, hx, h, ncx, T)
        if got is None:
            continue                                   # all pairs: complete by construction
        queried += 1
        for j, b2 in enumerate(boxes):
            if j != i and overlaps(b1, b2, sh[i], sh[j], period):
                pairs += 1
                assert j in got, (seed, i, j, b1, b2)
    assert queried > len(boxes) // 2 and pairs > 0

"""Scan formulation of the reference's nearest-pixel inpainting, in numpy.

compute_nearest (rvs/src/inpainting.cpp:104-136) runs column-major
Gauss-Seidel sweeps over an (x, y, dist) map, alternating forward (x and y
ascending) and reverse, until a sweep changes nothing.  After the forward
sweep 0 and the reverse sweep 1 the distances equal the exact L1 distance
transform, so sweep 2 never changes anything and the result is the state
after sweep 1.  Both sweeps are min-plus recurrences with a fixed
neighbour priority and can be evaluated with row and column scans:

  sweep 0: D0, S0 (p) = lexmin over q with q.x <= p.x, q.y <= p.y of
           (C(q).d + |p - q|, C(q).src.x, C(q).src.y), where C(q) is
           (0, q) for a non-hole and (1, down(q)) / (1, right(q)) for a
           hole whose down / right neighbour is a non-hole (down first);
  sweep 1: T(q) = best of stay (D0(q), S0(q)), left (D0+1, S0 of left),
           up (D0+1, S0 of up), in that priority; for a hole p the best
           candidate in its lower-right quadrant is taken from its own
           column (minimum y) when that column holds a minimum, otherwise
           the minimum with the largest y, then the smallest x; p changes
           only on strict improvement.

This module is the executable statement of that derivation.  The tests
check it against the oracle's literal sweeps on random masks, and the CUDA
inpainting kernels implement the same scans.
"""
import numpy as np

INF = 1 << 40


def inpaint_sources(hole):
    """hole: bool (H, W).  Returns int32 (H, W, 2) source (x, y) per pixel."""
    h, w = hole.shape
    big = w + h
    ys, xs = np.mgrid[0:h, 0:w]

    # ---- sweep 0: per-pixel candidate C(q) as (d, sx, sy)
    cd = np.full((h, w), INF, np.int64)
    csx = xs.copy()
    csy = ys.copy()
    cd[~hole] = 0
    down_ok = np.zeros((h, w), bool)
    down_ok[:-1, :] = hole[:-1, :] & ~hole[1:, :]
    right_ok = np.zeros((h, w), bool)
    right_ok[:, :-1] = hole[:, :-1] & ~hole[:, 1:]
    sel_r = right_ok & ~down_ok
    cd[down_ok] = 1
    csy[down_ok] += 1
    cd[sel_r] = 1
    csx[sel_r] += 1

    def lexmin(a, b):
        return a if a <= b else b

    # forward row scan: R(p) = min over q.x <= p.x of (cd + p.x - q.x, sx, sy)
    R = np.empty((h, w, 3), np.int64)
    for y in range(h):
        best = (INF, 0, 0)
        for x in range(w):
            best = (best[0] + 1, best[1], best[2])
            best = lexmin(best, (int(cd[y, x]), int(csx[y, x]), int(csy[y, x])))
            R[y, x] = best
    # forward column scan
    D0 = np.empty((h, w), np.int64)
    S0 = np.empty((h, w, 2), np.int64)
    for x in range(w):
        best = (INF, 0, 0)
        for y in range(h):
            best = (best[0] + 1, best[1], best[2])
            best = lexmin(best, tuple(int(v) for v in R[y, x]))
            if best[0] >= INF // 2:
                D0[y, x] = big
                S0[y, x] = (x, y)
            else:
                D0[y, x] = best[0]
                S0[y, x] = (best[1], best[2])
    D0[~hole] = 0
    S0[~hole] = np.stack([xs, ys], -1)[~hole]
    # A hole with no candidate keeps the initial state (big, itself).
    no = hole & (D0 >= big)
    D0[no] = big
    S0[no] = np.stack([xs, ys], -1)[no]

    # ---- sweep 1: T(q) (stay > left > up) and T'(q) (left > up)
    def opt(d, s):
        return (int(d), int(s[0]), int(s[1]))

    T = np.empty((h, w, 3), np.int64)
    Tp = np.empty((h, w, 3), np.int64)
    for y in range(h):
        for x in range(w):
            if not hole[y, x]:
                T[y, x] = (0, x, y)
                Tp[y, x] = (0, x, y)
                continue
            cands = [opt(D0[y, x], S0[y, x])]
            side = []
            if x > 0:
                side.append(opt(D0[y, x - 1] + 1, S0[y, x - 1]))
            if y > 0:
                side.append(opt(D0[y - 1, x] + 1, S0[y - 1, x]))
            best = None
            for c in cands + side:
                if best is None or c[0] < best[0]:
                    best = c
            T[y, x] = best
            bp = None
            for c in side:
                if bp is None or c[0] < bp[0]:
                    bp = c
            Tp[y, x] = bp if bp is not None else (INF, x, y)

    D1 = D0.copy()
    S1 = S0.copy()
    # off-column: backward row scan over q.x > x of (T.d + q.x, q.x)
    RR = np.empty((h, w, 2), np.int64)
    for y in range(h):
        best = (INF, 0)
        for x in range(w - 1, -1, -1):
            RR[y, x] = best
            best = min(best, (int(T[y, x, 0]) + x, x))
    for x in range(w):
        # column part: q = (x, y') with y' > y: (T.d + y', y'), plus q = p via T'
        colbest = (INF, 0)
        offbest = (INF, 0, 0)  # (cost + y', -y', qx)
        for y in range(h - 1, -1, -1):
            # off-column candidates of row y for column x
            if RR[y, x, 0] < INF:
                cand = (int(RR[y, x, 0]) - x + y, -y, int(RR[y, x, 1]))
                offbest = min(offbest, cand)
            if hole[y, x]:
                cc = (int(Tp[y, x, 0]), y)
                if colbest[0] < INF:
                    cc = min(cc, (colbest[0] - y, colbest[1]))
                oc = (offbest[0] - y, offbest[1], offbest[2]) if offbest[0] < INF else (INF, 0, 0)
                if cc[0] <= oc[0]:
                    cost = cc[0]
                    qy = cc[1]
                    src = Tp[y, x, 1:] if qy == y else T[qy, x, 1:]
                else:
                    cost = oc[0]
                    qy, qx = -oc[1], oc[2]
                    src = T[qy, qx, 1:]
                if cost < D0[y, x]:
                    D1[y, x] = cost
                    S1[y, x] = src
            colbest = min(colbest, (int(T[y, x, 0]) + y, y))
    return S1.astype(np.int32)

"""CPU restatement of StratifiedCombPopulationControl's bin targets
(population/CombPopulationControl.hpp:416-488) and of the copies appendCombBin
makes per bin (:347-413).  Test infrastructure: a checker for the engine's
stratified comb and for the reference build's, never called by the engine.

`expected_counts` returns, per (cell, bin), the number of census particles
the reference's activate writes for that bin: the target where the bin is
combed (each tooth below the target fires once the run's weights sum to the
bin weight), else one per kept particle plus ceil(w / ideal) per split one.
Weights given as dyadic numbers make every sum exact, so the restatement and
both implementations see the same bin and cell weights in any order.
"""
import math

import numpy as np


def bin_of(nu, bounds):
    """findGroup's rule on the bin edges: the first g with nu < bounds[g + 1], else the last."""
    B = len(bounds) - 1
    g = np.searchsorted(bounds[1:B], nu, side="right")
    return np.minimum(g, B - 1)


def bin_targets(bin_w, counts, total_w, ncells, nmin, factor, min_per_bin):
    """Targets per (cell, bin) as activate allocates them (:416-470).  bin_w
    and counts are (ncells, B); returns an integer array of the same shape."""
    N, B = bin_w.shape
    ntotal = int(float(ncells * nmin) * factor)
    out = np.zeros((N, B), dtype=np.int64)
    for c in range(N):
        cw = float(sum(bin_w[c]))
        if cw <= 0.0:
            continue
        cell_target = min(nmin * 20, max(nmin, int(ntotal * cw / total_w)))
        active = [g for g in range(B) if counts[c, g] > 0]
        if not active:
            continue
        target = [0] * B
        allocated = 0
        if len(active) * min_per_bin <= cell_target:
            for g in active:
                target[g] = min_per_bin
                allocated += min_per_bin
        else:
            active = sorted(active, key=lambda g: -bin_w[c, g])   # heaviest first, ties in bin order
            for g in active[:min(len(active), cell_target)]:
                target[g] = 1
                allocated += 1
        remaining = cell_target - allocated if cell_target > allocated else 0
        prop = 0
        frac = [0.0] * B
        for g in active:
            if target[g] == 0:
                continue
            exact = float(remaining) * bin_w[c, g] / cw
            extra = int(math.floor(exact))
            target[g] += extra
            prop += extra
            frac[g] = exact - extra
        while prop < remaining:
            best, bf = None, -1.0
            for g in active:
                if target[g] > 0 and frac[g] > bf:
                    best, bf = g, frac[g]
            if best is None:
                break
            target[best] += 1
            frac[best] = 0.0
            prop += 1
        out[c] = target
    return out


def expected_counts(cell, nu, w, bounds, ncells, nmin, factor, min_per_bin):
    """Output particles per (cell, bin) of activate on the census (cell, nu, w)."""
    B = len(bounds) - 1 if bounds is not None else 1
    keep = w > 0
    g = bin_of(nu, bounds) if B > 1 else np.zeros(len(w), np.int64)
    bin_w = np.zeros((ncells, B))
    counts = np.zeros((ncells, B), np.int64)
    np.add.at(bin_w, (cell[keep], g[keep]), w[keep])
    np.add.at(counts, (cell[keep], g[keep]), 1)
    target = bin_targets(bin_w, counts, float(w[keep].sum()), ncells, nmin, factor, min_per_bin)
    out = np.zeros((ncells, B), np.int64)
    for c, b in zip(*np.nonzero(counts)):
        tg, bw = target[c, b], bin_w[c, b]
        if tg == 0 or bw <= 0:
            continue
        if counts[c, b] > tg:
            out[c, b] = tg
        else:
            ideal = bw / tg
            ws = w[keep & (cell == c) & (g == b)]
            out[c, b] = sum(int(math.ceil(x / ideal)) if x > 2.0 * ideal else 1 for x in ws)
    return out, target, bin_w

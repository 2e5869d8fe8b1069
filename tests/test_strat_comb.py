"""StratifiedCombPopulationControl (population/CombPopulationControl.hpp:255-511)
through the reference build, against the restatement of its bin targets in
oracle/strat_comb.py: output particles per (cell, bin), weights and energy per
bin.  The census has dyadic weights, so every sum is exact in any order."""
import numpy as np

from oracle import strat_comb
from storm_b200 import problems


def strat_census(p, n, seed, Particles):
    """Census over the cells with frequencies log-uniform over the groups and
    distinct dyadic weights; a tenth of the cells hold a few heavy particles
    (the split path), the rest many light ones (the comb path)."""
    rng = np.random.default_rng(seed)
    N = p.ncells
    cell = rng.integers(0, N, n).astype(np.uint32)
    heavy = rng.choice(N, max(1, N // 10), replace=False)
    cell[np.isin(cell, heavy)] = rng.choice(np.setdiff1d(np.arange(N), heavy), np.isin(cell, heavy).sum())
    cell[:len(heavy)] = heavy
    k = rng.permutation(np.arange(1, 200 * n + 1))[:n].astype(np.float64)
    w = k * 2.0 ** -20
    w[:len(heavy)] *= 64.0
    w[rng.random(n) < 0.02] = 0.0
    b = p.group_bounds
    nu = np.exp(rng.uniform(np.log(b[0]), np.log(b[-1]), n))
    out = Particles(n)
    xc, yc, zc = p.cell_centers()
    out.x, out.y, out.z = xc[cell].copy(), yc[cell].copy(), zc[cell].copy()
    out.vx[:] = 3e10
    out.weight, out.initial_weight = w, w.copy()
    out.cell = cell
    out.frequency = nu
    out.id = np.arange(n, dtype=np.uint64)
    return out


def check_strat(p, pre, post):
    """Counts per (cell, bin) equal the restatement's; energy per (cell, bin)
    is conserved where the bin has a target; combed bins hold equal weights."""
    b = p.strat_bounds
    exp, target, bin_w = strat_comb.expected_counts(pre.cell.astype(np.int64), pre.frequency, pre.weight, b,
                                                    p.ncells, p.comb_nmin, p.comb_factor, p.strat_min_per_bin)
    g = strat_comb.bin_of(post.frequency, b)
    got = np.zeros_like(exp)
    np.add.at(got, (post.cell.astype(np.int64), g), 1)
    np.testing.assert_array_equal(got, exp)
    e_out = np.zeros_like(bin_w)
    np.add.at(e_out, (post.cell.astype(np.int64), g), post.weight)
    has = target > 0
    assert np.allclose(e_out[has], bin_w[has], rtol=1e-12, atol=0)
    assert (e_out[~has] == 0).all()
    # bins with fewer particles than their target are kept or split; the rest combed to equal weights
    pre_counts = np.zeros_like(exp)
    keep = pre.weight > 0
    np.add.at(pre_counts, (pre.cell[keep].astype(np.int64), strat_comb.bin_of(pre.frequency[keep], b)), 1)
    combed = has & (pre_counts > target)
    for c, q in zip(*np.nonzero(combed)):
        ws = post.weight[(post.cell == c) & (g == q)]
        assert np.allclose(ws, bin_w[c, q] / target[c, q], rtol=1e-15)
    assert combed.sum() > 10 and (has & ~combed).sum() > 5 and (~has & (pre_counts > 0)).sum() > 0
    return exp


def test_reference_stratified_comb_matches_restatement(ref_lib):
    p = problems.strat_cube()
    pre = strat_census(p, 4000, 5, ref_lib.Particles)
    post = ref_lib.Reference(p).comb(pre)
    check_strat(p, pre, post)

"""The engine's StratifiedCombPopulationControl (frequency bins) on the GPU:
on a given census, the output particles per (cell, bin), the energy per bin
and the combed weights equal what the reference's activate produces
(oracle/strat_comb.py restates it; tests/test_strat_comb.py pins the
restatement to the reference build); whole steps conserve energy and agree
with the reference's serial path within the seed-to-seed scatter."""
import numpy as np
import pytest

from storm_b200 import _abi as A
from storm_b200 import problems
from storm_b200.engine import Engine, Particles

from test_strat_comb import check_strat, strat_census

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [A.PRECISION_FP64, A.PRECISION_FP32_TRACK])
def test_stratified_comb_on_a_given_census(precision):
    p = problems.strat_cube(precision=precision)
    pre = strat_census(p, 4000, 5, Particles)
    e = Engine(p)
    post = e.population_control(pre)
    if precision == A.PRECISION_FP32_TRACK:
        # FP32 census records hold the frequency as a float: bin by the same float
        pre.frequency = pre.frequency.astype(np.float32).astype(np.float64)
    check_strat(p, pre, post)
    # the census radiation energy per cell is the combed census's
    np.testing.assert_allclose(e.cells()["erad_census"],
                               np.bincount(post.cell, weights=post.weight, minlength=p.ncells), rtol=1e-12)
    e.close()


def test_stratified_comb_matches_reference_counts(ref_lib):
    p = problems.strat_cube(seed=9)
    pre = strat_census(p, 5000, 8, ref_lib.Particles)
    ref = ref_lib.Reference(p).comb(pre)
    pre_e = strat_census(p, 5000, 8, Particles)
    e = Engine(p)
    got = e.population_control(pre_e)
    from oracle import strat_comb
    b = p.strat_bounds

    def counts(q):
        out = np.zeros((p.ncells, p.strat_bins), np.int64)
        np.add.at(out, (q.cell.astype(np.int64), strat_comb.bin_of(q.frequency, b)), 1)
        return out
    np.testing.assert_array_equal(counts(got), counts(ref))
    e.close()


def _balance(st):
    src = st["energy_census_in"] + st["energy_emitted"]
    sink = st["energy_deposited"] + st["energy_escaped"] + st["energy_census_pre_comb"]
    return abs(src - sink) / max(src, 1e-300)


def test_stratified_comb_steps_vs_reference(ref_lib):
    from batchcheck import assert_agree, run_batch

    def check(m, st):
        if isinstance(m, Engine):
            assert _balance(st) < 1e-10

    def prob(s):
        return problems.strat_cube(n=5, seed=s, comb_nmin=6)
    assert_agree(run_batch(Engine, prob, range(20, 36), 4, check), run_batch(ref_lib.Reference, prob, range(60, 76), 4),
                 "stratified comb cube 5^3: engine vs reference")

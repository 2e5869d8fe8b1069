"""The oracle (oracle/imc_oracle.c) pinned against the reference: live runs of the
reference build where it exists, and the committed golden fixtures everywhere."""
import numpy as np
import pytest

from conftest import golden
from storm_b200 import problems
from storm_b200.units import UNITS


def test_units_match_reference(ref_lib):
    u = ref_lib.units()
    for k in ("clight", "arad", "sigma_sb", "kev_kelvin", "k_boltz", "kev"):
        assert u[k] == UNITS[k], k


def test_philox_known_answers(oracle_lib):
    # Random123 known-answer vectors for Philox4x32-10
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, out in kat:
        assert list(oracle_lib.philox(ctr, key)) == out


def test_uniforms_open_interval(oracle_lib):
    u = np.array([oracle_lib.uniform(42, 1, s, p, d) for s in range(3) for p in range(20) for d in range(20)])
    assert (u > 0).all() and (u < 1).all()
    assert abs(u.mean() - 0.5) < 0.03


def _replay_oracle(orc, problem, g):
    o = orc.Oracle(problem)
    o.set_cell_physics(g["sigma_a"], np.zeros(problem.ncells), g["fleck"])
    b = orc.ReplayBatch(g["before"], g["cell"], g["tape_offset"], g["tape_length"], g["tape"])
    o.replay(b)
    return b


def _check_replay_exact(b, g, ncells):
    names = ["phys_x", "phys_y", "phys_z", "phys_vx", "phys_vy", "phys_vz", "phys_time_left", "phys_weight"]
    for k, nm in enumerate(names):
        np.testing.assert_array_equal(b[nm], g["after"][:, k], err_msg=nm)
    np.testing.assert_array_equal(b["phys_status"], g["status"])
    np.testing.assert_array_equal(b["draws_used"], g["tape_length"])
    np.testing.assert_array_equal(b["used_random_walk"], g["used_rw"])
    moved = g["status"] == 1
    np.testing.assert_array_equal(b["phys_next_cell"][moved].astype(np.int64), g["next"][moved])
    # tallies: re-adding our deposit to the reference's value before the call
    np.testing.assert_array_equal(g["tallies"][:, 2] + b["dep_erad"], g["tallies"][:, 3])
    mat = g["tallies"][:, 0] + b["dep_material"]
    scale = np.maximum(np.abs(g["tallies"][:, 1]), 1e-300)
    assert (np.abs(mat - g["tallies"][:, 1]) <= 4e-16 * scale).all()
    # manager handling: our post-manager state is the reference's next call's input
    ch = g["next_cell"] >= 0
    mgr = np.stack([b["mgr_x"], b["mgr_y"], b["mgr_z"], b["mgr_vx"], b["mgr_vy"], b["mgr_vz"]], 1)
    np.testing.assert_array_equal(mgr[ch], g["next_before"][ch])
    np.testing.assert_array_equal(b["mgr_cell"][ch].astype(np.int64), g["next_cell"][ch])


def test_replay_golden_slab(oracle_lib):
    g = golden("replay_slab.npz")
    p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50)
    b = _replay_oracle(oracle_lib, p, g)
    _check_replay_exact(b, g, p.ncells)
    # the fixture exercises boundary reflections and escapes
    assert ((g["status"] == 1) & (g["next"] >= p.ncells)).sum() > 50


def test_replay_golden_cube_random_walk(oracle_lib):
    g = golden("replay_cube_rw.npz")
    p = problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20)
    b = _replay_oracle(oracle_lib, p, g)
    _check_replay_exact(b, g, p.ncells)
    assert g["used_rw"].sum() > 500


@pytest.mark.parametrize("which", ["slab", "cube"])
def test_replay_live_reference(oracle_lib, ref_lib, which):
    if which == "slab":
        p = problems.gray_slab(new_photons_per_cell=4, face_packets=1500, comb_nmin=40, seed=7)
        warm = 3
    else:
        p = problems.step_cube(n=6, new_photons_per_cell=2, face_packets=30, comb_nmin=10, seed=9)
        warm = 2
    r = ref_lib.Reference(p)
    for _ in range(warm):
        r.step()
    r.record_begin(300000)
    r.step()
    r.record_end()
    rec = r.records()
    c = r.cells()
    g = dict(before=rec["before"], after=rec["after"], status=rec["status"], next=rec["next"].astype(np.int64),
             tallies=rec["tallies"], cell=rec["cell"], used_rw=rec["used_rw"], tape=rec["tape"],
             tape_offset=rec["tape_offset"], tape_length=rec["tape_length"], sigma_a=c["sigma_a"], fleck=c["fleck"])
    n = len(g["cell"])
    same = np.zeros(n, bool)
    same[:-1] = rec["id"][1:] == rec["id"][:-1]
    nb = np.full((n, 6), np.nan)
    nc = np.full(n, -1, np.int64)
    nb[:-1][same[:-1]] = rec["before"][1:][same[:-1], :6]
    nc[:-1][same[:-1]] = rec["cell"][1:][same[:-1]]
    g["next_before"], g["next_cell"] = nb, nc
    b = _replay_oracle(oracle_lib, p, g)
    _check_replay_exact(b, g, p.ncells)


def test_random_walk_golden(oracle_lib):
    g = golden("rw_samples.npz")
    L = oracle_lib.lib()
    leak = np.array([L.orc_rw_sample_leak(x) for x in g["xi_leak"]])
    rad = np.array([L.orc_rw_sample_radius(t, x) for t, x in zip(g["tau"], g["xi_rad"])])
    np.testing.assert_array_equal(leak, g["leak"])
    np.testing.assert_array_equal(rad, g["radius"])
    surv = np.array([L.orc_rw_survival(t) for t in g["t_grid"]])
    cdf = np.array([L.orc_rw_radial_cdf(x, t) for x, t in zip(g["x_grid"], g["t_grid"])])
    np.testing.assert_array_equal(surv, g["survival"])
    np.testing.assert_array_equal(cdf, g["cdf"])


def test_samplers_golden(oracle_lib):
    g = golden("samplers.npz")
    p = problems.step_cube(n=4)
    np.testing.assert_array_equal(p.x_edges, g["x_edges"])
    o = oracle_lib.Oracle(p)
    off = np.concatenate([[0], np.cumsum(g["cell_draws"])]).astype(np.int64)
    for q, c in enumerate(g["cells"]):
        pos = o.sample_in_cell(int(c), g["cell_tape"][off[q]:off[q + 1]])
        np.testing.assert_array_equal(pos, g["cell_pos"][q])
    for q in range(len(g["vel"])):
        np.testing.assert_array_equal(oracle_lib.isotropic(g["vel_tape"][2 * q:2 * q + 2], UNITS["clight"]), g["vel"][q])
    for q, f in enumerate(g["faces"]):
        np.testing.assert_array_equal(o.point_on_face(int(f), g["face_tape"][3 * q:3 * q + 3]), g["face_pos"][q])


def test_allocation_golden(oracle_lib):
    """Photon counts per cell (nPhotonsVec, RadiationIMC.hpp:2071-2087) are integers:
    bit-exact, including the cells whose share floors one below the even split."""
    g = golden("allocation_slab.npz")
    for s in range(len(g["photons"])):
        p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50)
        p.temperature = g["temperature"][s]
        p.internal_energy = g["internal_energy"][s]
        o = oracle_lib.Oracle(p)
        o.phase("begin"); o.phase("prestep"); o.phase("emit")
        counts, _ = o.emission()
        np.testing.assert_array_equal(counts, g["photons"][s])
        np.testing.assert_array_equal(o.cells()["sigma_a"], g["sigma_a"][s])
        np.testing.assert_array_equal(o.cells()["fleck"], g["fleck"][s])
    assert (g["photons"][0] == 49).any(), "fixture no longer covers the floor-below case"


def _balance(st):
    src = st["energy_census_in"] + st["energy_emitted"]
    sink = st["energy_deposited"] + st["energy_escaped"] + st["energy_census_pre_comb"]
    return abs(src - sink) / max(src, 1e-300)


def test_oracle_energy_conservation(oracle_lib):
    for p in (problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50),
              problems.step_cube(n=8, new_photons_per_cell=3, face_packets=40, comb_nmin=20)):
        o = oracle_lib.Oracle(p)
        for _ in range(3):
            st = o.step()
            assert _balance(st) < 1e-10
            assert abs(st["energy_census_out"] - st["energy_census_pre_comb"]) <= 1e-10 * st["energy_census_pre_comb"]


def _comb_invariants(before, after, p, exact_counts=True):
    N = p.ncells
    nmin, factor = p.comb_nmin, p.comb_factor
    W = np.bincount(before.cell, weights=before.weight, minlength=N)
    assert before.n > 0
    cnt = np.bincount(before.cell[before.weight > 0], minlength=N)
    tot = W.sum()
    ntotal = int(N * nmin * factor)
    share = np.floor(ntotal * W / tot).astype(np.int64)
    nin = np.minimum(nmin * 20, np.maximum(nmin, share))
    out_cnt = np.bincount(after.cell, minlength=N)
    out_W = np.bincount(after.cell, weights=after.weight, minlength=N)
    combed = cnt > nin
    assert combed.any() and (~combed & (cnt > 0)).any()
    if exact_counts:
        assert (out_cnt[combed] == nin[combed]).all()
    np.testing.assert_allclose(out_W, W, rtol=1e-12, atol=1e-300)
    for c in np.where(combed)[0][:50]:
        w = after.weight[after.cell == c]
        np.testing.assert_allclose(w, W[c] / nin[c], rtol=1e-15)


def synthetic_census(p, n, seed, Particles):
    """Census spread over the cells with lognormal weights; a few cells hold
    only heavy particles so the split path (CombPopulationControl.hpp:164-194)
    runs next to the comb path (:196-225)."""
    rng = np.random.default_rng(seed)
    N = p.ncells
    cell = rng.integers(0, N, n).astype(np.uint32)
    heavy = rng.choice(N, max(1, N // 10), replace=False)
    cell[: len(heavy) * 2] = np.repeat(heavy, 2)
    w = rng.lognormal(0.0, 1.0, n)
    w[: len(heavy) * 2] *= 50.0
    w[rng.random(n) < 0.02] = 0.0          # zero weights are skipped (:136-137)
    out = Particles(n)
    xc, yc, zc = p.cell_centers()
    out.x, out.y, out.z = xc[cell].copy(), yc[cell].copy(), zc[cell].copy()
    out.vx[:] = 3e10
    out.weight, out.initial_weight = w, w.copy()
    out.cell = cell
    out.id = np.arange(n, dtype=np.uint64)
    return out


def test_comb_invariants_reference_and_oracle(oracle_lib, ref_lib):
    p = problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=8, comb_factor=1.5)
    pre = synthetic_census(p, 3000, 3, ref_lib.Particles)
    post = ref_lib.Reference(p).comb(pre)
    _comb_invariants(pre, post, p)
    o = oracle_lib.Oracle(p)
    o.set_census(pre)
    o.phase("comb")
    _comb_invariants(pre, o.census(), p)


def test_oracle_matches_reference_statistically(oracle_lib, ref_lib):
    """Full time steps: the oracle (Philox streams) and the reference (its own
    mt19937_64 streams) agree cell by cell under the batch gate (per-cell Welch
    z of temperature, deposit and radiation energies, storm_b200.batchstats)."""
    from batchcheck import assert_agree, run_batch

    def prob(s):
        return problems.gray_slab(new_photons_per_cell=5, face_packets=3000, comb_nmin=50, seed=s)
    assert_agree(run_batch(ref_lib.Reference, prob, range(100, 116), 4),
                 run_batch(oracle_lib.Oracle, prob, range(200, 216), 4), "slab: reference vs oracle")

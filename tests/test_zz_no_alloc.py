"""The allocation-free emission allocation (storm_cuda_emission_allocation_noalloc)
against the regular path, through the C ABI.

It is for callers that cannot allocate device memory while they run (an
allocator that owns the device, a no-allocation loop).  This file
sorts last so that a run stopping at the first failure has run everything else;
it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(energy, new_per_cell):
    import torch
    from storm_b200.engine import lib
    L = lib()
    f = L.storm_cuda_emission_allocation_noalloc
    f.argtypes = [C.c_int, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    n = len(energy)
    d_energy = torch.tensor(energy, dtype=torch.float64, device="cuda:0")
    d_photons = torch.full((n,), -1, dtype=torch.int64, device="cuda:0")
    d_offsets = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    rc = f(0, d_energy.data_ptr(), n, new_per_cell, d_photons.data_ptr(), d_offsets.data_ptr(), stream)
    torch.cuda.synchronize()
    assert rc == 0, rc
    return d_photons.cpu().numpy().view(np.uint64), d_offsets.cpu().numpy().view(np.uint64)


def test_noalloc_matches_engine_on_consecutive_calls():
    from storm_b200 import problems
    from storm_b200.engine import Engine
    for p in (problems.gray_slab(new_photons_per_cell=5, face_packets=2000, comb_nmin=50),
              problems.step_cube(n=16, new_photons_per_cell=3, face_packets=50, comb_nmin=10)):
        e = Engine(p)
        for s in range(2):
            e.step()
            e.phase("begin")
            e.phase("prestep")
            e.phase("emit")
            photons, energy = e.emission()      # the regular entry point's result
            first = _noalloc(energy, p.new_photons_per_cell)
            second = _noalloc(energy, p.new_photons_per_cell)
            for ph, off in (first, second):
                np.testing.assert_array_equal(ph, photons)
                np.testing.assert_array_equal(off[:-1], np.concatenate([[0], np.cumsum(photons)[:-1]]))
                assert off[-1] == photons.sum()


def _allocation_formula(energy, new_per_cell):
    """The reference's count per cell (radiation/RadiationIMC.hpp:2058-2087) on
    the host: floor(E / S * N * n * 10) clamped to [n, 20 n], S the
    left-to-right sum (np.cumsum adds in order)."""
    total = np.cumsum(energy)[-1]
    tp = float(len(energy) * new_per_cell * 10)
    share = np.floor(energy / total * tp).astype(np.uint64)
    out = np.clip(share, new_per_cell, 20 * new_per_cell).astype(np.uint64)
    out[energy <= 0] = 0
    return out


@pytest.mark.parametrize("case", ["random", "uniform"])
def test_noalloc_large_meshes_take_no_device_memory(case):
    """More than 2^21 cells, so that the prefix sum's tile totals span several
    chunks.  "uniform": every cell's share is an exact integer, which puts each
    floor on the edge of the blocked total's error interval and sends the call
    down its exact left-to-right fallback on the device.  Two calls in a row
    give the host formula's counts, and the second changes neither torch's
    allocation nor the device's free memory."""
    import torch
    n = (1 << 21) + 4099
    rng = np.random.default_rng(7)
    if case == "random":
        energy = rng.lognormal(0.0, 2.0, n)
        energy[::97] = 0.0
    else:
        energy = np.full(n, 0.5)
    expect = _allocation_formula(energy, 3)
    first = _noalloc(energy, 3)
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info(0)[0], torch.cuda.memory_allocated(0)
    second = _noalloc(energy, 3)
    free1, alloc1 = torch.cuda.mem_get_info(0)[0], torch.cuda.memory_allocated(0)
    for ph, off in (first, second):
        np.testing.assert_array_equal(ph, expect)
        np.testing.assert_array_equal(off[:-1], np.concatenate([[0], np.cumsum(expect)[:-1]]))
        assert off[-1] == expect.sum()
    # the helper's own tensors are freed before the second measurement
    assert alloc1 == alloc0 and free1 == free0, (alloc0, alloc1, free0, free1)


def test_noalloc_rejects_sizes_beyond_limit():
    from storm_b200.engine import lib
    f = lib().storm_cuda_emission_allocation_noalloc
    f.argtypes = [C.c_int, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    dummy = C.c_void_p(16)
    assert f(0, dummy, (1 << 24) + 1, 5, dummy, dummy, None) == 1   # STORM_ERR_INVALID_ARG, nothing launched
    assert f(0, dummy, 0, 5, dummy, dummy, None) == 1

"""The allocation-free emission allocation (storm_cuda_emission_allocation_noalloc)
against the regular path, through the C ABI.

It is for callers that cannot allocate device memory while they run (graph
capture, an allocator that owns the device, a no-allocation loop).  This file
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


def test_noalloc_rejects_sizes_beyond_limit():
    from storm_b200.engine import lib
    f = lib().storm_cuda_emission_allocation_noalloc
    f.argtypes = [C.c_int, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    dummy = C.c_void_p(16)
    assert f(0, dummy, (1 << 24) + 1, 5, dummy, dummy, None) == 1   # STORM_ERR_INVALID_ARG, nothing launched
    assert f(0, dummy, 0, 5, dummy, dummy, None) == 1

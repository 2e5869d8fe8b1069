"""The C-ABI library loads without a GPU, exports every entry point the header
declares, and its struct layouts match the ctypes mirror."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT
from storm_b200 import _abi as A
from storm_b200 import engine, problems

HEADER = os.path.join(ROOT, "include", "storm_cuda.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(storm_cuda_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    L = engine.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert L.storm_cuda_abi_version() == A.ABI_VERSION


def test_struct_layout_matches_header():
    prog = r'''
#include <stddef.h>
#include <stdio.h>
#include "storm_cuda.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(StormProblemDesc), sizeof(StormParticlesSoA), sizeof(StormStepStats),
         sizeof(StormReplayBatch), sizeof(StormBoxFace));
  printf("%zu %zu %zu %zu\n", offsetof(StormProblemDesc, faces), offsetof(StormProblemDesc, seed),
         offsetof(StormProblemDesc, device), offsetof(StormReplayBatch, used_random_walk));
  printf("%zu %zu %zu\n", sizeof(StormServerConfig), sizeof(StormRequestResult), sizeof(StormServerStats));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write(prog)
        r = subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), src, "-o", exe], capture_output=True)
        if r.returncode != 0:
            pytest.skip("no C compiler")
        out = subprocess.run([exe], capture_output=True, text=True).stdout.split()
    sizes = [int(x) for x in out]
    assert sizes[:5] == [C.sizeof(A.StormProblemDesc), C.sizeof(A.StormParticlesSoA), C.sizeof(A.StormStepStats),
                         C.sizeof(A.StormReplayBatch), C.sizeof(A.StormBoxFace)]
    assert sizes[5:9] == [A.StormProblemDesc.faces.offset, A.StormProblemDesc.seed.offset,
                          A.StormProblemDesc.device.offset, A.StormReplayBatch.used_random_walk.offset]
    assert sizes[9:] == [C.sizeof(A.StormServerConfig), C.sizeof(A.StormRequestResult), C.sizeof(A.StormServerStats)]


def _create(desc):
    h = C.c_void_p()
    return engine.lib().storm_cuda_create(C.byref(desc), C.byref(h)), h


def test_create_rejects_invalid_descriptors():
    p = problems.gray_slab()
    d = p.to_desc()
    d.abi_version = 99
    assert _create(d)[0] == 1
    d = p.to_desc()
    d.new_photons_per_cell = 0          # RadiationIMC requires newPhotonsPerCell > 0
    assert _create(d)[0] == 1
    d = p.to_desc()
    d.nx = 0
    assert _create(d)[0] == 1
    d = p.to_desc()
    d.opacity_kind = 9
    assert _create(d)[0] == 6
    e = p.x_edges.copy()
    e[3] = e[2]                          # edges must increase strictly
    p2 = problems.gray_slab()
    p2.x_edges = e
    assert _create(p2.to_desc())[0] == 1


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    rc, _ = _create(problems.gray_slab().to_desc())
    assert rc == 7   # STORM_ERR_NO_DEVICE: no CPU fallback


def test_dropin_header_compiles_and_fails_loudly_without_device():
    """MonteCarloManagerCUDA compiled against the reference's types (built
    where the reference sources exist): it loads, and constructing it without a
    GPU throws the reference's StormError instead of falling back to the CPU."""
    path = os.path.join(ROOT, "oracle", "_ref", "libstormdropin.so")
    if not os.path.exists(path):
        pytest.skip("drop-in harness not built")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    L = C.CDLL(path)
    for s in ("dropin_create", "dropin_step", "dropin_destroy", "dropin_ref", "dropin_get_cells"):
        assert hasattr(L, s), s
    L.dropin_create.restype = C.c_void_p
    L.dropin_create.argtypes = [C.POINTER(A.StormProblemDesc), C.c_int, C.c_char_p, C.c_size_t]
    desc = problems.gray_slab().to_desc()
    err = C.create_string_buffer(512)
    assert not L.dropin_create(C.byref(desc), 0, err, 512)
    msg = err.value.decode()
    assert "MonteCarloManagerCUDA" in msg and "storm_cuda_create" in msg, msg


def test_server_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    cfg = A.StormServerConfig(0, 4, 2, 0, 0)
    h = C.c_void_p()
    assert engine.lib().storm_server_create(C.byref(cfg), C.byref(h)) == 7   # STORM_ERR_NO_DEVICE


def test_memory_cache_calls_without_device():
    """The device memory cache's counters read without a GPU (nothing allocated);
    releasing it needs a device and says so."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    c = engine.pool_counters()
    assert set(c) == {"mallocs", "frees", "cached_bytes", "live_bytes"}
    assert all(isinstance(v, int) and v >= 0 for v in c.values())
    with pytest.raises(engine.StormError):
        engine.release_cached(0)


def test_tuning_calls_reject_a_null_handle():
    L = engine.lib()
    b, t = C.c_uint32(), C.c_int()
    assert L.storm_cuda_autotune_transport(None, 1) == 1   # STORM_ERR_INVALID_ARG
    assert L.storm_cuda_transport_burst(None, C.byref(b), C.byref(t)) == 1


def test_serving_mix_is_seeded():
    a = problems.serving_mix(8)
    b = problems.serving_mix(8)
    assert [(p.shape, s, p.sigma_a[0], p.new_photons_per_cell) for p, s in a] == \
           [(p.shape, s, p.sigma_a[0], p.new_photons_per_cell) for p, s in b]
    assert all(16 <= p.shape[0] <= 48 and 5 <= s <= 20 for p, s in a)


def test_host_step_rejects_missing_arguments():
    """storm_cuda_step_host checks its handle and buffers before touching a device."""
    L = engine.lib()
    s = A.StormParticlesSoA()
    cnt = C.c_uint64()
    st = A.StormStepStats()
    assert L.storm_cuda_step_host(None, 1e-11, C.byref(s), C.byref(s), 0, C.byref(cnt), C.byref(st)) == 1

"""The entry point for callers that cannot allocate GPU memory.

ce_advance_device_noalloc runs the creature kernel with its scratch in a
fixed array inside the library, for callers that must not call cudaMalloc or
cudaFree (cudaFree waits for all work on the GPU, a stall on the evolution
loop's critical path) or whose device memory belongs to another allocator.
This test calls it through the C ABI twice in a row on the same batch and
checks both results against the regular device entry's, to the bit (the
engine's results are exact, so the tolerance is zero). The file sorts last so
that a run that stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def test_no_alloc_entry_matches_the_device_entry_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    w = WORKLOADS["game"]
    world = w.world(duration=2.0)
    wave = ce.pack(ce.generate(w.spec, 20_000), world)
    flags, rate = ce.world_flags(world), world.rate or 60
    params = ce.make_params(world, 0, len(wave), 0)
    d_lanes = torch.from_numpy(wave.lanes.view(np.int32)).to(dev)
    d_muscles = torch.from_numpy(wave.muscles).to(dev)
    d_heads = torch.from_numpy(wave.heads.view(np.int32).reshape(-1)).to(dev)
    stream = torch.cuda.current_stream(dev)

    # The regular entry, with scratch the caller allocates.
    with ce.Engine(0) as eng:
        d_res = torch.zeros(len(wave) * 19, dtype=torch.float32, device=dev)
        d_counter = torch.zeros(16, dtype=torch.int32, device=dev)
        d_scratch = torch.empty(eng.scratch_bytes(flags, rate, wave.max_nodes, wave.max_muscles, len(wave)), dtype=torch.uint8,
                                device=dev)
        eng.advance_device(d_lanes.data_ptr(), d_muscles.data_ptr(), d_heads.data_ptr(), d_res.data_ptr(),
                           d_counter.data_ptr(), d_scratch.data_ptr(), params, flags, rate, wave.max_nodes,
                           wave.max_muscles, stream.cuda_stream)
        torch.cuda.synchronize(dev)
        expected = d_res.cpu().numpy().view(np.uint32)

    lib = ce.lib()
    assert lib.ce_noalloc_scratch_bytes() == 32 << 20
    for call in range(2):
        d_out = torch.full((len(wave) * 19,), float("nan"), dtype=torch.float32, device=dev)
        status = lib.ce_advance_device_noalloc(d_lanes.data_ptr(), d_muscles.data_ptr(), d_heads.data_ptr(),
                                               d_out.data_ptr(), C.byref(params), flags, rate, wave.max_nodes,
                                               wave.max_muscles, C.c_void_p(stream.cuda_stream))
        assert status == ce.CE_OK, lib.ce_last_error().decode()
        torch.cuda.synchronize(dev)
        got = d_out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, expected), f"call {call}: {(got != expected).sum()} words differ"


def test_no_alloc_entry_rejects_bad_sizes():
    lib = ce.lib()
    params = ce.make_params(ce.make_world(), 0, 1, 0)
    dummy = C.c_void_p(16)
    assert lib.ce_advance_device_noalloc(dummy, dummy, dummy, dummy, C.byref(params), 1, 60, 40, 8,
                                         None) == ce.CE_ERR_INVALID
    assert b"unsupported" in lib.ce_last_error()

"""Generation dump rows written on the device (ce_dump_rows_device) from
resident results equal the host's rows (ce_dump_rows) to the byte."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS

pytestmark = pytest.mark.gpu


def test_device_dump_rows_equal_host_rows(engine):
    torch = pytest.importorskip("torch")
    w = WORKLOADS["effects"]
    world = w.world(duration=6.0, has_screen=1, screen_seconds=5.0, screen_bar=0.05, screen_bar_young=0.05,
                    screen_bar_reshaped=0.05)
    wave = ce.pack(ce.generate(w.spec, 60_000), world)
    results, _ = engine.run(wave, world)
    rng = np.random.default_rng(3)
    n = len(wave)
    heads = np.zeros(n, ce.DUMP_HEAD_DTYPE)
    heads["parent"] = rng.integers(0, 2 ** 63, n, dtype=np.uint64)
    heads["slot"] = np.arange(n, dtype=np.uint32)
    heads["op"] = rng.integers(0, 0x1000, n)
    heads["flags"] = rng.integers(0, 256, n) & 0xEF
    heads["kind"] = rng.integers(0, 16, n)
    heads["nodes"] = wave.heads[:, 0] & 255
    heads["muscles"] = wave.heads[:, 1]
    archive = (results["fitness"] - 0.01).astype(np.float32)
    dev = torch.device("cuda", 0)
    d_res = torch.from_numpy(results.view(np.float32).reshape(-1).copy()).to(dev)
    d_heads = torch.from_numpy(wave.heads.view(np.int32).reshape(-1)).to(dev)
    d_dump = torch.from_numpy(heads.view(np.uint8).copy()).to(dev)
    d_arch = torch.from_numpy(archive).to(dev)
    d_rows = torch.zeros(n * 64, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for af, d_af in ((None, 0), (archive, d_arch.data_ptr())):
        ce.dump_rows_device(d_res.data_ptr(), d_heads.data_ptr(), d_dump.data_ptr(), d_af, n, world,
                            d_rows.data_ptr(), stream)
        torch.cuda.synchronize(dev)
        rows = d_rows.cpu().numpy().reshape(n, 64)
        host = ce.dump_rows(results, wave, heads, world, af)
        assert (rows == host).all()
    assert (results["screened"] > 0).any()

"""The device metrics epilogue (ce_metrics_device) against the host's
to_metrics and niche cells (src/scheduler.rs:890-923, src/qd.rs:762-999):
every metrics row and every cell equal to the bit."""
import numpy as np
import pytest

import evolution_simulator_gpu_b200 as ce
from evolution_simulator_gpu_b200.configs import WORKLOADS, effects_world_kw

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload,screen", [("game", False), ("effects", True)])
def test_device_metrics_equal_host_metrics(engine, workload, screen):
    torch = pytest.importorskip("torch")
    w = WORKLOADS[workload]
    kw = dict(duration=6.0)
    if screen:
        kw.update(has_screen=1, screen_seconds=5.0, screen_bar=0.05, screen_bar_young=0.05,
                  screen_bar_reshaped=0.05)
    world = w.world(**kw)
    pop = ce.generate(w.spec, 100_000)
    wave = ce.pack(pop, world)
    results, _ = engine.run(wave, world)
    nodes = (wave.heads[:, 0] & 255).astype(np.uint32)
    host_m = ce.to_metrics(results, nodes, world)
    host_cells = {}
    for layout in (True, False):
        host_cells[layout] = ce.niche_cells(pop, host_m, indices=wave.slots, global_layout=layout)
    dev = torch.device("cuda", 0)
    d_res = torch.from_numpy(results.view(np.float32).reshape(-1).copy()).to(dev)
    d_heads = torch.from_numpy(wave.heads.view(np.int32).reshape(-1)).to(dev)
    for layout in (True, False):
        shapes = ce.shape_classes(pop, wave, global_layout=layout)
        d_shape = torch.from_numpy(shapes).to(dev)
        d_m = torch.zeros(len(wave) * ce.METRICS_DTYPE.itemsize // 4, dtype=torch.int32, device=dev)
        d_cells = torch.zeros(len(wave), dtype=torch.int64, device=dev)
        ce.metrics_device(d_res.data_ptr(), d_heads.data_ptr(), d_shape.data_ptr(), len(wave), world,
                          d_m.data_ptr(), d_cells.data_ptr(), torch.cuda.current_stream(dev).cuda_stream,
                          global_layout=layout)
        torch.cuda.synchronize(dev)
        dm = d_m.cpu().numpy().view(ce.METRICS_DTYPE)
        cells = d_cells.cpu().numpy()
        assert (dm.view(np.uint32) == host_m.view(np.uint32)).all()
        assert (cells == host_cells[layout]).all()
        assert (cells >= 0).all()
    if screen:
        assert (host_m["screened"] > 0).any()

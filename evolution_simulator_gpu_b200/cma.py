"""CMA-ES emitters on the GPU: a batch of the reference's CmaEmitter
(src/qd.rs:2130-2474), one emitter per template body, in either mode: a
separable CMA-ES optimizer (CmaEmitter::optimizer, physical units) or a
CMA-ME emitter (CmaEmitter::new, normalised coordinates and a rank-one step
along the evolution path). The emitters' state is resident in device memory
and ask and tell run as kernels (ce_cma_init / ce_cma_ask / ce_cma_tell).

    opt = CmaEmitters(templates)                # optimizers: sigma 0.5
    pop = opt.ask(count, seed=7, generation=3)  # sample g: emitter g mod E
    fit = evaluate(pop)                         # any evaluator
    opt.tell(pop, fit)                          # one update an emitter

Sample g draws from the reference's breeding stream Rng::stream(seed,
generation, round, slot g) (src/evolution.rs:455-600, restated on the
device), so its coordinates are the reference's sample_into's for that ring
slot given the same emitter state, whichever range of samples a call asks
for.
"""
from __future__ import annotations

import contextlib
import ctypes as C
from typing import Optional

import numpy as np

from . import api

# Config defaults the ask reads (src/config.rs:126, 145-148): the mutation
# strength and repair's diameter and friction ranges.
MUTATION = 1.0
SIZE = (0.06, 0.12)
FRICTION = (0.65, 1.0)


def dims(genomes: np.ndarray, exploring=None) -> np.ndarray:
    """The coordinates of each body: write_parameters' 4 a node, 5 a bone,
    1 period and 8 a muscle (src/qd.rs:2734-2770), or for a CMA-ME emitter
    exploring_parameters' 4 a node, 1 a bone and 8 a muscle
    (src/qd.rs:2504-2538)."""
    g = genomes
    n, b, m = (g[f].astype(np.int64) for f in ("node_count", "bone_count", "muscle_count"))
    opt = 4 * n + 5 * b + 1 + 8 * m
    if exploring is None:
        return opt
    return np.where(np.asarray(exploring, bool), 4 * n + b + 8 * m, opt)


class Genes(tuple):
    """The device byte tensors of one ask: (nodes, bones, muscles, strength
    or None, genomes); `rows` holds its node, bone and muscle rows and its
    sample count."""
    rows: tuple


class CmaEmitters:
    """One CMA-ES emitter per template body, on GPU `device`. `exploring`
    (one flag an emitter, or None) makes an emitter a CMA-ME emitter."""

    def __init__(self, templates: api.Population, exploring=None, device=None, stream=None):
        import torch
        from .refine import take
        self._torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.templates = take(templates, np.arange(len(templates)))  # genes packed in order from row 0
        E = len(self.templates)
        if E == 0:
            raise ValueError("CmaEmitters: no templates")
        self.exploring = None if exploring is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(exploring, bool), (E,)), np.uint8)
        L = api.lib()
        offsets = np.zeros(E + 1, np.uint64)
        api._check(L.ce_cma_offsets(api._ptr(self.templates.genomes), api._ptr(self.exploring), E,
                                    api._ptr(offsets)), "ce_cma_offsets")
        self.offsets = offsets.astype(np.int64)
        D = int(offsets[-1])

        def up(arr):
            return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(self.device)

        t = self.templates
        self._t = [up(t.nodes), up(t.bones), up(t.muscles), up(t.genomes)]
        self._ts = None if t.strength is None else up(t.strength)
        self._off = up(offsets)
        self._mode = None if self.exploring is None else up(self.exploring)
        f = dict(dtype=torch.float32, device=self.device)
        self.mean, self.covariance = torch.empty(D, **f), torch.empty(D, **f)
        self.path_c, self.path_sigma = torch.empty(D, **f), torch.empty(D, **f)
        self.sigma = torch.empty(E, **f)
        self._stream = torch.cuda.current_stream(self.device) if stream is None else stream
        self._c = api.CmaC(self._population_c(), None if self._mode is None else self._mode.data_ptr(),
                           self._off.data_ptr(), self.mean.data_ptr(), self.covariance.data_ptr(),
                           self.path_c.data_ptr(), self.path_sigma.data_ptr(), self.sigma.data_ptr())
        self.asked = 0  # samples drawn so far: the next ask starts there
        self._events = []
        api._check(L.ce_cma_init(C.byref(self._c), self._stream.cuda_stream), "ce_cma_init")

    def __len__(self) -> int:
        return len(self.templates)

    def _population_c(self) -> api.PopulationC:
        n, b, m, g = self._t
        return api.PopulationC(n.data_ptr(), b.data_ptr(), m.data_ptr(), g.data_ptr(), len(self.templates),
                               None if self._ts is None else self._ts.data_ptr())

    @staticmethod
    def draw(seed: int = 0, generation: int = 0, round: int = 0, first_id: int = 1, strength: float = MUTATION,
             size=SIZE, friction=FRICTION) -> api.CmaDraw:
        """What ce_cma_ask draws with: the breeding stream's coordinates,
        the ids, the mutation strength and repair's ranges."""
        return api.CmaDraw(seed, generation, 0, round, first_id, strength, size[0], size[1], friction[0],
                           friction[1])

    def ask_device(self, count: int, seed: int = 0, generation: int = 0, round: int = 0, first_id: int = 1,
                   first: Optional[int] = None, values: bool = False, strength: float = MUTATION, size=SIZE,
                   friction=FRICTION):
        """Samples [first, first + count) (first: where the last ask ended)
        as device byte tensors (nodes, bones, muscles, strength or None,
        genomes) plus the drawn coordinates ([count, max dims] float32, or
        None)."""
        torch = self._torch
        first = self.asked if first is None else int(first)
        draw = self.draw(seed, generation, round, first_id, strength, size, friction)
        L = api.lib()
        rn, rb, rm = C.c_size_t(), C.c_size_t(), C.c_size_t()
        api._check(L.ce_sample_rows(api._ptr(self.templates.genomes), len(self), first, count, C.byref(rn),
                                    C.byref(rb), C.byref(rm)), "ce_sample_rows")

        def out(rows, dtype):
            return torch.empty(max(rows * dtype.itemsize, 1), dtype=torch.uint8, device=self.device)

        on, ob, om = out(rn.value, api.NODE_DTYPE), out(rb.value, api.BONE_DTYPE), out(rm.value, api.MUSCLE_DTYPE)
        og = out(count, api.GENOME_DTYPE)
        ost = None if self._ts is None else out(rm.value, np.dtype(np.float32))
        stride = int(dims(self.templates.genomes, self.exploring).max())
        # Zeros past an emitter's own coordinates (the kernel writes its dims only).
        vals = torch.zeros((max(count, 1), stride), dtype=torch.float32, device=self.device) if values else None
        with self._timed():
            api._check(L.ce_cma_ask(C.byref(self._c), C.byref(draw), first, count, on.data_ptr(), ob.data_ptr(),
                                    om.data_ptr(), None if ost is None else ost.data_ptr(), og.data_ptr(),
                                    None if vals is None else vals.data_ptr(), stride, self._stream.cuda_stream),
                       "ce_cma_ask")
        self.asked = first + count
        genes = Genes((on, ob, om, ost, og))
        genes.rows = (rn.value, rb.value, rm.value, count)
        return genes, (None if vals is None else vals[:count])

    def download(self, genes) -> api.Population:
        """The genes of an ask_device (its Genes) as a host population."""
        on, ob, om, ost, og = genes
        self._stream.synchronize()
        rn, rb, rm, count = genes.rows

        def back(t, rows, dtype):
            return t.cpu().numpy()[:rows * dtype.itemsize].view(dtype).copy()

        return api.Population(back(on, rn, api.NODE_DTYPE), back(ob, rb, api.BONE_DTYPE),
                              back(om, rm, api.MUSCLE_DTYPE), back(og, count, api.GENOME_DTYPE),
                              None if ost is None else back(ost, rm, np.dtype(np.float32)))

    def ask(self, count: int, seed: int = 0, generation: int = 0, round: int = 0, first_id: int = 1,
            first: Optional[int] = None, **kw) -> api.Population:
        """ask_device, copied back to a host population."""
        genes, _ = self.ask_device(count, seed, generation, round, first_id, first, **kw)
        return self.download(genes)

    @contextlib.contextmanager
    def _timed(self):
        """CUDA events around the kernels a call launches (kernel_seconds)."""
        a, b = self._torch.cuda.Event(enable_timing=True), self._torch.cuda.Event(enable_timing=True)
        a.record(self._stream)
        yield
        b.record(self._stream)
        self._events.append((a, b))

    def kernel_seconds(self) -> float:
        """Device time of the ask and tell kernels since the last call."""
        self._stream.synchronize()
        s = sum(a.elapsed_time(b) for a, b in self._events) * 1e-3
        self._events = []
        return s

    def tell(self, samples: api.Population, keys, first: Optional[int] = None) -> None:
        """Updates every emitter from the samples [first, first + len) of an
        ask (first: where that ask began, by default the last ask's range)
        and their keys (fitness for an optimizer, the archive's improvement
        key for a CMA-ME emitter), one a sample, in the samples' order."""
        torch = self._torch
        count = len(samples)
        first = self.asked - count if first is None else int(first)

        def up(arr):
            return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(self.device)

        dn, db, dm, dg = up(samples.nodes), up(samples.bones), up(samples.muscles), up(samples.genomes)
        fit = torch.as_tensor(np.ascontiguousarray(keys, np.float32)).to(self.device)
        self.tell_device((dn, db, dm, dg), fit, first, count)
        self._stream.synchronize()

    def tell_device(self, genes, keys, first: int, count: int) -> None:
        """tell on device tensors: genes = (nodes, bones, muscles, genomes)
        byte tensors of the samples, keys float32 [count]."""
        dn, db, dm, dg = genes
        pc = api.PopulationC(dn.data_ptr(), db.data_ptr(), dm.data_ptr(), dg.data_ptr(), count, None)
        with self._timed():
            api._check(api.lib().ce_cma_tell(C.byref(self._c), C.byref(pc), keys.data_ptr(), first, count,
                                             self._stream.cuda_stream), "ce_cma_tell")

    def recenter(self, which, bodies: api.Population) -> np.ndarray:
        """CmaEmitter::recentered (src/qd.rs:2166-2177): emitter which[i]
        restarts from body i of `bodies` (its template replaced, the mean at
        the body's coordinates), keeping its covariance, paths and step size
        when the body's plan is the template's. Bodies whose counts differ
        from the template's are rejected (True in the returned mask) and
        leave their emitter as it was."""
        from .refine import take
        torch = self._torch
        which = np.ascontiguousarray(which, np.uint32)
        if len(np.unique(which)) != len(which):
            raise ValueError("recenter: the emitters must be distinct")
        if len(which) != len(bodies) or (len(which) and int(which.max()) >= len(self)):
            raise ValueError("recenter: one body an emitter, emitters of this batch")
        b = take(bodies, np.arange(len(bodies)))

        def up(arr):
            return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).reshape(-1).copy()).to(self.device)

        dn, db, dm, dg, dw = up(b.nodes), up(b.bones), up(b.muscles), up(b.genomes), up(which)
        ds = None if b.strength is None else up(b.strength)
        rej = torch.zeros(max(len(which), 1), dtype=torch.int32, device=self.device)
        pc = api.PopulationC(dn.data_ptr(), db.data_ptr(), dm.data_ptr(), dg.data_ptr(), len(b),
                             None if ds is None else ds.data_ptr())
        api._check(api.lib().ce_cma_recenter(C.byref(self._c), C.byref(pc), dw.data_ptr(), len(which),
                                             rej.data_ptr(), self._stream.cuda_stream), "ce_cma_recenter")
        rejected = rej.cpu().numpy()[:len(which)].astype(bool)
        # The host copy of the templates follows the device's.
        t = self.templates
        for i, e in enumerate(which):
            if rejected[i]:
                continue
            g, h = t.genomes[e], b.genomes[i]
            for arr, src, f in ((t.nodes, b.nodes, "node"), (t.bones, b.bones, "bone"), (t.muscles, b.muscles, "muscle")):
                a0, n = int(g[f + "_start"]), int(g[f + "_count"])
                arr[a0:a0 + n] = src[int(h[f + "_start"]):int(h[f + "_start"]) + n]
            if t.strength is not None and b.strength is not None:
                a0, n = int(g["muscle_start"]), int(g["muscle_count"])
                t.strength[a0:a0 + n] = b.strength[int(h["muscle_start"]):int(h["muscle_start"]) + n]
        return rejected

    def converged(self) -> np.ndarray:
        """CmaEmitter::converged (src/qd.rs:2184-2187): optimizers whose step
        size has fallen below 0.05."""
        self._stream.synchronize()
        sig = self.sigma.cpu().numpy()
        opt = np.ones(len(self), bool) if self.exploring is None else ~self.exploring.astype(bool)
        return opt & (sig < 0.05)

    def save(self, path) -> None:
        """The emitters as one .npz file: templates, modes, every emitter's
        mean, covariance, paths and step size, and where the next ask
        starts (the reference keeps its emitters in its search-state saves,
        tests/search_state.rs:769)."""
        self._stream.synchronize()
        t = self.templates
        extra = {} if t.strength is None else {"strength": t.strength}
        if self.exploring is not None:
            extra["exploring"] = self.exploring
        np.savez(path, nodes=t.nodes, bones=t.bones, muscles=t.muscles, genomes=t.genomes,
                 mean=self.mean.cpu().numpy(), covariance=self.covariance.cpu().numpy(),
                 path_c=self.path_c.cpu().numpy(), path_sigma=self.path_sigma.cpu().numpy(),
                 sigma=self.sigma.cpu().numpy(), asked=np.uint64(self.asked), **extra)

    @classmethod
    def load(cls, path, device=None, stream=None) -> "CmaEmitters":
        """Emitters as `save` left them, on GPU `device`."""
        d = np.load(path)
        t = api.Population(d["nodes"], d["bones"], d["muscles"], d["genomes"],
                           d["strength"] if "strength" in d else None)
        out = cls(t, exploring=d["exploring"] if "exploring" in d else None, device=device, stream=stream)
        torch = out._torch
        for name in ("mean", "covariance", "path_c", "path_sigma", "sigma"):
            getattr(out, name).copy_(torch.from_numpy(d[name]).to(out.device))
        out.asked = int(d["asked"])
        return out

    def state(self, e: int):
        """Emitter e's (mean, covariance, path_c, path_sigma, sigma) on the
        host."""
        self._stream.synchronize()
        a, b = int(self.offsets[e]), int(self.offsets[e + 1])
        return (self.mean[a:b].cpu().numpy(), self.covariance[a:b].cpu().numpy(), self.path_c[a:b].cpu().numpy(),
                self.path_sigma[a:b].cpu().numpy(), np.float32(self.sigma[e].item()))

    def set_state(self, e: int, mean, covariance, path_c, path_sigma, sigma) -> None:
        """Overwrites emitter e's state (host arrays)."""
        torch = self._torch
        a, b = int(self.offsets[e]), int(self.offsets[e + 1])
        for dst, src in ((self.mean, mean), (self.covariance, covariance), (self.path_c, path_c),
                         (self.path_sigma, path_sigma)):
            dst[a:b] = torch.as_tensor(np.asarray(src, np.float32)).to(self.device)
        self.sigma[e] = float(sigma)

"""Test infrastructure: a numpy float32 restatement of the reference's
CMA-ES emitters (CmaEmitter, src/qd.rs:2130-2474) in both modes, the checker
of the device's ce_cma_init / ce_cma_ask / ce_cma_tell. Only tests/ use it.

* ``finalize`` / ``keyed`` / ``stream_key`` / ``twelve_uniforms`` /
  ``gene_gaussian``: the reference's counter-based generator
  (src/evolution.rs:455-600), in integers.
* ``layout_of`` / ``scale`` / ``wraps`` / ``delta`` / ``moved``: Layout
  (src/qd.rs:2607-2699); ``phase_dimension``: is_phase_dimension
  (src/qd.rs:2480-2482).
* ``parameters``: write_parameters (src/qd.rs:2734-2770);
  ``explore_parameters``: exploring_parameters (src/qd.rs:2504-2538).
* ``apply`` / ``apply_explore``: apply_parameters (src/qd.rs:2773-2811) and
  apply_exploring_parameters (src/qd.rs:2579-2606), each followed by
  repair's clamps of single genes (src/evolution.rs:1230-1234, 1278-1330).
* ``sample``: sample_optimizing / sample_exploring (src/qd.rs:2244-2289,
  2381-2402) for the child of ring slot g.
* ``tell``: tell with tell_optimizing or tell_exploring (src/qd.rs:
  2213-2243, 2290-2376, 2405-2474), with ties in key broken by sample index.
* ``recentered``: CmaEmitter::recentered (src/qd.rs:2166-2177), for either
  mode.

Every operation is float32, in the reference's order; ln and exp are numpy's.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32
NODE_SCALES = np.array([0.02, 0.02, 0.005, 0.03], np.float32)
BONE_SCALES = np.array([0.02, 0.1, 0.1, 0.02, 0.05], np.float32)
MUSCLE_SCALES = np.array([0.05, 0.05, 0.02, 0.02, 0.05, 0.05, 0.1, 0.05], np.float32)
PERIOD_SCALE = f32(0.05)
MAX_BONE, MAX_STROKE, MIN_PERIOD = f32(2.0), f32(2.0), f32(0.2)
JOINT_LIMIT = f32(np.float32(120.0 * np.pi / 180.0))
FAILED = f32(-1.0e20)
PATH_WEIGHT = f32(0.3)
SIZE, FRICTION = (0.06, 0.12), (0.65, 1.0)  # repair's ranges at the default Config
M64 = (1 << 64) - 1
CURSOR = 0xffffffff


def finalize(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & M64
    z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & M64
    return z ^ (z >> 31)


def keyed(key: int, gene: int, draw: int) -> int:
    return finalize((key + ((gene << 32 | draw) * 0x9e3779b97f4a7c15)) & M64)


def stream_key(seed: int, generation: int, round_: int, slot: int) -> int:
    key = finalize((seed + 0x632be59bd9b4e019) & M64)
    for word in (generation, round_, slot):
        key = finalize(key ^ ((word * 0xd1342543de82ef95) & M64))
    return key


def twelve_uniforms(words) -> np.float32:
    total = sum((w & 0xffff) + (w >> 16 & 0xffff) + (w >> 32 & 0xffff) + (w >> 48) for w in words)
    return f32(f32(total - 6 * 65535) * f32(f32(1.0) / f32(65535.0)))


def gene_gaussian(genes: int, d: int) -> np.float32:
    return twelve_uniforms([keyed(genes, d, k) for k in range(3)])


def rem_euclid1(x):
    r = np.fmod(f32(x), f32(1.0))
    return f32(r + f32(1.0)) if r < 0 else f32(r)


def layout_of(bones):
    """Layout::of's typical bone length of a body from its bone genes."""
    if len(bones) == 0:
        return f32(1.0)
    s = f32(0.0)
    for b in bones["rest_length"]:
        s = f32(s + b)
    return f32(min(max(f32(s / f32(len(bones))), f32(0.05)), f32(10.0)))


def scale(n, b, size, d):
    ne, be = 4 * n, 4 * n + 5 * b
    if d < ne:
        return f32(NODE_SCALES[d % 4] * (size if d % 4 < 2 else f32(1.0)))
    if d < be:
        f = (d - ne) % 5
        return f32(BONE_SCALES[f] * (size if f == 0 else f32(1.0)))
    if d == be:
        return PERIOD_SCALE
    f = (d - be - 1) % 8
    return f32(MUSCLE_SCALES[f] * (size if f in (2, 3) else f32(1.0)))


def wraps(n, b, d):
    be = 4 * n + 5 * b
    return d > be and (d - be - 1) % 8 in (4, 7)


def phase_dimension(d, phase_start):
    return d >= phase_start and (d - phase_start) % 8 == 5


def wrap_phase(x):
    return f32(rem_euclid1(f32(x + f32(0.5))) - f32(0.5))


def delta(n, b, d, value, mean):
    if wraps(n, b, d):
        return f32(rem_euclid1(f32(f32(value - mean) + f32(0.5))) - f32(0.5))
    return f32(value - mean)


def moved(n, b, d, mean, step):
    return rem_euclid1(f32(mean + step)) if wraps(n, b, d) else f32(mean + step)


def parameters(nodes, bones, muscles):
    out = []
    for x in nodes:
        out += [x["x"], x["y"], x["diameter"], x["friction"]]
    for x in bones:
        out += [x["rest_length"], x["min_angle"], x["max_angle"], x["organ_mass"], x["organ_at"]]
    out.append(np.log(f32(max(f32(muscles[0]["period"]) if len(muscles) else f32(1.0), f32(1e-3)))))
    for x in muscles:
        out += [x["anchor_a"], x["anchor_b"], x["short"], x["long"], x["phase"], x["duty"],
                np.log(f32(max(f32(x["stiffness"]), f32(1e-3)))), x["reset"]]
    return np.array(out, np.float32)


def explore_parameters(nodes, bones, muscles):
    out = []
    for x in nodes:
        out += [f32(f32(x["x"] + f32(4.0)) / f32(8.0)), max(f32(x["y"] / f32(4.0)), f32(0.0)),
                clamp(f32(f32(x["diameter"] - f32(0.01)) / f32(0.99)), 0.0, 1.0), clamp(x["friction"], 0.0, 1.0)]
    for x in bones:
        out.append(clamp(f32(f32(x["rest_length"] - f32(0.03)) / f32(MAX_BONE - f32(0.03))), 0.0, 1.0))
    for x in muscles:
        out += [clamp(x["anchor_a"], 0.0, 1.0), clamp(x["anchor_b"], 0.0, 1.0),
                max(f32(f32(x["short"] - f32(0.01)) / f32(0.79)), f32(0.0)),
                max(f32(f32(x["long"] - f32(0.01)) / f32(0.99)), f32(0.0)),
                clamp(f32(f32(x["period"] - MIN_PERIOD) / f32(f32(10.0) - MIN_PERIOD)), 0.0, 1.0),
                clamp(x["phase"], 0.0, 1.0), clamp(f32(f32(x["duty"] - f32(0.05)) / f32(0.90)), 0.0, 1.0),
                clamp(f32(f32(x["stiffness"] - f32(1.0)) / f32(119.0)), 0.0, 1.0)]
    return np.array(out, np.float32)


def clamp(x, lo, hi):
    return f32(min(max(f32(x), f32(lo)), f32(hi)))


def apply(nodes, bones, muscles, values, size=SIZE, friction=FRICTION):
    """The genes of a template body moved to coordinates `values` (copies)."""
    nodes, bones, muscles = nodes.copy(), bones.copy(), muscles.copy()
    v = np.asarray(values, np.float32)
    i = 0
    for x in nodes:
        x["x"] = v[i]
        x["y"] = max(v[i + 1], f32(0.0))
        x["diameter"] = clamp(v[i + 2], *size)
        x["friction"] = clamp(v[i + 3], *friction)
        i += 4
    for x in bones:
        x["rest_length"] = clamp(v[i], 0.03, MAX_BONE)
        x["min_angle"] = clamp(v[i + 1], -JOINT_LIMIT, 0.0)
        x["max_angle"] = clamp(v[i + 2], 0.0, JOINT_LIMIT)
        x["organ_mass"] = max(v[i + 3], f32(0.0))
        x["organ_at"] = clamp(v[i + 4], 0.0, 1.0)
        i += 5
    base = max(f32(muscles[0]["period"]) if len(muscles) else f32(1.0), f32(1e-3))
    pscale = f32(clamp(np.exp(v[i]), MIN_PERIOD, 10.0) / base)
    i += 1
    for x in muscles:
        x["anchor_a"] = clamp(v[i], 0.0, 1.0)
        x["anchor_b"] = clamp(v[i + 1], 0.0, 1.0)
        x["short"] = clamp(v[i + 2], 0.01, f32(0.8) * MAX_STROKE)
        x["long"] = clamp(v[i + 3], x["short"], MAX_STROKE)
        x["period"] = clamp(f32(x["period"] * pscale), MIN_PERIOD, 10.0)
        x["phase"] = rem_euclid1(v[i + 4])
        x["duty"] = clamp(v[i + 5], 0.05, 0.95)
        x["stiffness"] = clamp(np.exp(v[i + 6]), 1.0, 120.0)
        x["reset"] = rem_euclid1(v[i + 7])
        i += 8
    return nodes, bones, muscles


def apply_explore(nodes, bones, muscles, values, size=SIZE, friction=FRICTION):
    """apply_exploring_parameters and repair's clamps (copies)."""
    nodes, bones, muscles = nodes.copy(), bones.copy(), muscles.copy()
    v = np.asarray(values, np.float32)
    i = 0
    for x in nodes:
        x["x"] = f32(f32(v[i] * f32(8.0)) - f32(4.0))
        x["y"] = f32(v[i + 1] * f32(4.0))
        x["diameter"] = clamp(f32(f32(0.01) + f32(v[i + 2] * f32(0.99))), *size)
        x["friction"] = clamp(v[i + 3], *friction)
        i += 4
    for x in bones:
        x["rest_length"] = f32(f32(0.03) + f32(v[i] * f32(MAX_BONE - f32(0.03))))
        i += 1
    for x in muscles:
        x["anchor_a"] = clamp(v[i], 0.0, 1.0)
        x["anchor_b"] = clamp(v[i + 1], 0.0, 1.0)
        short = f32(f32(0.01) + f32(v[i + 2] * f32(0.79)))
        long_ = max(f32(f32(0.01) + f32(v[i + 3] * f32(0.99))), short)
        x["short"] = clamp(short, 0.01, f32(0.8) * MAX_STROKE)
        x["long"] = clamp(long_, x["short"], MAX_STROKE)
        x["period"] = clamp(f32(MIN_PERIOD + f32(v[i + 4] * f32(f32(10.0) - MIN_PERIOD))), MIN_PERIOD, 10.0)
        ph = v[i + 5]
        x["phase"] = rem_euclid1(f32(ph - np.trunc(ph)))
        x["duty"] = clamp(f32(f32(0.05) + f32(v[i + 6] * f32(0.90))), 0.05, 0.95)
        x["stiffness"] = clamp(f32(f32(1.0) + f32(v[i + 7] * f32(119.0))), 1.0, 120.0)
        i += 8
    return nodes, bones, muscles


def sample(state, template, exploring, g, seed=0, generation=0, round_=0, strength=1.0):
    """The coordinates of the child of ring slot g drawn from an emitter in
    `state` (mean, covariance, path_c, path_sigma, sigma)."""
    mean, cov, pc, _, sigma = state
    n, b, m = map(len, template)
    D = len(mean)
    key = stream_key(seed, generation, round_, g)
    strength = f32(strength)
    out = np.zeros(D, np.float32)
    if not exploring:
        genes = keyed(key, CURSOR, 0)
        size = layout_of(template[1])
        for d in range(D):
            out[d] = f32(mean[d] + f32(f32(f32(f32(sigma * strength) * scale(n, b, size, d)) *
                                           f32(np.sqrt(cov[d]))) * gene_gaussian(genes, d)))
        return out
    norm = f32(0.0)
    for x in pc:
        norm = f32(norm + f32(x * x))
    norm = f32(np.sqrt(norm))
    cursor, path_scale = 0, f32(0.0)
    if norm > f32(1e-6):
        z = twelve_uniforms([keyed(key, CURSOR, k) for k in range(3)])
        path_scale = f32(f32(f32(f32(np.sqrt(PATH_WEIGHT)) * z) / norm) * f32(np.sqrt(f32(D))))
        cursor = 3
    genes = keyed(key, CURSOR, cursor)
    phase_start, node_end = 4 * n + b, 4 * n
    for d in range(D):
        step = f32(f32(f32(np.sqrt(cov[d])) * gene_gaussian(genes, d)) + f32(pc[d] * path_scale))
        value = f32(mean[d] + f32(f32(sigma * step) * strength))
        field = (d - phase_start) % 8 if d >= phase_start else None
        if phase_dimension(d, phase_start):
            out[d] = rem_euclid1(value)
        elif d < node_end and d % 4 == 0:
            out[d] = value
        elif (d < node_end and d % 4 == 1) or field in (2, 3):
            out[d] = max(value, f32(0.0))
        else:
            out[d] = clamp(value, 0.0, 1.0)
    return out


def same_plan(template, sample):
    """tell's body-plan filter (src/qd.rs:2217-2228): the sample's counts and
    its bone and muscle connections are the template's, gene by gene."""
    (tn, tb, tm), (sn, sb, sm) = template, sample
    if (len(tn), len(tb), len(tm)) != (len(sn), len(sb), len(sm)):
        return False
    pair = lambda a, b: (min(int(a), int(b)), max(int(a), int(b)))
    return (all(pair(x["a"], x["b"]) == pair(y["a"], y["b"]) for x, y in zip(tb, sb)) and
            all(pair(x["bone_a"], x["bone_b"]) == pair(y["bone_a"], y["bone_b"]) for x, y in zip(tm, sm)))


def _weights(mu):
    w = [f32(np.log(f32(f32(mu) + f32(0.5))) - np.log(f32(i + 1))) for i in range(mu)]
    wsum = f32(0.0)
    for x in w:
        wsum = f32(wsum + x)
    wsum = max(wsum, f32(np.finfo(np.float32).tiny))
    sq = f32(0.0)
    for i in range(mu):
        w[i] = f32(w[i] / wsum)
        sq = f32(sq + f32(w[i] * w[i]))
    return w, f32(f32(1.0) / max(sq, f32(1e-6)))


def _ranked(template, samples, keys):
    """tell's filter, truncation and sort: (key, sample index) best first."""
    pairs = [(f32(f), i) for i, f in enumerate(keys)
             if np.isfinite(f) and f32(f) > FAILED and same_plan(template, samples[i])]
    pairs.sort(key=lambda q: (-q[0], q[1]))
    return pairs[:1024]


def tell_explore(state, template, samples, keys):
    """tell + tell_exploring on one CMA-ME emitter (see ``tell``)."""
    mean, cov, pc, ps, sigma = (np.array(state[0], np.float32), np.array(state[1], np.float32),
                                np.array(state[2], np.float32), np.array(state[3], np.float32), f32(state[4]))
    pairs = _ranked(template, samples, keys)
    if len(pairs) < 2:
        return mean, cov, pc, ps, sigma
    mu = (len(pairs) + 1) // 2
    w, mu_eff = _weights(mu)
    n_, b_, _ = map(len, template)
    phase_start = 4 * n_ + b_
    D = len(mean)
    sig = max(sigma, f32(1e-6))
    vectors = [explore_parameters(*samples[i]) for _, i in pairs[:mu]]
    new_mean = np.zeros(D, np.float32)
    rank_mu = np.zeros(D, np.float32)
    for d in range(D):
        ph = phase_dimension(d, phase_start)
        acc, rm = f32(0.0), f32(0.0)
        for rank in range(mu):
            v = vectors[rank][d]
            acc = f32(acc + f32(w[rank] * (wrap_phase(f32(v - mean[d])) if ph else v)))
            delta = f32((wrap_phase(f32(v - mean[d])) if ph else f32(v - mean[d])) / sig)
            rm = f32(rm + f32(f32(w[rank] * delta) * delta))
        new_mean[d] = rem_euclid1(f32(mean[d] + acc)) if ph else acc
        rank_mu[d] = rm
    n = f32(D)
    c_sigma = f32(f32(mu_eff + f32(2.0)) / f32(f32(n + mu_eff) + f32(5.0)))
    d_sigma = f32(f32(f32(1.0) + f32(f32(2.0) * max(f32(np.sqrt(f32(max(f32(mu_eff - f32(1.0)), f32(0.0)) / f32(n + f32(1.0))))) - f32(1.0), f32(0.0)))) + c_sigma)
    c_c = f32(f32(f32(4.0) + f32(mu_eff / n)) / f32(f32(n + f32(4.0)) + f32(f32(f32(2.0) * mu_eff) / n)))
    a13 = f32(n + f32(1.3))
    c1 = f32(f32(2.0) / f32(f32(a13 * a13) + mu_eff))
    a2 = f32(n + f32(2.0))
    inner = max(f32(f32(mu_eff - f32(2.0)) + f32(f32(1.0) / mu_eff)), f32(0.0))
    c_mu = min(f32(f32(f32(2.0) * inner) / f32(f32(a2 * a2) + mu_eff)), f32(f32(1.0) - c1))
    y = np.zeros(D, np.float32)
    norm = f32(0.0)
    k_sigma = f32(np.sqrt(f32(f32(c_sigma * f32(f32(2.0) - c_sigma)) * mu_eff)))
    for d in range(D):
        md = wrap_phase(f32(new_mean[d] - mean[d])) if phase_dimension(d, phase_start) else f32(new_mean[d] - mean[d])
        y[d] = f32(md / sig)
        normalized = f32(y[d] / max(f32(np.sqrt(cov[d])), f32(1e-6)))
        ps[d] = f32(f32(f32(f32(1.0) - c_sigma) * ps[d]) + f32(k_sigma * normalized))
        norm = f32(norm + f32(ps[d] * ps[d]))
    norm = f32(np.sqrt(norm))
    chi = f32(f32(np.sqrt(n)) * f32(f32(f32(1.0) - f32(f32(1.0) / f32(f32(4.0) * n))) + f32(f32(1.0) / f32(f32(f32(21.0) * n) * n))))
    hsig = f32(norm / max(chi, f32(1e-6))) < f32(f32(1.4) + f32(f32(2.0) / f32(n + f32(1.0))))
    correction = f32(0.0) if hsig else f32(c_c * f32(f32(2.0) - c_c))
    k_c = f32(np.sqrt(f32(f32(c_c * f32(f32(2.0) - c_c)) * mu_eff)))
    a = f32(f32(f32(f32(1.0) - c1) - c_mu) + f32(c1 * correction))
    for d in range(D):
        pc[d] = f32(f32(f32(f32(1.0) - c_c) * pc[d]) + (f32(k_c * y[d]) if hsig else f32(0.0)))
        cov[d] = clamp(f32(f32(f32(a * cov[d]) + f32(f32(c1 * pc[d]) * pc[d])) + f32(c_mu * rank_mu[d])), 0.0025, 4.0)
    sigma = clamp(f32(sigma * np.exp(f32(f32(c_sigma / d_sigma) * f32(f32(norm / max(chi, f32(1e-6))) - f32(1.0))))),
                  0.005, 0.35)
    return new_mean, cov, pc, ps, sigma


def tell(state, template, samples, fitness, exploring=False):
    """tell + tell_optimizing on one emitter (tell_exploring with
    `exploring`). `state` = (mean, covariance, path_c, path_sigma, sigma),
    float32 arrays and a float32; `template` and each of `samples` = (nodes,
    bones, muscles) gene arrays; `fitness` one key a sample. Returns the new
    state (copies)."""
    if exploring:
        return tell_explore(state, template, samples, fitness)
    mean, cov, pc, ps, sigma = (np.array(state[0], np.float32), np.array(state[1], np.float32),
                                np.array(state[2], np.float32), np.array(state[3], np.float32), f32(state[4]))
    tn, tb, tm = template
    nn_, nb_ = len(tn), len(tb)
    size = layout_of(tb)
    pairs = _ranked(template, samples, fitness)
    if len(pairs) < 2:
        return mean, cov, pc, ps, sigma
    L = len(pairs)
    mu = (L + 1) // 2
    w, mu_eff = _weights(mu)
    D = len(mean)
    sig = max(sigma, f32(1e-6))
    vectors = [parameters(*samples[i]) for _, i in pairs[:mu]]
    step = np.zeros(D, np.float32)
    rank_mu = np.zeros(D, np.float32)
    for d in range(D):
        unit = f32(sig * scale(nn_, nb_, size, d))
        st, rm = f32(0.0), f32(0.0)
        for rank in range(mu):
            y = f32(delta(nn_, nb_, d, vectors[rank][d], mean[d]) / unit)
            st = f32(st + f32(w[rank] * y))
            rm = f32(rm + f32(f32(w[rank] * y) * y))
        step[d], rank_mu[d] = st, rm
    n = f32(D)
    c_sigma = f32(f32(mu_eff + f32(2.0)) / f32(f32(n + mu_eff) + f32(5.0)))
    d_sigma = f32(f32(f32(1.0) + f32(f32(2.0) * max(f32(np.sqrt(f32(max(f32(mu_eff - f32(1.0)), f32(0.0)) / f32(n + f32(1.0))))) - f32(1.0), f32(0.0)))) + c_sigma)
    c_c = f32(f32(f32(4.0) + f32(mu_eff / n)) / f32(f32(n + f32(4.0)) + f32(f32(f32(2.0) * mu_eff) / n)))
    separable = f32(f32(n + f32(2.0)) / f32(3.0))
    a13 = f32(n + f32(1.3))
    c1 = min(f32(f32(f32(2.0) / f32(f32(a13 * a13) + mu_eff)) * separable), f32(0.5))
    a2 = f32(n + f32(2.0))
    inner = max(f32(f32(mu_eff - f32(2.0)) + f32(f32(1.0) / mu_eff)), f32(0.0))
    c_mu = min(f32(f32(f32(f32(2.0) * inner) / f32(f32(a2 * a2) + mu_eff)) * separable), f32(f32(1.0) - c1))
    norm = f32(0.0)
    k_sigma = f32(np.sqrt(f32(f32(c_sigma * f32(f32(2.0) - c_sigma)) * mu_eff)))
    for d in range(D):
        ps[d] = f32(f32(f32(f32(1.0) - c_sigma) * ps[d]) + f32(f32(k_sigma * step[d]) / max(f32(np.sqrt(cov[d])), f32(1e-6))))
        norm = f32(norm + f32(ps[d] * ps[d]))
    norm = f32(np.sqrt(norm))
    chi = f32(f32(np.sqrt(n)) * f32(f32(f32(1.0) - f32(f32(1.0) / f32(f32(4.0) * n))) + f32(f32(1.0) / f32(f32(f32(21.0) * n) * n))))
    hsig = f32(norm / max(chi, f32(1e-6))) < f32(f32(1.4) + f32(f32(2.0) / f32(n + f32(1.0))))
    correction = f32(0.0) if hsig else f32(c_c * f32(f32(2.0) - c_c))
    k_c = f32(np.sqrt(f32(f32(c_c * f32(f32(2.0) - c_c)) * mu_eff)))
    a = f32(f32(f32(f32(1.0) - c1) - c_mu) + f32(c1 * correction))
    for d in range(D):
        pc[d] = f32(f32(f32(f32(1.0) - c_c) * pc[d]) + (f32(k_c * step[d]) if hsig else f32(0.0)))
        cov[d] = clamp(f32(f32(f32(a * cov[d]) + f32(f32(c1 * pc[d]) * pc[d])) + f32(c_mu * rank_mu[d])), 1e-4, 1e4)
        mean[d] = moved(nn_, nb_, d, mean[d], f32(f32(sig * scale(nn_, nb_, size, d)) * step[d]))
    sigma = clamp(f32(sigma * np.exp(f32(f32(c_sigma / d_sigma) * f32(f32(norm / max(chi, f32(1e-6))) - f32(1.0))))),
                  0.01, 30.0)
    if pairs[L // 2][0] < f32(f32(0.25) * pairs[0][0]):
        sigma = max(f32(sigma * f32(0.6)), f32(0.01))
    return mean, cov, pc, ps, sigma


def recentered(state, template, body, exploring=False):
    """The state an emitter restarts in from `body`: the mean at the body's
    coordinates; covariance, paths and step size kept when the body's plan
    is the template's, else the mode's constructor's (unit covariance, zero
    paths, 0.5 or 0.12)."""
    mean = explore_parameters(*body) if exploring else parameters(*body)
    if same_plan(template, body) and len(mean) == len(state[0]):
        return mean, np.array(state[1], np.float32), np.array(state[2], np.float32), \
            np.array(state[3], np.float32), f32(state[4])
    D = len(mean)
    return mean, np.ones(D, np.float32), np.zeros(D, np.float32), np.zeros(D, np.float32), \
        f32(0.12 if exploring else 0.5)

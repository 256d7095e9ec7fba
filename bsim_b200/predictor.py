"""Training data and training for the firing predictor (host side).

The predictor's features for population p at cycle t are its rates in cycles
t-1..t-8 and its mean in-degree; the target is its rate in cycle t+1 (rates are
spikes / size * 10, so 1.0 is 1 kHz at dt = 0.1 ms). This matches the inference
the step kernel runs (include/bsim_b200.h, "Firing predictor").
"""
import numpy as np

from . import Engine, mlp_init, mlp_train

LAGS = 8


def features(counts, size, mean_indeg):
    """counts [T, P] spikes per cycle and population -> (x [n, 9], y [n]) for every
    cycle t with 8 earlier cycles and one later cycle available."""
    counts = np.asarray(counts, np.float64)
    T, P = counts.shape
    rate = counts / np.asarray(size, np.float64)[None, :] * 10.0
    xs, ys = [], []
    for t in range(LAGS + 1, T - 1):
        lag = rate[t - 1 - np.arange(LAGS)]          # [8, P], most recent first
        x = np.concatenate([lag.T, (np.asarray(mean_indeg, np.float64) * 1e-3)[:, None]], axis=1)
        xs.append(x)
        ys.append(rate[t + 1])
    return np.concatenate(xs).astype(np.float32), np.concatenate(ys).astype(np.float32)


def collect(specs, steps, dt, settle=200, chunk=1000, opts=None):
    """Runs a plain engine and returns (counts [steps, P], size, mean_indeg)."""
    eng = Engine.generated(specs, dt, opts=opts)
    eng.enable_pop_stats(chunk + 2)
    eng.run(settle)
    out = []
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        eng.run(k)
        out.append(eng.pop_counts(k))
        done += k
    size, indeg, _ = eng.pop_info()
    eng.close()
    return np.concatenate(out), size, indeg


def train(x, y, epochs=30, batch=512, lr=2e-3, seed=1):
    """Trains from a deterministic initialisation on the GPU; returns (params, loss)."""
    return mlp_train(mlp_init(seed), x, y, epochs=epochs, batch=batch, lr=lr, seed=seed)


def fit_costs(events_per_cycle, ns_per_cycle):
    """Least-squares cost model of one delivery mode, ns per cycle = a + b * events
    per cycle, from per-chunk measurements at varied activity (a, b >= 0)."""
    e = np.asarray(events_per_cycle, np.float64)
    t = np.asarray(ns_per_cycle, np.float64)
    A = np.stack([np.ones_like(e), e], 1)
    (a, b), *_ = np.linalg.lstsq(A, t, rcond=None)
    if b < 0:
        a, b = float(t.mean()), 0.0
    if a < 0:
        a, b = 0.0, float((e * t).sum() / max((e * e).sum(), 1e-30))
    return [float(a), float(b)]

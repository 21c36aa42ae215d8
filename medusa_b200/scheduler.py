"""Training the learned superstep scheduler from timing traces.

The traces come from the graph families of the benchmark configurations,
at sizes that trace in seconds, with seeds distinct from the benchmark's:

  * uniform random (the PageRank configuration's family),
  * R-MAT (a,b,c,d) = (0.45,0.15,0.15,0.25) (the BFS/SSSP configuration's),
  * 2-D grid with 10% of the edges dropped and 0.5% shortcuts (road-like).

One model per loop kind: single-source BFS and SSSP (8 schedules each) and
64-source batched BFS (push vs pull).  All are FP32 6-32-32-8 MLPs trained
on the GPU by the library's own kernels.
"""
import numpy as np

from . import api


def trace_families(seed, scale=14):
    v = 1 << scale
    side = int(round((v / 2) ** 0.5))
    return [
        ("uniform", api.uniform_params(v, 16 * v, seed=seed, wmin=1, wmax=1000)),
        ("rmat", api.rmat_params(scale, 16 * v, 0.45, 0.15, 0.15, seed=seed, wmin=1, wmax=1000)),
        ("grid", api.grid_params(side, side, 0.1, 0.005, seed=seed, wmin=1, wmax=100)),
    ]


def collect(ctx, seeds, apps=(0, 1), scales=(14,)):
    """Concatenated traces (X [n,6], T [n,8], fixed choice [n]) over the
    families, sizes (log2 vertices) and seeds, for the given apps (0 BFS,
    1 SSSP, 2 batched BFS)."""
    if isinstance(scales, int):
        scales = (scales,)
    X, T, S = [], [], []
    for scale in scales:
        for seed in seeds:
            for _, p in trace_families(seed, scale):
                g = ctx.generate(p)
                try:
                    for app in apps:
                        x, t, s = ctx.scheduler_collect(g, app, 0)
                        X.append(x)
                        T.append(t)
                        S.append(s)
                finally:
                    g.close()
    return np.concatenate(X), np.concatenate(T), np.concatenate(S)


def train(ctx, seeds=(101, 102), scales=(14,), epochs=1500, lr=3e-3, seed=7, rounds=2):
    """Train both models; returns {model: (final loss, samples)}.

    The first training pass learns from traces along the fixed rule's
    trajectories.  Each further pass (`rounds` in all) collects traces along
    the trained policy's own trajectories (states where it departed from the
    fixed rule), adds them to the set and retrains (dataset aggregation)."""
    out = {}
    sets = {api.MB_MODEL_BFS: ((0,), [], []), api.MB_MODEL_SSSP: ((1,), [], []),
            api.MB_MODEL_BATCHED: ((2,), [], [])}
    saved = ctx.policy
    try:
        for r in range(rounds):
            ctx.set_policy(api.MB_POLICY_LEARNED if r else api.MB_POLICY_FIXED)
            for model, (apps, Xs, Ts) in sets.items():
                X, T, _ = collect(ctx, seeds, apps, scales)
                Xs.append(X)
                Ts.append(T)
            ctx.set_policy(api.MB_POLICY_FIXED)
            for model, (apps, Xs, Ts) in sets.items():
                X, T = np.concatenate(Xs), np.concatenate(Ts)
                out[model] = (ctx.scheduler_train(X, T, epochs, lr, seed, model), len(X))
    finally:
        ctx.set_policy(*saved)
    return out


def evaluate(ctx, X, T, S, model=api.MB_MODEL_BFS):
    """Summed per-superstep times of the fixed rule's choices, the model's
    choices and the per-superstep best schedule on traces (X, T, S), over
    the samples where both the fixed and the learned choice were timed.
    (SSSP replays are not always state-identical: relaxations inside a
    superstep race, so a replay can converge a step earlier and leave a
    schedule unmeasured.)"""
    pick = ctx.scheduler_pick(X, model, fallback=S)
    idx = np.arange(len(T))
    t_fixed = T[idx, S]
    t_learned = T[idx, pick]
    ok = (t_fixed > 0) & (t_learned > 0)
    best = np.where(T > 0, T, np.inf).min(axis=1)
    out = {"fixed_ms": float(t_fixed[ok].sum()), "learned_ms": float(t_learned[ok].sum()),
           "oracle_best_ms": float(best[ok].sum()), "samples": int(ok.sum()),
           "unmeasured": int((~ok).sum())}
    # the reference's single schedule (its edge-centric superstep,
    # MB_SCHED_PUSH_UNFUSED) where it was timed: what the model gains over it
    ref = T[:, api.MB_SCHED_PUSH_UNFUSED]
    ok_r = ok & (ref > 0)
    if ok_r.any():
        out["reference_schedule_ms"] = float(ref[ok_r].sum())
        out["learned_ms_on_those"] = float(t_learned[ok_r].sum())
        out["reference_samples"] = int(ok_r.sum())
    return out

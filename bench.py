#!/usr/bin/env python3
"""Benchmark: Medusa's BSP superstep on B200 -- BFS/SSSP GTEPS (and PageRank edges/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl medusa|reference]

Workload (N=1, the configuration the metric is quoted on): R-MAT with 2^20
vertices and 2^24 directed edges, (a,b,c,d) = (0.45,0.15,0.15,0.25), seeded,
duplicates kept; integer weights in [1,1000] stored as float32.  One step =
one BFS and one SSSP from source 0, each a whole BSP iteration loop.
`value` = (BFS + SSSP traversed edges) / device time of the two loops, in
GTEPS, where traversed edges = sum of out-degrees of reached vertices (the
reference's count).  Inputs are resident in HBM; L2 is flushed (256 MiB
write) before every step.  `e2e` = the same metric through the C ABI with
pinned host buffers: the source ids go host->device and the levels and
distances come back device->host inside the timed region.

`pagerank`: PageRank on the reference's CPU-runnable configuration (uniform,
2^18 vertices, 2^22 edges, 10 supersteps from 1/N), edges/s per superstep.

`configs`: C3 (1448x1448 road-like grid, BFS + SSSP from the corner, fixed
vs learned schedule), C4a (64 BFS + 32 SSSP sources on R-MAT 2^22/2^26,
batched and learned+batched vs one loop per source, identical outputs) and
C5 (R-MAT 2^24/2^28, (0.57,0.19,0.19,0.05):
BFS, SSSP and 20 PageRank supersteps, fixed vs learned schedule with HBM
roofline fractions, plus per-superstep fixed / learned / oracle-best costs)
and C4b (256 R-MAT graphs of uneven sizes, 20 PageRank supersteps + one BFS
each, in one persistent launch vs one library call per graph, identical
outputs).

`forms`: the same graph, 64 BFS sources (vertices 0..63) and 32 SSSP
sources (0..31) under four forms -- plain (fixed schedule rule, one loop per
source), learned (the trained MLP scheduler picks each superstep's
schedule), batched (64-bit / 32-lane source masks, one traversal per batch)
and learned+batched -- each form's GTEPS, its ratio to plain, and a check
that all four return identical levels and distances.  The scheduler is
trained first, on the GPU, from timing traces of the uniform / R-MAT / grid
generator families at 2^14, 2^17 and 2^20 vertices with seeds other than
the workload's.

Multi-GPU (torchrun): the path does not shard (one graph per GPU, as the
reference's single-GPU path); every rank runs the full workload on its own
replica, `value` sums all ranks' traversed edges over the max device time.

`--impl reference`: the reference's own CPU superstep code (oracle/_ref),
on this host's cores, on the same graph and metric; rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 1
C2 = dict(scale=20, num_edges=1 << 24, a=0.45, b=0.15, c=0.15, wmin=1, wmax=1000)
C1 = dict(num_vertices=1 << 18, num_edges=1 << 22)
PR_ITERS = 10
TRAIN_SCALES = (14, 17, 20)  # log2 vertices of the scheduler's trace graphs
TRAIN_ROUNDS = 3  # trace collections: fixed-rule trajectories, then the learned policy's
METRIC = "BFS/SSSP GTEPS (R-MAT 2^20 V / 2^24 E, source 0)"
WORKLOAD = ("R-MAT 2^20 vertices, 2^24 edges, (a,b,c,d)=(0.45,0.15,0.15,0.25), seed 1, "
            "weights int [1,1000] as f32; one step = BFS + SSSP from source 0")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def c2_params(api):
    return api.rmat_params(C2["scale"], C2["num_edges"], C2["a"], C2["b"], C2["c"], seed=SEED,
                           wmin=C2["wmin"], wmax=C2["wmax"])


def c1_params(api):
    return api.uniform_params(C1["num_vertices"], C1["num_edges"], seed=SEED)


def host_edges(kind, **params):
    """A workload's edge list made on the CPU by the oracle's generator (the
    same edges the product's generator makes; the CPU legs load nothing from
    the product library)."""
    from oracle import oracle as O
    return O.generate(kind, **params)


def c2_edges():
    return host_edges("rmat", scale=C2["scale"], num_edges=C2["num_edges"], a=C2["a"], b=C2["b"],
                      c=C2["c"], seed=SEED, wmin=C2["wmin"], wmax=C2["wmax"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                         "sw_power_cap"]
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def flush_l2(buf):
    buf.zero_()


def bfs_bytes(st, V):
    # algorithmic bytes of a BFS: 8 per reached edge, 20 per reached vertex, 4 per vertex
    return 8 * st["edges_traversed"] + 20 * st["vertices_reached"] + 4 * V


def sssp_bytes(st, V):
    return 12 * st["edges_traversed"] + 20 * st["vertices_reached"] + 4 * V


BRANCH_KERNELS = {0: "k_push_edge_q", 1: "k_push_warp_q", 4: "k_pull_stream", 5: "k_pull_warp",
                  6: "reference split", 7: "full pull", 17: "k_tail", 19: "k_push_edge_bm + k_nbm2q",
                  20: "k_push_edge_q (two CTAs per SM)"}
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dominant_kernel_traffic.md")


def measured_traffic_ratio(kernel):
    """DRAM bytes per algorithmic byte of `kernel`, from the committed ncu
    summary (a line "| <kernel> | ... | <ratio> |" in its table), or None."""
    try:
        for line in open(TRAFFIC_FILE):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if len(cells) >= 2 and cells[0] == kernel:
                return float(cells[-1])
    except (OSError, ValueError):
        pass
    return None


def kernel_roofline(ctx, g, V, pk, pk_kind):
    """The dominant kernel of one BFS + one SSSP: every superstep's branch
    timed alone (CUDA events, host-driven loop), algorithmic bytes per
    superstep from its frontier (BFS 8 B per frontier out-edge + 20 B per
    frontier vertex, SSSP 12 + 20), the branch with the largest total time."""
    ctx.set_tracing(True)
    try:
        g.bfs([0])
        g.sssp([0])
        tr = ctx.get_trace()
    finally:
        ctx.set_tracing(False)
    per = {}
    for r in tr:
        per_edge = 8 if r["app"] == 0 else 12
        key = (int(r["app"]), int(r["branch"]))
        ms, b, n = per.get(key, (0.0, 0.0, 0))
        per[key] = (ms + float(r["ms"]),
                    b + per_edge * float(r["frontier_edges"]) + 20.0 * float(r["frontier_vertices"]),
                    n + 1)
    (app, br), (ms, byts, n) = max(per.items(), key=lambda kv: kv[1][0])
    name = BRANCH_KERNELS.get(br % 8 if br < 16 else br, "branch %d" % br)
    achieved = byts / (ms / 1e3) / 1e9
    ratio = measured_traffic_ratio(name)
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk, "unit": "GB/s",
            "frac": round(achieved / pk, 4),
            "traffic": None if ratio is None else round(ratio * byts / n),
            "peak_kind": pk_kind,
            "kernel": "%s (%s, branch %d)" % (name, ("BFS", "SSSP")[app], br),
            "launches": n, "avg_launch_ms": round(ms / n, 4),
            "algorithmic_bytes_per_launch": round(byts / n),
            "share_of_traced_time": round(ms / sum(v[0] for v in per.values()), 3),
            "traffic_source": None if ratio is None else
            "DRAM bytes / algorithmic bytes of this kernel from profiles/dominant_kernel_traffic.md"}


def reset_tunables(ctx, api):
    for k in api.TUNABLES:
        ctx.set_tunable(k, -1)
    ctx.set_sssp_delta(0.0)


def verify_against_bsp(ctx, api, g, lv_out, d_out):
    """The timed runs' outputs (device tensors, source 0) against one run of
    the BSP loop with every tunable at its default and the asynchronous
    kernels off; the tuned settings are restored afterwards.  Returns
    {"bfs_levels": bool, "sssp_distances": bool} (bit for bit)."""
    import torch
    saved = {k: ctx.get_tunable(k) for k in api.TUNABLES}
    saved_delta = ctx.sssp_delta
    try:
        reset_tunables(ctx, api)
        ctx.set_tunable("sssp_async", 0)
        ctx.set_tunable("bfs_async", 0)
        lv = torch.empty_like(lv_out)
        dd = torch.empty_like(d_out)
        g.bfs([0], out=lv)
        g.sssp([0], out=dd)
        return {"bfs_levels": bool(torch.equal(lv, lv_out)),
                "sssp_distances": bool(torch.equal(dd.view(torch.int32), d_out.view(torch.int32)))}
    finally:
        for k, v in saved.items():
            ctx.set_tunable(k, v)
        ctx.set_sssp_delta(saved_delta)


def reduce_over_ranks(dev_ms, edges, dist=None, device="cpu"):
    """Replicas: the job's time is the slowest rank's device time and its
    work the sum of every rank's traversed edges (no data-path collective:
    each rank runs its own copy of the workload)."""
    import torch
    if dist is None:
        return float(dev_ms), float(edges)
    t = torch.tensor([dev_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e = torch.tensor([edges], dtype=torch.float64, device=device)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), float(e.item())


def run_medusa(args):
    import torch
    from medusa_b200 import api
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = api.Context(local)
    if args.hostloop:
        ctx.set_graph_capture(False)
    p = c2_params(api)
    g = ctx.generate(p)
    V = g.V
    tuned = {}
    if not args.no_autotune:
        # launch and routing parameters for this graph (results never change)
        from medusa_b200 import autotune
        tuned.update(autotune.tune_traversals(ctx, g, 0)[0])
    lv_dev = torch.empty(V, dtype=torch.int32, device=dev)
    d_dev = torch.empty(V, dtype=torch.float32, device=dev)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)  # 256 MiB > L2

    def step(out_l, out_d):
        _, sb = g.bfs([0], out=out_l)
        _, ss = g.sssp([0], out=out_d)
        return sb, ss

    for _ in range(args.warmup):
        step(lv_dev, d_dev)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    dev_ms, edges, launches, bts = 0.0, 0, 0, 0
    sb_last = ss_last = None
    wall0 = time.perf_counter()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            sb, ss = step(lv_dev, d_dev)
            dev_ms += sb["device_ms"] + ss["device_ms"]
            edges += sb["edges_traversed"] + ss["edges_traversed"]
            launches += sb["kernel_launches"] + ss["kernel_launches"]
            bts += bfs_bytes(sb, V) + sssp_bytes(ss, V)
            sb_last, ss_last = sb, ss
        torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    t_max, edges_all = reduce_over_ranks(dev_ms, edges, dist, dev)
    value = edges_all / (t_max / 1e3) / 1e9

    # end to end through the C ABI with pinned host buffers
    lv_h = torch.empty(V, dtype=torch.int32, pin_memory=True)
    d_h = torch.empty(V, dtype=torch.float32, pin_memory=True)
    e2e_wall, e2e_edges = 0.0, 0
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sb, ss = step(lv_h, d_h)
        e2e_wall += time.perf_counter() - t0
        e2e_edges += sb["edges_traversed"] + ss["edges_traversed"]
    e2e_val = e2e_edges / e2e_wall / 1e9
    # the timed (tuned) outputs against the plain BSP loop's, bit for bit
    # (after both measurements: switching the settings back and forth
    # re-instantiates the loop graphs)
    verified = verify_against_bsp(ctx, api, g, lv_dev, d_dev)

    pk, pk_kind = peaks()
    bfs_gb = bfs_bytes(sb_last, V) / 1e9
    sssp_gb = sssp_bytes(ss_last, V) / 1e9
    achieved = bts / (dev_ms / 1e3) / 1e9
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "vertices": V, "edges": g.E, "sources": [0],
                   "l2": "flushed (256 MiB write) before every step",
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "schedule_policy": "fixed (direction-optimising rule)",
                   "loop": ("host-driven loop (one flag read per superstep)" if args.hostloop
                            else "one CUDA graph per BSP loop (device-side convergence)"),
                   "autotuned": {k: float(v) for k, v in tuned.items()}},
        "bfs": {"gteps": round(sb_last["edges_traversed"] / sb_last["device_ms"] / 1e6, 3),
                "ms": round(sb_last["device_ms"], 4), "supersteps": sb_last["supersteps"],
                "edges_traversed": sb_last["edges_traversed"],
                "vertices_reached": sb_last["vertices_reached"],
                "schedule_count": sb_last["schedule_count"],
                "edges_scanned": sb_last["edges_scanned"]},
        "sssp": {"gteps": round(ss_last["edges_traversed"] / ss_last["device_ms"] / 1e6, 3),
                 "ms": round(ss_last["device_ms"], 4), "supersteps": ss_last["supersteps"],
                 "edges_traversed": ss_last["edges_traversed"],
                 "schedule_count": ss_last["schedule_count"],
                 "edges_scanned": ss_last["edges_scanned"]},
        "e2e": {"value": round(e2e_val, 3), "unit": "GTEPS", "h2d_bytes_per_step": 8,
                "d2h_bytes_per_step": 8 * V},
        "roofline": kernel_roofline(ctx, g, V, pk, pk_kind),
        "roofline_loops": {"bound": "hbm", "achieved": round(achieved, 1), "peak": pk,
                           "unit": "GB/s", "frac": round(achieved / pk, 4),
                           "peak_kind": pk_kind,
                           "what": "BFS + SSSP superstep loops (one CUDA graph each), whole step",
                           "bytes_per_step": {"bfs": round(bfs_gb, 4), "sssp": round(sssp_gb, 4),
                                              "unit": "GB",
                                              "formula": "BFS 8*E_r+20*V_r+4*V; SSSP 12*E_r+20*V_r+4*V"}},
        "gpu_launches": int(launches),
        "verified_against_bsp": verified,
        "wall_s": round(wall, 3),
        "clocks": clk.summary(),
    }
    if not args.no_forms:
        out["forms"] = bench_forms(ctx, api, args, flush, g)
    if not args.no_pagerank:
        out["pagerank"] = bench_pagerank(ctx, api, args, flush)
    g.close()
    reset_tunables(ctx, api)  # each configuration tunes its own
    if not args.no_configs and not args.no_forms:  # C5's learned arm needs the trained models
        out["configs"] = bench_configs(ctx, api, args, flush)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(api, args)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def bench_forms(ctx, api, args, flush, g):
    """plain / learned / batched / learned+batched on the workload graph."""
    import torch
    from medusa_b200 import scheduler
    t0 = time.perf_counter()
    trained = scheduler.train(ctx, seeds=(101, 102), scales=TRAIN_SCALES, rounds=TRAIN_ROUNDS)
    MODELS = (("bfs", api.MB_MODEL_BFS), ("sssp", api.MB_MODEL_SSSP),
              ("batched_bfs", api.MB_MODEL_BATCHED))
    train_s = time.perf_counter() - t0
    V = g.V
    bsrc, ssrc = list(range(64)), list(range(32))
    lv = torch.empty((64, V), dtype=torch.int32, device="cuda")
    dd = torch.empty((32, V), dtype=torch.float32, device="cuda")
    forms = {"plain": (api.MB_POLICY_FIXED, False), "learned": (api.MB_POLICY_LEARNED, False),
             "batched": (api.MB_POLICY_FIXED, True),
             "learned_batched": (api.MB_POLICY_LEARNED, True)}
    reps = max(1, min(args.steps, 3))
    res, ref_out, launches = {}, None, 0
    for name, (policy, batching) in forms.items():
        ctx.set_policy(policy)
        ctx.set_batching(batching)
        for _ in range(max(1, args.warmup // 3)):
            g.bfs(bsrc, out=lv)
            g.sssp(ssrc, out=dd)
        ms_b = ms_s = 0.0
        e_b = e_s = 0
        for _ in range(reps):
            flush_l2(flush)
            torch.cuda.synchronize()
            _, sb = g.bfs(bsrc, out=lv)
            flush_l2(flush)
            torch.cuda.synchronize()
            _, ss = g.sssp(ssrc, out=dd)
            ms_b += sb["device_ms"]
            ms_s += ss["device_ms"]
            e_b += sb["edges_traversed"]
            e_s += ss["edges_traversed"]
            launches += sb["kernel_launches"] + ss["kernel_launches"]
        outs = (lv.cpu().numpy().copy(), dd.cpu().numpy().view(np.uint32).copy())
        if ref_out is None:
            ref_out = outs
        same = bool(np.array_equal(outs[0], ref_out[0]) and np.array_equal(outs[1], ref_out[1]))
        res[name] = {"gteps": round((e_b + e_s) / ((ms_b + ms_s) / 1e3) / 1e9, 3),
                     "bfs_gteps": round(e_b / (ms_b / 1e3) / 1e9, 3),
                     "sssp_gteps": round(e_s / (ms_s / 1e3) / 1e9, 3),
                     "bfs_ms": round(ms_b / reps, 3), "sssp_ms": round(ms_s / reps, 3),
                     "identical_to_plain": same}
    ctx.set_policy(api.MB_POLICY_FIXED)
    ctx.set_batching(True)
    base = res["plain"]["gteps"]
    for name in res:
        res[name]["vs_plain"] = round(res[name]["gteps"] / base, 3)
    res["sources"] = {"bfs": "vertices 0..63", "sssp": "vertices 0..31"}
    res["scheduler_training"] = {
        "seconds": round(train_s, 1),
        "samples": {k: trained[m][1] for k, m in MODELS},
        "final_loss": {k: round(trained[m][0], 4) for k, m in MODELS},
        "traces": "uniform / R-MAT / grid families, 2^%s vertices, seeds 101 and 102"
                  % "/".join(str(x) for x in TRAIN_SCALES)}
    # per superstep on this graph (source 0): the fixed rule's choice, the
    # model's choice and the best of all schedules, each choice costed as
    # that superstep plus the 3 after it under the fixed rule
    per_step = {}
    for app, name, model in ((0, "bfs", api.MB_MODEL_BFS), (1, "sssp", api.MB_MODEL_SSSP),
                             (2, "batched_bfs", api.MB_MODEL_BATCHED)):
        X, T, F = ctx.scheduler_collect(g, app, 0)
        r = scheduler.evaluate(ctx, X, T, F, model)
        per_step[name] = {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()}
    res["per_superstep"] = per_step
    res["gpu_launches"] = launches
    return res


def _timed(fn, reps, flush):
    """Median device ms (library stats) of fn() over reps runs, L2 flushed before each."""
    import torch
    ms, st = [], None
    for _ in range(reps):
        flush_l2(flush)
        torch.cuda.synchronize()
        st = fn()
        ms.append(st["device_ms"])
    return float(np.median(ms)), st


def _trav(st, ms, nbytes, pk):
    ach = nbytes / (ms / 1e3) / 1e9
    return {"gteps": round(st["edges_traversed"] / (ms / 1e3) / 1e9, 3), "ms": round(ms, 4),
            "supersteps": st["supersteps"], "edges_traversed": st["edges_traversed"],
            "schedule_count": st["schedule_count"],
            "roofline": {"achieved_gbs": round(ach, 1), "frac": round(ach / pk, 4)}}


def bench_configs(ctx, api, args, flush):
    """The other configurations: C3 road-like grid, C4a batched sources on a
    2^22-vertex R-MAT, C5 2^24-vertex R-MAT at scale (fixed vs learned)."""
    import torch
    from medusa_b200 import autotune, scheduler
    pk, _ = peaks()
    reps = max(1, min(args.steps, 3))
    out = {}
    # C3: 1448x1448 grid, 10% of the edges dropped, 0.5% shortcuts, weights [1,100]
    g = ctx.generate(api.grid_params(1448, 1448, 0.1, 0.005, seed=SEED, wmin=1, wmax=100))
    V = g.V
    tuned3 = {} if args.no_autotune else autotune.tune_traversals(ctx, g, 0, reps=2)[0]
    lv = torch.empty(V, dtype=torch.int32, device="cuda")
    dd = torch.empty(V, dtype=torch.float32, device="cuda")
    # the fixed rule, then the learned scheduler (the same tuned parameters)
    arms, res = {}, {}
    for name, policy in (("learned", api.MB_POLICY_LEARNED), ("fixed", api.MB_POLICY_FIXED)):
        ctx.set_policy(policy)
        for _ in range(2):
            g.bfs([0], out=lv)
            g.sssp([0], out=dd)
        mb, sb = _timed(lambda: g.bfs([0], out=lv)[1], reps, flush)
        ms_, ss = _timed(lambda: g.sssp([0], out=dd)[1], reps, flush)
        arms[name] = {"bfs": _trav(sb, mb, bfs_bytes(sb, V), pk),
                      "sssp": _trav(ss, ms_, sssp_bytes(ss, V), pk)}
        res[name] = (lv.cpu().numpy().copy(), dd.cpu().numpy().view(np.uint32).copy())
    out["c3_grid"] = {"workload": "grid 1448x1448, 10% edges dropped, 0.5% shortcuts, weights "
                                  "int [1,100], seed 1, source 0 (corner)",
                      "vertices": V, "edges": g.E,
                      "bfs": arms["fixed"]["bfs"], "sssp": arms["fixed"]["sssp"],
                      "learned": arms["learned"],
                      "learned_identical": bool(np.array_equal(res["fixed"][0], res["learned"][0]) and
                                                np.array_equal(res["fixed"][1], res["learned"][1])),
                      "autotuned": {k: float(v) for k, v in tuned3.items()},
                      "verified_against_bsp": verify_against_bsp(ctx, api, g, lv, dd)}
    g.close()
    if not args.no_cpu_baseline:
        out["c3_grid"]["cpu_baseline"] = cpu_baseline_traversals(
            host_edges("grid", rows=1448, cols=1448, drop_frac=0.1, shortcut_frac=0.005,
                       seed=SEED, wmin=1, wmax=100),
            "one BFS + one SSSP from the corner on the full C3 graph (reference Medusa_Exec_CPU, "
            "OpenMP)")
    reset_tunables(ctx, api)
    del lv, dd
    # C4a: 64 BFS + 32 SSSP sources on R-MAT 2^22 / 2^26, batched vs one loop per source
    g = ctx.generate(api.rmat_params(22, 1 << 26, 0.45, 0.15, 0.15, seed=SEED, wmin=1, wmax=1000))
    V = g.V
    lv = torch.empty((64, V), dtype=torch.int32, device="cuda")
    dd = torch.empty((32, V), dtype=torch.float32, device="cuda")
    c4 = {"workload": "R-MAT 2^22 vertices, 2^26 edges, (0.45,0.15,0.15,0.25), seed 1; "
                      "BFS sources 0..63, SSSP sources 0..31", "vertices": V, "edges": g.E}
    outs = {}
    for name, batching, policy in (("plain", False, api.MB_POLICY_FIXED),
                                   ("batched", True, api.MB_POLICY_FIXED),
                                   ("learned_batched", True, api.MB_POLICY_LEARNED)):
        ctx.set_batching(batching)
        ctx.set_policy(policy)
        g.bfs(list(range(64)), out=lv)
        g.sssp(list(range(32)), out=dd)
        mb, sb = _timed(lambda: g.bfs(list(range(64)), out=lv)[1], 1, flush)
        ms_, ss = _timed(lambda: g.sssp(list(range(32)), out=dd)[1], 1, flush)
        outs[name] = (lv.cpu().numpy().copy(), dd.cpu().numpy().view(np.uint32).copy())
        c4[name] = {"bfs_gteps": round(sb["edges_traversed"] / (mb / 1e3) / 1e9, 3),
                    "sssp_gteps": round(ss["edges_traversed"] / (ms_ / 1e3) / 1e9, 3),
                    "gteps": round((sb["edges_traversed"] + ss["edges_traversed"])
                                   / ((mb + ms_) / 1e3) / 1e9, 3),
                    "bfs_ms": round(mb, 3), "sssp_ms": round(ms_, 3)}
    ctx.set_batching(True)
    ctx.set_policy(api.MB_POLICY_FIXED)
    for name in ("batched", "learned_batched"):
        c4[name]["vs_plain"] = round(c4[name]["gteps"] / c4["plain"]["gteps"], 3)
    c4["identical"] = all(np.array_equal(outs["plain"][k], outs[name][k])
                          for name in ("batched", "learned_batched") for k in (0, 1))
    out["c4a_batched"] = c4
    g.close()
    del lv, dd, outs
    # C5: R-MAT 2^24 / 2^28, (0.57,0.19,0.19,0.05), weights [1,1000]; fixed vs learned
    g = ctx.generate(api.rmat_params(24, 1 << 28, 0.57, 0.19, 0.19, seed=SEED, wmin=1, wmax=1000))
    V, E = g.V, g.E
    tuned5 = {} if args.no_autotune else autotune.tune_traversals(ctx, g, 0, reps=2)[0]
    lv = torch.empty(V, dtype=torch.int32, device="cuda")
    dd = torch.empty(V, dtype=torch.float32, device="cuda")
    rk = torch.empty(V, dtype=torch.float32, device="cuda")
    c5 = {"workload": "R-MAT 2^24 vertices, 2^28 edges, (0.57,0.19,0.19,0.05), seed 1, weights "
                      "int [1,1000]; BFS and SSSP from 0, PageRank 20 supersteps from 1/N",
          "vertices": V, "edges": E}
    res = {}
    for name, policy in (("fixed", api.MB_POLICY_FIXED), ("learned", api.MB_POLICY_LEARNED)):
        ctx.set_policy(policy)
        g.bfs([0], out=lv)
        g.sssp([0], out=dd)
        mb, sb = _timed(lambda: g.bfs([0], out=lv)[1], reps, flush)
        ms_, ss = _timed(lambda: g.sssp([0], out=dd)[1], reps, flush)
        res[name] = (lv.cpu().numpy().copy(), dd.cpu().numpy().view(np.uint32).copy())
        c5[name] = {"bfs": _trav(sb, mb, bfs_bytes(sb, V), pk),
                    "sssp": _trav(ss, ms_, sssp_bytes(ss, V), pk)}
    ctx.set_policy(api.MB_POLICY_FIXED)
    c5["learned_identical"] = bool(np.array_equal(res["fixed"][0], res["learned"][0]) and
                                   np.array_equal(res["fixed"][1], res["learned"][1]))
    lv.copy_(torch.from_numpy(res["fixed"][0]))
    dd.copy_(torch.from_numpy(res["fixed"][1].view(np.float32)))
    c5["verified_against_bsp"] = verify_against_bsp(ctx, api, g, lv, dd)
    per_step = {}
    for app, name, model in ((0, "bfs", api.MB_MODEL_BFS), (1, "sssp", api.MB_MODEL_SSSP)):
        X, T, F = ctx.scheduler_collect(g, app, 0, max_samples=32)
        r = scheduler.evaluate(ctx, X, T, F, model)
        per_step[name] = {k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()}
    c5["per_superstep"] = per_step
    c5["autotuned"] = {k: float(v) for k, v in tuned5.items()}
    reset_tunables(ctx, api)
    pres, pranks = time_pagerank_orders(ctx, api, g, 20, flush, reps, not args.no_autotune, rk)
    b = 8 * E + 16 * V + 4
    for name in pres:
        per = pres[name]["ms_per_superstep"]
        pres[name]["roofline"] = {"achieved_gbs": round(b / (per / 1e3) / 1e9, 1),
                                  "frac": round(b / (per / 1e3) / 1e9 / pk, 4)}
    c5["pagerank"] = dict(pres["reference_order"])
    c5["pagerank"]["summation_order"] = "the reference's (MEG slots, sequential float fold), default"
    c5["pagerank"]["fixed_order"] = pres["fixed_order"]
    g.close()
    del lv, dd, rk
    if not args.no_cpu_baseline:
        V_, s_, d_, _ = host_edges("rmat", scale=24, num_edges=1 << 28, a=0.57, b=0.19, c=0.19,
                                   seed=SEED)
        c5["pagerank"]["accuracy"] = pr_accuracy(V_, s_, d_, 20, pranks)
        del s_, d_
    out["c5_scale"] = c5
    out["c4b_many_graphs"] = bench_many_graphs(ctx, api, reps, not args.no_autotune)
    return out


def bench_many_graphs(ctx, api, reps, tune=True):
    """C4b: 256 R-MAT graphs of uneven sizes, 20 PageRank supersteps + one
    BFS each, in ONE persistent launch vs one library call per graph."""
    import torch
    from medusa_b200 import autotune
    ps = api.c4b_params(256, seed=SEED)
    b = ctx.batch_generate(ps)
    ranks = torch.empty(b.total_V, dtype=torch.float32, device="cuda")
    levels = torch.empty(b.total_V, dtype=torch.int32, device="cuda")
    tuned, table = ({}, []) if not tune else autotune.tune_batch(ctx, b, 20, reps=2, ranks=ranks,
                                                                levels=levels)
    b.run(20, None, ranks, levels)
    ms = []
    for _ in range(reps):
        torch.cuda.synchronize()
        _, _, st = b.run(20, None, ranks, levels)
        ms.append(st["device_ms"])
    one = float(np.median(ms))
    r_all = ranks.cpu().numpy()
    l_all = levels.cpu().numpy()
    # the same work one graph at a time through mb_pagerank / mb_bfs (the
    # many-graph kernel sums in the fixed order)
    ctx.set_pagerank_order(api.MB_PR_ORDER_FIXED)
    seq_ms, same = 0.0, True
    for i, p in enumerate(ps):
        g = ctx.generate(p)
        r, s1 = g.pagerank(20, 1.0 / g.V)
        lv, s2 = g.bfs([0])
        seq_ms += s1["device_ms"] + s2["device_ms"]
        same &= bool(np.array_equal(r.view(np.uint32), r_all[b.vbase[i]:b.vbase[i + 1]].view(np.uint32))
                     and np.array_equal(lv[0], l_all[b.vbase[i]:b.vbase[i + 1]]))
        g.close()
    ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
    edges = st["edges_traversed"]
    res = {"workload": "256 R-MAT graphs, (0.45,0.15,0.15,0.25), vertices 2^10..2^18 log-uniform, "
                       "average degree uniform [4,32], seed 1; 20 PageRank supersteps + one BFS "
                       "from vertex 0 each",
           "graphs": b.n, "vertices": int(b.total_V), "edges": int(b.total_E),
           "one_launch": {"ms": round(one, 3), "edges_per_s": round(edges / (one / 1e3), 1),
                          "kernel_launches": st["kernel_launches"]},
           "one_call_per_graph": {"ms": round(seq_ms, 3),
                                  "edges_per_s": round(edges / (seq_ms / 1e3), 1)},
           "vs_one_call_per_graph": round(seq_ms / one, 3),
           "identical": same,
           "autotuned": {k: int(v) for k, v in tuned.items()},
           "autotune_candidates": len(table)}
    b.close()
    ctx.set_tunable("batch_threads", -1)
    ctx.set_tunable("batch_edges_per_cta", -1)
    return res


def pr_accuracy(V, src, dst, iters, ranks):
    """PageRank errors, per run: each result's max relative error per vertex
    against the reference's FP32 ranks (the oracle's sequential fold in the
    reference's MEG order, bit-identical to the reference's CPU code on the
    golden graphs) and its L1 error against the FP64 oracle (absolute, and
    relative to the FP64 ranks' sum).  ranks: {name: float32 array}."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    aa = O.AAGraph(V, src, dst)
    ref = O.pagerank(V, aa, None, iters, 1.0 / V).astype(np.float64)
    r64 = O.pagerank(V, aa, None, iters, 1.0 / V, fp64=True)
    del aa
    out = {"reference_fp32_l1_vs_fp64": float(np.abs(ref - r64).sum()),
           "fp64_rank_sum": float(r64.sum())}
    for name, r in ranks.items():
        r = r.astype(np.float64)
        out[name] = {"max_rel_vs_reference": float((np.abs(r - ref) / ref).max()),
                     "vertices_above_1e-5": int(((np.abs(r - ref) / ref) > 1e-5).sum()),
                     "bit_identical_to_reference": bool(np.array_equal(r, ref)),
                     "l1_vs_fp64": float(np.abs(r - r64).sum()),
                     "l1_vs_fp64_relative": float(np.abs(r - r64).sum() / r64.sum())}
    out["oracle_seconds"] = round(time.perf_counter() - t0, 1)
    return out


def time_pagerank_orders(ctx, api, g, iters, flush, reps, tune, out):
    """Device ms per superstep and the ranks of both summation orders: the
    reference's (default; autotuned hub threshold and light packing) and the
    fixed parallel order (autotuned light packing and short-block pairing)."""
    from medusa_b200 import autotune
    res, ranks = {}, {}
    for name, order in (("reference_order", api.MB_PR_ORDER_REFERENCE),
                        ("fixed_order", api.MB_PR_ORDER_FIXED)):
        ctx.set_pagerank_order(order)
        tuned = {}
        if tune:
            tuned = autotune.tune_pagerank(ctx, g, iters, reps=2, out=out)[0]
        g.pagerank(iters, 1.0 / g.V, out=out)
        ms, st = _timed(lambda: g.pagerank(iters, 1.0 / g.V, out=out)[1], reps, flush)
        ranks[name] = out.cpu().numpy().copy()
        res[name] = {"ms_per_superstep": round(ms / iters, 5),
                     "edges_per_s": round(g.E / (ms / iters / 1e3), 1),
                     "kernel_launches": st["kernel_launches"],
                     "autotuned": {k: float(v) for k, v in tuned.items()}}
        for k in tuned:
            ctx.set_tunable(k, -1)
    ctx.set_pagerank_order(api.MB_PR_ORDER_REFERENCE)
    return res, ranks


def bench_pagerank(ctx, api, args, flush):
    """C1: uniform 2^18 / 2^22, 10 supersteps from 1/N, both summation orders
    with their errors, and the reference's own CPU PageRank on the same graph."""
    import torch
    p = c1_params(api)
    g = ctx.generate(p)
    V, E = g.V, g.E
    r = torch.empty(V, dtype=torch.float32, device="cuda")
    res, ranks = time_pagerank_orders(ctx, api, g, PR_ITERS, flush, max(args.steps, 3),
                                      not args.no_autotune, r)
    g.close()
    pk, _ = peaks()
    b = 8 * E + 16 * V + 4
    per_iter_ms = res["reference_order"]["ms_per_superstep"]
    ach = b / (per_iter_ms / 1e3) / 1e9
    out = {"workload": "uniform 2^18 vertices, 2^22 edges, seed 1, 10 supersteps from 1/N",
           "edges_per_s": round(E / (per_iter_ms / 1e3), 1), "ms_per_superstep": per_iter_ms,
           "summation_order": "the reference's (MEG slots, sequential float fold), default",
           "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": pk, "unit": "GB/s",
                        "frac": round(ach / pk, 4),
                        "bytes_per_superstep": b, "formula": "8*E + 16*V + 4"},
           "orders": res}
    if not args.no_cpu_baseline:
        V_, s_, d_, _ = host_edges("uniform", num_vertices=C1["num_vertices"],
                                   num_edges=C1["num_edges"], seed=SEED)
        out["accuracy"] = pr_accuracy(V_, s_, d_, PR_ITERS, ranks)
        out["cpu_baseline"] = cpu_baseline_pagerank(V_, s_, d_, PR_ITERS)
    return out


def cpu_baseline_pagerank(V, src, dst, iters):
    """The reference's own CPU PageRank (oracle/_ref: MPG's sortByDegree +
    buildMEG + its per-vertex send/update functions, OpenMP) on the graph."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"unavailable": "oracle/_ref not built"}
    nthr = min(os.cpu_count() or 1, 24)
    rp = O.RefGraph("pr", V, src, dst)
    ms = []
    for _ in range(3):
        _, m = rp.pagerank(iters, 1.0 / V, nthr)
        ms.append(m)
    rp.close()
    per = float(np.median(ms)) / iters
    return {"value": round(len(src) / (per / 1e3), 1), "unit": "edges/s per superstep",
            "ms_per_superstep": round(per, 3), "cores": nthr, "kind": "reference",
            "sample": "%d supersteps on the full C1 graph, median of 3 runs" % iters}


def cpu_baseline_traversals(edges, sample):
    """The reference's CPU BFS and SSSP (oracle/_ref, OpenMP) from vertex 0 of
    the graph `edges` = (V, src, dst, w)."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"unavailable": "oracle/_ref not built"}
    V, s, d, w = edges
    nthr = min(os.cpu_count() or 1, 24)
    gb = O.RefGraph("bfs", V, s, d)
    lv, ms_b = gb.bfs(0, nthr)
    gb.close()
    gs = O.RefGraph("sssp", V, s, d, w)
    dd, ms_s = gs.sssp(0, nthr)
    gs.close()
    outdeg = np.bincount(s, minlength=V)
    er = int(outdeg[lv >= 0].sum()) + int(outdeg[dd < 1e9].sum())
    return {"value": round(er / ((ms_b + ms_s) / 1e3) / 1e9, 5), "unit": "GTEPS", "cores": nthr,
            "kind": "reference", "sample": sample, "bfs_ms": round(ms_b, 2), "sssp_ms": round(ms_s, 2)}


def cpu_baseline(api, args):
    """The reference's CPU path (oracle/_ref) on the same graph: one BFS + one SSSP."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"unavailable": "oracle/_ref not built"}
    V, s, d, w = c2_edges()
    nthr = min(os.cpu_count() or 1, 24)
    gb = O.RefGraph("bfs", V, s, d)
    lv, ms_b = gb.bfs(0, nthr)
    gb.close()
    gs = O.RefGraph("sssp", V, s, d, w)
    dd, ms_s = gs.sssp(0, nthr)
    gs.close()
    outdeg = np.bincount(s, minlength=V)
    er = int(outdeg[lv >= 0].sum()) + int(outdeg[dd < 1e9].sum())
    return {"value": round(er / ((ms_b + ms_s) / 1e3) / 1e9, 5), "unit": "GTEPS",
            "cores": nthr, "kind": "reference",
            "sample": "one BFS + one SSSP from source 0 on the full workload graph "
                      "(reference Medusa_Exec_CPU, OpenMP)",
            "bfs_ms": round(ms_b, 2), "sssp_ms": round(ms_s, 2)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    V, s, d, w = c2_edges()
    nthr = min(os.cpu_count() or 1, 24)
    gb = O.RefGraph("bfs", V, s, d)
    gs = O.RefGraph("sssp", V, s, d, w)
    outdeg = np.bincount(s, minlength=V)
    for _ in range(args.warmup):
        gb.bfs(0, nthr)
        gs.sssp(0, nthr)
    ms, edges = 0.0, 0
    for _ in range(args.steps):
        lv, mb = gb.bfs(0, nthr)
        dd, msd = gs.sssp(0, nthr)
        ms += mb + msd
        edges += int(outdeg[lv >= 0].sum()) + int(outdeg[dd < 1e9].sum())
    val = edges / (ms / 1e3) / 1e9
    out = {"impl": "reference", "metric": METRIC, "value": round(val, 5), "unit": "GTEPS",
           "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "int32/f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "vertices": V, "edges": int(len(s)), "sources": [0]},
           "cpu_baseline": {"value": round(val, 5), "unit": "GTEPS", "cores": nthr,
                            "kind": "reference",
                            "sample": "each step: one BFS + one SSSP from source 0 on the full graph"},
           "e2e": {"value": round(val, 5), "unit": "GTEPS", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    gb.close()
    gs.close()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="medusa", choices=["medusa", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pagerank", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="run with the built-in launch parameters instead of tuned ones")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the C3 grid, C4a batched and C5 at-scale measurements")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the plain / learned / batched / learned+batched comparison")
    ap.add_argument("--hostloop", action="store_true",
                    help="host-driven superstep loop instead of one CUDA graph per loop")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_medusa(args)


if __name__ == "__main__":
    main()

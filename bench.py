"""Benchmark: batched river datagen solve on B200.

Workload (one "step"): 4096 independent seeded river subgames, each solved by
DCFR until exploitability <= 0.3% of its pot or 300 iterations, all in one
persistent launch (plus the per-board setup kernel), from a zeroed state.
Per-spot inputs follow the batched datagen configuration: 5-card boards,
weights ~Beta(0.5, 0.5) with 30% zeroed and board-masked, pot U[20, 200],
SPR U[0.5, 10], bet menu from {[50%, a], [33%, 75%, a], [25%, 50%, 100%,
150%, a]}, raise {100%, a}.  Data are synthetic (seeded numpy PCG64).

value  = spots solved per second, inputs resident in HBM (device events
         around the setup + solve kernels of each step).
e2e    = the same through the public API from host buffers: tree build,
         host->device copy (pinned), solve, results device->host, every
         step; batch k + 1 is built on a host thread while batch k solves,
         as a datagen job runs (--e2e-pipelined 0: one batch at a time).
Multi-GPU (torchrun): every rank solves its own 4096 spots (replicas,
weak scaling); the step time is the max over ranks.

`--impl reference` times the reference CPU algorithm (the oracle's C++
restatement of crates/range-solver, run spot-parallel on all host threads)
on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "river spots/s at <=0.3% pot exploitability"
UNIT = "spots/s"
TARGET_FRAC = 0.003
MAX_ITER = 300


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic_per_spot_iteration(kernel: str):
    """DRAM read + write bytes per spot-iteration of the committed ncu capture
    of the batched solve kernel that ran (profiles/<kernel>_river_datagen_1024.md),
    or None."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", f"{kernel}_river_datagen_1024.md")
    try:
        with open(path) as f:
            m = re.search(r"^traffic_bytes_per_spot_iteration:\s*([0-9.]+)", f.read(), re.M)
        return float(m.group(1)) if m else None
    except OSError:
        return None


def rank_max(x: float, dist, device: str) -> float:
    """Max of x over all ranks of the process group (x itself without one).
    Every rank must call it at the same point: it is a collective."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_throughput(spots_per_rank: int, world: int, step_ms_max: float) -> float:
    """Whole-job spots/s of `world` independent replicas, each solving
    spots_per_rank spots per step, timed by the slowest rank."""
    return world * spots_per_rank / (step_ms_max / 1e3)


def turn_game_measure(ps, spots, iters: int, cpu_iters: int):
    """One turn subgame (4-card board, 48 river deals, U[0,1] ranges, pot 100,
    stack 300, bets 33% / 75% / all-in, raise 60%) solved for a fixed number of
    iterations on the whole GPU (grid mode), timed through ps.solve from host
    to host (exploitability every 5 iterations and finalize included), beside
    the oracle's time for `cpu_iters` iterations with the chance children
    spread over all host threads."""
    import torch

    r, b, t = spots.turn_spot(2)
    warm = spots.product_game(r, b, t)
    ps.solve(warm, 5, 0.0)
    g = spots.product_game(r, b, t)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e = ps.solve(g, iters, 0.0)
    dt = time.perf_counter() - t0
    out = {"workload": "turn subgame: 4-card board, 48 river deals, pot 100, stack 300, bets 33%/75%/a, raise 60%",
           "nodes": g.num_nodes(), "hands": [g.num_private_hands(0), g.num_private_hands(1)],
           "iterations": iters, "gpu_ms_per_iteration": dt / iters * 1e3,
           "gpu_note": "ps.solve from host: iterations, exploitability every 5, finalize",
           "exploitability_pct_pot": 100.0 * e / t.starting_pot}
    if cpu_iters > 0:
        from oracle import oracle as O

        threads = os.cpu_count() or 1
        O.set_chance_threads(threads)  # river chance children in parallel, as the reference's rayon
        try:
            o = spots.oracle_game(r, b, t)
            t0 = time.perf_counter()
            o.solve(cpu_iters, 0.0)  # the same loop as the GPU side: checks every 5 iterations, finalize
            out["cpu_ms_per_iteration"] = (time.perf_counter() - t0) / cpu_iters * 1e3
        finally:
            O.set_chance_threads(1)
        out["cpu"] = {"threads": threads, "kind": "port", "iterations_timed": cpu_iters,
                      "note": "solve(): exploitability every 5 iterations and finalize, as the GPU side",
                      "parallel": "the 48 river chance children of each chance node, as solver.rs:264-326 with rayon"}
    return out


def river_game_measure(ps, spots, iters: int, cpu_iters: int):
    """One plain river subgame (5-card board, U[0,1] ranges masked by the
    board, pot 100, stack 200, bets 50% / 100% / all-in, raise 100%) solved
    for `iters` iterations through ps.solve (one launch on a 16-CTA
    thread-block cluster, whose hardware barrier ends each step; a single
    river game is latency-bound, so the line gives iterations/s and the
    exploitability reached), beside the oracle on
    one host thread (river nodes never parallelise in the reference,
    node.rs:347-349), timed through the same solve loop (checks every 5
    iterations, finalize).  The tree has no bet cap: the reference's tree
    builder has none, so both sides solve the same tree."""
    import torch

    r, b, t = spots.river_spot(1)
    ps.solve(spots.product_game(r, b, t), 5, 0.0)  # warm
    g = spots.product_game(r, b, t)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e = ps.solve(g, iters, 0.0)
    dt = time.perf_counter() - t0
    H0 = g.num_private_hands(0)
    root = g.strategy_at_index(0).reshape(-1, H0)
    out = {"workload": "river subgame: pot 100, stack 200, bets 50%/100%/a, raise 100%",
           "nodes": g.num_nodes(), "hands": [H0, g.num_private_hands(1)],
           "iterations": iters, "gpu_iterations_per_s": iters / dt, "gpu_ms_per_iteration": dt / iters * 1e3,
           "gpu_note": "ps.solve from host: iterations, exploitability every 5, finalize",
           "exploitability_pct_pot": 100.0 * e / t.starting_pot, "launch": g.schedule(),
           "root_action_frequencies": [float(x) for x in root.mean(axis=1)]}
    if cpu_iters > 0:
        o = spots.oracle_game(r, b, t)
        t0 = time.perf_counter()
        o.solve(cpu_iters, 0.0)
        out["cpu_iterations_per_s"] = cpu_iters / (time.perf_counter() - t0)
        out["cpu"] = {"threads": 1, "kind": "port", "iterations_timed": cpu_iters,
                      "note": "solve(): exploitability every 5 iterations and finalize, as the GPU side"}
    return out


def turn_adjoint_measure(ps, spots, n: int, iters: int, cpu_sample: int):
    """Depth-limited turn spots solved with seeded boundary values, then the
    gradient of loss = MSE(root cfvalues, seeded target) with respect to the
    boundary values through the batched adjoint (BatchSolvedValues): spots/s
    forward + backward on the device, beside the oracle's forward (the same
    iterations per spot, spot-parallel on the host cores) on a sample."""
    import torch
    from poker_solver_rust_b200.autograd import batch_solved_values

    sp = spots.turn_boundary_spots(n, seed=11)
    free0 = torch.cuda.mem_get_info()[0]
    torch.cuda.reset_peak_memory_stats()
    bs = ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp])
    rng = np.random.default_rng(12)
    V = spots.boundary_values(rng, bs)
    B = torch.tensor(V, device="cuda", requires_grad=True)
    target = torch.tensor(rng.normal(0, 1, (n, 2, 1326)).astype(np.float32), device="cuda") * \
        torch.tensor(0.25 * bs.starting_pots, device="cuda")[:, None, None]
    times = []
    for rep in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cfv = batch_solved_values(bs, B, iters)
        loss = ((cfv - target) ** 2).mean()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        B.grad = None
        loss.backward()
        torch.cuda.synchronize()
        times.append((t1 - t0, time.perf_counter() - t1))
    fwd, bwd = min(times, key=lambda x: x[0] + x[1])
    used = (free0 - torch.cuda.mem_get_info()[0]) / 1e9
    out = {"workload": f"{n} depth-limited turn spots (bets 33%/75%/a, raise 60%, boundary at each non-fold turn "
                       "terminal; Beta(0.5,0.5) ranges 30% zeroed, pot U[20,200], SPR U[0.5,10]), boundary values "
                       f"~N(0,(pot/4)^2), {iters} DCFR iterations, loss = MSE(root cfvalues, seeded target), "
                       "gradient w.r.t. the boundary values",
           "boundary_items": bs.num_boundary_items(), "iterations": iters,
           "spots_per_s_fwd_bwd": n / (fwd + bwd), "fwd_ms": fwd * 1e3, "bwd_ms": bwd * 1e3,
           "device_gb": used, "note": "host-timed with device synchronisation; device_gb = device memory held "
                                      "by the batch and the tensors at the end"}
    if cpu_sample > 0:
        threads = os.cpu_count() or 1
        sample = sp[:min(n, CPU_SPOTS_PER_THREAD * threads)]
        items = bs.boundary_items()

        def one(i):
            r, b, t = sample[i]
            o = spots.oracle_game(r, b, t)
            ks = np.nonzero(items["spot"] == i)[0]
            for j, k in enumerate(ks):
                for p in range(2):
                    cards = o.private_cards(p)
                    o.set_boundary_cfvs(j, p, np.ascontiguousarray(
                        V[k, p, [ps.card_pair_to_index(int(x), int(y)) for x, y in cards]]))
            for it in range(iters):
                o.solve_step(it)
            o.root_cfvalues(0)
            o.root_cfvalues(1)

        from concurrent.futures import ThreadPoolExecutor
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(one, range(len(sample))))
        dt = time.perf_counter() - t0
        out["cpu_forward"] = {"spots_per_s": len(sample) / dt, "cores": threads, "kind": "port",
                              "sample": f"first {len(sample)} spots: boundary values, {iters} iterations, root "
                                        "cfvalues (no gradient)"}
    return out


def turn_datagen_measure(ps, spots, n: int, iters: int, interval: int):
    """The on-device turn-datagen loop (solve_with_boundary_net) on n
    depth-limited turn spots with a stand-in boundary network (7 x 500 bf16
    MLP, seeded random weights): spots/s for `iters` iterations with the
    boundaries re-evaluated every `interval`."""
    import torch
    from poker_solver_rust_b200.datagen import solve_with_boundary_net

    sp = spots.turn_boundary_spots(n, seed=21)
    bs = ps.BatchSolver([spots.card_config(r, b) for r, b, _ in sp], [t for _, _, t in sp])
    torch.manual_seed(0)
    layers = [torch.nn.Linear(2720, 500), torch.nn.ReLU()]
    for _ in range(6):
        layers += [torch.nn.Linear(500, 500), torch.nn.ReLU()]
    net = torch.nn.Sequential(*layers, torch.nn.Linear(500, 1326)).cuda().to(torch.bfloat16)
    def timed(factored, reps):
        best = None
        for rep in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            solve_with_boundary_net(bs, net, iters, interval, bf16=True, factored=factored)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        return best

    best = timed(True, 3)
    e, _ = bs.results()
    dense = timed(False, 2)
    return {"workload": f"{n} depth-limited turn spots, {iters} iterations, boundary network re-evaluated every "
                        f"{interval} (7x500 bf16 MLP stand-in, 2720 -> 1326)",
            "boundary_items": bs.num_boundary_items(), "spots_per_s": n / best, "seconds": best,
            "first_layer": "factored (ps_boundary_first_layer)",
            "spots_per_s_dense_first_layer": n / dense,
            "mean_expl_pct_pot": float(np.mean(e / bs.starting_pots) * 100),
            "note": "host-timed end to end on the device: network (first layer factored over the river cards), "
                    "48-river average, boundary values, iterations; the dense variant writes the 2720-value "
                    "input rows and runs the first layer on them"}


def make_workload(n_spots: int, seed: int):
    from tests import spots

    return spots.datagen_spots(n_spots, seed=seed)


CPU_SPOTS_PER_THREAD = 16  # per timed step: enough that the last spots to finish do not set the step time


def cpu_sample(work, step: int, threads: int, per_thread: int = CPU_SPOTS_PER_THREAD):
    """The spots of CPU step `step`: per_thread spots per host thread, taken in
    order from the GPU arm's own spots (wrapping around)."""
    n = per_thread * threads
    return [work[(step * n + i) % len(work)] for i in range(n)]


def oracle_solve_sample(sample, threads: int):
    """Reference CPU algorithm, spot-parallel: each host thread takes the next
    spot as it finishes one (the reference's datagen workers, one game per
    thread, pipeline.rs:111-124).  Returns (seconds, iterations per spot)."""
    from tests import spots

    def one(spec):
        r, b, t = spec
        g = spots.oracle_game(r, b, t)
        g.solve(MAX_ITER, TARGET_FRAC * t.starting_pot)
        return g.iterations_run

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, sample))
    return time.perf_counter() - t0, np.array(res)


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    # each step: a bounded sample of the GPU arm's own 4096 spots (rank 0's seed)
    work = make_workload(args.spots, seed=args.seed)
    spt = args.cpu_spots_per_thread
    per_step = spt * threads
    for w in range(args.warmup):
        oracle_solve_sample(cpu_sample(work, w, threads, spt), threads)
    secs, its = [], []
    for k in range(args.steps):
        dt, it = oracle_solve_sample(cpu_sample(work, args.warmup + k, threads, spt), threads)
        secs.append(dt)
        its.append(it)
    tot = sum(secs)
    value = per_step * args.steps / tot
    mean_it = float(np.concatenate(its).mean())
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded PCG64)",
        "config": {"workload": f"batched river datagen: {args.spots} spots per GPU to <=0.3% pot or "
                               f"{MAX_ITER} iterations", "parallelism": f"host threads x{threads}",
                   "timed_sample": f"{per_step} spots per step ({spt} per host thread), taken in "
                                   f"order from the GPU arm's {args.spots} spots"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{per_step} spots per step ({spt} per thread) of the GPU arm's "
                                   f"spots, spot-parallel on {threads} threads",
                         "mean_iterations": mean_it},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--spots", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--cpu-sample", type=int, default=1, help="0 = skip the CPU baseline leg")
    ap.add_argument("--cpu-spots-per-thread", type=int, default=CPU_SPOTS_PER_THREAD,
                    help="spots per host thread in each CPU step (reference arm and CPU baseline leg)")
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--block", type=int, default=-1, help="threads per CTA; -1 = autotune, 0 = library default")
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=3, help="steps of the one-batch-at-a-time e2e leg")
    ap.add_argument("--e2e-pipelined", type=int, default=1,
                    help="1 = e2e over --steps batches, the next one built while the current one solves")
    ap.add_argument("--turn-iters", type=int, default=500, help="single turn game iterations (0 = skip)")
    ap.add_argument("--turn-cpu-iters", type=int, default=50)
    ap.add_argument("--river-iters", type=int, default=1000, help="single river game iterations (0 = skip)")
    ap.add_argument("--river-cpu-iters", type=int, default=200)
    ap.add_argument("--adjoint-spots", type=int, default=1024, help="depth-limited turn spots + adjoint (0 = skip)")
    ap.add_argument("--adjoint-iters", type=int, default=300)
    ap.add_argument("--datagen-spots", type=int, default=512, help="turn-datagen loop spots (0 = skip)")
    ap.add_argument("--stage", type=int, default=-1)
    ap.add_argument("--bufs", type=int, default=0, help="terminal scan buffers per CTA (0 = half the warps)")
    ap.add_argument("--inst", type=int, default=0, help="spots per CTA in lockstep (0 = library default)")
    ap.add_argument("--sched", type=int, default=0, help="0 = library default, 1 = step-synchronous, 2 = dataflow")
    ap.add_argument("--flow-threads", type=int, default=0, help="dataflow threads per CTA (0 = default/autotuned)")
    ap.add_argument("--spots-per-cta", type=int, default=0, help="dataflow spots per CTA (0 = default/autotuned)")
    ap.add_argument("--node-parts", type=int, default=0, help="dataflow node-op parts (0 = default/autotuned)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)

    import poker_solver_rust_b200 as ps
    from tests import spots

    work = make_workload(args.spots, seed=args.seed + 1000 * rank)
    cc = [spots.card_config(r, b) for r, b, _ in work]
    tcs = [t for _, _, t in work]
    targets = np.array([TARGET_FRAC * t.starting_pot for t in tcs], np.float32)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return rank_max(x, dist, "cuda")

    shape = dict(block_threads=args.block, ctas_per_sm=args.ctas_per_sm, stage_tables=args.stage,
                 scan_buffers=args.bufs, instances_per_cta=args.inst, scheduler=args.sched,
                 flow_threads=args.flow_threads, flow_spots_per_cta=args.spots_per_cta, node_parts=args.node_parts)
    bs = ps.BatchSolver(cc, tcs, **shape)
    for _ in range(args.warmup):
        bs.solve(MAX_ITER, targets)

    # ---- device-resident timing ----
    clk = ClockSampler(local)
    barrier()
    clk.start()
    solve_ms, setup_ms = [], []
    for _ in range(args.steps):
        bs.solve(MAX_ITER, targets)
        a, b = bs.last_timing()
        solve_ms.append(a)
        setup_ms.append(b)
    barrier()
    clocks = clk.stop()
    step_ms = max_over_ranks(sum(solve_ms) / args.steps + sum(setup_ms) / args.steps)
    expl, iters = bs.results()
    value = replicas_throughput(args.spots, world, step_ms)

    # roofline of the persistent solve kernel: algorithmic bytes / kernel time
    sbytes = np.array([bs.iteration_bytes(i) / 20.0 for i in range(args.spots)])
    checks = 1 + np.ceil(iters / 5.0)
    alg_bytes = float(np.sum(iters * 20.0 * sbytes + checks * 4.0 * sbytes))
    kernel_s = statistics.median(solve_ms) / 1e3
    achieved = alg_bytes / kernel_s / 1e9
    peak, peak_kind = _peaks()
    kernel = "k_flow" if bs.config()["scheduler"] == "dataflow" else "k_solve"
    tps = profiled_traffic_per_spot_iteration(kernel)
    traffic = float(tps * np.sum(iters)) if tps else None

    # ---- end to end through the public API (host buffers) ----
    # One batch at a time: build (configs, trees, upload), solve, read back.
    e2e_ms = []
    h2d = d2h = 0
    for k in range(min(args.steps, args.e2e_steps)):
        barrier()
        t0 = time.perf_counter()
        b2 = ps.BatchSolver(cc, tcs, **shape)
        b2.solve(MAX_ITER, targets)
        e2, _ = b2.results()
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        h2d, d2h = b2.io_bytes()
        del b2
    e2e_serial_step = max_over_ranks(statistics.median(e2e_ms)) if e2e_ms else float("nan")
    e2e_serial = replicas_throughput(args.spots, world, e2e_serial_step) if e2e_ms else None
    # A datagen job's steady state: batch k + 1 is built on a host thread
    # while batch k solves (ctypes releases the GIL inside the library).  Every
    # step still builds, uploads, solves and reads back its own batch; the
    # timed region starts before the first build and ends after the last read.
    e2e_value = None
    pipe_detail = None
    n_pipe = args.steps if args.e2e_pipelined else 0
    if n_pipe > 0:
        def pipeline(n: int):
            """n steps of a datagen job: batch k + 1 built on a host thread
            while batch k solves; returns the wall ms and per-step times."""
            build_ms, wait_ms, solve_host_ms = [], [], []
            io = (0, 0)

            def build():
                tb = time.perf_counter()
                b = ps.BatchSolver(cc, tcs, **shape)
                build_ms.append((time.perf_counter() - tb) * 1e3)
                return b

            barrier()
            t0 = time.perf_counter()
            with ThreadPoolExecutor(1) as ex:
                nxt = ex.submit(build)
                for k in range(n):
                    tw = time.perf_counter()
                    b2 = nxt.result()
                    wait_ms.append((time.perf_counter() - tw) * 1e3)
                    if k + 1 < n:
                        nxt = ex.submit(build)
                    ts = time.perf_counter()
                    b2.solve(MAX_ITER, targets)
                    b2.results()
                    solve_host_ms.append((time.perf_counter() - ts) * 1e3)
                    io = b2.io_bytes()
                    del b2
            torch.cuda.synchronize()
            return ((time.perf_counter() - t0) * 1e3, io,
                    {"build_ms": build_ms, "wait_ms": wait_ms, "solve_and_read_ms": solve_host_ms})

        # untimed warm-up: the library's device memory and stream pools grow to
        # two batches in flight (the first overlapped builds wait while they do)
        if args.warmup > 0:
            pipeline(args.warmup)
        wall, (h2d, d2h), pipe_detail = pipeline(n_pipe)
        pipe_step = max_over_ranks(wall / n_pipe)
        e2e_value = replicas_throughput(args.spots, world, pipe_step)
    elif e2e_ms:
        e2e_value = e2e_serial

    # ---- plain per-instance GPU path on a sample (one game, one launch per spot) ----
    plain = None
    if rank == 0 and args.plain_sample > 0:
        sample = work[:args.plain_sample]
        t0 = time.perf_counter()
        for r, b, t in sample:
            g = spots.product_game(r, b, t)
            ps.solve(g, MAX_ITER, TARGET_FRAC * t.starting_pot)
        plain_s = time.perf_counter() - t0
        plain = {"value": len(sample) / plain_s, "unit": UNIT, "sample": f"first {len(sample)} spots, one "
                 "game per spot through the single-game API (one solve launch per spot: on one 16-CTA "
                 "thread-block cluster for these small trees, on every SM for wide ones), host-synchronised"}

    # ---- single turn game (config 2 of the spec), grid mode ----
    turn = None
    if rank == 0 and args.turn_iters > 0:
        turn = turn_game_measure(ps, spots, args.turn_iters, args.turn_cpu_iters)

    # ---- single river game (config 1 of the spec) ----
    river = None
    if rank == 0 and args.river_iters > 0:
        river = river_game_measure(ps, spots, args.river_iters, args.river_cpu_iters)

    # ---- depth-limited turn spots: solve + adjoint, and the datagen loop ----
    adjoint = datagen = None
    if rank == 0 and args.adjoint_spots > 0:
        adjoint = turn_adjoint_measure(ps, spots, args.adjoint_spots, args.adjoint_iters, args.cpu_sample)
    if rank == 0 and args.datagen_spots > 0:
        datagen = turn_datagen_measure(ps, spots, args.datagen_spots, 100, 10)

    # ---- CPU baseline (oracle) on a bounded sample ----
    cpu = None
    if rank == 0 and args.cpu_sample > 0:
        threads = os.cpu_count() or 1
        sample = cpu_sample(work, 0, threads, args.cpu_spots_per_thread)
        dt, cit = oracle_solve_sample(sample, threads)
        cpu = {"value": len(sample) / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"first {len(sample)} spots of the job ({args.cpu_spots_per_thread} per thread), spot-parallel "
                         f"on {threads} threads",
               "mean_iterations": float(cit.mean()),
               "gpu_mean_iterations_same_spots": float(iters[:len(sample)].mean())}

    if rank == 0:
        cfg = bs.config()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG64)",
            "config": {"workload": f"batched river datagen: {args.spots} spots per GPU to <=0.3% pot or "
                                   f"{MAX_ITER} iterations", "parallelism": f"replicas x{world}",
                       "l2": "state (regrets + strategy sums) exceeds L2; no flush needed",
                       "scheduler": cfg["scheduler"], "block_threads": cfg["block_threads"],
                       "ctas_per_sm": cfg["ctas_per_sm"], "grid": cfg["grid"],
                       "scan_buffers": cfg["scan_buffers"], "spots_per_cta": cfg["spots_per_cta"],
                       "node_parts": cfg["node_parts"],
                       "autotune": bs.autotune_trials()},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": n_pipe or len(e2e_ms),
                    "pipelined": bool(n_pipe),
                    "note": ("batch k + 1 built on a host thread while batch k solves; every step builds, "
                             "uploads, solves and reads back its own batch" if n_pipe else
                             "one batch at a time"),
                    "serial_value": e2e_serial, "serial_steps": len(e2e_ms), "pipeline": pipe_detail},
            "gpu_launches": 2 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": kernel, "alg_bytes_per_launch": alg_bytes,
                         "traffic_note": "DRAM bytes per launch, scaled from the 1024-spot ncu capture by "
                                         f"spot-iterations (profiles/{kernel}_river_datagen_1024.md)"},
            "cpu_baseline": cpu,
            "plain_gpu": plain,
            "river_game": river,
            "turn_game": turn,
            "turn_adjoint": adjoint,
            "turn_datagen": datagen,
            "clocks": clocks,
            "detail": {"setup_ms": statistics.median(setup_ms), "solve_ms": statistics.median(solve_ms),
                       "mean_iterations": float(iters.mean()), "max_iterations": int(iters.max()),
                       "solved_fraction": float(np.mean(expl <= targets)),
                       "mean_expl_pct_pot": float(np.mean(expl / np.array([t.starting_pot for t in tcs])) * 100)},
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the batched cloth VBD step on B200.

Workload (default): 4,096 independent cloth instances, grid side n ~ U{16..128} vertices from a seed,
1 m x 1 m each, per-instance Young's modulus log-uniform in [1e3, 1e6] Pa (nu = 0.3, thickness 1e-3 m,
Lame mu = E h / (2 (1 + nu)), lambda = E h nu / (1 - nu^2)), bending stiffness log-uniform in
[1e-5, 1e-3], 1-4 random pinned corners, 0.2 kg/m^2, a ground plane, gravity -9.81, dt = 1/600 s,
10 VBD iterations per substep, FP32, one persistent launch per substep replayed from a CUDA graph.
A "step" is one substep of the whole batch. Inputs are synthetic (seeded); the working set
(~10 GB) is far larger than the 126 MB L2, so no flush is needed between steps.

metric: vertex-iterations/s = sum_i V_i x iterations x substeps / time of the solve (forward step,
all iterations, velocity update). Particle-shape contact generation runs every step before the
solve; it is timed separately and the rate including it is reported as well.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--instances 4096]

--impl reference times the CPU implementation of the same step (the oracle restatement of the
reference's SolverVBD, OpenMP over the vertices of a color, all host threads) on a bounded sample
of the same instances.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "VBD vertex-iters/s on 1 B200, batched FP32 vs plain; pos err <=1e-4 vs FP64"
UNIT = "vertex-iters/s"
ITERATIONS = 10
DT = 1.0 / 600.0


# DRAM bytes (read + write) per vertex-iteration of the solve kernel, from one ncu capture per layout of the
# first 512 instances of this workload; the traffic of a full launch scales with its vertex-iterations.
NCU_TRAFFIC_PER_VI = {
    "ell16": (508.0, "ncu capture of the first 512 instances of this batch, scaled by vertex-iterations"),
}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def instance_params(seed: int, count: int):
    rng = np.random.default_rng(seed)
    sides = rng.integers(16, 129, size=count)
    E = 10.0 ** rng.uniform(3.0, 6.0, size=count)
    bend = 10.0 ** rng.uniform(-5.0, -3.0, size=count)
    pins = [rng.choice(4, size=int(rng.integers(1, 5)), replace=False) for _ in range(count)]
    return sides, E, bend, pins


def build_instance(n, E, bend, pins):
    from newton_chysx_b200 import sim

    nu, h, density = 0.3, 1.0e-3, 0.2
    mu = E * h / (2.0 * (1.0 + nu))
    lam = E * h * nu / (1.0 - nu * nu)
    b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    cell = 1.0 / (n - 1)
    # every instance sits in its own frame, its corner at the origin: worlds do not interact, and far from the
    # origin FP32 positions would round to ~8e-6 m at 96 m (an offset grid of 64 x 64 instances 1.5 m apart)
    b.add_cloth_grid(pos=(0.0, 0.0, 0.6), rot=sim.quat_identity(), vel=(0.0, 0.0, 0.0), dim_x=n - 1,
                     dim_y=n - 1, cell_x=cell, cell_y=cell, mass=density / (n * n), tri_ke=mu, tri_ka=lam, tri_kd=0.0,
                     edge_ke=bend, edge_kd=0.0, particle_radius=5.0e-3)  # fmt: skip
    corners = [0, n - 1, n * (n - 1), n * n - 1]
    flags = b.particle_flags
    for c in pins:
        flags[corners[int(c)]] &= ~1
    b.set_particle_flags(flags)
    b.color(include_bending=True)
    return b


def _instance_from_template(tpl, n, E, bend, pins):
    """A copy of the side-n template builder with this instance's materials and pins.

    Topology, rest poses, areas, rest angles and the coloring depend only on n (materials scale
    the triangle/hinge stiffnesses but never zero them, so the coloring graph is unchanged)."""
    import copy

    nu, h = 0.3, 1.0e-3
    mu = E * h / (2.0 * (1.0 + nu))
    lam = E * h * nu / (1.0 - nu * nu)
    b = copy.copy(tpl)
    mats = tpl.tri_materials.copy()
    mats[:, 0], mats[:, 1] = mu, lam
    b._tri_mat = [mats]
    props = tpl.edge_bending_properties.copy()
    props[:, 0] = bend
    b._edge_prop = [props]
    b._q = [tpl.particle_q.copy()]
    flags = tpl.particle_flags.copy()
    corners = [0, n - 1, n * (n - 1), n * n - 1]
    for c in pins:
        flags[corners[int(c)]] &= ~1
    b._flags = [flags]
    return b


_TEMPLATES: dict[int, object] = {}


def templates(sides):
    """Side-n template builders (E 1e4, bending 1e-4, no pins), built once per side and shared by every
    batch this process builds."""
    for n in np.unique(np.asarray(sides)):
        if int(n) not in _TEMPLATES:
            _TEMPLATES[int(n)] = build_instance(int(n), 1.0e4, 1.0e-4, [])
    return _TEMPLATES


def build_batch_indices(seed: int, count: int, indices):
    """Instances `indices` (increasing) of the count-instance batch of `seed` as the worlds of one builder,
    each with its own materials and pins, and a ground plane."""
    from newton_chysx_b200 import sim

    sides, E, bend, pins = instance_params(seed, count)
    indices = np.asarray(indices, dtype=np.int64)
    tpl = templates(sides[indices])
    top = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    for i in indices:
        n = int(sides[i])
        top.add_world(_instance_from_template(tpl[n], n, float(E[i]), float(bend[i]), pins[i]))
    top.add_ground_plane()
    return top


def build_batch(seed: int, count: int):
    top = build_batch_indices(seed, count, np.arange(count))
    return top, instance_params(seed, count)[0]


def lpt_partition(costs, parts: int):
    """Longest-processing-time-first assignment: instances in decreasing cost, each to the shard with the
    least cost so far (ties to the lower shard). Returns each shard's instance indices in increasing order
    and the shards' total costs."""
    import heapq

    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, r) for r in range(parts)]
    shards: list[list[int]] = [[] for _ in range(parts)]
    load = np.zeros(parts)
    for i in order:
        c, r = heapq.heappop(heap)
        shards[r].append(int(i))
        load[r] = c + costs[i]
        heapq.heappush(heap, (load[r], r))
    return [np.sort(np.asarray(s, dtype=np.int64)) for s in shards], load


def shard_plan(seed: int, per_rank: int, world: int):
    """One global batch of per_rank x world instances, split over the ranks by LPT on V_i x C_i (vertices
    times colors, the persistent kernel's work per instance). Weak scaling: each rank gets about per_rank
    instances' worth of work. With one rank the shard is the whole batch in its original order."""
    total = per_rank * world
    sides = instance_params(seed, total)[0]
    tpl = templates(sides)
    colors = np.array([len(tpl[int(n)]._color_groups) for n in sides], dtype=np.float64)
    shards, load = lpt_partition(sides.astype(np.float64) ** 2 * colors, world)
    return total, shards, load


def run_e2e(args, dev, dist, states, shape, total, shard, vi_all_ranks):
    """End-to-end rate: host-resident state of the rank's shard, per substep H2D of (q, qd), contacts, step and
    D2H of (q, qd), over --e2e-chunks instance groups pipelined on separate streams."""
    import torch

    import newton_chysx_b200 as nb

    C = max(1, args.e2e_chunks)
    bounds = [round(len(shard) * c / C) for c in range(C + 1)]
    hq_all = states[0].particle_q.cpu()
    hqd_all = states[0].particle_qd.cpu()
    chunks, v0 = [], 0
    for c in range(C):
        model = build_batch_indices(args.seed, total, shard[bounds[c]:bounds[c + 1]]).finalize(dev)
        model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e3, 10.0, 0.5
        solver = nb.SolverVBD(model, iterations=ITERATIONS, **shape)
        pipe = nb.CollisionPipeline(model, soft_contact_margin=0.01)
        contacts = pipe.contacts()
        s_in, s_out = model.state(), model.state()
        n = model.particle_count
        hq = hq_all[v0:v0 + n].clone().pin_memory()
        hqd = hqd_all[v0:v0 + n].clone().pin_memory()
        v0 += n
        stream = torch.cuda.Stream(dev)
        stream.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(stream):
            s_in.particle_q.copy_(hq)
            s_in.particle_qd.copy_(hqd)
            pipe.collide(s_in, contacts)
            solver.step(s_in, s_out, None, contacts, DT)  # sizes every buffer before capture
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                pipe.collide(s_in, contacts)
                solver.step(s_in, s_out, None, contacts, DT)
        torch.cuda.current_stream(dev).wait_stream(stream)
        chunks.append(dict(model=model, solver=solver, graph=g, s_in=s_in, s_out=s_out, hq=hq, hqd=hqd,
                           oq=torch.empty_like(hq).pin_memory(), oqd=torch.empty_like(hqd).pin_memory(),
                           stream=stream))  # fmt: skip
    assert v0 == hq_all.shape[0], "the chunks must cover the batch"
    Ke = max(1, args.e2e_steps if args.e2e_steps > 0 else args.steps)  # default: as many substeps as the timed region
    cur = torch.cuda.current_stream(dev)

    def run(k):
        # each group's substeps run in order on its own stream; groups are independent until the final join
        for ch in chunks:
            ch["stream"].wait_stream(cur)
        for _ in range(k):
            for ch in chunks:
                with torch.cuda.stream(ch["stream"]):
                    ch["s_in"].particle_q.copy_(ch["hq"], non_blocking=True)
                    ch["s_in"].particle_qd.copy_(ch["hqd"], non_blocking=True)
                    ch["graph"].replay()
                    ch["oq"].copy_(ch["s_out"].particle_q, non_blocking=True)
                    ch["oqd"].copy_(ch["s_out"].particle_qd, non_blocking=True)
        for ch in chunks:
            cur.wait_stream(ch["stream"])

    run(1)  # warm-up
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run(Ke)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks([e0.elapsed_time(e1)], device=dev)[0]
    h2d = sum(2 * ch["hq"].numel() * 4 for ch in chunks)
    d2h = sum(2 * ch["oq"].numel() * 4 for ch in chunks)
    for ch in chunks:
        ch["graph"] = None
    return {"value": vi_all_ranks * Ke / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "steps": Ke, "chunks": C, "ms_per_step": ms / Ke}  # fmt: skip


def max_over_ranks(values, device=None):
    """Element-wise max of per-rank timings (the multi-GPU time is the slowest rank's)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def bytes_per_vertex_iteration(V, T, E, contacts=True):
    """Algorithmic bytes of one colour sweep (92 V + 68 T + 64 E + 96 V with contacts) per vertex."""
    return (92.0 * V + 68.0 * T + 64.0 * E + (96.0 * V if contacts else 0.0)) / V


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        import tempfile

        self.path = os.path.join(tempfile.gettempdir(), f"vbd_clocks_{os.getpid()}_{index}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)  # fmt: skip
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
            os.remove(self.path)
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if len(r) >= 9]
        smax = [float(r[2]) for r in rows if len(r) >= 9]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(sm)}  # fmt: skip


def run_ours(args):
    import torch

    import newton_chysx_b200 as nb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    t0 = time.time()
    total, shards, load = shard_plan(args.seed, args.instances, world)
    shard = shards[rank]
    sides_all = instance_params(args.seed, total)[0]
    if args.tune:
        # launch shape from the autotuner, timed on the shard's first instances (same size distribution)
        from newton_chysx_b200 import autotune

        sub_model = build_batch_indices(args.seed, total, shard[: args.tune_instances]).finalize(dev)
        sub_model.soft_contact_ke, sub_model.soft_contact_kd, sub_model.soft_contact_mu = 1.0e3, 10.0, 0.5
        shape = autotune.tune(sub_model, schedule="persistent", iterations=ITERATIONS, dt=DT)
        del sub_model
    else:
        shape = dict(schedule="persistent", lanes_per_vertex=args.lanes, block_size=args.block,
                     positions_in_shared=args.shared, layout=args.layout, min_blocks_per_sm=args.occ,
                     pair_vertices=args.pair)  # fmt: skip
    tune_s = time.time() - t0
    model = build_batch_indices(args.seed, total, shard).finalize(dev)
    model.soft_contact_ke, model.soft_contact_kd, model.soft_contact_mu = 1.0e3, 10.0, 0.5
    solver = nb.SolverVBD(model, iterations=ITERATIONS, **shape)
    pipe = nb.CollisionPipeline(model, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    setup_s = time.time() - t0
    V, T, E = model.particle_count, model.tri_count, model.edge_count
    assert V == int(np.sum(sides_all[shard].astype(np.int64) ** 2)), "the model must hold the shard's instances"
    vi_all_ranks = float(np.sum(sides_all.astype(np.float64) ** 2)) * ITERATIONS  # every rank's vertices
    states = [model.state(), model.state()]

    # settle the batch for a few substeps so that contacts and motion are present, then capture; substep n reads
    # states[n % 2] and writes states[(n + 1) % 2] through every phase, so the batch follows one trajectory
    nsub = 0
    for _ in range(max(args.warmup, 3)):
        pipe.collide(states[nsub % 2], contacts)
        solver.step(states[nsub % 2], states[(nsub + 1) % 2], None, contacts, DT)
        nsub += 1
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    g_collide = [torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()]
    g_solve = [torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()]
    with torch.cuda.stream(stream):
        for p in range(2):
            with torch.cuda.graph(g_collide[p], stream=stream):
                pipe.collide(states[p], contacts)
            with torch.cuda.graph(g_solve[p], stream=stream):
                solver.step(states[p], states[1 - p], None, contacts, DT)
    torch.cuda.current_stream(dev).wait_stream(stream)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        g_collide[nsub % 2].replay()
        g_solve[nsub % 2].replay()
        nsub += 1
    torch.cuda.synchronize()

    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = nsub
    with ClockSampler(dev.index) as clocks:
        ev0.record()
        for k in range(K):
            g_collide[(n0 + k) % 2].replay()
            ev[k][0].record()
            g_solve[(n0 + k) % 2].replay()
            ev[k][1].record()
        ev1.record()
        torch.cuda.synchronize()
    nsub += K
    solve_ms = sum(a.elapsed_time(b) for a, b in ev)
    total_ms = ev0.elapsed_time(ev1)
    solve_ms, total_ms = max_over_ranks([solve_ms, total_ms], device=dev)
    errors = solver.device_errors()

    vi_step = float(V) * ITERATIONS
    value = vi_all_ranks * K / (solve_ms * 1e-3)
    value_with_contacts = vi_all_ranks * K / (total_ms * 1e-3)
    peak, peak_src = _peaks()
    bvi = bytes_per_vertex_iteration(V, T, E, contacts=True)
    achieved = bvi * vi_step / (solve_ms / K * 1e-3) / 1e9

    # position error of the timed FP32 batch against FP64 on a sample of its instances (rank 0's shard)
    pos = None
    if rank == 0 and not args.no_pos_err:
        pos = position_error(args, dev, total, shard, model, states, nsub, g_collide, g_solve, shape)

    # end to end through the public API with host buffers: every substep, pinned H2D of the inputs (q, qd),
    # contact generation, the step and D2H of the result (q, qd). The batch is split into --e2e-chunks groups of
    # instances, each its own Model and SolverVBD on its own CUDA stream, so that the copies of one group overlap
    # the solve of another (the copy engines and the SMs work at the same time).
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, dev, dist, states, shape, total, shard, vi_all_ranks)
    # the plain drop-in on the same GPU: one SolverVBD per cloth, eager per-instance step calls
    plain = None
    if rank == 0 and args.plain_sample > 0:
        plain = run_plain(args, total, shard[: args.plain_sample])
    traffic, traffic_src = args.traffic, "--traffic (ncu capture)" if args.traffic is not None else None
    if traffic is None and solver.layout in NCU_TRAFFIC_PER_VI:
        per_vi, traffic_src = NCU_TRAFFIC_PER_VI[solver.layout]
        traffic = per_vi * vi_step
    out = None
    if rank == 0:
        out = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": K,
            "warmup": args.warmup,
            "ms_per_step": solve_ms / K,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded cloth grids, random-init materials)",
            "config": {
                "workload": f"batched cloth VBD, {args.instances} instances/GPU, side U{{16..128}}, ground contact",
                "instances_per_gpu": args.instances,
                "instances_total": total,
                "instances_rank0": len(shard),
                "shard_cost_spread": float(load.max() / load.min()) if world > 1 else 1.0,
                "vertices_per_gpu": V,
                "triangles_per_gpu": T,
                "hinges_per_gpu": E,
                "iterations": ITERATIONS,
                "dt": DT,
                "schedule": solver.schedule,
                "lanes_per_vertex": solver.lanes_per_vertex,
                "block_size": solver.block_size,
                "positions_in_shared_bytes": solver.shared_bytes,
                "layout": solver.layout,
                "launch_shape": shape,
                "autotuned": bool(args.tune),
                "tune_s": round(tune_s, 1),
                "l2": "inputs larger than L2 (~10 GB working set), no flush",
                "parallelism": f"instance sharding x{world}, LPT on vertices x colors (no collective)",
                "timed": "solve only (forward, iterations, velocity); contact generation outside the solve events",
                "setup_s": round(setup_s, 1),
            },
            "value_with_contact_generation": value_with_contacts,
            "ms_per_step_with_contact_generation": total_ms / K,
            "e2e": e2e,
            "gpu_launches": K * (1 + solver.launches_per_step),
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": traffic,
                "traffic_source": traffic_src,
                "peak_source": peak_src,
                "bytes_per_vertex_iteration": bvi,
                "kernel": "k_persistent (per-substep solve)",
            },
            "clocks": clocks.summary(),
            "device_errors": errors,
        }
        if pos is not None:
            out["pos_err"] = pos["value"]
            out["pos_err_detail"] = pos
        if plain is not None:
            out["plain"] = plain
            out["batched_over_plain"] = (value / world) / plain["value"]
        if not args.no_cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline(args, seconds=args.cpu_seconds)
    if dist:
        g_collide.clear()
        g_solve.clear()
        dist.barrier()
        dist.destroy_process_group()
    return out


def cpu_baseline(args, seconds=15.0):
    """The oracle (CPU restatement of the reference SolverVBD step) on a bounded sample of the batch."""
    from oracle import vbd_oracle as orc
    from tests.helpers import oracle_model_dict

    sides, E, bend, pins = instance_params(args.seed, args.instances)
    threads = orc.max_threads()
    done_vi = 0
    elapsed = 0.0
    used = 0
    for i in range(args.instances):
        b = build_instance(int(sides[i]), float(E[i]), float(bend[i]), pins[i])
        b.add_ground_plane()
        m = b.finalize("cpu")
        om = orc.Model(oracle_model_dict(m))
        q = m.particle_q.numpy().astype(np.float64)
        qd = np.zeros_like(q)
        t = time.perf_counter()
        cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(q, m.particle_radius.numpy(), m.particle_flags.numpy(),
                                                         m.shape_type, m.shape_transform, m.shape_scale, 0.01)  # fmt: skip
        contacts = orc.make_contacts(cnt, p, s, bp, bv, nn)
        orc.step(om, q, qd, None, contacts, DT, ITERATIONS, precision=32, nthreads=threads)
        elapsed += time.perf_counter() - t
        done_vi += m.particle_count * ITERATIONS
        used += 1
        if elapsed >= seconds:
            break
    return {"value": done_vi / elapsed, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {used} of {args.instances} instances, one substep each ({done_vi} vertex-iterations)"}  # fmt: skip


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from oracle import vbd_oracle as orc

    orc.lib()
    K, W = args.steps, args.warmup
    per_step = max(2.0, args.cpu_seconds / max(K, 1))
    for _ in range(min(W, 1)):
        cpu_baseline(args, seconds=0.5)
    vals = []
    t0 = time.perf_counter()
    for _ in range(K):
        vals.append(cpu_baseline(args, seconds=per_step))
    wall = time.perf_counter() - t0
    v = statistics.mean(x["value"] for x in vals)
    cb = dict(vals[-1])
    cb["value"] = v
    return {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": K,
        "warmup": W, "ms_per_step": wall * 1e3 / max(K, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded cloth grids, random-init materials)",
        "config": {"workload": f"batched cloth VBD, {args.instances} instances/GPU, side U{{16..128}}, ground contact",
                   "iterations": ITERATIONS, "dt": DT, "sample_per_step_s": per_step},
        "impl": "reference", "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }  # fmt: skip


def run_plain(args, total=None, indices=None):
    """The plain drop-in used per instance: one SolverVBD per cloth, one step call per instance per
    substep (per-color launches), on a sample of the batch; the rate is per vertex-iteration."""
    import torch

    import newton_chysx_b200 as nb

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    total = args.instances if total is None else total
    sides, E, bend, pins = instance_params(args.seed, total)
    idx = np.arange(min(args.plain_sample, total)) if indices is None else np.asarray(indices)
    t0 = time.time()
    items = []
    for i in idx:
        b = build_instance(int(sides[i]), float(E[i]), float(bend[i]), pins[i])
        b.add_ground_plane()
        m = b.finalize(dev)
        m.soft_contact_ke, m.soft_contact_kd, m.soft_contact_mu = 1.0e3, 10.0, 0.5
        solver = nb.SolverVBD(m, iterations=ITERATIONS, schedule="per_color", lanes_per_vertex=args.lanes or 4)
        pipe = nb.CollisionPipeline(m, soft_contact_margin=0.01)
        items.append((m, solver, pipe, pipe.contacts(), [m.state(), m.state()]))
    setup_s = time.time() - t0
    V = sum(m.particle_count for m, *_ in items)

    def substep(k):
        for m, solver, pipe, c, st in items:
            pipe.collide(st[k % 2], c)
            solver.step(st[k % 2], st[(k + 1) % 2], None, c, DT)

    W = max(args.warmup, 3)
    for k in range(W):
        substep(k)
    torch.cuda.synchronize()
    K = max(1, min(args.steps, args.plain_steps))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(W, W + K):
        substep(k)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"workload": "plain per-instance drop-in", "value": V * ITERATIONS * K / (ms * 1e-3), "unit": UNIT,
            "instances": len(items), "vertices": V, "steps": K, "ms_per_step": ms / K,
            "launches_per_instance_step": items[0][1].launches_per_step + 1, "setup_s": round(setup_s, 1),
            "note": "first instances of the batch, each its own Model and SolverVBD (per-color schedule); every substep "
                    "one eager collide + step call per instance from Python, no CUDA graph; contact generation "
                    "inside the timed region"}  # fmt: skip


def error_sample(sides, E, pool, count):
    """A sample of `count` instances of `pool` that holds the largest and the smallest side and both ends of
    Young's modulus, filled with instances spread evenly through the pool."""
    pool = np.asarray(pool)
    picks = [pool[np.argmax(sides[pool])], pool[np.argmin(sides[pool])], pool[np.argmin(E[pool])],
             pool[np.argmax(E[pool])]]  # fmt: skip
    seen = {int(p) for p in picks}
    for j in np.linspace(0, len(pool) - 1, max(count, 1)).round().astype(int):
        if len(seen) >= count:
            break
        seen.add(int(pool[j]))
    return np.array(sorted(seen), dtype=np.int64)


def position_error(args, dev, total, shard, model, states, nsub, g_collide, g_solve, shape):
    """Position error of the FP32 batch against FP64, on a sample of the shard's instances (error_sample),
    as max over vertices of |x_fp32 - x_fp64|_2 / L, with L = 1 m the cloth side.

    * per substep: after the timed region, each of --err-substeps more substeps of the whole batch (the
      benchmark's graphs) runs beside the FP64 solver (precision="fp64", the same step in double precision)
      stepping the sample from the same FP32 input state with contacts generated from the same positions;
    * trajectory: the sample alone, from the initial state, for as many substeps as the batch ran before its
      timed region ended, once in FP32 with the benchmark's launch shape and once in FP64."""
    import torch

    import newton_chysx_b200 as nb

    t0 = time.time()
    sides, E, _, _ = instance_params(args.seed, total)
    sample = error_sample(sides, E, shard, args.err_sample)
    local = np.searchsorted(shard, sample)  # world index in the rank's model
    ws = model.world_particle_start if model.world_particle_start is not None else np.array([0, model.particle_count])
    sel = torch.cat([torch.arange(int(ws[w]), int(ws[w + 1]), device=dev) for w in local])
    sm = build_batch_indices(args.seed, total, sample).finalize(dev)
    sm.soft_contact_ke, sm.soft_contact_kd, sm.soft_contact_mu = 1.0e3, 10.0, 0.5
    assert sm.particle_count == sel.numel()

    def f64_states():
        out = [sm.state(), sm.state()]
        for s in out:
            s.particle_q, s.particle_qd, s.particle_f = (t.double() for t in (s.particle_q, s.particle_qd, s.particle_f))
        return out

    def f32_view(s):
        v = type(s)()
        v.particle_q = s.particle_q.float()
        return v

    def err(a, b):
        return float(torch.linalg.norm(a.double() - b.double(), dim=1).max())

    s64 = nb.SolverVBD(sm, iterations=ITERATIONS, schedule="persistent", precision="fp64")
    pipe = nb.CollisionPipeline(sm, soft_contact_margin=0.01)
    c64 = pipe.contacts()
    a64, b64 = f64_states()
    per_substep = []
    for _ in range(args.err_substeps):
        src, dst = states[nsub % 2], states[(nsub + 1) % 2]
        a64.particle_q.copy_(src.particle_q[sel].double())
        a64.particle_qd.copy_(src.particle_qd[sel].double())
        pipe.collide(f32_view(a64), c64)
        s64.step(a64, b64, None, c64, DT)
        g_collide[nsub % 2].replay()
        g_solve[nsub % 2].replay()
        nsub += 1
        torch.cuda.synchronize()
        per_substep.append(err(dst.particle_q[sel], b64.particle_q))

    s32 = nb.SolverVBD(sm, iterations=ITERATIONS, **shape)
    c32 = pipe.contacts()
    t32 = [sm.state(), sm.state()]
    t64 = f64_states()
    n_traj = max(args.warmup, 3) + args.warmup + args.steps
    traj = []
    for k in range(n_traj):
        pipe.collide(t32[k % 2], c32)
        s32.step(t32[k % 2], t32[(k + 1) % 2], None, c32, DT)
        pipe.collide(f32_view(t64[k % 2]), c64)
        s64.step(t64[k % 2], t64[(k + 1) % 2], None, c64, DT)
        traj.append(err(t32[(k + 1) % 2].particle_q, t64[(k + 1) % 2].particle_q))
    torch.cuda.synchronize()
    worst = max(max(per_substep, default=0.0), max(traj, default=0.0))
    return {"value": worst, "unit": "m per m of cloth side (max vertex |x32 - x64|_2 / L, L = 1 m)",
            "bound": 1e-4, "within_bound": bool(worst <= 1e-4), "per_substep": per_substep,
            "per_substep_after_substep": nsub - len(per_substep), "trajectory_max": max(traj, default=0.0),
            "trajectory_substeps": n_traj, "fp32_layout": s32.layout,
            "reference": "precision='fp64' (the same step in FP64, held to the FP64 oracle at 1e-9 m by the tests)",
            "instances": [int(i) for i in sample], "sides": [int(sides[i]) for i in sample],
            "E_range": [float(E[sample].min()), float(E[sample].max())], "s": round(time.time() - t0, 1)}  # fmt: skip


SC_ITERATIONS = 20


def build_selfcontact_model(dev, n=256):
    """Plain drop-in at scale: an n x n sheet (1 m side, E = 1e4 Pa, nu = 0.3, h = 1e-3 m, 0.2 kg/m^2,
    bending 1e-4) flat at z = 0.5 m above a fixed sphere of radius 0.3 m at the origin."""
    import newton_chysx_b200 as nb

    E, nu, h = 1.0e4, 0.3, 1.0e-3
    b = nb.ModelBuilder(up_axis="Z", gravity=-9.81)
    b.add_cloth_grid(pos=(-0.5, -0.5, 0.5), rot=nb.quat_identity(), vel=(0.0, 0.0, 0.0), dim_x=n - 1, dim_y=n - 1,
                     cell_x=1.0 / (n - 1), cell_y=1.0 / (n - 1), mass=0.2 / (n * n), tri_ke=E * h / (2.0 * (1.0 + nu)),
                     tri_ka=E * h * nu / (1.0 - nu * nu), tri_kd=0.0, edge_ke=1e-4, edge_kd=0.0,
                     particle_radius=2e-3)  # fmt: skip
    b.add_shape_sphere(radius=0.3)
    b.color(include_bending=True)
    m = b.finalize(dev)
    m.soft_contact_ke, m.soft_contact_kd, m.soft_contact_mu = 1.0e4, 1.0e-2, 0.5
    return m


SC_KW = dict(particle_enable_self_contact=True, particle_self_contact_radius=2e-3, particle_self_contact_margin=3.5e-3,
             particle_collision_detection_interval=0, particle_topological_contact_filter_threshold=2)  # fmt: skip


def time_selfcontact_substeps(solver, pipe, contacts, s0, s1, q_settled, qd_settled, K):
    """ms per substep (collision generation + step) from the settled state, K substeps replayed from a CUDA graph
    of two substeps (a ping-pong pair), timed with CUDA events."""
    import torch

    s0.particle_q.copy_(q_settled)
    s0.particle_qd.copy_(qd_settled)
    pipe.collide(s0, contacts)  # one eager substep first: a solver sizes its contact buffers outside the capture
    solver.step(s0, s1, None, contacts, DT)
    graph = torch.cuda.CUDAGraph()
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream), torch.cuda.graph(graph, stream=stream):
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        pipe.collide(s1, contacts)
        solver.step(s1, s0, None, contacts, DT)
    torch.cuda.current_stream().wait_stream(stream)
    s0.particle_q.copy_(q_settled)
    s0.particle_qd.copy_(qd_settled)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(K // 2):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    del graph
    return e0.elapsed_time(e1) / K


def run_selfcontact(args):
    """Config of the plain drop-in at scale: one 256 x 256 cloth (65,536 vertices, 130,050 triangles)
    dropped onto a sphere with vertex-triangle and edge-edge self-contact, 20 iterations per substep,
    dt = 1/600 s. The sheet first falls and drapes untimed (--sc-settle-frames x 10 substeps); then K
    substeps (collision generation + step) are timed, replayed from a CUDA graph of one substep."""
    import torch

    import newton_chysx_b200 as nb

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    m = build_selfcontact_model(dev, args.sc_n)
    solver = nb.SolverVBD(m, iterations=SC_ITERATIONS, lanes_per_vertex=args.lanes, **SC_KW)
    pipe = nb.CollisionPipeline(m, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    s0, s1 = m.state(), m.state()
    t0 = time.perf_counter()
    settle = args.sc_settle_frames * 10 + args.warmup
    for k in range(settle):
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    settle_s = time.perf_counter() - t0
    q_settled, qd_settled = s0.particle_q.clone(), s0.particle_qd.clone()
    K = max(2, args.steps + (args.steps % 2))
    with ClockSampler(dev.index or 0) as clk:
        ms = time_selfcontact_substeps(solver, pipe, contacts, s0, s1, q_settled, qd_settled, K)
    pairs = solver.self_contact_counts()
    V = m.particle_count
    value = V * SC_ITERATIONS / (ms * 1e-3)
    out = {
        "metric": "VBD vertex-iters/s on 1 B200, plain drop-in with self-contact", "value": value, "unit": UNIT,
        "n_gpus": 1, "steps": K, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (cloth grid dropped on a sphere)",
        "config": {"workload": f"plain drop-in at scale: {args.sc_n}x{args.sc_n} cloth on a sphere, self-contact",
                   "vertices": V, "triangles": m.tri_count, "edges": m.edge_count, "iterations": SC_ITERATIONS,
                   "dt": DT, "self_contact": {k: v for k, v in SC_KW.items() if k != "particle_enable_self_contact"},
                   "settled_substeps": settle, "settle_s": round(settle_s, 2),
                   "timed": "sphere contact generation + step, one CUDA graph per two substeps",
                   "l2": "working set below L2; the step is launch- and latency-bound, see launches_per_step"},
        "launches_per_step": solver.launches_per_step + 1, "colors": len(m.particle_color_groups),
        "lanes_per_vertex": solver.lanes_per_vertex,
        "self_contact_pairs": {"vertex_triangle": pairs[0], "edge_edge": pairs[1], "overflow_flags": pairs[2]},
        "clocks": clk.summary(), "device_errors": solver.device_errors(),
        "finite": bool(torch.isfinite(s0.particle_q).all().item()),
    }  # fmt: skip
    if not args.no_e2e:  # public API with host state: H2D of (q, qd), step, D2H of q
        hq = q_settled.cpu().pin_memory()
        hqd = qd_settled.cpu().pin_memory()
        out_q = torch.empty_like(hq).pin_memory()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(K):
            s0.particle_q.copy_(hq, non_blocking=True)
            s0.particle_qd.copy_(hqd, non_blocking=True)
            pipe.collide(s0, contacts)
            solver.step(s0, s1, None, contacts, DT)
            out_q.copy_(s1.particle_q, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        ms_e = e0.elapsed_time(e1) / K
        out["e2e"] = {"value": V * SC_ITERATIONS / (ms_e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 2 * hq.numel() * 4,
                      "d2h_bytes_per_step": out_q.numel() * 4, "steps": K}  # fmt: skip
    # the mixed mode (FP64 contact terms and block solve on contact vertices) timed the same way
    mixed = nb.SolverVBD(m, iterations=SC_ITERATIONS, precision="mixed", lanes_per_vertex=args.lanes, **SC_KW)
    ms_mixed = time_selfcontact_substeps(mixed, pipe, contacts, s0, s1, q_settled, qd_settled, K)
    out["mixed"] = {"value": V * SC_ITERATIONS / (ms_mixed * 1e-3), "unit": UNIT, "ms_per_step": ms_mixed,
                    "device_errors": mixed.device_errors()}  # fmt: skip
    if not args.no_pos_err:
        out["pos_err"], out["pos_err_detail"] = selfcontact_position_error(args, m, solver, mixed, pipe, q_settled,
                                                                           qd_settled)  # fmt: skip
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_selfcontact(m, q_settled.cpu().numpy(), qd_settled.cpu().numpy())
        if not args.no_pos_err:
            ora = out["cpu_baseline"].pop("fp64_step_q")
            q32 = out["pos_err_detail"].pop("first_fp32_q")
            d = float(np.linalg.norm(q32 - ora, axis=1).max())
            out["pos_err_detail"]["vs_fp64_oracle_first_substep"] = d
            out["pos_err"] = max(out["pos_err"], d)
            out["pos_err_detail"]["within_bound"] = bool(out["pos_err"] <= 1e-4)
    if "pos_err_detail" in out:
        out["pos_err_detail"].pop("first_fp32_q", None)
    return out


def selfcontact_position_error(args, m, solver, mixed, pipe, q_settled, qd_settled):
    """Position error against FP64 on the settled, draped sheet with self-contact, as max over vertices of
    |x - x_fp64|_2 / L (L = 1 m), with the number of vertices past 1e-4 m:
    * per substep: each of --err-substeps FP32 substeps (collide + step, the timed calls) beside an FP64 substep
      (precision="fp64", the same step in double precision) from the same FP32 input with contacts from the same
      positions, and the mixed mode's substep from that input;
    * trajectory: FP32 and FP64 from the settled state for the same substeps;
    * floor: the FP64 step from the first input moved by Gaussian noise of 1e-8 m (below FP32 rounding of the
      positions) against the FP64 step from that input. The step is discontinuous where a contact's normal
      velocity is near zero: the damping stiffness kd ke / dt switches on and off with its sign, so any two
      arithmetics part by this much there."""
    import torch

    import newton_chysx_b200 as nb

    t0 = time.time()
    s64 = nb.SolverVBD(m, iterations=SC_ITERATIONS, precision="fp64", lanes_per_vertex=args.lanes, **SC_KW)
    c32, c64 = pipe.contacts(), pipe.contacts()
    a32, b32, bmx = m.state(), m.state(), m.state()
    a64, b64, t64a, t64b = m.state(), m.state(), m.state(), m.state()
    for s in (a64, b64, t64a, t64b):
        s.particle_q, s.particle_qd, s.particle_f = (t.double() for t in (s.particle_q, s.particle_qd, s.particle_f))
    a32.particle_q.copy_(q_settled)
    a32.particle_qd.copy_(qd_settled)
    t64a.particle_q.copy_(q_settled.double())
    t64a.particle_qd.copy_(qd_settled.double())

    def f32_view(s):
        v = type(s)()
        v.particle_q = s.particle_q.float()
        return v

    def dist(a, b):
        return torch.linalg.norm(a.double() - b.double(), dim=1)

    def stat(d):
        return {"max": float(d.max()), "above_1e-4": int((d > 1e-4).sum()), "above_1e-5": int((d > 1e-5).sum())}

    per32, permx, traj, first, first_stats = [], [], [], None, {}
    amx = m.state()
    for k in range(max(1, args.err_substeps)):
        # a step writes its result into its input state too (the reference's side effect): every solver starts
        # from its own copy of the input
        qin, qdin = a32.particle_q.clone(), a32.particle_qd.clone()
        pipe.collide(a32, c32)
        amx.particle_q.copy_(qin)
        amx.particle_qd.copy_(qdin)
        mixed.step(amx, bmx, None, c32, DT)
        solver.step(a32, b32, None, c32, DT)
        a64.particle_q.copy_(qin.double())
        a64.particle_qd.copy_(qdin.double())
        pipe.collide(f32_view(a64), c64)
        s64.step(a64, b64, None, c64, DT)
        pipe.collide(f32_view(t64a), c64)
        s64.step(t64a, t64b, None, c64, DT)
        torch.cuda.synchronize()
        d32, dmx = dist(b32.particle_q, b64.particle_q), dist(bmx.particle_q, b64.particle_q)
        if first is None:
            first = b32.particle_q.cpu().numpy().astype(np.float64)
            first_stats = {"fp32": stat(d32), "mixed": stat(dmx)}
            gen = torch.Generator(device=qin.device).manual_seed(7)
            fl = (m.particle_flags & 1).bool()
            noise = torch.randn(qin.shape, generator=gen, device=qin.device, dtype=torch.float64)
            p64, q64 = m.state(), m.state()
            for s in (p64, q64):
                s.particle_q, s.particle_qd, s.particle_f = (t.double() for t in (s.particle_q, s.particle_qd,
                                                                                  s.particle_f))  # fmt: skip
            p64.particle_q.copy_(qin.double() + 1e-8 * noise * fl[:, None])
            p64.particle_qd.copy_(qdin.double())
            s64.step(p64, q64, None, c64, DT)  # contacts of the unperturbed FP32 positions
            torch.cuda.synchronize()
            first_stats["fp64_floor"] = stat(dist(q64.particle_q, b64.particle_q))
        per32.append(float(d32.max()))
        permx.append(float(dmx.max()))
        traj.append(float(dist(b32.particle_q, t64b.particle_q).max()))
        a32, b32 = b32, a32
        t64a, t64b = t64b, t64a
    worst = max(per32)
    counts = s64.self_contact_counts()
    return worst, {"value": worst, "unit": "m per m of cloth side (max vertex |x32 - x64|_2 / L, L = 1 m)",
                   "bound": 1e-4, "within_bound": bool(worst <= 1e-4), "per_substep": per32,
                   "per_substep_mixed": permx, "first_substep": first_stats, "trajectory": traj,
                   "after_settled_substeps": args.sc_settle_frames * 10 + args.warmup,
                   "fp64_self_contact_pairs": {"vertex_triangle": counts[0], "edge_edge": counts[1]},
                   "reference": "precision='fp64' (the same step in FP64, held to the FP64 oracle at 1e-9 m by the "
                                "tests); with the CPU baseline on, also the FP64 oracle's own substep from the "
                                "settled state",
                   "first_fp32_q": first, "s": round(time.time() - t0, 1)}  # fmt: skip


def cpu_baseline_selfcontact(m, q, qd, fp64_step=True):
    """The oracle (FP32, all host threads, box-grid detection) on one substep of the same settled state; with
    fp64_step, also the FP64 oracle's substep from that state (untimed), returned as fp64_step_q."""
    from newton_chysx_b200.collision import build_contact_filters
    from oracle import vbd_oracle as orc
    from tests.helpers import oracle_model_dict

    threads = orc.max_threads()
    om = orc.Model(oracle_model_dict(m))
    vt, ee = build_contact_filters(m.particle_count, m.tri_indices, m.edge_indices, 2)
    sc = orc.SelfContact(m.particle_q.cpu().numpy().astype(np.float64), radius=SC_KW["particle_self_contact_radius"],
                         margin=SC_KW["particle_self_contact_margin"], vt_filter=vt, ee_filter=ee)  # fmt: skip
    q = q.astype(np.float64)
    t = time.perf_counter()
    cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(q, m.particle_radius.cpu().numpy(),
                                                     m.particle_flags.cpu().numpy(), m.shape_type, m.shape_transform,
                                                     m.shape_scale, 0.01)  # fmt: skip
    contacts = orc.make_contacts(cnt, p, s, bp, bv, nn)
    orc.step(om, q, qd.astype(np.float64), None, contacts, DT, SC_ITERATIONS, precision=32, nthreads=threads,
             self_contact=sc)  # fmt: skip
    el = time.perf_counter() - t
    out = {"value": m.particle_count * SC_ITERATIONS / el, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": "one substep of the same settled 256x256 state (self-contact detection on a box grid)"}  # fmt: skip
    if fp64_step:
        _, q64, _ = orc.step(om, q, qd.astype(np.float64), None, contacts, DT, SC_ITERATIONS, precision=64,
                             nthreads=threads, self_contact=sc)  # fmt: skip
        out["fp64_step_q"] = q64
    return out


def build_selfcontact_batch_model(dev, worlds, n=32, seed=9):
    """Batched self-contact: `worlds` copies of an n x n sheet (0.25 m side, the drop-in material, 0.2 kg/m^2,
    bending 1e-4) each over its own sphere of radius 0.06 m, dropped from a seeded height with a seeded sideways
    velocity so that each sheet drapes and folds onto itself differently. The worlds sit 0.5 m apart on a square
    grid: co-located worlds would share every cell of the collision grid (and on the per-color schedule, which
    lets worlds collide as the reference's union model does, interpenetrate)."""
    import torch

    import newton_chysx_b200 as nb

    E, nu, h, side = 1.0e4, 0.3, 1.0e-3, 0.25
    tpl = nb.ModelBuilder(up_axis="Z", gravity=-9.81)
    tpl.add_cloth_grid(pos=(-side / 2, -side / 2, 0.1), rot=nb.quat_identity(), vel=(0.0, 0.0, 0.0), dim_x=n - 1,
                       dim_y=n - 1, cell_x=side / (n - 1), cell_y=side / (n - 1), mass=0.2 * side * side / (n * n),
                       tri_ke=E * h / (2.0 * (1.0 + nu)), tri_ka=E * h * nu / (1.0 - nu * nu), tri_kd=0.0,
                       edge_ke=1e-4, edge_kd=0.0, particle_radius=2e-3)  # fmt: skip
    tpl.add_shape_sphere(radius=0.06)
    tpl.color(include_bending=True)
    b = nb.ModelBuilder(up_axis="Z", gravity=-9.81)
    for _ in range(worlds):
        b.add_world(tpl)
    m = b.finalize(dev)
    rng = np.random.default_rng(seed)
    n1 = tpl.particle_count
    k = int(math.ceil(math.sqrt(worlds)))
    off = np.stack([np.arange(worlds) % k * 0.5, np.arange(worlds) // k * 0.5, rng.uniform(0.0, 0.05, worlds)], 1)
    with torch.no_grad():
        m.particle_q += torch.as_tensor(np.repeat(off, n1, axis=0), dtype=torch.float32, device=dev)
        m.particle_qd[:, 0] = torch.as_tensor(np.repeat(rng.normal(0.0, 0.3, worlds), n1), dtype=torch.float32,
                                              device=dev)  # fmt: skip
    m.shape_transform[:, :2] += off[:, :2].astype(np.float32)  # each world's sphere under its sheet
    m.soft_contact_ke, m.soft_contact_kd, m.soft_contact_mu = 1.0e4, 1.0e-2, 0.5
    return m


def run_selfcontact_batch(args):
    """Self-contact on a batched model: --instances sheets (--sc-batch-n vertices a side, each over its own sphere)
    with vertex-triangle and edge-edge self-contact, 20 iterations, dt = 1/600 s. The sheets fall and drape untimed
    (--sc-settle-frames x 10 substeps); then K substeps (contact generation + step) are timed from a CUDA graph
    on the persistent self-contact schedule (one CTA per world, detections grid-wide) and on the per-color
    schedule, from the same settled state."""
    import torch

    import newton_chysx_b200 as nb

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    W = args.instances
    t0 = time.perf_counter()
    m = build_selfcontact_batch_model(dev, W, n=args.sc_batch_n)
    build_s = time.perf_counter() - t0
    kw = dict(SC_KW, lanes_per_vertex=args.lanes)
    solver = nb.SolverVBD(m, iterations=SC_ITERATIONS, **kw)
    assert solver.schedule == "persistent"
    pipe = nb.CollisionPipeline(m, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    s0, s1 = m.state(), m.state()
    settle = args.sc_settle_frames * 10 + args.warmup
    for _ in range(settle):
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    q_settled, qd_settled = s0.particle_q.clone(), s0.particle_qd.clone()
    K = max(2, args.steps + (args.steps % 2))
    with ClockSampler(dev.index or 0) as clk:
        ms = time_selfcontact_substeps(solver, pipe, contacts, s0, s1, q_settled, qd_settled, K)
    pairs = solver.self_contact_counts()
    per_color = nb.SolverVBD(m, iterations=SC_ITERATIONS, schedule="per_color", **kw)
    ms_pc = time_selfcontact_substeps(per_color, pipe, contacts, s0, s1, q_settled, qd_settled, K)
    V = m.particle_count
    n = args.sc_batch_n
    return {
        "metric": "VBD vertex-iters/s on 1 B200, batched cloth with self-contact", "value": V * SC_ITERATIONS / (ms * 1e-3),
        "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (sheets dropped on spheres)",
        "config": {"workload": f"{W} sheets of {n}x{n} with self-contact, each over its own sphere, 0.5 m apart",
                   "vertices": V, "iterations": SC_ITERATIONS, "dt": DT, "settled_substeps": settle,
                   "build_s": round(build_s, 1), "schedule": solver.schedule,
                   "lanes_per_vertex": solver.lanes_per_vertex,
                   "timed": "sphere contact generation + step, one CUDA graph per two substeps"},
        "launches_per_step": solver.launches_per_step + 1,
        "per_color": {"value": V * SC_ITERATIONS / (ms_pc * 1e-3), "unit": UNIT, "ms_per_step": ms_pc,
                      "launches_per_step": per_color.launches_per_step + 1,
                      "lanes_per_vertex": per_color.lanes_per_vertex},
        "persistent_over_per_color": ms_pc / ms,
        "self_contact_pairs": {"vertex_triangle": pairs[0], "edge_edge": pairs[1], "overflow_flags": pairs[2]},
        "clocks": clk.summary(), "device_errors": solver.device_errors() + per_color.device_errors(),
        "finite": bool(torch.isfinite(s0.particle_q).all().item()),
    }  # fmt: skip


def build_soft_model(dev, worlds, seed=5):
    """Volumetric batch: `worlds` tetrahedral blocks of 8 x 4 x 4 cells (5 tets per cell, 225 particles, 640
    tets; 2 cm cells, 500 kg/m^3, mu 2e4 Pa, lambda 3e4 Pa, damping 1e-3), each hung from a fixed anchor by
    four springs at its top corners, falling onto a ground plane from a seeded height and velocity."""
    import torch

    import newton_chysx_b200 as nb

    tpl = nb.ModelBuilder(up_axis="Z", gravity=-9.81)
    tpl.add_soft_grid(pos=(0.0, 0.0, 0.0), rot=nb.quat_identity(), vel=(0.0, 0.0, 0.0), dim_x=8, dim_y=4, dim_z=4,
                      cell_x=0.02, cell_y=0.02, cell_z=0.02, density=500.0, k_mu=2.0e4, k_lambda=3.0e4, k_damp=1.0e-3,
                      particle_radius=2e-3)  # fmt: skip
    nv = tpl.particle_count
    anchor = tpl.add_particle((0.08, 0.04, 0.5), (0.0, 0.0, 0.0), 0.0, 2e-3)
    for c in (nv - 1, nv - 9, nv - 1 - 9 * 4, nv - 9 - 9 * 4):
        tpl.add_spring(anchor, c, 50.0, 1e-2, 0.0)
    tpl.color()
    b = nb.ModelBuilder(up_axis="Z", gravity=-9.81)
    for _ in range(worlds):
        b.add_world(tpl)
    b.add_ground_plane()
    m = b.finalize(dev)
    rng = np.random.default_rng(seed)
    n1 = tpl.particle_count
    lift = np.repeat(rng.uniform(0.01, 0.05, worlds), n1)
    vx = np.repeat(rng.normal(0.0, 0.2, worlds), n1)
    block = np.tile(np.arange(n1) < nv, worlds)
    with torch.no_grad():
        m.particle_q[:, 2] += torch.as_tensor(np.where(block, lift, 0.0), dtype=torch.float32, device=dev)
        m.particle_qd[:, 0] = torch.as_tensor(np.where(block, vx, 0.0), dtype=torch.float32, device=dev)
        m.particle_qd[:, 2] = torch.as_tensor(np.where(block, -0.5, 0.0), dtype=torch.float32, device=dev)
    m.soft_contact_ke, m.soft_contact_kd, m.soft_contact_mu = 1.0e4, 1.0e-2, 0.5
    return m


def run_soft(args):
    """Soft bodies (tetrahedra + springs), batched: --instances blocks (default 4,096) on the persistent schedule
    (one CTA per block), 10 iterations, dt = 1/600 s, ground contact. The step is timed from a CUDA graph of two
    substeps. The per-instance working set (about 60 KB of tet records and adjacency) stays in L1/L2 for the
    instance's 10 iterations, so DRAM moves each instance's data about once per substep: the kernel is bound by
    its arithmetic and by gather latency, not by HBM; the roofline fraction says so."""
    import torch

    import newton_chysx_b200 as nb

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    W = args.instances
    t0 = time.perf_counter()
    m = build_soft_model(dev, W)
    build_s = time.perf_counter() - t0
    solver = nb.SolverVBD(m, iterations=ITERATIONS, schedule="persistent", lanes_per_vertex=args.lanes,
                          instance_per_warp=args.warp)  # fmt: skip
    pipe = nb.CollisionPipeline(m, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    s0, s1 = m.state(), m.state()
    for _ in range(args.warmup):
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    q_w, qd_w = s0.particle_q.clone(), s0.particle_qd.clone()
    graph = torch.cuda.CUDAGraph()
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream), torch.cuda.graph(graph, stream=stream):
        pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        pipe.collide(s1, contacts)
        solver.step(s1, s0, None, contacts, DT)
    torch.cuda.current_stream().wait_stream(stream)
    s0.particle_q.copy_(q_w)
    s0.particle_qd.copy_(qd_w)
    K = max(2, args.steps + (args.steps % 2))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler(dev.index or 0) as clk:
        e0.record()
        for _ in range(K // 2):
            graph.replay()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    V = m.particle_count
    value = V * ITERATIONS / (ms * 1e-3)
    # algorithmic DRAM bytes per substep: every instance's records read once (tet int4 + 3 float4 = 64 B, spring
    # int2 + float4 = 24 B, adjacency 4 B per incidence and 2 x 4 B offsets per vertex), the particle arrays the
    # step reads (q, qd, mass, inv mass, flags: 36 B) and writes (q twice, qd: 36 B)
    T, S = m.tet_count, m.spring_count
    alg = T * 64 + S * 24 + 4 * (4 * T + 2 * S) + V * (2 * 2 * 4) + V * 72
    peak, peak_src = _peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    out = {
        "metric": "VBD vertex-iters/s on 1 B200, batched soft bodies (tetrahedra + springs)", "value": value,
        "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded tetrahedral blocks on springs)",
        "config": {"workload": f"{W} tetrahedral blocks 8x4x4 cells hung by springs over a ground plane",
                   "vertices": V, "tets": T, "springs": S, "iterations": ITERATIONS, "dt": DT,
                   "schedule": solver.schedule, "lanes_per_vertex": solver.lanes_per_vertex,
                   "instance_per_warp": bool(args.warp), "shared_bytes": solver.shared_bytes,
                   "build_s": round(build_s, 1),
                   "timed": "ground contact generation + step, one CUDA graph per two substeps",
                   "l2": "per-instance working set stays on chip for its iterations; DRAM sees it once per substep"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_src, "algorithmic_bytes_per_step": alg,
                     "note": "algorithmic bytes per substep / substep time; compute- and latency-bound"},
        "gpu_launches": K * (solver.launches_per_step + 1), "colors": len(m.particle_color_groups),
        "clocks": clk.summary(), "device_errors": solver.device_errors(),
        "finite": bool(torch.isfinite(s0.particle_q).all().item()),
    }  # fmt: skip
    if not args.no_e2e:
        hq, hqd = q_w.cpu().pin_memory(), qd_w.cpu().pin_memory()
        out_q = torch.empty_like(hq).pin_memory()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(K):
            s0.particle_q.copy_(hq, non_blocking=True)
            s0.particle_qd.copy_(hqd, non_blocking=True)
            pipe.collide(s0, contacts)
            solver.step(s0, s1, None, contacts, DT)
            out_q.copy_(s1.particle_q, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        ms_e = e0.elapsed_time(e1) / K
        out["e2e"] = {"value": V * ITERATIONS / (ms_e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 2 * hq.numel() * 4,
                      "d2h_bytes_per_step": out_q.numel() * 4, "steps": K}  # fmt: skip
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_soft()
    return out


def cpu_baseline_soft(sample_worlds=256, seconds=10.0):
    """The oracle (FP32, all host threads) on `sample_worlds` blocks of the same workload, substep after substep
    until `seconds` have passed."""
    import torch

    from oracle import vbd_oracle as orc
    from tests.helpers import oracle_model_dict

    m = build_soft_model(torch.device("cpu"), sample_worlds)
    threads = orc.max_threads()
    om = orc.Model(oracle_model_dict(m))
    q = m.particle_q.double().numpy()
    qd = m.particle_qd.double().numpy()
    cnt, p, s, bp, bv, nn = orc.soft_contacts_shapes(q, m.particle_radius.numpy(), m.particle_flags.numpy(),
                                                     m.shape_type, m.shape_transform, m.shape_scale, 0.01)  # fmt: skip
    t = time.perf_counter()
    n = 0
    while n == 0 or time.perf_counter() - t < seconds:
        _, q, qd = orc.step(om, q, qd, None, orc.make_contacts(cnt, p, s, bp, bv, nn), DT, ITERATIONS, precision=32,
                            nthreads=threads)  # fmt: skip
        n += 1
    el = time.perf_counter() - t
    return {"value": n * m.particle_count * ITERATIONS / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} substeps of {sample_worlds} blocks of the same workload (contacts of the first substep)"}  # fmt: skip


def build_contact_scene(dev, n_particles, seed=7):
    """Particles spread over 2 m x 2 m x 0.8 m above nine static shapes, one of every kind the contact generator
    handles: ground plane, sphere, box, capsule, cone, ellipsoid, a 257 x 257 heightfield, an icosphere mesh
    (1,280 triangles, non-uniform scale) and a torus mesh (576 triangles, rotated)."""
    import numpy as np

    import newton_chysx_b200 as nb
    from tests.helpers import icosphere, torus_mesh

    rng = np.random.default_rng(seed)
    b = nb.ModelBuilder(up_axis="Z")
    pts = np.stack([rng.uniform(-1.0, 1.0, n_particles), rng.uniform(-1.0, 1.0, n_particles),
                    rng.uniform(-0.05, 0.75, n_particles)], 1)  # fmt: skip
    b.add_particles(pts, (0.0, 0.0, 0.0), 1.0, radius=0.005)
    q = nb.quat_from_axis_angle((0.2, 1.0, 0.3), 0.6)
    b.add_ground_plane()
    b.add_shape_sphere(xform=((0.5, 0.5, 0.3), nb.quat_identity()), radius=0.2)
    b.add_shape_box(xform=((-0.5, -0.5, 0.3), q), hx=0.2, hy=0.15, hz=0.1)
    b.add_shape_capsule(xform=((0.0, 0.6, 0.35), q), radius=0.08, half_height=0.2)
    b.add_shape_cone(xform=((-0.6, 0.4, 0.3), nb.quat_identity()), radius=0.2, half_height=0.2)
    b.add_shape_ellipsoid(xform=((0.6, -0.1, 0.5), q), rx=0.2, ry=0.15, rz=0.1)
    g = np.linspace(-1.0, 1.0, 257)
    gx, gy = np.meshgrid(g, g)
    b.add_shape_heightfield(xform=((0.0, 0.0, 0.05), nb.quat_identity()),
                            heightfield=nb.Heightfield(0.05 * np.sin(4 * gx) * np.cos(3 * gy), 257, 257, 1.0, 1.0))
    b.add_shape_mesh(xform=((0.1, -0.5, 0.3), nb.quat_identity()), mesh=nb.Mesh(*icosphere(0.2, 3)),
                     scale=(1.2, 1.0, 0.8))  # fmt: skip
    b.add_shape_mesh(xform=((-0.1, 0.0, 0.4), q), mesh=nb.Mesh(*torus_mesh(0.25, 0.06)))
    return b.finalize(dev)


def run_contacts(args):
    """Particle-shape contact generation (CollisionPipeline.collide -> vbd_soft_contacts_table): --contact-particles
    particles (default 8M) against nine shapes of every kind. One launch tests every (particle, shape) pair; the
    metric is pair tests per second. Algorithmic DRAM bytes per launch: each particle's position, radius and flags
    read once (20 B) plus each contact written (particle and shape ids, point, velocity, normal: 44 B); the mesh
    and heightfield queries are arithmetic- and gather-bound, which the roofline fraction shows."""
    import torch

    import newton_chysx_b200 as nb

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    N = args.contact_particles
    t0 = time.perf_counter()
    m = build_contact_scene(dev, N)
    build_s = time.perf_counter() - t0
    S = m.shape_count
    pipe = nb.CollisionPipeline(m, soft_contact_max=N, soft_contact_margin=0.01)
    contacts = pipe.contacts()
    state = m.state()
    for _ in range(args.warmup):
        pipe.collide(state, contacts)
    torch.cuda.synchronize()
    K = args.steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index or 0) as clk:
        e0.record()
        for _ in range(K):
            pipe.collide(state, contacts)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    count = int(contacts.soft_contact_count.item())
    pairs = N * S
    alg = 20 * N + 44 * min(count, N)
    peak, peak_src = _peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    out = {
        "metric": "particle-shape contact pair tests/s on 1 B200 (contact generation for the VBD step)",
        "value": pairs / (ms * 1e-3), "unit": "pairs/s", "n_gpus": 1, "steps": K, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded particles over nine analytic, heightfield and mesh shapes)",
        "config": {"workload": f"{N} particles x {S} static shapes (plane, sphere, box, capsule, cone, ellipsoid, "
                               "257x257 heightfield, 1280- and 576-triangle meshes)",
                   "particles": N, "shapes": S, "contacts_found": count, "margin": 0.01, "build_s": round(build_s, 1),
                   "l2": f"inputs {20 * N / 1e6:.0f} MB > L2, no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_src, "algorithmic_bytes_per_launch": alg,
                     "note": "one thread per (particle, shape): mesh BVH and heightfield queries make it "
                             "arithmetic- and gather-bound"},
        "gpu_launches": K, "clocks": clk.summary(),
    }  # fmt: skip
    if not args.no_e2e:
        hq = state.particle_q.cpu().pin_memory()
        hc = torch.empty(1, dtype=torch.int32).pin_memory()
        hn = torch.empty_like(contacts.soft_contact_normal, device="cpu").pin_memory()
        hp = torch.empty_like(contacts.soft_contact_particle, device="cpu").pin_memory()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(K):
            state.particle_q.copy_(hq, non_blocking=True)
            pipe.collide(state, contacts)
            hc.copy_(contacts.soft_contact_count, non_blocking=True)
            hp.copy_(contacts.soft_contact_particle, non_blocking=True)
            hn.copy_(contacts.soft_contact_normal, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        ms_e = e0.elapsed_time(e1) / K
        out["e2e"] = {"value": pairs / (ms_e * 1e-3), "unit": "pairs/s", "h2d_bytes_per_step": hq.numel() * 4,
                      "d2h_bytes_per_step": 4 + hp.numel() * 4 + hn.numel() * 4, "steps": K}  # fmt: skip
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_contacts(m, seconds=min(args.cpu_seconds, 10.0))
    return out


def cpu_baseline_contacts(m, seconds=10.0):
    """The oracle's contact generation (one host thread, a serial loop over particles and shapes) on leading
    slices of the same particles, grown until `seconds` have passed."""
    import numpy as np

    from oracle import vbd_oracle as orc

    q = m.particle_q.double().cpu().numpy()
    r = m.particle_radius.double().cpu().numpy()
    fl = m.particle_flags.cpu().numpy()
    args = (m.shape_type, m.shape_transform.astype(np.float64), m.shape_scale.astype(np.float64))
    kw = dict(heightfield_index=m.shape_heightfield_index, heightfields=m.heightfield_data,
              elevations=m.heightfield_elevations.cpu().numpy(), mesh_index=m.shape_mesh_index,
              meshes=[(x.vertices, x.indices) for x in m.meshes])  # fmt: skip
    n, done, t = 2048, 0, time.perf_counter()
    while time.perf_counter() - t < seconds and n <= len(r):
        orc.soft_contacts_shapes(q[:n], r[:n], fl[:n], *args, 0.01, max_contacts=n, **kw)
        done += n
        n *= 2
    el = time.perf_counter() - t
    return {"value": done * m.shape_count / el, "unit": "pairs/s", "cores": 1, "kind": "port",
            "sample": f"{done} particles x {m.shape_count} shapes (leading slices of the same particles; the oracle "
                      "queries meshes by brute force)"}


def run_adjoint(args):
    """Differentiable config: 64 x 64 hanging cloth (a curtain: the whole top row pinned, bending ke 1e-2),
    60 frames x 10 substeps x 10 iterations; loss = mean squared distance of the final positions to a
    seeded target (rest shape plus N(0, 0.05^2) per coordinate); gradient w.r.t. per-triangle Young's
    moduli (through the Lame map) and the initial velocity by the hand-written adjoint, checked against
    FP64 central differences (h = 1e-4) along 32 seeded random directions.

    Why a curtain with some bending stiffness: a sheet hung from two corners, or one whose bending is
    negligible (ke 1e-4), passes through compressed states where out-of-plane motion buckles
    exponentially; the derivative w.r.t. the initial velocity then grows to ~1e14 after 240 substeps and
    central differences agree with the adjoint only below h ~ 1e-7 (measured), so a check at h = 1e-4
    says nothing. With the top row pinned and ke = 1e-2 the 600-substep derivatives stay O(1e-4) and
    central differences agree to ~1e-6."""
    import torch

    import newton_chysx_b200 as nb
    from newton_chysx_b200.adjoint import DifferentiableVBD, lame_from_young

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    n, nu, h_th, frames = 64, 0.3, 1.0e-3, args.adjoint_frames
    substeps = frames * 10
    b = nb.ModelBuilder(up_axis="Z", gravity=-9.81)
    rot = nb.quat_from_axis_angle((1.0, 0.0, 0.0), np.pi * 0.5)
    b.add_cloth_grid(pos=(0.0, 0.0, 1.0), rot=rot, vel=(0.0, 0.0, 0.0), dim_x=n - 1, dim_y=n - 1, cell_x=1.0 / (n - 1),
                     cell_y=1.0 / (n - 1), mass=0.2 / (n * n), tri_ke=1.0, tri_ka=1.0, tri_kd=0.0, edge_ke=1e-2,
                     edge_kd=0.0, particle_radius=5e-3)  # fmt: skip
    flags = b.particle_flags
    for i in range(n * (n - 1), n * n):
        flags[i] &= ~int(nb.ParticleFlags.ACTIVE)
    b.set_particle_flags(flags)
    b.color(include_bending=True)
    model = b.finalize(dev)
    rng = np.random.default_rng(args.seed)
    T = model.tri_count
    E = torch.tensor(10.0 ** rng.uniform(3.5, 4.5, size=T), dtype=torch.float64, device=dev)
    q0 = model.particle_q.to(torch.float64)
    qd0 = torch.zeros_like(q0)
    target = q0 + torch.tensor(rng.normal(0.0, 0.05, size=q0.shape), dtype=torch.float64, device=dev)

    def loss_of(sim, mu, lam, v0):
        q, _ = sim.rollout(q0.to(sim.dtype), v0.to(sim.dtype), mu, lam, DT, substeps)
        return ((q.to(torch.float64) - target) ** 2).sum(dim=1).mean()

    out = {"workload": f"differentiable {n}x{n} curtain, {frames} frames x 10 substeps x 10 iterations",
           "vertices": model.particle_count, "triangles": T, "substeps": substeps}  # fmt: skip
    grads = {}
    for prec in ("fp64", "fp32"):
        sim = DifferentiableVBD(model, iterations=ITERATIONS, precision=prec)
        mu0, lam0 = lame_from_young(E, nu, h_th)
        times = []
        for rep in range(2):  # the first pass allocates the autograd buffers
            mu, lam = mu0.clone().requires_grad_(True), lam0.clone().requires_grad_(True)
            v0 = qd0.clone().requires_grad_(True)
            torch.cuda.synchronize()
            t = time.perf_counter()
            L = loss_of(sim, mu, lam, v0)
            torch.cuda.synchronize()
            tf = time.perf_counter() - t
            L.backward()
            torch.cuda.synchronize()
            times.append((tf, time.perf_counter() - t))
        grads[prec] = (sim, mu.grad.detach(), lam.grad.detach(), v0.grad.detach(), float(L.detach()))
        tf, tt = times[-1]
        vi = model.particle_count * ITERATIONS * substeps
        out[prec] = {"loss": float(L.detach()), "forward_s": tf, "forward_backward_s": tt,
                     "forward_vertex_iters_per_s": vi / tf, "backward_vertex_iters_per_s": vi / (tt - tf)}  # fmt: skip
    sim, gmu, glam, gv, _ = grads["fp64"]
    h = 1e-4
    worst, rels = 0.0, []
    drng = np.random.default_rng(args.seed + 1)
    for _ in range(args.adjoint_directions):
        dE = torch.tensor(drng.normal(size=T), device=dev, dtype=torch.float64)
        dv = torch.tensor(drng.normal(size=q0.shape), device=dev, dtype=torch.float64)
        dE, dv = dE / dE.abs().max(), dv / dv.norm()
        with torch.no_grad():
            mu_p, lam_p = lame_from_young(E * (1.0 + h * dE), nu, h_th)
            mu_m, lam_m = lame_from_young(E * (1.0 - h * dE), nu, h_th)
            fd = float(loss_of(sim, mu_p, lam_p, qd0 + h * dv) - loss_of(sim, mu_m, lam_m, qd0 - h * dv))
            # the model stores the Lame coefficients in float32: predict with the perturbation applied
            d_mu = mu_p.float().double() - mu_m.float().double()
            d_lam = lam_p.float().double() - lam_m.float().double()
            ad = float((gmu * d_mu).sum() + (glam * d_lam).sum() + (gv * (2.0 * h * dv)).sum())
        rel = abs(ad - fd) / max(abs(fd), 1e-30)
        rels.append(rel)
        worst = max(worst, rel)
    g32 = grads["fp32"]
    out["fd_check"] = {"directions": args.adjoint_directions, "h": h, "max_rel_err": worst,
                       "median_rel_err": float(np.median(rels)), "tolerance": 1e-3, "pass": worst <= 1e-3}  # fmt: skip
    out["fp32_vs_fp64_grad_rel"] = {
        "mu": float((g32[1].double() - gmu).norm() / gmu.norm()),
        "lambda": float((g32[2].double() - glam).norm() / glam.norm()),
        "velocity": float((g32[3].double() - gv).norm() / gv.norm()),
    }
    return out


def build_precision_model(n=1024, seed=4, sliver_fraction=1e-3):
    """1024 x 1024 sheet, per-triangle E log-uniform in [1e5, 1e8] Pa, 0.1% of vertex sites moved
    towards a neighbour so that incident triangles keep ~1e-6 of their nominal rest area."""
    from newton_chysx_b200 import sim

    rng = np.random.default_rng(seed)
    nu, h, density = 0.3, 1.0e-3, 0.2
    cell = 1.0 / (n - 1)
    xs, ys = np.meshgrid(np.arange(n), np.arange(n))
    verts = np.stack([xs.ravel() * cell, ys.ravel() * cell, np.zeros(n * n)], axis=1)
    sites = rng.choice(np.nonzero((xs.ravel() < n - 1) & (xs.ravel() > 0) & (ys.ravel() > 0) & (ys.ravel() < n - 1))[0],
                       size=int(sliver_fraction * n * n), replace=False)  # fmt: skip
    verts[sites, 0] += cell * (1.0 - 1.0e-6)  # next to its +x neighbour
    cx, cy = np.meshgrid(np.arange(1, n), np.arange(1, n))
    cx, cy = cx.ravel(), cy.ravel()
    v0, v1, v2, v3 = (cy - 1) * n + cx - 1, (cy - 1) * n + cx, cy * n + cx, cy * n + cx - 1
    idx = np.stack([v0, v1, v3, v1, v2, v3], axis=1).reshape(-1)
    T = len(idx) // 3
    E = 10.0 ** rng.uniform(5.0, 8.0, size=T)
    b = sim.ModelBuilder(up_axis="Z", gravity=-9.81)
    rot = sim.quat_from_axis_angle((1.0, 0.0, 0.0), np.pi * 0.5)
    start = b.add_particles(verts @ sim.quat_to_matrix(rot).astype(np.float32).astype(np.float64).T
                            + np.array([0.0, 0.0, 0.1]), (0, 0, 0), np.zeros(n * n), radius=5e-3)  # fmt: skip
    tri = (start + idx).reshape(-1, 3)
    areas = b.add_triangles(tri[:, 0], tri[:, 1], tri[:, 2], E * h / (2 * (1 + nu)), E * h * nu / (1 - nu * nu), 0.0)
    assert np.all(areas > 0.0), "a sliver lost its area"
    hinges = sim.mesh_hinges(b.tri_indices)
    b.add_edges(hinges[:, 0], hinges[:, 1], hinges[:, 2], hinges[:, 3], edge_ke=1e-4, edge_kd=0.0)
    mass = np.full(n * n, density / (n * n))
    flags = b.particle_flags
    for c in (n * (n - 1), n * n - 1):
        flags[c] = 0
        mass[c] = 0.0
    b.set_particle_mass(mass)
    b.set_particle_flags(flags)
    b.color(include_bending=True)
    return b, sites


def run_precision(args):
    """FP32 and mixed precision against all-FP64 runs of the same kernels on the precision stress sheet.

    Three figures per precision: (1) the error of one substep started from the same FP64 state (the
    arithmetic error of the step), sampled at several frames; (2) the trajectory error after all
    frames; (3) next to it, the spread of two FP64 trajectories whose initial positions differ by
    1e-12 m: past a bifurcation of the stiff, unconverged dynamics, any perturbation grows to the
    same size, so trajectory differences below that spread say nothing about arithmetic."""
    import torch

    import newton_chysx_b200 as nb

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    b, _ = build_precision_model(args.precision_n)
    model = b.finalize(dev)
    iters, frames = 30, args.precision_frames
    # sliver-adjacent vertices: those of triangles below 1e-3 of the median rest area
    areas = model.tri_areas.cpu().numpy()
    sliver = np.zeros(model.particle_count, dtype=bool)
    sliver[np.unique(model.tri_indices.cpu().numpy()[areas < 1e-3 * np.median(areas)].ravel())] = True
    out = {"workload": f"precision stress {args.precision_n}x{args.precision_n}", "frames": frames, "substeps": 10,
           "iterations": iters, "vertices": model.particle_count, "triangles": model.tri_count,
           "sliver_adjacent_vertices": int(sliver.sum())}  # fmt: skip
    solvers = {p: nb.SolverVBD(model, iterations=iters, precision=p, schedule="per_color") for p in ("fp64", "fp32", "mixed")}
    # mixed precision at further FP64-solve thresholds (one-substep errors only)
    extra = {f"mixed_threshold_{t:g}": nb.SolverVBD(model, iterations=iters, precision="mixed", schedule="per_color",
                                                     fp64_solve_threshold=t) for t in args.mixed_thresholds}  # fmt: skip
    solvers.update(extra)

    def states(dtype):
        s0, s1 = model.state(), model.state()
        for s_ in (s0, s1):
            s_.particle_q, s_.particle_qd, s_.particle_f = (t.to(dtype) for t in (s_.particle_q, s_.particle_qd, s_.particle_f))
        return s0, s1

    def run(prec, perturb=0.0, sample_frames=()):
        dtype = torch.float64 if prec == "fp64" else torch.float32
        s0, s1 = states(dtype)
        if perturb:
            g = torch.Generator(device=dev).manual_seed(1)
            s0.particle_q += perturb * torch.randn(s0.particle_q.shape, generator=g, device=dev, dtype=dtype)
        samples, traj = {}, []
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_ms = 0.0
        for f in range(frames):
            for k in range(10):
                if f in sample_frames and k == 0:
                    samples[f] = (s0.particle_q.clone(), s0.particle_qd.clone())
                e0.record()
                solvers[prec].step(s0, s1, None, None, DT)
                e1.record()
                torch.cuda.synchronize()
                t_ms += e0.elapsed_time(e1)
                s0, s1 = s1, s0
            traj.append(s0.particle_q.double().cpu().numpy())
        return traj, samples, t_ms

    def err(a, b):
        d = np.linalg.norm(a - b, axis=1)
        return {"max_m": float(d.max()), "rms_m": float(np.sqrt((d * d).mean()))}

    def err_split(a, b):
        d = np.linalg.norm(a - b, axis=1)
        return {"sliver_max_m": float(d[sliver].max()), "rest_max_m": float(d[~sliver].max()),
                "rest_rms_m": float(np.sqrt((d[~sliver] ** 2).mean()))}  # fmt: skip

    sample_frames = sorted({0, frames // 4, frames // 2, frames - 1})
    ref, samples, t64 = run("fp64", sample_frames=sample_frames)
    pert, _, _ = run("fp64", perturb=1e-12)
    out["fp64"] = {"vertex_iters_per_s": model.particle_count * iters * frames * 10 / (t64 * 1e-3),
                   "device_errors": solvers["fp64"].device_errors()}  # fmt: skip
    out["fp64_sensitivity_floor"] = {"perturbation_m": 1e-12,
                                     "per_frame_max_m": [err(a, b)["max_m"] for a, b in zip(ref, pert, strict=True)]}  # fmt: skip
    # the error of one substep that rounding the state to FP32 alone causes: the FP64 step from the FP32-rounded
    # state against the FP64 step from the exact state (no FP32 arithmetic at all)
    floor = {}
    for f, (q, qd) in samples.items():
        outs = []
        for rounded in (False, True):
            s_in, s_out = states(torch.float64)
            s_in.particle_q.copy_(q.float().double() if rounded else q)
            s_in.particle_qd.copy_(qd.float().double() if rounded else qd)
            solvers["fp64"].step(s_in, s_out, None, None, DT)
            outs.append(s_out.particle_q.cpu().numpy())
        torch.cuda.synchronize()
        floor[f"frame_{f}"] = err_split(outs[1], outs[0])
    out["fp64_from_fp32_rounded_state"] = floor
    for name in extra:
        one = {}
        for f, (q, qd) in samples.items():
            outs = []
            for key, dtype in (("fp64", torch.float64), (name, torch.float32)):
                s_in, s_out = states(dtype)
                s_in.particle_q.copy_(q)
                s_in.particle_qd.copy_(qd)
                solvers[key].step(s_in, s_out, None, None, DT)
                outs.append(s_out.particle_q.double().cpu().numpy())
            one[f"frame_{f}"] = err_split(outs[1], outs[0])
        out[name] = {"one_substep_error": one}
    for prec in ("fp32", "mixed"):
        traj, _, t = run(prec)
        o = {"vertex_iters_per_s": model.particle_count * iters * frames * 10 / (t * 1e-3),
             "trajectory_error_final": err(traj[-1], ref[-1]),
             "trajectory_error_per_frame_max_m": [err(a, b)["max_m"] for a, b in zip(traj, ref, strict=True)],
             "device_errors": solvers[prec].device_errors()}  # fmt: skip
        one = {}
        for f, (q, qd) in samples.items():
            s64_in, s64_out = states(torch.float64)
            s64_in.particle_q.copy_(q)
            s64_in.particle_qd.copy_(qd)
            solvers["fp64"].step(s64_in, s64_out, None, None, DT)
            s_in, s_out = states(torch.float32)
            s_in.particle_q.copy_(q)
            s_in.particle_qd.copy_(qd)
            solvers[prec].step(s_in, s_out, None, None, DT)
            torch.cuda.synchronize()
            a, b64 = s_out.particle_q.double().cpu().numpy(), s64_out.particle_q.cpu().numpy()
            one[f"frame_{f}"] = dict(err(a, b64), **err_split(a, b64))
        o["one_substep_error"] = one
        if prec == "mixed":
            o["residual_last_step"] = solvers[prec].residuals().tolist()
        out[prec] = o
    return out


def relaunch(gpus: int, argv) -> int:
    """Runs this script as `gpus` ranks under torch.distributed.run on 127.0.0.1 and returns its exit code."""
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *argv]  # fmt: skip
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["batched", "plain", "precision", "selfcontact", "selfcontact_batch",
                                           "adjoint", "soft", "contacts"], default="batched")  # fmt: skip
    ap.add_argument("--contact-particles", type=int, default=8 << 20, help="contacts workload: particle count")
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--shared", choices=["auto", "on", "off"], default="auto")
    ap.add_argument("--layout", choices=["auto", "ring", "ell16", "ell", "csr"], default="auto")
    ap.add_argument("--occ", type=int, default=0, help="resident 256-thread CTAs per SM the kernel is compiled for")
    ap.add_argument("--pair", action="store_true", help="ell16: two vertices per thread in paired FP32 instructions")
    ap.add_argument("--warp", action="store_true", help="soft workload: one warp per instance")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="use the launch-shape flags, not the autotuner")
    ap.add_argument("--tune-instances", type=int, default=1024)
    ap.add_argument("--e2e-steps", type=int, default=0, help="substeps of the end-to-end leg (0: --steps)")
    ap.add_argument("--e2e-chunks", type=int, default=4, help="instance groups pipelined on separate streams in e2e")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--plain-sample", type=int, default=256, help="instances of the plain drop-in leg (0: off)")
    ap.add_argument("--plain-steps", type=int, default=5, help="timed substeps of the plain drop-in leg")
    ap.add_argument("--err-sample", type=int, default=16, help="instances of the FP64 position-error leg")
    ap.add_argument("--err-substeps", type=int, default=3, help="substeps of the per-substep FP64 comparison")
    ap.add_argument("--no-pos-err", action="store_true")
    ap.add_argument("--precision-n", type=int, default=1024)
    ap.add_argument("--precision-frames", type=int, default=60)
    ap.add_argument("--mixed-thresholds", type=float, nargs="*", default=[],
                    help="precision workload: further FP64-solve thresholds of mixed precision to compare")
    ap.add_argument("--traffic", type=float, default=None, help="DRAM bytes per launch from an ncu capture")
    ap.add_argument("--sc-n", type=int, default=256, help="selfcontact workload: grid side (vertices)")
    ap.add_argument("--sc-settle-frames", type=int, default=40, help="selfcontact workload: untimed frames first")
    ap.add_argument("--sc-batch-n", type=int, default=32, help="selfcontact_batch workload: sheet side (vertices)")
    ap.add_argument("--adjoint-frames", type=int, default=60)
    ap.add_argument("--adjoint-directions", type=int, default=32)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch this command under torchrun (rank 0 prints the JSON line)
        sys.exit(relaunch(args.gpus, sys.argv[1:]))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}; the ranks decide", file=sys.stderr)
    if args.impl == "reference":
        out = run_reference(args)
    elif args.workload == "plain":
        out = run_plain(args)
    elif args.workload == "precision":
        out = run_precision(args)
    elif args.workload == "selfcontact":
        out = run_selfcontact(args)
    elif args.workload == "selfcontact_batch":
        out = run_selfcontact_batch(args)
    elif args.workload == "adjoint":
        out = run_adjoint(args)
    elif args.workload == "soft":
        out = run_soft(args)
    elif args.workload == "contacts":
        out = run_contacts(args)
    else:
        out = run_ours(args)
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()

"""Benchmark of the sparse D3Q19 MRT single-phase update on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): 256^3 overlapping-sphere mask, sphere radius uniform in
4-10 lu, porosity 0.35, seed 20260101; periodic, tau = 0.8 (nu = 0.1),
gx = 1e-6; populations stored as FP32 deviations f_i - w_i, FP32 collision
arithmetic.  A step is one fused collide + pull-stream pass over every fluid
node.  Inputs (2 x 19 x 4 B x 5.87 M nodes + table) are far larger than the
126 MB L2, so no flush is needed between steps.

value  fluid MLUPS, device-resident, CUDA events on the solver's stream
       around the K timed steps, max over ranks; N ranks run N independent
       replicas (the single-domain path has no data exchange: weak scaling).
e2e    the same metric through the C ABI from host memory: lbm_create from
       the host mask (compaction, table, upload), K steps with a diagnostics
       read-back (lbm_reduce) every 100 steps, and lbm_get_fields of rho/u to
       the host, all inside the timed region.
roofline  achieved = (2*19*4 + table) B per fluid update x nodes / step time,
          table = the pull-table bytes per node the step reads (lbm_table_info:
          18*2 + 18*4/32 + the int32 fallback share x 18*4 with the compact
          table, 18*4 with the int32 one),
          against the measured HBM copy bandwidth.
--impl reference  times the reference solver (SP3, compiled from its own
       source with -O3 -march=native, oracle/_ref/libref_sp3_fast.so) on the
       host cores: one process per core, each on a 64^3 sub-block of the same
       geometry (a bounded sample of the workload).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "jianhui-lbm_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "fluid MLUPS (sparse D3Q19 MRT, FP32 deviation storage)"
SHAPE = (256, 256, 256)
PHI, RADIUS, SEED = 0.35, (4.0, 10.0), 20260101
NU, GX = 0.1, 1e-6
BYTES_PER_LU = 2 * 19 * 4 + 18 * 4  # with the int32 pull table; the solver reports its own


def workload_mask():
    from lbm_b200 import geometry as G

    return G.overlapping_spheres(SHAPE, PHI, RADIUS, SEED)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """dram bytes per launch of the step kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "sp_step_f32_256cube.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch_full:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []  # (host time, csv line)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.time(), ln.strip()))

    def wait_first_sample(self, limit_s=5.0):
        """Blocks until nvidia-smi has delivered a sample (at most limit_s)."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < limit_s:
            time.sleep(0.02)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, window=None):
        """Median SM clock and throttle reasons over every sample; with
        window = (t0, t1), also how many samples fell inside it."""
        sm, smax, reasons, inside = [], None, set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            if window and window[0] <= t <= window[1]:
                inside += 1
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
               "reasons": sorted(reasons), "samples": len(sm)}
        if window:
            out["samples_in_timed_region"] = inside
            out["span"] = "warm-up, timed steps and the e2e leg"
        return out


def _strict(x):
    """JSON-safe copy: non-finite floats (the +-inf permeability of an axis
    without force, k = Q nu / (V g) with g = 0) become null."""
    if isinstance(x, float):
        return x if x == x and abs(x) != float("inf") else None
    if isinstance(x, dict):
        return {k: _strict(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_strict(v) for v in x]
    return x


def emit(line):
    print(json.dumps(_strict(line), allow_nan=False), flush=True)


def dist_setup():
    from lbm_b200 import dispatch

    world, rank, local = dispatch.dist_env()
    return world, rank, local, dispatch.init_process_group()


def allmax(pg, x):
    from lbm_b200 import dispatch

    return dispatch.max_over_ranks(pg, x)


def barrier(pg):
    from lbm_b200 import dispatch

    dispatch.barrier(pg)


# ------------------------------------------------------------ reference arm
def _ref_worker(args):
    sub, steps, warm = args
    # the reference prints progress on stdout; keep the bench's stdout to its JSON line
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    import oracle

    ref = oracle.ReferenceSP3(fast=True)
    count = ref.create(sub, NU, (GX, 0.0, 0.0), binary=True)
    ref.step(warm)
    t0 = time.perf_counter()
    ref.step(steps)
    return count, time.perf_counter() - t0


def reference_sample(mask, steps, warmup, procs=None, edge=64):
    """Reference SP3 (-O3 -march=native) on `procs` host cores, each process on
    its own edge^3 periodic sub-block of the workload geometry."""
    import multiprocessing as mp

    try:
        ncpu = len(os.sched_getaffinity(0))
    except AttributeError:
        ncpu = os.cpu_count() or 1
    procs = procs or ncpu
    nz, ny, nx = mask.shape
    blocks = []
    per = max(nx // edge, 1)
    for b in range(procs):
        i, j, k = b % per, (b // per) % per, (b // (per * per)) % per
        sub = np.ascontiguousarray(mask[k * edge:(k + 1) * edge, j * edge:(j + 1) * edge, i * edge:(i + 1) * edge])
        blocks.append((sub, steps, warmup))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, blocks)
    wall = time.perf_counter() - t0
    lu = sum(c for c, _ in res) * steps
    tmax = max(t for _, t in res)
    return {"value": lu / tmax / 1e6, "unit": "MLUPS", "cores": procs, "kind": "reference",
            "sample": f"{procs} processes x {edge}^3 sub-blocks of the workload geometry, {steps} steps each "
                      f"after {warmup} warm-up; SP3 built -O3 -march=native; slowest process timed",
            "wall_s": wall}


def _calib_worker(args):
    sub, steps = args
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    import oracle

    ref = oracle.ReferenceSP3(fast=True)
    count = ref.create(sub, NU, (GX, 0.0, 0.0), binary=True)
    ref.step(1)
    t0 = time.perf_counter()
    ref.step(steps)
    return count, time.perf_counter() - t0


def reference_calibration(mask, steps=2, edge=64):
    """One reference process on the whole 256^3 geometry beside one process on
    a 64^3 sub-block (the unit of the timed sample), each alone on the host,
    same number of steps: shows whether the sub-blocks run faster per core
    than the full domain (cache effects of the smaller arrays)."""
    import multiprocessing as mp

    sub = np.ascontiguousarray(mask[:edge, :edge, :edge])
    ctx = mp.get_context("spawn")
    out = {}
    for name, m in (("sub_block_64", sub), ("full_domain_256", mask)):
        with ctx.Pool(1) as pool:
            count, t = pool.map(_calib_worker, [(m, steps)])[0]
        out[name] = {"fluid_nodes": count, "steps": steps, "mlups_1core": count * steps / t / 1e6}
    out["full_over_sub"] = out["full_domain_256"]["mlups_1core"] / out["sub_block_64"]["mlups_1core"]
    return out


def run_reference(a):
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return 0
    import oracle

    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference solver library oracle/_ref not built"}))
        return 0
    mask = workload_mask()
    cb = reference_sample(mask, a.steps, a.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "MLUPS", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "256^3 overlapping spheres r=U[4,10], phi=0.35, tau=0.8, gx=1e-6 (bounded sample)",
                       "sample": cb["sample"]},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    emit(line)
    return 0


# ------------------------------------------------------------ our arm
def run_ours(a):
    world, rank, local, pg = dist_setup()
    import lbm_b200

    mask = workload_mask()
    # pick ordering / block size once (not timed), then build the timed solver with them
    if a.ordering == "auto":
        with lbm_b200.SinglePhase(mask, NU, (GX, 0, 0), precision="f32", ordering="reference", device=local) as s0:
            tune = s0.autotune(trial_steps=200)
            compact = s0.table_info()["compact"]
        order, block = tune["ordering"], tune["block"]
    else:
        # steady-state winner on this workload (reference order, 256 threads,
        # int32 table); the autotuner's short trials run at burst clocks
        order, block, compact = lbm_b200.ORDERINGS[a.ordering], a.block, 0

    s = lbm_b200.SinglePhase(mask, NU, (GX, 0, 0), precision="f32", ordering=order, block_size=block, device=local)
    s.set_table_mode(compact)
    count = s.count
    mem, tinfo = s.memory(), s.table_info()
    bytes_per_lu = mem["bytes_per_lu"]  # populations + the table form the step reads
    # the sampler runs from before the warm-up to the end of the e2e leg: a
    # short timed region (the driver's 20 steps take 4 ms) sees no sample of
    # its own, the steps around it do
    clk = ClockSampler(local).__enter__()
    clk.wait_first_sample()
    s.step(a.warmup)
    barrier(pg)
    t_timed0 = time.time()
    s.step(a.steps)  # lbm_step times the K steps with CUDA events on its stream
    t_timed1 = time.time()
    ms = s.last_step_ms()
    diag = s.reduce()
    # untimed: the field read path's kernels load once per process (lazy
    # module loading), before the end-to-end leg rather than inside it
    s.fields()
    s.close()
    ms_max = allmax(pg, ms)
    ms_step = ms_max / a.steps
    value = world * count * a.steps / (ms_max * 1e-3) / 1e6

    # end to end through the C ABI from host buffers
    barrier(pg)
    if a.skip_e2e:
        t_e2e, count_e2e = None, count
    t0 = time.perf_counter()
    e = lbm_b200.SinglePhase(mask, NU, (GX, 0, 0), precision="f32", ordering=order, block_size=block, device=local)
    e.set_table_mode(compact)
    left, reads = (0 if a.skip_e2e else a.steps), 0
    while left > 0:
        k = min(100, left)
        e.step(k)
        e.reduce()
        reads += 1
        left -= k
    rho, u = e.fields()
    t_e2e = time.perf_counter() - t0
    e.close()
    # the bit-exact FP64 kernel on the same workload (its own solver, the
    # default launch shape), timed the same way
    f64_steps = max(50, min(a.steps, 500))
    with lbm_b200.SinglePhase(mask, NU, (GX, 0, 0), precision="f64", device=local) as f:
        f.step(5)
        f.step(f64_steps)
        ms64 = f.last_step_ms() / f64_steps
        b64 = f.memory()["bytes_per_lu"]
    clk.__exit__(None, None, None)
    t_e2e = allmax(pg, t_e2e)
    e2e_value = None if a.skip_e2e else world * count * a.steps / t_e2e / 1e6
    # in reference order lbm_create uploads the mask (one byte per cell) and
    # builds the compaction and the pull table on the device
    h2d = mask.size
    d2h = reads * 64 + rho.nbytes + u.nbytes

    if rank != 0:
        return 0
    peak, peak_kind = measured_peak()
    achieved = bytes_per_lu * count / (ms_step * 1e-3) / 1e9
    traffic = profiled_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "256^3 overlapping spheres r=U[4,10], phi=0.35, seed 20260101, tau=0.8, gx=1e-6, "
                               "FP32 deviation storage",
                   "fluid_nodes": count, "ordering": order, "block": block, "parallelism": f"replicas x{world}",
                   "l2": "inputs > L2 (no flush)",
                   "pull_table": "compact" if tinfo["compact"] else "int32",
                   "table_wide_fraction": tinfo["wide_fraction"]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind, "bytes_per_lu": bytes_per_lu},
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": h2d / a.steps,
                "d2h_bytes_per_step": d2h / a.steps, "wall_s": t_e2e,
                "what": "lbm_create from the host mask (upload of nx*ny*nz bytes; compaction and pull table built "
                        "on the device), K steps with an lbm_reduce read-back every 100, lbm_get_fields of rho and "
                        "u (doubles, reference id order); at small K the creation and the field read-back "
                        "dominate the wall time"},
        "gpu_launches": a.steps,
        "clocks": clk.summary(window=(t_timed0, t_timed1)),
        "perm_x": diag["perm"][0],
        "fp64_exact": {"mlups": count / (ms64 * 1e-3) / 1e6, "ms_per_step": ms64, "steps": f64_steps,
                       "bytes_per_lu": b64, "gbs": b64 * count / (ms64 * 1e-3) / 1e9,
                       "what": "the FP64 kernel whose populations equal the reference's bit for bit "
                               "(FP64-pipe bound, not HBM)"},
    }
    if world == 1 and not a.no_cpu_baseline:
        try:
            cb = reference_sample(mask, steps=a.cpu_steps, warmup=1)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            if not a.no_cpu_calibration:
                line["cpu_baseline"]["calibration"] = reference_calibration(mask, steps=a.calib_steps)
        except Exception as ex:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unavailable": str(ex)[:200]}
    emit(line)
    return 0


# ------------------------------------------------------------ batch / serve
def shard(items, world, rank, weight):
    from lbm_b200 import dispatch

    return dispatch.shard([weight(x) for x in items], world, rank)


def size_breakdown(trace, per_inst):
    """Where each path spends its time: the pool's rate by the nodes stepping
    in a chain, the one-at-a-time path's by instance size (fluid nodes)."""
    bins = [0, 2e5, 5e5, 1e6, 2e6, 4e6, 8e6, 1e12]
    out = {"pool_by_stepping_nodes": [], "one_at_a_time_by_instance_nodes": []}
    tr = np.asarray(trace).reshape(-1, 3)
    tot = sum(n * st for n, st, _ in per_inst) or 1
    for lo, hi in zip(bins[:-1], bins[1:]):
        m = (tr[:, 0] >= lo) & (tr[:, 0] < hi)
        if m.any():
            ms = float(tr[m, 2].sum())
            out["pool_by_stepping_nodes"].append({"nodes": [lo, hi], "chains": int(m.sum()), "ms": ms,
                                                  "glups": float((tr[m, 0] * tr[m, 1]).sum() / (ms * 1e-3) / 1e9)})
        sel = [(n, st, t) for n, st, t in per_inst if lo <= n < hi]
        if sel:
            work = sum(n * st for n, st, _ in sel)
            secs = sum(t for _, _, t in sel)
            out["one_at_a_time_by_instance_nodes"].append({"nodes": [lo, hi], "instances": len(sel), "s": secs,
                                                           "glups": work / secs / 1e9, "share_of_work": work / tot})
    return out


def run_batch(a):
    """64 independent sphere packs to the 1e-6 stop test: one batched pool vs
    the plain one-at-a-time GPU path, same tolerance."""
    world, rank, local, pg = dist_setup()
    import lbm_b200
    from lbm_b200 import workloads as W

    inst_all = W.config4_instances(a.instances)
    mine = shard(inst_all, world, rank, lambda x: float((x[0] == 0).sum()))
    inst = [inst_all[i] for i in mine]
    tol, every, cap = 1e-6, 100, 400000
    clk = ClockSampler(local).__enter__()
    fixed = a.batch_block > 0
    # the CUDA context and the library's kernels load with the first solve of
    # the process: one small solve first, so neither timed path pays for it
    with lbm_b200.SinglePhase(np.zeros((8, 8, 8), dtype=np.uint8), 0.1, (1e-6, 0, 0), precision="f32",
                              device=local) as warm:
        warm.step(2)
    with lbm_b200.Batch([(np.zeros((8, 8, 8), dtype=np.uint8), 0.1, (1e-6, 0, 0))], precision="f32",
                        ordering="reference", block=256, device=local) as warm:
        warm.run(tol=1e-3, check_every=10, max_steps=20)
    # the layout and block size are picked first on a batch of their own (not
    # timed); the timed batch is created with them
    if fixed:
        tune = {"ordering": lbm_b200.ORDER_REFERENCE, "block": a.batch_block}
    else:
        with lbm_b200.Batch(inst, precision="f32", ordering="reference", block=256, device=local) as b:
            tune = b.autotune(trial_steps=30)
    order_name = {v: k for k, v in lbm_b200.ORDERINGS.items()}[tune["ordering"]]
    barrier(pg)
    t0 = time.perf_counter()
    with lbm_b200.Batch(inst, precision="f32", ordering=order_name, block=tune["block"], device=local) as b:
        t_batch_create = time.perf_counter() - t0
        barrier(pg)
        t0 = time.perf_counter()
        res = b.run(tol=tol, check_every=every, max_steps=cap)
        t_batch = time.perf_counter() - t0
        info = b.info()
        trace = b.trace()
    singles, t_single, t_single_create, per_inst, creates = [], 0.0, 0.0, [], []
    for (mask, nu, g) in inst:
        tc = time.perf_counter()
        with lbm_b200.SinglePhase(mask, nu, g, precision="f32", device=local) as s:
            t0 = time.perf_counter()
            d = s.run_to_convergence(tol=tol, check_every=every, max_steps=cap)
            dt = time.perf_counter() - t0
            t_single += dt
            t_single_create += t0 - tc
            creates.append(t0 - tc)
            singles.append(d)
            per_inst.append((s.count, d["step"], dt))
    # FP64 check of a seeded sample of the instances: the bit-exact FP64
    # kernel run to the same stop test is the reference's permeability
    rng = np.random.default_rng(11)
    sample = sorted(rng.choice(len(inst), size=min(a.fp64_sample, len(inst)), replace=False).tolist())
    errs = []
    for i in sample:
        mask, nu, g = inst[i]
        with lbm_b200.SinglePhase(mask, nu, g, precision="f64", device=local) as s:
            d = s.run_to_convergence(tol=tol, check_every=every, max_steps=cap)
        errs.append(abs(res[i]["perm"][0] - d["perm"][0]) / abs(d["perm"][0]))
    clk.__exit__(None, None, None)
    t_batch = allmax(pg, t_batch)
    t_single = allmax(pg, t_single)
    if rank != 0:
        return 0
    dk = max(abs(r["perm"][0] - s["perm"][0]) / abs(s["perm"][0]) for r, s in zip(res, singles))
    line = {"metric": "perm solves/s (batched)", "value": len(inst_all) / t_batch, "unit": "solves/s",
            "n_gpus": world, "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(inst_all)} sphere packs, edge log-U[48,160], porosity U[0.25,0.5], r=5, tau=0.8, "
                                   "gx=1e-6, stop test 1e-6 per 100 steps", "seed": 404,
                       "ordering": tune["ordering"], "block": tune["block"]},
            "one_at_a_time": {"value": len(inst_all) / t_single, "unit": "solves/s", "wall_s": t_single},
            "batched_wall_s": t_batch, "speedup_vs_one_at_a_time": t_single / t_batch,
            "fluid_nodes": info["total_nodes"], "node_steps": info["node_steps"],
            "mlups_batched": info["node_steps"] / t_batch / 1e6,
            "converged": sum(r["status"] == 0 for r in res), "max_rel_perm_diff_vs_one_at_a_time": dk,
            "with_creation": {"batched_s": t_batch_create + t_batch, "one_at_a_time_s": t_single_create + t_single,
                              "batch_create_s": t_batch_create, "one_at_a_time_create_s": t_single_create,
                              "one_at_a_time_create_s_first_median_max": [creates[0], float(np.median(creates)),
                                                                          max(creates)] if creates else None,
                              "batched_solves_per_s": len(inst_all) / (t_batch_create + t_batch),
                              "one_at_a_time_solves_per_s": len(inst_all) / (t_single_create + t_single),
                              "what": "host masks to converged results: lbm_batch_create (indexing, upload, pool) "
                                      "with the tuned layout and block + the run, against lbm_create + "
                                      "run_to_convergence per instance; the tuning itself (on a batch of its own) "
                                      "is not included"},
            "size_breakdown": size_breakdown(trace, per_inst),
            "fp64_check": {"sample": sample, "max_rel_perm_err": max(errs) if errs else None,
                           "anchor": "bit-exact FP64 kernel, same stop test"},
            "clocks": clk.summary()}
    emit(line)
    return 0


def run_serve(a):
    """Poisson request stream served by continuous batching; p50/p99 latency,
    solves/s and the permeability error of a sample against FP64."""
    world, rank, local, pg = dist_setup()
    import lbm_b200
    from lbm_b200 import workloads as W

    reqs_all = W.config5_requests(n=a.requests, rate_per_s=a.rate)
    mine = [i for i in range(len(reqs_all)) if i % world == rank]
    reqs = [reqs_all[i] for i in mine]
    tol, every = 1e-6, 100
    clk = ClockSampler(local).__enter__()
    lat, results, ids = [], {}, {}
    with lbm_b200.Server(capacity_nodes=a.pool_nodes, max_active=64, precision="f32", tol=tol, check_every=every,
                         max_steps=400000, device=local, target_active_nodes=a.target_nodes,
                         policy=a.policy) as srv:
        barrier(pg)
        t0 = srv.now()
        nxt = 0
        while len(results) < len(reqs):
            now = srv.now() - t0
            while nxt < len(reqs) and reqs[nxt][0] <= now:
                _, mask, nu, g = reqs[nxt]
                ids[srv.submit(mask, nu, g)] = nxt
                nxt += 1
            active, queued = srv.pump()
            for r in srv.poll():
                results[ids[r["request_id"]]] = r
            if active == 0 and queued == 0 and nxt < len(reqs):
                time.sleep(max(0.0, reqs[nxt][0] - (srv.now() - t0)))
        t_end = srv.now() - t0
    for i, r in results.items():
        lat.append(r["t_done"] - (t0 + reqs[i][0]))
    # the plain one-at-a-time GPU path on the same stream: each request's solo
    # solve time (single-domain FP32 solver, same stop test), served FIFO
    solo = []
    for (_, mask, nu, g) in reqs:
        ts = time.perf_counter()  # creation (indexing, upload) is part of a solo solve
        with lbm_b200.SinglePhase(mask, nu, g, precision="f32", device=local) as s:
            s.run_to_convergence(tol=tol, check_every=every, max_steps=400000)
        solo.append(time.perf_counter() - ts)
    free_at, fifo_lat = 0.0, []
    for (arr, _, _, _), d in zip(reqs, solo):
        start = max(arr, free_at)
        free_at = start + d
        fifo_lat.append(free_at - arr)
    fifo_lat = np.array(fifo_lat)
    fifo_span = free_at - reqs[0][0] if reqs else 0.0
    # FP64 check of a seeded sample of the requests
    rng = np.random.default_rng(7)
    sample = sorted(rng.choice(len(reqs), size=min(a.fp64_sample, len(reqs)), replace=False).tolist())
    errs = []
    for i in sample:
        _, mask, nu, g = reqs[i]
        with lbm_b200.SinglePhase(mask, nu, g, precision="f64", device=local) as s:
            d = s.run_to_convergence(tol=tol, check_every=every, max_steps=400000)
        errs.append(abs(results[i]["perm"][0] - d["perm"][0]) / abs(d["perm"][0]))
    clk.__exit__(None, None, None)
    if rank != 0:
        return 0
    lat = np.array(lat)
    line = {"metric": "perm solves/s (served), p50/p99 latency", "value": len(reqs) / t_end, "unit": "solves/s",
            "n_gpus": world, "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{a.requests} Poisson requests at {a.rate}/s, edge log-U[32,192], porosity "
                                   "U[0.2,0.5], r U[3,8], gx=1e-6, tau=0.8, stop test 1e-6 per 100 steps",
                       "seed": 505, "pool_nodes": a.pool_nodes, "target_active_nodes": a.target_nodes, "policy": a.policy},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "makespan_s": t_end, "converged": sum(r["status"] == 0 for r in results.values()),
            "one_at_a_time_fifo": {"solves_per_s": len(reqs) / (fifo_span + reqs[0][0]) if reqs else None,
                                   "p50": float(np.percentile(fifo_lat, 50)),
                                   "p99": float(np.percentile(fifo_lat, 99)),
                                   "gpu_busy_s": float(sum(solo))},
            "fp64_check": {"sample": sample, "max_rel_perm_err": max(errs) if errs else None,
                           "anchor": "bit-exact FP64 kernel, same stop test"},
            "clocks": clk.summary()}
    emit(line)
    return 0


def run_cfg2_accuracy(a):
    """The 256^3 workload run to its stop test (relative change of u_ave over
    100 steps below 1e-6, SP:812-816 with the configuration's tolerance) in
    each requested storage kind; the bit-exact FP64 kernel (identical to the
    reference's FP64 arithmetic, pinned against the compiled reference) is the
    anchor.  Reports the permeability error (Comput_Perm, SP3:3518-3650) and
    the velocity error max|u - u_64| / max|u_64| of each kind against it."""
    world, rank, local, pg = dist_setup()
    import lbm_b200

    mask = workload_mask()
    tol, every = 1e-6, 100
    out = {}
    with ClockSampler(local) as clk:
        for prec in [p.strip() for p in a.precisions.split(",") if p.strip()]:
            t0 = time.perf_counter()
            with lbm_b200.SinglePhase(mask, NU, (GX, 0, 0), precision=prec, device=local) as s:
                d = s.run_to_convergence(tol=tol, check_every=every, max_steps=a.max_steps)
                wall = time.perf_counter() - t0
                rho, u = s.fields()
                out[prec] = {"diag": d, "u": u[1:], "count": s.count, "wall_s": wall}
    if rank != 0:
        return 0
    anchor = out.get("f64")
    res = {}
    for prec, r in out.items():
        d = r["diag"]
        e = {"stop_step": d["step"], "converged": d["converged"] == 1, "status": d["status"],
             "perm": d["perm"], "u_ave": d["u_ave"], "wall_s": r["wall_s"],
             "fluid_mlups_wall": r["count"] * d["step"] / r["wall_s"] / 1e6}
        if anchor is not None and prec != "f64":
            k64 = anchor["diag"]["perm"]
            e["perm_err_vs_fp64"] = [abs(x - y) / abs(y) if y else None for x, y in zip(d["perm"], k64)]
            e["u_err_vs_fp64"] = float(np.abs(r["u"] - anchor["u"]).max() / np.abs(anchor["u"]).max())
            e["u_ave_err_vs_fp64"] = abs(d["u_ave"] - anchor["diag"]["u_ave"]) / abs(anchor["diag"]["u_ave"])
            e["stop_step_minus_fp64"] = d["step"] - anchor["diag"]["step"]
        res[prec] = e
    line = {"metric": "permeability error vs FP64 at the stop test", "workload": "cfg2-accuracy",
            "config": {"workload": "256^3 overlapping spheres r=U[4,10], phi=0.35, seed 20260101, tau=0.8, gx=1e-6; "
                                   "stop when |du_ave/u_ave| < 1e-6 over 100 steps", "fluid_nodes": out[next(iter(out))]["count"]},
            "anchor": "f64 = the bit-exact FP64 kernel" if anchor is not None else None,
            "results": res, "clocks": clk.summary(), "data": "synthetic", "n_gpus": world}
    emit(line)
    return 0


def run_cg(a):
    """Colour-gradient two-phase run (config 3) in FP32, compared with the FP64
    kernel (bit-identical to the reference colour-gradient solver) on the
    same input: saturation and phase fluxes."""
    world, rank, local, pg = dist_setup()
    import lbm_b200
    from lbm_b200 import workloads as W

    mask, psi = W.config3()
    kw = dict(nu_l=0.1, nu_g=0.1, psi_solid=0.70711, cap_a=1e-3, g=(1e-5, 0.0, 0.0), body_force_phase=-1,
              flux_psi=0.99, flux_umax=0.01)
    if a.cg_faces:
        # Sub_BC 1 pressure faces on both x faces, no body force
        kw["g"] = (0.0, 0.0, 0.0)
        kw["boundary"] = lbm_b200.Boundary.make(sub_bc=1, in_bc=1, pressure=(1, 1, 0, 0, 0, 0),
                                                rho=(1.0, 1.004, 1.0, 1.0, 1.0, 1.0))
    steps = a.cg_steps
    out = {}
    clk = ClockSampler(local).__enter__()
    for prec in ("f32", "f64"):
        with lbm_b200.ColourGradient(mask, psi, precision=prec, device=local, **kw) as s:
            s.step(20)
            s.step(steps - 20)
            ms = s.last_step_ms()
            out[prec] = (s.reduce(), ms / (steps - 20), s.count)
    clk.__exit__(None, None, None)
    if rank != 0:
        return 0
    (d32, ms32, n), (d64, ms64, _) = out["f32"], out["f64"]
    peak, peak_src = measured_peak()
    # FP32: colour pass 18*4 (table) + 8*4 (colour record) + 3*4 (rho_r, rho_b, psi);
    # collide pass 19*4 (f) + 18*4 (table) + 3*4 (psi, rho_r, rho_b) + 19*4 (f*) + 8*4 (record)
    cg_bytes = (72 + 32 + 12) + (19 * 4 + 72 + 12 + 19 * 4 + 32)
    achieved = n * cg_bytes / (ms32 * 1e-3) / 1e9
    line = {"metric": "colour-gradient fluid MLUPS (FP32)", "value": n / (ms32 * 1e-3) / 1e6, "unit": "MLUPS",
            "n_gpus": world, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "128^3 random cylinders r=3, porosity 0.6, blob phase field S_w=0.5, nu ratio 1, "
                                   "CapA=1e-3, psi_solid=cos45, " +
                                   ("Sub_BC 1 pressure faces rho 1.004 (x-) / 1.0 (x+), no body force" if a.cg_faces
                                    else "gx=1e-5 on the non-wetting phase"), "steps": steps,
                       "fluid_nodes": n},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_src, "bytes_per_lu": cg_bytes},
            "fp64_mlups": n / (ms64 * 1e-3) / 1e6,
            "saturation": {"f32": d32["saturation"], "f64": d64["saturation"]},
            "q_l_x": {"f32": d32["q_l"][0], "f64": d64["q_l"][0]},
            "q_g_x": {"f32": d32["q_g"][0], "f64": d64["q_g"][0]},
            "rel_err_vs_fp64": {"saturation": abs(d32["saturation"] - d64["saturation"]) / d64["saturation"],
                                "q_l": abs(d32["q_l"][0] - d64["q_l"][0]) / (abs(d64["q_l"][0]) + 1e-300),
                                "q_g": abs(d32["q_g"][0] - d64["q_g"][0]) / (abs(d64["q_g"][0]) + 1e-300)},
            "clocks": clk.summary()}
    emit(line)
    return 0


def run_solute(a):
    """D3Q7 solute transport on the config-2 geometry (256^3 spheres, 5.87 M
    fluid nodes) advected by the FP32 flow after 300 steps: solute MLUPS in
    FP32 and FP64, against the 2*6*s + 6*4 + 3*s bytes per update; the D3Q19
    solute step beside it (2*19*s + 18*4 + 3*s bytes per update)."""
    world, rank, local, pg = dist_setup()
    import lbm_b200

    mask = workload_mask()
    rng = np.random.default_rng(7)
    c0 = rng.uniform(0.0, 1.0, mask.shape)
    steps = max(a.steps // 4, 50)
    out = {}
    clk = ClockSampler(local).__enter__()
    with lbm_b200.SinglePhase(mask, NU, (GX, 0.0, 0.0), precision="f32", device=local) as flow:
        flow.step(300)
        for lat in (7, 19):
            for prec in ("f32", "f64"):
                with lbm_b200.Solute(None, c0, 0.01, flow=flow, precision=prec, device=local, lattice=lat) as s:
                    s.step(a.warmup)
                    s.step(steps)
                    key = prec if lat == 7 else f"{prec}_q19"
                    out[key] = (s.last_step_ms() / steps, s.count, float(s.concentration()[1:].sum()))
    clk.__exit__(None, None, None)
    if rank != 0:
        return 0
    peak, peak_src = measured_peak()
    (ms32, n, m32), (ms64, _, m64) = out["f32"], out["f64"]
    b32, b64 = 2 * 6 * 4 + 6 * 4 + 3 * 4, 2 * 6 * 8 + 6 * 4 + 3 * 8
    line = {"metric": "D3Q7 solute MLUPS (FP32)", "value": n / (ms32 * 1e-3) / 1e6, "unit": "MLUPS",
            "n_gpus": world, "higher_is_better": True, "dtype": "f32", "data": "synthetic", "steps": steps,
            "warmup": a.warmup,
            "config": {"workload": "256^3 overlapping spheres r=U[4,10], phi=0.35 (config-2 geometry), D=0.01, "
                                   "velocity of the FP32 flow after 300 steps", "fluid_nodes": n},
            "roofline": {"bound": "hbm", "achieved": n * b32 / (ms32 * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": n * b32 / (ms32 * 1e-3) / 1e9 / peak, "traffic": None, "peak_source": peak_src,
                         "bytes_per_lu": b32},
            "fp64": {"mlups": n / (ms64 * 1e-3) / 1e6, "gbs": n * b64 / (ms64 * 1e-3) / 1e9, "bytes_per_lu": b64},
            "mass_rel_diff_f32_vs_f64": abs(m32 - m64) / abs(m64), "clocks": clk.summary()}
    (q32, _, n32), (q64, _, n64) = out["f32_q19"], out["f64_q19"]
    c32, c64 = 2 * 19 * 4 + 18 * 4 + 3 * 4, 2 * 19 * 8 + 18 * 4 + 3 * 8
    line["d3q19"] = {"what": "the D3Q19 solute program's step (lbm_st19_create_from_flow), same flow and C0",
                     "f32": {"mlups": n / (q32 * 1e-3) / 1e6, "gbs": n * c32 / (q32 * 1e-3) / 1e9,
                             "frac": n * c32 / (q32 * 1e-3) / 1e9 / peak, "bytes_per_lu": c32},
                     "fp64": {"mlups": n / (q64 * 1e-3) / 1e6, "gbs": n * c64 / (q64 * 1e-3) / 1e9,
                              "frac": n * c64 / (q64 * 1e-3) / 1e9 / peak, "bytes_per_lu": c64},
                     "mass_rel_diff_f32_vs_f64": abs(n32 - n64) / abs(n64)}
    emit(line)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cg-steps", type=int, default=20000)
    ap.add_argument("--cg-faces", action="store_true", help="cg: pressure faces on x instead of the body force")
    ap.add_argument("--workload", default="cfg2", choices=["cfg2", "cfg2-accuracy", "batch", "serve", "cg", "solute"],
                    help="cfg2 = the headline single-domain bench; cfg2-accuracy = its FP32 error against the "
                         "bit-exact FP64 kernel at the stop test; batch / serve = configs 4 / 5")
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--instances", type=int, default=64, help="batch: number of config-4 solves")
    ap.add_argument("--batch-block", type=int, default=0, help="batch: fixed block size, reference order (0 = autotune)")
    ap.add_argument("--rate", type=float, default=8.0)
    ap.add_argument("--policy", default="fifo", choices=["fifo", "shortest"], help="serve: admission order")
    ap.add_argument("--pool-nodes", type=int, default=96 * 1024 * 1024)
    ap.add_argument("--fp64-sample", type=int, default=6)
    ap.add_argument("--target-nodes", type=int, default=1024 * 1024,
                    help="serve: resident-node target (0 = admit while memory allows)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cpu-calibration", action="store_true",
                    help="skip the one-process full-domain vs sub-block reference timing")
    ap.add_argument("--calib-steps", type=int, default=2)
    ap.add_argument("--precisions", default="f32,f64",
                    help="cfg2-accuracy: storage kinds run to the stop test (f64 = the bit-exact kernel, the anchor)")
    ap.add_argument("--max-steps", type=int, default=200000, help="cfg2-accuracy: step cap of each solve")
    ap.add_argument("--ordering", default="reference", choices=["auto", "reference", "morton", "hilbert", "brick"],
                    help="node order of the timed solve; auto = lbm_autotune (short trials at burst clocks)")
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--skip-e2e", action="store_true", help="profiling runs: no end-to-end pass")
    a = ap.parse_args()
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "batch":
        return run_batch(a)
    if a.workload == "serve":
        return run_serve(a)
    if a.workload == "cg":
        return run_cg(a)
    if a.workload == "cfg2-accuracy":
        return run_cfg2_accuracy(a)
    if a.workload == "solute":
        return run_solute(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())

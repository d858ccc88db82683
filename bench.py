#!/usr/bin/env python
"""SDOT serving benchmark: Newton solves/s and p50/p99 latency, batched vs the plain one-at-a-time GPU solve,
every solve to max |m - nu| / nu <= 1e-8.

Workload: the serving stream -- requests with Poisson arrivals, dimension 2 (70 %) or 3 (30 %), N log-uniform
in [1e3, 2e5], Diracs uniform in the unit box, target uniform or a 4-gaussian mixture (50/50; centres
U[0.2, 0.8]^d, sigma U[0.05, 0.15], equal masses, support clipped to the unit box), nu = 1/N.  Seeded
synthetic inputs; a STEP is one slice of `--requests-per-step` requests of that stream.  Requests this build
cannot solve (recorded in `config.skipped`) are left out of the stream before it is sliced.

  value      solves/s of the batched engine (sdot_solve_batch) on a step's requests, inputs already resident
             in HBM, CUDA events on the library's stream, max over ranks;
  e2e        solves/s of the served stream (sdot_server_*: host buffers in and out, continuous batching),
             arrivals at rate lambda = 2 x the plain solves/s, with p50 / p99 latency (arrival -> result);
  plain_gpu  solves/s of the one-at-a-time GPU solve (sdot_solve per request, host buffers).

Multi-GPU: replicas only (each rank owns its own slice of the stream, no collective on the data path).
`--impl reference` times the CPU oracle (the restatement of the reference's algorithm) instead.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sdot-ffi_b200"))

METRIC = "SDOT Newton solves/s + p50/p99 latency, batched vs plain GPU, mass err ≤1e-8"
RTOL = 1e-8
BYTES_PER_CELL = {2: 96.0, 3: 188.0}      # compulsory bytes of one cell per diagram (seed, weight, mass, centroid, upper facets)
# the statuses of a solve that met its tolerance: "converged", and "converged (aggregated)" -- the reference's `converged`
# (SdotPlanNd.py:984-988): seeds the doubles cannot separate meet it as clusters; the timed steps list those requests
CONVERGED = (1, 7)
AGGREGATED = []


def request(seed, k):
    """request k of the stream: (d, n, kind, gaussian params, arrival gap)"""
    rng = np.random.default_rng([seed, k])
    d = 2 if rng.uniform() < 0.7 else 3
    n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e5)))))
    gauss = rng.uniform() < 0.5
    c = rng.uniform(0.2, 0.8, size=(4, d))
    s = rng.uniform(0.05, 0.15, size=4)
    return dict(k=k, d=d, n=n, gauss=gauss, c=c, s=s, gap=rng.exponential())


def positions(seed, req):
    return np.random.default_rng([seed, req["k"], 1]).uniform(size=(req["n"], req["d"]))


def target_of(req):
    import sdot
    d = req["d"]
    if req["gauss"]:
        return sdot.SumOfGaussians(req["c"], req["s"], np.full(4, 0.25), support_box=(np.zeros(d), np.ones(d)))
    return sdot.Box(nb_dims=d)


def capabilities():
    """which (d, gaussian) kinds this build solves, probed on a tiny diagram"""
    import sdot
    caps = {}
    rng = np.random.default_rng(0)
    for d in (2, 3):
        for g in (False, True):
            r = dict(d=d, gauss=g, c=rng.uniform(0.2, 0.8, size=(4, d)), s=np.full(4, 0.1))
            try:
                sdot.PowerDiagram(rng.uniform(size=(16, d)), distribution=target_of(r)).measures
                caps[(d, g)] = True
            except NotImplementedError:
                caps[(d, g)] = False
    return caps


def stream(seed, count, probe):
    out, skipped, k = [], 0, 0
    while len(out) < count:
        r = request(seed, k)
        k += 1
        if probe(r):
            out.append(r)
        else:
            skipped += 1
    return out, skipped


def sixteen_gaussians_image(rng, res=1024):
    """the image target of the 2D Newton workload: 16 isotropic gaussians (centres uniform, sigma uniform in [0.02, 0.1],
    amplitudes uniform in [0.5, 2]) at the pixel centres of [0,1]^2, plus 1 % of the peak"""
    c = rng.uniform(size=(16, 2))
    s = rng.uniform(0.02, 0.1, size=16)
    a = rng.uniform(0.5, 2.0, size=16)
    xs = (np.arange(res) + 0.5) / res
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    v = np.zeros((res, res))
    for k in range(16):
        v += a[k] * np.exp(-((X - c[k, 0]) ** 2 + (Y - c[k, 1]) ** 2) / (2 * s[k] ** 2))
    return v + 0.01 * v.max()


def settings():
    from sdot import Iterative, Tuning
    return Iterative(tol=0.0, on_failure="ignore", tuning=Tuning(mass_rtol=RTOL))


# ---- clocks during a timed region ---------------------------------------------------------------------------------------------
class Clocks:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


# ---- the GPU arm ---------------------------------------------------------------------------------------------------------
def device_batch(reqs, seed, torch):
    """the step's inputs resident on the device, and the descriptors pointing at them"""
    import ctypes
    from sdot import _lib
    from sdot.PowerDiagram import _domain_box
    from sdot.SdotPlanNd import solver_options
    keep, descs, outs, h2d = [], (_lib.SolveDesc * len(reqs))(), (_lib.SolveOut * len(reqs))(), 0
    opts = solver_options(settings(), 0)
    for k, r in enumerate(reqs):
        pos = torch.from_numpy(positions(seed, r)).cuda()
        h2d += pos.numel() * 8
        t = target_of(r).normalized_version(nb_dims=r["d"])
        lo, hi = _domain_box(t.bounding_half_spaces(), r["d"])
        dens = t._sdot_density()
        dev = []
        if dens[0] == "gauss":
            arrs = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda() for a in dens[1:]]
            dev = arrs
            h2d += sum(a.numel() * 8 for a in arrs)
        sd = _lib.SolveDesc()
        sd.diagram.dim, sd.diagram.n = r["d"], r["n"]
        sd.diagram.positions = pos.data_ptr()
        sd.diagram.weights = None
        for a in range(r["d"]):
            sd.diagram.box_lo[a], sd.diagram.box_hi[a] = float(lo[a]), float(hi[a])
        D = _lib.Density()
        if dens[0] == "uniform":
            D.kind, D.value = _lib.DENSITY_UNIFORM, float(dens[1])
        else:
            D.kind, D.count = _lib.DENSITY_GAUSSIANS, 4
            D.centres, D.sigmas, D.masses = dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr()
        sd.diagram.density = D
        sd.diagram.memory = _lib.SDOT_DEVICE
        sd.nu = None
        for q, name in enumerate(_lib.OPTIONS):
            sd.options[q] = float(opts[name])
        descs[k] = sd
        o = dict(w=torch.empty(r["n"], dtype=torch.float64, device="cuda"), m=torch.empty(r["n"], dtype=torch.float64, device="cuda"),
                 b=torch.empty(r["n"] * r["d"], dtype=torch.float64, device="cuda"), c=torch.empty(1, dtype=torch.float64, device="cuda"))
        so = _lib.SolveOut()
        so.weights, so.masses, so.barycentres, so.cost = o["w"].data_ptr(), o["m"].data_ptr(), o["b"].data_ptr(), o["c"].data_ptr()
        outs[k] = so
        keep.append((pos, dev, o))
    return descs, outs, keep, h2d


def run_value_step(reqs, seed, torch, check):
    """one timed step of the batched engine on device-resident inputs: (seconds, launches)"""
    import ctypes
    from sdot import _lib
    L = _lib.load()
    ctx = _lib.context()
    descs, outs, keep, _ = device_batch(reqs, seed, torch)
    stream = torch.cuda.ExternalStream(_lib.stream())
    torch.cuda.synchronize()
    l0 = _lib.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sts = (_lib.Status * len(reqs))()
    code = L.sdot_solve_batch(ctx, len(reqs), descs, outs, sts)
    e1.record(stream)
    torch.cuda.synchronize()
    if code != 0:
        raise RuntimeError(f"sdot_solve_batch: {[s.message for s in sts if s.code][:1]}")
    secs = e0.elapsed_time(e1) / 1000
    worst, failed = 0.0, []
    for r, (_, _, o), so in zip(reqs, keep, outs):
        st = np.array(so.stats[:])
        if st[0] not in CONVERGED:
            failed.append((r["k"], int(st[0])))
            continue
        if st[0] == 7:                  # converged on the clusters of seeds the doubles cannot separate: their masses, not each cell's
            AGGREGATED.append((r["k"], float(st[29] * r["n"] / st[12]) if st[12] > 0 else None))
            continue
        m = o["m"].cpu().numpy()
        worst = max(worst, float(np.abs(m * r["n"] / st[12] - 1).max()) if st[12] > 0 else 1.0)
    if check and failed:
        print(f"warning: requests (k, status) that did not converge: {failed}", file=sys.stderr)
    return secs, _lib.kernel_launches() - l0, worst, failed


def run_plain(reqs, seed, keep_per_dim=4):
    """one-at-a-time GPU solves through the public API (host arrays): seconds, worst mass error, failures, and the fitted
    weights of the first `keep_per_dim` converged requests of each dimension ([(request, weights)])"""
    from sdot import OtProblem, SumOfDiracs
    from sdot.SdotPlanNd import SdotPlanNd
    t0 = time.perf_counter()
    worst, failed, fits = 0.0, 0, []
    for r in reqs:
        plan = OtProblem(SumOfDiracs(positions(seed, r)), target_of(r)).solve(settings())
        if not plan.converged:
            failed += 1
            continue
        if plan.stats["status"] == "converged":
            worst = max(worst, float(np.abs(plan.cell_masses / plan.target_masses - 1).max()))
        if sum(1 for q, _ in fits if q["d"] == r["d"]) < keep_per_dim:
            fits.append((r, np.asarray(plan.weights, dtype=np.float64)))
    return time.perf_counter() - t0, worst, failed, fits


def gather_model(fits, dim, seed):
    """the neighbour search's record reads per cell, from the device counters (sdot_context_set_counters), on one diagram at
    the fitted weights of the kept requests of dimension `dim` (untimed, after the timed legs).  These reads mostly hit L2:
    the bytes they add to the compulsory ones are a second denominator of the cell kernel's roofline, not DRAM traffic."""
    from sdot import PowerDiagram, _lib
    sel = [(r, w) for r, w in fits if r["d"] == dim]
    if not sel:
        return None
    _lib.gather_counters(dim, reset=True)
    _lib.set_counters(True)
    try:
        for r, w in sel:
            t = target_of(r).normalized_version(nb_dims=dim)
            PowerDiagram(positions(seed, r), w, boundaries=t.bounding_half_spaces(), distribution=t).measures
    finally:
        _lib.set_counters(False)
    c = _lib.gather_counters(dim, reset=True)
    cells = max(c["cells"], 1)
    per = {k: c[k] / cells for k in ("candidates", "grid_cells", "grid_ranges", "nodes")}
    rec = 8.0 * (dim + 1)              # a seed (position + weight) or a pyramid node (affine majorant)
    extra = per["candidates"] * rec + per["grid_cells"] * 8 + per["grid_ranges"] * 8 + per["nodes"] * rec
    return {"per_cell": {k: round(v, 2) for k, v in per.items()}, "bytes_per_cell": BYTES_PER_CELL[dim] + extra,
            "sample": f"one diagram at the fitted weights of {len(sel)} timed {dim}D requests (k = {[r['k'] for r, _ in sel]}, "
                      f"{c['cells']} cells), counted by the kernel's counting instantiation"}


def run_served(reqs, seed, lam):
    """the stream through the server: arrivals at rate `lam`; returns (seconds, latencies, h2d, d2h, worst, counters)"""
    from sdot.server import Server
    pos = [positions(seed, r) for r in reqs]
    tg = [target_of(r) for r in reqs]
    gaps = np.array([r["gap"] for r in reqs]) / lam
    arrivals = np.cumsum(gaps) - gaps[0]
    h2d = sum(p.nbytes for p in pos) + sum(32 * 4 * (r["d"] + 2) if r["gauss"] else 0 for r in reqs)
    d2h = sum(r["n"] * (2 + r["d"]) * 8 + 8 + 31 * 8 for r in reqs)
    done, lat, worst, failed = {}, [], [0.0], [0]
    with Server(max_active=0) as srv:
        tickets = [None] * len(reqs)
        start = time.perf_counter()

        def collect():
            for i in range(len(reqs)):
                while tickets[i] is None:
                    time.sleep(0.0002)
                res = srv.result(tickets[i])
                now = time.perf_counter() - start
                done[i] = now
                lat.append(now - arrivals[i])
                st = res["stats"]
                if st[0] not in CONVERGED:
                    failed[0] += 1
                    continue
                if st[0] == 1:
                    worst[0] = max(worst[0], float(np.abs(res["masses"] * reqs[i]["n"] / st[12] - 1).max()) if st[12] > 0 else 1.0)

        th = threading.Thread(target=collect)
        th.start()
        for i, r in enumerate(reqs):
            wait = arrivals[i] - (time.perf_counter() - start)
            if wait > 0:
                time.sleep(wait)
            tickets[i] = srv.submit(pos[i], tg[i], settings=settings())
        th.join()
        counters = srv.counters()
    return max(done.values()), np.array(lat), h2d, d2h, worst[0], counters, failed[0]


# ---- the CPU legs: the oracle in worker processes under hard wall limits ---------------------------------------------------
# measured oracle cost per seed of one solve (8 threads): 2D uniform ~40 us, 3D uniform ~110 us, 2D gaussians ~1.5 ms
# (13 continuation stages); 3D gaussians ~1 s (adaptive tetrahedral quadrature: 956 s for one solve of 1,000 seeds)


def cpu_worker(seed, ks):
    """(child process) the oracle's solve of each request k of `ks` in turn: a line when a solve starts, one when it ends"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    print(json.dumps({"threads": O.max_threads()}), flush=True)
    for k in ks:
        r = request(seed, k)
        t = target_of(r).normalized_version(nb_dims=r["d"])
        dens = t._sdot_density()
        od = ("uniform", dens[1]) if dens[0] == "uniform" else ("gauss", dens[1], dens[2], dens[3])
        lo, hi = t.box() if hasattr(t, "box") else (np.zeros(r["d"]), np.ones(r["d"]))
        print(json.dumps({"start": k}), flush=True)
        t0 = time.perf_counter()
        s = O.solve(positions(seed, r), box=(lo, hi), density=od, tol_abs=0.0, tol_rel=RTOL, lin_tol=1e-8, agg_margin=4.0)
        print(json.dumps({"k": k, "n": r["n"], "secs": time.perf_counter() - t0, "ok": s["stats"]["status"] in CONVERGED}), flush=True)


def cpu_sample(reqs, seed, budget_s=20.0, cap_s=5.0):
    """the oracle (the CPU restatement of the reference's algorithm) on a seeded random sample of `reqs` -- every kind and
    size of the stream, none left out -- each request solved in a worker process under a hard limit of `cap_s` seconds,
    the whole leg under `budget_s` of wall time.  A request past its limit is killed and counted unsolved with the limit
    as its time (it would take longer): value = solves that met the tolerance / seconds of the sampled requests, an UPPER
    bound of the CPU's throughput on this mix"""
    order = [reqs[i] for i in np.random.default_rng([seed, 7]).permutation(len(reqs))]
    todo = [r["k"] for r in order]
    by_k = {r["k"]: r for r in order}
    rows, threads, t_start = [], [None], time.perf_counter()
    while todo and time.perf_counter() - t_start < budget_s:
        cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", ",".join(map(str, todo)), "--seed", str(seed)]
        proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        cur = [None, 0.0]                   # the request being solved, and when it started
        lock = threading.Lock()

        def read():
            for line in proc.stdout:
                try:
                    d = json.loads(line)
                except ValueError:
                    continue
                with lock:
                    if "threads" in d:
                        threads[0] = d["threads"]
                    elif "start" in d:
                        cur[0], cur[1] = d["start"], time.perf_counter()
                    else:
                        rows.append(dict(d, capped=False))
                        todo.remove(d["k"])
                        cur[0] = None

        th = threading.Thread(target=read, daemon=True)
        th.start()
        killed = None
        while proc.poll() is None:
            time.sleep(0.02)
            with lock:
                over_cap = cur[0] is not None and time.perf_counter() - cur[1] > cap_s
                over_budget = time.perf_counter() - t_start > budget_s
                if over_cap or over_budget:
                    killed = (cur[0], time.perf_counter() - cur[1]) if cur[0] is not None else None
                    proc.kill()
        proc.wait()
        th.join(timeout=5)
        if killed is not None:
            k, el = killed
            rows.append(dict(k=k, n=by_k[k]["n"], secs=min(el, cap_s), ok=False, capped=True))
            todo.remove(k)
        if killed is None and proc.returncode not in (0, None) and not rows:
            break
    secs = sum(d["secs"] for d in rows)
    solved = sum(1 for d in rows if d["ok"])
    kinds = {}
    for d in rows:
        r = by_k[d["k"]]
        key = f"{r['d']}D {'gaussian' if r['gauss'] else 'uniform'}"
        e = kinds.setdefault(key, [0, 0, 0])
        e[0] += 1
        e[1] += bool(d["ok"])
        e[2] += bool(d["capped"])
    desc = ", ".join(f"{k}: {v[0]} ({v[1]} solved, {v[2]} past the limit)" for k, v in sorted(kinds.items()))
    return dict(value=solved / secs if secs > 0 else None, unit="solves/s", cores=threads[0] or os.cpu_count(), kind="port",
                sample=f"{len(rows)} requests drawn at random from the timed ones ({desc}; sum N = {sum(d['n'] for d in rows)}), each "
                       f"solved under a {cap_s:.0f} s limit within a {budget_s:.0f} s leg; a request past its limit counts as unsolved "
                       f"with the limit as its time, so the value is an upper bound of the CPU's solves/s on this mix. "
                       f"oracle/sdot_oracle.c FP64 + OpenMP, same tolerance: the CPU restatement of sdot's algorithm, not the "
                       f"reference binary")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_of(kernel, cells_per_launch):
    """DRAM bytes per launch of `kernel`: the per-cell traffic of the committed ncu capture (a smaller case, see
    profiles/), scaled to this run's cells per launch"""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            rec = json.load(f).get(kernel)
        return None if rec is None else rec["bytes_per_cell"] * cells_per_launch
    except (OSError, ValueError, KeyError, TypeError):
        return None


def rank_share(reqs, rank, world):
    """the requests of one rank: every world-th of the stream from its rank on, so the ranks' shares are disjoint,
    cover the stream, and hold the same mix of kinds and sizes"""
    return reqs[rank::world]


def over_ranks(secs, nfail, dist, device):
    """the timed seconds as the max over the ranks and the unconverged solves summed over them; every rank takes both
    collectives, in this order"""
    import torch
    t = torch.tensor([secs], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    f = torch.tensor([float(nfail)], dtype=torch.float64, device=device)
    dist.all_reduce(f, op=dist.ReduceOp.SUM)
    return float(t.item()), int(f.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--requests-per-step", type=int, default=8)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--cpu-budget", type=float, default=30.0, help="wall limit (s) of the GPU arm's CPU-baseline leg")
    ap.add_argument("--cpu-cap", type=float, default=10.0, help="wall limit (s) of one request's CPU solve (GPU arm's CPU leg)")
    ap.add_argument("--ref-budget", type=float, default=150.0, help="wall limit (s) of the reference arm's CPU solves")
    ap.add_argument("--ref-cap", type=float, default=15.0, help="wall limit (s) of one request's CPU solve (reference arm)")
    ap.add_argument("--cpu-worker", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cells-only", type=int, default=0, help="diagrams of this many uniform seeds (for a profiler), then exit")
    ap.add_argument("--cells-dim", type=int, default=2)
    ap.add_argument("--cells-repeat", type=int, default=0)
    ap.add_argument("--cells-density", default="uniform", choices=["uniform", "gauss", "image16"],
                    help="cells-only / solve-only target: uniform, a 4-gaussian mixture like the stream's, or (2D solve-only) the "
                         "1024 x 1024 image of 16 gaussians plus a 1 %% floor")
    ap.add_argument("--solve-only", type=int, default=0, help="one solve of this many uniform seeds (for a profiler), then exit")
    ap.add_argument("--value-only", action="store_true", help="the warm-up and timed batched steps alone, one short line (for a profiler)")
    ap.add_argument("--solve-linear", default="auto", choices=["auto", "cg", "mg"])
    ap.add_argument("--solve-step", default="auto", choices=["auto", "trials", "limits"])
    ap.add_argument("--solve-lin-precision", default="fp64", choices=["fp64", "mixed"])
    a = ap.parse_args()
    if a.cpu_worker is not None:
        cpu_worker(a.seed, [int(k) for k in a.cpu_worker.split(",") if k])
        return
    if a.solve_only:
        import sdot
        from sdot import Iterative, OtProblem, SumOfDiracs, Tuning, _lib
        d = a.cells_dim
        pos = np.random.default_rng(a.seed).uniform(size=(a.solve_only, d))
        dist = sdot.Box(nb_dims=d)
        if a.cells_density == "gauss":
            rq = request(a.seed, 0)
            dist = target_of(dict(rq, d=d, gauss=True, c=np.random.default_rng(a.seed + 2).uniform(0.2, 0.8, size=(4, d))))
        if a.cells_density == "image16":
            dist = sdot.Image(sixteen_gaussians_image(np.random.default_rng(a.seed + 3)), frame=[1 / 1024, 1 / 1024])
        _lib.set_timing(True)
        t0 = time.perf_counter()
        plan = OtProblem(SumOfDiracs(pos), dist).solve(Iterative(tol=0.0, tuning=Tuning(mass_rtol=RTOL, linear_solver=a.solve_linear,
                                                                                        step=a.solve_step,
                                                                                        linear_precision=a.solve_lin_precision)))
        secs = time.perf_counter() - t0
        st = plan.stats
        kst = _lib.kernel_stats()
        print(json.dumps({"solve_only": a.solve_only, "dim": d, "density": a.cells_density, "linear": a.solve_linear, "step": a.solve_step,
                          "lin_precision": a.solve_lin_precision,
                          "status": st["status"], "seconds": secs, "nb_iter": st["nb_iter"], "nb_diag": st["nb_diag"],
                          "lin_nb_iter": st["lin_nb_iter"], "kernel_ms": {k: round(v[0], 3) for k, v in kst.items()},
                          "kernel_launches": {k: v[1] for k, v in kst.items()}}))
        return
    if a.cells_only:
        import sdot
        from sdot import _lib
        d = a.cells_dim
        pos = np.random.default_rng(a.seed).uniform(size=(a.cells_only, d))
        w = np.random.default_rng(a.seed + 1).uniform(0, a.cells_only ** (-2.0 / d), size=a.cells_only)
        dist = None
        if a.cells_density == "gauss":
            rq = request(a.seed, 0)
            dist = target_of(dict(rq, d=d, gauss=True, c=np.random.default_rng(a.seed + 2).uniform(0.2, 0.8, size=(4, d))))
        pd = sdot.PowerDiagram(pos, w, boundaries=sdot.box_half_spaces(np.zeros(d), np.ones(d)), distribution=dist)
        m = pd.facets()
        _lib.set_timing(True)
        for _ in range(a.cells_repeat):
            pd.facets()
        ms, nl, units = _lib.kernel_stats()["cells2d" if d == 2 else "cells3d"]
        print(json.dumps({"cells_only": a.cells_only, "dim": d, "density": a.cells_density, "facets_per_cell": float(m[0].mean()), "launches": nl,
                          "ms_per_launch": ms / max(nl, 1), "ns_per_cell": 1e6 * ms / max(units, 1),
                          "algorithmic_GBps": units * BYTES_PER_CELL[d] / (ms / 1000) / 1e9 if ms else None}))
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    R = a.requests_per_step
    config = {"workload": "serving stream: Poisson arrivals, d=2 (70%) / 3 (30%), N log-uniform [1e3, 2e5], uniform or 4-gaussian "
                          "target (50/50), nu = 1/N, mass_rtol 1e-8",
              "requests_per_step": R, "seed": a.seed, "parallelism": f"replicas{world}" if world > 1 else "single",
              "l2": "inputs of a step (~R x 37k seeds x 1.2 KB of working set) exceed the 126 MB L2"}

    if a.impl == "reference":
        if rank != 0:
            return
        # the timed slices of the GPU arm's stream, solved by the oracle on every host core under a hard wall limit
        reqs, skipped = stream(a.seed, (a.warmup + a.steps) * R, lambda r: True)
        cpu = cpu_sample(reqs[a.warmup * R:], a.seed, budget_s=a.ref_budget, cap_s=a.ref_cap)
        v = cpu["value"]
        config["reference_step"] = f"a step's {R} requests at the measured CPU throughput (ms_per_step = R / value)"
        print(json.dumps({"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                          "ms_per_step": 1000.0 * R / v if v else None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f64", "data": "synthetic", "impl": "reference", "config": config,
                          "cpu_baseline": dict(cpu, value=v), "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                                                                      "d2h_bytes_per_step": 0}}))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    os.environ["SDOT_DEVICE"] = str(torch.cuda.current_device())
    from sdot import _lib

    caps = capabilities()

    def probe(r):
        return caps[(r["d"], r["gauss"])]

    total = (a.warmup + a.steps) * R * world
    reqs, skipped = stream(a.seed, total, probe)
    config["skipped"] = (f"{skipped} requests of kinds this build does not solve yet left out of the stream: "
                         + ", ".join(f"{d}D {'gaussian' if g else 'uniform'}" for (d, g), ok in caps.items() if not ok)) if skipped else "none"
    mine = rank_share(reqs, rank, world)
    warm, timed = mine[: a.warmup * R], mine[a.warmup * R:]

    legs = {}
    t_leg = time.perf_counter()
    # warm-up steps (untimed)
    for s in range(a.warmup):
        run_value_step(warm[s * R:(s + 1) * R], a.seed, torch, check=True)

    # the timed steps: batched engine, device-resident inputs
    _lib.set_timing(True)
    _lib.kernel_stats(reset=True)
    AGGREGATED.clear()
    secs, launches, worst, failed = 0.0, 0, 0.0, []
    with Clocks(torch.cuda.current_device()) as clk:
        for s in range(a.steps):
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            t, l, w, f = run_value_step(timed[s * R:(s + 1) * R], a.seed, torch, check=True)
            secs += t
            launches += l
            worst = max(worst, w)
            failed += f
    kst = _lib.kernel_stats()
    _lib.set_timing(False)
    legs["warmup_and_value"] = time.perf_counter() - t_leg
    if a.value_only:
        if rank == 0:
            print(json.dumps({"value_only": True, "value": (a.steps * R * world - len(failed)) / secs, "unit": "solves/s", "steps": a.steps,
                              "requests_per_step": R, "gpu_launches": int(launches),
                              "kernel_ms": {k: round(v[0], 3) for k, v in kst.items()}}))
        if world > 1:
            dist.destroy_process_group()
        return
    t_leg = time.perf_counter()
    # only the solves that reached the mass tolerance count
    nfail = len(failed)
    if world > 1:
        secs, nfail = over_ranks(secs, nfail, dist, "cuda")
    value = ( a.steps * R * world - nfail ) / secs

    # plain one-at-a-time on the same requests
    pr = timed
    p_secs, p_worst, p_failed, fits = run_plain(pr, a.seed)
    plain = (len(pr) - p_failed) / p_secs
    legs["plain"] = time.perf_counter() - t_leg
    t_leg = time.perf_counter()

    # served stream, arrivals at twice the plain throughput
    lam = 2.0 * plain
    e_secs, lat, h2d, d2h, e_worst, counters, e_failed = run_served(timed, a.seed, lam)
    e2e = (len(timed) - e_failed) / e_secs
    legs["served"] = time.perf_counter() - t_leg
    t_leg = time.perf_counter()

    hbm, peak_kind = peaks()
    # the dominant kernel of the timed region: the 2D or the 3D cells, whichever took more device time
    dom = 3 if kst["cells3d"][0] > kst["cells2d"][0] else 2
    ms, nl, units = kst[f"cells{dom}d"]
    cells_b = units * BYTES_PER_CELL[dom]
    achieved = cells_b / (ms / 1000) / 1e9 if ms > 0 else None
    cg_ms, cg_n, cg_rows = kst["cg"]
    gather = None
    if rank == 0 and achieved:
        try:
            gm = gather_model(fits, dom, a.seed)
            if gm is not None:
                ga = gm["bytes_per_cell"] * units / (ms / 1000) / 1e9
                gather = dict(gm, achieved=ga, frac=ga / hbm, unit="GB/s",
                              note="search reads counted on the device; they count L2-resident re-reads, not DRAM traffic")
        except Exception as e:          # a measurement aid: the line stands without it
            print(f"warning: gather model leg: {e}", file=sys.stderr)
    legs["gather"] = time.perf_counter() - t_leg
    t_leg = time.perf_counter()
    cpu = cpu_sample(timed, a.seed, a.cpu_budget, a.cpu_cap) if rank == 0 else None
    legs["cpu"] = time.perf_counter() - t_leg
    if rank != 0:
        dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1000 * secs / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config,
        "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d // max(1, a.steps), "d2h_bytes_per_step": d2h // max(1, a.steps),
                "p50_ms": float(np.percentile(lat, 50) * 1000), "p99_ms": float(np.percentile(lat, 99) * 1000), "lambda_per_s": lam,
                "max_active": counters["max_active"], "worst_mass_rel_err": e_worst, "unconverged": e_failed},
        "plain_gpu": {"value": plain, "unit": "solves/s", "requests": len(pr), "worst_mass_rel_err": p_worst, "unconverged": p_failed},
        "e2e_over_plain": e2e / plain,
        "worst_mass_rel_err": worst,
        "unconverged": {"count": nfail, "requests_status": failed[:16]},
        "aggregated": {"count": len(AGGREGATED), "requests_full_rel_err": AGGREGATED[:16]},
        "roofline": {"bound": "hbm", "kernel": f"cells{dom}d (k_cells{dom}d)", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm if achieved else None, "traffic": traffic_of(f"k_cells{dom}d", units / max(nl, 1)),
                     "peak_kind": peak_kind, "algorithmic_bytes_per_cell": BYTES_PER_CELL[dom], "cells_per_launch": units / max(nl, 1),
                     "avg_launch_ms": ms / max(nl, 1), "gather_model": gather, "cg_ms_share": cg_ms / max(1e-9, 1000 * secs),
                     "cells_ms_share": ms / max(1e-9, 1000 * secs),
                     "kernel_ms": {k: round(v[0], 3) for k, v in kst.items()},
                     "busy_share": sum(v[0] for v in kst.values()) / max(1e-9, 1000 * secs)},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "legs_wall_s": {k: round(v, 1) for k, v in legs.items()},
    }
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

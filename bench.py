"""Benchmark: converged isotherm points per second at 64^3 FP64.

Workload (the 64^3 configuration): the 276-atom cubic host (a = 17 A, seeded
random sequential addition, C:H:N:Zn = 96:120:48:12), united-atom methane,
T = 300 K, WBII + MFA + LJ external potential, 24 pressures log-spaced from
1e-3 to 100 bar, hybrid-Anderson (m = 5) to RES < 1e-8, started from
Ninit = rho_bulk (the reference notebook's start).  One step = one batched
solve of the whole isotherm.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--no-plain]

Prints one JSON line (rank 0).  `value` is device-resident throughput (the
functional and initial densities already on the GPU); `e2e` goes through the
public entry point solve_isotherm from host arrays (host atoms in, loadings
and densities out).  `--impl reference` times the numpy restatement of the
reference path (pinned against the reference) on the host cores.
Multi-GPU runs are replicas: every rank solves its own isotherm (weak scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NPTS = (64, 64, 64)
ROT_NPTS = (32, 32, 32)
NPRESS = 24
T = 300.0
THRESH = 1e-8
METRIC = "isotherm converged points/s at 64^3 FP64 (hybrid Anderson m=5, RES<1e-8)"
# the workload keys both arms report
ISOTHERM_CONFIG = {"workload": "isotherm-64cubed", "grid": list(NPTS), "host": "cubic a=17A 276 atoms seed 0",
                   "points_per_isotherm": NPRESS, "pressures_bar": [1e-3, 100.0], "solver": "hybridanderson m=5",
                   "tolerance": "RES<1e-8", "start": "Ninit=rho_bulk"}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "_fallback": True}


class ClockSampler(object):
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace('.', '').isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace('.', '').isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def ncu_traffic(plan):
    """DRAM bytes (read + write) of one captured pipeline launch, from the
    capture record committed beside the profile summaries: (bytes, want,
    instances), or None when there is no record for this grid."""
    fn = os.path.join(ROOT, "profiles", "pipeline_traffic_isotherm64.json")
    try:
        with open(fn) as f:
            rec = json.load(f)
    except (OSError, ValueError):
        return None
    if tuple(rec.get("grid", ())) != tuple(plan.npoints):
        return None
    return float(rec["dram_bytes"]), int(rec["want"]), int(rec["instances"])


def pipeline_bytes(plan, want, n_active):
    """Algorithmic HBM bytes of one functional-pipeline launch (3 kernels).

    S = one yz-spectrum of one instance (N1*N2*H3*16 B).  Column pass 1 reads
    rho_hat and writes 5 weighted-density spectra; the plane pass reads 5 and
    writes 5 dPhi spectra; column pass 2 reads 5 + rho_hat and writes the C1
    spectrum.  The MFA kernel spectrum (S) is read once per launch per pass
    that uses it.  Value-only launches (want & 1 == 0) skip the forward and the
    second column pass.  With want & 8 the plane pass also writes the 5
    weighted densities in real space (5 * N1*N2*N3*8 B).
    """
    S = plan.nspec * 16
    if want & 1:
        per = S * (1 + 5 + 5 + 5 + 5 + 1 + 1)
        shared = S * (2 if want & 2 else 1)
    else:
        per = S * (1 + 5 + 5)
        shared = S if want & 2 else 0
    if want & 8:
        per += 5 * plan.npts * 8
    return per * n_active + shared


def reduce_over_ranks(ms, nconv, world, device):
    """Max of the timed milliseconds and sum of converged points over ranks
    (replicas: no data-path collective; two scalars after the timed region)."""
    import torch
    if world <= 1:
        return float(ms), float(nconv)
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    nc = torch.tensor([float(nconv)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(nc, op=dist.ReduceOp.SUM)
    return float(t.item()), float(nc.item())


def setup_case(torch):
    from cmmdft_b200 import workload as W
    from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
    from cmmdft_b200.units import bar
    host = cubic_host_276(0)
    guest = methane_guest_params()
    pressures = np.logspace(-3, 2, NPRESS) * bar
    fn = W.build_functional(host, NPTS, T, guest)
    mus, bulks = W.isotherm_inputs(pressures, T, guest)
    return host, guest, pressures, fn, mus, bulks


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from cmmdft_b200 import batch as BT, workload as W, isotherm as ISO

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    host, guest, pressures, fn, mus, bulks = setup_case(torch)
    rho0 = W.initial_density(fn, mus, ninit=bulks)

    def one_solve(events=None, groups=None):
        s = BT.GroupedSolve(fn, mus, groups=args.groups if groups is None else groups, native=args.driver == "native", method="hybridanderson",
                            nsteps=args.max_iters,
                            threshold=THRESH, criterion="res", divergence_guard=True, anderson_coefs=args.coefs)
        s.pipeline_events = events
        N, rho, conv = s.solve(rho0)
        return s, conv

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        one_solve()
    events = []
    launches = 0
    nconv = 0
    iters = []
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(args.steps):
            s, conv = one_solve(events)
            launches += s.kernel_launches
            nconv += int(conv.sum())
            iters.append(int(s.steps.sum()))
            per_point = [int(x) for x in s.steps]
            diverged = [int(i) for i in np.where(s.diverged)[0]]
        e1.record()
        barrier()
    ms = e0.elapsed_time(e1)
    ms_max, nconv_all = reduce_over_ranks(ms, nconv, world, "cuda")
    value = nconv_all / (ms_max / 1e3)

    # roofline of the fused functional pipeline, from its events in the timed
    # region.  With concurrent groups a launch's events would also span the
    # other group's kernels, so the pipeline is then timed in a separate
    # pass of single-group solves (ms_ref: that pass's device time).
    ms_ref, n_rl = ms_max / args.steps, args.steps
    rl_pass = "timed region"
    if args.groups > 1:
        events = []
        nref = max(1, min(args.steps, 5))
        one_solve(None, groups=1)   # the single-group workspace, outside the pass
        barrier()
        e0.record()
        for _ in range(nref):
            one_solve(events, groups=1)
        e1.record()
        barrier()
        ms_ref, n_rl = e0.elapsed_time(e1) / nref, nref
        rl_pass = "%d single-group solves after the timed region" % nref
    tot_bytes = 0.0
    tot_ms = 0.0
    for a, b, want, nact in events:  # CUDA-event pairs (Python driver) or milliseconds (native driver)
        tot_ms += a.elapsed_time(b) if b is not None else a
        tot_bytes += pipeline_bytes(fn.plan, want, nact)
    pk = peaks()
    achieved = tot_bytes / (tot_ms / 1e3) / 1e9 if tot_ms > 0 else None
    # measured DRAM bytes per launch: the captured launch's bytes scaled by
    # the algorithmic bytes of the average timed launch
    cap = ncu_traffic(fn.plan)
    traffic = (cap[0] / pipeline_bytes(fn.plan, cap[1], cap[2]) * tot_bytes / len(events)) \
        if (cap and events) else None
    dram_gbs = traffic / (tot_ms / len(events) / 1e3) / 1e9 if (traffic and tot_ms > 0) else None
    roofline = {"bound": "hbm", "kernel": "functional pipeline (k_col_weights+k_plane_fmt+k_col_backconv)",
                "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": (achieved / pk["hbm_gbs"]) if achieved else None,
                "peak_source": "fallback" if pk.get("_fallback") else "measured",
                "traffic": traffic,
                "traffic_source": ("ncu DRAM bytes of one %d-instance launch (want %d), scaled by algorithmic bytes"
                                   % (cap[2], cap[1])) if cap else None,
                "dram_achieved": dram_gbs,
                "dram_frac": (dram_gbs / pk["hbm_gbs"]) if dram_gbs else None,
                "launches": len(events),
                "bytes_per_launch": tot_bytes / max(len(events), 1),
                "ms_per_launch": tot_ms / max(len(events), 1),
                "share_of_step": (tot_ms / n_rl) / ms_ref if ms_ref else None,
                "pass": rl_pass}

    # end to end through the public entry point (host arrays in, loadings + densities out)
    e2e = None
    if not args.no_e2e:
        out = None
        for _ in range(args.warmup):   # warm-up: pinned result buffers, plan tables, workspaces
            out = ISO.solve_isotherm(host, pressures, T, guest, NPTS, threshold=THRESH, groups=args.groups,
                                     native=args.driver == "native", anderson_coefs=args.coefs)
        barrier()
        t0 = time.perf_counter()
        h2d = d2h = 0
        ne = 0
        for _ in range(args.steps):
            out = ISO.solve_isotherm(host, pressures, T, guest, NPTS, threshold=THRESH, groups=args.groups,
                                     native=args.driver == "native", anderson_coefs=args.coefs)
            ne += int(out["converged"].sum())
            h2d += host.pos.nbytes + host.ffatype_ids.nbytes + 2 * 8 * len(host.ffatypes)
            d2h += out["rho"].nbytes + out["N"].nbytes
        barrier()
        dt = time.perf_counter() - t0
        dt_ms, ne = reduce_over_ranks(dt * 1e3, ne, world, "cuda")   # slowest rank, all ranks' points
        dt = dt_ms / 1e3
        e2e = {"value": ne / dt, "unit": "points/s", "h2d_bytes_per_step": h2d // args.steps,
               "d2h_bytes_per_step": d2h // args.steps,
               "includes": "EOS mu(P) + extpot + MFA kernel + solve + densities to pinned host memory"}

    plain = None
    if not args.no_plain and rank == 0:
        barrier()
        t0 = time.perf_counter()
        npl = 0
        pit = 0
        for i in range(NPRESS):
            cls = BT.NativeBatchSolve if args.driver == "native" else BT.BatchSolve
            s = cls(fn, mus[i:i + 1], method="hybridanderson", nsteps=args.max_iters,
                    threshold=THRESH, criterion="res", divergence_guard=True, anderson_coefs=args.coefs)
            N, rho, conv = s.solve(rho0[i:i + 1])
            npl += int(conv.sum())
            pit += int(s.steps.sum())
        torch.cuda.synchronize()
        dtp = time.perf_counter() - t0
        plain = {"value": npl / dtp, "unit": "points/s", "iterations": pit,
                 "batched_over_plain": value / (npl / dtp) / max(world, 1)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(one_point=True)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(ISOTHERM_CONFIG, instance_groups=args.groups, driver=args.driver,
                           anderson_coefs=args.coefs, iterations_per_isotherm=iters,
                           converged_points=nconv, steps_per_point=per_point, diverged_points=diverged,
                           divergence_note="points 21-23 (37-100 bar) diverge in the reference's own "
                                           "hybrid-Anderson from the Ninit=rho_bulk start; retired by the "
                                           "divergence guard",
                           parallelism="replicas" if world > 1 else "single",
                           l2="working set > L2 (24 x 2 MiB fields x ~30 live buffers)"),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "plain": plain,
            "gpu_launches": launches, "clocks": clk.summary()}
    print(json.dumps(line))


# ------------------------------------------------------------- CPU sides --
def _oracle_point(args):
    """One reference-path (numpy oracle) hybrid-Anderson solve at 64^3; returns (seconds, N, converged)."""
    idx, = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, ROOT)
    from oracle import cmm_oracle as O
    from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
    from cmmdft_b200.units import bar, kjmol
    host = cubic_host_276(0)
    sig, eps, mass = methane_guest_params()
    grid = O.OGrid(host.rvecs, npoints=list(NPTS))
    V = O.external_potential(grid.points[..., :3].reshape(-1, 3), host.ff, sig, eps, host.recentred_pos(),
                             host.ffatypes, host.ffatype_ids, host.rvecs).reshape(grid.npoints)
    V = O.cap_potential(V, 1e4 * kjmol)
    fe = O.build_functional(grid, sig, eps, mass, T, V)
    P = np.logspace(-3, 2, NPRESS)[idx] * bar
    mb = O.MBWR(mass, sig, eps)
    mu = O.eos_calculate_mu(mb, T, P)
    mb.set_temperature(T)
    rb = np.nanmin(O.eos_densities_from_chempots(mb, [mu]), axis=1)[0]
    rho0 = rb * np.exp(-np.maximum(V, 0) / (1.0 / fe.beta))
    t0 = time.perf_counter()
    s = O.Anderson(fe, nsteps=500, m=5, criterion="res", threshold=THRESH)
    N, rho, conv = s.solve(mu, rho0)
    return time.perf_counter() - t0, float(N), bool(conv), s.curr_step


def cpu_baseline_sample(one_point=True, nproc=1, points=None):
    """Time the numpy restatement of the reference path on host cores (spawned workers)."""
    import multiprocessing as mp
    if points is None:
        points = [NPRESS // 2]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        res = pool.map(_oracle_point, [(i,) for i in points])
    wall = time.perf_counter() - t0
    nconv = sum(1 for r in res if r[2])
    # points solved concurrently by nproc single-threaded processes: divide by
    # the longest per-process solve time (per-process setup excluded)
    per_proc = {}
    for i, r in enumerate(res):
        per_proc.setdefault(i % nproc, 0.0)
        per_proc[i % nproc] += r[0]
    solve_s = max(per_proc.values())
    return {"value": nconv / solve_s, "unit": "points/s", "cores": nproc,
            "kind": "port",
            "sample": "%d pressure point(s) %s of the 24-point 64^3 isotherm, numpy/scipy oracle "
                      "(pinned to the reference), scipy.fft workers=1, %d process(es); solve time only "
                      "(setup excluded), wall incl. setup %.1f s" % (len(points), points, nproc, wall),
            "iterations": [r[3] for r in res]}


_ORACLE = {}


def _oracle_init():
    """Worker set-up of the reference arm (once per process): the oracle's
    grid, external potential, functional and EOS of the 64^3 isotherm."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, ROOT)
    from oracle import cmm_oracle as O
    from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
    from cmmdft_b200.units import kjmol
    host = cubic_host_276(0)
    sig, eps, mass = methane_guest_params()
    grid = O.OGrid(host.rvecs, npoints=list(NPTS))
    V = O.external_potential(grid.points[..., :3].reshape(-1, 3), host.ff, sig, eps, host.recentred_pos(),
                             host.ffatypes, host.ffatype_ids, host.rvecs).reshape(grid.npoints)
    V = O.cap_potential(V, 1e4 * kjmol)
    _ORACLE.update(O=O, V=V, fe=O.build_functional(grid, sig, eps, mass, T, V), mb=O.MBWR(mass, sig, eps))


def _oracle_solve(idx):
    """One pressure point of the isotherm through the oracle in a set-up
    worker; returns (solve seconds, converged, steps)."""
    from cmmdft_b200.units import bar
    O, V, fe, mb = _ORACLE["O"], _ORACLE["V"], _ORACLE["fe"], _ORACLE["mb"]
    P = np.logspace(-3, 2, NPRESS)[idx] * bar
    mu = O.eos_calculate_mu(mb, T, P)
    mb.set_temperature(T)
    rb = np.nanmin(O.eos_densities_from_chempots(mb, [mu]), axis=1)[0]
    rho0 = rb * np.exp(-np.maximum(V, 0) / (1.0 / fe.beta))
    t0 = time.perf_counter()
    s = O.Anderson(fe, nsteps=500, m=5, criterion="res", threshold=THRESH)
    N, rho, conv = s.solve(mu, rho0)
    return time.perf_counter() - t0, bool(conv), s.curr_step


def _oracle_pid(_):
    time.sleep(0.2)
    return os.getpid()


def run_reference(args, budget_s=120.0):
    """The reference arm: the oracle (the reference's numpy path, pinned to
    it) on one process per host core (up to 21), each set up once; a step
    solves one pressure point per process (points cycling over the 21 the
    reference's algorithm converges; the top 3 diverge in it and would
    iterate to nsteps) and takes the wall time of the slowest (44 s on a
    16-core host).  At most one untimed warm-up step (numpy has nothing to
    warm beyond the set-up), then up to K timed steps, stopped once they
    pass ``budget_s`` (reported as steps and steps_requested)."""
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    try:
        ncores = len(os.sched_getaffinity(0))
    except Exception:
        ncores = os.cpu_count() or 1
    nproc = max(1, min(ncores, 21))
    ctx = mp.get_context("spawn")
    conv = 0
    iters = []
    t_setup = time.perf_counter()
    with ctx.Pool(nproc, initializer=_oracle_init) as pool:
        pids = set()   # every worker has run its set-up once it has answered
        while len(pids) < nproc and time.perf_counter() - t_setup < 600:
            pids.update(pool.map(_oracle_pid, range(nproc), chunksize=1))
        setup_s = time.perf_counter() - t_setup
        k = 0
        nwarm = min(1, max(0, args.warmup))
        for _ in range(nwarm):
            pool.map(_oracle_solve, [(k * nproc + i) % 21 for i in range(nproc)], chunksize=1)
            k += 1
        t0 = time.perf_counter()
        done = 0
        for _ in range(max(1, args.steps)):
            res = pool.map(_oracle_solve, [(k * nproc + i) % 21 for i in range(nproc)], chunksize=1)
            k += 1
            done += 1
            conv += sum(1 for r in res if r[1])
            iters += [r[2] for r in res]
            if time.perf_counter() - t0 > budget_s:
                break
        wall = time.perf_counter() - t0
    value = conv / wall
    sample = ("%d timed step(s) of %d pressure points each (one per process, cycling over the 21 points the "
              "reference's algorithm converges), numpy/scipy oracle pinned to the reference, scipy.fft workers=1 "
              "per process; per-process set-up (external potential, functional) once, %.1f s, outside the "
              "timed steps" % (done, nproc, setup_s))
    line = {"metric": METRIC, "value": value, "unit": "points/s", "n_gpus": 0, "steps": done,
            "warmup": nwarm, "ms_per_step": wall / done * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": dict(ISOTHERM_CONFIG, parallelism="%d host processes" % nproc),
            "cpu_baseline": {"value": value, "unit": "points/s", "cores": nproc, "kind": "port", "sample": sample,
                             "iterations": iters},
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if done < args.steps:
        line["steps_requested"] = args.steps
    print(json.dumps(line))


def run_uneven(args):
    """Secondary workload (not the headline line): 8 orthorhombic hosts with
    edges U(12, 40) A (seed 2), grids from a 0.25 A spacing (55-157 per axis),
    32 pressures 1e-3..100 bar each -- 256 solves through solve_batch, hosts
    concurrent on their own streams within a device-memory budget.  Timed by
    wall clock around the call with the device synchronised (the hosts run on
    several streams), after one untimed run."""
    import torch
    from cmmdft_b200 import isotherm as ISO
    from cmmdft_b200.hosts import uneven_hosts, methane_guest_params
    from cmmdft_b200.units import bar
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    hosts = uneven_hosts(8, 2)
    guest = methane_guest_params()
    P = np.logspace(-3, 2, 32) * bar
    schedules, tuning = None, None
    if args.autotune:
        from cmmdft_b200 import autotune as AT
        from cmmdft_b200.isotherm import grid_points
        t0 = time.perf_counter()
        schedules, tuning = [], []
        for h in hosts:
            shape = grid_points(h)
            best, table = AT.tune(shape, h.rvecs, batch=4)
            default = [t for t in table if t[0] == [0, 0, 0, -1, 0]]
            d_ms = default[0][2] if default else None
            npts = float(np.prod(shape))
            schedules.append(best)
            tuning.append({"grid": list(shape), "schedule": best, "radices": table[0][1],
                           "ns_per_point": table[0][2] * 1e6 / (4 * npts),
                           "default_ns_per_point": d_ms * 1e6 / (4 * npts) if d_ms else None,
                           "candidates": len(table)})
        tune_s = time.perf_counter() - t0
    ISO.solve_batch(hosts, P, T, guest, schedules=schedules)
    times, nconv, steps = [], 0, 0
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = ISO.solve_batch(hosts, P, T, guest, schedules=schedules)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        nconv += sum(int(r['converged'].sum()) for r in res)
        steps = sum(int(r['steps'].sum()) for r in res)
    dt = sum(times)
    line = {"metric": "uneven multi-host batch converged points/s (FP64, RES<1e-8)", "value": nconv / dt,
            "unit": "points/s", "n_gpus": 1, "steps": len(times), "warmup": 1, "ms_per_step": dt / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "uneven-8-hosts", "grids": [list(r['npoints']) for r in res],
                       "atoms": [int(h.natom) for h in hosts], "pressures_per_host": len(P),
                       "solves": len(P) * len(hosts), "converged_per_run": nconv // len(times),
                       "solver_steps_per_run": steps, "timing": "wall clock, device synchronised"}}
    if tuning is not None:
        line["config"]["fft_schedules"] = tuning
        line["config"]["autotune_s"] = tune_s
        line["config"]["schedule_note"] = ("per grid: the fastest of the candidate FFT schedules for one C1 "
                                           "evaluation of 4 instances (ns per grid point and instance), "
                                           "and the default schedule's time")
    print(json.dumps(line))


def run_gradient(args):
    """Secondary workload (not the headline line): the differentiation case --
    96^3 host (a = 24 A, 779 atoms), 16-point excess isotherm 0.01-10 bar,
    squared error against a target from +-10% perturbed LJ parameters (seed
    3), gradient with respect to the 10 parameters through the autograd
    function (forward solve + implicit adjoint).  Wall clock with the device
    synchronised; the central-difference cost is stated as 2 x 10 forward
    solves, not run."""
    import torch
    from cmmdft_b200 import adjoint as A
    from cmmdft_b200.hosts import cubic_host_779, methane_guest_params
    from cmmdft_b200.units import bar
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    model = A.IsothermModel(cubic_host_779(0), methane_guest_params(), T, (96, 96, 96),
                            np.logspace(-2, 1, 16) * bar, quantity="excess", threshold=1e-12, criterion="riue")
    th0 = model.theta0
    target_theta = th0 * (1 + np.random.default_rng(3).uniform(-0.1, 0.1, th0.shape))
    with torch.no_grad():
        target = model(torch.as_tensor(target_theta)).clone()
    fw, bw = [], []
    for _ in range(max(1, min(args.steps, 3))):
        theta = torch.tensor(th0.copy(), requires_grad=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = ((model(theta) - target) ** 2).sum()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        fw.append(t1 - t0)
        bw.append(t2 - t1)
    f_ms, b_ms = 1e3 * float(np.median(fw)), 1e3 * float(np.median(bw))
    line = {"metric": "excess-isotherm loss gradient, 10 LJ parameters, 96^3 FP64 (ms per gradient)",
            "value": f_ms + b_ms, "unit": "ms", "n_gpus": 1, "steps": len(fw), "warmup": 1,
            "ms_per_step": f_ms + b_ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "gradient-96cubed", "grid": [96, 96, 96], "atoms": 779, "pressures": 16,
                       "parameters": int(len(th0)), "tolerance": "RIUE<1e-12", "forward_ms": f_ms,
                       "adjoint_ms": b_ms, "central_difference_ms_estimate": 2 * len(th0) * f_ms,
                       "timing": "wall clock, device synchronised, median"}}
    print(json.dumps(line))


def run_large(args):
    """Secondary workload (not the headline line): the large-cell WDA case --
    cubic a = 64 A host (14,680 atoms, seed 4), 256^3 FP64 grid, WBII + MFA +
    the WDA correlation part + LJ external potential, 16 pressures
    1e-3..100 bar from Ninit = rho_bulk, hybrid Anderson m=5 to RES < 1e-8.
    The external potential (cell-list kernel, CUDA events) and the batched
    solve (CUDA events, inputs resident) are timed separately; the 16
    instances run as one batch when they fit in 85% of free device memory,
    else as sequential batches."""
    import torch
    from cmmdft_b200 import batch as BT, engine as E, workload as W
    from cmmdft_b200.hosts import cubic_host_64, methane_guest_params
    from cmmdft_b200.units import bar, angstrom, kjmol
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    host = cubic_host_64()
    guest = methane_guest_params()
    npts = (256, 256, 256)
    P = np.logspace(-3, 2, 16) * bar
    plan = E.GridPlan(npts, host.rvecs)
    sig, eps = W.host_type_arrays(host)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ext_ms = []
    for _ in range(2):
        ev[0].record()
        E.external_potential(plan, host.recentred_pos(), host.ffatype_ids, sig, eps, guest[0], guest[1],
                             12 * angstrom, 1e4 * kjmol)
        ev[1].record()
        torch.cuda.synchronize()
        ext_ms.append(ev[0].elapsed_time(ev[1]))
    fn = W.build_functional(host, npts, T, guest, wda=True, plan=plan)
    mus, bulks = W.isotherm_inputs(P, T, guest)
    n = int(np.prod(npts))
    S = plan.nspec * 2
    m, nwd = 5, fn.nwd
    per = 8 * ((2 * m + 3) * n + (17 + m) * S + (m + 1) * nwd * n + 2 * S)   # workspace of one instance
    free, _ = torch.cuda.mem_get_info()
    bmax = max(1, int(0.85 * free // per))
    nb = -(-len(P) // bmax)
    chunks = np.array_split(np.arange(len(P)), nb)

    def solve_all():
        out = []
        for idx in chunks:
            r0 = W.initial_density(fn, mus[idx], ninit=bulks[idx])
            s = BT.NativeBatchSolve(fn, mus[idx], method="hybridanderson", nsteps=args.max_iters, threshold=THRESH,
                                    criterion="res", divergence_guard=True)
            s.solve(r0)
            out.append(s)
            del r0
        return out
    solve_all()   # warm-up: plan tables, workspaces
    torch.cuda.synchronize()
    times, res = [], None
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(max(1, min(args.steps, 2))):
            ev[0].record()
            res = solve_all()
            ev[1].record()
            torch.cuda.synchronize()
            times.append(ev[0].elapsed_time(ev[1]))
    conv = np.concatenate([s.conv for s in res])
    steps = np.concatenate([s.steps for s in res])
    ms = float(np.mean(times))
    pairs = float(n) * host.natom
    line = {"metric": "large-cell WDA isotherm converged points/s (256^3 FP64, RES<1e-8)",
            "value": int(conv.sum()) / (ms / 1e3), "unit": "points/s", "n_gpus": 1, "steps": len(times),
            "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "large-wda-256cubed", "grid": list(npts), "host": "cubic a=64A 14680 atoms seed 4",
                       "functional": "WBII + MFA + WDA(MBWR-CS-MFA) + LJ", "pressures": len(P),
                       "pressures_bar": [1e-3, 100.0], "solver": "hybridanderson m=5", "tolerance": "RES<1e-8",
                       "start": "Ninit=rho_bulk", "batches": [len(c) for c in chunks],
                       "converged_points": int(conv.sum()), "steps_per_point": [int(x) for x in steps],
                       "workspace_gb_per_instance": per / 1e9},
            "extpot": {"ms": float(min(ext_ms)), "atom_point_pairs": pairs,
                       "pairs_per_s": pairs / (min(ext_ms) / 1e3),
                       "note": "cell-list kernel; pairs counted over all atoms x points (the all-atom work)"},
            "clocks": clk.summary()}
    print(json.dumps(line))


def _oracle_rot_sample(args):
    """Oracle (numpy restatement of the reference's generate_effective_potential
    and of its interpolated path) on ``m`` grid points; returns seconds."""
    kind, degree, m = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, ROOT)
    from oracle import cmm_oracle as O
    from cmmdft_b200.hosts import cubic_host_276, co2_trappe_guest
    from cmmdft_b200.rotations import combined_rotations
    from cmmdft_b200.units import angstrom, boltzmann
    host = cubic_host_276(0)
    g = co2_trappe_guest()
    rot, w = combined_rotations(degree)
    grid = O.OGrid(host.rvecs, npoints=list(ROT_NPTS))
    pts = grid.points[..., :3].reshape(-1, 3)[:: max(1, int(np.prod(ROT_NPTS)) // m)][:m]
    beta = 1 / T / boltzmann
    t0 = time.perf_counter()
    if kind == "direct":
        O.effective_potential(pts, g["pos"], g["masses"], g["site_sigma"], g["site_epsilon"], rot, w, beta, host.ff,
                              host.recentred_pos(), host.ffatypes, host.ffatype_ids, host.rvecs)
    else:
        st = [g["ffatypes"][i] for i in g["ffatype_ids"]]
        fine_n = [int(np.ceil(l / (0.15 * angstrom))) for l in np.linalg.norm(host.rvecs, axis=1)]
        O.interpolated_effective_potential(pts, g["pos"], g["masses"], st, g["ff"], rot, w, beta, host.ff,
                                           host.recentred_pos(), host.ffatypes, host.ffatype_ids, host.rvecs, fine_n,
                                           grid.points[0, 0, 0, :3], np.full(3, 0.15 * angstrom))
    return time.perf_counter() - t0


def run_rotavg(args):
    """Secondary workload (not the headline line): the orientation-averaged
    external potential of rigid TraPPE CO2 in the 276-atom cubic host at
    300 K on a 32^3 grid, Lebedev degree 9 x planar rotations (342),
    direct (k_extpot_rot) and tricubic-interpolated from 0.15 A derivative
    grids (k_extpot_deriv + k_extpot_rot_interp).  ``value``: grid points/s
    of the direct path on the device (inputs resident, CUDA events);
    ``e2e``: ExternalPotential.generate_potential through the public API
    (host arrays in, the potential back on the host); ``cpu_baseline``: the
    oracle's restatement of the reference path on a sample of points, one
    core."""
    import torch
    import multiprocessing as mp
    import cmmdft_b200 as cd
    from cmmdft_b200 import engine as E, workload as W
    from cmmdft_b200.hosts import cubic_host_276, co2_trappe_guest
    from cmmdft_b200.rotations import combined_rotations
    from cmmdft_b200.system import Grid, System
    from cmmdft_b200.units import angstrom, boltzmann, kjmol
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    degree = 9
    host = cubic_host_276(0)
    g = co2_trappe_guest()
    rot, w = combined_rotations(degree)
    beta = 1 / T / boltzmann
    plan = E.GridPlan(ROT_NPTS, host.rvecs)
    sig, eps = W.host_type_arrays(host)
    pos = host.recentred_pos()
    npt = int(np.prod(ROT_NPTS))

    def direct():
        return E.effective_potential(plan, pos, host.ffatype_ids, sig, eps, g["pos"], g["masses"], g["site_sigma"],
                                     g["site_epsilon"], rot, w, 12 * angstrom, beta, 1e4 * kjmol)
    nh = cd.NanoporousHost("synthetic", pos=host.pos, ffatypes=host.ffatypes, ffatype_ids=host.ffatype_ids,
                           rvecs=host.rvecs, ff=host.ff)
    guest = cd.NonSphericalGuest("CO2", pos=g["pos"], masses=g["masses"], ffatypes=g["ffatypes"],
                                 ffatype_ids=g["ffatype_ids"], ff=g["ff"])
    system = System(nh, guest)
    grid = Grid(nh.cell, npoints=ROT_NPTS)

    def api(interpolate):
        ext = cd.ExternalPotential(grid, system, degree=degree, interpolate=interpolate, cutoff=12 * angstrom)
        ext.generate_potential(temperature=T)
        return ext.potential          # on the host
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(max(1, args.warmup)):
        direct()
        api(False)
        api(True)
    torch.cuda.synchronize()
    nrep = max(1, min(args.steps, 5))
    dev_ms, e2e_s = [], {}
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(nrep):
            ev[0].record()
            direct()
            ev[1].record()
            torch.cuda.synchronize()
            dev_ms.append(ev[0].elapsed_time(ev[1]))
        for interp in (False, True):
            t0 = time.perf_counter()
            for _ in range(nrep):
                api(interp)
            e2e_s[interp] = (time.perf_counter() - t0) / nrep
    ms = float(np.median(dev_ms))
    pairs = float(npt) * len(w) * len(g["masses"]) * host.natom
    cpu = {}
    if not args.no_cpu:
        ctx = mp.get_context("spawn")
        with ctx.Pool(1) as pool:
            for kind, m in (("direct", 1024), ("interpolated", 64)):
                sec = pool.map(_oracle_rot_sample, [(kind, degree, m)])[0]
                cpu[kind] = {"value": m / sec, "unit": "points/s", "cores": 1, "kind": "port",
                             "sample": "%d of the %d grid points, numpy oracle of the reference's %s path "
                                       "(pinned to it bit for bit)" % (m, npt, kind)}
    line = {"metric": "orientation-averaged external potential, grid points/s (32^3, CO2, 342 rotations)",
            "value": npt / (ms / 1e3), "unit": "points/s", "n_gpus": 1, "steps": nrep, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "rotavg-co2-32cubed", "grid": list(ROT_NPTS),
                       "host": "cubic a=17A 276 atoms seed 0", "guest": "rigid TraPPE CO2 (3 sites)",
                       "degree": degree, "rotations": len(w), "temperature_K": T, "cutoff_A": 12.0},
            "roofline": {"bound": "fp64", "kernel": "k_extpot_rot", "site_atom_pairs": pairs,
                         "pairs_per_s": pairs / (ms / 1e3), "flop_per_pair": 25,
                         "achieved": 25 * pairs / (ms / 1e3) / 1e12, "unit": "TFLOP/s", "peak": None,
                         "note": "no measured FP64 peak on this pool; minimum-image LJ over all host atoms"},
            "e2e": {"direct": {"value": npt / e2e_s[False], "unit": "points/s"},
                    "interpolated": {"value": npt / e2e_s[True], "unit": "points/s"},
                    "includes": "ExternalPotential.generate_potential: host arrays to the device, rotation "
                                "set, kernels, potential back to the host"},
            "cpu_baseline": cpu or None, "clocks": clk.summary()}
    print(json.dumps(line))


def run_solvers(args):
    """Secondary workload (not the headline line): one pressure point (1 bar)
    of the 64^3 isotherm host from Ninit = rho_bulk through each solver the
    package carries: static Picard (device-resident loop), hybrid Anderson
    (the headline's solver, one instance), QuasiNewton (L-BFGS with the
    backtracking search) and FIRE ('abc-fire', mask rho0 > 0), each to its
    criterion; device time of one solve (CUDA events, after one untimed
    solve), solver steps and ms per step."""
    import torch
    from cmmdft_b200 import batch as BT, workload as W
    from cmmdft_b200.fire import FireSolve
    from cmmdft_b200.quasinewton import QuasiNewtonSolve
    from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
    from cmmdft_b200.units import bar
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    host, guest = cubic_host_276(0), methane_guest_params()
    fn = W.build_functional(host, NPTS, T, guest)
    mus, bulks = W.isotherm_inputs(np.array([1.0]) * bar, T, guest)
    mu = float(mus[0])
    rho0 = W.initial_density(fn, mus, ninit=bulks)

    def picard():
        s = BT.NativeBatchSolve(fn, mus, method="static", nsteps=2000, threshold=1e-6, criterion="res")
        s.solve(rho0)
        return int(s.steps[0]), bool(s.conv[0])

    def hybrid_anderson():
        s = BT.NativeBatchSolve(fn, mus, method="hybridanderson", nsteps=500, threshold=THRESH, criterion="res")
        s.solve(rho0)
        return int(s.steps[0]), bool(s.conv[0])

    def quasi_newton():
        s = QuasiNewtonSolve(fn, nsteps=500, method="bfgs", line_search="backtracking", threshold=THRESH,
                             criterion="res")
        _, _, conv = s.solve(mu, rho0[0])
        return int(s.steps), bool(conv)

    def fire():
        s = FireSolve(fn, (rho0[0] > 0).cpu().numpy(), nsteps=2000, method="abc-fire", threshold=1e-6,
                      criterion="res")
        _, _, conv = s.solve(mu, rho0[0])
        return int(s.steps), bool(conv)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    out = {}
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for name, f, crit in (("static Picard", picard, "RES<1e-6"), ("hybrid Anderson m=5", hybrid_anderson,
                                                                        "RES<1e-8"),
                              ("QuasiNewton bfgs backtracking", quasi_newton, "RES<1e-8"),
                              ("FIRE abc-fire", fire, "RES<1e-6")):
            f()
            torch.cuda.synchronize()
            ev[0].record()
            steps, conv = f()
            ev[1].record()
            torch.cuda.synchronize()
            ms = ev[0].elapsed_time(ev[1])
            out[name] = {"ms": ms, "steps": steps, "converged": conv, "ms_per_step": ms / max(steps, 1),
                         "criterion": crit}
    ha = out["hybrid Anderson m=5"]
    line = {"metric": "single-point solve time per solver, 64^3 FP64 at 1 bar (ms)", "value": ha["ms"],
            "unit": "ms", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": ha["ms"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "solvers-64cubed-1bar", "grid": list(NPTS), "host": "cubic a=17A 276 atoms seed 0",
                       "pressure_bar": 1.0, "start": "Ninit=rho_bulk"},
            "solvers": out, "clocks": clk.summary()}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)   # ~0.5 s of timed solves: host jitter averages out
    ap.add_argument("--groups", type=int, default=4,
                    help="instance groups on concurrent streams, each driven from its own host thread (one "
                         "group's host decisions overlap the others' kernels; 4 groups of 6 measured best)")
    ap.add_argument("--driver", choices=("native", "python"), default="native",
                    help="batched loop in the library (cmm_solve_batched) or in Python")
    ap.add_argument("--coefs", choices=("slsqp", "exact"), default="slsqp",
                    help="Anderson coefficients: the reference's SLSQP (same trajectory and result as the "
                         "reference) or the exact simplex minimiser (fewer steps, not the reference's result)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--max-iters", type=int, default=500, help="solver step cap (lower it only to profile)")
    ap.add_argument("--autotune", action="store_true",
                    help="uneven workload: tune each host grid's FFT schedule first and solve with it")
    ap.add_argument("--workload", choices=("isotherm64", "uneven", "gradient", "large", "rotavg", "solvers"),
                    default="isotherm64",
                    help="isotherm64: the headline 64^3 isotherm; uneven: 8 uneven hosts x 32 pressures; "
                         "gradient: the 96^3 excess-isotherm loss gradient; large: the 256^3 WDA isotherm of "
                         "the 64 A host; rotavg: the orientation-averaged CO2 potential at 32^3; solvers: one "
                         "64^3 point through each solver")
    args = ap.parse_args()
    if args.workload == "solvers":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "a per-solver timing line of the package only; "
                                                                "the reference arm times the isotherm workload"}))
        elif int(os.environ.get("RANK", "0")) == 0:
            run_solvers(args)
        return
    if args.workload == "rotavg":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                sec = _oracle_rot_sample(("direct", 9, 1024))
                print(json.dumps({"impl": "reference", "metric": "orientation-averaged external potential, grid "
                                  "points/s (32^3, CO2, 342 rotations)", "value": 1024 / sec, "unit": "points/s",
                                  "higher_is_better": True,
                                  "cpu_baseline": {"value": 1024 / sec, "kind": "port", "cores": 1,
                                                   "sample": "1024 of the 32768 grid points"},
                                  "e2e": {"value": 1024 / sec, "unit": "points/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}))
        elif int(os.environ.get("RANK", "0")) == 0:
            run_rotavg(args)
        return
    if args.workload == "large":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the 256^3 large-cell workload takes hours per "
                                                                "point in the reference's numpy path"}))
        elif int(os.environ.get("RANK", "0")) == 0:
            run_large(args)
        return
    if args.workload == "gradient":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no derivatives"}))
        elif int(os.environ.get("RANK", "0")) == 0:
            run_gradient(args)
        return
    if args.workload == "uneven":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the uneven multi-host workload is timed on the "
                                                                "GPU only (hours of CPU time in the reference)"}))
        elif int(os.environ.get("RANK", "0")) == 0:
            run_uneven(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

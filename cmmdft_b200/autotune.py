"""FFT-schedule autotuner for the functional pipeline.

A grid plan's FFT schedule -- the order of the radix stages on each axis,
the fused or staged form of the plane passes, the tile width of the
run-time-length column passes (cmm_grid_create_sched) -- does not change the
transforms beyond rounding, but it changes their speed, most for the grids
that the 0.25 angstrom spacing of the reference's Grid gives real cells:
lengths with prime factors 7..13 and above 16 (Rader or direct-DFT stages),
odd N3, planes beyond shared memory.  ``tune(npoints, rvecs, batch)``
times one functional evaluation (cmm_fmt_c1: C1 spectrum, free-energy sums,
n3 maximum) of a synthetic density for every candidate schedule on the
current device, CUDA events after a warm-up, and returns the fastest with
the table of all timings -- the default schedule unless another is faster
by more than ``margin`` (5 %): the timing covers the functional pipeline
only, while a non-default radix order moves every pass of the solve (the
plane update passes included) to the run-time-length kernels and the staged
form stages the update passes too, which costs more than a pipeline gain
within the timing noise recovers (the uneven eight-host workload ran 2x
slower on sub-1 % picks).  Results are cached per (shape, batch, version,
device) in memory and, when a cache file is given, on disk as JSON.

The candidates: for each axis the distinct radix orders (an order that
gives the same stage sequence as another is tried once), the staged plane
passes where the fused ones are possible, and column tiles 4, 8 and 16 for
the run-time-length column kernels; at most ``max_candidates`` are timed,
the default schedule always among them.
"""
import itertools
import json
import os

import numpy as np

from . import _lib as L
from . import engine as E

__all__ = ['candidates', 'tune', 'plan_for']

ORDERS = (0, 1, 2, 3)   # CMM_ORDER_DEFAULT, _NO8, _ODDFIRST, _ODDDESC
_cache = {}


def _stage_orders(n):
    """Distinct radix stage sequences of a length-n axis: {sequence: order}."""
    m, p2 = n, []
    out = {}
    for order in ORDERS:
        mm, pw = n, []
        while order != 1 and mm % 8 == 0:
            pw.append(8)
            mm //= 8
        while mm % 4 == 0:
            pw.append(4)
            mm //= 4
        while mm % 2 == 0:
            pw.append(2)
            mm //= 2
        odd = []
        q = 3
        while mm > 1:
            while mm % q == 0:
                odd.append(q)
                mm //= q
            q += 2
        if order in (2, 3):
            odd = odd[::-1]
        seq = tuple(odd + pw) if order == 2 else tuple(pw + odd)
        out.setdefault(seq, order)
    del m, p2
    return out


def candidates(npoints, max_candidates=48):
    """Candidate schedules [x order, y order, z order, staging, tile] for a
    grid, the default first."""
    n1, n2, n3 = [int(n) for n in npoints]
    zlen = n3 if n3 % 2 else n3 // 2
    orders = [sorted(set(_stage_orders(n).values())) for n in (n1, n2, zlen)]
    default = [0, 0, 0, -1, 0]
    out = [default]
    # radix orders first, then the plane-pass form, then column tiles: a
    # truncated list keeps the widest spread of orders
    for tile in (0, 8, 4):
        for st in (-1, 1, 2):
            for o in itertools.product(*orders):
                c = [o[0], o[1], o[2], st, tile]
                if c != default and c not in out:
                    out.append(c)
    return out[:max_candidates]


def _time_schedule(npoints, rvecs, sched, batch, version, R, reps=5):
    import torch
    plan = E.GridPlan(npoints, rvecs, schedule=sched)
    V = torch.zeros(plan.npoints, dtype=torch.float64, device="cuda")
    fn = E.Functional(plan, R, 1.0, 1.0, V, version)
    g = torch.Generator(device="cuda").manual_seed(1)
    # a smooth, dense synthetic density (packing fraction about 0.2)
    rho = 0.2 / (4.0 / 3.0 * np.pi * R ** 3) * (1 + 0.3 * torch.rand((batch,) + plan.npoints, dtype=torch.float64,
                                                                      device="cuda", generator=g))
    spec = plan.rfft_yz(rho)
    buf = E.Buffers(plan, batch, nwork=fn.nwork)
    chat = plan.new_spec(batch)
    fn.c1(buf, spec, chat, want=7)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn.c1(buf, spec, chat, want=7)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps, plan.schedule()[1]


def tune(npoints, rvecs, batch=4, version=L.WBII, R=3.0, max_candidates=48, cache_file=None, verbose=False,
         margin=0.05):
    """Fastest FFT schedule for one functional evaluation of ``batch``
    instances on this grid, the default one unless another beats it by more
    than ``margin``: (schedule, table) with table a list of (schedule,
    radices, ms) sorted by time."""
    import torch
    npoints = tuple(int(n) for n in npoints)
    dev = torch.cuda.get_device_name(torch.cuda.current_device())
    key = "%s|%d|%d|%s" % ("x".join(map(str, npoints)), int(batch), int(version), dev)
    if key in _cache:
        return _cache[key]
    disk = {}
    if cache_file and os.path.exists(cache_file):
        with open(cache_file) as f:
            disk = json.load(f)
        if key in disk:
            _cache[key] = (disk[key]["schedule"], disk[key]["table"])
            return _cache[key]
    table = []
    for sched in candidates(npoints, max_candidates):
        try:
            ms, radices = _time_schedule(npoints, rvecs, sched, batch, version, R)
        except L.CmmError:
            continue      # e.g. a tile too wide for shared memory
        table.append((sched, radices, ms))
        if verbose:
            print("  %s radices %s: %.3f ms" % (sched, radices, ms), flush=True)
    table.sort(key=lambda t: t[2])
    best = table[0][0]
    dflt = [t for t in table if t[0] == [0, 0, 0, -1, 0]]
    if dflt and table[0][2] > (1.0 - margin) * dflt[0][2]:
        best = dflt[0][0]
    _cache[key] = (best, table)
    if cache_file:
        disk[key] = {"schedule": best, "table": table}
        with open(cache_file, "w") as f:
            json.dump(disk, f)
    return best, table


def plan_for(npoints, rvecs, batch=4, version=L.WBII, R=3.0, **kw):
    """A GridPlan with the tuned schedule."""
    best, _ = tune(npoints, rvecs, batch=batch, version=version, R=R, **kw)
    return E.GridPlan(npoints, rvecs, schedule=best)

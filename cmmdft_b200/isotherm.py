"""Public batched entry point: a whole isotherm (or any set of chemical
potentials) on one host in one batched solve.

The reference solves an isotherm as a Python loop of Program.solve calls, one
per pressure (examples/methane_ZIF8.ipynb cells 7-11, cmmdft/program.py:
331-404).  ``solve_isotherm`` takes host arrays on the CPU, builds the
external potential and MFA kernel on the GPU, solves every point of the
isotherm as one batch, and returns loadings (and densities) on the CPU.
"""
import numpy as np
import torch

from . import batch as BT
from . import engine as E
from . import workload as W
from .units import angstrom, kjmol

__all__ = ['solve_isotherm', 'solve_batch', 'grid_points', 'excess_loading']


def solve_isotherm(host, pressures, temperature, guest, npoints, method='hybridanderson', threshold=1e-8,
                   criterion='res', nsteps=500, start='bulk', version='WBII', tailcorrections=False,
                   return_density=True, fn=None, m=5, alpha_mix=0.1, divergence_guard=True, groups=1, native=True,
                   anderson_coefs='slsqp'):
    """Solve the adsorption isotherm of a spherical LJ guest in ``host``.

    pressures: array in atomic units (e.g. ``np.logspace(-3, 2, 24) * bar``).
    start: 'bulk' -> rho0 = rho_bulk exp(-max(V,0)/kT) (Ninit=rho_bulk, the
    reference notebook's choice); 'ideal' -> exp(beta (mu - V)) / Lambda^3.
    groups: independent instance groups solved on concurrent streams (host
    decisions of one group overlap the device work of another).
    native: run the batched loop in the library (cmm_solve_batched); False
    runs the Python driver (the same kernels and decisions).
    anderson_coefs: 'slsqp' takes the reference's SLSQP coefficients (same
    trajectory and result as the reference at any tolerance); 'exact' the
    exact simplex minimiser (fewer steps, a different point within the
    tolerance).
    Returns a dict with mu, rho_bulk, N (absolute loading per cell),
    converged, steps, omega and (optionally) the densities [B, N1, N2, N3].
    """
    if fn is None:
        fn = W.build_functional(host, npoints, temperature, guest, version=version,
                                tailcorrections=tailcorrections)
    mus, bulks = W.isotherm_inputs(pressures, temperature, guest)
    rho0 = W.initial_density(fn, mus, ninit=bulks if start == 'bulk' else None)
    s = BT.GroupedSolve(fn, mus, groups=groups, native=native, method=method, nsteps=nsteps, threshold=threshold,
                        criterion=criterion, m=m, alpha_mix=alpha_mix, divergence_guard=divergence_guard,
                        anderson_coefs=anderson_coefs)
    # densities land in pinned host memory while the rest of the batch iterates
    host = torch.empty(tuple(rho0.shape), dtype=torch.float64, pin_memory=True) if return_density else None
    N, rho, conv = s.solve(rho0, host_out=host)
    out = dict(mu=mus, rho_bulk=bulks, N=np.array(N), converged=np.array(conv), steps=s.steps.copy(),
               diverged=s.diverged.copy(),
               solver=s, functional=fn)
    if return_density:
        out['rho'] = host.numpy()
    return out


def excess_loading(N, rho_bulk, he_fraction, cell_volume):
    """N_ex = N - rho_bulk * He_frac * V_cell (Calculator.return_loading, calculator.py:114-138)."""
    return np.asarray(N) - np.asarray(rho_bulk) * he_fraction * cell_volume


def grid_points(host, spacing=0.25 * angstrom):
    """N_a = ceil(L_a / spacing), L_a the length of cell vector a (Grid.__init__,
    cmmdft/system.py:262-266, which measures the columns of rvecs; the hosts
    here are orthorhombic, where rows and columns agree)."""
    lengths = np.linalg.norm(np.asarray(host.rvecs, dtype=float), axis=0)
    return tuple(int(np.ceil(l / spacing)) for l in lengths)


def solve_batch(hosts, pressures, temperature, guest, npoints=None, spacing=0.25 * angstrom,
                method='hybridanderson', threshold=1e-8, criterion='res', nsteps=500, m=5, alpha_mix=0.1,
                divergence_guard=True, anderson_coefs='slsqp', return_density=False, max_concurrent=4,
                version='WBII', tailcorrections=False, memory_budget=None, schedules=None):
    """Isotherms of several hosts of uneven cells and grids in one call.

    The reference solves every (host, pressure) point in its own Program.solve
    loop.  Here each host is one batched solve of all its pressures (its own
    grid plan, potential and MFA kernel, since the cell sets the k-vectors);
    up to ``max_concurrent`` hosts run at once, each driven by the native
    batched solver from its own host thread on one of ``max_concurrent``
    CUDA streams, so the host decisions of one host overlap the kernels of
    the others.  A host's device buffers (~520 B per grid point and pressure
    with m = 5) return to the caching allocator when its solve ends and serve
    the next host on the same stream.  A host starts only while the estimated
    buffers of the running ones stay within ``memory_budget`` bytes (default
    60% of the device's memory); a host larger than the budget runs alone.

    hosts: list of SyntheticHost-like hosts; pressures: one array for every
    host or a list with one array per host (atomic units); npoints: None
    (from ``spacing``), one shape for all hosts or a list of shapes.
    schedules: None (default FFT schedules) or one cmm_grid_create_sched
    schedule per host (e.g. from cmmdft_b200.autotune.tune); a schedule moves
    results only by rounding.
    Returns one dict per host as ``solve_isotherm`` does (without the solver
    and functional objects), in the order of ``hosts``.
    """
    import threading
    nh = len(hosts)
    if npoints is None:
        shapes = [grid_points(h, spacing) for h in hosts]
    elif np.ndim(npoints) == 1 and len(npoints) == 3 and not isinstance(npoints[0], (tuple, list)):
        shapes = [tuple(int(n) for n in npoints)] * nh
    else:
        shapes = [tuple(int(n) for n in s) for s in npoints]
    plist = pressures if (isinstance(pressures, (list, tuple)) and len(pressures) == nh and
                          np.ndim(pressures[0]) == 1) else [pressures] * nh
    results = [None] * nh
    errors = []
    cur = torch.cuda.current_stream()
    device = torch.cuda.current_device()
    if memory_budget is None:
        memory_budget = int(0.6 * torch.cuda.mem_get_info(device)[1])
    need = [(640 * len(np.atleast_1d(plist[i])) + 512) * int(np.prod(shapes[i])) for i in range(nh)]   # bytes, generous
    cond = threading.Condition()
    state = dict(bytes=0, running=0)
    # One stream per concurrency slot, reused by the hosts that take the slot:
    # the caching allocator hands a finished host's blocks to the next host on
    # the same stream, so hosts neither free device memory (which synchronises
    # the device under the hosts still running) nor allocate it afresh.
    # The slots' streams are the same ones on every call (BT._group_streams),
    # so a call's workspaces come from the blocks the previous call freed.
    free_streams = list(BT._group_streams(max(1, int(max_concurrent))))

    def admit(i):
        with cond:
            cond.wait_for(lambda: state['running'] == 0 or (state['running'] < max(1, int(max_concurrent)) and
                                                             state['bytes'] + need[i] <= memory_budget))
            state['bytes'] += need[i]
            state['running'] += 1
            return free_streams.pop()

    def leave(i, st):
        with cond:
            state['bytes'] -= need[i]
            state['running'] -= 1
            free_streams.append(st)
            cond.notify_all()

    def run(i):
        st = admit(i)
        try:
            torch.cuda.set_device(device)
            st.wait_stream(cur)
            with torch.cuda.stream(st):
                plan = None
                if schedules is not None and schedules[i] is not None:
                    plan = E.GridPlan(shapes[i], hosts[i].rvecs, schedule=schedules[i])
                fn = W.build_functional(hosts[i], shapes[i], temperature, guest, version=version,
                                        tailcorrections=tailcorrections, plan=plan)
                P = np.asarray(plist[i], dtype=float)
                mus, bulks = W.isotherm_inputs(P, temperature, guest)
                rho0 = W.initial_density(fn, mus, ninit=bulks)
                s = BT.NativeBatchSolve(fn, mus, method=method, nsteps=nsteps, threshold=threshold,
                                        criterion=criterion, m=m, alpha_mix=alpha_mix,
                                        divergence_guard=divergence_guard, anderson_coefs=anderson_coefs)
                host = (torch.empty(tuple(rho0.shape), dtype=torch.float64, pin_memory=True)
                        if return_density else None)
                N, rho, conv = s.solve(rho0, host_out=host)
                out = dict(mu=mus, rho_bulk=bulks, N=np.array(N), converged=np.array(conv),
                           steps=s.steps.copy(), diverged=s.diverged.copy(), omega=np.array(s.omega0),
                           npoints=shapes[i])
                st.synchronize()
                if return_density:
                    out['rho'] = host.numpy()
                results[i] = out
                del s, fn, rho, rho0
        except BaseException as e:  # re-raised on the calling thread
            errors.append(e)
        finally:
            leave(i, st)

    threads = [threading.Thread(target=run, args=(i,)) for i in range(nh)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return results

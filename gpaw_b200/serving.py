"""Many independent Poisson solves: batches and a continuous-batching server.

The model is the pair-density workload of the reference
(gpaw/lrtddft/omega_matrix.py:400 calls PoissonSolver.solve once per pair
density): many independent charge-neutral solves on grids of different sizes.

PoissonBatch(solvers)
    Solvers of any grid sizes captured as parallel branches of one CUDA
    graph; one launch runs every solve's V-cycle loop concurrently on the
    device, each stopping on its own criterion.

PoissonServer(...)
    Requests (grid size, rho) arrive over time and wait in a queue per grid
    size.  Solvers come in pods: single solvers, and `slots` solvers of one
    size captured as one PoissonBatch (plain graph branches), so that one
    graph launch carries up to `slots` requests.  Whenever fewer than
    `max_inflight` launches are in flight, the waiting requests of each size,
    oldest size first, take a pod (a single solver when one request waits,
    a batch pod when more do; a new pod within the device-memory budget if
    none is free and the GPU is idle or the size has none yet), fill its slots and launch it on the next stream,
    overlapping the launches already on the GPU; unused slots run nothing.
    Completions are found by polling the oldest launch of each stream, and
    each pod returns to its pool.  Latency is completion minus arrival.
    Solves never share buffers, so a result is the same alone and in the mix.
    Each pod owns its requests' potential buffers, so the serving loop makes
    no device allocation once the pods exist (an allocation would stall the
    launches in flight).

    Failures are per request, on the host: a request whose `deadline`
    (seconds after its arrival) passes while it waits is dropped
    ('expired'); one whose `cancel_at` (seconds from the start of the run)
    passes is dropped if it waits and its result discarded if it is in
    flight ('cancelled'; a launch on the GPU is never interrupted); a pod
    that cannot be created (over the memory budget, or the device allocation
    fails) leaves the request waiting while other launches are in flight and
    rejects it when nothing is ('rejected').
"""
import collections
import time

import numpy as np
import torch

from . import _lib
from .grid_descriptor import GridDescriptor
from .poisson import PoissonSolver


class PoissonBatch:
    """Independent solves launched together as one graph.  Solvers of one
    structure (same levels, smoothing, stencil and transfer orders and
    boundary conditions; any grid sizes; float64) run grouped: each V-cycle
    step is one persistent launch over all their grids, pulling work tiles
    from a queue, and each solve stops on its own criterion.  Groups and the
    other solvers run as parallel graph branches.  `grouped`: how many
    solvers run inside groups."""

    def __init__(self, solvers, group=True):
        """group=False: every solver runs as its own graph branch, never
        grouped (better when many batches are in flight at once)."""
        self.solvers = list(solvers)
        for s in self.solvers:
            if s.solver is None:
                s.initialize()
        handles = (_lib._vp * len(self.solvers))(*[s.solver for s in self.solvers])
        h = _lib._vp()
        _lib.check(_lib.lib.gfd_poisson_batch_create_ex(
            len(self.solvers), handles, 0 if group else _lib.GFD_BATCH_NO_GROUPS,
            _lib.ctypes.byref(h)), 'PoissonBatch')
        self.batch = h
        g = _lib.ctypes.c_int(0)
        _lib.check(_lib.lib.gfd_poisson_batch_grouped(h, _lib.ctypes.byref(g)))
        self.grouped = g.value

    def __del__(self):
        h = getattr(self, 'batch', None)
        lib = getattr(_lib, 'lib', None) if _lib is not None else None
        if h and lib is not None:  # at interpreter exit the module may be gone
            lib.gfd_poisson_batch_destroy(h)
            self.batch = None

    def solve_async(self, phis, rhos, eps=2e-10, maxcharge=1e-6, maxiter=1000, stream=None):
        """Enqueue every solve on `stream` (default: the current stream) and
        return at once.  phis[i] / rhos[i] are CUDA float64 arrays of solver
        i's grid, or both None to leave slot i unused in this launch (it runs
        no V-cycle).  Read the results with solvers[i].result() once the
        stream has passed the launch."""
        if len(phis) != len(self.solvers) or len(rhos) != len(self.solvers):
            raise ValueError('one phi and one rho per solver (None for an unused slot)')
        used = [p for p in phis if p is not None]
        if not used:
            raise ValueError('a launch needs at least one used slot')
        for s, p, r in zip(self.solvers, phis, rhos):
            if (p is None) != (r is None):
                raise ValueError('phi and rho of a slot must both be given or both None')
            if p is not None:
                s._check_arrays(p, r)
        if stream is None:
            stream = torch.cuda.current_stream(used[0].device)
        P = (_lib._vp * len(phis))(*[None if p is None else p.data_ptr() for p in phis])
        R = (_lib._vp * len(rhos))(*[None if r is None else r.data_ptr() for r in rhos])
        _lib.check(_lib.lib.gfd_poisson_batch_solve_async(
            self.batch, P, R, float(eps), float(maxcharge), int(maxiter), stream.cuda_stream),
            'PoissonBatch.solve')
        return stream

    def solve(self, phis, rhos, eps=2e-10, maxcharge=1e-6, maxiter=1000):
        """Solve all (unused slots: None); returns [(niter, error), ...] for
        the used slots, None for the unused ones; raises as
        PoissonSolver.solve for the first solver that failed."""
        stream = self.solve_async(phis, rhos, eps, maxcharge, maxiter)
        stream.synchronize()
        return [None if p is None else s.result() for s, p in zip(self.solvers, phis)]


def grid_for(N, h_bohr, pbc=False, device=None):
    """Zero-boundary (or periodic) cubic grid of N points per axis, spacing h."""
    return GridDescriptor((N, N, N), (N * h_bohr,) * 3, pbc, device=device)


class Request:
    """One solve: grid size N, arrival time (seconds from the start of the
    run), rho on the device; optional deadline (seconds after arrival by
    which it must be admitted) and cancel_at (seconds from the start)."""
    __slots__ = ('rid', 'N', 'arrival', 'rho', 'admit', 'done', 'niter', 'error', 'phi',
                 'status', 'deadline', 'cancel_at')

    def __init__(self, rid, N, arrival, rho, deadline=None, cancel_at=None):
        self.rid = rid
        self.N = N
        self.arrival = arrival
        self.rho = rho
        self.deadline = deadline
        self.cancel_at = cancel_at
        self.admit = None
        self.done = None
        self.niter = None
        self.error = None
        self.phi = None
        self.status = None


class _Pod:
    """`slots` solvers of one grid size that launch together: one graph
    launch (a PoissonBatch) serves up to `slots` requests; `phis` are the
    slots' potential buffers.  `ready`: an event that the pod's next launch
    must wait for (the copies of its last results, when they are kept)."""
    __slots__ = ('N', 'solvers', 'batch', 'nbytes', 'phis', 'ready')

    def __init__(self, N, solvers, batch, nbytes, phis):
        self.N = N
        self.solvers = solvers
        self.batch = batch
        self.nbytes = nbytes
        self.phis = phis
        self.ready = None


class PoissonServer:
    """Continuous batching of independent Poisson solves (see the module
    docstring).  slots: requests of one grid size that one launch can carry
    (1: every request is its own graph launch).  keep_results: True to copy
    every completed request's potential to `request.phi`, or a function of
    the request that says whether to keep its potential."""

    def __init__(self, h_bohr, nn=3, relax='J', eps=2e-10, precision='fp64',
                 budget_bytes=120 * 2**30, max_inflight=64, nstreams=32, device=None,
                 keep_results=False, slots=8):
        self.h = h_bohr
        self.nn = nn
        self.relax = relax
        self.eps = eps
        self.precision = precision
        self.budget = budget_bytes
        self.max_inflight = max_inflight
        self.slots = max(1, int(slots))
        self.device = torch.device(device) if device is not None else torch.device('cuda')
        self.streams = [torch.cuda.Stream(self.device) for _ in range(nstreams)]
        self.free = collections.defaultdict(list)   # (N, slots) -> [_Pod]
        self.npods = collections.defaultdict(int)   # N -> pods created
        self.used_bytes = 0
        self.keep_results = keep_results
        self.rejected = 0
        self.alloc_failures = 0

    # -- pod pool --------------------------------------------------------------
    def _new_pod(self, N, slots):
        """A pod of `slots` solvers of size N, or None when it would exceed
        the memory budget or its device allocations fail."""
        solvers, need = [], 0
        for _ in range(slots):
            ps = PoissonSolver(self.nn, self.relax, self.eps, precision=self.precision)
            ps.set_grid_descriptor(grid_for(N, self.h, device=self.device))
            need += ps.nbytes() + int(np.prod(ps.gd.n_c)) * 8  # + the slot's phi
            solvers.append(ps)
        if self.used_bytes + need > self.budget:
            return None
        try:
            for ps in solvers:
                ps.initialize()
            # Many pods are in flight at once: plain graph branches overlap
            # better there than grouped launches (measured on B200: 32^3
            # requests 2.7K/s against 1.2K/s grouped).
            batch = PoissonBatch(solvers, group=False) if slots > 1 else None
            shape = tuple(int(x) for x in solvers[0].gd.n_c)
            phis = [torch.empty(shape, dtype=torch.float64, device=self.device)
                    for _ in range(slots)]
        except MemoryError:
            self.alloc_failures += 1
            return None  # the solvers release what they hold when collected
        self.used_bytes += need
        return _Pod(N, solvers, batch, need, phis)

    def _launch(self, pod, reqs, stream):
        """Enqueue the requests on the pod's first slots (from phi = 0);
        returns their phis (the pod's buffers)."""
        phis = pod.phis[:len(reqs)]
        if pod.ready is not None:
            stream.wait_event(pod.ready)
            pod.ready = None
        with torch.cuda.stream(stream):
            for phi in phis:
                phi.zero_()
            if pod.batch is None:
                pod.solvers[0].solve_async(phis[0], reqs[0].rho)
            else:
                unused = [None] * (len(pod.solvers) - len(reqs))
                pod.batch.solve_async(phis + unused, [r.rho for r in reqs] + unused,
                                      eps=self.eps, stream=stream)
        return phis

    def warm(self, sizes, per_size=1, pod_requests=None):
        """Create, for each size, per_size single solvers and batch pods for
        pod_requests requests (default per_size), and run each once, so that
        admission pays for no allocation, graph capture or first launch."""
        want = {1: per_size}
        if self.slots > 1:
            want[self.slots] = per_size if pod_requests is None else pod_requests
        for N in sizes:
            for k, nreq in want.items():
                while len(self.free[N, k]) * k < nreq:
                    pod = self._new_pod(N, k)
                    if pod is None:
                        return
                    z = torch.zeros(tuple(int(x) for x in pod.solvers[0].gd.n_c),
                                    dtype=torch.float64, device=self.device)
                    stream = torch.cuda.current_stream(self.device)
                    self._launch(pod, [Request(-1, N, 0.0, z)], stream)
                    stream.synchronize()
                    self.free[N, k].append(pod)
                    self.npods[N] += 1

    def _acquire(self, N, waiting, busy):
        """A pod for `waiting` requests of size N: a single solver for one, a
        pod of `slots` for more (whichever is free, preferring that one).
        A new pod (within the memory budget) only when the GPU is idle
        (busy = 0) or no pod of this size exists: its allocation would stall
        the launches in flight.  None if none can be had now."""
        want = 1 if waiting == 1 or self.slots == 1 else self.slots
        other = self.slots if want == 1 else 1
        for k in (want, other):
            if self.free[N, k]:
                return self.free[N, k].pop()
        if busy and self.npods[N]:
            return None
        pod = self._new_pod(N, want)
        if pod is not None:
            self.npods[N] += 1
        return pod

    # -- serving loop ----------------------------------------------------------
    def run(self, requests, metrics=None):
        """Serve `requests` (Request objects with arrival times in seconds from
        the start of the run).  Returns a summary dict; per-request results are
        stored on the Request objects.  `metrics` (a timing.MetricsLog): one
        'request' record per request and one 'summary' record are written
        after the run, so that logging does not slow the serving loop."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queues = collections.OrderedDict()   # N -> arrived requests, not admitted
        # Work on one stream completes in order, so only the oldest launch of
        # each stream needs polling: O(streams) event queries per pass.
        lanes = [collections.deque() for _ in self.streams]
        ninflight = 0   # launches in flight
        ev_pool = []
        si = 0
        rejected0 = self.rejected
        deadlines = any(r.deadline is not None for r in requests)
        cancels = sorted((r for r in requests if r.cancel_at is not None),
                         key=lambda r: r.cancel_at)
        ci = 0
        t0 = time.perf_counter()
        while pending or ninflight or any(queues.values()):
            now = time.perf_counter() - t0
            # retire finished launches
            for li, lane in enumerate(lanes):
                while lane and lane[0][2].query():
                    pod, reqs, ev, phis = lane.popleft()
                    done = time.perf_counter() - t0
                    kept = False
                    for slot, (req, phi) in enumerate(zip(reqs, phis)):
                        req.done = done
                        if req.status == 'cancelled':
                            continue  # result discarded
                        try:
                            req.niter, req.error = pod.solvers[slot].result()
                            req.status = 'ok'
                        except Exception as e:  # reported per request
                            req.status = repr(e)
                        keep = self.keep_results
                        if keep is not True and callable(keep):
                            keep = keep(req)
                        if keep:
                            # copied on the pod's own stream; the pod's next
                            # launch (on any stream) waits for the copies
                            with torch.cuda.stream(self.streams[li]):
                                req.phi = phi.clone()
                            kept = True
                    if kept:
                        pod.ready = torch.cuda.Event()
                        pod.ready.record(self.streams[li])
                    ninflight -= 1
                    self.free[pod.N, len(pod.solvers)].append(pod)
                    ev_pool.append(ev)
            # cancellations due: waiting or not yet arrived requests are
            # dropped, in-flight ones have their results discarded
            while ci < len(cancels) and cancels[ci].cancel_at <= now:
                r = cancels[ci]
                ci += 1
                if r.status is None:
                    r.status = 'cancelled'
                    q = queues.get(r.N)
                    if q is not None and r in q:
                        q.remove(r)
            # arrivals join the queue of their grid size
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                if r.status == 'cancelled':
                    continue
                queues.setdefault(r.N, collections.deque()).append(r)
            # waiting requests whose admission deadline has passed
            if deadlines:
                for N, q in queues.items():
                    if any(r.deadline is not None and now > r.arrival + r.deadline for r in q):
                        keep = collections.deque()
                        for r in q:
                            if r.deadline is not None and now > r.arrival + r.deadline:
                                r.status = 'expired'
                            else:
                                keep.append(r)
                        queues[N] = keep
            # admit: sizes in order of their oldest waiting request; each
            # launch takes up to `slots` of that size's waiting requests
            for N in sorted((n for n in queues if queues[n]), key=lambda n: queues[n][0].arrival):
                q = queues[N]
                while q and ninflight < self.max_inflight:
                    pod = self._acquire(N, len(q), ninflight)
                    if pod is None:
                        if not ninflight:  # cannot fit now, nor after a retirement
                            req = q.popleft()
                            req.status = 'rejected: no device memory for a solver of this size'
                            self.rejected += 1
                            continue
                        break
                    m = min(len(pod.solvers), len(q))
                    reqs = [q.popleft() for _ in range(m)]
                    k = si % len(self.streams)
                    si += 1
                    phis = self._launch(pod, reqs, self.streams[k])
                    ev = ev_pool.pop() if ev_pool else torch.cuda.Event()
                    ev.record(self.streams[k])
                    admit = time.perf_counter() - t0
                    for r in reqs:
                        r.admit = admit
                    lanes[k].append((pod, reqs, ev, phis))
                    ninflight += 1
            if not ninflight and pending and not any(queues.values()):
                wait = pending[0].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 1e-3))
        wall = time.perf_counter() - t0
        done = [r for r in requests if r.status == 'ok']
        lat = np.array([r.done - r.arrival for r in done]) if done else np.zeros(1)
        summary = {'requests': len(requests), 'completed': len(done),
                'rejected': self.rejected - rejected0,
                'expired': sum(r.status == 'expired' for r in requests),
                'cancelled': sum(r.status == 'cancelled' for r in requests),
                'failed': sum(r.status not in (None, 'ok', 'expired', 'cancelled') and
                              not r.status.startswith('rejected') for r in requests),
                'wall_s': wall, 'solves_per_s': len(done) / wall if wall > 0 else 0.0,
                'p50_ms': float(np.percentile(lat, 50) * 1e3),
                'p99_ms': float(np.percentile(lat, 99) * 1e3),
                'max_residual': float(max([r.error for r in done], default=0.0)),
                'device_bytes': self.used_bytes}
        if metrics is not None:
            for r in requests:
                metrics.log('request', rid=r.rid, N=r.N, arrival_s=r.arrival, admit_s=r.admit,
                            done_s=r.done, status=r.status, niter=r.niter, residual=r.error)
            metrics.log('summary', precision=self.precision, **summary)
            metrics.flush()
        return summary


def pair_density(gd, seed, ngauss=8):
    """rho = psi1 * psi2 - mean(psi1 * psi2); each psi a sum of ngauss
    Gaussians (amplitude N(0,1), width U[0.4, 1.2] A, centres at least 2 A
    from the walls -- a quarter of the box on boxes too small for that),
    generated on the grid's device from a per-request seed."""
    bohr = 0.52917721092
    rng = np.random.default_rng(seed)
    dev = gd.device
    L = gd.cell_cv.diagonal()
    coords = [torch.arange(int(n), dtype=torch.float64, device=dev) + int(b)
              for n, b in zip(gd.n_c, gd.beg_c)]
    x = coords[0][:, None, None] * gd.h_cv[0, 0]
    y = coords[1][None, :, None] * gd.h_cv[1, 1]
    z = coords[2][None, None, :] * gd.h_cv[2, 2]
    rho = None
    for _ in range(2):
        psi = torch.zeros(tuple(int(n) for n in gd.n_c), dtype=torch.float64, device=dev)
        for _ in range(ngauss):
            a = rng.standard_normal()
            s = rng.uniform(0.4, 1.2) / bohr
            margin = np.minimum(2 / bohr, 0.25 * L)
            R = rng.uniform(margin, L - margin)
            psi += a * torch.exp(-((x - R[0]) ** 2 + (y - R[1]) ** 2 + (z - R[2]) ** 2) / (2 * s * s))
        rho = psi if rho is None else rho * psi
    return rho - rho.mean()

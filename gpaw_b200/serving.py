"""Many independent Poisson solves: batches and a continuous-batching server.

The model is the pair-density workload of the reference
(gpaw/lrtddft/omega_matrix.py:400 calls PoissonSolver.solve once per pair
density): many independent charge-neutral solves on grids of different sizes.

PoissonBatch(solvers)
    Solvers of any grid sizes captured as parallel branches of one CUDA
    graph; one launch runs every solve's V-cycle loop concurrently on the
    device, each stopping on its own criterion.

PoissonServer(...)
    Requests (grid size, rho) arrive over time.  A request is admitted as
    soon as it has arrived, a solver of its grid size is free (or can be
    created within the device-memory budget) and the number of solves in
    flight is below `max_inflight`; it is then launched on its own stream,
    so its kernels overlap with those of the solves already on the GPU.
    Completions are found by polling CUDA events, and each solver returns to
    its pool for the next request.  Latency is completion minus arrival.
    Solves never share buffers, so a result is the same alone and in the mix.
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

    def __init__(self, solvers):
        self.solvers = list(solvers)
        for s in self.solvers:
            if s.solver is None:
                s.initialize()
        handles = (_lib._vp * len(self.solvers))(*[s.solver for s in self.solvers])
        h = _lib._vp()
        _lib.check(_lib.lib.gfd_poisson_batch_create(len(self.solvers), handles,
                                                     _lib.ctypes.byref(h)), 'PoissonBatch')
        self.batch = h
        g = _lib.ctypes.c_int(0)
        _lib.check(_lib.lib.gfd_poisson_batch_grouped(h, _lib.ctypes.byref(g)))
        self.grouped = g.value

    def __del__(self):
        h = getattr(self, 'batch', None)
        if h:
            _lib.lib.gfd_poisson_batch_destroy(h)
            self.batch = None

    def solve(self, phis, rhos, eps=2e-10, maxcharge=1e-6, maxiter=1000):
        """Solve all; phis[i] / rhos[i] are CUDA float64 arrays of solver i's
        grid.  Returns [(niter, error), ...]; raises as PoissonSolver.solve
        for the first solver that failed."""
        if len(phis) != len(self.solvers) or len(rhos) != len(self.solvers):
            raise ValueError('one phi and one rho per solver')
        for s, p, r in zip(self.solvers, phis, rhos):
            s._check_arrays(p, r)
        stream = torch.cuda.current_stream(phis[0].device)
        P = (_lib._vp * len(phis))(*[p.data_ptr() for p in phis])
        R = (_lib._vp * len(rhos))(*[r.data_ptr() for r in rhos])
        _lib.check(_lib.lib.gfd_poisson_batch_solve_async(
            self.batch, P, R, float(eps), float(maxcharge), int(maxiter), stream.cuda_stream),
            'PoissonBatch.solve')
        stream.synchronize()
        return [s.result() for s in self.solvers]


def grid_for(N, h_bohr, pbc=False, device=None):
    """Zero-boundary (or periodic) cubic grid of N points per axis, spacing h."""
    return GridDescriptor((N, N, N), (N * h_bohr,) * 3, pbc, device=device)


class Request:
    __slots__ = ('rid', 'N', 'arrival', 'rho', 'admit', 'done', 'niter', 'error', 'phi',
                 'status')

    def __init__(self, rid, N, arrival, rho):
        self.rid = rid
        self.N = N
        self.arrival = arrival
        self.rho = rho
        self.admit = None
        self.done = None
        self.niter = None
        self.error = None
        self.phi = None
        self.status = None


class PoissonServer:
    def __init__(self, h_bohr, nn=3, relax='J', eps=2e-10, precision='fp64',
                 budget_bytes=120 * 2**30, max_inflight=64, nstreams=32, device=None,
                 keep_results=False):
        self.h = h_bohr
        self.nn = nn
        self.relax = relax
        self.eps = eps
        self.precision = precision
        self.budget = budget_bytes
        self.max_inflight = max_inflight
        self.device = torch.device(device) if device is not None else torch.device('cuda')
        self.streams = [torch.cuda.Stream(self.device) for _ in range(nstreams)]
        self.free = collections.defaultdict(list)   # N -> [PoissonSolver]
        self.used_bytes = 0
        self.keep_results = keep_results
        self.rejected = 0

    # -- solver pool ---------------------------------------------------------
    def _new_solver(self, N):
        ps = PoissonSolver(self.nn, self.relax, self.eps, precision=self.precision)
        ps.set_grid_descriptor(grid_for(N, self.h, device=self.device))
        need = ps.nbytes() + 2 * int(np.prod(ps.gd.n_c)) * 8  # + the request's phi
        if self.used_bytes + need > self.budget:
            return None
        ps.initialize()
        ps._bytes = need
        self.used_bytes += need
        return ps

    def warm(self, sizes, per_size=1):
        """Create solvers ahead of time, with their graphs captured, so that
        admission does not pay for allocation and capture."""
        for N in sizes:
            while len(self.free[N]) < per_size:
                ps = self._new_solver(N)
                if ps is None:
                    return
                ps.prepare()
                self.free[N].append(ps)

    def _acquire(self, N):
        if self.free[N]:
            return self.free[N].pop()
        return self._new_solver(N)

    # -- serving loop ----------------------------------------------------------
    def run(self, requests):
        """Serve `requests` (Request objects with arrival times in seconds from
        the start of the run).  Returns a summary dict; per-request results are
        stored on the Request objects."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        inflight = []
        ev_pool = []
        si = 0
        t0 = time.perf_counter()
        while pending or inflight:
            now = time.perf_counter() - t0
            # retire finished solves
            still = []
            for job in inflight:
                req, ps, ev, phi = job
                if ev.query():
                    req.done = time.perf_counter() - t0
                    try:
                        req.niter, req.error = ps.result()
                        req.status = 'ok'
                    except Exception as e:  # reported per request
                        req.status = repr(e)
                    if self.keep_results:
                        req.phi = phi
                    self.free[req.N].append(ps)
                    ev_pool.append(ev)
                else:
                    still.append(job)
            inflight = still
            # admit arrived requests
            while pending and pending[0].arrival <= now and len(inflight) < self.max_inflight:
                req = pending[0]
                ps = self._acquire(req.N)
                if ps is None:
                    if not inflight:  # cannot ever fit
                        pending.popleft()
                        req.status = 'rejected: over memory budget'
                        self.rejected += 1
                        continue
                    break
                pending.popleft()
                stream = self.streams[si % len(self.streams)]
                si += 1
                with torch.cuda.stream(stream):
                    phi = torch.zeros(tuple(int(x) for x in ps.gd.n_c), dtype=torch.float64,
                                      device=self.device)
                    ps.solve_async(phi, req.rho)
                    ev = ev_pool.pop() if ev_pool else torch.cuda.Event()
                    ev.record(stream)
                req.admit = time.perf_counter() - t0
                inflight.append((req, ps, ev, phi))
            if not inflight and pending:
                wait = pending[0].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 1e-3))
        wall = time.perf_counter() - t0
        done = [r for r in requests if r.status == 'ok']
        lat = np.array([r.done - r.arrival for r in done]) if done else np.zeros(1)
        return {'requests': len(requests), 'completed': len(done), 'rejected': self.rejected,
                'wall_s': wall, 'solves_per_s': len(done) / wall if wall > 0 else 0.0,
                'p50_ms': float(np.percentile(lat, 50) * 1e3),
                'p99_ms': float(np.percentile(lat, 99) * 1e3),
                'max_err': float(max([r.error for r in done], default=0.0)),
                'device_bytes': self.used_bytes}


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

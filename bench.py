"""Benchmark of the finite-difference path on B200.

Headline workload: band-batched complex Laplace apply (GPAW kinetic operator,
scale = -0.5, nn = 3: the 19-point 6th-order stencil) on 512 complex128 bands
of a 96^3 fully periodic grid, h = 0.18 A, Bloch phases for k = (0.25, 0, 0),
Re/Im ~ N(0, 1).  One step = one apply over all bands.  The metric is the
algorithmic HBM bandwidth, 32 bytes per point (one complex128 read, one
written), in GB/s.  The 7.25 GB input is far larger than the 126 MB L2, so no
flush is needed between steps.

The same JSON line carries, for the dominant kernel, the roofline against the
measured copy bandwidth (MEASURED_PEAKS.json), the end-to-end figure through
the public API with host buffers, the CPU baseline, the clocks seen during
the timed region, and the Poisson solves/s (128^3 zero-boundary grid, 64
Gaussians, eps = 2e-10) of the plain FP64 and the mixed-precision solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU: one process per GPU under torch.distributed.run; every rank applies
the operator to its own 512 bands (weak scaling, no collective on the data
path); the time is the max over ranks.
"""
import argparse
import collections
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BOHR = 0.52917721092
N = 96
NBANDS = 512
BYTES_PER_POINT = 32  # complex128 in + out
K_VEC = (0.25, 0.0, 0.0)
METRIC = 'stencil HBM GB/s (band-batched complex128 Laplace nn=3)'


def workload_config(nbands=NBANDS):
    return {'workload': 'complex128 Laplace nn=3, %d bands x %d^3 periodic, h=0.18 A, '
                        'k=(0.25,0,0)' % (nbands, N),
            'bands': nbands, 'grid': [N, N, N], 'nn': 3, 'dtype': 'complex128',
            'bytes_per_point': BYTES_PER_POINT,
            'l2_policy': 'inputs (7.25 GB) larger than L2 (126 MB); no flush needed'}


def measured_peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def ncu_traffic():
    """Per-launch DRAM bytes of the headline kernel from the committed ncu
    summary (profiles/star_kernel_c128_96.txt: a line 'traffic_bytes_per_launch: X')."""
    path = os.path.join(ROOT, 'profiles', 'star_kernel_c128_96.txt')
    try:
        for line in open(path):
            if line.startswith('traffic_bytes_per_launch:'):
                return float(line.split(':', 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# Clock sampling during the timed region (NVML).
# ---------------------------------------------------------------------------
class ClockSampler:
    REASONS = {0x4: 'sw_power_cap', 0x8: 'hw_slowdown', 0x20: 'sw_thermal_slowdown',
               0x40: 'hw_thermal_slowdown', 0x80: 'hw_power_brake_slowdown'}

    def __init__(self, period=0.02):
        self.period = period
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self.handle = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = self._handle()
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.handle = None

    def _handle(self):
        import torch
        pynvml = self.nvml
        try:
            props = torch.cuda.get_device_properties(torch.cuda.current_device())
            bus = '%08x:%02x:%02x.0' % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            vis = os.environ.get('CUDA_VISIBLE_DEVICES', '0').split(',')[0]
            return pynvml.nvmlDeviceGetHandleByIndex(int(vis) if vis.isdigit() else 0)

    def _sample(self):
        p = self.nvml
        try:
            self.samples.append(p.nvmlDeviceGetClockInfo(self.handle, p.NVML_CLOCK_SM))
            mask = p.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
            for bit, name in self.REASONS.items():
                if mask & bit:
                    self.reasons.add(name)
        except Exception:
            pass

    def _run(self):
        while not self._stop.is_set():
            self._sample()
            time.sleep(self.period)

    def __enter__(self):
        if self.handle is not None:
            self._sample()
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        return self

    def __exit__(self, *exc):
        if self.handle is not None:
            self._stop.set()
            self.thread.join()
            self._sample()

    def result(self):
        if not self.samples:
            return {'sm_mhz': None, 'sm_max_mhz': self.max_mhz, 'reasons': ['unavailable']}
        return {'sm_mhz': float(np.median(self.samples)), 'sm_max_mhz': self.max_mhz,
                'reasons': sorted(self.reasons), 'samples': len(self.samples)}


# ---------------------------------------------------------------------------
# Distributed plumbing (one process per GPU).
# ---------------------------------------------------------------------------
def dist_setup(ngpus):
    import torch
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device('cuda', local))
    else:
        torch.cuda.set_device(0)
    return rank, world


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    from gpaw_b200.parallel import max_over_ranks as mor
    return mor(x) if world > 1 else x


# ---------------------------------------------------------------------------
# CPU baseline / reference arm.
# ---------------------------------------------------------------------------
class CpuStencil:
    """The reference CPU path (oracle/_ref when it was built, else the oracle
    port) applying the workload's operator to a sample of its bands with all
    host threads."""

    def __init__(self, nbands_sample, impl='ref'):
        from oracle import geometry as G
        from oracle import kernels as K
        self.K = K
        self.impl = impl if (impl != 'ref' or K.have_ref()) else 'port'
        self.kind = 'reference' if self.impl == 'ref' else 'port'
        gd = G.Grid((N,) * 3, (N * 0.18 / BOHR,) * 3, 1)
        self.pbc = gd.pbc_c
        self.c, self.o = G.laplace_stencil(gd, -0.5, 3)
        rng = np.random.default_rng(2)
        shape = (nbands_sample,) + tuple(gd.n_c)
        self.a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        self.ph = G.bloch_phases(gd, K_VEC)
        self.threads = os.cpu_count() or 1
        self.isa = K.ISA
        self.nbands = nbands_sample
        self.bytes = BYTES_PER_POINT * nbands_sample * N ** 3

    def step(self):
        self.K.fd_apply(self.c, self.o, self.pbc, self.a, self.ph, nthreads=self.threads,
                        impl=self.impl)

    def rate(self, min_seconds):
        self.step()
        t0 = time.perf_counter()
        reps = 0
        while True:
            self.step()
            reps += 1
            dt = time.perf_counter() - t0
            if dt >= min_seconds:
                return self.bytes * reps / dt / 1e9, reps, dt


def run_reference_arm(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return 0
    cpu = CpuStencil(16)
    for _ in range(args.warmup):
        cpu.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu.step()
    total = time.perf_counter() - t0
    value = float(args.steps * cpu.bytes / total / 1e9)
    sample = '%d of the %d bands per step (%s C path, %d threads, %s build)' % (
        cpu.nbands, NBANDS, cpu.kind, cpu.threads, cpu.isa)
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'GB/s',
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': total / args.steps * 1e3, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'complex128', 'data': 'synthetic',
            'config': workload_config(),
            'cpu_baseline': {'value': value, 'unit': 'GB/s', 'cores': cpu.threads,
                             'kind': cpu.kind, 'sample': sample},
            'e2e': {'value': value, 'unit': 'GB/s', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# Poisson solves/s (128^3 zero boundary, 64 Gaussians, eps = 2e-10).
# ---------------------------------------------------------------------------
def poisson_rho(gd, ng, seed, wall=2.0):
    """ng normalised Gaussians (widths U[0.4, 1.2] A, centres at least `wall`
    A from the walls, charges +-1 summing to zero), mean removed."""
    from math import pi
    rng = np.random.default_rng(seed)
    r = gd.get_grid_point_coordinates()
    L = gd.cell_cv.diagonal()
    q = np.array([1.0] * (ng // 2) + [-1.0] * (ng // 2))
    rng.shuffle(q)
    rho = np.zeros(tuple(gd.n_c))
    for i in range(ng):
        s = rng.uniform(0.4, 1.2) / BOHR
        R = rng.uniform(wall / BOHR, L - wall / BOHR)
        d2 = sum((r[c] - R[c]) ** 2 for c in range(3))
        rho += q[i] * (2 * pi * s * s) ** -1.5 * np.exp(-d2 / (2 * s * s))
    return rho - rho.mean()


def poisson_bench(nsolves=8, tune=True, check=True):
    import torch
    from gpaw_b200.grid_descriptor import GridDescriptor
    from gpaw_b200.poisson import PoissonSolver
    Np = 128
    gd = GridDescriptor((Np,) * 3, (Np * 0.2 / BOHR,) * 3, 0)
    rho_h = poisson_rho(gd, 64, 3)
    rho = torch.from_numpy(rho_h).cuda()
    out = {'workload': '128^3 zero boundary, h=0.2 A, 64 Gaussians, nn=3, Jacobi, eps=2e-10'}
    phis = {}
    for prec in ('fp64', 'mixed'):
        ps = PoissonSolver(3, 'J', 2e-10, precision=prec)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        if tune:
            ps.autotune(reps=5)
        phi = torch.zeros_like(rho)
        ps.solve(phi, rho)  # warm-up
        lat = []
        for _ in range(nsolves):
            phi.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            niter = ps.solve(phi, rho)
            torch.cuda.synchronize()
            lat.append(time.perf_counter() - t0)
        phis[prec] = phi.cpu().numpy()
        lat = np.array(lat)
        out[prec] = {'solves_per_s': float(1.0 / lat.mean()), 'p50_ms': float(np.median(lat) * 1e3),
                     'p99_ms': float(np.percentile(lat, 99) * 1e3), 'vcycles': int(niter),
                     'residual': float(ps.error), 'autotuned': bool(tune)}
    out['mixed_vs_fp64_speedup'] = out['mixed']['solves_per_s'] / out['fp64']['solves_per_s']
    out['mixed_max_abs_vs_fp64'] = float(np.abs(phis['mixed'] - phis['fp64']).max())
    if check:
        out['oracle'] = poisson_oracle_check(gd, rho_h, phis, out)
    return out, phis, rho_h, gd


def poisson_oracle_check(gd, rho_h, phis, out):
    """The same solve by the CPU oracle (the reference's V-cycle restated
    over its C kernels): V-cycle count and max-abs error of the timed GPU
    potentials against it."""
    from oracle import geometry as G
    from oracle import poisson as OP
    og = G.Grid(gd.N_c, gd.cell_cv, gd.pbc_c)
    ps = OP.PoissonSolver(3, 'J', 2e-10)
    ps.set_grid_descriptor(og)
    ps.initialize()
    phi_o = np.zeros(tuple(og.n_c))
    t0 = time.perf_counter()
    n_o = ps.solve(phi_o, rho_h)
    dt = time.perf_counter() - t0
    return {'vcycles': int(n_o), 'residual': float(ps.errors[-1]), 'cpu_seconds': dt,
            'fp64_vcycles_match': int(n_o) == out['fp64']['vcycles'],
            'fp64_max_abs_vs_oracle': float(np.abs(phis['fp64'] - phi_o).max()),
            'mixed_max_abs_vs_oracle': float(np.abs(phis['mixed'] - phi_o).max()),
            'bars': {'fp64': 1e-10, 'mixed': 1e-9}}


# ---------------------------------------------------------------------------
# Poisson serving: requests arriving as a Poisson process, grids drawn from
# {32, 48, 64, 96, 128, 160}^3 (zero boundary, h = 0.2 A), rho a pair density
# of two 8-Gaussian orbitals, eps = 2e-10, 120 GB admission budget.
# ---------------------------------------------------------------------------
SERVING_SIZES = (32, 48, 64, 96, 128, 160)


def serving_bench(rates=(100.0, 300.0, 1000.0, 3000.0, 5000.0), nreq=10000,
                  precisions=('fp64', 'mixed'), seed=5, low_rate_seconds=3.0, ndens=256,
                  check=True):
    """The request stream: `nreq` requests per rate at 1000/s and above; at the
    lower rates about `low_rate_seconds` of arrivals (10,000 requests at
    100/s would take 100 s).  Each request's rho is one of `ndens` seeded
    pair densities of its grid size (request i of size N takes density
    i mod ndens).  check: a sample of requests -- the first two of each size
    up to 96^3 at the highest rate -- is compared with the FP64 oracle's
    solve of the same rho."""
    import torch
    from gpaw_b200.serving import PoissonServer, Request, grid_for, pair_density
    h = 0.2 / BOHR
    rng = np.random.default_rng(seed)
    dens = {N: [pair_density(grid_for(N, h), 1000 * N + k) for k in range(ndens)]
            for N in SERVING_SIZES}
    torch.cuda.synchronize()
    out = {'workload': '%d requests per rate >= 1000/s (%.0f s of arrivals below), grids %s^3 '
                       'zero boundary, h=0.2 A, pair densities (%d seeded per size), eps=2e-10, '
                       'budget 120 GB' % (nreq, low_rate_seconds, list(SERVING_SIZES), ndens)}
    streams = {}
    for lam in rates:
        m = nreq if lam >= 1000 else int(lam * low_rate_seconds)
        gaps = rng.exponential(1.0 / lam, m)
        t = np.cumsum(gaps) - gaps[0]
        streams[lam] = (t, rng.choice(SERVING_SIZES, m))
    sample = {}
    for prec in precisions:
        srv = PoissonServer(h, precision=prec, max_inflight=64, nstreams=32)
        srv.warm(SERVING_SIZES, per_size=24, pod_requests=64)
        res = {}
        for lam in rates:
            t, sizes = streams[lam]
            seen = collections.Counter()
            reqs = []
            for i, N in enumerate(sizes):
                N = int(N)
                reqs.append(Request(i, N, float(t[i]), dens[N][seen[N] % ndens]))
                seen[N] += 1
            last = lam == rates[-1]
            srv.keep_results = False
            srv.run([Request(-1, r.N, 0.0, r.rho) for r in reqs[:16]])  # warm (not timed)
            picked = collections.defaultdict(list)
            if check and last:
                # the sample: the first two requests of each size up to 96^3;
                # only their potentials are copied out during the run
                for r in reqs:
                    if r.N <= 96 and len(picked[r.N]) < 2:
                        picked[r.N].append(r)
                ids = {r.rid for rs in picked.values() for r in rs}
                srv.keep_results = lambda r: r.rid in ids
            stats = srv.run(reqs)
            res['%g/s' % lam] = {k: stats[k] for k in (
                'requests', 'completed', 'solves_per_s', 'wall_s', 'p50_ms', 'p99_ms',
                'max_residual', 'rejected', 'expired', 'cancelled', 'failed')}
            if check and last:
                sample[prec] = [(r.N, r.rho, r.phi.cpu().numpy())
                                for N in picked for r in picked[N] if r.status == 'ok']
            srv.keep_results = False
        res['device_bytes'] = srv.used_bytes
        out[prec] = res
        del srv
        torch.cuda.empty_cache()
    if check:
        out['oracle_check'] = serving_oracle_check(sample, h)
    return out


def serving_oracle_check(sample, h):
    """Max-abs error of sampled served potentials against the oracle's FP64
    solve of the same rho (the reference's V-cycle over its C kernels)."""
    from oracle import geometry as G
    from oracle import poisson as OP
    cache = {}
    worst = {}
    t0 = time.perf_counter()
    for prec, items in sample.items():
        errs = []
        for N, rho_t, phi in items:
            key = (N, id(rho_t))
            if key not in cache:
                og = G.Grid((N,) * 3, (N * h,) * 3, 0)
                ps = OP.PoissonSolver(3, 'J', 2e-10)
                ps.set_grid_descriptor(og)
                ps.initialize()
                phi_o = np.zeros(tuple(og.n_c))
                ps.solve(phi_o, rho_t.cpu().numpy())
                cache[key] = phi_o
            errs.append(float(np.abs(phi - cache[key]).max()))
        worst[prec] = {'requests_checked': len(items), 'max_abs_vs_oracle': max(errs, default=None)}
    worst['bars'] = {'fp64': 1e-10, 'mixed': 1e-9}
    worst['cpu_seconds'] = time.perf_counter() - t0
    return worst


def small_batch_bench(n=128, N=32):
    """n independent Gauss-Seidel solves of N^3 in one graph launch: small
    solvers of one structure run grouped (one persistent launch per V-cycle
    step over all grids, work tiles pulled from a queue)."""
    import torch
    from gpaw_b200.poisson import PoissonSolver
    from gpaw_b200.serving import PoissonBatch, grid_for
    h = 0.2 / BOHR
    solvers, rhos, phis = [], [], []
    for i in range(n):
        gd = grid_for(N, h)
        ps = PoissonSolver(3, 'GS', 2e-10)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        solvers.append(ps)
        rhos.append(torch.from_numpy(poisson_rho(gd, 4, 900 + i, wall=1.0)).cuda())
        phis.append(torch.zeros_like(rhos[-1]))
    batch = PoissonBatch(solvers)
    batch.solve(phis, rhos)
    best = None
    for _ in range(3):
        for p in phis:
            p.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = batch.solve(phis, rhos)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return {'workload': '%d solves of %d^3, GS, one launch' % (n, N), 'seconds': best,
            'solves_per_s': n / best, 'grouped_solvers': batch.grouped,
            'vcycles': sorted(set(r[0] for r in res)),
            'max_residual': max(r[1] for r in res)}


def batch_bench(transfer_bands=256, tune=True):
    """32 simultaneous solves (8 each of 48, 64, 80, 96 points per axis, 16
    Gaussians, multicolour Gauss-Seidel) in one graph launch, and band-
    batched restriction/interpolation of 256 float64 bands 224^3 <-> 112^3
    (nn=3, periodic).  tune: autotune the launch plans first (one solver per
    grid size; the others share its plans through the cache)."""
    import torch
    from gpaw_b200 import autotune
    from gpaw_b200.poisson import PoissonSolver
    from gpaw_b200.serving import PoissonBatch, grid_for
    from gpaw_b200.transformers import Transformer
    from gpaw_b200.grid_descriptor import GridDescriptor
    h = 0.2 / BOHR
    solvers, rhos, phis = [], [], []
    for i, N in enumerate([48] * 8 + [64] * 8 + [80] * 8 + [96] * 8):
        gd = grid_for(N, h)
        ps = PoissonSolver(3, 'GS', 2e-10)
        ps.set_grid_descriptor(gd)
        ps.initialize()
        if tune and i % 8 == 0:
            ps.autotune(reps=3)
        solvers.append(ps)
        rhos.append(torch.from_numpy(poisson_rho(gd, 16, 40 + i)).cuda())
        phis.append(torch.zeros_like(rhos[-1]))
    batch = PoissonBatch(solvers)  # captured with the tuned plans
    batch.solve(phis, rhos)  # warm-up (captures the graph)
    for p in phis:
        p.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = batch.solve(phis, rhos)
    dt = time.perf_counter() - t0
    small = small_batch_bench()
    out = {'poisson_batch_small': small,
           'poisson_batch': {'workload': '32 solves, 8 each of 48,64,80,96^3, GS, one launch',
                             'seconds': dt, 'solves_per_s': 32 / dt,
                             'vcycles': [r[0] for r in res], 'max_residual': max(r[1] for r in res),
                             'autotuned': bool(tune)}}
    coarse = GridDescriptor((112,) * 3, (112 * 0.3,) * 3, 1)
    fine = coarse.refine()
    g = torch.Generator(device='cuda')
    g.manual_seed(4)
    nb = transfer_bands
    c = torch.rand((nb, 112, 112, 112), dtype=torch.float64, device='cuda', generator=g) * 2 - 1
    f = torch.empty((nb, 224, 224, 224), dtype=torch.float64, device='cuda')
    ip = Transformer(coarse, fine, 3)
    rs = Transformer(fine, coarse, 3)
    plans = None
    if tune:
        plans = {'interpolate': autotune.tune_transformer(ip, nb, reps=2),
                 'restrict': autotune.tune_transformer(rs, nb, reps=2)}
    for _ in range(2):
        ip.apply(c, f)
        rs.apply(f, c)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    ip.apply(c, f)
    ev[1].record()
    rs.apply(f, c)
    ev[2].record()
    torch.cuda.synchronize()
    nfine = nb * 224 ** 3
    t_ip = ev[0].elapsed_time(ev[1]) * 1e-3
    t_rs = ev[1].elapsed_time(ev[2]) * 1e-3
    out['transfers'] = {'workload': '%d float64 bands, 112^3 <-> 224^3, nn=3, periodic' % nb,
                        'interpolate_GBps': 9 * nfine / t_ip / 1e9,
                        'restrict_GBps': 9 * nfine / t_rs / 1e9,
                        'interpolate_ms': t_ip * 1e3, 'restrict_ms': t_rs * 1e3,
                        'launch_plans': plans}
    del c, f
    return out


# ---------------------------------------------------------------------------
# Pseudo-Hamiltonian on the headline bands: kin psit + vt psit fused in one
# pass against the reference's two passes (kinetic apply, then
# Htpsit += psit * vt as a separate elementwise update).
# ---------------------------------------------------------------------------
def hamiltonian_bench(lap, a, b, phase, steps):
    import torch
    g = torch.Generator(device='cuda')
    g.manual_seed(9)
    vt = torch.rand(tuple(a.shape[1:]), dtype=torch.float64, device='cuda', generator=g) - 0.5

    def timed(fn):
        for _ in range(3):
            fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def two_pass():
        lap.apply(a, b, phase)
        b.addcmul_(a, vt)

    fused_ms = timed(lambda: lap.apply_with_potential(a, b, vt, phase))
    two_ms = timed(two_pass)
    nbytes = BYTES_PER_POINT * a.numel()
    return {'workload': 'kin psit + vt psit, %d complex128 bands x %d^3, k=(0.25,0,0)'
                        % (a.shape[0], a.shape[1]),
            'fused_ms': fused_ms, 'fused_GBps': nbytes / (fused_ms * 1e-3) / 1e9,
            'two_pass_ms': two_ms, 'speedup_vs_two_pass': two_ms / fused_ms,
            'bytes_per_point': BYTES_PER_POINT}


# ---------------------------------------------------------------------------
# The rest of the stencil configurations: Gradient(v, 1.0, n=3) on the
# headline bands, the complex64 (FP32) copy of the Laplace workload, and the
# plain FP64 Laplace of 16 x 47^3 (too small for bandwidth: its latency).
# ---------------------------------------------------------------------------
def stencil_variants_bench(gd, a, b, phase, steps):
    import torch
    from gpaw_b200.fd_operators import Gradient, Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor

    def timed(fn, n):
        for _ in range(3):
            fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {}
    nbytes = BYTES_PER_POINT * a.numel()
    for v in range(3):
        grad = Gradient(gd, v, 1.0, 3, complex)
        ms = timed(lambda: grad.apply(a, b, phase), steps)
        out['gradient%d_GBps' % v] = nbytes / (ms * 1e-3) / 1e9
    lap32 = Laplace(gd, -0.5, 3, np.complex64)
    a32 = a.to(torch.complex64)
    b32 = torch.empty_like(a32)
    ms = timed(lambda: lap32.apply(a32, b32, phase), steps)
    out['complex64_laplace_GBps'] = 16 * a32.numel() / (ms * 1e-3) / 1e9
    # the FP32 variant's error against the FP64 apply of the same bands
    Laplace(gd, -0.5, 3, complex).apply(a, b, phase)
    err = 0.0
    for i in range(0, a.shape[0], 64):
        d = (b32[i:i + 64].to(torch.complex128) - b[i:i + 64]).abs().max().item()
        err = max(err, d)
    out['complex64_laplace_max_rel_err_vs_fp64'] = err / b.abs().max().item()
    del a32, b32
    N1 = 48
    gd1 = GridDescriptor((N1,) * 3, (N1 * 0.2 / BOHR,) * 3, 0)
    lap1 = Laplace(gd1, -0.5, 3)
    g = torch.Generator(device='cuda')
    g.manual_seed(1)
    x = torch.rand((16,) + tuple(int(n) for n in gd1.n_c), dtype=torch.float64, device='cuda',
                   generator=g) * 2 - 1
    y = torch.empty_like(x)
    ms = timed(lambda: lap1.apply(x, y), 200)
    out['plain_fp64_16x47_us'] = ms * 1e3
    out['plain_fp64_16x47_GBps'] = 16 * x.numel() / (ms * 1e-3) / 1e9
    out['workload'] = ('Gradient v=0,1,2 and complex64 Laplace on %d bands x 96^3 (32 / 16 B '
                       'per point); float64 Laplace nn=3 on 16 x 47^3 zero boundary'
                       % a.shape[0])
    return out


# ---------------------------------------------------------------------------
# Band preconditioner (gpaw/preconditioner.py) on the headline bands: the
# eight-pass device form against the reference's nineteen-operation
# sequence written with this library's unfused calls.
# ---------------------------------------------------------------------------
def preconditioner_bench(gd, lap, a, b, phase, steps):
    import torch
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.preconditioner import Preconditioner
    from gpaw_b200.transformers import Transformer
    nb = a.shape[0]
    pc = Preconditioner(gd, lap, complex, block=nb)
    gd1 = gd.coarsen()
    gd2 = gd1.coarsen()
    kin1 = Laplace(gd1, -0.5, 1, complex)
    kin2 = Laplace(gd2, -0.5, 1, complex)
    r0, r1_ = Transformer(gd, gd1, 1, complex), Transformer(gd1, gd2, 1, complex)
    i2, i1 = Transformer(gd2, gd1, 1, complex), Transformer(gd1, gd, 1, complex)
    sh1 = (nb,) + tuple(int(x) for x in gd1.n_c)
    sh2 = (nb,) + tuple(int(x) for x in gd2.n_c)
    r1, d1, q1 = (torch.empty(sh1, dtype=a.dtype, device=a.device) for _ in range(3))
    r2, q2 = (torch.empty(sh2, dtype=a.dtype, device=a.device) for _ in range(2))
    step = pc.step

    class K:
        phase_cd = phase

    def unfused():
        # gpaw/preconditioner.py:48-70, one array operation per line
        r0.apply(-a, r1, phase)
        d1.copy_(4 * step * r1)
        kin1.apply(d1, q1, phase)
        q1.sub_(r1)
        r1_.apply(q1, r2, phase)
        d2 = 16 * step * r2
        kin2.apply(d2, q2, phase)
        q2.sub_(r2)
        d2.sub_(16 * step * q2)
        i2.apply(d2, q1, phase)
        d1.sub_(q1)
        kin1.apply(d1, q1, phase)
        q1.sub_(r1)
        d1.sub_(4 * step * q1)
        i1.apply(-d1, b, phase)
        q0 = torch.empty_like(b)
        lap.apply(b, q0, phase)
        q0.sub_(a)
        b.add_(q0, alpha=-step)
        b.mul_(-1.0)

    def timed(fn):
        for _ in range(2):
            fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    fused_ms = timed(lambda: pc(a, K))
    unfused_ms = timed(unfused)
    del pc
    return {'workload': 'Preconditioner (gpaw/preconditioner.py), %d complex128 bands x %d^3, '
                        'kin0 nn=3, k=(0.25,0,0)' % (nb, a.shape[1]),
            'device_passes_ms': fused_ms, 'reference_sequence_ms': unfused_ms,
            'speedup': unfused_ms / fused_ms}


def headline_oracle_check(lap, a, b, phase):
    """Max relative error (max |gpu - oracle| / max |oracle|) of the last
    timed apply on the first, middle and last band against the oracle."""
    from oracle import kernels as K
    idx = sorted({0, a.shape[0] // 2, a.shape[0] - 1})
    a_h = a[idx].cpu().numpy()
    b_h = b[idx].cpu().numpy()
    ref = K.fd_apply(lap.coef_p, lap.offset_pc, lap.gd.pbc_c, a_h, phase,
                     nthreads=os.cpu_count() or 1)
    err = float(np.abs(b_h - ref).max() / np.abs(ref).max())
    return {'bands_checked': idx, 'max_rel_err_vs_oracle': err, 'bar': 1e-13,
            'oracle': 'C restatement of c/bmgs/fd.c + c/bc.c (bit-equal to the reference C)'}


# ---------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------
def run_gpu_arm(args):
    import torch
    rank, world = dist_setup(args.gpus)
    from gpaw_b200.fd_operators import Laplace
    from gpaw_b200.grid_descriptor import GridDescriptor

    gd = GridDescriptor((N,) * 3, (N * 0.18 / BOHR,) * 3, 1)
    lap = Laplace(gd, -0.5, 3, complex)
    phase = np.exp(2j * np.pi * gd.sdisp_cd * np.array(K_VEC)[:, None])
    g = torch.Generator(device='cuda')
    g.manual_seed(2 + rank)
    nb = args.bands
    shape = (nb,) + tuple(int(x) for x in gd.n_c)
    a = torch.complex(torch.randn(shape, dtype=torch.float64, device='cuda', generator=g),
                      torch.randn(shape, dtype=torch.float64, device='cuda', generator=g))
    b = torch.empty_like(a)
    stream = torch.cuda.current_stream()
    nbytes = BYTES_PER_POINT * nb * N ** 3
    plan = None
    if not args.no_autotune:
        from gpaw_b200 import autotune
        plan = autotune.tune_operator(lap, nb, phase_cd=phase, reps=3)

    for _ in range(args.warmup):
        lap.apply(a, b, phase)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler() as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            lap.apply(a, b, phase)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = max_over_ranks(ms, world)
    value = world * nbytes / (ms_max * 1e-3) / 1e9
    kernel_gbs = nbytes / (ms * 1e-3) / 1e9

    # End to end through the public API with host buffers: every step copies
    # all bands in from pinned host memory, applies and copies the result
    # back (HostStreamer overlaps the copies in both directions and the
    # kernel, in chunks of bands).
    e2e = None
    if args.e2e_steps > 0:
        from gpaw_b200.streaming import HostStreamer
        e2e_steps = min(args.steps, args.e2e_steps)
        try:
            host_in = torch.empty(shape, dtype=torch.complex128, pin_memory=True)
            host_out = torch.empty(shape, dtype=torch.complex128, pin_memory=True)
            pinned = True
        except RuntimeError:  # page-locking refused (memlock limit): pageable copies
            host_in = torch.empty(shape, dtype=torch.complex128)
            host_out = torch.empty(shape, dtype=torch.complex128)
            pinned = False
        host_in.copy_(a)
        streamer = HostStreamer(lap, chunk_bands=16)
        streamer.apply(host_in, host_out, phase)  # warm-up (device buffers)
        torch.cuda.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            streamer.apply(host_in, host_out, phase)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, world)
        e2e = {'value': world * nbytes / (e2e_ms * 1e-3) / 1e9, 'unit': 'GB/s',
               'steps': e2e_steps, 'h2d_bytes_per_step': nbytes // 2,
               'd2h_bytes_per_step': nbytes // 2,
               'api': 'gpaw_b200.streaming.HostStreamer.apply, 16-band chunks',
               'pinned_host_memory': pinned}
        del host_in, host_out, streamer

    # The timed output, checked: three of this rank's bands against the
    # oracle (the reference's stencil and Bloch halo restated in C).
    check = headline_oracle_check(lap, a, b, phase) if not args.no_cpu else None

    ham = pcb = var = None
    if rank == 0 and world == 1 and not args.no_hamiltonian:
        ham = hamiltonian_bench(lap, a, b, phase, min(args.steps, 20))
        pcb = preconditioner_bench(gd, lap, a, b, phase, min(args.steps, 10))
        var = stencil_variants_bench(gd, a, b, phase, min(args.steps, 20))

    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic()
    line = {'metric': METRIC, 'value': value, 'unit': 'GB/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms_max,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'complex128', 'data': 'synthetic (seeded N(0,1) bands)',
            'config': dict(workload_config(nb), parallelism='bands sharded, %d per GPU' % nb),
            'roofline': {'bound': 'hbm', 'achieved': kernel_gbs, 'peak': peak, 'unit': 'GB/s',
                         'frac': kernel_gbs / peak, 'peak_kind': peak_kind,
                         'traffic': traffic, 'algorithmic_bytes_per_launch': nbytes,
                         'kernel': ('star_direct_kernel<cplx<double>,R=3>'
                                    if plan and plan['form'] == 'direct'
                                    else 'star_kernel<cplx<double>,R=3>')},
            'launch_plan': plan,
            'check': check,
            'e2e': e2e,
            'gpu_launches': args.steps,
            'clocks': clocks.result()}
    if ham is not None:
        line['hamiltonian'] = ham
    if pcb is not None:
        line['preconditioner'] = pcb
    if var is not None:
        line['stencil_variants'] = var
    if rank == 0 and world == 1 and not args.no_poisson:
        try:
            pb, _, _, _ = poisson_bench(tune=not args.no_autotune)
            line['poisson'] = pb
        except Exception as e:  # reported, never hidden
            line['poisson'] = {'error': repr(e)}
    if rank == 0 and world == 1 and not args.no_poisson and not args.no_serving:
        try:
            line['serving'] = serving_bench(nreq=args.requests, check=not args.no_cpu)
            line.update(batch_bench(tune=not args.no_autotune))
        except Exception as e:  # reported, never hidden
            line['serving'] = {'error': repr(e)}
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = CpuStencil(16)
        r, reps, dt = cpu.rate(args.cpu_seconds)
        line['cpu_baseline'] = {'value': r, 'unit': 'GB/s', 'cores': cpu.threads,
                                'kind': cpu.kind,
                                'sample': '16 of the 512 bands, %d passes in %.1f s '
                                          '(%s build)' % (reps, dt, cpu.isa)}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--e2e-steps', type=int, default=3, help='0 skips the end-to-end leg')
    ap.add_argument('--bands', type=int, default=NBANDS,
                    help='bands per GPU (smaller cases for profiling only)')
    ap.add_argument('--cpu-seconds', type=float, default=10.0)
    ap.add_argument('--no-poisson', action='store_true')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--only', choices=['poisson', 'serving', 'batch'], default=None,
                    help='run only the Poisson solves/s sub-benchmark (profiling)')
    ap.add_argument('--solves', type=int, default=8, help='timed solves per precision')
    ap.add_argument('--requests', type=int, default=10000,
                    help='serving requests per rate at 1000/s and above')
    ap.add_argument('--no-serving', action='store_true')
    ap.add_argument('--no-hamiltonian', action='store_true')
    ap.add_argument('--no-autotune', action='store_true',
                    help='keep the built-in launch rules (no plan tuning before timing)')
    ap.add_argument('--transfer-bands', type=int, default=256,
                    help='bands of the transfer sub-benchmark (--only batch; smaller for profiling)')
    args = ap.parse_args()
    if args.impl == 'reference':
        return run_reference_arm(args)
    if args.only:
        import torch
        torch.cuda.set_device(0)
        if args.only == 'poisson':
            pb, _, _, _ = poisson_bench(args.solves, not args.no_autotune)
            print(json.dumps({'poisson': pb}))
        elif args.only == 'serving':
            print(json.dumps({'serving': serving_bench(nreq=args.requests,
                                                       check=not args.no_cpu)}))
        else:
            print(json.dumps(batch_bench(args.transfer_bands, not args.no_autotune)))
        return 0
    return run_gpu_arm(args)


if __name__ == '__main__':
    sys.exit(main())

"""Nested timers and a JSON-lines metrics stream.

Timer follows the interface of gpaw/utilities/timing.py:86-166 (start /
stop by stack order, get_time by the tuple of nested names, write as an
inclusive / exclusive table, add).  The operators here are asynchronous, so a
host clock around a call measures its launch, not its work: CudaTimer keeps
the same interface but records a CUDA event pair on the current stream for
every region (and an NVTX range, so a profiler timeline shows the names), and
resolves the times when they are read.

MetricsLog writes one JSON object per line (per-request records of the
Poisson server, summaries, timer tables) to a file or a stream.
"""
import json
import sys
import time

import torch


class Timer:
    """Host-clock nested timer (gpaw/utilities/timing.py:86-166)."""

    def __init__(self, print_levels=1000):
        self.timers = {}
        self.t0 = time.time()
        self.running = []
        self.print_levels = print_levels

    def start(self, name):
        names = tuple(self.running + [name])
        self.timers[names] = self.timers.get(names, 0.0) - time.time()
        self.running.append(name)

    def _check_top(self, name):
        if not self.running:
            raise RuntimeError('No timer is running')
        if name is None:
            name = self.running[-1]
        if name != self.running[-1]:
            raise RuntimeError('Must stop timers by stack order.  Requested stopping '
                               'of %s but topmost is %s' % (name, self.running[-1]))

    def stop(self, name=None):
        self._check_top(name)
        names = tuple(self.running)
        self.running.pop()
        self.timers[names] += time.time()

    def get_time(self, *names):
        return self.totals()[names]

    def add(self, timer):
        for names, t in timer.totals().items():
            self.timers[names] = self.timers.get(names, 0.0) + t

    def totals(self):
        """Inclusive seconds per tuple of nested names (finished regions)."""
        return dict(self.timers)

    def table(self):
        """Rows (names, inclusive s, exclusive s) in sorted order, then
        ('Other',) for the wall time outside every top-level region; and the
        wall time since the timer was made.  Stops running regions first."""
        while self.running:
            self.stop()
        tot = time.time() - self.t0
        incl = self.totals()
        excl = dict(incl)
        other = tot
        for names, t in incl.items():
            if len(names) > 1:
                if len(names) <= self.print_levels and names[:-1] in excl:
                    excl[names[:-1]] -= t
            else:
                other -= t
        rows = [(names, incl[names], excl[names]) for names in sorted(incl)]
        rows.append((('Other',), other, other))
        return rows, tot

    def write(self, out=sys.stdout):
        rows, tot = self.table()
        if len(rows) == 1:
            return
        n = max(len(names[-1]) + len(names) for names, _, _ in rows) + 1
        bar = '=' * 60
        out.write('\n%s\n%-*s    incl.     excl.\n%s\n' % (bar, n, 'Timing:', bar))
        for names, ti, te in rows:
            if len(names) > self.print_levels:
                continue
            r = te / tot if tot > 0 else 0.0
            i = int(40 * r + 0.5)
            mark = '|' if i == 0 else '|%s|' % ('-' * (i - 1))
            name = (len(names) - 1) * ' ' + names[-1] + ':'
            out.write('%-*s%9.3f %9.3f %5.1f%% %s\n' % (n, name, ti, te, 100 * r, mark))
        out.write('%s\n%-*s%9.3f %5.1f%%\n%s\n' % (bar, n + 10, 'Total:', tot, 100.0, bar))
        out.write('date: %s\n' % time.asctime())


class NullTimer:
    """Same interface as Timer; does nothing."""

    def start(self, name):
        pass

    def stop(self, name=None):
        pass

    def add(self, timer):
        pass

    def write(self, out=sys.stdout):
        pass


class CudaTimer(Timer):
    """Device-time nested timer: each region is a CUDA event pair on the
    stream that is current at start (and an NVTX range).  Reading the times
    waits for the recorded events, not for the whole device."""

    def __init__(self, print_levels=1000, nvtx=True):
        super().__init__(print_levels)
        self.nvtx = nvtx
        self.open = []       # (names, start event, stream) of running regions
        self.pairs = {}      # names -> [(start, end)] not yet resolved

    def start(self, name):
        names = tuple(self.running + [name])
        stream = torch.cuda.current_stream()
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        if self.nvtx:
            torch.cuda.nvtx.range_push(name)
        self.running.append(name)
        self.open.append((names, ev, stream))

    def stop(self, name=None):
        self._check_top(name)
        names, ev0, stream = self.open.pop()
        ev1 = torch.cuda.Event(enable_timing=True)
        ev1.record(stream)
        if self.nvtx:
            torch.cuda.nvtx.range_pop()
        self.running.pop()
        self.pairs.setdefault(names, []).append((ev0, ev1))

    def totals(self):
        for names, pairs in self.pairs.items():
            t = 0.0
            for a, b in pairs:
                b.synchronize()
                t += a.elapsed_time(b) * 1e-3
            self.timers[names] = self.timers.get(names, 0.0) + t
        self.pairs = {}
        return dict(self.timers)


class MetricsLog:
    """JSON-lines writer: log(kind, **fields) writes
    {"t": seconds since creation, "kind": kind, ...fields} as one line.
    `target` is a path (opened for append) or a text stream."""

    def __init__(self, target):
        self.t0 = time.time()
        if isinstance(target, str):
            self.out = open(target, 'a')
            self.owned = True
        else:
            self.out = target
            self.owned = False

    def log(self, kind, **fields):
        rec = {'t': round(time.time() - self.t0, 6), 'kind': kind}
        rec.update(fields)
        self.out.write(json.dumps(rec, default=_plain) + '\n')

    def timer(self, timer, kind='timing'):
        """One record per region of a Timer / CudaTimer (nested name joined
        by '.', inclusive and exclusive seconds) and one for the total."""
        rows, tot = timer.table()
        for names, ti, te in rows:
            self.log(kind, region='.'.join(names), incl_s=ti, excl_s=te)
        self.log(kind, region='Total', incl_s=tot, excl_s=tot)

    def flush(self):
        self.out.flush()

    def close(self):
        self.out.flush()
        if self.owned:
            self.out.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _plain(x):
    """numpy / torch scalars to Python numbers for json."""
    try:
        return x.item()
    except AttributeError:
        return str(x)

"""Band operators on host arrays: copies and kernels overlapped in chunks.

GPAW keeps its wave functions in host memory (numpy arrays).  A caller that
applies a device operator to host bands pays two PCIe transfers per band;
done one after the other, transfer in, apply, transfer out, the PCIe link
works in one direction at a time and the GPU waits.  HostStreamer splits the
bands into chunks and runs three streams, so the host-to-device copy of chunk
k+1, the kernel on chunk k and the device-to-host copy of chunk k-1 overlap:
both link directions stay busy and the kernel time hides behind the copies.
"""
import torch

from .tensors import is_complex


class HostStreamer:
    """Apply `op` (an FDOperator: Laplace, Gradient, ...) to bands that live
    in host memory.  in/out host tensors should be pinned
    (tensor.pin_memory()) for the copies to overlap; chunk_bands bands move
    per copy, through two device buffers per direction."""

    def __init__(self, op, chunk_bands=16, device=None):
        self.op = op
        self.chunk = int(chunk_bands)
        if self.chunk < 1:
            raise ValueError('chunk_bands must be at least 1')
        self.device = torch.device(device) if device is not None else torch.device('cuda')
        self.h2d = torch.cuda.Stream(self.device)
        self.comp = torch.cuda.Stream(self.device)
        self.d2h = torch.cuda.Stream(self.device)
        self._buf = None

    def _buffers(self, shape, dtype):
        key = (tuple(shape), dtype)
        if self._buf is None or self._buf[0] != key:
            mk = lambda: torch.empty(shape, dtype=dtype, device=self.device)  # noqa: E731
            self._buf = (key, [mk(), mk()], [mk(), mk()])
        return self._buf[1], self._buf[2]

    def apply(self, in_host, out_host, phase_cd=None, vt_g=None):
        """out_host = op(in_host) (plus vt_g * in_host when a device potential
        vt_g is given: the fused pseudo-Hamiltonian).  The caller's current
        stream waits for the last copy back; synchronise it before reading
        out_host on the host."""
        if in_host.is_cuda or out_host.is_cuda:
            raise ValueError('HostStreamer.apply takes host tensors; use op.apply on device')
        if tuple(in_host.shape) != tuple(out_host.shape) or in_host.dtype != out_host.dtype:
            raise ValueError('input and output must have the same shape and dtype')
        if in_host.dim() != 4:
            raise ValueError('bands must have shape (nbands,) + grid')
        if is_complex(in_host.dtype) != is_complex(self.op.dtype):
            raise ValueError('operator built for %s arrays, got %s' % (self.op.dtype, in_host.dtype))
        nb = in_host.shape[0]
        shape = (min(self.chunk, nb),) + tuple(in_host.shape[1:])
        din, dout = self._buffers(shape, in_host.dtype)
        cur = torch.cuda.current_stream(self.device)
        for s in (self.h2d, self.comp, self.d2h):
            s.wait_stream(cur)
        ev = {name: [torch.cuda.Event(), torch.cuda.Event()] for name in ('in', 'run', 'out')}
        for k, b0 in enumerate(range(0, nb, self.chunk)):
            m = min(self.chunk, nb - b0)
            slot = k % 2
            with torch.cuda.stream(self.h2d):
                if k >= 2:
                    self.h2d.wait_event(ev['run'][slot])  # chunk k-2 has read din[slot]
                din[slot][:m].copy_(in_host[b0:b0 + m], non_blocking=True)
                ev['in'][slot].record(self.h2d)
            with torch.cuda.stream(self.comp):
                self.comp.wait_event(ev['in'][slot])
                if k >= 2:
                    self.comp.wait_event(ev['out'][slot])  # chunk k-2 has left dout[slot]
                if vt_g is None:
                    self.op.apply(din[slot][:m], dout[slot][:m], phase_cd)
                else:
                    self.op.apply_with_potential(din[slot][:m], dout[slot][:m], vt_g, phase_cd)
                ev['run'][slot].record(self.comp)
            with torch.cuda.stream(self.d2h):
                self.d2h.wait_event(ev['run'][slot])
                out_host[b0:b0 + m].copy_(dout[slot][:m], non_blocking=True)
                ev['out'][slot].record(self.d2h)
        cur.wait_stream(self.d2h)
        cur.wait_stream(self.comp)
        cur.wait_stream(self.h2d)
        return out_host

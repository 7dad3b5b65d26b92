"""Volumes larger than one launch, streamed through the GPU in chunks of slices.

The reference reconstructs a volume slice by slice in a process pool
(algorithms/art.py:289-295, sir.py:260).  Here the slices of a volume held in
(page-locked) host memory go through the GPU in chunks: each chunk is one
multi-slice plan launch (``nz`` = chunk slices in one persistent kernel).  Three
CUDA streams form a pipeline -- host-to-device copies, compute, device-to-host
copies -- over ``slots`` sets of device buffers, ordered by events: the copy in
of chunk c+1 and the copy out of chunk c-1 overlap the launches of chunk c,
while the launches themselves run one after another on the compute stream (so
two chunks never compete for L2) and share one plan.

    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.streaming import VolumeStreamer
    tp = cpr.projectors(2048, angles_deg, oper="dd")
    vs = VolumeStreamer(tp, chunk=16, slots=3)
    ms = vs.project(images, sinograms)          # host [nz][n][n] -> host [nz][na][n]
    ms = vs.backproject(sinograms, images)
    ms = vs.reconstruct(sinograms, images, "sirt", iters=100)

Host arrays are CPU torch tensors (``pin_memory=True`` for copies that
overlap; pageable ones still work, with copies that do not overlap) or numpy
arrays (wrapped without a copy, pageable).  Results are bit-identical to
slice-by-slice plans: a chunk runs the same kernels on the same slices.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .class_projectors_radon import _KIND
from .solvers import Solver


def _host(a):
    if isinstance(a, np.ndarray):
        if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
            raise ValueError("host arrays must be C-contiguous float32")
        return torch.from_numpy(a)
    if not (isinstance(a, torch.Tensor) and a.device.type == "cpu" and a.dtype == torch.float32
            and a.is_contiguous()):
        raise ValueError("host arrays must be contiguous float32 CPU tensors or numpy arrays")
    return a


class VolumeStreamer:
    """Chunked, pipelined projection and reconstruction of a slice stack."""

    def __init__(self, tp, chunk: int = 16, slots: int = 3, device=None):
        if chunk < 1 or slots < 2:
            raise ValueError("chunk must be >= 1 and slots >= 2")
        self.tp, self.chunk, self.slots = tp, int(chunk), int(slots)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.n, self.na = int(tp.npix), int(tp.nang)
        self.s_in, self.s_run, self.s_out = (torch.cuda.Stream(self.device) for _ in range(3))
        self._plans = {}
        self._bufs = {}
        self._solvers = {}

    def _plan(self, m: int):
        if m not in self._plans:
            with torch.cuda.device(self.device):
                self._plans[m] = _lib.Plan(_KIND[self.tp.oper], self.n, self.tp._angles_c, nz=m)
        return self._plans[m]

    def _buf(self, slot: int, which: str):
        key = (slot, which)
        if key not in self._bufs:
            shape = (self.chunk, self.n, self.n) if which == "img" else (self.chunk, self.na, self.n)
            self._bufs[key] = torch.empty(shape, dtype=torch.float32, device=self.device)
        return self._bufs[key]

    def _pipeline(self, src, dst, src_kind: str, dst_kind: str, compute):
        """For each chunk: copy src in (s_in), compute(slot, m, din, dout) (s_run),
        copy dout out (s_out).  A slot's buffers are refilled only after the
        chunk that used them last has been computed and copied out."""
        src, dst = _host(src), _host(dst)
        nz = int(src.shape[0])
        if int(dst.shape[0]) != nz:
            raise ValueError("source and destination hold different numbers of slices")
        cur = torch.cuda.current_stream(self.device)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(cur)
        for st in (self.s_in, self.s_run, self.s_out):
            st.wait_event(t0)
        ev_in = [torch.cuda.Event() for _ in range(self.slots)]
        ev_run = [torch.cuda.Event() for _ in range(self.slots)]
        ev_out = [torch.cuda.Event() for _ in range(self.slots)]
        used = [False] * self.slots
        for c, z0 in enumerate(range(0, nz, self.chunk)):
            m = min(self.chunk, nz - z0)
            k = c % self.slots
            din, dout = self._buf(k, src_kind)[:m], self._buf(k, dst_kind)[:m]
            with torch.cuda.stream(self.s_in):
                if used[k]:
                    self.s_in.wait_event(ev_run[k])   # din last read by the slot's previous compute
                din.copy_(src[z0:z0 + m], non_blocking=True)
                ev_in[k].record(self.s_in)
            with torch.cuda.stream(self.s_run):
                self.s_run.wait_event(ev_in[k])
                if used[k]:
                    self.s_run.wait_event(ev_out[k])  # dout last read by the slot's previous copy out
                compute(k, m, din, dout)
                ev_run[k].record(self.s_run)
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(ev_run[k])
                dst[z0:z0 + m].copy_(dout, non_blocking=True)
                ev_out[k].record(self.s_out)
            used[k] = True
        for st in (self.s_in, self.s_run, self.s_out):
            cur.wait_stream(st)
        t1.record(cur)
        t1.synchronize()
        return t0.elapsed_time(t1)

    def project(self, images, sinograms) -> float:
        """sinograms[z] = A images[z] for every slice; returns the device milliseconds."""
        return self._pipeline(images, sinograms, "img", "sino",
                              lambda k, m, din, dout: self._plan(m).forward(din, out=dout))

    def backproject(self, sinograms, images) -> float:
        """images[z] = A^T sinograms[z] for every slice; returns the device milliseconds."""
        return self._pipeline(sinograms, images, "sino", "img",
                              lambda k, m, din, dout: self._plan(m).adjoint(din, out=dout))

    def reconstruct(self, sinograms, images, algo: str = "sirt", iters: int = 100, x0: float = 1.0) -> float:
        """images[z] = ``iters`` iterations of the fused solver ``algo`` (sirt or em)
        on sinograms[z], from the constant start x0 (the reference starts SIRT at
        1, art.py:408); returns the device milliseconds.  Each slot's solver is
        bound to the slot's sinogram and iterate buffers and keeps its CUDA graph
        from chunk to chunk; SIRT's and MLEM's weights depend on the geometry only
        (SPS's depend on each sinogram, so SPS is not streamed here)."""
        if algo not in ("sirt", "em", "mlem"):
            raise ValueError("reconstruct streams sirt and em (SPS weights depend on each chunk's sinogram)")

        def compute(k, m, b, x):
            x.fill_(float(x0))
            key = (k, m, algo)
            if key not in self._solvers:  # created once per slot (it synchronises)
                self._solvers[key] = Solver(self._plan(m), algo, b.reshape(-1), device=self.device)
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(_lib.lib.tomo_solver_run(self._solvers[key]._h, ctypes.c_void_p(x.data_ptr()), int(iters),
                                                None, 1, ctypes.c_void_p(stream)), "tomo_solver_run")
        return self._pipeline(sinograms, images, "sino", "img", compute)

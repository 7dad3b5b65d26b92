"""Volumes larger than one launch, streamed through the GPU in chunks of slices.

The reference reconstructs a volume slice by slice in a process pool
(algorithms/art.py:289-295, sir.py:260).  Here the slices of a volume held in
(page-locked) host memory go through the GPU in chunks: each chunk is one
multi-slice plan launch (``nz`` = chunk slices in one persistent kernel), and
``streams`` CUDA streams take the chunks in turn, so that the host-to-device
copy of one chunk, the projector (or solver) launches of another and the
device-to-host copy of a third overlap.  Every stream owns its plan (its own
scratch) and its device buffers; a stream's next chunk reuses them only after
its previous chunk, in stream order, so no chunk waits on another stream.

    from iterative_tomographic_reconstruction_algorithms_b200 import class_projectors_radon as cpr
    from iterative_tomographic_reconstruction_algorithms_b200.streaming import VolumeStreamer
    tp = cpr.projectors(2048, angles_deg, oper="dd")
    vs = VolumeStreamer(tp, chunk=16, streams=3)
    ms = vs.project(images, sinograms)          # host [nz][n][n] -> host [nz][na][n]
    ms = vs.backproject(sinograms, images)
    ms = vs.reconstruct(sinograms, images, "sirt", iters=100)

Host arrays are CPU torch tensors (``pin_memory=True`` for copies that
overlap; pageable ones still work, with copies that do not overlap) or numpy
arrays (wrapped without a copy, pageable).  Results are bit-identical to
slice-by-slice plans: a chunk runs the same kernels on the same slices.
"""
from __future__ import annotations

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
    """Chunked, multi-stream projection and reconstruction of a slice stack."""

    def __init__(self, tp, chunk: int = 16, streams: int = 3, device=None):
        if chunk < 1 or streams < 1:
            raise ValueError("chunk and streams must be >= 1")
        self.tp, self.chunk, self.nstreams = tp, int(chunk), int(streams)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.n, self.na = int(tp.npix), int(tp.nang)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(self.nstreams)]
        self._plans = {}
        self._bufs = {}
        self._solvers = {}

    # one plan and one pair of buffers per (stream, slices in the chunk)
    def _plan(self, s: int, m: int):
        key = (s, m)
        if key not in self._plans:
            with torch.cuda.device(self.device):
                self._plans[key] = _lib.Plan(_KIND[self.tp.oper], self.n, self.tp._angles_c, nz=m)
        return self._plans[key]

    def _buf(self, s: int, which: str):
        key = (s, which)
        if key not in self._bufs:
            shape = (self.chunk, self.n, self.n) if which == "img" else (self.chunk, self.na, self.n)
            self._bufs[key] = torch.empty(shape, dtype=torch.float32, device=self.device)
        return self._bufs[key]

    def _run(self, src, dst, body):
        src, dst = _host(src), _host(dst)
        nz = int(src.shape[0])
        if int(dst.shape[0]) != nz:
            raise ValueError("source and destination hold different numbers of slices")
        cur = torch.cuda.current_stream(self.device)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(cur)
        for st in self.streams:
            st.wait_event(t0)
        for c, z0 in enumerate(range(0, nz, self.chunk)):
            m = min(self.chunk, nz - z0)
            s = c % self.nstreams
            with torch.cuda.stream(self.streams[s]):
                body(s, m, src[z0:z0 + m], dst[z0:z0 + m])
        for st in self.streams:
            cur.wait_stream(st)
        t1.record(cur)
        t1.synchronize()
        return t0.elapsed_time(t1)

    def project(self, images, sinograms) -> float:
        """sinograms[z] = A images[z] for every slice; returns the device milliseconds."""
        def body(s, m, src, dst):
            din, dout = self._buf(s, "img")[:m], self._buf(s, "sino")[:m]
            din.copy_(src, non_blocking=True)
            self._plan(s, m).forward(din, out=dout)
            dst.copy_(dout, non_blocking=True)
        return self._run(images, sinograms, body)

    def backproject(self, sinograms, images) -> float:
        """images[z] = A^T sinograms[z] for every slice; returns the device milliseconds."""
        def body(s, m, src, dst):
            din, dout = self._buf(s, "sino")[:m], self._buf(s, "img")[:m]
            din.copy_(src, non_blocking=True)
            self._plan(s, m).adjoint(din, out=dout)
            dst.copy_(dout, non_blocking=True)
        return self._run(sinograms, images, body)

    def reconstruct(self, sinograms, images, algo: str = "sirt", iters: int = 100, x0: float = 1.0) -> float:
        """images[z] = ``iters`` iterations of the fused solver ``algo`` (sirt or em)
        on sinograms[z], from the constant start x0 (the reference starts SIRT at
        1, art.py:408); returns the device milliseconds.  Each stream's solver is
        bound to its sinogram buffer and iterate buffer and keeps its CUDA graph
        from chunk to chunk; SIRT's and MLEM's weights depend on the geometry
        only (SPS's depend on each sinogram, so SPS is not streamed here)."""
        if algo not in ("sirt", "em", "mlem"):
            raise ValueError("reconstruct streams sirt and em (SPS weights depend on each chunk's sinogram)")
        import ctypes

        def body(s, m, src, dst):
            b, x = self._buf(s, "sino")[:m], self._buf(s, "img")[:m]
            b.copy_(src, non_blocking=True)
            x.fill_(float(x0))
            key = (s, m, algo)
            if key not in self._solvers:  # created once per stream (it synchronises)
                self._solvers[key] = Solver(self._plan(s, m), algo, b.reshape(-1), device=self.device)
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(_lib.lib.tomo_solver_run(self._solvers[key]._h, ctypes.c_void_p(x.data_ptr()), int(iters),
                                                None, 1, ctypes.c_void_p(stream)), "tomo_solver_run")
            dst.copy_(x, non_blocking=True)
        return self._run(sinograms, images, body)

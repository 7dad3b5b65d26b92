"""Projection filtering for filtered backprojection (host-side, numpy).

Restates ``common/operators/filters_module/filters.py`` of the reference:
``calc_filter`` (:35-76) builds a ramp (absorption) or Hilbert (differential
phase contrast, ``dpc=True``) kernel of length 2*nfreq with optional
Shepp-Logan / cosine / Hamming / Hanning apodisation, and ``filter_proj``
(:89-113) zero-pads each projection to 2*nfreq (nfreq = 2 * 2^ceil(log2 npix)),
filters it in Fourier space and keeps the first npix samples.  All rows are
transformed in one vectorised FFT instead of one at a time.
"""
from __future__ import annotations

import numpy as np

myfloat = np.float32
mycomplex = np.complex64


def calc_filter(nfreq: int, ftype: str = "ramp", dpc: bool = False) -> np.ndarray:
    if ftype == "none":
        return np.ones(2 * nfreq)
    if not dpc:
        filtarr = 2 * np.arange(nfreq + 1) / myfloat(2 * nfreq)
        w = 2 * np.pi * np.arange(nfreq + 1) / myfloat(2 * nfreq)
        d = 1.0
    else:
        filtarr = np.ones(nfreq + 1, dtype=mycomplex) * (1.0j) / (2 * np.pi)
        w, d = None, 1.0
    if ftype in ("shepp-logan", "cosine", "hamming", "hanning") and w is None:
        # the reference reads the undefined ramp frequencies here and raises
        raise NameError("calc_filter: apodised Hilbert filters are undefined in the reference")
    if ftype == "shepp-logan":
        filtarr[1:] *= np.sin(w[1:]) / (2.0 * d * 2.0 * d * w[1:])
    elif ftype == "cosine":
        filtarr[1:] *= np.cos(w[1:]) / (2.0 * d * w[1:])
    elif ftype == "hamming":
        filtarr[1:] *= (0.54 + 0.46 * np.cos(w[1:]) / d)
    elif ftype == "hanning":
        filtarr[1:] *= (1.0 + np.cos(w[1:] / d) / 2.0)
    if not dpc:
        return np.concatenate((filtarr, filtarr[nfreq - 1:0:-1]), axis=0)
    return np.concatenate((filtarr, np.conjugate(filtarr[nfreq - 1:0:-1])), axis=0)


def filter_proj(sino: np.ndarray, ftype: str = "ramp", dpc: bool = False) -> np.ndarray:
    nang, npix = sino.shape
    nfreq = 2 * int(2 ** (int(np.ceil(np.log2(npix)))))
    filtarr = calc_filter(nfreq, ftype=ftype, dpc=dpc)
    padded = np.concatenate((sino, np.zeros((nang, 2 * nfreq - npix))), axis=1)
    out = np.real(np.fft.ifft(np.fft.fft(padded, axis=1) * filtarr[None, :], axis=1))
    sino[:, :] = out[:, :npix]
    return sino


def filter_proj_device(sino, ftype: str = "ramp", dpc: bool = False):
    """``filter_proj`` for a CUDA tensor [..., nang, npix]: the same float64
    transform of the zero-padded rows (torch.fft on the device), result float32.
    Returns a new tensor; the input is not modified."""
    import torch
    npix = int(sino.shape[-1])
    nfreq = 2 * int(2 ** (int(np.ceil(np.log2(npix)))))
    filtarr = torch.from_numpy(np.asarray(calc_filter(nfreq, ftype=ftype, dpc=dpc)).astype(np.complex128))
    spec = torch.fft.fft(sino.to(torch.float64), n=2 * nfreq, dim=-1)
    out = torch.fft.ifft(spec * filtarr.to(sino.device), dim=-1).real[..., :npix]
    return out.to(torch.float32).contiguous()


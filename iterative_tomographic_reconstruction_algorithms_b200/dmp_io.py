"""DMP image files (reference: common/myimage/my_image_io.py:222-247).

Format: a header of three 16-bit integers (width, height, 0) followed by the
image as little-endian float32, row-major ``[height][width]``.  ``read_dmp``
can read straight into page-locked host memory so that the copy to the GPU is
a single asynchronous DMA (``to_device=True``), which is how a streamed stack
of slices is fed to a batched plan.

Difference: the header is read as unsigned 16-bit (the reference reads signed
``'h'``, which turns sizes above 32767 negative); files of either are the same
for sizes up to 32767.
"""
from __future__ import annotations

import os

import numpy as np


def read_dmp(path, pinned: bool = False, to_device: bool = False):
    """The image of a DMP file: numpy float32 [height, width], or a torch
    tensor in page-locked memory (``pinned``), or on the current CUDA device
    (``to_device``, copied from a page-locked buffer)."""
    with open(path, "rb") as fd:
        hdr = np.fromfile(fd, np.uint16, 3)
        if hdr.size != 3:
            raise ValueError(f"{path}: truncated DMP header")
        width, height = int(hdr[0]), int(hdr[1])
        count = width * height
        if not (pinned or to_device):
            data = np.fromfile(fd, np.float32, count)
            if data.size != count:
                raise ValueError(f"{path}: expected {count} values, found {data.size}")
            return data.reshape(height, width)
        import torch
        host = torch.empty((height, width), dtype=torch.float32, pin_memory=True)
        view = host.numpy().reshape(-1).view(np.uint8)
        got = fd.readinto(memoryview(view))
        if got != count * 4:
            raise ValueError(f"{path}: expected {count * 4} bytes, read {got}")
    if to_device:
        return host.to("cuda", non_blocking=True)
    return host


def write_dmp(path, image) -> None:
    """Writes a 2-D array as a DMP file (float32 data, header width, height, 0)."""
    if hasattr(image, "detach"):
        image = image.detach().cpu().numpy()
    a = np.ascontiguousarray(image, dtype=np.float32)
    if a.ndim != 2 or a.shape[0] > 65535 or a.shape[1] > 65535:
        raise ValueError("DMP holds 2-D images up to 65535 x 65535")
    with open(path, "wb") as fd:
        np.array([a.shape[1], a.shape[0], 0], np.uint16).tofile(fd)
        a.astype("<f4", copy=False).tofile(fd)

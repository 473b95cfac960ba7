"""Batch reader: MRC subtomograms (and CTF weight files) decoded by native threads straight
into pinned host batches, the next batch read while the current one aligns.

Mirrors the reader side of the reference's run loop: ``_read_worker`` and ``cpu_reader``
(src/matcha/utils/run_utils.py:23-41, 430-611) read each subtomogram with
``load_subtomogram_cpu`` and, with CTF correction on, its weights file (the path with
``_data.`` replaced by ``_weights.``) with ``load_ctf_relion5_cpu``
(src/matcha/utils/io_utils.py:229-253); a file that fails is skipped with a warning and
batches are filled to ``batch_size`` with the files that load, the last one partial.  Here the
decode is ``mtb_read_mrc`` (C++ threads, ``pread`` into the batch buffer, no per-file tensors,
no ``torch.stack``, no separate pinning copy), and two pinned batch slots alternate.
"""
from __future__ import annotations

import ctypes
import threading
import warnings
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _native as nat

READ_STATUS = {0: "ok", 1: "cannot open", 2: "not an MRC file or unsupported mode", 3: "unexpected shape",
               4: "file shorter than its data"}


class MrcReader:
    """``mtb_read_mrc`` on a pool of ``n_threads`` threads (0: one per hardware thread)."""

    def __init__(self, n_threads: int = 0):
        self._lib = nat.load()
        h = ctypes.c_void_p()
        nat.check(self._lib.mtb_reader_create(int(n_threads), ctypes.byref(h)), "mtb_reader_create")
        self._h = h

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._lib.mtb_reader_destroy(h)

    def read_into(self, paths, out: torch.Tensor, shape, crop=None) -> np.ndarray:
        """Decode ``paths`` of voxel shape ``shape`` (nz, ny, nx) into ``out`` (len(paths),
        *crop) float32 CPU tensor (crop: the leading box kept, default the whole volume).
        Returns the per-file status (``READ_STATUS``)."""
        n = len(paths)
        crop = tuple(shape) if crop is None else tuple(crop)
        if out.dtype != torch.float32 or out.device.type != "cpu" or not out.is_contiguous():
            raise ValueError("out must be a contiguous float32 CPU tensor")
        if tuple(out.shape) != (n,) + crop:
            raise ValueError(f"out has shape {tuple(out.shape)}, expected {(n,) + crop}")
        status = np.zeros(n, dtype=np.int32)
        if n == 0:
            return status
        enc = [str(p).encode() for p in paths]
        arr = (ctypes.c_char_p * n)(*enc)
        nat.check(self._lib.mtb_read_mrc(self._h, ctypes.cast(arr, ctypes.c_void_p), n, *map(int, shape),
                                         *map(int, crop), out.data_ptr(),
                                         status.ctypes.data_as(ctypes.c_void_p)), "mtb_read_mrc")
        return status

    def read(self, paths, shape, crop=None, pin: bool = False):
        crop = tuple(shape) if crop is None else tuple(crop)
        out = torch.empty((len(paths),) + crop, dtype=torch.float32, pin_memory=pin)
        return out, self.read_into(paths, out, shape, crop)


def write_mrc(path, data: np.ndarray):
    """A minimal MRC2014 float32 file (little-endian, no extended header) of a (nz, ny, nx)
    array, for making test and timing inputs."""
    data = np.ascontiguousarray(data, dtype="<f4")
    nz, ny, nx = data.shape
    words = np.zeros(256, dtype="<i4")
    words[0:4] = [nx, ny, nz, 2]
    words[7:10] = [nx, ny, nz]
    words[16:19] = [1, 2, 3]
    hdr = bytearray(words.tobytes())
    hdr[208:212] = b"MAP "
    hdr[212:216] = bytes([0x44, 0x44, 0, 0])
    with open(path, "wb") as f:
        f.write(bytes(hdr))
        f.write(data.tobytes())


def ctf_crop(N: int):
    """The leading box load_ctf_relion5_cpu keeps of an (N, N, N) weights file."""
    return (N // 2, N, N // 2 + 1)


class BatchReader:
    """Batches of (subtomograms, CTF weights or None, paths) in pinned host memory.

    ``batches(paths)`` yields ``(vols, ctfs, paths, release)``: ``vols`` (b, N, N, N) and
    ``ctfs`` (b, N/2, N, N/2+1) are views of one of two pinned slots, ``paths`` the b files
    that loaded.  While the caller aligns a batch the reader fills the other slot.  A caller
    whose host-to-device copies of a batch may still run when it asks for the next batch
    calls ``release(event)`` first with the CUDA event after which they are done (e.g. the
    ``copies_done`` event ``AlignmentStep.align_host`` returns); the slot is refilled only
    after that event.  Otherwise asking for the next batch releases the slot."""

    def __init__(self, N: int, batch_size: int, do_ctf_correction: bool = True, n_threads: int = 0,
                 base_str: str = "_data.", replace_str: str = "_weights.", pin: bool = True):
        self.N, self.batch_size, self.do_ctf = int(N), int(batch_size), bool(do_ctf_correction)
        self.base_str, self.replace_str = base_str, replace_str
        self.reader = MrcReader(n_threads)
        shape_v = (self.batch_size, N, N, N)
        self._vols = [torch.empty(shape_v, dtype=torch.float32, pin_memory=pin) for _ in range(2)]
        self._ctfs = ([torch.empty((self.batch_size,) + ctf_crop(N), dtype=torch.float32, pin_memory=pin)
                       for _ in range(2)] if self.do_ctf else [None, None])
        self.skipped = []  # (path, reason) of every file that failed

    def _fill(self, slot: int, paths, cursor: int):
        """Fill ``slot`` from ``paths[cursor:]`` up to batch_size loaded files."""
        N, vols, ctfs = self.N, self._vols[slot], self._ctfs[slot]
        good = []
        while len(good) < self.batch_size and cursor < len(paths):
            take = paths[cursor:cursor + self.batch_size - len(good)]
            cursor += len(take)
            lo = len(good)
            st = self.reader.read_into(take, vols[lo:lo + len(take)], (N, N, N))
            if self.do_ctf:
                cst = self.reader.read_into([p.replace(self.base_str, self.replace_str) for p in take],
                                            ctfs[lo:lo + len(take)], (N, N, N), ctf_crop(N))
            else:
                cst = np.zeros_like(st)
            for i, p in enumerate(take):
                if st[i] == 0 and cst[i] == 0:
                    k = len(good)
                    if k != lo + i:  # close the gap a skipped file left
                        vols[k].copy_(vols[lo + i])
                        if self.do_ctf:
                            ctfs[k].copy_(ctfs[lo + i])
                    good.append(p)
                else:
                    why = READ_STATUS.get(int(st[i] if st[i] else cst[i]), "error")
                    self.skipped.append((p, why))
                    warnings.warn(f"Skipping {p}: {why}")
        return good, cursor

    def batches(self, paths):
        paths = [str(p) for p in paths]
        released = [threading.Event(), threading.Event()]
        events = [None, None]
        for r in released:
            r.set()

        def fill(slot, cursor):
            released[slot].wait()
            if events[slot] is not None:
                events[slot].synchronize()
                events[slot] = None
            return self._fill(slot, paths, cursor)

        with ThreadPoolExecutor(max_workers=1) as ex:
            slot, fut = 0, ex.submit(fill, 0, 0)
            while True:
                good, cursor = fut.result()
                if not good:
                    return
                released[slot].clear()
                nxt = 1 - slot
                fut = ex.submit(fill, nxt, cursor) if cursor < len(paths) else None

                def release(event=None, _slot=slot):
                    events[_slot] = event
                    released[_slot].set()

                b = len(good)
                yield (self._vols[slot][:b], self._ctfs[slot][:b] if self.do_ctf else None, good, release)
                # asking for the next batch without release(event) means the caller is done with
                # this slot; refill it (two batches on) without waiting
                released[slot].set()
                if fut is None:
                    return
                slot = nxt

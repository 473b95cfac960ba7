"""Per-batch result bookkeeping of the alternation loop without per-value host syncs.

Drop-in for ``store_alignment_parameters`` (src/matcha/utils/io_utils.py:181-225): the same
arguments, the same rows appended to ``result_data`` and the same pickle, but the values every
row reads from device tensors (scores, the tracker's Euler angles, local and prior shifts) are
packed on the device by ``mtb_pack_results`` and copied to the host once per batch, where the
reference calls ``.item()`` / ``.cpu()`` per particle.  ``particle_token`` is the reference's
``_particle_token`` (io_utils.py:14-25).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

from . import _native as nat

COLUMNS = ("rotation_score", "alpha", "beta", "gamma", "tx", "ty", "tz", "px", "py", "pz", "shift_score")


def particle_token(path_like: str) -> str:
    """The particle name a result row carries (io_utils.py:14-25)."""
    path_norm = str(path_like).strip()
    if "@" in path_norm:
        path_norm = path_norm.split("@", 1)[1]
    path_norm = path_norm.replace("\\", "/")
    parts = Path(path_norm).parts
    token = "/".join(parts[-2:]) if len(parts) >= 2 else parts[-1]
    for suffix in ("_weights.mrc", "_ctf.mrc", "_data.mrc", ".mrc"):
        token = token.replace(suffix, "")
    return token.replace("_subtomo", "_").replace("//", "/")


@torch.no_grad()
def pack_results(rotation_scores: torch.Tensor, shift_scores: torch.Tensor, local_shifts: torch.Tensor,
                 rotation_tracker: torch.Tensor, prior_shifts: torch.Tensor, B: int) -> torch.Tensor:
    """(B, 11) float64 on the device, columns ``COLUMNS``; the first of each particle's
    entries when a tensor holds several per particle (the reference's argmax over a
    dimension of size one always picks it)."""
    dev = rotation_tracker.device
    nat.require_cuda(rotation_tracker, "rotation_tracker")

    def first(t, width, dtype):
        t = torch.as_tensor(t, device=dev).to(dtype)
        return t.reshape(B, -1, width)[:, 0].contiguous() if width > 1 else t.reshape(B, -1)[:, 0].contiguous()

    rs = first(rotation_scores, 1, torch.float32)
    ss = first(shift_scores, 1, torch.float32)
    ls = first(local_shifts, 3, torch.float32)
    ps = first(prior_shifts, 3, torch.float32)
    tr = first(rotation_tracker, 4, torch.float64)
    out = torch.empty((B, len(COLUMNS)), device=dev, dtype=torch.float64)
    with torch.cuda.device(dev):
        nat.check(nat.load().mtb_pack_results(nat.ptr(rs), nat.ptr(ss), nat.ptr(ls), nat.ptr(ps), nat.ptr(tr), B,
                                              nat.ptr(out), nat.stream_ptr(dev)), "mtb_pack_results")
    return out


def append_rows(result_data, packed: np.ndarray, tomogram_file_names, half: str, alternation_index=None):
    """Rows of ``store_alignment_parameters`` from a host copy of ``pack_results``: one per
    file name, in order (a padded batch has more packed rows than names)."""
    for i, name in enumerate(tomogram_file_names):
        r = packed[i]
        result_data.loc[len(result_data)] = {
            "path": name,
            "rotation_score": float(r[0]),
            "rotation": np.array(r[1:4], dtype=np.float64),
            "translation": r[4:7].astype(np.float32),
            "file_name": name.split("/")[-1],
            "prior_shift": r[7:10].astype(np.float32),
            "alternation_index": alternation_index if alternation_index is not None else 0,
            "shift_score": float(r[10]),
            "rlnTomoParticleName": particle_token(name),
            "half": half,
        }
    return result_data


def store_alignment_parameters(config, result_data, tomogram_file_names: list, rotation_scores: torch.Tensor,
                               shift_scores: torch.Tensor, local_shifts: torch.Tensor,
                               rotation_tracker: torch.Tensor, prior_shifts: torch.Tensor, half: str,
                               alternation_index: int = None):
    """io_utils.py:181-225 with one device-to-host copy per batch; ``rotation_tracker`` is the
    (B, 4) float64 device tracker (w, x, y, z)."""
    B = int(config["num_subtomograms_per_batch"])
    packed = pack_results(rotation_scores, shift_scores, local_shifts, rotation_tracker, prior_shifts, B).cpu().numpy()
    append_rows(result_data, packed, tomogram_file_names, half, alternation_index)
    result_data.to_pickle(f"{config['execution']['output_file_name']}.pkl")
    return result_data

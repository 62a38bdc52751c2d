"""Frame output in the reference's on-disk format (pfflip/io.py:10-29).

``save_frame`` writes one compressed ``.npz`` per frame with the keys and
dtypes downstream renderers read: ``t`` (float32), ``step`` (int32), ``dx``
(float32), ``phi`` (the cell phase field as float16) and, with
``particles=True``, every ``stride``-th particle's position (float16, the
caller's original order) and type (int8).  The float16 conversions run on
the device; only the converted arrays cross to the host.
"""

from __future__ import annotations

import os

import numpy as np
import torch

from ._arrays import as_tensor


def save_frame(sim, path: str, *, particles: bool = True, stride: int = 1):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    data = {
        "t": np.float32(sim.time),
        "step": np.int32(sim.step_index),
        "dx": np.float32(sim.cfg.dx),
        "phi": as_tensor(sim.phi_cell).to(torch.float16).cpu().numpy(),
    }
    if particles:
        n = sim.n_particles
        ids = sim._ids().long()
        pos = torch.empty((n, 3), dtype=torch.float16, device=sim.dev)
        pos[ids] = sim._pos4[:, :3].to(torch.float16)
        pt = torch.empty(n, dtype=torch.int8, device=sim.dev)
        pt[ids] = (sim._flags() & 1).to(torch.int8)
        data["px"] = pos[::stride].cpu().numpy()
        data["ptype"] = pt[::stride].cpu().numpy()
    np.savez_compressed(path, **data)


def load_frame(path: str) -> dict:
    """The arrays of a frame written by ``save_frame`` (or the reference's)."""
    with np.load(path) as f:
        return {k: f[k] for k in f.files}

"""Focus of a beam of traced electrons (traceon/focus.py:9-42) on the GPU.

`focus_position` takes the reference's argument, a list of (N, 6)
trajectories, and returns the same (x, y, z): the point nearest, in the
least-squares sense, to every trajectory's final straight-line extension.
The sums run on the device (`tb_focus_position`); device-resident traces use
`TraceResult.focus_position` directly.
"""
from __future__ import annotations

import numpy as np

from . import backend as B


def focus_position(positions):
    """traceon/focus.py:9-42: positions is an iterable of (N, 6) arrays of
    x, y, z, vx, vy, vz; the last row of each is used."""
    torch = B._torch()
    assert all(p.shape == (len(p), 6) for p in positions)
    last = np.array([np.asarray(p, dtype=np.float64)[-1] for p in positions]).reshape(-1, 6)
    out = B.dev_focus_position(B.to_dev(last, torch.float64))
    return out.cpu().numpy()

"""Device-resident batches of scenarios for the batched engine, CUDA graphs
and the server: PropagJob structures over torch device buffers.

* ``device_jobs``    -- jobs from (width, height, dx, dy, max_time, tile,
                        ignitions, terrain tensors) tuples, with their fire,
                        time, reference and boundary buffers
* ``ensemble_batch`` -- the ensemble of config 2: members sharing a
                        1024 x 1024 terrain, each with its own wind,
                        moisture and ignition (scenarios.config2)
* ``uneven_batch``   -- independent scenarios of uneven sizes (config 3)

No counterpart in the reference, which runs one scenario per call
(crates/propag/src/propag.rs:323-574).
"""
from __future__ import annotations

import numpy as np


def device_jobs(L, dev, items):
    """items: (width, height, dx, dy, max_time, tile, ignitions, terrain tensors).
    Returns the jobs, their terrain pointer structs and the buffers that keep
    them alive (terrain, fire rasters, ignitions, time, refs_x, refs_y, bits)."""
    import torch
    jobs, terrains, keep = [], [], []
    for (w, h, dx, dy, max_time, tile, ignitions, t) in items:
        n = w * h
        fire = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3)]
        ign = np.array(list(ignitions), dtype=[("x", "<u4"), ("y", "<u4"), ("t", "<f4")])
        ign_d = torch.from_numpy(np.frombuffer(ign.tobytes() or bytes(12), np.uint8).copy()).to(dev)
        out = torch.empty(n, dtype=torch.float32, device=dev)
        rx = torch.empty(n, dtype=torch.int16, device=dev)
        ry = torch.empty(n, dtype=torch.int16, device=dev)
        bnd = torch.empty((n + 31) // 32, dtype=torch.int32, device=dev)
        j = L.PropagJob()
        j.width, j.height, j.dx, j.dy, j.max_time, j.tile = w, h, dx, dy, max_time, tile
        j.speed_max, j.azimuth_max, j.eccentricity = (f.data_ptr() for f in fire)
        j.ignitions, j.n_ignitions = ign_d.data_ptr(), len(ign)
        j.time, j.refs_x, j.refs_y, j.boundaries = out.data_ptr(), rx.data_ptr(), ry.data_ptr(), bnd.data_ptr()
        jobs.append(j)
        terrains.append(L.PropagTerrainPtrs(*[t[k].data_ptr() for k in L.TERRAIN_FIELDS]))
        keep.append((t, fire, ign_d, out, rx, ry, bnd))
    return jobs, terrains, keep


def ensemble_batch(L, dev, n_members):
    """The ensemble on a shared 1024 x 1024 terrain: per-member wind speed and
    direction, dead moisture offset and ignition, max_time 21600 s."""
    import torch
    from py_propag import scenarios as S
    base, members = S.config2(n=n_members)
    N = base.width * base.height
    bt = {k: torch.from_numpy(np.ascontiguousarray(v).ravel()).to(dev) for k, v in base.terrain.items()}
    items = []
    for m in members:
        t = dict(bt)
        t["wind_speed"] = torch.full((N,), m["wind_speed"], dtype=torch.float32, device=dev)
        t["wind_azimuth"] = torch.full((N,), m["wind_azimuth"], dtype=torch.float32, device=dev)
        for k in ("d1hr", "d10hr", "d100hr"):
            t[k] = bt[k] + np.float32(m["dead_offset"])
        items.append((base.width, base.height, base.dx, base.dy, m["max_time"], 0, [m["ignition"]], t))
    desc = (f"config2: {n_members}-member ensemble on a shared {base.width}x{base.height} terrain, "
            f"per-member wind/moisture/ignition, max_time 21600 s")
    return device_jobs(L, dev, items), desc


def uneven_batch(L, dev, n):
    """Independent scenarios of uneven sizes: square grids log-uniform in
    128..2048 at 5-30 m, own terrain and fuel, 1-10 ignitions, 1-12 h."""
    import torch
    from py_propag import scenarios as S
    scs = S.config3(n=n)
    items = []
    for sc in scs:
        t = {k: torch.from_numpy(np.ascontiguousarray(v).ravel()).to(dev) for k, v in sc.terrain.items()}
        items.append((sc.width, sc.height, sc.dx, sc.dy, sc.max_time, 0, sc.ignitions, t))
    cells = sum(sc.width * sc.height for sc in scs)
    desc = (f"config3: {n} scenarios, square grids {min(s.width for s in scs)}.."
            f"{max(s.width for s in scs)} at 5-30 m ({cells / 1e6:.1f} M cells), own terrain, "
            f"1-10 ignitions, max_time 1-12 h")
    return device_jobs(L, dev, items), desc

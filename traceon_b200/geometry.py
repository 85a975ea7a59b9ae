"""Synthetic radially symmetric electrode geometries as line4 (cubic) meshes.

The reference builds meshes with ``traceon.geometry.Path(...).mesh()``, whose
``discretize_path`` spaces nodes uniformly (traceon/geometry.py:39-70).  The
lens workloads here are graded toward the corners of every straight segment,
which the reference mesher cannot do, so the mesh rows are written directly
in the reference's line4 layout: each element row is
``[start, end, 1/3-point, 2/3-point]`` (traceon/mesher.py:188-227 and the
vertex ordering of traceon/geometry.py:851-857).  All lengths are metres.
"""
from __future__ import annotations

import numpy as np

MM = 1e-3


def graded_nodes(n: int) -> np.ndarray:
    """n+1 Chebyshev-Lobatto nodes on [0, 1]: dense toward both ends."""
    k = np.arange(n + 1)
    s = 0.5 * (1.0 - np.cos(np.pi * k / n))
    s[0], s[-1] = 0.0, 1.0
    return s


def polyline_elements(points_rz, counts) -> np.ndarray:
    """Cubic line elements along a polyline of (r, z) corners.  ``counts[i]``
    elements on segment i, graded toward both ends.  Returns (N, 4, 3) rows
    (r, 0, z) in line4 order [start, end, 1/3, 2/3]."""
    pts = np.asarray(points_rz, dtype=np.float64)
    rows = []
    for (p0, p1), n in zip(zip(pts[:-1], pts[1:]), counts):
        s = graded_nodes(int(n))
        for a, b in zip(s[:-1], s[1:]):
            q = [p0 + (p1 - p0) * t for t in (a, b, a + (b - a) / 3, a + 2 * (b - a) / 3)]
            rows.append([[x[0], 0.0, x[1]] for x in q])
    return snap(np.array(rows, dtype=np.float64))


def snap(a: np.ndarray) -> np.ndarray:
    """Zero the low 16 mantissa bits of every coordinate.  The reference
    Mesh merges points after the same truncation (traceon/mesher.py:262-290),
    so snapped vertices pass through a reference Mesh unchanged."""
    a = np.array(a, dtype=np.float64)
    a.view(np.uint64)[...] &= np.uint64(0xFFFFFFFFFFFF0000)
    return a


def split_counts(total: int, lengths) -> list[int]:
    """Split ``total`` elements over segments proportionally to length; each
    segment gets at least 2 (at least 1 when total < 2 per segment).
    Raises ValueError when there are fewer elements than segments."""
    lengths = np.asarray(lengths, dtype=np.float64)
    if len(lengths) == 0 or total < len(lengths):
        raise ValueError(f'{total} elements cannot cover {len(lengths)} segments with at least one each')
    raw = total * lengths / lengths.sum()
    floor = 2 if total >= 2 * len(lengths) else 1
    c = np.maximum(floor, np.floor(raw).astype(int))
    while c.sum() < total:
        c[np.argmax(raw - c)] += 1
    while c.sum() > total:
        over = np.where(c > floor, c - raw, -np.inf)  # trim only above the minimum
        c[np.argmax(over)] -= 1
    return [int(x) for x in c]


def tube_counts(r_in: float, r_out: float, z0: float, z1: float, n: int) -> list[int]:
    """Elements on the three segments of aperture_tube (cap, tube, cap)."""
    return split_counts(n, [r_out - r_in, z1 - z0, r_out - r_in])


def aperture_tube(r_in: float, r_out: float, z0: float, z1: float, n: int) -> np.ndarray:
    """One einzel-lens electrode: a tube of radius r_in over [z0, z1] with
    annular end caps out to r_out, i.e. the polyline
    (r_out, z0) -> (r_in, z0) -> (r_in, z1) -> (r_out, z1)."""
    corners = [(r_out, z0), (r_in, z0), (r_in, z1), (r_out, z1)]
    return polyline_elements(corners, tube_counts(r_in, r_out, z0, z1, n))


def mesh_segments_device(segments, counts):
    """Graded cubic elements of straight segments (S, 4) = (r0, z0, r1, z1)
    with counts[s] elements each, meshed on the GPU (tb_mesh_segments); the
    rule of polyline_elements.  Returns a (N, 4, 3) device tensor."""
    from . import backend as B
    torch = B._torch()
    seg = np.ascontiguousarray(segments, dtype=np.float64).reshape(-1, 4)
    counts = np.asarray(counts, dtype=np.int64).reshape(-1)
    if len(counts) != len(seg) or (counts < 0).any() or not len(seg):
        raise ValueError('one non-negative element count per segment')
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    n = int(off[-1])
    out = torch.empty((n, 4, 3), dtype=torch.float64, device=B.device())
    seg_t, off_t = B.to_dev(seg, torch.float64), B.to_dev(off, torch.int64)
    B._call('tb_mesh_segments', seg_t.data_ptr(), off_t.data_ptr(), len(seg), out.data_ptr(), n, B._stream())
    return out


class LensGeometry:
    """A meshed electrode stack: vertices (N,4,3), per-element electrode index
    and the electrode names, in the element order used for the BEM matrix;
    `segments` (S, 4) lists the straight electrode segments (r0, z0, r1, z1)."""

    def __init__(self, vertices, electrode_index, names, segments=None, segment_counts=None):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.electrode_index = np.asarray(electrode_index, dtype=np.int64)
        self.names = list(names)
        self.segments = np.zeros((0, 4)) if segments is None else np.asarray(segments, dtype=np.float64)
        # elements per segment, when the mesh is exactly the graded mesh of `segments`
        self.segment_counts = None if segment_counts is None else np.asarray(segment_counts, dtype=np.int64)

    def vertices_device(self):
        """The same vertices meshed on the GPU from `segments` and
        `segment_counts` (tb_mesh_segments): a (N, 4, 3) device tensor."""
        if self.segment_counts is None:
            raise ValueError('this geometry does not record its segment counts')
        return mesh_segments_device(self.segments, self.segment_counts)

    def __len__(self):
        return len(self.vertices)

    def voltages_to_values(self, voltages) -> np.ndarray:
        v = np.asarray(voltages, dtype=np.float64)
        return v[self.electrode_index]

    def unit_rhs(self) -> np.ndarray:
        """One right-hand side per electrode at 1 V (the superposition basis of
        traceon/solver.py:364-400)."""
        F = np.zeros((len(self.names), len(self)))
        for e in range(len(self.names)):
            F[e, self.electrode_index == e] = 1.0
        return F


def einzel_lens(n_elements: int = 1000, r_tube: float = 1.0 * MM, r_cap: float = 2.0 * MM,
                spans=((-5 * MM, -1 * MM), (-0.5 * MM, 0.5 * MM), (1 * MM, 5 * MM))) -> LensGeometry:
    """Three coaxial tubes at r = 1 mm spanning z in [-5,-1], [-0.5,0.5],
    [1,5] mm with annular end caps to r = 2 mm; ``n_elements`` cubic elements
    split evenly across the electrodes and graded toward the tube edges."""
    k = len(spans)
    per = [n_elements // k + (1 if i < n_elements % k else 0) for i in range(k)]
    verts, idx, segs, counts = [], [], [], []
    for e, ((z0, z1), n) in enumerate(zip(spans, per)):
        v = aperture_tube(r_tube, r_cap, z0, z1, n)
        verts.append(v)
        idx.append(np.full(len(v), e))
        corners = [(r_cap, z0), (r_tube, z0), (r_tube, z1), (r_cap, z1)]
        segs += [(a[0], a[1], b[0], b[1]) for a, b in zip(corners[:-1], corners[1:])]
        counts += tube_counts(r_tube, r_cap, z0, z1, n)
    names = ['ground_in', 'lens', 'ground_out'][:k] if k == 3 else [f'electrode{i}' for i in range(k)]
    return LensGeometry(np.concatenate(verts), np.concatenate(idx), names, segs, counts)


def einzel_lens_voltages(seed: int) -> np.ndarray:
    """(0, V_mid, 0) with V_mid uniform in [500, 2000] V from the seed."""
    rng = np.random.default_rng(seed)
    return np.array([0.0, rng.uniform(500.0, 2000.0), 0.0])


def electron_beam(n: int, seed: int, energy_ev: float = 1000.0, z0: float = -9.5 * MM,
                  r_max: float = 0.2 * MM, angle_max: float = 5e-3, energy_spread: float = 0.0):
    """Start states of the lens workload: electrons at ``energy_ev`` (times
    U[1 - spread, 1 + spread]) starting at x = r ~ U[0, r_max], y = 0, z = z0,
    heading +z at an angle ~ U[-a, a] in the xz-plane.  Returns (positions
    (n,3), velocities (n,3)) in SI units; the speed follows
    traceon.tracing.velocity_vec (traceon/tracing.py:24-56)."""
    from scipy.constants import e, m_e
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, r_max, n)
    ang = rng.uniform(-angle_max, angle_max, n)
    energy = energy_ev * (rng.uniform(1 - energy_spread, 1 + energy_spread, n) if energy_spread else np.ones(n))
    speed = np.sqrt(2 * energy * e / m_e)[:, None]
    pos = np.stack([r, np.zeros(n), np.full(n, z0)], axis=1)
    vel = speed * np.stack([np.sin(ang), np.zeros(n), np.cos(ang)], axis=1)
    return pos, vel


def surrogate_beam(n: int, seed: int, r_max: float = 0.2 * MM):
    """The learned-surrogate workload's beam: 1 keV +-5 % (uniform), angles
    +-20 mrad, start radius up to r_max (default 0.2 mm, the plain-method
    workload's beam) at z = -9.5 mm."""
    return electron_beam(n, seed, r_max=r_max, angle_max=20e-3, energy_spread=0.05)


LENS_BOUNDS = np.array([[-2 * MM, 2 * MM], [-2 * MM, 2 * MM], [-10 * MM, 10 * MM]])
LENS_EXIT_Z = 9.5 * MM


def random_lens(seed: int, n_range=(500, 6000), tubes_range=(2, 5), r_range=(0.5 * MM, 3.0 * MM),
                gap_range=(0.2 * MM, 1.0 * MM), length_range=(1.0 * MM, 4.0 * MM), cap=0.5 * MM,
                volt_range=(-5000.0, 5000.0)):
    """A synthetic coaxial lens of the batching workload: N ~ U[n_range]
    elements over 2-5 tubes along z with radii ~ U[0.5, 3] mm, gaps between
    consecutive tubes ~ U[0.2, 1] mm, lengths ~ U[1, 4] mm, annular caps of
    0.5 mm; returns (geometry, voltages ~ U[-5, 5] kV per electrode)."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(n_range[0], n_range[1] + 1))
    k = int(rng.integers(tubes_range[0], tubes_range[1] + 1))
    radii = rng.uniform(*r_range, k)
    lengths = rng.uniform(*length_range, k)
    gaps = rng.uniform(*gap_range, k - 1)
    z = -0.5 * (lengths.sum() + gaps.sum())
    spans = []
    for i in range(k):
        spans.append((z, z + lengths[i]))
        z += lengths[i] + (gaps[i] if i < k - 1 else 0.0)
    # elements per electrode in proportion to its outline length
    outline = lengths + 2 * cap
    per = split_counts(n, outline) if k > 1 else [n]
    verts, idx, segs, counts = [], [], [], []
    for e, ((z0, z1), r, m) in enumerate(zip(spans, radii, per)):
        v = aperture_tube(r, r + cap, z0, z1, max(int(m), 6))
        verts.append(v)
        idx.append(np.full(len(v), e))
        corners = [(r + cap, z0), (r, z0), (r, z1), (r + cap, z1)]
        segs += [(a[0], a[1], b[0], b[1]) for a, b in zip(corners[:-1], corners[1:])]
        counts += tube_counts(r, r + cap, z0, z1, max(int(m), 6))
    geo = LensGeometry(np.concatenate(verts), np.concatenate(idx), [f'electrode{i}' for i in range(k)], segs, counts)
    return geo, rng.uniform(*volt_range, k)


class MirrorLens:
    """A lens of the batching workload: a random_lens stack followed by an
    electrostatic mirror (an aperture plate) at -1.1 x the beam voltage.
    geometry: LensGeometry whose last electrode is 'mirror'; voltages: one per
    electrode; z_start: where the beam starts (0.5 mm before the first tube);
    bounds: (3, 2) box the particles are traced in (a square inside the
    narrowest bore in x and y, from 0.5 mm behind the start to 1 mm past the
    mirror in z)."""

    def __init__(self, geometry, voltages, z_start, bounds):
        self.geometry, self.voltages, self.z_start, self.bounds = geometry, voltages, z_start, bounds


def mirror_lens(seed: int, n_range=(500, 6000), beam_voltage: float = 1000.0, mirror_gap=1.0 * MM,
                plate=0.2 * MM) -> MirrorLens:
    """random_lens(seed) with N ~ U[n_range] elements in all, the last ~10 %
    (at least 24) on a mirror plate: bore radius half the narrowest tube's, the
    same 0.5 mm cap, `plate` thick, `mirror_gap` after the last tube, at
    -1.1 x beam_voltage."""
    rng = np.random.default_rng(seed + 7919)
    n = int(rng.integers(n_range[0], n_range[1] + 1))
    n_mirror = max(24, n // 10)
    geo, volts = random_lens(seed, n_range=(n - n_mirror, n - n_mirror))
    segs = list(geo.segments)
    r_min = min(s[2] for s in segs[1::3])  # the tube segments' radius
    z_lo = min(min(s[1], s[3]) for s in segs)
    z_hi = max(max(s[1], s[3]) for s in segs)
    bore, cap = 0.5 * r_min, 0.5 * MM
    z0 = z_hi + mirror_gap
    v = aperture_tube(bore, bore + cap, z0, z0 + plate, n_mirror)
    corners = [(bore + cap, z0), (bore, z0), (bore, z0 + plate), (bore + cap, z0 + plate)]
    segs += [(a[0], a[1], b[0], b[1]) for a, b in zip(corners[:-1], corners[1:])]
    counts = list(geo.segment_counts) + tube_counts(bore, bore + cap, z0, z0 + plate, n_mirror)
    k = len(geo.names)
    lens = LensGeometry(np.concatenate([geo.vertices, v]), np.concatenate([geo.electrode_index, np.full(len(v), k)]),
                        list(geo.names) + ['mirror'], segs, counts)
    z_start = z_lo - 0.5 * MM
    h = 0.7 * bore
    bounds = np.array([[-h, h], [-h, h], [z_start - 0.5 * MM, z0 + plate + 1.0 * MM]])
    return MirrorLens(lens, np.concatenate([volts, [-1.1 * beam_voltage]]), z_start, bounds)


def mirror_beam(n: int, seed: int, z0: float, r_max: float = 0.05 * MM, angle_max: float = 50e-3,
                median_ev: float = 1000.0, sigma: float = 1.0, clip=(100.0, 10000.0)):
    """The batching workload's beam: electrons at energies lognormal (median
    1 keV, sigma 1, clipped to [100 eV, 10 keV]) from x = r ~ U[0, r_max],
    y = 0, z = z0, heading +z at angles ~ U[-50, 50] mrad in the xz-plane."""
    from scipy.constants import e, m_e
    rng = np.random.default_rng(seed)
    energy = np.clip(median_ev * np.exp(sigma * rng.standard_normal(n)), *clip)
    r = rng.uniform(0.0, r_max, n)
    ang = rng.uniform(-angle_max, angle_max, n)
    speed = np.sqrt(2 * energy * e / m_e)[:, None]
    pos = np.stack([r, np.zeros(n), np.full(n, z0)], axis=1)
    vel = speed * np.stack([np.sin(ang), np.zeros(n), np.cos(ang)], axis=1)
    return pos, vel


# ---------------------------------------------------------------- combined lens
# Outline of the iron pole piece of the combined workload's magnetic lens, in
# (r, z) mm: a closed C-shaped yoke whose bore (r = 2.5 mm) is open over
# |z| < 1 mm (the gap between the pole tips) and whose window r in
# (2.8, 7) mm, |z| < 5 mm holds the coils.
POLE_OUTLINE_MM = [(2.5, -6.0), (8.0, -6.0), (8.0, 6.0), (2.5, 6.0), (2.5, 1.0), (2.8, 1.0), (2.8, 5.0),
                   (7.0, 5.0), (7.0, -5.0), (2.8, -5.0), (2.8, -1.0), (2.5, -1.0), (2.5, -6.0)]


def outward_oriented(vertices: np.ndarray) -> np.ndarray:
    """The line4 elements of one closed outline, reversed if needed so that
    their normals point out of the enclosed body -- the test the reference
    mesher applies by default (traceon/mesher.py:730-739, divergence
    theorem: sum of r_mid n_r length > 0).  Reversal swaps start/end and the
    1/3 / 2/3 points of every element and the element order."""
    v = np.asarray(vertices, dtype=np.float64)
    d = v[:, 1] - v[:, 0]
    length = np.hypot(d[:, 0], d[:, 2])
    n_r = d[:, 2] / np.where(length > 0, length, 1.0)  # normal_2d: (dz, -dr) / |d|
    mid_r = 0.5 * (v[:, 0, 0] + v[:, 1, 0])
    if np.sum(mid_r * n_r * length) > 0:
        return v
    return v[::-1][:, [1, 0, 3, 2]].copy()


def coil_rings(r, z, current, half_width=0.1 * MM):
    """Current rings as the reference's current quadrature (N, 12) weights and
    (N, 12, 3) points (y = 0): each coil a square cross-section of side
    2 half_width around (r, z) sampled at 12 points (a 4 x 3 grid) of equal
    weight; current density x weights sums to the coil's A-turns.  Returns
    (current densities (N,), jac (N, 12), pos (N, 12, 3))."""
    r, z, current = (np.atleast_1d(np.asarray(a, dtype=np.float64)) for a in (r, z, current))
    area = (2 * half_width) ** 2
    ur = (np.arange(4) + 0.5) / 4 * 2 - 1
    uz = (np.arange(3) + 0.5) / 3 * 2 - 1
    gr, gz = np.meshgrid(ur, uz, indexing='ij')
    pos = np.zeros((len(r), 12, 3))
    pos[:, :, 0] = r[:, None] + half_width * gr.reshape(-1)[None]
    pos[:, :, 2] = z[:, None] + half_width * gz.reshape(-1)[None]
    jac = np.full((len(r), 12), area / 12)
    return current / area, jac, pos


class CombinedLens:
    """The combined electro-magnetostatic workload: the three-tube einzel
    lens (electrodes ground_in, lens, ground_out) inside the iron pole piece
    `pole` of a magnetic lens, magnetised by current coils.  `geometry` holds
    all elements (electrostatic first); coils: (r, z, A-turns) per coil."""

    def __init__(self, geometry, coils):
        self.geometry = geometry
        self.coil_r, self.coil_z, self.coil_current = (np.asarray(a, dtype=np.float64) for a in coils)

    def coil_sources(self, currents=None):
        """(current densities, jac, pos) of the coils (at `currents`, default
        their own A-turns)."""
        cur = self.coil_current if currents is None else np.asarray(currents, dtype=np.float64)
        return coil_rings(self.coil_r, self.coil_z, cur)


def combined_lens(seed: int, n_elec: int = 16384, n_mag: int = 16384, n_coils: int = 4) -> CombinedLens:
    """The combined workload's geometry: the einzel lens meshed to n_elec
    elements, the pole piece outline (POLE_OUTLINE_MM) meshed to n_mag
    elements graded toward its corners, normals out of the iron, and n_coils
    coils with r ~ U[3, 6] mm, z ~ U[-4, 4] mm, currents ~ U[0.5, 5] kA-turns
    from the seed."""
    lens = einzel_lens(n_elec)
    pts = np.array(POLE_OUTLINE_MM) * MM
    seg = np.hypot(*(pts[1:] - pts[:-1]).T)
    pole = outward_oriented(polyline_elements(pts, split_counts(n_mag, seg)))
    verts = np.concatenate([lens.vertices, pole])
    idx = np.concatenate([lens.electrode_index, np.full(len(pole), len(lens.names))])
    segs = np.concatenate([lens.segments, np.stack([pts[:-1, 0], pts[:-1, 1], pts[1:, 0], pts[1:, 1]], 1)])
    geo = LensGeometry(verts, idx, lens.names + ['pole'], segs)
    rng = np.random.default_rng(seed)
    coils = (rng.uniform(3e-3, 6e-3, n_coils), rng.uniform(-4e-3, 4e-3, n_coils),
             rng.uniform(500.0, 5000.0, n_coils))
    return CombinedLens(geo, coils)


def combined_beam(n: int, seed: int, r_max: float = 0.2 * MM, angle_max: float = 10e-3):
    """The combined workload's beam: electrons at 5 keV with a lognormal
    energy spread of 2 % (sigma of log E = 0.02), start radius up to r_max at
    z = -9.5 mm, angles U[-a, a] in the xz-plane."""
    from scipy.constants import e, m_e
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, r_max, n)
    ang = rng.uniform(-angle_max, angle_max, n)
    energy = 5000.0 * np.exp(rng.normal(0.0, 0.02, n))
    speed = np.sqrt(2 * energy * e / m_e)[:, None]
    pos = np.stack([r, np.zeros(n), np.full(n, -9.5 * MM)], axis=1)
    vel = speed * np.stack([np.sin(ang), np.zeros(n), np.cos(ang)], axis=1)
    return pos, vel

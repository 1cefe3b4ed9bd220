"""Procedural soccar arena mesh, passed to a BatchSim as ``ArenaLayout.meshes[0]`` (uu).

The game's collision meshes are not available, so both the oracle and this package take the same deterministic
synthetic arena: a box x in [-4096, 4096], y in [-5120, 5120], z in [0, 2044] with 45-degree corner bevels 1152 uu
wide, 256-uu quarter-cylinder fillets at the floor/wall and wall/ceiling edges tessellated at ``fillet_segments``
segments, and one goal recess 1786 (x) x 642 (z) x 880 (y deep) behind each end wall.

Construction: the wall cross-section (floor fillet, wall, ceiling fillet) is swept around the bevelled octagon: every
profile point (inset d, height z) becomes a ring made of the octagon inset by d, and neighbouring rings are joined by
quads. The floor and ceiling are concentric inset rings down to the centre. The goal mouth (|x| <= 893, z <= 642) is
cut out of the end-wall strips and a five-sided recess box is added behind it, with the floor fillet ends capped.
All arithmetic is float64 numpy and the result is rounded once to float32, so it is identical on every host.
"""
from __future__ import annotations

import numpy as np

HALF_X = 4096.0
HALF_Y = 5120.0
HEIGHT = 2044.0
BEVEL = 1152.0
FILLET_R = 256.0
GOAL_HALF_W = 893.0
GOAL_H = 642.0
GOAL_DEPTH = 880.0


def _octagon(d: float) -> np.ndarray:
    """Corners of the bevelled footprint inset by d (counter-clockwise, starting on the +y end wall's right end)."""
    hx, hy = HALF_X - d, HALF_Y - d
    # a 45-degree bevel moves by d * (sqrt(2) - 1) along each axis when inset by d
    b = BEVEL - d * (np.sqrt(2.0) - 1.0)
    b = max(b, 0.0)
    return np.array([
        [hx - b, hy], [-(hx - b), hy], [-hx, hy - b], [-hx, -(hy - b)],
        [-(hx - b), -hy], [hx - b, -hy], [hx, -(hy - b)], [hx, hy - b],
    ])


def _edge_params(seg_len: float) -> list[np.ndarray]:
    """Per octagon edge, the break parameters t in [0, 1] (shared by every ring so rings stay aligned).

    Edges 0 (+y end wall, going -x) and 4 (-y end wall, going +x) also break at the goal posts x = -+893.
    """
    outer = _octagon(0.0)
    params = []
    for e in range(8):
        a, b = outer[e], outer[(e + 1) % 8]
        length = float(np.hypot(*(b - a)))
        n = max(1, int(np.ceil(length / seg_len)))
        ts = list(np.linspace(0.0, 1.0, n + 1))
        if e in (0, 4):
            for post in (-GOAL_HALF_W, GOAL_HALF_W):
                t = (post - a[0]) / (b[0] - a[0])
                ts.append(t)
            ts = sorted(set(round(t, 12) for t in ts))
            # drop breaks that land too close to a goal post
            posts = [(p - a[0]) / (b[0] - a[0]) for p in (-GOAL_HALF_W, GOAL_HALF_W)]
            ts = [t for t in ts if any(abs(t - p) < 1e-9 for p in posts) or t in (0.0, 1.0)
                  or min(abs(t - p) for p in posts) * length > 0.3 * seg_len]
        params.append(np.array(ts))
    return params


def _ring(d: float, z: float, params: list[np.ndarray]) -> tuple[np.ndarray, list[tuple[int, int]]]:
    """Ring vertices at inset d, height z; returns (points [n, 3], per point (edge, index within edge))."""
    oc = _octagon(d)
    pts, tags = [], []
    for e in range(8):
        a, b = oc[e], oc[(e + 1) % 8]
        for k, t in enumerate(params[e][:-1]):
            p = a + (b - a) * t
            pts.append([p[0], p[1], z])
            tags.append((e, k))
    return np.array(pts), tags


def _in_goal_mouth(p: np.ndarray) -> bool:
    return abs(p[1]) > HALF_Y - FILLET_R - 1e-6 and abs(p[0]) < GOAL_HALF_W - 1e-6


def generate(fillet_segments: int = 16, seg_len: float = 384.0, wall_bands: int = 4, floor_rings: int = 10):
    """Returns (vertices float32 [V, 3] in uu, indices int32 [3T])."""
    params = _edge_params(seg_len)
    r = FILLET_R
    profile = []
    for i in range(fillet_segments + 1):
        th = 0.5 * np.pi * i / fillet_segments
        profile.append((r - r * np.sin(th), r - r * np.cos(th)))
    wall_z = list(np.linspace(r, HEIGHT - r, wall_bands + 1)[1:-1])
    if GOAL_H not in wall_z:
        wall_z.append(GOAL_H)
    for z in sorted(wall_z):
        profile.append((0.0, z))
    for i in range(fillet_segments + 1):
        ph = 0.5 * np.pi * i / fillet_segments
        profile.append((r - r * np.cos(ph), HEIGHT - r + r * np.sin(ph)))

    verts: list[np.ndarray] = []
    tris: list[tuple[int, int, int]] = []
    nv = 0

    def add_vertices(p: np.ndarray) -> int:
        nonlocal nv
        base = nv
        verts.append(np.asarray(p, dtype=np.float64).reshape(-1, 3))
        nv += len(verts[-1])
        return base

    # wall sweep
    rings = []
    for d, z in profile:
        pts, _ = _ring(d, z, params)
        rings.append((add_vertices(pts), pts))
    n = len(rings[0][1])
    for j in range(len(rings) - 1):
        (b0, p0), (b1, p1) = rings[j], rings[j + 1]
        z_hi = max(profile[j][1], profile[j + 1][1])
        for k in range(n):
            k1 = (k + 1) % n
            mid = 0.5 * (p0[k] + p0[k1])
            if _in_goal_mouth(np.array([mid[0], np.sign(mid[1]) * HALF_Y])) and z_hi <= GOAL_H + 1e-6 \
                    and abs(mid[1]) > 0.0 and abs(abs(mid[1]) - (HALF_Y - profile[j][0])) < 1e-6:
                continue
            # the normal faces into the arena: rings run counter-clockwise seen from above, z grows with j
            tris.append((b0 + k, b1 + k, b0 + k1))
            tris.append((b0 + k1, b1 + k, b1 + k1))

    # floor and ceiling: concentric rings from the fillet edge inward, closed by a fan at the centre
    for z, up in ((0.0, True), (HEIGHT, False)):
        ds = np.linspace(r, HALF_X - 64.0, floor_rings + 1)
        frings = []
        for d in ds:
            pts, _ = _ring(d, z, params)
            frings.append((add_vertices(pts), pts))
        for j in range(len(frings) - 1):
            (b0, p0), (b1, _) = frings[j], frings[j + 1]
            for k in range(n):
                k1 = (k + 1) % n
                if up:
                    tris.append((b0 + k, b0 + k1, b1 + k))
                    tris.append((b0 + k1, b1 + k1, b1 + k))
                else:
                    tris.append((b0 + k, b1 + k, b0 + k1))
                    tris.append((b0 + k1, b1 + k, b1 + k1))
        bl, _ = frings[-1]
        c = add_vertices(np.array([[0.0, 0.0, z]]))
        for k in range(n):
            k1 = (k + 1) % n
            tris.append((bl + k, bl + k1, c) if up else (bl + k, c, bl + k1))

    # goal mouth floor strip, fillet end caps and recess boxes
    for s in (1.0, -1.0):
        y0, y1 = s * (HALF_Y - r), s * HALF_Y
        y2 = s * (HALF_Y + GOAL_DEPTH)
        w, h = GOAL_HALF_W, GOAL_H

        def quad(a, b, c, d, flip):
            base = add_vertices(np.array([a, b, c, d]))
            if (s > 0) != flip:
                tris.append((base, base + 1, base + 2))
                tris.append((base, base + 2, base + 3))
            else:
                tris.append((base, base + 2, base + 1))
                tris.append((base, base + 3, base + 2))

        quad([-w, y0, 0.0], [w, y0, 0.0], [w, y1, 0.0], [-w, y1, 0.0], False)      # mouth floor (up)
        quad([-w, y1, 0.0], [w, y1, 0.0], [w, y2, 0.0], [-w, y2, 0.0], False)      # recess floor (up)
        quad([-w, y1, h], [-w, y2, h], [w, y2, h], [w, y1, h], False)              # recess ceiling (down)
        quad([-w, y2, 0.0], [w, y2, 0.0], [w, y2, h], [-w, y2, h], False)          # back wall (toward field)
        for sx in (-1.0, 1.0):
            x = sx * w
            a, b, c, d = [x, y1, 0.0], [x, y2, 0.0], [x, y2, h], [x, y1, h]
            quad(a, b, c, d, sx < 0)                                              # side walls (inward)
            # cap the floor fillet's end at the post: fan over the fillet cross-section
            cap = [[x, s * HALF_Y, 0.0]]
            for i in range(fillet_segments + 1):
                th = 0.5 * np.pi * i / fillet_segments
                cap.append([x, s * (HALF_Y - (r - r * np.sin(th))), r - r * np.cos(th)])
            cb = add_vertices(np.array(cap))
            for i in range(1, fillet_segments + 1):
                if (sx > 0) == (s > 0):
                    tris.append((cb, cb + i, cb + i + 1))
                else:
                    tris.append((cb, cb + i + 1, cb + i))
        # wall above the goal mouth up to z = h between the posts is part of the sweep (kept); the fillet rings
        # between the posts below h were skipped above.

    v = np.concatenate(verts, axis=0).astype(np.float32)
    idx = np.asarray(tris, dtype=np.int32).reshape(-1)
    return v, idx


def generate_dense(fillet_segments: int = 64):
    """The ~40k-triangle variant (64-segment fillets, finer panels)."""
    return generate(fillet_segments=fillet_segments, seg_len=224.0, wall_bands=8, floor_rings=16)


def generate_fine(fillet_segments: int = 64):
    """The contact-heavy stress workload's second geometry: 64-segment fillets and finer panels, ~42k triangles."""
    return generate(fillet_segments=fillet_segments, seg_len=256.0, wall_bands=6, floor_rings=12)

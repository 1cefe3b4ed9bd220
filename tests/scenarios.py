"""Seeded synthetic scenarios shared by the parity tests, the golden-fixture script and bench.py.

Ball-only arenas: each arena's ball starts at a seeded position inside the procedural arena with a seeded velocity
(uniform direction, speed U[0, vmax] uu/s) and angular velocity, as the contact-heavy stress config draws the ball's
start (random velocity up to 6000 uu/s in a uniform direction). Everything is derived from numpy's PCG64 with the
given seed, so every host produces the same inputs.
"""
from __future__ import annotations

import numpy as np

BALL_BYTES = 288
OFF_POS, OFF_VEL, OFF_ANG = 40, 68, 80


def ball_states(default_ball: np.ndarray, n: int, seed: int, vmax: float = 6000.0, z_range=(150.0, 1800.0),
                xy_scale=(3000.0, 4000.0)) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = np.tile(np.asarray(default_ball, np.uint8).reshape(1, BALL_BYTES), (n, 1))
    pos = np.stack([rng.uniform(-xy_scale[0], xy_scale[0], n), rng.uniform(-xy_scale[1], xy_scale[1], n),
                    rng.uniform(z_range[0], z_range[1], n)], 1).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    vel = (d * rng.uniform(0.0, vmax, (n, 1))).astype(np.float32)
    ang = rng.uniform(-4.0, 4.0, (n, 3)).astype(np.float32)
    out[:, OFF_POS:OFF_POS + 12] = pos.view(np.uint8).reshape(n, 12)
    out[:, OFF_VEL:OFF_VEL + 12] = vel.view(np.uint8).reshape(n, 12)
    out[:, OFF_ANG:OFF_ANG + 12] = ang.view(np.uint8).reshape(n, 12)
    return out


def free_flight_states(default_ball: np.ndarray, n: int, seed: int) -> np.ndarray:
    """Balls high in the middle of the arena, slow enough to stay clear of every surface for 60 ticks."""
    return ball_states(default_ball, n, seed, vmax=300.0, z_range=(900.0, 1300.0), xy_scale=(2000.0, 3000.0))


def ball_pos(b: np.ndarray) -> np.ndarray:
    return b[:, OFF_POS:OFF_POS + 12].copy().view(np.float32)

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


# ---- cars -------------------------------------------------------------------------------------------------------------
CAR_BYTES, CONTROLS_BYTES = 880, 24
CAR_POS, CAR_ROT, CAR_VEL, CAR_ANG, CAR_ON_GROUND = 0, 12, 28, 40, 122


def _yaw_quat(yaw):
    return np.stack([np.cos(yaw / 2), np.zeros_like(yaw), np.zeros_like(yaw), np.sin(yaw / 2)], 1)


def airborne_cars(template: np.ndarray, n: int, seed: int, z: float = 1000.0) -> np.ndarray:
    """One car per row high above the floor: seeded position, uniform random orientation, slow linear and angular
    velocity, not on the ground (the cars fall freely for about 100 ticks)."""
    rng = np.random.default_rng(seed)
    out = np.tile(np.asarray(template, np.uint8).reshape(1, CAR_BYTES), (n, 1))
    pos = np.stack([rng.uniform(-2000, 2000, n), rng.uniform(-3000, 3000, n), np.full(n, z)], 1).astype(np.float32)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    out[:, CAR_POS:CAR_POS + 12] = pos.view(np.uint8).reshape(n, 12)
    out[:, CAR_ROT:CAR_ROT + 16] = q.astype(np.float32).view(np.uint8).reshape(n, 16)
    out[:, CAR_VEL:CAR_VEL + 12] = rng.uniform(-300, 300, (n, 3)).astype(np.float32).view(np.uint8).reshape(n, 12)
    out[:, CAR_ANG:CAR_ANG + 12] = rng.uniform(-2, 2, (n, 3)).astype(np.float32).view(np.uint8).reshape(n, 12)
    out[:, CAR_ON_GROUND] = 0
    return out


def grounded_cars(template: np.ndarray, n: int, seed: int) -> np.ndarray:
    """One car per row resting on its wheels near the middle of the floor with a seeded heading and speed."""
    rng = np.random.default_rng(seed)
    out = np.tile(np.asarray(template, np.uint8).reshape(1, CAR_BYTES), (n, 1))
    pos = np.stack([rng.uniform(-1500, 1500, n), rng.uniform(-2500, 2500, n), np.full(n, 17.0)], 1).astype(np.float32)
    yaw = rng.uniform(-np.pi, np.pi, n)
    q = _yaw_quat(yaw)
    speed = rng.uniform(0, 1500, n)
    vel = np.stack([np.cos(yaw) * speed, np.sin(yaw) * speed, np.zeros(n)], 1).astype(np.float32)
    out[:, CAR_POS:CAR_POS + 12] = pos.view(np.uint8).reshape(n, 12)
    out[:, CAR_ROT:CAR_ROT + 16] = q.astype(np.float32).view(np.uint8).reshape(n, 16)
    out[:, CAR_VEL:CAR_VEL + 12] = vel.view(np.uint8).reshape(n, 12)
    return out


class ControlStream:
    """Seeded random controls: axes U[-1, 1], jump / boost / handbrake Bernoulli(p_jump / 0.3 / 0.1), each car's sample
    held for U{1..hold_max} ticks."""

    def __init__(self, rows: int, seed: int, p_jump: float = 0.1, hold_max: int = 1):
        self.rng = np.random.default_rng(seed)
        self.rows, self.p_jump, self.hold_max = rows, p_jump, hold_max
        self.cur = np.zeros((rows, CONTROLS_BYTES), np.uint8)
        self.left = np.zeros(rows, np.int64)

    def next(self) -> np.ndarray:
        renew = self.left <= 0
        k = int(renew.sum())
        if k:
            f = self.rng.uniform(-1, 1, (k, 5)).astype(np.float32)
            row = np.zeros((k, CONTROLS_BYTES), np.uint8)
            row[:, :20] = f.view(np.uint8).reshape(k, 20)
            row[:, 20] = self.rng.random(k) < self.p_jump
            row[:, 21] = self.rng.random(k) < 0.3
            row[:, 22] = self.rng.random(k) < 0.1
            self.cur[renew] = row
            self.left[renew] = self.rng.integers(1, self.hold_max + 1, k)
        self.left -= 1
        return self.cur.copy()


def chase_ball_controls(cars: np.ndarray, balls: np.ndarray, max_cars: int, rng: np.random.Generator,
                        p_jump: float = 0.02) -> np.ndarray:
    """A ball-chasing driver for every car slot (dense car rows [envs * max_cars, CAR_BYTES], balls [envs, BALL_BYTES]):
    full throttle and boost, steering proportional to the heading error toward the arena's ball, rare jumps, seeded
    air-control noise. The game's quaternions are (w, x, y, z); forward is the body x axis."""
    n = cars.shape[0]
    pos = cars[:, CAR_POS:CAR_POS + 12].copy().view(np.float32).astype(np.float64)
    q = cars[:, CAR_ROT:CAR_ROT + 16].copy().view(np.float32).astype(np.float64)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    yaw = np.arctan2(2.0 * (x * y + w * z), 1.0 - 2.0 * (y * y + z * z))
    bpos = np.repeat(balls[:, OFF_POS:OFF_POS + 12].copy().view(np.float32).astype(np.float64), max_cars, axis=0)
    want = np.arctan2(bpos[:, 1] - pos[:, 1], bpos[:, 0] - pos[:, 0])
    err = (want - yaw + np.pi) % (2.0 * np.pi) - np.pi
    ctrl = np.zeros((n, CONTROLS_BYTES), np.uint8)
    f = np.zeros((n, 5), np.float32)
    f[:, 0] = 1.0
    f[:, 1] = np.clip(2.5 * err, -1.0, 1.0)
    f[:, 2:5] = rng.uniform(-0.3, 0.3, (n, 3))
    ctrl[:, :20] = f.view(np.uint8).reshape(n, 20)
    ctrl[:, 20] = rng.random(n) < p_jump
    ctrl[:, 21] = 1
    return ctrl


# ---- episodes ---------------------------------------------------------------------------------------------------------
ENV_COMMAND_BYTES = 16
CAR_LATEST_TOUCH = 520  # CarState.latest_touch_tick (u64)
ENV_TICK, ENV_BLUE, ENV_ORANGE = 0, 4, 8


def _splitmix(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)).astype(np.uint64)
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)).astype(np.uint64)
    return x ^ (x >> np.uint64(31))


class EpisodeClock:
    """Host statement of rg_batch_episode_commands for the oracle side: after each step, an env whose score is non-zero
    (a goal this episode) or whose ball no car touched for `no_touch_ticks` ticks gets a fresh-episode reset
    (reset_to_kickoff = reset_scoreboard = reset_tick_count = 1) for the next step's first tick. Touches are seen
    through each car's latest_touch_tick changing between checks; `stagger_seed` starts each env's clock at a seeded
    age in [0, no_touch_ticks)."""

    def __init__(self, envs: np.ndarray, cars: np.ndarray, max_cars: int, no_touch_ticks: int, stagger_seed: int = 0):
        n = envs.shape[0]
        self.max_cars, self.no_touch = max_cars, no_touch_ticks
        self.seen = cars[:, CAR_LATEST_TOUCH:CAR_LATEST_TOUCH + 8].copy().view(np.uint64).reshape(n, max_cars)
        tick = envs[:, ENV_TICK:ENV_TICK + 4].copy().view(np.uint32).ravel().astype(np.int64)
        age = np.zeros(n, np.int64)
        if stagger_seed:
            with np.errstate(over="ignore"):
                h = _splitmix(np.uint64(stagger_seed) ^ np.arange(n, dtype=np.uint64))
            age = (h % np.uint64(no_touch_ticks)).astype(np.int64)
        self.touch = tick - age

    def commands(self, envs: np.ndarray, cars: np.ndarray, counts: np.ndarray) -> np.ndarray:
        n = envs.shape[0]
        latest = cars[:, CAR_LATEST_TOUCH:CAR_LATEST_TOUCH + 8].copy().view(np.uint64).reshape(n, self.max_cars)
        active = np.arange(self.max_cars)[None, :] < np.asarray(counts)[:, None]
        changed = active & (latest != self.seen)
        self.seen = np.where(changed, latest, self.seen)
        valid = changed & (latest != np.uint64(0xFFFFFFFFFFFFFFFF))
        cand = np.where(valid, latest.astype(np.int64), np.iinfo(np.int64).min)
        self.touch = np.maximum(self.touch, cand.max(axis=1))
        tick = envs[:, ENV_TICK:ENV_TICK + 4].copy().view(np.uint32).ravel().astype(np.int64)
        score = envs[:, ENV_BLUE:ENV_BLUE + 4].copy().view(np.uint32).ravel() | \
            envs[:, ENV_ORANGE:ENV_ORANGE + 4].copy().view(np.uint32).ravel()
        reset = (score != 0) | (tick - self.touch >= self.no_touch)
        self.touch = np.where(reset, 0, self.touch)
        out = np.zeros((n, ENV_COMMAND_BYTES), np.uint8)
        out[reset, 0:3] = 1
        return out


def contact_heavy(cars: np.ndarray, balls: np.ndarray, counts: np.ndarray, max_cars: int, seed: int):
    """The contact-heavy stress start: each arena's ball at a seeded point in the middle of the field with a velocity
    of up to 6000 uu/s in a uniform random direction, and its cars spawned within 600 uu of the ball (on the floor or
    in the air), heading toward the ball at up to supersonic speed. `cars` [envs * max_cars] and `balls` [envs] are the kickoff states to start
    from; returns the states to upload."""
    rng = np.random.default_rng(seed)
    n = balls.shape[0]
    b = balls.copy()
    bpos = np.stack([rng.uniform(-2500, 2500, n), rng.uniform(-3500, 3500, n), rng.uniform(150, 900, n)], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    bvel = d * rng.uniform(0, 6000, (n, 1))
    b[:, OFF_POS:OFF_POS + 12] = bpos.astype(np.float32).view(np.uint8).reshape(n, 12)
    b[:, OFF_VEL:OFF_VEL + 12] = bvel.astype(np.float32).view(np.uint8).reshape(n, 12)
    c = cars.copy()
    for e in range(n):
        for s in range(int(counts[e])):
            row = e * max_cars + s
            off = rng.normal(size=3)
            off /= np.linalg.norm(off)
            off *= rng.uniform(200, 600)
            p = bpos[e] + off
            p[2] = max(17.0, min(p[2], 1200.0))
            # heading toward the ball give or take 30 degrees, up to supersonic speed
            yaw = np.arctan2(bpos[e, 1] - p[1], bpos[e, 0] - p[0]) + rng.uniform(-0.5, 0.5)
            q = _yaw_quat(np.array([yaw]))[0]
            v = np.array([np.cos(yaw), np.sin(yaw), 0.0]) * rng.uniform(800, 2300)
            c[row, CAR_POS:CAR_POS + 12] = p.astype(np.float32).view(np.uint8)
            c[row, CAR_ROT:CAR_ROT + 16] = q.astype(np.float32).view(np.uint8)
            c[row, CAR_VEL:CAR_VEL + 12] = v.astype(np.float32).view(np.uint8)
            c[row, CAR_ON_GROUND] = 1 if p[2] <= 17.0 else 0
    return c, b

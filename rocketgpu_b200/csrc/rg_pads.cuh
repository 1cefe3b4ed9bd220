// Boost pads of one arena: cooldown countdown before the tick, the swept pickup test and the touch bookkeeping after
// it, and the give / respawn rules (reference include/rocketgpu/detail/step/env_step.hpp:1946-2030, 2160-2907,
// a layout's own pad list as BatchSim runs it for a custom ArenaLayout).
#pragma once

#include "rg_car.cuh"

namespace rg {

// The layout's pads (a custom layout keeps the game's 34 soccar pads unless it lists its own).
struct PadLayout {
    V3 pos[64];
    uint8_t is_big[64];
    int count;
};

RG_HDI uint16_t pad_frac_q(float frame_frac) {
    return static_cast<uint16_t>(fmin_(fmax_(frame_frac, 0.0f), 1.0f) * 65535.0f + 0.5f);
}
RG_HDI void pad_pre_tick(PadState& p, float dt) {
    if (!p.is_active || p.cooldown > 0.0f) {
        p.cooldown -= dt;
        p.is_active = 0;
    }
    if (p.cur_locked_car_id != 0) p.cur_locked_car_id = 0;
}
RG_HDI bool pad_respawn_due(const PadState& p, float dt, float frame_frac) {
    const float left = floorf(p.cooldown / dt + 0.5f) + 1.0f;
    return left < 0.0f || (left == 0.0f && p.pickup_frac_q < pad_frac_q(frame_frac));
}
RG_HDI V3 pad_rb_pos_uu(V3 pos_bt) {
    const V3 p = pos_bt * 50.0f;
    return V3{quant_round_pos(p.x, 100.0f), quant_round_pos(p.y, 100.0f), quant_round_pos(p.z, 100.0f)};
}
RG_HDI V3 pad_frame_pos(const CarState& c, float frame_frac) {
    const V3 p0 = pad_rb_pos_uu(c.tick_start_pos_bt);
    const V3 p1 = pad_rb_pos_uu(c.pos_bt);
    return p0 + (p1 - p0) * frame_frac;
}
RG_HDI void pad_frame_axes(const CarState& c, const TickConfig& tc, V3 axes[3]) {
    car_basis(c, axes[0], axes[1], axes[2]);
    const V3 w = c.is_demoed ? c.ang_vel : clamp_length(c.ang_vel, tc.car_max_ang_speed);
    const V3 spin_back = w * (-(1.0f - tc.frame_frac) * tc.tick_dt);
    for (int a = 0; a < 3; ++a) axes[a] = axes[a] + cross(spin_back, axes[a]);
}
RG_HDI V3 pad_sweep_from_bt(const CarState& c, V3 car_bt) {
    if (c.pad_frame_pos_valid) {
        const V3 moved = car_bt - c.pad_frame_pos_bt;
        if (dot(moved, moved) <= (240.0f / 50.0f) * (240.0f / 50.0f)) return c.pad_frame_pos_bt;
    }
    const V3 p0 = pad_rb_pos_uu(c.tick_start_pos_bt);
    const V3 p1 = pad_rb_pos_uu(c.pos_bt);
    return car_bt - (p1 - p0) * (1.0f / 50.0f);
}
RG_HDI void pad_store_frame_pos(CarState& c, const TickConfig& tc) {
    c.pad_frame_pos_bt = pad_frame_pos(c, tc.frame_frac) * (1.0f / 50.0f);
    c.pad_frame_pos_valid = c.is_demoed ? 0 : 1;
}
// Entry of the car's swept point into the pad's cylinder (reference BoostPadSweepEnterBt).
RG_HDI bool pad_sweep_enter(V3 pad_pos_uu, bool is_big, V3 from_bt, V3 to_bt, float& enter) {
    const float rad_bt = (is_big ? 160.0f + 48.0f : 128.0f + 48.0f) * kUuToBt;
    const float half_z_bt = (64.0f + 32.0f) * kUuToBt;
    const float pad_z_bt = (pad_pos_uu.z - (is_big ? 1.0f : 5.92f)) * kUuToBt;
    float s0 = 0.0f, s1 = 1.0f;
    const float z0 = from_bt.z - pad_z_bt;
    const float dz = to_bt.z - from_bt.z;
    if (fabs_(dz) < 1e-7f) {
        if (fabs_(z0) >= half_z_bt) return false;
    } else {
        const float ta = (-half_z_bt - z0) / dz;
        const float tb = (half_z_bt - z0) / dz;
        s0 = fmax_(s0, fmin_(ta, tb));
        s1 = fmin_(s1, fmax_(ta, tb));
    }
    const float ax = from_bt.x - pad_pos_uu.x * kUuToBt;
    const float ay = from_bt.y - pad_pos_uu.y * kUuToBt;
    const float dx = to_bt.x - from_bt.x;
    const float dy = to_bt.y - from_bt.y;
    const float a = dx * dx + dy * dy;
    const float b = ax * dx + ay * dy;
    const float cc = ax * ax + ay * ay - rad_bt * rad_bt;
    if (a < 1e-12f) {
        enter = s0;
        return false;
    }
    const float disc = b * b - a * cc;
    if (disc <= 0.0f) return false;
    const float root = sqrtf(disc);
    enter = fmax_(s0, (-b - root) / a);
    return enter < fmin_(s1, (-b + root) / a);
}
// Oriented-box overlap of the car's hitbox with the pad's box (reference BoostPadBoxOverlap, :2300-2342).
RG_HDI bool pad_box_overlap(V3 pad_pos_uu, bool is_big, V3 car_uu, const V3 axes[3], const CarConfig& cfg) {
    const float pad_r = is_big ? 160.0f : 128.0f;
    const float h[3] = {pad_r, pad_r, 64.0f};
    const float e[3] = {cfg.hitbox_size.x * 0.5f - 1.25f, cfg.hitbox_size.y * 0.5f - 1.25f,
                        cfg.hitbox_size.z * 0.5f - 1.25f};
    const V3 centre = car_uu + axes[0] * cfg.hitbox_offset.x + axes[1] * cfg.hitbox_offset.y +
                      axes[2] * cfg.hitbox_offset.z;
    const float t[3] = {centre.x - pad_pos_uu.x, centre.y - pad_pos_uu.y,
                        centre.z - (pad_pos_uu.z - (is_big ? 1.0f : 5.917984f))};
    float r[3][3], ar[3][3];
    for (int j = 0; j < 3; ++j) {
        const float cj[3] = {axes[j].x, axes[j].y, axes[j].z};
        for (int i = 0; i < 3; ++i) {
            r[i][j] = cj[i];
            ar[i][j] = fabs_(cj[i]) + 1e-6f;
        }
    }
    for (int i = 0; i < 3; ++i)
        if (fabs_(t[i]) > h[i] + e[0] * ar[i][0] + e[1] * ar[i][1] + e[2] * ar[i][2]) return false;
    for (int j = 0; j < 3; ++j) {
        const float tb = t[0] * r[0][j] + t[1] * r[1][j] + t[2] * r[2][j];
        if (fabs_(tb) > h[0] * ar[0][j] + h[1] * ar[1][j] + h[2] * ar[2][j] + e[j]) return false;
    }
    for (int i = 0; i < 3; ++i) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
        for (int j = 0; j < 3; ++j) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            const float ra = h[i1] * ar[i2][j] + h[i2] * ar[i1][j];
            const float rb = e[j1] * ar[i][j2] + e[j2] * ar[i][j1];
            if (fabs_(t[i2] * r[i1][j] - t[i1] * r[i2][j]) > ra + rb) return false;
        }
    }
    return true;
}

// Pads whose cylinder the car's frame-interpolated point swept through this tick, and the overlaps of the car's box
// with those pads and with the pad it is touching (reference BoostPadContactsForCar, :2412-2505, custom-layout branch).
RG_HDI uint64_t pad_contacts_for_car(const CarState& c, const CarConfig& cfg, const PadState* pads,
                                     const PadLayout& L, const TickConfig& tc, uint64_t& overlap, V3& frame_pos_bt) {
    uint64_t hits = 0u;
    overlap = 0u;
    const V3 car_pos = pad_frame_pos(c, tc.frame_frac);
    const V3 car_bt = car_pos * (1.0f / 50.0f);
    frame_pos_bt = car_bt;
    const V3 prev = pad_sweep_from_bt(c, car_bt);
    const V3 lo = vmin(car_bt, prev), hi = vmax(car_bt, prev);
    for (int p = 0; p < L.count; ++p) {
        const V3 pad_bt = L.pos[p] * kUuToBt;
        if (pad_bt.x < lo.x - 240.0f * kUuToBt || pad_bt.x > hi.x + 240.0f * kUuToBt ||
            pad_bt.y < lo.y - 240.0f * kUuToBt || pad_bt.y > hi.y + 240.0f * kUuToBt ||
            pad_bt.z < lo.z - 135.0f * kUuToBt || pad_bt.z > hi.z + 135.0f * kUuToBt)
            continue;
        float enter = 0.0f;
        if (pad_sweep_enter(L.pos[p], pads[p].is_big != 0, prev, car_bt, enter)) hits |= 1ull << p;
    }
    uint64_t check = hits;
    if (c.boost_pad_touching != 0) check |= 1ull << (c.boost_pad_touching - 1);
    if (check != 0u) {
        V3 axes[3];
        pad_frame_axes(c, tc, axes);
        for (; check != 0u; check &= check - 1u) {
            const int p = ctz64(check);
            if (pad_box_overlap(L.pos[p], pads[p].is_big != 0, car_pos, axes, cfg)) overlap |= 1ull << p;
        }
    }
    return hits;
}

// A car's pad contacts for the pads' tail, computed by the car's own thread after its post-tick: the pads whose
// sweep the car entered this tick, the pads its box overlaps among those and the pad it was touching, and its frame
// position. Exact ahead of the arena's pad pass: the geometry reads only the car and the pads' fixed sizes; an
// earlier car's pickup may clear this car's touching pad, which only makes one overlap bit unused.
struct PadContacts {
    uint64_t hits, overlap;
    V3 frame_pos_bt;
};
RG_HDI void pad_contacts_stage(const CarState& c, const CarConfig& cfg, const PadState* pads, const PadLayout& L,
                               const TickConfig& tc, PadContacts& out) {
    out.hits = out.overlap = 0u;
    out.frame_pos_bt = V3{0.0f, 0.0f, 0.0f};
    if (!c.is_demoed) out.hits = pad_contacts_for_car(c, cfg, pads, L, tc, out.overlap, out.frame_pos_bt);
}

RG_HDI bool pad_eligible(const CarState& c, const TickConfig& tc) {
    return !c.is_demoed && !c.driving_disabled && c.boost < tc.boost_max;
}
RG_HDI void pad_touch_step(PadState& pad, int p, CarState& c, uint32_t car_id, bool in_cylinder, bool overlapping,
                           bool eligible) {
    if (!pad.is_active || pad.cur_locked_car_id != 0) return;
    const uint8_t touching = static_cast<uint8_t>(p + 1);
    if (c.boost_pad_touching == touching) {
        if (!overlapping) c.boost_pad_touching = 0;
    } else if (in_cylinder) {
        if (eligible) {
            c.boost_pad_touching = touching;
            pad.cur_locked_car_id = car_id;
        } else if (overlapping) {
            c.boost_pad_touching = touching;
        }
    }
}
// Pickup: the car gets the pad's boost, the pad starts its cooldown (reference BoostPadGive, :2562-2585).
// `cars` is the arena's car array; car ids are global slot + 1.
RG_HDI void pad_give(CarState* cars, int car_base, int max_cars, PadState& pad, int p, uint32_t car_id,
                     const TickConfig& tc) {
    CarState& c = cars[static_cast<int>(car_id - 1u) - car_base];
    const float boost_before = c.boost;
    car_set_boost_amount(c, fmin_(tc.boost_max / 100.0f, car_boost_amount(c) + (pad.is_big ? 1.0f : 0.12f)));
    pad.is_active = 0;
    pad.cooldown = (pad.is_big ? tc.boost_pad_cooldown_big : tc.boost_pad_cooldown_small) - tc.tick_dt;
    pad.pickup_frac_q = pad_frac_q(tc.frame_frac);
    for (int i = 0; i < max_cars; ++i)
        if (cars[i].boost_pad_touching == p + 1) cars[i].boost_pad_touching = 0;
    if (tc.events.windows) {
        PhysicsEvent e = new_event(kEventBoostPickup);
        e.car_id = car_id;
        e.pad_index = static_cast<uint32_t>(p);
        e.is_big_pad = pad.is_big;
        e.boost_before = boost_before;
        e.boost_after = c.boost;
        emit_event(tc.events, static_cast<uint32_t>(car_base / max_cars), e);
    }
}
// More than one pad hit in one tick: visit them in order of entry (reference BoostPadSweepTouchSteps, :2587-2637).
RG_HDI void pad_sweep_touch_steps(CarState* cars, int car_base, int max_cars, int slot, PadState* pads,
                                  const PadLayout& L, const TickConfig& tc, uint64_t hits, uint64_t overlap) {
    CarState& c = cars[slot];
    const uint32_t car_id = static_cast<uint32_t>(car_base + slot + 1);
    const V3 to_bt = pad_frame_pos(c, tc.frame_frac) * (1.0f / 50.0f);
    const V3 from_bt = pad_sweep_from_bt(c, to_bt);
    if (c.boost_pad_touching != 0 && ((hits >> (c.boost_pad_touching - 1)) & 1u) == 0u) {
        const int p = c.boost_pad_touching - 1;
        pad_touch_step(pads[p], p, c, car_id, false, ((overlap >> p) & 1u) != 0u, false);
    }
    for (uint64_t left = hits; left != 0u;) {
        int p = -1;
        float best = 0.0f;
        for (uint64_t m = left; m != 0u; m &= m - 1u) {
            const int q = ctz64(m);
            float s = 0.0f;
            pad_sweep_enter(L.pos[q], pads[q].is_big != 0, from_bt, to_bt, s);
            if (p < 0 || s < best) {
                p = q;
                best = s;
            }
        }
        if (p < 0) break;
        left &= ~(1ull << p);
        PadState& pad = pads[p];
        if (!pad.is_active || pad.cur_locked_car_id != 0) continue;
        if (c.boost_pad_touching == p + 1) {
            if (((overlap >> p) & 1u) == 0u) c.boost_pad_touching = 0;
            continue;
        }
        if (pad_eligible(c, tc)) {
            c.boost_pad_touching = static_cast<uint8_t>(p + 1);
            pad.cur_locked_car_id = car_id;
            pad_give(cars, car_base, max_cars, pad, p, car_id, tc);
        } else if (((overlap >> p) & 1u) != 0u) {
            c.boost_pad_touching = static_cast<uint8_t>(p + 1);
        }
    }
}

// The pads' part of the tick tail (reference BoostPadTouchPassForEnv, :2706-2835, and PostTickBoostPadsForEnv,
// :2851-2892). `order` lists the car slots in visit order.
// `staged` (null: computed here) holds car slot i's pad contacts (pad_contacts_stage) at byte offset
// i * staged_stride.
RG_NOINL void pads_tail(CarState* cars, int car_base, int max_cars, const CarConfig* cfgs, int count, const int* order,
                      PadState* pads, const PadLayout& L, const TickConfig& tc, const PadContacts* staged = nullptr,
                      size_t staged_stride = sizeof(PadContacts)) {
    if (!tc.enable_boost_pads || tc.frame_frac < 0.0f) return;
    for (int k = 0; k < count; ++k) {
        const int i = order[k];
        CarState& c = cars[i];
        uint64_t overlap = 0u, hits = 0u;
        V3 frame_pos_bt{0.0f, 0.0f, 0.0f};
        if (staged) {
            const PadContacts& pc = *reinterpret_cast<const PadContacts*>(
                reinterpret_cast<const unsigned char*>(staged) + static_cast<size_t>(i) * staged_stride);
            hits = pc.hits;
            overlap = pc.overlap;
            frame_pos_bt = pc.frame_pos_bt;
        } else if (!c.is_demoed) {
            hits = pad_contacts_for_car(c, cfgs[i], pads, L, tc, overlap, frame_pos_bt);
        }
        if ((hits & (hits - 1u)) != 0u) {
            pad_sweep_touch_steps(cars, car_base, max_cars, i, pads, L, tc, hits, overlap);
        } else {
            const bool eligible = pad_eligible(c, tc);
            uint64_t near = hits;
            if (c.boost_pad_touching != 0) near |= 1ull << (c.boost_pad_touching - 1);
            for (; near != 0u; near &= near - 1u) {
                const int p = ctz64(near);
                pad_touch_step(pads[p], p, c, static_cast<uint32_t>(car_base + i + 1), ((hits >> p) & 1u) != 0u,
                               ((overlap >> p) & 1u) != 0u, eligible);
            }
        }
        if (c.is_demoed) {
            pad_store_frame_pos(c, tc);
        } else {
            c.pad_frame_pos_bt = frame_pos_bt;
            c.pad_frame_pos_valid = 1;
        }
    }
    // respawns (reference BoostPadRespawnStep, :2528-2553)
    for (int p = 0; p < L.count; ++p) {
        PadState& pad = pads[p];
        if (pad.is_active || !pad_respawn_due(pad, tc.tick_dt, tc.frame_frac)) continue;
        pad.cooldown = 0.0f;
        pad.is_active = 1;
        for (int k = count - 1; k >= 0; --k) {
            CarState& c = cars[order[k]];
            if (c.is_demoed) continue;
            const V3 car_uu = pad_frame_pos(c, tc.frame_frac);
            V3 axes[3];
            pad_frame_axes(c, tc, axes);
            if (pad_box_overlap(L.pos[p], pad.is_big != 0, car_uu, axes, cfgs[order[k]]))
                c.boost_pad_touching = static_cast<uint8_t>(p + 1);
        }
    }
    // the touch list (reference BoostPadTouchListStep, :2555-2561)
    for (int k = count - 1; k >= 0; --k) {
        const int i = order[k];
        CarState& c = cars[i];
        if (c.boost_pad_touching != 0) {
            const int p = c.boost_pad_touching - 1;
            PadState& pad = pads[p];
            if (pad.is_active && pad.cur_locked_car_id == 0 && pad_eligible(c, tc)) {
                pad.cur_locked_car_id = static_cast<uint32_t>(car_base + i + 1);
                const int whole = x86_f2i(c.boost);
                c.rlbotv5_boost_hold = static_cast<uint8_t>(
                    (254 < whole + (static_cast<float>(whole) < c.boost ? 1 : 0)
                         ? 254
                         : whole + (static_cast<float>(whole) < c.boost ? 1 : 0)) +
                    1);
            }
        }
    }
    // post tick: a pad locked by a car gives its boost
    if (count > 0) {
        for (int p = 0; p < L.count; ++p) {
            PadState& pad = pads[p];
            const uint32_t locked = pad.cur_locked_car_id;
            if ((locked | pad.prev_locked_car_id) == 0u) continue;
            if (locked != 0 && pad.is_active) pad_give(cars, car_base, max_cars, pad, p, locked, tc);
            pad.prev_locked_car_id = locked;
        }
    }
}

}  // namespace rg

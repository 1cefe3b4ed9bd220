// A car body's contacts with the arena mesh, host+device: triangle queries, box-triangle GJK/EPA, the per-car
// candidate list and its retained manifold, and the contact rows it feeds the solver.
//
// Reference: AppendCarWorldMeshContactRowsBody (include/rocketgpu/detail/step/car_world_contacts.hpp:1270-2146) on the
// path a custom single-mesh soccar layout takes (the car/mesh manifold listed in the broadphase, no staged or replayed
// candidates); CarWorldTriangleQueryTest (:1014-1062) with its gap tests (:982-1012); ComputeCarWorldTriangleHit
// (:652-695); the Bullet-style replacement rule (:805-860); the retained manifold merge (:1740-1830); emit_candidates
// (:1478-1599); the row builders InitializeCarWorldSplitContactRow / InitializeCarWorldVelocityContactRow /
// InitializeCarWorldFrictionContactRow (arena_geometry.hpp:2404-2530, 2767-2815); the car's predictive (CCD) rows
// (AppendPredictiveContactRows, env_step.hpp:4206-4255).
#pragma once

#include "rg_ball_world.cuh"
#include "rg_car.cuh"
#include "rg_gjk.cuh"

namespace rg {

// One retained contact point of a car's mesh manifold (Bullet units; reference CarWorldMeshRetainedPoint).
struct CarMeshPoint {
    V3 local_a, local_b, normal;
    float distance;
};
// Persistent per car slot: the car/mesh manifold (reference CarWorldMeshRetainedManifold; one arena mesh, one slot).
struct alignas(16) CarWorldScratch {
    CarMeshPoint pts[4];
    int32_t count;
    int32_t pad[3];
};

// ---- the car's box ------------------------------------------------------------------------------------------------
// reference BulletHitboxSize (math.hpp:1554-1560)
RG_HDI V3 bullet_hitbox_size(const CarConfig& cfg) {
    const V3 sized = cfg.hitbox_published + V3{2.5f, 2.5f, 2.5f};
    const bool has =
        sized.x == cfg.hitbox_size.x && sized.y == cfg.hitbox_size.y && sized.z == cfg.hitbox_size.z;
    const V3 published = has ? cfg.hitbox_published : cfg.hitbox_size - V3{2.5f, 2.5f, 2.5f};
    const V3 half_bt = (published * 0.02f) * 0.5f + V3{0.025f, 0.025f, 0.025f};
    return (half_bt * 50.0f) * 2.0f;
}
// reference BulletBoxHalfExtentWithMarginBt (host_validation_and_contact_debug.hpp:43-54)
RG_HDI V3 car_box_half_bt(const CarConfig& cfg) {
    const V3 half = (bullet_hitbox_size(cfg) * (1.0f / 50.0f)) / 2.0f;
    const float mn = fmin_(half.x, fmin_(half.y, half.z));
    const float safe = 0.1f * mn;
    const float m = safe < 0.04f ? safe : 0.04f;
    return half - V3{m, m, m} + V3{m, m, m};
}
// reference CarContactBreakingThresholdBt (arena_geometry.hpp:6787-6798)
RG_HDI float car_contact_threshold_bt(const CarConfig& cfg) {
    const V3 half = (bullet_hitbox_size(cfg) * 0.02f) * 0.5f;
    const float m = fmin_(0.1f * fmin_(fmin_(half.x, half.y), half.z), 0.04f);
    const V3 mv{m, m, m};
    const V3 hm = (half - mv) + mv;
    const V3 c = cfg.hitbox_offset * 0.02f;
    const V3 lo = c - hm, hi = c + hm;
    const V3 sc = (lo + hi) * 0.5f;
    const float r = len(hi - lo) * 0.5f;
    return (r + len(sc)) * 0.02f;
}
// Body-space <-> world points through the car's basis (reference CarBodyLocalPointBt / CarBodyWorldPointBt,
// triangle_and_carcar.hpp:172-202).
RG_HD V3 car_local_point(V3 f, V3 r, V3 u, V3 pos, V3 p) {
    const V3 d = p - pos;
    return V3{f.x * d.x + f.y * d.y + f.z * d.z, r.x * d.x + r.y * d.y + r.z * d.z, u.x * d.x + u.y * d.y + u.z * d.z};
}
RG_HD V3 car_world_point(V3 f, V3 r, V3 u, V3 pos, V3 l) {
    return V3{(l.x * f.x + l.y * r.x + l.z * u.x) + pos.x, (l.x * f.y + l.y * r.y + l.z * u.y) + pos.y,
              (l.x * f.z + l.y * r.z + l.z * u.z) + pos.z};
}

// The car box's world frame for mesh queries (reference ComputeCarWorldMeshQueryFrame, car_world_contacts.hpp:869-905).
struct CarQueryFrame {
    V3 ax, ay, az;
    V3 center, half, extent, lo, hi;
};
RG_HDI CarQueryFrame car_query_frame(const CarState& c, const CarConfig& cfg) {
    CarQueryFrame f;
    car_basis(c, f.ax, f.ay, f.az);
    const V3 r0{f.ax.x, f.ay.x, f.az.x}, r1{f.ax.y, f.ay.y, f.az.y}, r2{f.ax.z, f.ay.z, f.az.z};
    const V3 p = cfg.hitbox_offset * (1.0f / 50.0f);
    f.center = V3{dot(p, r0) + c.pos_bt.x, dot(p, r1) + c.pos_bt.y, dot(p, r2) + c.pos_bt.z};
    const V3 h = car_box_half_bt(cfg);
    f.half = h;
    f.extent = V3{fabs_(f.ax.x) * h.x + fabs_(f.ay.x) * h.y + fabs_(f.az.x) * h.z,
                  fabs_(f.ax.y) * h.x + fabs_(f.ay.y) * h.y + fabs_(f.az.y) * h.z,
                  fabs_(f.ax.z) * h.x + fabs_(f.ay.z) * h.y + fabs_(f.az.z) * h.z};
    f.lo = f.center - f.extent;
    f.hi = f.center + f.extent;
    return f;
}

// 0: the triangle's bounds miss the box's AABB; 1: the broadphase pairs them but a separating axis (triangle normal,
// box axis or edge x axis) keeps them apart by more than the threshold; 2: run the narrowphase
// (reference CarWorldTriangleQueryTest, car_world_contacts.hpp:982-1062).
RG_HDI int car_triangle_query(const DevTri& t, const CarQueryFrame& f, float thr) {
    if (fmin_(fmin_(t.a.z, t.b.z), t.c.z) > f.hi.z || fmax_(fmax_(t.a.z, t.b.z), t.c.z) < f.lo.z ||
        fmin_(fmin_(t.a.x, t.b.x), t.c.x) > f.hi.x || fmax_(fmax_(t.a.x, t.b.x), t.c.x) < f.lo.x ||
        fmin_(fmin_(t.a.y, t.b.y), t.c.y) > f.hi.y || fmax_(fmax_(t.a.y, t.b.y), t.c.y) < f.lo.y)
        return 0;
    const V3 n = normalize_fallback(t.normal, V3{0.0f, 0.0f, 1.0f});
    const float cp = dot(n, f.center);
    const float se = fabs_(dot(n, f.ax)) * f.half.x + fabs_(dot(n, f.ay)) * f.half.y + fabs_(dot(n, f.az)) * f.half.z;
    const float tp = dot(n, t.a);
    if (tp - (cp + se) > thr || (cp - se) - tp > thr) return 1;
    const float reject = thr + 1.0e-3f;
    auto axis_gap = [&](V3 axis, float h) {
        const float c = dot(axis, f.center);
        const float pa = dot(axis, t.a), pb = dot(axis, t.b), pc = dot(axis, t.c);
        return fmax_(fmin_(pa, fmin_(pb, pc)) - (c + h), (c - h) - fmax_(pa, fmax_(pb, pc)));
    };
    if (axis_gap(f.ax, f.half.x) > reject || axis_gap(f.ay, f.half.y) > reject || axis_gap(f.az, f.half.z) > reject)
        return 1;
    const V3 e[3] = {t.b - t.a, t.c - t.b, t.a - t.c};
    const V3 ax[3] = {f.ax, f.ay, f.az};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            const V3 u = cross(e[i], ax[j]);
            const float l = sqrtf(dot(u, u));
            if (!(l > 1e-6f)) continue;
            const float c = dot(u, f.center);
            const float r = fabs_(dot(u, f.ax)) * f.half.x + fabs_(dot(u, f.ay)) * f.half.y +
                            fabs_(dot(u, f.az)) * f.half.z;
            const float pa = dot(u, t.a), pb = dot(u, t.b), pc = dot(u, t.c);
            if (fmax_(fmin_(pa, fmin_(pb, pc)) - (c + r), (c - r) - fmax_(pa, fmax_(pb, pc))) > reject * l) return 1;
        }
    }
    return 2;
}

// Narrowphase of the box against one triangle: GJK/EPA distance and the point on the triangle, then the triangle's
// face normal corrected at internal edges (reference ComputeCarWorldTriangleHit).
struct CarTriHit {
    V3 normal, raw_normal, point_b, raw_point_b;
    float distance;
    bool hit;
};
RG_HDI CarTriHit car_triangle_hit(V3 f, V3 r, V3 u, V3 pos_bt, const CarConfig& cfg, const DevTri& t, float thr) {
    CarTriHit out;
    out.hit = false;
    float distance = 0.0f;
    V3 point_b{0.0f, 0.0f, 0.0f};
    const V3 raw_half = (bullet_hitbox_size(cfg) * 0.5f) * (1.0f / 50.0f);
    if (!gjk::box_triangle_contact(f, r, u, pos_bt, cfg.hitbox_offset * (1.0f / 50.0f), raw_half, t.a, t.b, t.c,
                                   distance, point_b) ||
        distance > thr)
        return out;
    const V3 e1 = t.b - t.a, e2 = t.c - t.a;
    const V3 n{e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
    const float inv = 1.0f / sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
    V3 normal{n.x * inv, n.y * inv, n.z * inv};
    out.raw_normal = normal;
    out.raw_point_b = point_b;
    const V3 point_a = point_b + normal * distance;
    adjust_internal_edge(t, point_a, distance, point_b, normal);
    out.normal = normal;
    out.point_b = point_b;
    out.distance = distance;
    out.hit = true;
    return out;
}

// A contact candidate of the car's mesh manifold for this tick (reference MeshContactCandidate).
struct MeshCandidate {
    V3 normal, raw_normal, local_a, point_b, rel_bt;
    float distance, add_distance;
    int32_t seed;  // -1 for a new contact, else the retained point it continues
};

// Bullet's replacement rule for a full 4-point cache: keep the deepest point, maximise the area
// (reference SelectCarWorldMeshContactReplaceIndexBulletStyle, car_world_contacts.hpp:805-860).
RG_HDI int mesh_replace_index(const MeshCandidate* c, const MeshCandidate& p) {
    int max_i = -1;
    float max_pen = p.add_distance;
    for (int i = 0; i < 4; ++i) {
        if (c[i].add_distance < max_pen) {
            max_i = i;
            max_pen = c[i].add_distance;
        }
    }
    float r0 = 0.0f, r1 = 0.0f, r2 = 0.0f, r3 = 0.0f;
    if (max_i != 0) r0 = len2(cross(p.local_a - c[1].local_a, c[3].local_a - c[2].local_a));
    if (max_i != 1) r1 = len2(cross(p.local_a - c[0].local_a, c[3].local_a - c[2].local_a));
    if (max_i != 2) r2 = len2(cross(p.local_a - c[0].local_a, c[3].local_a - c[1].local_a));
    if (max_i != 3) r3 = len2(cross(p.local_a - c[0].local_a, c[2].local_a - c[1].local_a));
    int best = 0;
    float v = r0;
    if (r1 > v) {
        best = 1;
        v = r1;
    }
    if (r2 > v) {
        best = 2;
        v = r2;
    }
    if (r3 > v) best = 3;
    return best;
}

// ---- contact rows (Bullet units, as the solver runs them) -------------------------------------------------------
struct CarVelRow {
    V3 normal, rel_cross, ang;
    float inv_mass, jac, rhs, applied;
    int32_t body, tag;
};
struct CarFricRow {
    V3 tangent, rel_cross, ang;
    float inv_mass, jac, rhs, applied, friction;
    int32_t body, normal_row;
};
struct CarSplitRow {
    V3 normal, rel_cross, ang;
    float inv_mass, jac, rhs, applied;
    int32_t body, tag;
};
constexpr int kMaxCarWorldRows = 5 * 8;  // per car: up to 4 mesh contacts and 1 predictive contact
// Car/world contact rows with room for N of each kind: an arena's rows (N = kMaxCarWorldRows, slot order), or one
// car's mesh rows staged by the per-car kernel (N = kCarStageRows: the retained manifold holds at most 4 points).
template <int N>
struct CarWorldRowsN {
    static constexpr int kCap = N;
    CarVelRow vel[N];
    CarFricRow fric[N];
    CarSplitRow split[N];
    int nv, nf, ns;
};
using CarWorldRows = CarWorldRowsN<kMaxCarWorldRows>;
constexpr int kCarStageRows = 4;
using CarStageRows = CarWorldRowsN<kCarStageRows>;

// Appends one car's staged rows to the arena's rows; its friction rows' normal-row indices move with its normal rows.
// The arena's rows never fill up (at most 6 cars x 4 mesh contacts + 6 predictive contacts < kMaxCarWorldRows), so
// appending builds exactly the rows the car's query would have appended in place.
RG_HDI void append_car_rows(CarWorldRows& dst, const CarStageRows& src) {
    const int base = dst.nv;
    for (int k = 0; k < src.nv; ++k) dst.vel[dst.nv++] = src.vel[k];
    for (int k = 0; k < src.nf; ++k) {
        CarFricRow r = src.fric[k];
        r.normal_row += base;
        dst.fric[dst.nf++] = r;
    }
    for (int k = 0; k < src.ns; ++k) dst.split[dst.ns++] = src.split[k];
}

// The car's inverse inertia in uu (reference MakeCarInvInertiaRowsUu, host_validation_and_contact_debug.hpp:86-129),
// used by the row builders' validity checks.
RG_HDI void car_inv_inertia_uu(const CarState& c, const CarConfig& cfg, float mass, V3& o0, V3& o1, V3& o2) {
    if (c.restored_inv_inertia_valid) {
        o0 = c.restored_inv_inertia_bt[0] * 0.0004f;
        o1 = c.restored_inv_inertia_bt[1] * 0.0004f;
        o2 = c.restored_inv_inertia_bt[2] * 0.0004f;
        return;
    }
    const V3 h = car_box_half_bt(cfg) * 50.0f;
    const float x = h.x * 2.0f, y = h.y * 2.0f, z = h.z * 2.0f;
    const float x2 = x * x, y2 = y * y, z2 = z * z;
    const float s = mass / 12.0f;
    const V3 in{s * (y2 + z2), s * (x2 + z2), s * (x2 + y2)};
    const V3 il{in.x != 0.0f ? 1.0f / in.x : 0.0f, in.y != 0.0f ? 1.0f / in.y : 0.0f,
                in.z != 0.0f ? 1.0f / in.z : 0.0f};
    inv_inertia_world_from_columns(c.tick_start_basis_forward, c.tick_start_basis_right, c.tick_start_basis_up, il, o0,
                                   o1, o2);
}
RG_HD V3 mul_rows(V3 r0, V3 r1, V3 r2, V3 v) { return V3{dot(r0, v), dot(r1, v), dot(r2, v)}; }

// Builds one contact's split, normal and friction rows (reference InitializeCarWorld*ContactRow with the Bullet-unit
// overrides the mesh and predictive callers pass). `ang_bt` / `tang_ang_bt`: inverse world inertia times (r x n) and
// (r x t); `split_ang_uu`: the uu-inertia term of the split row's validity check. Returns whether a normal row was
// made.
template <class Rows>
RG_HDI bool car_contact_rows(Rows& rows, int body, int tag, const CarState& c, V3 normal, V3 rel_bt,
                             float distance_bt, V3 ang_bt, V3 tang_ang_bt, V3 tangent, V3 split_ang_uu,
                             float inv_mass, float restitution, float friction, float dt) {
    const float pen_uu = fmax_(0.0f, -distance_bt) * 50.0f;
    // split (position) row
    if (!(pen_uu <= 0.0f || dt <= 0.0f) && rows.ns < Rows::kCap) {
        const V3 rel_uu = rel_bt * 50.0f;
        const float denom = inv_mass + dot(normal, cross(split_ang_uu, rel_uu));
        if (denom > 1e-8f) {
            const float jac_uu = 1.0f / denom;
            const float denom_bt = inv_mass + dot(normal, cross(ang_bt, rel_bt));
            const float jac = denom_bt > 1e-8f ? 1.0f / denom_bt : jac_uu;
            CarSplitRow& s = rows.split[rows.ns++];
            s.normal = normal;
            s.rel_cross = cross(rel_bt, normal);
            s.ang = ang_bt;
            s.inv_mass = inv_mass;
            s.jac = jac;
            const float pen_bt = -distance_bt;
            s.rhs = ((pen_bt * 0.8f) / dt) * jac;
            s.applied = 0.0f;
            s.body = body;
            s.tag = tag;
        }
    }
    // normal row
    if (rows.nv >= Rows::kCap) return false;
    const V3 rel_uu = rel_bt * 50.0f;
    const V3 ang_uu = ang_bt * (1.0f / 50.0f);
    const float denom = inv_mass + dot(normal, cross(ang_uu, rel_uu));
    if (denom <= 1e-8f) return false;
    float jac = 1.0f / denom;
    const float bt_denom = inv_mass + dot(normal, cross(ang_bt, rel_bt));
    if (bt_denom > 1e-8f) jac = 1.0f / bt_denom;
    const V3 rel_cross = cross(rel_bt, normal);
    const V3 vel_bt = c.vel_bt;
    const V3 ang_vel = c.ang_vel;
    const float rv_rest = dot(normal, vel_bt + cross(ang_vel, rel_bt));
    const float rv = dot(normal, vel_bt + c.ext_force_impulse_bt) + dot(rel_cross, ang_vel + c.ext_torque_impulse);
    const float rest = fmax_(restitution * -rv_rest, 0.0f);
    const int vi = rows.nv++;
    CarVelRow& v = rows.vel[vi];
    v.normal = normal;
    v.rel_cross = rel_cross;
    v.ang = ang_bt;
    v.inv_mass = inv_mass;
    v.jac = jac;
    v.rhs = (rest - rv) * jac;
    v.applied = 0.0f;
    v.body = body;
    v.tag = tag;
    // friction row
    if (!(friction <= 0.0f) && rows.nf < Rows::kCap) {
        const V3 tang_ang_uu = tang_ang_bt * (1.0f / 50.0f);
        const float fden = inv_mass + dot(tangent, cross(tang_ang_uu, rel_uu));
        if (fden > 1e-8f) {
            float fjac = 1.0f / fden;
            const float fbt = inv_mass + dot(tangent, cross(tang_ang_bt, rel_bt));
            if (fbt > 1e-8f) fjac = 1.0f / fbt;
            CarFricRow& fr = rows.fric[rows.nf++];
            fr.tangent = tangent;
            fr.rel_cross = cross(rel_bt, tangent);
            fr.ang = tang_ang_bt;
            fr.inv_mass = inv_mass;
            fr.jac = fjac;
            const float v1 = dot(tangent, vel_bt + c.ext_force_impulse_bt) + dot(fr.rel_cross, ang_vel);
            const float relv = v1 + 0.0f;
            fr.rhs = (0.0f - relv) * fjac;
            fr.applied = 0.0f;
            fr.friction = friction;
            fr.body = body;
            fr.normal_row = vi;
        }
    }
    return true;
}

// The sliding direction of a contact: the lateral part of the body's velocity (with this tick's external impulses)
// at the contact, else Bullet's first plane-space axis (reference emit_candidates, car_world_contacts.hpp:1547-1556).
RG_HDI V3 contact_tangent(V3 normal, V3 vel_nd_bt) {
    const float rn = dot(normal, vel_nd_bt);
    const V3 lat = vel_nd_bt - normal * rn;
    const float l2 = len2(lat);
    if (l2 > 1.1920928955078125e-7f) return lat * (1.0f / sqrtf(l2));
    constexpr float kSqrt12 = 0.7071067811865475244008443621048490f;
    if (fabs_(normal.z) > kSqrt12) {
        const float a = normal.y * normal.y + normal.z * normal.z;
        const float k = 1.0f / sqrtf(a);
        return V3{0.0f, -normal.z * k, normal.y * k};
    }
    const float a = normal.x * normal.x + normal.y * normal.y;
    const float k = 1.0f / sqrtf(a);
    return V3{-normal.y * k, normal.x * k, 0.0f};
}

// What a car's arena contacts leave for the car's world-contact record (reference ContactAccumulator).
struct CarWorldContactResult {
    bool hit;
    V3 latest_normal;
};
// The query's car-world events: one per manifold point made into rows, with the point's normal (reference
// ContactAccumulator::add and its event, arena_geometry.hpp:21-46, arena_ball.hpp:563-573); the arena emits them where
// the reference's query runs, with the car's position, velocity and ground flag at that moment.
struct MeshContactEvents {
    uint32_t count;
    V3 normal[4];
};

// The car's contacts with the arena mesh for this tick: refresh the retained manifold, collect candidates from the
// triangles the box overlaps, merge them into the manifold and emit rows (body index `body`, source tag 100).
// `listed`: the car/mesh manifold exists in the broadphase list.
// The car does not change here: a hit (res.hit) is recorded by the caller (car_record_world_surface(c, true), once
// for the points the reference records one by one: the record is idempotent), at the place in the tick where the
// reference's query runs.
template <class Rows>
RG_NOINL CarWorldContactResult car_mesh_contacts(const CarState& c, const CarConfig& cfg, CarWorldScratch& ws,
                                               bool listed, const MeshDevice& mesh, const TickConfig& tc, int body,
                                               Rows& rows, MeshContactEvents* events = nullptr) {
    CarWorldContactResult res;
    res.hit = false;
    res.latest_normal = V3{0.0f, 0.0f, 1.0f};
    if (events) events->count = 0;
    if (!listed) {
        ws.count = 0;
        return res;
    }
    const float thr = car_contact_threshold_bt(cfg);
    V3 f, r, u;
    car_basis(c, f, r, u);
    const V3 pos = c.pos_bt;
    MeshCandidate cand[4];
    int n = 0;
    CarMeshPoint seeds[4];
    // retained points: distances refreshed at the current pose; points that drifted away leave
    auto refresh = [&]() {
        V3 wa[4], wb[4];
        for (int i = 0; i < ws.count; ++i) {
            wa[i] = car_world_point(f, r, u, pos, ws.pts[i].local_a);
            wb[i] = ws.pts[i].local_b;
            ws.pts[i].distance = dot(wa[i] - wb[i], ws.pts[i].normal);
        }
        for (int i = ws.count - 1; i >= 0; --i) {
            const CarMeshPoint& p = ws.pts[i];
            const V3 pd = wb[i] - (wa[i] - p.normal * p.distance);
            if (p.distance > thr || dot(pd, pd) > thr * thr) {
                const int last = ws.count - 1;
                if (i != last) {
                    ws.pts[i] = ws.pts[last];
                    wa[i] = wa[last];
                    wb[i] = wb[last];
                }
                ws.count = last;
            }
        }
    };
    bool seeded = false;
    if (ws.count > 0) {
        refresh();
        for (int k = 0; k < ws.count; ++k) {
            const CarMeshPoint& p = ws.pts[k];
            const V3 pwa = car_world_point(f, r, u, pos, p.local_a);
            MeshCandidate& m = cand[k];
            m.normal = p.normal;
            m.raw_normal = V3{0.0f, 0.0f, 1.0f};
            m.local_a = p.local_a;
            m.point_b = p.local_b;
            m.rel_bt = pwa - pos;
            m.distance = p.distance;
            m.add_distance = p.distance;
            m.seed = k;
            seeds[k] = p;
        }
        n = ws.count;
        seeded = true;
    }
    V3 last_normal{0.0f, 0.0f, 1.0f};
    const CarQueryFrame qf = car_query_frame(c, cfg);
    mesh_query_box(mesh, qf.lo, qf.hi, [&](const DevTri& t) {
        if (car_triangle_query(t, qf, thr) != 2) return;
        const CarTriHit h = car_triangle_hit(f, r, u, pos, cfg, t, thr);
        if (!h.hit || h.distance > thr) return;
        MeshCandidate m;
        m.normal = h.normal;
        m.raw_normal = h.raw_normal;
        m.add_distance = h.distance;
        const V3 manifold_a = h.raw_point_b + h.raw_normal * h.distance;
        m.local_a = car_local_point(f, r, u, pos, manifold_a);
        m.point_b = h.point_b;
        const V3 ra = car_world_point(f, r, u, pos, m.local_a);
        m.distance = dot(ra - m.point_b, m.normal);
        m.rel_bt = ra - pos;
        m.seed = -1;
        int merge = -1;
        float shortest = thr * thr;
        for (int i = 0; i < n; ++i) {
            const V3 d = cand[i].local_a - m.local_a;
            const float dd = dot(d, d);
            if (dd < shortest) {
                shortest = dd;
                merge = i;
            }
        }
        last_normal = h.raw_normal;
        if (m.distance > thr) {
            if (merge >= 0) {
                for (int i = merge; i + 1 < n; ++i) cand[i] = cand[i + 1];
                --n;
            }
            return;
        }
        if (merge >= 0) {
            cand[merge] = m;
            return;
        }
        if (n < 4) {
            cand[n++] = m;
            return;
        }
        cand[mesh_replace_index(cand, m)] = m;
    });
    // the manifold keeps this tick's candidates (seeded points carry over unchanged)
    if (seeded) {
        refresh();
        ws.count = 0;
    } else if (n == 0) {
        return res;
    }
    for (int k = 0; k < n; ++k) {
        if (seeded && cand[k].seed >= 0) {
            ws.pts[ws.count++] = seeds[cand[k].seed];
            continue;
        }
        CarMeshPoint p;
        p.local_a = cand[k].local_a;
        p.local_b = cand[k].point_b;
        p.normal = cand[k].normal;
        p.distance = dot(car_world_point(f, r, u, pos, p.local_a) - p.local_b, p.normal);
        ws.pts[ws.count++] = p;
    }
    n = ws.count;
    if (n <= 0) return res;
    // rows (reference emit_candidates)
    V3 i0, i1, i2, u0, u1, u2;
    car_inv_inertia_world_bt(c, cfg, tc.car_mass, i0, i1, i2);
    car_inv_inertia_uu(c, cfg, tc.car_mass, u0, u1, u2);
    const float inv_mass = 1.0f / tc.car_mass;
    const V3 vel_ext = c.vel_bt + c.ext_force_impulse_bt;
    const V3 ang_ext = c.ang_vel + c.ext_torque_impulse;
    V3 normal_sum{0.0f, 0.0f, 0.0f};
    bool any_row = false;
    for (int k = 0; k < n && k < 4; ++k) {
        const CarMeshPoint& p = ws.pts[k];
        const V3 pwa = car_world_point(f, r, u, pos, p.local_a);
        const V3 rel_bt = pwa - pos;
        res.hit = true;
        if (events) events->normal[events->count++] = p.normal;
        const V3 ang_bt = mul_rows(i0, i1, i2, cross(rel_bt, p.normal));
        const float pen_uu = fmax_(0.0f, -p.distance) * 50.0f;
        V3 split_ang_uu{0.0f, 0.0f, 0.0f};
        if (!(pen_uu <= 0.0f || tc.tick_dt <= 0.0f)) split_ang_uu = mul_rows(u0, u1, u2, cross(rel_bt * 50.0f, p.normal));
        const V3 tangent = contact_tangent(p.normal, vel_ext + cross(ang_ext, rel_bt));
        const V3 tang_ang_bt = mul_rows(i0, i1, i2, cross(rel_bt, tangent));
        if (car_contact_rows(rows, body, 100, c, p.normal, rel_bt, p.distance, ang_bt, tang_ang_bt, tangent,
                             split_ang_uu, inv_mass, tc.arena_restitution, tc.arena_friction, tc.tick_dt)) {
            normal_sum += p.normal;
            any_row = true;
        }
    }
    res.latest_normal = last_normal;
    // the game's contact normal: the sum of the normal rows' normals, normalized (reference
    // ApplyGameCarWorldContactNormal, arena_ball.hpp:95-166, with every row on the one mesh tag)
    if (any_row) {
        const float l2 = dot(normal_sum, normal_sum);
        if (l2 >= 1e-8f) {
            const V3 nn = normal_sum * (1.0f / sqrtf(l2));
            res.latest_normal = V3{0.0f + nn.x, 0.0f + nn.y, 0.0f + nn.z};
        }
    }
    return res;
}

}  // namespace rg

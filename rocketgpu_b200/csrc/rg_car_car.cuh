// Contacts between two cars of an arena: the box/box separating-axis test with the game's contact points, the
// retained 4-point manifold of each car pair, the pair's two-body contact rows for the unified solves, and the game's
// bump and demolition rules with the demolition's time-of-impact pose.
//
// Reference (the path WorldStepSoccar takes for car pairs, env_step.hpp:4916-5042, ResolveCarCarCollisionImpl with
// shared rows, env_step.hpp:736-851):
//   CarCarCcmGateMasks (env_step.hpp:139-203), PrepareSharedCarCarCollisionContacts (:207-380),
//   EmitSharedCarCarContactRows (:382-706), retained-manifold refresh / insert (:43-131);
//   ComputeObbContact / ComputeObbContactGameOrder (triangle_and_carcar.hpp:2221-2388), the face clip and edge/edge
//   anchors (:1806-2202), ComputeApproxCarCarContactAnchorPairsWithBtObb (:3093-3226);
//   ResolveCarCarDirectionalContact / BumpCone / RecordCarHit (:2790-3091), ShouldDemolish / InForwardConePose
//   (:2757-2788), CarCarTimeOfImpact and its GJK closest points (:2400-2755); DemolishCar (arena_ball.hpp:3087-3090).
// The pair contact cache of the reference is cleared at every world step's start and only ever written afterwards,
// so no row starts warm: it is not kept here.
#pragma once

#include "rg_ball_car.cuh"
#include "rg_car_world.cuh"
#include "rg_gjk.cuh"

namespace rg {

// ---- retained manifold --------------------------------------------------------------------------------------------
struct CarCarPoint {
    V3 local_a, local_b, pos_a, pos_b, normal;
    float distance;
};
struct CarCarManifold {
    int32_t count;
    CarCarPoint p[4];
};
RG_HD int car_pair_slot(int lo, int hi) { return hi * (hi - 1) / 2 + lo; }

RG_HDI void car_car_refresh(CarCarManifold& m, const CarState& a, const CarState& b, float thr) {
    const int count = m.count;
    if (count <= 0) return;
    V3 fa, ra, ua, fb, rb, ub;
    car_basis(a, fa, ra, ua);
    car_basis(b, fb, rb, ub);
    for (int i = 0; i < count; ++i) {
        CarCarPoint& p = m.p[i];
        p.pos_a = car_world_point(fa, ra, ua, a.pos_bt, p.local_a);
        p.pos_b = car_world_point(fb, rb, ub, b.pos_bt, p.local_b);
        p.distance = dot(p.pos_b - p.pos_a, p.normal);
    }
    const float thr_sq = thr * thr;
    int kept = count;
    for (int i = count - 1; i >= 0; --i) {
        const CarCarPoint p = m.p[i];
        bool remove = p.distance > thr;
        if (!remove) {
            const V3 projected = p.pos_b - p.normal * p.distance;
            const V3 diff = p.pos_a - projected;
            remove = dot(diff, diff) > thr_sq;
        }
        if (remove) {
            m.p[i] = m.p[kept - 1];
            --kept;
        }
    }
    m.count = kept;
}

RG_HD float car_car_res(V3 l, V3 p1, V3 p2, V3 p3) {
    const V3 c = cross(l - p1, p2 - p3);
    return dot(c, c);
}

RG_HDI void car_car_add(CarCarManifold& m, const CarCarPoint& pt, float thr) {
    const int count = m.count;
    float shortest = thr * thr;
    int nearest = -1;
    for (int i = 0; i < count; ++i) {
        const V3 d = m.p[i].local_b - pt.local_b;
        const float d2 = dot(d, d);
        if (d2 < shortest) {
            shortest = d2;
            nearest = i;
        }
    }
    if (nearest >= 0) {
        m.p[nearest] = pt;
        return;
    }
    if (count < 4) {
        m.p[count] = pt;
        m.count = count + 1;
        return;
    }
    int max_pen_idx = 4;
    float max_pen = pt.distance;
    for (int i = 0; i < 4; ++i) {
        if (m.p[i].distance < max_pen) {
            max_pen_idx = i;
            max_pen = m.p[i].distance;
        }
    }
    const V3 l = pt.local_b, p0 = m.p[0].local_b, p1 = m.p[1].local_b, p2 = m.p[2].local_b, p3 = m.p[3].local_b;
    const float r0 = max_pen_idx == 0 ? 0.0f : car_car_res(l, p1, p3, p2);
    const float r1 = max_pen_idx == 1 ? 0.0f : car_car_res(l, p0, p3, p2);
    const float r2 = max_pen_idx == 2 ? 0.0f : car_car_res(l, p0, p3, p1);
    const float r3 = max_pen_idx == 3 ? 0.0f : car_car_res(l, p0, p2, p1);
    int biggest = 0;
    float max_area = r0;
    if (r1 > max_area) {
        biggest = 1;
        max_area = r1;
    }
    if (r2 > max_area) {
        biggest = 2;
        max_area = r2;
    }
    if (r3 > max_area) biggest = 3;
    m.p[biggest] = pt;
}

// Pairs whose retained manifold is empty and whose cars are apart (bounding spheres) or inactive skip the pair test
// this tick: bit car_pair_slot(lo, hi) of the result.
RG_HD float car_bounding_sphere_radius(const CarConfig& cfg) {
    const V3 e = cfg.hitbox_size * 0.5f;
    return len(e) + len(cfg.hitbox_offset) + 5.0f;
}
RG_HDI uint32_t car_car_reject_mask(const CarState* cars, const CarConfig* cfgs, const CarCarManifold* mans,
                                    int count) {
    if (count < 2) return 0u;
    const int n = count < 8 ? count : 8;
    uint32_t live = 0u, reject = 0u;
    for (int k = 0; k < n; ++k)
        live |= static_cast<uint32_t>((cars[k].is_demoed == 0) & (cars[k].just_respawned == 0)) << k;
    for (int hi = 1; hi < n; ++hi) {
        for (int lo = 0; lo < hi; ++lo) {
            const int slot = car_pair_slot(lo, hi);
            const uint32_t pair_live = (live >> lo) & (live >> hi) & 1u;
            const uint32_t empty = mans[slot].count == 0 ? 1u : 0u;
            const float md = car_bounding_sphere_radius(cfgs[hi]) + car_bounding_sphere_radius(cfgs[lo]);
            const uint32_t beyond = !(len2(cars[lo].pos - cars[hi].pos) < md * md) ? 1u : 0u;
            reject |= (empty & (beyond | (pair_live ^ 1u))) << slot;
        }
    }
    return reject;
}

// ---- oriented boxes -----------------------------------------------------------------------------------------------
struct Obb {
    V3 center, axis[3], half;
};
constexpr uint8_t kObbFaceA = 0, kObbFaceB = 1, kObbEdgeEdge = 2;
struct ObbFeature {
    uint8_t kind, axis_a, axis_b;
};
RG_HD float comp3(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// the car's hitbox in Bullet units (reference MakeCarObbBulletTransformBt)
RG_HDI Obb make_car_obb_bt(const CarState& c, const CarConfig& cfg) {
    Obb o;
    car_basis(c, o.axis[0], o.axis[1], o.axis[2]);
    o.center = c.pos_bt + rotate_via_basis(o.axis[0], o.axis[1], o.axis[2], cfg.hitbox_offset * (1.0f / 50.0f));
    o.half = car_box_half_bt(cfg);
    return o;
}

// Separating-axis test of two boxes with the game's axis choice (reference ComputeObbContact): the axis of least
// penetration among the 6 face normals and 9 edge crosses (edge axes favoured by 5 %), pointing from a to b.
RG_HDI bool obb_contact(const Obb& a, const Obb& b, float threshold, V3& out_normal, float& out_overlap,
                        ObbFeature& out_feature) {
    constexpr float kEps = 1e-5f;
    float R[3][3], AbsR[3][3], AbsRF[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            R[i][j] = dot(a.axis[i], b.axis[j]);
            AbsRF[i][j] = fabs_(R[i][j]);
            AbsR[i][j] = AbsRF[i][j] + kEps;
        }
    const V3 tw = b.center - a.center;
    const float t[3] = {dot(tw, a.axis[0]), dot(tw, a.axis[1]), dot(tw, a.axis[2])};
    constexpr float kEdgeFudge = 1.05f;
    constexpr float kEdgeSepEps = 1.1920929e-7f;
    bool have = false;
    float best_s2 = -1.0e30f;
    V3 best_axis{1.0f, 0.0f, 0.0f};
    bool best_invert = false;
    ObbFeature best{kObbEdgeEdge, 0, 0};
    auto face = [&](V3 axis, float e1, float e2, uint8_t kind, uint8_t ia, uint8_t ib) {
        const float s2 = fabs_(e1) - e2;
        if (s2 > threshold) return false;
        if (!have || s2 > best_s2) {
            have = true;
            best_s2 = s2;
            best_axis = axis;
            best_invert = e1 < 0.0f;
            best = ObbFeature{kind, ia, ib};
        }
        return true;
    };
    auto edge = [&](V3 nl, float e1, float e2, uint8_t ia, uint8_t ib) {
        const float s2_raw = fabs_(e1) - e2;
        if (s2_raw > kEdgeSepEps) return false;
        const float al = sqrtf(nl.x * nl.x + nl.y * nl.y + nl.z * nl.z);
        if (al <= kEdgeSepEps) return true;
        const float s2 = s2_raw / al;
        if (!have || s2 * kEdgeFudge > best_s2) {
            have = true;
            best_s2 = s2;
            const V3 nc{nl.x / al, nl.y / al, nl.z / al};
            best_axis = V3{a.axis[0].x * nc.x + a.axis[1].x * nc.y + a.axis[2].x * nc.z,
                           a.axis[0].y * nc.x + a.axis[1].y * nc.y + a.axis[2].y * nc.z,
                           a.axis[0].z * nc.x + a.axis[1].z * nc.y + a.axis[2].z * nc.z};
            best_invert = e1 < 0.0f;
            best = ObbFeature{kObbEdgeEdge, ia, ib};
        }
        return true;
    };
    for (int i = 0; i < 3; ++i) {
        const float e2 = ((comp3(a.half, i) + b.half.x * AbsRF[i][0]) + b.half.y * AbsRF[i][1]) + b.half.z * AbsRF[i][2];
        if (!face(a.axis[i], t[i], e2, kObbFaceA, static_cast<uint8_t>(i), 0)) return false;
    }
    for (int j = 0; j < 3; ++j) {
        const float e1 = dot(tw, b.axis[j]);
        const float e2 =
            ((a.half.x * AbsRF[0][j] + a.half.y * AbsRF[1][j]) + a.half.z * AbsRF[2][j]) + comp3(b.half, j);
        if (!face(b.axis[j], e1, e2, kObbFaceB, 0, static_cast<uint8_t>(j))) return false;
    }
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
            V3 nl;
            if (i == 0) {
                nl = V3{0.0f, -R[2][j], R[1][j]};
            } else if (i == 1) {
                nl = V3{R[2][j], 0.0f, -R[0][j]};
            } else {
                nl = V3{-R[1][j], R[0][j], 0.0f};
            }
            const int a_lo = i == 0 ? 1 : 0, a_hi = i == 2 ? 1 : 2;
            const int b_lo = j == 0 ? 1 : 0, b_hi = j == 2 ? 1 : 2;
            const float e1 = t[i2] * R[i1][j] - t[i1] * R[i2][j];
            const float e2 = ((comp3(a.half, a_lo) * AbsR[a_hi][j] + comp3(a.half, a_hi) * AbsR[a_lo][j]) +
                              comp3(b.half, b_lo) * AbsR[i][b_hi]) +
                             comp3(b.half, b_hi) * AbsR[i][b_lo];
            if (!edge(nl, e1, e2, static_cast<uint8_t>(i), static_cast<uint8_t>(j))) return false;
        }
    }
    if (!have) return false;
    if (best_invert) best_axis = -best_axis;
    out_normal = best_axis;
    out_overlap = -best_s2;
    out_feature = best;
    return true;
}
// the same test run from b to a, reported from a to b (reference ComputeObbContactGameOrder)
RG_HDI bool obb_contact_game_order(const Obb& a, const Obb& b, float threshold, V3& n, float& overlap, ObbFeature& f) {
    V3 nba;
    ObbFeature fba;
    if (!obb_contact(b, a, threshold, nba, overlap, fba)) return false;
    n = -nba;
    f.kind = fba.kind == kObbFaceA ? kObbFaceB : (fba.kind == kObbFaceB ? kObbFaceA : fba.kind);
    f.axis_a = fba.axis_b;
    f.axis_b = fba.axis_a;
    return true;
}

// ---- contact points -----------------------------------------------------------------------------------------------
// Clips the quad `quad` (4 points, 2D) against the rectangle |x| < h[0], |y| < h[1] (reference IntersectRectQuad2).
RG_HDI int intersect_rect_quad2(const float h[2], const float quad[8], float out[16]) {
    int in_count = 4, out_count = 0;
    float buffer[16];
    const float* in_poly = quad;
    float* out_poly = out;
    for (int axis = 0; axis <= 1; ++axis) {
        for (int sign = -1; sign <= 1; sign += 2) {
            const float* ip = in_poly;
            float* op = out_poly;
            out_count = 0;
            for (int i = in_count; i > 0; --i) {
                const bool inside_cur = sign * ip[axis] < h[axis];
                if (inside_cur) {
                    op[0] = ip[0];
                    op[1] = ip[1];
                    op += 2;
                    ++out_count;
                    if (out_count & 8) {
                        in_poly = out_poly;
                        goto done;
                    }
                }
                const float* np = (i > 1) ? (ip + 2) : in_poly;
                const bool inside_next = sign * np[axis] < h[axis];
                if (inside_cur != inside_next) {
                    op[1 - axis] = ip[1 - axis] + (np[1 - axis] - ip[1 - axis]) / (np[axis] - ip[axis]) *
                                                      (sign * h[axis] - ip[axis]);
                    op[axis] = sign * h[axis];
                    op += 2;
                    ++out_count;
                    if (out_count & 8) {
                        in_poly = out_poly;
                        goto done;
                    }
                }
                ip += 2;
            }
            in_poly = out_poly;
            out_poly = (in_poly == out) ? buffer : out;
            in_count = out_count;
        }
    }
done:
    if (in_poly != out)
        for (int k = 0; k < out_count * 2; ++k) out[k] = in_poly[k];
    return out_count;
}

// Keeps `max_points` of `count` clipped points: the deepest, then the ones nearest to evenly spaced angles around the
// polygon's centroid (reference CullFacePoints2; the angles are the double-precision atan2 it calls).
RG_HDI void cull_face_points2(int count, const float* points, int max_points, int deepest, int out_idx[8]) {
    float cx = 0.0f, cy = 0.0f;
    if (count == 1) {
        cx = points[0];
        cy = points[1];
    } else if (count == 2) {
        cx = 0.5f * (points[0] + points[2]);
        cy = 0.5f * (points[1] + points[3]);
    } else {
        float area = 0.0f, q = 0.0f;
        for (int i = 0; i < count - 1; ++i) {
            q = points[i * 2] * points[i * 2 + 3] - points[i * 2 + 2] * points[i * 2 + 1];
            area += q;
            cx += q * (points[i * 2] + points[i * 2 + 2]);
            cy += q * (points[i * 2 + 1] + points[i * 2 + 3]);
        }
        q = points[count * 2 - 2] * points[1] - points[0] * points[count * 2 - 1];
        const float denom = area + q;
        const float scale = fabs_(denom) > 1.1920929e-7f ? (1.0f / (3.0f * denom)) : 1.0e18f;
        cx = scale * (cx + q * (points[count * 2 - 2] + points[0]));
        cy = scale * (cy + q * (points[count * 2 - 1] + points[1]));
    }
    float angles[8];
    for (int i = 0; i < count; ++i)
        angles[i] = static_cast<float>(atan2(static_cast<double>(points[i * 2 + 1] - cy),
                                             static_cast<double>(points[i * 2] - cx)));
    int avail[8];
    for (int i = 0; i < count; ++i) avail[i] = 1;
    avail[deepest] = 0;
    out_idx[0] = deepest;
    for (int slot = 1; slot < max_points; ++slot) {
        float target = static_cast<float>(slot) * (2.0f * 3.14159265f / static_cast<float>(max_points)) +
                       angles[deepest];
        if (target > 3.14159265f) target -= 2.0f * 3.14159265f;
        float best_diff = 1.0e9f;
        int best = deepest;
        for (int i = 0; i < count; ++i) {
            if (!avail[i]) continue;
            float diff = fabs_(angles[i] - target);
            if (diff > 3.14159265f) diff = 2.0f * 3.14159265f - diff;
            if (diff < best_diff) {
                best_diff = diff;
                best = i;
            }
        }
        avail[best] = 0;
        out_idx[slot] = best;
    }
}

// Face contact: the incident box's face nearest to the reference face, clipped to it (reference
// ComputeFaceClippedCarCarContactAnchorPairs). Returns the number of points (<= 4).
RG_HDI int face_clipped_anchor_pairs(const Obb& ref, int ref_axis, const Obb& inc, V3 ref_to_inc, V3* out_ref,
                                     V3* out_inc, int max_points, int ref_is_a, V3* out_game, float* out_depths) {
    const float sign = dot(ref.axis[ref_axis], ref_to_inc) >= 0.0f ? 1.0f : -1.0f;
    const V3 rn = ref.axis[ref_axis] * sign;
    const float nr[3] = {dot(inc.axis[0], rn), dot(inc.axis[1], rn), dot(inc.axis[2], rn)};
    const float anr[3] = {fabs_(nr[0]), fabs_(nr[1]), fabs_(nr[2])};
    int lanr, a1, a2;
    if (anr[1] > anr[0]) {
        if (anr[1] > anr[2]) {
            a1 = 0;
            lanr = 1;
            a2 = 2;
        } else {
            a1 = 0;
            a2 = 1;
            lanr = 2;
        }
    } else {
        if (anr[0] > anr[2]) {
            lanr = 0;
            a1 = 1;
            a2 = 2;
        } else {
            a1 = 0;
            a2 = 1;
            lanr = 2;
        }
    }
    const V3 center = nr[lanr] < 0.0f ? (inc.center - ref.center + inc.axis[lanr] * comp3(inc.half, lanr))
                                      : (inc.center - ref.center - inc.axis[lanr] * comp3(inc.half, lanr));
    const int code1 = ref_axis == 0 ? 1 : 0;
    const int code2 = ref_axis == 2 ? 1 : 2;
    const float c1 = dot(center, ref.axis[code1]), c2 = dot(center, ref.axis[code2]);
    const float m11 = dot(ref.axis[code1], inc.axis[a1]), m12 = dot(ref.axis[code1], inc.axis[a2]);
    const float m21 = dot(ref.axis[code2], inc.axis[a1]), m22 = dot(ref.axis[code2], inc.axis[a2]);
    const float k1 = m11 * comp3(inc.half, a1), k2 = m21 * comp3(inc.half, a1);
    const float k3 = m12 * comp3(inc.half, a2), k4 = m22 * comp3(inc.half, a2);
    const float quad[8] = {c1 - k1 - k3, c2 - k2 - k4, c1 - k1 + k3, c2 - k2 + k4,
                           c1 + k1 + k3, c2 + k2 + k4, c1 + k1 - k3, c2 + k2 - k4};
    const float rect[2] = {comp3(ref.half, code1), comp3(ref.half, code2)};
    float clipped[16];
    const int poly = intersect_rect_quad2(rect, quad, clipped);
    if (poly < 1) return 0;
    const float det = m11 * m22 - m12 * m21;
    if (fabs_(det) <= 1.0e-8f) return 0;
    const float det_inv = 1.0f / det;
    const float im11 = m11 * det_inv, im12 = m12 * det_inv, im21 = m21 * det_inv, im22 = m22 * det_inv;
    V3 coords[8];
    float depths[8];
    int n = 0;
    for (int i = 0; i < poly; ++i) {
        const float u = clipped[i * 2 + 0], v = clipped[i * 2 + 1];
        const float ik1 = im22 * (u - c1) - im12 * (v - c2);
        const float ik2 = -im21 * (u - c1) + im11 * (v - c2);
        const V3 local = center + inc.axis[a1] * ik1 + inc.axis[a2] * ik2;
        coords[n] = local;
        const float depth = comp3(ref.half, ref_axis) - dot(rn, local);
        depths[n] = depth;
        if (depth >= 0.0f) {
            clipped[n * 2 + 0] = u;
            clipped[n * 2 + 1] = v;
            ++n;
        }
    }
    if (n < 1) return 0;
    int outc = n < max_points ? n : max_points;
    if (outc > 4) outc = 4;
    if (outc < 1) outc = 1;
    int sel[8];
    if (n <= outc) {
        for (int i = 0; i < n; ++i) sel[i] = i;
        outc = n;
    } else {
        int deepest = 0;
        float dd = depths[0];
        for (int i = 1; i < n; ++i)
            if (depths[i] > dd) {
                dd = depths[i];
                deepest = i;
            }
        cull_face_points2(n, clipped, outc, deepest, sel);
    }
    for (int i = 0; i < outc; ++i) {
        const int idx = sel[i];
        const V3 ip = ref.center + coords[idx];
        const V3 rp = ip + rn * depths[idx];
        out_ref[i] = rp;
        out_inc[i] = ref_is_a ? ip : (rp + rn * (-depths[idx]));
        if (out_game) out_game[i] = ref_is_a ? rp : ip;
        if (out_depths) out_depths[i] = -depths[idx];
    }
    return outc;
}

// Edge/edge contact: the closest points of the two edges of the separating cross axis (reference
// ComputeEdgeEdgeCarCarContactAnchorsBulletStyle with ComputeLineClosestApproachParams).
RG_HDI bool edge_edge_anchors(const Obb& a, int axis_a, const Obb& b, int axis_b, V3& out_normal, V3& out_pa,
                              V3& out_pb, float& out_game_s) {
    if (axis_a < 0 || axis_a > 2 || axis_b < 0 || axis_b > 2) return false;
    const Obb& box1 = b;
    const Obb& box2 = a;
    const int i = axis_b, j = axis_a;
    const V3 p = box2.center - box1.center;
    const float pp[3] = {dot(box1.axis[0], p), dot(box1.axis[1], p), dot(box1.axis[2], p)};
    float r[3];
    for (int k = 0; k < 3; ++k) r[k] = dot(box1.axis[k], box2.axis[j]);
    float e1;
    V3 nc;
    if (i == 0) {
        e1 = pp[2] * r[1] - pp[1] * r[2];
        nc = V3{0.0f, -r[2], r[1]};
    } else if (i == 1) {
        e1 = pp[0] * r[2] - pp[2] * r[0];
        nc = V3{r[2], 0.0f, -r[0]};
    } else {
        e1 = pp[1] * r[0] - pp[0] * r[1];
        nc = V3{-r[1], r[0], 0.0f};
    }
    const float l = sqrtf(nc.x * nc.x + nc.y * nc.y + nc.z * nc.z);
    if (!(l > 1.1920929e-07f)) return false;
    {
        constexpr float kFudge2 = 1.0e-5f;
        const int lo = i == 0 ? 1 : 0, hi = i == 2 ? 1 : 2;
        const int k1 = j == 0 ? 1 : 0, k2 = j == 2 ? 1 : 2;
        const float q_hi_j = fabs_(r[hi]) + kFudge2, q_lo_j = fabs_(r[lo]) + kFudge2;
        const float q_i_k2 = fabs_(dot(box1.axis[i], box2.axis[k2])) + kFudge2;
        const float q_i_k1 = fabs_(dot(box1.axis[i], box2.axis[k1])) + kFudge2;
        const float e2 = ((comp3(box1.half, lo) * q_hi_j + comp3(box1.half, hi) * q_lo_j) +
                          comp3(box2.half, k1) * q_i_k2) +
                         comp3(box2.half, k2) * q_i_k1;
        out_game_s = (fabs_(e1) - e2) / l;
    }
    nc = V3{nc.x / l, nc.y / l, nc.z / l};
    V3 normal{box1.axis[0].x * nc.x + box1.axis[1].x * nc.y + box1.axis[2].x * nc.z,
              box1.axis[0].y * nc.x + box1.axis[1].y * nc.y + box1.axis[2].y * nc.z,
              box1.axis[0].z * nc.x + box1.axis[1].z * nc.y + box1.axis[2].z * nc.z};
    if (e1 < 0.0f) normal = V3{-normal.x, -normal.y, -normal.z};
    V3 pa = box1.center;
    for (int k = 0; k < 3; ++k) {
        const float s = dot(normal, box1.axis[k]) > 0.0f ? 1.0f : -1.0f;
        pa += box1.axis[k] * (s * comp3(box1.half, k));
    }
    V3 pb = box2.center;
    for (int k = 0; k < 3; ++k) {
        const float s = dot(normal, box2.axis[k]) > 0.0f ? -1.0f : 1.0f;
        pb += box2.axis[k] * (s * comp3(box2.half, k));
    }
    const V3 ua = box1.axis[i], ub = box2.axis[j];
    float alpha = 0.0f, beta = 0.0f;
    {
        const V3 pd = pb - pa;
        const float uaub = dot(ua, ub);
        const float q1 = dot(ua, pd);
        const float q2 = -dot(ub, pd);
        float d = 1.0f - uaub * uaub;
        if (d > 1.0e-4f) {
            d = 1.0f / d;
            alpha = (q1 + uaub * q2) * d;
            beta = (uaub * q1 + q2) * d;
        }
    }
    out_normal = normal;
    out_pa = pb + ub * beta;
    out_pb = pa + ua * alpha;
    return true;
}

// A body-space round trip of a world point (reference CarBodyManifoldWorldPointBt).
RG_HDI V3 car_manifold_point(const CarState& c, V3 p) {
    V3 f, r, u;
    car_basis(c, f, r, u);
    return car_world_point(f, r, u, c.pos_bt, car_local_point(f, r, u, c.pos_bt, p));
}
RG_HDI V3 car_inverse_rotate(const CarState& c, V3 v) {
    if (!c.basis_authoritative) return quat_inverse_rotate(c.rot, v);
    return V3{dot(c.basis_forward, v), dot(c.basis_right, v), dot(c.basis_up, v)};
}
// the hitbox corner furthest along a body-space direction, uu (reference SupportPointOnCarHitboxLocal)
RG_HDI V3 car_hitbox_support_local(const CarConfig& cfg, V3 d) {
    const float m = ball_car_shape_margin(cfg);
    const V3 h = (bullet_hitbox_size(cfg) * 0.5f) - V3{m, m, m} + V3{m, m, m};
    return cfg.hitbox_offset + V3{d.x >= 0.0f ? h.x : -h.x, d.y >= 0.0f ? h.y : -h.y, d.z >= 0.0f ? h.z : -h.z};
}

// The pair's contact points for a fresh contact (reference ComputeApproxCarCarContactAnchorPairsWithBtObb with the
// game's face contacts): face clip, edge/edge anchors, else the two hitbox support points.
struct CarCarAnchors {
    int count;
    V3 a_bt[4], b_bt[4];
    V3 a_uu[4], b_uu[4];  // the same points in uu as the reference carries them (not always a_bt * 50)
    V3 game_a_bt[4];
    float game_depth[4];
    bool game_valid;
    V3 game_normal;
};
RG_HDI void car_car_anchors(const CarState& a, const CarConfig& ca, const Obb& oa, const CarState& b,
                            const CarConfig& cb, const Obb& ob, V3 normal, const ObbFeature& f, float overlap_uu,
                            CarCarAnchors& out) {
    out.count = 0;
    out.game_valid = false;
    if (f.kind == kObbFaceA || f.kind == kObbFaceB) {
        const bool fa = f.kind == kObbFaceA;
        V3 ref_pts[4], inc_pts[4];
        const int n = face_clipped_anchor_pairs(fa ? oa : ob, fa ? f.axis_a : f.axis_b, fa ? ob : oa,
                                                fa ? normal : -normal, ref_pts, inc_pts, 4, fa ? 1 : 0, out.game_a_bt,
                                                out.game_depth);
        if (n > 0) {
            out.game_valid = true;
            out.game_normal = normal;
            for (int i = 0; i < n; ++i) {
                out.a_bt[i] = car_manifold_point(a, fa ? ref_pts[i] : inc_pts[i]);
                out.b_bt[i] = car_manifold_point(b, fa ? inc_pts[i] : ref_pts[i]);
                out.a_uu[i] = out.a_bt[i] * 50.0f;
                out.b_uu[i] = out.b_bt[i] * 50.0f;
            }
            out.count = n;
            return;
        }
        return;  // game face contacts: a face clip that keeps nothing has no points
    }
    {
        V3 pa, pb, gn;
        float gs = 0.0f;
        if (edge_edge_anchors(oa, f.axis_a, ob, f.axis_b, gn, pa, pb, gs)) {
            float overlap_bt = overlap_uu * (1.0f / 50.0f);
            {
                V3 sn;
                float so = 0.0f;
                ObbFeature sf;
                if (obb_contact_game_order(oa, ob, 0.0f, sn, so, sf) && sf.kind == kObbEdgeEdge &&
                    sf.axis_a == f.axis_a && sf.axis_b == f.axis_b)
                    overlap_bt = so;
            }
            const V3 raw_a = pa;
            out.game_a_bt[0] = raw_a;
            out.game_depth[0] = gs;
            out.game_normal = -gn;
            out.game_valid = true;
            const V3 raw_b = overlap_bt > 0.0f ? (raw_a + gn * overlap_bt) : pb;
            out.b_bt[0] = car_manifold_point(b, raw_b);
            out.a_bt[0] = car_manifold_point(a, raw_a);
            out.a_uu[0] = out.a_bt[0] * 50.0f;
            out.b_uu[0] = out.b_bt[0] * 50.0f;
            out.count = 1;
            return;
        }
    }
    const V3 pa_uu = a.pos + car_rotate(a, car_hitbox_support_local(ca, car_inverse_rotate(a, normal)));
    const V3 pb_uu = b.pos + car_rotate(b, car_hitbox_support_local(cb, car_inverse_rotate(b, -normal)));
    out.a_uu[0] = pa_uu;
    out.b_uu[0] = pb_uu;
    out.a_bt[0] = pa_uu * (1.0f / 50.0f);
    out.b_bt[0] = pb_uu * (1.0f / 50.0f);
    out.count = 1;
}

// Refreshes the pair's retained manifold and adds this tick's points (reference PrepareSharedCarCarCollisionContacts
// without a cached contact). Returns false when the pair has no contact; `demo_x_*` are the contact points' body-space
// x of each car, for the bumper test.
RG_HDI bool car_car_prepare(const CarState& a, const CarConfig& ca, const CarState& b, const CarConfig& cb,
                            float min_dist_sq, CarCarManifold& m, V3& normal, int& demo_count, float* demo_xa,
                            float* demo_xb) {
    const float thr = fmin_(car_contact_threshold_bt(ca), car_contact_threshold_bt(cb));
    car_car_refresh(m, a, b, thr);
    const bool fresh_gate = len2(b.pos - a.pos) < min_dist_sq;
    if (!fresh_gate && m.count == 0) return false;
    const Obb oa = make_car_obb_bt(a, ca), ob = make_car_obb_bt(b, cb);
    bool overlap = true;
    for (int k = 0; k < 3; ++k) {
        float ea = 0.0f, eb = 0.0f;
        for (int i = 0; i < 3; ++i) {
            ea += fabsf(comp3(oa.axis[i], k)) * comp3(oa.half, i);
            eb += fabsf(comp3(ob.axis[i], k)) * comp3(ob.half, i);
        }
        const float cA = comp3(oa.center, k), cB = comp3(ob.center, k);
        overlap = overlap && !(cA - ea > cB + eb || cA + ea < cB - eb);
    }
    if (!overlap) {
        m.count = 0;
        return false;
    }
    V3 cur_n{1.0f, 0.0f, 0.0f};
    ObbFeature cur_f{kObbEdgeEdge, 0, 0};
    float cur_overlap_bt = 0.0f;
    const bool have_current = fresh_gate && obb_contact_game_order(oa, ob, 0.0f, cur_n, cur_overlap_bt, cur_f);
    const float cur_overlap_uu = cur_overlap_bt * 50.0f;
    bool have = false;
    if (have_current) {
        normal = cur_n;
        have = true;
    }
    const bool fresh = have;
    if (!have && m.count > 0) {
        normal = m.p[0].normal;
        have = true;
    }
    if (!have) return false;
    CarCarAnchors an;
    int n = 1;
    V3 pts_a_uu[4], pts_b_uu[4];
    if (!fresh) {
        n = m.count < 4 ? m.count : 4;
        for (int k = 0; k < n; ++k) {
            pts_a_uu[k] = m.p[k].pos_a * 50.0f;
            pts_b_uu[k] = m.p[k].pos_b * 50.0f;
        }
    } else {
        car_car_anchors(a, ca, oa, b, cb, ob, normal, cur_f, cur_overlap_uu, an);
        n = an.count;
        for (int k = 0; k < n; ++k) {
            pts_a_uu[k] = an.a_uu[k];
            pts_b_uu[k] = an.b_uu[k];
        }
    }
    demo_count = 0;
    if ((have_current || !fresh) && n > 0) {
        demo_count = n;
        for (int k = 0; k < n; ++k) {
            demo_xa[k] = car_inverse_rotate(a, pts_a_uu[k] - a.pos).x;
            demo_xb[k] = car_inverse_rotate(b, pts_b_uu[k] - b.pos).x;
        }
    }
    if (fresh && n > 0) {
        V3 fa_, ra_, ua_, fb_, rb_, ub_;
        car_basis(a, fa_, ra_, ua_);
        car_basis(b, fb_, rb_, ub_);
        for (int k = 0; k < n; ++k) {
            const V3 on_a = an.game_valid ? an.game_a_bt[k] : an.a_bt[k];
            const float depth = an.game_valid ? an.game_depth[k] : dot(an.b_bt[k] - on_a, normal);
            if (depth > thr) continue;
            const V3 pn = an.game_valid ? an.game_normal : normal;
            CarCarPoint pt;
            pt.normal = pn;
            pt.local_a = car_local_point(fa_, ra_, ua_, a.pos_bt, on_a);
            pt.local_b = car_local_point(fb_, rb_, ub_, b.pos_bt, on_a + pn * depth);
            pt.pos_a = pt.pos_b = V3{0.0f, 0.0f, 0.0f};
            pt.distance = depth;
            car_car_add(m, pt, thr);
        }
        car_car_refresh(m, a, b, thr);
    }
    return true;
}

// ---- pair rows ----------------------------------------------------------------------------------------------------
// Two-body rows between cars a and b of an arena, in Bullet units (normal_a points from b into a).
struct PairVelRow {
    V3 normal_a, rel_a_cross, rel_b_cross, ang_a, ang_b;
    float inv_mass, jac, rhs, applied;
    int32_t a, b;
};
struct PairFricRow {
    V3 tangent_a, rel_a_cross, rel_b_cross, ang_a, ang_b;
    float inv_mass, jac, rhs, applied, friction;
    int32_t a, b, normal_row;
};
struct PairSplitRow {
    V3 normal_a, rel_a_cross, rel_b_cross, ang_a, ang_b;
    float inv_mass, jac, rhs, applied;
    int32_t a, b;
    uint8_t has_bt;
};
constexpr int kMaxPairRows = 4 * 15;  // 4 points per pair, up to 15 pairs (6 cars)
struct CarCarRows {
    PairVelRow vel[kMaxPairRows];
    PairFricRow fric[kMaxPairRows];
    PairSplitRow split[kMaxPairRows];
    int nv, nf, ns;
};

RG_HD V3 plane_space1_first(V3 n) {
    constexpr float kSqrt12 = 0.7071067811865475244008443621048490f;
    if (fabs_(n.z) > kSqrt12) {
        const float a = n.y * n.y + n.z * n.z;
        const float k = 1.0f / sqrtf(a);
        return V3{0.0f, -n.z * k, n.y * k};
    }
    const float a = n.x * n.x + n.y * n.y;
    const float k = 1.0f / sqrtf(a);
    return V3{-n.y * k, n.x * k, 0.0f};
}

// The pair's rows from its retained points (reference EmitSharedCarCarContactRows).
RG_HDI void car_car_rows(const CarState& a, const CarState& b, const CarConfig& ca, const CarConfig& cb,
                         const TickConfig& tc, const PreContactCar& pa, const PreContactCar& pb, float dt, int ia,
                         int ib, const CarCarManifold& m, CarCarRows& rows) {
    const int n = m.count < 4 ? m.count : 4;
    if (n == 0) return;
    float max_pen_uu = 0.0f;
    for (int k = 0; k < n; ++k) max_pen_uu = fmax_(max_pen_uu, -m.p[k].distance * 50.0f);
    const float penetration = fmax_(0.0f, max_pen_uu);
    V3 ia0, ia1, ia2, ib0, ib1, ib2, ua0, ua1, ua2, ub0, ub1, ub2;
    car_inv_inertia_world_bt(a, ca, tc.car_mass, ia0, ia1, ia2);
    car_inv_inertia_world_bt(b, cb, tc.car_mass, ib0, ib1, ib2);
    car_inv_inertia_uu(a, ca, tc.car_mass, ua0, ua1, ua2);
    car_inv_inertia_uu(b, cb, tc.car_mass, ub0, ub1, ub2);
    const float inv_mass = 1.0f / tc.car_mass;
    const V3 lin_a = pa.vel_bt, lin_b = pb.vel_bt;
    const V3 ext_lin_a = a.ext_force_impulse_bt, ext_lin_b = b.ext_force_impulse_bt;
    const V3 ext_ang_a = a.ext_torque_impulse, ext_ang_b = b.ext_torque_impulse;
    const V3 base_lin_a = lin_a + ext_lin_a, base_lin_b = lin_b + ext_lin_b;
    for (int k = 0; k < n; ++k) {
        const CarCarPoint& pt = m.p[k];
        const V3 np = pt.normal;
        const V3 ra_bt = pt.pos_a - a.pos_bt, rb_bt = pt.pos_b - b.pos_bt;
        const V3 ra = ra_bt * 50.0f, rb = rb_bt * 50.0f;
        const V3 na = -np, nb = np;
        const V3 ra_x_n = cross(ra_bt, na);
        const V3 dang_a = mul_rows(ia0, ia1, ia2, ra_x_n);
        const float den_a = inv_mass + dot(na, cross(dang_a, ra_bt));
        const V3 rb_x_n = cross(rb_bt, -na);
        const V3 dang_b = mul_rows(ib0, ib1, ib2, rb_x_n);
        const float den_b = inv_mass + dot(na, cross(-dang_b, rb_bt));
        const float den = den_a + den_b;
        if (!(den <= 1.0e-6f) && rows.nv < kMaxPairRows) {
            const float v1 = dot(na, base_lin_a) + dot(ra_x_n, pa.ang_vel + ext_ang_a);
            const float v2 = dot(nb, base_lin_b) + dot(rb_x_n, pb.ang_vel + ext_ang_b);
            const float base_vn = v1 + v2;
            const float jac = 1.0f / den;
            const V3 va = lin_a + cross(pa.ang_vel, ra_bt);
            const V3 vb = lin_b + cross(pb.ang_vel, rb_bt);
            const float vn_no_ext = dot(nb, vb - va);
            const float rest = fmax_(0.1f * -vn_no_ext, 0.0f);
            const int vi = rows.nv++;
            PairVelRow& r = rows.vel[vi];
            r.normal_a = na;
            r.rel_a_cross = ra_x_n;
            r.rel_b_cross = rb_x_n;
            r.ang_a = dang_a;
            r.ang_b = dang_b;
            r.inv_mass = inv_mass;
            r.jac = jac;
            r.rhs = (rest - base_vn) * jac;
            r.applied = 0.0f;
            r.a = ia;
            r.b = ib;
            if (rows.nf < kMaxPairRows) {
                const V3 bva = base_lin_a + cross(pa.ang_vel + ext_ang_a, ra_bt);
                const V3 bvb = base_lin_b + cross(pb.ang_vel + ext_ang_b, rb_bt);
                const V3 brv = bvb - bva;
                V3 t = brv - np * dot(brv, np);
                const float lat = len2(t);
                const float tl = sqrtf(lat);
                t = lat > 1.1920928955078125e-07f ? t * (1.0f / tl) : plane_space1_first(np);
                const V3 ta = t, tb = -t;
                const V3 ra_x_t = cross(ra_bt, ta), rb_x_t = cross(rb_bt, tb);
                const V3 tang_a = mul_rows(ia0, ia1, ia2, ra_x_t);
                const V3 tang_b = mul_rows(ib0, ib1, ib2, rb_x_t);
                const float dta = inv_mass + dot(ta, cross(tang_a, ra_bt));
                const float dtb = inv_mass + dot(ta, cross(-tang_b, rb_bt));
                const float dt_ = dta + dtb;
                if (!(dt_ <= 1.0e-6f)) {
                    PairFricRow& fr = rows.fric[rows.nf++];
                    fr.tangent_a = ta;
                    fr.rel_a_cross = ra_x_t;
                    fr.rel_b_cross = rb_x_t;
                    fr.ang_a = tang_a;
                    fr.ang_b = tang_b;
                    fr.inv_mass = inv_mass;
                    fr.jac = 1.0f / dt_;
                    const float w1 = dot(ta, base_lin_a) + dot(ra_x_t, pa.ang_vel);
                    const float w2 = dot(tb, base_lin_b) + dot(rb_x_t, pb.ang_vel);
                    fr.rhs = -(w1 + w2) * fr.jac;
                    fr.applied = 0.0f;
                    fr.friction = 0.09f;
                    fr.a = ia;
                    fr.b = ib;
                    fr.normal_row = vi;
                }
            }
        }
        if (penetration > 0.0f && dt > 0.0f) {
            const V3 cpa = pt.pos_a * 50.0f, cpb = pt.pos_b * 50.0f;
            const V3 sra = (cpa * (1.0f / 50.0f) - a.pos_bt) * 50.0f;
            const V3 srb = (cpb * (1.0f / 50.0f) - b.pos_bt) * 50.0f;
            const float ppen = fmax_(0.0f, -dot(cpb - cpa, np));
            if (!(ppen <= 0.0f)) {
                const V3 sa_x = cross(sra, na), sb_x = cross(srb, nb);
                const V3 sang_a = mul_rows(ua0, ua1, ua2, sa_x);
                const V3 sang_b = mul_rows(ub0, ub1, ub2, sb_x);
                float sden = 0.0f;
                sden += inv_mass + dot(na, cross(sang_a, sra));
                sden += inv_mass + dot(nb, cross(sang_b, srb));
                if (!(sden <= 1.0e-8f)) {
                    const float jac_uu = 1.0f / sden;
                    const float rhs_uu = ((ppen * 0.8f) / dt) * jac_uu;
                    const float ppen_bt = fmax_(0.0f, -dot(pt.pos_b - pt.pos_a, np));
                    float dbt = 0.0f;
                    dbt += inv_mass + dot(na, cross(dang_a, ra_bt));
                    dbt += inv_mass + dot(nb, cross(dang_b, rb_bt));
                    const float jac_bt = dbt > 1.0e-8f ? 1.0f / dbt : 0.0f;
                    const float rhs_bt = ((ppen_bt * 0.8f) / dt) * jac_bt;
                    if (rhs_uu > 0.0f && jac_uu > 0.0f && rows.ns < kMaxPairRows) {
                        PairSplitRow& s = rows.split[rows.ns++];
                        s.normal_a = na;
                        s.rel_a_cross = ra_x_n;
                        s.rel_b_cross = rb_x_n;
                        s.ang_a = dang_a;
                        s.ang_b = dang_b;
                        s.inv_mass = inv_mass;
                        s.jac = jac_bt;
                        s.rhs = rhs_bt;
                        s.applied = 0.0f;
                        s.a = ia;
                        s.b = ib;
                        s.has_bt = (jac_bt > 0.0f && ppen_bt > 0.0f) ? 1 : 0;
                    }
                }
            }
        }
    }
}

// ---- bumps and demolitions ----------------------------------------------------------------------------------------
RG_HDI void demolish_car(CarState& c, const TickConfig& tc) {
    c.is_demoed = 1;
    c.demo_respawn_timer = tc.demo_respawn_time + tc.tick_dt;
}
// The hitter's bump / demolition counters, and the car-bump event (reference RecordCarHit and the CarBump emits
// beside it, triangle_and_carcar.hpp:2883-2895, 2953-2965).
RG_HDI void record_car_hit(CarState& hitter, uint32_t hitter_id, uint32_t victim_id, bool is_demo, uint8_t hitter_team,
                           const EventStream& events) {
    const uint32_t k = ((victim_id - hitter_id) & 7u) - 1u;
    if (is_demo) {
        hitter.bump_event_demos[k] = static_cast<uint8_t>(hitter.bump_event_demos[k] + 1u);
    } else {
        hitter.bump_event_bumps[k] = static_cast<uint8_t>(hitter.bump_event_bumps[k] + 1u);
    }
    if (events.windows) {
        PhysicsEvent e = new_event(kEventCarBump);
        e.car_id = hitter_id;
        e.other_car_id = victim_id;
        e.team = hitter_team;
        e.is_demo = is_demo ? 1 : 0;
        e.car_on_ground = hitter.is_on_ground;
        e.position = hitter.pos;
        e.car_velocity = hitter.vel;
        emit_event_for_car(events, hitter_id, e);
    }
}
RG_HDI void ue3_rotator_axes(const Ue3Rotator& r, V3& x, V3& y, V3& z) {
    const float sp = ue3_rotator_sin(r.pitch), cp = ue3_rotator_sin(r.pitch + 16384);
    const float sy = ue3_rotator_sin(r.yaw), cy = ue3_rotator_sin(r.yaw + 16384);
    const float sr = ue3_rotator_sin(r.roll), cr = ue3_rotator_sin(r.roll + 16384);
    const float sp_sr = sp * sr, cr_sp = cr * sp;
    x = V3{cy * cp, cp * sy, sp};
    y = V3{sp_sr * cy - cr * sy, cy * cr + sp_sr * sy, -sr * cp};
    z = V3{-(cr_sp * cy + sy * sr), cy * sr - cr_sp * sy, cp * cr};
}
// Whether the victim's hitbox centre lies in the hitter's forward cone (reference InForwardConePose).
RG_HDI bool in_forward_cone(V3 a_pos, Q4 a_rot, const CarConfig& a_cfg, V3 v_pos, Q4 v_rot, const CarConfig& v_cfg,
                            bool reverse, float max_yaw_deg) {
    V3 fwd, right, up, vx, vy, vz;
    ue3_rotator_axes(ue3_quat_to_rotator(a_rot), fwd, right, up);
    ue3_rotator_axes(ue3_quat_to_rotator(v_rot), vx, vy, vz);
    const V3 ao = a_cfg.hitbox_offset, vo = v_cfg.hitbox_offset;
    const V3 pa = a_pos + V3{dot(fwd, ao), dot(right, ao), dot(up, ao)};
    const V3 pv = v_pos + V3{dot(vx, vo), dot(vy, vo), dot(vz, vo)};
    V3 d = pv - pa;
    const float d2 = len2(d);
    if (d2 != 1.0f) d = d2 < 1e-8f ? V3{0.0f, 0.0f, 0.0f} : d * (1.0f / sqrtf(d2));
    const V3 f = reverse ? fwd * -1.0f : fwd;
    auto angle_deg = [&](V3 axis) {
        float k = dot(d, axis);
        k = k >= 0.0f ? (k / 1.01f) : (k * 1.01f);
        V3 p = d - axis * k;
        const float p2 = len2(p);
        if (p2 != 1.0f) p = p2 < 1e-8f ? V3{0.0f, 0.0f, 0.0f} : p * (1.0f / sqrtf(p2));
        float c = dot(f, p);
        c = c < -1.0f ? -1.0f : (c > 1.0f ? 1.0f : c);
        return ucrt_acosf(c) * 57.29578f;
    };
    if (angle_deg(right) > 36.8698959f) return false;
    return angle_deg(up) <= max_yaw_deg;
}

// ---- the demolition's time of impact ------------------------------------------------------------------------------
struct ToiXf {
    V3 fwd, right, up, origin;
};
RG_HDI ToiXf toi_integrate(const ToiXf& t, V3 lin, V3 ang, float dt) {
    ToiXf o = t;
    o.origin = V3{dt * lin.x + t.origin.x, dt * lin.y + t.origin.y, dt * lin.z + t.origin.z};
    Q4 q{1.0f, 0.0f, 0.0f, 0.0f};
    game_integrate_orientation(o.fwd, o.right, o.up, q, ang, dt);
    return o;
}
RG_HDI V3 toi_angular_velocity(const ToiXf& t0, const ToiXf& t1) {
    const float m00 = t0.fwd.x, m01 = t0.right.x, m02 = t0.up.x;
    const float m10 = t0.fwd.y, m11 = t0.right.y, m12 = t0.up.y;
    const float m20 = t0.fwd.z, m21 = t0.right.z, m22 = t0.up.z;
    const float co0 = m11 * m22 - m12 * m21, co1 = m12 * m20 - m10 * m22, co2 = m10 * m21 - m11 * m20;
    const float s = 1.0f / ((m00 * co0 + m01 * co1) + m02 * co2);
    const float i00 = co0 * s, i01 = (m02 * m21 - m01 * m22) * s, i02 = (m01 * m12 - m02 * m11) * s;
    const float i10 = co1 * s, i11 = (m00 * m22 - m02 * m20) * s, i12 = (m02 * m10 - m00 * m12) * s;
    const float i20 = co2 * s, i21 = (m01 * m20 - m00 * m21) * s, i22 = (m00 * m11 - m01 * m10) * s;
    auto row = [&](float b0, float b1, float b2) {
        return V3{(i00 * b0 + i10 * b1) + i20 * b2, (i01 * b0 + i11 * b1) + i21 * b2,
                  (i02 * b0 + i12 * b1) + i22 * b2};
    };
    const V3 d0 = row(t1.fwd.x, t1.right.x, t1.up.x);
    const V3 d1 = row(t1.fwd.y, t1.right.y, t1.up.y);
    const V3 d2 = row(t1.fwd.z, t1.right.z, t1.up.z);
    const Q4 q = game_quat_normalize(
        game_rot_from_basis(V3{d0.x, d1.x, d2.x}, V3{d0.y, d1.y, d2.y}, V3{d0.z, d1.z, d2.z}), -1.0f);
    float w = q.w;
    w = -1.0f <= w ? w : -1.0f;
    w = w <= 1.0f ? w : 1.0f;
    const float half = ucrt_acosf(w);
    const float angle = half + half;
    const float l2 = (q.x * q.x + q.y * q.y) + q.z * q.z;
    V3 axis{1.0f, 0.0f, 0.0f};
    if (l2 >= 1.42108547e-14f) {
        const float inv = 1.0f / sqrtf(l2);
        axis = V3{inv * q.x, q.y * inv, inv * q.z};
    }
    return V3{axis.x * angle, axis.y * angle, axis.z * angle};
}
RG_HDI float toi_angular_motion_disc(const gjk::Shape& box) {
    const float m = box.margin;
    const float ex = box.half.x + m, ey = box.half.y + m, ez = box.half.z + m;
    const float dx = ex - -ex, dy = ey - -ey, dz = ez - -ez;
    return sqrtf((dx * dx + dy * dy) + dz * dz) * 0.5f;
}
RG_HDI Q4 ue_quat_slerp(Q4 q1, Q4 q2, float t) {
    const float raw = ((q1.x * q2.x + q1.y * q2.y) + q1.z * q2.z) + q1.w * q2.w;
    const float cosom = raw >= 0.0f ? raw : -raw;
    float s0, s1;
    if (cosom < 0.9999f) {
        const float c = -1.0f > cosom ? -1.0f : (cosom < 1.0f ? cosom : 1.0f);
        const float omega = ucrt_acosf(c);
        const float inv_sin = 1.0f / ucrt_sinf(omega);
        s0 = ucrt_sinf((1.0f - t) * omega) * inv_sin;
        s1 = ucrt_sinf(omega * t) * inv_sin;
    } else {
        s0 = 1.0f - t;
        s1 = t;
    }
    if (!(raw >= 0.0f)) s1 = -s1;
    return Q4{s1 * q2.w + q1.w * s0, s1 * q2.x + q1.x * s0, s1 * q2.y + q1.y * s0, s1 * q2.z + q1.z * s0};
}
RG_HDI gjk::Xform toi_xform(const ToiXf& t) { return gjk::basis_xform(t.fwd, t.right, t.up, t.origin); }
// the box's AABB centre in a transform (btBoxShape::getAabb)
RG_HDI V3 toi_aabb_center(const gjk::Shape& s, const gjk::Xform& x) {
    const V3 h = s.half + V3{s.margin, s.margin, s.margin};
    const V3 e{gjk::bdot(V3{fabs_(x.b.r[0].x), fabs_(x.b.r[0].y), fabs_(x.b.r[0].z)}, h),
               gjk::bdot(V3{fabs_(x.b.r[1].x), fabs_(x.b.r[1].y), fabs_(x.b.r[1].z)}, h),
               gjk::bdot(V3{fabs_(x.b.r[2].x), fabs_(x.b.r[2].y), fabs_(x.b.r[2].z)}, h)};
    return ((x.o + e) + (x.o - e)) * 0.5f;
}
// Closest points of the two boxes (reference CarToiClosestPoints): the GJK pair detector, EPA when they touch.
RG_NOINL bool toi_closest_points(const gjk::Shape& sa, const ToiXf& ca, const gjk::Shape& sb, const ToiXf& cb,
                                 float& out_distance, V3& out_normal, V3& out_point) {
    using namespace gjk;
    constexpr float kMaxDistSq = 1.0e18f;
    const float margin_a = sa.margin, margin_b = sb.margin;
    Xform xa = toi_xform(ca), xb = toi_xform(cb);
    const V3 offset = (xa.o + xb.o) * 0.5f;
    xa.o = xa.o - offset;
    xb.o = xb.o - offset;
    V3 cached{0.0f, 1.0f, 0.0f};
    float sq = 1.0e30f;
    bool valid = false;
    int degenerate = 0;
    float distance = 0.0f;
    V3 normal{0.0f, 0.0f, 0.0f}, pa{0.0f, 0.0f, 0.0f}, pb{0.0f, 0.0f, 0.0f};
    if (!pair_detector(sa, xa, sb, xb, kMaxDistSq, cached, degenerate, sq, pa, pb)) return false;
    const float l2 = len2(cached);
    if (l2 <= 0.0001f) degenerate = 5;
    const float s = sqrtf(sq);
    if (l2 > 1.1920929e-7f * 1.1920929e-7f) {
        const float inv_len = 1.0f / sqrtf(l2);
        normal = cached * inv_len;
        if (s > 0.0f) {
            pa = pa - cached * (margin_a / s);
            pb = pb + cached * (margin_b / s);
            distance = (1.0f / inv_len) - (margin_a + margin_b);
            valid = true;
        }
    }
    if (!valid || (degenerate && ((distance + (margin_a + margin_b)) <= 0.01f))) {
        const V3 delta_origin = xb.o - xa.o;
        const float dl2 = blen2(delta_origin);
        const V3 guess = dl2 > 1.0e-20f ? bdiv(delta_origin, sqrtf(dl2)) : V3{0.0f, 0.0f, 0.0f};
        Results r;
        V3 sep{0.0f, 0.0f, 0.0f}, wa{0.0f, 0.0f, 0.0f}, wb{0.0f, 0.0f, 0.0f};
        bool pen = false;
        if (penetration(sa, xa, sb, xb, guess, r)) {
            wa = r.witness0;
            wb = r.witness1;
            sep = r.normal;
            pen = true;
        } else if (gjk::distance(sa, xa, sb, xb, guess, r)) {
            wa = r.witness0;
            wb = r.witness1;
            sep = r.normal;
        }
        if (pen) {
            V3 tn = wb - wa;
            float lp = blen2(tn);
            if (lp <= 1.1920929e-7f * 1.1920929e-7f) {
                tn = sep;
                lp = blen2(sep);
            }
            if (lp > 1.1920929e-7f * 1.1920929e-7f) {
                tn = bdiv(tn, sqrtf(lp));
                const float d2 = -len(wa - wb);
                if (!valid || d2 < distance) {
                    distance = d2;
                    pa = wa;
                    pb = wb;
                    normal = tn;
                    valid = true;
                }
            }
        } else if (blen2(sep) > 0.0f) {
            const float d2 = len(wa - wb) - (margin_a + margin_b);
            if (!valid || d2 < distance) {
                pa = wa - sep * margin_a;
                pb = wb + sep * margin_b;
                normal = normalize_fallback(sep, normal);
                distance = d2;
                valid = true;
            }
        }
    }
    if (!valid || !((distance < 0.0f) || (distance * distance < kMaxDistSq))) return false;
    {
        const V3 ca_ = toi_aabb_center(sa, xa), cb_ = toi_aabb_center(sb, xb);
        V3 nb = normal;
        if (bdot(ca_ - cb_, nb) < 0.0f) nb = nb * -1.0f;
        out_normal = nb;
    }
    out_point = pb + offset;
    out_distance = distance;
    return distance < 1.0e18f;
}
// Both cars moved back to the moment their hitboxes first touched within this tick (reference CarCarTimeOfImpact):
// conservative advancement over the tick's motion from the start velocities; the poses stay put when no impact is
// found.
RG_NOINL void car_car_time_of_impact(const CarState& a, const CarConfig& acfg, V3 a_vel, const CarState& v,
                                     const CarConfig& vcfg, V3 v_vel, float dt, V3& pos_a, Q4& rot_a, V3& pos_v,
                                     Q4& rot_v) {
    constexpr float kAllowed = 0.04f;
    constexpr float kEps = 1.1920929e-7f;
    constexpr float kUuToBtF = 1.0f / 50.0f;
    auto sweep = [&](const CarState& s, V3 vel, ToiXf& from, ToiXf& to) {
        ToiXf t0;
        game_basis_from_rot(s.rot, t0.fwd, t0.right, t0.up);
        t0.origin = V3{s.pos.x * kUuToBtF, s.pos.y * kUuToBtF, s.pos.z * kUuToBtF};
        const V3 lin{vel.x * kUuToBtF, vel.y * kUuToBtF, vel.z * kUuToBtF};
        from = toi_integrate(t0, V3{-lin.x, -lin.y, -lin.z}, V3{-s.ang_vel.x, -s.ang_vel.y, -s.ang_vel.z}, dt);
        to = toi_integrate(t0, lin, s.ang_vel, dt);
    };
    auto child = [&](const ToiXf& t, const CarConfig& cfg) {
        ToiXf c = t;
        c.origin = gjk::xform(toi_xform(t), cfg.hitbox_offset * kUuToBtF);
        return c;
    };
    const gjk::Shape box_a = gjk::make_box((bullet_hitbox_size(acfg) * 0.5f) * kUuToBtF, 0.04f);
    const gjk::Shape box_b = gjk::make_box((bullet_hitbox_size(vcfg) * 0.5f) * kUuToBtF, 0.04f);
    ToiXf ca0, cb0;
    V3 lin_a, lin_b, ang_a, ang_b;
    {
        ToiXf fa, ta, fb, tb;
        sweep(a, a_vel, fa, ta);
        sweep(v, v_vel, fb, tb);
        ca0 = child(fa, acfg);
        const ToiXf ca1 = child(ta, acfg);
        cb0 = child(fb, vcfg);
        const ToiXf cb1 = child(tb, vcfg);
        lin_a = V3{ca1.origin.x - ca0.origin.x, ca1.origin.y - ca0.origin.y, ca1.origin.z - ca0.origin.z};
        lin_b = V3{cb1.origin.x - cb0.origin.x, cb1.origin.y - cb0.origin.y, cb1.origin.z - cb0.origin.z};
        ang_a = toi_angular_velocity(ca0, ca1);
        ang_b = toi_angular_velocity(cb0, cb1);
    }
    const float max_ang = sqrtf((ang_a.x * ang_a.x + ang_a.y * ang_a.y) + ang_a.z * ang_a.z) *
                              toi_angular_motion_disc(box_a) +
                          sqrtf((ang_b.x * ang_b.x + ang_b.y * ang_b.y) + ang_b.z * ang_b.z) *
                              toi_angular_motion_disc(box_b);
    const V3 rel{lin_b.x - lin_a.x, lin_b.y - lin_a.y, lin_b.z - lin_a.z};
    if (sqrtf((rel.x * rel.x + rel.y * rel.y) + rel.z * rel.z) + max_ang == 0.0f) return;
    float d = 0.0f;
    V3 n{0.0f, 0.0f, 0.0f}, cpt{0.0f, 0.0f, 0.0f};
    if (!toi_closest_points(box_a, ca0, box_b, cb0, d, n, cpt)) return;
    float dist = d + kAllowed;
    if (((rel.x * n.x + rel.y * n.y) + rel.z * n.z) + max_ang <= kEps) return;
    float lambda = 0.0f, fraction = 0.0f;
    int iter = 0;
    while (dist > 0.001f) {
        const float proj = ((rel.x * n.x + rel.y * n.y) + rel.z * n.z) + max_ang;
        if (proj <= kEps) return;
        fraction = lambda + dist / proj;
        if (fraction > 1.0f || fraction < 0.0f || fraction <= lambda) return;
        const ToiXf ia = toi_integrate(ca0, lin_a, ang_a, fraction);
        const ToiXf ib = toi_integrate(cb0, lin_b, ang_b, fraction);
        if (!toi_closest_points(box_a, ia, box_b, ib, d, n, cpt)) return;
        dist = d + kAllowed;
        if (++iter > 64) return;
        lambda = fraction;
    }
    if (!(fraction < 1.0f)) return;
    auto pose = [&](V3& pos, Q4& rot, const CarState& s, V3 vel) {
        ToiXf from, to;
        sweep(s, vel, from, to);
        pos = V3{(to.origin.x * 50.0f - from.origin.x * 50.0f) * fraction + from.origin.x * 50.0f,
                 (to.origin.y * 50.0f - from.origin.y * 50.0f) * fraction + from.origin.y * 50.0f,
                 (to.origin.z * 50.0f - from.origin.z * 50.0f) * fraction + from.origin.z * 50.0f};
        rot = game_quat_normalize(ue_quat_slerp(game_rot_from_basis(from.fwd, from.right, from.up),
                                                game_rot_from_basis(to.fwd, to.right, to.up), fraction),
                                  1e-8f);
    };
    pose(pos_a, rot_a, a, a_vel);
    pose(pos_v, rot_v, v, v_vel);
}
// reference ShouldDemolish with the victim's start velocity
RG_HDI bool should_demolish(const CarState& a, const CarConfig& acfg, V3 a_start_vel, const CarState& v,
                            const CarConfig& vcfg, V3 v_start_vel, const TickConfig& tc) {
    if (!a.is_supersonic) return false;
    const V3 fwd = ue3_rotator_forward(ue3_quat_to_rotator(a.rot));
    const float fs = dot(a_start_vel, fwd);
    const bool reverse = fs < 0.0f;
    if (fabsf(fs) < tc.supersonic_maintain_min_speed) return false;
    V3 pa = a.pos, pv = v.pos;
    Q4 ra = a.rot, rv = v.rot;
    car_car_time_of_impact(a, acfg, a_start_vel, v, vcfg, v_start_vel, tc.tick_dt, pa, ra, pv, rv);
    return in_forward_cone(pa, ra, acfg, pv, rv, vcfg, reverse, 45.5729942f);
}

// The hitter's bumper cone: a demolition when supersonic (not this tick's path: the demolition test above already
// ran), else a bump impulse queued on the victim (reference BumpCone).
RG_HDI bool bump_cone(CarState& h, uint32_t hid, uint8_t hteam, const CarConfig& hcfg, V3 h_start_vel, CarState& v,
                      uint32_t vid, const CarConfig& vcfg, const TickConfig& tc) {
    const bool bumper = in_forward_cone(h.pos, h.rot, hcfg, v.pos, v.rot, vcfg, false, 70.0f);
    if (bumper) {
        const float speed = sqrtf(len2(h_start_vel));
        const V3 vel_dir = h_start_vel * (1.0f / speed);
        auto curve = [speed](float y0, float y1, float y2) {
            if (speed <= 0.0f) return y0;
            if (speed < 1400.0f) return y0 + (y1 - y0) * (speed / 1400.0f);
            if (speed < 2200.0f) return y1 + (y2 - y1) * ((speed - 1400.0f) / 800.0f);
            return y2;
        };
        V3 impulse;
        if (v.is_on_ground != 0) {
            const V3 up_dir = ue3_rotator_up_axis(ue3_quat_to_rotator(v.rot));
            impulse = vel_dir * curve(150.0f, 200000.0f, 275000.0f) + up_dir * curve(50.0f, 50000.0f, 75000.0f);
        } else {
            impulse = vel_dir * curve(150.0f, 250000.0f, 350000.0f);
        }
        const V3 impulse_bt = ((impulse * tc.bump_force_scale) * (1.0f / 50.0f)) * (1.0f / tc.car_mass);
        v.vel_impulse_cache_bt += impulse_bt;
        v.vel_impulse_cache += impulse_bt * 50.0f;
        if (v.pending_bump_count < 7) {
            int slot = v.pending_bump_count++;
            for (; slot > 0 && v.pending_bump_hitter[slot - 1] > hid; --slot) {
                v.pending_bump_bt[slot] = v.pending_bump_bt[slot - 1];
                v.pending_bump_hitter[slot] = v.pending_bump_hitter[slot - 1];
            }
            v.pending_bump_bt[slot] = impulse_bt;
            v.pending_bump_hitter[slot] = hid;
        }
    }
    h.car_contact.other_car_id = vid;
    h.car_contact.cooldown_timer = tc.bump_cooldown_time + tc.tick_dt * 0.5f;
    if (bumper) record_car_hit(h, hid, vid, false, hteam, tc.events);
    return false;
}

// One direction of a car pair's game contact (reference ResolveCarCarDirectionalContact with the start velocities).
RG_HDI bool car_car_directional(CarState& h, uint32_t hid, uint8_t hteam, const CarConfig& hcfg, CarState& v,
                                uint32_t vid, uint8_t vteam, const CarConfig& vcfg, V3 h_start_vel, V3 v_start_vel,
                                bool demo_only, const TickConfig& tc) {
    if ((h.is_demoed && !demo_only) || v.is_demoed || h.just_respawned || v.just_respawned) return false;
    const bool in_cooldown = h.car_contact.other_car_id == vid && h.car_contact.cooldown_timer > 0.0f;
    const V3 vel = h_start_vel;
    const float speed = sqrtf(len2(vel));
    if (!(speed > 0.0f)) return false;
    const V3 dpos = v.pos - h.pos;
    V3 hit_dir{0.0f, 0.0f, 0.0f};
    {
        const float l2 = len2(dpos);
        const float l = l2 > 0.0f ? sqrtf(l2) : 0.0f;
        if (l > 1.1920928955078125e-7f * 1.1920928955078125e-7f) hit_dir = V3{dpos.x / l, dpos.y / l, dpos.z / l};
    }
    const float towards = dot(hit_dir, vel);
    if (towards <= 0.0f) return false;
    const V3 vel_dir = vel * (1.0f / speed);
    if (dot(v_start_vel, vel_dir) >= towards) return false;
    bool demo = tc.enable_demos && should_demolish(h, hcfg, vel, v, vcfg, v_start_vel, tc);
    if (demo && !tc.enable_team_demos) demo = hteam != vteam;
    if (demo) {
        demolish_car(v, tc);
        record_car_hit(h, hid, vid, true, hteam, tc.events);
        return true;
    }
    if (in_cooldown) return false;
    return bump_cone(h, hid, hteam, hcfg, vel, v, vid, vcfg, tc);
}

// A car pair's contact for this tick (reference ResolveCarCarCollisionImpl<shared rows>): the retained manifold, the
// game's bumps and demolitions in both directions, then the pair's rows. `ia`/`ib` are the cars' slots in the arena.
RG_NOINL void car_car_resolve(CarState& a, uint32_t id_a, uint8_t team_a, const CarConfig& ca, CarState& b,
                              uint32_t id_b, uint8_t team_b, const CarConfig& cb, const TickConfig& tc,
                              const PreContactCar& pa, const PreContactCar& pb, V3 start_a, V3 start_b, int ia,
                              int ib, CarCarManifold& m, CarCarRows& rows) {
    if (a.is_demoed || b.is_demoed || a.just_respawned || b.just_respawned) {
        m.count = 0;
        return;
    }
    const float md = car_bounding_sphere_radius(ca) + car_bounding_sphere_radius(cb);
    V3 normal{1.0f, 0.0f, 0.0f};
    int demo_count = 0;
    float xa[4], xb[4];
    if (!car_car_prepare(a, ca, b, cb, md * md, m, normal, demo_count, xa, xb)) return;
    if (demo_count > 0) {
        const bool a_lower = id_a > id_b;
        CarState& h1 = a_lower ? a : b;
        CarState& v1 = a_lower ? b : a;
        const uint32_t h1_id = a_lower ? id_a : id_b, v1_id = a_lower ? id_b : id_a;
        const uint8_t h1_team = a_lower ? team_a : team_b, v1_team = a_lower ? team_b : team_a;
        const CarConfig& h1_cfg = a_lower ? ca : cb;
        const CarConfig& v1_cfg = a_lower ? cb : ca;
        const V3 h1_start = a_lower ? start_a : start_b, v1_start = a_lower ? start_b : start_a;
        bool h1_demoed_here = false, v1_demoed_here = false;
        for (int k = 0; k < demo_count; ++k) {
            if (a.is_demoed && b.is_demoed) break;
            if (!v1.is_demoed && (!h1.is_demoed || h1_demoed_here)) {
                car_car_directional(h1, h1_id, h1_team, h1_cfg, v1, v1_id, v1_team, v1_cfg, h1_start, v1_start,
                                    h1.is_demoed != 0, tc);
                v1_demoed_here = v1_demoed_here || v1.is_demoed;
            }
            if (a.is_demoed && b.is_demoed) break;
            if (!h1.is_demoed && (!v1.is_demoed || v1_demoed_here)) {
                car_car_directional(v1, v1_id, v1_team, v1_cfg, h1, h1_id, h1_team, h1_cfg, v1_start, h1_start,
                                    v1.is_demoed != 0, tc);
                h1_demoed_here = h1_demoed_here || h1.is_demoed;
            }
        }
    }
    car_car_rows(a, b, ca, cb, tc, pa, pb, tc.tick_dt, ia, ib, m, rows);
    if (m.count > 0) {
        // the pair's rows write each car's velocity, angular velocity and origin back (reference
        // EmitSharedCarCarContactRows, env_step.hpp:665-680): unchanged for finite values except the origin's uu copy,
        // recomputed from bt, which later bumps and the car's events read
        auto write_back = [](CarState& c) {
            const V3 dv = c.vel - c.vel;
            if (dv.x != 0.0f || dv.y != 0.0f || dv.z != 0.0f) car_set_vel_uu(c, c.vel + dv);
            c.ang_vel = c.ang_vel + (c.ang_vel - c.ang_vel);
            car_set_pos_bt(c, c.pos_bt + (c.pos_bt - c.pos_bt));
        };
        write_back(a);
        write_back(b);
    }
}

}  // namespace rg

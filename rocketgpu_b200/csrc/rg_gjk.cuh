// Convex-convex distance and penetration for the car's hitbox against arena triangles, host+device.
//
// Three published algorithms, restated in the reference's float operation order (Bullet Physics 2.8x, zlib licence):
//   * the Voronoi-region simplex solver and the GJK pair-detector loop (btVoronoiSimplexSolver / btGjkPairDetector),
//     as the reference drives it for a box against a triangle (GjkSimplexSolver,
//     include/rocketgpu/detail/step/raycast_wheels_and_contact_prep.hpp:4090-4470; RunCarArenaTriangleGjkSimplex,
//     triangle_and_carcar.hpp:206-300);
//   * btGjkEpa2's GJK and EPA (include/rocketgpu/detail/bullet_gjk_epa2_port.hpp:560-1730), used as the penetration
//     depth solver when the shapes overlap (BulletPortCalcPenDepth, triangle_and_carcar.hpp:100-157);
//   * the contact point / distance assembly of ComputeCarArenaTriangleContact (triangle_and_carcar.hpp:301-535).
// EPA's recursive horizon expansion is written with an explicit stack; its polytope (64 vertices, 128 faces) lives in
// the calling thread's local memory.
#pragma once

#include "rg_math.cuh"

namespace rg {
namespace gjk {

// ---- Bullet-style vector ops (division multiplies by the reciprocal, as btVector3 does) ------------------------------
RG_HD float bdot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
RG_HD V3 bcross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
RG_HD float blen2(V3 a) { return bdot(a, a); }
RG_HD float blen(V3 a) { return sqrtf(blen2(a)); }
RG_HD V3 bdiv(V3 a, float s) {
    const float inv = 1.0f / s;
    return V3{a.x * inv, a.y * inv, a.z * inv};
}
RG_HD V3 bnormalized(V3 v) {  // btVector3::normalize (no-op below 1e-20)
    const float l2 = blen2(v);
    return l2 > 1.0e-20f ? bdiv(v, sqrtf(l2)) : v;
}
RG_HD float comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
RG_HD void set_comp(V3& v, int i, float s) {
    if (i == 0) v.x = s;
    else if (i == 1) v.y = s;
    else v.z = s;
}

// Rows of a 3x3 matrix and a rigid transform (btMatrix3x3 / btTransform semantics).
struct Mat3 {
    V3 r[3];
};
struct Xform {
    Mat3 b;
    V3 o;
};
RG_HD V3 mat_mul(const Mat3& m, V3 v) { return V3{bdot(m.r[0], v), bdot(m.r[1], v), bdot(m.r[2], v)}; }
RG_HD V3 vec_mul_mat(V3 v, const Mat3& m) {  // v * M
    return V3{m.r[0].x * v.x + m.r[1].x * v.y + m.r[2].x * v.z, m.r[0].y * v.x + m.r[1].y * v.y + m.r[2].y * v.z,
              m.r[0].z * v.x + m.r[1].z * v.y + m.r[2].z * v.z};
}
RG_HD Mat3 transpose_times(const Mat3& a, const Mat3& m) {  // a^T * m
    Mat3 o;
    const float c[3][3] = {{a.r[0].x, a.r[1].x, a.r[2].x}, {a.r[0].y, a.r[1].y, a.r[2].y}, {a.r[0].z, a.r[1].z, a.r[2].z}};
    for (int i = 0; i < 3; ++i)
        o.r[i] = V3{c[i][0] * m.r[0].x + c[i][1] * m.r[1].x + c[i][2] * m.r[2].x,
                    c[i][0] * m.r[0].y + c[i][1] * m.r[1].y + c[i][2] * m.r[2].y,
                    c[i][0] * m.r[0].z + c[i][1] * m.r[1].z + c[i][2] * m.r[2].z};
    return o;
}
RG_HD V3 xform(const Xform& t, V3 v) {  // t * v = (v . b0, v . b1, v . b2) + o
    return V3{bdot(v, t.b.r[0]), bdot(v, t.b.r[1]), bdot(v, t.b.r[2])} + t.o;
}
RG_HD Xform inverse_times(const Xform& t, const Xform& other) {
    Xform out;
    out.b = transpose_times(t.b, other.b);
    out.o = vec_mul_mat(other.o - t.o, t.b);
    return out;
}
RG_HD V3 inv_xform(const Xform& t, V3 v) {
    const V3 d = v - t.o;
    const V3 c0{t.b.r[0].x, t.b.r[1].x, t.b.r[2].x};
    const V3 c1{t.b.r[0].y, t.b.r[1].y, t.b.r[2].y};
    const V3 c2{t.b.r[0].z, t.b.r[1].z, t.b.r[2].z};
    return V3{bdot(c0, d), bdot(c1, d), bdot(c2, d)};
}

// ---- shapes: a box (half extents without margin + margin) and a triangle -----------------------------------------
enum ShapeKind : uint8_t { kTriangle = 0, kBox = 1, kSphere = 2 };
struct Shape {
    uint8_t kind;
    V3 half;      // box: implicit dimensions
    V3 v[3];      // triangle vertices
    float margin; // sphere: the radius
};
RG_HD V3 support_no_margin(const Shape& s, V3 d) {
    if (s.kind == kBox) {
        return V3{d.x >= 0.0f ? s.half.x : -s.half.x, d.y >= 0.0f ? s.half.y : -s.half.y,
                  d.z >= 0.0f ? s.half.z : -s.half.z};
    }
    if (s.kind == kSphere) return V3{0.0f, 0.0f, 0.0f};
    const V3 dots{bdot(d, s.v[0]), bdot(d, s.v[1]), bdot(d, s.v[2])};
    const int ax = dots.x < dots.y ? (dots.y < dots.z ? 2 : 1) : (dots.x < dots.z ? 2 : 0);
    return s.v[ax];
}
RG_HD V3 support_margin(const Shape& s, V3 d) {
    V3 n = d;
    if (blen2(n) < (1.1920929e-7f * 1.1920929e-7f)) n = V3{-1.0f, -1.0f, -1.0f};
    n = bnormalized(n);
    return support_no_margin(s, n) + n * s.margin;
}
// The reference's box shape from half extents with the margin included (MakeBulletPortBoxShape).
RG_HDI Shape make_box(V3 half_with_margin, float margin) {
    Shape s;
    s.kind = kBox;
    const float min_dim = fmin_(half_with_margin.x, fmin_(half_with_margin.y, half_with_margin.z));
    const float safe_margin = fmin_(margin, 0.1f * min_dim);
    s.half = half_with_margin - V3{safe_margin, safe_margin, safe_margin};
    s.margin = safe_margin;
    s.v[0] = s.v[1] = s.v[2] = V3{0.0f, 0.0f, 0.0f};
    return s;
}
RG_HDI Shape make_sphere(float radius) {
    Shape s;
    s.kind = kSphere;
    s.half = V3{0.0f, 0.0f, 0.0f};
    s.v[0] = s.v[1] = s.v[2] = V3{0.0f, 0.0f, 0.0f};
    s.margin = radius;
    return s;
}
RG_HDI Shape make_triangle(V3 a, V3 b, V3 c) {
    Shape s;
    s.kind = kTriangle;
    s.half = V3{0.0f, 0.0f, 0.0f};
    s.v[0] = a;
    s.v[1] = b;
    s.v[2] = c;
    s.margin = 0.0f;
    return s;
}

// ---- btGjkEpa2 ---------------------------------------------------------------------------------------------------
constexpr int kGjkMaxIterations = 128;
constexpr float kGjkAccuracy = 0.0001f;
constexpr float kGjkMinDistance = 0.0001f;
constexpr float kGjkDuplicatedEps = 0.0001f;
constexpr int kEpaMaxVertices = 64;
constexpr int kEpaMaxIterations = 255;
constexpr float kEpaAccuracy = 0.0001f;
constexpr float kEpaPlaneEps = 0.00001f;
constexpr int kEpaMaxFaces = kEpaMaxVertices * 2;

struct Minkowski {
    const Shape* s0;
    const Shape* s1;
    Mat3 to1;   // shape1 <- shape0 rotation
    Xform to0;  // shape0 <- shape1 transform
    bool margins;
    RG_HD V3 support0(V3 d) const { return margins ? support_margin(*s0, d) : support_no_margin(*s0, d); }
    RG_HD V3 support1(V3 d) const {
        const V3 l = mat_mul(to1, d);
        return xform(to0, margins ? support_margin(*s1, l) : support_no_margin(*s1, l));
    }
    RG_HD V3 support(V3 d) const { return support0(d) - support1(-d); }
};
RG_HDI Minkowski make_minkowski(const Shape& s0, const Xform& w0, const Shape& s1, const Xform& w1, bool margins) {
    Minkowski m;
    m.s0 = &s0;
    m.s1 = &s1;
    m.to1 = transpose_times(w1.b, w0.b);
    m.to0 = inverse_times(w0, w1);
    m.margins = margins;
    return m;
}

struct SV {
    V3 d, w;
};
struct Simplex {
    int c[4];  // indices into the vertex store
    float p[4];
    int rank;
};

enum GjkStatus { kGjkValid, kGjkInside, kGjkFailed };

struct Gjk {
    Minkowski shape;
    V3 ray;
    float distance;
    Simplex simplices[2];
    SV store[4];
    int free_[4];
    int nfree;
    int current;
    int simplex;  // index of the result simplex
    GjkStatus status;

    RG_HD void getsupport(V3 d, SV& sv) const {
        sv.d = bdiv(d, blen(d));
        sv.w = shape.support(sv.d);
    }
    RG_HD void removevertice(Simplex& s) { free_[nfree++] = s.c[--s.rank]; }
    RG_HD void appendvertice(Simplex& s, V3 v) {
        s.p[s.rank] = 0.0f;
        s.c[s.rank] = free_[--nfree];
        getsupport(v, store[s.c[s.rank++]]);
    }
    RG_HD static float det(V3 a, V3 b, V3 c) {
        return (a.y * b.z * c.x + a.z * b.x * c.y - a.x * b.z * c.y - a.y * b.x * c.z + a.x * b.y * c.z -
                a.z * b.y * c.x);
    }
    RG_HDI static float project2(V3 a, V3 b, float* w, unsigned& m) {
        const V3 d = b - a;
        const float l = blen2(d);
        if (l > 0.0f) {
            const float t = l > 0.0f ? -bdot(a, d) / l : 0.0f;
            if (t >= 1.0f) {
                w[0] = 0.0f;
                w[1] = 1.0f;
                m = 2;
                return blen2(b);
            } else if (t <= 0.0f) {
                w[0] = 1.0f;
                w[1] = 0.0f;
                m = 1;
                return blen2(a);
            } else {
                w[1] = t;
                w[0] = 1.0f - t;
                m = 3;
                return blen2(a + d * t);
            }
        }
        return -1.0f;
    }
    RG_HDI static float project3(V3 a, V3 b, V3 c, float* w, unsigned& m) {
        const int imd3[3] = {1, 2, 0};
        const V3 vt[3] = {a, b, c};
        const V3 dl[3] = {a - b, b - c, c - a};
        const V3 n = bcross(dl[0], dl[1]);
        const float l = blen2(n);
        if (l > 0.0f) {
            float mindist = -1.0f;
            float subw[2] = {0.0f, 0.0f};
            unsigned subm = 0;
            for (int i = 0; i < 3; ++i) {
                if (bdot(vt[i], bcross(dl[i], n)) > 0.0f) {
                    const int j = imd3[i];
                    const float subd = project2(vt[i], vt[j], subw, subm);
                    if ((mindist < 0.0f) || (subd < mindist)) {
                        mindist = subd;
                        m = static_cast<unsigned>(((subm & 1) ? 1 << i : 0) + ((subm & 2) ? 1 << j : 0));
                        w[i] = subw[0];
                        w[j] = subw[1];
                        w[imd3[j]] = 0.0f;
                    }
                }
            }
            if (mindist < 0.0f) {
                const float d = bdot(a, n);
                const float s = sqrtf(l);
                const V3 p = n * (d / l);
                mindist = blen2(p);
                m = 7;
                w[0] = blen(bcross(dl[1], b - p)) / s;
                w[1] = blen(bcross(dl[2], c - p)) / s;
                w[2] = 1.0f - (w[0] + w[1]);
            }
            return mindist;
        }
        return -1.0f;
    }
    RG_HDI static float project4(V3 a, V3 b, V3 c, V3 d, float* w, unsigned& m) {
        const int imd3[3] = {1, 2, 0};
        const V3 vt[4] = {a, b, c, d};
        const V3 dl[3] = {a - d, b - d, c - d};
        const float vl = det(dl[0], dl[1], dl[2]);
        const bool ng = (vl * bdot(a, bcross(b - c, a - b))) <= 0.0f;
        if (ng && (fabs_(vl) > 0.0f)) {
            float mindist = -1.0f;
            float subw[3] = {0.0f, 0.0f, 0.0f};
            unsigned subm = 0;
            for (int i = 0; i < 3; ++i) {
                const int j = imd3[i];
                const float s = vl * bdot(d, bcross(dl[i], dl[j]));
                if (s > 0.0f) {
                    const float subd = project3(vt[i], vt[j], d, subw, subm);
                    if ((mindist < 0.0f) || (subd < mindist)) {
                        mindist = subd;
                        m = static_cast<unsigned>((subm & 1 ? 1 << i : 0) + (subm & 2 ? 1 << j : 0) + (subm & 4 ? 8 : 0));
                        w[i] = subw[0];
                        w[j] = subw[1];
                        w[imd3[j]] = 0.0f;
                        w[3] = subw[2];
                    }
                }
            }
            if (mindist < 0.0f) {
                mindist = 0.0f;
                m = 15;
                w[0] = det(c, b, d) / vl;
                w[1] = det(a, c, d) / vl;
                w[2] = det(b, a, d) / vl;
                w[3] = 1.0f - (w[0] + w[1] + w[2]);
            }
            return mindist;
        }
        return -1.0f;
    }

    RG_HDI GjkStatus evaluate(V3 guess) {
        int iterations = 0;
        float sqdist = 0.0f;
        float alpha = 0.0f;
        V3 lastw[4];
        int clastw = 0;
        for (int i = 0; i < 4; ++i) free_[i] = i;
        nfree = 4;
        current = 0;
        status = kGjkValid;
        distance = 0.0f;
        simplices[0].rank = 0;
        ray = guess;
        const float sqrl = blen2(ray);
        appendvertice(simplices[0], sqrl > 0.0f ? -ray : V3{1.0f, 0.0f, 0.0f});
        simplices[0].p[0] = 1.0f;
        ray = store[simplices[0].c[0]].w;
        sqdist = sqrl;
        lastw[0] = lastw[1] = lastw[2] = lastw[3] = ray;
        do {
            const int next = 1 - current;
            Simplex& cs = simplices[current];
            Simplex& ns = simplices[next];
            const float rl = blen(ray);
            if (rl < kGjkMinDistance) {
                status = kGjkInside;
                break;
            }
            appendvertice(cs, -ray);
            const V3 w = store[cs.c[cs.rank - 1]].w;
            bool found = false;
            for (int i = 0; i < 4; ++i) {
                if (blen2(w - lastw[i]) < kGjkDuplicatedEps) {
                    found = true;
                    break;
                }
            }
            if (found) {
                removevertice(simplices[current]);
                break;
            }
            clastw = (clastw + 1) & 3;
            lastw[clastw] = w;
            const float omega = bdot(ray, w) / rl;
            alpha = omega > alpha ? omega : alpha;
            if (((rl - alpha) - (kGjkAccuracy * rl)) <= 0.0f) {
                removevertice(simplices[current]);
                break;
            }
            float weights[4];
            unsigned mask = 0;
            switch (cs.rank) {
                case 2: sqdist = project2(store[cs.c[0]].w, store[cs.c[1]].w, weights, mask); break;
                case 3: sqdist = project3(store[cs.c[0]].w, store[cs.c[1]].w, store[cs.c[2]].w, weights, mask); break;
                case 4:
                    sqdist = project4(store[cs.c[0]].w, store[cs.c[1]].w, store[cs.c[2]].w, store[cs.c[3]].w, weights,
                                      mask);
                    break;
            }
            if (sqdist >= 0.0f) {
                ns.rank = 0;
                ray = V3{0.0f, 0.0f, 0.0f};
                current = next;
                for (int i = 0, ni = cs.rank; i < ni; ++i) {
                    if (mask & (1u << i)) {
                        ns.c[ns.rank] = cs.c[i];
                        ns.p[ns.rank++] = weights[i];
                        ray += store[cs.c[i]].w * weights[i];
                    } else {
                        free_[nfree++] = cs.c[i];
                    }
                }
                if (mask == 15) status = kGjkInside;
            } else {
                removevertice(simplices[current]);
                break;
            }
            if ((++iterations) >= kGjkMaxIterations) status = kGjkFailed;
        } while (status == kGjkValid);
        simplex = current;
        switch (status) {
            case kGjkValid: distance = blen(ray); break;
            case kGjkInside: distance = 0.0f; break;
            default: break;
        }
        return status;
    }

    // Grow a degenerate simplex to a tetrahedron that encloses the origin (btGjkEpa2 EncloseOrigin).
    RG_HDI bool enclose4() {
        const Simplex& s = simplices[simplex];
        return fabs_(det(store[s.c[0]].w - store[s.c[3]].w, store[s.c[1]].w - store[s.c[3]].w,
                         store[s.c[2]].w - store[s.c[3]].w)) > 0.0f;
    }
    RG_HDI bool enclose3() {
        Simplex& s = simplices[simplex];
        const V3 n = bcross(store[s.c[1]].w - store[s.c[0]].w, store[s.c[2]].w - store[s.c[0]].w);
        if (blen2(n) > 0.0f) {
            appendvertice(s, n);
            if (enclose4()) return true;
            removevertice(s);
            appendvertice(s, -n);
            if (enclose4()) return true;
            removevertice(s);
        }
        return false;
    }
    RG_HDI bool enclose2() {
        Simplex& s = simplices[simplex];
        const V3 d = store[s.c[1]].w - store[s.c[0]].w;
        for (int i = 0; i < 3; ++i) {
            V3 axis{0.0f, 0.0f, 0.0f};
            set_comp(axis, i, 1.0f);
            const V3 p = bcross(d, axis);
            if (blen2(p) > 0.0f) {
                appendvertice(s, p);
                if (enclose3()) return true;
                removevertice(s);
                appendvertice(s, -p);
                if (enclose3()) return true;
                removevertice(s);
            }
        }
        return false;
    }
    RG_HDI bool enclose1() {
        Simplex& s = simplices[simplex];
        for (int i = 0; i < 3; ++i) {
            V3 axis{0.0f, 0.0f, 0.0f};
            set_comp(axis, i, 1.0f);
            appendvertice(s, axis);
            if (enclose2()) return true;
            removevertice(s);
            appendvertice(s, -axis);
            if (enclose2()) return true;
            removevertice(s);
        }
        return false;
    }
    RG_HDI bool enclose_origin() {
        switch (simplices[simplex].rank) {
            case 1: return enclose1();
            case 2: return enclose2();
            case 3: return enclose3();
            case 4: return enclose4();
        }
        return false;
    }
};

enum EpaStatus { kEpaValid, kEpaTouching, kEpaDegenerated, kEpaNonConvex, kEpaInvalidHull, kEpaOutOfFaces,
                 kEpaOutOfVertices, kEpaAccuracyReached, kEpaFallBack, kEpaFailed };

struct Epa {
    struct Face {
        V3 n;
        float d;
        int16_t c[3];  // vertex: 0..63 EPA store, 64+k GJK store k
        int16_t f[3];
        int16_t l[2];
        uint8_t e[3];
        uint8_t pass;
    };
    struct List {
        int16_t root;
        int count;
    };
    EpaStatus status;
    int16_t result_c[3];
    float result_p[3];
    int result_rank;
    V3 normal;
    float depth;
    SV sv_store[kEpaMaxVertices];
    Face fc[kEpaMaxFaces];
    int nextsv;
    // The free faces: `stock` holds the faces given back (most recent first), `fresh` the first never-used slot.
    // btGjkEpa2 links all faces into its stock at initialisation and takes the head; taking given-back faces first,
    // then fresh slots in index order, hands out the same faces in the same order without touching all 128.
    List hull, stock;
    int16_t fresh;
    const Gjk* gjk;

    RG_HD const SV& vtx(int16_t i) const { return i >= kEpaMaxVertices ? gjk->store[i - kEpaMaxVertices] : sv_store[i]; }
    RG_HD void bind(int16_t fa, int ea, int16_t fb, int eb) {
        fc[fa].e[ea] = static_cast<uint8_t>(eb);
        fc[fa].f[ea] = fb;
        fc[fb].e[eb] = static_cast<uint8_t>(ea);
        fc[fb].f[eb] = fa;
    }
    RG_HD void append(List& list, int16_t face) {
        fc[face].l[0] = -1;
        fc[face].l[1] = list.root;
        if (list.root >= 0) fc[list.root].l[0] = face;
        list.root = face;
        ++list.count;
    }
    RG_HD void remove(List& list, int16_t face) {
        if (fc[face].l[1] >= 0) fc[fc[face].l[1]].l[0] = fc[face].l[0];
        if (fc[face].l[0] >= 0) fc[fc[face].l[0]].l[1] = fc[face].l[1];
        if (face == list.root) list.root = fc[face].l[1];
        --list.count;
    }
    RG_HDI void initialize() {
        status = kEpaFailed;
        normal = V3{0.0f, 0.0f, 0.0f};
        depth = 0.0f;
        nextsv = 0;
        hull.root = stock.root = -1;
        hull.count = stock.count = 0;
        fresh = 0;
    }
    RG_HDI bool getedgedist(int16_t face, int16_t a, int16_t b, float& dist) {
        const V3 aw = vtx(a).w, bw = vtx(b).w;
        const V3 ba = bw - aw;
        const V3 n_ab = bcross(ba, fc[face].n);
        const float a_dot_nab = bdot(aw, n_ab);
        if (a_dot_nab < 0.0f) {
            const float ba_l2 = blen2(ba);
            const float a_dot_ba = bdot(aw, ba);
            const float b_dot_ba = bdot(bw, ba);
            if (a_dot_ba > 0.0f) {
                dist = blen(aw);
            } else if (b_dot_ba < 0.0f) {
                dist = blen(bw);
            } else {
                const float a_dot_b = bdot(aw, bw);
                const float v = (blen2(aw) * blen2(bw) - a_dot_b * a_dot_b) / ba_l2;
                dist = sqrtf(v > 0.0f ? v : 0.0f);
            }
            return true;
        }
        return false;
    }
    RG_HDI int16_t newface(int16_t a, int16_t b, int16_t c, bool forced) {
        if (stock.root >= 0 || fresh < kEpaMaxFaces) {
            int16_t face;
            if (stock.root >= 0) {
                face = stock.root;
                remove(stock, face);
            } else {
                face = fresh++;
            }
            append(hull, face);
            Face& F = fc[face];
            F.pass = 0;
            F.c[0] = a;
            F.c[1] = b;
            F.c[2] = c;
            F.n = bcross(vtx(b).w - vtx(a).w, vtx(c).w - vtx(a).w);
            const float l = blen(F.n);
            if (l > kEpaAccuracy) {
                if (!getedgedist(face, a, b, F.d) && !getedgedist(face, b, c, F.d) && !getedgedist(face, c, a, F.d)) {
                    F.d = bdot(vtx(a).w, F.n) / l;
                }
                F.n = bdiv(F.n, l);
                if (forced || (F.d >= -kEpaPlaneEps)) return face;
                status = kEpaNonConvex;
            } else {
                status = kEpaDegenerated;
            }
            remove(hull, face);
            append(stock, face);
            return -1;
        }
        status = kEpaOutOfFaces;
        return -1;
    }
    RG_HDI int16_t findbest() {
        int16_t minf = hull.root;
        float mind = fc[minf].d * fc[minf].d;
        for (int16_t f = fc[minf].l[1]; f >= 0; f = fc[f].l[1]) {
            const float sqd = fc[f].d * fc[f].d;
            if (sqd < mind) {
                minf = f;
                mind = sqd;
            }
        }
        return minf;
    }
    struct Horizon {
        int16_t cf, ff;
        int nf;
    };
    // Recursive horizon walk of btGjkEpa2 (expand) with an explicit stack of (face, edge, stage) frames.
    RG_HDI bool expand(int pass, int16_t w, int16_t f0, int e0, Horizon& horizon) {
        const int i1m3[3] = {1, 2, 0};
        const int i2m3[3] = {2, 0, 1};
        struct Frame {
            int16_t f;
            uint8_t e, stage;
        };
        Frame frames[kEpaMaxFaces];
        int sp = 0;
        frames[sp++] = Frame{f0, static_cast<uint8_t>(e0), 0};
        bool ret = false;
        while (sp > 0) {
            Frame& top = frames[sp - 1];
            Face& cf = fc[top.f];
            const int ce = top.e;
            if (top.stage == 0) {
                if (cf.pass != pass) {
                    const int e1 = i1m3[ce];
                    if ((bdot(cf.n, vtx(w).w) - cf.d) < -kEpaPlaneEps) {
                        const int16_t nf = newface(cf.c[e1], cf.c[ce], w, false);
                        if (nf >= 0) {
                            bind(nf, 0, top.f, ce);
                            if (horizon.cf >= 0)
                                bind(horizon.cf, 1, nf, 2);
                            else
                                horizon.ff = nf;
                            horizon.cf = nf;
                            ++horizon.nf;
                            ret = true;
                        } else {
                            ret = false;
                        }
                        --sp;
                        continue;
                    }
                    cf.pass = static_cast<uint8_t>(pass);
                    top.stage = 1;
                    if (sp < kEpaMaxFaces) {
                        frames[sp++] = Frame{cf.f[e1], cf.e[e1], 0};
                        continue;
                    }
                    ret = false;
                    --sp;
                    continue;
                }
                ret = false;
                --sp;
                continue;
            }
            if (top.stage == 1) {
                if (!ret) {
                    --sp;
                    continue;
                }
                const int e2 = i2m3[ce];
                top.stage = 2;
                if (sp < kEpaMaxFaces) {
                    frames[sp++] = Frame{cf.f[e2], cf.e[e2], 0};
                    continue;
                }
                ret = false;
                --sp;
                continue;
            }
            if (ret) {
                remove(hull, top.f);
                append(stock, top.f);
            }
            --sp;
        }
        return ret;
    }
    RG_HDI EpaStatus evaluate(Gjk& g, V3 guess) {
        gjk = &g;
        Simplex& simplex = g.simplices[g.simplex];
        if ((simplex.rank > 1) && g.enclose_origin()) {
            while (hull.root >= 0) {
                const int16_t f = hull.root;
                remove(hull, f);
                append(stock, f);
            }
            status = kEpaValid;
            nextsv = 0;
            const V3 w0 = g.store[simplex.c[0]].w, w1 = g.store[simplex.c[1]].w, w2 = g.store[simplex.c[2]].w,
                     w3 = g.store[simplex.c[3]].w;
            if (Gjk::det(w0 - w3, w1 - w3, w2 - w3) < 0.0f) {
                const int tc = simplex.c[0];
                simplex.c[0] = simplex.c[1];
                simplex.c[1] = tc;
                const float tp = simplex.p[0];
                simplex.p[0] = simplex.p[1];
                simplex.p[1] = tp;
            }
            const int16_t s0 = static_cast<int16_t>(kEpaMaxVertices + simplex.c[0]);
            const int16_t s1 = static_cast<int16_t>(kEpaMaxVertices + simplex.c[1]);
            const int16_t s2 = static_cast<int16_t>(kEpaMaxVertices + simplex.c[2]);
            const int16_t s3 = static_cast<int16_t>(kEpaMaxVertices + simplex.c[3]);
            const int16_t tetra[4] = {newface(s0, s1, s2, true), newface(s1, s0, s3, true), newface(s2, s1, s3, true),
                                      newface(s0, s2, s3, true)};
            if (hull.count == 4) {
                int16_t best = findbest();
                Face outer = fc[best];
                int pass = 0;
                bind(tetra[0], 0, tetra[1], 0);
                bind(tetra[0], 1, tetra[2], 0);
                bind(tetra[0], 2, tetra[3], 0);
                bind(tetra[1], 1, tetra[3], 2);
                bind(tetra[1], 2, tetra[2], 1);
                bind(tetra[2], 2, tetra[3], 1);
                status = kEpaValid;
                for (int iterations = 0; iterations < kEpaMaxIterations; ++iterations) {
                    if (nextsv < kEpaMaxVertices) {
                        Horizon horizon{-1, -1, 0};
                        const int16_t w = static_cast<int16_t>(nextsv++);
                        bool valid = true;
                        fc[best].pass = static_cast<uint8_t>(++pass);
                        g.getsupport(fc[best].n, sv_store[w]);
                        const float wdist = bdot(fc[best].n, sv_store[w].w) - fc[best].d;
                        if (wdist > kEpaAccuracy) {
                            for (int j = 0; (j < 3) && valid; ++j) {
                                valid &= expand(pass, w, fc[best].f[j], fc[best].e[j], horizon);
                            }
                            if (valid && (horizon.nf >= 3)) {
                                bind(horizon.cf, 1, horizon.ff, 2);
                                remove(hull, best);
                                append(stock, best);
                                best = findbest();
                                outer = fc[best];
                            } else {
                                status = kEpaInvalidHull;
                                break;
                            }
                        } else {
                            status = kEpaAccuracyReached;
                            break;
                        }
                    } else {
                        status = kEpaOutOfVertices;
                        break;
                    }
                }
                const V3 projection = outer.n * outer.d;
                normal = outer.n;
                depth = outer.d;
                result_rank = 3;
                result_c[0] = outer.c[0];
                result_c[1] = outer.c[1];
                result_c[2] = outer.c[2];
                result_p[0] = blen(bcross(vtx(outer.c[1]).w - projection, vtx(outer.c[2]).w - projection));
                result_p[1] = blen(bcross(vtx(outer.c[2]).w - projection, vtx(outer.c[0]).w - projection));
                result_p[2] = blen(bcross(vtx(outer.c[0]).w - projection, vtx(outer.c[1]).w - projection));
                const float sum = result_p[0] + result_p[1] + result_p[2];
                result_p[0] /= sum;
                result_p[1] /= sum;
                result_p[2] /= sum;
                return status;
            }
        }
        status = kEpaFallBack;
        normal = -guess;
        const float nl = blen(normal);
        normal = nl > 0.0f ? bdiv(normal, nl) : V3{1.0f, 0.0f, 0.0f};
        depth = 0.0f;
        result_rank = 1;
        result_c[0] = static_cast<int16_t>(kEpaMaxVertices + simplex.c[0]);
        result_p[0] = 1.0f;
        return status;
    }
};

struct Results {
    V3 witness0, witness1, normal;
    float distance;
};

// btGjkEpaSolver2::Penetration (with margins).
RG_NOINL bool penetration(const Shape& s0, const Xform& w0, const Shape& s1, const Xform& w1, V3 guess, Results& r) {
    r.witness0 = r.witness1 = V3{0.0f, 0.0f, 0.0f};
    Gjk g;
    g.shape = make_minkowski(s0, w0, s1, w1, true);
    g.ray = V3{0.0f, 0.0f, 0.0f};
    g.nfree = 0;
    g.status = kGjkFailed;
    g.current = 0;
    g.distance = 0.0f;
    if (g.evaluate(-guess) != kGjkInside) return false;
    Epa epa;
    epa.initialize();
    if (epa.evaluate(g, -guess) == kEpaFailed) return false;
    V3 wsum{0.0f, 0.0f, 0.0f};
    for (int i = 0; i < epa.result_rank; ++i) {
        V3 dn = epa.vtx(epa.result_c[i]).d;
        if (blen2(dn) < (1.1920929e-7f * 1.1920929e-7f)) dn = V3{-1.0f, -1.0f, -1.0f};
        dn = bnormalized(dn);
        const V3 sup = support_no_margin(s0, dn) + dn * s0.margin;
        wsum += sup * epa.result_p[i];
    }
    r.witness0 = xform(w0, wsum);
    r.witness1 = xform(w0, wsum - epa.normal * epa.depth);
    r.normal = -epa.normal;
    r.distance = -epa.depth;
    return true;
}
// btGjkEpaSolver2::Distance (no margins). Returns false when the shapes overlap or GJK fails.
RG_NOINL bool distance(const Shape& s0, const Xform& w0, const Shape& s1, const Xform& w1, V3 guess, Results& r) {
    r.witness0 = r.witness1 = V3{0.0f, 0.0f, 0.0f};
    Gjk g;
    g.shape = make_minkowski(s0, w0, s1, w1, false);
    g.ray = V3{0.0f, 0.0f, 0.0f};
    g.nfree = 0;
    g.status = kGjkFailed;
    g.current = 0;
    g.distance = 0.0f;
    if (g.evaluate(guess) != kGjkValid) return false;
    V3 a{0.0f, 0.0f, 0.0f}, b{0.0f, 0.0f, 0.0f};
    const Simplex& s = g.simplices[g.simplex];
    for (int i = 0; i < s.rank; ++i) {
        const float p = s.p[i];
        a += g.shape.support0(g.store[s.c[i]].d) * p;
        b += g.shape.support1(-g.store[s.c[i]].d) * p;
    }
    r.witness0 = xform(w0, a);
    r.witness1 = xform(w0, b);
    r.normal = a - b;
    r.distance = blen(r.normal);
    r.normal = bdiv(r.normal, r.distance > kGjkMinDistance ? r.distance : 1.0f);
    return true;
}

// ---- the Voronoi simplex solver of the GJK pair detector ----------------------------------------------------------
struct SubResult {
    V3 closest;
    bool ua, ub, uc, ud;
    float bc[4];
    bool degenerate;
    RG_HD void reset() {
        closest = V3{0.0f, 0.0f, 0.0f};
        ua = ub = uc = ud = false;
        bc[0] = bc[1] = bc[2] = bc[3] = 0.0f;
        degenerate = false;
    }
    RG_HD void set_bc(float a, float b, float c, float d) {
        bc[0] = a;
        bc[1] = b;
        bc[2] = c;
        bc[3] = d;
    }
    RG_HD bool valid() const { return bc[0] >= 0.0f && bc[1] >= 0.0f && bc[2] >= 0.0f && bc[3] >= 0.0f; }
};

struct VoronoiSimplex {
    int n;
    V3 w[4], p[4], q[4];
    V3 cp1, cp2, cv;
    V3 last_w;
    SubResult bc;
    bool valid_closest, needs_update;

    RG_HD void reset() {
        valid_closest = false;
        n = 0;
        needs_update = true;
        last_w = V3{1.0e18f, 1.0e18f, 1.0e18f};
        bc.reset();
        cp1 = cp2 = cv = V3{0.0f, 0.0f, 0.0f};
    }
    RG_HD void add(V3 ww, V3 pp, V3 qq) {
        last_w = ww;
        needs_update = true;
        w[n] = ww;
        p[n] = pp;
        q[n] = qq;
        ++n;
    }
    RG_HD bool full() const { return n == 4; }
    RG_HD bool in_simplex(V3 ww) const {
        for (int i = 0; i < n; ++i)
            if (len2(w[i] - ww) <= 0.0001f) return true;
        return ww.x == last_w.x && ww.y == last_w.y && ww.z == last_w.z;
    }
    RG_HD void remove_vertex(int i) {
        --n;
        w[i] = w[n];
        p[i] = p[n];
        q[i] = q[n];
    }
    RG_HD void reduce(const SubResult& u) {
        if (n >= 4 && !u.ud) remove_vertex(3);
        if (n >= 3 && !u.uc) remove_vertex(2);
        if (n >= 2 && !u.ub) remove_vertex(1);
        if (n >= 1 && !u.ua) remove_vertex(0);
    }
    RG_HDI static void closest_triangle(V3 pt, V3 a, V3 b, V3 c, SubResult& r) {
        r.ua = r.ub = r.uc = r.ud = false;
        const V3 ab = b - a, ac = c - a, ap = pt - a;
        const float d1 = dot(ab, ap), d2 = dot(ac, ap);
        if (d1 <= 0.0f && d2 <= 0.0f) {
            r.closest = a;
            r.ua = true;
            r.set_bc(1.0f, 0.0f, 0.0f, 0.0f);
            return;
        }
        const V3 bp = pt - b;
        const float d3 = dot(ab, bp), d4 = dot(ac, bp);
        if (d3 >= 0.0f && d4 <= d3) {
            r.closest = b;
            r.ub = true;
            r.set_bc(0.0f, 1.0f, 0.0f, 0.0f);
            return;
        }
        const float vc = d1 * d4 - d3 * d2;
        if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
            const float v = d1 / (d1 - d3);
            r.closest = a + ab * v;
            r.ua = r.ub = true;
            r.set_bc(1.0f - v, v, 0.0f, 0.0f);
            return;
        }
        const V3 cp = pt - c;
        const float d5 = dot(ab, cp), d6 = dot(ac, cp);
        if (d6 >= 0.0f && d5 <= d6) {
            r.closest = c;
            r.uc = true;
            r.set_bc(0.0f, 0.0f, 1.0f, 0.0f);
            return;
        }
        const float vb = d5 * d2 - d1 * d6;
        if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
            const float ww = d2 / (d2 - d6);
            r.closest = a + ac * ww;
            r.ua = r.uc = true;
            r.set_bc(1.0f - ww, 0.0f, ww, 0.0f);
            return;
        }
        const float va = d3 * d6 - d5 * d4;
        if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
            const float ww = (d4 - d3) / ((d4 - d3) + (d5 - d6));
            r.closest = b + (c - b) * ww;
            r.ub = r.uc = true;
            r.set_bc(0.0f, 1.0f - ww, ww, 0.0f);
            return;
        }
        const float denom = 1.0f / (va + vb + vc);
        const float v = vb * denom;
        const float ww = vc * denom;
        r.closest = a + ab * v + ac * ww;
        r.ua = r.ub = r.uc = true;
        r.set_bc(1.0f - v - ww, v, ww, 0.0f);
    }
    RG_HDI static int outside_plane(V3 pt, V3 a, V3 b, V3 c, V3 d) {
        const V3 nrm = cross(b - a, c - a);
        const float signp = dot(pt - a, nrm);
        const float signd = dot(d - a, nrm);
        if (signd * signd < (1.0e-4f * 1.0e-4f)) return -1;
        return signp * signd < 0.0f;
    }
    RG_HDI static bool closest_tetra(V3 pt, V3 a, V3 b, V3 c, V3 d, SubResult& fin) {
        SubResult t;
        t.reset();
        fin.closest = pt;
        fin.ua = fin.ub = fin.uc = fin.ud = true;
        const int oabc = outside_plane(pt, a, b, c, d);
        const int oacd = outside_plane(pt, a, c, d, b);
        const int oadb = outside_plane(pt, a, d, b, c);
        const int obdc = outside_plane(pt, b, d, c, a);
        if (oabc < 0 || oacd < 0 || oadb < 0 || obdc < 0) {
            fin.degenerate = true;
            return false;
        }
        if (!oabc && !oacd && !oadb && !obdc) return false;
        float best = 3.402823466e+38f;
        if (oabc) {
            closest_triangle(pt, a, b, c, t);
            const float sq = len2(t.closest - pt);
            if (sq < best) {
                best = sq;
                fin.closest = t.closest;
                fin.ua = t.ua;
                fin.ub = t.ub;
                fin.uc = t.uc;
                fin.ud = false;
                fin.set_bc(t.bc[0], t.bc[1], t.bc[2], 0.0f);
            }
        }
        if (oacd) {
            closest_triangle(pt, a, c, d, t);
            const float sq = len2(t.closest - pt);
            if (sq < best) {
                best = sq;
                fin.closest = t.closest;
                fin.ua = t.ua;
                fin.ub = false;
                fin.uc = t.ub;
                fin.ud = t.uc;
                fin.set_bc(t.bc[0], 0.0f, t.bc[1], t.bc[2]);
            }
        }
        if (oadb) {
            closest_triangle(pt, a, d, b, t);
            const float sq = len2(t.closest - pt);
            if (sq < best) {
                best = sq;
                fin.closest = t.closest;
                fin.ua = t.ua;
                fin.ub = t.uc;
                fin.uc = false;
                fin.ud = t.ub;
                fin.set_bc(t.bc[0], t.bc[2], 0.0f, t.bc[1]);
            }
        }
        if (obdc) {
            closest_triangle(pt, b, d, c, t);
            const float sq = len2(t.closest - pt);
            if (sq < best) {
                best = sq;
                fin.closest = t.closest;
                fin.ua = false;
                fin.ub = t.ua;
                fin.uc = t.uc;
                fin.ud = t.ub;
                fin.set_bc(0.0f, t.bc[0], t.bc[2], t.bc[1]);
            }
        }
        return true;
    }
    RG_HDI bool update() {
        if (needs_update) {
            bc.reset();
            needs_update = false;
            switch (n) {
                case 0: valid_closest = false; break;
                case 1:
                    cp1 = p[0];
                    cp2 = q[0];
                    cv = cp1 - cp2;
                    bc.reset();
                    bc.set_bc(1.0f, 0.0f, 0.0f, 0.0f);
                    valid_closest = bc.valid();
                    break;
                case 2: {
                    const V3 from = w[0], to = w[1];
                    const V3 diff = -from;
                    const V3 v = to - from;
                    float t = dot(v, diff);
                    if (t > 0.0f) {
                        const float vv = dot(v, v);
                        if (t < vv) {
                            t /= vv;
                            bc.ua = bc.ub = true;
                        } else {
                            t = 1.0f;
                            bc.ub = true;
                        }
                    } else {
                        t = 0.0f;
                        bc.ua = true;
                    }
                    bc.set_bc(1.0f - t, t, 0.0f, 0.0f);
                    cp1 = p[0] + (p[1] - p[0]) * t;
                    cp2 = q[0] + (q[1] - q[0]) * t;
                    cv = cp1 - cp2;
                    reduce(bc);
                    valid_closest = bc.valid();
                    break;
                }
                case 3:
                    closest_triangle(V3{0.0f, 0.0f, 0.0f}, w[0], w[1], w[2], bc);
                    cp1 = p[0] * bc.bc[0] + p[1] * bc.bc[1] + p[2] * bc.bc[2];
                    cp2 = q[0] * bc.bc[0] + q[1] * bc.bc[1] + q[2] * bc.bc[2];
                    cv = cp1 - cp2;
                    reduce(bc);
                    valid_closest = bc.valid();
                    break;
                case 4: {
                    if (closest_tetra(V3{0.0f, 0.0f, 0.0f}, w[0], w[1], w[2], w[3], bc)) {
                        cp1 = p[0] * bc.bc[0] + p[1] * bc.bc[1] + p[2] * bc.bc[2] + p[3] * bc.bc[3];
                        cp2 = q[0] * bc.bc[0] + q[1] * bc.bc[1] + q[2] * bc.bc[2] + q[3] * bc.bc[3];
                        cv = cp1 - cp2;
                        reduce(bc);
                        valid_closest = bc.valid();
                    } else if (bc.degenerate) {
                        valid_closest = false;
                    } else {
                        valid_closest = true;
                        cv = V3{0.0f, 0.0f, 0.0f};
                    }
                    break;
                }
                default: valid_closest = false; break;
            }
        }
        return valid_closest;
    }
};

// ---- box vs triangle -----------------------------------------------------------------------------------------------
// The box's world transform from the car basis (columns) and a centre (MakeBulletPortBoxWorldTransform).
RG_HDI Xform basis_xform(V3 f, V3 r, V3 u, V3 origin) {
    Xform t;
    t.b.r[0] = V3{f.x, r.x, u.x};
    t.b.r[1] = V3{f.y, r.y, u.y};
    t.b.r[2] = V3{f.z, r.z, u.z};
    t.o = origin;
    return t;
}

// Bullet's GJK pair detector loop between shape `a` (in `xa`) and `b` (in `xb`), without margins
// (reference RunCarArenaTriangleGjkSimplex / RunBallCarGjkSimplex, triangle_and_carcar.hpp:206-300, 538-624):
// iterates the Voronoi simplex toward the origin until a termination rule fires. Returns whether it ended on a rule
// that yields closest points (`pa`, `pb`, world space); `degenerate` records which rule.
RG_NOINL bool pair_detector(const Shape& a, const Xform& xa, const Shape& b, const Xform& xb, float max_dist_sq,
                          V3& cached_axis, int& degenerate, float& squared_distance, V3& pa, V3& pb) {
    constexpr float kRelError2 = 1.0e-6f;
    bool check_simplex = false;
    VoronoiSimplex sx;
    sx.reset();
    int cur_iter = 0;
    while (true) {
        const V3 sep_a = vec_mul_mat(-cached_axis, xa.b);
        const V3 sep_b = vec_mul_mat(cached_axis, xb.b);
        const V3 pw = xform(xa, support_no_margin(a, sep_a));
        const V3 qw = xform(xb, support_no_margin(b, sep_b));
        const V3 w = pw - qw;
        const float delta = dot(cached_axis, w);
        if ((delta > 0.0f) && (delta * delta > squared_distance * max_dist_sq)) {
            degenerate = 10;
            check_simplex = true;
            break;
        }
        if (sx.in_simplex(w)) {
            degenerate = 1;
            check_simplex = true;
            break;
        }
        const float f0 = squared_distance - delta;
        const float f1 = squared_distance * kRelError2;
        if (f0 <= f1) {
            degenerate = f0 <= 0.0f ? 2 : 11;
            check_simplex = true;
            break;
        }
        sx.add(w, pw, qw);
        const bool ok = sx.update();
        const V3 new_axis = sx.cv;
        if (!ok) {
            degenerate = 3;
            check_simplex = true;
            break;
        }
        if (len2(new_axis) < kRelError2) {
            cached_axis = new_axis;
            degenerate = 6;
            check_simplex = true;
            break;
        }
        const float prev = squared_distance;
        squared_distance = len2(new_axis);
        if (prev - squared_distance <= 1.1920929e-7f * prev) {
            check_simplex = true;
            degenerate = 12;
            break;
        }
        cached_axis = new_axis;
        if (cur_iter++ > 1000) break;
        if (sx.full()) {
            degenerate = 13;
            break;
        }
    }
    if (check_simplex) {
        sx.update();
        pa = sx.cp1;
        pb = sx.cp2;
    }
    return check_simplex;
}

// Closest points / penetration of the car's hitbox (half extents `raw_half_bt`, Bullet margin 0.04) and a triangle
// (reference ComputeCarArenaTriangleContact). Returns false when there is no contact within 10 bt; otherwise the
// signed distance and the witness point on the triangle.
RG_NOINL bool box_triangle_contact(V3 basis_f, V3 basis_r, V3 basis_u, V3 car_pos_bt, V3 child_offset_bt, V3 raw_half_bt,
                                 V3 ta, V3 tb, V3 tc, float& out_distance_bt, V3& out_point_on_b_bt) {
    const Shape box = make_box(raw_half_bt, 0.04f);
    const Shape tri = make_triangle(ta, tb, tc);
    const float margin_a = box.margin, margin_b = tri.margin;
    Xform ta_x = basis_xform(basis_f, basis_r, basis_u, car_pos_bt);
    ta_x.o = xform(ta_x, child_offset_bt);
    const float margin = margin_a + margin_b;
    Xform tb_x;
    tb_x.b.r[0] = V3{1.0f, 0.0f, 0.0f};
    tb_x.b.r[1] = V3{0.0f, 1.0f, 0.0f};
    tb_x.b.r[2] = V3{0.0f, 0.0f, 1.0f};
    tb_x.o = V3{0.0f, 0.0f, 0.0f};
    const V3 offset = (ta_x.o + tb_x.o) * 0.5f;
    ta_x.o = ta_x.o - offset;
    tb_x.o = tb_x.o - offset;
    V3 cached_axis{0.0f, 1.0f, 0.0f};
    bool is_valid = false;
    int degenerate = 0;
    float squared_distance = 1.0e30f;
    float distance_bt = 0.0f;
    V3 point_a{0.0f, 0.0f, 0.0f}, point_b{0.0f, 0.0f, 0.0f};

    // GJK pair-detector loop (RunCarArenaTriangleGjkSimplex)
    const bool check_simplex =
        pair_detector(box, ta_x, tri, tb_x, 100.0f, cached_axis, degenerate, squared_distance, point_a, point_b);
    if (check_simplex) {
        const float l2 = len2(cached_axis);
        if (l2 <= 0.0001f) degenerate = 5;
        if (l2 > 1.1920929e-7f * 1.1920929e-7f) {
            const float rlen = 1.0f / sqrtf(l2);
            const float s = sqrtf(squared_distance);
            if (s > 0.0f) {
                point_a = point_a - cached_axis * (margin_a / s);
                point_b = point_b + cached_axis * (margin_b / s);
                distance_bt = (1.0f / rlen) - margin;
                is_valid = true;
            }
        }
    }
    const bool catch_degenerate = degenerate && ((distance_bt + margin) <= 0.01f);
    if (!is_valid || catch_degenerate) {
        // penetration depth (BulletPortCalcPenDepth): EPA with the box-to-triangle origin delta as the guess
        const V3 delta_origin = tb_x.o - ta_x.o;  // btVector3::safeNormalize
        const float dl2 = blen2(delta_origin);
        const V3 guess = dl2 > 1.0e-20f ? bdiv(delta_origin, sqrtf(dl2)) : V3{0.0f, 0.0f, 0.0f};
        Results r;
        V3 sep{0.0f, 0.0f, 0.0f}, wa{0.0f, 0.0f, 0.0f}, wb{0.0f, 0.0f, 0.0f};
        bool pen = false;
        if (penetration(box, ta_x, tri, tb_x, guess, r)) {
            wa = r.witness0;
            wb = r.witness1;
            sep = r.normal;
            pen = true;
        } else if (distance(box, ta_x, tri, tb_x, guess, r)) {
            wa = r.witness0;
            wb = r.witness1;
            sep = r.normal;
        }
        if (pen) {
            V3 nb = wb - wa;
            float l2 = blen2(nb);
            if (l2 <= (1.1920929e-7f * 1.1920929e-7f)) {
                nb = sep;
                l2 = blen2(sep);
            }
            if (l2 > (1.1920929e-7f * 1.1920929e-7f)) {
                const float d2 = -len(wa - wb);
                if (!is_valid || (d2 < distance_bt)) {
                    distance_bt = d2;
                    point_a = wa;
                    point_b = wb;
                    is_valid = true;
                }
            }
        } else if (blen2(sep) > 0.0f) {
            const float d2 = len(wa - wb) - margin;
            if (!is_valid || (d2 < distance_bt)) {
                point_a = wa - sep * margin_a;
                point_b = wb + sep * margin_b;
                distance_bt = d2;
                is_valid = true;
            }
        }
    }
    if (!is_valid) return false;
    if (!((distance_bt < 0.0f) || (distance_bt * distance_bt < 100.0f))) return false;
    point_b = point_b + offset;
    out_distance_bt = distance_bt;
    out_point_on_b_bt = point_b;
    return true;
}

// ---- box vs sphere ---------------------------------------------------------------------------------------------
// World AABB centre of a box or sphere under `t` (btConvexShape::getAabb), as the normal-direction fix reads it.
RG_HDI V3 aabb_center(const Shape& s, const Xform& t) {
    if (s.kind == kBox) {
        const V3 h = s.half + V3{s.margin, s.margin, s.margin};
        const V3 a0{fabs_(t.b.r[0].x), fabs_(t.b.r[0].y), fabs_(t.b.r[0].z)};
        const V3 a1{fabs_(t.b.r[1].x), fabs_(t.b.r[1].y), fabs_(t.b.r[1].z)};
        const V3 a2{fabs_(t.b.r[2].x), fabs_(t.b.r[2].y), fabs_(t.b.r[2].z)};
        const V3 e{bdot(h, a0), bdot(h, a1), bdot(h, a2)};
        return ((t.o + e) + (t.o - e)) * 0.5f;
    }
    const V3 e{s.margin, s.margin, s.margin};
    return ((t.o + e) + (t.o - e)) * 0.5f;
}

struct BallBoxContact {
    V3 normal;          // from the car toward the ball
    float distance_bt;  // signed separation
    V3 rel_ball_bt, rel_car_bt;    // contact points relative to the ball / car origins
    V3 ball_local_bt, car_local_bt;  // the same points in the bodies' frames
};
// The car's hitbox (raw half extents, Bullet margin 0.04) against the ball's sphere (reference
// ComputeBallCarContactGeometryGjk, triangle_and_carcar.hpp:626-821): the GJK pair detector, EPA when they overlap,
// the contact kept within the breaking threshold. False leaves the caller to the sphere-box fallback.
RG_NOINL bool ball_box_contact(V3 cf, V3 cr, V3 cu, V3 car_pos_bt, V3 child_offset_bt, V3 raw_half_bt, V3 bx, V3 by,
                             V3 bz, V3 ball_pos_bt, float radius_bt, float threshold_bt, BallBoxContact& out) {
    const Shape box = make_box(raw_half_bt, 0.04f);
    const Shape sphere = make_sphere(radius_bt);
    const float margin_a = box.margin, margin_b = sphere.margin;
    float max_dist_sq = margin_a + margin_b + threshold_bt;
    max_dist_sq *= max_dist_sq;
    Xform xa = basis_xform(cf, cr, cu, car_pos_bt);
    xa.o = xform(xa, child_offset_bt);
    Xform xb = basis_xform(bx, by, bz, ball_pos_bt);
    const V3 offset = (xa.o + xb.o) * 0.5f;
    xa.o = xa.o - offset;
    xb.o = xb.o - offset;
    V3 cached_axis{0.0f, 1.0f, 0.0f};
    float squared_distance = 1.0e30f;
    bool is_valid = false;
    int degenerate = 0;
    float distance_bt = 0.0f;
    V3 normal{0.0f, 0.0f, 0.0f}, pa{0.0f, 0.0f, 0.0f}, pb{0.0f, 0.0f, 0.0f};
    if (!pair_detector(box, xa, sphere, xb, max_dist_sq, cached_axis, degenerate, squared_distance, pa, pb))
        return false;
    const float len_sqr = len2(cached_axis);
    if (len_sqr <= 0.0001f) degenerate = 5;
    const float s = sqrtf(squared_distance);
    if (len_sqr > 1.1920929e-7f * 1.1920929e-7f) {
        const float inv_len = 1.0f / sqrtf(len_sqr);
        normal = cached_axis * inv_len;
        if (s > 0.0f) {
            pa = pa - cached_axis * (margin_a / s);
            pb = pb + cached_axis * (margin_b / s);
            distance_bt = (1.0f / inv_len) - (margin_a + margin_b);
            is_valid = true;
        }
    }
    const bool catch_degenerate = degenerate && ((distance_bt + (margin_a + margin_b)) <= 0.01f);
    if (!is_valid || catch_degenerate) {
        const V3 delta_origin = xb.o - xa.o;
        const float dl2 = blen2(delta_origin);
        const V3 guess = dl2 > 1.0e-20f ? bdiv(delta_origin, sqrtf(dl2)) : V3{0.0f, 0.0f, 0.0f};
        Results r;
        V3 sep{0.0f, 0.0f, 0.0f}, wa{0.0f, 0.0f, 0.0f}, wb{0.0f, 0.0f, 0.0f};
        bool pen = false;
        if (penetration(box, xa, sphere, xb, guess, r)) {
            wa = r.witness0;
            wb = r.witness1;
            sep = r.normal;
            pen = true;
        } else if (distance(box, xa, sphere, xb, guess, r)) {
            wa = r.witness0;
            wb = r.witness1;
            sep = r.normal;
        }
        if (pen) {
            V3 nb = wb - wa;
            float l2 = blen2(nb);
            if (l2 <= 1.1920929e-7f * 1.1920929e-7f) {
                nb = sep;
                l2 = blen2(sep);
            }
            if (l2 > 1.1920929e-7f * 1.1920929e-7f) {
                nb = bdiv(nb, sqrtf(l2));
                const float d2 = -len(wa - wb);
                if (!is_valid || d2 < distance_bt) {
                    distance_bt = d2;
                    pa = wa;
                    pb = wb;
                    normal = nb;
                    is_valid = true;
                }
            }
        } else if (blen2(sep) > 0.0f) {
            const float d2 = len(wa - wb) - (margin_a + margin_b);
            if (!is_valid || d2 < distance_bt) {
                pa = wa - sep * margin_a;
                pb = wb + sep * margin_b;
                const float l2 = dot(sep, sep);
                normal = l2 <= 1e-12f ? normal : sep * (1.0f / sqrtf(l2));
                distance_bt = d2;
                is_valid = true;
            }
        }
    }
    if (!is_valid) return false;
    if (!((distance_bt < 0.0f) || (distance_bt * distance_bt < max_dist_sq))) return false;
    if (distance_bt > threshold_bt) return false;
    const V3 point_on_ball = pb + offset;
    // the normal made to point from the sphere toward the box (FixArenaTriangleContactNormalDirectionBullet)
    const V3 diff = aabb_center(box, xa) - aabb_center(sphere, xb);
    V3 bn = normal;
    if (bdot(diff, bn) < 0.0f) bn = bn * -1.0f;
    const V3 point_on_car = point_on_ball + bn * distance_bt;
    out.normal = -bn;
    out.distance_bt = distance_bt;
    const V3 car_local = vec_mul_mat(point_on_car - car_pos_bt, xa.b);
    const V3 ball_local = vec_mul_mat(point_on_ball - ball_pos_bt, xb.b);
    const V3 car_ref = V3{bdot(car_local, xa.b.r[0]), bdot(car_local, xa.b.r[1]), bdot(car_local, xa.b.r[2])} +
                       car_pos_bt;
    const V3 ball_ref = V3{bdot(ball_local, xb.b.r[0]), bdot(ball_local, xb.b.r[1]), bdot(ball_local, xb.b.r[2])} +
                        ball_pos_bt;
    out.rel_ball_bt = ball_ref - ball_pos_bt;
    out.rel_car_bt = car_ref - car_pos_bt;
    out.ball_local_bt = ball_local;
    out.car_local_bt = car_local;
    return true;
}

}  // namespace gjk
}  // namespace rg

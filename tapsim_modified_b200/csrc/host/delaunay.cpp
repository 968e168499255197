#include "delaunay.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <sstream>

#include "predicates.h"

namespace tg_host {
namespace {

// Face opposite vertex k, ordered so that orient(face, v_k) > 0 for a
// positively oriented tetrahedron (v0,v1,v2,v3).
const int kFace[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};

inline uint64_t spread3(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

inline uint64_t morton(const IPoint& p) {
    const uint64_t off = 1ull << 40;
    return spread3((uint64_t)(p.x + off) >> 20) | spread3((uint64_t)(p.y + off) >> 20) << 1 |
           spread3((uint64_t)(p.z + off) >> 20) << 2;
}

struct Builder {
    int n, INF;
    std::vector<IPoint> P;
    struct Tet { int32_t v[4]; int32_t n[4]; };
    std::vector<Tet> T;
    std::vector<int32_t> freeList;
    std::vector<uint32_t> mark;
    uint32_t stamp = 0;
    int lastTet = 0;
    unsigned rot = 0;

    struct BFace { int32_t f0, f1, f2, outer, outerSlot; };
    std::vector<int32_t> cavity;
    std::vector<BFace> bfaces;
    std::vector<int32_t> newTets;
    struct GlueSlot { uint64_t key; int32_t val; uint32_t gen; };
    std::vector<GlueSlot> glue;
    uint32_t glueGen = 0;

    bool infinite(int t) const {
        const int32_t* v = &T[t].v[0];
        return v[0] == INF || v[1] == INF || v[2] == INF || v[3] == INF;
    }

    int alloc() {
        if (!freeList.empty()) {
            const int t = freeList.back();
            freeList.pop_back();
            return t;
        }
        const int t = (int)T.size();
        T.emplace_back();
        mark.push_back(0);
        return t;
    }

    void release(int t) {
        T[t].v[0] = -2;  // dead marker
        freeList.push_back(t);
    }

    // p strictly inside the circle through the non-degenerate triangle abc;
    // p is coplanar with abc.
    bool in_circle(const IPoint& a, const IPoint& b, const IPoint& c, const IPoint& p) const {
        const i128 ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
        const i128 vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
        const i128 nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
        const i128 ax_ = nx < 0 ? -nx : nx, ay_ = ny < 0 ? -ny : ny, az_ = nz < 0 ? -nz : nz;
        IPoint q = a;
        const int64_t off = 1ll << 38;
        if (ax_ >= ay_ && ax_ >= az_) q.x += off;
        else if (ay_ >= az_) q.y += off;
        else q.z += off;
        const int o = orient(a, b, c, q);
        const int s = insphere(a, b, c, q, p);
        return o > 0 ? s > 0 : s < 0;
    }

    bool conflict(int t, int pi) const {
        const int32_t* v = &T[t].v[0];
        int k = -1;
        for (int i = 0; i < 4; i++)
            if (v[i] == INF) k = i;
        const IPoint& p = P[pi];
        if (k < 0) return insphere(P[v[0]], P[v[1]], P[v[2]], P[v[3]], p) > 0;
        const IPoint& a = P[v[kFace[k][0]]];
        const IPoint& b = P[v[kFace[k][1]]];
        const IPoint& c = P[v[kFace[k][2]]];
        const int o = orient(a, b, c, p);
        if (o > 0) return true;
        if (o < 0) return false;
        return in_circle(a, b, c, p);
    }

    int locate(int pi, int start) {
        int t = start;
        if (t < 0 || T[t].v[0] == -2) t = 0;
        while (T[t].v[0] == -2) t++;
        if (infinite(t)) {
            for (int k = 0; k < 4; k++)
                if (T[t].v[k] == INF) { t = T[t].n[k]; break; }
        }
        const IPoint& p = P[pi];
        const long maxSteps = 64 + (long)T.size() * 2;
        for (long step = 0; step < maxSteps; step++) {
            const int32_t* v = &T[t].v[0];
            const unsigned r = rot++;
            int next = -1;
            for (int j = 0; j < 4; j++) {
                const int k = (int)((r + j) & 3);
                if (orient(P[v[kFace[k][0]]], P[v[kFace[k][1]]], P[v[kFace[k][2]]], p) < 0) {
                    next = T[t].n[k];
                    break;
                }
            }
            if (next < 0) return t;
            if (infinite(next)) return next;
            t = next;
        }
        // visibility walks terminate on Delaunay meshes; scan as a last resort
        for (int s = 0; s < (int)T.size(); s++)
            if (T[s].v[0] != -2 && conflict(s, pi)) return s;
        return -1;
    }

    void glue_new_tets() {
        size_t cap = glue.size() < 64 ? 64 : glue.size();
        while (cap < newTets.size() * 6) cap <<= 1;
        if (cap != glue.size()) {
            glue.assign(cap, GlueSlot{0, 0, 0});
            glueGen = 0;
        }
        glueGen++;
        if (glueGen == 0) {
            for (GlueSlot& g : glue) g.gen = 0;
            glueGen = 1;
        }
        for (int32_t nt : newTets) {
            for (int m = 0; m < 3; m++) {
                const int32_t a = T[nt].v[(m + 1) % 3], b = T[nt].v[(m + 2) % 3];
                const uint64_t key = ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
                size_t h = (size_t)((key * 0x9E3779B97F4A7C15ull) >> 20) & (cap - 1);
                while (true) {
                    GlueSlot& g = glue[h];
                    if (g.gen != glueGen) {
                        g.key = key;
                        g.val = nt * 4 + m;
                        g.gen = glueGen;
                        break;
                    }
                    if (g.key == key) {
                        const int32_t other = g.val;
                        T[nt].n[m] = other / 4;
                        T[other / 4].n[other % 4] = nt;
                        g.key = ~0ull;  // paired: each edge pairs exactly once
                        break;
                    }
                    h = (h + 1) & (cap - 1);
                }
            }
        }
    }

    std::string insert(int pi) {
        int t0 = locate(pi, lastTet);
        if (t0 < 0 || !conflict(t0, pi)) {
            std::ostringstream os;
            os << "delaunay: point " << pi << " could not be inserted (duplicate or degenerate input)";
            return os.str();
        }
        stamp += 2;
        if (stamp < 2) {  // wrapped: reset marks
            std::fill(mark.begin(), mark.end(), 0u);
            stamp = 2;
        }
        const uint32_t IN = stamp, OUT = stamp + 1;
        cavity.clear();
        bfaces.clear();
        mark[t0] = IN;
        cavity.push_back(t0);
        for (size_t q = 0; q < cavity.size(); q++) {
            const int t = cavity[q];
            for (int k = 0; k < 4; k++) {
                const int o = T[t].n[k];
                if (mark[o] == IN) continue;
                if (mark[o] != OUT) {
                    if (conflict(o, pi)) {
                        mark[o] = IN;
                        cavity.push_back(o);
                        continue;
                    }
                    mark[o] = OUT;
                }
                BFace f;
                f.f0 = T[t].v[kFace[k][0]];
                f.f1 = T[t].v[kFace[k][1]];
                f.f2 = T[t].v[kFace[k][2]];
                f.outer = o;
                f.outerSlot = -1;
                for (int m = 0; m < 4; m++)
                    if (T[o].n[m] == t) f.outerSlot = m;
                bfaces.push_back(f);
            }
        }
        for (int t : cavity) release(t);
        newTets.clear();
        for (const BFace& f : bfaces) {
            const int nt = alloc();
            T[nt].v[0] = f.f0;
            T[nt].v[1] = f.f1;
            T[nt].v[2] = f.f2;
            T[nt].v[3] = pi;
            T[nt].n[3] = f.outer;
            T[f.outer].n[f.outerSlot] = nt;
            mark[nt] = 0;
            newTets.push_back(nt);
        }
        glue_new_tets();
        lastTet = newTets.front();
        for (int32_t nt : newTets)
            if (!infinite(nt)) { lastTet = nt; break; }
        return std::string();
    }

    std::string init(const std::vector<int>& order, size_t* used) {
        // four affinely independent points from the start of the order
        const int i0 = order[0];
        int i1 = -1, i2 = -1, i3 = -1;
        size_t s = 1;
        for (; s < order.size() && i1 < 0; s++) {
            const IPoint& q = P[order[s]];
            if (q.x != P[i0].x || q.y != P[i0].y || q.z != P[i0].z) i1 = order[s];
        }
        for (; s < order.size() && i2 < 0; s++) {
            const IPoint &a = P[i0], &b = P[i1], &c = P[order[s]];
            const i128 ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
            const i128 vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
            if (uy * vz - uz * vy != 0 || uz * vx - ux * vz != 0 || ux * vy - uy * vx != 0) i2 = order[s];
        }
        for (; s < order.size() && i3 < 0; s++)
            if (orient(P[i0], P[i1], P[i2], P[order[s]]) != 0) i3 = order[s];
        if (i3 < 0) return "delaunay: all points are coplanar";
        if (orient(P[i0], P[i1], P[i2], P[i3]) < 0) std::swap(i1, i2);
        const int T0 = alloc();
        const int32_t v0[4] = {i0, i1, i2, i3};
        for (int k = 0; k < 4; k++) T[T0].v[k] = v0[k];
        newTets.clear();
        for (int k = 0; k < 4; k++) {
            const int it = alloc();
            const int32_t g0 = v0[kFace[k][0]], g1 = v0[kFace[k][1]], g2 = v0[kFace[k][2]];
            T[it].v[0] = g0;
            T[it].v[1] = g2;
            T[it].v[2] = g1;
            T[it].v[3] = INF;
            T[it].n[3] = T0;
            T[T0].n[k] = it;
            newTets.push_back(it);
        }
        glue_new_tets();
        lastTet = T0;
        // mark the four seed points as used
        *used = 0;
        (void)used;
        seeds[0] = i0; seeds[1] = i1; seeds[2] = i2; seeds[3] = i3;
        return std::string();
    }
    int seeds[4];
};

}  // namespace

std::string delaunay_tetrahedralize(const float* xyz, int n, uint64_t seed, Tetrahedralization* out) {
    if (n < 4) return "delaunay: fewer than four points";
    Builder B;
    B.n = n;
    B.INF = n;
    // snap to a power-of-two integer grid with |coordinate| <= 2^40
    double amax = 0.0;
    for (long i = 0; i < 3L * n; i++) amax = std::max(amax, std::fabs((double)xyz[i]));
    if (!(amax > 0.0) || !std::isfinite(amax)) return "delaunay: invalid coordinates";
    const int e = (int)std::floor(std::log2(std::ldexp(1.0, 40) / amax));
    const double scale = std::ldexp(1.0, e);
    B.P.resize(n);
    for (int i = 0; i < n; i++) {
        B.P[i].x = std::llround((double)xyz[3 * i] * scale);
        B.P[i].y = std::llround((double)xyz[3 * i + 1] * scale);
        B.P[i].z = std::llround((double)xyz[3 * i + 2] * scale);
    }
    {
        std::vector<int> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        std::sort(idx.begin(), idx.end(), [&](int a, int b) {
            const IPoint &p = B.P[a], &q = B.P[b];
            if (p.x != q.x) return p.x < q.x;
            if (p.y != q.y) return p.y < q.y;
            return p.z < q.z;
        });
        for (int i = 1; i < n; i++) {
            const IPoint &p = B.P[idx[i - 1]], &q = B.P[idx[i]];
            if (p.x == q.x && p.y == q.y && p.z == q.z) {
                std::ostringstream os;
                os << "delaunay: duplicate points " << idx[i - 1] << " and " << idx[i];
                return os.str();
            }
        }
    }
    // biased randomized insertion order
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed);
    std::shuffle(order.begin(), order.end(), rng);
    {
        std::vector<uint64_t> key(n);
        for (int i = 0; i < n; i++) key[i] = morton(B.P[i]);
        size_t lo = 0, hi = std::min<size_t>(n, 64);
        while (lo < (size_t)n) {
            std::sort(order.begin() + lo, order.begin() + hi, [&](int a, int b) { return key[a] < key[b]; });
            lo = hi;
            hi = std::min<size_t>(n, hi * 2);
            if ((size_t)n - hi < hi / 4) hi = n;
        }
    }
    B.T.reserve((size_t)n * 7);
    B.mark.reserve((size_t)n * 7);
    size_t used = 0;
    std::string err = B.init(order, &used);
    if (!err.empty()) return err;
    for (int i = 0; i < n; i++) {
        const int pi = order[i];
        if (pi == B.seeds[0] || pi == B.seeds[1] || pi == B.seeds[2] || pi == B.seeds[3]) continue;
        err = B.insert(pi);
        if (!err.empty()) return err;
    }
    // keep finite tetrahedra, ordered along a Morton curve of their first vertex
    const int slots = (int)B.T.size();
    std::vector<int> keep;
    keep.reserve(slots);
    for (int t = 0; t < slots; t++)
        if (B.T[t].v[0] != -2 && !B.infinite(t)) keep.push_back(t);
    {
        std::vector<uint64_t> key(slots, 0);
        for (int t : keep) {
            const IPoint &a = B.P[B.T[t].v[0]], &b = B.P[B.T[t].v[1]], &c = B.P[B.T[t].v[2]], &d = B.P[B.T[t].v[3]];
            IPoint m;
            m.x = (a.x + b.x + c.x + d.x) / 4;
            m.y = (a.y + b.y + c.y + d.y) / 4;
            m.z = (a.z + b.z + c.z + d.z) / 4;
            key[t] = morton(m);
        }
        std::stable_sort(keep.begin(), keep.end(), [&](int a, int b) { return key[a] < key[b]; });
    }
    std::vector<int32_t> remap(slots, -1);
    for (size_t i = 0; i < keep.size(); i++) remap[keep[i]] = (int32_t)i;
    out->vertices.resize(keep.size() * 4);
    out->neighbours.resize(keep.size() * 4);
    for (size_t i = 0; i < keep.size(); i++) {
        const int t = keep[i];
        for (int k = 0; k < 4; k++) {
            out->vertices[4 * i + k] = B.T[t].v[k];
            out->neighbours[4 * i + k] = remap[B.T[t].n[k]];
        }
    }
    return std::string();
}

}  // namespace tg_host

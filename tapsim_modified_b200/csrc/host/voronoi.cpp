#include "voronoi.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <thread>

namespace tg_host {
namespace {

struct D3 {
    double x, y, z;
};
inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 scale(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(D3 a) { return std::sqrt(dot(a, a)); }

void parallel_for(int n, int threads, const std::function<void(int, int)>& body) {
    if (threads <= 1 || n < 4096) {
        body(0, n);
        return;
    }
    std::atomic<int> next(0);
    const int chunk = 2048;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back([&]() {
            while (true) {
                const int s = next.fetch_add(chunk);
                if (s >= n) break;
                body(s, std::min(n, s + chunk));
            }
        });
    for (auto& th : pool) th.join();
}

// Circumcentre of a tetrahedron (tetCenter, geometry_3d.cpp:830-870 solves
// the same 3x3 system by LU; closed form here).
D3 circumcentre(D3 a, D3 b, D3 c, D3 d) {
    const D3 u = sub(b, a), v = sub(c, a), w = sub(d, a);
    const double det = 2.0 * dot(u, cross(v, w));
    const D3 num = add(add(scale(cross(v, w), dot(u, u)), scale(cross(w, u), dot(v, v))), scale(cross(u, v), dot(w, w)));
    return add(a, scale(num, 1.0 / det));
}

struct Ring {
    std::vector<int32_t> tets;  // ordered around the edge
    bool closed = false;
    D3 d1{0, 0, 0}, d2{0, 0, 0};  // outward directions at the front / back hull ends
};

// Area of the Voronoi face given its ordered vertices, with open faces
// extended by `f` along d1 (front) and d2 (back).  Mirrors the centre and fan
// of VoronoiFace::finiteCenter / finiteArea (geometry_3d.cpp:243-360): the
// closed list repeats its first vertex at the end, open faces add the two
// far points to the centre, and the fan never closes the far edge.
double face_area(const std::vector<D3>& v, bool closed, D3 d1, D3 d2, double f) {
    const size_t m = v.size();
    D3 c{0, 0, 0};
    for (const D3& p : v) c = add(c, p);
    double cnt = (double)m;
    if (closed) {
        c = add(c, v[0]);
        cnt += 1.0;
    } else {
        c = add(c, add(v[0], scale(d1, f)));
        c = add(c, add(v[m - 1], scale(d2, f)));
        cnt += 2.0;
    }
    c = scale(c, 1.0 / cnt);
    double area = 0.0;
    for (size_t k = 0; k + 1 < m; k++) area += 0.5 * norm(cross(sub(v[k], c), sub(v[k + 1], c)));
    if (closed) {
        area += 0.5 * norm(cross(sub(v[m - 1], c), sub(v[0], c)));
    } else {
        area += 0.5 * norm(cross(sub(add(v[0], scale(d1, f)), c), sub(v[0], c)));
        area += 0.5 * norm(cross(sub(v[m - 1], c), sub(add(v[m - 1], scale(d2, f)), c)));
    }
    return area;
}

}  // namespace

std::string build_mesh_tables(const float* xyz, int n, const int32_t* tet_v, const int32_t* tet_n, int num_tets,
                              int threads, MeshTables* out) {
    if (threads <= 0) threads = std::max(1u, std::thread::hardware_concurrency());
    MeshTables& M = *out;
    M.num_nodes = n;
    M.num_tets = num_tets;
    auto P = [&](int i) { return D3{(double)xyz[3 * i], (double)xyz[3 * i + 1], (double)xyz[3 * i + 2]}; };

    // node -> incident tetrahedra, ascending tet index
    std::vector<int32_t> tptr(n + 1, 0), tidx((size_t)num_tets * 4);
    for (long t = 0; t < num_tets; t++)
        for (int k = 0; k < 4; k++) {
            const int v = tet_v[4 * t + k];
            if (v < 0 || v >= n) return "mesh: tetrahedron vertex out of range";
            tptr[v + 1]++;
        }
    for (int i = 0; i < n; i++) tptr[i + 1] += tptr[i];
    {
        std::vector<int32_t> fill(tptr.begin(), tptr.end() - 1);
        for (long t = 0; t < num_tets; t++)
            for (int k = 0; k < 4; k++) tidx[fill[tet_v[4 * t + k]]++] = (int32_t)t;
    }
    M.node_tet.assign(n, -1);
    for (int i = 0; i < n; i++) {
        if (tptr[i + 1] == tptr[i]) return "mesh: node without tetrahedron";
        M.node_tet[i] = tidx[tptr[i + 1] - 1];
    }
    // hull nodes: vertices of faces without a neighbour
    M.hull.assign(n, 0);
    for (long t = 0; t < num_tets; t++)
        for (int k = 0; k < 4; k++)
            if (tet_n[4 * t + k] < 0)
                for (int m = 0; m < 4; m++)
                    if (m != k) M.hull[tet_v[4 * t + m]] = 1;

    // Delaunay adjacency
    M.row_ptr.assign(n + 1, 0);
    std::vector<std::vector<int32_t>> rows(n);
    parallel_for(n, threads, [&](int s, int e) {
        std::vector<int32_t> buf;
        for (int i = s; i < e; i++) {
            buf.clear();
            for (int q = tptr[i]; q < tptr[i + 1]; q++)
                for (int k = 0; k < 4; k++) {
                    const int v = tet_v[4 * (long)tidx[q] + k];
                    if (v != i) buf.push_back(v);
                }
            std::sort(buf.begin(), buf.end());
            buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
            rows[i] = buf;
        }
    });
    for (int i = 0; i < n; i++) M.row_ptr[i + 1] = M.row_ptr[i] + (int32_t)rows[i].size();
    const long nnz = M.row_ptr[n];
    M.col.resize(nnz);
    for (int i = 0; i < n; i++) std::copy(rows[i].begin(), rows[i].end(), M.col.begin() + M.row_ptr[i]);
    std::vector<std::vector<int32_t>>().swap(rows);
    M.rev.resize(nnz);
    M.dist.resize(nnz);
    parallel_for(n, threads, [&](int s, int e) {
        for (int i = s; i < e; i++)
            for (int q = M.row_ptr[i]; q < M.row_ptr[i + 1]; q++) {
                const int j = M.col[q];
                const int32_t* b = M.col.data() + M.row_ptr[j];
                const int32_t* bEnd = M.col.data() + M.row_ptr[j + 1];
                const int32_t* f = std::lower_bound(b, bEnd, (int32_t)i);
                M.rev[q] = (int32_t)(f - M.col.data());
                M.dist[q] = norm(sub(P(i), P(j)));
            }
    });
    // half mean neighbour distance per node (computeCharge's infinity factor)
    std::vector<double> halfMean(n);
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int q = M.row_ptr[i]; q < M.row_ptr[i + 1]; q++) s += M.dist[q];
        halfMean[i] = 0.5 * s / std::max(1, M.row_ptr[i + 1] - M.row_ptr[i]);
    }

    // circumcentres
    std::vector<D3> cc(num_tets);
    parallel_for(num_tets, threads, [&](int s, int e) {
        for (int t = s; t < e; t++)
            cc[t] = circumcentre(P(tet_v[4 * (long)t]), P(tet_v[4 * (long)t + 1]), P(tet_v[4 * (long)t + 2]),
                                 P(tet_v[4 * (long)t + 3]));
    });

    // face areas, one ring walk per edge (i < j), mirrored to (j, i)
    M.area_half.assign(nnz, 0.0);
    M.area_pos.assign(nnz, 0);
    std::vector<double> areaVol(nnz, 0.0);
    std::atomic<int> ringError(0);
    parallel_for(n, threads, [&](int s, int e) {
        Ring ring;
        std::vector<int32_t> back;
        std::vector<D3> verts;
        for (int i = s; i < e; i++) {
            for (int q = M.row_ptr[i]; q < M.row_ptr[i + 1]; q++) {
                const int j = M.col[q];
                if (j < i) continue;
                // a tetrahedron holding the edge
                int t0 = -1;
                for (int r = tptr[i]; r < tptr[i + 1] && t0 < 0; r++) {
                    const int32_t* v = &tet_v[4 * (long)tidx[r]];
                    if (v[0] == j || v[1] == j || v[2] == j || v[3] == j) t0 = tidx[r];
                }
                if (t0 < 0) { ringError = 1; continue; }
                auto othersOf = [&](int t, int* a, int* b) {
                    int c = 0;
                    for (int k = 0; k < 4; k++) {
                        const int v = tet_v[4 * (long)t + k];
                        if (v != i && v != j) { if (c++ == 0) *a = v; else *b = v; }
                    }
                };
                auto posOf = [&](int t, int v) {
                    for (int k = 0; k < 4; k++)
                        if (tet_v[4 * (long)t + k] == v) return k;
                    return -1;
                };
                // outward unit normal of the hull face (i, j, third) of tet t,
                // pointing away from the tet's remaining vertex `inner`
                auto outward = [&](int third, int inner) {
                    D3 nrm = cross(sub(P(third), P(i)), sub(P(j), P(i)));
                    if (dot(nrm, sub(P(inner), P(i))) > 0.0) nrm = scale(nrm, -1.0);
                    const double l = norm(nrm);
                    return l > 0.0 ? scale(nrm, 1.0 / l) : nrm;
                };
                int a0, b0;
                othersOf(t0, &a0, &b0);
                ring.tets.clear();
                ring.tets.push_back(t0);
                ring.closed = false;
                // forward: cross the face opposite `ex`, keep `keep`
                int t = t0, ex = a0, keep = b0;
                int guard = 0;
                while (true) {
                    const int nt = tet_n[4 * (long)t + posOf(t, ex)];
                    if (nt < 0) { ring.d2 = outward(keep, ex); break; }
                    if (nt == t0) { ring.closed = true; break; }
                    int x, y;
                    othersOf(nt, &x, &y);
                    const int c = (x == keep) ? y : x;
                    ring.tets.push_back(nt);
                    ex = keep;
                    keep = c;
                    t = nt;
                    if (++guard > 100000) { ringError = 2; break; }
                }
                if (!ring.closed) {
                    back.clear();
                    t = t0; ex = b0; keep = a0;
                    while (true) {
                        const int nt = tet_n[4 * (long)t + posOf(t, ex)];
                        if (nt < 0) { ring.d1 = outward(keep, ex); break; }
                        int x, y;
                        othersOf(nt, &x, &y);
                        const int c = (x == keep) ? y : x;
                        back.push_back(nt);
                        ex = keep;
                        keep = c;
                        t = nt;
                        if (++guard > 100000) { ringError = 2; break; }
                    }
                    std::reverse(back.begin(), back.end());
                    back.insert(back.end(), ring.tets.begin(), ring.tets.end());
                    ring.tets.swap(back);
                }
                verts.clear();
                for (int32_t tt : ring.tets) verts.push_back(cc[tt]);
                const double d = M.dist[q];
                const double aHalf = face_area(verts, ring.closed, ring.d1, ring.d2, 0.5 * d);
                const double aOne = ring.closed ? aHalf : face_area(verts, false, ring.d1, ring.d2, 1.0);
                const double aVi = ring.closed ? aHalf : face_area(verts, false, ring.d1, ring.d2, halfMean[i]);
                const double aVj = ring.closed ? aHalf : face_area(verts, false, ring.d1, ring.d2, halfMean[j]);
                const int r = M.rev[q];
                M.area_half[q] = M.area_half[r] = aHalf;
                M.area_pos[q] = M.area_pos[r] = aOne > 0.0 ? 1 : 0;
                areaVol[q] = aVi;
                areaVol[r] = aVj;
            }
        }
    });
    if (ringError) return "mesh: inconsistent tetrahedron adjacency";
    M.volume.assign(n, 0.0);
    for (int i = 0; i < n; i++) {
        double v = 0.0;
        for (int q = M.row_ptr[i]; q < M.row_ptr[i + 1]; q++) v += areaVol[q] * M.dist[q] / 6.0;
        M.volume[i] = v;
    }
    return std::string();
}

}  // namespace tg_host

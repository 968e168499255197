// Ion flights: one thread per ion.  Restates Trajectory_3d (tapsim/
// trajectory_3d.cpp) in FP64: the embedded Cash-Karp Runge-Kutta step
// (o5_integrator, :583-676, tableau of Cash & Karp 1990), the
// error-restricted step control (errorRestricted_stepper, :358-425), the
// loop that ends when the ion leaves the mesh (integrate, :130-209) and the
// linear extrapolation to the top plane (extrapolate, :303-332).  The field
// at a point is the barycentric interpolation of the per-vertex field_o1 of
// the enclosing tetrahedron (Grid_3d::FastField::compute,
// grid_3d.cpp:1663-1721, with the weights of tetWeights,
// geometry_3d.cpp:916-980); the tetrahedron comes from a visibility walk
// (findTetrahedron, geometry_3d.cpp:988-1044) whose start face rotates
// instead of being drawn with rand().
#include <algorithm>

#include "kernels.cuh"

namespace tgd {
namespace {

constexpr int kBlock = 128;

__constant__ int kFaceDev[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};

struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 ld3(const float* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

__device__ __forceinline__ double orient(V3 a, V3 b, V3 c, V3 p) {
    const double ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
    const double vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
    const double wx = p.x - a.x, wy = p.y - a.y, wz = p.z - a.z;
    return ux * (vy * wz - vz * wy) - uy * (vx * wz - vz * wx) + uz * (vx * wy - vy * wx);
}

// Sign of orient(a,b,c,p), exact for the points snapped to the power-of-two
// grid the host Delaunay builder uses (|coordinate| <= 2^40 quanta): a double
// evaluation with a forward error bound, and an exact 128-bit integer
// evaluation when the bound does not certify the sign.  The walk thereby
// decides every face consistently (a point on a shared face, such as an ion
// starting at a mesh vertex, is never "beyond" it from both sides), which is
// what makes the visibility walk terminate, as the reference's exact
// Predicates::orient3d does (geometry_3d.cpp:1750-1768).
__device__ int orient_sign(V3 a, V3 b, V3 c, V3 p, double snap) {
    const double ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
    const double vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
    const double wx = p.x - a.x, wy = p.y - a.y, wz = p.z - a.z;
    const double m0 = vy * wz - vz * wy, m1 = vx * wz - vz * wx, m2 = vx * wy - vy * wx;
    const double det = ux * m0 - uy * m1 + uz * m2;
    const double perm = fabs(ux) * (fabs(vy * wz) + fabs(vz * wy)) + fabs(uy) * (fabs(vx * wz) + fabs(vz * wx)) +
                        fabs(uz) * (fabs(vx * wy) + fabs(vy * wx));
    const double bound = 16.0 * 1.1102230246251565e-16 * perm;
    if (det > bound) return 1;
    if (det < -bound) return -1;
    const double lim = 1.0995116277760000e12;  // 2^40
    const double px = p.x * snap, py = p.y * snap, pz = p.z * snap;
    if (fabs(px) > lim || fabs(py) > lim || fabs(pz) > lim) return det > 0.0 ? 1 : (det < 0.0 ? -1 : 0);
    const long long ax = __double2ll_rn(a.x * snap), ay = __double2ll_rn(a.y * snap), az = __double2ll_rn(a.z * snap);
    const long long Ux = __double2ll_rn(b.x * snap) - ax, Uy = __double2ll_rn(b.y * snap) - ay, Uz = __double2ll_rn(b.z * snap) - az;
    const long long Vx = __double2ll_rn(c.x * snap) - ax, Vy = __double2ll_rn(c.y * snap) - ay, Vz = __double2ll_rn(c.z * snap) - az;
    const long long Wx = __double2ll_rn(px) - ax, Wy = __double2ll_rn(py) - ay, Wz = __double2ll_rn(pz) - az;
    const __int128 M0 = (__int128)Vy * Wz - (__int128)Vz * Wy;
    const __int128 M1 = (__int128)Vx * Wz - (__int128)Vz * Wx;
    const __int128 M2 = (__int128)Vx * Wy - (__int128)Vy * Wx;
    const __int128 e = (__int128)Ux * M0 - (__int128)Uy * M1 + (__int128)Uz * M2;
    return e > 0 ? 1 : (e < 0 ? -1 : 0);
}

// Returns the tetrahedron holding p, -1 when p is outside the mesh, -2 when
// the walk exceeded `limit` steps.
__device__ int locate(const DevMesh& m, V3 p, int t, int limit, unsigned& rot) {
    if (t < 0) return -1;
    for (int step = 0; step < limit; step++) {
        const int* v = m.tet_v + 4 * t;
        int next = -1;
        bool moved = false;
        const unsigned r = rot++;
        for (int j = 0; j < 4; j++) {
            const int k = (int)((r + j) & 3);
            const V3 a = ld3(m.xyz, v[kFaceDev[k][0]]), b = ld3(m.xyz, v[kFaceDev[k][1]]), c = ld3(m.xyz, v[kFaceDev[k][2]]);
            if (orient_sign(a, b, c, p, m.snap) < 0) {
                next = m.tet_n[4 * t + k];
                moved = true;
                break;
            }
        }
        if (!moved) return t;
        if (next < 0) return -1;
        t = next;
    }
    return -2;
}

// Barycentric weights (tetWeights): |sub-volume| / |volume|, 1/4 each for a
// flat tetrahedron.
__device__ void weights(const DevMesh& m, int t, V3 p, double w[4]) {
    const int* v = m.tet_v + 4 * t;
    const V3 P[4] = {ld3(m.xyz, v[0]), ld3(m.xyz, v[1]), ld3(m.xyz, v[2]), ld3(m.xyz, v[3])};
    const double vol = fabs(orient(P[0], P[1], P[2], P[3]));
    if (vol == 0.0) {
        w[0] = w[1] = w[2] = w[3] = 0.25;
        return;
    }
    w[0] = fabs(orient(p, P[1], P[2], P[3])) / vol;
    w[1] = fabs(orient(P[0], p, P[2], P[3])) / vol;
    w[2] = fabs(orient(P[0], P[1], p, P[3])) / vol;
    w[3] = fabs(orient(P[0], P[1], P[2], p)) / vol;
}

// Vertex fields of one flight call: every node's field_o1 is computed once,
// in bulk, from the current potentials before the flights start, and the
// potentials are copied beside them (the flights read only these two
// snapshots, so a flight may overlap the next event's relaxation) (the
// FastField buffer of the reference, grid_3d.cpp:1672-1702, filled for all
// vertices at once instead of on first use).  Four lanes share a row; a
// singular node stores NaN in x, which the flight reports as S_SINGULAR when
// it interpolates from that vertex, as the on-demand computation would.
// With a cell list, only the listed cells are computed: the event loop lists
// the cells that are free or have a free neighbour, since the field of a
// Dirichlet cell among Dirichlet cells depends only on potentials and
// couplings that never change.
constexpr int kLanesPerRow = 4;
__global__ void k_vertex_fields(DevMesh m, const int32_t* __restrict__ cells, int count) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = gid / kLanesPerRow;
    const int lane = gid % kLanesPerRow;
    const bool live = t < (cells ? count : m.n);
    const int ii = live ? (cells ? cells[t] : t) : m.n - 1;
    const int i = ii;
    const bool hull = (m.flags[ii] & F_HULL) != 0;
    const double xi = m.xyz[3 * ii], yi = m.xyz[3 * ii + 1], zi = m.xyz[3 * ii + 2];
    const double pi = m.phi64[ii];
    double a00 = 0, a01 = 0, a02 = 0, a11 = 0, a12 = 0, a22 = 0, b0 = 0, b1 = 0, b2 = 0;
    const int q1 = hull ? 0 : m.row_ptr[ii + 1];
    for (int q = (hull ? 0 : m.row_ptr[ii]) + lane; q < q1; q += kLanesPerRow) {
        if (m.cnz[q] == 0) continue;
        const int j = m.col[q];
        const double dx = (double)m.xyz[3 * j] - xi, dy = (double)m.xyz[3 * j + 1] - yi, dz = (double)m.xyz[3 * j + 2] - zi;
        const double dp = m.phi64[j] - pi;
        a00 += dx * dx; a01 += dx * dy; a02 += dx * dz;
        a11 += dy * dy; a12 += dy * dz; a22 += dz * dz;
        b0 += dp * dx; b1 += dp * dy; b2 += dp * dz;
    }
    for (int o = kLanesPerRow / 2; o > 0; o >>= 1) {
        a00 += __shfl_xor_sync(0xffffffffu, a00, o); a01 += __shfl_xor_sync(0xffffffffu, a01, o);
        a02 += __shfl_xor_sync(0xffffffffu, a02, o); a11 += __shfl_xor_sync(0xffffffffu, a11, o);
        a12 += __shfl_xor_sync(0xffffffffu, a12, o); a22 += __shfl_xor_sync(0xffffffffu, a22, o);
        b0 += __shfl_xor_sync(0xffffffffu, b0, o); b1 += __shfl_xor_sync(0xffffffffu, b1, o);
        b2 += __shfl_xor_sync(0xffffffffu, b2, o);
    }
    if (!live || lane != 0) return;
    if (m.phiTrace != m.phi64) m.phiTrace[i] = pi;
    double* out = m.vfield + 3 * (size_t)i;
    if (hull) {
        out[0] = out[1] = out[2] = 0.0;
        return;
    }
    const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    if (det == 0.0 || !(det == det)) {
        out[0] = __longlong_as_double(0x7ff8000000000000ll);
        out[1] = out[2] = 0.0;
        return;
    }
    const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
    const double inv = 1.0 / det;
    out[0] = -(c00 * b0 + c01 * b1 + c02 * b2) * inv;
    out[1] = -(c01 * b0 + c11 * b1 + c12 * b2) * inv;
    out[2] = -(c02 * b0 + c12 * b1 + c22 * b2) * inv;
}

// Packed tetrahedron records, 128 bytes each: vertex 0 (3 floats) and the
// six-fold volume (float), the gradients n1, n2, n3 of the barycentric
// coordinates of vertices 1..3 (9 doubles: lambda_k(p) = n_k.(p - v0),
// lambda_0 = 1 - lambda_1 - lambda_2 - lambda_3), the neighbours (4 ints)
// and the vertex ids (4 ints).  A walk step then tests the four faces with
// three dot products, and the same lambdas are the interpolation weights
// |sub-volume| / volume of tetWeights (geometry_3d.cpp:916-980).  A flat
// tetrahedron stores zero gradients and volume 0.
constexpr int kTetWords = 32;
__global__ void k_pack_tets(DevMesh m, float* pack) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.ntets) return;
    float* o = pack + kTetWords * (size_t)t;
    int v[4];
    V3 P[4];
    for (int k = 0; k < 4; k++) {
        v[k] = m.tet_v[4 * t + k];
        P[k] = ld3(m.xyz, v[k]);
    }
    const V3 e1{P[1].x - P[0].x, P[1].y - P[0].y, P[1].z - P[0].z};
    const V3 e2{P[2].x - P[0].x, P[2].y - P[0].y, P[2].z - P[0].z};
    const V3 e3{P[3].x - P[0].x, P[3].y - P[0].y, P[3].z - P[0].z};
    const V3 c23{e2.y * e3.z - e2.z * e3.y, e2.z * e3.x - e2.x * e3.z, e2.x * e3.y - e2.y * e3.x};
    const V3 c31{e3.y * e1.z - e3.z * e1.y, e3.z * e1.x - e3.x * e1.z, e3.x * e1.y - e3.y * e1.x};
    const V3 c12{e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
    const double vol6 = e1.x * c23.x + e1.y * c23.y + e1.z * c23.z;
    const double inv = vol6 != 0.0 ? 1.0 / vol6 : 0.0;
    o[0] = m.xyz[3 * v[0]];
    o[1] = m.xyz[3 * v[0] + 1];
    o[2] = m.xyz[3 * v[0] + 2];
    o[3] = (float)vol6;
    if (vol6 != 0.0 && o[3] == 0.0f) o[3] = 1e-38f;  // keep "not flat" when the float underflows
    double* g = reinterpret_cast<double*>(o + 4);
    g[0] = c23.x * inv; g[1] = c23.y * inv; g[2] = c23.z * inv;
    g[3] = c31.x * inv; g[4] = c31.y * inv; g[5] = c31.z * inv;
    g[6] = c12.x * inv; g[7] = c12.y * inv; g[8] = c12.z * inv;
    int* oi = reinterpret_cast<int*>(o);
    for (int k = 0; k < 4; k++) {
        oi[22 + k] = m.tet_n[4 * t + k];
        oi[26 + k] = v[k];
    }
    oi[30] = oi[31] = 0;
}

__device__ V3 vertex_field(const DevMesh& m, int i) {
    const V3 E{m.vfield[3 * i], m.vfield[3 * i + 1], m.vfield[3 * i + 2]};
    if (E.x != E.x) {
        atomicOr(m.status, S_SINGULAR);
        return V3{0, 0, 0};
    }
    return E;
}

// The last tetrahedron an ion touched, from its packed record, with the
// vertex fields once interpolated from: RK stages that stay inside it need
// no memory traffic.  A record comes in one round trip; the vertex
// fields of the final tetrahedron of a walk take a second.  Every member is
// addressed with compile-time indices so that the cache lives in registers.
struct TetSlot {
    int t;
    int nb0, nb1, nb2, nb3;
    int v0, v1, v2, v3;
    V3 P0;
    V3 G1, G2, G3;
    float vol6;
    V3 F0, F1, F2, F3;
    bool hasF;
};
// `a` is the tetrahedron of the last lookup
struct TetCache {
    TetSlot a;
};

__device__ __forceinline__ int pick4(int k, int x0, int x1, int x2, int x3) {
    return k == 0 ? x0 : (k == 1 ? x1 : (k == 2 ? x2 : x3));
}

__device__ void load_slot(const DevMesh& m, TetSlot& s, int t) {
    const float4* p = reinterpret_cast<const float4*>(m.tetpack + kTetWords * (size_t)t);
    const float4 q0 = __ldg(p);
    const double2 g0 = __ldg(reinterpret_cast<const double2*>(p + 1));
    const double2 g1 = __ldg(reinterpret_cast<const double2*>(p + 2));
    const double2 g2 = __ldg(reinterpret_cast<const double2*>(p + 3));
    const double2 g3 = __ldg(reinterpret_cast<const double2*>(p + 4));
    const double2 g4 = __ldg(reinterpret_cast<const double2*>(p + 5));  // g[8], neighbours 0, 1
    const int4 q6 = __ldg(reinterpret_cast<const int4*>(p + 6));       // neighbours 2, 3, vertices 0, 1
    const int4 q7 = __ldg(reinterpret_cast<const int4*>(p + 7));       // vertices 2, 3, padding
    s.t = t;
    s.P0 = V3{q0.x, q0.y, q0.z};
    s.vol6 = q0.w;
    s.G1 = V3{g0.x, g0.y, g1.x};
    s.G2 = V3{g1.y, g2.x, g2.y};
    s.G3 = V3{g3.x, g3.y, g4.x};
    const long long nb01 = __double_as_longlong(g4.y);
    s.nb0 = (int)(unsigned)(nb01 & 0xffffffffll);
    s.nb1 = (int)(unsigned)((unsigned long long)nb01 >> 32);
    s.nb2 = q6.x;
    s.nb3 = q6.y;
    s.v0 = q6.z;
    s.v1 = q6.w;
    s.v2 = q7.x;
    s.v3 = q7.y;
    s.hasF = false;
}

// Barycentric coordinates of p in the slot's tetrahedron and bounds on their
// rounding error (about a thousand ulps of the terms summed)
struct Bary {
    double l0, l1, l2, l3, e0, e1, e2, e3;
};
__device__ __forceinline__ Bary lambdas(const TetSlot& S, V3 p) {
    const double dx = p.x - S.P0.x, dy = p.y - S.P0.y, dz = p.z - S.P0.z;
    Bary b;
    b.l1 = S.G1.x * dx + S.G1.y * dy + S.G1.z * dz;
    b.l2 = S.G2.x * dx + S.G2.y * dy + S.G2.z * dz;
    b.l3 = S.G3.x * dx + S.G3.y * dy + S.G3.z * dz;
    const double a1 = fabs(S.G1.x * dx) + fabs(S.G1.y * dy) + fabs(S.G1.z * dz);
    const double a2 = fabs(S.G2.x * dx) + fabs(S.G2.y * dy) + fabs(S.G2.z * dz);
    const double a3 = fabs(S.G3.x * dx) + fabs(S.G3.y * dy) + fabs(S.G3.z * dz);
    b.l0 = 1.0 - b.l1 - b.l2 - b.l3;
    b.e1 = 1e-13 * a1;
    b.e2 = 1e-13 * a2;
    b.e3 = 1e-13 * a3;
    b.e0 = 1e-13 * (1.0 + a1 + a2 + a3);
    return b;
}

// Makes `a` hold tetrahedron t (loading it unless it is already there)
__device__ __forceinline__ void cache_tet(const DevMesh& m, TetCache& c, int t) {
    if (c.a.t == t) return;
    load_slot(m, c.a, t);
}

// Side of face k (opposite vertex k) that p lies on: -1 beyond it.  The
// barycentric coordinate decides unless it is within its rounding bound of
// zero, or the tetrahedron is flat; then the exact predicate on the vertex
// coordinates decides (as Predicates::orient3d does in the reference).
__device__ __noinline__ int face_side_exact(const float* xyz, double snap, int i0, int i1, int i2, V3 p) {
    return orient_sign(ld3(xyz, i0), ld3(xyz, i1), ld3(xyz, i2), p, snap);
}
__device__ __forceinline__ bool beyond(const DevMesh& m, const TetSlot& S, int k, V3 p, double lam, double err) {
    if (S.vol6 != 0.0f) {
        if (lam < -err) return true;
        if (lam > err) return false;
    }
    const int i0 = pick4(kFaceDev[k][0], S.v0, S.v1, S.v2, S.v3);
    const int i1 = pick4(kFaceDev[k][1], S.v0, S.v1, S.v2, S.v3);
    const int i2 = pick4(kFaceDev[k][2], S.v0, S.v1, S.v2, S.v3);
    return face_side_exact(m.xyz, m.snap, i0, i1, i2, p) < 0;
}

// findTetrahedron through the cache: on return c.a holds p's tetrahedron
// (result 0; *found, when given, p's barycentric coordinates in it), or -1
// when p is outside the mesh, -2 when the walk exceeded its bound.  The faces are tested in an order rotating from walk step to
// walk step; the walk leaves through the first face p lies beyond.
__device__ __forceinline__ int locate_cached(const DevMesh& m, TetCache& c, V3 p, int t, int limit, unsigned& rot,
                                             Bary* found = nullptr) {
    if (t < 0) return -1;
    for (int step = 0; step < limit; step++) {
        cache_tet(m, c, t);
        const TetSlot& S = c.a;
        const Bary b = lambdas(S, p);
        const int r = (int)(rot++ & 3u);
        int next = 0;
        bool moved = false;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = (r + j) & 3;
            if (!moved) {
                const double lam = k == 0 ? b.l0 : (k == 1 ? b.l1 : (k == 2 ? b.l2 : b.l3));
                const double err = k == 0 ? b.e0 : (k == 1 ? b.e1 : (k == 2 ? b.e2 : b.e3));
                if (beyond(m, S, k, p, lam, err)) {
                    next = pick4(k, S.nb0, S.nb1, S.nb2, S.nb3);
                    moved = true;
                }
            }
        }
        if (!moved) {
            if (found) *found = b;
            return 0;
        }
        if (next < 0) return -1;
        t = next;
    }
    return -2;
}

// Field at p: walk from `guess`, interpolate the vertex fields with the
// weights |lambda_k| (1/4 each in a flat tetrahedron).  *located is the
// tetrahedron holding p (unchanged when p is outside the mesh).
__device__ __forceinline__ bool fast_field(const DevMesh& m, TetCache& c, V3 p, int guess, int limit, unsigned& rot, V3* E,
                           int* located) {
    *E = V3{0, 0, 0};
    Bary b;  // the walk's last coordinates: p's in the tetrahedron it found
    const int sl = locate_cached(m, c, p, guess, limit, rot, &b);
    if (sl == -2) return false;
    if (sl < 0) return true;
    TetSlot& S = c.a;
    *located = S.t;
    if (!S.hasF) {
        S.F0 = vertex_field(m, S.v0);
        S.F1 = vertex_field(m, S.v1);
        S.F2 = vertex_field(m, S.v2);
        S.F3 = vertex_field(m, S.v3);
        S.hasF = true;
    }
    double w0 = 0.25, w1 = 0.25, w2 = 0.25, w3 = 0.25;
    if (S.vol6 != 0.0f) {
        w0 = fabs(b.l0);
        w1 = fabs(b.l1);
        w2 = fabs(b.l2);
        w3 = fabs(b.l3);
    }
    E->x = w0 * S.F0.x + w1 * S.F1.x + w2 * S.F2.x + w3 * S.F3.x;
    E->y = w0 * S.F0.y + w1 * S.F1.y + w2 * S.F2.y + w3 * S.F3.y;
    E->z = w0 * S.F0.z + w1 * S.F1.z + w2 * S.F2.z + w3 * S.F3.z;
    return true;
}

__device__ double potential_at(const DevMesh& m, const double* phi, V3 p, int t) {
    const int* v = m.tet_v + 4 * t;
    double w[4];
    weights(m, t, p, w);
    return w[0] * phi[v[0]] + w[1] * phi[v[1]] + w[2] * phi[v[2]] + w[3] * phi[v[3]];
}

// Tetrahedron t2 shares a vertex with t1 and is not t1: membership of the
// set Geometry_3d::Table::adjacentTetrahedra (geometry_3d.cpp:1046-1096)
// builds for t1 by a walk over face neighbours.
__device__ bool shares_vertex(const DevMesh& m, int t1, int t2) {
    if (t2 < 0 || t2 == t1) return false;
    for (int a = 0; a < 4; a++) {
        const int va = m.tet_v[4 * t1 + a];
        for (int b = 0; b < 4; b++)
            if (va == m.tet_v[4 * t2 + b]) return true;
    }
    return false;
}

// Geometry_3d::Table::isBoundaryTetrahedron (geometry_3d.cpp:819-828)
__device__ bool boundary_tet(const DevMesh& m, int t) {
    for (int a = 0; a < 4; a++)
        if (m.flags[m.tet_v[4 * t + a]] & F_HULL) return true;
    return false;
}

// The accept / retry rule of the steppers other than the error-restricted
// one of the main path: 0 NONE takes every step; 2 geometryRestricted_stepper
// (trajectory_3d.cpp:427-452) accepts a point in a tetrahedron sharing a
// vertex with the current one (or outside the mesh from a boundary
// tetrahedron), grows dt by 1.1 while the point stays in the current
// tetrahedron and shrinks it by 0.9 otherwise; 3 adaptive_stepper
// (:454-532) shrinks dt by 0.1 when the point leaves that set, then applies
// the error rule.  Returns 1 to accept, 0 to retry with the updated dt; *nt
// is the located tetrahedron when *located.
__device__ __forceinline__ int stepper_verdict(const DevMesh& m, TetCache& fc, const TraceParams& tp, V3 nx, int tet,
                                            int& cur, unsigned& rot, double rel, double* dt, int* nt, bool* located) {
    *located = false;
    if (tp.stepper == 0) return 1;
    if (tp.stepper == 2 || tp.stepper == 3) {
        const int nsl = locate_cached(m, fc, nx, cur, tp.walk_limit, rot);
        *nt = nsl >= 0 ? fc.a.t : nsl;
        if (*nt == -2) atomicOr(m.status, S_WALK_LIMIT);
        if (*nt >= 0) cur = *nt;
        *located = true;
        if (tp.stepper == 2) {
            if (*nt < 0 && boundary_tet(m, tet)) return 1;
            if (shares_vertex(m, tet, *nt)) return 1;
            if (*nt == tet) {
                *dt *= 1.1;
            } else {
                if (*dt == tp.dt_min) return 1;
                *dt *= 0.9;
            }
            *located = false;
            return 0;
        }
        if (*nt >= 0 && *nt != tet && !shares_vertex(m, tet, *nt)) {
            *dt *= 0.1;
            *located = false;
            return 0;
        }
    }
    if (rel < tp.tol || *dt == tp.dt_min) {
        if (rel != 0.0) {
            const double tmp = *dt * pow(tp.tol / rel, 0.25) * 0.9;
            if (tmp < *dt) *dt *= 1.1; else *dt = tmp;
        }
        return 1;
    }
    const double tmp = *dt * pow(tp.tol / rel, 0.25) * 0.9;
    if (tmp > *dt) *dt *= 0.9; else *dt = tmp;
    *located = false;
    return 0;
}

// Point idx of the path of ion `slot` (Trajectory_3d::phaseVector,
// trajectory_3d.h:40-80), dropped beyond the path's capacity.
__device__ __forceinline__ void path_point(const TraceParams& tp, int slot, int idx, double t, V3 x, V3 v, int tet) {
    if (idx >= tp.path_cap) return;
    float4* p = reinterpret_cast<float4*>(tp.path + ((size_t)slot * tp.path_cap + idx) * 8);
    p[0] = make_float4((float)t, (float)x.x, (float)x.y, (float)x.z);
    p[1] = make_float4((float)v.x, (float)v.y, (float)v.z, __int_as_float(tet < 0 ? -1 : tet));
}

// The error vector of the latest trial step, parked in words 6..11 of the
// ion's error record so that it holds no registers across the stepper's
// point location.
__device__ __forceinline__ void path_trial_error(const TraceParams& tp, int slot, V3 ex, V3 ev) {
    float* e = tp.path_err + 12 * (size_t)slot + 6;
    e[0] = (float)ex.x; e[1] = (float)ex.y; e[2] = (float)ex.z;
    e[3] = (float)ev.x; e[4] = (float)ev.y; e[5] = (float)ev.z;
}

// Trajectory_3d::cumulative_error (trajectory_3d.cpp:683-700) with the
// accepted step's error: each of the six components becomes
// sqrt(current^2 + step^2), in float as the reference keeps it.
__device__ __forceinline__ void path_error(const TraceParams& tp, int slot) {
    float* e = tp.path_err + 12 * (size_t)slot;
#pragma unroll
    for (int j = 0; j < 6; j++) e[j] = sqrtf(e[j] * e[j] + e[6 + j] * e[6 + j]);
}

// One Cash-Karp trial step (o5_integrator, trajectory_3d.cpp:583-676) of
// length dt from (x, v), its arithmetic in R: FP64, or FP32 as the reference
// integrates.  The state enters and leaves in double (rounded to R on the
// way in, so in FP32 it is the float state); the points of the stages are
// located and their fields interpolated as in FP64, then rounded to R.
// *rel: the largest relative error of a position or velocity component (as
// errorRestricted_stepper forms it, trajectory_3d.cpp:366-387).  Returns
// false when a walk exceeded its bound.  s0: the first stage's field, kept
// across the trials of a step.
// The stages run as a loop that is not unrolled, the tableau's rows read from
// constant memory: the kernel then holds one copy of the point location and
// interpolation in its hot loop instead of six.  A flight is a long chain of
// dependent steps on few warps per SM, and the unrolled body stalled on
// instruction fetch more than on anything else; the arithmetic, and so every
// result, is the same.
__constant__ double kCashKarpB[6][5] = {{0, 0, 0, 0, 0},
                                        {1.0 / 5.0, 0, 0, 0, 0},
                                        {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
                                        {3.0 / 10.0, -9.0 / 10.0, 6.0 / 5.0, 0, 0},
                                        {-11.0 / 54.0, 5.0 / 2.0, -70.0 / 27.0, 35.0 / 27.0, 0},
                                        {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0,
                                         253.0 / 4096.0}};
// The first stage's field of the current state.  Every trial of a step
// evaluates its first stage at the same point, so a retried trial (after the
// stepper shrank dt) takes the field from here and starts its next walk from
// the tetrahedron it was found in.  The tetrahedron holding a point does not
// depend on where a walk to it starts (short of a point on a shared face,
// where both sides interpolate the same field), so the flights are those of
// the recomputation; on 4096 probe ions in each precision they were
// identical bit for bit.
struct Stage0 {
    V3 E;
    int tet;
    bool have;
};
template <typename R>
__device__ __forceinline__ bool ck_trial(const DevMesh& m, TetCache& fc, const TraceParams& tp, unsigned& rot, int& cur,
                                         V3 x, V3 v, double k, double dt, V3* nxo, V3* nvo, V3* exo, V3* evo,
                                         double* relo, Stage0& s0) {
    constexpr double C5[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};
    constexpr double C4[6] = {2825.0 / 27648.0, 0.0, 18575.0 / 48384.0, 13525.0 / 55296.0, 277.0 / 14336.0, 1.0 / 4.0};
    const R xx = (R)x.x, xy = (R)x.y, xz = (R)x.z, vx = (R)v.x, vy = (R)v.y, vz = (R)v.z;
    const R kk = (R)k, h = (R)dt;
    R dx[6][3], dv[6][3];
    bool walkOk = true;
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
        R px = xx, py = xy, pz = xz, qx = vx, qy = vy, qz = vz;
#pragma unroll 1
        for (int j = 0; j < s; j++) {
            const R b = (R)kCashKarpB[s][j];
            px += b * dx[j][0]; py += b * dx[j][1]; pz += b * dx[j][2];
            qx += b * dv[j][0]; qy += b * dv[j][1]; qz += b * dv[j][2];
        }
        V3 E;
        if (s == 0 && s0.have) {
            E = s0.E;
            cur = s0.tet;
        } else {
            walkOk &= fast_field(m, fc, V3{(double)px, (double)py, (double)pz}, cur, tp.walk_limit, rot, &E, &cur);
            if (s == 0) {
                s0.E = E;
                s0.tet = cur;
                s0.have = true;
            }
        }
        dv[s][0] = (R)E.x * kk * h; dv[s][1] = (R)E.y * kk * h; dv[s][2] = (R)E.z * kk * h;
        dx[s][0] = qx * h; dx[s][1] = qy * h; dx[s][2] = qz * h;
    }
    R nx[3] = {xx, xy, xz}, nv[3] = {vx, vy, vz}, ex[3] = {0, 0, 0}, ev[3] = {0, 0, 0};
#pragma unroll
    for (int s = 0; s < 6; s++) {
        const R c5 = (R)C5[s], dc = (R)(C5[s] - C4[s]);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            nx[c] += c5 * dx[s][c];
            nv[c] += c5 * dv[s][c];
            ex[c] += dc * dx[s][c];
            ev[c] += dc * dv[s][c];
        }
    }
    R rel = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (nx[c] != (R)0) rel = fmax(rel, fabs(ex[c] / nx[c]));
        if (nv[c] != (R)0) rel = fmax(rel, fabs(ev[c] / nv[c]));
    }
    *nxo = V3{(double)nx[0], (double)nx[1], (double)nx[2]};
    *nvo = V3{(double)nv[0], (double)nv[1], (double)nv[2]};
    *exo = V3{(double)ex[0], (double)ex[1], (double)ex[2]};
    *evo = V3{(double)ev[0], (double)ev[1], (double)ev[2]};
    *relo = (double)rel;
    return walkOk;
}

// errorRestricted_stepper's rule (trajectory_3d.cpp:396-421) in R: accept
// when rel is below the threshold or the step is at its floor, and adjust
// dt by (tol / rel)^(1/4) with the safety factor 0.9, growing by at most
// 1.1 and shrinking by at least 0.9.  Returns true to accept.
template <typename R>
__device__ __forceinline__ bool error_rule(double relIn, const TraceParams& tp, double* dtIo) {
    const R rel = (R)relIn, tol = (R)tp.tol;
    R dt = (R)*dtIo;
    const bool accept = rel < tol || dt == (R)tp.dt_min;
    if (!accept || rel != (R)0) {
        const R tmp = dt * (R)pow(tol / rel, (R)0.25) * (R)0.9;
        if (accept) dt = tmp < dt ? dt * (R)1.1 : tmp;
        else dt = tmp > dt ? dt * (R)0.9 : tmp;
    }
    *dtIo = (double)dt;
    return accept;
}

// One ion from x0 (velocity v0, charge/mass k) into *out; with kPath its
// path and error estimate go to slot `slot` of tp's path buffers (a
// separate instantiation, so that the flights without a path keep their
// registers).
// kPrec: the arithmetic of the Cash-Karp steps (TraceParams::precision),
// fixed per instantiation so that each kernel holds only its own registers.
template <bool kPath, int kPrec>
__device__ __forceinline__ void trace_ion(const DevMesh& m, V3 x, V3 v, double k, int guessTet, const TraceParams& tp,
                                          unsigned rot, int slot, ImpactOut* out) {
    const V3 x0 = x;
    ImpactOut res;
    TetCache fc;
    fc.a.t = -1;
    fc.a.hasF = false;
    double time = 0.0;
    int tet = locate(m, x, guessTet, tp.walk_limit, rot);
    res.steps = 0;
    res.trials = 0;
    res.last_tet = tet;
    res.last_pos[0] = (float)x.x; res.last_pos[1] = (float)x.y; res.last_pos[2] = (float)x.z;
    res.last_phi = 0.0f;
    if (kPath) {
        float* e = tp.path_err + 12 * (size_t)slot;
#pragma unroll
        for (int j = 0; j < 12; j++) e[j] = 0.0f;
        if (tet >= 0) path_point(tp, slot, 0, 0.0, x, v, tet);  // Trajectory_3d::init (:99-123)
    }
    if (tet < 0) {
        if (tet == -2) atomicOr(m.status, S_WALK_LIMIT);
        res.status = -1;  // Trajectory_3d::init: initial point is outside
        res.stop[0] = (float)x.x; res.stop[1] = (float)x.y; res.stop[2] = (float)x.z;
        res.stop_time = 0.0f;
        *out = res;
        return;
    }
    V3 E0;
    int cur = tet;  // tetrahedron of the last located point: the next walk starts there
    if (!fast_field(m, fc, x, tet, tp.walk_limit, rot, &E0, &cur)) atomicOr(m.status, S_WALK_LIMIT);
    int status;
    if (E0.x == 0.0 && E0.y == 0.0 && E0.z == 0.0) {
        status = 1;  // NO_FIELD
    } else {
        status = 3;  // ITERATION_LIMIT_PASSED unless another exit is taken
        double dt = tp.dt0;
        for (int it = 0; it < tp.max_steps; it++) {
            V3 nx, nv;
            double used = dt;
            bool accepted = false;
            bool located = false;  // the accepted trial point is already located (steppers 2, 3)
            int nt = -1;
            // FP32 arithmetic for this step: always with precision 1, and
            // with precision 2 once the ion is beyond fp64_radius of its start
            const double ddx = x.x - x0.x, ddy = x.y - x0.y, ddz = x.z - x0.z;
            const bool lo = kPrec != 0 && tp.integrator == 1 &&
                            (kPrec == 1 || ddx * ddx + ddy * ddy + ddz * ddz > tp.fp64_radius2);
            Stage0 s0;
            s0.have = false;
            for (int tries = 0; tries < tp.stepper_limit; tries++) {
                res.trials++;
                if (lo) {
                    if ((float)dt < (float)tp.dt_min) dt = (double)(float)tp.dt_min;
                } else if (dt < tp.dt_min) {
                    dt = tp.dt_min;
                }
                used = dt;
                if (tp.integrator == 0) {
                    // o1_integrator (trajectory_3d.cpp:560-581): Euler; the
                    // error estimate is the next state times dt^2
                    V3 E;
                    if (!fast_field(m, fc, x, cur, tp.walk_limit, rot, &E, &cur)) atomicOr(m.status, S_WALK_LIMIT);
                    nv = V3{v.x + dt * E.x * k, v.y + dt * E.y * k, v.z + dt * E.z * k};
                    nx = V3{x.x + dt * v.x, x.y + dt * v.y, x.z + dt * v.z};
                    const bool any = nx.x != 0.0 || nx.y != 0.0 || nx.z != 0.0 || nv.x != 0.0 || nv.y != 0.0 ||
                                     nv.z != 0.0;
                    const double rel = any ? dt * dt : 0.0;
                    const int verdict = stepper_verdict(m, fc, tp, nx, tet, cur, rot, rel, &dt, &nt, &located);
                    if (verdict > 0) {
                        accepted = true;
                        break;
                    }
                    continue;
                }
                V3 ex, evv;
                double rel;
                bool walkOk;
                if (kPrec == 1) walkOk = ck_trial<float>(m, fc, tp, rot, cur, x, v, k, dt, &nx, &nv, &ex, &evv, &rel, s0);
                else if (kPrec == 0) walkOk = ck_trial<double>(m, fc, tp, rot, cur, x, v, k, dt, &nx, &nv, &ex, &evv, &rel, s0);
                else walkOk = lo ? ck_trial<float>(m, fc, tp, rot, cur, x, v, k, dt, &nx, &nv, &ex, &evv, &rel, s0)
                                 : ck_trial<double>(m, fc, tp, rot, cur, x, v, k, dt, &nx, &nv, &ex, &evv, &rel, s0);
                if (!walkOk) atomicOr(m.status, S_WALK_LIMIT);
                if (kPath) path_trial_error(tp, slot, ex, evv);
                if (tp.stepper != 1) {
                    const int verdict = stepper_verdict(m, fc, tp, nx, tet, cur, rot, rel, &dt, &nt, &located);
                    if (verdict > 0) {
                        accepted = true;
                        break;
                    }
                    continue;
                }
                if (kPrec == 0 ? error_rule<double>(rel, tp, &dt)
                               : (lo ? error_rule<float>(rel, tp, &dt) : error_rule<double>(rel, tp, &dt))) {
                    accepted = true;
                    break;
                }
            }
            if (!accepted) {
                status = 2;  // STEPPER_LIMIT_PASSED
                break;
            }
            if (!located) {
                const int nsl = locate_cached(m, fc, nx, cur, tp.walk_limit, rot);
                nt = nsl >= 0 ? fc.a.t : nsl;
                if (nt == -2) atomicOr(m.status, S_WALK_LIMIT);
            }
            res.steps++;
            if (kPath) {
                // the error of the accepted step: o1_integrator's is the new
                // state times dt^2 (trajectory_3d.cpp:568-576)
                if (tp.integrator == 0) {
                    const double d2 = used * used;
                    path_trial_error(tp, slot, V3{nx.x * d2, nx.y * d2, nx.z * d2}, V3{nv.x * d2, nv.y * d2, nv.z * d2});
                }
                path_error(tp, slot);
                path_point(tp, slot, res.steps, time + used, nx, nv, nt);
            }
            const double tnext = lo ? (double)((float)time + (float)used) : time + used;
            if (nt < 0) {
                // left the mesh: the previous point is the last inside it
                res.last_tet = tet;
                res.last_pos[0] = (float)x.x; res.last_pos[1] = (float)x.y; res.last_pos[2] = (float)x.z;
                x = nx;
                v = nv;
                time = tnext;
                tet = -1;
                status = 5;  // SYSTEM_LIMIT_PASSED
                break;
            }
            x = nx;
            v = nv;
            time = tnext;
            tet = nt;
            cur = nt;
        }
    }
    if (tet >= 0) {
        res.last_tet = tet;
        res.last_pos[0] = (float)x.x; res.last_pos[1] = (float)x.y; res.last_pos[2] = (float)x.z;
    }
    res.last_phi = res.last_tet >= 0 ? (float)potential_at(m, m.phiTrace, V3{res.last_pos[0], res.last_pos[1],
                                                                              res.last_pos[2]},
                                                           res.last_tet)
                                     : 0.0f;
    // extrapolate to the top plane along the last velocity
    const double dtz = (tp.top_z - x.z) / v.z;
    res.stop[0] = (float)(x.x + dtz * v.x);
    res.stop[1] = (float)(x.y + dtz * v.y);
    res.stop[2] = (float)(x.z + dtz * v.z);
    res.stop_time = (float)(time + dtz);
    res.status = status;
    if (kPath) {
        // Trajectory_3d::extrapolate (trajectory_3d.cpp:303-332): the last
        // point, located from the last tetrahedron (outside stays outside;
        // a flight at rest, NO_FIELD, extrapolates to a non-finite point)
        const V3 p{x.x + dtz * v.x, x.y + dtz * v.y, x.z + dtz * v.z};
        int pt = -1;
        if (tet >= 0 && isfinite(p.x) && isfinite(p.y) && isfinite(p.z)) {
            pt = locate(m, p, tet, tp.walk_limit, rot);
            if (pt == -2) atomicOr(m.status, S_WALK_LIMIT);
        }
        path_point(tp, slot, res.steps + 1, time + dtz, p, v, pt);
        const float fdt = (float)dtz;
        if (fdt > 0.0f) {
            float* e = tp.path_err + 12 * (size_t)slot;
#pragma unroll
            for (int j = 0; j < 3; j++) e[j] += fdt * e[3 + j];
        }
    }
    *out = res;
}

// perWarp: the ions each warp carries (its first perWarp lanes; the rest
// return at once).  A flight is a chain of dependent loads whose branches
// (walk lengths, rejected steps) differ from ion to ion, so a warp runs its
// lanes' flights largely one after another: few ions per warp over every
// warp the SMs can hold beats full warps on a fraction of them.
template <bool kPath, int kPrec>
__global__ void k_trace(DevMesh m, int nIons, int perWarp, const float* start, const float* vel, const float* qm,
                        const int32_t* guess, TraceParams tp, ImpactOut* out) {
    const int lane = threadIdx.x & 31;
    const int ion = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * perWarp + lane;
    if (lane >= perWarp || ion >= nIons) return;
    const V3 x{start[3 * ion], start[3 * ion + 1], start[3 * ion + 2]};
    const V3 v = vel ? V3{vel[3 * ion], vel[3 * ion + 1], vel[3 * ion + 2]} : V3{0, 0, 0};
    trace_ion<kPath, kPrec>(m, x, v, qm[ion], guess ? guess[ion] : 0, tp, (unsigned)ion * 7u, ion, out + ion);
}

// A single ion from rest, its start passed by value (no staging copy)
template <bool kPath, int kPrec>
__global__ void k_trace_one(DevMesh m, float x, float y, float z, float vx, float vy, float vz, float qm, int guess,
                            TraceParams tp, ImpactOut* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    trace_ion<kPath, kPrec>(m, V3{x, y, z}, V3{vx, vy, vz}, qm, guess, tp, 0u, 0, out);
}

__global__ void k_potential_at(DevMesh m, int n, const float* xyz, const int32_t* guess, int limit, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned rot = (unsigned)i;
    const V3 p{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    const int t = locate(m, p, guess ? guess[i] : 0, limit, rot);
    if (t == -2) atomicOr(m.status, S_WALK_LIMIT);
    out[i] = t >= 0 ? (float)potential_at(m, m.phi64, p, t) : 0.0f;
}

}  // namespace

void launch_trace(const DevMesh& m, int nIons, const float* start, const float* vel, const float* qm,
                  const int32_t* guess, TraceParams tp, ImpactOut* out, cudaStream_t s) {
    if (nIons <= 0) return;
    count_launch();
    // ions per warp: as few as fill every warp slot the SMs hold at this
    // kernel's register count (one wave), one warp per block
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto go = [&](auto kernel) {
        int perSM = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, 32, 0) != cudaSuccess || perSM < 1) perSM = 1;
        const long long slots = (long long)perSM * sms;
        const int perWarp = (int)std::min<long long>(32, std::max<long long>(1, (nIons + slots - 1) / slots));
        const int warps = (nIons + perWarp - 1) / perWarp;
        kernel<<<warps, 32, 0, s>>>(m, nIons, perWarp, start, vel, qm, guess, tp, out);
    };
    const int prec = tp.precision == 1 ? 1 : (tp.precision == 2 ? 2 : 0);
    if (tp.path) {
        if (prec == 0) go(k_trace<true, 0>); else if (prec == 1) go(k_trace<true, 1>); else go(k_trace<true, 2>);
    } else {
        if (prec == 0) go(k_trace<false, 0>); else if (prec == 1) go(k_trace<false, 1>); else go(k_trace<false, 2>);
    }
}
void launch_pack_tets(const DevMesh& m, float* pack, cudaStream_t s) {
    if (m.ntets > 0) { count_launch(); k_pack_tets<<<(m.ntets + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, pack); }
}
void launch_vertex_fields(const DevMesh& m, cudaStream_t s, const int32_t* cells, int count) {
    const long long items = cells ? count : m.n;
    if (m.n > 0 && items > 0) {
        count_launch();
        const long long threads = items * kLanesPerRow;
        k_vertex_fields<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(m, cells, (int)items);
    }
}
void launch_trace_one(const DevMesh& m, const float start[3], const float vel[3], float qm, int guess, TraceParams tp,
                      ImpactOut* out, cudaStream_t s) {
    count_launch();
    auto go = [&](auto kernel) {
        kernel<<<1, 32, 0, s>>>(m, start[0], start[1], start[2], vel[0], vel[1], vel[2], qm, guess, tp, out);
    };
    const int prec = tp.precision == 1 ? 1 : (tp.precision == 2 ? 2 : 0);
    if (tp.path) {
        if (prec == 0) go(k_trace_one<true, 0>); else if (prec == 1) go(k_trace_one<true, 1>); else go(k_trace_one<true, 2>);
    } else {
        if (prec == 0) go(k_trace_one<false, 0>); else if (prec == 1) go(k_trace_one<false, 1>);
        else go(k_trace_one<false, 2>);
    }
}
void launch_potential_at(const DevMesh& m, int n, const float* xyz, const int32_t* guess, int walkLimit, float* out,
                         cudaStream_t s) {
    if (n > 0) { count_launch(); k_potential_at<<<(n + kBlock - 1) / kBlock, kBlock, 0, s>>>(m, n, xyz, guess, walkLimit, out); }
}

}  // namespace tgd

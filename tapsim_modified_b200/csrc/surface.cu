// Surface kernels: per-cell field (first-order least squares gradient), the
// evaporation-field ratio with its argmax, surface-set maintenance, the
// cell-flip removal with its in-place coupling update, the coordination
// rewrite and the local surface normal.
#include "kernels.cuh"

namespace tgd {
namespace {

constexpr int kBlock = 256;

// Grid_3d::Table::field_o1 (tapsim/grid_3d.cpp:909-991): least-squares fit
// of (phi_j - phi_i) against (x_j - x_i) over neighbours with a non-zero
// coupling, E = -grad phi; zero on hull nodes.  FP64 throughout (the
// reference evaluates the same normal equations in float).
__device__ bool field_o1(const DevMesh& m, int i, double E[3]) {
    E[0] = E[1] = E[2] = 0.0;
    if (m.flags[i] & F_HULL) return true;
    const double xi = m.xyz[3 * i], yi = m.xyz[3 * i + 1], zi = m.xyz[3 * i + 2];
    const double pi = m.phi64[i];
    double a00 = 0, a01 = 0, a02 = 0, a11 = 0, a12 = 0, a22 = 0, b0 = 0, b1 = 0, b2 = 0;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) {
        if (m.c64[q] == 0.0) continue;
        const int j = m.col[q];
        const double dx = (double)m.xyz[3 * j] - xi, dy = (double)m.xyz[3 * j + 1] - yi, dz = (double)m.xyz[3 * j + 2] - zi;
        const double dp = m.phi64[j] - pi;
        a00 += dx * dx; a01 += dx * dy; a02 += dx * dz;
        a11 += dy * dy; a12 += dy * dz; a22 += dz * dz;
        b0 += dp * dx; b1 += dp * dy; b2 += dp * dz;
    }
    // symmetric 3x3 solve by cofactors
    const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    if (det == 0.0 || !(det == det)) return false;
    const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
    const double inv = 1.0 / det;
    const double g0 = (c00 * b0 + c01 * b1 + c02 * b2) * inv;
    const double g1 = (c01 * b0 + c11 * b1 + c12 * b2) * inv;
    const double g2 = (c02 * b0 + c12 * b1 + c22 * b2) * inv;
    E[0] = -g0;
    E[1] = -g1;
    E[2] = -g2;
    return (g0 == g0) && (g1 == g1) && (g2 == g2);
}

__global__ void k_field_o1(DevMesh m, const int32_t* nodes, int count, double* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    double E[3];
    if (!field_o1(m, nodes[t], E)) atomicOr(m.status, S_SINGULAR);
    out[3 * t] = E[0];
    out[3 * t + 1] = E[1];
    out[3 * t + 2] = E[2];
}

// Grid_3d::Table::force (grid_3d.cpp:1201-1236) in FP64: the dielectric
// force on cell i, sum over its neighbours j of
// eps0 c_ij (phi_j - phi_i)^2 (1/eps_j - 1/eps_i) (x_j - x_i) / |x_j - x_i|^2.
__device__ void cell_force(const DevMesh& m, int i, double F[3]) {
    F[0] = F[1] = F[2] = 0.0;
    const double xi = m.xyz[3 * i], yi = m.xyz[3 * i + 1], zi = m.xyz[3 * i + 2];
    const double pi = m.phi64[i];
    const double ei = 1.0 / (double)m.types[m.type[i]].epsilon;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) {
        const int j = m.col[q];
        const double dp = m.phi64[j] - pi;
        const double mag = dp * dp * kEpsilon0 * m.c64[q] * (1.0 / (double)m.types[m.type[j]].epsilon - ei);
        const double dx = (double)m.xyz[3 * j] - xi, dy = (double)m.xyz[3 * j + 1] - yi, dz = (double)m.xyz[3 * j + 2] - zi;
        const double s = mag / (dx * dx + dy * dy + dz * dz);
        F[0] += dx * s;
        F[1] += dy * s;
        F[2] += dz * s;
    }
}

// Potential, field_o1 and force of cells nodes[0..count) (all cells when
// nodes is null), as float: the values File_Io::LogGrid::push
// (logGrid.cpp:119-143) and LogSurface::prepare (logSurface.cpp:159-201)
// collect.  Any output may be null.
__global__ void k_cell_values(DevMesh m, const int32_t* nodes, int count, float* phi, float* field, float* force) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int i = nodes ? nodes[k] : k;
    if (phi) phi[k] = (float)m.phi64[i];
    if (field) {
        double E[3];
        if (!field_o1(m, i, E)) atomicOr(m.status, S_SINGULAR);
        field[3 * (size_t)k] = (float)E[0];
        field[3 * (size_t)k + 1] = (float)E[1];
        field[3 * (size_t)k + 2] = (float)E[2];
    }
    if (force) {
        double F[3];
        cell_force(m, i, F);
        force[3 * (size_t)k] = (float)F[0];
        force[3 * (size_t)k + 1] = (float)F[1];
        force[3 * (size_t)k + 2] = (float)F[2];
    }
}

// A removable, non-vacuum cell with a vacuum neighbour across a face of
// positive area (Surface_3d::Table::init/update, surface_3d.cpp:50-119).
__device__ bool is_surface_candidate(const DevMesh& m, int i, int vacuumId) {
    const int t = m.type[i];
    if (t == vacuumId) return false;
    if (t < 0 || !m.types[t].present) {
        atomicOr(m.status, S_UNKNOWN_TYPE);
        return false;
    }
    if (!m.types[t].removable) return false;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++)
        if (m.type[m.col[q]] == vacuumId && m.area_pos[q]) return true;
    return false;
}

__device__ void surface_insert(const DevMesh& m, Surface sf, int i) {
    if (m.flags[i] & F_SURFACE) return;
    const int s = atomicAdd(sf.count, 1);
    if (s < sf.capacity) {
        sf.list[s] = i;
        sf.slot[i] = s;
        m.flags[i] |= F_SURFACE;
    }
}

__global__ void k_surface_init(DevMesh m, Surface sf, int vacuumId) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    m.flags[i] &= ~F_SURFACE;
    if (is_surface_candidate(m, i, vacuumId)) {
        const int s = atomicAdd(sf.count, 1);
        if (s < sf.capacity) {
            sf.list[s] = i;
            sf.slot[i] = s;
            m.flags[i] |= F_SURFACE;
        }
    }
}

// keys[0]: (ratio, lowest index) argmax; keys[1]: (z, lowest index) apex;
// acc[0]: sum of ratios.  The reference keeps the first maximum in ascending
// index order (evapMaximum's strict '<', surface_3d.cpp:427-428; apex,
// surface_3d.cpp:171-190): the low word holds ~index so that ties resolve to
// the smallest index.
// Grid_3d::Table::field_o2 (tapsim/grid_3d.cpp:993-1199): least-squares fit
// of the second-order Taylor model (basis x, y, z, x^2/2, xy, xz, y^2/2, yz,
// z^2/2) over all neighbours, solved by Gaussian elimination with partial
// pivoting in FP64; E = -gradient, charge = -eps0 * Laplacian; zeros on hull
// nodes.  Returns false when the system is singular.
__device__ bool field_o2(const DevMesh& m, int i, double E[3], double* charge) {
    E[0] = E[1] = E[2] = 0.0;
    *charge = 0.0;
    if (m.flags[i] & F_HULL) return true;
    double a[81], b[9];
    for (int k = 0; k < 81; k++) a[k] = 0.0;
    for (int k = 0; k < 9; k++) b[k] = 0.0;
    const double xi = m.xyz[3 * i], yi = m.xyz[3 * i + 1], zi = m.xyz[3 * i + 2];
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) {
        const int j = m.col[q];
        const double x = (double)m.xyz[3 * j] - xi, y = (double)m.xyz[3 * j + 1] - yi, z = (double)m.xyz[3 * j + 2] - zi;
        const double f[9] = {x, y, z, 0.5 * x * x, x * y, x * z, 0.5 * y * y, y * z, 0.5 * z * z};
        const double dp = m.phi64[j] - m.phi64[i];
        for (int r = 0; r < 9; r++) {
            b[r] += dp * f[r];
            for (int c = r; c < 9; c++) a[r * 9 + c] += f[r] * f[c];
        }
    }
    for (int r = 0; r < 9; r++)
        for (int c = 0; c < r; c++) a[r * 9 + c] = a[c * 9 + r];
    for (int k = 0; k < 9; k++) {
        int p = k;
        for (int r = k + 1; r < 9; r++)
            if (fabs(a[r * 9 + k]) > fabs(a[p * 9 + k])) p = r;
        if (a[p * 9 + k] == 0.0) return false;
        if (p != k) {
            for (int c = 0; c < 9; c++) {
                const double t = a[k * 9 + c];
                a[k * 9 + c] = a[p * 9 + c];
                a[p * 9 + c] = t;
            }
            const double t = b[k];
            b[k] = b[p];
            b[p] = t;
        }
        for (int r = k + 1; r < 9; r++) {
            const double f = a[r * 9 + k] / a[k * 9 + k];
            for (int c = k; c < 9; c++) a[r * 9 + c] -= f * a[k * 9 + c];
            b[r] -= f * b[k];
        }
    }
    for (int k = 8; k >= 0; k--) {
        double acc = b[k];
        for (int c = k + 1; c < 9; c++) acc -= a[k * 9 + c] * b[c];
        b[k] = acc / a[k * 9 + k];
    }
    E[0] = -b[0];
    E[1] = -b[1];
    E[2] = -b[2];
    *charge = -(b[3] + b[6] + b[8]) * kEpsilon0;
    return b[0] == b[0] && b[1] == b[1] && b[2] == b[2];
}

// Score of a surface cell before normalisation, by probability mode
// (Surface_3d::evap_compute_probabilities, surface_3d.cpp:222-399):
// 0 |E|/E_evap; 1 Boltzmann exp(-(1 - |E|/E_evap) Q / (2 kB T)); 2 linear
// force q |E| / E_evap^2 from field_o2; 3 Voronoi flux force |F| / A / E_evap^2
// with F = sum_j -eps0 (phi_j - phi_i)^2 c_ij (1/eps_j - 1/eps_i) d_ij / |d_ij|^2
// and A = sum_j c_ij |d_ij| (1/eps_i + 1/eps_j) / 2 (the capped face areas).
__device__ double select_score(const DevMesh& m, int i, int mode, float temperature, double ratio) {
    const DType& t = m.types[m.type[i]];
    if (mode == 0) return ratio;
    if (mode == 1) return exp(-(1.0 - ratio) * (double)t.evap_energy / ((double)temperature * 8.6173431e-5) / 2.0);
    const double ef = (double)t.evap_field;
    if (mode == 2) {
        double E[3], q;
        if (!field_o2(m, i, E, &q)) atomicOr(m.status, S_SINGULAR);
        return q * sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]) / (ef * ef);
    }
    const double ei = 1.0 / (double)t.epsilon;
    const double xi = m.xyz[3 * i], yi = m.xyz[3 * i + 1], zi = m.xyz[3 * i + 2];
    double F0 = 0.0, F1 = 0.0, F2 = 0.0, area = 0.0;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) {
        const int j = m.col[q];
        const double ej = 1.0 / (double)m.types[m.type[j]].epsilon;
        const double dp = m.phi64[j] - m.phi64[i];
        const double v = -kEpsilon0 * dp * dp * m.c64[q] * (ej - ei);
        const double dx = (double)m.xyz[3 * j] - xi, dy = (double)m.xyz[3 * j + 1] - yi, dz = (double)m.xyz[3 * j + 2] - zi;
        const double d2 = dx * dx + dy * dy + dz * dz;
        area += m.c64[q] * sqrt(d2) / 2.0 * (ei + ej);
        F0 += dx / d2 * v;
        F1 += dy / d2 * v;
        F2 += dz / d2 * v;
    }
    return sqrt(F0 * F0 + F1 * F1 + F2 * F2) / area / (ef * ef);
}

__global__ void k_surface_select(DevMesh m, Surface sf, int slots, int mode, float temperature,
                                 unsigned long long* keys, double* acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long kr = 0ull, kz = 0ull, kmin = 0ull, kmax = 0ull;
    double r = 0.0, sc = 0.0;
    if (t < slots) {
        const int i = sf.list[t];
        if (i >= 0) {
            double E[3];
            if (!field_o1(m, i, E)) atomicOr(m.status, S_SINGULAR);
            const double len = sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
            const float ratio = (float)(len / (double)m.types[m.type[i]].evap_field);
            sf.ratio[t] = ratio;
            if (!(ratio == ratio)) atomicOr(m.status, S_NAN);
            r = (double)ratio;
            const float score = (float)select_score(m, i, mode, temperature, (double)ratio);
            sf.score[t] = score;
            sc = (double)score;
            const uint32_t low = ~(uint32_t)i;
            kr = ((unsigned long long)float_order_key(ratio) << 32) | low;
            kz = ((unsigned long long)float_order_key(m.xyz[3 * i + 2]) << 32) | low;
            kmin = (unsigned long long)low;   // max of ~i = smallest node
            kmax = (unsigned long long)(uint32_t)i + 1ull;
        } else {
            sf.ratio[t] = -1.0f;
            sf.score[t] = 0.0f;
        }
    }
    block_max_atomic_u64<kBlock>(kr, &keys[0]);
    block_max_atomic_u64<kBlock>(kz, &keys[1]);
    block_max_atomic_u64<kBlock>(kmin, &keys[2]);
    block_max_atomic_u64<kBlock>(kmax, &keys[3]);
    block_sum2_atomic<kBlock>(r, sc, &acc[0], &acc[1]);
}

// probability key: (p, ~node) so that the maximum is the first maximum in
// ascending node order; a NaN probability (zero or NaN sum) keys as 0, so
// the first surface cell wins, as evapMaximum keeps it (surface_3d.cpp:423-431)
__device__ __forceinline__ unsigned long long prob_key(float p, int i) {
    const uint32_t hi = (p == p) ? float_order_key(p) : 0u;
    return ((unsigned long long)hi << 32) | (~(uint32_t)i);
}

// The node of a (value, node) key: the low word holds ~node.
__device__ __forceinline__ int key_node(unsigned long long key) { return (int)(~(uint32_t)key); }

// keys[4]: the first maximum of score / sum, sum = acc[1] as float (the
// reference normalises in float); nothing on an empty surface (keys[0] == 0)
__global__ void k_surface_best(Surface sf, int slots, const double* acc, unsigned long long* keys) {
    if (keys[0] == 0ull) return;
    const float sum = (float)acc[1];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long k = 0ull;
    if (t < slots) {
        const int i = sf.list[t];
        if (i >= 0) k = prob_key(sf.score[t] / sum, i);
    }
    block_max_atomic_u64<kBlock>(k, &keys[4]);
}

// keys[5]: the runner-up probability (the candidate of keys[4] left out),
// keys[6]: the runner-up ratio (the best-ratio node of keys[0] left out)
__global__ void k_surface_second(Surface sf, int slots, const double* acc, unsigned long long* keys) {
    if (keys[0] == 0ull) return;
    const float sum = (float)acc[1];
    const int candidate = key_node(keys[4]), bestRatioNode = key_node(keys[0]);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long kp = 0ull, kr = 0ull;
    if (t < slots) {
        const int i = sf.list[t];
        if (i >= 0 && i != candidate) kp = prob_key(sf.score[t] / sum, i);
        if (i >= 0 && i != bestRatioNode) kr = ((unsigned long long)float_order_key(sf.ratio[t]) << 32) | (~(uint32_t)i);
    }
    block_max_atomic_u64<kBlock>(kp, &keys[5]);
    block_max_atomic_u64<kBlock>(kr, &keys[6]);
}

// sum of the normalised probabilities of the surface nodes <= upTo
__global__ void k_surface_prefix(Surface sf, int slots, float sum, int upTo, double* acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double p = 0.0;
    if (t < slots) {
        const int i = sf.list[t];
        if (i >= 0 && i <= upTo) p = (double)(sf.score[t] / sum);
    }
    block_sum_atomic<kBlock>(p, acc);
}

// Coupling of the pair (n1, n2) as Grid_3d::Table::computeCoupling
// (grid_3d.cpp:1392-1409) evaluates it: zero from a non-Neumann cell to a
// Neumann cell, else the harmonic mean of the permittivities times the
// capped face area over the distance (geom).
__device__ double pair_coupling(const DevMesh& m, int n1, int n2, double geom) {
    const bool neu1 = (m.flags[n1] & F_NEUMANN) != 0, neu2 = (m.flags[n2] & F_NEUMANN) != 0;
    if (!neu1 && neu2) return 0.0;
    const double e1 = m.types[m.type[n1]].epsilon, e2 = m.types[m.type[n2]].epsilon;
    return 2.0 * e1 * e2 / (e1 + e2) * geom;
}

__device__ void recompute_diag(const DevMesh& m, int i) {
    double d = 0.0;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) d += m.ceff64[q];
    m.diag64[i] = d;
    m.diag32[i] = (float)d;
}

// Flip node i to the vacuum type and resync its couplings in place
// (Grid_3d::Table::fastResync, grid_3d.cpp:555-589), executed by one warp.
__device__ void flip_and_resync(const DevMesh& m, RowLists rl, int i, int vacuumId) {
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        m.type[i] = (int8_t)vacuumId;
        const DType& vt = m.types[vacuumId];
        uint8_t f = m.flags[i] & (F_HULL | F_SURFACE | F_FREE);
        if (vt.dirichlet) f |= F_DIRICHLET;
        if (vt.neumann) f |= F_NEUMANN;
        if (!vt.dirichlet && !(f & F_FREE)) {
            const int c = m.colour[i];
            if (vt.neumann) {
                rl.rowsN[rl.segStart[c] + atomicAdd(&rl.countN[c], 1)] = i;
                rl.allN[atomicAdd(&rl.countAll[1], 1)] = i;
            } else {
                rl.rowsV[rl.segStart[c] + atomicAdd(&rl.countV[c], 1)] = i;
                rl.allV[atomicAdd(&rl.countAll[0], 1)] = i;
            }
            f |= F_FREE;
        }
        m.flags[i] = f;
        m.q64[i] = m.volume ? m.volume[i] * (double)vt.charge_density / kEpsilon0 : 0.0;
    }
    __syncwarp();
    const bool neuI = (m.flags[i] & F_NEUMANN) != 0;
    for (int q = m.row_ptr[i] + lane; q < m.row_ptr[i + 1]; q += 32) {
        const int j = m.col[q];
        const int r = m.rev[q];
        const double c = pair_coupling(m, i, j, m.geom[q]);
        const bool neuJ = (m.flags[j] & F_NEUMANN) != 0;
        m.c64[q] = c;
        m.c64[r] = c;
        const double ci = (!neuI && neuJ) ? 0.0 : c;
        const double cj = (!neuJ && neuI) ? 0.0 : c;
        m.ceff64[q] = ci;
        m.ceff32[q] = (float)ci;
        m.ceff64[r] = cj;
        m.ceff32[r] = (float)cj;
    }
    __syncwarp();
    if (lane == 0) recompute_diag(m, i);
    for (int q = m.row_ptr[i] + lane; q < m.row_ptr[i + 1]; q += 32) recompute_diag(m, m.col[q]);
    __syncwarp();
}

// Surface_3d::Table::update (surface_3d.cpp:83-119) for a removed node.
__device__ bool surface_update(const DevMesh& m, Surface sf, int i, int vacuumId) {
    const int lane = threadIdx.x & 31;
    bool ok = true;
    if (lane == 0) {
        if (!(m.flags[i] & F_SURFACE)) {
            ok = false;
        } else {
            sf.list[sf.slot[i]] = -1;
            m.flags[i] &= ~F_SURFACE;
        }
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    if (!ok) return false;
    // lanes take distinct neighbours, so no node is inserted twice
    for (int q = m.row_ptr[i] + lane; q < m.row_ptr[i + 1]; q += 32) {
        const int j = m.col[q];
        if (is_surface_candidate(m, j, vacuumId)) surface_insert(m, sf, j);
    }
    __syncwarp();
    return true;
}

// evap_takeAway (surface_3d.cpp:507-564), one warp.
__global__ void k_take_away(DevMesh m, RowLists rl, Surface sf, int node, int vacuumId, int32_t* result, int resultCap) {
    const int lane = threadIdx.x & 31;
    __shared__ int lonely[256];
    __shared__ int nLonely;
    if (lane == 0) {
        result[0] = 0;
        nLonely = 0;
    }
    __syncwarp();
    if (!(m.flags[node] & F_SURFACE)) {
        if (lane == 0) {
            atomicOr(m.status, S_NOT_SURFACE);
            result[0] = -1;
        }
        return;
    }
    flip_and_resync(m, rl, node, vacuumId);
    surface_update(m, sf, node, vacuumId);
    // detached neighbours: non-vacuum cells whose neighbours are all vacuum,
    // collected in neighbour order before any of them is removed
    const int q0 = m.row_ptr[node], q1 = m.row_ptr[node + 1];
    for (int base = q0; base < q1; base += 32) {
        const int q = base + lane;
        bool isLonely = false;
        if (q < q1) {
            const int j = m.col[q];
            if (m.type[j] != vacuumId) {
                isLonely = true;
                for (int p = m.row_ptr[j]; p < m.row_ptr[j + 1]; p++)
                    if (m.type[m.col[p]] != vacuumId) { isLonely = false; break; }
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, isLonely);
        if (isLonely) {
            const int pos = nLonely + __popc(mask & ((1u << lane) - 1u));
            if (pos < 256) lonely[pos] = m.col[q];
        }
        __syncwarp();
        if (lane == 0) nLonely += __popc(mask);
        __syncwarp();
    }
    const int nl = min(nLonely, 256);
    for (int k = 0; k < nl; k++) {
        const int j = lonely[k];
        flip_and_resync(m, rl, j, vacuumId);
        if (!surface_update(m, sf, j, vacuumId) && lane == 0) atomicOr(m.status, S_NOT_SURFACE);
        if (lane == 0 && k + 1 < resultCap) result[1 + k] = j;
    }
    if (lane == 0) result[0] = nl;
}

// update_coordination (surface_3d.cpp:568-593): every cell with id >= 10
// adds its number of id >= 10 neighbours to its id.  The id >= 10 predicate
// is read from a copy of the ids taken before the pass; the reference's
// in-order update reads the same values unless an id wraps past 127.
__global__ void k_coordination(DevMesh m, const int8_t* before) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const int id = before[i];
    if (id < 10) return;
    int cnt = 0;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++)
        if (before[m.col[q]] >= 10) cnt++;
    m.type[i] = (int8_t)(id + cnt);
}

// Surface_3d::Table::normal (surface_3d.cpp:123-169): plane fit through the
// 3-hop surface neighbourhood (smallest-eigenvalue eigenvector of the
// uncentred scatter matrix of p_node - p_k, find_best_plane,
// geometry_3d.cpp:1806-1870), oriented towards the vacuum cells of the
// neighbourhood.  One block; Jacobi eigen-iteration in FP64.
constexpr int kNHash = 4096;
__device__ void surface_normal(const DevMesh& m, int node, int vacuumId, float* out) {
    __shared__ int32_t keys[kNHash];
    __shared__ int32_t frontier[kNHash];
    __shared__ int fs, fe, tail;
    __shared__ double S[6], V[3];
    for (int k = threadIdx.x; k < kNHash; k += blockDim.x) keys[k] = -1;
    if (threadIdx.x < 6) S[threadIdx.x] = 0.0;
    if (threadIdx.x < 3) V[threadIdx.x] = 0.0;
    if (threadIdx.x == 0) {
        frontier[0] = node;
        fs = 0;
        fe = 1;
        tail = 1;
    }
    __syncthreads();
    for (int h = 0; h < 3; h++) {
        const int a = fs, b = fe;
        for (int f = a + threadIdx.x; f < b; f += blockDim.x) {
            const int u = frontier[f];
            for (int q = m.row_ptr[u]; q < m.row_ptr[u + 1]; q++) {
                const int v = m.col[q];
                uint32_t hsh = ((uint32_t)v * 2654435761u) & (kNHash - 1);
                for (int probe = 0; probe < kNHash; probe++) {
                    const int prev = atomicCAS(&keys[hsh], -1, v);
                    if (prev == -1) {
                        const int pos = atomicAdd(&tail, 1);
                        if (pos < kNHash) frontier[pos] = v;
                        break;
                    }
                    if (prev == v) break;
                    hsh = (hsh + 1) & (kNHash - 1);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            fs = b;
            fe = min(tail, kNHash);
        }
        __syncthreads();
    }
    const int members = min(tail, kNHash);
    const double px = m.xyz[3 * node], py = m.xyz[3 * node + 1], pz = m.xyz[3 * node + 2];
    for (int f = 1 + threadIdx.x; f < members; f += blockDim.x) {
        const int v = frontier[f];
        if (v == node) continue;
        const double dx = m.xyz[3 * v] - px, dy = m.xyz[3 * v + 1] - py, dz = m.xyz[3 * v + 2] - pz;
        if (m.type[v] == vacuumId) {
            atomicAdd(&V[0], dx);
            atomicAdd(&V[1], dy);
            atomicAdd(&V[2], dz);
        }
        if (m.flags[v] & F_SURFACE) {
            atomicAdd(&S[0], dx * dx);
            atomicAdd(&S[1], dx * dy);
            atomicAdd(&S[2], dx * dz);
            atomicAdd(&S[3], dy * dy);
            atomicAdd(&S[4], dy * dz);
            atomicAdd(&S[5], dz * dz);
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double a[3][3] = {{S[0], S[1], S[2]}, {S[1], S[3], S[4]}, {S[2], S[4], S[5]}};
    double ev[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 64; sweep++) {
        const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
        if (off == 0.0) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(tt * tt + 1.0), s = tt * c;
                for (int k = 0; k < 3; k++) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; k++) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    const double vkp = ev[k][p], vkq = ev[k][q];
                    ev[k][p] = c * vkp - s * vkq;
                    ev[k][q] = s * vkp + c * vkq;
                }
            }
    }
    int idx = 0;
    for (int k = 1; k < 3; k++)
        if (a[k][k] < a[idx][idx]) idx = k;
    double n0 = ev[0][idx], n1 = ev[1][idx], n2 = ev[2][idx];
    const double len = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (len > 0.0) { n0 /= len; n1 /= len; n2 /= len; }
    if (n0 * V[0] + n1 * V[1] + n2 * V[2] < 0.0) { n0 = -n0; n1 = -n1; n2 = -n2; }
    out[0] = (float)n0;
    out[1] = (float)n1;
    out[2] = (float)n2;
}

__global__ void k_surface_normal(DevMesh m, int node, int vacuumId, float* out) {
    surface_normal(m, node, vacuumId, out);
}

// The normals of cells nodes[0..count), one block each.
__global__ void k_surface_normals(DevMesh m, const int32_t* nodes, int vacuumId, float* out) {
    surface_normal(m, nodes[blockIdx.x], vacuumId, out + 3 * (size_t)blockIdx.x);
}

inline int blocks(int n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

void launch_surface_init(const DevMesh& m, Surface sf, int vacuumId, cudaStream_t s) {
    { count_launch(); k_surface_init<<<blocks(m.n), kBlock, 0, s>>>(m, sf, vacuumId); }
}
void launch_surface_select(const DevMesh& m, Surface sf, int slots, int mode, float temperature,
                           unsigned long long* keys, double* acc, cudaStream_t s) {
    if (slots > 0) {
        count_launch();
        k_surface_select<<<blocks(slots), kBlock, 0, s>>>(m, sf, slots, mode, temperature, keys, acc);
    }
}
void launch_surface_best(Surface sf, int slots, const double* acc, unsigned long long* keys, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_surface_best<<<blocks(slots), kBlock, 0, s>>>(sf, slots, acc, keys); }
}
void launch_surface_second(Surface sf, int slots, const double* acc, unsigned long long* keys, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_surface_second<<<blocks(slots), kBlock, 0, s>>>(sf, slots, acc, keys); }
}
void launch_surface_prefix(Surface sf, int slots, float sum, int upTo, double* acc, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_surface_prefix<<<blocks(slots), kBlock, 0, s>>>(sf, slots, sum, upTo, acc); }
}
void launch_field_o1(const DevMesh& m, const int32_t* nodes, int count, double* out, cudaStream_t s) {
    if (count > 0) { count_launch(); k_field_o1<<<blocks(count), kBlock, 0, s>>>(m, nodes, count, out); }
}
void launch_take_away(const DevMesh& m, RowLists rl, Surface sf, int node, int vacuumId, int32_t* result, int resultCap,
                      cudaStream_t s) {
    { count_launch(); k_take_away<<<1, 32, 0, s>>>(m, rl, sf, node, vacuumId, result, resultCap); }
}
void launch_update_coordination(const DevMesh& m, int8_t* scratchType, cudaStream_t s) {
    cudaMemcpyAsync(scratchType, m.type, (size_t)m.n, cudaMemcpyDeviceToDevice, s);
    { count_launch(); k_coordination<<<blocks(m.n), kBlock, 0, s>>>(m, scratchType); }
}
void launch_surface_normal(const DevMesh& m, Surface sf, int node, int vacuumId, float* out, cudaStream_t s) {
    (void)sf;
    { count_launch(); k_surface_normal<<<1, 256, 0, s>>>(m, node, vacuumId, out); }
}
void launch_surface_normals(const DevMesh& m, const int32_t* nodes, int count, int vacuumId, float* out,
                            cudaStream_t s) {
    if (count > 0) { count_launch(); k_surface_normals<<<count, 256, 0, s>>>(m, nodes, vacuumId, out); }
}
void launch_cell_values(const DevMesh& m, const int32_t* nodes, int count, float* phi, float* field, float* force,
                        cudaStream_t s) {
    if (count > 0) { count_launch(); k_cell_values<<<blocks(count), kBlock, 0, s>>>(m, nodes, count, phi, field, force); }
}

}  // namespace tgd

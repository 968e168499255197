/* CPU restatement of TAPSim's per-event hot path in FP64 (test oracle).
 * Test infrastructure only; see tapsim_oracle.h. */
#include "tapsim_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int is_neumann(const orc_mesh* m, int i) { return m->types[(int)m->type[i]].neumann; }
static int is_dirichlet(const orc_mesh* m, int i) { return m->types[(int)m->type[i]].dirichlet; }

/* weight of neighbour entry q in the update of row i: computePotential
 * (tapsim/grid_3d.cpp:1317-1371) skips Neumann neighbours of non-Neumann rows */
static double row_weight(const orc_mesh* m, int i, int q) {
    if (!is_neumann(m, i) && is_neumann(m, m->col[q])) return 0.0;
    return m->c[q];
}

double orc_residual(const orc_mesh* m) {
    double r2 = 0.0, b2 = 0.0;
    for (int i = 0; i < m->n; i++) {
        if (is_dirichlet(m, i)) continue;
        double s = 0.0, d = 0.0, b = 0.0;
        for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
            const double w = row_weight(m, i, q);
            const int j = m->col[q];
            s += w * m->phi[j];
            d += w;
            if (is_dirichlet(m, j)) b += w * m->phi[j];
        }
        const double r = s - d * m->phi[i] - m->q[i];
        b -= m->q[i];
        r2 += r * r;
        b2 += b * b;
    }
    return b2 > 0.0 ? sqrt(r2 / b2) : sqrt(r2);
}

static double sweep(orc_mesh* m, double omega) {
    double dev = 0.0;
    for (int i = 0; i < m->n; i++) {
        if (is_dirichlet(m, i)) continue;
        double s = 0.0, d = 0.0;
        for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
            const double w = row_weight(m, i, q);
            s += w * m->phi[m->col[q]];
            d += w;
        }
        const double v = (s - m->q[i]) / d;
        const double nv = m->phi[i] + omega * (v - m->phi[i]);
        const double dl = fabs(nv - m->phi[i]);
        if (dl > dev) dev = dl;
        m->phi[i] = nv;
    }
    return dev;
}

int64_t orc_solve(orc_mesh* m, double tol, int64_t max_sweeps, double omega, double* rel_out) {
    int64_t s = 0;
    double rel = orc_residual(m);
    while (rel > tol) {
        if (s >= max_sweeps) {
            if (rel_out) *rel_out = rel;
            return -1;
        }
        for (int k = 0; k < 10; k++) sweep(m, omega);
        s += 10;
        rel = orc_residual(m);
    }
    if (rel_out) *rel_out = rel;
    return s;
}

/* Grid_3d::Table::find_localNodes (grid_3d.cpp:1284-1315) followed by the
 * removal of Dirichlet cells that localRelax does (:707-721): the cells
 * reached from `node` in 1..shell steps through the Delaunay neighbours,
 * node itself only when a neighbour leads back to it (shell >= 2), minus
 * the Dirichlet cells; written in ascending order (a std::set<int>).
 * Returns the count (at most cap are written). */
int32_t orc_local_set(const orc_mesh* m, int32_t node, int32_t shell, int32_t* out, int32_t cap) {
    uint8_t* seen = calloc((size_t)m->n, 1);
    int32_t* front = malloc(sizeof(int32_t) * (size_t)m->n);
    int32_t* next = malloc(sizeof(int32_t) * (size_t)m->n);
    int32_t nf = 1, total = 0;
    front[0] = node;
    for (int32_t h = 0; h < shell; h++) {
        int32_t nn = 0;
        for (int32_t f = 0; f < nf; f++)
            for (int32_t q = m->row_ptr[front[f]]; q < m->row_ptr[front[f] + 1]; q++) {
                const int32_t j = m->col[q];
                if (seen[j]) continue;
                seen[j] = 1;
                next[nn++] = j;
            }
        int32_t* t = front;
        front = next;
        next = t;
        nf = nn;
    }
    for (int32_t i = 0; i < m->n; i++)
        if (seen[i] && !is_dirichlet(m, i)) {
            if (total < cap) out[total] = i;
            total++;
        }
    free(seen);
    free(front);
    free(next);
    return total;
}

/* The fixed point of localRelax (grid_3d.cpp:722-795): the potentials of
 * the listed cells that satisfy computePotential (:1317-1371) with every
 * other cell held at its value; Gauss-Seidel over the list until a sweep
 * changes no potential by more than tol.  Returns the sweeps, -1 on the cap. */
int64_t orc_local_solve(orc_mesh* m, const int32_t* cells, int32_t count, double tol, int64_t max_sweeps) {
    for (int64_t s = 1; s <= max_sweeps; s++) {
        double dev = 0.0;
        for (int32_t k = 0; k < count; k++) {
            const int32_t i = cells[k];
            double sum = 0.0, d = 0.0;
            for (int32_t q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
                const double w = row_weight(m, i, q);
                sum += w * m->phi[m->col[q]];
                d += w;
            }
            const double v = (sum - m->q[i]) / d;
            if (fabs(v - m->phi[i]) > dev) dev = fabs(v - m->phi[i]);
            m->phi[i] = v;
        }
        if (dev <= tol) return s;
    }
    return -1;
}

/* The stagnation rule of Grid_3d::Table::relax(thr, cycle, queue) and
 * localRelax (grid_3d.cpp:625-654): with a full queue of the last `queue`
 * deviations, the least-squares slope of deviation over sweep index,
 * sum (x - xm)(y - ym) / (queue (queue^2 - 1) cycle / 12); 1 when it is
 * exactly zero (RelaxationFault), else 0 (also while the queue is short). */
int32_t orc_stagnated(const double* dev, int32_t count, int32_t queue, int32_t cycle) {
    if (queue <= 0 || count < queue) return 0;
    const double* y = dev + count - queue;
    const double xMean = (queue - 1) / 2.0f;
    double yMean = 0.0;
    for (int32_t k = 0; k < queue; k++) yMean += y[k];
    yMean /= queue;
    double num = 0.0;
    for (int32_t k = 0; k < queue; k++) num += (k - xMean) * (y[k] - yMean);
    double den = queue;
    den *= queue;
    den -= 1;
    den *= queue;
    den *= cycle;
    den /= 12.0f;
    return num / den == 0.0;
}

double orc_relax_cycles(orc_mesh* m, int32_t n) {
    double dev = 0.0;
    for (int k = 0; k < n; k++) dev = sweep(m, 1.0);
    return dev;
}

/* Grid_3d::Table::force (grid_3d.cpp:1201-1236) in FP64: sum over the
 * neighbours of eps0 c_ij (phi_j - phi_i)^2 (1/eps_j - 1/eps_i) d / |d|^2,
 * d = x_j - x_i */
void orc_force(const orc_mesh* m, int32_t i, double F[3]) {
    const double eps0 = 8.85418781762e-12;
    const double ei = 1.0 / m->types[m->type[i]].epsilon;
    F[0] = F[1] = F[2] = 0.0;
    for (int32_t q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
        const int32_t j = m->col[q];
        const double dp = m->phi[j] - m->phi[i];
        const double mag = eps0 * m->c[q] * dp * dp * (1.0 / m->types[m->type[j]].epsilon - ei);
        double d[3], d2 = 0.0;
        for (int k = 0; k < 3; k++) {
            d[k] = (double)m->xyz[3 * j + k] - (double)m->xyz[3 * i + k];
            d2 += d[k] * d[k];
        }
        for (int k = 0; k < 3; k++) F[k] += d[k] * mag / d2;
    }
}

/* Grid_3d::Table::field_o1 (grid_3d.cpp:909-991) in FP64 */
int orc_field_o1(const orc_mesh* m, int32_t i, double E[3]) {
    E[0] = E[1] = E[2] = 0.0;
    if (m->hull && m->hull[i]) return 1;
    double A[3][3] = {{0}}, b[3] = {0};
    for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
        if (m->c[q] == 0.0) continue;
        const int j = m->col[q];
        double d[3];
        for (int k = 0; k < 3; k++) d[k] = (double)m->xyz[3 * j + k] - (double)m->xyz[3 * i + k];
        const double dp = m->phi[j] - m->phi[i];
        for (int r = 0; r < 3; r++) {
            for (int s = 0; s < 3; s++) A[r][s] += d[r] * d[s];
            b[r] += dp * d[r];
        }
    }
    /* Gaussian elimination with partial pivoting */
    int piv[3] = {0, 1, 2};
    for (int k = 0; k < 3; k++) {
        int p = k;
        for (int r = k + 1; r < 3; r++)
            if (fabs(A[r][k]) > fabs(A[p][k])) p = r;
        if (A[p][k] == 0.0) return 0;
        if (p != k) {
            for (int s = 0; s < 3; s++) {
                const double t = A[k][s];
                A[k][s] = A[p][s];
                A[p][s] = t;
            }
            const double t = b[k];
            b[k] = b[p];
            b[p] = t;
            const int ti = piv[k];
            piv[k] = piv[p];
            piv[p] = ti;
        }
        for (int r = k + 1; r < 3; r++) {
            const double f = A[r][k] / A[k][k];
            for (int s = k; s < 3; s++) A[r][s] -= f * A[k][s];
            b[r] -= f * b[k];
        }
    }
    double g[3];
    for (int k = 2; k >= 0; k--) {
        double s = b[k];
        for (int r = k + 1; r < 3; r++) s -= A[k][r] * g[r];
        g[k] = s / A[k][k];
    }
    for (int k = 0; k < 3; k++) E[k] = -g[k];
    return 1;
}

/* Surface_3d::Table::init / update candidate test (surface_3d.cpp:50-119) */
static int surface_candidate(const orc_mesh* m, int i, int vac) {
    const int t = m->type[i];
    if (t == vac) return 0;
    if (!m->types[t].removable) return 0;
    for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++)
        if (m->type[m->col[q]] == vac && m->area_pos[q]) return 1;
    return 0;
}

int32_t orc_surface_init(orc_mesh* m, int32_t vac) {
    int32_t cnt = 0;
    for (int i = 0; i < m->n; i++) {
        m->surface[i] = (uint8_t)surface_candidate(m, i, vac);
        cnt += m->surface[i];
    }
    return cnt;
}

/* evap_compute_specificFields + probLinear_field + evapMaximum + apex
 * (surface_3d.cpp:171-219, 267-297, 423-431): ascending node order, first
 * maximum wins */
void orc_select(const orc_mesh* m, float* ratio_out, orc_select_info* info) {
    info->candidate = -1;
    info->apex = -1;
    info->num_surface = 0;
    info->best = -1.0f;
    info->second = 0.0f;
    info->sum = 0.0;
    float zmax = 0.0f;
    for (int i = 0; i < m->n; i++) {
        if (!m->surface[i]) continue;
        double E[3];
        orc_field_o1(m, i, E);
        const float r = (float)(sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]) / m->types[(int)m->type[i]].evap_field);
        if (ratio_out) ratio_out[i] = r;
        info->sum += r;
        if (info->candidate < 0 || r > info->best) {
            if (info->candidate >= 0) info->second = info->best > info->second ? info->best : info->second;
            info->best = r;
            info->candidate = i;
        } else if (r > info->second) {
            info->second = r;
        }
        if (info->apex < 0 || m->xyz[3 * i + 2] > zmax) {
            zmax = m->xyz[3 * i + 2];
            info->apex = i;
        }
        info->num_surface++;
    }
}

/* Gaussian elimination with partial pivoting on a 9x9 system (the
 * reference uses LU with partial pivoting, utils.h:52-210); returns 0 when
 * a pivot vanishes */
static int solve9(double a[81], double b[9]) {
    for (int k = 0; k < 9; k++) {
        int p = k;
        for (int r = k + 1; r < 9; r++)
            if (fabs(a[r * 9 + k]) > fabs(a[p * 9 + k])) p = r;
        if (a[p * 9 + k] == 0.0) return 0;
        if (p != k) {
            for (int j = 0; j < 9; j++) {
                const double t = a[k * 9 + j];
                a[k * 9 + j] = a[p * 9 + j];
                a[p * 9 + j] = t;
            }
            const double t = b[k];
            b[k] = b[p];
            b[p] = t;
        }
        for (int r = k + 1; r < 9; r++) {
            const double f = a[r * 9 + k] / a[k * 9 + k];
            for (int j = k; j < 9; j++) a[r * 9 + j] -= f * a[k * 9 + j];
            b[r] -= f * b[k];
        }
    }
    for (int k = 8; k >= 0; k--) {
        double s = b[k];
        for (int j = k + 1; j < 9; j++) s -= a[k * 9 + j] * b[j];
        b[k] = s / a[k * 9 + k];
    }
    return 1;
}

/* basis of the second-order fit: x, y, z, x^2/2, xy, xz, y^2/2, yz, z^2/2 */
static void basis9(double x, double y, double z, double f[9]) {
    f[0] = x; f[1] = y; f[2] = z;
    f[3] = 0.5 * x * x; f[4] = x * y; f[5] = x * z;
    f[6] = 0.5 * y * y; f[7] = y * z; f[8] = 0.5 * z * z;
}

int orc_field_o2(const orc_mesh* m, int32_t i, double E[3], double* charge) {
    E[0] = E[1] = E[2] = 0.0;
    *charge = 0.0;
    if (m->hull[i]) return 1;
    double a[81] = {0}, b[9] = {0};
    for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
        const int j = m->col[q];
        double f[9];
        basis9((double)m->xyz[3 * j] - m->xyz[3 * i], (double)m->xyz[3 * j + 1] - m->xyz[3 * i + 1],
               (double)m->xyz[3 * j + 2] - m->xyz[3 * i + 2], f);
        const double dp = m->phi[j] - m->phi[i];
        for (int r = 0; r < 9; r++) {
            b[r] += dp * f[r];
            for (int s = 0; s < 9; s++) a[r * 9 + s] += f[r] * f[s];
        }
    }
    if (!solve9(a, b)) return 0;
    E[0] = -b[0];
    E[1] = -b[1];
    E[2] = -b[2];
    *charge = -(b[3] + b[6] + b[8]) * 8.85418781762e-12;
    return 1;
}

double orc_score(const orc_mesh* m, int32_t i, int32_t mode, double temperature) {
    const orc_type* t = &m->types[(int)m->type[i]];
    if (mode == 1 || mode == 0) {
        double E[3];
        orc_field_o1(m, i, E);
        const double ratio = sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]) / t->evap_field;
        if (mode == 0) return ratio;
        /* probBoltzmann (surface_3d.cpp:222-264) */
        return exp(-(1.0 - ratio) * t->evap_energy / (temperature * 8.6173431e-5) / 2.0);
    }
    if (mode == 2) {
        /* probLinear_force (surface_3d.cpp:299-330) */
        double E[3], q;
        orc_field_o2(m, i, E, &q);
        return q * sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]) / (t->evap_field * t->evap_field);
    }
    /* probVoronoiFluxForce (surface_3d.cpp:332-399) */
    const double eps0 = 8.85418781762e-12;
    double F[3] = {0, 0, 0}, area = 0.0;
    const double ei = 1.0 / t->epsilon;
    for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
        const int j = m->col[q];
        const double ej = 1.0 / m->types[(int)m->type[j]].epsilon;
        const double dp = m->phi[j] - m->phi[i];
        const double v = -eps0 * dp * dp * m->c[q] * (ej - ei);
        const double dx = (double)m->xyz[3 * j] - m->xyz[3 * i], dy = (double)m->xyz[3 * j + 1] - m->xyz[3 * i + 1],
                     dz = (double)m->xyz[3 * j + 2] - m->xyz[3 * i + 2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        area += m->c[q] * sqrt(d2) / 2.0 * (ei + ej);
        F[0] += dx / d2 * v;
        F[1] += dy / d2 * v;
        F[2] += dz / d2 * v;
    }
    return sqrt(F[0] * F[0] + F[1] * F[1] + F[2] * F[2]) / area / (t->evap_field * t->evap_field);
}

void orc_select_mode(const orc_mesh* m, int32_t mode, double temperature, float* score_out, orc_select_info* info) {
    info->candidate = -1;
    info->apex = -1;
    info->num_surface = 0;
    info->best = -1.0f;
    info->second = 0.0f;
    info->sum = 0.0;
    float zmax = 0.0f;
    for (int i = 0; i < m->n; i++) {
        if (!m->surface[i]) continue;
        const float s = (float)orc_score(m, i, mode, temperature);
        score_out[i] = s;
        info->sum += s;
        if (info->apex < 0 || m->xyz[3 * i + 2] > zmax) {
            zmax = m->xyz[3 * i + 2];
            info->apex = i;
        }
        info->num_surface++;
    }
    /* evapMaximum on the normalised probabilities: the first maximum (a NaN
     * probability, as from a zero sum, never replaces the first cell) */
    const float sum = (float)info->sum;
    for (int i = 0; i < m->n; i++) {
        if (!m->surface[i]) continue;
        const float p = score_out[i] / sum;
        if (info->candidate < 0) {
            info->candidate = i;
            info->best = p;
        } else if (info->best < p) {
            if (info->best > info->second) info->second = info->best;
            info->best = p;
            info->candidate = i;
        } else if (p > info->second) {
            info->second = p;
        }
    }
}

int32_t orc_pick(const orc_mesh* m, const float* score, double sum, double u) {
    const float fs = (float)sum;
    double cum = 0.0;
    int32_t last = -1;
    for (int i = 0; i < m->n; i++) {
        if (!m->surface[i]) continue;
        cum += (double)(score[i] / fs);
        last = i;
        if (!(u > cum)) return i;
    }
    return last;
}

/* computeCoupling (grid_3d.cpp:1392-1409) for the pair (n1, n2) */
static double pair_coupling(const orc_mesh* m, int n1, int n2, double geom) {
    if (!is_neumann(m, n1) && is_neumann(m, n2)) return 0.0;
    const double e1 = m->types[(int)m->type[n1]].epsilon, e2 = m->types[(int)m->type[n2]].epsilon;
    return 2.0 * e1 * e2 / (e1 + e2) * geom;
}

static int find_entry(const orc_mesh* m, int i, int j) {
    for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++)
        if (m->col[q] == j) return q;
    return -1;
}

/* setId(vacuum) + fastResync (grid_3d.cpp:555-589) */
static void flip(orc_mesh* m, int i, int vac) {
    m->type[i] = (int8_t)vac;
    for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
        const int j = m->col[q];
        const double c = pair_coupling(m, i, j, m->geom[q]);
        m->c[q] = c;
        m->c[find_entry(m, j, i)] = c;
    }
    m->q[i] = m->volume ? m->volume[i] * m->types[vac].charge_density / 8.85418781762e-12 : 0.0;
}

/* Surface_3d::Table::update (surface_3d.cpp:83-119) */
static int surface_update(orc_mesh* m, int i, int vac) {
    if (!m->surface[i]) return 0;
    m->surface[i] = 0;
    for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
        const int j = m->col[q];
        if (!m->surface[j] && surface_candidate(m, j, vac)) m->surface[j] = 1;
    }
    return 1;
}

/* evap_takeAway (surface_3d.cpp:507-564) */
int32_t orc_take_away(orc_mesh* m, int32_t node, int32_t vac, int32_t* detached, int32_t cap) {
    if (!m->surface[node]) return -1;
    flip(m, node, vac);
    surface_update(m, node, vac);
    int32_t nd = 0;
    int32_t lonely[512];
    for (int q = m->row_ptr[node]; q < m->row_ptr[node + 1]; q++) {
        const int j = m->col[q];
        if (m->type[j] == vac) continue;
        int all = 1;
        for (int p = m->row_ptr[j]; p < m->row_ptr[j + 1]; p++)
            if (m->type[m->col[p]] != vac) { all = 0; break; }
        if (all && nd < 512) lonely[nd++] = j;
    }
    for (int k = 0; k < nd; k++) {
        flip(m, lonely[k], vac);
        surface_update(m, lonely[k], vac);
        if (detached && k < cap) detached[k] = lonely[k];
    }
    return nd;
}

/* update_coordination (surface_3d.cpp:568-593), in node order as the reference */
void orc_update_coordination(orc_mesh* m) {
    for (int i = 0; i < m->n; i++) {
        if (m->type[i] < 10) continue;
        int cnt = 0;
        for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++)
            if (m->type[m->col[q]] >= 10) cnt++;
        m->type[i] = (int8_t)(m->type[i] + cnt);
    }
}

/* ---- flights -------------------------------------------------------------- */

static double orient(const double* a, const double* b, const double* c, const double* p) {
    const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const double w[3] = {p[0] - a[0], p[1] - a[1], p[2] - a[2]};
    return u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) + u[2] * (v[0] * w[1] - v[1] * w[0]);
}

static void node_xyz(const orc_mesh* m, int i, double* o) {
    o[0] = m->xyz[3 * i];
    o[1] = m->xyz[3 * i + 1];
    o[2] = m->xyz[3 * i + 2];
}

static const int kFace[4][3] = {{1, 3, 2}, {0, 2, 3}, {0, 3, 1}, {0, 1, 2}};

/* power-of-two scale to an integer grid with |coordinate| <= 2^40 */
static double snap_scale(const orc_mesh* m) {
    static const float* cached_xyz = 0;
    static int cached_n = -1;
    static double cached = 1.0;
    if (cached_xyz == m->xyz && cached_n == m->n) return cached;
    double amax = 0.0;
    for (int i = 0; i < 3 * m->n; i++)
        if (fabs((double)m->xyz[i]) > amax) amax = fabs((double)m->xyz[i]);
    cached = amax > 0.0 ? ldexp(1.0, (int)floor(log2(ldexp(1.0, 40) / amax))) : 1.0;
    cached_xyz = m->xyz;
    cached_n = m->n;
    return cached;
}

/* exact sign of orient(a,b,c,p) for the points snapped to that grid (the
 * reference walks with Shewchuk's exact orient3d) */
static int orient_exact(const double* a, const double* b, const double* c, const double* p, double s) {
    const double o = orient(a, b, c, p);
    const double lim = ldexp(1.0, 40);
    if (fabs(p[0] * s) > lim || fabs(p[1] * s) > lim || fabs(p[2] * s) > lim) return o > 0 ? 1 : (o < 0 ? -1 : 0);
    long long A[3], U[3], V[3], W[3];
    for (int k = 0; k < 3; k++) {
        A[k] = llround(a[k] * s);
        U[k] = llround(b[k] * s) - A[k];
        V[k] = llround(c[k] * s) - A[k];
        W[k] = llround(p[k] * s) - A[k];
    }
    const __int128 m0 = (__int128)V[1] * W[2] - (__int128)V[2] * W[1];
    const __int128 m1 = (__int128)V[0] * W[2] - (__int128)V[2] * W[0];
    const __int128 m2 = (__int128)V[0] * W[1] - (__int128)V[1] * W[0];
    const __int128 e = (__int128)U[0] * m0 - (__int128)U[1] * m1 + (__int128)U[2] * m2;
    return e > 0 ? 1 : (e < 0 ? -1 : 0);
}

/* findTetrahedron (geometry_3d.cpp:988-1044): visibility walk, faces tried in
 * a fixed order; -1 outside the mesh */
static int locate(const orc_mesh* m, const double* p, int t) {
    const double s = snap_scale(m);
    for (int step = 0; step < 4 * m->ntets + 16; step++) {
        if (t < 0) return -1;
        const int* v = m->tet_v + 4 * t;
        int next = -2;
        for (int k = 0; k < 4; k++) {
            double a[3], b[3], c[3];
            node_xyz(m, v[kFace[k][0]], a);
            node_xyz(m, v[kFace[k][1]], b);
            node_xyz(m, v[kFace[k][2]], c);
            if (orient_exact(a, b, c, p, s) < 0) {
                next = m->tet_n[4 * t + k];
                break;
            }
        }
        if (next == -2) return t;
        t = next;
    }
    return -1;
}

static void weights(const orc_mesh* m, int t, const double* p, double* w) {
    double P[4][3];
    for (int k = 0; k < 4; k++) node_xyz(m, m->tet_v[4 * t + k], P[k]);
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

/* FastField::compute (grid_3d.cpp:1663-1721) */
static void field_at(const orc_mesh* m, const double* p, int guess, double* E) {
    E[0] = E[1] = E[2] = 0.0;
    const int t = locate(m, p, guess);
    if (t < 0) return;
    double w[4];
    weights(m, t, p, w);
    for (int k = 0; k < 4; k++) {
        double Ek[3];
        orc_field_o1(m, m->tet_v[4 * t + k], Ek);
        for (int d = 0; d < 3; d++) E[d] += w[k] * Ek[d];
    }
}

double orc_potential_at(const orc_mesh* m, const double p[3], int32_t guess) {
    const int t = locate(m, p, guess);
    if (t < 0) return 0.0;
    double w[4];
    weights(m, t, p, w);
    double v = 0.0;
    for (int k = 0; k < 4; k++) v += w[k] * m->phi[m->tet_v[4 * t + k]];
    return v;
}

/* Trajectory_3d (trajectory_3d.cpp:130-209, 303-332, 358-425, 583-676) */
/* tetrahedron t2 shares a vertex with t1 (t1's entry in the set that
 * Geometry_3d::Table::adjacentTetrahedra, geometry_3d.cpp:1046-1096, builds
 * by a walk over face neighbours; t1 itself is excluded) */
static int shares_vertex(const orc_mesh* m, int t1, int t2) {
    if (t2 < 0 || t2 == t1) return 0;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
            if (m->tet_v[4 * t1 + a] == m->tet_v[4 * t2 + b]) return 1;
    return 0;
}

/* Geometry_3d::Table::isBoundaryTetrahedron (geometry_3d.cpp:819-828) */
static int boundary_tet(const orc_mesh* m, int t) {
    for (int a = 0; a < 4; a++)
        if (m->hull[m->tet_v[4 * t + a]]) return 1;
    return 0;
}

void orc_trace(const orc_mesh* m, const double start[3], double qm, int32_t guess, double dt0, double dt_min,
               double tol, int32_t max_steps, int32_t stepper_limit, double top_z, orc_impact* out) {
    const double v0[3] = {0.0, 0.0, 0.0};
    orc_trace_ext(m, start, v0, qm, guess, dt0, dt_min, tol, max_steps, stepper_limit, top_z, 1, 1, out);
}

/* point k of a recorded path: time, position, velocity, tetrahedron */
static void put_point(double* path, int32_t cap, int32_t k, double t, const double* x, const double* v, int tet) {
    if (!path || k >= cap) return;
    double* p = path + 8 * (size_t)k;
    p[0] = t;
    for (int d = 0; d < 3; d++) {
        p[1 + d] = x[d];
        p[4 + d] = v[d];
    }
    p[7] = tet < 0 ? -1.0 : (double)tet;
}

/* Trajectory_3d::cumulative_error (trajectory_3d.cpp:683-700) */
static void add_error(double* err, const double* ex, const double* ev) {
    if (!err) return;
    for (int d = 0; d < 3; d++) {
        err[d] = sqrt(err[d] * err[d] + ex[d] * ex[d]);
        err[3 + d] = sqrt(err[3 + d] * err[3 + d] + ev[d] * ev[d]);
    }
}

static void trace_core(const orc_mesh* m, const double start[3], const double vel[3], double qm, int32_t guess,
                       double dt0, double dt_min, double tol, int32_t max_steps, int32_t stepper_limit, double top_z,
                       int32_t integrator, int32_t stepper, orc_impact* out, int32_t cap, double* path,
                       double* err);

void orc_trace_ext(const orc_mesh* m, const double start[3], const double vel[3], double qm, int32_t guess,
                   double dt0, double dt_min, double tol, int32_t max_steps, int32_t stepper_limit, double top_z,
                   int32_t integrator, int32_t stepper, orc_impact* out) {
    trace_core(m, start, vel, qm, guess, dt0, dt_min, tol, max_steps, stepper_limit, top_z, integrator, stepper, out,
               0, NULL, NULL);
}

void orc_trace_path(const orc_mesh* m, const double start[3], const double vel[3], double qm, int32_t guess,
                    double dt0, double dt_min, double tol, int32_t max_steps, int32_t stepper_limit, double top_z,
                    int32_t integrator, int32_t stepper, orc_impact* out, int32_t cap, double* path, double* err) {
    trace_core(m, start, vel, qm, guess, dt0, dt_min, tol, max_steps, stepper_limit, top_z, integrator, stepper, out,
               cap, path, err);
}

static void trace_core(const orc_mesh* m, const double start[3], const double vel[3], double qm, int32_t guess,
                       double dt0, double dt_min, double tol, int32_t max_steps, int32_t stepper_limit, double top_z,
                       int32_t integrator, int32_t stepper, orc_impact* out, int32_t cap, double* path,
                       double* err) {
    static const double B[6][5] = {{0, 0, 0, 0, 0},
                                   {1.0 / 5.0, 0, 0, 0, 0},
                                   {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
                                   {3.0 / 10.0, -9.0 / 10.0, 6.0 / 5.0, 0, 0},
                                   {-11.0 / 54.0, 5.0 / 2.0, -70.0 / 27.0, 35.0 / 27.0, 0},
                                   {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};
    static const double C5[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};
    static const double C4[6] = {2825.0 / 27648.0, 0.0, 18575.0 / 48384.0, 13525.0 / 55296.0, 277.0 / 14336.0, 0.25};
    double x[3] = {start[0], start[1], start[2]}, v[3] = {vel[0], vel[1], vel[2]};
    double time = 0.0;
    memset(out, 0, sizeof(*out));
    if (err) memset(err, 0, 6 * sizeof(double));
    int tet = locate(m, x, guess);
    out->last_tet = tet;
    memcpy(out->last_pos, x, sizeof(x));
    if (tet >= 0) put_point(path, cap, 0, 0.0, x, v, tet); /* Trajectory_3d::init (trajectory_3d.cpp:99-123) */
    if (tet < 0) {
        out->status = -1;
        memcpy(out->stop, x, sizeof(x));
        return;
    }
    double E0[3];
    field_at(m, x, tet, E0);
    int status;
    if (E0[0] == 0.0 && E0[1] == 0.0 && E0[2] == 0.0) {
        status = 1;
    } else {
        status = 3;
        double dt = dt0;
        for (int it = 0; it < max_steps; it++) {
            double nx[3], nv[3], used = dt;
            double ex[3] = {0, 0, 0}, ev[3] = {0, 0, 0}; /* error vector of the trial step */
            int accepted = 0, nt = -1;
            for (int tries = 0; tries < stepper_limit; tries++) {
                if (dt < dt_min) dt = dt_min;
                used = dt;
                double rel = 0.0;
                if (integrator == 0) {
                    /* o1_integrator (trajectory_3d.cpp:560-581): Euler step;
                     * error = next state times dt^2 */
                    double E[3];
                    field_at(m, x, tet, E);
                    for (int d = 0; d < 3; d++) {
                        nv[d] = v[d] + dt * E[d] * qm;
                        nx[d] = x[d] + dt * v[d];
                    }
                    for (int d = 0; d < 3; d++) {
                        if (nx[d] != 0.0 && dt * dt > rel) rel = dt * dt;
                        if (nv[d] != 0.0 && dt * dt > rel) rel = dt * dt;
                        ex[d] = nx[d] * dt * dt;
                        ev[d] = nv[d] * dt * dt;
                    }
                } else {
                    double dx[6][3], dv[6][3];
                    for (int s = 0; s < 6; s++) {
                        double ps[3], vs[3];
                        for (int d = 0; d < 3; d++) {
                            ps[d] = x[d];
                            vs[d] = v[d];
                            for (int j = 0; j < s; j++) {
                                ps[d] += B[s][j] * dx[j][d];
                                vs[d] += B[s][j] * dv[j][d];
                            }
                        }
                        double E[3];
                        field_at(m, ps, tet, E);
                        for (int d = 0; d < 3; d++) {
                            dv[s][d] = E[d] * qm * dt;
                            dx[s][d] = vs[d] * dt;
                        }
                    }
                    for (int d = 0; d < 3; d++) {
                        nx[d] = x[d];
                        nv[d] = v[d];
                        ex[d] = ev[d] = 0.0;
                        for (int s = 0; s < 6; s++) {
                            nx[d] += C5[s] * dx[s][d];
                            nv[d] += C5[s] * dv[s][d];
                            ex[d] += (C5[s] - C4[s]) * dx[s][d];
                            ev[d] += (C5[s] - C4[s]) * dv[s][d];
                        }
                    }
                    for (int d = 0; d < 3; d++) {
                        if (nx[d] != 0.0 && fabs(ex[d] / nx[d]) > rel) rel = fabs(ex[d] / nx[d]);
                        if (nv[d] != 0.0 && fabs(ev[d] / nv[d]) > rel) rel = fabs(ev[d] / nv[d]);
                    }
                }
                nt = locate(m, nx, tet);
                if (stepper == 0) { /* NONE: every step is taken */
                    accepted = 1;
                    break;
                }
                if (stepper == 2) { /* geometryRestricted_stepper (trajectory_3d.cpp:427-452) */
                    if (nt < 0 && boundary_tet(m, tet)) { accepted = 1; break; }
                    if (shares_vertex(m, tet, nt)) { accepted = 1; break; }
                    if (nt == tet) {
                        dt *= 1.1;
                    } else {
                        if (dt == dt_min) { accepted = 1; break; }
                        dt *= 0.9;
                    }
                    continue;
                }
                if (stepper == 3 && nt >= 0 && nt != tet && !shares_vertex(m, tet, nt)) {
                    /* adaptive_stepper (trajectory_3d.cpp:454-532): leaving the star */
                    dt *= 0.1;
                    continue;
                }
                /* errorRestricted_stepper (trajectory_3d.cpp:358-425) */
                if (rel < tol || dt == dt_min) {
                    if (rel != 0.0) {
                        const double tmp = dt * pow(tol / rel, 0.25) * 0.9;
                        if (tmp < dt) dt *= 1.1; else dt = tmp;
                    }
                    accepted = 1;
                    break;
                }
                const double tmp = dt * pow(tol / rel, 0.25) * 0.9;
                if (tmp > dt) dt *= 0.9; else dt = tmp;
            }
            if (!accepted) {
                status = 2;
                break;
            }
            out->steps++;
            add_error(err, ex, ev);
            put_point(path, cap, out->steps, time + used, nx, nv, nt);
            if (nt < 0) {
                out->last_tet = tet;
                memcpy(out->last_pos, x, sizeof(x));
                memcpy(x, nx, sizeof(x));
                memcpy(v, nv, sizeof(v));
                time += used;
                tet = -1;
                status = 5;
                break;
            }
            memcpy(x, nx, sizeof(x));
            memcpy(v, nv, sizeof(v));
            time += used;
            tet = nt;
        }
    }
    if (tet >= 0) {
        out->last_tet = tet;
        memcpy(out->last_pos, x, sizeof(x));
    }
    out->last_phi = out->last_tet >= 0 ? orc_potential_at(m, out->last_pos, out->last_tet) : 0.0;
    const double dtz = (top_z - x[2]) / v[2];
    for (int d = 0; d < 3; d++) out->stop[d] = x[d] + dtz * v[d];
    out->stop_time = time + dtz;
    out->status = status;
    /* Trajectory_3d::extrapolate (trajectory_3d.cpp:303-332) */
    const int finite = isfinite(out->stop[0]) && isfinite(out->stop[1]) && isfinite(out->stop[2]);
    put_point(path, cap, out->steps + 1, time + dtz, out->stop, v, tet >= 0 && finite ? locate(m, out->stop, tet) : -1);
    if (err && dtz > 0.0)
        for (int d = 0; d < 3; d++) err[d] += dtz * err[3 + d];
}

#include "tipgen.h"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace tg_host {
namespace {

// Axially symmetric tip: spherical cap of radius R centred on the axis at
// z_c, tangent to a cone of half angle alpha that widens towards the base
// plane z = 0.  alpha = 0 gives a hemisphere on a cylinder of radius R.
struct Shape {
    double R, alpha, zt, zc, rt, rb, apex, tana;
    Shape(const TipParams& p) {
        R = p.cap_radius;
        alpha = p.half_angle_deg * M_PI / 180.0;
        tana = std::tan(alpha);
        zt = p.shank_length;
        zc = zt - R * std::sin(alpha);
        rt = R * std::cos(alpha);
        rb = rt + zt * tana;
        apex = zc + R;
    }
    double radius_at(double z) const { return rt + (zt - z) * tana; }
    bool inside(double x, double y, double z) const {
        if (z < 0.0) return false;
        const double rho2 = x * x + y * y;
        if (z <= zt) {
            const double r = radius_at(z);
            return rho2 <= r * r;
        }
        const double dz = z - zc;
        return rho2 + dz * dz <= R * R;
    }
    // Euclidean distance from an outside point to the tip body (0 inside).
    double dist(double x, double y, double z) const {
        if (inside(x, y, z)) return 0.0;
        const double rho = std::sqrt(x * x + y * y);
        double best = 1e300;
        // cap arc: nearest sphere point lies on the arc above the tangent line
        {
            const double dz = z - zc;
            const double len = std::sqrt(rho * rho + dz * dz);
            if (len > 0.0 && dz / len >= std::sin(alpha)) best = std::min(best, len - R);
        }
        // shank generator segment from (rt, zt) to (rb, 0)
        {
            const double ax = rt, az = zt, bx = rb, bz = 0.0;
            const double ux = bx - ax, uz = bz - az;
            double t = ((rho - ax) * ux + (z - az) * uz) / (ux * ux + uz * uz);
            t = std::min(1.0, std::max(0.0, t));
            const double px = ax + t * ux, pz = az + t * uz;
            best = std::min(best, std::hypot(rho - px, z - pz));
        }
        // base disc edge region (points below the tip base plane are not generated)
        // and the tangent point itself are covered by the two cases above.
        return std::max(0.0, best);
    }
};

struct Builder {
    const TipParams& p;
    Shape shape;
    TipMesh mesh;
    double W, H;
    std::vector<double> levelSpacing, levelOuter;  // spacing h_k and outer distance D_k

    Builder(const TipParams& params) : p(params), shape(params) {
        W = p.box_half_width;
        H = p.box_height;
        if (shape.rb + p.fine_shell >= W || shape.apex + p.fine_shell >= H)
            throw std::runtime_error("generate_tip: specimen does not fit into the vacuum box");
        // level 0 is the lattice continuation; its nominal spacing is the mean
        // bcc point spacing (2 points per a^3)
        const double h0 = p.lattice_a / std::cbrt(2.0);
        levelSpacing.push_back(h0);
        levelOuter.push_back(p.fine_shell);
        // farthest box point from the tip bounds the number of levels
        const double far = std::sqrt(2.0 * W * W + H * H);
        double h = h0, D = p.fine_shell;
        while (D < far) {
            h *= p.coarsen;
            if (p.max_spacing > 0.0) h = std::min(h, p.max_spacing);
            D += p.layers_per_level * h;
            levelSpacing.push_back(h);
            levelOuter.push_back(D);
        }
        levelOuter.back() = 1e300;
    }

    int level_of(double d) const {
        for (size_t k = 0; k < levelOuter.size(); k++)
            if (d <= levelOuter[k]) return (int)k;
        return (int)levelOuter.size() - 1;
    }

    void push(double x, double y, double z, int id) {
        mesh.xyz.push_back((float)x);
        mesh.xyz.push_back((float)y);
        mesh.xyz.push_back((float)z);
        mesh.id.push_back((short)id);
    }

    // Points on one face of the box.  (u,v) span the face, the fixed
    // coordinate is `fixedVal` on axis `axis`.  Points are jittered in the
    // face and kept at least 0.2 h away from the face edges.
    void boundary_face(int axis, double fixedVal, double u0, double u1, double v0, double v1, int id, int faceTag) {
        for (size_t k = 0; k < levelSpacing.size(); k++) {
            const double h = levelSpacing[k];
            const double dIn = k == 0 ? -1.0 : levelOuter[k - 1];
            const double dOut = levelOuter[k];
            // restrict enumeration to where this level can occur
            double lu0 = u0, lu1 = u1, lv0 = v0, lv1 = v1;
            if (dOut < 1e299) {
                const double reach = std::max(shape.rb, shape.R) + dOut;
                if (axis == 2) {
                    lu0 = std::max(u0, -reach); lu1 = std::min(u1, reach);
                    lv0 = std::max(v0, -reach); lv1 = std::min(v1, reach);
                } else {
                    lu0 = std::max(u0, -reach); lu1 = std::min(u1, reach);
                    lv0 = std::max(v0, 0.0); lv1 = std::min(v1, shape.apex + dOut);
                }
                if (lu0 >= lu1 || lv0 >= lv1) continue;
            }
            const int64_t i0 = (int64_t)std::floor(lu0 / h) - 1, i1 = (int64_t)std::ceil(lu1 / h) + 1;
            const int64_t j0 = (int64_t)std::floor(lv0 / h) - 1, j1 = (int64_t)std::ceil(lv1 / h) + 1;
            for (int64_t i = i0; i <= i1; i++)
                for (int64_t j = j0; j <= j1; j++) {
                    double u = (i + 0.5 + 0.6 * (hash_unit(p.seed, 1000 + faceTag, (int64_t)k, i, j, 0) - 0.5)) * h;
                    double v = (j + 0.5 + 0.6 * (hash_unit(p.seed, 1000 + faceTag, (int64_t)k, i, j, 1) - 0.5)) * h;
                    if (u <= u0 + 0.2 * h || u >= u1 - 0.2 * h || v <= v0 + 0.2 * h || v >= v1 - 0.2 * h) continue;
                    double x, y, z;
                    if (axis == 0) { x = fixedVal; y = u; z = v; }
                    else if (axis == 1) { x = u; y = fixedVal; z = v; }
                    else { x = u; y = v; z = fixedVal; }
                    const double d = shape.dist(x, y, z);
                    if (d <= dIn || d > dOut) continue;
                    push(x, y, z, id);
                    mesh.num_boundary++;
                }
        }
    }

    // Interior points of one box edge from (x0,y0,z0) to (x1,y1,z1), sampled
    // with the spacing of the level the edge midpoint falls into.
    void boundary_edge(double x0, double y0, double z0, double x1, double y1, double z1, int tag) {
        const double mx = 0.5 * (x0 + x1), my = 0.5 * (y0 + y1), mz = 0.5 * (z0 + z1);
        const double h = levelSpacing[level_of(shape.dist(mx, my, mz))];
        const double len = std::sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0) + (z1 - z0) * (z1 - z0));
        const int64_t n = std::max<int64_t>(1, (int64_t)std::floor(len / h));
        for (int64_t i = 1; i <= n; i++) {
            const double t = (i + 0.4 * (hash_unit(p.seed, 2000 + tag, i, 0, 0, 0) - 0.5)) / (n + 1);
            push(x0 + t * (x1 - x0), y0 + t * (y1 - y0), z0 + t * (z1 - z0), p.sides_id);
            mesh.num_boundary++;
        }
    }

    void boundaries() {
        // top (counter electrode) and bottom planes
        boundary_face(2, H, -W, W, -W, W, p.top_id, 0);
        boundary_face(2, 0.0, -W, W, -W, W, p.bottom_id, 1);
        // sides
        boundary_face(0, -W, -W, W, 0.0, H, p.sides_id, 2);
        boundary_face(0, W, -W, W, 0.0, H, p.sides_id, 3);
        boundary_face(1, -W, -W, W, 0.0, H, p.sides_id, 4);
        boundary_face(1, W, -W, W, 0.0, H, p.sides_id, 5);
        // box edges
        int tag = 0;
        for (int sx = 0; sx < 2; sx++)
            for (int sy = 0; sy < 2; sy++)
                boundary_edge(sx ? W : -W, sy ? W : -W, 0.0, sx ? W : -W, sy ? W : -W, H, tag++);
        for (int sz = 0; sz < 2; sz++)
            for (int s = 0; s < 2; s++) {
                const double z = sz ? H : 0.0, c = s ? W : -W;
                boundary_edge(-W, c, z, W, c, z, tag++);
                boundary_edge(c, -W, z, c, W, z, tag++);
            }
        // corners
        for (int sx = 0; sx < 2; sx++)
            for (int sy = 0; sy < 2; sy++)
                for (int sz = 0; sz < 2; sz++) {
                    push(sx ? W : -W, sy ? W : -W, sz ? H : 0.0, p.sides_id);
                    mesh.num_boundary++;
                }
    }

    // Jittered cubic-grid vacuum points for the coarse levels (k >= 1).
    void coarse_vacuum() {
        for (size_t k = 1; k < levelSpacing.size(); k++) {
            const double h = levelSpacing[k];
            const double dIn = levelOuter[k - 1], dOut = levelOuter[k];
            const double reach = (dOut < 1e299) ? std::max(shape.rb, shape.R) + dOut : 1e300;
            const double x0 = std::max(-W, -reach), x1 = std::min(W, reach);
            const double z1 = (dOut < 1e299) ? std::min(H, shape.apex + dOut) : H;
            const int64_t i0 = (int64_t)std::floor(x0 / h) - 1, i1 = (int64_t)std::ceil(x1 / h) + 1;
            const int64_t k1 = (int64_t)std::ceil(z1 / h) + 1;
            for (int64_t i = i0; i <= i1; i++)
                for (int64_t j = i0; j <= i1; j++)
                    for (int64_t l = 0; l <= k1; l++) {
                        const double x = (i + 0.5 + 0.6 * (hash_unit(p.seed, 3000, (int64_t)k, i, j, l * 4 + 0) - 0.5)) * h;
                        const double y = (j + 0.5 + 0.6 * (hash_unit(p.seed, 3000, (int64_t)k, i, j, l * 4 + 1) - 0.5)) * h;
                        const double z = (l + 0.5 + 0.6 * (hash_unit(p.seed, 3000, (int64_t)k, i, j, l * 4 + 2) - 0.5)) * h;
                        const double m = 0.2 * h;
                        if (x <= -W + m || x >= W - m || y <= -W + m || y >= W - m || z <= m || z >= H - m) continue;
                        const double d = shape.dist(x, y, z);
                        if (d <= dIn || d > dOut) continue;
                        push(x, y, z, p.vacuum_id);
                        mesh.num_vacuum++;
                    }
        }
    }

    // bcc lattice with [110] along z: cubic coordinates (x,y,z) map to
    // x' = (x - y)/sqrt2, y' = z, z' = (x + y)/sqrt2, shifted up by half a
    // (110) interplanar spacing so that no lattice plane lies in z = 0.
    void lattice(std::vector<double>& atoms, std::vector<double>& shellVac) {
        const double a = p.lattice_a;
        const double s2 = std::sqrt(2.0);
        const double shift = a / (2.0 * s2);
        const double P = shape.rb + p.fine_shell + a;
        const double Zm = shape.apex + p.fine_shell + a;
        const double xmin = -P / s2, xmax = (P + Zm) / s2;
        const int64_t i0 = (int64_t)std::floor(xmin / a) - 1, i1 = (int64_t)std::ceil(xmax / a) + 1;
        const int64_t k0 = (int64_t)std::floor(-P / a) - 1, k1 = (int64_t)std::ceil(P / a) + 1;
        for (int64_t i = i0; i <= i1; i++)
            for (int64_t j = i0; j <= i1; j++)
                for (int64_t k = k0; k <= k1; k++)
                    for (int b = 0; b < 2; b++) {
                        const double cx = (i + 0.5 * b) * a, cy = (j + 0.5 * b) * a, cz = (k + 0.5 * b) * a;
                        const double x = (cx - cy) / s2;
                        const double y = cz;
                        const double z = (cx + cy) / s2 + shift;
                        if (z <= 0.0 || z >= Zm) continue;
                        if (std::fabs(x) > P || std::fabs(y) > P) continue;
                        if (shape.inside(x, y, z)) {
                            atoms.push_back(x); atoms.push_back(y); atoms.push_back(z);
                        } else if (shape.dist(x, y, z) <= p.fine_shell) {
                            // vacuum sites continue the lattice but are jittered by
                            // up to 2% of a: a truncated lattice has co-spherical
                            // point sets at its outer edge, and the jitter makes
                            // the Delaunay mesh unique there
                            const double jx = 0.04 * a * (hash_unit(p.seed, 5000, i, j, k, 3 * b + 0) - 0.5);
                            const double jy = 0.04 * a * (hash_unit(p.seed, 5000, i, j, k, 3 * b + 1) - 0.5);
                            const double jz = 0.04 * a * (hash_unit(p.seed, 5000, i, j, k, 3 * b + 2) - 0.5);
                            shellVac.push_back(x + jx); shellVac.push_back(y + jy); shellVac.push_back(z + jz);
                        }
                    }
    }

    void alloy(const std::vector<double>& atoms, std::vector<char>& solute) {
        const size_t n = atoms.size() / 3;
        solute.assign(n, 0);
        if (p.solute_fraction <= 0.0) return;
        // precipitate volume estimate from the atom count (bcc: 2 atoms per a^3)
        const double volume = n * p.lattice_a * p.lattice_a * p.lattice_a / 2.0;
        const int64_t nPrecip = (int64_t)std::llround(p.precip_density * volume);
        std::vector<double> centres;  // x y z r
        uint64_t ctr = 0;
        while ((int64_t)centres.size() / 4 < nPrecip && ctr < (uint64_t)nPrecip * 1000 + 1000) {
            const size_t pick = (size_t)(hash_unit(p.seed, 4000, (int64_t)ctr, 0, 0, 0) * n);
            ctr++;
            const double u1 = std::max(1e-12, hash_unit(p.seed, 4001, (int64_t)ctr, 0, 0, 0));
            const double u2 = hash_unit(p.seed, 4002, (int64_t)ctr, 0, 0, 0);
            const double g = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
            double r = 1e-9 * std::exp(p.precip_mu + p.precip_sigma * g);
            r = std::min(p.precip_rmax, std::max(p.precip_rmin, r));
            centres.push_back(atoms[3 * pick]);
            centres.push_back(atoms[3 * pick + 1]);
            centres.push_back(atoms[3 * pick + 2]);
            centres.push_back(r);
        }
        int64_t count = 0;
        for (size_t i = 0; i < n; i++) {
            for (size_t c = 0; c < centres.size(); c += 4) {
                const double dx = atoms[3 * i] - centres[c], dy = atoms[3 * i + 1] - centres[c + 1], dz = atoms[3 * i + 2] - centres[c + 2];
                if (dx * dx + dy * dy + dz * dz <= centres[c + 3] * centres[c + 3]) { solute[i] = 1; count++; break; }
            }
        }
        // the remainder of the solute goes to random matrix sites
        const int64_t target = (int64_t)std::llround(p.solute_fraction * n);
        const int64_t matrixLeft = (int64_t)n - count;
        if (target > count && matrixLeft > 0) {
            const double q = (double)(target - count) / (double)matrixLeft;
            for (size_t i = 0; i < n; i++)
                if (!solute[i] && hash_unit(p.seed, 4100, (int64_t)i, 0, 0, 0) < q) solute[i] = 1;
        }
    }

    TipMesh run() {
        std::vector<double> atoms, shellVac;
        lattice(atoms, shellVac);
        std::vector<char> solute;
        alloy(atoms, solute);
        boundaries();
        for (size_t i = 0; i < shellVac.size(); i += 3) {
            push(shellVac[i], shellVac[i + 1], shellVac[i + 2], p.vacuum_id);
            mesh.num_vacuum++;
        }
        coarse_vacuum();
        for (size_t i = 0; i < atoms.size() / 3; i++) {
            push(atoms[3 * i], atoms[3 * i + 1], atoms[3 * i + 2], solute[i] ? p.solute_id : p.matrix_id);
            mesh.num_atoms++;
            mesh.num_solute += solute[i];
        }
        mesh.apex_z = shape.apex;
        return mesh;
    }
};

}  // namespace

TipMesh generate_tip(const TipParams& params) {
    Builder b(params);
    return b.run();
}

}  // namespace tg_host

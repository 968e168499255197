#include "samplegen.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <thread>
#include <unordered_map>

#include "tipgen.h"  // hash_unit

namespace tg_host {
namespace {

// Balanced k-d tree in implicit layout: the median of the index range
// [lo, hi) sits at mid = (lo + hi) / 2 with its split axis, and the two
// halves [lo, mid) and [mid + 1, hi) hold the points below and above it.
class KdTree {
  public:
    explicit KdTree(const std::vector<float>& xyz) {
        const int n = (int)(xyz.size() / 3);
        std::vector<int> idx(n);
        std::iota(idx.begin(), idx.end(), 0);
        axis_.assign(n, 0);
        build(xyz, idx, 0, n);
        p_.resize(3 * (size_t)n);
        for (int k = 0; k < n; k++)
            for (int a = 0; a < 3; a++) p_[3 * (size_t)k + a] = xyz[3 * (size_t)idx[k] + a];
        index_.swap(idx);
        for (int a = 0; a < 3; a++) {
            lo_[a] = 1e300;
            hi_[a] = -1e300;
        }
        for (int k = 0; k < n; k++)
            for (int a = 0; a < 3; a++) {
                lo_[a] = std::min(lo_[a], p_[3 * (size_t)k + a]);
                hi_[a] = std::max(hi_[a], p_[3 * (size_t)k + a]);
            }
    }
    // the original indices of the points within sqrt(r2) of q, ascending
    void within(const double q[3], double r2, std::vector<int>& out) const {
        out.clear();
        collect(0, size(), q, r2, out);
        std::sort(out.begin(), out.end());
    }
    // the original index of tree position k
    int index(int k) const { return index_[k]; }
    int size() const { return (int)(p_.size() / 3); }
    // squared distance from q to the nearest point other than tree position `skip`
    double nearest2(const double q[3], int skip = -1) const {
        double best = 1e300;
        if (size() > 0) query(0, size(), q, skip, best, lo_, hi_);
        return best;
    }
    const double* point(int k) const { return &p_[3 * (size_t)k]; }

  private:
    std::vector<double> p_;
    std::vector<int8_t> axis_;
    std::vector<int> index_;
    double lo_[3], hi_[3];  // the points' bounding box

    void collect(int lo, int hi, const double q[3], double r2, std::vector<int>& out) const {
        while (hi > lo) {
            const int mid = lo + (hi - lo) / 2;
            const double* p = point(mid);
            const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
            if (dx * dx + dy * dy + dz * dz <= r2) out.push_back(index_[mid]);
            if (hi - lo == 1) return;
            const int a = axis_[mid];
            const double diff = q[a] - p[a];
            if (diff <= 0.0 || diff * diff <= r2) collect(lo, mid, q, r2, out);
            if (diff < 0.0 && diff * diff > r2) return;
            lo = mid + 1;
        }
    }

    void build(const std::vector<float>& xyz, std::vector<int>& idx, int lo, int hi) {
        while (hi - lo > 1) {
            float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
            for (int k = lo; k < hi; k++)
                for (int a = 0; a < 3; a++) {
                    const float v = xyz[3 * (size_t)idx[k] + a];
                    mn[a] = std::min(mn[a], v);
                    mx[a] = std::max(mx[a], v);
                }
            int a = 0;
            for (int b = 1; b < 3; b++)
                if (mx[b] - mn[b] > mx[a] - mn[a]) a = b;
            const int mid = lo + (hi - lo) / 2;
            std::nth_element(idx.begin() + lo, idx.begin() + mid, idx.begin() + hi, [&](int u, int v) {
                const float fu = xyz[3 * (size_t)u + a], fv = xyz[3 * (size_t)v + a];
                return fu < fv || (fu == fv && u < v);
            });
            axis_[mid] = (int8_t)a;
            build(xyz, idx, lo, mid);
            lo = mid + 1;
        }
    }

    // Nearest-point search over tree positions [lo, hi), whose points lie in
    // the box [blo, bhi].  A subtree is skipped when its box lies at least
    // the best distance so far from q: a point r inside has |q_a - r_a| >=
    // the box's gap on every axis, in floating point too, so its squared
    // distance is no smaller and the result is the exact minimum.  Far from
    // the points (the coarse vacuum levels) the box test prunes what the
    // split planes alone cannot.
    void query(int lo, int hi, const double q[3], int skip, double& best, const double blo[3],
               const double bhi[3]) const {
        if (hi <= lo) return;
        double box = 0.0;
        for (int a = 0; a < 3; a++) {
            const double e = q[a] < blo[a] ? blo[a] - q[a] : (q[a] > bhi[a] ? q[a] - bhi[a] : 0.0);
            box += e * e;
        }
        if (box >= best) return;
        const int mid = lo + (hi - lo) / 2;
        const double* p = point(mid);
        if (mid != skip) {
            const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
            best = std::min(best, dx * dx + dy * dy + dz * dz);
        }
        if (hi - lo == 1) return;
        const int a = axis_[mid];
        // the children: [lo, mid) below the split value, [mid+1, hi) above
        double lhi[3] = {bhi[0], bhi[1], bhi[2]}, rlo[3] = {blo[0], blo[1], blo[2]};
        lhi[a] = p[a];
        rlo[a] = p[a];
        const double diff = q[a] - p[a];
        // the side that holds q first, the other only if the split plane is
        // nearer than the best point so far
        if (diff < 0.0) {
            query(lo, mid, q, skip, best, blo, lhi);
            if (diff * diff < best) query(mid + 1, hi, q, skip, best, rlo, bhi);
        } else {
            query(mid + 1, hi, q, skip, best, rlo, bhi);
            if (diff * diff < best) query(lo, mid, q, skip, best, blo, lhi);
        }
    }
};

// body(slab) for slab = 0 .. count-1 on `threads` host threads; the first
// exception of any worker is rethrown here after every thread has joined.
template <class F>
void for_slabs(int threads, int64_t count, F body) {
    std::atomic<int64_t> next(0);
    std::exception_ptr err;
    std::mutex mu;
    auto work = [&] {
        try {
            for (int64_t s; (s = next.fetch_add(1)) < count;) body(s);
        } catch (...) {
            std::lock_guard<std::mutex> g(mu);
            if (!err) err = std::current_exception();
            next.store(count);
        }
    };
    std::vector<std::thread> pool;
    try {
        for (int t = 1; t < threads; t++) pool.emplace_back(work);
    } catch (...) {
        next.store(count);
        for (auto& t : pool) t.join();
        throw;
    }
    work();
    for (auto& t : pool) t.join();
    if (err) std::rethrow_exception(err);
}

struct Builder {
    const SampleParams& p;
    const KdTree& tree;
    const std::vector<float>& atoms;
    int threads;
    // level-0 vacuum sites continuing the sample's lattice (3 per site) and
    // a hash grid over them with cells of h0
    std::vector<double> sites;
    std::unordered_map<uint64_t, std::vector<int>> siteCells;
    double W, H, h0;
    double bmin[3], bmax[3];  // the sample's bounding box
    std::vector<double> levelSpacing, levelOuter;
    // atoms per cell of a grid with cells of fine_shell over the bounding
    // box (one cell of margin): a point whose 27 cells hold no atom lies
    // farther than the fine shell from the sample
    std::vector<uint8_t> occ;
    int64_t occN[3] = {0, 0, 0};
    SampleMesh mesh;

    Builder(const SampleParams& params, const KdTree& t, int nThreads, const std::vector<float>& xyz)
        : p(params), tree(t), atoms(xyz), threads(std::max(1, nThreads)) {
        W = p.box_half_width;
        H = p.box_height;
        for (int a = 0; a < 3; a++) {
            bmin[a] = 1e300;
            bmax[a] = -1e300;
        }
        for (size_t k = 0; k < xyz.size(); k += 3)
            for (int a = 0; a < 3; a++) {
                bmin[a] = std::min(bmin[a], (double)xyz[k + a]);
                bmax[a] = std::max(bmax[a], (double)xyz[k + a]);
            }
        if (bmin[2] <= 0.0) throw std::runtime_error("generate_sample_mesh: the sample must lie above the bottom plane z = 0");
        const double S = p.fine_shell;
        if (bmin[0] - S <= -W || bmax[0] + S >= W || bmin[1] - S <= -W || bmax[1] + S >= W || bmax[2] + S >= H)
            throw std::runtime_error("generate_sample_mesh: the sample and its fine shell do not fit into the vacuum box");
        h0 = spacing();
        if (!(h0 > 0.0)) throw std::runtime_error("generate_sample_mesh: the sample has coincident points only");
        if (S < 2.0 * h0) throw std::runtime_error("generate_sample_mesh: fine_shell must be at least two point spacings");
        levelSpacing.push_back(h0);
        levelOuter.push_back(S);
        const double far = std::sqrt(2.0 * W * W + H * H);
        double h = h0, D = S;
        while (D < far) {
            h *= p.coarsen;
            if (p.max_spacing > 0.0) h = std::min(h, p.max_spacing);
            D += p.layers_per_level * h;
            levelSpacing.push_back(h);
            levelOuter.push_back(D);
        }
        levelOuter.back() = 1e300;
        mesh.spacing = h0;
        for (int a = 0; a < 3; a++) occN[a] = (int64_t)std::ceil((bmax[a] - bmin[a]) / S) + 3;
        occ.assign((size_t)(occN[0] * occN[1] * occN[2]), 0);
        for (size_t k = 0; k < xyz.size(); k += 3) {
            int64_t c[3];
            for (int a = 0; a < 3; a++) c[a] = occ_cell(xyz[k + a], a);
            occ[(size_t)((c[0] * occN[1] + c[1]) * occN[2] + c[2])] = 1;
        }
    }

    int64_t occ_cell(double v, int a) const { return (int64_t)std::floor((v - (bmin[a] - p.fine_shell)) / p.fine_shell); }
    // false when no atom lies within fine_shell of q (its 27 cells are empty)
    bool atom_in_reach(double x, double y, double z) const {
        const double q[3] = {x, y, z};
        int64_t c[3];
        for (int a = 0; a < 3; a++) c[a] = occ_cell(q[a], a);
        for (int64_t i = c[0] - 1; i <= c[0] + 1; i++)
            for (int64_t j = c[1] - 1; j <= c[1] + 1; j++)
                for (int64_t k = c[2] - 1; k <= c[2] + 1; k++) {
                    if (i < 0 || j < 0 || k < 0 || i >= occN[0] || j >= occN[1] || k >= occN[2]) continue;
                    if (occ[(size_t)((i * occN[1] + j) * occN[2] + k)]) return true;
                }
        return false;
    }

    // median nearest-neighbour distance over up to 4096 evenly spaced atoms
    double spacing() const {
        const int n = tree.size();
        const int m = std::min(n, 4096);
        std::vector<double> d(m);
        for (int k = 0; k < m; k++) {
            const int pos = (int)((int64_t)k * n / m);
            const double* q = tree.point(pos);
            const double qq[3] = {q[0], q[1], q[2]};
            d[k] = std::sqrt(tree.nearest2(qq, pos));
        }
        std::vector<double> pos;
        for (double v : d)
            if (v > 0.0 && v < 1e299) pos.push_back(v);
        if (pos.empty()) return 0.0;
        std::nth_element(pos.begin(), pos.begin() + pos.size() / 2, pos.end());
        return pos[pos.size() / 2];
    }

    // lower bound of the distance from (x, y, z) to the sample: the distance
    // to its bounding box
    double box_distance(double x, double y, double z) const {
        const double q[3] = {x, y, z};
        double s = 0.0;
        for (int a = 0; a < 3; a++) {
            const double e = std::max({bmin[a] - q[a], 0.0, q[a] - bmax[a]});
            s += e * e;
        }
        return std::sqrt(s);
    }

    double distance(double x, double y, double z) const {
        const double q[3] = {x, y, z};
        return std::sqrt(tree.nearest2(q));
    }

    int64_t cell(double v) const { return (int64_t)std::floor(v / h0); }
    static uint64_t cell_key(int64_t i, int64_t j, int64_t k) {
        return ((uint64_t)(i & 0x1FFFFF) << 42) | ((uint64_t)(j & 0x1FFFFF) << 21) | (uint64_t)(k & 0x1FFFFF);
    }
    // The cells, of the 3 x 3 x 3 around q's, that can hold a point within r
    // of q: on each axis those that [q - r, q + r] reaches (widened by a
    // hair for rounding).  Any such point lies in them, so a scan of them
    // finds what a scan of all 27 does.
    void cell_range(const double q[3], double r, int64_t lo[3], int64_t hi[3]) const {
        const double m = 1e-9 * h0;
        for (int a = 0; a < 3; a++) {
            const int64_t c = cell(q[a]);
            lo[a] = std::max(c - 1, (int64_t)std::floor((q[a] - r - m) / h0));
            hi[a] = std::min(c + 1, (int64_t)std::floor((q[a] + r + m) / h0));
        }
    }
    // a lattice site within r (<= h0) of q
    bool site_near(const double q[3], double r) const {
        int64_t lo[3], hi[3];
        cell_range(q, r, lo, hi);
        for (int64_t i = lo[0]; i <= hi[0]; i++)
            for (int64_t j = lo[1]; j <= hi[1]; j++)
                for (int64_t k = lo[2]; k <= hi[2]; k++) {
                    auto it = siteCells.find(cell_key(i, j, k));
                    if (it == siteCells.end()) continue;
                    for (int s : it->second) {
                        const double dx = q[0] - sites[3 * (size_t)s], dy = q[1] - sites[3 * (size_t)s + 1],
                                     dz = q[2] - sites[3 * (size_t)s + 2];
                        if (dx * dx + dy * dy + dz * dz < r * r) return true;
                    }
                }
        return false;
    }
    // the lattice sites within r of q in the 3 x 3 x 3 cells around q's (all
    // of them for r <= h0), ascending
    void sites_within(const double q[3], double r, std::vector<int>& out) const {
        out.clear();
        int64_t lo[3], hi[3];
        cell_range(q, r, lo, hi);
        for (int64_t i = lo[0]; i <= hi[0]; i++)
            for (int64_t j = lo[1]; j <= hi[1]; j++)
                for (int64_t k = lo[2]; k <= hi[2]; k++) {
                    auto it = siteCells.find(cell_key(i, j, k));
                    if (it == siteCells.end()) continue;
                    for (int s : it->second) {
                        const double dx = q[0] - sites[3 * (size_t)s], dy = q[1] - sites[3 * (size_t)s + 1],
                                     dz = q[2] - sites[3 * (size_t)s + 2];
                        if (dx * dx + dy * dy + dz * dz <= r * r) out.push_back(s);
                    }
                }
        std::sort(out.begin(), out.end());
    }

    // Level 0 continues the sample's lattice.  For a point A of a
    // centrosymmetric lattice and a nearest neighbour B of it (within 1.2
    // h0), A + (A - B) is a lattice point too; one with no atom and no site
    // within 0.5 h0, at least `exclusion` h0 and at most fine_shell from the
    // nearest atom, inside the box, becomes a vacuum site.  The first
    // generation reflects through the atoms with fewer neighbours than most
    // (the surface), each later one through the sites found last, until a
    // generation finds none.  Candidates are tested against the atoms in
    // parallel and against the sites in order, so that the sites do not
    // depend on the thread count.
    void lattice_shell() {
        const int n = (int)(atoms.size() / 3);
        const double rN = 1.2 * h0, excl = p.exclusion * h0, S = p.fine_shell, m = 0.2 * h0;
        std::vector<int> coord(n);
        const int64_t chunk = 4096;
        for_slabs(threads, (n + chunk - 1) / chunk, [&](int64_t c) {
            std::vector<int> nb;
            for (int64_t k = c * chunk; k < std::min<int64_t>(n, (c + 1) * chunk); k++) {
                const double q[3] = {atoms[3 * k], atoms[3 * k + 1], atoms[3 * k + 2]};
                tree.within(q, rN * rN, nb);
                coord[k] = (int)nb.size() - 1;
            }
        });
        std::vector<int> hist(64, 0);
        for (int c : coord) hist[std::min(63, std::max(0, c))]++;
        const int full = (int)(std::max_element(hist.begin(), hist.end()) - hist.begin());
        // frontier: points to reflect through (positions)
        std::vector<double> frontier;
        for (int k = 0; k < n; k++)
            if (coord[k] < full)
                for (int a = 0; a < 3; a++) frontier.push_back(atoms[3 * (size_t)k + a]);
        while (!frontier.empty()) {
            const int64_t nf = (int64_t)(frontier.size() / 3);
            std::vector<std::vector<double>> found((size_t)((nf + 255) / 256));
            for_slabs(threads, (int64_t)found.size(), [&](int64_t c) {
                std::vector<int> nbA, nbS;
                std::vector<double>& out = found[(size_t)c];
                for (int64_t f = c * 256; f < std::min<int64_t>(nf, (c + 1) * 256); f++) {
                    const double* A = &frontier[3 * (size_t)f];
                    tree.within(A, rN * rN, nbA);
                    sites_within(A, rN, nbS);
                    auto reflect = [&](const double* B) {
                        const double q[3] = {2.0 * A[0] - B[0], 2.0 * A[1] - B[1], 2.0 * A[2] - B[2]};
                        if (q[0] <= -W + m || q[0] >= W - m || q[1] <= -W + m || q[1] >= W - m || q[2] <= m ||
                            q[2] >= H - m)
                            return;
                        // cheap tests first (the merge below would reject
                        // these too): a site of an earlier generation there
                        // already, or no atom within the fine shell
                        if (site_near(q, 0.5 * h0) || !atom_in_reach(q[0], q[1], q[2])) return;
                        const double d = std::sqrt(tree.nearest2(q));
                        if (d < std::max(excl, 0.5 * h0) || d > S) return;
                        out.insert(out.end(), q, q + 3);
                    };
                    for (int b : nbA) {
                        const double B[3] = {atoms[3 * (size_t)b], atoms[3 * (size_t)b + 1], atoms[3 * (size_t)b + 2]};
                        reflect(B);
                    }
                    for (int b : nbS) reflect(&sites[3 * (size_t)b]);
                }
            });
            std::vector<double> next;
            for (const auto& c : found)
                for (size_t k = 0; k < c.size(); k += 3) {
                    const double* q = &c[k];
                    if (site_near(q, 0.5 * h0)) continue;
                    const int id = (int)(sites.size() / 3);
                    sites.insert(sites.end(), q, q + 3);
                    siteCells[cell_key(cell(q[0]), cell(q[1]), cell(q[2]))].push_back(id);
                    next.insert(next.end(), q, q + 3);
                }
            frontier.swap(next);
        }
        // out, jittered by up to 1% of h0 per coordinate (a truncated
        // lattice has co-spherical point sets at its outer edge)
        for (size_t k = 0; k < sites.size() / 3; k++) {
            double q[3];
            for (int a = 0; a < 3; a++)
                q[a] = sites[3 * k + a] + 0.02 * h0 * (hash_unit(p.seed, 7000, (int64_t)k, a, 0, 0) - 0.5);
            push(q[0], q[1], q[2], p.vacuum_id);
            mesh.num_vacuum++;
        }
    }

    void push(double x, double y, double z, int id) {
        mesh.xyz.push_back((float)x);
        mesh.xyz.push_back((float)y);
        mesh.xyz.push_back((float)z);
        mesh.id.push_back((short)id);
    }

    // Jittered cubic-grid points of level k in the slab range of x indices
    // [i0, i1]: kept where the nearest atom lies in (dIn, dOut] (and at least
    // the exclusion distance off); one slab per x index, in index order.
    void volume_level(size_t k, double x0, double x1, double y0, double y1, double z0, double z1, int tag) {
        const double h = levelSpacing[k];
        const double dIn = k == 0 ? -1.0 : levelOuter[k - 1], dOut = levelOuter[k];
        const double excl = p.exclusion * h0;
        const int64_t i0 = (int64_t)std::floor(x0 / h) - 1, i1 = (int64_t)std::ceil(x1 / h) + 1;
        const int64_t j0 = (int64_t)std::floor(y0 / h) - 1, j1 = (int64_t)std::ceil(y1 / h) + 1;
        const int64_t l0 = std::max<int64_t>(0, (int64_t)std::floor(z0 / h) - 1), l1 = (int64_t)std::ceil(z1 / h) + 1;
        std::vector<std::vector<float>> slabs((size_t)(i1 - i0 + 1));
        for_slabs(threads, i1 - i0 + 1, [&](int64_t s) {
            const int64_t i = i0 + s;
            std::vector<float>& out = slabs[(size_t)s];
            for (int64_t j = j0; j <= j1; j++)
                for (int64_t l = l0; l <= l1; l++) {
                    const double x = (i + 0.5 + 0.6 * (hash_unit(p.seed, tag, (int64_t)k, i, j, l * 4 + 0) - 0.5)) * h;
                    const double y = (j + 0.5 + 0.6 * (hash_unit(p.seed, tag, (int64_t)k, i, j, l * 4 + 1) - 0.5)) * h;
                    const double z = (l + 0.5 + 0.6 * (hash_unit(p.seed, tag, (int64_t)k, i, j, l * 4 + 2) - 0.5)) * h;
                    const double m = 0.2 * h;
                    if (x <= -W + m || x >= W - m || y <= -W + m || y >= W - m || z <= m || z >= H - m) continue;
                    if (box_distance(x, y, z) > dOut) continue;
                    if (k == 0) {
                        // level 0 ends at the fine shell, and the lattice's
                        // sites fill it in a crystal: two cheap tests first
                        const double q[3] = {x, y, z};
                        if (!atom_in_reach(x, y, z) || site_near(q, excl)) continue;
                    }
                    const double d = distance(x, y, z);
                    if (d <= dIn || d > dOut || d < excl) continue;
                    out.push_back((float)x);
                    out.push_back((float)y);
                    out.push_back((float)z);
                }
        });
        for (const auto& s : slabs)
            for (size_t q = 0; q < s.size(); q += 3) {
                push(s[q], s[q + 1], s[q + 2], p.vacuum_id);
                mesh.num_vacuum++;
            }
    }

    void vacuum() {
        for (size_t k = 0; k < levelSpacing.size(); k++) {
            const double dOut = levelOuter[k];
            const double reach = dOut < 1e299 ? dOut : 1e300;
            const double x0 = std::max(-W, bmin[0] - reach), x1 = std::min(W, bmax[0] + reach);
            const double y0 = std::max(-W, bmin[1] - reach), y1 = std::min(W, bmax[1] + reach);
            const double z0 = std::max(0.0, bmin[2] - reach), z1 = std::min(H, bmax[2] + reach);
            volume_level(k, x0, x1, y0, y1, z0, z1, 6000);
        }
    }

    // Points on one face of the box; (u, v) span the face, the fixed
    // coordinate is `fixedVal` on axis `axis`.  Jittered in the face and kept
    // 0.2 h away from its edges.
    void boundary_face(int axis, double fixedVal, double u0, double u1, double v0, double v1, int id, int faceTag) {
        // the two in-face axes
        const int au = axis == 0 ? 1 : 0, av = axis == 2 ? 1 : 2;
        for (size_t k = 0; k < levelSpacing.size(); k++) {
            const double h = levelSpacing[k];
            const double dIn = k == 0 ? -1.0 : levelOuter[k - 1];
            const double dOut = levelOuter[k];
            double lu0 = u0, lu1 = u1, lv0 = v0, lv1 = v1;
            if (dOut < 1e299) {
                lu0 = std::max(u0, bmin[au] - dOut);
                lu1 = std::min(u1, bmax[au] + dOut);
                lv0 = std::max(v0, bmin[av] - dOut);
                lv1 = std::min(v1, bmax[av] + dOut);
                if (lu0 >= lu1 || lv0 >= lv1) continue;
            }
            const int64_t i0 = (int64_t)std::floor(lu0 / h) - 1, i1 = (int64_t)std::ceil(lu1 / h) + 1;
            const int64_t j0 = (int64_t)std::floor(lv0 / h) - 1, j1 = (int64_t)std::ceil(lv1 / h) + 1;
            std::vector<std::vector<float>> slabs((size_t)(i1 - i0 + 1));
            for_slabs(threads, i1 - i0 + 1, [&](int64_t s) {
                const int64_t i = i0 + s;
                std::vector<float>& out = slabs[(size_t)s];
                for (int64_t j = j0; j <= j1; j++) {
                    const double u = (i + 0.5 + 0.6 * (hash_unit(p.seed, 8000 + faceTag, (int64_t)k, i, j, 0) - 0.5)) * h;
                    const double v = (j + 0.5 + 0.6 * (hash_unit(p.seed, 8000 + faceTag, (int64_t)k, i, j, 1) - 0.5)) * h;
                    if (u <= u0 + 0.2 * h || u >= u1 - 0.2 * h || v <= v0 + 0.2 * h || v >= v1 - 0.2 * h) continue;
                    double q[3];
                    q[axis] = fixedVal;
                    q[au] = u;
                    q[av] = v;
                    if (box_distance(q[0], q[1], q[2]) > dOut) continue;
                    const double d = distance(q[0], q[1], q[2]);
                    // a face point may sit nearer the sample than a volume
                    // point (the sample's base rests on the bottom plane)
                    if (d <= dIn || d > dOut || d < 0.25 * h0) continue;
                    out.push_back((float)q[0]);
                    out.push_back((float)q[1]);
                    out.push_back((float)q[2]);
                }
            });
            for (const auto& s : slabs)
                for (size_t q = 0; q < s.size(); q += 3) {
                    push(s[q], s[q + 1], s[q + 2], id);
                    mesh.num_boundary++;
                }
        }
    }

    // interior points of one box edge, at the spacing of the level its
    // midpoint falls into
    void boundary_edge(double x0, double y0, double z0, double x1, double y1, double z1, int tag) {
        const double mx = 0.5 * (x0 + x1), my = 0.5 * (y0 + y1), mz = 0.5 * (z0 + z1);
        const double d = distance(mx, my, mz);
        size_t k = 0;
        while (k + 1 < levelOuter.size() && d > levelOuter[k]) k++;
        const double h = levelSpacing[k];
        const double len = std::sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0) + (z1 - z0) * (z1 - z0));
        const int64_t n = std::max<int64_t>(1, (int64_t)std::floor(len / h));
        for (int64_t i = 1; i <= n; i++) {
            const double t = (i + 0.4 * (hash_unit(p.seed, 9000 + tag, i, 0, 0, 0) - 0.5)) / (n + 1);
            push(x0 + t * (x1 - x0), y0 + t * (y1 - y0), z0 + t * (z1 - z0), p.sides_id);
            mesh.num_boundary++;
        }
    }

    // meshgen's markers: bottom (z = 0), top (z = H), sides for the side
    // faces and for every node on an edge or corner of the box
    void boundaries() {
        boundary_face(2, H, -W, W, -W, W, p.top_id, 0);
        boundary_face(2, 0.0, -W, W, -W, W, p.bottom_id, 1);
        boundary_face(0, -W, -W, W, 0.0, H, p.sides_id, 2);
        boundary_face(0, W, -W, W, 0.0, H, p.sides_id, 3);
        boundary_face(1, -W, -W, W, 0.0, H, p.sides_id, 4);
        boundary_face(1, W, -W, W, 0.0, H, p.sides_id, 5);
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
        for (int sx = 0; sx < 2; sx++)
            for (int sy = 0; sy < 2; sy++)
                for (int sz = 0; sz < 2; sz++) {
                    push(sx ? W : -W, sy ? W : -W, sz ? H : 0.0, p.sides_id);
                    mesh.num_boundary++;
                }
    }
};

}  // namespace

std::string generate_sample_mesh(const std::vector<float>& xyz, const std::vector<short>& id,
                                 const SampleParams& params, int threads, SampleMesh* out) {
    if (!out) return "generate_sample_mesh: null output";
    if (xyz.size() != 3 * id.size() || id.empty()) return "generate_sample_mesh: empty or inconsistent sample";
    if (!(params.box_half_width > 0.0) || !(params.box_height > 0.0) || !(params.fine_shell > 0.0) ||
        !(params.coarsen > 1.0) || params.layers_per_level < 1 || !(params.exclusion > 0.0))
        return "generate_sample_mesh: bad parameters";
    for (short s : id)
        if (s == params.vacuum_id || s == params.top_id || s == params.bottom_id || s == params.sides_id)
            return "generate_sample_mesh: a sample atom carries a vacuum or boundary marker id";
    try {
        const KdTree tree(xyz);
        Builder b(params, tree, threads, xyz);
        b.boundaries();
        b.lattice_shell();
        b.vacuum();
        // the sample last (meshgen/meshgen.cpp:3908)
        for (size_t k = 0; k < id.size(); k++) b.push(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], id[k]);
        b.mesh.num_sample = (int)id.size();
        *out = std::move(b.mesh);
    } catch (const std::exception& e) {
        return e.what();
    }
    return std::string();
}

}  // namespace tg_host

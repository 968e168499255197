// Synthetic atom-probe specimens: a bcc lattice cut to a tip shape (spherical
// cap on a conical or cylindrical shank), embedded in a vacuum region that is
// coarsened geometrically with distance from the tip up to a planar
// counter-electrode.  The output is the point set and per-point type id of a
// TAPSim node file (meshgen output layout: generated vacuum and boundary
// points first, specimen atoms appended last, meshgen/meshgen.cpp:3908).
//
// The point set is built to be in general position (no five points on a
// sphere, no four coplanar points on a circle): the bcc lattice is
// non-degenerate, vacuum points off the lattice are jittered, and points on
// the flat boundary planes are jittered within their plane.  Its Delaunay
// tetrahedralization is therefore unique, so any correct Delaunay code (the
// reference's TetGen or the builder in delaunay.cpp) yields the same mesh.
#pragma once

#include <cstdint>
#include <vector>

namespace tg_host {

// SplitMix64 finaliser (the point jitter of the generated meshes)
inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform in [0,1) from a hash of (seed, a, b, c, d, e).
inline double hash_unit(uint64_t seed, int64_t a, int64_t b, int64_t c, int64_t d, int64_t e) {
    uint64_t h = mix64(seed);
    h = mix64(h ^ (uint64_t)a);
    h = mix64(h ^ (uint64_t)b);
    h = mix64(h ^ (uint64_t)c);
    h = mix64(h ^ (uint64_t)d);
    h = mix64(h ^ (uint64_t)e);
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

struct TipParams {
    double lattice_a = 0.2866e-9;      // bcc lattice constant [m]
    double cap_radius = 5e-9;          // R [m]
    double shank_length = 10e-9;       // height of the shank below the cap tangent line [m]
    double half_angle_deg = 0.0;       // shank half angle (0 = cylinder)
    double box_half_width = 0.5e-6;    // vacuum box |x|,|y| <= W [m]
    double box_height = 1.0e-6;        // counter-electrode plane z = H [m]
    double fine_shell = 1.0e-9;        // thickness of the lattice-continuation vacuum shell [m]
    int layers_per_level = 4;          // point layers per coarsening level
    double coarsen = 2.0;              // spacing ratio between levels
    double max_spacing = 0.0;          // cap on the coarse spacing (0 = none) [m]
    // binary alloy (second species on lattice sites)
    double solute_fraction = 0.0;      // total solute atom fraction
    double precip_density = 0.0;       // precipitate number density [1/m^3]
    double precip_rmin = 1e-9, precip_rmax = 2e-9;  // lognormal radius, clipped [m]
    double precip_mu = 0.0, precip_sigma = 0.25;    // lognormal of r / 1 nm
    uint64_t seed = 1;
    // type ids (meshgen markers and the specimen species)
    int vacuum_id = 0, top_id = 1, bottom_id = 2, sides_id = 3;
    int matrix_id = 4, solute_id = 5;
};

struct TipMesh {
    std::vector<float> xyz;     // 3 per node [m]
    std::vector<short> id;      // type id per node
    int num_atoms = 0;          // specimen atoms (the trailing block)
    int num_solute = 0;
    int num_vacuum = 0;
    int num_boundary = 0;
    double apex_z = 0.0;        // apex height of the tip shape [m]
};

// Builds the specimen and its vacuum region.  Deterministic in params.seed.
TipMesh generate_tip(const TipParams& params);

}  // namespace tg_host

// Vacuum mesh around an arbitrary sample: the role of the reference's
// MeshGen (meshgen/meshgen.cpp:2506-3986).  MeshGen reads a sample node file
// (readSample, :197-360), builds cascaded TetGen levels of vacuum around it,
// marks the outer box's nodes as bottom (z = 0), top (z = extent) or sides
// (:3855-3892) and appends the sample's points last (:3908).
//
// This builder places the vacuum points itself, as the tip generator does,
// but grades them by the distance to the nearest sample atom (a k-d tree
// over the sample) instead of an analytic tip shape:
//   - level 0, out to `fine_shell`: the sample's lattice continued into the
//     vacuum (every reflection A + (A - B) of a nearest neighbour B through
//     a surface atom or an earlier vacuum site A that lands on no atom),
//     then a jittered cubic grid at the sample's point spacing h0 (the
//     median nearest-neighbour distance) where that left room, every point
//     `exclusion` h0 or more off the atoms;
//   - levels k >= 1: jittered cubic grids whose spacing grows by `coarsen`
//     every `layers_per_level` layers, out to the box;
//   - the box faces (top z = H, bottom z = 0, sides |x|, |y| = W), their
//     edges and corners at the spacing of the level they fall into.
// The sample must lie inside the box, above the bottom plane z = 0, and
// away from the other faces by at least its fine shell.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tg_host {

struct SampleParams {
    double box_half_width = 0.5e-6;    // vacuum box |x|,|y| <= W, centred on x = y = 0 [m]
    double box_height = 1.0e-6;        // top plane z = H [m]
    double fine_shell = 1.0e-9;        // thickness of the level-0 vacuum [m]
    double exclusion = 0.8;            // vacuum points keep this many h0 off every atom
    int layers_per_level = 4;          // point layers per coarsening level
    double coarsen = 2.0;              // spacing ratio between levels
    double max_spacing = 0.0;          // cap on the coarse spacing (0 = none) [m]
    uint64_t seed = 1;
    // meshgen's markers (VACUUM_MARKER, TOP_MARKER, BOTTOM_MARKER, SIDES_MARKER)
    int vacuum_id = 0, top_id = 1, bottom_id = 2, sides_id = 3;
};

struct SampleMesh {
    std::vector<float> xyz;        // 3 per node [m]: generated nodes, then the sample
    std::vector<short> id;         // type id per node
    int num_sample = 0;            // the trailing block
    int num_vacuum = 0;
    int num_boundary = 0;
    double spacing = 0.0;          // h0 [m]
};

// Builds the vacuum and boundary nodes around the sample (xyz: 3 floats per
// atom, id: type ids) and appends the sample.  Deterministic in the seed,
// whatever the thread count.  Returns an empty string or the error.
std::string generate_sample_mesh(const std::vector<float>& xyz, const std::vector<short>& id,
                                 const SampleParams& params, int threads, SampleMesh* out);

}  // namespace tg_host

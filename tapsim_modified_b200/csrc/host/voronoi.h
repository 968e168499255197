// Mesh tables derived from a Delaunay tetrahedralization: the Delaunay
// adjacency as CSR, the Voronoi face geometry of every edge (FP64), hull
// flags and the per-node tetrahedron hint.
//
// Follows the reference's geometry routines:
//   adjacency            Geometry_3d::Table::adjacentNodes      geometry_3d.cpp:1098-1110
//   hull flag            Geometry_3d::Table::setBoundary        geometry_3d.cpp:1688-1710
//   tetrahedron hint     Geometry_3d::Table::setAssociatedTetrahedra  geometry_3d.cpp:1712-1722
//   Voronoi face walk    Geometry_3d::Table::get_voronoiFace    geometry_3d.cpp:1211-1382
//   capped face area     VoronoiFace::finiteCenter/finiteArea   geometry_3d.cpp:243-360
//   circumcentre         Geometry_3d::Table::tetCenter          geometry_3d.cpp:830-870
//   capped cell volume   VoronoiCell::finiteVolume              geometry_3d.cpp:437-453
// The reference evaluates face areas in float from float-rounded
// circumcentres; here every step is FP64.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tg_host {

struct MeshTables {
    int num_nodes = 0;
    int num_tets = 0;
    std::vector<int32_t> row_ptr;     // n+1
    std::vector<int32_t> col;         // nnz, ascending within a row
    std::vector<int32_t> rev;         // nnz, position of the mirrored entry (j,i)
    std::vector<double> dist;         // nnz, |p_i - p_j| [m]
    std::vector<double> area_half;    // nnz, face area capped with infinity factor 0.5*d [m^2]
    std::vector<uint8_t> area_pos;    // nnz, face area capped with factor 1.0 is > 0
    std::vector<uint8_t> hull;        // n, node lies on the convex hull
    std::vector<int32_t> node_tet;    // n, last tetrahedron (in tet order) containing the node
    std::vector<double> volume;       // n, capped Voronoi volume with the factor of
                                      // Grid_3d::Table::computeCharge (grid_3d.cpp:1373-1390):
                                      // half the mean neighbour distance [m^3]
};

// Builds all tables.  xyz: 3 floats per node; tets as produced by
// delaunay_tetrahedralize (or read from a TAPSIM geometry table).
std::string build_mesh_tables(const float* xyz, int n, const int32_t* tet_v, const int32_t* tet_n,
                              int num_tets, int threads, MeshTables* out);

}  // namespace tg_host

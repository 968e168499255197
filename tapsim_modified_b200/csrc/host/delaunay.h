// Delaunay tetrahedralization of a 3D point set (host, built once per mesh).
//
// Replaces the reference's TetGen call in Geometry_3d::Table::tetrahedralize
// (tapsim/geometry_3d.cpp:759-810, TetGen switches "znNFCQ": zero-based
// indices, neighbour list, no boundary output, quiet).  Output layout matches
// what the reference keeps from TetGen: per tetrahedron four vertex indices
// and four neighbour indices, neighbour k opposite vertex k, -1 on the convex
// hull, and every tetrahedron positively oriented in the sense of
// Geometry_3d::Table::setOrientation (geometry_3d.cpp:1778-1788).
//
// Algorithm: incremental Bowyer-Watson insertion with an infinite vertex for
// the convex hull, biased randomized insertion order (rounds of doubling size,
// each sorted along a Morton curve), visibility-walk point location, and
// exact predicates on snapped integer coordinates (predicates.h).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tg_host {

struct Tetrahedralization {
    std::vector<int32_t> vertices;    // 4 per tet
    std::vector<int32_t> neighbours;  // 4 per tet, -1 on the hull
    int num_tets() const { return (int)(vertices.size() / 4); }
};

// Returns an empty string on success, otherwise an error message.
// `xyz` holds 3 floats per point.  Duplicate points are rejected.
std::string delaunay_tetrahedralize(const float* xyz, int n, uint64_t seed, Tetrahedralization* out);

}  // namespace tg_host

// Byte-compatible readers and writers for the reference's file formats.
//
//   node file   File_Io::readGeomGrid / writeGeomGrid   tapsim/file_io.cpp:765-1011
//               (meshgen writes the same layout, meshgen/meshgen.cpp:362-446)
//   config      File_Io::readConfig / writeConfig       tapsim/file_io.cpp:100-460
//   ini         File_Io::readInitialization            tapsim/file_io.cpp:58-92
//   dump        File_Io::writeSystem / readSystem       tapsim/file_io.cpp:1013-1062 with the
//               binary tables of Configuration::Table   tapsim/configuration.cpp:62-210,
//               Geometry_3d::Table                      tapsim/geometry_3d.cpp:530-640,
//               Grid_3d::Table                          tapsim/grid_3d.cpp:248-381
//   results     File_Io::LogResults                     tapsim/logResults.cpp:135-381
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace tg_host {

struct NodeFile {
    std::vector<float> xyz;
    std::vector<short> id;
    std::vector<uint32_t> number;  // read, or assigned as readGeomGrid does
    bool has_numbers = false;      // the file carries numbers
    std::vector<float> phi;        // empty when the file carries no potentials
};

// Reads ASCII or BINARY node files.  Numbers that are absent or invalid (0)
// are assigned as readGeomGrid does (file_io.cpp:975-1000).
std::string read_node_file(const std::string& path, NodeFile* out);
std::string write_node_file(const std::string& path, const NodeFile& nf, bool binary);

struct CellType {
    int id = -1;
    std::string name;
    float charge_density = 0.0f;   // [C/m^3]
    float epsilon = 1.0f;
    bool removable = true;
    bool neumann = false;
    bool dirichlet = false;
    float phi = 0.0f;              // [V]
    float mass = 0.0f;             // [amu]
    short evap_charge = 0;
    float evap_field = 0.0f;       // [V/m]
    float evap_energy = 0.0f;      // [eV]
};

struct ConfigTable {
    float temperature = 0.0f;
    std::map<int, CellType> types;  // by id
    int id_of(const std::string& name) const;
};

std::string read_config(const std::string& path, ConfigTable* out);
std::string write_config_ascii(const std::string& path, const ConfigTable& table);

std::string read_ini(const std::string& path, std::map<std::string, std::string>* out);

// TAPSIM DUMP contents.
struct Dump {
    uint32_t last_index = 0;
    ConfigTable config;
    float min[3], max[3], cmin[3], cmax[3];
    std::vector<float> xyz;
    std::vector<uint8_t> hull;
    std::vector<int32_t> node_tet;
    std::vector<int32_t> tet_v, tet_n;
    double relaxation_factor = 0.0;
    int32_t phi_switch = 0;
    std::vector<int8_t> id;
    std::vector<uint32_t> number;
    std::vector<float> phi0, phi1, charge;
    std::vector<uint8_t> boundary, dirichlet, neumann;
    std::vector<int32_t> row_ptr, col;
    std::vector<float> coupling;
};

std::string read_dump(const std::string& path, Dump* out);
std::string write_dump(const std::string& path, const Dump& d);

// One record of the results log (LogResults::Dataset, logResults.h:41-66).
struct ResultRecord {
    uint32_t index;
    short id;
    uint32_t number;
    float voltage;
    float start[3], stop[3];
    float tof;
    float probability;
    float phi_before, field_before[3];
    float phi_after, field_after[3];
    float normal[3], apex[3];
};

// Results files; with chunk > 0 split as LogResults' writer thread does
// (path.%08u after the index opening each chunk, the header text in the
// first file only).
std::string write_results(const std::string& path, const std::vector<ResultRecord>& recs, bool binary,
                          const std::string& header, int chunk = 0);

// One trajectory of the trajectory log (LogTrajectory::Dataset).
struct TrajectoryRecord {
    uint32_t index, number;
    float time_scale;
    int32_t status;
    float charge, mass;
    int32_t num_points;
    const float* points;  // 8 words a point: time, position, velocity, tetrahedron bits
    float error[6];
};
std::string write_trajectories(const std::string& path, const std::vector<TrajectoryRecord>& recs, bool binary,
                               int chunk = 0);

// One grid snapshot as File_Io::LogGrid writes it (logGrid.cpp:197-245):
// per cell the type id, unique number, potential, field_o1 [3] and
// force [3].
struct GridLog {
    int n;
    const int32_t* id;
    const uint32_t* number;
    const float* phi;
    const float* field;
    const float* force;
};
std::string write_grid_log(const std::string& path, bool binary, const GridLog& g);

// One surface snapshot as File_Io::LogSurface::writer writes it
// (logSurface.cpp:203-293): the surface cells in ascending index order with
// type, unique number, probability and optionally their neighbour lists
// (neighbour_ptr null: none), then the cells and all their neighbours in
// ascending order with potential, field_o1 [3] and normal [3] (zero for
// cells off the surface).
struct SurfaceLog {
    int cells;
    const int32_t* cell;
    const int32_t* type;
    const uint32_t* number;
    const float* probability;
    const int32_t* neighbour_ptr;  // [cells + 1]
    const int32_t* neighbours;
    int nodes;
    const int32_t* node;
    const float* phi;
    const float* field;
    const float* normal;
};
std::string write_surface_log(const std::string& path, bool binary, const SurfaceLog& s);

}  // namespace tg_host

// Host-side mesh objects behind tg_mesh_* (include/tapsim_gpu.h): build the
// arrays of a tg_mesh_desc from the tip generator, from a node file plus
// configuration (the reference's Process::initialization path:
// readConfig, readGeomGrid, tetrahedralize, fastSync; process.cpp:47-129), or
// from a TAPSIM dump (File_Io::readSystem, the resumption path).
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/tapsim_gpu.h"
#include "delaunay.h"
#include "formats.h"
#include "samplegen.h"
#include "tipgen.h"
#include "voronoi.h"

using namespace tg_host;

struct tg_mesh {
    std::vector<float> xyz;
    std::vector<int8_t> type;
    std::vector<uint8_t> hull;
    std::vector<float> phi;
    std::vector<int32_t> row_ptr, col;
    std::vector<double> coupling, geom, volume;
    std::vector<uint8_t> area_pos;
    std::vector<int32_t> tet_v, tet_n, node_tet;
    std::vector<uint32_t> number;
    ConfigTable config;
    std::vector<tg_type> types;
    bool has_geom = false;
    uint32_t dump_index = 0;  // LAST_INDEX of the dump the mesh was read from
};

namespace tgapi {
void set_process_error(const std::string& msg);  // handle.cu: read by tg_last_error(NULL)
}

namespace {

int mesh_fail(const std::string& m) {
    tgapi::set_process_error(m);
    return TG_ERR_HOST;
}

void fill_types(tg_mesh* m) {
    m->types.clear();
    for (const auto& kv : m->config.types) {
        const CellType& c = kv.second;
        tg_type t;
        t.id = c.id;
        t.charge_density = c.charge_density;
        t.epsilon = c.epsilon;
        t.removable = c.removable;
        t.neumann = c.neumann;
        t.dirichlet = c.dirichlet;
        t.phi = c.phi;
        t.mass = c.mass;
        t.evap_charge = c.evap_charge;
        t.evap_field = c.evap_field;
        t.evap_energy = c.evap_energy;
        m->types.push_back(t);
    }
}

// Coupling of every entry as Grid_3d::Table::fastSync leaves it
// (grid_3d.cpp:491-553): the pair is evaluated once, from its lower index,
// by computeCoupling (grid_3d.cpp:1392-1409), and mirrored.
int couplings_from_tables(tg_mesh* m, const MeshTables& t) {
    const int n = (int)m->type.size();
    m->coupling.assign(t.col.size(), 0.0);
    m->geom.assign(t.col.size(), 0.0);
    for (int i = 0; i < n; i++) {
        for (int q = t.row_ptr[i]; q < t.row_ptr[i + 1]; q++) {
            const int j = t.col[q];
            const int lo = std::min(i, j), hi = std::max(i, j);
            auto ilo = m->config.types.find(m->type[lo]);
            auto ihi = m->config.types.find(m->type[hi]);
            if (ilo == m->config.types.end() || ihi == m->config.types.end())
                return mesh_fail("mesh: node type missing from the configuration");
            const CellType &a = ilo->second, &b = ihi->second;
            const double g = t.dist[q] > 0.0 ? t.area_half[q] / t.dist[q] : 0.0;
            m->geom[q] = g;
            if (!a.neumann && b.neumann) continue;
            m->coupling[q] = 2.0 * (double)a.epsilon * (double)b.epsilon / ((double)a.epsilon + (double)b.epsilon) * g;
        }
    }
    return TG_OK;
}

int build_from_points(tg_mesh* m, int threads, uint64_t seed) {
    const int n = (int)m->type.size();
    Tetrahedralization T;
    std::string err = delaunay_tetrahedralize(m->xyz.data(), n, seed, &T);
    if (!err.empty()) return mesh_fail(err);
    MeshTables t;
    err = build_mesh_tables(m->xyz.data(), n, T.vertices.data(), T.neighbours.data(), T.num_tets(), threads, &t);
    if (!err.empty()) return mesh_fail(err);
    m->tet_v.swap(T.vertices);
    m->tet_n.swap(T.neighbours);
    m->row_ptr.swap(t.row_ptr);
    m->col.swap(t.col);
    m->hull.swap(t.hull);
    m->node_tet.swap(t.node_tet);
    m->area_pos.swap(t.area_pos);
    m->volume.swap(t.volume);
    t.row_ptr = m->row_ptr;
    t.col = m->col;
    const int rc = couplings_from_tables(m, t);
    m->has_geom = true;
    return rc;
}

ConfigTable default_tip_config() {
    ConfigTable ct;
    auto add = [&](int id, const char* name, bool rem, bool neu, bool dir, float phi, float mass, short q, float E) {
        CellType t;
        t.id = id;
        t.name = name;
        t.removable = rem;
        t.neumann = neu;
        t.dirichlet = dir;
        t.phi = phi;
        t.mass = mass;
        t.evap_charge = q;
        t.evap_field = E;
        t.evap_energy = rem ? 1.0f : 0.0f;
        ct.types[id] = t;
    };
    // meshgen markers (meshgen/meshgen.cpp:491-595) with Neumann sides, and
    // the specimen species: bcc Fe (E_evap 33 V/nm) and Cu (30 V/nm), tip at 1 V
    add(0, "Vacuum", false, false, false, 0.0f, 0.0f, 0, 0.0f);
    add(1, "Top", false, false, true, 0.0f, 0.0f, 0, 0.0f);
    add(2, "Bottom", false, true, false, 0.0f, 0.0f, 0, 0.0f);
    add(3, "Sides", false, true, false, 0.0f, 0.0f, 0, 0.0f);
    add(4, "Fe", true, false, true, 1.0f, 55.845f, 2, 33e9f);
    add(5, "Cu", true, false, true, 1.0f, 63.546f, 2, 30e9f);
    return ct;
}

// The configuration template meshgen writes beside its node file
// (writeConfig, meshgen/meshgen.cpp:491-595): vacuum; top and sides
// Dirichlet at 0 V; bottom Neumann; every other id in the node set a
// removable Dirichlet cell at 1000 V and charge state 1, whose mass and
// evaporation field (left for the user to fill in there) are 0 here.
ConfigTable sample_config_template(const SampleParams& sp, const std::vector<short>& ids) {
    ConfigTable ct;
    auto add = [&](int id, const char* name, bool rem, bool neu, bool dir, float phi, short q, float energy) {
        CellType t;
        t.id = id;
        t.name = name;
        t.removable = rem;
        t.neumann = neu;
        t.dirichlet = dir;
        t.phi = phi;
        t.evap_charge = q;
        t.evap_energy = energy;
        ct.types[id] = t;
    };
    add(sp.vacuum_id, "Vacuum", false, false, false, 0.0f, 0, 0.0f);
    add(sp.top_id, "Top", false, false, true, 0.0f, 0, 0.0f);
    add(sp.bottom_id, "Bottom", false, true, false, 1000.0f, 0, 0.0f);
    add(sp.sides_id, "Sides", false, false, true, 0.0f, 0, 0.0f);
    for (short id : ids)
        if (!ct.types.count(id)) add(id, "Sample", true, false, true, 1000.0f, 1, 1.0f);
    return ct;
}

}  // namespace

extern "C" {

void tg_sample_params_default(tg_sample_params* p) {
    SampleParams d;
    p->box_half_width = d.box_half_width;
    p->box_height = d.box_height;
    p->fine_shell = d.fine_shell;
    p->exclusion = d.exclusion;
    p->layers_per_level = d.layers_per_level;
    p->coarsen = d.coarsen;
    p->max_spacing = d.max_spacing;
    p->vacuum_id = d.vacuum_id;
    p->top_id = d.top_id;
    p->bottom_id = d.bottom_id;
    p->sides_id = d.sides_id;
    p->seed = d.seed;
}

int tg_mesh_from_sample(const char* sampleFile, const char* configFile, const tg_sample_params* p, int32_t threads,
                        tg_mesh** out) {
    if (!sampleFile || !p || !out) return mesh_fail("tg_mesh_from_sample: null argument");
    NodeFile nf;
    std::string err = read_node_file(sampleFile, &nf);
    if (!err.empty()) return mesh_fail(err);
    SampleParams sp;
    sp.box_half_width = p->box_half_width;
    sp.box_height = p->box_height;
    sp.fine_shell = p->fine_shell;
    sp.exclusion = p->exclusion;
    sp.layers_per_level = p->layers_per_level;
    sp.coarsen = p->coarsen;
    sp.max_spacing = p->max_spacing;
    sp.vacuum_id = p->vacuum_id;
    sp.top_id = p->top_id;
    sp.bottom_id = p->bottom_id;
    sp.sides_id = p->sides_id;
    sp.seed = p->seed;
    const int nThreads = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    SampleMesh sm;
    err = generate_sample_mesh(nf.xyz, nf.id, sp, nThreads, &sm);
    if (!err.empty()) return mesh_fail(err);
    tg_mesh* m = new tg_mesh();
    if (configFile) {
        err = read_config(configFile, &m->config);
        if (!err.empty()) {
            delete m;
            return mesh_fail(err);
        }
    } else {
        m->config = sample_config_template(sp, nf.id);
    }
    fill_types(m);
    const int n = (int)sm.id.size();
    const int nGen = n - sm.num_sample;
    m->xyz.swap(sm.xyz);
    m->type.resize(n);
    m->phi.resize(n);
    m->number.resize(n);
    // numbers as readGeomGrid gives them to meshgen's output
    // (file_io.cpp:975-1000): the sample keeps the numbers its file carries
    // and the generated nodes before it count on from the largest; without
    // numbers in the file every node is numbered in node order
    uint32_t next = 1;
    if (nf.has_numbers)
        for (uint32_t v : nf.number) next = std::max(next, v + 1);
    for (int i = 0; i < n; i++) {
        if (sm.id[i] < -128 || sm.id[i] > 127) {
            delete m;
            return mesh_fail("tg_mesh_from_sample: type id outside -128..127");
        }
        m->type[i] = (int8_t)sm.id[i];
        auto it = m->config.types.find(m->type[i]);
        if (it == m->config.types.end()) {
            delete m;
            return mesh_fail("tg_mesh_from_sample: node type missing from the configuration");
        }
        const bool sample = i >= nGen;
        m->phi[i] = sample && !nf.phi.empty() ? nf.phi[i - nGen] : it->second.phi;
        m->number[i] = !nf.has_numbers ? (uint32_t)(i + 1) : sample ? nf.number[i - nGen] : next++;
    }
    const int rc = build_from_points(m, nThreads, sp.seed);
    if (rc != TG_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return TG_OK;
}

void tg_tip_params_default(tg_tip_params* p) {
    TipParams d;
    p->lattice_a = d.lattice_a;
    p->cap_radius = d.cap_radius;
    p->shank_length = d.shank_length;
    p->half_angle_deg = d.half_angle_deg;
    p->box_half_width = d.box_half_width;
    p->box_height = d.box_height;
    p->fine_shell = d.fine_shell;
    p->layers_per_level = d.layers_per_level;
    p->coarsen = d.coarsen;
    p->max_spacing = d.max_spacing;
    p->solute_fraction = d.solute_fraction;
    p->precip_density = d.precip_density;
    p->precip_rmin = d.precip_rmin;
    p->precip_rmax = d.precip_rmax;
    p->precip_mu = d.precip_mu;
    p->precip_sigma = d.precip_sigma;
    p->seed = d.seed;
}

int tg_mesh_from_tip(const tg_tip_params* p, int32_t threads, tg_mesh** out) {
    if (!p || !out) return mesh_fail("tg_mesh_from_tip: null argument");
    TipParams tp;
    tp.lattice_a = p->lattice_a;
    tp.cap_radius = p->cap_radius;
    tp.shank_length = p->shank_length;
    tp.half_angle_deg = p->half_angle_deg;
    tp.box_half_width = p->box_half_width;
    tp.box_height = p->box_height;
    tp.fine_shell = p->fine_shell;
    tp.layers_per_level = p->layers_per_level;
    tp.coarsen = p->coarsen;
    tp.max_spacing = p->max_spacing;
    tp.solute_fraction = p->solute_fraction;
    tp.precip_density = p->precip_density;
    tp.precip_rmin = p->precip_rmin;
    tp.precip_rmax = p->precip_rmax;
    tp.precip_mu = p->precip_mu;
    tp.precip_sigma = p->precip_sigma;
    tp.seed = p->seed;
    TipMesh tm;
    try {
        tm = generate_tip(tp);
    } catch (const std::exception& e) {
        return mesh_fail(e.what());
    }
    tg_mesh* m = new tg_mesh();
    m->xyz.swap(tm.xyz);
    m->type.assign(tm.id.begin(), tm.id.end());
    m->config = default_tip_config();
    fill_types(m);
    const int n = (int)m->type.size();
    m->phi.resize(n);
    for (int i = 0; i < n; i++) m->phi[i] = m->config.types[m->type[i]].phi;
    m->number.resize(n);
    for (int i = 0; i < n; i++) m->number[i] = i + 1;
    const int rc = build_from_points(m, threads, p->seed);
    if (rc != TG_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return TG_OK;
}

int tg_mesh_from_files(const char* nodeFile, const char* configFile, int32_t threads, tg_mesh** out) {
    if (!nodeFile || !configFile || !out) return mesh_fail("tg_mesh_from_files: null argument");
    NodeFile nf;
    std::string err = read_node_file(nodeFile, &nf);
    if (!err.empty()) return mesh_fail(err);
    tg_mesh* m = new tg_mesh();
    err = read_config(configFile, &m->config);
    if (!err.empty()) {
        delete m;
        return mesh_fail(err);
    }
    fill_types(m);
    const int n = (int)nf.id.size();
    m->xyz.swap(nf.xyz);
    m->type.assign(nf.id.begin(), nf.id.end());
    m->number.swap(nf.number);
    m->phi.resize(n);
    for (int i = 0; i < n; i++) {
        auto it = m->config.types.find(m->type[i]);
        if (it == m->config.types.end()) {
            delete m;
            return mesh_fail("tg_mesh_from_files: node type missing from the configuration");
        }
        // initial potentials: preset values unless the file carries them
        // (Process::initialization, process.cpp:63-79)
        m->phi[i] = nf.phi.empty() ? it->second.phi : nf.phi[i];
    }
    const int rc = build_from_points(m, threads, 1);
    if (rc != TG_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return TG_OK;
}

int tg_mesh_from_dump(const char* dumpFile, const char* configFile, tg_mesh** out) {
    if (!dumpFile || !out) return mesh_fail("tg_mesh_from_dump: null argument");
    Dump d;
    std::string err = read_dump(dumpFile, &d);
    if (!err.empty()) return mesh_fail(err);
    tg_mesh* m = new tg_mesh();
    if (configFile) {
        err = read_config(configFile, &m->config);
        if (!err.empty()) {
            delete m;
            return mesh_fail(err);
        }
    } else {
        m->config = d.config;
    }
    fill_types(m);
    const int n = (int)d.id.size();
    m->xyz.swap(d.xyz);
    m->type.assign(d.id.begin(), d.id.end());
    m->hull.swap(d.hull);
    m->number.swap(d.number);
    // Grid_3d::Table::potential(i) reads phi[(phiSwitch + 1) % 2] (grid_3d.h:184)
    m->phi = ((d.phi_switch + 1) % 2) ? d.phi1 : d.phi0;
    m->dump_index = d.last_index;
    m->row_ptr.swap(d.row_ptr);
    m->col.swap(d.col);
    m->coupling.assign(d.coupling.begin(), d.coupling.end());
    m->tet_v.swap(d.tet_v);
    m->tet_n.swap(d.tet_n);
    m->node_tet.swap(d.node_tet);
    for (int i = 0; i < n; i++)
        for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++)
            if (q > m->row_ptr[i] && m->col[q] <= m->col[q - 1]) {
                delete m;
                return mesh_fail("tg_mesh_from_dump: neighbour lists are not ascending");
            }
    for (int32_t c : m->col)
        if (c < 0 || c >= n) {
            delete m;
            return mesh_fail("tg_mesh_from_dump: neighbour index out of range");
        }
    // The dump's couplings were computed with the dump's own type table
    // (computeCoupling, grid_3d.cpp:1392-1409: 2 e1 e2 / (e1 + e2) times
    // area / distance).  Dividing that table's permittivity factor out gives
    // each entry's geometric factor, so that a removal resynced under another
    // configuration sees the true geometry, as the reference's does.
    auto eps = [&](int id) {
        const auto it = d.config.types.find(id);
        return it == d.config.types.end() ? 1.0 : (double)it->second.epsilon;
    };
    m->geom.resize(m->coupling.size());
    for (int i = 0; i < n; i++)
        for (int q = m->row_ptr[i]; q < m->row_ptr[i + 1]; q++) {
            const double e1 = eps(m->type[i]), e2 = eps(m->type[m->col[q]]);
            m->geom[q] = m->coupling[q] / (2.0 * e1 * e2 / (e1 + e2));
        }
    m->has_geom = true;
    *out = m;
    return TG_OK;
}

void tg_mesh_destroy(tg_mesh* m) { delete m; }

float tg_mesh_temperature(const tg_mesh* m) { return m ? m->config.temperature : 0.0f; }

int32_t tg_mesh_type_id(const tg_mesh* m, const char* name) {
    if (!m || !name) return -1;
    return m->config.id_of(name);
}

int tg_mesh_describe(const tg_mesh* m, tg_mesh_desc* d, int32_t* nnz) {
    if (!m || !d) return mesh_fail("tg_mesh_describe: null argument");
    std::memset(d, 0, sizeof(*d));
    d->num_nodes = (int32_t)m->type.size();
    d->xyz = m->xyz.data();
    d->type_id = m->type.data();
    d->hull = m->hull.empty() ? nullptr : m->hull.data();
    d->phi = m->phi.data();
    d->row_ptr = m->row_ptr.data();
    d->col = m->col.data();
    d->coupling = m->coupling.data();
    d->geom = m->has_geom ? m->geom.data() : nullptr;
    d->area_pos = m->area_pos.empty() ? nullptr : m->area_pos.data();
    d->volume = m->volume.empty() ? nullptr : m->volume.data();
    d->num_tets = (int32_t)(m->tet_v.size() / 4);
    d->tet_v = m->tet_v.data();
    d->tet_n = m->tet_n.data();
    d->node_tet = m->node_tet.data();
    d->num_types = (int32_t)m->types.size();
    d->types = m->types.data();
    if (nnz) *nnz = (int32_t)m->col.size();
    return TG_OK;
}

int tg_mesh_write_node_file(const tg_mesh* m, const char* path, int32_t binary) {
    if (!m || !path) return mesh_fail("tg_mesh_write_node_file: null argument");
    NodeFile nf;
    nf.xyz = m->xyz;
    nf.id.assign(m->type.begin(), m->type.end());
    const std::string err = write_node_file(path, nf, binary != 0);
    return err.empty() ? TG_OK : mesh_fail(err);
}

int tg_mesh_write_grid_nodes(const tg_mesh* m, const char* path, int32_t binary, const float* phi) {
    if (!m || !path) return mesh_fail("tg_mesh_write_grid_nodes: null argument");
    const size_t n = m->type.size();
    NodeFile nf;
    nf.xyz = m->xyz;
    nf.id.assign(m->type.begin(), m->type.end());
    nf.number.resize(n);
    for (size_t i = 0; i < n; i++) nf.number[i] = m->number.size() == n ? m->number[i] : (uint32_t)(i + 1);
    const float* p = phi ? phi : m->phi.data();
    nf.phi.assign(p, p + n);
    const std::string err = write_node_file(path, nf, binary != 0);
    return err.empty() ? TG_OK : mesh_fail(err);
}

int tg_mesh_write_config(const tg_mesh* m, const char* path) {
    if (!m || !path) return mesh_fail("tg_mesh_write_config: null argument");
    const std::string err = write_config_ascii(path, m->config);
    return err.empty() ? TG_OK : mesh_fail(err);
}

uint32_t tg_mesh_dump_index(const tg_mesh* m) { return m ? m->dump_index : 0u; }

int tg_mesh_numbers(const tg_mesh* m, uint32_t* out) {
    if (!m || !out) return mesh_fail("tg_mesh_numbers: null argument");
    const size_t n = m->type.size();
    for (size_t i = 0; i < n; i++) out[i] = m->number.size() == n ? m->number[i] : (uint32_t)(i + 1);
    return TG_OK;
}

int tg_results_write(const char* path, int32_t binary, const char* header, int32_t count, const tg_result_row* rows,
                     int32_t chunk) {
    if (!path || count < 0 || (count && !rows) || chunk < 0) return mesh_fail("tg_results_write: bad argument");
    std::vector<ResultRecord> recs(count);
    for (int32_t k = 0; k < count; k++) {
        const tg_result_row& a = rows[k];
        ResultRecord& r = recs[k];
        r.index = a.index;
        r.id = (short)a.id;
        r.number = a.number;
        r.voltage = a.voltage;
        for (int j = 0; j < 3; j++) {
            r.start[j] = a.start[j];
            r.stop[j] = a.stop[j];
            r.field_before[j] = a.field_before[j];
            r.field_after[j] = a.field_after[j];
            r.normal[j] = a.normal[j];
            r.apex[j] = a.apex[j];
        }
        r.tof = a.tof;
        r.probability = a.probability;
        r.phi_before = a.potential_before;
        r.phi_after = a.potential_after;
    }
    const std::string err = write_results(path, recs, binary != 0, header ? header : "", chunk);
    return err.empty() ? TG_OK : mesh_fail(err);
}

int tg_trajectory_write(const char* path, int32_t binary, int32_t count, const tg_trajectory_item* items,
                        int32_t chunk) {
    if (!path || count < 0 || (count && !items) || chunk < 0) return mesh_fail("tg_trajectory_write: bad argument");
    std::vector<TrajectoryRecord> recs(count);
    for (int32_t k = 0; k < count; k++) {
        const tg_trajectory_item& a = items[k];
        if (a.num_points < 0 || (a.num_points && !a.points)) return mesh_fail("tg_trajectory_write: bad points");
        TrajectoryRecord& t = recs[k];
        t.index = a.index;
        t.number = a.number;
        t.time_scale = a.time_scale;
        t.status = a.status;
        t.charge = a.charge;
        t.mass = a.mass;
        t.num_points = a.num_points;
        t.points = reinterpret_cast<const float*>(a.points);
        for (int j = 0; j < 6; j++) t.error[j] = a.error[j];
    }
    const std::string err = write_trajectories(path, recs, binary != 0, chunk);
    return err.empty() ? TG_OK : mesh_fail(err);
}

int tg_grid_log_write(const char* path, int32_t binary, int32_t n, const int32_t* id, const uint32_t* number,
                      const float* phi, const float* field, const float* force) {
    if (!path || n < 0 || (n && (!id || !number || !phi || !field || !force)))
        return mesh_fail("tg_grid_log_write: bad argument");
    GridLog g{n, id, number, phi, field, force};
    const std::string err = write_grid_log(path, binary != 0, g);
    return err.empty() ? TG_OK : mesh_fail(err);
}

int tg_surface_log_write(const char* path, int32_t binary, int32_t nCells, const int32_t* cells, const int32_t* type,
                         const uint32_t* number, const float* probability, const int32_t* neighbourPtr,
                         const int32_t* neighbours, int32_t nNodes, const int32_t* nodes, const float* phi,
                         const float* field, const float* normal) {
    if (!path || nCells < 0 || nNodes < 0 || (nCells && (!cells || !type || !number || !probability)) ||
        (nNodes && (!nodes || !phi || !field || !normal)) || (neighbourPtr && nCells && !neighbours &&
                                                               neighbourPtr[nCells] > 0))
        return mesh_fail("tg_surface_log_write: bad argument");
    SurfaceLog sl{nCells, cells, type, number, probability, neighbourPtr, neighbours, nNodes, nodes, phi, field, normal};
    const std::string err = write_surface_log(path, binary != 0, sl);
    return err.empty() ? TG_OK : mesh_fail(err);
}

int tg_mesh_write_dump(const tg_mesh* m, const char* path, const float* phi) {
    if (!m || !path) return mesh_fail("tg_mesh_write_dump: null argument");
    Dump d;
    d.last_index = m->dump_index;  // File_Io::writeSystem with the index read (tapsim.cpp:141-145)
    d.config = m->config;
    const int n = (int)m->type.size();
    for (int k = 0; k < 3; k++) {
        d.min[k] = 1e30f;
        d.max[k] = -1e30f;
    }
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            d.min[k] = std::min(d.min[k], m->xyz[3 * i + k]);
            d.max[k] = std::max(d.max[k], m->xyz[3 * i + k]);
        }
    for (int k = 0; k < 3; k++) {
        d.cmin[k] = d.min[k];
        d.cmax[k] = d.max[k];
    }
    d.xyz = m->xyz;
    d.hull = m->hull;
    d.node_tet = m->node_tet;
    d.tet_v = m->tet_v;
    d.tet_n = m->tet_n;
    d.id.assign(m->type.begin(), m->type.end());
    d.number = m->number;
    if (d.number.size() != (size_t)n) {
        d.number.resize(n);
        for (int i = 0; i < n; i++) d.number[i] = i + 1;
    }
    d.phi0.resize(n);
    for (int i = 0; i < n; i++) d.phi0[i] = phi ? phi[i] : m->phi[i];
    d.phi1 = d.phi0;
    d.charge.assign(n, 0.0f);
    d.boundary.resize(n);
    d.dirichlet.resize(n);
    d.neumann.resize(n);
    for (int i = 0; i < n; i++) {
        const CellType& t = m->config.types.at(m->type[i]);
        d.boundary[i] = m->hull.empty() ? 0 : m->hull[i];
        d.dirichlet[i] = t.dirichlet;
        d.neumann[i] = t.neumann;
        if (!m->volume.empty()) d.charge[i] = (float)(m->volume[i] * t.charge_density / 8.85418781762e-12);
    }
    d.row_ptr = m->row_ptr;
    d.col = m->col;
    d.coupling.assign(m->coupling.begin(), m->coupling.end());
    const std::string err = write_dump(path, d);
    return err.empty() ? TG_OK : mesh_fail(err);
}

}  // extern "C"

// tapsim_b200: the evaporation loop of TAPSim (Process::evaporation,
// tapsim/process.cpp:441-1124) as a C++ host program over the C ABI of
// libtapsim_b200.so (include/tapsim_gpu.h).  The device runs steps I-VI of
// every event (choice, removal, relaxation, fields, flight); this host keeps
// the voltage queue and time scale (process.cpp:985-1036) in float, as the
// reference does, and writes the results file with LogResults' layout.
//
// Command line, as the reference's (commands.cpp:55-841):
//   tapsim_b200 make-ini [filename]
//   tapsim_b200 [options] relaxation iconfig inode [onode]
//   tapsim_b200 [options] relaxation --read-dump=? oconfig onode
//     (--write-dump=?, --threshold=?, --cycle-size=?, --queue-size=?,
//     --init-potentials / --reset-potentials)
//   tapsim_b200 [options] evaporation iconfig inode [results]
//   tapsim_b200 [options] evaporation --input-dump=? iconfig [results]
//   tapsim_b200 [options] resumption idump [results]
//   tapsim_b200 [options] meshgen isample onodes   (meshgen's role,
//     meshgen/meshgen.cpp:2506-3986: graded vacuum and the marked box around
//     the sample node file; --create-config-template=? writes meshgen's
//     configuration template, --box-half-width=?, --box-height=?,
//     --fine-shell=? [m] size the box, --write-ascii the node file)
// Options taken from the reference: --ini-file=?, --threads=?, --write-ascii,
// --write-binary, --no-file-output, --skip-relaxation, --init-potentials,
// --reset-potentials, --threshold=?, --cycle-size=?, --queue-size=? (the
// initial relaxation), --event-limit=?, --last-event=?, --shrink-limit=?,
// --voltage-queue-size=? (--voltage-queue-limit=?), --vacuum-identifier=?,
// --no-chunks, --chunk-size=?, --trajectory-error-threshold=?,
// --evap-threshold=?, --evap-shell-size=?, --evap-cycle-size=?,
// --evap-queue-size=?, --evap-global-cycles=?, --refresh-interval=?,
// --refresh-threshold=?, --refresh-cycle-size=?, --refresh-queue-size=?;
// --no-trajectories, --no-grids, --no-surfaces and --no-dump are accepted
// (this program writes the results file only), and the options that ask
// for those files are refused.
// Options of this build: --relax-mode=solve|reference (solve: every event
// relaxed to --rel-tol, 1e-8; reference: the ini's local/global/refresh
// sweeps), --warm-start=0|1, --batch=? (events per library call),
// --records=? (every event's record as the library returned it, raw).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../../include/tapsim_gpu.h"

namespace {

// The initialization file's keys and defaults in makeIniList's order
// (commands.cpp:1249-1325), an empty key for each blank line; make-ini
// writes them out, and every key a run reads defaults to them.
const std::vector<std::pair<const char*, const char*>> kIniList = {
    {"RESULTS_FILENAME", "results_data"}, {"RESULTS_BINARY_OUTPUT", "0"}, {"RESULTS_CHUNK_SIZE", "10000"}, {"", ""},
    {"TRAJECTORY_FILENAME", "trajectory_data"}, {"TRAJECTORY_BINARY_OUTPUT", "1"}, {"TRAJECTORY_CHUNK_SIZE", "10000"},
    {"", ""},
    {"GRID_FILENAME", "grid_data"}, {"GRID_BINARY_OUTPUT", "1"}, {"GRID_INTERVAL", "2147483647"}, {"", ""},
    {"SURFACE_FILENAME", "surface_data"}, {"SURFACE_BINARY_OUTPUT", "1"}, {"SURFACE_INTERVAL", "2147483647"}, {"", ""},
    {"GEOMETRY_FILENAME", "geometry.dat"}, {"GEOMETRY_BINARY_OUTPUT", "1"}, {"GEOMETRY_CONTENTS", "0xff"}, {"", ""},
    {"DUMP_FILENAME", "dump"}, {"DUMP_INTERVAL", "10000"}, {"", ""},
    {"OUTPUT_DELAY_TIME", "60"}, {"", ""},
    {"METHOD_EVAPORATION_PROBABILITY", "0"}, {"METHOD_EVAPORATION_CHOICE", "0"}, {"", ""},
    {"VACUUM_CELL_IDENTIFIER", "Vacuum"}, {"", ""},
    {"TRAJECTORY_INTEGRATOR_TYPE", "1"}, {"TRAJECTORY_STEPPER_TYPE", "1"}, {"TRAJECTORY_INITIAL_TIME_STEP", "1e-14"},
    {"TRAJECTORY_MINIMUM_TIME_STEP", "1e-16"}, {"TRAJECTORY_ERROR_THRESHOLD", "1e-6"},
    {"TRAJECTORY_NON_RANDOM_START_POSITION", "1"}, {"TRAJECTORY_NO_INITIAL_VELOCITY", "1"}, {"", ""},
    {"VOLTAGE_QUEUE_SIZE", "250"}, {"", ""},
    {"LOCAL_RELAXATION_ERROR_THRESHOLD", "1e-2"}, {"LOCAL_RELAXATION_SHELL_SIZE", "3"},
    {"LOCAL_RELAXATION_CYCLE_SIZE", "5"}, {"LOCAL_RELAXATION_QUEUE_SIZE", "5"}, {"GLOBAL_RELAXATION_STEPS", "1"},
    {"", ""},
    {"REFRESH_RELAXATION_INTERVAL", "0"}, {"REFRESH_RELAXATION_ERROR_THRESHOLD", "0.0"},
    {"REFRESH_RELAXATION_CYCLE_SIZE", "100"}, {"REFRESH_RELAXATION_QUEUE_SIZE", "25"}, {"", ""},
};
// the default initialization file (tapsim.cpp:64), read when present and
// no --ini-file is given (commands.cpp:1038-1044)
const char* kDefaultIni = "tapsim.ini";

struct Args {
    std::string command, config, nodes, dump, results, ini;
    int threads = 0;
    int binary = -1;          // -1: the ini's RESULTS_BINARY_OUTPUT
    bool fileOutput = true;
    bool skipRelaxation = false;
    long eventLimit = -1;     // -1: until the surface is empty
    int queueSize = -1;
    std::string vacuum;
    int chunkSize = -1;       // -1: the ini's; 0: one file
    bool relaxReference = false;
    double relTol = 1e-8;
    int warmStart = 0;
    int batch = 64;
    std::string records;      // --records: every event's tg_event_record, raw, in order
    std::string sample, configTemplate;  // meshgen
    std::string iniOut;                  // make-ini
    // relaxation (RelaxationCommands, commands.cpp:861-894)
    std::string readDump, writeDump, oconfig, onodes;
    // the initial relaxation of evaporation (Grid_3d::Table::relax), -1: the
    // ini's refresh parameters (commands.cpp:929-933); relaxation's own
    // defaults are 0, 100 and 25 (commands.cpp:876-894)
    float threshold = -1.0f;
    int cycleSize = -1, relaxQueue = -1;
    bool resetPotentials = false;
    std::map<std::string, std::string> iniOverrides;  // command-line values of ini keys
    long lastEvent = -1;       // resumption: the index before the first event (-1: the dump's)
    float shrinkLimit = -1.0f; // stop once the apex sank this far [m] (-1: never)
    double boxHalfWidth = -1.0, boxHeight = -1.0, fineShell = -1.0;
};

[[noreturn]] void die(const std::string& msg) {
    std::fprintf(stderr, "tapsim_b200: %s\n", msg.c_str());
    std::exit(1);
}

void check(int rc, const tg_handle* h, const char* what) {
    if (rc != TG_OK) die(std::string(what) + " failed (" + std::to_string(rc) + "): " + tg_last_error(h));
}

bool opt(const std::string& a, const char* name, std::string* value) {
    const std::string p = std::string("--") + name + "=";
    if (a.compare(0, p.size(), p) != 0) return false;
    *value = a.substr(p.size());
    return true;
}

Args parse(int argc, char** argv) {
    Args a;
    std::vector<std::string> pos;
    for (int k = 1; k < argc; k++) {
        const std::string s = argv[k];
        std::string v;
        if (opt(s, "ini-file", &v)) a.ini = v;
        else if (opt(s, "threads", &v)) a.threads = std::atoi(v.c_str());
        else if (s == "--write-ascii") a.binary = 0;
        else if (s == "--write-binary") a.binary = 1;
        else if (s == "--no-file-output") a.fileOutput = false;
        else if (s == "--skip-relaxation") a.skipRelaxation = true;
        else if (opt(s, "event-limit", &v)) a.eventLimit = std::atol(v.c_str());
        else if (opt(s, "voltage-queue-size", &v) || opt(s, "voltage-queue-limit", &v)) a.queueSize = std::atoi(v.c_str());
        else if (opt(s, "vacuum-identifier", &v)) a.vacuum = v;
        else if (s == "--no-chunks") a.chunkSize = 0;
        else if (opt(s, "chunk-size", &v)) a.chunkSize = std::atoi(v.c_str());
        else if (opt(s, "input-dump", &v)) a.dump = v;
        else if (opt(s, "relax-mode", &v)) {
            if (v != "solve" && v != "reference") die("--relax-mode is solve or reference");
            a.relaxReference = v == "reference";
        } else if (opt(s, "rel-tol", &v)) a.relTol = std::atof(v.c_str());
        else if (opt(s, "warm-start", &v)) a.warmStart = std::atoi(v.c_str());
        else if (opt(s, "batch", &v)) a.batch = std::max(1, std::atoi(v.c_str()));
        else if (opt(s, "records", &v)) a.records = v;
        else if (opt(s, "create-config-template", &v)) a.configTemplate = v;
        else if (opt(s, "box-half-width", &v)) a.boxHalfWidth = std::atof(v.c_str());
        else if (opt(s, "box-height", &v)) a.boxHeight = std::atof(v.c_str());
        else if (opt(s, "fine-shell", &v)) a.fineShell = std::atof(v.c_str());
        else if (opt(s, "read-dump", &v)) a.readDump = v;
        else if (opt(s, "write-dump", &v)) a.writeDump = v;
        else if (opt(s, "threshold", &v)) a.threshold = (float)std::atof(v.c_str());
        else if (opt(s, "cycle-size", &v)) a.cycleSize = std::atoi(v.c_str());
        else if (opt(s, "queue-size", &v)) a.relaxQueue = std::atoi(v.c_str());
        else if (s == "--init-potentials" || s == "--reset-potentials") a.resetPotentials = true;
        // evaporation and resumption (commands.cpp:280-841): ini values
        else if (opt(s, "evap-threshold", &v)) a.iniOverrides["LOCAL_RELAXATION_ERROR_THRESHOLD"] = v;
        else if (opt(s, "evap-shell-size", &v)) a.iniOverrides["LOCAL_RELAXATION_SHELL_SIZE"] = v;
        else if (opt(s, "evap-cycle-size", &v)) a.iniOverrides["LOCAL_RELAXATION_CYCLE_SIZE"] = v;
        else if (opt(s, "evap-queue-size", &v)) {
            // the reference's handler falls through into --evap-global-cycles
            // (commands.cpp:511-516), so the value sets both
            a.iniOverrides["LOCAL_RELAXATION_QUEUE_SIZE"] = v;
            a.iniOverrides["GLOBAL_RELAXATION_STEPS"] = v;
        } else if (opt(s, "evap-global-cycles", &v)) a.iniOverrides["GLOBAL_RELAXATION_STEPS"] = v;
        else if (opt(s, "refresh-interval", &v)) a.iniOverrides["REFRESH_RELAXATION_INTERVAL"] = v;
        else if (opt(s, "refresh-threshold", &v)) a.iniOverrides["REFRESH_RELAXATION_ERROR_THRESHOLD"] = v;
        else if (opt(s, "refresh-cycle-size", &v)) a.iniOverrides["REFRESH_RELAXATION_CYCLE_SIZE"] = v;
        else if (opt(s, "refresh-queue-size", &v)) a.iniOverrides["REFRESH_RELAXATION_QUEUE_SIZE"] = v;
        else if (opt(s, "trajectory-error-threshold", &v)) a.iniOverrides["TRAJECTORY_ERROR_THRESHOLD"] = v;
        else if (opt(s, "shrink-limit", &v)) a.shrinkLimit = (float)std::atof(v.c_str());
        else if (opt(s, "last-event", &v)) a.lastEvent = std::atol(v.c_str());
        // outputs this program does not write: asking for none is accepted
        else if (s == "--no-trajectories" || s == "--no-grids" || s == "--no-surfaces" || s == "--no-dump") {
        } else if (opt(s, "write-trajectories", &v) || opt(s, "write-grids", &v) || opt(s, "write-surfaces", &v) ||
                   opt(s, "snapshot-interval", &v) || opt(s, "dump-interval", &v)) {
            die("\"" + s + "\": tapsim_b200 writes the results file only (the Python host's Evaporation writes "
                "trajectories and grid and surface snapshots)");
        }
        else if (s.compare(0, 2, "--") == 0) die("unknown or invalid argument in command line: \"" + s + "\"");
        else pos.push_back(s);
    }
    if (pos.empty()) die("usage: tapsim_b200 [options] make-ini|relaxation|evaporation|resumption|meshgen ...");
    a.command = pos[0];
    if (a.command == "evaporation") {
        if (!a.dump.empty()) {
            if (pos.size() < 2) die("missing arguments for processing in 'evaporation'-mode");
            a.config = pos[1];
            if (pos.size() > 2) a.results = pos[2];
        } else {
            if (pos.size() < 3) die("missing arguments for processing in 'evaporation'-mode");
            a.config = pos[1];
            a.nodes = pos[2];
            if (pos.size() > 3) a.results = pos[3];
        }
    } else if (a.command == "resumption") {
        if (pos.size() < 2) die("missing arguments for processing in 'resumption'-mode");
        a.dump = pos[1];
        if (pos.size() > 2) a.results = pos[2];
    } else if (a.command == "make-ini") {
        // make-ini [filename] (commands.cpp:55-140)
        if (pos.size() > 2) die("missing arguments for processing in 'make-ini'-mode");
        a.iniOut = pos.size() > 1 ? pos[1] : kDefaultIni;
    } else if (a.command == "relaxation") {
        // relaxation iconfig inode [onode] | --read-dump=? oconfig onode
        // (commands.cpp:142-277; iconfig inode alone writes the relaxed
        // nodes over inode, as the reference does)
        if (!a.readDump.empty()) {
            if (pos.size() != 3) die("missing arguments for processing in 'relaxation'-mode");
            a.oconfig = pos[1];
            a.onodes = pos[2];
        } else {
            if (pos.size() != 3 && pos.size() != 4) die("missing arguments for processing in 'relaxation'-mode");
            a.config = pos[1];
            a.nodes = pos[2];
            a.onodes = pos.size() == 4 ? pos[3] : pos[2];
        }
    } else if (a.command == "meshgen") {
        if (pos.size() < 3) die("missing arguments for 'meshgen': isample onodes");
        a.sample = pos[1];
        a.nodes = pos[2];
    } else {
        die("unknown command " + a.command);
    }
    return a;
}

std::map<std::string, std::string> read_ini(const std::string& path) {
    std::map<std::string, std::string> ini;
    for (const auto& kv : kIniList)
        if (kv.first[0]) ini[kv.first] = kv.second;
    if (path.empty()) return ini;
    std::ifstream f(path);
    if (!f) die("cannot read ini file " + path);
    std::string line;
    while (std::getline(f, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        auto trim = [](std::string s) {
            const size_t b = s.find_first_not_of(" \t\r"), e = s.find_last_not_of(" \t\r");
            return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
        };
        ini[trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
    return ini;
}

// MathVector3d<float>::length() in float
float length3(const float v[3]) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

}  // namespace

// meshgen's role: the sample's vacuum mesh, written as a node file (binary
// unless --write-ascii, as meshgen's ASCII_OUTPUT_MODE 0) and, with
// --create-config-template, the configuration template beside it
int meshgen(const Args& a) {
    tg_sample_params p;
    tg_sample_params_default(&p);
    if (a.boxHalfWidth > 0.0) p.box_half_width = a.boxHalfWidth;
    if (a.boxHeight > 0.0) p.box_height = a.boxHeight;
    if (a.fineShell > 0.0) p.fine_shell = a.fineShell;
    tg_mesh* mesh = nullptr;
    check(tg_mesh_from_sample(a.sample.c_str(), nullptr, &p, a.threads, &mesh), nullptr, "meshing the sample");
    check(tg_mesh_write_node_file(mesh, a.nodes.c_str(), a.binary == 0 ? 0 : 1), nullptr, "writing the node file");
    if (!a.configTemplate.empty())
        check(tg_mesh_write_config(mesh, a.configTemplate.c_str()), nullptr, "writing the configuration template");
    tg_mesh_desc desc;
    int32_t nnz = 0;
    check(tg_mesh_describe(mesh, &desc, &nnz), nullptr, "tg_mesh_describe");
    std::printf("meshgen: %d nodes, %d couplings, %d tetrahedra\n", desc.num_nodes, nnz, desc.num_tets);
    tg_mesh_destroy(mesh);
    return 0;
}

// make-ini (doMakeIni, tapsim.cpp:66-85): the default initialization file,
// as File_Io::writeInitialization lays it out (file_io.cpp:96-112)
int make_ini(const Args& a) {
    std::ofstream f(a.iniOut, std::ios::trunc);
    if (!f) die("cannot write " + a.iniOut);
    for (const auto& kv : kIniList) {
        if (kv.first[0]) f << kv.first << " = " << kv.second;
        f << '\n';
    }
    if (!f) die("cannot write " + a.iniOut);
    std::printf("make-ini: default initialization file \"%s\"\n", a.iniOut.c_str());
    return 0;
}

// Grid_3d::Table::randomReset (grid_3d.cpp:811-848): free cells uniform in
// [min, max] of the types' potentials, in float, from the stream main()
// seeds with srand(99) (tapsim.cpp:235); Dirichlet cells at their type's
void random_reset(tg_handle* h, const tg_mesh_desc& desc) {
    const int n = desc.num_nodes;
    std::map<int, const tg_type*> types;
    for (int k = 0; k < desc.num_types; k++) types[desc.types[k].id] = &desc.types[k];
    if (types.empty()) die("the configuration has no cell types");
    float minPhi = types.begin()->second->phi, maxPhi = minPhi;
    for (const auto& kv : types) {
        minPhi = std::min(minPhi, kv.second->phi);
        maxPhi = std::max(maxPhi, kv.second->phi);
    }
    std::srand(99);
    std::vector<double> phi(n);
    for (int i = 0; i < n; i++) {
        const auto t = types.find(desc.type_id[i]);
        if (t == types.end()) die("a node of an unknown cell type");
        float p;
        if (t->second->dirichlet) {
            p = t->second->phi;
        } else {
            p = (float)std::rand();
            p /= (float)RAND_MAX;
            p *= maxPhi - minPhi;
            p += minPhi;
        }
        phi[i] = p;
    }
    check(tg_set_phi(h, phi.data()), h, "tg_set_phi");
    std::printf("potential values are reset\n");
}

// relaxation (doRelaxation, tapsim.cpp:87-148): the system from a dump or a
// configuration and node file, its potentials reset at random on request,
// relaxed, then the configuration (with --read-dump), the node file with
// numbers and potentials, and a dump (--write-dump) written.  --relax-mode
// as for evaporation: solve (default) relaxes to --rel-tol; reference runs
// Grid_3d::Table::relax(threshold, cycle, queue) (Process::relaxation,
// process.cpp:133-157), whose stagnation fault ends it without an error.
int relaxation(const Args& a) {
    tg_mesh* mesh = nullptr;
    if (!a.readDump.empty()) check(tg_mesh_from_dump(a.readDump.c_str(), nullptr, &mesh), nullptr, "reading the dump");
    else check(tg_mesh_from_files(a.nodes.c_str(), a.config.c_str(), a.threads, &mesh), nullptr, "reading the mesh");
    tg_mesh_desc desc;
    int32_t nnz = 0;
    check(tg_mesh_describe(mesh, &desc, &nnz), nullptr, "tg_mesh_describe");
    const int n = desc.num_nodes;
    tg_handle* h = nullptr;
    check(tg_create(&desc, &h), nullptr, "tg_create");
    if (a.resetPotentials) random_reset(h, desc);
    if (a.relaxReference) {
        int64_t it = 0;
        double dev = 0.0;
        const int rc = tg_relax_threshold(h, a.threshold >= 0.0f ? a.threshold : 0.0f, a.cycleSize >= 0 ? a.cycleSize : 100,
                                          a.relaxQueue >= 0 ? a.relaxQueue : 25, 2000000, &it, &dev);
        if (rc == TG_ERR_RELAX_FAULT || rc == TG_ERR_ITERATION_CAP)
            std::printf("relaxation: numerical limit reached after %lld steps (deviation = %g)\n", (long long)it, dev);
        else check(rc, h, "relaxation");
        if (rc == TG_OK) std::printf("relaxation: %lld steps, deviation %g\n", (long long)it, dev);
    } else {
        tg_solve_opts so{};
        so.rel_tol = a.relTol;
        so.max_outer = 50;
        so.max_inner = 20000;
        so.inner_rtol = 1e-4;
        so.warm_start = 0;
        so.preconditioner = 1;
        tg_solve_info info;
        check(tg_solve(h, &so, &info), h, "relaxation");
        std::printf("relaxation: relative residual %.3e after %d outer steps\n", info.rel_residual, info.outer);
    }
    std::vector<double> phi64(n);
    check(tg_get_phi(h, phi64.data()), h, "tg_get_phi");
    std::vector<float> phi(n);
    for (int i = 0; i < n; i++) phi[i] = (float)phi64[i];
    if (!a.oconfig.empty()) check(tg_mesh_write_config(mesh, a.oconfig.c_str()), nullptr, "writing the configuration");
    if (!a.onodes.empty())
        check(tg_mesh_write_grid_nodes(mesh, a.onodes.c_str(), 0, phi.data()), nullptr, "writing the node file");
    if (!a.writeDump.empty()) check(tg_mesh_write_dump(mesh, a.writeDump.c_str(), phi.data()), nullptr, "writing the dump");
    tg_destroy(h);
    tg_mesh_destroy(mesh);
    return 0;
}

int main(int argc, char** argv) {
    Args a = parse(argc, argv);
    if (a.command == "meshgen") return meshgen(a);
    if (a.command == "make-ini") return make_ini(a);
    if (a.command == "relaxation") return relaxation(a);
    if (a.ini.empty() && std::ifstream(kDefaultIni).good()) a.ini = kDefaultIni;
    if (!a.writeDump.empty()) die("--write-dump: tapsim_b200 writes no dumps during an evaporation");
    std::map<std::string, std::string> ini = read_ini(a.ini);
    for (const auto& kv : a.iniOverrides) ini[kv.first] = kv.second;
    auto I = [&](const char* k) { return std::atoi(ini.at(k).c_str()); };
    auto F = [&](const char* k) { return std::atof(ini.at(k).c_str()); };

    // Process::initialization / readSystem: the mesh with its couplings
    tg_mesh* mesh = nullptr;
    int rc;
    if (!a.dump.empty()) rc = tg_mesh_from_dump(a.dump.c_str(), a.config.empty() ? nullptr : a.config.c_str(), &mesh);
    else rc = tg_mesh_from_files(a.nodes.c_str(), a.config.c_str(), a.threads, &mesh);
    check(rc, nullptr, "reading the mesh");
    tg_mesh_desc desc;
    int32_t nnz = 0;
    check(tg_mesh_describe(mesh, &desc, &nnz), nullptr, "tg_mesh_describe");
    const int n = desc.num_nodes;
    std::vector<uint32_t> numbers(n);
    check(tg_mesh_numbers(mesh, numbers.data()), nullptr, "tg_mesh_numbers");
    const std::string vacuumName = a.vacuum.empty() ? ini.at("VACUUM_CELL_IDENTIFIER") : a.vacuum;
    const int vacuumId = tg_mesh_type_id(mesh, vacuumName.c_str());
    if (vacuumId < 0) die("no cell type named " + vacuumName + " in the configuration");
    std::map<int, tg_type> types;
    for (int k = 0; k < desc.num_types; k++) types[desc.types[k].id] = desc.types[k];
    // the index before the first event: 0 for an evaporation, the dump's
    // (or --last-event) for a resumption (tapsim.cpp:206-225)
    const long initEvent = a.command == "resumption" ? (a.lastEvent >= 0 ? a.lastEvent : (long)tg_mesh_dump_index(mesh)) : 0;
    tg_handle* h = nullptr;
    check(tg_create(&desc, &h), nullptr, "tg_create");
    if (a.resetPotentials) random_reset(h, desc);

    tg_solve_opts solve{};
    solve.rel_tol = a.relTol;
    solve.max_outer = 50;
    solve.max_inner = 20000;
    solve.inner_rtol = 1e-4;
    solve.warm_start = a.warmStart;
    solve.preconditioner = 1;
    // initial relaxation (Process::relaxation with the refresh parameters,
    // commands.cpp:931-933), unless --skip-relaxation
    if (!a.skipRelaxation) {
        if (a.relaxReference) {
            int64_t it = 0;
            double dev = 0.0;
            rc = tg_relax_threshold(h, a.threshold >= 0.0f ? a.threshold : F("REFRESH_RELAXATION_ERROR_THRESHOLD"),
                                    a.cycleSize >= 0 ? a.cycleSize : I("REFRESH_RELAXATION_CYCLE_SIZE"),
                                    a.relaxQueue >= 0 ? a.relaxQueue : I("REFRESH_RELAXATION_QUEUE_SIZE"), 2000000,
                                    &it, &dev);
            if (rc != TG_OK && rc != TG_ERR_RELAX_FAULT && rc != TG_ERR_ITERATION_CAP) check(rc, h, "relaxation");
        } else {
            tg_solve_opts s0 = solve;
            s0.warm_start = 0;
            tg_solve_info info;
            check(tg_solve(h, &s0, &info), h, "relaxation");
        }
    }

    tg_event_opts o{};
    o.vacuum_id = vacuumId;
    o.relax_mode = a.relaxReference ? 0 : 1;
    o.local_threshold = F("LOCAL_RELAXATION_ERROR_THRESHOLD");
    o.local_shell = I("LOCAL_RELAXATION_SHELL_SIZE");
    o.local_cycle = I("LOCAL_RELAXATION_CYCLE_SIZE");
    o.local_queue = I("LOCAL_RELAXATION_QUEUE_SIZE");
    o.global_steps = I("GLOBAL_RELAXATION_STEPS");
    o.refresh_interval = I("REFRESH_RELAXATION_INTERVAL");
    o.refresh_threshold = F("REFRESH_RELAXATION_ERROR_THRESHOLD");
    o.refresh_cycle = I("REFRESH_RELAXATION_CYCLE_SIZE");
    o.refresh_queue = I("REFRESH_RELAXATION_QUEUE_SIZE");
    o.refresh_max_sweeps = 2000000;
    o.solve = solve;
    o.trace.time_step = F("TRAJECTORY_INITIAL_TIME_STEP");
    o.trace.min_time_step = F("TRAJECTORY_MINIMUM_TIME_STEP");
    o.trace.error_threshold = F("TRAJECTORY_ERROR_THRESHOLD");
    o.trace.max_steps = 100000;
    o.trace.stepper_limit = 200;
    o.trace.walk_limit = 100000;
    o.trace.integrator = I("TRAJECTORY_INTEGRATOR_TYPE");
    o.trace.stepper = I("TRAJECTORY_STEPPER_TYPE");
    o.trace_enabled = 1;
    o.normal_enabled = 1;
    o.prob_mode = I("METHOD_EVAPORATION_PROBABILITY");
    o.choice_mode = I("METHOD_EVAPORATION_CHOICE");
    o.temperature = tg_mesh_temperature(mesh);
    o.rng_seed = 99;  // std::srand(99) in main (tapsim.cpp:235)
    o.initial_velocity = I("TRAJECTORY_NO_INITIAL_VELOCITY") ? 0 : 1;

    // steps I-VI on the device, VI (voltage, time scale) and VII (results)
    // here, one batch of events per library call
    const size_t queueSize = a.queueSize >= 0 ? (size_t)a.queueSize : (size_t)I("VOLTAGE_QUEUE_SIZE");
    std::deque<float> voltageQueue;
    float voltageQueueSum = 0.0f;
    std::vector<tg_result_row> rows;
    std::vector<tg_event_record> recs((size_t)a.batch);
    FILE* rawOut = a.records.empty() ? nullptr : std::fopen(a.records.c_str(), "wb");
    if (!a.records.empty() && !rawOut) die("cannot write " + a.records);
    long events = 0;
    float initApexZ = 0.0f;
    bool shrunk = false;
    for (;;) {
        long want = a.batch;
        if (a.eventLimit >= 0) want = std::min<long>(want, a.eventLimit - events);
        if (want <= 0) break;
        int32_t done = 0;
        // the refresh schedule tests (initial index + event index) % interval
        // (process.cpp:876), the event index counting on from the initial one
        rc = tg_run_events(h, &o, (int32_t)(initEvent + initEvent + events + 1), (int32_t)want, recs.data(), &done);
        if (rc != TG_OK && rc != TG_ERR_NO_SURFACE) check(rc, h, "tg_run_events");
        for (int k = 0; k < done; k++) {
            const tg_event_record& r = recs[k];
            const tg_type& t = types.at(r.type_id);
            float voltage, timeScale;
            const float fb = length3(r.field_before);
            if (r.impact.last_tet >= 0 && fb != 0.0f) {
                float v = r.phi_before;
                v -= r.impact.last_phi;
                v *= t.evap_field;
                v /= fb;
                v /= r.scaling_reference;
                voltageQueue.push_back(v);
                voltageQueueSum += v;
                while (voltageQueue.size() > queueSize) {
                    voltageQueueSum -= voltageQueue.front();
                    voltageQueue.pop_front();
                }
                voltage = voltageQueueSum / voltageQueue.size();
                timeScale = r.phi_after;
                timeScale -= r.impact.last_phi;
                timeScale /= voltage;
                timeScale = std::sqrt(timeScale);
            } else {
                voltage = fb == 0.0f ? 1.0f : 0.0f;
                timeScale = 1.0f;
            }
            tg_result_row row{};
            row.index = (uint32_t)(initEvent + events + k + 1);
            row.id = r.type_id;
            row.number = numbers[r.node];
            row.voltage = voltage;
            for (int c = 0; c < 3; c++) {
                row.start[c] = desc.xyz[3 * (size_t)r.node + c];
                row.stop[c] = r.impact.stop[c];
                row.field_before[c] = r.field_before[c];
                row.field_after[c] = r.field_after[c];
                row.normal[c] = r.normal[c];
                row.apex[c] = r.apex[c];
            }
            row.tof = r.impact.stop_time * timeScale;
            row.probability = r.probability;
            row.potential_before = r.phi_before;
            row.potential_after = r.phi_after;
            rows.push_back(row);
            if (events + k == 0) initApexZ = r.apex[2];
            // --shrink-limit: the run ends after the event whose apex lies
            // that far below the first one's (process.cpp:1108)
            if (a.shrinkLimit >= 0.0f && initApexZ - r.apex[2] >= a.shrinkLimit) {
                shrunk = true;
                done = k + 1;
                break;
            }
        }
        if (rawOut && done > 0) std::fwrite(recs.data(), sizeof(tg_event_record), (size_t)done, rawOut);
        events += done;
        if (shrunk || done < want) break;  // shrunk, or the surface ran out
    }
    if (rawOut) std::fclose(rawOut);
    std::printf("events %ld\n", events);
    if (a.fileOutput) {
        const std::string path = a.results.empty() ? ini.at("RESULTS_FILENAME") : a.results;
        const int binary = a.binary >= 0 ? a.binary : I("RESULTS_BINARY_OUTPUT");
        const int chunk = a.chunkSize >= 0 ? a.chunkSize : I("RESULTS_CHUNK_SIZE");
        if (!path.empty())
            check(tg_results_write(path.c_str(), binary, nullptr, (int32_t)rows.size(), rows.data(), chunk), nullptr,
                  "tg_results_write");
    }
    tg_destroy(h);
    tg_mesh_destroy(mesh);
    return 0;
}

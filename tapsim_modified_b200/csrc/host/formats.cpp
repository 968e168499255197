#include "formats.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>

namespace tg_host {
namespace {

std::string trim(const std::string& s) {
    const char* ws = " \t\n\r";
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return std::string();
    const size_t b = s.find_last_not_of(ws);
    return s.substr(a, b - a + 1);
}

template <class T>
bool rd(std::istream& is, T* v) {
    is.read(reinterpret_cast<char*>(v), sizeof(T));
    return (bool)is;
}
template <class T>
void wr(std::ostream& os, const T& v) {
    os.write(reinterpret_cast<const char*>(&v), sizeof(T));
}
bool rd_cstr(std::istream& is, std::string* s) {
    s->clear();
    char c;
    while (is.get(c)) {
        if (c == '\0') return true;
        s->push_back(c);
    }
    return false;
}

const char* kConfigKeys[13] = {"TEMPERATURE", "ID", "NAME", "CHARGE_DENSITY", "DIELECTRICITY", "REMOVABLE",
                               "NEUMANN_BOUNDARY", "DIRICHLET_BOUNDARY", "POTENTIAL", "MASS",
                               "EVAPORATION_CHARGE_STATE", "EVAPORATION_FIELD_STRENGTH",
                               "EVAPORATION_ACTIVATION_ENERGY"};

template <class T>
bool parse(const std::string& s, T* v) {
    std::istringstream is(s);
    is >> *v;
    return !is.fail();
}

}  // namespace

int ConfigTable::id_of(const std::string& name) const {
    for (const auto& kv : types)
        if (kv.second.name == name) return kv.first;
    return -1;
}

std::string read_node_file(const std::string& path, NodeFile* out) {
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) return "node file: cannot open " + path;
    std::string header;
    do {
        if (!std::getline(f, header)) return "node file: missing header";
    } while (header.empty() || header[0] == '#');
    bool ascii;
    if (header.compare(0, 5, "ASCII") == 0) { ascii = true; header = header.substr(5); }
    else if (header.compare(0, 6, "BINARY") == 0) { ascii = false; header = header.substr(6); }
    else return "node file: unknown mode";
    long n = 0;
    int withNumbers = 0, withPotentials = 0;
    {
        std::istringstream hs(header);
        hs >> n >> withNumbers >> withPotentials;
        if (hs.fail() || n < 0) return "node file: bad header";
    }
    out->xyz.assign(3 * n, 0.0f);
    out->id.assign(n, -1);
    out->number.assign(n, 0);
    out->has_numbers = withNumbers != 0;
    out->phi.assign(withPotentials ? n : 0, 0.0f);
    for (long i = 0; i < n; i++) {
        if (ascii) {
            std::string line;
            do {
                if (!std::getline(f, line)) return "node file: truncated";
            } while (!line.empty() && line[0] == '#');
            std::vector<std::string> v;
            std::istringstream ls(line);
            std::string tok;
            while (std::getline(ls, tok, '\t')) v.push_back(tok);
            const size_t need = 4 + (withNumbers ? 1 : 0) + (withPotentials ? 1 : 0);
            if (v.size() < need) return "node file: short line";
            for (int k = 0; k < 3; k++)
                if (!parse(v[k], &out->xyz[3 * i + k])) return "node file: bad coordinate";
            if (!parse(v[3], &out->id[i])) return "node file: bad id";
            size_t c = 4;
            if (withNumbers && !parse(v[c++], &out->number[i])) return "node file: bad number";
            if (withPotentials && !parse(v[c++], &out->phi[i])) return "node file: bad potential";
        } else {
            if (!rd(f, &out->xyz[3 * i]) || !rd(f, &out->xyz[3 * i + 1]) || !rd(f, &out->xyz[3 * i + 2]) ||
                !rd(f, &out->id[i]))
                return "node file: truncated";
            if (withNumbers && !rd(f, &out->number[i])) return "node file: truncated";
            if (withPotentials && !rd(f, &out->phi[i])) return "node file: truncated";
        }
    }
    // unique numbering (file_io.cpp:975-1000)
    std::set<uint32_t> seen;
    uint32_t next = 1;
    for (long i = 0; i < n; i++) {
        if (out->number[i] == 0) continue;
        if (!seen.insert(out->number[i]).second) return "node file: non unique numbering";
        if (out->number[i] >= next) next = out->number[i] + 1;
    }
    for (long i = 0; i < n; i++)
        if (out->number[i] == 0) out->number[i] = next++;
    return std::string();
}

std::string write_node_file(const std::string& path, const NodeFile& nf, bool binary) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.good()) return "node file: cannot write " + path;
    const long n = (long)nf.id.size();
    const int withNumbers = nf.number.empty() ? 0 : 1;
    const int withPotentials = nf.phi.empty() ? 0 : 1;
    if (binary) {
        f << "BINARY " << n << " " << withNumbers << " " << withPotentials << '\n';
        for (long i = 0; i < n; i++) {
            wr(f, nf.xyz[3 * i]);
            wr(f, nf.xyz[3 * i + 1]);
            wr(f, nf.xyz[3 * i + 2]);
            wr(f, nf.id[i]);
            if (withNumbers) wr(f, nf.number[i]);
            if (withPotentials) wr(f, nf.phi[i]);
        }
    } else {
        f << "ASCII " << n << " " << withNumbers << " " << withPotentials << '\n';
        char buf[256];
        for (long i = 0; i < n; i++) {
            int len = snprintf(buf, sizeof(buf), "%.8e\t%.8e\t%.8e\t%d", (double)nf.xyz[3 * i], (double)nf.xyz[3 * i + 1],
                               (double)nf.xyz[3 * i + 2], (int)nf.id[i]);
            f.write(buf, len);
            if (withNumbers) { len = snprintf(buf, sizeof(buf), "\t%u", nf.number[i]); f.write(buf, len); }
            if (withPotentials) { len = snprintf(buf, sizeof(buf), "\t%.8e", (double)nf.phi[i]); f.write(buf, len); }
            f << '\n';
        }
    }
    return f.good() ? std::string() : "node file: write error";
}

std::string read_config(const std::string& path, ConfigTable* out) {
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) return "config: cannot open " + path;
    out->types.clear();
    out->temperature = 0.0f;
    std::string first;
    do {
        if (!std::getline(f, first)) return "config: empty";
    } while (first.empty() || first[0] == '#');
    first = trim(first);
    if (first == "BINARY") {
        int size = 0;
        if (!rd(f, &out->temperature) || !rd(f, &size)) return "config: truncated";
        for (int i = 0; i < size; i++) {
            CellType t;
            char id;
            bool b;
            if (!rd(f, &id) || !rd_cstr(f, &t.name)) return "config: truncated";
            t.id = id;
            rd(f, &t.charge_density);
            rd(f, &t.epsilon);
            rd(f, &b); t.removable = b;
            rd(f, &b); t.neumann = b;
            rd(f, &b); t.dirichlet = b;
            rd(f, &t.phi);
            rd(f, &t.mass);
            rd(f, &t.evap_charge);
            rd(f, &t.evap_field);
            if (!rd(f, &t.evap_energy)) return "config: truncated";
            out->types[t.id] = t;
        }
        return std::string();
    }
    if (first != "ASCII") return "config: unknown mode";
    std::string line;
    while (true) {
        std::map<std::string, std::string> block;
        bool any = false;
        while (std::getline(f, line)) {
            const std::string t = trim(line);
            if (t.empty()) {
                if (any) break;
                continue;
            }
            if (t[0] == '#') continue;
            const size_t pos = t.find(" = ");
            if (pos == std::string::npos) return "config: bad line '" + t + "'";
            if (!block.insert(std::make_pair(trim(t.substr(0, pos)), trim(t.substr(pos + 3)))).second)
                return "config: duplicate key";
            any = true;
        }
        if (!any) break;
        if (block.size() == 1) {
            if (block.begin()->first != kConfigKeys[0]) return "config: bad global key";
            if (!parse(block.begin()->second, &out->temperature)) return "config: bad temperature";
        } else if (block.size() == 12) {
            CellType t;
            short idv = -1;
            int removable = 0, neumann = 0, dirichlet = 0;
            for (const auto& kv : block) {
                int k = 1;
                while (k < 13 && kv.first != kConfigKeys[k]) k++;
                bool ok = true;
                switch (k) {
                    case 1: ok = parse(kv.second, &idv); break;
                    case 2: t.name = kv.second; break;
                    case 3: ok = parse(kv.second, &t.charge_density); break;
                    case 4: ok = parse(kv.second, &t.epsilon); break;
                    case 5: ok = parse(kv.second, &removable); break;
                    case 6: ok = parse(kv.second, &neumann); break;
                    case 7: ok = parse(kv.second, &dirichlet); break;
                    case 8: ok = parse(kv.second, &t.phi); break;
                    case 9: ok = parse(kv.second, &t.mass); break;
                    case 10: ok = parse(kv.second, &t.evap_charge); break;
                    case 11: ok = parse(kv.second, &t.evap_field); break;
                    case 12: ok = parse(kv.second, &t.evap_energy); break;
                    default: return "config: unknown key " + kv.first;
                }
                if (!ok) return "config: bad value for " + kv.first;
            }
            if (idv < 0 || idv > 127) return "config: invalid id";
            t.id = idv;
            t.removable = removable != 0;
            t.neumann = neumann != 0;
            t.dirichlet = dirichlet != 0;
            out->types[t.id] = t;
        } else {
            return "config: incomplete type block";
        }
        if (!f) break;
    }
    return std::string();
}

std::string write_config_ascii(const std::string& path, const ConfigTable& table) {
    std::ofstream f(path, std::ios::trunc);
    if (!f.good()) return "config: cannot write " + path;
    f.precision(8);
    f << "ASCII\n\n" << kConfigKeys[0] << " = " << table.temperature << "\n\n";
    for (const auto& kv : table.types) {
        const CellType& t = kv.second;
        f << "ID = " << t.id << "\n"
          << "NAME = " << t.name << "\n"
          << "CHARGE_DENSITY = " << t.charge_density << "\n"
          << "DIELECTRICITY = " << t.epsilon << "\n"
          << "REMOVABLE = " << (t.removable ? 1 : 0) << "\n"
          << "NEUMANN_BOUNDARY = " << (t.neumann ? 1 : 0) << "\n"
          << "DIRICHLET_BOUNDARY = " << (t.dirichlet ? 1 : 0) << "\n"
          << "POTENTIAL = " << t.phi << "\n"
          << "MASS = " << t.mass << "\n"
          << "EVAPORATION_CHARGE_STATE = " << t.evap_charge << "\n"
          << "EVAPORATION_FIELD_STRENGTH = " << t.evap_field << "\n"
          << "EVAPORATION_ACTIVATION_ENERGY = " << t.evap_energy << "\n\n";
    }
    return f.good() ? std::string() : "config: write error";
}

std::string read_ini(const std::string& path, std::map<std::string, std::string>* out) {
    std::ifstream f(path);
    if (!f.good()) return "ini: cannot open " + path;
    out->clear();
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        const size_t pos = line.find(" = ");
        if (pos == std::string::npos) return "ini: bad line '" + line + "'";
        if (!out->insert(std::make_pair(trim(line.substr(0, pos)), trim(line.substr(pos + 3)))).second)
            return "ini: duplicate key";
    }
    return std::string();
}

std::string read_dump(const std::string& path, Dump* d) {
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) return "dump: cannot open " + path;
    std::string line;
    std::getline(f, line);
    if (line.compare(0, 23, "TAPSIM DUMP INFORMATION") != 0) return "dump: wrong file type";
    std::getline(f, line);
    if (line.compare(0, 10, "LAST_INDEX") != 0 || !parse(trim(line.substr(10)), &d->last_index)) return "dump: bad index";
    std::string ver;
    // configuration table
    if (!rd_cstr(f, &ver) || ver != "1.0") return "dump: config version";
    int size = 0;
    rd(f, &d->config.temperature);
    rd(f, &size);
    d->config.types.clear();
    for (int i = 0; i < size; i++) {
        CellType t;
        char id;
        bool b;
        rd(f, &id);
        t.id = id;
        rd_cstr(f, &t.name);
        rd(f, &t.charge_density);
        rd(f, &t.epsilon);
        rd(f, &b); t.removable = b;
        rd(f, &b); t.neumann = b;
        rd(f, &b); t.dirichlet = b;
        rd(f, &t.phi);
        rd(f, &t.mass);
        // the reference writes the short charge state with sizeof(float)
        // bytes (configuration.cpp:145,204); the first two carry the value
        char cs[4];
        f.read(cs, 4);
        std::memcpy(&t.evap_charge, cs, 2);
        rd(f, &t.evap_field);
        if (!rd(f, &t.evap_energy)) return "dump: truncated config";
        d->config.types[t.id] = t;
    }
    // geometry table
    if (!rd_cstr(f, &ver) || ver != "1.0") return "dump: geometry version";
    for (int k = 0; k < 3; k++) rd(f, &d->min[k]);
    for (int k = 0; k < 3; k++) rd(f, &d->max[k]);
    for (int k = 0; k < 3; k++) rd(f, &d->cmin[k]);
    for (int k = 0; k < 3; k++) rd(f, &d->cmax[k]);
    int n = 0;
    rd(f, &n);
    d->xyz.resize(3L * n);
    d->hull.resize(n);
    d->node_tet.resize(n);
    for (int i = 0; i < n; i++) {
        rd(f, &d->xyz[3 * i]);
        rd(f, &d->xyz[3 * i + 1]);
        rd(f, &d->xyz[3 * i + 2]);
        bool b;
        rd(f, &b);
        d->hull[i] = b;
        if (!rd(f, &d->node_tet[i])) return "dump: truncated geometry";
    }
    int nt = 0;
    rd(f, &nt);
    d->tet_v.resize(4L * nt);
    d->tet_n.resize(4L * nt);
    for (long t = 0; t < nt; t++) {
        f.read(reinterpret_cast<char*>(&d->tet_v[4 * t]), 16);
        f.read(reinterpret_cast<char*>(&d->tet_n[4 * t]), 16);
    }
    if (!f) return "dump: truncated tetrahedra";
    // grid table
    if (!rd_cstr(f, &ver) || ver != "1.0") return "dump: grid version";
    float inf;
    rd(f, &inf);
    rd(f, &d->relaxation_factor);
    rd(f, &d->phi_switch);
    int gn = 0;
    rd(f, &gn);
    if (gn != n) return "dump: node count mismatch";
    d->id.resize(n);
    d->number.resize(n);
    d->phi0.resize(n);
    d->phi1.resize(n);
    d->charge.resize(n);
    d->boundary.resize(n);
    d->dirichlet.resize(n);
    d->neumann.resize(n);
    d->row_ptr.assign(n + 1, 0);
    d->col.clear();
    d->coupling.clear();
    for (int i = 0; i < n; i++) {
        rd(f, &d->id[i]);
        rd(f, &d->number[i]);
        rd(f, &d->phi0[i]);
        rd(f, &d->phi1[i]);
        rd(f, &d->charge[i]);
        bool b;
        rd(f, &b); d->boundary[i] = b;
        rd(f, &b); d->dirichlet[i] = b;
        rd(f, &b); d->neumann[i] = b;
        int nn = 0;
        if (!rd(f, &nn) || nn < 0) return "dump: truncated grid";
        for (int k = 0; k < nn; k++) {
            int c;
            float v;
            rd(f, &c);
            rd(f, &v);
            d->col.push_back(c);
            d->coupling.push_back(v);
        }
        d->row_ptr[i + 1] = (int32_t)d->col.size();
    }
    if (!f) return "dump: truncated grid";
    return std::string();
}

std::string write_dump(const std::string& path, const Dump& d) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.good()) return "dump: cannot write " + path;
    f << "TAPSIM DUMP INFORMATION" << '\n' << "LAST_INDEX " << d.last_index << '\n';
    f.write("1.0", 4);
    wr(f, d.config.temperature);
    wr(f, (int)d.config.types.size());
    for (const auto& kv : d.config.types) {
        const CellType& t = kv.second;
        wr(f, (char)t.id);
        f.write(t.name.c_str(), t.name.size() + 1);
        wr(f, t.charge_density);
        wr(f, t.epsilon);
        wr(f, (bool)t.removable);
        wr(f, (bool)t.neumann);
        wr(f, (bool)t.dirichlet);
        wr(f, t.phi);
        wr(f, t.mass);
        // The reference writes the 16-bit charge state with sizeof(float)
        // bytes (configuration.cpp:204) and reads it back the same way
        // (configuration.cpp:145), so two bytes beyond the short travel with
        // it.  In the reference as built from its sources, those bytes are
        // the low half of the type count on the writer's stack, and its
        // reader stores them back into that count: they must hold the count
        // for the reference to read the rest of the dump.
        char cs[4];
        const uint16_t ntypes = (uint16_t)d.config.types.size();
        std::memcpy(cs, &t.evap_charge, 2);
        std::memcpy(cs + 2, &ntypes, 2);
        f.write(cs, 4);
        wr(f, t.evap_field);
        wr(f, t.evap_energy);
    }
    f.write("1.0", 4);
    for (int k = 0; k < 3; k++) wr(f, d.min[k]);
    for (int k = 0; k < 3; k++) wr(f, d.max[k]);
    for (int k = 0; k < 3; k++) wr(f, d.cmin[k]);
    for (int k = 0; k < 3; k++) wr(f, d.cmax[k]);
    const uint32_t n = (uint32_t)d.hull.size();
    wr(f, n);
    for (uint32_t i = 0; i < n; i++) {
        wr(f, d.xyz[3 * i]);
        wr(f, d.xyz[3 * i + 1]);
        wr(f, d.xyz[3 * i + 2]);
        wr(f, (bool)d.hull[i]);
        wr(f, d.node_tet[i]);
    }
    const uint32_t nt = (uint32_t)(d.tet_v.size() / 4);
    wr(f, nt);
    for (uint32_t t = 0; t < nt; t++) {
        f.write(reinterpret_cast<const char*>(&d.tet_v[4 * (size_t)t]), 16);
        f.write(reinterpret_cast<const char*>(&d.tet_n[4 * (size_t)t]), 16);
    }
    f.write("1.0", 4);
    wr(f, 1e2f);
    wr(f, d.relaxation_factor);
    wr(f, d.phi_switch);
    wr(f, n);
    for (uint32_t i = 0; i < n; i++) {
        wr(f, d.id[i]);
        wr(f, d.number[i]);
        wr(f, d.phi0[i]);
        wr(f, d.phi1[i]);
        wr(f, d.charge[i]);
        wr(f, (bool)d.boundary[i]);
        wr(f, (bool)d.dirichlet[i]);
        wr(f, (bool)d.neumann[i]);
        const int nn = d.row_ptr[i + 1] - d.row_ptr[i];
        wr(f, nn);
        for (int q = d.row_ptr[i]; q < d.row_ptr[i + 1]; q++) {
            wr(f, d.col[q]);
            wr(f, d.coupling[q]);
        }
    }
    return f.good() ? std::string() : "dump: write error";
}

namespace {

// File name of a chunk: path.%08u after the index that opens it.
std::string chunk_name(const std::string& path, uint32_t index) {
    char suffix[16];
    snprintf(suffix, sizeof(suffix), ".%08u", index);
    return path + suffix;
}

void results_header(std::ostream& f, bool binary, const std::string& header) {
    static const char* fields[] = {"index [1]", "id [1]", "number [1]", "voltage [V]", "startX [m]", "startY [m]",
                                   "startZ [m]", "stopX [m]", "stopY [m]", "stopZ [m]", "tof [s]",
                                   "probability [1]", "potentialBefore [V]", "fieldBeforeX [V/m]",
                                   "fieldBeforeY [V/m]", "fieldBeforeZ [V/m]", "potentialAfter [V]",
                                   "fieldAfterX [V/m]", "fieldAfterY [V/m]", "fieldAfterZ [V/m]", "normalX [m]",
                                   "normalY [m]", "normalZ [m]", "apexX [m]", "apexY [m]", "apexZ [m]"};
    static const char* types[] = {"int", "int", "unsigned int", "float", "float", "float", "float", "float", "float",
                                  "float", "float", "float", "float", "float", "float", "float", "float", "float",
                                  "float", "float", "float", "float", "float", "float", "float", "float"};
    f << "TAPSIM RESULTS DATA\nVERSION 1.0\n" << header;
    for (int k = 0; k < 26; k++) {
        std::string name = fields[k];
        if (binary) {
            // the binary header names potentials with unit [1]
            if (k == 12) name = "potentialBefore [1]";
            if (k == 16) name = "potentialAfter [1]";
            f << "# " << name << " (" << types[k] << ")\n";
        } else {
            f << "# " << name << "\n";
        }
    }
    f << (binary ? "BINARY\n" : "ASCII\n");
}

}  // namespace

std::string write_results(const std::string& path, const std::vector<ResultRecord>& recs, bool binary,
                          const std::string& header, int chunk) {
    std::ofstream f;
    auto open = [&](const std::string& name, bool first) {
        if (f.is_open()) f.close();
        f.open(name, std::ios::binary | std::ios::trunc);
        if (f.good()) results_header(f, binary, first ? header : std::string());
        return f.good();
    };
    if (recs.empty() && !open(path, true)) return "results: cannot write " + path;
    for (size_t k = 0; k < recs.size(); k++) {
        const ResultRecord& r = recs[k];
        if (k == 0 || (chunk > 0 && r.index % (uint32_t)chunk == 0)) {
            const std::string name = chunk > 0 ? chunk_name(path, r.index) : path;
            if (!open(name, k == 0)) return "results: cannot write " + name;
        }
        if (binary) {
            wr(f, r.index);
            wr(f, r.id);
            wr(f, r.number);
            wr(f, r.voltage);
            for (int j = 0; j < 3; j++) wr(f, r.start[j]);
            for (int j = 0; j < 3; j++) wr(f, r.stop[j]);
            wr(f, r.tof);
            wr(f, r.probability);
            wr(f, r.phi_before);
            for (int j = 0; j < 3; j++) wr(f, r.field_before[j]);
            wr(f, r.phi_after);
            for (int j = 0; j < 3; j++) wr(f, r.field_after[j]);
            for (int j = 0; j < 3; j++) wr(f, r.normal[j]);
            for (int j = 0; j < 3; j++) wr(f, r.apex[j]);
        } else {
            char buf[1024];
            int len = snprintf(buf, sizeof(buf),
                               "%u\t%d\t%u\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\t%e\n",
                               r.index, (int)r.id, r.number, r.voltage, r.start[0], r.start[1], r.start[2], r.stop[0],
                               r.stop[1], r.stop[2], r.tof, r.probability, r.phi_before, r.field_before[0],
                               r.field_before[1], r.field_before[2], r.phi_after, r.field_after[0], r.field_after[1],
                               r.field_after[2], r.normal[0], r.normal[1], r.normal[2], r.apex[0], r.apex[1], r.apex[2]);
            f.write(buf, len);
        }
    }
    return f.good() ? std::string() : "results: write error";
}

namespace {

void trajectory_header(std::ostream& f, bool binary) {
    static const char* cols[] = {"time [s]", "positionX [m]", "positionY [m]", "positionZ [m]", "velocityX [m/s]",
                                 "velocityY [m/s]", "velocityZ [m/s]", "tetrahedron [1]"};
    f << "TAPSIM TRAJECTORY DATA\nVERSION 1.0\n";
    for (int k = 0; k < 8; k++) {
        f << "# " << cols[k];
        if (binary) f << (k == 7 ? " (int)" : " (float)");
        f << '\n';
    }
    f << '\n';
}

const char* status_name(int s) {
    switch (s) {
        case 0: return "NO_INTEGRATION";
        case 1: return "NO_FIELD";
        case 2: return "STEPPER_LIMIT_PASSED";
        case 3: return "ITERATION_LIMIT_PASSED";
        case 4: return "GEOMETRY_LIMIT_PASSED";
        case 5: return "SYSTEM_LIMIT_PASSED";
        default: return "INVALID";
    }
}

}  // namespace

std::string write_trajectories(const std::string& path, const std::vector<TrajectoryRecord>& recs, bool binary,
                               int chunk) {
    std::ofstream f;
    auto open = [&](const std::string& name) {
        if (f.is_open()) f.close();
        f.open(name, std::ios::binary | std::ios::trunc);
        if (f.good()) trajectory_header(f, binary);
        return f.good();
    };
    if (recs.empty() && !open(path)) return "trajectories: cannot write " + path;
    char line[512];
    for (size_t k = 0; k < recs.size(); k++) {
        const TrajectoryRecord& t = recs[k];
        if (k == 0 || (chunk > 0 && t.index % (uint32_t)chunk == 0)) {
            const std::string name = chunk > 0 ? chunk_name(path, t.index) : path;
            if (!open(name)) return "trajectories: cannot write " + name;
        }
        int len = snprintf(line, sizeof(line),
                           "# index = %u\n# unique number = %u\n# time scale = %e\n# integrator status = %d => %s\n"
                           "# charge [C] / mass [kg] = %e / %e\n%s %d\n",
                           t.index, t.number, t.time_scale, t.status, status_name(t.status), t.charge, t.mass,
                           binary ? "BINARY" : "ASCII", t.num_points);
        f.write(line, len);
        if (binary) {
            f.write(reinterpret_cast<const char*>(t.points), 32 * (std::streamsize)t.num_points);
            f << '\n';
        } else {
            for (int p = 0; p < t.num_points; p++) {
                const float* q = t.points + 8 * (size_t)p;
                int32_t tet;
                std::memcpy(&tet, q + 7, sizeof(tet));
                len = snprintf(line, sizeof(line), "%e\t%e\t%e\t%e\t%e\t%e\t%e\t%d\n", q[0], q[1], q[2], q[3], q[4],
                               q[5], q[6], tet);
                f.write(line, len);
            }
        }
        len = snprintf(line, sizeof(line),
                       "# final error estimate (position) = (%e/%e/%e)\n# final error estimate (velocity) = (%e/%e/%e)\n\n",
                       t.error[0], t.error[1], t.error[2], t.error[3], t.error[4], t.error[5]);
        f.write(line, len);
    }
    return f.good() ? std::string() : "trajectories: write error";
}

std::string write_grid_log(const std::string& path, bool binary, const GridLog& g) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.good()) return "grid log: cannot write " + path;
    f << "TAPSIM GRID DATA\nVERSION 1.0\n" << (binary ? "BINARY " : "ASCII ") << g.n << '\n';
    std::string buf;
    for (int i = 0; i < g.n; i++) {
        const float* E = g.field + 3 * (size_t)i;
        const float* F = g.force + 3 * (size_t)i;
        if (binary) {
            wr(f, (short)g.id[i]);
            wr(f, g.number[i]);
            wr(f, g.phi[i]);
            for (int k = 0; k < 3; k++) wr(f, E[k]);
            for (int k = 0; k < 3; k++) wr(f, F[k]);
        } else {
            char line[512];
            const int len = snprintf(line, sizeof(line), "%d\t%u\t%e\t%e\t%e\t%e\t%e\t%e\t%e\n", (int)(short)g.id[i],
                                     g.number[i], g.phi[i], E[0], E[1], E[2], F[0], F[1], F[2]);
            buf.append(line, len);
            if (buf.size() > (1u << 20)) {
                f.write(buf.data(), buf.size());
                buf.clear();
            }
        }
    }
    f.write(buf.data(), buf.size());
    return f.good() ? std::string() : "grid log: write error";
}

std::string write_surface_log(const std::string& path, bool binary, const SurfaceLog& s) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.good()) return "surface log: cannot write " + path;
    f << "TAPSIM SURFACE DATA\nVERSION 1.0\n" << (binary ? "BINARY" : "ASCII") << "\n\n";
    f << "CELLS " << s.cells << '\n';
    char line[512];
    for (int c = 0; c < s.cells; c++) {
        const int q0 = s.neighbour_ptr ? s.neighbour_ptr[c] : 0, q1 = s.neighbour_ptr ? s.neighbour_ptr[c + 1] : 0;
        if (binary) {
            wr(f, s.cell[c]);
            wr(f, (short)s.type[c]);
            wr(f, s.number[c]);
            wr(f, s.probability[c]);
            wr(f, (uint32_t)(q1 - q0));
            for (int q = q0; q < q1; q++) wr(f, s.neighbours[q]);
        } else {
            int len = snprintf(line, sizeof(line), "%d\t%d\t%u\t%e", s.cell[c], (int)(short)s.type[c], s.number[c],
                               s.probability[c]);
            f.write(line, len);
            if (s.neighbour_ptr) {
                len = snprintf(line, sizeof(line), "\t%d", q1 - q0);
                f.write(line, len);
                for (int q = q0; q < q1; q++) {
                    len = snprintf(line, sizeof(line), "\t%d", s.neighbours[q]);
                    f.write(line, len);
                }
            }
            f << '\n';
        }
    }
    f << '\n' << "NODES " << s.nodes << '\n';
    for (int k = 0; k < s.nodes; k++) {
        const float* E = s.field + 3 * (size_t)k;
        const float* N = s.normal + 3 * (size_t)k;
        if (binary) {
            wr(f, s.node[k]);
            wr(f, s.phi[k]);
            for (int j = 0; j < 3; j++) wr(f, E[j]);
            for (int j = 0; j < 3; j++) wr(f, N[j]);
        } else {
            const int len = snprintf(line, sizeof(line), "%d\t%e\t%e\t%e\t%e\t%e\t%e\t%e\n", s.node[k], s.phi[k], E[0],
                                     E[1], E[2], N[0], N[1], N[2]);
            f.write(line, len);
        }
    }
    return f.good() ? std::string() : "surface log: write error";
}

}  // namespace tg_host

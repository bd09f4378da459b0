// Host-side model I/O and DOF numbering (include/ofea_host.h): the .inp subset
// OpenFEA reads, set_BCs numbering / load vector, legacy-VTK output.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <string_view>
#include <vector>

#include "../../../include/ofea_gpu.h"
#include "../../../include/ofea_host.h"

struct ofea_model {
    int nd = 0, ne = 0;
    std::vector<double> xyz;
    std::vector<int> topo, etype, fix, load_set;
    int load_dof = 0;
    double load_value = 0;
    double E = 0, nu = 0, density = 0;
    int has_elastic = 0;
};

namespace {

struct IoError {
    std::string msg;
};

// The whole file in one buffer and the [begin, end) of every line, line
// breaks \n, \r\n and \r as the reference's safeGetline accepts them.  The
// lines are parsed in place (no per-line strings): a 1.56M-DOF model reads
// in a fraction of a second.
struct Lines {
    std::string buf;
    std::vector<std::pair<size_t, size_t>> ln;
    size_t size() const { return ln.size(); }
    std::string_view operator[](size_t i) const {
        return std::string_view(buf.data() + ln[i].first, ln[i].second - ln[i].first);
    }
};

Lines read_lines(const char *path) {
    Lines L;
    FILE *f = std::fopen(path, "rb");
    if (!f) throw IoError{std::string("cannot open ") + path};
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    L.buf.resize(size > 0 ? (size_t)size : 0);
    const size_t got = size > 0 ? std::fread(&L.buf[0], 1, (size_t)size, f) : 0;
    std::fclose(f);
    if (size < 0 || got != (size_t)size) throw IoError{std::string("cannot read ") + path};
    const std::string &all = L.buf;
    size_t b = 0;
    for (size_t i = 0; i < all.size(); ++i) {
        const char ch = all[i];
        if (ch == '\n' || ch == '\r') {
            L.ln.emplace_back(b, i);
            if (ch == '\r' && i + 1 < all.size() && all[i + 1] == '\n') ++i;
            b = i + 1;
        }
    }
    if (b < all.size()) L.ln.emplace_back(b, all.size());
    return L;
}

bool has(std::string_view s, const char *key) { return s.find(key) != std::string_view::npos; }

std::string_view strip(std::string_view s) {
    size_t b = s.find_first_not_of(" \t"), e = s.find_last_not_of(" \t");
    return b == std::string_view::npos ? std::string_view() : s.substr(b, e - b + 1);
}

// The numbers of a "*Node" line: whitespace and commas separate them (the
// reference replaces ',' by ' ' and reads with >>, src/data2cae.cpp:103-115).
bool parse_doubles(std::string_view s, double *v, int count) {
    const char *p = s.data(), *e = p + s.size();
    for (int k = 0; k < count; ++k) {
        while (p < e && (*p == ' ' || *p == '\t' || *p == ',')) ++p;
        if (p < e && *p == '+') ++p;
        const auto r = std::from_chars(p, e, v[k]);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
    }
    return true;
}

// The comma-separated integers of an "*Element" line (each token stripped).
int parse_ints(std::string_view s, int *v, int cap) {
    int n = 0;
    size_t pos = 0;
    while (pos <= s.size()) {
        size_t c = s.find(',', pos);
        if (c == std::string_view::npos) c = s.size();
        std::string_view t = strip(s.substr(pos, c - pos));
        if (!t.empty()) {
            if (n >= cap) return -1;
            const char *p = t.data(), *e = p + t.size();
            if (*p == '+') ++p;
            const auto r = std::from_chars(p, e, v[n]);
            if (r.ec != std::errc()) return -1;
            ++n;
        }
        pos = c + 1;
    }
    return n;
}

// Whitespace tokens with one trailing comma removed, as the reference's
// "iss >> node_id; erase last ','" (src/data2cae.cpp:334-341).
std::vector<int> id_list(std::string_view line) {
    std::istringstream iss{std::string(line)};
    std::string tok;
    std::vector<int> out;
    while (iss >> tok) {
        if (!tok.empty() && tok.back() == ',') tok.pop_back();
        if (!tok.empty()) out.push_back(std::atoi(tok.c_str()));
    }
    return out;
}

// Value of the second token of a "a, b, c" generate line (read_ele_node_num).
int generate_count(std::string_view line) {
    std::istringstream iss{std::string(line)};
    std::string t1, t2;
    iss >> t1 >> t2;
    return std::atoi(t2.c_str());
}

void parse(const Lines &L, ofea_model &m) {
    // counts from the first *Nset / *Elset generate lines (src/data2cae.cpp:28-47)
    int nd_gen = -1, ne_gen = -1;
    for (size_t i = 0; i + 1 < L.size(); ++i) {
        if (has(L[i], "*Nset")) nd_gen = generate_count(L[i + 1]);
        if (has(L[i], "*Elset")) {
            ne_gen = generate_count(L[i + 1]);
            break;
        }
    }
    // nodes and elements (src/data2cae.cpp:89-163), up to *End Assembly
    bool in_node = false, in_elem = false;
    int etype = -1;
    for (size_t i = 0; i < L.size(); ++i) {
        const std::string_view s = L[i];
        if (has(s, "*End Assembly")) break;
        if (has(s, "*")) {
            in_node = has(s, "*Node") && !has(s, "*Nset") && !has(s, "*Node Output");
            in_elem = false;
            if (has(s, "*Element") && !has(s, "*Element Output")) {
                size_t eq = s.find('=');
                std::string_view t = eq == std::string_view::npos ? std::string_view() : strip(s.substr(eq + 1));
                size_t comma = t.find(',');
                if (comma != std::string_view::npos) t = strip(t.substr(0, comma));
                if (t == "C3D4")
                    etype = 0;
                else if (t == "C3D8")
                    etype = 1;
                else
                    throw IoError{"unsupported element type '" + std::string(t) + "' (C3D4, C3D8 only)"};
                in_elem = true;
            }
            continue;
        }
        if (in_node) {
            double v[4];  // id, x, y, z
            if (!parse_doubles(s, v, 4)) throw IoError{"bad *Node line: " + std::string(s)};
            // stored in file order, ids not used (src/data2cae.cpp:103-115)
            m.xyz.push_back(v[1]);
            m.xyz.push_back(v[2]);
            m.xyz.push_back(v[3]);
        } else if (in_elem) {
            int v[10];
            const int npe = etype == 1 ? 8 : 4;
            if (parse_ints(s, v, 10) != npe + 1) throw IoError{"bad *Element line: " + std::string(s)};
            for (int a = 0; a < 8; ++a) m.topo.push_back(a < npe ? v[1 + a] : 0);
            m.etype.push_back(etype);
        }
    }
    m.nd = (int)(m.xyz.size() / 3);
    m.ne = (int)m.etype.size();
    if (m.nd == 0 || m.ne == 0) throw IoError{"no *Node or *Element data"};
    if ((nd_gen >= 0 && nd_gen != m.nd) || (ne_gen >= 0 && ne_gen != m.ne))
        throw IoError{"*Nset/*Elset generate counts disagree with the *Node/*Element data"};
    for (int v : m.topo)
        if (v < 0 || v > m.nd) throw IoError{"element references a node id outside 1..nd"};
    // Set-load / Set-fix node lists before *End Assembly (src/data2cae.cpp:321-350, 382-411)
    auto node_set = [&](const char *key, std::vector<int> &out) {
        for (size_t i = 0; i < L.size(); ++i) {
            if (has(L[i], "*End Assembly")) break;
            if (has(L[i], key)) {
                size_t j = i + 1;
                for (; j < L.size() && !has(L[j], "*"); ++j) {
                    auto ids = id_list(L[j]);
                    out.insert(out.end(), ids.begin(), ids.end());
                }
                i = j - 1;
            }
        }
    };
    node_set("Set-load", m.load_set);
    node_set("Set-fix", m.fix);
    // Cload after *End Assembly: "set, dof, value" (src/data2cae.cpp:352-369)
    bool after = false;
    for (size_t i = 0; i < L.size(); ++i) {
        if (has(L[i], "*End Assembly")) after = true;
        if (after && has(L[i], "Cload") && i + 1 < L.size()) {
            std::istringstream iss{std::string(L[i + 1])};
            std::string name, dof, val;
            iss >> name >> dof >> val;
            if (!dof.empty() && dof.back() == ',') dof.pop_back();
            m.load_dof = std::atoi(dof.c_str());
            m.load_value = std::strtod(val.c_str(), nullptr);
            break;
        }
    }
    // *Density, *Elastic (last occurrence wins, src/data2cae.cpp:422-442)
    for (size_t i = 0; i + 1 < L.size(); ++i) {
        if (has(L[i], "*Density")) {
            std::istringstream iss{std::string(L[i + 1])};
            std::string d;
            iss >> d;
            if (!d.empty() && d.back() == ',') d.pop_back();
            m.density = std::strtod(d.c_str(), nullptr);
        }
        if (has(L[i], "*Elastic")) {
            std::istringstream iss{std::string(L[i + 1])};
            std::string e, nu;
            iss >> e >> nu;
            if (!e.empty() && e.back() == ',') e.pop_back();
            m.E = std::strtod(e.c_str(), nullptr);
            m.nu = std::strtod(nu.c_str(), nullptr);
            m.has_elastic = 1;
        }
    }
}

// The CA change file (ReadInfo::CA_read_change, src/data2cae.cpp:520-661):
// "*nodes_all, N" then N lines "x, y, z" (every node of the original model,
// modified coordinates); "*eles_change, M, type=C3D4|C3D8" then M lines
// "kind, n1, .., nk" (kind 0 deleted, 1 moved, 2 added; node ids 0-based into
// the node list), several such blocks allowed; "*End Assembly";
// "*idref2new, N" then N lines: the node's id in the modified model, or -1.
struct CaInfo {
    std::vector<double> xyz;
    std::vector<int> kind, etype, topo, map;
};

void parse_ca_info(const Lines &L, CaInfo &ci) {
    size_t i = 0;
    auto count_after_comma = [](std::string_view line) {
        const size_t c = line.find(',');
        if (c == std::string_view::npos) throw IoError{"missing count"};
        std::string_view t = line.substr(c + 1);
        const size_t e = t.find(',');
        if (e != std::string_view::npos) t = t.substr(0, e);
        t = strip(t);
        int v = 0;
        const auto r = std::from_chars(t.data(), t.data() + t.size(), v);
        if (r.ec != std::errc() || v < 0) throw IoError{"bad count"};
        return v;
    };
    int nd = -1;
    for (; i < L.size(); ++i) {
        std::string_view line = L[i];
        if (has(line, "*nodes_all")) {
            nd = count_after_comma(line);
            ci.xyz.resize(3 * (size_t)nd);
            for (int k = 0; k < nd; ++k) {
                if (++i >= L.size() || !parse_doubles(L[i], &ci.xyz[3 * (size_t)k], 3))
                    throw IoError{"bad node line in *nodes_all"};
            }
        } else if (has(line, "*eles_change")) {
            if (nd < 0) throw IoError{"*eles_change before *nodes_all"};
            const int m = count_after_comma(line);
            const size_t eq = line.find('=');
            if (eq == std::string_view::npos) throw IoError{"*eles_change without type="};
            std::string_view ty = strip(line.substr(eq + 1));
            int et, nn;
            if (ty == "C3D4") et = 0, nn = 4;
            else if (ty == "C3D8" || ty == "C3D8R") et = 1, nn = 8;
            else throw IoError{"unknown element type in *eles_change"};
            for (int k = 0; k < m; ++k) {
                if (++i >= L.size()) throw IoError{"truncated *eles_change"};
                int v[9];
                if (parse_ints(L[i], v, 9) != nn + 1) throw IoError{"bad line in *eles_change"};
                if (v[0] < 0 || v[0] > 2) throw IoError{"change kind must be 0, 1 or 2"};
                ci.kind.push_back(v[0]);
                ci.etype.push_back(et);
                for (int j = 0; j < 8; ++j) {
                    const int node = j < nn ? v[j + 1] : -1;
                    if (j < nn && (node < 0 || node >= nd)) throw IoError{"node id out of range in *eles_change"};
                    ci.topo.push_back(node);
                }
            }
        } else if (has(line, "*idref2new")) {
            if (nd < 0) throw IoError{"*idref2new before *nodes_all"};
            const int m = count_after_comma(line);
            if (m != nd) throw IoError{"*idref2new count differs from *nodes_all"};
            ci.map.resize(nd);
            for (int k = 0; k < nd; ++k) {
                if (++i >= L.size() || parse_ints(L[i], &ci.map[k], 1) != 1 || ci.map[k] < -1)
                    throw IoError{"bad line in *idref2new"};
            }
        }
    }
    if (nd < 0) throw IoError{"no *nodes_all section"};
    if (ci.map.empty() && nd > 0) throw IoError{"no *idref2new section"};
}

}  // namespace

extern "C" {

int ofea_ca_info_read(const char *path, int *n_nodes, int *n_changes, double *xyz, int *kind, int *etype,
                      int *topo, int *node_map) {
    if (!path || !n_nodes || !n_changes) return OFEA_ERR_INVALID_ARG;
    try {
        CaInfo ci;
        parse_ca_info(read_lines(path), ci);
        *n_nodes = (int)ci.map.size();
        *n_changes = (int)ci.kind.size();
        if (xyz) std::copy(ci.xyz.begin(), ci.xyz.end(), xyz);
        if (kind) std::copy(ci.kind.begin(), ci.kind.end(), kind);
        if (etype) std::copy(ci.etype.begin(), ci.etype.end(), etype);
        if (topo) std::copy(ci.topo.begin(), ci.topo.end(), topo);
        if (node_map) std::copy(ci.map.begin(), ci.map.end(), node_map);
        return OFEA_OK;
    } catch (...) {
        return OFEA_ERR_IO;
    }
}

int ofea_inp_read(const char *path, ofea_model **out) {
    if (!path || !out) return OFEA_ERR_INVALID_ARG;
    *out = nullptr;
    try {
        auto lines = read_lines(path);
        auto *m = new ofea_model();
        try {
            parse(lines, *m);
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
        return OFEA_OK;
    } catch (const IoError &) {
        return OFEA_ERR_IO;
    } catch (...) {
        return OFEA_ERR_IO;
    }
}

void ofea_model_free(ofea_model *m) { delete m; }

int ofea_model_sizes(const ofea_model *m, int *nd, int *ne, int *nfix, int *nload) {
    if (!m) return OFEA_ERR_INVALID_ARG;
    if (nd) *nd = m->nd;
    if (ne) *ne = m->ne;
    if (nfix) *nfix = (int)m->fix.size();
    if (nload) *nload = (int)m->load_set.size();
    return OFEA_OK;
}

int ofea_model_arrays(const ofea_model *m, double *xyz, int *topo, int *etype, int *fix,
                      int *load_set) {
    if (!m) return OFEA_ERR_INVALID_ARG;
    if (xyz) std::copy(m->xyz.begin(), m->xyz.end(), xyz);
    if (topo) std::copy(m->topo.begin(), m->topo.end(), topo);
    if (etype) std::copy(m->etype.begin(), m->etype.end(), etype);
    if (fix) std::copy(m->fix.begin(), m->fix.end(), fix);
    if (load_set) std::copy(m->load_set.begin(), m->load_set.end(), load_set);
    return OFEA_OK;
}

int ofea_model_material(const ofea_model *m, double *E, double *nu, double *density,
                        int *has_elastic) {
    if (!m) return OFEA_ERR_INVALID_ARG;
    if (E) *E = m->E;
    if (nu) *nu = m->nu;
    if (density) *density = m->density;
    if (has_elastic) *has_elastic = m->has_elastic;
    return OFEA_OK;
}

int ofea_model_cload(const ofea_model *m, int *dof, double *value) {
    if (!m) return OFEA_ERR_INVALID_ARG;
    if (dof) *dof = m->load_dof;
    if (value) *value = m->load_value;
    return OFEA_OK;
}

int ofea_build_free_index(int nd, int nfix, const int *fix_ids, int *free_map, int *nfree) {
    if (nd <= 0 || nfix <= 0 || !fix_ids || !free_map) return OFEA_ERR_INVALID_ARG;
    std::vector<int> s(fix_ids, fix_ids + nfix);
    std::sort(s.begin(), s.end());
    for (int k = 0; k < nfix; ++k)
        if (s[k] < 1 || s[k] > nd || (k > 0 && s[k] == s[k - 1])) return OFEA_ERR_INVALID_ARG;
    // walk the nodes against the sorted fixed ids (src/set_bc.cpp:25-42)
    int next = 0, c = 0;
    for (int i = 0; i < nd; ++i) {
        if (c < nfix && i == s[c] - 1) {
            free_map[i] = -1;
            ++c;
        } else {
            free_map[i] = next++;
        }
    }
    if (nfree) *nfree = next;
    return OFEA_OK;
}

int ofea_build_single_load(int nd, const int *free_map, int nload, const int *load_set, int dof,
                           double value, double *f) {
    if (nd <= 0 || !free_map || (nload > 0 && !load_set) || !f) return OFEA_ERR_INVALID_ARG;
    if (dof < 1 || dof > 3) return OFEA_ERR_INVALID_ARG;
    int nfree = 0;
    for (int i = 0; i < nd; ++i) nfree += free_map[i] >= 0;
    std::fill(f, f + 3L * nfree, 0.0);
    for (int k = 0; k < nload; ++k) {
        int id = load_set[k];
        if (id < 1 || id > nd) return OFEA_ERR_INVALID_ARG;
        int r = free_map[id - 1];
        if (r >= 0) f[3L * r + dof - 1] = value;
    }
    return OFEA_OK;
}

int ofea_full_displacement(int nd, const int *free_map, const double *u, double *u_full) {
    if (nd <= 0 || !free_map || !u || !u_full) return OFEA_ERR_INVALID_ARG;
    for (int i = 0; i < nd; ++i) {
        int r = free_map[i];
        for (int c = 0; c < 3; ++c) u_full[3L * i + c] = r >= 0 ? u[3L * r + c] : 0.0;
    }
    return OFEA_OK;
}

int ofea_write_vtk(const char *path, int nd, const double *xyz, int ne, const int *topo,
                   const int *etype, const double *u_full, double scale) {
    return ofea_write_vtk_stress(path, nd, xyz, ne, topo, etype, u_full, scale, nullptr);
}

int ofea_write_vtk_stress(const char *path, int nd, const double *xyz, int ne, const int *topo, const int *etype,
                          const double *u_full, double scale, const double *node_stress) {
    if (!path || nd <= 0 || ne < 0 || !xyz || !topo || !etype || !u_full) return OFEA_ERR_INVALID_ARG;
    // same header, separators and default 6-significant-digit formatting as
    // the reference writer (src/data2vtk.cpp:56-100, 143-196); the text is
    // built in one buffer with std::to_chars (general format, precision 6 is
    // what an ostream prints by default) and written once
    std::string out;
    out.reserve((size_t)nd * 120 + (size_t)ne * 64 + 1024);
    char tmp[64];
    auto put = [&](const char *str) { out.append(str); };
    auto put_d = [&](double v) {
        const auto r = std::to_chars(tmp, tmp + sizeof(tmp), v, std::chars_format::general, 6);
        out.append(tmp, r.ptr);
    };
    auto put_i = [&](long v) {
        const auto r = std::to_chars(tmp, tmp + sizeof(tmp), v);
        out.append(tmp, r.ptr);
    };
    put("# vtk DataFile Version 3.0\n");
    put("The density field of the optimized results\n");
    put("ASCII\n");
    put("DATASET UNSTRUCTURED_GRID\n\n");
    put("POINTS\t");
    put_i(nd);
    put("\tdouble\n");
    for (int i = 0; i < nd; ++i) {
        put_d(xyz[3L * i] + scale * u_full[3L * i]);
        put("\t\t");
        put_d(xyz[3L * i + 1] + scale * u_full[3L * i + 1]);
        put("\t\t");
        put_d(xyz[3L * i + 2] + scale * u_full[3L * i + 2]);
        put("\n");
    }
    long n4 = 0, n8 = 0;
    for (int e = 0; e < ne; ++e) (etype[e] == 1 ? n8 : n4)++;
    put("CELLS\t");
    put_i(ne);
    put("\t");
    put_i(n8 * 9 + n4 * 5);
    put("\n");
    for (int e = 0; e < ne; ++e) {
        const int *t = topo + 8L * e;
        if (etype[e] == 1) {
            static const int ord[8] = {0, 1, 3, 2, 4, 5, 7, 6};  // VTK_VOXEL order
            put("8");
            for (int a = 0; a < 8; ++a) {
                put("\t");
                put_i(t[ord[a]] - 1);
            }
        } else {
            static const int ord[4] = {0, 2, 1, 3};
            put("4");
            for (int a = 0; a < 4; ++a) {
                put("\t");
                put_i(t[ord[a]] - 1);
            }
        }
        put("\n");
    }
    put("CELL_TYPES\t\t");
    put_i(ne);
    put("\n");
    for (int e = 0; e < ne; ++e) put(etype[e] == 1 ? "11\n" : "10\n");
    const char *names[3] = {"u_x", "u_y", "u_z"};
    put("\nPOINT_DATA\t");
    put_i(nd);
    for (int c = 0; c < 3; ++c) {
        put("\nSCALARS ");
        put(names[c]);
        put(" double 1\nLOOKUP_TABLE  table");
        put_i(c + 1);
        put("\n");
        for (int i = 0; i < nd; ++i) {
            put_d(u_full[3L * i + c]);
            put("\n");
        }
    }
    put("\nSCALARS u_magnitude double 1\nLOOKUP_TABLE  table4\n");
    for (int i = 0; i < nd; ++i) {
        const double *u = u_full + 3L * i;
        put_d(std::sqrt(u[2] * u[2] + u[1] * u[1] + u[0] * u[0]));
        put("\n");
    }
    if (node_stress) {  // src/data2vtk.cpp:211-262
        const char *sn[7] = {"S_xx", "S_yy", "S_zz", "S_xy", "S_yz", "S_xz", "S_Mises"};
        for (int k = 0; k < 7; ++k) {
            put("\nSCALARS ");
            put(sn[k]);
            put(" double 1\nLOOKUP_TABLE  table");
            put_i(k + 5);
            put("\n");
            for (int i = 0; i < nd; ++i) {
                put_d(node_stress[(long)k * nd + i]);
                put("\n");
            }
        }
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return OFEA_ERR_IO;
    const size_t w = std::fwrite(out.data(), 1, out.size(), f);
    const int rc = std::fclose(f);
    return (w == out.size() && rc == 0) ? OFEA_OK : OFEA_ERR_IO;
}

}  // extern "C"

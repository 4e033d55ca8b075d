// Configuration IO of the reference, host side only: the restart / trajectory
// writer WriteConfig (src/WriteConfig.cpp) in its four formats, the reader
// ReadConfig (src/ReadConfig.cpp), and the fixes' restart chunks
// (FixPair::restartChunkPairParams / readFromRestart, FixPair.cpp:211-265;
// FixRigid::restartChunk / readFromRestart, FixRigid.cu:1438-1514).
//
// File layout written by "base64" (writeXMLfileBase64, WriteConfig.cpp:91-162):
//   <data>
//   <configuration turn= numAtoms= dimension= periodic="111" rCut= padding= dt=>
//   <bounds base64="1" xlo= ylo= zlo= xhi= yhi= zhi= />     each one double, base64
//   <atomParams numTypes=><handle>..</handle><mass>..</mass></atomParams>
//   <position base64="1">..</position>  velocity, force: 3 doubles per atom
//   <groupTag base64="1">               uint32 per atom; type, id: int32; q: double
//   <groupInfo><groupHandles>..</groupHandles><groupBits>..</groupBits></groupInfo>
//   <molecules><m>ids </m>..</molecules>
//   </configuration>
//   </data>
// "xml" (writeXMLfile, WriteConfig.cpp:253-343) writes the same with plain
// text numbers ("%f"), bounds base64="0", and a <fixes> block of the fixes'
// restart chunks; "xyz" and "lammpstrj" are the trajectory formats of
// writeXYZFile / writeLAMMPSTRJFile (WriteConfig.cpp:165-251).  Byte data is
// little-endian as the reference's raw memory dumps on x86.
//
// The reader keeps a small DOM of the file (elements, attributes, text) in
// place of pugixml and walks its configurations with next / prev / moveBy.
#include <algorithm>
#include <cctype>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <unistd.h>
#include <vector>

#include "engine.hpp"

namespace mdx {

// ---------------------------------------------------------------- base64
// RFC 4648 alphabet with '=' padding and no line breaks (the form the
// reference's base64_encode writes and its base64_decode reads)
static const char kB64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

std::string b64_encode(const void *data, size_t n) {
    const unsigned char *p = static_cast<const unsigned char *>(data);
    std::string out;
    out.reserve((n + 2) / 3 * 4);
    size_t i = 0;
    for (; i + 3 <= n; i += 3) {
        const uint32_t v = (uint32_t)p[i] << 16 | (uint32_t)p[i + 1] << 8 | p[i + 2];
        out += kB64[v >> 18];
        out += kB64[(v >> 12) & 63];
        out += kB64[(v >> 6) & 63];
        out += kB64[v & 63];
    }
    if (i < n) {
        uint32_t v = (uint32_t)p[i] << 16;
        if (i + 1 < n) v |= (uint32_t)p[i + 1] << 8;
        out += kB64[v >> 18];
        out += kB64[(v >> 12) & 63];
        out += i + 1 < n ? kB64[(v >> 6) & 63] : '=';
        out += '=';
    }
    return out;
}

static int b64_value(char c) {
    if (c >= 'A' && c <= 'Z') return c - 'A';
    if (c >= 'a' && c <= 'z') return c - 'a' + 26;
    if (c >= '0' && c <= '9') return c - '0' + 52;
    if (c == '+') return 62;
    if (c == '/') return 63;
    return -1;
}

// decodes until the first '=' or the end; false on a character outside the
// alphabet
bool b64_decode(const std::string &s, std::vector<unsigned char> &out) {
    out.clear();
    uint32_t acc = 0;
    int bits = 0;
    for (char c : s) {
        if (c == '=') break;
        const int v = b64_value(c);
        if (v < 0) return false;
        acc = acc << 6 | (uint32_t)v;
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out.push_back((unsigned char)((acc >> bits) & 0xff));
        }
    }
    return true;
}

// ---------------------------------------------------------------- XML DOM
struct XNode {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XNode> kids;
    std::string text;  // the element's character data (all text runs joined)
    const char *attr(const char *k) const {
        for (const auto &a : attrs)
            if (a.first == k) return a.second.c_str();
        return nullptr;
    }
    const XNode *child(const char *k) const {
        for (const auto &c : kids)
            if (c.name == k) return &c;
        return nullptr;
    }
};

struct XParser {
    const std::string &s;
    size_t i = 0;
    std::string err;
    explicit XParser(const std::string &src) : s(src) {}
    bool fail(const char *what) {
        if (err.empty()) {
            char b[160];
            std::snprintf(b, sizeof(b), "%s at byte %zu", what, i);
            err = b;
        }
        return false;
    }
    void ws() {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) i++;
    }
    bool starts(const char *p) const { return s.compare(i, std::strlen(p), p) == 0; }
    bool skip_to(const char *p) {
        const size_t k = s.find(p, i);
        if (k == std::string::npos) return fail("unterminated markup");
        i = k + std::strlen(p);
        return true;
    }
    static std::string unescape(const std::string &t) {
        if (t.find('&') == std::string::npos) return t;
        std::string o;
        for (size_t k = 0; k < t.size(); k++) {
            if (t[k] != '&') {
                o += t[k];
                continue;
            }
            static const char *const ent[5][2] = {
                {"&lt;", "<"}, {"&gt;", ">"}, {"&amp;", "&"}, {"&quot;", "\""}, {"&apos;", "'"}};
            bool hit = false;
            for (const auto &e : ent)
                if (t.compare(k, std::strlen(e[0]), e[0]) == 0) {
                    o += e[1];
                    k += std::strlen(e[0]) - 1;
                    hit = true;
                    break;
                }
            if (!hit) o += '&';
        }
        return o;
    }
    bool name(std::string &out) {
        const size_t b = i;
        while (i < s.size() && (std::isalnum((unsigned char)s[i]) || s[i] == '_' || s[i] == '-' || s[i] == ':' ||
                                s[i] == '.'))
            i++;
        if (i == b) return fail("expected a name");
        out = s.substr(b, i - b);
        return true;
    }
    // skips the prolog, comments and processing instructions between elements
    bool misc() {
        for (;;) {
            ws();
            if (starts("<?")) {
                if (!skip_to("?>")) return false;
            } else if (starts("<!--")) {
                if (!skip_to("-->")) return false;
            } else if (starts("<!")) {
                if (!skip_to(">")) return false;
            } else {
                return true;
            }
        }
    }
    bool element(XNode &n, int depth) {
        if (depth > 64) return fail("elements nested too deeply");
        if (i >= s.size() || s[i] != '<') return fail("expected '<'");
        i++;
        if (!name(n.name)) return false;
        for (;;) {
            ws();
            if (i >= s.size()) return fail("unterminated start tag");
            if (s[i] == '/') {
                if (i + 1 >= s.size() || s[i + 1] != '>') return fail("expected '/>'");
                i += 2;
                return true;
            }
            if (s[i] == '>') {
                i++;
                break;
            }
            std::string k;
            if (!name(k)) return false;
            ws();
            if (i >= s.size() || s[i] != '=') return fail("expected '=' after an attribute name");
            i++;
            ws();
            if (i >= s.size() || (s[i] != '"' && s[i] != '\'')) return fail("expected a quoted attribute value");
            const char q = s[i++];
            const size_t e = s.find(q, i);
            if (e == std::string::npos) return fail("unterminated attribute value");
            n.attrs.push_back({k, unescape(s.substr(i, e - i))});
            i = e + 1;
        }
        // content
        for (;;) {
            const size_t lt = s.find('<', i);
            if (lt == std::string::npos) return fail("unterminated element");
            if (lt > i) n.text += unescape(s.substr(i, lt - i));
            i = lt;
            if (starts("</")) {
                i += 2;
                std::string close;
                if (!name(close)) return false;
                if (close != n.name) return fail("mismatched end tag");
                ws();
                if (i >= s.size() || s[i] != '>') return fail("expected '>'");
                i++;
                return true;
            }
            if (starts("<!--")) {
                if (!skip_to("-->")) return false;
                continue;
            }
            if (starts("<![CDATA[")) {
                const size_t e = s.find("]]>", i);
                if (e == std::string::npos) return fail("unterminated CDATA");
                n.text += s.substr(i + 9, e - i - 9);
                i = e + 3;
                continue;
            }
            if (starts("<?")) {
                if (!skip_to("?>")) return false;
                continue;
            }
            n.kids.emplace_back();
            if (!element(n.kids.back(), depth + 1)) return false;
        }
    }
    bool document(XNode &root) {
        if (!misc()) return false;
        if (!element(root, 0)) return false;
        if (!misc()) return false;
        if (i != s.size()) return fail("content after the document element");
        return true;
    }
};

// ---------------------------------------------------------------- numbers
// the C++ stream default the reference writes with (6 significant digits)
static std::string fmt_g(double v) {
    char b[64];
    std::snprintf(b, sizeof(b), "%g", v);
    return b;
}

static std::vector<std::string> tokens(const std::string &t) {
    std::vector<std::string> out;
    std::istringstream ss(t);
    std::string x;
    while (ss >> x) out.push_back(x);
    return out;
}

static bool parse_double(const char *p, double *out) {
    if (!p) return false;
    char *end = nullptr;
    const double v = std::strtod(p, &end);
    if (end == p) return false;
    while (*end == ' ' || *end == '\t' || *end == '\n' || *end == '\r') end++;
    if (*end) return false;
    *out = v;
    return true;
}

static bool parse_i64(const char *p, int64_t *out) {
    if (!p) return false;
    char *end = nullptr;
    const long long v = std::strtoll(p, &end, 10);
    if (end == p || *end) return false;
    *out = v;
    return true;
}

// standard atomic weights (IUPAC, abridged) for AtomParams::guessAtomicNumbers
// (AtomParams.cpp:60-77): a species takes the element whose weight is within
// 1 % of its mass, else -1
static const double kElementMass[] = {
    0,       1.008,   4.0026,  6.94,    9.0122,  10.81,   12.011,  14.007,  15.999,  18.998,  20.180,
    22.990,  24.305,  26.982,  28.085,  30.974,  32.06,   35.45,   39.95,   39.098,  40.078,  44.956,
    47.867,  50.942,  51.996,  54.938,  55.845,  58.933,  58.693,  63.546,  65.38,   69.723,  72.630,
    74.922,  78.971,  79.904,  83.798};

static int guess_atomic_number(double mass) {
    const int n = (int)(sizeof(kElementMass) / sizeof(kElementMass[0]));
    for (int z = 1; z < n; z++)
        if (std::fabs(kElementMass[z] - mass) / kElementMass[z] < 0.01) return z;
    return -1;
}

// ---------------------------------------------------------------- writer
struct ConfigWriter {
    State *state = nullptr;
    std::string fn, handle, format, groupHandle;
    int writeEvery = 1;
    uint32_t groupBit = 1;
    bool isXML = true, oneFilePerWrite = false, unwrapMolecules = false;
    bool writingVelocities = false, writingForces = false;
    bool finished = false;
};

// WriteConfig::getCurrentFn (WriteConfig.cpp:346-366): the format's suffix,
// and the turn in place of '*' when each write opens its own file
static std::string current_fn(const ConfigWriter &w, int64_t turn) {
    std::string f = w.fn;
    if (w.format == "xyz") f += ".xyz";
    else if (w.format == "lammpstrj") f += ".lammpstrj";
    else f += ".xml";
    if (w.oneFilePerWrite) {
        const size_t pos = f.find('*');
        f = f.substr(0, pos) + std::to_string(turn) + f.substr(pos + 1);
    }
    return f;
}

// positions with each molecule made whole and its centre of mass wrapped
// into the box (State::unwrapMolecules, State.cpp:329-370): a walk over the
// fixes' bonds among the molecule's atoms from its last id, each atom put at
// the minimum image of the atom it was reached from
static void unwrapped_positions(const State &s, std::vector<double> &x) {
    const int n = (int)s.atoms.size();
    x.resize(3 * (size_t)n);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) x[3 * (size_t)i + d] = s.atoms[i].pos[d];
    if (s.molecules.empty()) return;
    std::vector<char> inmol(n, 0);
    for (const auto &m : s.molecules)
        for (int id : m)
            if (id >= 0 && id < n) inmol[id] = 1;
    std::vector<std::vector<int>> adj(n);
    std::vector<std::pair<int, int>> bonds;
    for (Fix *f : s.fixes) f->getBonds(bonds);
    for (const auto &b : bonds) {
        if (b.first < 0 || b.second < 0 || b.first >= n || b.second >= n) continue;
        if (!inmol[b.first] || !inmol[b.second]) continue;
        adj[b.first].push_back(b.second);
        adj[b.second].push_back(b.first);
    }
    double L[3];
    for (int d = 0; d < 3; d++) L[d] = s.hi[d] - s.lo[d];
    std::vector<int> seen(n, -1);
    for (size_t mi = 0; mi < s.molecules.size(); mi++) {
        const auto &m = s.molecules[mi];
        if (m.empty()) continue;
        const int root = m.back();
        if (root < 0 || root >= n) continue;
        std::vector<int> stack{root};
        seen[root] = (int)mi;
        while (!stack.empty()) {
            const int a = stack.back();
            stack.pop_back();
            for (int b : adj[a]) {
                if (seen[b] == (int)mi) continue;
                seen[b] = (int)mi;
                for (int d = 0; d < 3; d++) {
                    double dr = x[3 * (size_t)b + d] - x[3 * (size_t)a + d];
                    dr -= L[d] * std::round(dr / L[d]);
                    x[3 * (size_t)b + d] = x[3 * (size_t)a + d] + dr;
                }
                stack.push_back(b);
            }
        }
        double com[3] = {0, 0, 0}, mt = 0;
        for (int id : m) {
            if (id < 0 || id >= n) continue;
            const double w = s.atoms[id].mass;
            mt += w;
            for (int d = 0; d < 3; d++) com[d] += w * x[3 * (size_t)id + d];
        }
        if (mt <= 0) continue;
        for (int d = 0; d < 3; d++) {
            com[d] /= mt;
            const double wrapped = com[d] - L[d] * std::floor((com[d] - s.lo[d]) / L[d]);
            const double shift = wrapped - com[d];
            for (int id : m)
                if (id >= 0 && id < n) x[3 * (size_t)id + d] += shift;
        }
    }
}

static const char *fix_type_for_restart(const Fix &f) { return f.type.c_str(); }

// FixPair::restartChunkPairParams (FixPair.cpp:243-265): each raw table in
// handle order, one value per line, unset entries as DEFAULT_FILL (-1000).
// Values carry 9 significant digits so that a float round-trips (the
// reference streams 6).
static std::string pair_restart_chunk(FixPair &p) {
    p.ensureSize();
    std::map<std::string, std::vector<double>> tabs = p.params;
    const size_t nt = p.state->species.size();
    if (p.lj_kind == 3) tabs["FCutHandle"] = std::vector<double>(nt * nt, std::nan(""));
    std::ostringstream ss;
    char b[64];
    for (const auto &kv : tabs) {
        ss << "<parameter handle=\"" << kv.first << "\">\n";
        for (double v : kv.second) {
            const double w = std::isnan(v) ? -1000.0 : (double)(float)v;
            std::snprintf(b, sizeof(b), "%.9g\n", w);
            ss << b;
        }
        ss << "</parameter>\n";
    }
    return ss.str();
}

// FixRigid::restartChunk (FixRigid.cu:1438-1456); a three-site molecule's
// fourth id is written as 0, as the reference stores it
static std::string rigid_restart_chunk(FixRigid &r) {
    std::ostringstream ss;
    ss << "<atomsInMolecule n=\"" << r.mol_ids.size() << "\">\n";
    for (const int4 &m : r.mol_ids) ss << m.x << " " << m.y << " " << m.z << " " << (m.w < 0 ? 0 : m.w) << "\n";
    ss << "</atomsInMolecule>\n";
    ss << "<style type='" << r.style << "'>\n</style>\n";
    ss << "<model fourSite='" << (r.foursite ? "true" : "false") << "'/>\n";
    return ss.str();
}

static std::string fix_restart_chunk(Fix &f) {
    if (f.kind == FixKind::Pair) return pair_restart_chunk(static_cast<FixPair &>(f));
    if (f.kind == FixKind::Rigid) return rigid_restart_chunk(static_cast<FixRigid &>(f));
    return "";
}

static void put_config_head(std::ostream &o, const State &s, int64_t turn) {
    char b[400];
    std::snprintf(b, sizeof(b),
                  "<configuration turn=\"%" PRId64 "\" numAtoms=\"%d\" dimension=\"%d\" periodic=\"%d%d%d\" "
                  "rCut=\"%f\" padding=\"%f\" dt=\"%f\">\n",
                  turn, (int)s.atoms.size(), 3, s.periodic[0], s.periodic[1], s.periodic[2], s.rCut, s.padding,
                  s.dt);
    o << b;
}

static void put_atom_params(std::ostream &o, const State &s) {
    o << "<atomParams numTypes=\"" << s.species.size() << "\">\n<handle>\n";
    for (const auto &sp : s.species) o << sp.handle << "\n";
    o << "</handle>\n<mass>\n";
    for (const auto &sp : s.species) o << fmt_g(sp.mass) << "\n";
    o << "</mass>\n</atomParams>\n";
}

static void put_groups_molecules(std::ostream &o, const State &s) {
    o << "<groupInfo>\n<groupHandles>\n";
    for (const auto &g : s.groupTags) o << g.first << "\n";
    o << "</groupHandles>\n<groupBits>\n";
    for (const auto &g : s.groupTags) o << g.second << "\n";
    o << "</groupBits>\n</groupInfo>\n<molecules>\n";
    for (const auto &m : s.molecules) {
        o << "<m>\n";
        for (int id : m) o << id << " ";
        o << "</m>\n";
    }
    o << "</molecules>\n";
}

template <typename T>
static void put_b64(std::ostream &o, const char *tag, const std::vector<T> &v) {
    o << "<" << tag << " base64=\"1\">\n" << b64_encode(v.data(), v.size() * sizeof(T)) << "</" << tag << ">\n";
}

static int write_xml(ConfigWriter &w, const std::string &path, int64_t turn, bool base64) {
    State &s = *w.state;
    std::ofstream o(path, w.oneFilePerWrite ? std::ios::out : std::ios::app);
    if (!o) {
        set_error(MDX_ERR_ARG, "cannot open '%s' for writing", path.c_str());
        return MDX_ERR_ARG;
    }
    if (w.oneFilePerWrite) o << "<data>\n";
    put_config_head(o, s, turn);
    const int n = (int)s.atoms.size();
    std::vector<double> x;
    if (w.unwrapMolecules) unwrapped_positions(s, x);
    else {
        x.resize(3 * (size_t)n);
        for (int i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) x[3 * (size_t)i + d] = s.atoms[i].pos[d];
    }
    char b[400];
    if (base64) {
        double dims[6] = {s.lo[0], s.lo[1], s.lo[2], s.hi[0], s.hi[1], s.hi[2]};
        std::string e[6];
        for (int k = 0; k < 6; k++) e[k] = b64_encode(dims + k, 8);
        std::snprintf(b, sizeof(b), "<bounds base64=\"1\" xlo=\"%s\" ylo=\"%s\" zlo=\"%s\" xhi=\"%s\" yhi=\"%s\" zhi=\"%s\" />\n",
                      e[0].c_str(), e[1].c_str(), e[2].c_str(), e[3].c_str(), e[4].c_str(), e[5].c_str());
        o << b;
        put_atom_params(o, s);
        std::vector<double> v(3 * (size_t)n), f(3 * (size_t)n), q(n);
        std::vector<uint32_t> g(n);
        std::vector<int32_t> t(n), id(n);
        for (int i = 0; i < n; i++) {
            const HostAtom &a = s.atoms[i];
            for (int d = 0; d < 3; d++) {
                v[3 * (size_t)i + d] = a.vel[d];
                f[3 * (size_t)i + d] = a.force[d];
            }
            g[i] = a.groupTag;
            t[i] = a.type;
            id[i] = i;
            q[i] = a.q;
        }
        put_b64(o, "position", x);
        put_b64(o, "velocity", v);
        put_b64(o, "force", f);
        put_b64(o, "groupTag", g);
        put_b64(o, "type", t);
        put_b64(o, "id", id);
        put_b64(o, "q", q);
    } else {
        std::snprintf(b, sizeof(b), "<bounds base64=\"0\" xlo=\"%f\" ylo=\"%f\" zlo=\"%f\" xhi=\"%f\" yhi=\"%f\" zhi=\"%f\" />\n",
                      s.lo[0], s.lo[1], s.lo[2], s.hi[0], s.hi[1], s.hi[2]);
        o << b;
        put_atom_params(o, s);
        o << "<fixes>\n";
        for (Fix *f : s.fixes) {
            std::snprintf(b, sizeof(b), "<fix type=\"%s\" handle=\"%s\">", fix_type_for_restart(*f), f->handle.c_str());
            o << b << "\n" << fix_restart_chunk(*f) << "</fix>\n";
        }
        o << "</fixes>\n";
        auto vec3 = [&](const char *tag, auto get) {
            o << "<" << tag << ">\n";
            for (int i = 0; i < n; i++) {
                const double *p = get(i);
                std::snprintf(b, sizeof(b), "%f %f %f\n", p[0], p[1], p[2]);
                o << b;
            }
            o << "</" << tag << ">\n";
        };
        vec3("position", [&](int i) { return &x[3 * (size_t)i]; });
        vec3("velocity", [&](int i) { return s.atoms[i].vel; });
        vec3("force", [&](int i) { return s.atoms[i].force; });
        o << "<groupTag>\n";
        for (int i = 0; i < n; i++) o << s.atoms[i].groupTag << "\n";
        o << "</groupTag>\n<type>\n";
        for (int i = 0; i < n; i++) o << s.atoms[i].type << "\n";
        o << "</type>\n<id>\n";
        for (int i = 0; i < n; i++) o << i << "\n";
        o << "</id>\n<q>\n";
        for (int i = 0; i < n; i++) {
            std::snprintf(b, sizeof(b), "%f\n", s.atoms[i].q);
            o << b;
        }
        o << "</q>\n";
    }
    put_groups_molecules(o, s);
    o << "</configuration>\n";
    if (w.oneFilePerWrite) o << "</data>\n";
    o.close();
    if (!o) {
        set_error(MDX_ERR_ARG, "write to '%s' failed", path.c_str());
        return MDX_ERR_ARG;
    }
    return 0;
}

// writeLAMMPSTRJFile (WriteConfig.cpp:165-203) and writeXYZFile
// (WriteConfig.cpp:206-251): the group's atoms, numbers as the C++ stream
// default
static int write_traj(ConfigWriter &w, const std::string &path, int64_t turn, bool lammps, bool guessed_z) {
    State &s = *w.state;
    std::ofstream o(path, w.oneFilePerWrite ? std::ios::out : std::ios::app);
    if (!o) {
        set_error(MDX_ERR_ARG, "cannot open '%s' for writing", path.c_str());
        return MDX_ERR_ARG;
    }
    const int n = (int)s.atoms.size();
    std::vector<double> x;
    if (w.unwrapMolecules) unwrapped_positions(s, x);
    else {
        x.resize(3 * (size_t)n);
        for (int i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) x[3 * (size_t)i + d] = s.atoms[i].pos[d];
    }
    int count = 0;
    for (int i = 0; i < n; i++)
        if (w.groupBit == 1u || (s.atoms[i].groupTag & w.groupBit)) count++;
    auto g = [](double v) { return fmt_g(v); };
    if (lammps) {
        o << "ITEM: TIMESTEP\n" << turn << "\nITEM: NUMBER OF ATOMS\n" << count << "\nITEM: BOX BOUNDS pp pp pp\n";
        for (int d = 0; d < 3; d++) o << g(s.lo[d]) << " " << g(s.hi[d]) << "\n";
        o << "ITEM: ATOMS id type x y z\n";
        for (int i = 0; i < n; i++) {
            if (!(s.atoms[i].groupTag & w.groupBit)) continue;
            o << i << " " << s.atoms[i].type << " " << g(x[3 * (size_t)i]) << " " << g(x[3 * (size_t)i + 1]) << " "
              << g(x[3 * (size_t)i + 2]) << "\n";
        }
    } else {
        std::vector<int> z(s.species.size());
        bool use_z = true;
        for (size_t t = 0; t < s.species.size(); t++) {
            z[t] = guessed_z ? guess_atomic_number(s.species[t].mass) : s.species[t].atomic_num;
            if (z[t] == -1) use_z = false;
        }
        o << count << "\nbounds lo (" << g(s.lo[0]) << ", " << g(s.lo[1]) << ", " << g(s.lo[2]) << ") hi ("
          << g(s.hi[0]) << ", " << g(s.hi[1]) << ", " << g(s.hi[2]) << ")";
        for (int i = 0; i < n; i++) {
            const HostAtom &a = s.atoms[i];
            if (!(a.groupTag & w.groupBit)) continue;
            o << "\n" << (use_z ? z[a.type] : a.type);
            o << " " << g(x[3 * (size_t)i]) << " " << g(x[3 * (size_t)i + 1]) << " " << g(x[3 * (size_t)i + 2]);
            if (w.writingVelocities) o << " " << g(a.vel[0]) << " " << g(a.vel[1]) << " " << g(a.vel[2]);
            if (w.writingForces) o << " " << g(a.force[0]) << " " << g(a.force[1]) << " " << g(a.force[2]);
        }
        o << "\n";
    }
    o.close();
    if (!o) {
        set_error(MDX_ERR_ARG, "write to '%s' failed", path.c_str());
        return MDX_ERR_ARG;
    }
    return 0;
}

// WriteConfig::write (WriteConfig.cpp:427-432); from_python = writePy, which
// first guesses the species' atomic numbers from their masses in real units
static int writer_write(ConfigWriter &w, int64_t turn, bool from_python) {
    if (!w.state) {
        set_error(MDX_ERR_STATE, "the writer's state no longer exists");
        return MDX_ERR_STATE;
    }
    if (w.finished) {
        set_error(MDX_ERR_STATE, "the writer has been finished");
        return MDX_ERR_STATE;
    }
    State &s = *w.state;
    if (int e = s.download()) return e;
    const std::string path = current_fn(w, turn);
    if (w.format == "xyz")
        return write_traj(w, path, turn, false, from_python && s.units.type == MDX_UNITS_REAL);
    if (w.format == "lammpstrj") return write_traj(w, path, turn, true, false);
    return write_xml(w, path, turn, w.format == "base64");
}

static void writer_finish(ConfigWriter &w) {
    if (w.finished) return;
    w.finished = true;
    if (w.isXML && !w.oneFilePerWrite) {
        std::ofstream o(current_fn(w, 0), std::ios::app);
        o << "</data>\n";
    }
}

int64_t config_next_write(const State &s, int64_t t) {
    int64_t best = -1;
    for (const ConfigWriter *w : s.writers) {
        if (w->writeEvery <= 0 || w->finished) continue;
        const int64_t W = w->writeEvery;
        const int64_t T = ((t + W - 1) / W) * W;
        if (best < 0 || T < best) best = T;
    }
    return best;
}

int config_write_due(State &s, int64_t turn) {
    for (ConfigWriter *w : s.writers) {
        if (w->writeEvery <= 0 || w->finished || turn % w->writeEvery) continue;
        if (int e = writer_write(*w, turn, false)) return e;
    }
    return 0;
}

// ---------------------------------------------------------------- reader
struct ConfigReader {
    std::string fn;
    XNode doc;
    int cur = -1;  // index of the current configuration among doc.kids
    bool haveReadYet = false;
    const XNode *config() const { return cur >= 0 && cur < (int)doc.kids.size() ? &doc.kids[cur] : nullptr; }
};

// xml_assign (xml_func.h:14-65): a per-atom chunk either as base64 of the
// raw values (base64="1") or as whitespace-separated text
template <typename T>
static int read_chunk(const XNode &cfg, const char *tag, int width, int n, std::vector<T> &out) {
    const XNode *c = cfg.child(tag);
    if (!c) {
        set_error(MDX_ERR_ARG, "configuration has no <%s> chunk", tag);
        return MDX_ERR_ARG;
    }
    out.assign((size_t)n * width, T());
    const char *b64 = c->attr("base64");
    if (b64 && std::strcmp(b64, "1") == 0) {
        const auto tok = tokens(c->text);
        std::vector<unsigned char> raw;
        if (tok.empty() || !b64_decode(tok.back(), raw)) {
            set_error(MDX_ERR_ARG, "<%s>: bad base64 data", tag);
            return MDX_ERR_ARG;
        }
        if (raw.size() != (size_t)n * width * sizeof(T)) {
            set_error(MDX_ERR_ARG, "<%s>: %zu bytes for %d atoms", tag, raw.size(), n);
            return MDX_ERR_ARG;
        }
        std::memcpy(out.data(), raw.data(), raw.size());
        return 0;
    }
    const auto tok = tokens(c->text);
    if (tok.size() != (size_t)n * width) {
        set_error(MDX_ERR_ARG, "<%s>: %zu values for %d atoms", tag, tok.size(), n);
        return MDX_ERR_ARG;
    }
    for (size_t k = 0; k < tok.size(); k++) {
        double v;
        if (!parse_double(tok[k].c_str(), &v)) {
            set_error(MDX_ERR_ARG, "<%s>: bad number '%s'", tag, tok[k].c_str());
            return MDX_ERR_ARG;
        }
        out[k] = (T)v;
    }
    return 0;
}

// ReadConfig::read (ReadConfig.cpp:176-257): the state's atoms, species,
// bounds, groups and molecules are replaced by the configuration's.  Atom ids
// are this library's indices, so the ids read must be 0..n-1 in some order.
static int read_config(State &s, const XNode &cfg) {
    int64_t turn = 0, natoms = 0;
    double rc = 0, pad = 0, dt = 0;
    if (!parse_i64(cfg.attr("turn"), &turn) || !parse_i64(cfg.attr("numAtoms"), &natoms) || natoms < 0 ||
        !parse_double(cfg.attr("rCut"), &rc) || !parse_double(cfg.attr("padding"), &pad) ||
        !parse_double(cfg.attr("dt"), &dt)) {
        set_error(MDX_ERR_ARG, "configuration: bad turn / numAtoms / rCut / padding / dt attribute");
        return MDX_ERR_ARG;
    }
    const char *dim = cfg.attr("dimension");
    if (dim && std::strcmp(dim, "2") == 0) {
        set_error(MDX_ERR_UNSUPPORTED, "two-dimensional configurations are not supported");
        return MDX_ERR_UNSUPPORTED;
    }
    const char *per = cfg.attr("periodic");
    int periodic[3] = {1, 1, 1};
    if (per) {
        if (std::strlen(per) != 3) {
            set_error(MDX_ERR_ARG, "configuration: bad periodic attribute '%s'", per);
            return MDX_ERR_ARG;
        }
        for (int d = 0; d < 3; d++) periodic[d] = per[d] - '0';
    }
    if (periodic[0] != 1 || periodic[1] != 1 || periodic[2] != 1) {
        set_error(MDX_ERR_UNSUPPORTED, "only fully periodic boxes are supported (periodic=\"%s\")", per);
        return MDX_ERR_UNSUPPORTED;
    }
    const int n = (int)natoms;
    std::vector<double> x, v, f, q;
    std::vector<uint32_t> g;
    std::vector<int32_t> t, id;
    if (int e = read_chunk(cfg, "position", 3, n, x)) return e;
    if (int e = read_chunk(cfg, "velocity", 3, n, v)) return e;
    if (int e = read_chunk(cfg, "force", 3, n, f)) return e;
    if (int e = read_chunk(cfg, "groupTag", 1, n, g)) return e;
    if (int e = read_chunk(cfg, "type", 1, n, t)) return e;
    if (int e = read_chunk(cfg, "id", 1, n, id)) return e;
    if (int e = read_chunk(cfg, "q", 1, n, q)) return e;
    // loadAtomParams (ReadConfig.cpp:21-54)
    const XNode *ap = cfg.child("atomParams");
    if (!ap) {
        set_error(MDX_ERR_ARG, "configuration has no <atomParams>");
        return MDX_ERR_ARG;
    }
    int64_t ntypes = 0;
    if (!parse_i64(ap->attr("numTypes"), &ntypes) || ntypes < 0) {
        set_error(MDX_ERR_ARG, "<atomParams>: bad numTypes");
        return MDX_ERR_ARG;
    }
    const XNode *hn = ap->child("handle"), *mn = ap->child("mass");
    const auto handles = hn ? tokens(hn->text) : std::vector<std::string>();
    const auto masses = mn ? tokens(mn->text) : std::vector<std::string>();
    if ((int64_t)handles.size() != ntypes || (int64_t)masses.size() != ntypes) {
        set_error(MDX_ERR_ARG, "<atomParams>: %zu handles and %zu masses for %lld types", handles.size(),
                  masses.size(), (long long)ntypes);
        return MDX_ERR_ARG;
    }
    std::vector<Species> species;
    for (int64_t k = 0; k < ntypes; k++) {
        double m;
        if (!parse_double(masses[k].c_str(), &m)) {
            set_error(MDX_ERR_ARG, "<atomParams>: bad mass '%s'", masses[k].c_str());
            return MDX_ERR_ARG;
        }
        species.push_back({handles[k], m, -1});
    }
    // loadBounds (ReadConfig.cpp:56-113)
    const XNode *bn = cfg.child("bounds");
    double lo[3], hi[3];
    if (!bn) {
        set_error(MDX_ERR_ARG, "configuration has no <bounds>");
        return MDX_ERR_ARG;
    }
    {
        const char *b64 = bn->attr("base64");
        const bool enc = b64 && std::strcmp(b64, "1") == 0;
        const char *keys[6] = {"xlo", "ylo", "zlo", "xhi", "yhi", "zhi"};
        for (int k = 0; k < 6; k++) {
            const char *val = bn->attr(keys[k]);
            double r = 0;
            bool ok = val != nullptr;
            if (ok && enc) {
                std::vector<unsigned char> raw;
                ok = b64_decode(val, raw) && raw.size() == 8;
                if (ok) std::memcpy(&r, raw.data(), 8);
            } else if (ok) {
                ok = parse_double(val, &r);
            }
            if (!ok) {
                set_error(MDX_ERR_ARG, "<bounds>: bad or missing %s", keys[k]);
                return MDX_ERR_ARG;
            }
            (k < 3 ? lo[k] : hi[k - 3]) = r;
        }
        for (int d = 0; d < 3; d++)
            if (!(hi[d] > lo[d])) {
                set_error(MDX_ERR_ARG, "<bounds>: hi must exceed lo");
                return MDX_ERR_ARG;
            }
    }
    // loadGroupInfo (ReadConfig.cpp:115-139)
    std::map<std::string, uint32_t> groups{{"all", 1u}};
    if (const XNode *gi = cfg.child("groupInfo")) {
        const XNode *gh = gi->child("groupHandles"), *gb = gi->child("groupBits");
        const auto hs = gh ? tokens(gh->text) : std::vector<std::string>();
        const auto bs = gb ? tokens(gb->text) : std::vector<std::string>();
        if (hs.size() != bs.size()) {
            set_error(MDX_ERR_ARG, "bad group tag restart data");
            return MDX_ERR_ARG;
        }
        for (size_t k = 0; k < hs.size(); k++) {
            int64_t bit;
            if (!parse_i64(bs[k].c_str(), &bit)) {
                set_error(MDX_ERR_ARG, "<groupBits>: bad value '%s'", bs[k].c_str());
                return MDX_ERR_ARG;
            }
            groups[hs[k]] = (uint32_t)bit;
        }
    }
    // loadMolecules (ReadConfig.cpp:141-156)
    std::vector<std::vector<int>> mols;
    if (const XNode *ms = cfg.child("molecules")) {
        for (const XNode &m : ms->kids) {
            std::vector<int> ids;
            for (const auto &tk : tokens(m.text)) {
                int64_t k;
                if (!parse_i64(tk.c_str(), &k) || k < 0 || k >= n) {
                    set_error(MDX_ERR_ARG, "<molecules>: bad atom id '%s'", tk.c_str());
                    return MDX_ERR_ARG;
                }
                ids.push_back((int)k);
            }
            mols.push_back(ids);
        }
    }
    // atoms by id
    std::vector<HostAtom> atoms(n);
    std::vector<char> have(n, 0);
    for (int i = 0; i < n; i++) {
        const int k = id[i];
        if (k < 0 || k >= n || have[k]) {
            set_error(MDX_ERR_UNSUPPORTED, "atom ids must be 0..numAtoms-1, each once (id %d)", k);
            return MDX_ERR_UNSUPPORTED;
        }
        if (t[i] < 0 || t[i] >= ntypes) {
            set_error(MDX_ERR_ARG, "atom %d has type %d of %lld", k, t[i], (long long)ntypes);
            return MDX_ERR_ARG;
        }
        have[k] = 1;
        HostAtom &a = atoms[k];
        for (int d = 0; d < 3; d++) {
            a.pos[d] = x[3 * (size_t)i + d];
            a.vel[d] = v[3 * (size_t)i + d];
            a.force[d] = f[3 * (size_t)i + d];
        }
        a.type = t[i];
        a.mass = species[t[i]].mass;
        a.q = q[i];
        a.ndf = 3;
        a.groupTag = g[i];
    }
    // commit
    if (s.stream) cudaStreamSynchronize(s.stream);
    s.atoms.swap(atoms);
    s.species = species;
    for (int d = 0; d < 3; d++) {
        s.lo[d] = lo[d];
        s.hi[d] = hi[d];
        s.periodic[d] = periodic[d];
    }
    s.bounds_set = true;
    s.groupTags = groups;
    s.molecules = mols;
    s.turn = turn;
    s.rCut = rc;
    s.padding = pad;
    s.dt = dt;
    s.prepared = false;
    s.uploaded = false;
    return 0;
}

static const XNode *reader_fix_node(const State &s, const Fix &f) {
    if (!s.reader || !s.reader->haveReadYet) return nullptr;
    const XNode *cfg = s.reader->config();
    if (!cfg) return nullptr;
    const XNode *fx = cfg->child("fixes");
    if (!fx) return nullptr;
    for (const XNode &k : fx->kids) {
        const char *t = k.attr("type"), *h = k.attr("handle");
        if (t && h && f.type == t && f.handle == h) return &k;
    }
    return nullptr;
}

int config_fix_restart(State &s, Fix &f) {
    const XNode *node = reader_fix_node(s, f);
    if (!node) return 0;
    if (f.kind == FixKind::Pair) {
        // FixPair::readFromRestart (FixPair.cpp:211-240)
        FixPair &p = static_cast<FixPair &>(f);
        p.ensureSize();
        for (const XNode &c : node->kids) {
            if (c.name != "parameter") continue;
            const char *h = c.attr("handle");
            const std::string hs = h ? h : "";
            if (p.lj_kind == 3 && hs == "FCutHandle") continue;  // derived from rCut, sig, eps at prepare
            auto it = p.params.find(hs);
            if (it == p.params.end()) {
                set_error(MDX_ERR_ARG, "Invalid restart data for fix %s: parameter '%s'", f.handle.c_str(),
                          hs.c_str());
                return MDX_ERR_ARG;
            }
            const auto tok = tokens(c.text);
            if (tok.size() > it->second.size()) {
                set_error(MDX_ERR_ARG, "restart data for fix %s: %zu values of '%s' for %zu entries",
                          f.handle.c_str(), tok.size(), hs.c_str(), it->second.size());
                return MDX_ERR_ARG;
            }
            for (size_t k = 0; k < tok.size(); k++) {
                double v;
                if (!parse_double(tok[k].c_str(), &v)) {
                    set_error(MDX_ERR_ARG, "restart data for fix %s: bad number '%s'", f.handle.c_str(),
                              tok[k].c_str());
                    return MDX_ERR_ARG;
                }
                it->second[k] = v == -1000.0 ? std::numeric_limits<double>::quiet_NaN() : v;
            }
        }
        return 0;
    }
    if (f.kind == FixKind::Rigid) {
        // FixRigid::readFromRestart (FixRigid.cu:1458-1514)
        FixRigid &r = static_cast<FixRigid &>(f);
        bool four = true;
        std::vector<int4> ids;
        for (const XNode &c : node->kids) {
            if (c.name == "model") {
                const char *fs = c.attr("fourSite");
                four = fs && (std::strcmp(fs, "true") == 0 || std::strcmp(fs, "1") == 0);
            } else if (c.name == "style") {
                if (const char *st = c.attr("type")) r.style = st;
            }
        }
        for (const XNode &c : node->kids) {
            if (c.name != "atomsInMolecule") continue;
            const auto tok = tokens(c.text);
            if (tok.size() % 4) {
                set_error(MDX_ERR_ARG, "restart data for fix %s: atomsInMolecule holds %zu ids", f.handle.c_str(),
                          tok.size());
                return MDX_ERR_ARG;
            }
            for (size_t k = 0; k < tok.size(); k += 4) {
                int64_t a[4];
                for (int j = 0; j < 4; j++)
                    if (!parse_i64(tok[k + j].c_str(), &a[j])) {
                        set_error(MDX_ERR_ARG, "restart data for fix %s: bad atom id", f.handle.c_str());
                        return MDX_ERR_ARG;
                    }
                ids.push_back(make_int4((int)a[0], (int)a[1], (int)a[2], four ? (int)a[3] : -1));
            }
        }
        r.mol_ids.clear();
        r.foursite = r.threesite = false;
        for (const int4 &m : ids)
            if (int e = r.createRigid(m.x, m.y, m.z, m.w)) return e;
        return 0;
    }
    return 0;
}

void config_state_detach(State &s) {
    for (ConfigWriter *w : s.writers) w->state = nullptr;
    s.writers.clear();
    delete s.reader;
    s.reader = nullptr;
}

static int reader_load(State &s, const char *fn) {
    std::ifstream in(fn, std::ios::binary);
    if (!in) {
        set_error(MDX_ERR_ARG, "cannot open '%s'", fn);
        return MDX_ERR_ARG;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string src = ss.str();
    auto *r = new ConfigReader();
    r->fn = fn;
    XParser p(src);
    if (!p.document(r->doc)) {
        set_error(MDX_ERR_ARG, "XML [%s] parsed with errors: %s", fn, p.err.c_str());
        delete r;
        return MDX_ERR_ARG;
    }
    delete s.reader;
    s.reader = r;
    return 0;
}

// ReadConfig::next / prev / moveBy (ReadConfig.cpp:259-315); a negative
// moveBy steps back through the file
static int reader_move(State &s, int op, int by, int *found) {
    *found = 0;
    ConfigReader *r = s.reader;
    if (!r) {
        set_error(MDX_ERR_STATE, "no configuration file loaded (readConfig.loadFile)");
        return MDX_ERR_STATE;
    }
    const int nk = (int)r->doc.kids.size();
    int cur = r->cur;
    const bool fresh = cur < 0 || !r->haveReadYet;
    if (op == 0) {
        cur = fresh ? 0 : cur + 1;
    } else if (op == 1) {
        cur = fresh ? nk - 1 : cur - 1;
    } else {
        if (by == 0) {
            *found = r->config() != nullptr;
            return 0;
        }
        if (fresh) {
            if (by < 0) return 0;
            cur = 0;
            by--;
        }
        cur += by;
    }
    if (cur < 0 || cur >= nk) {
        r->cur = -1;
        return 0;
    }
    r->cur = cur;
    r->haveReadYet = true;
    if (int e = read_config(s, r->doc.kids[cur])) return e;
    *found = 1;
    return 0;
}

}  // namespace mdx

using namespace mdx;

struct mdx_writer {
    ConfigWriter *w;
};

#define IO_ARG(cond, msg)                  \
    do {                                   \
        if (!(cond)) {                     \
            set_error(MDX_ERR_ARG, "%s", msg); \
            return MDX_ERR_ARG;            \
        }                                  \
    } while (0)

extern "C" {

int mdx_write_config_create(mdx_state *st, const char *fn, const char *handle, const char *format, int write_every,
                            const char *group_handle, int unwrap_molecules, mdx_writer **out) {
    IO_ARG(st && fn && handle && format && out, "null argument");
    IO_ARG(write_every >= 0, "writeEvery must be >= 0");
    State &s = *st->s;
    auto *w = new ConfigWriter();
    w->state = &s;
    w->fn = fn;
    w->handle = handle;
    w->format = format;
    w->writeEvery = write_every;
    w->groupHandle = group_handle ? group_handle : "all";
    w->unwrapMolecules = unwrap_molecules != 0;
    auto g = s.groupTags.find(w->groupHandle);
    if (g == s.groupTags.end()) {
        delete w;
        set_error(MDX_ERR_ARG, "no group '%s'", group_handle);
        return MDX_ERR_ARG;
    }
    w->groupBit = g->second;
    w->isXML = !(w->format == "xyz" || w->format == "lammpstrj");
    w->oneFilePerWrite = w->fn.find('*') != std::string::npos;
    if (!w->oneFilePerWrite) {
        // WriteConfig::WriteConfig (WriteConfig.cpp:389-416): start the file
        const std::string path = current_fn(*w, 0);
        unlink(path.c_str());
        if (w->isXML) {
            std::ofstream o(path, std::ios::app);
            if (!o) {
                delete w;
                set_error(MDX_ERR_ARG, "cannot open '%s' for writing", path.c_str());
                return MDX_ERR_ARG;
            }
            o << "<data>\n";
        }
    }
    *out = new mdx_writer{w};
    return 0;
}

int mdx_write_config_set(mdx_writer *w, const char *key, int64_t value) {
    IO_ARG(w && key, "null argument");
    const std::string k = key;
    if (k == "writeEvery") {
        IO_ARG(value >= 0, "writeEvery must be >= 0");
        w->w->writeEvery = (int)value;
    } else if (k == "unwrapMolecules") w->w->unwrapMolecules = value != 0;
    else if (k == "writingVelocities") w->w->writingVelocities = value != 0;
    else if (k == "writingForces") w->w->writingForces = value != 0;
    else {
        set_error(MDX_ERR_ARG, "unknown WriteConfig key '%s'", key);
        return MDX_ERR_ARG;
    }
    return 0;
}

int mdx_write_config_write(mdx_writer *w, int64_t turn) {
    IO_ARG(w, "null writer");
    try {
        if (w->w->state && turn < 0) {
            if (int e = w->w->state->download()) return e;
            turn = w->w->state->turn;
        }
        return writer_write(*w->w, turn, true);
    } catch (const std::exception &ex) {
        set_error(MDX_ERR_STATE, "exception: %s", ex.what());
        return MDX_ERR_STATE;
    }
}

int mdx_write_config_destroy(mdx_writer *w) {
    if (!w) return 0;
    writer_finish(*w->w);
    if (State *s = w->w->state) {
        auto &v = s->writers;
        v.erase(std::remove(v.begin(), v.end(), w->w), v.end());
    }
    delete w->w;
    delete w;
    return 0;
}

int mdx_state_activate_write_config(mdx_state *st, mdx_writer *w) {
    IO_ARG(st && w, "null argument");
    IO_ARG(w->w->state == st->s, "the writer belongs to another state");
    auto &v = st->s->writers;
    if (std::find(v.begin(), v.end(), w->w) == v.end()) v.push_back(w->w);
    return 0;
}

int mdx_state_deactivate_write_config(mdx_state *st, mdx_writer *w) {
    IO_ARG(st && w, "null argument");
    auto &v = st->s->writers;
    auto it = std::find(v.begin(), v.end(), w->w);
    if (it == v.end()) {
        set_error(MDX_ERR_ARG, "the writer is not active");
        return MDX_ERR_ARG;
    }
    v.erase(it);
    return 0;
}

int mdx_read_config_load(mdx_state *st, const char *fn) {
    IO_ARG(st && fn, "null argument");
    try {
        return reader_load(*st->s, fn);
    } catch (const std::exception &ex) {
        set_error(MDX_ERR_STATE, "exception: %s", ex.what());
        return MDX_ERR_STATE;
    }
}

int mdx_read_config_move(mdx_state *st, int op, int by, int *found) {
    IO_ARG(st && found, "null argument");
    IO_ARG(op >= 0 && op <= 2, "op must be 0 (next), 1 (prev) or 2 (moveBy)");
    try {
        return reader_move(*st->s, op, by, found);
    } catch (const std::exception &ex) {
        set_error(MDX_ERR_STATE, "exception: %s", ex.what());
        return MDX_ERR_STATE;
    }
}

int mdx_state_create_group(mdx_state *st, const char *handle, int n, const int *ids) {
    IO_ARG(st && handle && n >= 0 && (n == 0 || ids), "null argument");
    State &s = *st->s;
    if (s.groupTags.count(handle)) {
        set_error(MDX_ERR_ARG, "group '%s' already exists", handle);
        return MDX_ERR_ARG;
    }
    uint32_t used = 0;
    for (const auto &g : s.groupTags) used |= g.second;
    uint32_t bit = 0;
    for (int k = 1; k < 32; k++)
        if (!(used & (1u << k))) {
            bit = 1u << k;
            break;
        }
    if (!bit) {
        set_error(MDX_ERR_ARG, "no free group bits (32 groups at most)");
        return MDX_ERR_ARG;
    }
    for (int i = 0; i < n; i++)
        IO_ARG(ids[i] >= 0 && ids[i] < (int)s.atoms.size(), "createGroup: atom id out of range");
    if (n) {
        // the tag bits ride in the device force stream: bring the host copy
        // up to date, and upload again at the next prepare
        if (int e = s.download()) return e;
        s.prepared = false;
    }
    s.groupTags[handle] = bit;
    for (int i = 0; i < n; i++) s.atoms[ids[i]].groupTag |= bit;
    return 0;
}

int mdx_write_output(mdx_state *st) {
    IO_ARG(st, "null state");
    State &s = *st->s;
    try {
        if (int e = s.download()) return e;
        for (ConfigWriter *w : s.writers)
            if (int e = writer_write(*w, s.turn, false)) return e;
    } catch (const std::exception &ex) {
        set_error(MDX_ERR_STATE, "exception: %s", ex.what());
        return MDX_ERR_STATE;
    }
    return 0;
}

int mdx_state_get_bounds(mdx_state *st, double lo[3], double hi[3]) {
    IO_ARG(st && lo && hi, "null argument");
    IO_ARG(st->s->bounds_set, "bounds not set");
    for (int d = 0; d < 3; d++) {
        lo[d] = st->s->lo[d];
        hi[d] = st->s->hi[d];
    }
    return 0;
}

int mdx_state_get_species(mdx_state *st, int k, char *handle, int cap, double *mass, int *atomic_num, int *count) {
    IO_ARG(st, "null state");
    const State &s = *st->s;
    if (count) *count = (int)s.species.size();
    if (k < 0) return 0;
    IO_ARG(k < (int)s.species.size(), "species index out of range");
    const Species &sp = s.species[k];
    if (handle) {
        IO_ARG(cap > (int)sp.handle.size(), "handle buffer too small");
        std::memcpy(handle, sp.handle.c_str(), sp.handle.size() + 1);
    }
    if (mass) *mass = sp.mass;
    if (atomic_num) *atomic_num = sp.atomic_num;
    return 0;
}

int mdx_state_group_tag(mdx_state *st, const char *handle, uint32_t *bit) {
    IO_ARG(st && handle && bit, "null argument");
    auto it = st->s->groupTags.find(handle);
    if (it == st->s->groupTags.end()) {
        set_error(MDX_ERR_ARG, "no group '%s'", handle);
        return MDX_ERR_ARG;
    }
    *bit = it->second;
    return 0;
}

int mdx_state_create_molecule(mdx_state *st, int n, const int *ids) {
    IO_ARG(st && n > 0 && ids, "null argument");
    State &s = *st->s;
    for (int i = 0; i < n; i++) IO_ARG(ids[i] >= 0 && ids[i] < (int)s.atoms.size(), "createMolecule: bad atom id");
    s.molecules.emplace_back(ids, ids + n);
    return 0;
}

}  // extern "C"

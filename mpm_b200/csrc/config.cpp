// config.cpp -- YAML scene configuration, .xyz point clouds and the solver
// builder (include/mpm_b200_config.h).
//
// Follows parseYAML (src/mpm3d_parser.cpp:20-71), readXYZFile and the two
// builders (src/mpm_solver3d_builder.cu:10-129) of the reference.  The YAML
// reader is a small self-contained subset parser: block mappings and
// sequences by indentation, "- key: value" sequence items, flow sequences
// [a, b, c], plain and quoted scalars, and # comments -- everything the
// reference's configuration files use.
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../../include/mpm_b200.h"
#include "../../include/mpm_b200_config.h"

namespace mpm {

mpm_status recordError(mpm_status st, const char* msg);

namespace {

// ---------------------------------------------------------------------------
// YAML subset
// ---------------------------------------------------------------------------
struct YNode {
    enum Kind { SCALAR, MAP, SEQ } kind = SCALAR;
    std::string scalar;
    std::vector<std::pair<std::string, YNode>> map;
    std::vector<YNode> seq;
    int line = 0;

    const YNode* get(const std::string& k) const {
        if (kind != MAP) return nullptr;
        for (auto& kv : map)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

struct YLine {
    int indent;
    std::string text;  // without indentation and comment
    int number;
};

struct ParseError {
    std::string msg;
};

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

std::string stripComment(const std::string& s) {
    bool sq = false, dq = false;
    for (size_t i = 0; i < s.size(); ++i) {
        char c = s[i];
        if (c == '\'' && !dq) sq = !sq;
        else if (c == '"' && !sq) dq = !dq;
        else if (c == '#' && !sq && !dq && (i == 0 || std::isspace((unsigned char)s[i - 1]))) return s.substr(0, i);
    }
    return s;
}

std::string unquote(const std::string& s) {
    if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
        return s.substr(1, s.size() - 2);
    return s;
}

// Position of the "key:" separator (a colon followed by space or end), or npos.
size_t keyColon(const std::string& s) {
    bool sq = false, dq = false;
    for (size_t i = 0; i < s.size(); ++i) {
        char c = s[i];
        if (c == '\'' && !dq) sq = !sq;
        else if (c == '"' && !sq) dq = !dq;
        else if (c == ':' && !sq && !dq && (i + 1 == s.size() || s[i + 1] == ' ' || s[i + 1] == '\t')) return i;
    }
    return std::string::npos;
}

YNode parseFlowOrScalar(const std::string& raw, int line) {
    std::string v = trim(raw);
    YNode n;
    n.line = line;
    if (!v.empty() && v.front() == '[') {
        if (v.back() != ']') throw ParseError{"line " + std::to_string(line) + ": unterminated flow sequence"};
        n.kind = YNode::SEQ;
        std::string body = v.substr(1, v.size() - 2);
        int depth = 0;
        std::string cur;
        for (char c : body) {
            if (c == '[') ++depth;
            if (c == ']') --depth;
            if (c == ',' && depth == 0) {
                if (!trim(cur).empty()) n.seq.push_back(parseFlowOrScalar(cur, line));
                cur.clear();
            } else {
                cur += c;
            }
        }
        if (!trim(cur).empty()) n.seq.push_back(parseFlowOrScalar(cur, line));
        return n;
    }
    n.kind = YNode::SCALAR;
    n.scalar = unquote(v);
    return n;
}

class YParser {
public:
    explicit YParser(const std::string& text) {
        std::istringstream in(text);
        std::string l;
        int no = 0;
        while (std::getline(in, l)) {
            ++no;
            for (auto& c : l)
                if (c == '\t') c = ' ';
            std::string s = stripComment(l);
            if (trim(s).empty()) continue;
            if (trim(s) == "---" || trim(s) == "...") continue;
            int ind = 0;
            while (ind < (int)s.size() && s[ind] == ' ') ++ind;
            lines_.push_back({ind, trim(s), no});
        }
    }

    YNode parse() {
        if (lines_.empty()) {
            YNode n;
            n.kind = YNode::MAP;
            return n;
        }
        size_t i = 0;
        YNode root = parseBlock(i, lines_[0].indent);
        if (i != lines_.size())
            throw ParseError{"line " + std::to_string(lines_[i].number) + ": unexpected indentation"};
        return root;
    }

private:
    std::vector<YLine> lines_;

    YNode parseBlock(size_t& i, int indent) {
        if (lines_[i].text.rfind("- ", 0) == 0 || lines_[i].text == "-") return parseSeq(i, indent);
        return parseMap(i, indent, nullptr);
    }

    // Mapping whose keys sit at column `indent`.  `first` is an already
    // split first line (used by "- key: value" sequence items).
    YNode parseMap(size_t& i, int indent, const std::string* first) {
        YNode m;
        m.kind = YNode::MAP;
        m.line = i < lines_.size() ? lines_[i].number : 0;
        bool use_first = first != nullptr;
        while (use_first || (i < lines_.size() && lines_[i].indent == indent)) {
            std::string text;
            int lineno;
            if (use_first) {
                text = *first;
                lineno = lines_[i - 1].number;
                use_first = false;
            } else {
                text = lines_[i].text;
                lineno = lines_[i].number;
                if (text.rfind("- ", 0) == 0 || text == "-") break;
                ++i;
            }
            size_t c = keyColon(text);
            if (c == std::string::npos) throw ParseError{"line " + std::to_string(lineno) + ": expected 'key: value'"};
            std::string key = unquote(trim(text.substr(0, c)));
            std::string val = trim(text.substr(c + 1));
            YNode child;
            if (!val.empty()) {
                child = parseFlowOrScalar(val, lineno);
            } else if (i < lines_.size() && lines_[i].indent > indent) {
                child = parseBlock(i, lines_[i].indent);
            } else if (i < lines_.size() && lines_[i].indent == indent &&
                       (lines_[i].text.rfind("- ", 0) == 0 || lines_[i].text == "-")) {
                child = parseSeq(i, indent);  // "key:\n- item" at the key's column
            } else {
                child.kind = YNode::SCALAR;  // empty value
                child.line = lineno;
            }
            m.map.emplace_back(key, std::move(child));
        }
        return m;
    }

    YNode parseSeq(size_t& i, int indent) {
        YNode s;
        s.kind = YNode::SEQ;
        s.line = lines_[i].number;
        while (i < lines_.size() && lines_[i].indent == indent &&
               (lines_[i].text.rfind("- ", 0) == 0 || lines_[i].text == "-")) {
            const std::string& t = lines_[i].text;
            std::string rest = t == "-" ? std::string() : trim(t.substr(1));
            // column of the item's first key: after the dash and its spaces
            const size_t key_pos = t.find_first_not_of(' ', 1);
            const int item_col = indent + (int)(key_pos == std::string::npos ? 2 : key_pos);
            ++i;
            if (rest.empty()) {
                if (i < lines_.size() && lines_[i].indent > indent) s.seq.push_back(parseBlock(i, lines_[i].indent));
                else s.seq.push_back(YNode{});
            } else if (keyColon(rest) != std::string::npos && rest.front() != '[') {
                // "- key: value" opens a mapping whose later keys align with `key`
                s.seq.push_back(parseMap(i, item_col, &rest));
            } else {
                s.seq.push_back(parseFlowOrScalar(rest, lines_[i - 1].number));
            }
        }
        return s;
    }
};

// ---------------------------------------------------------------------------
// Typed access
// ---------------------------------------------------------------------------
const YNode& need(const YNode& n, const char* key, const std::string& where) {
    const YNode* c = n.get(key);
    if (!c) throw ParseError{"missing key " + where + key};
    return *c;
}

double asDouble(const YNode& n, const std::string& what) {
    if (n.kind != YNode::SCALAR || n.scalar.empty()) throw ParseError{what + ": expected a number"};
    char* end = nullptr;
    errno = 0;
    double v = std::strtod(n.scalar.c_str(), &end);
    if (end == n.scalar.c_str() || *end != '\0' || errno == ERANGE)
        throw ParseError{what + ": '" + n.scalar + "' is not a number"};
    return v;
}

long asInt(const YNode& n, const std::string& what) {
    double v = asDouble(n, what);
    if (v != (double)(long)v) throw ParseError{what + ": '" + n.scalar + "' is not an integer"};
    return (long)v;
}

bool asBool(const YNode& n, const std::string& what) {
    std::string s;
    for (char c : n.scalar) s += (char)std::tolower((unsigned char)c);
    if (s == "true" || s == "yes" || s == "on" || s == "1") return true;
    if (s == "false" || s == "no" || s == "off" || s == "0") return false;
    throw ParseError{what + ": '" + n.scalar + "' is not a boolean"};
}

void asVec3(const YNode& n, const std::string& what, double* out) {
    if (n.kind != YNode::SEQ || n.seq.size() != 3) throw ParseError{what + ": expected [x, y, z]"};
    for (int i = 0; i < 3; ++i) out[i] = asDouble(n.seq[i], what);
}

// parseConstitutiveModel / parseInterpolationType (src/mpm3d_parser.cpp:7-18)
int constitutiveModel(const std::string& s) {
    if (s == "FixedCorotated") return MPM_MODEL_FIXED_COROTATED;
    if (s == "NeoHookean") return MPM_MODEL_NEO_HOOKEAN;
    throw ParseError{"Unsupported constitutive model: " + s};
}
int interpolationType(const std::string& s) {
    if (s == "Linear") return MPM_INTERP_LINEAR;
    if (s == "QuadraticBSpline") return MPM_INTERP_QUADRATIC_BSPLINE;
    if (s == "CubicBSpline") return MPM_INTERP_CUBIC_BSPLINE;
    throw ParseError{"Unsupported interpolation type: " + s};
}

void copyStr(char* dst, size_t cap, const std::string& s) {
    std::strncpy(dst, s.c_str(), cap - 1);
    dst[cap - 1] = '\0';
}

mpm_config* buildConfig(const YNode& root, const std::string& base_dir) {
    if (root.kind != YNode::MAP) throw ParseError{"top level must be a mapping"};
    std::unique_ptr<mpm_config> cfg(new mpm_config());
    std::memset(cfg.get(), 0, sizeof(mpm_config));
    const YNode& groups = need(root, "ParticleGroups", "");
    if (groups.kind != YNode::SEQ) throw ParseError{"ParticleGroups must be a sequence"};
    std::vector<mpm_config_group> gv;
    for (size_t i = 0; i < groups.seq.size(); ++i) {
        const YNode& g = groups.seq[i];
        std::string w = "ParticleGroups[" + std::to_string(i) + "].";
        mpm_config_group cg;
        std::memset(&cg, 0, sizeof(cg));
        copyStr(cg.file, sizeof(cg.file), need(g, "File", w).scalar);
        cg.mass = (float)asDouble(need(g, "Mass", w), w + "Mass");
        double v[3];
        asVec3(need(g, "Velocity", w), w + "Velocity", v);
        for (int a = 0; a < 3; ++a) cg.velocity[a] = (float)v[a];
        cg.material.youngs_modulus = (float)asDouble(need(g, "YoungModulus", w), w + "YoungModulus");
        cg.material.poisson_ratio = (float)asDouble(need(g, "PoissonRatio", w), w + "PoissonRatio");
        cg.material.hardening = (float)asDouble(need(g, "HardeningCoefficient", w), w + "HardeningCoefficient");
        cg.material.critical_compression = (float)asDouble(need(g, "CriticalCompression", w), w + "CriticalCompression");
        cg.material.critical_stretch = (float)asDouble(need(g, "CriticalStretch", w), w + "CriticalStretch");
        cg.material.model = constitutiveModel(need(g, "ConstitutiveModel", w).scalar);
        gv.push_back(cg);
    }
    const YNode& grid = need(root, "Grid", "");
    double o[3], r[3];
    asVec3(need(grid, "Origin", "Grid."), "Grid.Origin", o);
    asVec3(need(grid, "Resolution", "Grid."), "Grid.Resolution", r);
    for (int a = 0; a < 3; ++a) {
        cfg->origin[a] = (float)o[a];
        if (r[a] != (double)(long)r[a]) throw ParseError{"Grid.Resolution: integers expected"};
        cfg->resolution[a] = (int32_t)r[a];
    }
    cfg->stride = (float)asDouble(need(grid, "Stride", "Grid."), "Grid.Stride");
    cfg->friction = (float)asDouble(need(grid, "BoundaryFrictionCoefficient", "Grid."), "Grid.BoundaryFrictionCoefficient");
    cfg->blend = (float)asDouble(need(need(root, "Transfer", ""), "BlendCoefficient", "Transfer."), "Transfer.BlendCoefficient");
    cfg->interpolation = interpolationType(need(need(root, "Interpolation", ""), "Type", "Interpolation.").scalar);
    const YNode& sim = need(root, "Simulate", "");
    cfg->dt = (float)asDouble(need(sim, "deltaTime", "Simulate."), "Simulate.deltaTime");
    if (const YNode* render = root.get("Render")) {
        if (const YNode* off = render->get("Offline")) cfg->offline = asBool(*off, "Render.Offline") ? 1 : 0;
        if (const YNode* sh = render->get("ParticleFragmentShader"))
            copyStr(cfg->particle_frag_shader, sizeof(cfg->particle_frag_shader), sh->scalar);
    }
    // extensions
    cfg->gravity = 9.80665f;
    if (const YNode* gr = sim.get("Gravity")) cfg->gravity = (float)asDouble(*gr, "Simulate.Gravity");
    cfg->transfer = -1;
    if (const YNode* t = sim.get("Transfer")) {
        if (t->scalar == "APIC") cfg->transfer = MPM_TRANSFER_APIC;
        else if (t->scalar == "PICFLIP" || t->scalar == "PIC-FLIP") cfg->transfer = MPM_TRANSFER_PIC_FLIP;
        else throw ParseError{"Unsupported transfer: " + t->scalar};
    }
    cfg->boundary = MPM_BOUNDARY_REFERENCE;
    cfg->sticky_cells = 3;
    if (const YNode* b = grid.get("Boundary")) {
        if (b->scalar == "Reference") cfg->boundary = MPM_BOUNDARY_REFERENCE;
        else if (b->scalar == "Sticky") cfg->boundary = MPM_BOUNDARY_STICKY;
        else throw ParseError{"Unsupported boundary: " + b->scalar};
    }
    if (const YNode* sc = grid.get("StickyCells")) cfg->sticky_cells = (int32_t)asInt(*sc, "Grid.StickyCells");
    copyStr(cfg->base_dir, sizeof(cfg->base_dir), base_dir);
    cfg->ngroups = (int32_t)gv.size();
    cfg->groups = (mpm_config_group*)std::calloc(gv.size() ? gv.size() : 1, sizeof(mpm_config_group));
    if (!cfg->groups) throw std::bad_alloc();
    for (size_t i = 0; i < gv.size(); ++i) cfg->groups[i] = gv[i];
    return cfg.release();
}

std::string dirOf(const std::string& path) {
    size_t p = path.find_last_of('/');
    return p == std::string::npos ? std::string(".") : path.substr(0, p == 0 ? 1 : p);
}

bool readFile(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

}  // namespace
}  // namespace mpm

using mpm::ParseError;

extern "C" {

mpm_status mpm_config_parse_yaml_string(const char* text, const char* base_dir, mpm_config** out) {
    if (!text || !out) return mpm::recordError(MPM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    try {
        mpm::YParser p(text);
        mpm::YNode root = p.parse();
        *out = mpm::buildConfig(root, base_dir ? base_dir : ".");
        return MPM_OK;
    } catch (const ParseError& e) {
        return mpm::recordError(MPM_ERR_PARSE, e.msg.c_str());
    } catch (const std::bad_alloc&) {
        return mpm::recordError(MPM_ERR_OOM, "host allocation failed");
    }
}

mpm_status mpm_config_parse_yaml(const char* path, mpm_config** out) {
    if (!path || !out) return mpm::recordError(MPM_ERR_INVALID_ARG, "null argument");
    std::string text;
    if (!mpm::readFile(path, text))
        return mpm::recordError(MPM_ERR_IO, (std::string("cannot open ") + path).c_str());
    return mpm_config_parse_yaml_string(text.c_str(), mpm::dirOf(path).c_str(), out);
}

mpm_status mpm_config_free(mpm_config* cfg) {
    if (!cfg) return MPM_OK;
    std::free(cfg->groups);
    delete cfg;
    return MPM_OK;
}

void mpm_free(void* p) { std::free(p); }

// readXYZFile (src/mpm_solver3d_builder.cu:10-30) and the builder's
// `config.stride * coords[j]` (:44).  Blank lines are skipped; a malformed
// line is an error (the reference stops reading there and keeps the points
// read so far without telling the caller).
mpm_status mpm_read_xyz(const char* path, const char* base_dir, float stride, float** points, size_t* n) {
    if (!path || !points || !n) return mpm::recordError(MPM_ERR_INVALID_ARG, "null argument");
    *points = nullptr;
    *n = 0;
    std::string text;
    std::string p = path;
    if (!mpm::readFile(p, text)) {
        bool ok = false;
        if (base_dir && p.size() && p[0] != '/') {
            p = std::string(base_dir) + "/" + path;
            ok = mpm::readFile(p, text);
        }
        if (!ok) return mpm::recordError(MPM_ERR_IO, (std::string("cannot open file ") + path).c_str());
    }
    std::vector<float> v;
    std::istringstream in(text);
    std::string line;
    int no = 0;
    while (std::getline(in, line)) {
        ++no;
        if (mpm::trim(line).empty()) continue;
        std::stringstream ss(line);
        float x, y, z;
        if (!(ss >> x >> y >> z))
            return mpm::recordError(MPM_ERR_PARSE, (std::string("cannot parse line ") + std::to_string(no) +
                                                    " of " + p).c_str());
        v.push_back(stride * x);
        v.push_back(stride * y);
        v.push_back(stride * z);
    }
    float* out = (float*)std::malloc(sizeof(float) * (v.size() ? v.size() : 1));
    if (!out) return mpm::recordError(MPM_ERR_OOM, "host allocation failed");
    if (!v.empty()) std::memcpy(out, v.data(), sizeof(float) * v.size());
    *points = out;
    *n = v.size() / 3;
    return MPM_OK;
}

// buildMPMSolver3DFromYAML / buildAPICMPMSolver3DFromYAML
// (src/mpm_solver3d_builder.cu:32-129).
mpm_status mpm_solver_create_from_config(const mpm_config* cfg, int32_t transfer, mpm_solver** out,
                                         int32_t* particles_number) {
    if (!cfg || !out) return mpm::recordError(MPM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (transfer < 0) transfer = cfg->transfer;
    if (transfer != MPM_TRANSFER_PIC_FLIP && transfer != MPM_TRANSFER_APIC)
        return mpm::recordError(MPM_ERR_INVALID_ARG, "no transfer given (PIC-FLIP or APIC)");
    std::vector<float> x, v, m;
    std::vector<uint16_t> mat;
    std::vector<mpm_material> mats;
    for (int32_t g = 0; g < cfg->ngroups; ++g) {
        const mpm_config_group& grp = cfg->groups[g];
        float* pts = nullptr;
        size_t n = 0;
        mpm_status st = mpm_read_xyz(grp.file, cfg->base_dir, cfg->stride, &pts, &n);
        if (st != MPM_OK) return st;
        x.insert(x.end(), pts, pts + 3 * n);
        mpm_free(pts);
        for (size_t i = 0; i < n; ++i) {
            for (int a = 0; a < 3; ++a) v.push_back(grp.velocity[a]);
            m.push_back(grp.mass);
            mat.push_back((uint16_t)g);
        }
        mats.push_back(grp.material);
    }
    if (mats.empty()) return mpm::recordError(MPM_ERR_INVALID_ARG, "configuration has no particle groups");
    mpm_scene_desc d;
    std::memset(&d, 0, sizeof(d));
    for (int a = 0; a < 3; ++a) {
        d.origin[a] = cfg->origin[a];
        d.resolution[a] = cfg->resolution[a];
    }
    d.stride = cfg->stride;
    d.friction = cfg->friction;
    d.blend = cfg->blend;
    d.dt = cfg->dt;
    d.gravity = cfg->gravity;
    d.transfer = transfer;
    d.interpolation = cfg->interpolation;
    d.boundary = cfg->boundary;
    d.sticky_cells = cfg->sticky_cells;
    d.volume_mode = MPM_VOLUME_GRID_ESTIMATE;
    d.particles_collision = 0;
    mpm_particles_in p;
    std::memset(&p, 0, sizeof(p));
    p.n = m.size();
    p.position = x.data();
    p.velocity = v.data();
    p.mass = m.data();
    p.material = mats.size() > 1 ? mat.data() : nullptr;
    p.materials = mats.data();
    p.nmaterials = (int32_t)mats.size();
    mpm_status st = mpm_solver_create(&d, &p, out);
    if (st == MPM_OK && particles_number) *particles_number = (int32_t)m.size();
    return st;
}

}  // extern "C"

// Dependency-free readers for milupHPC's two configuration surfaces.
//
// .info: Boost property-tree INFO syntax as read by ConfigParser
// (src/utils/config_parser.cpp:6-15) — `key value` pairs, `;` comments,
// quoted strings, `{ }` sub-trees.  The keys and their meaning are those read
// in src/main.cpp:165-237 (`smoothing` is eps^2, `theta` the opening
// parameter, `sfc` 0/1, `integrator` 0/1/2, ...).
//
// .cfg: the libconfig `materials = ( { ... }, ... );` list read by
// MaterialHandler(const char*) (src/materials/material_handler.cpp:58-150):
// ID, interactions, sml, artificial_viscosity {alpha, beta},
// eos {type, polytropic_K, polytropic_gamma, rho_0, bulk_modulus, n,
// shear_modulus}.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mhpc.h"

namespace {

std::string read_file(const char* path, bool* ok) {
    std::ifstream f(path);
    if (!f) { *ok = false; return {}; }
    std::stringstream ss;
    ss << f.rdbuf();
    *ok = true;
    return ss.str();
}

// --------------------------------------------------------------- .info
void parse_info(const std::string& text, std::map<std::string, std::string>& kv) {
    std::istringstream in(text);
    std::string line;
    int depth = 0;
    while (std::getline(in, line)) {
        std::string cur;
        bool quoted = false;
        std::vector<std::string> tok;
        for (size_t i = 0; i < line.size(); ++i) {
            char c = line[i];
            if (quoted) {
                if (c == '"') { quoted = false; tok.push_back(cur); cur.clear(); }
                else cur += c;
                continue;
            }
            if (c == ';') break;
            if (c == '"') { quoted = true; continue; }
            if (c == '{') { if (!cur.empty()) { tok.push_back(cur); cur.clear(); } ++depth; continue; }
            if (c == '}') { if (!cur.empty()) { tok.push_back(cur); cur.clear(); } --depth; continue; }
            if (std::isspace((unsigned char)c)) { if (!cur.empty()) { tok.push_back(cur); cur.clear(); } continue; }
            cur += c;
        }
        if (!cur.empty()) tok.push_back(cur);
        if (depth == 0 && tok.size() >= 2) kv[tok[0]] = tok[1];
        else if (depth == 0 && tok.size() == 1) kv[tok[0]] = "";
    }
}

bool as_bool(const std::string& v) {
    return v == "true" || v == "1" || v == "True" || v == "TRUE" || v == "yes";
}

// --------------------------------------------------------------- .cfg
struct Val {
    enum Kind { Scalar, Group, List } kind = Scalar;
    std::string s;
    std::map<std::string, std::shared_ptr<Val>> g;
    std::vector<std::shared_ptr<Val>> l;
};

struct Lexer {
    const std::string& t;
    size_t i = 0;
    explicit Lexer(const std::string& s) : t(s) {}
    void skip() {
        for (;;) {
            while (i < t.size() && std::isspace((unsigned char)t[i])) ++i;
            if (i < t.size() && t[i] == '#') { while (i < t.size() && t[i] != '\n') ++i; continue; }
            if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '/') { while (i < t.size() && t[i] != '\n') ++i; continue; }
            if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '*') {
                size_t e = t.find("*/", i + 2);
                i = e == std::string::npos ? t.size() : e + 2;
                continue;
            }
            break;
        }
    }
    char peek() { skip(); return i < t.size() ? t[i] : '\0'; }
    std::string word() {
        skip();
        std::string w;
        if (i < t.size() && t[i] == '"') {
            ++i;
            while (i < t.size() && t[i] != '"') w += t[i++];
            if (i < t.size()) ++i;
            return w;
        }
        while (i < t.size() && (std::isalnum((unsigned char)t[i]) || t[i] == '_' || t[i] == '.' || t[i] == '-' ||
                                t[i] == '+'))
            w += t[i++];
        return w;
    }
};

std::shared_ptr<Val> parse_value(Lexer& L, bool* ok, int depth);

void parse_settings(Lexer& L, std::map<std::string, std::shared_ptr<Val>>& g, char close, bool* ok, int depth) {
    while (*ok) {
        char c = L.peek();
        if (c == close || c == '\0') { if (c == close && close) ++L.i; return; }
        std::string name = L.word();
        if (name.empty()) { *ok = false; return; }
        c = L.peek();
        if (c != '=' && c != ':') { *ok = false; return; }
        ++L.i;
        g[name] = parse_value(L, ok, depth + 1);
        c = L.peek();
        if (c == ';' || c == ',') ++L.i;
    }
}

std::shared_ptr<Val> parse_value(Lexer& L, bool* ok, int depth) {
    auto v = std::make_shared<Val>();
    if (depth > 64) { *ok = false; return v; }
    char c = L.peek();
    if (c == '{') {
        ++L.i;
        v->kind = Val::Group;
        parse_settings(L, v->g, '}', ok, depth);
    } else if (c == '(' || c == '[') {
        char close = c == '(' ? ')' : ']';
        ++L.i;
        v->kind = Val::List;
        while (*ok) {
            char d = L.peek();
            if (d == close) { ++L.i; break; }
            if (d == '\0') { *ok = false; break; }
            v->l.push_back(parse_value(L, ok, depth + 1));
            d = L.peek();
            if (d == ',') ++L.i;
        }
    } else {
        v->s = L.word();
        if (v->s.empty()) *ok = false;
    }
    return v;
}

double num(const std::shared_ptr<Val>& g, const char* key, double def) {
    if (!g || g->kind != Val::Group) return def;
    auto it = g->g.find(key);
    if (it == g->g.end() || it->second->kind != Val::Scalar) return def;
    return std::atof(it->second->s.c_str());
}

// libconfig literal types: a float has a decimal point or an exponent
bool is_float_literal(const std::string& w) {
    if (w.empty()) return false;
    bool digit = false;
    for (char c : w) digit |= std::isdigit((unsigned char)c) != 0;
    return digit && (w.find('.') != std::string::npos || w.find('e') != std::string::npos ||
                     w.find('E') != std::string::npos);
}

bool is_int_literal(const std::string& w) {
    size_t i = (!w.empty() && (w[0] == '-' || w[0] == '+')) ? 1 : 0;
    if (i >= w.size()) return false;
    for (; i < w.size(); ++i)
        if (!std::isdigit((unsigned char)w[i])) return false;
    return true;
}

std::shared_ptr<Val> sub(const std::shared_ptr<Val>& g, const char* key) {
    if (!g || g->kind != Val::Group) return nullptr;
    auto it = g->g.find(key);
    return it == g->g.end() ? nullptr : it->second;
}

}  // namespace

extern "C" {

void mhpc_config_default(mhpc_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->integrator = 2;
    c->time_step = 0.025;
    c->max_time_step = 0.025;
    c->time_end = 1.0;
    c->sfc = 0;
    c->theta = 0.5;
    c->smoothing = 0.0;
    c->smoothing_kernel = 1;
    c->gravity_force_version = 0;
    c->sph_frnn_version = 0;
    c->gravity = 1;
    c->sph = 0;
    c->max_num_interactions = 180;
    c->nb_tolerance = 5;
    c->max_sml_iterations = 5;
    c->precision = 0;
    c->theta_mixed = 0.25;
    c->softening_h_factor = 0.0;
    c->node_pool_factor = 1.0;
    c->gravity_mac = 0;
    c->mac_alpha = 0.003;
    c->balsara = 0;
    c->mac_quad_alpha = 0.0;
    c->sml_band_rounds = 0;
    c->learned_refresh_every = 10;
    c->learned_refresh_iters = 32;
}

int mhpc_config_from_info(const char* path, mhpc_config* c) {
    if (!path || !c) return MHPC_ERR_ARG;
    bool ok;
    std::string text = read_file(path, &ok);
    if (!ok) return MHPC_ERR_CONFIG;
    std::map<std::string, std::string> kv;
    parse_info(text, kv);
    auto f = [&](const char* k, double* dst) { auto it = kv.find(k); if (it != kv.end()) *dst = std::atof(it->second.c_str()); };
    auto i = [&](const char* k, int* dst) { auto it = kv.find(k); if (it != kv.end()) *dst = std::atoi(it->second.c_str()); };
    auto b = [&](const char* k, int* dst) { auto it = kv.find(k); if (it != kv.end()) *dst = as_bool(it->second) ? 1 : 0; };
    i("integrator", &c->integrator);
    f("timeStep", &c->time_step);
    f("maxTimeStep", &c->max_time_step);
    f("timeEnd", &c->time_end);
    i("sfc", &c->sfc);
    f("theta", &c->theta);
    f("smoothing", &c->smoothing);
    i("smoothingKernel", &c->smoothing_kernel);
    i("gravityForceVersion", &c->gravity_force_version);
    i("sphFixedRadiusNNVersion", &c->sph_frnn_version);
    b("calculateEnergy", &c->calculate_energy);
    b("calculateAngularMomentum", &c->calculate_angular_momentum);
    b("calculateCenterOfMass", &c->calculate_center_of_mass);
    b("removeParticles", &c->remove_particles);
    i("removeParticlesCriterion", &c->remove_particles_criterion);
    f("removeParticlesDimension", &c->remove_particles_dimension);
    // run-time forms of parameter.h switches and of this library's options
    b("gravity", &c->gravity);
    b("sph", &c->sph);
    b("integrateEnergy", &c->integrate_energy);
    b("integrateDensity", &c->integrate_density);
    b("integrateSml", &c->integrate_sml);
    b("variableSml", &c->variable_sml);
    b("siUnits", &c->si_units);
    i("maxNumInteractions", &c->max_num_interactions);
    i("precision", &c->precision);
    f("thetaMixed", &c->theta_mixed);
    b("learnedSml", &c->learned_h);
    i("softeningMode", &c->softening_mode);
    f("softeningHFactor", &c->softening_h_factor);
    i("gravityMac", &c->gravity_mac);
    f("macAlpha", &c->mac_alpha);
    b("balsaraSwitch", &c->balsara);
    f("macQuadAlpha", &c->mac_quad_alpha);
    i("smlBandRounds", &c->sml_band_rounds);
    i("learnedRefreshEvery", &c->learned_refresh_every);
    i("learnedRefreshIters", &c->learned_refresh_iters);
    if (c->sml_band_rounds < 0 || c->learned_refresh_every < 0 || c->learned_refresh_iters < 0)
        return MHPC_ERR_CONFIG;
    if (c->gravity_mac < 0 || c->gravity_mac > 1 || (c->gravity_mac == 1 && c->mac_alpha <= 0))
        return MHPC_ERR_CONFIG;
    if (c->integrator < 0 || c->integrator > 2 || c->sfc < 0 || c->sfc > 1 || c->theta <= 0 ||
        c->smoothing_kernel < 0 || c->smoothing_kernel > 4 || c->max_num_interactions <= 0)
        return MHPC_ERR_CONFIG;
    return MHPC_OK;
}

int mhpc_materials_from_cfg(const char* path, mhpc_material* out, int cap, int* count) {
    if (!path || !out || !count || cap <= 0) return MHPC_ERR_ARG;
    bool ok;
    std::string text = read_file(path, &ok);
    if (!ok) return MHPC_ERR_CONFIG;
    Lexer L(text);
    auto root = std::make_shared<Val>();
    root->kind = Val::Group;
    ok = true;
    parse_settings(L, root->g, '\0', &ok, 0);
    if (!ok) return MHPC_ERR_CONFIG;
    auto mats = sub(root, "materials");
    if (!mats || mats->kind != Val::List) return MHPC_ERR_CONFIG;
    int nmat = (int)mats->l.size();
    // IDs must be 0..n-1 (material_handler.cpp:34-52)
    int maxid = -1;
    for (auto& m : mats->l) {
        if (m->kind != Val::Group || !sub(m, "ID")) return MHPC_ERR_CONFIG;
        int id = (int)num(m, "ID", -1);
        if (id < 0) return MHPC_ERR_CONFIG;
        if (id > maxid) maxid = id;
    }
    if (maxid != nmat - 1 || nmat > cap) return MHPC_ERR_CONFIG;
    // The reference reads every float through one variable `temp` declared
    // before the loop over materials (material_handler.cpp:80-134) with
    // libconfig's config_setting_lookup_float, which leaves it unchanged when
    // the setting is missing or is not a float (an integer literal, without
    // libconfig's auto-convert option): such a field takes the value of the
    // previous float read.  Integer fields (ID, interactions, eos type) are
    // read with config_setting_lookup_int, which likewise needs an integer
    // literal and otherwise leaves the field as it was (zero here).
    double temp = 0.0;
    auto lookup_float = [&](const std::shared_ptr<Val>& g, const char* key) {
        auto v = sub(g, key);
        if (v && v->kind == Val::Scalar && is_float_literal(v->s)) temp = std::atof(v->s.c_str());
        return temp;
    };
    auto lookup_int = [&](const std::shared_ptr<Val>& g, const char* key) {
        auto v = sub(g, key);
        return (v && v->kind == Val::Scalar && is_int_literal(v->s)) ? std::atoi(v->s.c_str()) : 0;
    };
    for (auto& m : mats->l) {
        int id = (int)num(m, "ID", 0);
        mhpc_material& o = out[id];
        std::memset(&o, 0, sizeof(o));
        o.id = id;
        o.interactions = lookup_int(m, "interactions");
        o.sml = lookup_float(m, "sml");
        auto av = sub(m, "artificial_viscosity");
        o.alpha = lookup_float(av, "alpha");
        o.beta = lookup_float(av, "beta");
        auto eos = sub(m, "eos");
        o.eos_type = lookup_int(eos, "type");
        o.polytropic_K = lookup_float(eos, "polytropic_K");
        o.polytropic_gamma = lookup_float(eos, "polytropic_gamma");
        o.rho_0 = lookup_float(eos, "rho_0");
        o.bulk_modulus = lookup_float(eos, "bulk_modulus");
        o.n = lookup_float(eos, "n");
        o.shear_modulus = lookup_float(eos, "shear_modulus");
    }
    *count = nmat;
    return MHPC_OK;
}

}  // extern "C"

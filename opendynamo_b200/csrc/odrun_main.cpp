// odrun — command-line solver: the reference binary's main (src/main.rs)
// over the C ABI. Reads ./config.toml (or the path given as the first
// argument), validates it against the reference's schema (src/config.rs)
// and runs od_run.
//
// odrun --make-initial-state [config.toml] writes the config's fresh
// initial state instead, as the reference's IC script does
// (scripts/make_initial_state.py:311-356): od_make_initial_state, saved as
// <output_dir>/<prefix>_<u_real>_000000.h5 at label 0, t = 0.
//
// The TOML reader covers what config files of this schema use: [table]
// headers, key = value with integers, floats, booleans and basic / literal
// strings, and comments. Unknown keys are ignored (serde's default); missing
// required keys and invalid enum spellings are errors.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "opendynamo.h"

namespace {

struct Value {
    enum Kind { Int, Float, Bool, Str } kind;
    long long i = 0;
    double f = 0;
    bool b = false;
    std::string s;
};

using Table = std::map<std::string, Value>;
using Doc = std::map<std::string, Table>;

[[noreturn]] void die(const std::string& msg) {
    std::fprintf(stderr, "Error: %s\n", msg.c_str());
    std::exit(1);
}

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
    return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

Value parse_value(const std::string& raw, int line) {
    const std::string v = trim(raw);
    Value out{};
    auto bad = [&]() -> Value { die("config.toml line " + std::to_string(line) + ": unsupported value '" + v + "'"); };
    if (v.empty()) return bad();
    if (v[0] == '"' || v[0] == '\'') {
        const char q = v[0];
        std::string s;
        size_t i = 1;
        for (; i < v.size() && v[i] != q; ++i) {
            if (q == '"' && v[i] == '\\' && i + 1 < v.size()) {
                const char e = v[++i];
                s += e == 'n' ? '\n' : e == 't' ? '\t' : e;
            } else {
                s += v[i];
            }
        }
        if (i >= v.size() || trim(v.substr(i + 1)).size()) return bad();
        out.kind = Value::Str;
        out.s = s;
        return out;
    }
    if (v == "true" || v == "false") {
        out.kind = Value::Bool;
        out.b = v == "true";
        return out;
    }
    std::string num;
    for (char c : v)
        if (c != '_') num += c;
    const bool is_float = num.find_first_of(".eE") != std::string::npos || num.find("inf") != std::string::npos ||
                          num.find("nan") != std::string::npos;
    char* end = nullptr;
    if (is_float) {
        out.kind = Value::Float;
        out.f = std::strtod(num.c_str(), &end);
    } else {
        out.kind = Value::Int;
        out.i = std::strtoll(num.c_str(), &end, 0);
    }
    if (!end || *end) return bad();
    return out;
}

Doc parse_toml(const std::string& text) {
    Doc doc;
    std::string table;
    std::istringstream in(text);
    std::string line;
    int ln = 0;
    while (std::getline(in, line)) {
        ++ln;
        // strip a comment outside strings
        bool sq = false, dq = false;
        for (size_t i = 0; i < line.size(); ++i) {
            const char c = line[i];
            if (c == '"' && !sq && (i == 0 || line[i - 1] != '\\')) dq = !dq;
            if (c == '\'' && !dq) sq = !sq;
            if (c == '#' && !sq && !dq) {
                line.resize(i);
                break;
            }
        }
        line = trim(line);
        if (line.empty()) continue;
        if (line[0] == '[') {
            if (line.back() != ']' || line.size() < 3 || line[1] == '[')
                die("config.toml line " + std::to_string(ln) + ": unsupported table header");
            table = trim(line.substr(1, line.size() - 2));
            if (doc.count(table)) die("config.toml: duplicate table [" + table + "]");
            doc[table];
            continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos) die("config.toml line " + std::to_string(ln) + ": expected key = value");
        std::string key = trim(line.substr(0, eq));
        if (key.size() >= 2 && (key[0] == '"' || key[0] == '\'')) key = key.substr(1, key.size() - 2);
        if (doc[table].count(key)) die("config.toml: duplicate key " + key);
        doc[table][key] = parse_value(line.substr(eq + 1), ln);
    }
    return doc;
}

struct Reader {
    const Doc& doc;
    const Table& tab(const std::string& t) const {
        auto it = doc.find(t);
        if (it == doc.end()) die("missing [" + t + "] table");
        return it->second;
    }
    const Value* get(const std::string& t, const std::string& k) const {
        auto it = doc.find(t);
        if (it == doc.end()) return nullptr;
        auto jt = it->second.find(k);
        return jt == it->second.end() ? nullptr : &jt->second;
    }
    const Value& req(const std::string& t, const std::string& k) const {
        tab(t);
        const Value* v = get(t, k);
        if (!v) die("[" + t + "] missing required key(s): " + k);
        return *v;
    }
    long long integer(const Value& v, const std::string& k) const {
        if (v.kind != Value::Int) die(k + " must be an integer");
        return v.i;
    }
    double number(const Value& v, const std::string& k) const {
        if (v.kind == Value::Int) return (double)v.i;
        if (v.kind != Value::Float) die(k + " must be a number");
        return v.f;
    }
    std::string str(const Value& v, const std::string& k) const {
        if (v.kind != Value::Str) die(k + " must be a string");
        return v.s;
    }
    double f32(double x) const { return (double)(float)x; }
};

std::string enum_of(const std::string& v, std::initializer_list<const char*> allowed, const char* what) {
    std::string list;
    for (const char* a : allowed) {
        if (v == a) return v;
        list += std::string(list.empty() ? "" : ", ") + a;
    }
    die(std::string("invalid ") + what + " '" + v + "': expected one of " + list);
}

}  // namespace

int main(int argc, char** argv) {
    bool make_ic = false;
    const char* path = "config.toml";
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "--make-initial-state") == 0)
            make_ic = true;
        else
            path = argv[i];
    }
    std::ifstream f(path);
    if (!f) die(std::string("Failed to load ") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const Doc doc = parse_toml(ss.str());
    Reader R{doc};

    od_params p;
    od_default_params(&p);
    // [mesh] (config.rs:13-38); extents are f32 in the reference
    p.nx = (int)R.integer(R.req("mesh", "nx"), "nx");
    p.ny = (int)R.integer(R.req("mesh", "ny"), "ny");
    p.nz = (int)R.integer(R.req("mesh", "nz"), "nz");
    if (p.nx <= 0 || p.ny <= 0 || p.nz <= 0) die("[mesh] nx, ny, nz must be positive integers");
    const float pi = 3.14159265358979323846f;
    p.lx = R.get("mesh", "lx") ? R.f32(R.number(*R.get("mesh", "lx"), "lx")) : (double)(4.0f * pi);
    p.ly = R.get("mesh", "ly") ? R.f32(R.number(*R.get("mesh", "ly"), "ly")) : 2.0;
    p.lz = R.get("mesh", "lz") ? R.f32(R.number(*R.get("mesh", "lz"), "lz")) : (double)((4.0f / 3.0f) * pi);
    // [physics]
    R.number(R.req("physics", "mach_bulk"), "mach_bulk");
    std::string ybc = R.get("physics", "y_boundary") ? R.str(*R.get("physics", "y_boundary"), "y_boundary") : "wall";
    p.y_wall = enum_of(ybc, {"wall", "periodic"}, "y_boundary") == "wall";
    if (const Value* v = R.get("physics", "viscosity_model")) enum_of(R.str(*v, "viscosity_model"), {"fixed", "sutherland"}, "viscosity_model");
    std::string ic_kind = "channel";
    if (const Value* v = R.get("physics", "initial_condition"))
        ic_kind = enum_of(R.str(*v, "initial_condition"), {"channel", "uniform"}, "initial_condition");
    const Value* ist = R.get("physics", "initial_state");
    const std::string initial_state = ist ? R.str(*ist, "initial_state") : "";
    // [solver]
    const long long n_steps = R.integer(R.req("solver", "n_steps"), "n_steps");
    if (n_steps < 0) die("[solver] n_steps must be a non-negative integer");
    const double dt = R.f32(R.number(R.req("solver", "dt"), "dt"));
    const std::string flux = enum_of(R.str(R.req("solver", "flux_scheme"), "flux_scheme"), {"slau2", "ausm+", "rusanov"},
                                     "flux_scheme");
    p.flux = flux == "slau2" ? OD_FLUX_SLAU2 : flux == "ausm+" ? OD_FLUX_AUSMPLUS : OD_FLUX_RUSANOV;
    if (const Value* v = R.get("solver", "fast_math")) {
        if (v->kind != Value::Bool) die("fast_math must be a boolean");
        p.fast_math = v->b;
    }
    // [io]
    const long long save_freq = R.integer(R.req("io", "save_freq"), "save_freq");
    if (save_freq <= 0) die("[io] save_freq must be a positive integer");
    const std::string output_dir = R.str(R.req("io", "output_dir"), "output_dir");
    const std::string prefix = R.str(R.req("io", "prefix"), "prefix");
    const long long ckpt = R.get("io", "checkpoint_freq") ? R.integer(*R.get("io", "checkpoint_freq"), "checkpoint_freq") : 0;
    if (ckpt < 0) die("[io] checkpoint_freq must be a non-negative integer");
    const std::string comp = R.get("io", "compression") ? R.str(*R.get("io", "compression"), "compression") : "blosc-lz4";
    enum_of(comp, {"none", "gzip1", "gzip2", "gzip3", "gzip4", "gzip5", "gzip6", "gzip7", "gzip8", "gzip9", "blosc-lz4", "blosc-zstd"},
            "compression");
    // [precision]
    int* slots[4] = {&p.u_real, &p.q_real, &p.rhs_real, &p.compute_real};
    const char* names[4] = {"u_real", "q_real", "rhs_real", "compute_real"};
    for (int i = 0; i < 4; ++i)
        *slots[i] = enum_of(R.str(R.req("precision", names[i]), names[i]), {"f32", "f64"}, names[i]) == "f64" ? OD_F64 : OD_F32;
    // [b200] extensions (absent = the reference's physics)
    if (const Value* v = R.get("b200", "mu")) p.mu = R.number(*v, "mu");
    if (const Value* v = R.get("b200", "forcing")) p.forcing = R.number(*v, "forcing");
    if (const Value* v = R.get("b200", "precision_form")) {
        const std::string form = enum_of(R.str(*v, "precision_form"), {"reference", "mixed"}, "precision_form");
        p.mixed = form == "mixed";
        if (p.mixed && (p.u_real != OD_F64 || p.compute_real != OD_F32))
            die("precision_form = \"mixed\" needs u_real = \"f64\" and compute_real = \"f32\"");
    }
    if (const Value* v = R.get("b200", "device")) p.device = (int)R.integer(*v, "device");
    if (const Value* v = R.get("b200", "viscosity_model")) {
        if (enum_of(R.str(*v, "viscosity_model"), {"reference", "sutherland"}, "[b200] viscosity_model") == "sutherland") {
            p.viscosity_model = OD_VISC_SUTHERLAND;
            p.t_ref = R.get("physics", "t_ref") ? R.f32(R.number(*R.get("physics", "t_ref"), "t_ref")) : (double)273.15f;
            p.s_suth = R.get("physics", "s_suth") ? R.f32(R.number(*R.get("physics", "s_suth"), "s_suth")) : (double)110.4f;
        }
    }
    if (const Value* v = R.get("b200", "re_bulk")) {
        const double re = R.number(*v, "re_bulk");
        if (!(re > 0)) die("[b200] re_bulk must be a positive number");
        p.mu = R.f32(R.number(R.req("physics", "mach_bulk"), "mach_bulk")) * (0.5 * p.ly) / re;
    }

    if (make_ic) {
        // the script's own defaults for what the config leaves out
        od_ic_params ic{};
        ic.nx = p.nx;
        ic.ny = p.ny;
        ic.nz = p.nz;
        ic.lx = p.lx;
        ic.ly = p.ly;
        ic.lz = p.lz;
        ic.mach_bulk = R.number(R.req("physics", "mach_bulk"), "mach_bulk");
        ic.initial_condition = ic_kind == "uniform" ? OD_IC_UNIFORM : OD_IC_CHANNEL;
        const Value* amp = R.get("physics", "perturbation_amplitude");
        const Value* modes = R.get("physics", "perturbation_modes");
        const Value* seed = R.get("physics", "perturbation_seed");
        ic.perturbation_amplitude = amp ? R.number(*amp, "perturbation_amplitude") : 0.0;
        ic.perturbation_modes = modes ? (int)R.integer(*modes, "perturbation_modes") : 16;
        ic.perturbation_seed = seed ? (int)R.integer(*seed, "perturbation_seed") : 7;
        const int u_f64 = p.u_real == OD_F64;
        const size_t n = (size_t)5 * p.nx * p.ny * p.nz * 64;
        std::vector<double> buf(u_f64 ? n : (n + 1) / 2);
        if (od_make_initial_state(&ic, buf.data(), n * (u_f64 ? 8 : 4), u_f64) != OD_OK)
            die("initial state: invalid [mesh] / [physics] values");
        std::error_code ec;
        std::filesystem::create_directories(output_dir, ec);
        if (ec) die("Failed to create output directory " + output_dir + ": " + ec.message());
        const std::string out = (std::filesystem::path(output_dir) /
                                 (prefix + (u_f64 ? "_f64" : "_f32") + "_000000.h5")).string();
        if (od_state_save(out.c_str(), buf.data(), u_f64, p.nx, p.ny, p.nz, 0, 0.0, p.lx, p.ly, p.lz, comp.c_str()) != OD_OK)
            die(od_state_error());
        std::printf("Initial state written: %s\n", out.c_str());
        return 0;
    }

    const char* tn[2] = {"F32", "F64"};
    std::printf("Configuring pipeline with precisions:\n");
    std::printf("  U:       %s\n  Q:       %s\n  RHS:     %s\n  COMPUTE: %s\n", tn[p.u_real], tn[p.q_real], tn[p.rhs_real],
                tn[p.compute_real]);
    std::printf("  SCHEME:  %s\n", flux == "slau2" ? "Slau2" : flux == "ausm+" ? "AusmPlus" : "Rusanov");

    od_run_opts o{};
    o.initial_state = initial_state.empty() ? nullptr : initial_state.c_str();
    o.n_steps = n_steps;
    o.dt = dt;
    o.save_freq = save_freq;
    o.checkpoint_freq = ckpt;
    o.compression = comp.c_str();
    o.output_dir = output_dir.c_str();
    o.prefix = prefix.c_str();
    od_run_result r;
    char err[1024] = {0};
    const int rc = od_run(&p, &o, &r, err, sizeof err);
    if (rc) die(err);
    return 0;
}

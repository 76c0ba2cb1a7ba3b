// q2d_host — command-line host of the B200 path that reads a Q2D case directory in the
// reference's own input formats and runs it through the C ABI (include/q2d_gpu.h).
//
// It stands where the Fortran host stands in the reference: Q2D_setup (Wrap_Setup.f90:10-167)
// reads input.ini, INPUT/bc.txt, INPUT/ic.tec, INPUT/phase.txt + thermo.dat and, with
// area-variation sources, INPUT/block<b>_area.dat; Q2D_solve (Wrap_Solve.f90:10-34) calls
// Explicit_Step until TODO = END and writes OUTPUT/field.tec at every IO request and at the end.
// Here every Explicit_Step is a q2d_gpu_step call on the GPU.
//
//   q2d_host CASE_DIR [--precision fp64|fp32-flux] [--steps-per-call N] [--max-steps M]
//            [--gamma G|table] [--out FILE] [--check] [--ignore-unsupported] [--quiet]
//
// --check parses every input and prints a JSON summary without touching the GPU.
// Readers follow: input.ini keys Register_Numerics.f90:31-76, Register_Sim_Param.f90:26-29,
// Register_IO.f90:23-39, Register_Sources.f90:33, Register_Physics.f90:24; limiter keywords
// Mod_Space.f90:18-76; Riemann keywords Mod_Riemann.f90:25-109; bc.txt Read_BCfile
// (IO_BC.f90:163-440, direction tokens parse_dir_tok :473-487); Tecplot BLOCK ic.tec with x, y
// nodal and rho1, u, v, p cell-centred, i fastest, one zone per block (Read_IC,
// IO_Solution.f90:38-129, layout of test/1D/ShuOsher-LIMO3/gen_case.py:60-75); the nodal
// cross-section file (Lib_Source_Areavariation.f90:53-101).
#include <cctype>
#include <cerrno>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/q2d_gpu.h"

namespace {

struct Fail {
    std::string msg;
};

[[noreturn]] void die(const std::string& m) { throw Fail{m}; }

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// ---- input.ini ------------------------------------------------------------------------
using Ini = std::map<std::string, std::map<std::string, std::string>>;

Ini read_ini(const std::string& path) {
    std::ifstream in(path);
    if (!in) die("cannot open " + path);
    Ini ini;
    std::string line, sec;
    while (std::getline(in, line)) {
        const size_t c = line.find_first_of("#;!");
        if (c != std::string::npos) line = line.substr(0, c);
        line = trim(line);
        if (line.empty()) continue;
        if (line.front() == '[') {
            const size_t e = line.find(']');
            if (e == std::string::npos) die("input.ini: bad section line '" + line + "'");
            sec = trim(line.substr(1, e - 1));
            continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos) die("input.ini: expected key = value, got '" + line + "'");
        ini[sec][trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
    return ini;
}

const std::string* ini_get(const Ini& ini, const std::string& sec, const std::string& key) {
    auto s = ini.find("Q2D-" + sec);
    if (s == ini.end()) return nullptr;
    auto k = s->second.find(key);
    return k == s->second.end() ? nullptr : &k->second;
}

double to_double(const std::string& v, const std::string& what) {
    std::string t = v;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'e';   // Fortran exponent letter
    char* end = nullptr;
    errno = 0;
    const double x = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || errno == ERANGE) die(what + ": not a number: '" + v + "'");
    return x;
}

long long to_int(const std::string& v, const std::string& what) {
    const double x = to_double(v, what);
    if (x != std::floor(x)) die(what + ": not an integer: '" + v + "'");
    return (long long)x;
}

bool to_bool(const std::string& v, const std::string& what) {
    const std::string t = lower(v);
    if (t == "true" || t == ".true." || t == "t" || t == "1" || t == "yes") return true;
    if (t == "false" || t == ".false." || t == "f" || t == "0" || t == "no") return false;
    die(what + ": not a logical: '" + v + "'");
}

// A point probe (IO_Probes.f90, registered by Register_IO.f90:44-82): its output file
// OUTPUT/<file>.txt, the variables written, the iteration and time frequencies, and its cell
// (block, i, j, 1-based), given or placed at the grid node nearest to `position`.
struct Probe {
    std::string file;
    std::vector<std::string> vars;
    double dtime = 1e30;
    long long diter = 1000000000;
    int b = 0, i = 0, j = 0;
    double x = 0.0, y = 0.0;
    long long ntime = 1;
    FILE* f = nullptr;
};

struct Setup {
    q2d_options opt;
    std::vector<std::string> unsupported;   // keys or values outside the built path
    int shell_diter = 1;
    bool area = false;
    bool newrun = true;   // newrun = false: restart from OUTPUT/field.tec (Register_Sim_Param.f90:26)
    bool sol_overwrite = true;   // sol-overwrite (Register_IO.f90:28)
    std::string sol_format = "tecplot ascii";   // sol-format (Register_IO.f90:24)
    std::vector<Probe> probes;
    std::string limiter_name, riemann_name, scheme_name, source_name;
};

Setup read_options(const Ini& ini) {
    Setup s;
    q2d_options_default(&s.opt);
    q2d_options& o = s.opt;
    if (const std::string* v = ini_get(ini, "Physics", "equations")) {
        if (lower(*v) != "euler") s.unsupported.push_back("[Q2D-Physics] equations = " + *v);
    }
    for (const char* k : {"turbulence", "chemistry", "soot-generation", "rotational-frame"}) {
        const std::string* v = ini_get(ini, "Physics", k);
        if (v && lower(*v) != "none" && !(std::string(k) == "chemistry" && lower(*v) == "frozen"))
            s.unsupported.push_back(std::string("[Q2D-Physics] ") + k + " = " + *v);
    }
    s.scheme_name = "euler";
    if (const std::string* v = ini_get(ini, "Numerics", "time-scheme")) {
        s.scheme_name = *v;
        const std::string t = lower(*v);
        if (t == "euler") o.n_rk = 1;
        else if (t == "rk2") o.n_rk = 2;
        else if (t == "rk3") o.n_rk = 3;
        else s.unsupported.push_back("[Q2D-Numerics] time-scheme = " + *v);
    }
    if (const std::string* v = ini_get(ini, "Numerics", "cfl")) o.cfl = to_double(*v, "cfl");
    if (const std::string* v = ini_get(ini, "Numerics", "cfl-rise-threshold"))
        o.rampa_iter = (int)to_int(*v, "cfl-rise-threshold");
    if (const std::string* v = ini_get(ini, "Numerics", "time-accurate"))
        o.time_accurate = to_bool(*v, "time-accurate") ? 1 : 0;
    // implicit residual smoothing: on when irs-beta > 0 (Assign_Setup.f90:61); 'irs = true' with
    // beta 0 smooths by the identity
    if (const std::string* v = ini_get(ini, "Numerics", "irs-beta")) {
        o.irs_beta = to_double(*v, "irs-beta");
        if (o.irs_beta < 0.0) die("irs-beta must be >= 0");
    }
    if (const std::string* v = ini_get(ini, "Numerics", "integration-variables"))
        if (lower(*v) != "cons") s.unsupported.push_back("[Q2D-Numerics] integration-variables = " + *v);
    // Setup_Space_Scheme (Mod_Space.f90:18-41) then Assign_Limiter (:44-78): the limiter keyword
    // is case-sensitive; MUSCL with 'none' means van Leer; anything else unknown is first order
    std::string recon, lim;
    if (const std::string* v = ini_get(ini, "Numerics", "space-reconstruction")) recon = *v;
    if (const std::string* v = ini_get(ini, "Numerics", "flux-limiter")) lim = *v;
    if (recon.find("MUSCL") != std::string::npos) {
        if (lim == "none") lim = "vanleer";
        o.shock_detector = recon.find("SD") != std::string::npos ? 1 : 0;   // MUSCL-SD (:25-27)
    }
    static const std::map<std::string, int> kLim = {{"minmod", Q2D_LIM_MINMOD},     {"vanleer", Q2D_LIM_VANLEER},
                                                    {"vanalbada", Q2D_LIM_VANALBADA}, {"mc", Q2D_LIM_MC},
                                                    {"superbee", Q2D_LIM_SUPERBEE}, {"LIMO3", Q2D_LIM_LIMO3}};
    auto li = kLim.find(lim);
    o.limiter = li == kLim.end() ? Q2D_LIM_IORD : li->second;
    s.limiter_name = li == kLim.end() ? "iord" : lim;
    // Assign_Riemann_Solver (Mod_Riemann.f90:25-109): HLLC by default
    s.riemann_name = "HLLC";
    if (const std::string* v = ini_get(ini, "Numerics", "riemann-solver")) s.riemann_name = *v;
    if (s.riemann_name == "HLLC") o.riemann = Q2D_RIEMANN_HLLC;
    else if (s.riemann_name == "HLLE") o.riemann = Q2D_RIEMANN_HLLE;
    else if (s.riemann_name == "LLF" || s.riemann_name == "Rusanov") o.riemann = Q2D_RIEMANN_LLF;
    else if (s.riemann_name == "SLAU") o.riemann = Q2D_RIEMANN_SLAU;
    else if (s.riemann_name == "SLAU2") o.riemann = Q2D_RIEMANN_SLAU2;
    else if (s.riemann_name == "HLLC+") o.riemann = Q2D_RIEMANN_HLLCP;
    else if (s.riemann_name == "HLLE++") o.riemann = Q2D_RIEMANN_HLLEPP;
    else if (s.riemann_name == "HLLEM") o.riemann = Q2D_RIEMANN_HLLEM;
    else if (s.riemann_name == "HLLC Rotated") o.riemann = Q2D_RIEMANN_HLLC_ROTATED;
    else if (s.riemann_name == "PLLF") o.riemann = Q2D_RIEMANN_PLLF;
    else if (s.riemann_name == "exact" || s.riemann_name == "Exact") o.riemann = Q2D_RIEMANN_EXACT;
    else if (s.riemann_name == "Hanel") o.riemann = Q2D_RIEMANN_HANEL;
    else if (s.riemann_name == "AUSM+") o.riemann = Q2D_RIEMANN_AUSMP;
    else if (s.riemann_name == "AUSM+-up") o.riemann = Q2D_RIEMANN_AUSMP_UP;
    else if (s.riemann_name == "AUSM+-up2") o.riemann = Q2D_RIEMANN_AUSMP_UP2;
    else o.riemann = Q2D_RIEMANN_HLLC;   // case default (:101-104)
    if (const std::string* v = ini_get(ini, "Numerics", "riemann-options-Minf")) {
        o.riemann_minf = to_double(*v, "riemann-options-Minf");
        if (o.riemann_minf < 0.0) die("riemann-options-Minf must be >= 0");
    }
    if ((o.riemann == Q2D_RIEMANN_AUSMP_UP || o.riemann == Q2D_RIEMANN_AUSMP_UP2) && !(o.riemann_minf > 0.0))
        die("AUSM+-up solver selected. Minf must be defined in input (riemann-options-Minf)");
    if (const std::string* v = ini_get(ini, "Parameters", "res-threshold")) o.res_threshold = to_double(*v, "res-threshold");
    if (const std::string* v = ini_get(ini, "Parameters", "time-threshold")) o.time_threshold = to_double(*v, "time-threshold");
    if (const std::string* v = ini_get(ini, "Parameters", "iter-threshold")) o.itermax = to_int(*v, "iter-threshold");
    if (const std::string* v = ini_get(ini, "Parameters", "newrun")) s.newrun = to_bool(*v, "newrun");
    if (const std::string* v = ini_get(ini, "IO", "res-diter")) o.res_diter = (int)to_int(*v, "res-diter");
    if (const std::string* v = ini_get(ini, "IO", "sol-diter")) o.sol_diter = (int)std::min<long long>(to_int(*v, "sol-diter"), 1000000000);
    if (const std::string* v = ini_get(ini, "IO", "sol-dtime")) o.sol_dtime = to_double(*v, "sol-dtime");
    if (const std::string* v = ini_get(ini, "IO", "shell-diter")) s.shell_diter = (int)to_int(*v, "shell-diter");
    // Register_IO.f90:23-28: initial conditions in ASCII Tecplot; solutions in ASCII Tecplot or
    // VTK (ascii, raw)
    if (const std::string* v = ini_get(ini, "IO", "ini-format"))
        if (lower(*v) != "tecplot ascii") s.unsupported.push_back("[Q2D-IO] ini-format = " + *v);
    if (const std::string* v = ini_get(ini, "IO", "sol-format")) {
        const std::string t = lower(*v);
        if (t == "tecplot ascii" || t == "vtk ascii" || t == "vtk raw") s.sol_format = t;
        else s.unsupported.push_back("[Q2D-IO] sol-format = " + *v);
    }
    if (const std::string* v = ini_get(ini, "IO", "sol-overwrite")) s.sol_overwrite = to_bool(*v, "sol-overwrite");
    // [Q2D-Probes] probe1, probe2, ... name sections of their own (Backend_INI.f90:65-75,
    // Register_IO.f90:44-82)
    if (ini.count("Q2D-Probes")) {
        for (int n = 1;; ++n) {
            const std::string* name = ini_get(ini, "Probes", "probe" + std::to_string(n));
            if (!name) break;
            Probe pr;
            pr.file = *name;
            auto sec = ini.find(*name);
            auto get = [&](const char* k) -> const std::string* {
                if (sec == ini.end()) return nullptr;
                auto it = sec->second.find(k);
                return it == sec->second.end() ? nullptr : &it->second;
            };
            if (const std::string* v = get("variables")) {
                std::istringstream is(*v);
                std::string w;
                while (is >> w) pr.vars.push_back(w);
            }
            for (const std::string& w : pr.vars)
                if (w != "rho(1)" && w != "u" && w != "v" && w != "p" && w != "T" && w != "M")
                    die("probe " + *name + ": unknown variable '" + w + "'");
            if (const std::string* v = get("dtime")) pr.dtime = to_double(*v, "dtime");
            if (const std::string* v = get("diter")) pr.diter = to_int(*v, "diter");
            if (pr.diter < 1 || !(pr.dtime > 0.0)) die("probe " + *name + ": dtime and diter must be > 0");
            if (const std::string* v = get("index-position")) {
                std::istringstream is(*v);
                if (!(is >> pr.b >> pr.i >> pr.j)) die("probe " + *name + ": index-position needs b i j");
            }
            if (const std::string* v = get("position")) {
                std::istringstream is(*v);
                std::string a, b;
                if (!(is >> a >> b)) die("probe " + *name + ": position needs x y");
                pr.x = to_double(a, "position");
                pr.y = to_double(b, "position");
            }
            s.probes.push_back(pr);
        }
    }
    s.source_name = "none";
    if (const std::string* v = ini_get(ini, "Sources", "active")) {
        s.source_name = *v;
        const std::string t = lower(*v);
        if (t == "axisymmetric") o.source = Q2D_SRC_AXI;
        else if (t == "area_variation") { o.source = Q2D_SRC_AREA; s.area = true; }
        else if (t != "none") s.unsupported.push_back("[Q2D-Sources] active = " + *v);
    }
    return s;
}

// ---- tokens of Fortran list-directed input ---------------------------------------------
std::vector<std::string> split_list(const std::string& line) {
    std::vector<std::string> t;
    std::string cur;
    for (char c : line) {
        if (std::isspace((unsigned char)c) || c == ',') {
            if (!cur.empty()) t.push_back(cur), cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) t.push_back(cur);
    return t;
}

// A list-directed READ of n items: values are taken from as many lines as needed; whatever is
// left on the last line is skipped (the next READ starts on a new record).
struct ListReader {
    std::ifstream in;
    std::string path;
    int line_no = 0;
    bool next(int n, std::vector<std::string>& out) {
        out.clear();
        std::string line;
        while ((int)out.size() < n) {
            if (!std::getline(in, line)) {
                if (out.empty()) return false;
                die(path + ": record ends early at line " + std::to_string(line_no));
            }
            ++line_no;
            for (const std::string& t : split_list(line))
                if ((int)out.size() < n) out.push_back(t);
        }
        return true;
    }
};

double dir_tok(const std::string& t) {   // parse_dir_tok (IO_BC.f90:473-487)
    if (t.find("normal") != std::string::npos) return DBL_MAX;
    char* end = nullptr;
    std::string u = t;
    for (char& c : u)
        if (c == 'd' || c == 'D') c = 'e';
    const double x = std::strtod(u.c_str(), &end);
    return end == u.c_str() ? 0.0 : x;
}

std::vector<q2d_bc_rec> read_bc(const std::string& path, std::vector<std::string>& unsupported) {
    ListReader r;
    r.in.open(path);
    r.path = path;
    if (!r.in) die("cannot open " + path);
    std::vector<q2d_bc_rec> recs;
    std::vector<std::string> t;
    std::map<int, int> odd;
    while (r.next(5, t)) {
        q2d_bc_rec b;
        std::memset(&b, 0, sizeof(b));
        b.b = (int)to_int(t[0], path);
        b.i = (int)to_int(t[1], path);
        b.j = (int)to_int(t[2], path);
        b.f = (int)to_int(t[3], path);
        b.type = (int)to_int(t[4], path);
        b.rel_fac = 1.0;
        switch (b.type) {
            case 101: case 201: case 103:   // bs, is, js, fs, d11, d12, d21, d22
                r.next(8, t);
                b.bs = (int)to_int(t[0], path); b.is = (int)to_int(t[1], path);
                b.js = (int)to_int(t[2], path); b.fs = (int)to_int(t[3], path);
                b.d11 = (int)to_int(t[4], path); b.d12 = (int)to_int(t[5], path);
                b.d21 = (int)to_int(t[6], path); b.d22 = (int)to_int(t[7], path);
                break;
            case 301: case 302: case 303: r.next(3, t); break;
            case 304: r.next(2, t); break;
            case 401:   // T0, p0, alpha, beta, rel_fac, massf(1)
                r.next(6, t);
                b.T0 = to_double(t[0], path); b.p0 = to_double(t[1], path);
                b.alpha = dir_tok(t[2]); b.rel_fac = to_double(t[4], path);
                break;
            case 402: case 403: case 404: r.next(6, t); break;
            case 405:   // mach, T, p, alpha, beta, rel_fac, massf(1)
                r.next(7, t);
                b.mach = to_double(t[0], path); b.T0 = to_double(t[1], path);
                b.pamb = to_double(t[2], path); b.alpha = dir_tok(t[3]);
                b.rel_fac = to_double(t[5], path);
                break;
            case 406:   // p_back, rel_fac
                r.next(2, t);
                b.pamb = to_double(t[0], path); b.rel_fac = to_double(t[1], path);
                break;
            case 407: r.next(7, t); break;
            case 410: die(path + ": BC type 410 (mapped state) is not supported (IO_BC.f90:371-378)");
            case 420: r.next(8, t); break;
            case 501: r.next(2, t); break;
            case 102: case 502: die(path + ": BC type " + std::to_string(b.type) + " is not supported");
            default: break;   // no property line (IO_BC.f90:427-431)
        }
        switch (b.type) {
            case 0: case 101: case 201: case 300: case 400: case 401: case 405: case 406: break;
            default: odd[b.type] += 1;
        }
        recs.push_back(b);
    }
    for (auto& kv : odd)
        unsupported.push_back("bc.txt: " + std::to_string(kv.second) + " records of type " + std::to_string(kv.first));
    return recs;
}

// ---- Tecplot BLOCK ic.tec --------------------------------------------------------------
struct Block {
    int ni = 0, nj = 0;
    std::vector<double> nodes;   // x, y per node, i fastest
    std::vector<double> prim;    // interior rho, u, v, p: [var][j][i]
    std::vector<double> area;    // nodal cross-section, empty if none
    std::string title;
};

int zone_int(const std::string& z, const std::string& key) {
    const std::string up = z;
    size_t p = 0;
    while ((p = up.find(key, p)) != std::string::npos) {
        const bool start = p == 0 || !std::isalnum((unsigned char)up[p - 1]);
        size_t q = p + key.size();
        while (q < up.size() && up[q] == ' ') ++q;
        if (start && q < up.size() && up[q] == '=') return std::atoi(up.c_str() + q + 1);
        p += key.size();
    }
    return -1;
}

std::string zone_str(const std::string& z, const std::string& key) {
    const size_t p = z.find(key);
    if (p == std::string::npos) return "";
    size_t q = z.find('=', p);
    if (q == std::string::npos) return "";
    ++q;
    while (q < z.size() && z[q] == ' ') ++q;
    size_t e = q;
    int depth = 0;
    while (e < z.size() && (depth > 0 || z[e] != ',')) {
        if (z[e] == '(') ++depth;
        if (z[e] == ')') --depth;
        ++e;
    }
    return trim(z.substr(q, e - q));
}

std::vector<Block> read_tec(const std::string& path, double* time0) {
    std::ifstream in(path);
    if (!in) die("cannot open " + path);
    std::vector<Block> blocks;
    std::string line, vars;
    std::vector<double> vals;
    Block* cur = nullptr;
    size_t need = 0;
    auto finish = [&]() {
        if (!cur) return;
        if (vals.size() != need)
            die(path + ": zone " + cur->title + " has " + std::to_string(vals.size()) + " values, expected " +
                std::to_string(need));
        const size_t nn = (size_t)(cur->ni + 1) * (cur->nj + 1), nc = (size_t)cur->ni * cur->nj;
        cur->nodes.resize(2 * nn);
        for (size_t k = 0; k < nn; ++k) {
            cur->nodes[2 * k] = vals[k];
            cur->nodes[2 * k + 1] = vals[nn + k];
        }
        cur->prim.assign(vals.begin() + 2 * nn, vals.end());
        (void)nc;
        vals.clear();
    };
    while (std::getline(in, line)) {
        const std::string t = trim(line);
        if (t.empty()) continue;
        const std::string u = lower(t);
        if (u.rfind("variables", 0) == 0) {
            vars = t;
            continue;
        }
        if (u.rfind("title", 0) == 0) continue;
        if (u.rfind("zone", 0) == 0) {
            finish();
            std::string z = t;
            std::string zu = z;
            for (char& c : zu) c = (char)std::toupper((unsigned char)c);
            const int I = zone_int(zu, "I"), J = zone_int(zu, "J");
            if (I < 2 || J < 2) die(path + ": zone without I, J >= 2: '" + t + "'");
            if (zone_str(zu, "DATAPACKING") != "BLOCK") die(path + ": only DATAPACKING=BLOCK is read");
            blocks.emplace_back();
            cur = &blocks.back();
            cur->ni = I - 1;
            cur->nj = J - 1;
            cur->title = zone_str(z, "T");
            need = 2 * (size_t)I * J + 4 * (size_t)cur->ni * cur->nj;
            const std::string st = zone_str(zu, "SOLUTIONTIME");
            if (time0 && !st.empty()) *time0 = to_double(st, path);
            continue;
        }
        if (!cur) die(path + ": data before the first ZONE");
        for (const std::string& tok : split_list(t)) vals.push_back(to_double(tok, path));
    }
    finish();
    // variables: x, y, then the cell-centred state; one species only on this path
    std::vector<std::string> names;
    {
        size_t p = 0;
        while ((p = vars.find('"', p)) != std::string::npos) {
            const size_t q = vars.find('"', p + 1);
            if (q == std::string::npos) break;
            names.push_back(vars.substr(p + 1, q - p - 1));
            p = q + 1;
        }
    }
    if (names.size() != 6 || names[2] != "rho1" || names[3] != "u" || names[4] != "v" || names[5] != "p")
        die(path + ": expected VARIABLES = \"x\" \"y\" \"rho1\" \"u\" \"v\" \"p\" (one species)");
    if (blocks.empty()) die(path + ": no zones");
    return blocks;
}

std::vector<double> read_area(const std::string& path, const Block& B) {
    std::ifstream in(path);
    if (!in) die("cannot open " + path + " (needed by [Q2D-Sources] active = area_variation)");
    std::vector<double> a;
    std::string tok;
    while (in >> tok) a.push_back(to_double(tok, path));
    if (a.size() != (size_t)(B.ni + 1) * (B.nj + 1))
        die(path + ": " + std::to_string(a.size()) + " values, expected (ni+1)(nj+1) = " +
            std::to_string((B.ni + 1) * (B.nj + 1)));
    return a;
}

// Gas of the single-species tables: R = Runiv / W from phase.txt; with "table" gamma from the
// first thermo.dat row, and when cp varies with temperature the whole table (Temperature, Cp,
// Enthalpy rows at 1, 2, .. K; knot 0 extrapolated from knots 1 and 2) for the thermally
// perfect gas (q2d_gpu_set_thermo_table); else gamma is the given value.
void read_gas(const std::string& dir, const std::string& gamma_arg, q2d_options& o, std::string& note,
              std::vector<double>& h_tab, std::vector<double>& cp_tab) {
    const double runiv = 8314.46;   // docs/theory/thermo.md:56
    std::ifstream ph(dir + "/INPUT/phase.txt");
    if (!ph) {
        note = "no INPUT/phase.txt: R = " + std::to_string(o.gas_R);
    } else {
        std::string line;
        std::getline(ph, line);
        std::vector<std::vector<std::string>> species;
        while (std::getline(ph, line)) {
            auto t = split_list(line);
            if (!t.empty()) species.push_back(t);
        }
        if (species.size() != 1 || species[0].size() < 2) die("INPUT/phase.txt: one species expected");
        o.gas_R = runiv / to_double(species[0][1], "phase.txt");
        note = "R = " + std::to_string(o.gas_R) + " (" + species[0][0] + ")";
    }
    if (gamma_arg == "table") {
        std::ifstream th(dir + "/INPUT/thermo.dat");
        if (!th) die("--gamma table needs INPUT/thermo.dat");
        // a constant cp (the reference's Air table: 1004.5 J/(kg K) on every row, 1-10000 K) is
        // the calorically perfect closure exactly; a temperature-dependent cp takes the table
        // lerp (Lib_Riemann_HLL.f90:258-303) of the plain FP64 form
        std::string line;
        double cp0 = 0.0;
        long long rows = 0;
        bool varies = false;
        std::vector<double> hs(1, 0.0), cps(1, 0.0);
        while (std::getline(th, line)) {
            auto t = split_list(line);
            if (t.size() >= 3 && (std::isdigit((unsigned char)t[0][0]) || t[0][0] == '.')) {
                const double T = to_double(t[0], "thermo.dat"), cp = to_double(t[1], "thermo.dat");
                if (T != (double)(rows + 1)) die("INPUT/thermo.dat: rows must be at T = 1, 2, .. K");
                if (rows++ == 0) cp0 = cp;
                else if (std::fabs(cp - cp0) > 1e-12 * std::fabs(cp0)) varies = true;
                cps.push_back(cp);
                hs.push_back(to_double(t[2], "thermo.dat"));
            }
        }
        if (rows == 0) die("INPUT/thermo.dat: no table rows");
        o.gas_gamma = cp0 / (cp0 - o.gas_R);
        if (varies) {
            if (rows < 2) die("INPUT/thermo.dat: a variable-cp table needs two rows or more");
            hs[0] = 2.0 * hs[1] - hs[2];
            cps[0] = 2.0 * cps[1] - cps[2];
            h_tab = std::move(hs);
            cp_tab = std::move(cps);
            note += ", thermally perfect table of " + std::to_string(rows) + " K";
        }
    } else {
        o.gas_gamma = to_double(gamma_arg, "--gamma");
    }
}

// P(4, -1:ni+2, -1:nj+2) of the reference with the interior filled.
std::vector<double> ghosted(const Block& B) {
    std::vector<double> P(4 * (size_t)(B.ni + 4) * (B.nj + 4), 0.0);
    const size_t nc = (size_t)B.ni * B.nj;
    for (int j = 0; j < B.nj; ++j)
        for (int i = 0; i < B.ni; ++i)
            for (int v = 0; v < 4; ++v)
                P[v + 4 * ((size_t)(i + 2) + (size_t)(B.ni + 4) * (j + 2))] = B.prim[v * nc + (size_t)j * B.ni + i];
    return P;
}

// The restart field of newrun = false (Read_IC, IO_Solution.f90:78-96): OUTPUT/field.tec, else
// the last of OUTPUT/field1.tec, field2.tec, ... that exists.
std::string restart_field(const std::string& dir) {
    const std::string base = dir + "/OUTPUT/field";
    if (std::ifstream(base + ".tec")) return base + ".tec";
    std::string found;
    for (int i = 1;; ++i) {
        const std::string t = base + std::to_string(i) + ".tec";
        if (!std::ifstream(t)) break;
        found = t;
    }
    if (found.empty()) die("[ERROR] reading input file " + base + ".tec");
    return found;
}

// Fortran Ew.d edit descriptor (w = 20, d = 10): 0.dddddddddd E+xx, right-justified.
std::string fortran_e20_10(double v) {
    char buf[64];
    if (v == 0.0) {
        std::snprintf(buf, sizeof buf, "%20s", "0.0000000000E+00");
        return buf;
    }
    char m[32];
    std::snprintf(m, sizeof m, "%.9E", v);   // [-]d.dddddddddE[+-]xx: the 10 significant digits
    const bool neg = m[0] == '-';
    const char* p = m + (neg ? 1 : 0);
    std::string digits;
    digits += p[0];
    digits.append(p + 2, 9);
    const int e = std::atoi(std::strchr(p, 'E') + 1) + 1;
    char out[40];
    std::snprintf(out, sizeof out, "%s0.%sE%c%02d", neg ? "-" : "", digits.c_str(), e < 0 ? '-' : '+', e < 0 ? -e : e);
    std::snprintf(buf, sizeof buf, "%20s", out);
    return buf;
}

void write_tec(const std::string& path, const std::vector<Block>& blocks, const std::vector<std::vector<double>>& P,
               double time) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) die("cannot write " + path);
    std::fprintf(f, " VARIABLES =\"x\"  \"y\"  \"rho1\"  \"u\"  \"v\"  \"p\"\n");
    for (size_t b = 0; b < blocks.size(); ++b) {
        const Block& B = blocks[b];
        std::fprintf(f, " ZONE  T = B%zu, I=%d, J=%d, K=1, DATAPACKING=BLOCK, "
                        "VARLOCATION=([1-2]=NODAL,[3-6]=CELLCENTERED), SOLUTIONTIME=%.17E\n",
                     b + 1, B.ni + 1, B.nj + 1, time);
        const size_t nn = (size_t)(B.ni + 1) * (B.nj + 1);
        for (int c = 0; c < 2; ++c)
            for (size_t k = 0; k < nn; ++k) std::fprintf(f, " %.17E\n", B.nodes[2 * k + c]);
        for (int v = 0; v < 4; ++v)
            for (int j = 0; j < B.nj; ++j)
                for (int i = 0; i < B.ni; ++i)
                    std::fprintf(f, " %.17E\n", P[b][v + 4 * ((size_t)(i + 2) + (size_t)(B.ni + 4) * (j + 2))]);
    }
    std::fclose(f);
}

// Cell (i, j) (1-based) of a ghosted reference-layout array P(4, -1:ni+2, -1:nj+2).
inline const double* cell_at(const std::vector<double>& P, int ni, int i, int j) {
    return &P[4 * ((size_t)(i + 1) + (size_t)(ni + 4) * (j + 1))];
}

// VTK XML structured grids (Write_vtk_tec, IO_Solution.f90:234-326, sol-format 'vtk ascii' or
// 'vtk raw'): one OUTPUT/vtk/<stem>_Block<b>.vts per block with the node coordinates and the cell
// variables rho(1), u, v, p, T (the reference's Ovarnames, T = p / (rho R)), and the multiblock
// index OUTPUT/<stem>.vtm; the time as field data.
void write_vtk(const std::string& outdir, const std::string& stem, const std::vector<Block>& blocks,
               const std::vector<std::vector<double>>& P, double time, double R, bool raw) {
    const std::string vdir = outdir + "/vtk";
    if (std::system(("mkdir -p '" + vdir + "'").c_str()) != 0) die("cannot create " + vdir);
    static const char* names[5] = {"rho(1)", "u", "v", "p", "T"};
    for (size_t b = 0; b < blocks.size(); ++b) {
        const Block& B = blocks[b];
        const std::string path = vdir + "/" + stem + "_Block" + std::to_string(b + 1) + ".vts";
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) die("cannot write " + path);
        const size_t nn = (size_t)(B.ni + 1) * (B.nj + 1), nc = (size_t)B.ni * B.nj;
        std::vector<std::vector<double>> arrays;   // points (3 per node), then the cell variables
        arrays.emplace_back(3 * nn);
        for (size_t k = 0; k < nn; ++k) {
            arrays[0][3 * k] = B.nodes[2 * k];
            arrays[0][3 * k + 1] = B.nodes[2 * k + 1];
            arrays[0][3 * k + 2] = 0.0;
        }
        for (int v = 0; v < 5; ++v) {
            std::vector<double> a(nc);
            for (int j = 0; j < B.nj; ++j)
                for (int i = 0; i < B.ni; ++i) {
                    const double* q = cell_at(P[b], B.ni, i + 1, j + 1);
                    a[(size_t)j * B.ni + i] = v < 4 ? q[v] : q[3] / (q[0] * R);
                }
            arrays.push_back(std::move(a));
        }
        std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"StructuredGrid\" version=\"1.0\" "
                        "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
        std::fprintf(f, "  <StructuredGrid WholeExtent=\"0 %d 0 %d 0 0\">\n", B.ni, B.nj);
        std::fprintf(f, "    <FieldData>\n      <DataArray type=\"Float64\" Name=\"TIME\" NumberOfTuples=\"1\" "
                        "format=\"ascii\">%.17E</DataArray>\n    </FieldData>\n", time);
        std::fprintf(f, "    <Piece Extent=\"0 %d 0 %d 0 0\">\n", B.ni, B.nj);
        unsigned long long offset = 0;
        auto array = [&](size_t k, const char* name, int ncomp) {
            std::fprintf(f, "        <DataArray type=\"Float64\"");
            if (name) std::fprintf(f, " Name=\"%s\"", name);
            if (ncomp > 1) std::fprintf(f, " NumberOfComponents=\"%d\"", ncomp);
            if (raw) {
                std::fprintf(f, " format=\"appended\" offset=\"%llu\"/>\n", offset);
                offset += 8 + 8 * arrays[k].size();
                return;
            }
            std::fprintf(f, " format=\"ascii\">\n");
            for (size_t q = 0; q < arrays[k].size(); ++q) std::fprintf(f, " %.17E\n", arrays[k][q]);
            std::fprintf(f, "        </DataArray>\n");
        };
        std::fprintf(f, "      <Points>\n");
        array(0, nullptr, 3);
        std::fprintf(f, "      </Points>\n      <CellData>\n");
        for (int v = 0; v < 5; ++v) array(1 + v, names[v], 1);
        std::fprintf(f, "      </CellData>\n    </Piece>\n  </StructuredGrid>\n");
        if (raw) {
            std::fprintf(f, "  <AppendedData encoding=\"raw\">\n_");
            for (const std::vector<double>& a : arrays) {
                const unsigned long long nb = 8ull * a.size();
                std::fwrite(&nb, sizeof nb, 1, f);
                std::fwrite(a.data(), sizeof(double), a.size(), f);
            }
            std::fprintf(f, "\n  </AppendedData>\n");
        }
        std::fprintf(f, "</VTKFile>\n");
        std::fclose(f);
    }
    const std::string vtm = outdir + "/" + stem + ".vtm";
    FILE* f = std::fopen(vtm.c_str(), "w");
    if (!f) die("cannot write " + vtm);
    std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"vtkMultiBlockDataSet\" version=\"1.0\" "
                    "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n  <vtkMultiBlockDataSet>\n");
    for (size_t b = 0; b < blocks.size(); ++b)
        std::fprintf(f, "    <DataSet index=\"%zu\" name=\"Block%zu\" file=\"vtk/%s_Block%zu.vts\"/>\n", b, b + 1,
                     stem.c_str(), b + 1);
    std::fprintf(f, "  </vtkMultiBlockDataSet>\n</VTKFile>\n");
    std::fclose(f);
}

// gfortran list-directed output (write(unit, *)) of an integer and of a REAL(8): I12, and 17
// significant digits in F form for 0.1 <= |x| < 1e16, E form with a 3-digit exponent otherwise.
std::string ld_int(long long v) {
    char b[32];
    std::snprintf(b, sizeof b, "%12lld", v);
    return b;
}
std::string ld_real(double v) {
    char b[64];
    const double a = std::fabs(v);
    if (v == 0.0 || (a >= 0.1 && a < 1e16)) {
        const int e = v == 0.0 ? 0 : (int)std::floor(std::log10(a));
        std::snprintf(b, sizeof b, "%*.*f     ", 21, std::max(0, 16 - e), v);
    } else {
        char m[40];
        std::snprintf(m, sizeof m, "%.16E", v);
        char* ep = std::strchr(m, 'E');
        const int ex = std::atoi(ep + 1);
        *ep = 0;
        std::snprintf(b, sizeof b, "%24sE%c%03d", m, ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    }
    return std::string(" ") + b;
}

void json_str(FILE* f, const std::string& s) {
    std::fputc('"', f);
    for (char c : s) {
        if (c == '"' || c == '\\') std::fputc('\\', f);
        std::fputc(c, f);
    }
    std::fputc('"', f);
}

struct Args {
    std::string dir, precision = "fp64", gamma = "1.4", out;
    int per_call = 100;
    long long max_steps = -1;
    bool check = false, ignore = false, quiet = false;
};

Args parse_args(int argc, char** argv) {
    Args a;
    for (int k = 1; k < argc; ++k) {
        const std::string s = argv[k];
        auto val = [&]() -> std::string {
            if (k + 1 >= argc) die("missing value after " + s);
            return argv[++k];
        };
        if (s == "--precision") a.precision = val();
        else if (s == "--steps-per-call") a.per_call = (int)to_int(val(), s);
        else if (s == "--max-steps") a.max_steps = to_int(val(), s);
        else if (s == "--gamma") a.gamma = val();
        else if (s == "--out") a.out = val();
        else if (s == "--check") a.check = true;
        else if (s == "--ignore-unsupported") a.ignore = true;
        else if (s == "--quiet") a.quiet = true;
        else if (!s.empty() && s[0] == '-') die("unknown option " + s);
        else if (a.dir.empty()) a.dir = s;
        else die("more than one case directory");
    }
    if (a.dir.empty()) die("usage: q2d_host CASE_DIR [--precision fp64|fp32-flux] [--steps-per-call N] "
                           "[--max-steps M] [--gamma G|table] [--out FILE] [--check] [--ignore-unsupported]");
    if (a.precision != "fp64" && a.precision != "fp32-flux") die("--precision: fp64 or fp32-flux");
    if (a.per_call < 1) die("--steps-per-call must be >= 1");
    return a;
}

// Setup_Probes (IO_Probes.f90:43-114): a probe without an index position sits at the grid node
// nearest to its position (Place, :118-136: nodes i = 1..ni, j = 0..nj of every block, the first
// nearest in block, j, i order); its cell is (b, i, j) of that node. A row-0 node reads the
// boundary cell (j = 1): the ghost row the reference would read is not kept.
void place_probes(std::vector<Probe>& probes, const std::vector<Block>& blocks) {
    for (Probe& pr : probes) {
        if (pr.b == 0 && pr.i == 0 && pr.j == 0) {
            double d0 = HUGE_VAL;
            for (size_t b = 0; b < blocks.size(); ++b) {
                const Block& B = blocks[b];
                for (int j = 0; j <= B.nj; ++j)
                    for (int i = 1; i <= B.ni; ++i) {
                        const double* xy = &B.nodes[2 * ((size_t)j * (B.ni + 1) + i)];
                        const double d = std::hypot(pr.x - xy[0], pr.y - xy[1]);
                        if (d < d0) { d0 = d; pr.b = (int)b + 1; pr.i = i; pr.j = j; }
                    }
            }
        }
        if (pr.b < 1 || pr.b > (int)blocks.size() || pr.i < 1 || pr.i > blocks[pr.b - 1].ni || pr.j < 0 ||
            pr.j > blocks[pr.b - 1].nj)
            die("probe " + pr.file + ": cell outside the grid");
        if (pr.j == 0) pr.j = 1;
    }
}

int run(int argc, char** argv) {
    const Args A = parse_args(argc, argv);
    const Ini ini = read_ini(A.dir + "/input.ini");
    Setup S = read_options(ini);
    S.opt.precision = A.precision == "fp64" ? Q2D_PREC_FP64 : Q2D_PREC_FP32_FLUX;
    std::string gas_note;
    std::vector<double> h_tab, cp_tab;
    read_gas(A.dir, A.gamma, S.opt, gas_note, h_tab, cp_tab);
    // newrun: INPUT/ic.tec, its SOLUTIONTIME ignored; restart: the last field written, time-accurate
    // cases resume at its SOLUTIONTIME, steady ones count iterations from int(SOLUTIONTIME)
    // (Wrap_Setup.f90:132-149; the writer stores -iterations there, Wrap_Postprocess.f90:41-47)
    const std::string icpath = S.newrun ? A.dir + "/INPUT/ic.tec" : restart_field(A.dir);
    double time0 = 0.0;
    std::vector<Block> blocks = read_tec(icpath, &time0);
    const double case_time = (!S.newrun && S.opt.time_accurate) ? time0 : 0.0;
    const long long iter_base = (!S.newrun && !S.opt.time_accurate) ? (long long)time0 : 0;
    if (S.area)
        for (size_t b = 0; b < blocks.size(); ++b)
            blocks[b].area = read_area(A.dir + "/INPUT/block" + std::to_string(b + 1) + "_area.dat", blocks[b]);
    std::vector<q2d_bc_rec> recs = read_bc(A.dir + "/INPUT/bc.txt", S.unsupported);
    const q2d_options& o = S.opt;
    place_probes(S.probes, blocks);

    if (A.check) {   // parse summary, no GPU
        FILE* f = stdout;
        std::fprintf(f, "{\"limiter\": %d, \"riemann\": %d, \"n_rk\": %d, \"time_accurate\": %d, \"source\": %d, "
                        "\"precision\": %d, \"rampa_iter\": %d, \"res_diter\": %d, \"sol_diter\": %d, "
                        "\"itermax\": %lld, \"cfl\": %.17g, \"res_threshold\": %.17g, \"time_threshold\": %.17g, "
                        "\"sol_dtime\": %.17g, \"gas_R\": %.17g, \"gas_gamma\": %.17g, \"shell_diter\": %d, "
                        "\"irs_beta\": %.17g, \"shock_detector\": %d, \"riemann_minf\": %.17g, \"newrun\": %d, "
                        "\"case_time\": %.17g, \"iter_base\": %lld,\n",
                     o.limiter, o.riemann, o.n_rk, o.time_accurate, o.source, o.precision, o.rampa_iter, o.res_diter,
                     o.sol_diter, o.itermax, o.cfl, o.res_threshold, o.time_threshold, o.sol_dtime, o.gas_R,
                     o.gas_gamma, S.shell_diter, o.irs_beta, o.shock_detector, o.riemann_minf, S.newrun ? 1 : 0,
                     case_time, iter_base);
        std::fprintf(f, " \"initial_field\": ");
        json_str(f, icpath);
        std::fprintf(f, ",\n");
        std::fprintf(f, " \"blocks\": [");
        for (size_t b = 0; b < blocks.size(); ++b) {
            double s = 0.0, sa = 0.0;
            for (double x : blocks[b].prim) s += x;
            for (double x : blocks[b].area) sa += x;
            std::fprintf(f, "%s{\"ni\": %d, \"nj\": %d, \"prim_sum\": %.17g, \"area_sum\": %.17g}", b ? ", " : "",
                         blocks[b].ni, blocks[b].nj, s, sa);
        }
        std::fprintf(f, "],\n \"bcs\": [");
        for (size_t k = 0; k < recs.size(); ++k) {
            const q2d_bc_rec& r = recs[k];
            std::fprintf(f, "%s[%d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %.17g, %.17g, %.17g, %.17g, %.17g, %.17g]",
                         k ? ", " : "", r.b, r.i, r.j, r.f, r.type, r.bs, r.is, r.js, r.fs, r.d11, r.d12, r.d21, r.d22,
                         r.T0, r.p0, r.pamb, r.mach, r.alpha >= 0.5 * DBL_MAX ? -1.0 : r.alpha, r.rel_fac);
        }
        std::fprintf(f, "],\n \"thermo_knots\": %zu, \"sol_format\": ", h_tab.size());
        json_str(f, S.sol_format);
        std::fprintf(f, ", \"sol_overwrite\": %d, \"probes\": [", S.sol_overwrite ? 1 : 0);
        for (size_t k = 0; k < S.probes.size(); ++k) {
            const Probe& pr = S.probes[k];
            std::fprintf(f, "%s{\"file\": ", k ? ", " : "");
            json_str(f, pr.file);
            std::fprintf(f, ", \"variables\": [");
            for (size_t q = 0; q < pr.vars.size(); ++q) {
                if (q) std::fprintf(f, ", ");
                json_str(f, pr.vars[q]);
            }
            std::fprintf(f, "], \"diter\": %lld, \"dtime\": %.17g, \"cell\": [%d, %d, %d]}", pr.diter, pr.dtime,
                         pr.b, pr.i, pr.j);
        }
        std::fprintf(f, "],\n \"unsupported\": [");
        for (size_t k = 0; k < S.unsupported.size(); ++k) {
            if (k) std::fprintf(f, ", ");
            json_str(f, S.unsupported[k]);
        }
        std::fprintf(f, "]}\n");
        return 0;
    }
    if (!S.unsupported.empty()) {
        for (const std::string& u : S.unsupported)
            std::fprintf(stderr, "q2d_host: %s: %s\n", A.ignore ? "warning, ignored" : "not on the built path", u.c_str());
        if (!A.ignore) return 2;
    }

    q2d_ctx* ctx = nullptr;
    auto check = [&](int st, const char* what) {
        if (st != Q2D_OK) {
            const char* m = ctx ? q2d_gpu_last_error(ctx) : nullptr;
            die(std::string(what) + ": " + q2d_gpu_errstr(st) + (m && *m ? std::string(" (") + m + ")" : ""));
        }
    };
    check(q2d_gpu_create(&ctx, &o), "q2d_gpu_create");
    if (!h_tab.empty())
        check(q2d_gpu_set_thermo_table(ctx, (int)h_tab.size(), h_tab.data(), cp_tab.data()),
              "q2d_gpu_set_thermo_table");
    int cid = -1;
    std::vector<int> bid(blocks.size());
    std::vector<std::vector<double>> P(blocks.size());
    try {
        check(q2d_gpu_add_case(ctx, &cid), "q2d_gpu_add_case");
        for (size_t b = 0; b < blocks.size(); ++b) {
            const Block& B = blocks[b];
            check(q2d_gpu_add_block(ctx, cid, B.ni, B.nj, B.nodes.data(), B.area.empty() ? nullptr : B.area.data(),
                                    &bid[b]),
                  "q2d_gpu_add_block");
            P[b] = ghosted(B);
            check(q2d_gpu_upload_prim(ctx, bid[b], P[b].data()), "q2d_gpu_upload_prim");
        }
        check(q2d_gpu_set_bcs(ctx, cid, recs.data(), (int)recs.size()), "q2d_gpu_set_bcs");
        if (case_time != 0.0) check(q2d_gpu_set_case_time(ctx, cid, case_time), "q2d_gpu_set_case_time");
        check(q2d_gpu_commit(ctx), "q2d_gpu_commit");
        if (!A.quiet)
            std::printf("q2d_host: %zu blocks, %lld cells, %zu boundary records, %s, limiter %s, %s, RK%d, cfl %g, %s\n",
                        blocks.size(), q2d_gpu_num_cells(ctx), recs.size(), A.precision.c_str(), S.limiter_name.c_str(),
                        S.riemann_name.c_str(), o.n_rk, o.cfl, gas_note.c_str());
        const std::string outdir = A.dir + "/OUTPUT";
        const std::string out = A.out.empty() ? outdir + "/field.tec" : A.out;
        if (A.out.empty()) {
            std::string cmd = "mkdir -p '" + outdir + "'";
            if (std::system(cmd.c_str()) != 0) die("cannot create " + outdir);
        }
        // Write_Solution (Wrap_Postprocess.f90:104-106, 120-125): OUTPUT/field at the end and, with
        // sol-overwrite = false, OUTPUT/field<k> for the k-th intermediate solution; Tecplot or VTK
        int id_stampa = 0;
        auto write_solution = [&](bool intermediate, double t) {
            std::string stem = "field";
            if (intermediate) {
                ++id_stampa;
                if (!S.sol_overwrite) stem += std::to_string(id_stampa);
            }
            if (!A.out.empty()) {
                write_tec(out, blocks, P, t);
            } else if (S.sol_format == "tecplot ascii") {
                write_tec(outdir + "/" + stem + ".tec", blocks, P, t);
            } else {
                write_vtk(outdir, stem, blocks, P, t, o.gas_R, S.sol_format == "vtk raw");
            }
            return stem;
        };
        for (Probe& pr : S.probes) {
            const std::string path = outdir + "/" + pr.file + ".txt";
            if (!S.newrun && !std::ifstream(path))
                die("[ERROR] You restarted from an old solution but the probes files were not found.");
            pr.f = std::fopen(path.c_str(), S.newrun ? "w" : "a");
            if (!pr.f) die("cannot write " + path);
        }
        bool probe_dtime = false;
        for (const Probe& pr : S.probes) probe_dtime = probe_dtime || pr.dtime < 1e30;
        // Write_Probes_Data (IO_Probes.f90:187-207) after an iteration that needs no solution output
        // (TODO = 1, Wrap_Postprocess.f90:246-257): every diter iterations the iteration and the
        // variables, else once the time passes the next multiple of dtime, the time and the variables
        auto write_probes = [&](long long iter_general, double t) {
            std::vector<char> have(blocks.size(), 0);
            for (Probe& pr : S.probes) {
                const bool by_iter = iter_general % pr.diter == 0;
                const bool by_time = !by_iter && t >= pr.dtime * (double)pr.ntime;
                if (!by_iter && !by_time) continue;
                const int b = pr.b - 1;
                if (!have[b]) {
                    check(q2d_gpu_download_prim(ctx, bid[b], P[b].data()), "q2d_gpu_download_prim");
                    have[b] = 1;
                }
                const double* q = cell_at(P[b], blocks[b].ni, pr.i, pr.j);
                std::string line = by_iter ? ld_int(iter_general) : ld_real(t);
                for (const std::string& w : pr.vars) {
                    double x;
                    if (w == "rho(1)") x = q[0];
                    else if (w == "u") x = q[1];
                    else if (w == "v") x = q[2];
                    else if (w == "p") x = q[3];
                    else if (w == "T") x = q[3] / (q[0] * o.gas_R);
                    else x = std::hypot(q[1], q[2]) / std::sqrt(o.gas_gamma * q[3] / q[0]);
                    line += ld_real(x);
                }
                std::fprintf(pr.f, "%s\n", line.c_str());
                if (by_time) pr.ntime += 1;
            }
        };
        FILE* hist = std::fopen((A.out.empty() ? outdir + "/residuals.dat" : A.out + ".residuals").c_str(), "w");
        if (!hist) die("cannot write the residual history");
        std::fprintf(hist, "# iter time dtglobal res_rho res_u res_v res_p\n");
        // the reference's residual history (Wrap_Setup.f90:114-127, Wrap_Postprocess.f90:128-133,
        // 248-253): iter_general, time (-1 for steady runs), the 4 residuals, (I8,E20.10,4E20.10),
        // every res-diter iterations; appended to on a restart
        FILE* rh = A.out.empty() ? std::fopen((outdir + "/residual-history.dat").c_str(), S.newrun ? "w" : "a")
                                 : nullptr;
        if (A.out.empty() && !rh) die("cannot write OUTPUT/residual-history.dat");
        // SOLUTIONTIME of a written field: the time, or -iter_general for steady runs
        auto sol_time = [&](const q2d_step_info& in) {
            return o.time_accurate ? in.time : -(double)(iter_base + in.iter);
        };
        q2d_step_info info{};
        long long done = 0, last_shell = 0;
        int rc = 0;
        for (;;) {
            int n = A.per_call;
            n = (int)std::min<long long>(n, o.res_diter - done % o.res_diter);   // land on res-diter multiples
            for (const Probe& pr : S.probes)   // and on the probes' iterations
                n = (int)std::min<long long>(n, pr.diter - (iter_base + done) % pr.diter);
            if (probe_dtime) n = 1;            // time-based probes: every step is checked
            if (A.max_steps >= 0) n = (int)std::min<long long>(n, A.max_steps - done);
            if (n <= 0) break;
            const int st = q2d_gpu_step(ctx, n, &info);
            done = info.iter;
            std::fprintf(hist, "%lld %.17g %.17g %.17g %.17g %.17g %.17g\n", info.iter, info.time, info.dtglobal,
                         info.residual[0], info.residual[1], info.residual[2], info.residual[3]);
            if (rh && st == Q2D_OK && info.iter % o.res_diter == 0) {
                std::string line;
                char ib[32];
                std::snprintf(ib, sizeof ib, "%8lld", iter_base + info.iter);
                line += ib;
                line += fortran_e20_10(o.time_accurate ? info.time : -1.0);
                for (int k = 0; k < 4; ++k) line += fortran_e20_10(info.residual[k]);
                std::fprintf(rh, "%s\n", line.c_str());
            }
            if (!A.quiet && (info.iter - last_shell >= S.shell_diter || info.todo != Q2D_TODO_CONTINUE || st)) {
                std::printf("iter %lld  time %.6e  dt %.6e  res %.6e %.6e %.6e %.6e\n", info.iter, info.time,
                            info.dtglobal, info.residual[0], info.residual[1], info.residual[2], info.residual[3]);
                last_shell = info.iter;
            }
            if (st != Q2D_OK) {
                std::fprintf(stderr, "q2d_host: step failed: %s at block %d cell (%d,%d) stage %d\n",
                             q2d_gpu_errstr(st), info.err_b, info.err_i, info.err_j, info.err_stage);
                rc = 3;
                break;
            }
            if (info.todo == Q2D_TODO_IO || info.todo == Q2D_TODO_END) {   // Write_Solution
                for (size_t b = 0; b < blocks.size(); ++b)
                    check(q2d_gpu_download_prim(ctx, bid[b], P[b].data()), "q2d_gpu_download_prim");
                write_solution(info.todo == Q2D_TODO_IO, sol_time(info));
            } else if (!S.probes.empty()) {
                write_probes(iter_base + info.iter, info.time);
            }
            if (info.todo == Q2D_TODO_END) break;
        }
        if (rc == 0 && info.todo != Q2D_TODO_END) {   // stopped by --max-steps
            for (size_t b = 0; b < blocks.size(); ++b)
                check(q2d_gpu_download_prim(ctx, bid[b], P[b].data()), "q2d_gpu_download_prim");
            write_solution(false, sol_time(info));
        }
        for (Probe& pr : S.probes) std::fclose(pr.f);
        std::fclose(hist);
        if (rh) std::fclose(rh);
        if (!A.quiet)
            std::printf("q2d_host: %s after %lld steps, wrote %s\n",
                        rc ? "stopped on error" : (info.todo == Q2D_TODO_END ? "converged/ended" : "stopped"), done,
                        out.c_str());
        q2d_gpu_destroy(ctx);
        return rc;
    } catch (...) {
        q2d_gpu_destroy(ctx);
        throw;
    }
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const Fail& f) {
        std::fprintf(stderr, "q2d_host: %s\n", f.msg.c_str());
        return 1;
    }
}

// case.cpp -- a CompLaB.xml run description turned into library calls: the reference's
// initialize_complab (complab_functions.hh:825-1602) for the parameters of the reactive-transport
// path, and the set-up phases of its main program (complab.cpp:1036-1290): geometry, flow solve with
// the Peclet rescale, the physical-unit chain that gives every species its relaxation rate and the
// time step, species lattices, biofilm automaton, equilibrium chemistry, precipitation. It is
// written against the public C ABI only, as a host program of the reference would be.
//
// What the file may hold and how it is read follows the reference: element names, defaults
// (tau 0.8, ns_max_iT 100000, ns_converge_iT1 1e-8 / iT2 1e-6, update intervals 1, unit um), the
// boundary-type words (Dirichlet, Neumann, closed / noflux / no_flux / wall, any case), nx counting
// interior planes (two ghost planes are added), Pe = 0 when delta_P is below 1e-14, a biofilm
// viscosity ratio n giving the permeability ratio 1/n. Compiled rate laws (the reference's
// defineRxnKinetics) are chosen after set-up with clb_set_kinetics; the run-time ones the file names
// (<symbolic> .sym laws, <graphnet> networks, per the organisms' reaction_type) are bound at set-up.
#include "../../include/clb.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_case_err;

clb_status case_fail(const std::string& m) {
    g_case_err = m;
    return CLB_INVALID_ARG;
}

// ------------------------------------------------------------------ a small XML reader
// Elements, text and nesting; comments, processing instructions and declarations are skipped,
// attributes are ignored (CompLaB.xml carries none that matter).
struct XNode {
    std::string name, text;
    std::vector<XNode> kids;
    const XNode* child(const std::string& n) const {
        for (const XNode& k : kids)
            if (k.name == n) return &k;
        return nullptr;
    }
};

struct XParser {
    const std::string& s;
    size_t p = 0;
    std::string err;
    explicit XParser(const std::string& src) : s(src) {}

    bool starts(const char* t) const { return s.compare(p, std::strlen(t), t) == 0; }
    bool skip_to(const char* t) {
        const size_t q = s.find(t, p);
        if (q == std::string::npos) return false;
        p = q + std::strlen(t);
        return true;
    }
    // skips comments, <?...?> and <!...> between elements; false on a malformed one
    bool skip_misc() {
        for (;;) {
            if (starts("<!--")) {
                if (!skip_to("-->")) return false;
            } else if (starts("<?")) {
                if (!skip_to("?>")) return false;
            } else if (starts("<!")) {
                if (!skip_to(">")) return false;
            } else {
                return true;
            }
            while (p < s.size() && std::isspace((unsigned char)s[p]) && s[p] != '<') ++p;
        }
    }
    bool element(XNode& out) {
        if (p >= s.size() || s[p] != '<') { err = "expected an element"; return false; }
        ++p;
        const size_t n0 = p;
        while (p < s.size() && !std::isspace((unsigned char)s[p]) && s[p] != '>' && s[p] != '/') ++p;
        out.name = s.substr(n0, p - n0);
        if (out.name.empty()) { err = "empty element name"; return false; }
        const size_t close = s.find('>', p);
        if (close == std::string::npos) { err = "unterminated tag <" + out.name; return false; }
        const bool empty = s[close - 1] == '/';
        p = close + 1;
        if (empty) return true;
        for (;;) {
            const size_t lt = s.find('<', p);
            if (lt == std::string::npos) { err = "unterminated element <" + out.name + ">"; return false; }
            out.text += s.substr(p, lt - p);
            p = lt;
            if (starts("</")) {
                p += 2;
                const size_t gt = s.find('>', p);
                if (gt == std::string::npos) { err = "unterminated end tag"; return false; }
                std::string nm = s.substr(p, gt - p);
                while (!nm.empty() && std::isspace((unsigned char)nm.back())) nm.pop_back();
                if (nm != out.name) { err = "<" + out.name + "> closed by </" + nm + ">"; return false; }
                p = gt + 1;
                return true;
            }
            if (starts("<!--") || starts("<?") || starts("<!")) {
                if (!skip_misc()) { err = "unterminated comment"; return false; }
                continue;
            }
            out.kids.emplace_back();
            if (!element(out.kids.back())) return false;
        }
    }
    bool document(XNode& root) {
        while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
        if (!skip_misc()) { err = "unterminated comment or declaration"; return false; }
        while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
        return element(root);
    }
};

std::string trim(const std::string& t) {
    size_t a = 0, b = t.size();
    while (a < b && std::isspace((unsigned char)t[a])) ++a;
    while (b > a && std::isspace((unsigned char)t[b - 1])) --b;
    return t.substr(a, b - a);
}

std::string lower(std::string t) {
    std::transform(t.begin(), t.end(), t.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return t;
}

// ------------------------------------------------------------------ the run description
struct Species {
    std::string name;
    double c0 = 0, d_pore = 0, d_bio = 0, left_bc = 0, right_bc = 0;
    int left = CLB_NEUMANN, right = CLB_NEUMANN, mobile = 1;
    double omega_pore = 0, omega_bio = 0;  // from the unit chain
};

struct Microbe {
    std::string name;
    int solver = 0;                       // 2: cellular automaton (the only kind this path runs)
    std::vector<int> codes;               // biofilm material numbers
    std::vector<double> b0;               // initial density per material number
    double visc_ratio = 0;                // viscosity_ratio_in_biofilm (permeability ratio 1/n)
    int rxn = 1;                          // reaction_type: 0 none, 1 kinetics (a compiled law the host
                                          // chooses), 3 a .srg surrogate, 8 a .sym law, 9 a .gnn network
    std::string sym_file;                 // <microbeN><expressions_file>: its own .sym law
    // a surrogate organism's uptake parameters (complab3d_metabolic.hh:814-960)
    std::vector<double> kc, vmax;         // half_saturation_constants, (fba_)maximum_uptake_flux
    double mw = 24.6, kd = 0.0;           // biomass_molar_mass (default 24.6), decay_coefficient (1/s)
};

}  // namespace

struct clb_case_s {
    std::string xml_dir, src_path = "src", input_path = "input", output_path = "output";
    // domain
    int nx = 0, ny = 0, nz = 0;           // nx with the two ghost planes
    double dx = 0, char_length = 0;       // dx in metres, the characteristic length in lattice units
    std::string geometry;
    std::vector<int> pore{2};
    int solid = 0, bounce_back = 1;
    // flow
    double delta_p = 0, peclet = 0, tau = 0.8;
    int ns_max1 = 100000, ns_max2 = 100000, ns_update = 1, ade_update = 1;
    double ns_eps1 = 1e-8, ns_eps2 = 1e-6;
    long long ade_max = 10000000;
    int vtk_interval = 0, chk_interval = 0;
    // chemistry, biology
    std::vector<Species> sp;
    std::vector<Microbe> mic;
    double bmax = 0, bfrac = 0;
    int ca_half = 0;
    bool enable_kinetics = false, enable_abiotic = false, biotic = false;
    // equilibrium
    bool eq_on = false;
    std::vector<std::string> components;
    std::vector<std::vector<double>> stoich;
    std::vector<double> logk;
    // run-time rate laws: <symbolic> (.sym files) and <graphnet> (.gnn networks)
    bool sym_on = false, gnn_on = false, srg_on = false;
    std::string sym_file, sym_abiotic, gnn_file, gnn_abiotic, srg_file;
    int srg_microbe = -1;                 // <surrogate><microbe>: the one organism, -1 every surrogate one
    // precipitation (one phase)
    bool prc_on = false;
    int prc_sub = -1, prc_interval = 1, prc_surface = 1;
    double prc_full = 0, prc_perm = 0;
    // derived
    std::map<std::string, double> val;
};

namespace {

// ---- typed reads along a path of element names; absent -> false (the reference's try/catch)
const XNode* at(const XNode& r, std::initializer_list<const char*> path) {
    const XNode* n = &r;
    for (const char* k : path) {
        n = n->child(k);
        if (!n) return nullptr;
    }
    return n;
}

bool read_str(const XNode* n, std::string& v) {
    if (!n) return false;
    v = trim(n->text);
    return true;
}

bool read_num(const XNode* n, double& v) {
    if (!n) return false;
    const std::string t = trim(n->text);
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    if (t.empty() || end != t.c_str() + t.size()) throw std::runtime_error("<" + n->name + "> is not a number: '" + t + "'");
    return true;
}

bool read_int(const XNode* n, int& v) {
    double d;
    if (!read_num(n, d)) return false;
    if (d != std::floor(d) || std::fabs(d) > 2e9) throw std::runtime_error("<" + n->name + "> is not an integer");
    v = (int)d;
    return true;
}

bool read_vec(const XNode* n, std::vector<double>& v) {
    if (!n) return false;
    std::istringstream in(n->text);
    v.clear();
    std::string tok;
    while (in >> tok) {
        char* end = nullptr;
        const double d = std::strtod(tok.c_str(), &end);
        if (end != tok.c_str() + tok.size()) throw std::runtime_error("<" + n->name + "> holds a non-number '" + tok + "'");
        v.push_back(d);
    }
    return true;
}

bool read_bool(const XNode* n, bool& v) {
    std::string t;
    if (!read_str(n, t)) return false;
    t = lower(t);
    if (t == "true" || t == "yes" || t == "1") v = true;
    else if (t == "false" || t == "no" || t == "0") v = false;
    else throw std::runtime_error("<" + n->name + "> should be true or false, not '" + t + "'");
    return true;
}

int face_type(const std::string& w, const std::string& what) {
    const std::string t = lower(w);
    if (t == "dirichlet") return CLB_DIRICHLET;
    if (t == "neumann") return CLB_NEUMANN;
    if (t == "closed" || t == "noflux" || t == "no_flux" || t == "wall") return CLB_CLOSED;
    throw std::runtime_error(what + " (" + w + ") should be Dirichlet, Neumann or closed");
}

void parse(clb_case_s& c, const XNode& root) {
    if (root.name != "parameters") throw std::runtime_error("the root element is <" + root.name + ">, not <parameters>");
    read_str(at(root, {"path", "src_path"}), c.src_path);
    read_str(at(root, {"path", "input_path"}), c.input_path);
    read_str(at(root, {"path", "output_path"}), c.output_path);
    read_bool(at(root, {"simulation_mode", "biotic_mode"}), c.biotic);
    read_bool(at(root, {"simulation_mode", "enable_kinetics"}), c.enable_kinetics);
    read_bool(at(root, {"simulation_mode", "enable_abiotic_kinetics"}), c.enable_abiotic);
    // LB_numerics (required: nx, ny, nz, dx, filename; complab_functions.hh:995-1003)
    const XNode* dom = at(root, {"LB_numerics", "domain"});
    if (!dom) throw std::runtime_error("<LB_numerics><domain> is missing");
    int nx = 0;
    if (!read_int(dom->child("nx"), nx) || !read_int(dom->child("ny"), c.ny) || !read_int(dom->child("nz"), c.nz))
        throw std::runtime_error("<domain> needs nx, ny and nz");
    if (nx < 1 || c.ny < 1 || c.nz < 1) throw std::runtime_error("<domain> sizes must be positive");
    c.nx = nx + 2;
    if (!read_num(dom->child("dx"), c.dx) || !(c.dx > 0)) throw std::runtime_error("<domain> needs a positive dx");
    if (!read_str(dom->child("filename"), c.geometry)) throw std::runtime_error("<domain> needs the geometry filename");
    read_num(at(root, {"LB_numerics", "delta_P"}), c.delta_p);
    read_num(at(root, {"LB_numerics", "Peclet"}), c.peclet);
    if (c.delta_p < 1e-14) c.peclet = 0;
    read_num(at(root, {"LB_numerics", "tau"}), c.tau);
    double cl = 0;
    const bool has_cl = read_num(dom->child("characteristic_length"), cl);
    if (!has_cl && c.peclet > 1e-14)
        throw std::runtime_error("characteristic_length must be given for a run with Pe > 0");
    std::string unit = "um";
    read_str(dom->child("unit"), unit);
    // the characteristic length is in the unit of dx: in lattice units it is cl / dx
    c.char_length = cl / c.dx;
    if (unit == "m") {
    } else if (unit == "mm") {
        c.dx *= 1e-3;
    } else if (unit == "um") {
        c.dx *= 1e-6;
    } else {
        throw std::runtime_error("unit (" + unit + ") must be m, mm or um");
    }
    if (const XNode* mn = dom->child("material_numbers")) {
        std::vector<double> v;
        if (read_vec(mn->child("pore"), v) && !v.empty()) {
            c.pore.clear();
            for (double d : v) c.pore.push_back((int)d);
        }
        read_int(mn->child("solid"), c.solid);
        read_int(mn->child("bounce_back"), c.bounce_back);
    }
    const XNode* it = at(root, {"LB_numerics", "iteration"});
    if (it) {
        read_int(it->child("ns_max_iT1"), c.ns_max1);
        read_int(it->child("ns_max_iT2"), c.ns_max2);
        read_num(it->child("ns_converge_iT1"), c.ns_eps1);
        read_num(it->child("ns_converge_iT2"), c.ns_eps2);
        read_int(it->child("ns_update_interval"), c.ns_update);
        read_int(it->child("ade_update_interval"), c.ade_update);
        double am = 0;
        if (read_num(it->child("ade_max_iT"), am)) c.ade_max = (long long)am;
    }
    read_int(at(root, {"IO", "save_VTK_interval"}), c.vtk_interval);
    read_int(at(root, {"IO", "save_CHK_interval"}), c.chk_interval);
    // chemistry (complab_functions.hh:1004-1030, 1281-1300; complab.cpp:441-458 <immobile>)
    int ns = 0;
    if (!read_int(at(root, {"chemistry", "number_of_substrates"}), ns) || ns < 0)
        throw std::runtime_error("<chemistry><number_of_substrates> is missing");
    if (ns > CLB_MAX_SPECIES) throw std::runtime_error("more substrates than the library's 16");
    for (int s = 0; s < ns; ++s) {
        const std::string nm = "substrate" + std::to_string(s);
        const XNode* n = at(root, {"chemistry", nm.c_str()});
        if (!n) throw std::runtime_error("<" + nm + "> is missing");
        Species S;
        if (!read_str(n->child("name_of_substrates"), S.name)) S.name = "substrate_" + std::to_string(s);
        std::string lt, rt;
        if (!read_str(n->child("left_boundary_type"), lt) || !read_str(n->child("right_boundary_type"), rt))
            throw std::runtime_error("<" + nm + "> needs left_boundary_type and right_boundary_type");
        S.left = face_type(lt, "left_boundary_type");
        S.right = face_type(rt, "right_boundary_type");
        if (!read_num(n->child("left_boundary_condition"), S.left_bc) ||
            !read_num(n->child("right_boundary_condition"), S.right_bc))
            throw std::runtime_error("<" + nm + "> needs left_boundary_condition and right_boundary_condition");
        if (!read_num(at(*n, {"substrate_diffusion_coefficients", "in_pore"}), S.d_pore) ||
            !read_num(at(*n, {"substrate_diffusion_coefficients", "in_biofilm"}), S.d_bio))
            throw std::runtime_error("<" + nm + "> needs its diffusion coefficients in pore and biofilm");
        if (!read_num(n->child("initial_concentration"), S.c0)) throw std::runtime_error("<" + nm + "> needs initial_concentration");
        bool imm = false;
        read_bool(n->child("immobile"), imm);
        S.mobile = imm ? 0 : 1;
        c.sp.push_back(S);
    }
    // microbiology: cellular-automaton microbes (complab_functions.hh:1036-1131, 1223-1236, 1380-1440)
    int nm = 0;
    read_int(at(root, {"microbiology", "number_of_microbes"}), nm);
    if (nm < 0 || nm > CLB_MAX_MICROBES) throw std::runtime_error("number_of_microbes out of range");
    for (int m = 0; m < nm; ++m) {
        const std::string bn = "microbe" + std::to_string(m);
        const XNode* n = at(root, {"microbiology", bn.c_str()});
        if (!n) throw std::runtime_error("<" + bn + "> is missing");
        Microbe M;
        if (!read_str(n->child("name_of_microbes"), M.name)) M.name = bn;
        std::string st;
        if (!read_str(n->child("solver_type"), st)) throw std::runtime_error("<" + bn + "> needs solver_type");
        const std::string stl = lower(st);
        if (stl == "ca" || stl == "cellular automata" || stl == "cellular_automata") M.solver = 2;
        else if (stl == "fd" || stl == "finite difference") M.solver = 1;
        else if (stl == "lbm" || stl == "lattice boltzmann") M.solver = 3;
        else throw std::runtime_error("solver_type " + st + " is not FD, CA or LBM");
        if (M.solver != 2)
            throw std::runtime_error("<" + bn + ">: only cellular-automaton microbes are on this path (FD and LBM biomass are not)");
        read_vec(n->child("initial_densities"), M.b0);
        std::vector<double> codes;
        read_vec(at(root, {"LB_numerics", "domain", "material_numbers", bn.c_str()}), codes);
        for (double d : codes) M.codes.push_back((int)d);
        if (M.codes.empty()) throw std::runtime_error("<material_numbers><" + bn + "> is missing for a biofilm microbe");
        if (M.codes.size() != M.b0.size())
            throw std::runtime_error("the material numbers and initial_densities of " + bn + " differ in length");
        if (!read_num(n->child("viscosity_ratio_in_biofilm"), M.visc_ratio))
            throw std::runtime_error("<" + bn + "> needs viscosity_ratio_in_biofilm (a cellular-automaton microbe)");
        // reaction_type (rxntype::parse, complab3d_metabolic.hh:207-236; kinetics when absent)
        std::string rt;
        if (read_str(n->child("reaction_type"), rt)) {
            const std::string r = lower(rt);
            if (r == "none" || r == "no" || r == "0") M.rxn = 0;
            else if (r == "kinetics" || r == "kns" || r == "1") M.rxn = 1;
            else if (r == "symbolic" || r == "sym" || r == "sym_law" || r == "rate_law" || r == "8") M.rxn = 8;
            else if (r == "graphnet" || r == "gnn" || r == "graph_network" || r == "graph" || r == "9") M.rxn = 9;
            else if (r == "symbolic_and_kinetics" || r == "symbolic+kinetics" || r == "10" ||
                     r == "graphnet_and_kinetics" || r == "graphnet+kinetics" || r == "11")
                throw std::runtime_error("<" + bn + ">: reaction_type " + rt +
                                         " (a run-time law and a compiled one on the same organism) is not on this path");
            else if (r == "surrogate" || r == "srg" || r == "ann" || r == "3") M.rxn = 3;
            else if (r == "glpk" || r == "fba" || r == "fba_glpk" || r == "cobrapy" || r == "cpy" ||
                     r == "fba_cobrapy" || r == "2" || r == "4" || r == "5" || r == "6" || r == "7" ||
                     r.find("_and_kinetics") != std::string::npos || r.find("+kinetics") != std::string::npos)
                throw std::runtime_error("<" + bn + ">: reaction_type " + rt +
                                         " (a flux-balance linear program, or one with a compiled law) is not on this path");
            else
                throw std::runtime_error("<" + bn + ">: reaction_type " + rt + " is not defined");
        }
        read_str(n->child("expressions_file"), M.sym_file);
        if (M.rxn == 3) {
            read_vec(n->child("half_saturation_constants"), M.kc);
            if (!read_vec(n->child("fba_maximum_uptake_flux"), M.vmax)) read_vec(n->child("maximum_uptake_flux"), M.vmax);
            for (double& v : M.vmax) v = std::fabs(v);
            read_num(n->child("biomass_molar_mass"), M.mw);
            read_num(n->child("decay_coefficient"), M.kd);
            if (!(M.mw > 0)) throw std::runtime_error("<" + bn + "> needs a positive biomass_molar_mass");
        }
        c.mic.push_back(M);
    }
    if (nm > 0) {
        if (!read_num(at(root, {"microbiology", "maximum_biomass_density"}), c.bmax))
            throw std::runtime_error("<microbiology> needs maximum_biomass_density");
        if (!read_num(at(root, {"microbiology", "thrd_biofilm_fraction"}), c.bfrac))
            throw std::runtime_error("<microbiology> needs thrd_biofilm_fraction");
        std::string cm;
        if (read_str(at(root, {"microbiology", "CA_method"}), cm)) {
            cm = lower(cm);
            if (cm == "half" || cm == "1" || cm == "yes") c.ca_half = 1;
            else if (cm == "fraction" || cm == "0" || cm == "no") c.ca_half = 0;
            else throw std::runtime_error("CA_method should be half or fraction");
        }
    }
    // equilibrium (complab.cpp:614-723)
    // run-time rate laws (complab3d_integration.hh:263-313): one .sym file for every symbolic
    // organism unless the organism names its own, one .gnn network for every graphnet organism, and
    // an abiotic file of either kind
    read_bool(at(root, {"symbolic", "enabled"}), c.sym_on);
    if (c.sym_on) {
        read_str(at(root, {"symbolic", "expressions_file"}), c.sym_file);
        read_str(at(root, {"symbolic", "abiotic_file"}), c.sym_abiotic);
    }
    read_bool(at(root, {"surrogate", "enabled"}), c.srg_on);
    if (c.srg_on) {
        read_str(at(root, {"surrogate", "weights_file"}), c.srg_file);
        read_int(at(root, {"surrogate", "microbe"}), c.srg_microbe);
        if (c.srg_file.empty()) throw std::runtime_error("<surrogate> is enabled but <weights_file> is not set");
    }
    read_bool(at(root, {"graphnet", "enabled"}), c.gnn_on);
    if (c.gnn_on) {
        read_str(at(root, {"graphnet", "network_file"}), c.gnn_file);
        read_str(at(root, {"graphnet", "abiotic_file"}), c.gnn_abiotic);
        if (c.gnn_file.empty() && c.gnn_abiotic.empty())
            throw std::runtime_error("<graphnet> is enabled but neither <network_file> nor <abiotic_file> is set");
    }
    for (size_t m = 0; m < c.mic.size(); ++m) {
        const Microbe& M = c.mic[m];
        if (M.rxn == 8 && (!c.sym_on || (c.sym_file.empty() && M.sym_file.empty())))
            throw std::runtime_error("microbe" + std::to_string(m) +
                                     " has reaction_type symbolic but <symbolic> names no file for it");
        if (M.rxn == 3 && (!c.srg_on || (c.srg_microbe >= 0 && c.srg_microbe != (int)m)))
            throw std::runtime_error("microbe" + std::to_string(m) +
                                     " has reaction_type surrogate but <surrogate> names no weights_file for it");
        if (M.rxn == 3 && (M.kc.size() != c.sp.size() || (!M.vmax.empty() && M.vmax.size() != c.sp.size())))
            throw std::runtime_error("microbe" + std::to_string(m) +
                                     ": half_saturation_constants and maximum_uptake_flux need one value per substrate");
        if (M.rxn == 9 && (!c.gnn_on || c.gnn_file.empty()))
            throw std::runtime_error("microbe" + std::to_string(m) +
                                     " has reaction_type graphnet but <graphnet> names no network_file");
    }
    if (c.sym_on && c.sym_file.empty() && c.sym_abiotic.empty()) {
        bool any = false;
        for (const Microbe& M : c.mic) any = any || !M.sym_file.empty();
        if (!any) throw std::runtime_error("<symbolic> is enabled but neither <expressions_file> nor <abiotic_file> is set");
    }
    if (c.sym_on && !c.sym_abiotic.empty() && c.gnn_on && !c.gnn_abiotic.empty())
        throw std::runtime_error("<symbolic> and <graphnet> both name an abiotic file; a run has one abiotic law");
    read_bool(at(root, {"equilibrium", "enabled"}), c.eq_on);
    if (c.eq_on) {
        std::string comp;
        if (!read_str(at(root, {"equilibrium", "components"}), comp)) throw std::runtime_error("<equilibrium> needs components");
        std::istringstream in(comp);
        std::string w;
        while (in >> w) c.components.push_back(w);
        for (int s = 0; s < ns; ++s) {
            const std::string k = "species" + std::to_string(s);
            std::vector<double> row;
            if (!read_vec(at(root, {"equilibrium", "stoichiometry", k.c_str()}), row)) row.assign(c.components.size(), 0.0);
            if (row.size() != c.components.size()) throw std::runtime_error("stoichiometry of " + k + " does not match the components");
            double lk = 0;
            read_num(at(root, {"equilibrium", "logK", k.c_str()}), lk);
            c.stoich.push_back(row);
            c.logk.push_back(lk);
        }
    }
    // precipitation (complab.cpp:470-500), one precipitate phase
    read_bool(at(root, {"precipitation", "enabled"}), c.prc_on);
    if (c.prc_on) {
        if (!read_int(at(root, {"precipitation", "solid_substrate"}), c.prc_sub) || c.prc_sub < 0 || c.prc_sub >= ns)
            throw std::runtime_error("<precipitation><solid_substrate> must name a substrate index");
        if (!read_num(at(root, {"precipitation", "max_precipRho"}), c.prc_full) || !(c.prc_full > 0))
            throw std::runtime_error("<precipitation><max_precipRho> must be positive");
        read_num(at(root, {"precipitation", "perm_ratio"}), c.prc_perm);
        read_int(at(root, {"precipitation", "update_interval"}), c.prc_interval);
        read_int(at(root, {"precipitation", "surface_only"}), c.prc_surface);
    }
    // the numbers by name
    auto& v = c.val;
    v["nx"] = c.nx; v["ny"] = c.ny; v["nz"] = c.nz; v["dx"] = c.dx; v["char_length"] = c.char_length;
    v["tau"] = c.tau; v["delta_P"] = c.delta_p; v["Peclet"] = c.peclet;
    v["ns_max_iT1"] = c.ns_max1; v["ns_max_iT2"] = c.ns_max2; v["ns_converge_iT1"] = c.ns_eps1;
    v["ns_converge_iT2"] = c.ns_eps2; v["ns_update_interval"] = c.ns_update; v["ade_update_interval"] = c.ade_update;
    v["ade_max_iT"] = (double)c.ade_max; v["n_substrates"] = ns; v["n_microbes"] = nm;
    v["save_VTK_interval"] = c.vtk_interval; v["equilibrium"] = c.eq_on; v["precipitation"] = c.prc_on;
    for (int s = 0; s < ns; ++s) {
        const std::string p = "substrate." + std::to_string(s) + ".";
        v[p + "c0"] = c.sp[s].c0; v[p + "d_pore"] = c.sp[s].d_pore; v[p + "d_biofilm"] = c.sp[s].d_bio;
        v[p + "left_type"] = c.sp[s].left; v[p + "right_type"] = c.sp[s].right;
        v[p + "left_bc"] = c.sp[s].left_bc; v[p + "right_bc"] = c.sp[s].right_bc; v[p + "mobile"] = c.sp[s].mobile;
    }
    for (int m = 0; m < nm; ++m) {
        const std::string p = "microbe." + std::to_string(m) + ".";
        v[p + "code"] = c.mic[m].codes[0];
        v[p + "perm_ratio"] = c.mic[m].visc_ratio > 1e-14 ? 1.0 / c.mic[m].visc_ratio : 0.0;
        v[p + "reaction_type"] = c.mic[m].rxn;
    }
    v["symbolic"] = c.sym_on;
    v["graphnet"] = c.gnn_on;
    v["surrogate"] = c.srg_on;
}

// The relaxation rates and the time step (complab.cpp:1221-1253). Substrate 0's pore diffusivity is
// the reference: ade_dt = refNu dx^2 / D_0, every species' lattice diffusivity is refNu D / D_0,
// tau = nu / cs2 + 1/2 with the D3Q7 cs2 = 1/4.
clb_status unit_chain(clb_case_s& c, double pore_mean_u) {
    const double cs2 = 0.25, thrd = 1e-14;
    double ref_nu, ref_tau;
    if (c.peclet > thrd) {
        ref_nu = pore_mean_u * c.char_length / c.peclet;
        ref_tau = ref_nu / cs2 + 0.5;
        if (ref_tau > 2 || ref_tau <= 0.5)
            return case_fail("the reference relaxation time " + std::to_string(ref_tau) + " is outside (0.5, 2]");
    } else {
        ref_tau = c.tau;
        ref_nu = cs2 * (ref_tau - 0.5);
    }
    if (c.sp.empty()) return CLB_OK;
    const double d0 = c.sp[0].d_pore;
    if (!(d0 > 0)) return case_fail("substrate 0 needs a positive pore diffusivity: every species is scaled against it");
    const double dt = ref_nu * c.dx * c.dx / d0;
    c.val["refNu"] = ref_nu;
    c.val["refTau"] = ref_tau;
    c.val["ade_dt"] = dt;
    for (size_t s = 0; s < c.sp.size(); ++s) {
        Species& S = c.sp[s];
        const double nu = s == 0 ? ref_nu : ref_nu * S.d_pore / d0;
        S.omega_pore = 1.0 / (nu / cs2 + 0.5);
        S.omega_bio = 1.0 / (ref_nu * S.d_bio / d0 / cs2 + 0.5);
        if (S.mobile) {
            const double tp = 1.0 / S.omega_pore, tb = 1.0 / S.omega_bio;
            if (!(tp > 0.5 && tp <= 2.0) || !(tb > 0.5 && tb <= 2.0))
                return case_fail("substrate " + S.name + ": relaxation time outside (0.5, 2] (pore " + std::to_string(tp) +
                                 ", biofilm " + std::to_string(tb) + ")");
        } else {
            S.omega_pore = S.omega_bio = 1.0;  // an immobile species never collides
        }
        const std::string p = "substrate." + std::to_string(s) + ".";
        c.val[p + "omega_pore"] = S.omega_pore;
        c.val[p + "omega_biofilm"] = S.omega_bio;
    }
    return CLB_OK;
}

std::string join_path(const std::string& a, const std::string& b) {
    if (b.empty() || b[0] == '/' || a.empty()) return b;
    return a + "/" + b;
}

}  // namespace

extern "C" {

const char* clb_case_error(void) { return g_case_err.c_str(); }

clb_status clb_case_load(const char* xml_path, clb_case** out) {
    if (!xml_path || !out) return case_fail("null argument");
    *out = nullptr;
    std::ifstream f(xml_path, std::ios::binary);
    if (!f) return case_fail(std::string("cannot open ") + xml_path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string src = ss.str();
    XNode root;
    XParser P(src);
    if (!P.document(root)) return case_fail(std::string(xml_path) + ": " + P.err);
    clb_case_s* c = new clb_case_s();
    try {
        parse(*c, root);
    } catch (const std::exception& e) {
        delete c;
        return case_fail(std::string(xml_path) + ": " + e.what());
    }
    if (c->peclet <= 1e-14) {
        // no flow: the unit chain needs nothing from a solve (refTau = tau)
        const clb_status st = unit_chain(*c, 0.0);
        if (st != CLB_OK) {
            delete c;
            return st;
        }
    }
    const std::string p = xml_path;
    const size_t slash = p.find_last_of('/');
    c->xml_dir = slash == std::string::npos ? "." : p.substr(0, slash);
    *out = c;
    return CLB_OK;
}

clb_status clb_case_free(clb_case* c) {
    delete c;
    return CLB_OK;
}

clb_status clb_case_get(const clb_case* c, const char* key, double* value) {
    if (!c || !key || !value) return case_fail("null argument");
    auto it = c->val.find(key);
    if (it == c->val.end()) return case_fail(std::string("no value named '") + key + "' (yet)");
    *value = it->second;
    return CLB_OK;
}

clb_status clb_case_setup(clb_case* c, int flow_precision, int ade_precision, clb_handle** out) {
    if (!c || !out) return case_fail("null argument");
    *out = nullptr;
    // geometry: <input_path>/<filename> beside the XML, interior planes, ghost planes duplicated
    const std::string gpath = join_path(join_path(c->xml_dir, c->input_path), c->geometry);
    std::vector<int8_t> mat((size_t)c->nx * c->ny * c->nz);
    clb_status st = clb_geom_read_dat(gpath.c_str(), c->nx - 2, c->ny, c->nz, mat.data());
    if (st != CLB_OK) return case_fail(clb_global_error());
    clb_domain_desc d;
    std::memset(&d, 0, sizeof d);
    d.nx = c->nx; d.ny = c->ny; d.nz = c->nz;
    d.flow_precision = flow_precision;
    d.ade_precision = ade_precision;
    d.solid_code = c->solid;
    d.bounce_back_code = c->bounce_back;
    d.n_pore_codes = (int32_t)std::min<size_t>(c->pore.size(), CLB_MAX_PORE_CODES);
    for (int i = 0; i < d.n_pore_codes; ++i) d.pore_codes[i] = c->pore[i];
    // biofilm materials: each microbe's first material number first (the automaton marks a voxel
    // with it), then the further numbers of every microbe, each with its microbe's permeability
    int nb = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (size_t m = 0; m < c->mic.size(); ++m)
            for (size_t k = pass == 0 ? 0 : 1; k < (pass == 0 ? 1 : c->mic[m].codes.size()); ++k) {
                if (nb >= CLB_MAX_MICROBES) return case_fail("more biofilm material numbers than the library's 8");
                d.bio_codes[nb] = c->mic[m].codes[k];
                d.perm_ratio[nb] = c->mic[m].visc_ratio > 1e-14 ? 1.0 / c->mic[m].visc_ratio : 0.0;
                ++nb;
            }
    d.n_microbes = nb;
    d.tau = c->tau;
    clb_handle* h = nullptr;
    if ((st = clb_create(&d, mat.data(), &h)) != CLB_OK) return case_fail(clb_global_error());
    auto bad = [&](clb_status s) {
        g_case_err = clb_last_error(h);
        clb_destroy(h);
        return s;
    };
    // flow (complab.cpp:1093-1183): skipped at Pe = 0
    double pore_mean_u = 0;
    if (c->peclet > 1e-14) {
        if ((st = clb_flow_init(h, c->delta_p)) != CLB_OK) return bad(st);
        int it = 0;
        double dp = c->delta_p;
        st = clb_flow_solve_peclet(h, c->peclet, c->char_length, 0.8, c->ns_max1, c->ns_eps1, &dp, &it);
        if (st != CLB_OK && st != CLB_NOT_CONVERGED) return bad(st);
        c->val["flow_converged"] = st == CLB_OK;
        c->val["flow_iterations"] = it;
        c->val["delta_P_used"] = dp;
        // PoreMeanU: over the pore and biofilm voxels of x = 1..nx-2 with biofilm materials present
        // and no rescale, else over every voxel of those planes (complab.cpp:1128-1150, 1173)
        std::vector<double> u((size_t)3 * mat.size());
        if ((st = clb_get_field(h, CLB_FIELD_FLOW_VELOCITY, 0, u.data(), 0)) != CLB_OK) return bad(st);
        const size_t N = mat.size(), P = (size_t)c->ny * c->nz;
        auto norm = [&](size_t n) { return std::sqrt(u[n] * u[n] + u[N + n] * u[N + n] + u[2 * N + n] * u[2 * N + n]); };
        const bool rescaled = std::fabs(dp - c->delta_p) > 0.0;
        if (!c->mic.empty() && !rescaled) {
            double tv = 0;
            long long tc = 0;
            for (int pc : c->pore) {
                double sum = 0;
                long long cnt = 0;
                for (size_t n = P; n < N - P; ++n)
                    if (mat[n] == pc) { sum += norm(n); ++cnt; }
                if (cnt) { tv += sum; tc += cnt; }
            }
            for (const Microbe& M : c->mic) {
                long long cnt = 0;
                double sum0 = 0;
                long long cnt0 = 0;
                for (size_t n = P; n < N - P; ++n) {
                    for (int code : M.codes)
                        if (mat[n] == code) ++cnt;
                    if (mat[n] == M.codes[0]) { sum0 += norm(n); ++cnt0; }
                }
                if (cnt0) tv += sum0 / (double)cnt0 * (double)cnt;
                tc += cnt;
            }
            pore_mean_u = tc ? tv / (double)tc : 0.0;
        } else {
            double sum = 0;
            for (size_t n = P; n < N - P; ++n) sum += norm(n);
            pore_mean_u = sum / (double)(N - 2 * P);
        }
        c->val["pore_mean_u"] = pore_mean_u;
    }
    if ((st = unit_chain(*c, pore_mean_u)) != CLB_OK) {
        clb_destroy(h);
        return st;
    }
    // species lattices (soluteDomainSetup), the velocity coupled
    std::vector<clb_species_desc> sd(c->sp.size());
    for (size_t s = 0; s < c->sp.size(); ++s) {
        const Species& S = c->sp[s];
        sd[s].omega_pore = S.omega_pore;
        sd[s].omega_biofilm = S.omega_bio;
        sd[s].mobile = S.mobile;
        sd[s].left_type = S.left;
        sd[s].right_type = S.right;
        sd[s].left_bc = S.left_bc;
        sd[s].right_bc = S.right_bc;
        sd[s].c0 = S.c0;
    }
    if (!sd.empty()) {
        if ((st = clb_ade_init(h, sd.data(), (int)sd.size())) != CLB_OK) return bad(st);
        if (c->peclet > 1e-14 && (st = clb_couple_velocity(h)) != CLB_OK) return bad(st);
        // the rates of every later kinetics law apply per time step ade_dt (set with no law yet)
        if ((st = clb_set_kinetics(h, CLB_LAW_NONE, nullptr, 0, c->val["ade_dt"])) != CLB_OK) return bad(st);
    }
    // biofilm: initial densities on their material numbers, then the automaton
    if (!c->mic.empty() && !sd.empty()) {
        const size_t N = mat.size();
        std::vector<double> bio(c->mic.size() * N, 0.0);
        for (size_t m = 0; m < c->mic.size(); ++m)
            for (size_t n = 0; n < N; ++n)
                for (size_t k = 0; k < c->mic[m].codes.size(); ++k)
                    if (mat[n] == c->mic[m].codes[k]) bio[m * N + n] = c->mic[m].b0[k];
        if ((st = clb_set_biomass(h, (int)c->mic.size(), bio.data())) != CLB_OK) return bad(st);
        clb_ca_desc cd;
        std::memset(&cd, 0, sizeof cd);
        cd.max_biomass = c->bmax;
        cd.biofilm_fraction = c->bfrac;
        cd.seed = 1;
        cd.push_mode = c->ca_half ? CLB_PUSH_HALF : CLB_PUSH_FRACTION;
        if ((st = clb_ca_setup(h, &cd)) != CLB_OK) return bad(st);
    }
    // run-time rate laws, bound to the substrates by name (files beside the XML): every symbolic
    // organism its .sym law, every graphnet organism the network, then the abiotic law
    if (!sd.empty() && (c->sym_on || c->gnn_on || c->srg_on)) {
        std::vector<const char*> names;
        for (const Species& S : c->sp) names.push_back(S.name.c_str());
        for (size_t m = 0; m < c->mic.size(); ++m) {
            const Microbe& M = c->mic[m];
            if (M.rxn == 8) {
                const std::string f = join_path(c->xml_dir, M.sym_file.empty() ? c->sym_file : M.sym_file);
                if ((st = clb_set_symbolic_kinetics(h, f.c_str(), names.data(), (int)m, M.name.c_str())) != CLB_OK)
                    return bad(st);
            } else if (M.rxn == 3) {
                const std::string f = join_path(c->xml_dir, c->srg_file);
                clb_surrogate_desc q;
                std::memset(&q, 0, sizeof q);
                for (size_t s = 0; s < c->sp.size(); ++s) {
                    q.half_saturation[s] = M.kc[s];
                    q.max_uptake_flux[s] = M.vmax.empty() ? 0.0 : M.vmax[s];
                }
                q.biomass_molar_mass = M.mw;
                q.decay = M.kd;
                if ((st = clb_set_surrogate_organism(h, f.c_str(), names.data(), (int)m, &q)) != CLB_OK) return bad(st);
            } else if (M.rxn == 9) {
                const std::string f = join_path(c->xml_dir, c->gnn_file);
                if ((st = clb_set_graph_network(h, f.c_str(), names.data(), (int)m)) != CLB_OK) return bad(st);
            }
        }
        if (c->sym_on && !c->sym_abiotic.empty()) {
            const std::string f = join_path(c->xml_dir, c->sym_abiotic);
            if ((st = clb_set_symbolic_kinetics(h, f.c_str(), names.data(), -1, "")) != CLB_OK) return bad(st);
        }
        if (c->gnn_on && !c->gnn_abiotic.empty()) {
            const std::string f = join_path(c->xml_dir, c->gnn_abiotic);
            if ((st = clb_set_graph_network(h, f.c_str(), names.data(), -1)) != CLB_OK) return bad(st);
        }
    }
    // equilibrium chemistry: rows are the substrates, columns the named components
    if (c->eq_on) {
        clb_speciation_desc q;
        std::memset(&q, 0, sizeof q);
        q.n_species = (int32_t)c->sp.size();
        q.n_components = (int32_t)c->components.size();
        if (q.n_species > CLB_MAX_EQ_SPECIES || q.n_components > CLB_MAX_COMPONENTS) {
            clb_destroy(h);
            return case_fail("the equilibrium tableau is larger than the library's 16 x 8");
        }
        for (int s = 0; s < q.n_species; ++s) {
            for (int j = 0; j < q.n_components; ++j) q.stoich[s][j] = c->stoich[s][j];
            q.logK[s] = c->logk[s];
        }
        for (int j = 0; j < q.n_components; ++j) {
            q.component_species[j] = -1;
            for (size_t s = 0; s < c->sp.size(); ++s)
                if (c->sp[s].name == c->components[j]) q.component_species[j] = (int32_t)s;
        }
        q.tolerance = 1e-10;
        q.max_iterations = 200;
        if ((st = clb_speciation_setup(h, &q)) != CLB_OK) return bad(st);
        if ((st = clb_set_speciation_mode(h, CLB_SPEC_NR)) != CLB_OK) return bad(st);
    }
    if (c->prc_on) {
        clb_precip_desc pd;
        std::memset(&pd, 0, sizeof pd);
        pd.mineral_species = c->prc_sub;
        pd.full_density = c->prc_full;
        pd.precip_code = -1;
        pd.seal_flow = c->peclet > 1e-14 ? 1 : 0;
        pd.seal_perm_ratio = c->prc_perm;
        pd.flow_max_iterations = c->ns_max2;
        pd.flow_eps = c->ns_eps2;
        pd.reopen_fraction = 0.9;
        pd.pore_code = -1;
        pd.dissolution_surface_only = 1;
        if ((st = clb_precip_setup(h, &pd)) != CLB_OK) return bad(st);
    }
    *out = h;
    return CLB_OK;
}

clb_status clb_case_run(clb_case* c, clb_handle* h, int iterations, const char* output_dir, clb_run_report* report) {
    if (!c || !h) return case_fail("null argument");
    clb_run_report total;
    std::memset(&total, 0, sizeof total);
    const int n = iterations >= 0 ? iterations : (int)std::min<long long>(c->ade_max, 2000000000LL);
    const int chunk = (output_dir && c->vtk_interval > 0) ? c->vtk_interval : n;
    clb_run_desc d;
    std::memset(&d, 0, sizeof d);
    d.ca = c->mic.empty() ? 0 : 1;
    d.ade_update_interval = c->ade_update;
    d.ns_update_interval = c->peclet > 1e-14 ? c->ns_update : 0;
    d.geometry_interval = c->prc_on ? c->prc_interval : 0;
    d.flow_max_iterations = c->ns_max2;
    d.flow_eps = c->ns_eps2;
    int done = 0;
    clb_status st = CLB_OK;
    while (done < n && st == CLB_OK) {
        d.iterations = std::min(chunk, n - done);
        clb_run_report r;
        st = clb_run(h, &d, &r);
        total.iterations += r.iterations; total.ca_sweeps += r.ca_sweeps; total.mask_changes += r.mask_changes;
        total.flow_resolves += r.flow_resolves; total.flow_iterations += r.flow_iterations;
        total.flow_unconverged += r.flow_unconverged; total.sealed += r.sealed; total.reopened += r.reopened;
        total.ms_transport += r.ms_transport; total.ms_ca += r.ms_ca; total.ms_flow += r.ms_flow;
        total.ms_geometry += r.ms_geometry; total.seconds += r.seconds; total.launches += r.launches;
        done += (int)r.iterations;
        if (st != CLB_OK) break;
        if (output_dir && c->vtk_interval > 0) {
            // writeAdvVTI: <name>_<7-digit iteration>.vti per substrate (complab_functions.hh:96-176)
            for (size_t s = 0; s < c->sp.size(); ++s) {
                char name[64];
                std::snprintf(name, sizeof name, "_%07d.vti", done);
                const std::string path = join_path(output_dir, c->sp[s].name + name);
                if ((st = clb_write_vti(h, CLB_FIELD_CONCENTRATION, (int)s, path.c_str())) != CLB_OK) break;
            }
        }
    }
    if (report) *report = total;
    if (st != CLB_OK) g_case_err = clb_last_error(h);
    return st;
}

}  // extern "C"

// runner.cpp -- RuNNer parameter-file reader of the engine.
//
// Follows parseRuNNerInput (hdnnps.f90:34-233): the keywords honoured, the
// element order (sorted by atomic number, stable), the symmetry-function
// order (stable sort on the key that symfunctionstring builds with the edit
// descriptors (I2,3F9.5,I3) / (I2,4F9.5,3I3) and lambda+10, hdnnps.f90:254-265),
// the scaling.data record order and index check (:283-294) and the
// weights.NNN.data order (for each layer: for iin: for iout: W(iout,iin),
// then the biases; :318-327).  Keyword order rules are those of the
// reference: 'elements' needs 'number_of_elements' first and
// 'global_nodes_short' needs 'global_hidden_layers_short' first.
//
// Hardening over the reference (which prints and stops): errors are
// returned; no cap of 200 symmetry functions per element; symmetry-function
// types other than 2 and 3 and inconsistent network sizes are rejected;
// 'cutoff_type' must be 2 when it is given.  The reference ignores the
// keyword and always evaluates the tanh^3 cutoff of
// symmetryFunctions.f90:310-327, which is RuNNer's cutoff_type 2 (the
// reference's own example, example/hdnnp-params/input.nn:70); a potential
// trained with another cutoff would load there without complaint and give
// wrong energies and forces, so it is refused here.  A file without the
// keyword loads, as in the reference.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "model.h"

namespace hdnnp {

static const char* const kSymbols[kMaxZ] = {
    "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",  "Cl", "Ar",
    "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr",
    "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe",
    "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf",
    "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th",
    "Pa", "U",  "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr", "Rf", "Db", "Sg", "Bh", "Hs",
    "Mt", "Ds", "Rg", "Cn", "Nh", "Fl", "Mc", "Lv", "Ts", "Og"};

int symbol_to_z(const std::string& s) {
    for (int i = 0; i < kMaxZ; ++i)
        if (s == kSymbols[i]) return i + 1;
    return -1;
}

namespace {

std::vector<std::string> tokens(const std::string& line) {
    std::vector<std::string> out;
    std::istringstream is(line);
    std::string t;
    while (is >> t) out.push_back(t);
    return out;
}

bool to_real(const std::string& s, double& v) {
    std::string t(s);
    for (auto& c : t)
        if (c == 'd' || c == 'D') c = 'e';  // Fortran double-precision exponent
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end != t.c_str();
}

bool to_int(const std::string& s, int& v) {
    char* end = nullptr;
    long x = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str()) return false;
    v = static_cast<int>(x);
    return true;
}

std::string fmt_f(double x) {  // Fortran F9.5 (asterisks on overflow)
    char b[64];
    int n = std::snprintf(b, sizeof b, "%9.5f", x);
    return n > 9 ? std::string(9, '*') : std::string(b);
}

std::string fmt_i(int x, int w) {  // Fortran Iw
    char b[32];
    int n = std::snprintf(b, sizeof b, "%*d", w, x);
    return n > w ? std::string(w, '*') : std::string(b);
}

std::string sort_key(const SymFn& f) {
    if (f.type == 2) return fmt_i(2, 2) + fmt_f(f.rcut) + fmt_f(f.eta) + fmt_f(f.rs) + fmt_i(f.z1, 3);
    return fmt_i(3, 2) + fmt_f(f.rcut) + fmt_f(f.eta) + fmt_f(f.zeta) + fmt_f(f.lambda + 10.0) + fmt_i(f.z1, 3) +
           fmt_i(f.z2, 3);
}

}  // namespace

bool load_runner(const std::string& dir_in, HostModel& m, std::string& err) {
    std::string dir = dir_in;
    if (dir.empty() || dir.back() != '/') dir += '/';
    std::ifstream in(dir + "input.nn");
    if (!in) {
        err = dir + "input.nn not found";
        return false;
    }
    int n_el = -1, n_hidden = -1;
    std::vector<std::string> syms;
    std::vector<int> nodes;
    std::vector<char> acts;
    std::vector<std::vector<SymFn>> by_z(kMaxZ + 1);
    double atom_e[kMaxZ + 1] = {0};
    std::string line;
    int lineno = 0;
    auto bad = [&](const std::string& what) {
        err = "input.nn line " + std::to_string(lineno) + ": " + what;
        return false;
    };
    while (std::getline(in, line)) {
        ++lineno;
        auto w = tokens(line);
        if (w.empty()) continue;
        const std::string& key = w[0];
        if (key == "number_of_elements") {
            if (w.size() < 2 || !to_int(w[1], n_el) || n_el < 1 || n_el > kMaxElements)
                return bad("number_of_elements must be 1.." + std::to_string(kMaxElements));
        } else if (key == "elements") {
            if (n_el < 0) return bad("'elements' before 'number_of_elements'");
            if ((int)w.size() < n_el + 1) return bad("fewer symbols than number_of_elements");
            syms.assign(w.begin() + 1, w.begin() + 1 + n_el);
            for (auto& s : syms)
                if (symbol_to_z(s) < 1) return bad("unknown element '" + s + "'");
        } else if (key == "atom_energy") {
            double e;
            int z = w.size() >= 3 ? symbol_to_z(w[1]) : -1;
            if (z < 1 || !to_real(w[2], e)) return bad("bad atom_energy");
            atom_e[z] = e;
        } else if (key == "cutoff_type") {
            int ct = -1;
            if (w.size() < 2 || !to_int(w[1], ct)) return bad("bad cutoff_type");
            if (ct != 2)
                return bad("cutoff_type " + w[1] +
                           " is not supported: the symmetry functions use the tanh^3 cutoff (cutoff_type 2)");
        } else if (key == "scale_symmetry_functions") {
            m.scalesf = true;
        } else if (key == "center_symmetry_functions") {
            m.centersf = true;
        } else if (key == "global_hidden_layers_short") {
            if (w.size() < 2 || !to_int(w[1], n_hidden) || n_hidden < 0 || n_hidden + 1 > kMaxLayers)
                return bad("global_hidden_layers_short must be 0.." + std::to_string(kMaxLayers - 1));
            nodes.assign(n_hidden + 1, 1);
            acts.assign(n_hidden + 1, 'l');
        } else if (key == "global_nodes_short") {
            if (n_hidden < 0) return bad("'global_nodes_short' before 'global_hidden_layers_short'");
            if ((int)w.size() < n_hidden + 1) return bad("too few entries in global_nodes_short");
            for (int i = 0; i < n_hidden; ++i)
                if (!to_int(w[1 + i], nodes[i]) || nodes[i] < 1 || nodes[i] > kMaxWidth)
                    return bad("layer width must be 1.." + std::to_string(kMaxWidth));
            nodes[n_hidden] = 1;
        } else if (key == "global_activation_short") {
            if (n_hidden < 0) return bad("'global_activation_short' before 'global_hidden_layers_short'");
            if ((int)w.size() < n_hidden + 2) return bad("too few entries in global_activation_short");
            for (int i = 0; i <= n_hidden; ++i) {
                char a = w[1 + i][0];
                if (a != 'l' && a != 't' && a != 'p' && a != 'r') return bad(std::string("unknown activation '") + a + "'");
                acts[i] = a;
            }
        } else if (key == "symfunction_short") {
            int type;
            if (w.size() < 3 || !to_int(w[2], type)) return bad("bad symfunction_short");
            SymFn f;
            f.type = type;
            int zc = symbol_to_z(w[1]);
            if (type == 2) {
                if (w.size() < 7) return bad("type-2 symfunction needs 7 fields");
                f.z1 = symbol_to_z(w[3]);
                if (!to_real(w[4], f.eta) || !to_real(w[5], f.rs) || !to_real(w[6], f.rcut))
                    return bad("bad type-2 symfunction numbers");
            } else if (type == 3) {
                if (w.size() < 9) return bad("type-3 symfunction needs 9 fields");
                f.z1 = symbol_to_z(w[3]);
                f.z2 = symbol_to_z(w[4]);
                if (!to_real(w[5], f.eta) || !to_real(w[6], f.lambda) || !to_real(w[7], f.zeta) ||
                    !to_real(w[8], f.rcut))
                    return bad("bad type-3 symfunction numbers");
                if (f.z2 < 1) return bad("unknown element in symfunction");
            } else {
                return bad("symmetry function type " + std::to_string(type) + " is not supported (only 2 and 3)");
            }
            if (zc < 1 || f.z1 < 1) return bad("unknown element in symfunction");
            if (std::find(syms.begin(), syms.end(), w[1]) == syms.end())
                return bad("symfunction for an element not listed in 'elements'");
            if (!(f.rcut > 0)) return bad("symfunction cutoff must be positive");
            by_z[zc].push_back(f);
        }
    }
    if (syms.empty()) {
        err = "input.nn: no 'elements' keyword";
        return false;
    }
    if (n_hidden < 0) {
        err = "input.nn: no 'global_hidden_layers_short' keyword";
        return false;
    }
    std::vector<int> zs;
    for (auto& s : syms) zs.push_back(symbol_to_z(s));
    std::stable_sort(zs.begin(), zs.end());
    for (size_t i = 1; i < zs.size(); ++i)
        if (zs[i] == zs[i - 1]) {
            err = "input.nn: element listed twice";
            return false;
        }
    m.el.clear();
    m.max_rc = 0;
    for (size_t e = 0; e < zs.size(); ++e) {
        ElementModel em;
        em.z = zs[e];
        em.atom_energy = atom_e[em.z];
        auto& v = by_z[em.z];
        std::vector<std::pair<std::string, size_t>> keyed;
        for (size_t i = 0; i < v.size(); ++i) keyed.emplace_back(sort_key(v[i]), i);
        std::stable_sort(keyed.begin(), keyed.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        for (auto& k : keyed) em.sfs.push_back(v[k.second]);
        for (auto& f : em.sfs) {
            if (m.z2e[f.z1] < 0 && std::find(zs.begin(), zs.end(), f.z1) == zs.end()) {
                err = "symfunction refers to an element that is not in the potential";
                return false;
            }
            if (f.type == 3 && std::find(zs.begin(), zs.end(), f.z2) == zs.end()) {
                err = "symfunction refers to an element that is not in the potential";
                return false;
            }
            // all SFs of one element share one cutoff (symmetryFunctions.f90:195-198)
            if ((f.rcut - em.sfs[0].rcut) * (f.rcut - em.sfs[0].rcut) > 1e-10) {
                err = "all symmetry functions of one element must share the cutoff";
                return false;
            }
            m.max_rc = std::max(m.max_rc, f.rcut);
        }
        if (em.sfs.empty()) {
            err = "element without symmetry functions";
            return false;
        }
        m.z2e[em.z] = (int)e;
        m.el.push_back(std::move(em));
    }

    // scaling.data
    {
        std::ifstream sc(dir + "scaling.data");
        if (!sc) {
            err = dir + "scaling.data not found";
            return false;
        }
        for (size_t e = 0; e < m.el.size(); ++e) {
            auto& v = m.el[e].sfs;
            for (size_t s = 0; s < v.size(); ++s) {
                std::vector<std::string> w;
                while (w.empty() && std::getline(sc, line)) w = tokens(line);
                int ie, is;
                if (w.size() < 5 || !to_int(w[0], ie) || !to_int(w[1], is) || !to_real(w[2], v[s].smin) ||
                    !to_real(w[3], v[s].smax) || !to_real(w[4], v[s].smean)) {
                    err = "scaling.data: malformed or short";
                    return false;
                }
                if (ie != (int)e + 1 || is != (int)s + 1) {
                    err = "scaling.data: wrong index (expected element " + std::to_string(e + 1) + ", SF " +
                          std::to_string(s + 1) + ")";
                    return false;
                }
                if (m.scalesf && !(v[s].smax - v[s].smin != 0.0)) {
                    err = "scaling.data: zero range (max == min) with scale_symmetry_functions";
                    return false;
                }
            }
        }
        std::vector<std::string> w;
        while (w.empty() && std::getline(sc, line)) w = tokens(line);
        if (w.size() < 2 || !to_real(w[0], m.emin) || !to_real(w[1], m.emax)) {
            err = "scaling.data: missing 'emin emax' record";
            return false;
        }
    }

    // weights.NNN.data
    for (auto& em : m.el) {
        int nin = (int)em.sfs.size();
        em.net.clear();
        for (int l = 0; l <= n_hidden; ++l) {
            Layer L;
            L.nin = nin;
            L.nout = nodes[l];
            L.act = acts[l];
            L.w.assign((size_t)L.nin * L.nout, 0.0);
            L.b.assign(L.nout, 0.0);
            em.net.push_back(L);
            nin = L.nout;
        }
        char fn[32];
        std::snprintf(fn, sizeof fn, "weights.%03d.data", em.z);
        std::ifstream wf(dir + fn);
        if (!wf) {
            err = dir + fn + " not found";
            return false;
        }
        auto next = [&](double& v) {
            while (std::getline(wf, line)) {
                auto w = tokens(line);
                if (!w.empty()) return to_real(w[0], v);
            }
            return false;
        };
        for (auto& L : em.net) {
            for (int i = 0; i < L.nin; ++i)
                for (int o = 0; o < L.nout; ++o)
                    if (!next(L.w[(size_t)o * L.nin + i])) {
                        err = std::string(fn) + ": too few values";
                        return false;
                    }
            for (int o = 0; o < L.nout; ++o)
                if (!next(L.b[o])) {
                    err = std::string(fn) + ": too few values";
                    return false;
                }
        }
    }
    return true;
}

}  // namespace hdnnp

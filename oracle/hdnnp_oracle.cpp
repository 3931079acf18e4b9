// hdnnp_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A CPU, FP64 restatement of the reference HDNNP prediction path
// (Jonas-Finkler/High-Dimensional-Neural-Network-Potential, Fortran 2008).
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
// load this library, and only as the checker / the timed CPU baseline.  The
// product (libhdnnp_b200.so) never links or calls it.
//
// Parity status: the reference cannot be compiled in this image (no Fortran
// compiler: gfortran/flang/ifort/lfortran are all absent) and it ships no
// golden outputs, so this restatement is NOT pinned against reference
// binaries ("parity unpinned" w.r.t. reference outputs).  It is pinned
// instead by tests/test_oracle.py against (i) an independent torch-autograd
// FP64 restatement of the energy, (ii) central finite differences of E for
// forces and for dE/dh, (iii) the fused vs. the single-SF routines, (iv) the
// cell-list vs. the O(N^2) neighbour list, and (v) invariances.
//
// Every routine below names the reference routine (file:line) it follows.
// Loop orders, the integer-zeta power path, the eta cache, the neighbour-list
// enumeration order and the scaling semantics follow the reference.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp).

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------- elements
// Element symbols in order of atomic number (constants.f90:29 holds the same
// table; the element -> number mapping is the standard periodic table).
static const char* kSym[118] = {
    "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar",
    "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr",
    "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe",
    "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu",
    "Hf", "Ta", "W", "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn",
    "Fr", "Ra", "Ac", "Th", "Pa", "U", "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr",
    "Rf", "Db", "Sg", "Bh", "Hs", "Mt", "Ds", "Rg", "Cn", "Nh", "Fl", "Mc", "Lv", "Ts", "Og"};

// elemSymToNum (constants.f90:95): exact, case-sensitive match; -1 if unknown.
static int sym_to_z(const std::string& s) {
    for (int i = 0; i < 118; ++i)
        if (s == kSym[i]) return i + 1;
    return -1;
}

// ---------------------------------------------------------------- model
struct SymFn {              // symFunction (symmetryFunctions.f90:7-16)
    int type = 0;           // 2 (radial G2) or 3 (angular G4)
    int el1 = 0, el2 = 0;   // neighbour elements (el2 only for type 3)
    double rcut = 0, eta = 0, lambda = 0, zeta = 0, rs = 0;
    double smin = 0, smax = 0, smean = 0;
};

struct Layer {              // nnLayer (neuralNetworks.f90:12-22)
    int nin = 0, nout = 0;
    char act = 'l';
    std::vector<double> w;  // weights(nOut, nIn), column-major: w[o + nout*i]
    std::vector<double> b;
};

struct Model {              // type hdnnp (hdnnps.f90:13-21)
    std::vector<int> elements;                 // atomic numbers sorted by Z
    std::vector<std::vector<SymFn>> sfs;       // indexed by Z (0..118)
    std::vector<std::vector<Layer>> nets;      // indexed by Z
    double maxRc = 0, emin = 0, emax = 0;
    double atomenergy[119] = {0};
    bool scalesf = false, centersf = false;
    Model() : sfs(119), nets(119) {}
};

static thread_local std::string g_err;

static bool fail(const std::string& m) {
    g_err = m;
    return false;
}

// splitString (util.f90:128): blank separated words.
static std::vector<std::string> split_words(const std::string& line) {
    std::vector<std::string> w;
    std::string cur;
    for (char c : line) {
        if (c == ' ' || c == '\t' || c == '\r' || c == '\n') {
            if (!cur.empty()) { w.push_back(cur); cur.clear(); }
        } else {
            cur.push_back(c);
        }
    }
    if (!cur.empty()) w.push_back(cur);
    return w;
}

// Fortran list-directed REAL read: accepts d/D exponents.
static bool read_real(const std::string& s, double& v) {
    std::string t = s;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'e';
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end != t.c_str();
}

static bool read_int(const std::string& s, int& v) {
    char* end = nullptr;
    long x = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str()) return false;
    v = (int)x;
    return true;
}

// symfunctionstring (hdnnps.f90:254-265): the sort key, formatted like the
// Fortran edit descriptors (I2,3F9.5,I3) and (I2,4F9.5,3I3) with lambda+10.
static std::string f95(double x) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%9.5f", x);
    std::string s(buf);
    if (s.size() > 9) s = std::string(9, '*');  // Fortran overflow fill
    return s;
}
static std::string ii(int x, int w) {
    char buf[32];
    std::snprintf(buf, sizeof buf, "%*d", w, x);
    std::string s(buf);
    if ((int)s.size() > w) s = std::string(w, '*');
    return s;
}
static std::string sf_key(const SymFn& f) {
    if (f.type == 2) return ii(2, 2) + f95(f.rcut) + f95(f.eta) + f95(f.rs) + ii(f.el1, 3);
    return ii(3, 2) + f95(f.rcut) + f95(f.eta) + f95(f.zeta) + f95(f.lambda + 10.0) + ii(f.el1, 3) +
           ii(f.el2, 3);
}

// parseRuNNerInput (hdnnps.f90:34-233) + sortSymFunctions (:235-252) +
// readScaling (:269-300) + readWeights (:302-330).
// cap_sfs > 0 reproduces the reference's nmaxSFs limit (hdnnps.f90:48).
static bool load_runner(const std::string& path, int cap_sfs, Model& m) {
    std::ifstream in(path + "input.nn");
    if (!in) return fail(path + "input.nn not found");
    int nEls = -1, nlayers = -1;
    std::vector<std::string> elsyms;
    std::vector<int> nnodes;
    std::vector<char> act;
    bool have_elements = false;
    std::string line;
    double maxrc = 0;
    while (std::getline(in, line)) {
        auto w = split_words(line);
        if (w.empty()) continue;
        const std::string& k = w[0];
        if (k == "number_of_elements") {
            if (w.size() < 2 || !read_int(w[1], nEls) || nEls <= 0) return fail("bad number_of_elements");
        } else if (k == "elements") {
            if (nEls < 0) return fail("'elements' before 'number_of_elements'");
            if ((int)w.size() < 1 + nEls) return fail("too few symbols after 'elements'");
            elsyms.assign(w.begin() + 1, w.begin() + 1 + nEls);
            for (auto& s : elsyms) {
                int z = sym_to_z(s);
                if (z < 1) return fail("unknown element " + s);
                m.sfs[z].clear();
            }
            have_elements = true;
        } else if (k == "atom_energy") {
            double e;
            if (w.size() < 3 || !read_real(w[2], e)) return fail("bad atom_energy line");
            int z = sym_to_z(w[1]);
            if (z < 1) return fail("unknown element in atom_energy: " + w[1]);
            m.atomenergy[z] = e;
        } else if (k == "scale_symmetry_functions") {
            m.scalesf = true;
        } else if (k == "center_symmetry_functions") {
            m.centersf = true;
        } else if (k == "global_hidden_layers_short") {
            if (w.size() < 2 || !read_int(w[1], nlayers) || nlayers < 0) return fail("bad global_hidden_layers_short");
            nnodes.assign(nlayers + 1, 0);
            act.assign(nlayers + 1, 'l');
        } else if (k == "global_nodes_short") {
            if (nlayers < 0) return fail("'global_nodes_short' before 'global_hidden_layers_short'");
            if ((int)w.size() < 1 + nlayers) return fail("too few entries in global_nodes_short");
            for (int i = 0; i < nlayers; ++i)
                if (!read_int(w[1 + i], nnodes[i])) return fail("bad global_nodes_short");
            nnodes[nlayers] = 1;
        } else if (k == "global_activation_short") {
            if (nlayers < 0) return fail("'global_activation_short' before 'global_hidden_layers_short'");
            if ((int)w.size() < 2 + nlayers) return fail("too few entries in global_activation_short");
            for (int i = 0; i <= nlayers; ++i) act[i] = w[1 + i][0];
            nnodes[nlayers] = 1;
        } else if (k == "symfunction_short") {
            if (w.size() < 3) return fail("bad symfunction_short line");
            int t;
            if (!read_int(w[2], t)) return fail("bad symfunction type");
            SymFn f;
            int zc;
            if (t == 2) {
                if (w.size() < 7) return fail("short type-2 symfunction line");
                zc = sym_to_z(w[1]);
                f.type = 2;
                f.el1 = sym_to_z(w[3]);
                if (!read_real(w[4], f.eta) || !read_real(w[5], f.rs) || !read_real(w[6], f.rcut))
                    return fail("bad type-2 symfunction numbers");
            } else if (t == 3) {
                if (w.size() < 9) return fail("short type-3 symfunction line");
                zc = sym_to_z(w[1]);
                f.type = 3;
                f.el1 = sym_to_z(w[3]);
                f.el2 = sym_to_z(w[4]);
                if (!read_real(w[5], f.eta) || !read_real(w[6], f.lambda) || !read_real(w[7], f.zeta) ||
                    !read_real(w[8], f.rcut))
                    return fail("bad type-3 symfunction numbers");
            } else {
                continue;  // the reference silently ignores other types
            }
            if (zc < 1) return fail("unknown centre element " + w[1]);
            if (!have_elements || std::find(elsyms.begin(), elsyms.end(), w[1]) == elsyms.end())
                return fail("symfunction for element not in 'elements': " + w[1]);
            if (f.rcut > maxrc) maxrc = f.rcut;
            if (cap_sfs > 0 && (int)m.sfs[zc].size() + 1 > cap_sfs)
                return fail("more symmetry functions in input file than nmaxSFs allows");
            m.sfs[zc].push_back(f);
        }
    }
    if (!have_elements) return fail("no 'elements' keyword");
    if (nlayers < 0) return fail("no 'global_hidden_layers_short' keyword");
    m.maxRc = maxrc;

    // elements sorted by Z with a stable sort (mergesort, sorting.f90:26).
    std::vector<int> zs;
    for (auto& s : elsyms) zs.push_back(sym_to_z(s));
    std::stable_sort(zs.begin(), zs.end());
    m.elements = zs;

    // sortSymFunctions: stable sort by the formatted key (mergesortStr, sorting.f90:105).
    for (int z : zs) {
        auto& v = m.sfs[z];
        std::vector<std::pair<std::string, int>> keyed;
        for (int i = 0; i < (int)v.size(); ++i) keyed.push_back({sf_key(v[i]), i});
        std::stable_sort(keyed.begin(), keyed.end(),
                         [](const std::pair<std::string, int>& a, const std::pair<std::string, int>& b) {
                             return a.first < b.first;
                         });
        std::vector<SymFn> sorted;
        for (auto& kv : keyed) sorted.push_back(v[kv.second]);
        v = sorted;
    }

    // readScaling
    {
        std::ifstream sc(path + "scaling.data");
        if (!sc) return fail(path + "scaling.data not found");
        for (int ie = 0; ie < (int)zs.size(); ++ie) {
            auto& v = m.sfs[zs[ie]];
            for (int isf = 0; isf < (int)v.size(); ++isf) {
                if (!std::getline(sc, line)) return fail("scaling.data too short");
                auto w = split_words(line);
                int riel, risf;
                if (w.size() < 5 || !read_int(w[0], riel) || !read_int(w[1], risf) || !read_real(w[2], v[isf].smin) ||
                    !read_real(w[3], v[isf].smax) || !read_real(w[4], v[isf].smean))
                    return fail("bad scaling.data line");
                if (riel != ie + 1 || risf != isf + 1) return fail("wrong index reading scaling.data");
            }
        }
        if (!std::getline(sc, line)) return fail("scaling.data: missing emin emax");
        auto w = split_words(line);
        if (w.size() < 2 || !read_real(w[0], m.emin) || !read_real(w[1], m.emax))
            return fail("scaling.data: bad emin emax");
    }

    // nn_new + readWeights
    for (int z : zs) {
        auto& layers = m.nets[z];
        layers.clear();
        int nin = (int)m.sfs[z].size();
        for (int l = 0; l <= nlayers; ++l) {
            Layer L;
            L.nin = nin;
            L.nout = nnodes[l];
            L.act = act[l];
            L.w.assign((size_t)L.nin * L.nout, 0.0);
            L.b.assign(L.nout, 0.0);
            layers.push_back(L);
            nin = L.nout;
        }
        char fn[64];
        std::snprintf(fn, sizeof fn, "weights.%03d.data", z);
        std::ifstream wf(path + fn);
        if (!wf) return fail(path + fn + " not found");
        auto next = [&](double& v) -> bool {
            while (std::getline(wf, line)) {
                auto w = split_words(line);
                if (w.empty()) continue;
                return read_real(w[0], v);
            }
            return false;
        };
        for (auto& L : layers) {
            for (int i = 0; i < L.nin; ++i)
                for (int o = 0; o < L.nout; ++o)
                    if (!next(L.w[o + (size_t)L.nout * i])) return fail(std::string("short weights file ") + fn);
            for (int o = 0; o < L.nout; ++o)
                if (!next(L.b[o])) return fail(std::string("short weights file ") + fn);
        }
    }
    return true;
}

// ---------------------------------------------------------------- 3x3 algebra
// Matrices are Fortran column-major 3x3: M(r,c) = a[r + 3*c]; lattice vector
// c is the column a[3c..3c+2] (atomicStructure.f90:20).
static inline double M(const double* a, int r, int c) { return a[r + 3 * c]; }

// det3D (linalg.f90:227)
static double det3(const double* a) {
    return M(a, 0, 0) * M(a, 1, 1) * M(a, 2, 2) + M(a, 0, 1) * M(a, 1, 2) * M(a, 2, 0) +
           M(a, 0, 2) * M(a, 1, 0) * M(a, 2, 1) - M(a, 0, 0) * M(a, 1, 2) * M(a, 2, 1) -
           M(a, 0, 1) * M(a, 1, 0) * M(a, 2, 2) - M(a, 0, 2) * M(a, 1, 1) * M(a, 2, 0);
}

// inv3DM (linalg.f90:264): adjugate divided by the determinant.
static void inv3(const double* a, double* b) {
    double r0[3] = {M(a, 0, 0), M(a, 0, 1), M(a, 0, 2)};
    double r1[3] = {M(a, 1, 0), M(a, 1, 1), M(a, 1, 2)};
    double r2[3] = {M(a, 2, 0), M(a, 2, 1), M(a, 2, 2)};
    double d = det3(a);
    double c0[3] = {r1[1] * r2[2] - r1[2] * r2[1], r0[2] * r2[1] - r0[1] * r2[2], r0[1] * r1[2] - r0[2] * r1[1]};
    double c1[3] = {r1[2] * r2[0] - r1[0] * r2[2], r0[0] * r2[2] - r0[2] * r2[0], r0[2] * r1[0] - r0[0] * r1[2]};
    double c2[3] = {r1[0] * r2[1] - r1[1] * r2[0], r0[1] * r2[0] - r0[0] * r2[1], r0[0] * r1[1] - r0[1] * r1[0]};
    for (int k = 0; k < 3; ++k) {
        b[0 + 3 * k] = c0[k] / d;
        b[1 + 3 * k] = c1[k] / d;
        b[2 + 3 * k] = c2[k] / d;
    }
}

// matMulVec3 (linalg.f90:194)
static inline void mv3(const double* a, const double* v, double* r) {
    for (int i = 0; i < 3; ++i) r[i] = M(a, i, 0) * v[0] + M(a, i, 1) * v[1] + M(a, i, 2) * v[2];
}

static inline void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// getNcells (pointsets.f90:220-243): image cells per lattice direction
// needed to reach every point within `cut`.
static void n_cells(const double* lat, double cut, int* n) {
    double axb[3], axc[3], bxc[3];
    cross3(lat + 0, lat + 3, axb);
    cross3(lat + 0, lat + 6, axc);
    cross3(lat + 3, lat + 6, bxc);
    auto nrm = [](double* v) {
        double s = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] /= s; v[1] /= s; v[2] /= s;
    };
    nrm(axb); nrm(axc); nrm(bxc);
    double p[3];
    p[0] = lat[0] * bxc[0] + lat[1] * bxc[1] + lat[2] * bxc[2];
    p[1] = lat[3] * axc[0] + lat[4] * axc[1] + lat[5] * axc[2];
    p[2] = lat[6] * axb[0] + lat[7] * axb[1] + lat[8] * axb[2];
    for (int i = 0; i < 3; ++i) n[i] = (int)std::ceil(cut / std::fabs(p[i]));
}

// moveAtomsIntoCell (pointsets.f90:201-217): fractional coordinates modulo 1.
static void wrap_into_cell(int nat, const double* lat, double* pos) {
    double inv[9];
    inv3(lat, inv);
    for (int i = 0; i < nat; ++i) {
        double s[3];
        mv3(inv, pos + 3 * i, s);
        for (int d = 0; d < 3; ++d) s[d] = s[d] - std::floor(s[d]);
        mv3(lat, s, pos + 3 * i);
    }
}

// ---------------------------------------------------------------- neighbours
struct NeiList {  // type neighborList (neighborLists.f90:10-16); entry 0 = the atom itself
    std::vector<double> pos;  // 3 per entry
    std::vector<int> idx;
    int n() const { return (int)idx.size(); }
};

// buildNeighborListGrid (neighborLists.f90:104-230), same enumeration order.
// `pos` are the positions handed to the builder (already wrapped for periodic
// input by hdnnpCalcNeighborLists, hdnnps.f90:379-386).
static void neighbours_grid(int nat, const double* pos, bool periodic, const double* lat_in, double rc,
                            std::vector<NeiList>& out) {
    out.assign(nat, NeiList());
    for (int i = 0; i < nat; ++i) {
        out[i].pos.assign(pos + 3 * i, pos + 3 * i + 3);
        out[i].idx.push_back(i);
    }
    std::vector<double> t(pos, pos + 3 * (size_t)nat);
    double lat[9], org[3] = {0, 0, 0};
    if (periodic) {
        std::memcpy(lat, lat_in, sizeof lat);
    } else {  // artificial box around the molecule (:131-138)
        for (int k = 0; k < 9; ++k) lat[k] = 0;
        for (int d = 0; d < 3; ++d) {
            double mn = t[d];
            for (int i = 1; i < nat; ++i) mn = std::min(mn, t[3 * i + d]);
            org[d] = mn - 1.e-4;
            double mx = -1e300;
            for (int i = 0; i < nat; ++i) {
                t[3 * i + d] -= org[d];
                mx = std::max(mx, t[3 * i + d]);
            }
            lat[d + 3 * d] = mx + 1.e-4;
        }
    }
    int ng[3];
    double grid[9];
    const double target = rc * 0.6;
    for (int d = 0; d < 3; ++d) {
        double len = std::sqrt(lat[3 * d] * lat[3 * d] + lat[3 * d + 1] * lat[3 * d + 1] + lat[3 * d + 2] * lat[3 * d + 2]);
        ng[d] = (int)(len / target) + 1;
        for (int r = 0; r < 3; ++r) grid[r + 3 * d] = lat[r + 3 * d] / ng[d];
    }
    wrap_into_cell(nat, lat, t.data());
    std::vector<double> rel(t);
    {
        double inv[9];
        inv3(lat, inv);
        for (int i = 0; i < nat; ++i) mv3(inv, t.data() + 3 * i, rel.data() + 3 * i);
    }
    auto cell_of = [&](int i, int d) {
        int c = (int)(rel[3 * i + d] * ng[d]);
        return std::min(std::max(c, 0), ng[d] - 1);  // guard for s == 1.0 after rounding
    };
    std::vector<std::vector<int>> cells((size_t)ng[0] * ng[1] * ng[2]);
    auto cid = [&](int x, int y, int z) { return ((size_t)x * ng[1] + y) * ng[2] + z; };
    for (int i = 0; i < nat; ++i) cells[cid(cell_of(i, 0), cell_of(i, 1), cell_of(i, 2))].push_back(i);
    int nc[3];
    n_cells(grid, rc, nc);
    const double rc2 = rc * rc;

#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nat; ++i) {
        int ix = cell_of(i, 0), iy = cell_of(i, 1), iz = cell_of(i, 2);
        for (int jx = -nc[0]; jx <= nc[0]; ++jx) {
            for (int jy = -nc[1]; jy <= nc[1]; ++jy) {
                for (int jz = -nc[2]; jz <= nc[2]; ++jz) {
                    double dl[3] = {0, 0, 0};
                    int cx = ix + jx, cy = iy + jy, cz = iz + jz;
                    if (cz < 0 || cz >= ng[2]) {
                        if (!periodic) continue;
                        int dd = (int)std::floor((double)cz / ng[2]);
                        cz -= ng[2] * dd;
                        for (int r = 0; r < 3; ++r) dl[r] += lat_in[r + 6] * dd;
                    }
                    if (cy < 0 || cy >= ng[1]) {
                        if (!periodic) continue;
                        int dd = (int)std::floor((double)cy / ng[1]);
                        cy -= ng[1] * dd;
                        for (int r = 0; r < 3; ++r) dl[r] += lat_in[r + 3] * dd;
                    }
                    if (cx < 0 || cx >= ng[0]) {
                        if (!periodic) continue;
                        int dd = (int)std::floor((double)cx / ng[0]);
                        cx -= ng[0] * dd;
                        for (int r = 0; r < 3; ++r) dl[r] += lat_in[r + 0] * dd;
                    }
                    const bool home = (jx == 0 && jy == 0 && jz == 0);
                    for (int j : cells[cid(cx, cy, cz)]) {
                        if (j == i && home) continue;
                        double p[3], d[3];
                        for (int r = 0; r < 3; ++r) {
                            p[r] = t[3 * j + r] + dl[r];
                            d[r] = t[3 * i + r] - p[r];
                        }
                        if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < rc2) {
                            for (int r = 0; r < 3; ++r) out[i].pos.push_back(p[r] + org[r]);
                            out[i].idx.push_back(j);
                        }
                    }
                }
            }
        }
    }
}

// buildNeighborList (neighborLists.f90:21-81): O(N^2) cross-check.
static void neighbours_brute(int nat, const double* pos, bool periodic, const double* lat, double rc,
                             std::vector<NeiList>& out) {
    out.assign(nat, NeiList());
    for (int i = 0; i < nat; ++i) {
        out[i].pos.assign(pos + 3 * i, pos + 3 * i + 3);
        out[i].idx.push_back(i);
    }
    int nc[3] = {0, 0, 0};
    if (periodic) n_cells(lat, rc, nc);
    for (int i = 0; i < nat; ++i)
        for (int ix = 0; ix <= nc[0]; ++ix)
            for (int iy = (ix == 0 ? 0 : -nc[1]); iy <= nc[1]; ++iy)
                for (int iz = ((ix == 0 && iy == 0) ? 0 : -nc[2]); iz <= nc[2]; ++iz) {
                    double dl[3];
                    for (int r = 0; r < 3; ++r) dl[r] = ix * lat[r] + iy * lat[r + 3] + iz * lat[r + 6];
                    int j0 = (ix == 0 && iy == 0 && iz == 0) ? i + 1 : 0;
                    for (int j = j0; j < nat; ++j) {
                        double d[3];
                        for (int r = 0; r < 3; ++r) d[r] = pos[3 * i + r] - (pos[3 * j + r] + dl[r]);
                        if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < rc * rc) {
                            for (int r = 0; r < 3; ++r) out[i].pos.push_back(pos[3 * j + r] + dl[r]);
                            out[i].idx.push_back(j);
                            for (int r = 0; r < 3; ++r) out[j].pos.push_back(pos[3 * i + r] - dl[r]);
                            out[j].idx.push_back(i);
                        }
                    }
                }
}

// ---------------------------------------------------------------- symmetry functions
// cutoff (symmetryFunctions.f90:310-327): tanh^3 cutoff; dfc is (dfc/dr)/r.
static inline void cutoff(double r, double rc, double& fc, double& dfc) {
    if (r < rc) {
        double t = std::tanh(1.0 - r / rc);
        double tt = t * t;
        fc = tt * t;
        dfc = -3.0 / (rc * r) * (tt - tt * tt);
    } else {
        fc = 0;
        dfc = 0;
    }
}

// x**n for integer n by binary exponentiation (what a Fortran real**integer
// power evaluates to); negative n gives 1/x**|n|.
static inline double powi(double x, int n) {
    bool neg = n < 0;
    unsigned k = neg ? (unsigned)(-n) : (unsigned)n;
    double r = 1.0, b = x;
    while (k) {
        if (k & 1u) r *= b;
        b *= b;
        k >>= 1u;
    }
    return neg ? 1.0 / r : r;
}

// calcAllSymmetryFunctions (symmetryFunctions.f90:158-308).  Neighbour entry 0
// is the centre.  G[nsf]; dG[nsf][nNei][3] (may be null).
static bool sf_fused(int nn, const double* npos, const int* nel, const std::vector<SymFn>& L, double* G,
                     double* dG) {
    const int ns = (int)L.size();
    if (ns == 0) return true;
    int s3 = -1;
    const double rc = L[0].rcut;
    for (int s = 0; s < ns; ++s) {
        if (L[s].type == 3 && s3 < 0)
            s3 = s;
        else if (L[s].type == 2 && s3 >= 0)
            return fail("SFs are not sorted");
        if ((L[s].rcut - rc) * (L[s].rcut - rc) > 1.e-10) return fail("expecting same rc for all symfunctions");
    }
    if (s3 < 0) s3 = ns;
    for (int s = 0; s < ns; ++s) G[s] = 0;
    if (dG) std::fill(dG, dG + (size_t)ns * nn * 3, 0.0);
    auto D = [&](int s, int n) { return dG + ((size_t)s * nn + n) * 3; };

    std::vector<double> dij(3 * (size_t)nn), rij(nn), fcs(nn), dfcs(nn);
    for (int j = 1; j < nn; ++j) {
        for (int r = 0; r < 3; ++r) dij[3 * j + r] = npos[r] - npos[3 * j + r];
        rij[j] = std::sqrt(dij[3 * j] * dij[3 * j] + dij[3 * j + 1] * dij[3 * j + 1] + dij[3 * j + 2] * dij[3 * j + 2]);
        cutoff(rij[j], rc, fcs[j], dfcs[j]);
    }
    for (int j = 1; j < nn; ++j) {
        const double* a = &dij[3 * j];
        const double ra = rij[j], fa = fcs[j], dfa = dfcs[j];
        for (int s = 0; s < s3; ++s) {  // radial (G2)
            const SymFn& f = L[s];
            if (f.el1 != nel[j]) continue;
            double e = std::exp(-f.eta * (ra - f.rs) * (ra - f.rs));
            if (dG) {
                for (int r = 0; r < 3; ++r) {
                    double g = -1.0 * e * dfa * a[r] + 2.0 * f.eta * (ra - f.rs) * a[r] / ra * e * fa;
                    D(s, j)[r] = g;
                    D(s, 0)[r] -= g;
                }
            }
            G[s] += e * fa;
        }
        for (int k = j + 1; k < nn; ++k) {  // angular (G4), unordered pairs j<k
            const double* b = &dij[3 * k];
            const double rb = rij[k], fb = fcs[k], dfb = dfcs[k];
            double djk[3];
            for (int r = 0; r < 3; ++r) djk[r] = npos[3 * j + r] - npos[3 * k + r];
            double rjk = std::sqrt(djk[0] * djk[0] + djk[1] * djk[1] + djk[2] * djk[2]);
            double fjk, dfjk;
            cutoff(rjk, rc, fjk, dfjk);
            double t1 = -1.0 / (ra * rb);
            double cth = 0.5 * (rjk * rjk - ra * ra - rb * rb) * t1;
            double ab = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
            double dcj[3], dck[3], dfpj[3], dfpk[3];
            for (int r = 0; r < 3; ++r) {
                dcj[r] = t1 * b[r] + a[r] * ab / (ra * ra * ra * rb);
                dck[r] = t1 * a[r] + b[r] * ab / (rb * rb * rb * ra);
                dfpj[r] = fb * (dfjk * djk[r] * fa - dfa * a[r] * fjk);
                dfpk[r] = -1.0 * fa * (dfjk * djk[r] * fb + dfb * b[r] * fjk);
            }
            const double fcp = fa * fb * fjk;
            double last_eta = 0.0, ep = 1.0, depj[3] = {0, 0, 0}, depk[3] = {0, 0, 0};
            for (int s = s3; s < ns; ++s) {
                const SymFn& f = L[s];
                if (!((nel[j] == f.el1 && nel[k] == f.el2) || (nel[j] == f.el2 && nel[k] == f.el1))) continue;
                int iz = (int)f.zeta;
                double base = 1.0 + f.lambda * cth;
                double pf, t2;
                if (std::fabs(f.zeta - iz) < 1.e-10) {
                    pf = powi(2.0, 1 - iz);
                    t2 = powi(base, iz - 1);
                } else {
                    pf = std::pow(2.0, 1.0 - f.zeta);
                    t2 = std::pow(base, f.zeta - 1.0);
                }
                double cp = t2 * base;
                if (std::fabs(f.eta - last_eta) > 1.e-10) {
                    ep = std::exp(-f.eta * (ra * ra + rb * rb + rjk * rjk));
                    for (int r = 0; r < 3; ++r) {
                        depj[r] = ep * f.eta * 2.0 * (a[r] - djk[r]);
                        depk[r] = ep * f.eta * 2.0 * (b[r] + djk[r]);
                    }
                    last_eta = f.eta;
                }
                if (dG) {
                    for (int r = 0; r < 3; ++r) {
                        double gj = pf * (cp * ep * dfpj[r] + cp * depj[r] * fcp +
                                          t2 * f.lambda * f.zeta * dcj[r] * ep * fcp);
                        double gk = pf * (cp * ep * dfpk[r] + cp * depk[r] * fcp +
                                          t2 * f.lambda * f.zeta * dck[r] * ep * fcp);
                        D(s, j)[r] += gj;
                        D(s, k)[r] += gk;
                        D(s, 0)[r] -= (gj + gk);
                    }
                }
                G[s] += pf * cp * ep * fcp;
            }
        }
    }
    return true;
}

// symmetryFunction2 (symmetryFunctions.f90:41-74): one radial SF.
static void sf2_single(int nn, const double* npos, const int* nel, const SymFn& f, double& G, double* dG) {
    G = 0;
    std::fill(dG, dG + 3 * (size_t)nn, 0.0);
    for (int i = 1; i < nn; ++i) {
        if (nel[i] != f.el1) continue;
        double r[3];
        for (int q = 0; q < 3; ++q) r[q] = npos[q] - npos[3 * i + q];
        double d = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        double fc, dfc;
        cutoff(d, f.rcut, fc, dfc);
        double e = std::exp(-f.eta * (d - f.rs) * (d - f.rs));
        for (int q = 0; q < 3; ++q) {
            double g = -1.0 * e * dfc * r[q] + 2 * f.eta * (d - f.rs) * r[q] / d * e * fc;
            dG[3 * i + q] = g;
            dG[q] -= g;
        }
        G += e * fc;
    }
}

// symmetryFunction3 (symmetryFunctions.f90:77-152): one angular SF with a
// real-valued power.
static void sf3_single(int nn, const double* npos, const int* nel, const SymFn& f, double& G, double* dG) {
    G = 0;
    std::fill(dG, dG + 3 * (size_t)nn, 0.0);
    for (int j = 1; j < nn; ++j) {
        if (nel[j] != f.el1 && nel[j] != f.el2) continue;
        double a[3];
        for (int q = 0; q < 3; ++q) a[q] = npos[q] - npos[3 * j + q];
        double ra = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        double fa, dfa;
        cutoff(ra, f.rcut, fa, dfa);
        for (int k = j + 1; k < nn; ++k) {
            if (!((nel[j] == f.el1 && nel[k] == f.el2) || (nel[j] == f.el2 && nel[k] == f.el1))) continue;
            double b[3], c[3];
            for (int q = 0; q < 3; ++q) {
                b[q] = npos[q] - npos[3 * k + q];
                c[q] = npos[3 * j + q] - npos[3 * k + q];
            }
            double rb = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
            double rcc = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
            double fb, dfb, fjk, dfjk;
            cutoff(rb, f.rcut, fb, dfb);
            cutoff(rcc, f.rcut, fjk, dfjk);
            double cth = (rcc * rcc - ra * ra - rb * rb) / (-2.0 * ra * rb);
            double ab = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
            double fcp = fa * fb * fjk;
            double pf = std::pow(2.0, 1.0 - f.zeta);
            double cp = std::pow(1.0 + f.lambda * cth, f.zeta);
            double dcpf = f.zeta * std::pow(1.0 + f.lambda * cth, f.zeta - 1.0) * f.lambda;
            double ep = std::exp(-f.eta * (ra * ra + rb * rb + rcc * rcc));
            for (int q = 0; q < 3; ++q) {
                double dcj = -1.0 * b[q] / (ra * rb) + a[q] * ab / (ra * ra * ra * rb);
                double dck = -1.0 * a[q] / (ra * rb) + b[q] * ab / (rb * rb * rb * ra);
                double dfpj = fb * (dfjk * c[q] * fa - dfa * a[q] * fjk);
                double dfpk = -1.0 * fa * (dfjk * c[q] * fb + dfb * b[q] * fjk);
                double depj = ep * f.eta * 2.0 * (a[q] - c[q]);
                double depk = ep * f.eta * 2.0 * (b[q] + c[q]);
                double gj = pf * (cp * ep * dfpj + cp * depj * fcp + dcpf * dcj * ep * fcp);
                double gk = pf * (cp * ep * dfpk + cp * depk * fcp + dcpf * dck * ep * fcp);
                dG[3 * j + q] += gj;
                dG[3 * k + q] += gk;
                dG[q] -= (gj + gk);
            }
            G += pf * cp * ep * fcp;
        }
    }
}

// ---------------------------------------------------------------- network
// activate / deactivate (neuralNetworks.f90:33-84)
static inline double act_f(char a, double x) {
    switch (a) {
        case 't': return std::tanh(x);
        case 'p': return std::log(1.0 + std::exp(x));
        case 'r': return x > 0 ? x : 0.0;
        default: return x;
    }
}
static inline double act_d(char a, double x) {
    switch (a) {
        case 't': { double t = std::tanh(x); return 1.0 - t * t; }
        case 'p': return 1.0 / (1.0 + std::exp(-1.0 * x));
        case 'r': return x > 0 ? 1.0 : 0.0;
        default: return 1.0;
    }
}

// nn_forward + nn_backward(gradOut = 1) for one atom (neuralNetworks.f90:94-158,
// 220-313): returns the output and dOut/dInput.
static double nn_eval(const std::vector<Layer>& net, const double* x, double* dx) {
    std::vector<std::vector<double>> c(net.size());
    std::vector<double> in(x, x + net[0].nin);
    for (size_t l = 0; l < net.size(); ++l) {
        const Layer& L = net[l];
        c[l].assign(L.nout, 0.0);
        std::vector<double> out(L.nout);
        for (int o = 0; o < L.nout; ++o) {
            double s = 0;
            for (int i = 0; i < L.nin; ++i) s += L.w[o + (size_t)L.nout * i] * in[i];
            c[l][o] = s + L.b[o];
            out[o] = act_f(L.act, c[l][o]);
        }
        in.swap(out);
    }
    const double y = in[0];
    if (dx) {
        std::vector<double> g(1, 1.0);
        for (int l = (int)net.size() - 1; l >= 0; --l) {
            const Layer& L = net[l];
            std::vector<double> t(L.nout), gi(L.nin, 0.0);
            for (int o = 0; o < L.nout; ++o) t[o] = g[o] * act_d(L.act, c[l][o]);
            for (int i = 0; i < L.nin; ++i)
                for (int o = 0; o < L.nout; ++o) gi[i] += t[o] * L.w[o + (size_t)L.nout * i];
            g.swap(gi);
        }
        std::copy(g.begin(), g.end(), dx);
    }
    return y;
}

// ---------------------------------------------------------------- evaluation
struct Eval {
    int nat;
    std::vector<NeiList> nl;
    std::vector<int> Z;
};

// hdnnpCalcNeighborLists (hdnnps.f90:373-388)
static void calc_neighbours(const Model& m, int nat, const int* Z, const double* pos, bool periodic,
                            const double* lat, bool brute, std::vector<NeiList>& nl) {
    std::vector<double> p(pos, pos + 3 * (size_t)nat);
    if (periodic) wrap_into_cell(nat, lat, p.data());
    if (brute)
        neighbours_brute(nat, p.data(), periodic, lat, m.maxRc, nl);
    else
        neighbours_grid(nat, p.data(), periodic, lat, m.maxRc, nl);
    (void)Z;
}

// scaling part of hdnnpCalcSymfunctions (hdnnps.f90:471-481)
static void scale_sf(const Model& m, const std::vector<SymFn>& L, double* G, double* dG, int nn) {
    for (size_t s = 0; s < L.size(); ++s) {
        if (m.centersf) G[s] = G[s] - L[s].smean;
        if (m.scalesf) {
            double w = L[s].smax - L[s].smin;
            G[s] = G[s] / w;
            if (dG)
                for (int q = 0; q < 3 * nn; ++q) dG[(size_t)s * nn * 3 + q] /= w;
        }
    }
}

// symmetry functions of one atom (fused or single-SF routines), scaled.
static bool atom_sfs(const Model& m, const NeiList& nl, const int* Z, int zc, bool separate, double* G,
                     double* dG) {
    const auto& L = m.sfs[zc];
    const int nn = nl.n();
    std::vector<int> nel(nn);
    for (int q = 0; q < nn; ++q) nel[q] = Z[nl.idx[q]];
    if (!separate) {
        if (!sf_fused(nn, nl.pos.data(), nel.data(), L, G, dG)) return false;
    } else {
        std::vector<double> tmp(3 * (size_t)nn);
        for (size_t s = 0; s < L.size(); ++s) {
            if (L[s].type == 2)
                sf2_single(nn, nl.pos.data(), nel.data(), L[s], G[s], tmp.data());
            else
                sf3_single(nn, nl.pos.data(), nel.data(), L[s], G[s], tmp.data());
            if (dG) std::copy(tmp.begin(), tmp.end(), dG + s * 3 * (size_t)nn);
        }
    }
    scale_sf(m, L, G, dG, nn);
    return true;
}

// hdnnpEnergyAndForces (hdnnps.f90:333-371) = neighbour lists + symmetry
// functions + hdnnpCalcNNs (:487-562).  dsf is produced per atom and
// contracted immediately (the reference stores all of it first; the
// arithmetic per atom is the same).
static bool eval(const Model& m, int nat, const int* Z, const double* pos, bool periodic, const double* lat,
                 double* E, double* F, double* dEdLat, double* atE, double* dEdG, int dEdG_stride, bool brute,
                 bool separate) {
    for (int i = 0; i < nat; ++i)
        if (Z[i] < 1 || Z[i] > 118 || m.nets[Z[i]].empty()) return fail("atom with element not in the potential");
    std::vector<NeiList> nl;
    calc_neighbours(m, nat, Z, pos, periodic, lat, brute, nl);
    double inv[9] = {0};
    if (dEdLat) {
        if (!periodic) return fail("dEdLat requested for a non-periodic structure");
        inv3(lat, inv);
    }
    std::vector<double> ae(nat, 0.0);
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    std::vector<std::vector<double>> fpart(nthr, std::vector<double>(3 * (size_t)nat, 0.0));
    std::vector<std::array<double, 9>> lpart(nthr);
    for (auto& a : lpart) a.fill(0.0);
    volatile bool ok = true;
    std::string errmsg;

#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < nat; ++i) {
        if (!ok) continue;
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        const int z = Z[i];
        const auto& L = m.sfs[z];
        const int ns = (int)L.size(), nn = nl[i].n();
        std::vector<double> G(ns), dG((size_t)ns * nn * 3), dE(ns);
        if (!atom_sfs(m, nl[i], Z, z, separate, G.data(), dG.data())) {
#pragma omp critical
            { ok = false; errmsg = g_err; }
            continue;
        }
        ae[i] = nn_eval(m.nets[z], G.data(), dE.data()) + m.atomenergy[z];
        if (dEdG)
            for (int s = 0; s < ns; ++s) dEdG[(size_t)i * dEdG_stride + s] = dE[s];
        double* f = fpart[tid].data();
        for (int s = 0; s < ns; ++s)
            for (int q = 0; q < nn; ++q) {
                int a = nl[i].idx[q];
                for (int r = 0; r < 3; ++r) f[3 * a + r] = f[3 * a + r] + (-1.0 * dE[s] * dG[((size_t)s * nn + q) * 3 + r]);
            }
        if (dEdLat) {
            auto& lp = lpart[tid];
            for (int s = 0; s < ns; ++s)
                for (int q = 0; q < nn; ++q) {
                    double rel[3];
                    mv3(inv, &nl[i].pos[3 * q], rel);
                    for (int x = 0; x < 3; ++x)
                        for (int r = 0; r < 3; ++r) lp[r + 3 * x] += dE[s] * dG[((size_t)s * nn + q) * 3 + r] * rel[x];
                }
        }
    }
    if (!ok) return fail(errmsg);
    double e = 0;
    for (int i = 0; i < nat; ++i) e += ae[i];
    *E = e;
    if (atE) std::copy(ae.begin(), ae.end(), atE);
    if (F) {
        std::fill(F, F + 3 * (size_t)nat, 0.0);
        for (int t = 0; t < nthr; ++t)
            for (size_t q = 0; q < 3 * (size_t)nat; ++q) F[q] += fpart[t][q];
    }
    if (dEdLat) {
        for (int k = 0; k < 9; ++k) dEdLat[k] = 0;
        for (int t = 0; t < nthr; ++t)
            for (int k = 0; k < 9; ++k) dEdLat[k] += lpart[t][k];
    }
    return true;
}

}  // namespace orc

// ================================================================ C API (ctypes)
using namespace orc;

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// parseRuNNerInput.  path must end with '/'.  cap_sfs=200 reproduces nmaxSFs.
void* orc_model_load(const char* path, int cap_sfs) {
    Model* m = new Model();
    if (!load_runner(path, cap_sfs, *m)) {
        delete m;
        return nullptr;
    }
    return m;
}

void orc_model_free(void* h) { delete (Model*)h; }

// Elements (sorted by Z), their SF counts, maxRc.
int orc_model_info(void* h, int* nel, int* zs, int* nsf, double* maxrc) {
    Model* m = (Model*)h;
    *nel = (int)m->elements.size();
    for (size_t i = 0; i < m->elements.size(); ++i) {
        zs[i] = m->elements[i];
        nsf[i] = (int)m->sfs[m->elements[i]].size();
    }
    *maxrc = m->maxRc;
    return 0;
}

// SF parameters of element z in the sorted order: per SF 11 doubles
// (type, el1, el2, rcut, eta, lambda, zeta, rs, smin, smax, smean).
int orc_model_sfs(void* h, int z, double* out) {
    Model* m = (Model*)h;
    const auto& L = m->sfs[z];
    for (size_t s = 0; s < L.size(); ++s) {
        double* o = out + 11 * s;
        o[0] = L[s].type; o[1] = L[s].el1; o[2] = L[s].el2; o[3] = L[s].rcut; o[4] = L[s].eta;
        o[5] = L[s].lambda; o[6] = L[s].zeta; o[7] = L[s].rs; o[8] = L[s].smin; o[9] = L[s].smax; o[10] = L[s].smean;
    }
    return (int)L.size();
}

// Network of element z: layer count, then per layer (nin, nout, act) and the
// weights (column-major nout x nin) + biases when w is non-null.
int orc_model_net(void* h, int z, int* nl, int* dims, char* acts, double* w) {
    Model* m = (Model*)h;
    const auto& net = m->nets[z];
    *nl = (int)net.size();
    size_t off = 0;
    for (size_t l = 0; l < net.size(); ++l) {
        dims[2 * l] = net[l].nin;
        dims[2 * l + 1] = net[l].nout;
        acts[l] = net[l].act;
        if (w) {
            std::copy(net[l].w.begin(), net[l].w.end(), w + off);
            off += net[l].w.size();
            std::copy(net[l].b.begin(), net[l].b.end(), w + off);
            off += net[l].b.size();
        }
    }
    return 0;
}

int orc_model_flags(void* h, int* scalesf, int* centersf, double* atomenergy119) {
    Model* m = (Model*)h;
    *scalesf = m->scalesf;
    *centersf = m->centersf;
    for (int z = 0; z < 119; ++z) atomenergy119[z] = m->atomenergy[z];
    return 0;
}

// Neighbour lists.  counts[nat] (incl. the self entry); idx/pos hold up to
// cap entries per atom at stride cap.  Returns the max count (>cap means the
// arrays were truncated).  mode 0 = cell list, 1 = O(N^2).
int orc_neighbours(void* h, int nat, const int* Z, const double* pos, int periodic, const double* lat, int mode,
                   int cap, int* counts, int* idx, double* npos) {
    Model* m = (Model*)h;
    std::vector<NeiList> nl;
    calc_neighbours(*m, nat, Z, pos, periodic != 0, lat, mode == 1, nl);
    int mx = 0;
    for (int i = 0; i < nat; ++i) {
        int n = nl[i].n();
        mx = std::max(mx, n);
        counts[i] = n;
        for (int q = 0; q < std::min(n, cap); ++q) {
            idx[(size_t)i * cap + q] = nl[i].idx[q];
            for (int r = 0; r < 3; ++r) npos[((size_t)i * cap + q) * 3 + r] = nl[i].pos[3 * q + r];
        }
    }
    return mx;
}

// Scaled symmetry functions G[nat][stride] (and optionally the centre-first
// derivatives dG[nat][stride][cap][3] for atoms with <= cap entries).
// separate=1 uses the single-SF routines.
int orc_symfunctions(void* h, int nat, const int* Z, const double* pos, int periodic, const double* lat,
                     int separate, int stride, double* G, int cap, double* dG) {
    Model* m = (Model*)h;
    std::vector<NeiList> nl;
    calc_neighbours(*m, nat, Z, pos, periodic != 0, lat, false, nl);
    for (int i = 0; i < nat; ++i) {
        const int z = Z[i];
        const int ns = (int)m->sfs[z].size(), nn = nl[i].n();
        std::vector<double> g(ns), d((size_t)ns * nn * 3);
        if (!atom_sfs(*m, nl[i], Z, z, separate != 0, g.data(), d.data())) return -1;
        for (int s = 0; s < ns; ++s) G[(size_t)i * stride + s] = g[s];
        if (dG && nn <= cap)
            for (int s = 0; s < ns; ++s)
                for (int q = 0; q < nn; ++q)
                    for (int r = 0; r < 3; ++r)
                        dG[(((size_t)i * stride + s) * cap + q) * 3 + r] = d[((size_t)s * nn + q) * 3 + r];
    }
    return 0;
}

// hdnnpEnergyAndForces.  pos[3*nat] (xyz per atom, Bohr), lat[9] column-major
// (columns = lattice vectors).  F, dEdLat, atE, dEdG may be null.
int orc_eval(void* h, int nat, const int* Z, const double* pos, int periodic, const double* lat, double* E,
             double* F, double* dEdLat, double* atE, double* dEdG, int dEdG_stride, int brute, int separate) {
    Model* m = (Model*)h;
    return eval(*m, nat, Z, pos, periodic != 0, lat, E, F, dEdLat, atE, dEdG, dEdG_stride, brute != 0,
                separate != 0)
               ? 0
               : -1;
}

// dEdLat2Stress (atomicStructure.f90:679-686): stress = -1/det(h) dEdLat h^T.
void orc_dEdLat_to_stress(const double* lat, const double* dEdLat, double* stress) {
    double d = det3(lat);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += dEdLat[i + 3 * k] * lat[j + 3 * k];
            stress[i + 3 * j] = -1.0 / d * s;
        }
}

}  // extern "C"

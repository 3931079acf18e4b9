// model.h -- host-side potential (parsed RuNNer files) and its device layout.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace hdnnp {

constexpr int kMaxZ = 118;
constexpr int kMaxElements = 16;   // elements in one potential
constexpr int kMaxLayers = 8;      // network layers (hidden + output)
constexpr int kMaxWidth = 128;     // neurons per hidden layer

struct SymFn {
    int type = 0;          // 2 = radial (G2), 3 = angular (G4)
    int z1 = 0, z2 = 0;    // neighbour element(s), atomic numbers
    double rcut = 0, eta = 0, lambda = 0, zeta = 0, rs = 0;
    double smin = 0, smax = 0, smean = 0;
};

struct Layer {
    int nin = 0, nout = 0;
    char act = 'l';
    std::vector<double> w;  // row-major [nout][nin]
    std::vector<double> b;
};

struct ElementModel {
    int z = 0;
    std::vector<SymFn> sfs;   // in the reference's sorted order
    std::vector<Layer> net;
    double atom_energy = 0;
};

struct HostModel {
    std::vector<ElementModel> el;  // sorted by Z
    int z2e[kMaxZ + 1];           // atomic number -> element index, -1 if absent
    double max_rc = 0, emin = 0, emax = 0;
    bool scalesf = false, centersf = false;
    HostModel() {
        for (int i = 0; i <= kMaxZ; ++i) z2e[i] = -1;
    }
};

// Parses input.nn, scaling.data and weights.NNN.data from `dir`.
// Returns false and sets `err` on failure.
bool load_runner(const std::string& dir, HostModel& m, std::string& err);

// atomic number of an element symbol, -1 if unknown
int symbol_to_z(const std::string& s);

}  // namespace hdnnp

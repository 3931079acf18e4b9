// capi.cu -- C ABI of the engine (include/hdnnp_gpu.h): model upload,
// evaluation contexts, host-side structure set-up and the stage pipeline.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hdnnp_gpu.h"
#include "engine.h"
#include "fastmath.cuh"
#include "model.h"

using namespace hdnnp;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CUDA_TRY(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(HDNNP_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

// ------------------------------------------------------------------ 3x3 helpers
// column-major 3x3: a[r + 3c]
double det3(const double* a) {
    return a[0] * a[4] * a[8] + a[3] * a[7] * a[2] + a[6] * a[1] * a[5] - a[0] * a[7] * a[5] - a[3] * a[1] * a[8] -
           a[6] * a[4] * a[2];
}

// inverse by adjugate / determinant (inv3DM, linalg.f90:264)
void inv3(const double* a, double* b) {
    auto A = [&](int r, int c) { return a[r + 3 * c]; };
    double d = det3(a);
    double r0[3] = {A(0, 0), A(0, 1), A(0, 2)}, r1[3] = {A(1, 0), A(1, 1), A(1, 2)}, r2[3] = {A(2, 0), A(2, 1), A(2, 2)};
    double c0[3] = {r1[1] * r2[2] - r1[2] * r2[1], r0[2] * r2[1] - r0[1] * r2[2], r0[1] * r1[2] - r0[2] * r1[1]};
    double c1[3] = {r1[2] * r2[0] - r1[0] * r2[2], r0[0] * r2[2] - r0[2] * r2[0], r0[2] * r1[0] - r0[0] * r1[2]};
    double c2[3] = {r1[0] * r2[1] - r1[1] * r2[0], r0[1] * r2[0] - r0[0] * r2[1], r0[0] * r1[1] - r0[1] * r1[0]};
    for (int k = 0; k < 3; ++k) {
        b[0 + 3 * k] = c0[k] / d;
        b[1 + 3 * k] = c1[k] / d;
        b[2 + 3 * k] = c2[k] / d;
    }
}

// getNcells (pointsets.f90:220-243)
void n_cells(const double* lat, double cut, int* n) {
    auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
    };
    double axb[3], axc[3], bxc[3];
    cross(lat, lat + 3, axb);
    cross(lat, lat + 6, axc);
    cross(lat + 3, lat + 6, bxc);
    for (double* v : {axb, axc, bxc}) {
        double s = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; ++k) v[k] /= s;
    }
    double p0 = lat[0] * bxc[0] + lat[1] * bxc[1] + lat[2] * bxc[2];
    double p1 = lat[3] * axc[0] + lat[4] * axc[1] + lat[5] * axc[2];
    double p2 = lat[6] * axb[0] + lat[7] * axb[1] + lat[8] * axb[2];
    n[0] = (int)std::ceil(cut / std::fabs(p0));
    n[1] = (int)std::ceil(cut / std::fabs(p1));
    n[2] = (int)std::ceil(cut / std::fabs(p2));
}

// Grid set-up of buildNeighborListGrid (neighborLists.f90:129-169).
int struct_setup(int nat, const double* pos, int periodic, const double* lat, double rc, StructInfo& S) {
    std::memset(&S, 0, sizeof S);
    S.periodic = periodic ? 1 : 0;
    if (nat <= 0) return fail(HDNNP_E_INPUT, "structure without atoms");
    // host positions are checked here; device-resident ones by the wrap kernel
    if (pos)
        for (int i = 0; i < 3 * nat; ++i)
            if (!std::isfinite(pos[i])) return fail(HDNNP_E_INPUT, "non-finite position");
    if (!pos && !periodic) return fail(HDNNP_E_INPUT, "a molecule needs host positions for its bounding box");
    if (periodic) {
        std::memcpy(S.h, lat, sizeof S.h);
        for (int k = 0; k < 9; ++k)
            if (!std::isfinite(lat[k])) return fail(HDNNP_E_INPUT, "non-finite lattice");
        double d = det3(S.h);
        if (!(std::fabs(d) > 1e-12)) return fail(HDNNP_E_INPUT, "singular lattice");
    } else {
        for (int d = 0; d < 3; ++d) {
            double mn = pos[d], mx = pos[d];
            for (int i = 1; i < nat; ++i) {
                mn = std::min(mn, pos[3 * i + d]);
                mx = std::max(mx, pos[3 * i + d]);
            }
            S.org[d] = mn - 1.e-4;
            double ext = 0.0;
            for (int i = 0; i < nat; ++i) ext = std::max(ext, pos[3 * i + d] - S.org[d]);
            S.h[d + 3 * d] = ext + 1.e-4;
        }
    }
    inv3(S.h, S.hinv);
    const double target = rc * 0.6;
    double grid[9];
    long long ncell = 1;
    for (int d = 0; d < 3; ++d) {
        double len = std::sqrt(S.h[3 * d] * S.h[3 * d] + S.h[3 * d + 1] * S.h[3 * d + 1] + S.h[3 * d + 2] * S.h[3 * d + 2]);
        S.ngrid[d] = (int)(len / target) + 1;
        ncell *= S.ngrid[d];
    }
    // Very sparse molecules: coarsen the grid (same neighbour set, other order).
    const long long limit = 64LL * nat + 4096;
    while (ncell > limit) {
        ncell = 1;
        for (int d = 0; d < 3; ++d) {
            S.ngrid[d] = std::max(1, S.ngrid[d] / 2);
            ncell *= S.ngrid[d];
        }
    }
    for (int d = 0; d < 3; ++d)
        for (int r = 0; r < 3; ++r) grid[r + 3 * d] = S.h[r + 3 * d] / S.ngrid[d];
    n_cells(grid, rc, S.nsearch);
    // A molecule's cells beyond its grid are empty: offsets of ngrid or more
    // find nothing (the reference visits and skips them), so the search stops
    // there -- flat or linear molecules (an extent of 2e-4 Bohr) stay cheap.
    if (!periodic)
        for (int d = 0; d < 3; ++d) S.nsearch[d] = std::min(S.nsearch[d], S.ngrid[d] - 1);
    if (periodic) {
        int nl[3];
        n_cells(S.h, rc, nl);
        if (nl[0] > 100 || nl[1] > 100 || nl[2] > 100)
            return fail(HDNNP_E_CAPACITY, "cell too small for the cutoff (more than 100 images per direction)");
    }
    for (int d = 0; d < 3; ++d)
        if (S.nsearch[d] > 64) return fail(HDNNP_E_CAPACITY, "cell too skewed for the cell-list search");
    return HDNNP_OK;
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    int ensure(size_t n) {
        if (n <= cap && p) return HDNNP_OK;
        if (p) cudaFree(p);
        p = nullptr;
        size_t want = std::max<size_t>(n + n / 4, 64);
        if (cudaMalloc(&p, want * sizeof(T)) != cudaSuccess) {
            cap = 0;
            return fail(HDNNP_E_CUDA, "cudaMalloc of the workspace failed");
        }
        cap = want;
        return HDNNP_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace

struct hdnnp_model {
    HostModel host;
    DevModel dev;
    int device = 0;
    void* dmem = nullptr;
};

struct hdnnp_ctx {
    hdnnp_model* model = nullptr;
    cudaStream_t stream = nullptr;
    int precision = HDNNP_PREC_FP64;
    int generic_sf = 0;
    int runtime_zeta = 0;
    int mlp_simt = 0;
    int sf_split = 0;          // launch shape of the fast SF kernels (0: defaults)
    int sf_blocks_per_sm = 0;
    int nei_warp = 0;          // neighbour-list form (0: by batch size)
    int launches = 0;
    // device buffers
    DevBuf<StructInfo> info;
    DevBuf<int> Z, sid, elem, cell_of, cell_cnt, cell_start, cell_atoms, nei_cnt, nei_off, nei_j, nei_s, nei_rev,
        el_count, el_start, el_atoms, scan_tmp, status;
    DevBuf<double> pos, wpos, G, dEdG, atE, gent, gself, vir, force, energy, dEdLat;
    DevBuf<float> Gf, dEdGf, atEf, gentf, gselff, virf;  // mixed-precision intermediates
    DevBuf<double> cm_acc, cm_E, cm_std;                  // committee: dE/dG sum, member energies, std
    DevBuf<unsigned> pairs;                               // contributing-pair lists (fast kernels)
    DevBuf<int> npairs;
    DevBuf<int> cnei_cnt, cnei_off, cnei_j, cnei_s, cnei_rev, cnei_map;  // compacted Verlet-skin lists
    DevBuf<int> pad;                                      // padded neighbour rows (int2 pairs)
    DevBuf<double4> posc;                                 // cell-ordered wrapped positions
    DevBuf<unsigned short> slab;                          // slab prefixes of the padded rows
    int m_est = 0;  // largest neighbour count counted on the host by hdnnp_eval_batch (0: none yet)
    bool last_fast = false, last_mixed = false;  // kernel family and precision of the last lists stage
    int stage_seq = 0;  // stage API: 1 after hdnnp_calc_neighbor_lists, 2 after hdnnp_calc_symfunctions
    int stage_periodic = 0;
    // One molecule of at most kSmallMolecule atoms per call in FP64: the
    // single-block kernel of fused_md.cu in evaluation mode (option
    // "small_eval", default on).  se_dev: the io block (see small_eval_io)
    // and the kernel's global homes; se_host: its mapped pinned mirror.
    int small_eval = 1;
    // the resident form of that kernel (option "small_resident", default on):
    // a single-block kernel that stays on one SM between calls and serves
    // them from a mapped-memory mailbox (no launch per call, warm caches); it
    // exits by itself after a few idle milliseconds
    int small_resident = 1;
    ResidentBox* rs_box = nullptr;     // mailbox, mapped pinned host memory
    ResidentBox* rs_dbox = nullptr;    // its device address
    cudaStream_t rs_stream = nullptr;  // non-blocking stream of the resident kernel
    int rs_natoms = 0;                 // atoms the running kernel serves (0: none launched)
    int rs_seq = 0;                    // number of the last request
    void* se_dev = nullptr;
    unsigned char* se_host = nullptr;
    unsigned char* se_hdev = nullptr;  // device address of the mapped se_host
    Batch se_b{};
    // profiling: events around each stage, accumulated stage times and counters
    bool profile = false;
    bool prof_pending = false;
    cudaEvent_t ev[8] = {};
    double stage_ms[8] = {0};
    long long host_counts[2] = {0, 0};
    DevBuf<unsigned long long> stats;
    // pinned host staging
    int* h_status = nullptr;
    Batch last{};
    bool have_last = false;
    std::vector<StructInfo> hinfo;
    ~hdnnp_ctx() {
        if (rs_natoms && rs_box) {  // stop the resident kernel first (a cudaFree would wait for it)
            rs_box->quit = 1;
            std::atomic_thread_fence(std::memory_order_seq_cst);
            cudaStreamSynchronize(rs_stream);
            rs_natoms = 0;
        }
        for (auto* b : {&Z, &sid, &elem, &cell_of, &cell_cnt, &cell_start, &cell_atoms, &nei_cnt, &nei_off, &nei_j,
                        &nei_s, &nei_rev, &el_count, &el_start, &el_atoms, &scan_tmp, &status})
            b->release();
        for (auto* b : {&pos, &wpos, &G, &dEdG, &atE, &gent, &gself, &vir, &force, &energy, &dEdLat, &cm_acc, &cm_E,
                        &cm_std})
            b->release();
        for (auto* b : {&Gf, &dEdGf, &atEf, &gentf, &gselff, &virf}) b->release();
        info.release();
        stats.release();
        pairs.release();
        npairs.release();
        for (auto* b : {&cnei_cnt, &cnei_off, &cnei_j, &cnei_s, &cnei_rev, &cnei_map, &pad}) b->release();
        slab.release();
        posc.release();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (h_status) cudaFreeHost(h_status);
        if (rs_box) cudaFreeHost((void*)rs_box);
        if (rs_stream) cudaStreamDestroy(rs_stream);
        if (se_dev) cudaFree(se_dev);
        if (se_host) cudaFreeHost(se_host);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Build device tables from the parsed model.
int upload_model(hdnnp_model* m) {
    const HostModel& H = m->host;
    DevModel& D = m->dev;
    std::memset(&D, 0, sizeof D);
    const int nel = (int)H.el.size();
    if (nel > kMaxEl) return fail(HDNNP_E_CAPACITY, "too many elements");
    D.nel = nel;
    D.max_rc = H.max_rc;
    for (int z = 0; z < 120; ++z) D.z2e[z] = (z <= kMaxZ) ? H.z2e[z] : -1;
    int nsf_max = 0;
    for (auto& e : H.el) nsf_max = std::max(nsf_max, (int)e.sfs.size());
    D.nsf_max = nsf_max;
    int nblk = 0;
    for (int a = 0; a < nel; ++a)
        for (int b = a; b < nel; ++b) {
            D.blk_a[nblk] = a;
            D.blk_b[nblk] = b;
            ++nblk;
        }
    D.nblk = nblk;
    std::vector<double> rc(nel), smean((size_t)nel * nsf_max, 0.0), swidth((size_t)nel * nsf_max, 1.0), ae(nel);
    std::vector<int> nsf(nel), g2_off, g4_off;
    std::vector<SF2> g2;
    std::vector<SF4> g4;
    int gmax = 1;
    for (int c = 0; c < nel; ++c) {
        const auto& E = H.el[c];
        rc[c] = E.sfs[0].rcut;
        nsf[c] = (int)E.sfs.size();
        ae[c] = E.atom_energy;
        for (int s = 0; s < nsf[c]; ++s) {
            if (H.centersf) smean[(size_t)c * nsf_max + s] = E.sfs[s].smean;
            if (H.scalesf) swidth[(size_t)c * nsf_max + s] = E.sfs[s].smax - E.sfs[s].smin;
        }
        for (int ne = 0; ne < nel; ++ne) {
            g2_off.push_back((int)g2.size());
            for (int s = 0; s < nsf[c]; ++s) {
                const SymFn& f = E.sfs[s];
                if (f.type == 2 && f.z1 == H.el[ne].z) g2.push_back(SF2{s, ne, f.eta, f.rs});
            }
        }
        for (int t = 0; t < nblk; ++t) {
            g4_off.push_back((int)g4.size());
            const int za = H.el[D.blk_a[t]].z, zb = H.el[D.blk_b[t]].z;
            std::vector<SF4> grp;
            for (int s = 0; s < nsf[c]; ++s) {
                const SymFn& f = E.sfs[s];
                if (f.type != 3) continue;
                if (!((f.z1 == za && f.z2 == zb) || (f.z1 == zb && f.z2 == za))) continue;
                SF4 q;
                q.sf = s;
                int iz = (int)f.zeta;
                q.izeta = (std::fabs(f.zeta - iz) < 1e-10 && iz >= 1) ? iz : -1;
                q.eta = f.eta;
                q.lambda = f.lambda;
                q.zeta = f.zeta;
                q.pf = q.izeta >= 1 ? std::ldexp(1.0, 1 - iz) : std::pow(2.0, 1.0 - f.zeta);
                grp.push_back(q);
            }
            std::stable_sort(grp.begin(), grp.end(), [](const SF4& x, const SF4& y) { return x.eta < y.eta; });
            gmax = std::max(gmax, (int)grp.size());
            g4.insert(g4.end(), grp.begin(), grp.end());
        }
    }
    g2_off.push_back((int)g2.size());
    g4_off.push_back((int)g4.size());
    D.gmax = gmax;

    // Angular-SF grid for the fast kernels: distinct lambda, zeta, eta over
    // all G4 SFs; every group must map one-to-one into lambda x zeta x eta.
    std::vector<short> pmap;
    {
        std::vector<double> lams, zets, etas;
        auto idx_of = [](std::vector<double>& v, double x) {
            for (size_t i = 0; i < v.size(); ++i)
                if (std::fabs(v[i] - x) <= 1e-12 * std::max(1.0, std::fabs(x))) return (int)i;
            v.push_back(x);
            return (int)v.size() - 1;
        };
        for (auto& E : H.el)
            for (auto& f : E.sfs)
                if (f.type == 3) {
                    idx_of(lams, f.lambda);
                    idx_of(zets, f.zeta);
                    idx_of(etas, f.eta);
                }
        std::sort(zets.begin(), zets.end());
        std::sort(etas.begin(), etas.end());
        int shape = 0;
        bool ints_ok = true;
        int maxz = 1;
        for (double z : zets) {
            int iz = (int)z;
            if (std::fabs(z - iz) < 1e-10 && iz >= 1) maxz = std::max(maxz, iz);
            if (z > 31.0) ints_ok = false;
        }
        // a compiled zeta set that matches exactly (same count of zeta and eta)
        for (int id = 5; id < kNumFastShapes && ints_ok && !shape; ++id) {
            bool match = (int)lams.size() <= kFastShapes[id][0] && (int)zets.size() == kFastShapes[id][1] &&
                         (int)etas.size() == kFastShapes[id][2];
            for (size_t z = 0; match && z < zets.size(); ++z) match = zets[z] == (double)kFastZeta[id][z];
            if (match) shape = id;
        }
        for (int id = 1; id <= 4 && ints_ok && !shape; ++id)
            if ((int)lams.size() <= kFastShapes[id][0] && (int)zets.size() <= kFastShapes[id][1] &&
                (int)etas.size() <= kFastShapes[id][2]) {
                shape = id;
                break;
            }
        if (!lams.empty() && shape) {
            const int NL = kFastShapes[shape][0], NZ = kFastShapes[shape][1], NE = kFastShapes[shape][2];
            const int P = NL * NZ * NE;
            pmap.assign((size_t)nel * nblk * P, (short)-1);
            bool ok = true;
            for (int c = 0; c < nel && ok; ++c)
                for (int t = 0; t < nblk && ok; ++t) {
                    const int za = H.el[D.blk_a[t]].z, zb = H.el[D.blk_b[t]].z;
                    for (int s = 0; s < nsf[c]; ++s) {
                        const SymFn& f = H.el[c].sfs[s];
                        if (f.type != 3 || !((f.z1 == za && f.z2 == zb) || (f.z1 == zb && f.z2 == za))) continue;
                        const int l = idx_of(lams, f.lambda), z = idx_of(zets, f.zeta), e = idx_of(etas, f.eta);
                        short& slot = pmap[((size_t)c * nblk + t) * P + (l * NZ + z) * NE + e];
                        if (slot >= 0) ok = false;  // two SFs on one grid point: generic kernels
                        slot = (short)s;
                    }
                }
            if (ok) {
                D.fast = shape;
                D.fl = (int)lams.size();
                D.fz = (int)zets.size();
                D.fe = (int)etas.size();
                for (int l = 0; l < D.fl; ++l) D.lam[l] = lams[l];
                for (int z = 0; z < D.fz; ++z) {
                    D.zet[z] = zets[z];
                    const int iz = (int)zets[z];
                    D.zint[z] = (std::fabs(zets[z] - iz) < 1e-10 && iz >= 1) ? iz - 1 : -1;
                    D.pfz[z] = D.zint[z] >= 0 ? std::ldexp(1.0, -D.zint[z]) : std::pow(2.0, 1.0 - zets[z]);
                }
                for (int e = 0; e < D.fe; ++e) D.eta4[e] = etas[e];
                // integer eta ratios: exp(-eta_e R) = exp(-eta_0 R)^k_e
                bool ints = D.fe > 1 && etas[0] > 0.0;
                for (int e = 1; e < D.fe && ints; ++e) {
                    const double k = etas[e] / etas[0], kr = std::nearbyint(k);
                    ints = kr >= 2.0 && kr <= 64.0 && std::fabs(k - kr) <= 1e-12 * kr;
                    D.eta_k[e] = (int)kr;
                }
                if (!ints)
                    for (int e = 0; e < 8; ++e) D.eta_k[e] = 0;
                else
                    D.eta_k[0] = 1;
                int bit = 0;
                while ((1 << (bit + 1)) <= maxz) ++bit;
                D.zmaxbit = bit;
            } else {
                pmap.clear();
            }
        }
        if (!D.fast) pmap.assign(1, (short)-1);
    }

    // networks: all elements share the hidden widths (global_nodes_short)
    const int L = (int)H.el[0].net.size();
    if (L > kMaxLayers) return fail(HDNNP_E_CAPACITY, "too many layers");
    D.nlayers = L;
    for (int l = 0; l < L; ++l) {
        D.width[l + 1] = H.el[0].net[l].nout;
        D.act[l] = H.el[0].net[l].act;
    }
    D.width[0] = nsf_max;
    std::vector<double> w, wt, bias;
    std::vector<long long> w_off, b_off;
    for (int c = 0; c < nel; ++c) {
        D.nin_el[c] = nsf[c];
        for (int l = 0; l < L; ++l) {
            const Layer& ly = H.el[c].net[l];
            w_off.push_back((long long)w.size());
            b_off.push_back((long long)bias.size());
            w.insert(w.end(), ly.w.begin(), ly.w.end());
            for (int i = 0; i < ly.nin; ++i)
                for (int o = 0; o < ly.nout; ++o) wt.push_back(ly.w[(size_t)o * ly.nin + i]);
            bias.insert(bias.end(), ly.b.begin(), ly.b.end());
        }
    }
    // one device allocation for all tables
    struct Part {
        size_t off;
        const void* src;
        size_t bytes;
    };
    std::vector<Part> parts;
    size_t off = 0;
    auto add = [&](const void* src, size_t bytes) {
        size_t o = off;
        parts.push_back({o, src, bytes});
        off += (std::max<size_t>(bytes, 8) + 255) & ~size_t(255);
        return o;
    };
    std::vector<double> sinvw(swidth.size());
    for (size_t q = 0; q < swidth.size(); ++q) sinvw[q] = 1.0 / swidth[q];
    size_t o_rc = add(rc.data(), rc.size() * 8), o_nsf = add(nsf.data(), nsf.size() * 4),
           o_g2o = add(g2_off.data(), g2_off.size() * 4), o_g2 = add(g2.data(), g2.size() * sizeof(SF2)),
           o_g4o = add(g4_off.data(), g4_off.size() * 4), o_g4 = add(g4.data(), g4.size() * sizeof(SF4)),
           o_sm = add(smean.data(), smean.size() * 8), o_sw = add(swidth.data(), swidth.size() * 8),
           o_siw = add(sinvw.data(), sinvw.size() * 8),
           o_w = add(w.data(), w.size() * 8), o_wt = add(wt.data(), wt.size() * 8), o_b = add(bias.data(), bias.size() * 8),
           o_wo = add(w_off.data(), w_off.size() * 8), o_bo = add(b_off.data(), b_off.size() * 8),
           o_ae = add(ae.data(), ae.size() * 8);
    std::vector<float> wf(w.begin(), w.end()), wtf(wt.begin(), wt.end()), bf(bias.begin(), bias.end());

    // First layer for the tensor-core network kernel: scale W1 by a power of
    // two (max |s1 W1| in [1, 2)), split into FP16 hi + lo, pack K-major
    // core matrices (8 rows x 16 B, row groups 128 B apart, K chunks of 8).
    std::vector<unsigned short> tcf, tcb;
    {
        const int kH = 32;
        bool ok = L >= 2 && L <= 4;
        for (int l = 0; l < L && ok; ++l) ok = D.width[l + 1] <= kH;
        const int kp = (nsf_max + 15) / 16 * 16;
        int np = kp;
        const int nch = (np + 255) / 256;
        const int chn = ((np + nch - 1) / nch + 15) / 16 * 16;
        np = nch * chn;
        ok = ok && (kH + np) <= 512 && kp <= 512;
        const size_t szA = (size_t)2 * 128 * kp * 2, szBf = (size_t)2 * kH * kp * 2, szBb = (size_t)2 * np * kH * 2,
                     szAb = (size_t)2 * 128 * kH * 2;
        // b1, then each later layer's W and bias zero-padded to kH x kH and kH
        const size_t wsmall = kH + (size_t)(L - 1) * (kH * kH + kH);
        // (after GEMM 1 the A_fwd region holds B_bwd, A_bwd and the hidden
        // layers' activation exchange, two 128 x 36 FP32 buffers)
        const size_t total = std::max(szA, szBb + szAb + (size_t)2 * 128 * 36 * 4) + szBf +
                             ((wsmall * 4 + 15) & ~size_t(15)) + 64;
        ok = ok && total <= 227 * 1024;
        if (ok) {
            auto cm = [](int row, int k, int rows) {
                return (size_t)((k >> 3) * (rows >> 3) * 128 + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2) / 2;
            };
            const size_t fper = (size_t)kH * kp, bper = (size_t)np * kH;  // halfwords per hi (or lo) part
            tcf.assign((size_t)nel * 2 * fper, 0);
            tcb.assign((size_t)nel * 2 * bper, 0);
            for (int c = 0; c < nel; ++c) {
                const Layer& l0 = H.el[c].net[0];
                double mx = 0.0;
                for (double v : l0.w) mx = std::max(mx, std::fabs(v));
                const double s1 = mx > 0 ? std::ldexp(1.0, -(int)std::floor(std::log2(mx))) : 1.0;
                D.tc_inv_s1[c] = (float)(1.0 / s1);
                unsigned short* F = tcf.data() + (size_t)c * 2 * fper;
                unsigned short* B = tcb.data() + (size_t)c * 2 * bper;
                for (int n = 0; n < l0.nout; ++n)
                    for (int k = 0; k < l0.nin; ++k) {
                        const double wv = l0.w[(size_t)n * l0.nin + k] * s1;
                        const __half hi = __float2half_rn((float)wv);
                        const __half lo = __float2half_rn((float)(wv - (double)__half2float(hi)));
                        const unsigned short uh = __half_as_ushort(hi), ul = __half_as_ushort(lo);
                        F[cm(n, k, kH)] = uh;
                        F[fper + cm(n, k, kH)] = ul;
                        B[cm(k, n, np)] = uh;  // transposed: row = input index, K = hidden index
                        B[bper + cm(k, n, np)] = ul;
                    }
            }
            D.tc_ok = 1;
            D.tc_kp = kp;
            D.tc_np = np;
            D.tc_nch = nch;
            D.tc_chn = chn;
            D.tc_sdelta = 64.0f;
        } else {
            tcf.assign(8, 0);
            tcb.assign(8, 0);
        }
    }
    // First layer in the register-fragment order of the FP64 tensor-core
    // network kernel (mma m8n8k4 f64: lane t holds B[t % 4][t / 4]); each
    // fragment is one coalesced 256-byte load.
    std::vector<double> dmf, dmb;
    {
        bool ok = L >= 1 && L <= 8 && D.width[L] == 1;
        for (int l = 1; l <= L && ok; ++l) ok = D.width[l] <= 32;
        D.dm_ok = ok ? 1 : 0;
        for (int c = 0; c < nel && ok; ++c) {
            const Layer& l0 = H.el[c].net[0];
            const int nin = l0.nin, H1 = l0.nout, KS = (nin + 3) / 4, NB = (nin + 7) / 8, KB = (H1 + 3) / 4;
            D.dm_off_f[c] = (long long)dmf.size();
            D.dm_off_b[c] = (long long)dmb.size();
            for (int ks = 0; ks < KS; ++ks)
                for (int nt = 0; nt < 4; ++nt)
                    for (int t = 0; t < 32; ++t) {
                        const int n = nt * 8 + t / 4, k = 4 * ks + t % 4;  // B[k][n] = W1[n][k]
                        dmf.push_back(n < H1 && k < nin ? l0.w[(size_t)n * nin + k] : 0.0);
                    }
            for (int nb = 0; nb < NB; ++nb)
                for (int ks = 0; ks < KB; ++ks)
                    for (int t = 0; t < 32; ++t) {
                        const int k = 4 * ks + t % 4, n = nb * 8 + t / 4;  // B[k][n] = W1[k][n]
                        dmb.push_back(k < H1 && n < nin ? l0.w[(size_t)k * nin + n] : 0.0);
                    }
        }
        if (dmf.empty()) dmf.assign(1, 0.0);
        if (dmb.empty()) dmb.assign(1, 0.0);
    }
    size_t o_pm = add(pmap.data(), pmap.size() * sizeof(short)), o_wf = add(wf.data(), wf.size() * 4),
           o_wtf = add(wtf.data(), wtf.size() * 4), o_bf = add(bf.data(), bf.size() * 4),
           o_tcf = add(tcf.data(), tcf.size() * 2), o_tcb = add(tcb.data(), tcb.size() * 2),
           o_dmf = add(dmf.data(), dmf.size() * 8), o_dmb = add(dmb.data(), dmb.size() * 8);
    CUDA_TRY(cudaSetDevice(m->device));
    CUDA_TRY(cudaMalloc(&m->dmem, off));
    char* base = (char*)m->dmem;
    for (auto& p : parts)
        if (p.src && p.bytes) CUDA_TRY(cudaMemcpy(base + p.off, p.src, p.bytes, cudaMemcpyHostToDevice));
    D.rc = (const double*)(base + o_rc);
    D.nsf = (const int*)(base + o_nsf);
    D.g2_off = (const int*)(base + o_g2o);
    D.g2max = 0;
    for (int c = 0; c < nel; ++c) D.g2max = std::max(D.g2max, g2_off[(size_t)c * nel + nel] - g2_off[(size_t)c * nel]);
    D.g2 = (const SF2*)(base + o_g2);
    D.g4_off = (const int*)(base + o_g4o);
    D.g4 = (const SF4*)(base + o_g4);
    D.smean = (const double*)(base + o_sm);
    D.swidth = (const double*)(base + o_sw);
    D.sinvw = (const double*)(base + o_siw);
    D.w = (const double*)(base + o_w);
    D.wt = (const double*)(base + o_wt);
    D.b = (const double*)(base + o_b);
    D.w_off = (const long long*)(base + o_wo);
    D.b_off = (const long long*)(base + o_bo);
    D.atom_energy = (const double*)(base + o_ae);
    D.pmap = (const short*)(base + o_pm);
    D.wf = (const float*)(base + o_wf);
    D.wtf = (const float*)(base + o_wtf);
    D.bf = (const float*)(base + o_bf);
    D.tc_fwd = (const unsigned short*)(base + o_tcf);
    D.tc_bwd = (const unsigned short*)(base + o_tcb);
    D.dm_fwd = (const double*)(base + o_dmf);
    D.dm_bwd = (const double*)(base + o_dmb);
    return HDNNP_OK;
}

bool h_status_ok(const hdnnp_ctx* c) { return c->h_status != nullptr; }

int check_status(hdnnp_ctx* c) {
    int f = c->h_status[0];
    if (f & 1) return fail(HDNNP_E_INPUT, "atom with an element that is not in the potential");
    if (f & 2) return fail(HDNNP_E_STATE, "internal error: neighbour list is not symmetric");
    if (f & 4) return fail(HDNNP_E_CAPACITY, "neighbour count above the kernel capacity");
    if (f & 8)
        return fail(HDNNP_E_INPUT, "non-finite position (structure " + std::to_string(c->h_status[1] - 1) + ")");
    if (f & 16) return fail(HDNNP_E_TIMEOUT, "tensor-core network kernel: bounded wait expired");
    return HDNNP_OK;
}

int collect_profile(hdnnp_ctx* c) {
    if (!c->prof_pending) return HDNNP_OK;
    CUDA_TRY(cudaEventSynchronize(c->ev[7]));
    for (int k = 0; k < 7; ++k) {
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]));
        c->stage_ms[k] += ms;
    }
    c->prof_pending = false;
    return HDNNP_OK;
}

// Core pipeline; inputs already on the device in c->Z / c->pos (or external
// device pointers), structure set-up in c->hinfo.
// Stages of one evaluation, as the reference splits hdnnpEnergyAndForces
// (hdnnps.f90:346-368): neighbour lists (with the wrap and the element
// groups), symmetry-function values, and the networks with the force and
// dE/dh contraction.  A call may run a suffix of them on the lists (and
// values) the previous call left in the context.
enum StageBits { kStageLists = 1, kStageSF = 2, kStageNN = 4, kStageAll = 7 };

int run_pipeline(hdnnp_ctx* c, int nstruct, int natoms, const int32_t* Zd, const double* posd, double* energy_d,
                 double* force_d, double* dEdLat_d, cudaStream_t st, PipePlan* pp = nullptr,
                 const Committee* cm = nullptr, int stages = kStageAll, const DevModel* nn_model = nullptr) {
    hdnnp_model* m = c->model;
    DevModel D = m->dev;
    // runtime-zeta variant of a compiled-zeta shape (same product layout)
    if (c->runtime_zeta && D.fast == 5) D.fast = 1;
    if (c->runtime_zeta && D.fast == 6) D.fast = 2;
    int r;
    if (stages & kStageLists) c->stage_seq = 0;  // the stage API's lists are replaced
    // stage events only when a call runs the whole evaluation
    const bool prof = c->profile && stages == kStageAll;
    int L = 0;
    Batch b{};
    bool fast = false, mixed = false;
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (pp) CUDA_TRY(cudaStreamIsCapturing(st, &capturing));
    auto mark = [&](int k) -> int {
        if (!prof) return HDNNP_OK;
        // inside a stream capture only an external record becomes a graph node
        if (capturing == cudaStreamCaptureStatusActive)
            CUDA_TRY(cudaEventRecordWithFlags(c->ev[k], st, cudaEventRecordExternal));
        else
            CUDA_TRY(cudaEventRecord(c->ev[k], st));
        return HDNNP_OK;
    };
    if (!(stages & kStageLists)) {
        // later stages on the lists (and values) of the previous call
        if (!c->have_last) return fail(HDNNP_E_STATE, "no neighbour lists on this context");
        b = c->last;
        b.force = force_d;
        b.energy = energy_d;
        b.dEdLat = dEdLat_d;
        fast = c->last_fast;
        mixed = c->last_mixed;
        if (!h_status_ok(c)) return fail(HDNNP_E_STATE, "no neighbour lists on this context");
        CUDA_TRY(cudaMemsetAsync(b.status, 0, sizeof(int), st));
    } else {
    int ncells = 0;
    if (!pp || pp->upload) {
        for (auto& S : c->hinfo) {
            S.cell_off = ncells;
            // a molecule of a plan gets the largest grid its box may take
            ncells += (pp && pp->dev_boxes && !S.periodic) ? 64 * S.nat + 4096 : S.ngrid[0] * S.ngrid[1] * S.ngrid[2];
        }
        if ((r = c->info.ensure(nstruct))) return r;
        CUDA_TRY(cudaMemcpyAsync(c->info.p, c->hinfo.data(), sizeof(StructInfo) * nstruct, cudaMemcpyHostToDevice, st));
        if (pp) pp->ncells = ncells;
    } else {
        ncells = pp->ncells;
    }
    const size_t N = natoms;
    if ((r = c->sid.ensure(N)) || (r = c->elem.ensure(N)) || (r = c->wpos.ensure(3 * N)) || (r = c->cell_of.ensure(N)) ||
        (r = c->cell_cnt.ensure(ncells + 1)) || (r = c->cell_start.ensure(ncells + 1)) ||
        (r = c->cell_atoms.ensure(N)) || (r = c->posc.ensure(N)) || (r = c->nei_cnt.ensure(N + 1)) ||
        (r = c->nei_off.ensure(N + 1)) ||
        (r = c->el_count.ensure(kMaxEl + 1)) || (r = c->el_start.ensure(kMaxEl + 1)) || (r = c->el_atoms.ensure(N)) ||
        (r = c->scan_tmp.ensure(std::max<size_t>(N, ncells) / 1024 + 256)) || (r = c->status.ensure(4)) ||
        (r = c->G.ensure(N * D.nsf_max)) || (r = c->dEdG.ensure(N * D.nsf_max)) || (r = c->atE.ensure(N)) ||
        (r = c->gself.ensure(3 * N)) || (r = c->vir.ensure(9 * N)))
        return r;
    if (!c->h_status) CUDA_TRY(cudaMallocHost(&c->h_status, 4 * sizeof(int)));
    b.nstruct = nstruct;
    b.natoms = natoms;
    b.ncells = ncells;
    b.info = c->info.p;
    b.Z = Zd;
    b.pos = posd;
    b.sid = c->sid.p;
    b.elem = c->elem.p;
    b.wpos = c->wpos.p;
    b.cell_of = c->cell_of.p;
    b.cell_cnt = c->cell_cnt.p;
    b.cell_start = c->cell_start.p;
    b.cell_atoms = c->cell_atoms.p;
    b.posc = c->posc.p;
    b.nei_cnt = c->nei_cnt.p;
    b.nei_off = c->nei_off.p;
    b.el_count = c->el_count.p;
    b.el_start = c->el_start.p;
    b.el_atoms = c->el_atoms.p;
    b.scan_tmp = c->scan_tmp.p;
    b.status = c->status.p;
    b.G = c->G.p;
    b.dEdG = c->dEdG.p;
    b.atE = c->atE.p;
    b.gself = c->gself.p;
    b.vir = c->vir.p;
    b.force = force_d;
    b.energy = energy_d;
    b.dEdLat = dEdLat_d;
    b.sf_split = c->sf_split;
    b.sf_blocks_per_sm = c->sf_blocks_per_sm;
    b.nei_warp = c->nei_warp;
    b.rc_list = pp ? pp->rc_list : 0.0;
    b.rebuild = pp ? pp->rebuild : nullptr;
    b.wshift = pp ? pp->wshift : nullptr;
    b.pos_ref = pp ? pp->pos_ref : nullptr;
    if (prof) {
        // a plan collects the stage times of its replays itself (ctx_profile_replay)
        if ((!pp || pp->eager) && (r = collect_profile(c))) return r;
        for (auto& e : c->ev)
            if (!e) CUDA_TRY(cudaEventCreate(&e));
        if (!c->stats.p) {
            if ((r = c->stats.ensure(8))) return r;
            CUDA_TRY(cudaMemset(c->stats.p, 0, 8 * sizeof(unsigned long long)));
        }
        b.stats = c->stats.p;
        if (!pp || pp->eager) {
            c->host_counts[0] += 1;
            c->host_counts[1] += natoms;
        }
    }
    CUDA_TRY(cudaMemsetAsync(b.status, 0, 4 * sizeof(int), st));
    if ((r = mark(0))) return r;
    if (pp && pp->pad_lists && pp->e_cap > 0) {
        // capacities known: one search pass into padded rows (buffer sized by the probe)
        if ((r = c->pad.ensure(2 * N * (size_t)pp->m_cap)) || (r = c->slab.ensure(N * (size_t)kSlabStride)))
            return r;
        b.pad = reinterpret_cast<int2*>(c->pad.p);
        b.pad_cap = pp->m_cap;
        b.slab = c->slab.p;
    }
    if (pp && pp->dev_boxes) L += launch_molecule_boxes(b, pp->rc_list > 0.0 ? pp->rc_list : D.max_rc, st);
    L += launch_neighbour_build_a(b, D, st, pp && !pp->upload);
    size_t E = 0;
    if (pp && pp->e_cap > 0) {
        // planned: no host read; overflow of the capacities is flagged on the device
        L += launch_capacity_guard(b, pp->e_cap, pp->m_cap, st);
        E = (size_t)pp->e_cap;
        b.mmax = pp->m_cap;
    } else {
        // entry total and the largest count
        CUDA_TRY(cudaMemcpyAsync(c->h_status + 2, b.nei_off + natoms, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(c->h_status + 3, b.status + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(c->h_status, b.status, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(c->h_status + 1, b.status + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        if ((r = check_status(c))) return r;
        if (c->h_status[2] < 0) return fail(HDNNP_E_CAPACITY, "more than 2^31 neighbour entries");
        E = (size_t)c->h_status[2];
        b.mmax = c->h_status[3];
        if (pp) {
            // probe evaluation of a plan: capacities with headroom
            const double f = 1.0 + std::max(pp->margin, 0.0);
            const double ecap = std::ceil((double)E * f) + 1024.0;
            if (ecap > (double)INT32_MAX) return fail(HDNNP_E_CAPACITY, "planned neighbour entries above 2^31");
            pp->e_cap = (long long)ecap;
            pp->m_cap = (((int)std::ceil(b.mmax * f) + 8) + 31) / 32 * 32;
            E = (size_t)pp->e_cap;
            b.mmax = pp->m_cap;
            if (pp->pad_lists && ((r = c->pad.ensure(2 * N * (size_t)pp->m_cap)) ||
                                  (r = c->slab.ensure(N * (size_t)kSlabStride))))
                return r;
        }
    }
    if ((r = c->nei_j.ensure(E + 1)) || (r = c->nei_s.ensure(E + 1)) || (r = c->nei_rev.ensure(E + 1)) ||
        (r = c->gent.ensure(3 * E + 3)))
        return r;
    b.nentries = (int)E;
    b.nei_j = c->nei_j.p;
    b.nei_s = c->nei_s.p;
    b.nei_rev = c->nei_rev.p;
    b.gent = c->gent.p;
    // Verlet-skin lists: the stages after the list read a compacted copy
    const bool compact = b.rc_list > D.max_rc;
    if (compact && ((r = c->cnei_cnt.ensure(N + 1)) || (r = c->cnei_off.ensure(N + 1)) ||
                    (r = c->cnei_j.ensure(E + 1)) || (r = c->cnei_s.ensure(E + 1)) ||
                    (r = c->cnei_rev.ensure(E + 1)) || (r = c->cnei_map.ensure(E + 1))))
        return r;
    // mixed precision runs on the fast (lambda x zeta x eta) kernels; potentials
    // outside their shapes evaluate in FP64 with the generic kernels
    fast = D.fast && !c->generic_sf;
    mixed = c->precision == HDNNP_PREC_MIXED && fast;
    if (fast) {
        if ((r = c->pairs.ensure(N * (size_t)kPairCap)) || (r = c->npairs.ensure(N))) return r;
        b.pairs = c->pairs.p;
        b.npairs = c->npairs.p;
        b.pcap = kPairCap;
    }
    if (mixed) {
        if ((r = c->Gf.ensure(N * D.nsf_max)) || (r = c->dEdGf.ensure(N * D.nsf_max)) || (r = c->atEf.ensure(N)) ||
            (r = c->gentf.ensure(3 * E + 3)) || (r = c->gselff.ensure(3 * N)) || (r = c->virf.ensure(9 * N)))
            return r;
        b.Gf = c->Gf.p;
        b.dEdGf = c->dEdGf.p;
        b.atEf = c->atEf.p;
        b.gentf = c->gentf.p;
        b.gselff = c->gselff.p;
        b.virf = c->virf.p;
    }
    {
        int mm = ((b.mmax + 31) / 32) * 32;
        const size_t sf_smem =
            fast ? sf_fast_smem_per_warp(mm, D.g2max, D.nblk, fast_shape_p(D.fast), true, mixed) * 4
                   : sf_smem_per_warp(mm, true) * 4;
        if (sf_smem > 220 * 1024 || (fast && mm > 1024))
            return fail(HDNNP_E_CAPACITY, "too many neighbours per atom for the symmetry-function kernels");
        if (mlp_smem_bytes(D, mixed ? sizeof(float) : sizeof(double)) > 220 * 1024)
            return fail(HDNNP_E_CAPACITY, "network too wide for the MLP kernel");
        if (cm) {
            for (int q = 0; q < cm->k; ++q)
                if (mlp_smem_bytes(*cm->members[q], mixed ? sizeof(float) : sizeof(double)) > 220 * 1024)
                    return fail(HDNNP_E_CAPACITY, "committee member " + std::to_string(q) + ": network too wide");
            if ((r = c->cm_acc.ensure(N * D.nsf_max)) || (r = c->cm_E.ensure((size_t)cm->k * nstruct))) return r;
        }
    }
    if ((r = mark(1))) return r;  // after the host read: stage 1 starts here
    L += launch_neighbour_build_b(b, D, st);
    if (compact) {
        const CompactLists cl{c->cnei_cnt.p, c->cnei_off.p, c->cnei_j.p, c->cnei_s.p, c->cnei_rev.p, c->cnei_map.p};
        L += launch_compact_lists(b, D.max_rc, cl, st);
        b.nei_cnt = cl.cnt;
        b.nei_off = cl.off;
        b.nei_j = cl.nj;
        b.nei_s = cl.ns;
        b.nei_rev = cl.rev;
        b.rc_list = D.max_rc;  // entries beyond an element's own cutoff are still dropped
    }
    if ((r = mark(2))) return r;
    L += launch_element_groups(b, D, st);
    if ((r = mark(3))) return r;
    c->last_fast = fast;
    c->last_mixed = mixed;
    }  // lists stage
    if (stages & kStageSF) {
        L += fast ? launch_sf_values_fast(b, D, mixed, st) : launch_sf_values(b, D, st);
        if ((r = mark(4))) return r;
    }
    if (stages & kStageNN) {
        // networks of the context's potential, of another potential with the
        // same elements and input widths (nn_model), or of a committee
        const DevModel& M = nn_model ? *nn_model : D;
        if (cm)
            L += launch_committee_networks(b, *cm, mixed, !c->mlp_simt, c->cm_acc.p, c->cm_E.p, st);
        else if (mixed && M.tc_ok && !c->mlp_simt)
            L += launch_mlp_tc(b, M, st);
        else
            L += mixed ? launch_mlp_fp32(b, M, st) : launch_mlp(b, M, st);
        if ((r = mark(5))) return r;
        L += fast ? launch_sf_gradients_fast(b, D, mixed, st) : launch_sf_gradients(b, D, st);
        if ((r = mark(6))) return r;
        L += mixed ? launch_forces_and_reduce_fp32(b, D, dEdLat_d != nullptr, st)
                   : launch_forces_and_reduce(b, D, dEdLat_d != nullptr, st);
        if (cm) L += launch_committee_finish(b, *cm, c->cm_E.p, st);  // mean energies (and std)
        if ((r = mark(7))) return r;
    }
    if (prof && (!pp || pp->eager)) c->prof_pending = true;
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(c->h_status, b.status, sizeof(int), cudaMemcpyDeviceToHost, st));
    // without the mid-pipeline host read, the structure a non-finite position
    // blames comes back here (not inside a graph capture: plans read acc)
    if (pp && pp->e_cap > 0 && capturing != cudaStreamCaptureStatusActive)
        CUDA_TRY(cudaMemcpyAsync(c->h_status + 1, b.status + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
    c->launches = L;
    c->last = b;
    c->have_last = true;
    return HDNNP_OK;
}

// Io block of the small-molecule evaluation (bytes from the start of
// se_dev, mirrored in se_host): positions, element indices and the status
// accumulator go in (one copy); the status, energy and forces come out (one
// copy).  Sized for kSmallMolecule atoms.
struct SmallEvalIo {
    static constexpr size_t pos = 0;                                   // double[3 * kSmallMolecule]
    static constexpr size_t elem = pos + 8 * 3 * kSmallMolecule;       // int[kSmallMolecule]
    static constexpr size_t acc = elem + 4 * kSmallMolecule;           // int[2]
    static constexpr size_t energy = acc + 8;                          // double
    static constexpr size_t force = energy + 8;                        // double[3 * kSmallMolecule]
    static constexpr size_t info = (force + 8 * 3 * kSmallMolecule + 255) & ~size_t(255);  // StructInfo
    static constexpr size_t homes = (info + sizeof(StructInfo) + 255) & ~size_t(255);
    static constexpr size_t in_bytes = energy - pos;   // pos, elem, acc
    static constexpr size_t out_off = acc;             // acc, energy, force
};

// Device homes of the single-block kernel for a molecule of up to
// kSmallMolecule atoms (the per-step arrays its shared memory cannot hold):
// allocated once per context.
int small_eval_setup(hdnnp_ctx* c) {
    if (c->se_dev) return HDNNP_OK;
    const DevModel& D = c->model->dev;
    const size_t N = kSmallMolecule, NN = N * N, nsf = (size_t)D.nsf_max;
    const size_t nd = 2 * N * nsf + 3 * NN + 9 * N, ni = 3 * NN;
    const size_t bytes = SmallEvalIo::homes + nd * 8 + ni * 4;
    CUDA_TRY(cudaMalloc(&c->se_dev, bytes));
    CUDA_TRY(cudaHostAlloc((void**)&c->se_host, SmallEvalIo::homes, cudaHostAllocMapped));
    std::memset(c->se_host, 0, SmallEvalIo::homes);
    CUDA_TRY(cudaHostGetDevicePointer((void**)&c->se_hdev, c->se_host, 0));
    unsigned char* base = (unsigned char*)c->se_dev;
    double* d = (double*)(base + SmallEvalIo::homes);
    int* q = (int*)(d + nd);
    Batch& b = c->se_b;
    b = Batch{};
    b.nstruct = 1;
    b.G = d; d += N * nsf;
    b.dEdG = d; d += N * nsf;
    b.gent = d; d += 3 * NN;
    b.vir = d;
    b.nei_j = q; q += NN;
    b.nei_s = q; q += NN;
    b.nei_rev = q;
    b.elem = (int*)(base + SmallEvalIo::elem);
    b.info = (const StructInfo*)(base + SmallEvalIo::info);
    StructInfo S{};
    for (int k = 0; k < 9; ++k) S.h[k] = S.hinv[k] = (k % 4 == 0) ? 1.0 : 0.0;
    S.ngrid[0] = S.ngrid[1] = S.ngrid[2] = 1;
    CUDA_TRY(cudaMemcpy(base + SmallEvalIo::info, &S, sizeof S, cudaMemcpyHostToDevice));
    return HDNNP_OK;
}

// Stops the context's resident kernel (if one runs) and waits for it.
int resident_stop(hdnnp_ctx* c) {
    if (!c->rs_natoms) return HDNNP_OK;
    c->rs_box->quit = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    CUDA_TRY(cudaStreamSynchronize(c->rs_stream));
    c->rs_natoms = 0;
    return HDNNP_OK;
}

// One molecule through the resident item-parallel kernel: the inputs and a
// request number go into the mailbox, the kernel (launched on the first
// call, or again when the molecule's size changes or the kernel left after
// idling) answers with the outputs and the number.  Every field of the
// mailbox has one writer, so a kernel that left just before the request
// came is seen (exited) and replaced, and the new kernel serves the pending
// request.  The host waits at most 2 s.
int small_eval_resident(hdnnp_ctx* c, int nat, const int32_t* Z, const double* pos, double* energy, double* force) {
    const DevModel& D = c->model->dev;
    if (!c->rs_box) {
        CUDA_TRY(cudaHostAlloc((void**)&c->rs_box, sizeof(ResidentBox), cudaHostAllocMapped));
        std::memset((void*)c->rs_box, 0, sizeof(ResidentBox));
        CUDA_TRY(cudaHostGetDevicePointer((void**)&c->rs_dbox, (void*)c->rs_box, 0));
        CUDA_TRY(cudaStreamCreateWithFlags(&c->rs_stream, cudaStreamNonBlocking));
    }
    ResidentBox* bx = c->rs_box;
    int r;
    if (c->rs_natoms && c->rs_natoms != nat && (r = resident_stop(c))) return r;
    bx->natoms = nat;
    std::memcpy(bx->pos, pos, sizeof(double) * 3 * nat);
    for (int i = 0; i < nat; ++i) bx->elem[i] = D.z2e[Z[i]];
    bx->acc[0] = bx->acc[1] = 0;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    const int seq = ++c->rs_seq;
    bx->req = seq;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    c->launches = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        if (!c->rs_natoms) {
            bx->quit = 0;
            bx->exited = 0;
            std::atomic_thread_fence(std::memory_order_seq_cst);
            if (!launch_small_resident(D, nat, c->rs_dbox, c->rs_stream))
                return fail(HDNNP_E_STATE, "molecule does not take the resident single-block form");
            CUDA_TRY(cudaGetLastError());
            c->rs_natoms = nat;
            c->launches = 1;
        }
        if (bx->ack == seq) break;
        if (bx->exited) {  // it left, idle, before it saw this request: replace it
            CUDA_TRY(cudaStreamSynchronize(c->rs_stream));
            c->rs_natoms = 0;
            continue;
        }
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(2)) {
            resident_stop(c);
            return fail(HDNNP_E_STATE, "the resident single-block kernel did not answer within 2 s");
        }
    }
    std::atomic_thread_fence(std::memory_order_seq_cst);
    c->have_last = false;
    const int st = bx->acc[0];
    if (st & 8) return fail(HDNNP_E_INPUT, "non-finite position (structure 0)");
    if (st) return fail(HDNNP_E_STATE, "single-block evaluation: device flags " + std::to_string(st));
    *energy = bx->energy;
    std::memcpy(force, bx->force, sizeof(double) * 3 * nat);
    return HDNNP_OK;
}

// One molecule of nat <= kSmallMolecule atoms in FP64 through the
// single-block kernel (fused_md.cu, evaluation mode): one kernel and one
// wait (plus a host-to-device and a device-to-host copy when the
// warp-per-atom form runs), or a request to the context's resident kernel
// (item-parallel form, option small_resident).  Z must be validated.
int small_eval(hdnnp_ctx* c, int nat, const int32_t* Z, const double* pos, double* energy, double* force) {
    int r;
    const DevModel& D = c->model->dev;
    if (c->small_resident && small_md_tiny(D, nat)) return small_eval_resident(c, nat, Z, pos, energy, force);
    if ((r = small_eval_setup(c))) return r;
    unsigned char* h = c->se_host;
    unsigned char* dv = (unsigned char*)c->se_dev;
    std::memcpy(h + SmallEvalIo::pos, pos, sizeof(double) * 3 * nat);
    int* he = (int*)(h + SmallEvalIo::elem);
    for (int i = 0; i < nat; ++i) he[i] = D.z2e[Z[i]];
    int* hacc = (int*)(h + SmallEvalIo::acc);
    hacc[0] = hacc[1] = 0;
    cudaStream_t st = c->stream;
    Batch b = c->se_b;
    // The item-parallel form gets its inputs with the launch (kernel
    // parameters) and writes its results once, straight into the mapped host
    // block (no copies).  The warp-per-atom form reads the element indices
    // throughout and gets device copies.
    const bool mapped = small_md_tiny(D, nat);
    if (mapped) {
        dv = c->se_hdev;
        b.elem = (int*)(dv + SmallEvalIo::elem);
    } else {
        CUDA_TRY(cudaMemcpyAsync(dv, h, SmallEvalIo::in_bytes, cudaMemcpyHostToDevice, st));
    }
    b.natoms = nat;
    b.mmax = nat - 1;
    b.nentries = nat * nat;
    SmallMdArgs a{};
    a.natoms = nat;
    a.nsteps = 1;
    a.dt = 0.0;
    a.pos = (double*)(dv + SmallEvalIo::pos);
    a.force = (double*)(dv + SmallEvalIo::force);
    a.energy = (double*)(dv + SmallEvalIo::energy);
    a.acc = (int*)(dv + SmallEvalIo::acc);
    a.eval_only = 1;
    if (mapped) {
        // the item-parallel form takes the positions and element indices with
        // the launch and writes its results into the mapped block
        a.inline_pos = (const double*)(h + SmallEvalIo::pos);
        a.inline_elem = he;
    }
    launch_small_md(b, D, a, st);
    CUDA_TRY(cudaGetLastError());
    const size_t out = SmallEvalIo::force + sizeof(double) * 3 * nat - SmallEvalIo::out_off;
    if (!mapped)
        CUDA_TRY(cudaMemcpyAsync(h + SmallEvalIo::out_off, dv + SmallEvalIo::out_off, out, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    c->launches = 1;
    c->have_last = false;  // the intermediates are not in the context's arrays
    if (hacc[0] & 8) return fail(HDNNP_E_INPUT, "non-finite position (structure 0)");
    if (hacc[0]) return fail(HDNNP_E_STATE, "single-block evaluation: device flags " + std::to_string(hacc[0]));
    std::memcpy(energy, h + SmallEvalIo::energy, sizeof(double));
    std::memcpy(force, h + SmallEvalIo::force, sizeof(double) * 3 * nat);
    return HDNNP_OK;
}

int prepare_structs(hdnnp_ctx* c, int nstruct, const int64_t* off, const int32_t* Z, const double* pos,
                    const int32_t* periodic, const double* lat, bool validate_Z) {
    const HostModel& H = c->model->host;
    c->hinfo.resize(nstruct);
    if (off[0] != 0) return fail(HDNNP_E_INPUT, "atom_off[0] must be 0");
    for (int s = 0; s < nstruct; ++s) {
        int64_t a0 = off[s], a1 = off[s + 1];
        if (a1 <= a0) return fail(HDNNP_E_INPUT, "structure " + std::to_string(s) + " has no atoms");
        if (a1 > INT32_MAX) return fail(HDNNP_E_CAPACITY, "more than 2^31 atoms");
        int per = periodic ? periodic[s] : 0;
        int r = struct_setup((int)(a1 - a0), pos ? pos + 3 * a0 : nullptr, per, lat + 9 * s, H.max_rc, c->hinfo[s]);
        if (r) return fail(r, "structure " + std::to_string(s) + ": " + g_err);
        c->hinfo[s].atom_off = (int)a0;
        c->hinfo[s].nat = (int)(a1 - a0);
    }
    if (validate_Z)
        for (int64_t i = 0; i < off[nstruct]; ++i)
            if (Z[i] < 1 || Z[i] > kMaxZ || H.z2e[Z[i]] < 0)
                return fail(HDNNP_E_INPUT, "atom " + std::to_string(i) + " has element Z=" + std::to_string(Z[i]) +
                                               " that is not in the potential");
    return HDNNP_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

const char* hdnnp_last_error(void) { return g_err.c_str(); }

int hdnnp_model_load_runner(const char* path, int device, hdnnp_model** out) {
    if (!path || !out) return fail(HDNNP_E_INPUT, "null argument");
    *out = nullptr;
    auto* m = new hdnnp_model();
    m->device = device;
    std::string err;
    if (!load_runner(path, m->host, err)) {
        delete m;
        return fail(HDNNP_E_IO, err);
    }
    int r = upload_model(m);
    if (r) {
        if (m->dmem) cudaFree(m->dmem);
        delete m;
        return r;
    }
    *out = m;
    return HDNNP_OK;
}

int hdnnp_model_info(const hdnnp_model* m, int* nelem, int* Z, int* nsf, double* max_rc) {
    if (!m) return fail(HDNNP_E_INPUT, "null model");
    if (nelem) *nelem = (int)m->host.el.size();
    for (size_t e = 0; e < m->host.el.size(); ++e) {
        if (Z) Z[e] = m->host.el[e].z;
        if (nsf) nsf[e] = (int)m->host.el[e].sfs.size();
    }
    if (max_rc) *max_rc = m->host.max_rc;
    return HDNNP_OK;
}

int hdnnp_model_flags(const hdnnp_model* m, int* scalesf, int* centersf, double* emin, double* emax,
                      double* atomenergies) {
    if (!m) return fail(HDNNP_E_INPUT, "null model");
    const HostModel& H = m->host;
    if (scalesf) *scalesf = H.scalesf ? 1 : 0;
    if (centersf) *centersf = H.centersf ? 1 : 0;
    if (emin) *emin = H.emin;
    if (emax) *emax = H.emax;
    if (atomenergies) {
        for (int z = 0; z < kMaxZ; ++z) atomenergies[z] = 0.0;
        for (const auto& e : H.el) atomenergies[e.z - 1] = e.atom_energy;
    }
    return HDNNP_OK;
}

namespace {
const ElementModel* element_of(const hdnnp_model* m, int Z) {
    if (!m || Z < 1 || Z > kMaxZ || m->host.z2e[Z] < 0) return nullptr;
    return &m->host.el[m->host.z2e[Z]];
}
}  // namespace

int hdnnp_model_symfunctions(const hdnnp_model* m, int Z, int* nsf, double* params) {
    const ElementModel* e = element_of(m, Z);
    if (!e || !nsf) return fail(HDNNP_E_INPUT, "null argument or element not in the potential");
    *nsf = (int)e->sfs.size();
    if (params)
        for (size_t s = 0; s < e->sfs.size(); ++s) {
            const SymFn& f = e->sfs[s];
            const double row[11] = {(double)f.type, (double)f.z1, (double)f.z2, f.rcut, f.eta, f.lambda,
                                    f.zeta, f.rs, f.smin, f.smax, f.smean};
            std::memcpy(params + 11 * s, row, sizeof row);
        }
    return HDNNP_OK;
}

int hdnnp_model_network(const hdnnp_model* m, int Z, int* nlayers, int* dims, char* acts, double* values) {
    const ElementModel* e = element_of(m, Z);
    if (!e || !nlayers) return fail(HDNNP_E_INPUT, "null argument or element not in the potential");
    *nlayers = (int)e->net.size();
    size_t o = 0;
    for (size_t l = 0; l < e->net.size(); ++l) {
        const Layer& ly = e->net[l];
        if (dims) {
            dims[2 * l] = ly.nin;
            dims[2 * l + 1] = ly.nout;
        }
        if (acts) acts[l] = ly.act;
        if (values) {
            // weights(nOut, nInp) column-major, as nnLayer%weights, then bias(nOut)
            for (int i = 0; i < ly.nin; ++i)
                for (int k = 0; k < ly.nout; ++k) values[o + (size_t)i * ly.nout + k] = ly.w[(size_t)k * ly.nin + i];
            o += (size_t)ly.nin * ly.nout;
            for (int k = 0; k < ly.nout; ++k) values[o + k] = ly.b[k];
            o += ly.nout;
        }
    }
    return HDNNP_OK;
}

void hdnnp_model_free(hdnnp_model* m) {
    if (!m) return;
    if (m->dmem) {
        cudaSetDevice(m->device);
        cudaFree(m->dmem);
    }
    delete m;
}

int hdnnp_ctx_create(hdnnp_model* m, hdnnp_ctx** out) {
    if (!m || !out) return fail(HDNNP_E_INPUT, "null argument");
    CUDA_TRY(cudaSetDevice(m->device));
    auto* c = new hdnnp_ctx();
    c->model = m;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return fail(HDNNP_E_CUDA, "cudaStreamCreate failed");
    }
    *out = c;
    return HDNNP_OK;
}

void hdnnp_ctx_free(hdnnp_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->model->device);
    cudaStreamSynchronize(c->stream);
    delete c;
}

int hdnnp_ctx_set_precision(hdnnp_ctx* c, int precision) {
    if (!c) return fail(HDNNP_E_INPUT, "null context");
    if (precision != HDNNP_PREC_FP64 && precision != HDNNP_PREC_MIXED) return fail(HDNNP_E_INPUT, "unknown precision");
    c->precision = precision;
    return HDNNP_OK;
}

int hdnnp_ctx_set_option(hdnnp_ctx* c, const char* name, int value) {
    if (!c || !name) return fail(HDNNP_E_INPUT, "null argument");
    if (std::string(name) == "generic_sf") {
        c->generic_sf = value != 0;
        return HDNNP_OK;
    }
    if (std::string(name) == "mlp_simt") {
        c->mlp_simt = value != 0;
        return HDNNP_OK;
    }
    if (std::string(name) == "runtime_zeta") {
        c->runtime_zeta = value != 0;
        return HDNNP_OK;
    }
    if (std::string(name) == "sf_split") {
        if (value < -1 || value > 1024) return fail(HDNNP_E_INPUT, "sf_split must be -1, 0 or 1..1024");
        c->sf_split = value;
        return HDNNP_OK;
    }
    if (std::string(name) == "sf_blocks_per_sm") {
        if (value < 0 || value > 64) return fail(HDNNP_E_INPUT, "sf_blocks_per_sm must be 0..64");
        c->sf_blocks_per_sm = value;
        return HDNNP_OK;
    }
    if (std::string(name) == "small_resident") {
        c->small_resident = value != 0;
        return c->small_resident ? HDNNP_OK : resident_stop(c);
    }
    if (std::string(name) == "small_eval") {
        c->small_eval = value != 0;
        return HDNNP_OK;
    }
    if (std::string(name) == "nei_warp") {
        if (value < -1 || value > 1) return fail(HDNNP_E_INPUT, "nei_warp must be -1, 0 or 1");
        c->nei_warp = value;
        return HDNNP_OK;
    }
    return fail(HDNNP_E_INPUT, std::string("unknown option ") + name);
}

int hdnnp_eval_batch(hdnnp_ctx* c, int nstruct, const int64_t* atom_off, const int32_t* Z, const double* pos,
                     const int32_t* periodic, const double* lat, double* energy, double* force, double* dEdLat) {
    if (!c || nstruct <= 0 || !atom_off || !Z || !pos || !lat || !energy || !force)
        return fail(HDNNP_E_INPUT, "null argument or empty batch");
    CUDA_TRY(cudaSetDevice(c->model->device));
    if (dEdLat && periodic) {
        // dEdLat rows of molecules are written as zeros
    }
    int r = prepare_structs(c, nstruct, atom_off, Z, pos, periodic, lat, true);
    if (r) return r;
    const int natoms = (int)atom_off[nstruct];
    const size_t N = natoms;
    cudaStream_t st = c->stream;
    // one small molecule in FP64 (the reference's MD example): one kernel
    if (nstruct == 1 && !(periodic && periodic[0]) && natoms <= kSmallMolecule && c->small_eval &&
        c->precision == HDNNP_PREC_FP64 && !c->profile &&
        small_md_smem_bytes(c->model->dev, natoms) <= 226 * 1024) {
        c->stage_seq = 0;
        if (dEdLat) std::memset(dEdLat, 0, 9 * sizeof(double));
        return small_eval(c, natoms, Z, pos, energy, force);
    }
    if ((r = c->Z.ensure(N)) || (r = c->pos.ensure(3 * N)) || (r = c->force.ensure(3 * N)) ||
        (r = c->energy.ensure(nstruct)) || (r = c->dEdLat.ensure(9 * (size_t)nstruct)))
        return r;
    CUDA_TRY(cudaMemcpyAsync(c->Z.p, Z, sizeof(int32_t) * N, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(c->pos.p, pos, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    auto results = [&]() -> int {
        CUDA_TRY(cudaMemcpyAsync(energy, c->energy.p, sizeof(double) * nstruct, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(force, c->force.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, st));
        if (dEdLat)
            CUDA_TRY(cudaMemcpyAsync(dEdLat, c->dEdLat.p, sizeof(double) * 9 * nstruct, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        return HDNNP_OK;
    };
    // After a call that counted its lists on the host, one search pass into
    // padded rows of 1.25 x the densest atom seen + 8 (no host read inside
    // the pipeline); an atom above that is flagged on the device, and the
    // call runs again with counted lists before returning.
    const int pad = c->m_est > 0 ? ((int)std::ceil(1.25 * c->m_est) + 8 + 31) / 32 * 32 : 0;
    if (pad > 0 && (double)N * pad < (double)INT32_MAX) {
        PipePlan lp{};
        lp.eager = true;
        lp.pad_lists = true;
        lp.m_cap = pad;
        lp.e_cap = (long long)N * pad;
        if ((r = run_pipeline(c, nstruct, natoms, c->Z.p, c->pos.p, c->energy.p, c->force.p,
                              dEdLat ? c->dEdLat.p : nullptr, st, &lp)) ||
            (r = results()))
            return r;
        if (!(c->h_status[0] & 32)) return check_status(c);
        if ((r = check_status(c))) return r;
        c->m_est = 0;
    }
    r = run_pipeline(c, nstruct, natoms, c->Z.p, c->pos.p, c->energy.p, c->force.p, dEdLat ? c->dEdLat.p : nullptr, st);
    if (r) return r;
    c->m_est = std::max(c->m_est, c->h_status[3]);  // the largest count, read by the pipeline
    if ((r = results())) return r;
    return check_status(c);
}

int hdnnp_eval_batch_device(hdnnp_ctx* c, int nstruct, const int64_t* atom_off_host, const int64_t* atom_off_dev,
                            const int32_t* Z_dev, const double* pos_dev, const int32_t* periodic_host,
                            const double* lat_host, double* energy_dev, double* force_dev, double* dEdLat_dev,
                            void* stream) {
    (void)atom_off_dev;
    if (!c || nstruct <= 0 || !atom_off_host || !Z_dev || !pos_dev || !lat_host || !energy_dev || !force_dev)
        return fail(HDNNP_E_INPUT, "null argument or empty batch");
    CUDA_TRY(cudaSetDevice(c->model->device));
    // molecules need their bounding box: only periodic structures are allowed here
    for (int s = 0; s < nstruct; ++s)
        if (!periodic_host || !periodic_host[s])
            return fail(HDNNP_E_INPUT, "hdnnp_eval_batch_device: all structures must be periodic");
    int r = prepare_structs(c, nstruct, atom_off_host, nullptr, nullptr, periodic_host, lat_host, false);
    if (r) return r;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    r = run_pipeline(c, nstruct, (int)atom_off_host[nstruct], Z_dev, pos_dev, energy_dev, force_dev, dEdLat_dev, st);
    if (r) return r;
    return HDNNP_OK;
}

int hdnnp_energy_and_forces(hdnnp_ctx* c, int nat, const int32_t* Z, const double* pos, int periodic,
                            const double* lat, double* energy, double* force, double* dEdLat) {
    if (dEdLat && !periodic) return fail(HDNNP_E_INPUT, "dEdLat needs a periodic structure");
    int64_t off[2] = {0, nat};
    int32_t per = periodic ? 1 : 0;
    double dummy[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    return hdnnp_eval_batch(c, 1, off, Z, pos, &per, lat ? lat : dummy, energy, force, dEdLat);
}

// ---------------------------------------------------------------- stages
// hdnnpCalcNeighborLists (hdnnps.f90:373-388): wrap, cell lists and the
// neighbour lists of one structure, kept in the context.
int hdnnp_calc_neighbor_lists(hdnnp_ctx* c, int nat, const int32_t* Z, const double* pos, int periodic,
                              const double* lat, int* nentries) {
    if (!c || nat <= 0 || !Z || !pos) return fail(HDNNP_E_INPUT, "null argument or no atoms");
    if (periodic && !lat) return fail(HDNNP_E_INPUT, "periodic structure without a lattice");
    CUDA_TRY(cudaSetDevice(c->model->device));
    c->stage_seq = 0;
    int64_t off[2] = {0, nat};
    int32_t per = periodic ? 1 : 0;
    const double ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    int r = prepare_structs(c, 1, off, Z, pos, &per, periodic ? lat : ident, true);
    if (r) return r;
    const size_t N = nat;
    cudaStream_t st = c->stream;
    if ((r = c->Z.ensure(N)) || (r = c->pos.ensure(3 * N)) || (r = c->force.ensure(3 * N)) ||
        (r = c->energy.ensure(1)) || (r = c->dEdLat.ensure(9)))
        return r;
    CUDA_TRY(cudaMemcpyAsync(c->Z.p, Z, sizeof(int32_t) * N, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(c->pos.p, pos, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    r = run_pipeline(c, 1, nat, c->Z.p, c->pos.p, c->energy.p, c->force.p, c->dEdLat.p, st, nullptr, nullptr,
                     kStageLists);
    if (r) return r;
    CUDA_TRY(cudaStreamSynchronize(st));
    if ((r = check_status(c))) return r;
    if (nentries) *nentries = c->h_status[2];
    c->stage_seq = 1;
    c->stage_periodic = periodic ? 1 : 0;
    return HDNNP_OK;
}

// The lists of the last hdnnp_calc_neighbor_lists in the reference's
// neighborList layout (neighborLists.f90:10-16): per atom nNeis = count + 1
// entries, entry 1 the atom itself (a cell's atoms at their wrapped
// positions, a molecule's where they were given), then its neighbours
// (index, Cartesian image position in the frame of the input) in list order.
int hdnnp_neighbor_lists_fetch(hdnnp_ctx* c, int* nneis, int* ineis, double* neis) {
    if (!c || !nneis) return fail(HDNNP_E_INPUT, "null argument");
    if (c->stage_seq < 1) return fail(HDNNP_E_STATE, "no lists: call hdnnp_calc_neighbor_lists first");
    CUDA_TRY(cudaSetDevice(c->model->device));
    const Batch& b = c->last;
    const int nat = b.natoms;
    std::vector<int> cnt(nat), off(nat + 1);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    CUDA_TRY(cudaMemcpy(cnt.data(), b.nei_cnt, sizeof(int) * nat, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(off.data(), b.nei_off, sizeof(int) * (nat + 1), cudaMemcpyDeviceToHost));
    for (int i = 0; i < nat; ++i) nneis[i] = cnt[i] + 1;
    if (!ineis && !neis) return HDNNP_OK;
    const size_t E = (size_t)off[nat];
    std::vector<int> nj(E), ns(E);
    std::vector<double> w(3 * (size_t)nat);
    if (E) {
        CUDA_TRY(cudaMemcpy(nj.data(), b.nei_j, sizeof(int) * E, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(ns.data(), b.nei_s, sizeof(int) * E, cudaMemcpyDeviceToHost));
    }
    CUDA_TRY(cudaMemcpy(w.data(), b.wpos, sizeof(double) * 3 * nat, cudaMemcpyDeviceToHost));
    const StructInfo& S = c->hinfo[0];
    size_t o = 0;
    for (int i = 0; i < nat; ++i) {
        if (ineis) ineis[o] = i;
        if (neis)
            for (int d = 0; d < 3; ++d) neis[3 * o + d] = w[3 * (size_t)i + d] + S.org[d];
        ++o;
        for (int q = off[i]; q < off[i + 1]; ++q, ++o) {
            const int j = nj[q];
            if (ineis) ineis[o] = j;
            if (!neis) continue;
            int sx, sy, sz;
            unpack_shift(ns[q], sx, sy, sz);
            // image shift summed z, y, x as in the neighbour search
            double l[3] = {0.0, 0.0, 0.0};
            for (int d = 0; d < 3; ++d) {
                if (sz) l[d] += S.h[6 + d] * sz;
                if (sy) l[d] += S.h[3 + d] * sy;
                if (sx) l[d] += S.h[0 + d] * sx;
            }
            // a molecule's box origin added back (neighborLists.f90:217)
            for (int d = 0; d < 3; ++d) neis[3 * o + d] = (w[3 * (size_t)j + d] + l[d]) + S.org[d];
        }
    }
    return HDNNP_OK;
}

// hdnnpCalcSymfunctions (hdnnps.f90:390-485): the scaled symmetry-function
// values of the structure whose lists the context holds; G (host, nat x
// nsf_max, row stride nsf_max, unused columns of elements with fewer
// functions are zero) may be NULL.  Derivatives are not stored: the
// contraction recomputes them (hdnnp_calc_nns).
int hdnnp_calc_symfunctions(hdnnp_ctx* c, double* G) {
    if (!c) return fail(HDNNP_E_INPUT, "null context");
    if (c->stage_seq < 1) return fail(HDNNP_E_STATE, "hdnnp_calc_symfunctions needs hdnnp_calc_neighbor_lists first");
    CUDA_TRY(cudaSetDevice(c->model->device));
    const int nat = c->last.natoms;
    cudaStream_t st = c->stream;
    int r = run_pipeline(c, 1, nat, c->Z.p, c->pos.p, c->energy.p, c->force.p, nullptr, st, nullptr, nullptr,
                         kStageSF);
    if (r) return r;
    c->last.dEdLat = nullptr;
    const size_t n = (size_t)nat * c->model->dev.nsf_max;
    std::vector<float> tmp;
    if (G) {
        if (c->last_mixed) {
            tmp.resize(n);
            CUDA_TRY(cudaMemcpyAsync(tmp.data(), c->last.Gf, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        } else {
            CUDA_TRY(cudaMemcpyAsync(G, c->last.G, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        }
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    if ((r = check_status(c))) return r;
    if (G && c->last_mixed)
        for (size_t q = 0; q < n; ++q) G[q] = (double)tmp[q];
    c->stage_seq = 2;
    return HDNNP_OK;
}

// hdnnpCalcNNs (hdnnps.f90:487-562): the networks of `nn` (NULL: the
// context's potential) on the symmetry functions the context holds, and the
// contraction into energy, forces and (periodic structures) dE/dh.  As in the
// reference's committee (globalHdnnps.f90:47-57) the functions and their
// derivatives are those of the context's potential, and `nn` must have the
// same elements and network input widths.  May be called repeatedly.
int hdnnp_calc_nns(hdnnp_ctx* c, const hdnnp_model* nn, double* energy, double* force, double* dEdLat) {
    if (!c || !energy || !force) return fail(HDNNP_E_INPUT, "null argument");
    if (c->stage_seq < 2) return fail(HDNNP_E_STATE, "hdnnp_calc_nns needs hdnnp_calc_symfunctions first");
    if (dEdLat && !c->stage_periodic) return fail(HDNNP_E_INPUT, "dEdLat needs a periodic structure");
    const HostModel& H0 = c->model->host;
    if (nn && nn != c->model) {
        if (nn->device != c->model->device) return fail(HDNNP_E_INPUT, "the network's potential lives on another device");
        const HostModel& Hq = nn->host;
        if (Hq.el.size() != H0.el.size()) return fail(HDNNP_E_INPUT, "the network's potential has other elements");
        for (size_t e = 0; e < H0.el.size(); ++e)
            if (Hq.el[e].z != H0.el[e].z || Hq.el[e].net.empty() || Hq.el[e].net[0].nin != (int)H0.el[e].sfs.size())
                return fail(HDNNP_E_INPUT, "the network's potential: elements or network input widths differ from the "
                                           "symmetry functions of the context's potential");
        const size_t tc = mlp_smem_bytes(nn->dev, c->last_mixed ? sizeof(float) : sizeof(double));
        if (tc > 220 * 1024) return fail(HDNNP_E_CAPACITY, "network too wide for the MLP kernel");
    }
    CUDA_TRY(cudaSetDevice(c->model->device));
    const int nat = c->last.natoms;
    cudaStream_t st = c->stream;
    int r = run_pipeline(c, 1, nat, c->Z.p, c->pos.p, c->energy.p, c->force.p, dEdLat ? c->dEdLat.p : nullptr, st,
                         nullptr, nullptr, kStageNN, (nn && nn != c->model) ? &nn->dev : nullptr);
    if (r) return r;
    CUDA_TRY(cudaMemcpyAsync(energy, c->energy.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(force, c->force.p, sizeof(double) * 3 * (size_t)nat, cudaMemcpyDeviceToHost, st));
    if (dEdLat) CUDA_TRY(cudaMemcpyAsync(dEdLat, c->dEdLat.p, sizeof(double) * 9, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return check_status(c);
}

int hdnnp_committee_eval_batch(hdnnp_ctx* c, hdnnp_model* const* members, int nmembers, int nstruct,
                               const int64_t* atom_off, const int32_t* Z, const double* pos, const int32_t* periodic,
                               const double* lat, double* energy, double* force, double* dEdLat, double* std_dev) {
    if (!c || !members || nmembers < 1 || nstruct <= 0 || !atom_off || !Z || !pos || !lat || !energy || !force)
        return fail(HDNNP_E_INPUT, "null argument, empty batch or empty committee");
    if (members[0] != c->model)
        return fail(HDNNP_E_INPUT, "the context must belong to the first member (it provides the symmetry functions)");
    const HostModel& H0 = c->model->host;
    std::vector<const DevModel*> dms((size_t)nmembers);
    for (int q = 0; q < nmembers; ++q) {
        const hdnnp_model* mq = members[q];
        if (!mq) return fail(HDNNP_E_INPUT, "committee member " + std::to_string(q) + " is null");
        if (mq->device != c->model->device)
            return fail(HDNNP_E_INPUT, "committee member " + std::to_string(q) + " lives on another device");
        const HostModel& Hq = mq->host;
        if (Hq.el.size() != H0.el.size())
            return fail(HDNNP_E_INPUT, "committee member " + std::to_string(q) + " has other elements");
        for (size_t e = 0; e < H0.el.size(); ++e)
            if (Hq.el[e].z != H0.el[e].z || Hq.el[e].net.empty() || Hq.el[e].net[0].nin != (int)H0.el[e].sfs.size())
                return fail(HDNNP_E_INPUT, "committee member " + std::to_string(q) +
                                               ": elements or network input widths differ from the first member's "
                                               "symmetry functions");
        dms[q] = &mq->dev;
    }
    CUDA_TRY(cudaSetDevice(c->model->device));
    int r = prepare_structs(c, nstruct, atom_off, Z, pos, periodic, lat, true);
    if (r) return r;
    const int natoms = (int)atom_off[nstruct];
    const size_t N = natoms;
    cudaStream_t st = c->stream;
    if ((r = c->Z.ensure(N)) || (r = c->pos.ensure(3 * N)) || (r = c->force.ensure(3 * N)) ||
        (r = c->energy.ensure(nstruct)) || (r = c->dEdLat.ensure(9 * (size_t)nstruct)) ||
        (r = c->cm_std.ensure(nstruct)))
        return r;
    CUDA_TRY(cudaMemcpyAsync(c->Z.p, Z, sizeof(int32_t) * N, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(c->pos.p, pos, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    Committee cm{dms.data(), nmembers, c->cm_std.p};
    r = run_pipeline(c, nstruct, natoms, c->Z.p, c->pos.p, c->energy.p, c->force.p, dEdLat ? c->dEdLat.p : nullptr,
                     st, nullptr, &cm);
    if (r) return r;
    CUDA_TRY(cudaMemcpyAsync(energy, c->energy.p, sizeof(double) * nstruct, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(force, c->force.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, st));
    if (dEdLat) CUDA_TRY(cudaMemcpyAsync(dEdLat, c->dEdLat.p, sizeof(double) * 9 * nstruct, cudaMemcpyDeviceToHost, st));
    if (std_dev) CUDA_TRY(cudaMemcpyAsync(std_dev, c->cm_std.p, sizeof(double) * nstruct, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return check_status(c);
}

int hdnnp_committee_energy_and_forces(hdnnp_ctx* c, hdnnp_model* const* members, int nmembers, int nat,
                                      const int32_t* Z, const double* pos, int periodic, const double* lat,
                                      double* energy, double* force, double* dEdLat, double* std_dev) {
    if (dEdLat && !periodic) return fail(HDNNP_E_INPUT, "dEdLat needs a periodic structure");
    int64_t off[2] = {0, nat};
    int32_t per = periodic ? 1 : 0;
    double dummy[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    return hdnnp_committee_eval_batch(c, members, nmembers, 1, off, Z, pos, &per, lat ? lat : dummy, energy, force,
                                      dEdLat, std_dev);
}

int hdnnp_dEdLat_to_stress(const double* lat, const double* dEdLat, double* stress) {
    if (!lat || !dEdLat || !stress) return fail(HDNNP_E_INPUT, "null argument");
    double d = det3(lat);
    if (d == 0.0) return fail(HDNNP_E_INPUT, "singular lattice");
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += dEdLat[i + 3 * k] * lat[j + 3 * k];
            stress[i + 3 * j] = -1.0 / d * s;
        }
    return HDNNP_OK;
}

int hdnnp_debug_fetch(hdnnp_ctx* c, const char* what, void* host, size_t bytes) {
    if (!c || !what || !host) return fail(HDNNP_E_INPUT, "null argument");
    if (!c->have_last) return fail(HDNNP_E_STATE, "no evaluation yet");
    const Batch& b = c->last;
    const void* src = nullptr;
    size_t n = 0;
    std::string w(what);
    int tmp = 0;
    if (w == "G") { src = b.G; n = sizeof(double) * (size_t)b.natoms * c->model->dev.nsf_max; }
    else if (w == "dEdG") { src = b.dEdG; n = sizeof(double) * (size_t)b.natoms * c->model->dev.nsf_max; }
    else if (w == "atom_energy") { src = b.atE; n = sizeof(double) * b.natoms; }
    else if (w == "nei_count") { src = b.nei_cnt; n = sizeof(int) * b.natoms; }
    else if (w == "nei_offset") { src = b.nei_off; n = sizeof(int) * (b.natoms + 1); }
    else if (w == "nei_index") { src = b.nei_j; n = sizeof(int) * b.nentries; }
    else if (w == "nei_shift") { src = b.nei_s; n = sizeof(int) * b.nentries; }
    else if (w == "nei_rev") { src = b.nei_rev; n = sizeof(int) * b.nentries; }
    else if (w == "nsf_max") { tmp = c->model->dev.nsf_max; n = sizeof(int); }
    else if (w == "nentries") { tmp = b.nentries; n = sizeof(int); }
    else return fail(HDNNP_E_INPUT, "unknown item " + w);
    // list arrays: nentries is the reserved size (padded lists reserve more
    // than they fill); the leading entries the caller sized for are copied
    if (src && (src == b.nei_j || src == b.nei_s || src == b.nei_rev)) n = std::min(n, bytes);
    if (bytes < n) return fail(HDNNP_E_CAPACITY, "buffer too small");
    if (!src) {
        std::memcpy(host, &tmp, n);
        return HDNNP_OK;
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    CUDA_TRY(cudaMemcpy(host, src, n, cudaMemcpyDeviceToHost));
    return HDNNP_OK;
}

int hdnnp_ctx_set_profiling(hdnnp_ctx* c, int on) {
    if (!c) return fail(HDNNP_E_INPUT, "null context");
    c->profile = on != 0;
    return HDNNP_OK;
}

int hdnnp_profile_read(hdnnp_ctx* c, double* stage_ms, int64_t* counters, int reset) {
    if (!c) return fail(HDNNP_E_INPUT, "null context");
    CUDA_TRY(cudaSetDevice(c->model->device));
    int r = collect_profile(c);
    if (r) return r;
    unsigned long long dc[8] = {0};
    if (c->stats.p) {
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        CUDA_TRY(cudaMemcpy(dc, c->stats.p, sizeof dc, cudaMemcpyDeviceToHost));
    }
    if (stage_ms)
        for (int k = 0; k < 8; ++k) stage_ms[k] = k < 7 ? c->stage_ms[k] : 0.0;
    if (counters) {
        counters[0] = c->host_counts[0];
        counters[1] = c->host_counts[1];
        for (int k = 2; k < 8; ++k) counters[k] = (int64_t)dc[k];
    }
    if (reset) {
        for (auto& x : c->stage_ms) x = 0.0;
        c->host_counts[0] = c->host_counts[1] = 0;
        if (c->stats.p) CUDA_TRY(cudaMemset(c->stats.p, 0, 8 * sizeof(unsigned long long)));
    }
    return HDNNP_OK;
}

int hdnnp_last_launch_count(hdnnp_ctx* c, int* launches) {
    if (!c || !launches) return fail(HDNNP_E_INPUT, "null argument");
    *launches = c->launches;
    return HDNNP_OK;
}

}  // extern "C"

// ====================================================================== math check
// hdnnp_debug_math: the branch-free FP64 functions of fastmath.cuh (used by
// the symmetry-function kernels) evaluated on the device over a host array,
// so that tests can hold them against the library functions.
namespace {
__global__ void k_math_check(int which, int n, const double* x, double* y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x[i];
    double r = 0.0, ir = 0.0;
    switch (which) {
        case 0: r = exp_clamped(v); break;
        case 1: r = tanh01(v); break;
        case 2: sqrt_rsqrt(v, r, ir); break;
        default: r = rsqrt_pos(v); break;
    }
    y[i] = r;
}
}  // namespace

extern "C" int hdnnp_debug_math(int which, int n, const double* x, double* y) {
    if (which < 0 || which > 3) return fail(HDNNP_E_INPUT, "which must be 0 (exp), 1 (tanh), 2 (sqrt) or 3 (1/sqrt)");
    if (n < 0 || (n > 0 && (!x || !y))) return fail(HDNNP_E_INPUT, "null argument or negative count");
    if (n == 0) return HDNNP_OK;
    double* d = nullptr;
    const size_t bytes = sizeof(double) * (size_t)n;
    CUDA_TRY(cudaMalloc(&d, 2 * bytes));
    cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_math_check<<<(n + 255) / 256, 256>>>(which, n, d, d + n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(HDNNP_E_CUDA, std::string("hdnnp_debug_math: ") + cudaGetErrorString(e));
    return HDNNP_OK;
}

// ====================================================================== no-allocation entry point
// hdnnp_energy_and_forces_noalloc: the evaluation of hdnnp_energy_and_forces
// for callers that cannot allocate GPU memory at evaluation time, such as an
// MD or Monte Carlo host code that runs under a fixed device-memory budget
// handed out at start-up, or a language binding without access to the CUDA
// allocator.  All intermediates live in one static device array instead of a
// context workspace; inputs and outputs are the caller's host arrays, as for
// hdnnp_energy_and_forces.  It copies synchronously on the legacy default
// stream, so it must not run while any stream of the device is being captured
// in the global capture mode (those copies would end that capture).
#include <mutex>

namespace {

// Size of the static scratch.  The array is part of the library's device
// code: under lazy module loading (CUDA's default) a device reserves it when
// this entry point first runs there; with CUDA_MODULE_LOADING=EAGER every
// device the process initialises reserves it when the library is loaded.
// Either way it stays reserved until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch, looked up once per device.  In host
// code the symbol g_noalloc_scratch only names a host-side stand-in; a kernel
// must be given this address instead.
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};
std::mutex g_noalloc_mu[kNoAllocMaxDevices];

int noalloc_setup(int dev) {
    if (g_noalloc_ptr[dev]) return HDNNP_OK;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
        return fail(HDNNP_E_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (unsigned char*)p;
    return HDNNP_OK;
}

// Device error flags of a no-allocation call, mapped as for a context
// (check_status); the structure index of flag 8 is always 0 here.
int noalloc_flags(int f) {
    if (f & 1) return fail(HDNNP_E_INPUT, "atom with an element that is not in the potential");
    if (f & 2) return fail(HDNNP_E_STATE, "internal error: neighbour list is not symmetric");
    if (f & 4) return fail(HDNNP_E_CAPACITY, "neighbour count above the kernel capacity");
    if (f & 8) return fail(HDNNP_E_INPUT, "non-finite position");
    if (f & 16) return fail(HDNNP_E_TIMEOUT, "bounded wait expired");
    return HDNNP_OK;
}

// Bump carving of the static scratch (256-byte aligned regions).
struct Carve {
    unsigned char* base;
    size_t used = 0;
    bool over = false;
    template <typename T>
    T* take(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        if (used + bytes > kNoAllocScratchBytes) {
            over = true;
            return nullptr;
        }
        T* p = (T*)(base + used);
        used += bytes;
        return p;
    }
};

}  // namespace

extern "C" int hdnnp_energy_and_forces_noalloc(const hdnnp_model* m, int nat, const int32_t* Z, const double* pos,
                                               int periodic, const double* lat, double* energy, double* force,
                                               double* dEdLat) {
    if (!m || nat <= 0 || !Z || !pos || !energy || !force) return fail(HDNNP_E_INPUT, "null argument or no atoms");
    if (periodic && !lat) return fail(HDNNP_E_INPUT, "periodic structure without a lattice");
    if (dEdLat && !periodic) return fail(HDNNP_E_INPUT, "dEdLat needs a periodic structure");
    const int dev = m->device;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(HDNNP_E_INPUT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu[dev]);
    // the caller's current device is restored on every return
    int caller_dev = -1;
    CUDA_TRY(cudaGetDevice(&caller_dev));
    struct RestoreDevice {
        int d;
        ~RestoreDevice() {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{caller_dev};
    CUDA_TRY(cudaSetDevice(dev));
    int r = noalloc_setup(dev);
    if (r) return r;
    const HostModel& H = m->host;
    const DevModel& D = m->dev;
    for (int i = 0; i < nat; ++i)
        if (Z[i] < 1 || Z[i] > kMaxZ || H.z2e[Z[i]] < 0)
            return fail(HDNNP_E_INPUT, "atom " + std::to_string(i) + " has element Z=" + std::to_string(Z[i]) +
                                           " that is not in the potential");
    double ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    StructInfo S;
    r = struct_setup(nat, pos, periodic, periodic ? lat : ident, H.max_rc, S);
    if (r) return r;
    S.atom_off = 0;
    S.nat = nat;
    S.cell_off = 0;
    const int ncells = S.ngrid[0] * S.ngrid[1] * S.ngrid[2];
    const size_t N = nat;

    Carve cv{g_noalloc_ptr[dev]};
    Batch b{};
    b.nstruct = 1;
    b.natoms = nat;
    b.ncells = ncells;
    StructInfo* info = cv.take<StructInfo>(1);
    int32_t* Zd = cv.take<int32_t>(N);
    double* posd = cv.take<double>(3 * N);
    b.sid = cv.take<int>(N);
    b.elem = cv.take<int>(N);
    b.wpos = cv.take<double>(3 * N);
    b.cell_of = cv.take<int>(N);
    b.cell_cnt = cv.take<int>(ncells + 1);
    b.cell_start = cv.take<int>(ncells + 1);
    b.cell_atoms = cv.take<int>(N);
    b.nei_cnt = cv.take<int>(N + 1);
    b.nei_off = cv.take<int>(N + 1);
    b.el_count = cv.take<int>(kMaxEl + 1);
    b.el_start = cv.take<int>(kMaxEl + 1);
    b.el_atoms = cv.take<int>(N);
    b.scan_tmp = cv.take<int>(std::max<size_t>(N, ncells) / 1024 + 256);
    b.status = cv.take<int>(4);
    b.G = cv.take<double>(N * D.nsf_max);
    b.dEdG = cv.take<double>(N * D.nsf_max);
    b.atE = cv.take<double>(N);
    b.gself = cv.take<double>(3 * N);
    b.vir = cv.take<double>(9 * N);
    double* Fd = cv.take<double>(3 * N);
    double* Ed = cv.take<double>(1);
    double* Ld = cv.take<double>(9);
    if (cv.over)
        return fail(HDNNP_E_CAPACITY, "structure too large for the " + std::to_string(kNoAllocScratchBytes >> 20) +
                                          " MiB static scratch of hdnnp_energy_and_forces_noalloc (" +
                                          std::to_string(nat) + " atoms)");
    b.info = info;
    b.Z = Zd;
    b.pos = posd;
    b.force = Fd;
    b.energy = Ed;
    b.dEdLat = dEdLat ? Ld : nullptr;
    b.stats = nullptr;
    cudaStream_t st = 0;  // legacy default stream: nothing is created
    CUDA_TRY(cudaMemcpy(info, &S, sizeof S, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(Zd, Z, sizeof(int32_t) * N, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(posd, pos, sizeof(double) * 3 * N, cudaMemcpyHostToDevice));
    // the scratch keeps the previous call's contents: clear what must start at zero
    CUDA_TRY(cudaMemsetAsync(b.status, 0, 4 * sizeof(int), st));
    launch_neighbour_build_a(b, D, st);
    int h[3] = {0, 0, 0};
    CUDA_TRY(cudaMemcpy(&h[0], b.status, sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&h[1], b.nei_off + nat, sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&h[2], b.status + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if ((r = noalloc_flags(h[0]))) return r;
    if (h[1] < 0) return fail(HDNNP_E_CAPACITY, "more than 2^31 neighbour entries");
    const size_t E = (size_t)h[1];
    b.nentries = (int)E;
    b.mmax = h[2];
    b.nei_j = cv.take<int>(E + 1);
    b.nei_s = cv.take<int>(E + 1);
    b.nei_rev = cv.take<int>(E + 1);
    b.gent = cv.take<double>(3 * E + 3);
    if (cv.over)
        return fail(HDNNP_E_CAPACITY, "too many neighbour entries (" + std::to_string(E) + ") for the " +
                                          std::to_string(kNoAllocScratchBytes >> 20) +
                                          " MiB static scratch of hdnnp_energy_and_forces_noalloc");
    {
        int mm = ((b.mmax + 31) / 32) * 32;
        if (sf_smem_per_warp(mm, true) * 4 > 220 * 1024)
            return fail(HDNNP_E_CAPACITY, "too many neighbours per atom for the symmetry-function kernels");
        if (mlp_smem_bytes(D, sizeof(double)) > 220 * 1024) return fail(HDNNP_E_CAPACITY, "network too wide for the MLP kernel");
    }
    launch_neighbour_build_b(b, D, st);
    launch_element_groups(b, D, st);
    launch_sf_values(b, D, st);
    launch_mlp(b, D, st);
    launch_sf_gradients(b, D, st);
    launch_forces_and_reduce(b, D, dEdLat != nullptr, st);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpy(energy, Ed, sizeof(double), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(force, Fd, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
    if (dEdLat) CUDA_TRY(cudaMemcpy(dEdLat, Ld, sizeof(double) * 9, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(&h[0], b.status, sizeof(int), cudaMemcpyDeviceToHost));
    return noalloc_flags(h[0]);
}

// ====================================================================== internal (C++) entry points of the server
namespace hdnnp {

int model_device(const hdnnp_model* m) { return m->device; }

const DevModel& model_devmodel(const hdnnp_model* m) { return m->dev; }

int set_error(int code, const std::string& msg) { return fail(code, msg); }

// Device-resident batch (as hdnnp_eval_batch_device) in which molecules are
// allowed: mol_pos[s] is a host copy of a non-periodic structure's positions,
// read only for its bounding box (null for periodic structures).
int eval_resident(hdnnp_ctx* c, int nstruct, const int64_t* off, const int32_t* Z_dev, const double* pos_dev,
                  const double* const* mol_pos, const int32_t* periodic, const double* lat, double* energy_dev,
                  double* force_dev, double* dEdLat_dev, cudaStream_t st, PipePlan* pp, double rc_list) {
    if (!c || nstruct <= 0 || !off || !Z_dev || !pos_dev || !periodic || !lat || !energy_dev || !force_dev)
        return fail(HDNNP_E_INPUT, "null argument or empty batch");
    CUDA_TRY(cudaSetDevice(c->model->device));
    const HostModel& H = c->model->host;
    c->hinfo.resize(nstruct);
    if (off[0] != 0) return fail(HDNNP_E_INPUT, "atom_off[0] must be 0");
    for (int s = 0; s < nstruct; ++s) {
        const int64_t a0 = off[s], a1 = off[s + 1];
        if (a1 <= a0) return fail(HDNNP_E_INPUT, "structure " + std::to_string(s) + " has no atoms");
        const double* mp = periodic[s] ? nullptr : (mol_pos ? mol_pos[s] : nullptr);
        int r = struct_setup((int)(a1 - a0), mp, periodic[s], lat + 9 * s, rc_list > 0.0 ? rc_list : H.max_rc,
                             c->hinfo[s]);
        if (r) return fail(r, "structure " + std::to_string(s) + ": " + g_err);
        c->hinfo[s].atom_off = (int)a0;
        c->hinfo[s].nat = (int)(a1 - a0);
    }
    return run_pipeline(c, nstruct, (int)off[nstruct], Z_dev, pos_dev, energy_dev, force_dev, dEdLat_dev, st, pp);
}

// Neighbour-list arrays of c (device), for callers that keep lists between
// evaluations (the server's Verlet skin): after a build they hold the lists
// of the last evaluation; before an evaluation in keep mode (PipePlan with a
// rebuild flag of 0) the caller fills elem, nei_cnt, nei_j, nei_s and nei_rev
// for natoms atoms and nentries entries (nei_off follows from nei_cnt).
int ctx_list_arrays(hdnnp_ctx* c, size_t natoms, size_t nentries, CtxLists* out) {
    int r;
    if ((r = c->elem.ensure(natoms)) || (r = c->nei_cnt.ensure(natoms + 1)) || (r = c->nei_off.ensure(natoms + 1)) ||
        (r = c->nei_j.ensure(nentries + 1)) || (r = c->nei_s.ensure(nentries + 1)) ||
        (r = c->nei_rev.ensure(nentries + 1)))
        return r;
    out->elem = c->elem.p;
    out->cnt = c->nei_cnt.p;
    out->off = c->nei_off.p;
    out->nj = c->nei_j.p;
    out->ns = c->nei_s.p;
    out->rev = c->nei_rev.p;
    return HDNNP_OK;
}

// Device error flags of the last evaluation on c (valid after its stream has
// been synchronised).
int ctx_check_status(hdnnp_ctx* c) { return check_status(c); }

// Host set-up of a resident plan: periodic structures as struct_setup with
// the list cutoff; molecules get their box on the device every evaluation.
int ctx_plan_setup(hdnnp_ctx* c, int nstruct, const int64_t* off, const int32_t* periodic, const double* lat,
                   double rc_list) {
    c->hinfo.resize(nstruct);
    if (off[0] != 0) return fail(HDNNP_E_INPUT, "atom_off[0] must be 0");
    for (int s = 0; s < nstruct; ++s) {
        const int64_t a0 = off[s], a1 = off[s + 1];
        if (a1 <= a0) return fail(HDNNP_E_INPUT, "structure " + std::to_string(s) + " has no atoms");
        if (a1 > INT32_MAX) return fail(HDNNP_E_CAPACITY, "more than 2^31 atoms");
        StructInfo& S = c->hinfo[s];
        if (periodic[s]) {
            int r = struct_setup((int)(a1 - a0), nullptr, 1, lat + 9 * s, rc_list, S);
            if (r) return fail(r, "structure " + std::to_string(s) + ": " + g_err);
        } else {
            std::memset(&S, 0, sizeof S);
            S.ngrid[0] = S.ngrid[1] = S.ngrid[2] = 1;
        }
        S.atom_off = (int)a0;
        S.nat = (int)(a1 - a0);
    }
    return HDNNP_OK;
}

int ctx_run_planned(hdnnp_ctx* c, int nstruct, int natoms, const int32_t* Z_dev, const double* pos_dev,
                    double* energy_dev, double* force_dev, double* dEdLat_dev, cudaStream_t st, PipePlan& pp) {
    CUDA_TRY(cudaSetDevice(c->model->device));
    return run_pipeline(c, nstruct, natoms, Z_dev, pos_dev, energy_dev, force_dev, dEdLat_dev, st, &pp);
}

// A plan replay with profiling has finished: accumulate the stage times of
// its (last) evaluation and count `evals` evaluations of `atoms` atoms.
int ctx_profile_replay(hdnnp_ctx* c, long long evals, long long atoms) {
    if (!c->profile || !c->ev[7]) return HDNNP_OK;
    c->prof_pending = true;
    int r = collect_profile(c);
    c->host_counts[0] += evals;
    c->host_counts[1] += atoms;
    return r;
}

// Device error flags of c's evaluations ([4] ints, flags in [0]).
int* ctx_status_dev(hdnnp_ctx* c) { return c->status.p; }

// Flags of the last evaluation on c as read back to the host (after its
// stream was synchronised), and the largest neighbour count of the last
// evaluation that read its counts on the host.
int ctx_last_flags(hdnnp_ctx* c) { return c->h_status ? c->h_status[0] : 0; }
int ctx_last_mmax(hdnnp_ctx* c) { return c->h_status ? c->h_status[3] : 0; }

// Batch index of a structure with a non-finite position in the last
// evaluation on c, or -1.
int ctx_bad_struct(hdnnp_ctx* c) {
    return (c->h_status && (c->h_status[0] & 8) && c->h_status[1] > 0) ? c->h_status[1] - 1 : -1;
}

}  // namespace hdnnp

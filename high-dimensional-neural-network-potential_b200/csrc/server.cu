// server.cu -- serving form: continuous batching of energy/force/stress
// requests from many MD and Monte Carlo walkers (include/hdnnp_gpu.h,
// "serving").
//
// No reference counterpart: the reference evaluates one structure per call
// (hdnnpEnergyAndForces, src/potentials/hdnnps.f90:333) from a user-written
// MD loop (src/potentials/hdnnpExample.f90:59-72).  Here each walker's state
// lives in device memory and a request names a walker and a step kind:
//   EVAL      evaluate the current positions
//   MC_TRIAL  keep positions and forces, displace every coordinate by
//             N(0, sigma) drawn on the device, evaluate
//   MC_REJECT restore what the last trial kept (no evaluation)
//   MD_STEP   velocity Verlet (hdnnpExample.f90:61-64) with the walker's last
//             forces: drift kernel, evaluation, kick kernel
// Worker threads (one evaluation context and CUDA stream each) take pending
// requests in arrival order and pack those of idle walkers into one batch of
// at most max_batch_atoms atoms; the walkers' positions are gathered into the
// batch arrays by device copies, the batched pipeline runs, and forces go
// back into the walkers' device state.  Only energies, forces and dE/dh of
// the batch travel to the host (pinned staging, one copy each).  With two or
// more workers one batch is formed and launched while the previous one is on
// the GPU, so requests that arrive meanwhile are admitted into the next batch
// and the batches overlap on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/hdnnp_gpu.h"
#include "engine.h"
#include "integrate.cuh"

namespace hdnnp {
int model_device(const hdnnp_model* m);
int set_error(int code, const std::string& msg);
int eval_resident(hdnnp_ctx* c, int nstruct, const int64_t* off, const int32_t* Z_dev, const double* pos_dev,
                  const double* const* mol_pos, const int32_t* periodic, const double* lat, double* energy_dev,
                  double* force_dev, double* dEdLat_dev, cudaStream_t st, PipePlan* pp = nullptr,
                  double rc_list = 0.0);
int ctx_list_arrays(hdnnp_ctx* c, size_t natoms, size_t nentries, CtxLists* out);
int ctx_check_status(hdnnp_ctx* c);
int ctx_bad_struct(hdnnp_ctx* c);
int ctx_last_flags(hdnnp_ctx* c);
int ctx_last_mmax(hdnnp_ctx* c);
}  // namespace hdnnp

using namespace hdnnp;

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kThreads = 256;

inline int blocks(int n) { return (n + kThreads - 1) / kThreads; }

// ------------------------------------------------------------------ server state
struct Walker {
    int id = 0, nat = 0, periodic = 0;
    double lat[9] = {0};
    // device state; force_keep/pos_keep hold the state before the last trial,
    // force_prev the forces of the previous MD step
    double *pos = nullptr, *pos_keep = nullptr, *mom = nullptr, *mass = nullptr, *force = nullptr,
           *force_keep = nullptr, *force_prev = nullptr;
    int32_t* Z = nullptr;
    bool md = false, busy = false;
    unsigned long long steps = 0;
    size_t bytes = 0;
    // Verlet-skin list (server option skin > 0): the walker's own CSR list
    // (atom and entry indices local to the walker), the wrap translation and
    // the positions of its last build
    int *l_off = nullptr, *l_cnt = nullptr, *l_elem = nullptr, *l_j = nullptr, *l_s = nullptr, *l_rev = nullptr;
    double *l_wsh = nullptr, *l_pref = nullptr;
    int l_entries = 0, l_cap = 0, l_mmax = 0;
    bool l_valid = false;
};

// One walker of a batch for the skin-list kernels (blockIdx.y = walker).
struct WRef {
    const double* pos;  // the walker's current positions
    int *off, *cnt, *elem, *j, *s, *rev;
    double *wsh, *pref;
    int nat, a0, e0;  // atoms, first atom and first entry in the batch
};

struct Request {
    int walker = 0, kind = 0;
    double dt = 0, sigma = 0;
    unsigned long long seed = 0;
    Clock::time_point t_submit, t_done;
    bool done = false;
    int status = 0;
    std::string err;
    double energy = 0;
    double dEdLat[9] = {0};
    std::vector<double> forces;
};

struct Worker {
    hdnnp_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    // largest per-atom neighbour count seen in a batch that counted its
    // entries on the host (0: none yet); later batches that build their lists
    // search once into padded rows of 1.25 x this + 8
    int m_est = 0;
    std::thread th;
    double* pos = nullptr;  // batch arrays (device)
    int32_t* Z = nullptr;
    double *E = nullptr, *F = nullptr, *L = nullptr;
    double *hE = nullptr, *hF = nullptr, *hL = nullptr, *hpos = nullptr;  // pinned staging
    // skin lists: batch wrap translations and reference positions, rebuild
    // flags (1 and 0), per-walker flags, list offsets read back, walker tables
    double *wshift = nullptr, *pos_ref = nullptr;
    int *flag1 = nullptr, *flag0 = nullptr, *d_flags = nullptr, *h_flags = nullptr, *h_off = nullptr;
    WRef *d_ref = nullptr, *h_ref = nullptr;
};

// Device bytes per walker atom: positions, kept positions, momenta, forces,
// kept forces, previous forces (3 doubles each), mass, Z.
constexpr size_t kWalkerBytesPerAtom = 6 * 24 + 8 + 4;
// With a skin, a walker also keeps its neighbour list: charged as 80 entries
// of 12 B per atom plus the per-atom offsets, counts, elements, wrap
// translations and reference positions.
constexpr size_t kSkinBytesPerAtom = 80 * 12 + 12 + 48;
constexpr int kOne = 1;

}  // namespace

struct hdnnp_server {
    hdnnp_model* model = nullptr;
    hdnnp_server_opts opts{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_req, cv_done;
    std::deque<uint64_t> pending;
    std::deque<uint64_t> finished;  // completion order, for hdnnp_server_next_done
    std::unordered_map<uint64_t, Request> reqs;
    std::map<int, Walker> walkers;
    std::vector<Worker> workers;
    std::atomic<bool> stop{false};
    uint64_t next_ticket = 1;
    int next_walker = 0;
    size_t hbm_walkers = 0, hbm_workspace = 0;
    // statistics since the last reset
    std::vector<double> lat_ms;
    long long atoms_done = 0, batches = 0, batched_requests = 0;
    std::atomic<long long> list_builds{0}, list_reuses{0};  // walker lists built / kept (skin > 0)
    Clock::time_point t_first, t_last;
    bool have_first = false;
};

namespace {

// Worker workspace per batch atom: the context's FP64 and FP32 per-atom
// arrays (G, dE/dG, positions, forces, virials ...), about 100 neighbour
// entries (batches that build their lists in one pass reserve 1.25 x the
// densest atom + 8) of 12 B (index, shift, reverse) + 24 B (FP64 entry
// gradient) + 12 B (FP32 copy) + 8 B (padded row), the batch arrays and
// pinned staging.
size_t workspace_bytes_per_atom(const hdnnp_model* m) {
    int nel = 0, zs[128], ns[128];
    double rc = 0;
    hdnnp_model_info(m, &nel, zs, ns, &rc);
    int nsf = 0;
    for (int e = 0; e < nel; ++e) nsf = std::max(nsf, ns[e]);
    return (size_t)nsf * 24 + 100 * 56 + 400;
}

// Records a completion for hdnnp_server_next_done (server lock held).  Tickets
// already consumed by hdnnp_server_wait are dropped from the front so the
// queue stays short when next_done is not used.
void note_finished(hdnnp_server* s, uint64_t t) {
    s->finished.push_back(t);
    while (s->finished.size() > 4096 && !s->reqs.count(s->finished.front())) s->finished.pop_front();
}

void fail_batch(hdnnp_server* s, const std::vector<uint64_t>& batch, std::vector<Request*>& rq,
                std::vector<Walker*>& ws, int status, const std::string& err) {
    const auto now = Clock::now();
    std::lock_guard<std::mutex> g(s->mu);
    for (size_t k = 0; k < rq.size(); ++k) {
        rq[k]->status = status;
        rq[k]->err = err;
        rq[k]->done = true;
        rq[k]->t_done = now;
        ws[k]->busy = false;
        note_finished(s, batch[k]);
    }
    s->cv_done.notify_all();
    s->cv_req.notify_all();
}

// ------------------------------------------------------------ skin lists
// flags[q] = 1 if an atom of walker q moved by more than sqrt(thr2) since its
// list was built (or is not finite)
__global__ void k_walker_moved(const WRef* t, double thr2, int* flags) {
    const WRef w = t[blockIdx.y];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.nat) return;
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double x = w.pos[3 * i + d] - w.pref[3 * i + d];
        d2 += x * x;
    }
    if (!(d2 <= thr2)) atomicOr(&flags[blockIdx.y], 1);
}

// The batch's lists of walker q (just built) into the walker's storage,
// indices made local.
__global__ void k_lists_out(const WRef* t, CtxLists L, const double* wsh, const double* pref) {
    const WRef w = t[blockIdx.y];
    const int la = blockIdx.x * blockDim.x + threadIdx.x;
    if (la >= w.nat) return;
    const int a = w.a0 + la;
    w.cnt[la] = L.cnt[a];
    w.elem[la] = L.elem[a];
    w.off[la] = L.off[a] - w.e0;
    if (la == w.nat - 1) w.off[w.nat] = L.off[a + 1] - w.e0;
    for (int d = 0; d < 3; ++d) {
        w.wsh[3 * la + d] = wsh[3 * a + d];
        w.pref[3 * la + d] = pref[3 * a + d];
    }
    for (int e = L.off[a]; e < L.off[a + 1]; ++e) {
        const int le = e - w.e0;
        w.j[le] = L.nj[e] - w.a0;
        w.s[le] = L.ns[e];
        w.rev[le] = L.rev[e] - w.e0;
    }
}

// Walker q's kept list into the batch arrays at its atom and entry offsets.
__global__ void k_lists_in(const WRef* t, CtxLists L, double* wsh, double* pref) {
    const WRef w = t[blockIdx.y];
    const int la = blockIdx.x * blockDim.x + threadIdx.x;
    if (la >= w.nat) return;
    const int a = w.a0 + la;
    L.cnt[a] = w.cnt[la];
    L.elem[a] = w.elem[la];
    for (int d = 0; d < 3; ++d) {
        wsh[3 * a + d] = w.wsh[3 * la + d];
        pref[3 * a + d] = w.pref[3 * la + d];
    }
    for (int le = w.off[la]; le < w.off[la + 1]; ++le) {
        const int e = w.e0 + le;
        L.nj[e] = w.j[le] + w.a0;
        L.ns[e] = w.s[le];
        L.rev[e] = w.rev[le] + w.e0;
    }
}

dim3 walker_grid(const std::vector<std::pair<Request*, Walker*>>& items) {
    int nmax = 1;
    for (auto& it : items) nmax = std::max(nmax, it.second->nat);
    return dim3((unsigned)blocks(nmax), (unsigned)items.size());
}

enum class ListMode { Build, BuildKeep, Keep };

// Evaluates the walkers of `items` (pre-step kernels already queued) as one
// batch on the worker's stream: gather into the batch arrays, batched
// pipeline, post-step (MD kick or force copy into the walker), results into
// the requests.  Returns the batch status (message in `err`).  With a skin,
// BuildKeep builds lists with cutoff rc + skin and keeps them in the walkers,
// Keep evaluates on the walkers' kept lists.
int evaluate_set(hdnnp_server* srv, Worker& w, const std::vector<std::pair<Request*, Walker*>>& items, std::string& err,
                 ListMode mode, int ab, int sb) {
    // this part's walker table: entries sb.. (the other part's copy may be in flight)
    cudaStream_t st = w.stream;
    double* bpos = w.pos + 3 * (size_t)ab;
    int32_t* bZ = w.Z + ab;
    double* bhpos = w.hpos + 3 * (size_t)ab;
    const size_t n = items.size();
    std::vector<int64_t> off(n + 1, 0);
    std::vector<int32_t> per(n);
    std::vector<double> lat(9 * n);
    std::vector<const double*> mol(n, nullptr);
    bool have_mol = false;
    for (size_t q = 0; q < n; ++q) {
        const Walker& wk = *items[q].second;
        off[q + 1] = off[q] + wk.nat;
        per[q] = wk.periodic;
        std::memcpy(&lat[9 * q], wk.lat, sizeof wk.lat);
        cudaMemcpyAsync(bpos + 3 * off[q], wk.pos, 24 * (size_t)wk.nat, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(bZ + off[q], wk.Z, 4 * (size_t)wk.nat, cudaMemcpyDeviceToDevice, st);
        if (!wk.periodic) {
            // a molecule's cell grid spans its bounding box: its positions come to the host
            cudaMemcpyAsync(bhpos + 3 * off[q], wk.pos, 24 * (size_t)wk.nat, cudaMemcpyDeviceToHost, st);
            mol[q] = bhpos + 3 * off[q];
            have_mol = true;
        }
    }
    cudaError_t ce = have_mol ? cudaStreamSynchronize(st) : cudaSuccess;
    if (ce != cudaSuccess) {
        err = cudaGetErrorString(ce);
        return HDNNP_E_CUDA;
    }
    const double skin = srv->opts.skin;
    double rc_list = 0.0;
    PipePlan pp{};
    PipePlan* ppp = nullptr;
    if (mode != ListMode::Build) {
        int nel = 0, zs[128], ns[128];
        double max_rc = 0;
        hdnnp_model_info(srv->model, &nel, zs, ns, &max_rc);
        rc_list = max_rc + skin;
        pp.rc_list = rc_list;
        pp.wshift = w.wshift;
        pp.pos_ref = w.pos_ref;
        ppp = &pp;
    }
    // lists built without a skin: one search pass into padded rows sized by
    // the densest batch so far, no host read of the entry total
    const int pad_cap = w.m_est > 0 ? ((int)std::ceil(1.25 * w.m_est) + 8 + 31) / 32 * 32 : 0;
    const bool padded = mode == ListMode::Build && pad_cap > 0 && (double)off[n] * pad_cap < (double)INT32_MAX;
    if (padded) {
        pp.pad_lists = true;
        pp.m_cap = pad_cap;
        pp.e_cap = (long long)off[n] * pad_cap;
        ppp = &pp;
    }
    if (mode == ListMode::BuildKeep) {
        pp.rebuild = w.flag1;  // build, recording the wrap translations and reference positions
    } else if (mode == ListMode::Keep) {
        // the walkers' lists into the batch arrays
        long long ent = 0;
        int mmax = 0;
        for (size_t q = 0; q < n; ++q) {
            const Walker& wk = *items[q].second;
            w.h_ref[sb + q] = WRef{nullptr, wk.l_off, wk.l_cnt, wk.l_elem, wk.l_j, wk.l_s, wk.l_rev, wk.l_wsh, wk.l_pref,
                              wk.nat, (int)off[q], (int)ent};
            ent += wk.l_entries;
            mmax = std::max(mmax, wk.l_mmax);
        }
        if (ent > INT32_MAX) return set_error(HDNNP_E_CAPACITY, "more than 2^31 neighbour entries in a batch");
        CtxLists L{};
        int r = ctx_list_arrays(w.ctx, (size_t)off[n], (size_t)ent, &L);
        if (r) {
            err = hdnnp_last_error();
            return r;
        }
        cudaMemcpyAsync(w.d_ref + sb, w.h_ref + sb, sizeof(WRef) * n, cudaMemcpyHostToDevice, st);
        k_lists_in<<<walker_grid(items), kThreads, 0, st>>>(w.d_ref + sb, L, w.wshift, w.pos_ref);
        pp.rebuild = w.flag0;
        pp.e_cap = ent;
        pp.m_cap = std::max(32, (mmax + 31) / 32 * 32);
    }
    int status = eval_resident(w.ctx, (int)n, off.data(), bZ, bpos, mol.data(), per.data(), lat.data(), w.E + sb,
                               w.F + 3 * (size_t)ab, w.L + 9 * (size_t)sb, st, ppp, rc_list);
    if (status) {
        err = hdnnp_last_error();
        cudaStreamSynchronize(st);
        return status;
    }
    ce = cudaStreamSynchronize(st);  // the device error flags of this batch
    if (ce != cudaSuccess) {
        err = cudaGetErrorString(ce);
        return HDNNP_E_CUDA;
    }
    if ((status = ctx_check_status(w.ctx))) {
        err = hdnnp_last_error();
        return status;
    }
    if (padded && (ctx_last_flags(w.ctx) & 32)) {
        // an atom with more neighbours than the padded rows hold: this batch
        // again with its counts read on the host (results are not yet used)
        w.m_est = 0;
        return evaluate_set(srv, w, items, err, mode, ab, sb);
    }
    if (mode == ListMode::Build && !padded) w.m_est = std::max(w.m_est, ctx_last_mmax(w.ctx));
    if (mode == ListMode::BuildKeep) {
        // keep each walker's new list: offsets to the host, storage, copy-out
        CtxLists L{};
        int r = ctx_list_arrays(w.ctx, (size_t)off[n], 0, &L);
        if (r) {
            err = hdnnp_last_error();
            return r;
        }
        cudaMemcpyAsync(w.h_off, L.off, sizeof(int) * (size_t)(off[n] + 1), cudaMemcpyDeviceToHost, st);
        if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) {
            err = cudaGetErrorString(ce);
            return HDNNP_E_CUDA;
        }
        for (size_t q = 0; q < n; ++q) {
            Walker& wk = *items[q].second;
            const int e0 = w.h_off[off[q]], e1 = w.h_off[off[q + 1]];
            int mmax = 0;
            for (int64_t a = off[q]; a < off[q + 1]; ++a) mmax = std::max(mmax, w.h_off[a + 1] - w.h_off[a]);
            const int ne = e1 - e0;
            const size_t n3 = 3 * (size_t)wk.nat;
            bool ok = true;
            if (!wk.l_off)
                ok = cudaMalloc(&wk.l_off, 4 * ((size_t)wk.nat + 1)) == cudaSuccess &&
                     cudaMalloc(&wk.l_cnt, 4 * (size_t)wk.nat) == cudaSuccess &&
                     cudaMalloc(&wk.l_elem, 4 * (size_t)wk.nat) == cudaSuccess &&
                     cudaMalloc(&wk.l_wsh, 8 * n3) == cudaSuccess && cudaMalloc(&wk.l_pref, 8 * n3) == cudaSuccess;
            if (ok && ne > wk.l_cap) {
                for (int* p : {wk.l_j, wk.l_s, wk.l_rev})
                    if (p) cudaFree(p);
                wk.l_j = wk.l_s = wk.l_rev = nullptr;
                wk.l_cap = ne + ne / 4 + 64;
                ok = cudaMalloc(&wk.l_j, 4 * (size_t)wk.l_cap) == cudaSuccess &&
                     cudaMalloc(&wk.l_s, 4 * (size_t)wk.l_cap) == cudaSuccess &&
                     cudaMalloc(&wk.l_rev, 4 * (size_t)wk.l_cap) == cudaSuccess;
            }
            if (!ok) {
                err = "skin-list storage could not be allocated";
                return HDNNP_E_CUDA;
            }
            wk.l_entries = ne;
            wk.l_mmax = mmax;
            w.h_ref[sb + q] = WRef{nullptr, wk.l_off, wk.l_cnt, wk.l_elem, wk.l_j, wk.l_s, wk.l_rev, wk.l_wsh, wk.l_pref,
                              wk.nat, (int)off[q], e0};
        }
        cudaMemcpyAsync(w.d_ref + sb, w.h_ref + sb, sizeof(WRef) * n, cudaMemcpyHostToDevice, st);
        k_lists_out<<<walker_grid(items), kThreads, 0, st>>>(w.d_ref + sb, L, w.wshift, w.pos_ref);
        for (auto& it : items) it.second->l_valid = true;
        srv->list_builds += (long long)n;
    } else if (mode == ListMode::Keep) {
        srv->list_reuses += (long long)n;
    }
    return HDNNP_OK;
}

// Post-steps (MD kick or force copy into the walker) and results of the
// walkers of `items`, evaluated from atom ab and structure sb of the batch
// buffers; the whole batch's results come to the host at once.
int finish_batch(Worker& w, const std::vector<std::pair<Request*, Walker*>>& items, std::string& err) {
    cudaStream_t st = w.stream;
    const size_t n = items.size();
    std::vector<int64_t> off(n + 1, 0);
    for (size_t q = 0; q < n; ++q) off[q + 1] = off[q] + items[q].second->nat;
    for (size_t q = 0; q < n; ++q) {
        const Request& r = *items[q].first;
        Walker& wk = *items[q].second;
        const int n3 = 3 * wk.nat;
        if (r.kind == HDNNP_REQ_MD_STEP)
            k_md_kick<<<blocks(n3), kThreads, 0, st>>>(wk.mom, w.F + 3 * off[q], wk.force_prev, wk.force, n3, r.dt);
        else
            cudaMemcpyAsync(wk.force, w.F + 3 * off[q], 24 * (size_t)wk.nat, cudaMemcpyDeviceToDevice, st);
    }
    cudaMemcpyAsync(w.hE, w.E, 8 * n, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(w.hF, w.F, 24 * (size_t)off[n], cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(w.hL, w.L, 72 * n, cudaMemcpyDeviceToHost, st);
    cudaError_t ce;
    if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) {
        err = cudaGetErrorString(ce);
        return HDNNP_E_CUDA;
    }
    for (size_t q = 0; q < n; ++q) {
        Request& r = *items[q].first;
        r.energy = w.hE[q];
        r.forces.assign(w.hF + 3 * off[q], w.hF + 3 * off[q + 1]);
        std::memcpy(r.dEdLat, w.hL + 9 * q, sizeof r.dEdLat);
    }
    return HDNNP_OK;
}

// Without a skin: one batch.  With a skin: walkers whose atoms all stayed
// within skin/2 of their list's reference positions are evaluated on their
// kept lists, the others (and walkers without a list) build new ones -- two
// pipeline runs at most, each batched over its walkers, into separate parts
// of the batch buffers; post-steps only once both have succeeded.  On
// failure *bad names the item whose input the device flags blame, or -1.
int evaluate(hdnnp_server* srv, Worker& w, const std::vector<std::pair<Request*, Walker*>>& items, std::string& err,
             int* bad) {
    *bad = -1;
    using Items = std::vector<std::pair<Request*, Walker*>>;
    auto blame = [&](const Items& part) {
        const int k = ctx_bad_struct(w.ctx);
        if (k >= 0 && k < (int)part.size())
            for (size_t q = 0; q < items.size(); ++q)
                if (items[q].second == part[k].second) *bad = (int)q;
    };
    int r;
    if (!(srv->opts.skin > 0.0) || items.size() > 65535) {
        // (the skin-list kernels index walkers by grid y, at most 65535)
        if ((r = evaluate_set(srv, w, items, err, ListMode::Build, 0, 0))) {
            blame(items);
            return r;
        }
        return finish_batch(w, items, err);
    }
    cudaStream_t st = w.stream;
    Items keep, build, cand;
    for (auto& it : items) (it.second->l_valid ? cand : build).push_back(it);
    if (!cand.empty()) {
        for (size_t q = 0; q < cand.size(); ++q) {
            const Walker& wk = *cand[q].second;
            w.h_ref[q] = WRef{wk.pos, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, wk.l_pref,
                              wk.nat, 0, 0};
        }
        cudaMemcpyAsync(w.d_ref, w.h_ref, sizeof(WRef) * cand.size(), cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(w.d_flags, 0, sizeof(int) * cand.size(), st);
        const double half = 0.5 * srv->opts.skin;
        k_walker_moved<<<walker_grid(cand), kThreads, 0, st>>>(w.d_ref, half * half, w.d_flags);
        cudaMemcpyAsync(w.h_flags, w.d_flags, sizeof(int) * cand.size(), cudaMemcpyDeviceToHost, st);
        const cudaError_t ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) {
            err = cudaGetErrorString(ce);
            return HDNNP_E_CUDA;
        }
        for (size_t q = 0; q < cand.size(); ++q) (w.h_flags[q] ? build : keep).push_back(cand[q]);
    }
    int nb_atoms = 0;
    for (auto& it : build) nb_atoms += it.second->nat;
    if (!build.empty() && (r = evaluate_set(srv, w, build, err, ListMode::BuildKeep, 0, 0))) {
        blame(build);
        return r;
    }
    if (!keep.empty() && (r = evaluate_set(srv, w, keep, err, ListMode::Keep, nb_atoms, (int)build.size()))) {
        blame(keep);
        return r;
    }
    Items all(build);
    all.insert(all.end(), keep.begin(), keep.end());
    return finish_batch(w, all, err);
}

void process_batch(hdnnp_server* s, Worker& w, const std::vector<uint64_t>& batch) {
    std::vector<Walker*> ws;
    std::vector<Request*> rq;
    {
        // element references stay valid across inserts into the containers;
        // busy walkers and unfinished requests are never erased
        std::lock_guard<std::mutex> g(s->mu);
        for (auto t : batch) {
            Request& r = s->reqs.at(t);
            rq.push_back(&r);
            ws.push_back(&s->walkers.at(r.walker));
        }
    }
    cudaStream_t st = w.stream;
    // per-walker steps before the evaluation
    std::vector<std::pair<Request*, Walker*>> ev;
    for (size_t k = 0; k < rq.size(); ++k) {
        Request& r = *rq[k];
        Walker& wk = *ws[k];
        const int n3 = 3 * wk.nat;
        r.status = HDNNP_OK;
        if (r.kind == HDNNP_REQ_MC_TRIAL) {
            const unsigned long long key = mix64(r.seed ^ mix64(wk.steps + 0x2545F4914F6CDD1Dull));
            k_mc_trial<<<blocks(n3), kThreads, 0, st>>>(wk.pos, wk.pos_keep, wk.force, wk.force_keep, n3, r.sigma,
                                                        key);
        } else if (r.kind == HDNNP_REQ_MC_REJECT) {
            k_mc_reject<<<blocks(n3), kThreads, 0, st>>>(wk.pos, wk.pos_keep, wk.force, wk.force_keep, n3);
            continue;
        } else if (r.kind == HDNNP_REQ_MD_STEP) {
            k_md_drift<<<blocks(n3), kThreads, 0, st>>>(wk.pos, wk.mom, wk.mass, wk.force, wk.force_prev, n3, r.dt);
        }
        ev.emplace_back(&r, &wk);
    }
    std::string err;
    int status = HDNNP_OK;
    if (!ev.empty()) {
        // A walker whose own input fails (a position that its trajectory
        // made non-finite, a walker too dense for the kernels) fails alone:
        // the walker named by the device flags leaves the batch and the rest
        // is evaluated again; without a name each walker is evaluated alone.
        while (!ev.empty()) {
            int bad = -1;
            status = evaluate(s, w, ev, err, &bad);
            if (status != HDNNP_E_INPUT && status != HDNNP_E_CAPACITY) break;
            if (ev.size() == 1) {
                ev[0].first->status = status;
                ev[0].first->err = err;
                status = HDNNP_OK;
                break;
            }
            if (bad >= 0 && bad < (int)ev.size()) {
                ev[bad].first->status = status;
                ev[bad].first->err = err;
                ev.erase(ev.begin() + bad);
                continue;
            }
            status = HDNNP_OK;
            for (auto& it : ev) {
                std::string e1;
                int b1 = -1;
                it.first->status = evaluate(s, w, {it}, e1, &b1);
                it.first->err = e1;
                if (it.first->status == HDNNP_E_CUDA) {
                    status = HDNNP_E_CUDA;
                    err = e1;
                    break;
                }
            }
            break;
        }
    } else {
        cudaError_t ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) {
            status = HDNNP_E_CUDA;
            err = cudaGetErrorString(ce);
        }
    }
    if (status) {
        fail_batch(s, batch, rq, ws, status, err);
        return;
    }
    const auto now = Clock::now();
    std::lock_guard<std::mutex> g(s->mu);
    for (size_t k = 0; k < rq.size(); ++k) {
        Request& r = *rq[k];
        Walker& wk = *ws[k];
        if (r.kind != HDNNP_REQ_MC_REJECT && r.status == HDNNP_OK) s->atoms_done += wk.nat;
        wk.steps += 1;
        wk.busy = false;
        r.done = true;
        r.t_done = now;
        note_finished(s, batch[k]);
        s->lat_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count());
    }
    s->t_last = now;
    s->batches += 1;
    s->batched_requests += (long long)rq.size();
    s->cv_done.notify_all();
    s->cv_req.notify_all();  // walkers became idle: their next requests can be batched
}

// Batch formation under the server lock: requests in arrival order; a request
// whose walker is busy is skipped (it keeps its place); the first request of
// an idle walker that does not fit ends the batch, so later small requests
// never overtake it indefinitely.
void take_batch(hdnnp_server* s, std::vector<uint64_t>& batch) {
    long long atoms = 0;
    const long long cap = s->opts.max_batch_atoms;
    for (auto it = s->pending.begin(); it != s->pending.end();) {
        Request& r = s->reqs.at(*it);
        Walker& wk = s->walkers.at(r.walker);
        if (wk.busy) {
            ++it;
            continue;
        }
        const long long need = (r.kind == HDNNP_REQ_MC_REJECT) ? 0 : wk.nat;
        if (atoms + need > cap) break;
        wk.busy = true;
        atoms += need;
        batch.push_back(*it);
        it = s->pending.erase(it);
        if (atoms == cap) break;
    }
}

void worker_loop(hdnnp_server* s, Worker* w) {
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<uint64_t> batch;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->stop.load()) return;
                take_batch(s, batch);
                if (!batch.empty()) break;
                s->cv_req.wait_for(lk, std::chrono::milliseconds(100));
            }
        }
        process_batch(s, *w, batch);
    }
}

void free_walker(Walker& w) {
    for (void* p : {(void*)w.pos, (void*)w.pos_keep, (void*)w.mom, (void*)w.mass, (void*)w.force,
                    (void*)w.force_keep, (void*)w.force_prev, (void*)w.Z, (void*)w.l_off, (void*)w.l_cnt,
                    (void*)w.l_elem, (void*)w.l_j, (void*)w.l_s, (void*)w.l_rev, (void*)w.l_wsh, (void*)w.l_pref})
        if (p) cudaFree(p);
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

int hdnnp_server_create(hdnnp_model* m, const hdnnp_server_opts* opts, hdnnp_server** out) {
    if (!m || !opts || !out) return set_error(HDNNP_E_INPUT, "null argument");
    if (opts->workers < 1 || opts->workers > 8) return set_error(HDNNP_E_INPUT, "workers must be 1..8");
    if (opts->max_batch_atoms < 1) return set_error(HDNNP_E_INPUT, "max_batch_atoms must be positive");
    if (opts->precision != HDNNP_PREC_FP64 && opts->precision != HDNNP_PREC_MIXED)
        return set_error(HDNNP_E_INPUT, "unknown precision");
    if (!(opts->skin >= 0.0) || !std::isfinite(opts->skin)) return set_error(HDNNP_E_INPUT, "skin must be finite and >= 0");
    const size_t ws = (size_t)opts->workers * opts->max_batch_atoms * workspace_bytes_per_atom(m);
    if (opts->hbm_budget && ws > opts->hbm_budget)
        return set_error(HDNNP_E_CAPACITY, "HBM budget (" + std::to_string(opts->hbm_budget) +
                                               " B) below the workers' workspace (" + std::to_string(ws) + " B)");
    auto* s = new hdnnp_server();
    s->model = m;
    s->opts = *opts;
    s->device = model_device(m);
    s->hbm_workspace = ws;
    if (cudaSetDevice(s->device) != cudaSuccess) {
        delete s;
        return set_error(HDNNP_E_CUDA, "cudaSetDevice failed");
    }
    s->workers.resize(opts->workers);
    const size_t na = opts->max_batch_atoms;
    for (auto& w : s->workers) {
        int r = hdnnp_ctx_create(m, &w.ctx);
        if (!r) r = hdnnp_ctx_set_precision(w.ctx, opts->precision);
        const bool ok = !r && cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) == cudaSuccess &&
                        cudaMalloc(&w.pos, na * 24) == cudaSuccess && cudaMalloc(&w.Z, na * 4) == cudaSuccess &&
                        cudaMalloc(&w.E, na * 8) == cudaSuccess && cudaMalloc(&w.F, na * 24) == cudaSuccess &&
                        cudaMalloc(&w.L, na * 72) == cudaSuccess && cudaMallocHost(&w.hE, na * 8) == cudaSuccess &&
                        cudaMallocHost(&w.hF, na * 24) == cudaSuccess &&
                        cudaMallocHost(&w.hL, na * 72) == cudaSuccess &&
                        cudaMallocHost(&w.hpos, na * 24) == cudaSuccess;
        const bool ok2 = !ok || !(opts->skin > 0.0) ||
                         (cudaMalloc(&w.wshift, na * 24) == cudaSuccess && cudaMalloc(&w.pos_ref, na * 24) == cudaSuccess &&
                          cudaMalloc(&w.flag1, 4) == cudaSuccess && cudaMalloc(&w.flag0, 4) == cudaSuccess &&
                          cudaMemcpy(w.flag1, &kOne, 4, cudaMemcpyHostToDevice) == cudaSuccess &&
                          cudaMemset(w.flag0, 0, 4) == cudaSuccess &&
                          cudaMalloc(&w.d_flags, 4 * na) == cudaSuccess &&
                          cudaMallocHost(&w.h_flags, 4 * na) == cudaSuccess &&
                          cudaMallocHost(&w.h_off, 4 * (na + 1)) == cudaSuccess &&
                          cudaMalloc(&w.d_ref, sizeof(WRef) * na) == cudaSuccess &&
                          cudaMallocHost(&w.h_ref, sizeof(WRef) * na) == cudaSuccess);
        if (!ok || !ok2) {
            std::string msg = r ? std::string(hdnnp_last_error()) : "server buffers could not be allocated";
            hdnnp_server_destroy(s);
            return set_error(r ? r : HDNNP_E_CUDA, msg);
        }
    }
    for (auto& w : s->workers) w.th = std::thread(worker_loop, s, &w);
    *out = s;
    return HDNNP_OK;
}

void hdnnp_server_destroy(hdnnp_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop.store(true);
    }
    s->cv_req.notify_all();
    for (auto& w : s->workers)
        if (w.th.joinable()) w.th.join();
    cudaSetDevice(s->device);
    for (auto& w : s->workers) {
        if (w.stream) cudaStreamSynchronize(w.stream);
        for (void* p : {(void*)w.pos, (void*)w.Z, (void*)w.E, (void*)w.F, (void*)w.L, (void*)w.wshift,
                        (void*)w.pos_ref, (void*)w.flag1, (void*)w.flag0, (void*)w.d_flags, (void*)w.d_ref})
            if (p) cudaFree(p);
        for (void* p : {(void*)w.hE, (void*)w.hF, (void*)w.hL, (void*)w.hpos, (void*)w.h_flags, (void*)w.h_off,
                        (void*)w.h_ref})
            if (p) cudaFreeHost(p);
        if (w.stream) cudaStreamDestroy(w.stream);
        if (w.ctx) hdnnp_ctx_free(w.ctx);
    }
    for (auto& kv : s->walkers) free_walker(kv.second);
    delete s;
}

int hdnnp_server_add_walker(hdnnp_server* s, int nat, const int32_t* Z, const double* pos, int periodic,
                            const double* lat, const double* masses, const double* momenta, int* walker) {
    if (!s || nat <= 0 || !Z || !pos || !walker || (periodic && !lat))
        return set_error(HDNNP_E_INPUT, "null argument or no atoms");
    if (nat > s->opts.max_batch_atoms)
        return set_error(HDNNP_E_CAPACITY, "walker of " + std::to_string(nat) + " atoms above max_batch_atoms");
    int nel = 0, zs[128], ns[128];
    double rc = 0;
    hdnnp_model_info(s->model, &nel, zs, ns, &rc);
    for (int i = 0; i < nat; ++i)
        if (std::find(zs, zs + nel, Z[i]) == zs + nel)
            return set_error(HDNNP_E_INPUT, "atom " + std::to_string(i) + " has element Z=" + std::to_string(Z[i]) +
                                                " that is not in the potential");
    for (int i = 0; i < 3 * nat; ++i)
        if (!std::isfinite(pos[i])) return set_error(HDNNP_E_INPUT, "non-finite position");
    if (masses)
        for (int i = 0; i < nat; ++i)
            if (!(masses[i] > 0)) return set_error(HDNNP_E_INPUT, "masses must be positive");
    const size_t bytes = (size_t)nat * (kWalkerBytesPerAtom + (s->opts.skin > 0.0 ? kSkinBytesPerAtom : 0));
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->opts.hbm_budget && s->hbm_walkers + bytes + s->hbm_workspace > s->opts.hbm_budget)
            return set_error(HDNNP_E_CAPACITY, "HBM budget exhausted: walker of " + std::to_string(bytes) +
                                                   " B not admitted");
        s->hbm_walkers += bytes;  // charged before allocating
    }
    cudaSetDevice(s->device);
    Walker w;
    w.nat = nat;
    w.periodic = periodic ? 1 : 0;
    if (periodic) std::memcpy(w.lat, lat, sizeof w.lat);
    w.md = masses != nullptr;
    w.bytes = bytes;
    const size_t n3 = 3 * (size_t)nat;
    bool ok = cudaMalloc(&w.pos, n3 * 8) == cudaSuccess && cudaMalloc(&w.pos_keep, n3 * 8) == cudaSuccess &&
              cudaMalloc(&w.mom, n3 * 8) == cudaSuccess && cudaMalloc(&w.mass, (size_t)nat * 8) == cudaSuccess &&
              cudaMalloc(&w.force, n3 * 8) == cudaSuccess && cudaMalloc(&w.force_keep, n3 * 8) == cudaSuccess &&
              cudaMalloc(&w.force_prev, n3 * 8) == cudaSuccess && cudaMalloc(&w.Z, (size_t)nat * 4) == cudaSuccess;
    if (ok) {
        std::vector<double> zero(n3, 0.0), one((size_t)nat, 1.0);
        ok = cudaMemcpy(w.pos, pos, n3 * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(w.pos_keep, pos, n3 * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(w.mom, momenta ? momenta : zero.data(), n3 * 8, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(w.mass, masses ? masses : one.data(), (size_t)nat * 8, cudaMemcpyHostToDevice) ==
                 cudaSuccess &&
             cudaMemset(w.force, 0, n3 * 8) == cudaSuccess && cudaMemset(w.force_keep, 0, n3 * 8) == cudaSuccess &&
             cudaMemset(w.force_prev, 0, n3 * 8) == cudaSuccess &&
             cudaMemcpy(w.Z, Z, (size_t)nat * 4, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (!ok) {
        free_walker(w);
        s->hbm_walkers -= bytes;
        return set_error(HDNNP_E_CUDA, "walker buffers could not be allocated");
    }
    w.id = s->next_walker++;
    *walker = w.id;
    s->walkers.emplace(w.id, w);
    return HDNNP_OK;
}

int hdnnp_server_remove_walker(hdnnp_server* s, int walker) {
    if (!s) return set_error(HDNNP_E_INPUT, "null server");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->walkers.find(walker);
    if (it == s->walkers.end()) return set_error(HDNNP_E_INPUT, "unknown walker");
    if (it->second.busy) return set_error(HDNNP_E_STATE, "walker has a request in flight");
    for (auto t : s->pending)
        if (s->reqs.at(t).walker == walker) return set_error(HDNNP_E_STATE, "walker has pending requests");
    cudaSetDevice(s->device);
    free_walker(it->second);
    s->hbm_walkers -= it->second.bytes;
    s->walkers.erase(it);
    return HDNNP_OK;
}

int hdnnp_server_submit(hdnnp_server* s, int walker, int kind, double dt, double sigma, uint64_t seed,
                        uint64_t* ticket) {
    if (!s || !ticket) return set_error(HDNNP_E_INPUT, "null argument");
    if (kind < HDNNP_REQ_EVAL || kind > HDNNP_REQ_MD_STEP) return set_error(HDNNP_E_INPUT, "unknown request kind");
    if (!std::isfinite(dt) || !std::isfinite(sigma) || sigma < 0)
        return set_error(HDNNP_E_INPUT, "dt and sigma must be finite, sigma >= 0");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->walkers.find(walker);
    if (it == s->walkers.end()) return set_error(HDNNP_E_INPUT, "unknown walker");
    if (kind == HDNNP_REQ_MD_STEP && !it->second.md) return set_error(HDNNP_E_INPUT, "MD step on a walker without masses");
    Request r;
    r.walker = walker;
    r.kind = kind;
    r.dt = dt;
    r.sigma = sigma;
    r.seed = seed;
    r.t_submit = Clock::now();
    if (!s->have_first) {
        s->t_first = r.t_submit;
        s->t_last = r.t_submit;
        s->have_first = true;
    }
    const uint64_t t = s->next_ticket++;
    s->reqs.emplace(t, std::move(r));
    s->pending.push_back(t);
    *ticket = t;
    s->cv_req.notify_one();
    return HDNNP_OK;
}

int hdnnp_server_wait(hdnnp_server* s, uint64_t ticket, int timeout_ms, double* energy, double* forces,
                      double* dEdLat, double* latency_ms) {
    if (!s) return set_error(HDNNP_E_INPUT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_error(HDNNP_E_INPUT, "unknown ticket");
    Request* r = &it->second;
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(std::max(timeout_ms, 0)), [&] { return r->done; }))
        return set_error(HDNNP_E_TIMEOUT, "request not finished within the timeout");
    Request done = std::move(*r);
    s->reqs.erase(ticket);
    lk.unlock();
    if (done.status) return set_error(done.status, done.err);
    if (energy) *energy = done.energy;
    if (forces) std::copy(done.forces.begin(), done.forces.end(), forces);
    if (dEdLat) std::memcpy(dEdLat, done.dEdLat, sizeof done.dEdLat);
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(done.t_done - done.t_submit).count();
    return HDNNP_OK;
}

int hdnnp_server_next_done(hdnnp_server* s, int timeout_ms, uint64_t* ticket) {
    if (!s || !ticket) return set_error(HDNNP_E_INPUT, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] {
        while (!s->finished.empty() && !s->reqs.count(s->finished.front())) s->finished.pop_front();
        return !s->finished.empty();
    };
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(std::max(timeout_ms, 0)), ready))
        return set_error(HDNNP_E_TIMEOUT, "no request finished within the timeout");
    *ticket = s->finished.front();
    s->finished.pop_front();
    return HDNNP_OK;
}

int hdnnp_server_read_walker(hdnnp_server* s, int walker, double* pos, double* momenta) {
    if (!s) return set_error(HDNNP_E_INPUT, "null server");
    std::lock_guard<std::mutex> g(s->mu);  // keeps the walker idle while copying
    auto it = s->walkers.find(walker);
    if (it == s->walkers.end()) return set_error(HDNNP_E_INPUT, "unknown walker");
    const Walker& w = it->second;
    if (w.busy) return set_error(HDNNP_E_STATE, "walker has a request in flight");
    cudaSetDevice(s->device);
    if (pos && cudaMemcpy(pos, w.pos, 24 * (size_t)w.nat, cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_error(HDNNP_E_CUDA, "walker position copy failed");
    if (momenta && cudaMemcpy(momenta, w.mom, 24 * (size_t)w.nat, cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_error(HDNNP_E_CUDA, "walker momentum copy failed");
    return HDNNP_OK;
}

int hdnnp_server_list_stats(hdnnp_server* s, int64_t* built, int64_t* kept) {
    if (!s) return set_error(HDNNP_E_INPUT, "null server");
    if (built) *built = s->list_builds.load();
    if (kept) *kept = s->list_reuses.load();
    return HDNNP_OK;
}

int hdnnp_server_stats(hdnnp_server* s, double* p50_ms, double* p99_ms, double* atom_steps_per_s,
                       double* mean_batch_requests, size_t* hbm_charged, int reset) {
    if (!s) return set_error(HDNNP_E_INPUT, "null server");
    std::lock_guard<std::mutex> g(s->mu);
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    // nearest-rank percentile
    auto pct = [&](double q) {
        if (v.empty()) return 0.0;
        size_t k = (size_t)std::ceil(q * (double)v.size());
        return v[std::min(v.size() - 1, k ? k - 1 : 0)];
    };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (atom_steps_per_s) {
        const double sec = s->have_first ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0.0;
        *atom_steps_per_s = sec > 0 ? (double)s->atoms_done / sec : 0.0;
    }
    if (mean_batch_requests) *mean_batch_requests = s->batches ? (double)s->batched_requests / s->batches : 0.0;
    if (hbm_charged) *hbm_charged = s->hbm_walkers + s->hbm_workspace;
    if (reset) {
        s->lat_ms.clear();
        s->atoms_done = s->batches = s->batched_requests = 0;
        s->have_first = false;
    }
    return HDNNP_OK;
}

}  // extern "C"

// plan.cu -- resident plans: a fixed batch evaluated (and optionally advanced
// by velocity-Verlet MD) from a CUDA graph, with Verlet-skin neighbour lists.
//
// No reference counterpart.  The reference re-does all set-up on every call
// of hdnnpEnergyAndForces (src/potentials/hdnnps.f90:333-371) and rebuilds the
// neighbour lists each time (hdnnps.f90:347).  A plan fixes the structures,
// their atom counts, periodic flags, lattices and element numbers, and the
// device buffers of positions and results.  Creating it runs one evaluation
// that measures the neighbour counts, reserves capacities with headroom, and
// captures the evaluation -- or `steps_per_launch` MD steps -- into a CUDA
// graph, so every launch is one graph launch without host work or host reads.
// Molecules get their bounding box on the device.  With a skin, lists are
// built with cutoff rc + skin and kept until an atom has moved more than
// skin / 2 since the last build (checked on the device each evaluation);
// every evaluation copies the entries within rc into a compacted list that
// the later stages read (launch_compact_lists).  Overflow of the planned capacities is flagged
// on the device (no access leaves the reserved arrays) and reported by
// hdnnp_plan_sync as HDNNP_E_CAPACITY; the plan must then be recreated.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/hdnnp_gpu.h"
#include "engine.h"
#include "integrate.cuh"

namespace hdnnp {
int model_device(const hdnnp_model* m);
int set_error(int code, const std::string& msg);
int ctx_plan_setup(hdnnp_ctx* c, int nstruct, const int64_t* off, const int32_t* periodic, const double* lat,
                   double rc_list);
int ctx_run_planned(hdnnp_ctx* c, int nstruct, int natoms, const int32_t* Z_dev, const double* pos_dev,
                    double* energy_dev, double* force_dev, double* dEdLat_dev, cudaStream_t st, PipePlan& pp);
int* ctx_status_dev(hdnnp_ctx* c);
int ctx_profile_replay(hdnnp_ctx* c, long long evals, long long atoms);
const DevModel& model_devmodel(const hdnnp_model* m);
}  // namespace hdnnp

using namespace hdnnp;

namespace {

constexpr int kThreads = 256;
inline unsigned blocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// acc[0] |= status flags of the evaluation; acc[1] += 1 if it rebuilt its lists
__global__ void k_accumulate(const int* status, const int* rebuild, int* acc) {
    if (blockIdx.x || threadIdx.x) return;
    acc[0] |= status[0];
    acc[1] += rebuild ? *rebuild : 1;
}

// Verlet-skin test: rebuild when an atom moved more than skin/2 since the
// last build (pos_ref = +inf before the first build forces one).
__global__ void k_skin_check(const double* pos, const double* pos_ref, int natoms, double half_skin2, int* rebuild) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natoms) return;
    const double dx = pos[3 * i] - pos_ref[3 * i], dy = pos[3 * i + 1] - pos_ref[3 * i + 1],
                 dz = pos[3 * i + 2] - pos_ref[3 * i + 2];
    if (!(dx * dx + dy * dy + dz * dz <= half_skin2)) *rebuild = 1;  // NaN (first build) rebuilds too
}

__global__ void k_fill(double* p, long long n, double v) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

}  // namespace

struct hdnnp_plan {
    hdnnp_model* model = nullptr;
    hdnnp_ctx* ctx = nullptr;  // private: its workspace must not move under the graph
    int device = 0;
    int nstruct = 0, natoms = 0;
    std::vector<int64_t> off;
    const int32_t* Z = nullptr;
    double* pos = nullptr;
    double *E = nullptr, *F = nullptr, *L = nullptr;
    hdnnp_plan_opts o{};
    PipePlan pp;
    // device state of the plan
    int* acc = nullptr;      // [2]: OR of flags, list builds
    int* rebuild = nullptr;  // [1]
    double* wshift = nullptr;
    double* pos_ref = nullptr;
    double* fprev = nullptr;
    int* h_acc = nullptr;    // pinned
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0, launches_synced = 0;
    int kernels_per_launch = 0;
    // autotuner result (launch shape of the symmetry-function kernels)
    int tuned_split = 0, tuned_per_sm = 0;
    double tuned_ms = 0.0;
    // single-block MD of a small molecule (fused_md.cu) instead of the graph
    bool small = false;
    Batch sb{};
    SmallMdArgs sa{};
    void* sscratch = nullptr;
};

namespace {

// One evaluation (skin test, pipeline, accumulation) on the plan's stream.
int plan_eval(hdnnp_plan* p, cudaStream_t st) {
    int L = 0;
    if (p->rebuild) {
        cudaMemsetAsync(p->rebuild, 0, sizeof(int), st);
        k_skin_check<<<blocks(p->natoms), kThreads, 0, st>>>(p->pos, p->pos_ref, p->natoms,
                                                             0.25 * p->o.skin * p->o.skin, p->rebuild);
        ++L;
    }
    int r = ctx_run_planned(p->ctx, p->nstruct, p->natoms, p->Z, p->pos, p->E, p->F, p->L, st, p->pp);
    if (r) return -r;
    int n = 0;
    hdnnp_last_launch_count(p->ctx, &n);
    L += n;
    k_accumulate<<<1, 32, 0, st>>>(ctx_status_dev(p->ctx), p->rebuild, p->acc);
    return L + 1;
}

// The work of one launch: an evaluation, or steps_per_launch MD steps.
int plan_body(hdnnp_plan* p, cudaStream_t st) {
    if (!p->o.momenta_dev) return plan_eval(p, st);
    const long long n3 = 3LL * p->natoms;
    int L = 0;
    for (int k = 0; k < p->o.steps_per_launch; ++k) {
        k_md_drift<<<blocks(n3), kThreads, 0, st>>>(p->pos, p->o.momenta_dev, p->o.masses_dev, p->F, p->fprev,
                                                    (int)n3, p->o.dt);
        const int r = plan_eval(p, st);
        if (r < 0) return r;
        k_md_kick<<<blocks(n3), kThreads, 0, st>>>(p->o.momenta_dev, p->F, p->fprev, p->F, (int)n3, p->o.dt);
        if (p->o.energy_hist_dev)
            cudaMemcpyAsync(p->o.energy_hist_dev + (size_t)k * p->nstruct, p->E, sizeof(double) * p->nstruct,
                            cudaMemcpyDeviceToDevice, st);
        L += r + 2;
    }
    return L;
}

// Autotuner: times the two symmetry-function stages (values + gradients) of
// the plan's own batch on its stream for each candidate launch shape -- the
// neighbour count that splits the two launches (or one launch) and the
// persistent grid in blocks per SM -- and keeps the fastest.  Each candidate
// runs twice, the second run is timed with the stage events.
int plan_autotune(hdnnp_plan* p) {
    static const int kSplits[] = {-1, 32, 48, 64, 96};
    static const int kPerSm[] = {8, 16, 32};
    hdnnp_ctx* c = p->ctx;
    int r = hdnnp_ctx_set_profiling(c, 1);
    double best = 1e300;
    int bs = 0, bp = 0;
    for (int sp : kSplits) {
        if (sp > 0 && sp >= p->pp.m_cap) continue;  // same as one launch
        for (int ps : kPerSm) {
            if ((r = hdnnp_ctx_set_option(c, "sf_split", sp)) || (r = hdnnp_ctx_set_option(c, "sf_blocks_per_sm", ps)))
                return r;
            double ms[8] = {0};
            for (int rep = 0; rep < 2; ++rep) {
                if ((r = hdnnp_profile_read(c, nullptr, nullptr, 1))) return r;
                const int L = plan_eval(p, p->stream);
                if (L < 0) return -L;
                if (cudaStreamSynchronize(p->stream) != cudaSuccess) return set_error(HDNNP_E_CUDA, "autotune run failed");
                if ((r = ctx_profile_replay(c, 1, p->natoms))) return r;
            }
            if ((r = hdnnp_profile_read(c, ms, nullptr, 1))) return r;
            const double t = ms[3] + ms[5];
            if (t < best) {
                best = t;
                bs = sp;
                bp = ps;
            }
        }
    }
    if ((r = hdnnp_ctx_set_option(c, "sf_split", bs)) || (r = hdnnp_ctx_set_option(c, "sf_blocks_per_sm", bp)) ||
        (r = hdnnp_ctx_set_profiling(c, p->o.profile ? 1 : 0)) || (r = hdnnp_profile_read(c, nullptr, nullptr, 1)))
        return r;
    p->tuned_split = bs;
    p->tuned_per_sm = bp;
    p->tuned_ms = best;
    cudaMemset(p->acc, 0, 2 * sizeof(int));
    return HDNNP_OK;
}

// Scratch and arguments of the single-block MD kernel (fused_md.cu): element
// indices (host-built from Z) and the structure record it copies into shared
// memory, and global homes of up to N*N neighbour entries and the per-atom SF
// arrays for what its shared-memory layout cannot hold.
int plan_setup_small(hdnnp_plan* p) {
    const DevModel& D = model_devmodel(p->model);
    const int N = p->natoms;
    std::vector<int32_t> Z((size_t)N);
    if (cudaMemcpy(Z.data(), p->Z, sizeof(int32_t) * N, cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_error(HDNNP_E_CUDA, "reading Z failed");
    std::vector<int> elem((size_t)N);
    for (int i = 0; i < N; ++i) {
        elem[i] = (Z[i] >= 1 && Z[i] <= 118) ? D.z2e[Z[i]] : -1;
        if (elem[i] < 0) return set_error(HDNNP_E_INPUT, "atom with an element that is not in the potential");
    }
    // global scratch: the source copies of the element indices and the
    // structure record, and the per-step arrays that the kernel's shared
    // memory layout leaves in global memory (large molecules / wide SF sets)
    const size_t NN = (size_t)N * N, nsf = (size_t)D.nsf_max;
    const size_t nd = 2 * N * nsf + 3 * NN + 9 * N;
    const size_t ni = 3 * NN + N;
    const size_t bytes = nd * 8 + sizeof(StructInfo) + ni * 4;
    if (cudaMalloc(&p->sscratch, bytes) != cudaSuccess) return set_error(HDNNP_E_CUDA, "small-MD scratch allocation");
    double* d = (double*)p->sscratch;
    StructInfo* info = (StructInfo*)(d + nd);
    int* q = (int*)(info + 1);
    Batch& b = p->sb;
    b = Batch{};
    b.nstruct = 1;
    b.natoms = N;
    b.G = d; d += N * nsf;
    b.dEdG = d; d += N * nsf;
    b.gent = d; d += 3 * NN;
    b.vir = d;
    b.info = info;
    b.nei_j = q; q += NN;
    b.nei_s = q; q += NN;
    b.nei_rev = q; q += NN;
    b.elem = q;
    b.Z = p->Z;
    b.mmax = N - 1;
    b.nentries = (int)NN;
    StructInfo S{};
    for (int k = 0; k < 9; ++k) S.h[k] = S.hinv[k] = (k % 4 == 0) ? 1.0 : 0.0;
    S.ngrid[0] = S.ngrid[1] = S.ngrid[2] = 1;
    S.nat = N;
    if (cudaMemcpy(info, &S, sizeof S, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b.elem, elem.data(), sizeof(int) * N, cudaMemcpyHostToDevice) != cudaSuccess)
        return set_error(HDNNP_E_CUDA, "small-MD set-up copies failed");
    SmallMdArgs& a = p->sa;
    a.natoms = N;
    a.nsteps = p->o.steps_per_launch;
    a.dt = p->o.dt;
    a.pos = p->pos;
    a.mom = p->o.momenta_dev;
    a.mass = p->o.masses_dev;
    a.force = p->F;
    a.energy = p->E;
    a.hist = p->o.energy_hist_dev;
    a.acc = p->acc;
    return HDNNP_OK;
}

void plan_release(hdnnp_plan* p) {
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->stream) cudaStreamSynchronize(p->stream);
    for (void* q : {(void*)p->acc, (void*)p->rebuild, (void*)p->wshift, (void*)p->pos_ref, (void*)p->fprev})
        if (q) cudaFree(q);
    if (p->h_acc) cudaFreeHost(p->h_acc);
    if (p->sscratch) cudaFree(p->sscratch);
    if (p->stream) cudaStreamDestroy(p->stream);
    if (p->ctx) hdnnp_ctx_free(p->ctx);
}

}  // namespace

extern "C" {

int hdnnp_plan_create(hdnnp_model* m, const hdnnp_plan_opts* o, int nstruct, const int64_t* atom_off,
                      const int32_t* periodic, const double* lat, const int32_t* Z_dev, double* pos_dev,
                      double* energy_dev, double* force_dev, double* dEdLat_dev, hdnnp_plan** out) {
    if (!m || !o || nstruct <= 0 || !atom_off || !periodic || !Z_dev || !pos_dev || !energy_dev || !force_dev || !out)
        return set_error(HDNNP_E_INPUT, "null argument or empty batch");
    if (!(o->skin >= 0.0) || !std::isfinite(o->skin) || !(o->margin >= 0.0))
        return set_error(HDNNP_E_INPUT, "skin and margin must be finite and >= 0");
    if (o->momenta_dev && (!o->masses_dev || o->steps_per_launch < 1 || !std::isfinite(o->dt)))
        return set_error(HDNNP_E_INPUT, "MD plan needs masses, steps_per_launch >= 1 and a finite dt");
    bool any_periodic = false;
    for (int s = 0; s < nstruct; ++s) any_periodic |= periodic[s] != 0;
    if (any_periodic && !lat) return set_error(HDNNP_E_INPUT, "periodic structures need lattices");
    auto* p = new hdnnp_plan();
    p->model = m;
    p->o = *o;
    p->device = model_device(m);
    p->nstruct = nstruct;
    p->off.assign(atom_off, atom_off + nstruct + 1);
    p->natoms = (int)atom_off[nstruct];
    p->Z = Z_dev;
    p->pos = pos_dev;
    p->E = energy_dev;
    p->F = force_dev;
    p->L = dEdLat_dev;
    auto bail = [&](int code, const std::string& msg) {
        std::string keep = msg;
        plan_release(p);
        delete p;
        return set_error(code, keep);
    };
    if (cudaSetDevice(p->device) != cudaSuccess) return bail(HDNNP_E_CUDA, "cudaSetDevice failed");
    int r = hdnnp_ctx_create(m, &p->ctx);
    if (!r) r = hdnnp_ctx_set_precision(p->ctx, o->precision);
    if (!r && o->profile) r = hdnnp_ctx_set_profiling(p->ctx, 1);
    if (r) return bail(r, hdnnp_last_error());
    int nel = 0, zs[128], ns[128];
    double max_rc = 0;
    hdnnp_model_info(m, &nel, zs, ns, &max_rc);
    const double rc_list = max_rc + o->skin;
    std::vector<double> latv(9 * (size_t)nstruct, 0.0);
    if (lat) latv.assign(lat, lat + 9 * (size_t)nstruct);
    r = ctx_plan_setup(p->ctx, nstruct, atom_off, periodic, latv.data(), rc_list);
    if (r) return bail(r, hdnnp_last_error());
    const size_t n3 = 3 * (size_t)p->natoms;
    bool ok = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&p->acc, 2 * sizeof(int)) == cudaSuccess &&
              cudaMallocHost(&p->h_acc, 2 * sizeof(int)) == cudaSuccess &&
              cudaMemset(p->acc, 0, 2 * sizeof(int)) == cudaSuccess;
    if (ok && o->skin > 0.0)
        ok = cudaMalloc(&p->rebuild, sizeof(int)) == cudaSuccess && cudaMalloc(&p->wshift, n3 * 8) == cudaSuccess &&
             cudaMalloc(&p->pos_ref, n3 * 8) == cudaSuccess;
    if (ok && o->momenta_dev) ok = cudaMalloc(&p->fprev, n3 * 8) == cudaSuccess;
    if (!ok) return bail(HDNNP_E_CUDA, "plan buffers could not be allocated");
    if (p->pos_ref) k_fill<<<blocks((long long)n3), kThreads, 0, p->stream>>>(p->pos_ref, (long long)n3, INFINITY);
    p->pp.margin = o->margin;
    p->pp.pad_lists = true;
    // molecules get their box on the device (periodic cells keep their set-up)
    p->pp.dev_boxes = false;
    for (int s = 0; s < nstruct; ++s) p->pp.dev_boxes = p->pp.dev_boxes || !periodic[s];
    p->pp.rc_list = o->skin > 0.0 ? rc_list : 0.0;
    p->pp.rebuild = p->rebuild;
    p->pp.wshift = p->wshift;
    p->pp.pos_ref = p->pos_ref;
    // probe: one plain evaluation on the stream, which sizes the capacities
    // and gives the forces the first MD step starts from
    p->pp.upload = true;
    r = plan_eval(p, p->stream);
    if (r < 0) return bail(-r, hdnnp_last_error());
    if (cudaStreamSynchronize(p->stream) != cudaSuccess) return bail(HDNNP_E_CUDA, "probe evaluation failed");
    cudaMemcpy(p->h_acc, p->acc, 2 * sizeof(int), cudaMemcpyDeviceToHost);
    if (p->h_acc[0]) {
        const int f = p->h_acc[0];
        return bail((f & 1) || (f & 8) ? HDNNP_E_INPUT : (f & 16) ? HDNNP_E_TIMEOUT : HDNNP_E_CAPACITY,
                    "probe evaluation flagged the input (device flags " + std::to_string(f) + ")");
    }
    cudaMemset(p->acc, 0, 2 * sizeof(int));
    if (o->profile) hdnnp_profile_read(p->ctx, nullptr, nullptr, 1);  // the probe is not a launch
    if (o->autotune && (r = plan_autotune(p))) return bail(r, hdnnp_last_error());
    // one small molecule in FP64: every MD step of a launch in one kernel
    {
        const DevModel& D = model_devmodel(m);
        p->small = o->momenta_dev && nstruct == 1 && !periodic[0] && p->natoms <= kSmallMolecule &&
                   o->precision == HDNNP_PREC_FP64 && !o->profile && o->single_block >= 0 &&
                   small_md_smem_bytes(D, p->natoms) <= 226 * 1024;
        if (p->small) {
            if ((r = plan_setup_small(p))) return bail(r, hdnnp_last_error());
            p->kernels_per_launch = 1;
            *out = p;
            return HDNNP_OK;
        }
    }
    // capture one launch
    p->pp.upload = false;
    if (cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess)
        return bail(HDNNP_E_CUDA, "cudaStreamBeginCapture failed");
    const int L = plan_body(p, p->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(p->stream, &g);
    p->graph = g;
    if (L < 0) return bail(-L, hdnnp_last_error());
    if (ce != cudaSuccess || !g) return bail(HDNNP_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    if (cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) return bail(HDNNP_E_CUDA, "cudaGraphInstantiate failed");
    p->kernels_per_launch = L;
    *out = p;
    return HDNNP_OK;
}

int hdnnp_plan_launch(hdnnp_plan* p, void* stream) {
    if (!p || (!p->exec && !p->small)) return set_error(HDNNP_E_INPUT, "null plan");
    cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
    if (p->small) {
        launch_small_md(p->sb, model_devmodel(p->model), p->sa, st);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_error(HDNNP_E_CUDA, std::string("single-block MD: ") + cudaGetErrorString(e));
        ++p->launches;
        return HDNNP_OK;
    }
    const cudaError_t e = cudaGraphLaunch(p->exec, st);
    if (e != cudaSuccess) return set_error(HDNNP_E_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
    ++p->launches;
    return HDNNP_OK;
}

int hdnnp_plan_sync(hdnnp_plan* p, void* stream, int64_t* list_builds) {
    if (!p) return set_error(HDNNP_E_INPUT, "null plan");
    cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
    cudaMemcpyAsync(p->h_acc, p->acc, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemsetAsync(p->acc, 0, 2 * sizeof(int), st);
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(HDNNP_E_CUDA, cudaGetErrorString(e));
    if (list_builds) *list_builds = p->h_acc[1];
    if (p->o.profile && p->launches > p->launches_synced) {
        const long long evals = (p->launches - p->launches_synced) * (p->o.momenta_dev ? p->o.steps_per_launch : 1);
        const int r = ctx_profile_replay(p->ctx, evals, evals * p->natoms);
        if (r) return r;
    }
    p->launches_synced = p->launches;
    const int f = p->h_acc[0];
    if (f & 1) return set_error(HDNNP_E_INPUT, "atom with an element that is not in the potential");
    if (f & 8) return set_error(HDNNP_E_INPUT, "non-finite position");
    if (f & (4 | 32))
        return set_error(HDNNP_E_CAPACITY, "neighbour counts above the plan's capacities: create the plan again");
    if (f & 2) return set_error(HDNNP_E_STATE, "internal error: neighbour list is not symmetric");
    if (f & 16) return set_error(HDNNP_E_TIMEOUT, "tensor-core network kernel: bounded wait expired");
    return HDNNP_OK;
}

int hdnnp_plan_profile(hdnnp_plan* p, double* stage_ms, int64_t* counters, int reset) {
    if (!p) return set_error(HDNNP_E_INPUT, "null plan");
    return hdnnp_profile_read(p->ctx, stage_ms, counters, reset);
}

int hdnnp_plan_tuning(const hdnnp_plan* p, int* sf_split, int* sf_blocks_per_sm, double* sf_ms) {
    if (!p) return set_error(HDNNP_E_INPUT, "null plan");
    if (sf_split) *sf_split = p->tuned_split;
    if (sf_blocks_per_sm) *sf_blocks_per_sm = p->tuned_per_sm;
    if (sf_ms) *sf_ms = p->tuned_ms;
    return HDNNP_OK;
}

int hdnnp_plan_info(const hdnnp_plan* p, int64_t* entry_capacity, int* kernels_per_launch) {
    if (!p) return set_error(HDNNP_E_INPUT, "null plan");
    if (entry_capacity) *entry_capacity = p->pp.e_cap;
    if (kernels_per_launch) *kernels_per_launch = p->kernels_per_launch;
    return HDNNP_OK;
}

void hdnnp_plan_free(hdnnp_plan* p) {
    if (!p) return;
    cudaSetDevice(p->device);
    plan_release(p);
    delete p;
}

}  // extern "C"

/* hdnnp_gpu.h -- C ABI of the B200-native HDNNP prediction engine.
 *
 * Drop-in boundary for the reference's Fortran potential API
 * (Jonas-Finkler/High-Dimensional-Neural-Network-Potential,
 * src/potentials/hdnnps.f90).  Every call is plain C: pointers, sizes and
 * status codes; no CUDA or C++ types appear in the signatures (streams are
 * passed as void*).  A Fortran ISO_C_BINDING binding of these entry points is
 * in fortran/hdnnps_gpu.f90.
 *
 * Conventions (same as the reference):
 *   positions   double[3*nat]  x,y,z per atom, Bohr      (atStruct%ats(3,nat))
 *   lattice     double[9]      column-major 3x3, column c = lattice vector c
 *                                                        (atStruct%lat(3,3))
 *   Z           int32[nat]     atomic numbers           (atStruct%el)
 *   forces      double[3*nat]  -dE/dr
 *   dEdLat      double[9]      dE/dh (column-major, like lat); periodic only
 *   energy      double         sum of atomic NN outputs + atom_energy
 * Energies come out in the units of the potential (the reference converts
 * nothing, atomicStructure.f90:157).
 *
 * All entry points return HDNNP_OK (0) or an error code; they never abort.
 * hdnnp_last_error() returns a message for the calling thread.
 */
#ifndef HDNNP_GPU_H
#define HDNNP_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    HDNNP_OK = 0,
    HDNNP_E_INPUT = 1,    /* bad argument, unknown element, singular cell ...  */
    HDNNP_E_IO = 2,       /* a RuNNer file is missing or malformed             */
    HDNNP_E_CAPACITY = 3, /* a size limit of the engine is exceeded            */
    HDNNP_E_TIMEOUT = 4,  /* a bounded wait expired                            */
    HDNNP_E_CUDA = 5,     /* a CUDA runtime call failed                        */
    HDNNP_E_STATE = 6     /* call not valid in the current state               */
} hdnnp_status;

typedef enum {
    HDNNP_PREC_FP64 = 0,  /* FP64 everywhere (parity form)                                  */
    HDNNP_PREC_MIXED = 1  /* FP32 symmetry functions, FP16 tensor-core MLP with hi+lo split,
                             FP64 wrapping, energy and virial reductions                      */
} hdnnp_precision;

typedef struct hdnnp_model hdnnp_model; /* parsed potential + its device copy */
typedef struct hdnnp_ctx hdnnp_ctx;     /* evaluation context: stream + workspace */

/* Message of the last failed call on this thread ("" if none). */
const char* hdnnp_last_error(void);

/* ---------------------------------------------------------------- model
 * Replaces parseRuNNerInput(handle, path) (hdnnps.f90:34-233) together with
 * sortSymFunctions (:235), readScaling (:269) and readWeights (:302).
 * `path` is a directory; like the reference it is joined with the file names
 * (a trailing '/' is added if missing).  Differences from the reference,
 * which stops the process instead: errors are returned; there is no
 * 200-symmetry-function cap (nmaxSFs, hdnnps.f90:48); symmetry-function types
 * other than 2 and 3 are rejected instead of skipped.  The model is uploaded
 * to `device` (CUDA ordinal).                                              */
int hdnnp_model_load_runner(const char* path, int device, hdnnp_model** out);

/* Elements (sorted by Z) and their symmetry-function counts; arrays of
 * length >= 118.  max_rc = largest cutoff (hdnnp%maxRc, hdnnps.f90:16).    */
int hdnnp_model_info(const hdnnp_model* m, int* nelem, int* Z, int* nsf, double* max_rc);

/* The components of type(hdnnp) (hdnnps.f90:13-21) as parsed, for callers
 * that read them: scalesf, centersf, emin, emax (read by readScaling,
 * :269-300, and unused by the prediction) and atomenergies(118), indexed by
 * atomic number - 1 (0 for elements not in the potential); each may be NULL. */
int hdnnp_model_flags(const hdnnp_model* m, int* scalesf, int* centersf, double* emin, double* emax,
                      double* atomenergies);

/* sfLists(Z) (type symFunctionList, symmetryFunctions.f90:18-21) in the
 * reference's sorted order: nsf and, if params != NULL, 11 doubles per
 * function: name (2 or 3), sfEls(1), sfEls(2) (atomic numbers; 0 for type 2),
 * rcut, eta, lambda, zeta, Rs, sfmin, sfmax, sfmean.  HDNNP_E_INPUT if Z is
 * not an element of the potential.                                          */
int hdnnp_model_symfunctions(const hdnnp_model* m, int Z, int* nsf, double* params);

/* nnList(Z) (type neuralNetwork, neuralNetworks.f90:24-28): nlayers and, when
 * non-NULL, dims[2*l] = nInp and dims[2*l+1] = nOut of layer l, acts[l] its
 * activation ('l', 't', 'p', 'r'), and values = for each layer
 * weights(nOut, nInp) in Fortran (column-major) order, then bias(nOut).     */
int hdnnp_model_network(const hdnnp_model* m, int Z, int* nlayers, int* dims, char* acts, double* values);

void hdnnp_model_free(hdnnp_model* m);

/* ---------------------------------------------------------------- context
 * A context owns a CUDA stream and a growable device workspace.  It is used
 * by one host thread at a time; several contexts may share one model.      */
int hdnnp_ctx_create(hdnnp_model* m, hdnnp_ctx** out);
void hdnnp_ctx_free(hdnnp_ctx* c);
int hdnnp_ctx_set_precision(hdnnp_ctx* c, int precision);

/* Context options (for tests and tuning): "sf_split" (-1: one launch; 0:
 * default 64; n: atoms with more than n neighbours in a second launch) and
 * "sf_blocks_per_sm" (0: default 32) shape the launches of the
 * lambda x zeta x eta kernels; "generic_sf" = 1 forces the
 * generic symmetry-function kernels (one parameter record per SF) instead of
 * the lambda x zeta x eta kernels; "runtime_zeta" = 1 makes the
 * lambda x zeta x eta kernels read the zeta set from the model even when a
 * kernel with that zeta set compiled in exists.  Results agree within
 * rounding.  "nei_warp" chooses how neighbour lists are built: 1 one warp per
 * atom, -1 one thread per atom, 0 (default) a warp per atom below 131,072
 * atoms in the batch; both give the same lists, entry for entry.
 * "small_eval" (default 1): a call of one molecule of at most 64 atoms in
 * FP64 (the reference's own MD example is one) runs as one kernel launch, a
 * thread block that builds the lists by direct search and keeps every
 * intermediate on chip, between one copy in and one copy out; 0 runs it
 * through the general pipeline (same results within rounding; the
 * intermediates of hdnnp_debug_fetch exist only then).
 * "small_resident" (default 1): such molecules that fit the kernel's
 * item-parallel form are served by a resident copy of it that stays on one
 * SM between calls and takes each call from a mailbox in mapped host memory
 * (no launch per call, warm caches; same results).  It leaves by itself
 * after a few milliseconds without a call, and when the context is freed or
 * the option is set to 0; while it waits it holds one SM and a
 * device-wide synchronisation waits for it to leave.                        */
int hdnnp_ctx_set_option(hdnnp_ctx* c, const char* name, int value);

/* ---------------------------------------------------------------- evaluation
 * Replaces hdnnpEnergyAndForces(handle, ats, energy, force, dEdLat)
 * (hdnnps.f90:333-371): neighbour lists (hdnnpCalcNeighborLists :373),
 * symmetry functions (hdnnpCalcSymfunctions :390) and the networks with the
 * force/dEdLat contraction (hdnnpCalcNNs :487).  Host arrays in, host arrays
 * out, synchronous.  dEdLat may be NULL; it requires periodic != 0 (the
 * reference reads an uninitialised lattice otherwise, hdnnps.f90:509).     */
int hdnnp_energy_and_forces(hdnnp_ctx* c, int nat, const int32_t* Z, const double* pos, int periodic,
                            const double* lat, double* energy, double* force, double* dEdLat);

/* The three stages of hdnnp_energy_and_forces as separate calls, as the
 * reference makes them public for its committee (globalHdnnps.f90:47-57).
 * Lists and values stay in the context's device memory between the calls
 * (the reference hands neiLists and sfs back to the caller).
 *
 * hdnnpCalcNeighborLists (hdnnps.f90:373-388): wraps the structure, builds
 * its neighbour lists and keeps them in `c`; nentries (may be NULL) receives
 * the number of neighbour entries, not counting the atoms themselves (the
 * reference stores each atom as entry 1 of its own list).                   */
int hdnnp_calc_neighbor_lists(hdnnp_ctx* c, int nat, const int32_t* Z, const double* pos, int periodic,
                              const double* lat, int* nentries);

/* The lists of the last hdnnp_calc_neighbor_lists on `c` in the layout of
 * the reference's type neighborList (neighborLists.f90:10-16): nneis[nat]
 * entries per atom (count + 1); if non-NULL, ineis[sum nneis] the 0-based
 * atom index of each entry and neis[3 * sum nneis] its Cartesian position
 * (image of the wrapped position), atom by atom, entry 1 of each atom being
 * the atom itself.  Size ineis and neis from nneis (a first call with both
 * NULL).                                                                     */
int hdnnp_neighbor_lists_fetch(hdnnp_ctx* c, int* nneis, int* ineis, double* neis);

/* hdnnpCalcSymfunctions (hdnnps.f90:390-485): the centred and scaled
 * symmetry functions of the structure of the last hdnnp_calc_neighbor_lists
 * on `c`.  G (may be NULL) receives them on the host, nat x nsf_max with row
 * stride nsf_max (nsf_max = the largest symmetry-function count of the
 * potential; unused columns are zero).  Their derivatives are not stored:
 * hdnnp_calc_nns recomputes them in its contraction, where the reference
 * keeps dsf(3, nNei) for every function and atom.  HDNNP_E_STATE without
 * lists.                                                                     */
int hdnnp_calc_symfunctions(hdnnp_ctx* c, double* G);

/* hdnnpCalcNNs (hdnnps.f90:487-562): the networks of `nn` (NULL: the
 * potential of `c`) on the symmetry functions of the last
 * hdnnp_calc_symfunctions on `c`, and the contraction into energy, forces and
 * dEdLat (NULL, or a periodic structure).  `nn` must have the elements and
 * network input widths of the potential of `c`, whose symmetry functions and
 * derivatives are used (as globalHdnnpEnergyAndForces does, :51-57).  May be
 * called several times on the same values.  HDNNP_E_STATE without values.
 * The chain of the three calls gives bitwise the results of
 * hdnnp_energy_and_forces.                                                   */
int hdnnp_calc_nns(hdnnp_ctx* c, const hdnnp_model* nn, double* energy, double* force, double* dEdLat);

/* Batch of nstruct independent structures in CSR form (no reference
 * counterpart: the reference evaluates one structure per call).
 * atom_off[nstruct+1] (atom_off[0] = 0); Z, pos, force indexed by global
 * atom; periodic[nstruct]; lat[9*nstruct]; energy[nstruct];
 * dEdLat[9*nstruct] or NULL (rows of non-periodic structures are zero).    */
int hdnnp_eval_batch(hdnnp_ctx* c, int nstruct, const int64_t* atom_off, const int32_t* Z, const double* pos,
                     const int32_t* periodic, const double* lat, double* energy, double* force, double* dEdLat);

/* Same, with every array already in device memory of the context's device
 * (inputs resident in HBM; no host copies).  Asynchronous on `stream`
 * (a cudaStream_t, or NULL for the context's own stream) except for one
 * small device-to-host read of the neighbour-entry total.  atom_off_host is
 * a HOST copy of the offsets (used to size the workspace).                  */
int hdnnp_eval_batch_device(hdnnp_ctx* c, int nstruct, const int64_t* atom_off_host, const int64_t* atom_off_dev,
                            const int32_t* Z_dev, const double* pos_dev, const int32_t* periodic_host,
                            const double* lat_host, double* energy_dev, double* force_dev, double* dEdLat_dev,
                            void* stream);

/* ---------------------------------------------------------------- committee
 * Replaces globalHdnnpEnergyAndForces(ats, energy, forces, dEdLat, std)
 * (globalHdnnps.f90:31-70): neighbour lists and symmetry functions -- with
 * their scaling -- come from members[0] (:47, :51), and every member's
 * networks run on them (:55-57); energy, forces and dEdLat are the member
 * means and std the population standard deviation of the member energies
 * (:60-68).  `c` must be a context of members[0]; every member must have the
 * same elements and a network input as wide as members[0]'s symmetry-function
 * list (the reference assumes this silently).  The members' dE/dG are averaged
 * before the one force/virial contraction (linear; equal within rounding to
 * averaging member forces).  std may be NULL.  The batch form takes the
 * arrays of hdnnp_eval_batch plus std[nstruct].                              */
int hdnnp_committee_energy_and_forces(hdnnp_ctx* c, hdnnp_model* const* members, int nmembers, int nat,
                                      const int32_t* Z, const double* pos, int periodic, const double* lat,
                                      double* energy, double* force, double* dEdLat, double* std);
int hdnnp_committee_eval_batch(hdnnp_ctx* c, hdnnp_model* const* members, int nmembers, int nstruct,
                               const int64_t* atom_off, const int32_t* Z, const double* pos, const int32_t* periodic,
                               const double* lat, double* energy, double* force, double* dEdLat, double* std);

/* ---------------------------------------------------------------- no-allocation variant
 * No counterpart in the reference.  The same evaluation as
 * hdnnp_energy_and_forces (host arrays in and out, same arguments and
 * results), for callers that cannot allocate GPU memory when they evaluate:
 * an MD or Monte Carlo host code that runs under a fixed device-memory budget
 * handed out at start-up, or a language binding without access to the CUDA
 * allocator.  It needs no context and calls no cudaMalloc, cudaFree or
 * allocating library routine: all intermediates live in one static 32 MiB
 * device array compiled into the library.
 * Memory: under lazy module loading (CUDA's default) a device reserves the
 * 32 MiB when this entry point first runs on it, so make that first call at
 * start-up, before a memory budget is handed out; with
 * CUDA_MODULE_LOADING=EAGER every process that loads the library reserves
 * them on every device it initialises.  The array stays reserved until the
 * process exits.
 * Limit: the structure must fit that array (for a 280-SF potential about
 * 5,000 atoms with ~52 neighbours each; in general about
 * nat * (16 * nsf_max + 210) + neighbour_entries * 36 bytes); larger inputs
 * return HDNNP_E_CAPACITY with the size that did not fit.
 * Set-up: the first call on a device looks up the device address of the
 * static array (cudaGetSymbolAddress) with that device current.
 * Streams: the call copies synchronously and runs its kernels on the legacy
 * default stream, and returns when they are done.  It must not run while any
 * stream of the device is being captured in the global capture mode.  The
 * caller's current device is restored before it returns.
 * Sharing: every call uses the same array and it keeps the last call's
 * contents (the call clears what must start at zero).  Calls are serialised
 * per device inside one process; calls that overlap on the GPU from other
 * processes or other copies of the library race on the array.               */
int hdnnp_energy_and_forces_noalloc(const hdnnp_model* m, int nat, const int32_t* Z, const double* pos,
                                    int periodic, const double* lat, double* energy, double* force,
                                    double* dEdLat);

/* ---------------------------------------------------------------- stress
 * dEdLat2Stress (atomicStructure.f90:679-686): stress = -1/det(h) dEdLat h^T. */
int hdnnp_dEdLat_to_stress(const double* lat, const double* dEdLat, double* stress);

/* ---------------------------------------------------------------- inspection
 * Copies an intermediate of the last evaluation on `c` to host memory, for
 * tests and profiling.  what: "G" (scaled symmetry functions, nat x nsf_max,
 * row stride nsf_max), "dEdG" (same layout), "atom_energy" (nat),
 * "nei_count" (nat, excluding the atom itself), "nei_index" (entries),
 * "nei_shift" (entries, packed image shift), "nsf_max" (1 int).
 * `bytes` is the size of `host`; returns HDNNP_E_CAPACITY if too small.  The
 * list arrays ("nei_index", "nei_shift", "nei_rev") copy their first `bytes`
 * (size the buffer from "nei_count"): their reserved size can exceed the
 * entries filled.                                                             */
int hdnnp_debug_fetch(hdnnp_ctx* c, const char* what, void* host, size_t bytes);

/* Kernel launches issued by the last evaluation on `c` (0 when the
 * context's resident single-block kernel served it: option "small_resident"). */
int hdnnp_last_launch_count(hdnnp_ctx* c, int* launches);

/* The branch-free FP64 functions that the symmetry-function kernels use for
 * their bounded arguments, evaluated on the current device: y[i] = f(x[i]),
 * which = 0 exp (arguments clamped to [-708, 709]), 1 tanh (u in [0, 1]),
 * 2 sqrt, 3 1/sqrt.  No reference counterpart (a test hook; the reference
 * calls the Fortran intrinsics exp, tanh and sqrt in
 * symmetryFunctions.f90:201-327).                                            */
int hdnnp_debug_math(int which, int n, const double* x, double* y);

/* ---------------------------------------------------------------- profiling
 * Tracing hook in place of the reference's per-stage cpu_time prints
 * (hdnnps.f90:346-368), which are always on there.  With profiling enabled
 * every evaluation records CUDA events around each stage on its stream and
 * counts work units; the totals accumulate until reset.
 * Stages (index): 0 neighbour count, 1 neighbour fill + reverse index,
 * 2 element grouping, 3 symmetry-function values, 4 networks,
 * 5 symmetry-function gradients, 6 force gather + structure reduction.
 * Counters (index): 0 evaluations, 1 atoms, 2 neighbour entries,
 * 3 candidate angular pairs, 4 contributing angular pairs (r_jk < rc),
 * 5 angular SF terms, 6 radial SF terms.                                    */
int hdnnp_ctx_set_profiling(hdnnp_ctx* c, int on);
int hdnnp_profile_read(hdnnp_ctx* c, double* stage_ms /* [8] */, int64_t* counters /* [8] */, int reset);

/* ---------------------------------------------------------------- resident plans
 * No counterpart in the reference, which repeats every set-up step and
 * rebuilds the neighbour lists on each hdnnpEnergyAndForces call
 * (hdnnps.f90:333-371).  A plan fixes a batch (atom_off, periodic, lat as for
 * hdnnp_eval_batch; Z, positions and results in device memory) and captures
 * one evaluation -- or, with momenta, `steps_per_launch` velocity-Verlet steps
 * (hdnnpExample.f90:61-64) -- into a CUDA graph; hdnnp_plan_launch replays it
 * with no host work.  Positions may be changed in place between launches
 * (lattices and atom counts may not).  Molecules get their bounding box on
 * the device.  skin > 0: Verlet-skin lists with cutoff max_rc + skin, rebuilt
 * on the device when an atom has moved more than skin/2 since the last build.
 * Creating a plan runs one evaluation (results valid afterwards; the MD
 * steps start from its forces) and reserves neighbour capacity with
 * `margin` headroom; a later launch that needs more flags it and
 * hdnnp_plan_sync returns HDNNP_E_CAPACITY (results of that launch are not
 * valid; create the plan again).  The plan owns a private workspace.       */
typedef struct hdnnp_plan hdnnp_plan;

typedef struct {
    int precision;           /* HDNNP_PREC_FP64 or HDNNP_PREC_MIXED                     */
    double margin;           /* capacity headroom, e.g. 0.25                            */
    double skin;             /* Verlet skin in Bohr; 0 = rebuild every evaluation      */
    double* momenta_dev;     /* NULL: evaluation plan; else MD plan (3*natoms doubles) */
    const double* masses_dev;/* natoms doubles (MD)                                    */
    double dt;               /* MD time step                                           */
    int steps_per_launch;    /* MD steps per launch                                    */
    double* energy_hist_dev; /* NULL or steps_per_launch*nstruct energies per launch    */
    int profile;             /* 1: stage events captured in the graph (hdnnp_plan_profile) */
    int autotune;            /* 1: before capture, time the symmetry-function kernels of this
                                batch for each candidate launch shape (neighbour-count split
                                of the two launches, persistent grid per SM) and keep the
                                fastest (hdnnp_plan_tuning)                               */
    int single_block;        /* 0: an MD plan of one molecule of at most 64 atoms in FP64
                                runs all steps of a launch in one thread block (one kernel
                                launch, neighbour lists by direct search); -1: never  */
} hdnnp_plan_opts;

int hdnnp_plan_create(hdnnp_model* m, const hdnnp_plan_opts* opts, int nstruct, const int64_t* atom_off,
                      const int32_t* periodic, const double* lat, const int32_t* Z_dev, double* pos_dev,
                      double* energy_dev, double* force_dev, double* dEdLat_dev, hdnnp_plan** out);
/* Asynchronous on `stream` (NULL: the plan's own stream). */
int hdnnp_plan_launch(hdnnp_plan* p, void* stream);
/* Waits for `stream` and returns the device status of the launches since the
 * last sync; list_builds (may be NULL) = neighbour-list builds among them.  */
int hdnnp_plan_sync(hdnnp_plan* p, void* stream, int64_t* list_builds);
int hdnnp_plan_info(const hdnnp_plan* p, int64_t* entry_capacity, int* kernels_per_launch);
/* Profile of a plan created with profile = 1, as hdnnp_profile_read: stage
 * times accumulate over the launches that hdnnp_plan_sync collected (the
 * last evaluation of the last launch before each sync); the work counters
 * cover every evaluation.                                                     */
int hdnnp_plan_profile(hdnnp_plan* p, double* stage_ms, int64_t* counters, int reset);
/* Kernel launches per hdnnp_plan_launch are reported by hdnnp_plan_info
 * (1 for the single-block MD of a small molecule).                           */
/* Launch shape the autotuner chose (0, 0 without autotune: defaults) and the
 * symmetry-function time it measured for it (ms per evaluation).           */
int hdnnp_plan_tuning(const hdnnp_plan* p, int* sf_split, int* sf_blocks_per_sm, double* sf_ms);
void hdnnp_plan_free(hdnnp_plan* p);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference, which evaluates one structure per call
 * from a user-written MD loop (src/potentials/hdnnpExample.f90:59-72).
 * A server keeps many walkers (MD or Monte Carlo trajectories) resident in
 * device memory -- positions, momenta, masses, last forces and the state
 * before the last trial move -- and evaluates their requests by continuous
 * batching: worker threads, each with its own evaluation context and CUDA
 * stream, take pending requests in arrival order, pack those of idle walkers
 * into a batch of at most max_batch_atoms atoms and evaluate it with the
 * batched pipeline; requests that arrive meanwhile join the next batch, and
 * with workers >= 2 consecutive batches overlap on the GPU.  Requests of one
 * walker run in submission order.  A walker's result does not depend on
 * which other walkers share its batch (bitwise for the FP64 form).
 * Admission: walkers and the workers' workspaces are charged against
 * hbm_budget; hdnnp_server_add_walker returns HDNNP_E_CAPACITY when a walker
 * does not fit (remove walkers to admit new ones).                          */
typedef struct hdnnp_server hdnnp_server;

typedef struct {
    size_t hbm_budget;   /* bytes for walkers + workspaces; 0 = no limit         */
    int max_batch_atoms; /* atom slots of one batch (also the largest walker)    */
    int workers;         /* concurrent batches, 1..8                             */
    int precision;       /* HDNNP_PREC_FP64 or HDNNP_PREC_MIXED                  */
    double skin;         /* Verlet skin (Bohr) of the walkers' neighbour lists; 0:
                            lists are built for every request.  With a skin each
                            walker keeps its list (cutoff rc + skin) and builds
                            it again only when one of its atoms has moved by more
                            than skin/2 since; a batch evaluates its walkers that
                            need a list and those that keep one as two parts    */
} hdnnp_server_opts;

typedef enum {
    HDNNP_REQ_EVAL = 0,      /* energy, forces, dEdLat of the current positions  */
    HDNNP_REQ_MC_TRIAL = 1,  /* keep the state, displace every coordinate by
                                N(0, sigma) (generator keyed by seed and the
                                walker's step count), then evaluate              */
    HDNNP_REQ_MC_REJECT = 2, /* restore the state kept by the last trial; no
                                evaluation and no result besides the status      */
    HDNNP_REQ_MD_STEP = 3    /* velocity Verlet step of length dt with the last
                                forces (hdnnpExample.f90:61-64), then evaluate;
                                needs masses and a previous EVAL                 */
} hdnnp_request_kind;

int hdnnp_server_create(hdnnp_model* m, const hdnnp_server_opts* opts, hdnnp_server** out);
/* Stops the workers after their current batch; pending requests are dropped. */
void hdnnp_server_destroy(hdnnp_server* s);

/* Z[nat], pos[3*nat]; lat[9] is used when periodic != 0.  masses[nat] and
 * momenta[3*nat] may be NULL (no MD; momenta default to zero).             */
int hdnnp_server_add_walker(hdnnp_server* s, int nat, const int32_t* Z, const double* pos, int periodic,
                            const double* lat, const double* masses, const double* momenta, int* walker);
/* Frees a walker's device memory; HDNNP_E_STATE while it has requests.      */
int hdnnp_server_remove_walker(hdnnp_server* s, int walker);

int hdnnp_server_submit(hdnnp_server* s, int walker, int kind, double dt, double sigma, uint64_t seed,
                        uint64_t* ticket);
/* Waits up to timeout_ms (0 = poll) for a request; HDNNP_E_TIMEOUT if it is
 * not finished (the ticket stays valid).  On completion the ticket is
 * consumed and energy, forces[3*nat], dEdLat[9] (zero for molecules) and the
 * submit-to-completion latency are written where the pointers are non-NULL. */
int hdnnp_server_wait(hdnnp_server* s, uint64_t ticket, int timeout_ms, double* energy, double* forces,
                      double* dEdLat, double* latency_ms);
/* Waits up to timeout_ms for the next finished request not yet reported by
 * this call (completion order) and returns its ticket, still to be consumed
 * by hdnnp_server_wait; HDNNP_E_TIMEOUT if none.  Tickets consumed by
 * hdnnp_server_wait before they are reported are skipped.                    */
int hdnnp_server_next_done(hdnnp_server* s, int timeout_ms, uint64_t* ticket);
/* Current positions and momenta of an idle walker (HDNNP_E_STATE if busy).  */
int hdnnp_server_read_walker(hdnnp_server* s, int walker, double* pos, double* momenta);
/* Latency percentiles over the finished requests, evaluated atoms per second
 * between the first submit and the last completion, mean requests per batch,
 * and HBM bytes charged to walkers + workspaces.  reset != 0 clears them.    */
int hdnnp_server_stats(hdnnp_server* s, double* p50_ms, double* p99_ms, double* atom_steps_per_s,
                       double* mean_batch_requests, size_t* hbm_charged, int reset);

/* Walker neighbour lists built and kept since the server started (skin > 0;
 * both 0 otherwise).  No reference counterpart: the reference builds the
 * lists on every call (hdnnps.f90:347).                                      */
int hdnnp_server_list_stats(hdnnp_server* s, int64_t* built, int64_t* kept);

#ifdef __cplusplus
}
#endif

#endif /* HDNNP_GPU_H */

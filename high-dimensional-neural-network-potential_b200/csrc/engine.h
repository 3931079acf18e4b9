// engine.h -- device data layout and kernel launchers of the HDNNP engine.
//
// One evaluation of a batch of structures runs these stages on one stream:
//   K1 wrap_and_bin     fractional wrap (FP64, h^-1 of each structure) + cell id
//   K2 cell lists       counting sort of atoms into the cells of their structure
//   K3 neighbours       per-atom count -> scan -> fill (CSR), reverse-entry index
//   K4 sf_values        G2/G4 values, centred and scaled          (pass 1)
//   K5 mlp              per-element network forward + dE/dG       (grouped by element)
//   K6 sf_gradients     dE/dG-weighted G derivatives per neighbour entry (pass 2)
//   K7 force_gather     F_a = -(g_self(a) + sum of reverse entries), deterministic
//   K8 struct_reduce    compensated energy sum, virial -> dE/dh (FP64)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hdnnp {

constexpr int kMaxEl = 16;

// Per-structure set-up computed on the host in FP64 (same formulas as the
// reference: artificial box for molecules, grid of >= 0.6 rc cells, search
// range getNcells(grid, rc)).
struct StructInfo {
    double h[9];      // column-major lattice used for wrapping and image shifts
    double hinv[9];   // its inverse (adjugate / det)
    double org[3];    // box origin for molecules (0 for periodic cells)
    int ngrid[3];     // cells per lattice direction
    int nsearch[3];   // neighbouring cells searched per direction
    int periodic;
    int cell_off;     // first cell of this structure in the global cell arrays
    int atom_off;     // first atom
    int nat;
};

// Radial SF entry, grouped by (centre element, neighbour element).
struct SF2 {
    int sf;      // index in the centre element's SF list
    int nel;     // neighbour element index
    double eta, rs;
};

// Angular SF entry, grouped by (centre element, unordered element pair),
// ordered by eta inside each group (one exp per distinct eta and pair).
struct SF4 {
    int sf;
    int izeta;   // zeta if it is an integer (|zeta - int| < 1e-10), else -1
    double eta, lambda, zeta, pf;  // pf = 2^(1-zeta)
};

// Device copy of the potential (pointers into one device allocation).
struct DevModel {
    int nel;
    int nsf_max;
    int nblk;                 // nel*(nel+1)/2 unordered element pairs
    int gmax;                 // largest angular group
    double max_rc;
    int z2e[120];
    int blk_a[kMaxEl * (kMaxEl + 1) / 2];
    int blk_b[kMaxEl * (kMaxEl + 1) / 2];
    const double* rc;         // [nel] cutoff of each centre element
    const int* nsf;           // [nel]
    const int* g2_off;        // [nel*nel+1]
    int g2max;                // most radial SFs of one centre element
    const SF2* g2;
    const int* g4_off;        // [nel*nblk+1]
    const SF4* g4;
    const double* smean;      // [nel*nsf_max] (0 when not centring)
    const double* swidth;     // [nel*nsf_max] (1 when not scaling)
    const double* sinvw;      // [nel*nsf_max] 1 / swidth (fast kernels multiply)
    // networks
    int nlayers;
    int width[9];             // width[0] = input (per element: nsf), width[l+1] = out of layer l
    char act[8];
    int nin_el[kMaxEl];       // input width per element
    const double* w;          // per element, per layer: W row-major [nout][nin]
    const double* wt;         // same, transposed [nin][nout]
    const double* b;
    const long long* w_off;   // [nel*nlayers] offset of each layer's W / WT
    const long long* b_off;   // [nel*nlayers]
    const double* atom_energy;// [nel]
    // Angular-SF grid of the potential: the distinct lambda, zeta and eta of
    // all G4 SFs.  When every (centre element, element pair) group maps
    // one-to-one into the product lambda x zeta x eta of a compiled shape
    // (NL, NZ, NE), the fast kernels evaluate per pair one power table and one
    // exponential per eta and contract in that product space.
    int fast;                 // 0: generic kernels; else the shape id (1..4)
    int fl, fz, fe;           // model counts (<= NL, NZ, NE of the shape)
    double lam[2];
    double zet[8];
    int zint[8];              // zeta - 1 if zeta is an integer >= 1, else -1
    double pfz[8];            // 2^(1 - zeta)
    double eta4[8];
    // eta4[e] / eta4[0] when every ratio is an integer 2..64 (ascending
    // etas), else 0: the FP64 kernels then take exp(-eta_e R) as
    // exp(-eta_0 R)^k_e by squaring, one exponential per pair
    int eta_k[8];
    int zmaxbit;              // highest bit of the integer zeta - 1 values
    const short* pmap;        // [nel][nblk][P]: SF index of product entry p, or -1
    // FP32 copies of the network weights (mixed-precision form)
    const float* wf;
    const float* wtf;
    const float* bf;
    // First layer packed for the tensor-core network kernel (mlp_tc.cu):
    // FP16 hi | lo of s1 * W1 per element in the K-major core-matrix layouts
    // of the forward GEMM (32 x tc_kp) and of the input-gradient GEMM
    // (tc_np x 32).  tc_ok = 0 if the network does not fit the kernel.
    int tc_ok;
    int tc_kp, tc_np, tc_nch, tc_chn;
    float tc_sdelta;              // power-of-two scale of delta1 before the split
    float tc_inv_s1[kMaxEl];      // 1 / s1 per element
    const unsigned short* tc_fwd;
    const unsigned short* tc_bwd;
    // First layer in the register-fragment order of the FP64 tensor-core
    // network kernel (mma m8n8k4 f64, mlp.cu), zero-padded: forward
    // B[k][n] = W1[n][k] as [ceil(nin/4)][4 n-tiles][32 lanes], input
    // gradient B[k][n] = W1[k][n] as [ceil(nin/8)][ceil(H1/4)][32 lanes];
    // per-element offsets in doubles.  dm_ok = 0 if the network does not fit.
    int dm_ok;
    long long dm_off_f[kMaxEl];
    long long dm_off_b[kMaxEl];
    const double* dm_fwd;
    const double* dm_bwd;
};

// Workspace pointers for one batch evaluation (all device memory).
struct Batch {
    int nstruct;
    int natoms;
    int ncells;
    int nentries;             // neighbour entries (excluding the atoms themselves)
    int mmax;                 // largest neighbour count of one atom
    const StructInfo* info;   // [nstruct]
    const int* Z;             // [natoms]
    const double* pos;        // [3*natoms]
    int* sid;                 // [natoms] structure of each atom
    int* elem;                // [natoms] element index
    double* wpos;             // [3*natoms] wrapped positions
    int* cell_of;             // [natoms]
    int* cell_cnt;            // [ncells+1]
    int* cell_start;          // [ncells+1]
    int* cell_atoms;          // [natoms]
    double4* posc;            // [natoms] wrapped position and index of cell_atoms[p] (cell order), or null
    int* nei_cnt;             // [natoms+1]
    int* nei_off;             // [natoms+1]
    int* nei_j;               // [nentries]
    int* nei_s;               // [nentries] packed image shift
    int* nei_rev;             // [nentries]
    double* G;                // [natoms*nsf_max]
    double* dEdG;             // [natoms*nsf_max]
    double* atE;              // [natoms]
    double* gent;             // [3*nentries]
    double* gself;            // [3*natoms]
    double* vir;              // [9*natoms]
    double* force;            // [3*natoms]
    double* energy;           // [nstruct]
    double* dEdLat;           // [9*nstruct] or null
    int* el_count;            // [nel+1]
    int* el_start;            // [nel+1]
    int* el_atoms;            // [natoms] atoms grouped by element
    int* scan_tmp;            // scan block sums
    int* status;              // [4] device error flags
    unsigned long long* stats;  // [8] work counters or null
    // FP32 intermediates of the mixed-precision form (same layouts)
    float* Gf;
    float* dEdGf;
    float* atEf;
    float* gentf;
    float* gselff;
    float* virf;
    // Resident plans (plan.cu).  rc_list: neighbour-list cutoff (0: the
    // potential's max_rc; max_rc + skin for Verlet-skin lists, which the
    // stages after the list read compacted to max_rc, with rc_list = max_rc;
    // the symmetry-function kernels drop entries beyond an element's own rc
    // when rc_list is above it).  rebuild: device flag,
    // null = build every evaluation; when it is 0 the list, cells and wrap
    // translations of the last build are kept and positions are translated
    // by wshift instead of wrapped.  wshift[3*natoms]: wrapped - raw position
    // of each atom at the last build; pos_ref[3*natoms]: raw positions at the
    // last build.
    double rc_list;
    const int* rebuild;
    double* wshift;
    double* pos_ref;
    // Contributing angular pairs of each atom, written by the fast value pass
    // (j | k << 10 | element-pair block << 20, enumeration order) and read by
    // the gradient pass instead of screening the candidates again; atoms with
    // more than pcap pairs are screened again.  Null: no list.
    unsigned* pairs;          // [natoms * pcap]
    int* npairs;              // [natoms]
    int pcap;
    // Launch shape of the fast symmetry-function kernels (0: defaults): the
    // neighbour count splitting the two launches (-1: one launch) and the
    // persistent grid in blocks per SM.  Set by the plans' autotuner.
    int sf_split;
    int sf_blocks_per_sm;
    int nei_warp;             // neighbour lists: 1 warp per atom, -1 thread per atom, 0 by batch size
    // Plans: the neighbour search writes each atom's entries (j, packed
    // shift) into a padded row of pad_cap in one pass, copied into the CSR
    // arrays after the scan (pad_cap = 0: count pass, then fill pass).
    int2* pad;                // [natoms * pad_cap]
    int pad_cap;
    // With padded rows: per atom, the row position at the start of each
    // (jx, jy) column of its search ("slab"; K = (2 nsearch_x + 1) (2
    // nsearch_y + 1) <= kMaxSlabs of them) and the count at the end.  The
    // search also tags each row entry with its slab (bits 24-31 of the
    // shift word).  The reverse entry of (i -> j) lies in the mirrored slab
    // K - 1 - s of j's row, so the copy into the CSR arrays finds it with a
    // scan of that slab alone.  Null: no slab table (full-row search).
    unsigned short* slab;     // [natoms * kSlabStride]
};

constexpr int kMaxSlabs = 64;
constexpr int kSlabStride = kMaxSlabs + 2;  // K + 1 prefix values, padded to an even count

constexpr int kPairCap = 1024;  // listed pairs per atom (the dense workloads average ~550)

// Resident-plan mode of the pipeline (plan.cu): capacities fixed in advance
// so that an evaluation needs no host read and can be captured in a CUDA
// graph.  e_cap == 0 on the first (probe) evaluation: the pipeline reads the
// counts, sets e_cap / m_cap with `margin` headroom and sizes the workspace.
struct PipePlan {
    long long e_cap = 0;     // neighbour entries
    int m_cap = 0;           // largest per-atom count (multiple of 32)
    double margin = 0.25;
    int ncells = 0;          // cells reserved (molecules: the largest grid allowed)
    bool upload = true;      // host set-up -> device (false inside a capture)
    bool dev_boxes = false;  // molecules: boxes recomputed on the device
    double rc_list = 0.0;    // neighbour-list cutoff (max_rc + skin)
    int* rebuild = nullptr;  // Verlet-skin flag (null: rebuild every time)
    double* wshift = nullptr;
    double* pos_ref = nullptr;
    bool pad_lists = false;  // one search pass into padded rows of m_cap (after the probe)
    bool eager = false;      // an eager call (hdnnp_eval_batch): profiled like one
};

// Device neighbour-list arrays of a context (ctx_list_arrays in capi.cu).
struct CtxLists {
    int *elem, *cnt, *off, *nj, *ns, *rev;
};

// Compacted copy of a Verlet-skin list (launch_compact_lists in
// neighbors.cu): cnt/off [natoms+1], nj/ns/rev [entries], map [entries of
// the full list] (compacted index or -1).
struct CompactLists {
    int *cnt, *off, *nj, *ns, *rev, *map;
};
int launch_compact_lists(const Batch& b, double rc, const CompactLists& c, cudaStream_t s);

// Committee of potentials (committee.cu; globalHdnnpEnergyAndForces,
// globalHdnnps.f90:31-70): neighbour lists and symmetry functions of the
// first member, every member's networks on them; dE/dG is averaged before the
// (linear) force/virial contraction, energies are averaged per structure and
// their population standard deviation is written to std_dev[nstruct].
struct Committee {
    const DevModel* const* members;  // host array of K device models; members[0] gives the SFs
    int k;
    double* std_dev;                 // device [nstruct] or null
};

// Single-block MD of one small molecule (fused_md.cu): every stage of
// `nsteps` velocity-Verlet steps in one kernel launch.
constexpr int kSmallMolecule = 64;  // atoms
struct SmallMdArgs {
    int natoms, nsteps;
    double dt;
    double* pos;
    double* mom;
    const double* mass;
    double* force;
    double* energy;
    double* hist;       // [nsteps] energies or null
    int* acc;           // [2]: OR of status flags, evaluations
    int eval_only;      // 1: one evaluation of pos (nsteps 1), no MD; mom and mass unused
    // host copies of the positions and element indices of an evaluation,
    // passed with the launch of the item-parallel form (null: read pos and
    // the batch's element indices from memory)
    const double* inline_pos = nullptr;
    const int* inline_elem = nullptr;
};

// packed image shift: three signed 8-bit lattice multiples
__host__ __device__ inline int pack_shift(int x, int y, int z) {
    return (x & 0xff) | ((y & 0xff) << 8) | ((z & 0xff) << 16);
}
__host__ __device__ inline void unpack_shift(int p, int& x, int& y, int& z) {
    x = (int)(signed char)(p & 0xff);
    y = (int)(signed char)((p >> 8) & 0xff);
    z = (int)(signed char)((p >> 16) & 0xff);
}

// ------------------------------------------------------------------ launchers
// Each returns the number of kernel launches it issued.
// wrap, bin, count; sid_valid: the atom -> structure map of an earlier
// evaluation of the same batch is still in place (plan replays)
int launch_neighbour_build_a(const Batch& b, const DevModel& m, cudaStream_t s, bool sid_valid = false);
int launch_scan(int* data, int n, int* tmp, int* total_out_dev, cudaStream_t s);   // exclusive scan in place, total in data[n]
int launch_scan_from(const int* src, int* data, int n, int* tmp, cudaStream_t s);  // the same from src (src may be data)
int launch_neighbour_build_b(const Batch& b, const DevModel& m, cudaStream_t s);  // fill + reverse
// Planned evaluations (no host read between the count and the fill pass):
// flag 32 and empty lists when the entries or the largest count exceed the
// capacities; molecules' boxes and grids recomputed on the device.
int launch_capacity_guard(const Batch& b, long long e_cap, int m_cap, cudaStream_t s);
int launch_molecule_boxes(const Batch& b, double rc, cudaStream_t s);
int launch_sf_values(const Batch& b, const DevModel& m, cudaStream_t s);
int launch_mlp(const Batch& b, const DevModel& m, cudaStream_t s);
int launch_sf_gradients(const Batch& b, const DevModel& m, cudaStream_t s);
int launch_forces_and_reduce(const Batch& b, const DevModel& m, int want_dEdLat, cudaStream_t s);
int launch_element_groups(const Batch& b, const DevModel& m, cudaStream_t s);
int launch_mlp_fp32(const Batch& b, const DevModel& m, cudaStream_t s);
int launch_forces_and_reduce_fp32(const Batch& b, const DevModel& m, int want_dEdLat, cudaStream_t s);
size_t mlp_smem_bytes(const DevModel& m, size_t elem);
int launch_mlp_tc(const Batch& b, const DevModel& m, cudaStream_t s);
// per-structure compensated sums of the atomic energies (FP64 or FP32 atE) into out[nstruct]
int launch_struct_energies(const Batch& b, bool fp32, double* out, cudaStream_t s);
// Committee: every member's network (acc: natoms*nsf_max accumulator of the
// working precision, Ek: K*nstruct member energies), then dE/dG = mean; the
// finish step writes the mean energies and their standard deviation.
int launch_committee_networks(const Batch& b, const Committee& cm, bool mixed, bool use_tc, void* acc, double* Ek,
                              cudaStream_t s);
int launch_committee_finish(const Batch& b, const Committee& cm, const double* Ek, cudaStream_t s);
size_t mlp_tc_smem_bytes(const DevModel& m);

size_t sf_smem_per_warp(int mmax, bool grad);
int device_sm_count();  // multiprocessors of the current device (cached per device)
// Mailbox of the resident single-block kernel (mapped pinned host memory,
// one per context): the host writes a request's inputs and then `req`; the
// kernel serves it, writes the outputs and then `ack`.  Every field has one
// writer (host: req, quit, natoms, pos, elem; kernel: ack, exited, acc,
// energy, force).
struct ResidentBox {
    volatile int req;      // sequence number of the newest request
    volatile int ack;      // sequence number of the last request served
    volatile int quit;     // 1: leave the loop now
    volatile int exited;   // 1: the kernel has left its loop
    int natoms;
    int acc[2];            // status flags of the last request, evaluations (1)
    int pad;
    double energy;
    double pos[3 * kSmallMolecule];
    int elem[kSmallMolecule];
    double force[3 * kSmallMolecule];
};
// Polls of an idle resident kernel before it exits (each poll a read of
// host memory, about a microsecond: a few milliseconds).
constexpr int kResidentPolls = 4000;

size_t small_md_smem_bytes(const DevModel& m, int natoms);  // dynamic shared memory of the kernel
// true when the item-parallel form runs: it reads its inputs once into
// shared memory and writes its outputs once (host-mapped buffers are fine)
bool small_md_tiny(const DevModel& m, int natoms);
int launch_small_md(const Batch& b, const DevModel& m, const SmallMdArgs& a, cudaStream_t s);
// The item-parallel single-block kernel in resident mode for molecules of
// `natoms` atoms: it serves evaluation requests from the mailbox `box` (its
// device address) until `quit` or until it has polled kResidentPolls times
// without a request.  Returns 0 if the molecule does not take the
// item-parallel form.
int launch_small_resident(const DevModel& m, int natoms, ResidentBox* box, cudaStream_t s);

// Compiled product-space shapes of the fast SF kernels: id -> (NL, NZ, NE).
// Ids 1-4 read zeta from the model; ids 5-6 have the zeta set compiled in
// (kFastZeta) and are preferred when the potential's zeta set matches.
constexpr int kNumFastShapes = 7;
constexpr int kFastShapes[kNumFastShapes][3] = {{0, 0, 0}, {2, 2, 1}, {2, 4, 2}, {2, 4, 4},
                                                {2, 8, 2}, {2, 2, 1}, {2, 4, 2}};
constexpr int kFastZeta[kNumFastShapes][4] = {{0}, {0}, {0}, {0}, {0}, {1, 4, 0, 0}, {1, 2, 4, 16}};
inline int fast_shape_p(int id) { return kFastShapes[id][0] * kFastShapes[id][1] * kFastShapes[id][2]; }

// Fast (product-space) symmetry-function kernels, FP64 (T = double) or FP32.
int launch_sf_values_fast(const Batch& b, const DevModel& m, bool fp32, cudaStream_t s);
int launch_sf_gradients_fast(const Batch& b, const DevModel& m, bool fp32, cudaStream_t s);
size_t sf_fast_smem_per_warp(int mmax, int g2max, int nblk, int P, bool grad, bool fp32);

}  // namespace hdnnp

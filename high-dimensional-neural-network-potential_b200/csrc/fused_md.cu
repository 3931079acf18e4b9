// fused_md.cu -- velocity-Verlet MD of one small molecule in ONE kernel launch.
//
// The reference's example runs MD of an 8-atom molecule, one
// hdnnpEnergyAndForces call per step (src/potentials/hdnnpExample.f90:58-64).
// Through the general pipeline such a step is ~26 tiny kernels, so its time is
// launch and pipeline latency, not work.  Here one thread block runs every
// stage of every step of a launch -- kick + drift, neighbour lists, symmetry
// functions, networks, gradients, forces -- separated by block barriers, with
// the per-atom routines of the generic symmetry-function kernels
// (symfn_generic.cuh).  Molecules only (no images), at most 64 atoms, FP64.
//
// Latency is the cost, so the state of the molecule (positions, momenta,
// forces) stays in shared memory for the whole launch and the per-step arrays
// are placed there too, in order of how often they are read, as far as the
// 227 KB allow (the rest stay in the plan's global scratch):
//   * neighbour lists from one 64-bit mask per atom (warp ballots over the
//     candidates): counts are popcounts, the reverse entry of (i -> j) is
//     off[j] + popc(mask[j] below i) -- no search;
//   * the networks of all atoms in one pass (rows of any element; the layer
//     widths are common to the elements, the input width is the element's),
//     reading G where the symmetry-function pass wrote it.
// Neighbours are listed in atom-index order (the reference walks its cell
// grid; for a molecule both give the same set, the sums differ only in
// rounding).
#include <atomic>

#include "engine.h"
#include "mlp_tile.cuh"
#include "symfn_generic.cuh"

namespace hdnnp {

namespace {

// arrays of one step; the first kMandatory always live in shared memory
enum Slot {
    kPos, kMom, kForce, kFprev, kMass, kElem, kSid, kOff, kAtE, kGself, kInfo, kStatus,
    kNeiJ, kNeiRev, kNeiS, kG, kDEdG, kGent, kVir, kSlots
};
constexpr int kMandatory = kNeiJ;

struct FusedArgs {
    int natoms, nsteps, mm, rows, maxw;  // rows: network rows per pass
    double dt, rc2;
    size_t warp_bytes;                   // symmetry-function shared memory per warp
    int slot[kSlots];                    // byte offset in dynamic shared memory, -1: global scratch
    double* pos;
    double* mom;
    const double* mass;
    double* force;
    double* energy;
    double* hist;                        // [nsteps] or null
    int* acc;                            // [2]: OR of status flags, evaluations
    int eval_only;                       // 1: one evaluation of pos, no MD (mom, mass unused)
};

template <typename P>
__device__ __forceinline__ void place(P*& p, unsigned char* smem, int off) {
    if (off >= 0) p = reinterpret_cast<P*>(smem + off);
}

// Networks (forward and dE/dG) of atoms r0 .. r0+R-1 in one pass over the
// layers; activations in buf.  Per row the same arithmetic, in the same
// order, as mlp_tile (one element tile of the batched kernel).
__device__ __forceinline__ void mlp_rows(const Batch& b, const DevModel& m, int r0, int R, int maxw, double* buf) {
    const int L = m.nlayers, tid = threadIdx.x, nt = blockDim.x;
    double* cb[8];
    double* yb[8];
    double* p = buf;
    for (int l = 0; l < L; ++l) {
        cb[l] = p;
        p += R * m.width[l + 1];
        yb[l] = p;
        p += R * m.width[l + 1];
    }
    double* dcur = p;
    double* dnext = p + R * maxw;
    for (int l = 0; l < L; ++l) {
        const int wout = m.width[l + 1];
        const char act = m.act[l];
        for (int idx = tid; idx < R * wout; idx += nt) {
            const int a = idx / wout, o = idx % wout, atom = r0 + a, e = b.elem[atom];
            const double* WT = m.wt + m.w_off[e * L + l];
            const double* in;
            int win;
            if (l == 0) {
                in = b.G + (size_t)atom * m.nsf_max;
                win = m.nin_el[e];
            } else {
                in = yb[l - 1] + a * m.width[l];
                win = m.width[l];
            }
            double s = 0.0;
            for (int i = 0; i < win; ++i) s += WT[(size_t)i * wout + o] * in[i];
            const double c = s + m.b[m.b_off[e * L + l] + o];
            cb[l][idx] = c;
            yb[l][idx] = act_f(act, c);
        }
        __syncthreads();
    }
    {
        const int w = m.width[L];
        for (int a = tid; a < R; a += nt) b.atE[r0 + a] = yb[L - 1][a * w] + m.atom_energy[b.elem[r0 + a]];
        for (int idx = tid; idx < R * w; idx += nt) dcur[idx] = act_d(m.act[L - 1], cb[L - 1][idx], yb[L - 1][idx]);
    }
    __syncthreads();
    for (int l = L - 1; l >= 0; --l) {
        const int wout = m.width[l + 1];
        const int W = (l == 0) ? m.nsf_max : m.width[l];
        for (int idx = tid; idx < R * W; idx += nt) {
            const int a = idx / W, i = idx % W, atom = r0 + a, e = b.elem[atom];
            const int wi = (l == 0) ? m.nin_el[e] : W;
            if (i >= wi) continue;
            const double* Wm = m.w + m.w_off[e * L + l];
            const double* da = dcur + a * wout;
            double s = 0.0;
            for (int o = 0; o < wout; ++o) s += da[o] * Wm[(size_t)o * wi + i];
            if (l == 0)
                b.dEdG[(size_t)atom * m.nsf_max + i] = s;
            else
                dnext[a * W + i] = s * act_d(m.act[l - 1], cb[l - 1][a * W + i], yb[l - 1][a * W + i]);
        }
        __syncthreads();
        double* t = dcur;
        dcur = dnext;
        dnext = t;
    }
}

template <int GM>
__global__ void __launch_bounds__(kThreads, 1) k_small_md(Batch g, DevModel m, FusedArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long mask[kSmallMolecule];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    const int N = a.natoms, n3 = 3 * N;
    const double dt = a.dt;
    // the step's arrays: shared memory where the layout put them
    Batch b = g;
    double *pos = nullptr, *mom = nullptr, *F = nullptr, *Fp = nullptr, *mass = nullptr;
    StructInfo* info = nullptr;
    place(pos, smem, a.slot[kPos]);
    place(mom, smem, a.slot[kMom]);
    place(F, smem, a.slot[kForce]);
    place(Fp, smem, a.slot[kFprev]);
    place(mass, smem, a.slot[kMass]);
    place(b.elem, smem, a.slot[kElem]);
    place(b.sid, smem, a.slot[kSid]);
    place(b.nei_off, smem, a.slot[kOff]);
    place(b.atE, smem, a.slot[kAtE]);
    place(b.gself, smem, a.slot[kGself]);
    place(info, smem, a.slot[kInfo]);
    place(b.status, smem, a.slot[kStatus]);
    place(b.nei_j, smem, a.slot[kNeiJ]);
    place(b.nei_rev, smem, a.slot[kNeiRev]);
    place(b.nei_s, smem, a.slot[kNeiS]);
    place(b.G, smem, a.slot[kG]);
    place(b.dEdG, smem, a.slot[kDEdG]);
    place(b.gent, smem, a.slot[kGent]);
    place(b.vir, smem, a.slot[kVir]);
    b.info = info;
    b.wpos = pos;
    b.stats = nullptr;
    for (int q = tid; q < n3; q += blockDim.x) {
        pos[q] = a.pos[q];
        mom[q] = a.eval_only ? 0.0 : a.mom[q];
        F[q] = a.eval_only ? 0.0 : a.force[q];
    }
    for (int i = tid; i < N; i += blockDim.x) {
        mass[i] = a.eval_only ? 1.0 : a.mass[i];
        b.elem[i] = g.elem[i];
        b.sid[i] = 0;
    }
    if (tid < (int)(sizeof(StructInfo) / sizeof(int)))
        reinterpret_cast<int*>(info)[tid] = reinterpret_cast<const int*>(g.info)[tid];
    if (tid == 0) b.status[0] = 0;
    __syncthreads();
    for (int step = 0; step < a.nsteps; ++step) {
        // kick of the previous step and drift (hdnnpExample.f90:61-64),
        // element by element in the same thread
        for (int q = tid; q < n3; q += blockDim.x) {
            if (a.eval_only) {  // positions as given
                if (!isfinite(pos[q])) atomicOr(b.status, 8);
                continue;
            }
            const double mi = mass[q / 3];
            double p = mom[q];
            if (step > 0) p += 0.5 * dt * (F[q] + Fp[q]);
            mom[q] = p;
            const double x = pos[q] + (p / mi * dt + 0.5 * F[q] / mi * dt * dt);
            if (!isfinite(x)) atomicOr(b.status, 8);  // the list build's non-finite flag
            pos[q] = x;
            Fp[q] = F[q];
        }
        __syncthreads();
        // neighbour masks: one warp per atom, ballots over the candidates
        for (int i = w; i < N; i += nw) {
            const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
            unsigned long long mk = 0;
            for (int c = 0; c < N; c += 32) {
                const int j = c + lane;
                bool in = false;
                if (j < N && j != i) {
                    const double dx = xi - pos[3 * j], dy = yi - pos[3 * j + 1], dz = zi - pos[3 * j + 2];
                    in = dx * dx + dy * dy + dz * dz < a.rc2;
                }
                mk |= (unsigned long long)__ballot_sync(0xffffffffu, in) << c;
            }
            if (lane == 0) mask[i] = mk;
        }
        __syncthreads();
        // offsets: warp 0 scans the counts (two atoms per lane)
        if (w == 0) {
            const int i0 = 2 * lane, i1 = 2 * lane + 1;
            const int c0 = i0 < N ? __popcll(mask[i0]) : 0, c1 = i1 < N ? __popcll(mask[i1]) : 0;
            int incl = c0 + c1;
            for (int d = 1; d < 32; d <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += t;
            }
            const int excl = incl - c0 - c1;
            if (i0 < N) b.nei_off[i0] = excl;
            if (i1 < N) b.nei_off[i1] = excl + c0;
            if (lane == 31) b.nei_off[N] = incl;
        }
        __syncthreads();
        // entries in index order; reverse entry without search
        for (int i = w; i < N; i += nw) {
            const unsigned long long mi = mask[i];
            const int o = b.nei_off[i];
            for (int c = 0; c < N; c += 32) {
                const int j = c + lane;
                if (j < N && ((mi >> j) & 1ull)) {
                    const int e = o + __popcll(mi & ((1ull << j) - 1ull));
                    b.nei_j[e] = j;
                    b.nei_s[e] = 0;
                    b.nei_rev[e] = b.nei_off[j] + __popcll(mask[j] & ((1ull << i) - 1ull));
                }
            }
        }
        __syncthreads();
        // symmetry functions (one warp per atom)
        {
            Smem<double> s = carve<double>(smem + w * a.warp_bytes, a.mm, m.nsf_max, false);
            for (int i = w; i < N; i += nw) sfv_atom<GM>(b, m, a.mm, s, i, lane);
        }
        __syncthreads();
        // networks of all atoms, a.rows per pass
        for (int r0 = 0; r0 < N; r0 += a.rows)
            mlp_rows(b, m, r0, N - r0 < a.rows ? N - r0 : a.rows, a.maxw, reinterpret_cast<double*>(smem));
        // dE/dG-weighted gradients
        {
            Smem<double> s = carve<double>(smem + w * a.warp_bytes, a.mm, m.nsf_max, true);
            for (int i = w; i < N; i += nw) sfg_atom(b, m, a.mm, s, i, lane);
        }
        __syncthreads();
        // forces F_i = -(g_self(i) + sum of the reverse entries); the last
        // thread sums the energy (Neumaier) meanwhile
        for (int i = tid; i < N; i += blockDim.x) {
            double fx = b.gself[3 * i], fy = b.gself[3 * i + 1], fz = b.gself[3 * i + 2];
            for (int e = b.nei_off[i]; e < b.nei_off[i + 1]; ++e) {
                const int r = b.nei_rev[e];
                fx += b.gent[3 * r];
                fy += b.gent[3 * r + 1];
                fz += b.gent[3 * r + 2];
            }
            F[3 * i] = -fx;
            F[3 * i + 1] = -fy;
            F[3 * i + 2] = -fz;
        }
        if (tid == blockDim.x - 1) {
            double sum = 0.0, c = 0.0;
            for (int i = 0; i < N; ++i) {
                const double x = b.atE[i], t = sum + x;
                c += fabs(sum) >= fabs(x) ? (sum - t) + x : (x - t) + sum;
                sum = t;
            }
            if (a.hist) a.hist[step] = sum + c;
            if (step == a.nsteps - 1) a.energy[0] = sum + c;
        }
        __syncthreads();
    }
    // last kick; the state back to the plan's arrays
    for (int q = tid; q < n3; q += blockDim.x) {
        if (!a.eval_only) {
            a.mom[q] = mom[q] + 0.5 * dt * (F[q] + Fp[q]);
            a.pos[q] = pos[q];
        }
        a.force[q] = F[q];
    }
    if (tid == 0) {
        a.acc[0] |= b.status[0];
        a.acc[1] += a.nsteps;
    }
}

size_t align16z(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared-memory layout: the work area (per-warp symmetry-function staging or
// the network activations) first, then the step's arrays while they fit.
size_t small_md_layout(const DevModel& m, int N, FusedArgs* a) {
    const int mm = ((N - 1 + 31) / 32) * 32 < 32 ? 32 : ((N - 1 + 31) / 32) * 32;
    const size_t wb = warp_bytes<double>(mm, m.nsf_max, true);
    size_t row = 0;
    int maxw = 1;
    for (int l = 0; l < m.nlayers; ++l) {
        row += 2 * (size_t)m.width[l + 1];
        maxw = m.width[l + 1] > maxw ? m.width[l + 1] : maxw;
    }
    row = (row + 2 * (size_t)maxw) * sizeof(double);
    size_t work = wb * (kThreads / 32);
    const size_t rows_min = N < 32 ? (size_t)N : 32;
    if (row * rows_min > work) work = row * rows_min;
    const int rows = (int)((work / row) < (size_t)N ? work / row : (size_t)N);
    const size_t n = (size_t)N, NN = n * n, nsf = (size_t)m.nsf_max;
    const size_t bytes[kSlots] = {24 * n,     24 * n,     24 * n, 24 * n,         8 * n,          4 * n,
                                  4 * n,      4 * (n + 1), 8 * n, 24 * n,         sizeof(StructInfo), 16,
                                  4 * NN,     4 * NN,     4 * NN, 8 * n * nsf,    8 * n * nsf,    24 * NN,
                                  72 * n};
    const size_t budget = 226 * 1024;
    size_t off = align16z(work);
    for (int k = 0; k < kSlots; ++k) {
        const size_t sz = align16z(bytes[k]);
        if (k < kMandatory || off + sz <= budget) {
            if (a) a->slot[k] = (int)off;
            off += sz;
        } else if (a) {
            a->slot[k] = -1;
        }
    }
    if (a) {
        a->mm = mm;
        a->rows = rows;
        a->maxw = maxw;
        a->warp_bytes = wb;
    }
    return off;
}

// ---------------------------------------------------------------------------
// Item-parallel form for molecules whose whole step fits in shared memory
// (the reference's 8-atom example and other molecules of a few atoms).  A warp
// per atom leaves most lanes idle when an atom has a handful of neighbours, so
// every stage here hands out one small item per thread instead -- a list
// entry, an angular pair (j, k) of one centre, or one (atom, symmetry
// function) -- and every sum is taken in a fixed order by one thread
// (deterministic):
//   entries: geometry, cutoff and the radial exponentials of the entry's
//            (centre, neighbour element) group;
//   pairs:   the angular geometry of (j, k) (oriented like the element pair
//            block: j of its first element) and, per function of the block,
//            exp(-eta (rij^2 + rik^2 + rjk^2)) and (1 + lambda cos)^(zeta-1);
//   values:  G of one (atom, function) from the entry / pair terms;
//   network: one (atom, neuron) per thread, layer by layer; stores
//            dE/dG / width;
//   pair gradients: the d/dr_j and d/dr_k parts of one pair (no
//            transcendental: the pair stage kept them);
//   entry gradients: radial part + the pair parts of one entry.
// The formulas are those of the generic per-atom routines (symfn_generic.cuh,
// after symmetryFunctions.f90:129-297 of the reference).

enum TSlot {
    tPos, tMom, tF, tFp, tMass, tAtE, tG, tW, tEG, tERC, tGent, tPS, tPE, tPT, tPG, tMlp,
    tMask, tElem, tOff, tPoff, tNJ, tRev, tOwn, tPblk, tPjk, tRecBlk, tBlkOf, tStatus, tSlots
};

struct TinyArgs {
    int natoms, nsteps, g2w, g4w, maxw;
    double dt, rc2;                 // list cutoff^2
    int slot[tSlots];               // byte offsets in dynamic shared memory
    double* pos;
    double* mom;
    const double* mass;
    double* force;
    double* energy;
    double* hist;
    int* acc;
    const int* elem;
    int eval_only;                  // 1: one evaluation of pos, no MD (mom, mass unused)
    // 1: positions and element indices are the copies below, passed with the
    // launch (the plain call of one molecule: no copy and no read of host
    // memory from the kernel)
    int inline_in;
    double in_pos[3 * kSmallMolecule];
    int in_elem[kSmallMolecule];
    // resident mode: serve evaluation requests from this mailbox (device
    // address of mapped host memory) until told to quit or idle
    ResidentBox* box;
};

// pair r of one centre's list (0 <= p < q): r = q (q - 1) / 2 + p
__device__ __forceinline__ void tri_pair(int r, int& p, int& q) {
    int t = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)r)) * 0.5f);
    while (t * (t - 1) / 2 > r) --t;
    while ((t + 1) * t / 2 <= r) ++t;
    q = t;
    p = r - t * (t - 1) / 2;
}

// largest i in [0, n) with off[i] <= x (off nondecreasing, off[0] = 0)
__device__ __forceinline__ int owner_of(const int* off, int n, int x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kThreads, 1) k_tiny_md(DevModel m, TinyArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
    const int N = a.natoms, n3 = 3 * N, nel = m.nel, nblk = m.nblk, nsf = m.nsf_max;
    const int g2w = a.g2w, g4w = a.g4w;
    const double dt = a.dt;
    double* pos = (double*)(smem + a.slot[tPos]);
    double* mom = (double*)(smem + a.slot[tMom]);
    double* F = (double*)(smem + a.slot[tF]);
    double* Fp = (double*)(smem + a.slot[tFp]);
    double* mass = (double*)(smem + a.slot[tMass]);
    double* atE = (double*)(smem + a.slot[tAtE]);
    double* G = (double*)(smem + a.slot[tG]);
    double* Wt = (double*)(smem + a.slot[tW]);       // dE/dG / width
    double* eg = (double*)(smem + a.slot[tEG]);      // per entry: dx dy dz r fc dfc
    double* erc = (double*)(smem + a.slot[tERC]);    // per entry: radial exponentials
    double* gent = (double*)(smem + a.slot[tGent]);  // per entry: dE_i/dr_j
    double* ps = (double*)(smem + a.slot[tPS]);      // per pair: fjk dfjk t1 cos fcp
    double* pe = (double*)(smem + a.slot[tPE]);      // per pair and function: exp
    double* pt = (double*)(smem + a.slot[tPT]);      // per pair and function: base^(zeta-1)
    double* pg = (double*)(smem + a.slot[tPG]);      // per pair: d/dr_j, d/dr_k
    double* mlp = (double*)(smem + a.slot[tMlp]);
    unsigned long long* mask = (unsigned long long*)(smem + a.slot[tMask]);
    int* elem = (int*)(smem + a.slot[tElem]);
    int* off = (int*)(smem + a.slot[tOff]);
    int* poff = (int*)(smem + a.slot[tPoff]);
    int* nj = (int*)(smem + a.slot[tNJ]);
    int* rev = (int*)(smem + a.slot[tRev]);
    int* own = (int*)(smem + a.slot[tOwn]);
    int* pblk = (int*)(smem + a.slot[tPblk]);        // block | swap << 8, or -1
    int* pjk = (int*)(smem + a.slot[tPjk]);          // entry of j | entry of k << 16
    int* recblk = (int*)(smem + a.slot[tRecBlk]);    // block of each angular record
    int* blkof = (int*)(smem + a.slot[tBlkOf]);      // block of an element pair
    int* status = (int*)(smem + a.slot[tStatus]);
    for (int x = tid; x < nel * nblk; x += nt)
        for (int g = m.g4_off[x]; g < m.g4_off[x + 1]; ++g) recblk[g] = x % nblk;
    for (int t = tid; t < nblk; t += nt) {
        blkof[m.blk_a[t] * nel + m.blk_b[t]] = t;
        blkof[m.blk_b[t] * nel + m.blk_a[t]] = t;
    }
    // Resident mode: one round per request of the mailbox.  Thread 0 polls
    // (bounded: kResidentPolls reads of host memory, then the kernel exits)
    // and broadcasts the request through shared memory; -1 ends the loop.
    ResidentBox* box = a.box;
    int served = box ? box->ack : 0;
    int* cmd = status + 1;
    for (int round = 0;; ++round) {
        if (box) {
            if (tid == 0) {
                // one read of host memory per poll (about a microsecond over
                // the bus); the quit flag every 16 polls
                int r = -1;
                for (int it = 0; it < kResidentPolls; ++it) {
                    const int q = box->req;
                    if (q != served) {
                        r = q;
                        break;
                    }
                    if ((it & 15) == 15 && box->quit) break;
                }
                __threadfence_system();  // the request's inputs are read after its number
                cmd[0] = r;
            }
            __syncthreads();
            const int r = cmd[0];
            __syncthreads();
            if (r < 0) break;
            served = r;
        } else if (round > 0) {
            break;
        }
    // a request's inputs are read past the caches (the host rewrites them)
    for (int q = tid; q < n3; q += nt) {
        pos[q] = a.inline_in ? a.in_pos[q] : box ? ((volatile const double*)a.pos)[q] : a.pos[q];
        mom[q] = a.eval_only ? 0.0 : a.mom[q];
        F[q] = a.eval_only ? 0.0 : a.force[q];
    }
    for (int i = tid; i < N; i += nt) {
        mass[i] = a.eval_only ? 1.0 : a.mass[i];
        elem[i] = a.inline_in ? a.in_elem[i] : box ? ((volatile const int*)a.elem)[i] : a.elem[i];
    }
    if (tid == 0) status[0] = 0;
    __syncthreads();
    for (int step = 0; step < a.nsteps; ++step) {
        // kick of the previous step and drift (hdnnpExample.f90:61-64)
        for (int q = tid; q < n3; q += nt) {
            if (a.eval_only) {  // positions as given
                if (!isfinite(pos[q])) atomicOr(status, 8);
                continue;
            }
            const double mi = mass[q / 3];
            double p = mom[q];
            if (step > 0) p += 0.5 * dt * (F[q] + Fp[q]);
            mom[q] = p;
            const double x = pos[q] + (p / mi * dt + 0.5 * F[q] / mi * dt * dt);
            if (!isfinite(x)) atomicOr(status, 8);
            pos[q] = x;
            Fp[q] = F[q];
        }
        __syncthreads();
        // neighbour masks (warp per atom)
        for (int i = w; i < N; i += nw) {
            const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
            unsigned long long mk = 0;
            for (int c = 0; c < N; c += 32) {
                const int j = c + lane;
                bool in = false;
                if (j < N && j != i) {
                    const double dx = xi - pos[3 * j], dy = yi - pos[3 * j + 1], dz = zi - pos[3 * j + 2];
                    in = dx * dx + dy * dy + dz * dz < a.rc2;
                }
                mk |= (unsigned long long)__ballot_sync(0xffffffffu, in) << c;
            }
            if (lane == 0) mask[i] = mk;
        }
        __syncthreads();
        // entry and pair offsets (warp 0, two atoms per lane)
        if (w == 0) {
            const int i0 = 2 * lane, i1 = 2 * lane + 1;
            const int c0 = i0 < N ? __popcll(mask[i0]) : 0, c1 = i1 < N ? __popcll(mask[i1]) : 0;
            const int q0 = c0 * (c0 - 1) / 2, q1 = c1 * (c1 - 1) / 2;
            int ie = c0 + c1, ip = q0 + q1;
            for (int d = 1; d < 32; d <<= 1) {
                const int te = __shfl_up_sync(0xffffffffu, ie, d), tp = __shfl_up_sync(0xffffffffu, ip, d);
                if (lane >= d) {
                    ie += te;
                    ip += tp;
                }
            }
            const int xe = ie - c0 - c1, xp = ip - q0 - q1;
            if (i0 < N) {
                off[i0] = xe;
                poff[i0] = xp;
            }
            if (i1 < N) {
                off[i1] = xe + c0;
                poff[i1] = xp + q0;
            }
            if (lane == 31) {
                off[N] = ie;
                poff[N] = ip;
            }
        }
        __syncthreads();
        // entries: index order, reverse entry by popcount, geometry, radial exponentials
        for (int i = w; i < N; i += nw) {
            const unsigned long long mi = mask[i];
            const int o = off[i], c = elem[i];
            const double rc = m.rc[c];
            const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
            for (int cc = 0; cc < N; cc += 32) {
                const int j = cc + lane;
                if (j < N && ((mi >> j) & 1ull)) {
                    const int e = o + __popcll(mi & ((1ull << j) - 1ull));
                    nj[e] = j;
                    own[e] = i;
                    rev[e] = off[j] + __popcll(mask[j] & ((1ull << i) - 1ull));
                    const double dx = xi - pos[3 * j], dy = yi - pos[3 * j + 1], dz = zi - pos[3 * j + 2];
                    const double r = sqrt(dx * dx + dy * dy + dz * dz);
                    double fc, dfc;
                    cutoff(r, rc, fc, dfc);
                    double* ge = eg + 6 * e;
                    ge[0] = dx;
                    ge[1] = dy;
                    ge[2] = dz;
                    ge[3] = r;
                    ge[4] = fc;
                    ge[5] = dfc;
                    const int el = elem[j], f0 = m.g2_off[c * nel + el], f1 = m.g2_off[c * nel + el + 1];
                    for (int f = f0; f < f1; ++f) {
                        const SF2 q = m.g2[f];
                        const double x = r - q.rs;
                        erc[(size_t)e * g2w + (f - f0)] = exp(-q.eta * x * x);
                    }
                }
            }
        }
        __syncthreads();
        // angular pairs
        const int npair = poff[N];
        for (int P = tid; P < npair; P += nt) {
            const int i = owner_of(poff, N, P);
            int p, q;
            tri_pair(P - poff[i], p, q);
            const int ep = off[i] + p, eq = off[i] + q, c = elem[i];
            const int elp = elem[nj[ep]], elq = elem[nj[eq]];
            const int t = blkof[elp * nel + elq];
            const int gb = m.g4_off[c * nblk + t], ge = m.g4_off[c * nblk + t + 1];
            pblk[P] = -1;
            if (gb == ge) continue;
            const bool swap = elp != elq && elp != m.blk_a[t];
            const int j = swap ? eq : ep, k = swap ? ep : eq;
            const double* aj = eg + 6 * j;
            const double* ak = eg + 6 * k;
            const double cx = ak[0] - aj[0], cy = ak[1] - aj[1], cz = ak[2] - aj[2];
            const double mrc = m.rc[c];
            const double rjk2 = cx * cx + cy * cy + cz * cz;
            if (!(rjk2 < mrc * mrc)) continue;
            const double rj = aj[3], rk = ak[3];
            const double rjk = sqrt(rjk2);
            double fjk, dfjk;
            cutoff(rjk, mrc, fjk, dfjk);
            const double t1 = -1.0 / (rj * rk);
            const double cth = 0.5 * (rjk * rjk - rj * rj - rk * rk) * t1;
            const double fcp = aj[4] * ak[4] * fjk;
            const double rsum = rj * rj + rk * rk + rjk * rjk;
            double last_eta = -1.0, ex = 0.0;
            for (int u = 0; u < ge - gb; ++u) {
                const SF4 f = m.g4[gb + u];
                if (f.eta != last_eta) {
                    ex = exp(-f.eta * rsum);
                    last_eta = f.eta;
                }
                const double base = 1.0 + f.lambda * cth;
                pe[(size_t)P * g4w + u] = ex;
                pt[(size_t)P * g4w + u] = f.izeta >= 0 ? ipow(base, f.izeta - 1) : pow(base, f.zeta - 1.0);
            }
            double* s = ps + 5 * (size_t)P;
            s[0] = fjk;
            s[1] = dfjk;
            s[2] = t1;
            s[3] = cth;
            s[4] = fcp;
            pblk[P] = t | (swap ? 256 : 0);
            pjk[P] = j | (k << 16);
        }
        __syncthreads();
        // symmetry-function values, one (atom, function) per thread
        for (int x = tid; x < N * nsf; x += nt) {
            const int i = x / nsf, u = x - i * nsf, c = elem[i];
            const int r0 = m.g2_off[c * nel], n2 = m.g2_off[c * nel + nel] - r0;
            const int a0 = m.g4_off[c * nblk], n4 = m.g4_off[c * nblk + nblk] - a0;
            double acc = 0.0;
            int sf;
            if (u < n2) {
                const SF2 q = m.g2[r0 + u];
                const int f0 = m.g2_off[c * nel + q.nel], col = r0 + u - f0;
                for (int e = off[i]; e < off[i + 1]; ++e)
                    if (elem[nj[e]] == q.nel) acc += erc[(size_t)e * g2w + col] * eg[6 * e + 4];
                sf = q.sf;
            } else if (u < n2 + n4) {
                const int g = a0 + u - n2, t = recblk[g], col = g - m.g4_off[c * nblk + t];
                const SF4 f = m.g4[g];
                for (int P = poff[i]; P < poff[i + 1]; ++P) {
                    const int pb = pblk[P];
                    if (pb < 0 || (pb & 255) != t) continue;
                    const double* s = ps + 5 * (size_t)P;
                    const double base = 1.0 + f.lambda * s[3];
                    acc += f.pf * (pt[(size_t)P * g4w + col] * base) * pe[(size_t)P * g4w + col] * s[4];
                }
                sf = f.sf;
            } else {
                continue;
            }
            const size_t k = (size_t)c * nsf + sf;
            G[(size_t)i * nsf + sf] = (acc - m.smean[k]) / m.swidth[k];
        }
        __syncthreads();
        // networks: one (atom, neuron) per thread and layer; activations in mlp
        {
            const int L = m.nlayers;
            int lo = 0;  // offset of layer l's pre-activations in mlp (N rows)
            for (int l = 0; l < L; ++l) {
                const int wout = m.width[l + 1];
                const int win = l == 0 ? 0 : m.width[l];
                const double* yin = mlp + lo - N * win;  // previous layer's activations
                double* cb = mlp + lo;
                double* yb = cb + N * wout;
                const char act = m.act[l];
                for (int x = tid; x < N * wout; x += nt) {
                    const int i = x / wout, o = x - i * wout, e = elem[i];
                    const double* WT = m.wt + m.w_off[e * L + l];
                    const double* in = l == 0 ? G + (size_t)i * nsf : yin + i * win;
                    const int n = l == 0 ? m.nin_el[e] : win;
                    double s = 0.0;
                    for (int k = 0; k < n; ++k) s += WT[(size_t)k * wout + o] * in[k];
                    const double cv = s + m.b[m.b_off[e * L + l] + o];
                    cb[x] = cv;
                    yb[x] = act_f(act, cv);
                }
                lo += 2 * N * wout;
                __syncthreads();
            }
            // output layer: atomic energy and the delta of the output neuron
            const int wl = m.width[L];
            const double* cl = mlp + lo - 2 * N * wl;
            const double* yl = cl + N * wl;
            double* d0 = mlp + lo;
            double* d1 = d0 + N * a.maxw;
            for (int i = tid; i < N; i += nt) atE[i] = yl[i * wl] + m.atom_energy[elem[i]];
            for (int x = tid; x < N * wl; x += nt) d0[x] = act_d(m.act[L - 1], cl[x], yl[x]);
            __syncthreads();
            for (int l = L - 1; l >= 0; --l) {
                const int wout = m.width[l + 1];
                lo -= 2 * N * wout;  // now the offset of layer l
                const int W = l == 0 ? nsf : m.width[l];
                const double* cp = mlp + lo - 2 * N * W;  // layer l-1 (when l > 0)
                const double* yp = cp + N * W;
                for (int x = tid; x < N * W; x += nt) {
                    const int i = x / W, k = x - i * W, e = elem[i];
                    const int wi = l == 0 ? m.nin_el[e] : W;
                    if (k >= wi) continue;
                    const double* Wm = m.w + m.w_off[e * L + l];
                    const double* da = d0 + i * wout;
                    double s = 0.0;
                    for (int o = 0; o < wout; ++o) s += da[o] * Wm[(size_t)o * wi + k];
                    if (l == 0)
                        Wt[(size_t)i * nsf + k] = s / m.swidth[(size_t)e * nsf + k];
                    else
                        d1[x] = s * act_d(m.act[l - 1], cp[x], yp[x]);
                }
                __syncthreads();
                double* tmp = d0;
                d0 = d1;
                d1 = tmp;
            }
        }
        // pair gradients: d/dr_j and d/dr_k of one pair's terms
        for (int P = tid; P < npair; P += nt) {
            const int pb = pblk[P];
            if (pb < 0) continue;
            const int t = pb & 255, jk = pjk[P], j = jk & 0xffff, k = jk >> 16;
            const int i = own[j], c = elem[i];
            const int gb = m.g4_off[c * nblk + t], ge = m.g4_off[c * nblk + t + 1];
            const double* aj = eg + 6 * j;
            const double* ak = eg + 6 * k;
            const double* s = ps + 5 * (size_t)P;
            const double ajx = aj[0], ajy = aj[1], ajz = aj[2], akx = ak[0], aky = ak[1], akz = ak[2];
            const double rj = aj[3], rk = ak[3], fj = aj[4], fk = ak[4], dfj = aj[5], dfk = ak[5];
            const double cx = akx - ajx, cy = aky - ajy, cz = akz - ajz;
            const double fjk = s[0], dfjk = s[1], t1 = s[2], cth = s[3], fcp = s[4];
            const double dot = ajx * akx + ajy * aky + ajz * akz;
            const double cj = dot / (rj * rj * rj * rk), ck = dot / (rk * rk * rk * rj);
            double A = 0.0, B = 0.0, C = 0.0;
            for (int u = 0; u < ge - gb; ++u) {
                const SF4 f = m.g4[gb + u];
                const double t2 = pt[(size_t)P * g4w + u];
                const double wpe = Wt[(size_t)i * nsf + f.sf] * f.pf * pe[(size_t)P * g4w + u];
                const double cp = t2 * (1.0 + f.lambda * cth);
                A += wpe * cp;
                B += wpe * cp * f.eta;
                C += wpe * t2 * f.lambda * f.zeta;
            }
            const double B2 = 2.0 * B * fcp, Cf = C * fcp;
            double* g = pg + 6 * (size_t)P;
            g[0] = A * fk * (dfjk * cx * fj - dfj * ajx * fjk) + B2 * (ajx - cx) + Cf * (t1 * akx + ajx * cj);
            g[1] = A * fk * (dfjk * cy * fj - dfj * ajy * fjk) + B2 * (ajy - cy) + Cf * (t1 * aky + ajy * cj);
            g[2] = A * fk * (dfjk * cz * fj - dfj * ajz * fjk) + B2 * (ajz - cz) + Cf * (t1 * akz + ajz * cj);
            g[3] = -A * fj * (dfjk * cx * fk + dfk * akx * fjk) + B2 * (akx + cx) + Cf * (t1 * ajx + akx * ck);
            g[4] = -A * fj * (dfjk * cy * fk + dfk * aky * fjk) + B2 * (aky + cy) + Cf * (t1 * ajy + aky * ck);
            g[5] = -A * fj * (dfjk * cz * fk + dfk * akz * fjk) + B2 * (akz + cz) + Cf * (t1 * ajz + akz * ck);
        }
        __syncthreads();
        // entry gradients: radial part, then the pair parts in pair order
        const int nent = off[N];
        for (int e = tid; e < nent; e += nt) {
            const int i = own[e], c = elem[i], p = e - off[i], M = off[i + 1] - off[i];
            const int el = elem[nj[e]], f0 = m.g2_off[c * nel + el], f1 = m.g2_off[c * nel + el + 1];
            const double* ge = eg + 6 * e;
            const double r = ge[3], fc = ge[4], dfc = ge[5];
            double coef = 0.0;
            for (int f = f0; f < f1; ++f) {
                const SF2 q = m.g2[f];
                const double x = r - q.rs;
                const double ex = erc[(size_t)e * g2w + (f - f0)];
                coef += Wt[(size_t)i * nsf + q.sf] * (-ex * dfc + 2.0 * q.eta * x / r * ex * fc);
            }
            double gx = coef * ge[0], gy = coef * ge[1], gz = coef * ge[2];
            for (int qq = 0; qq < M; ++qq) {
                if (qq == p) continue;
                const int lo = qq < p ? qq : p, hi = qq < p ? p : qq;
                const int P = poff[i] + hi * (hi - 1) / 2 + lo;
                const int pb = pblk[P];
                if (pb < 0) continue;
                const bool is_j = (p == lo) != ((pb & 256) != 0);
                const double* g = pg + 6 * (size_t)P + (is_j ? 0 : 3);
                gx += g[0];
                gy += g[1];
                gz += g[2];
            }
            gent[3 * e] = gx;
            gent[3 * e + 1] = gy;
            gent[3 * e + 2] = gz;
        }
        __syncthreads();
        // forces F_i = sum of own entries - sum of reverse entries; energy (Neumaier)
        for (int i = tid; i < N; i += nt) {
            double sx = 0.0, sy = 0.0, sz = 0.0;
            for (int e = off[i]; e < off[i + 1]; ++e) {
                sx -= gent[3 * e];
                sy -= gent[3 * e + 1];
                sz -= gent[3 * e + 2];
            }
            double fx = sx, fy = sy, fz = sz;
            for (int e = off[i]; e < off[i + 1]; ++e) {
                const int r = rev[e];
                fx += gent[3 * r];
                fy += gent[3 * r + 1];
                fz += gent[3 * r + 2];
            }
            F[3 * i] = -fx;
            F[3 * i + 1] = -fy;
            F[3 * i + 2] = -fz;
        }
        if (tid == nt - 1) {
            double sum = 0.0, cmp = 0.0;
            for (int i = 0; i < N; ++i) {
                const double x = atE[i], t = sum + x;
                cmp += fabs(sum) >= fabs(x) ? (sum - t) + x : (x - t) + sum;
                sum = t;
            }
            if (a.hist) a.hist[step] = sum + cmp;
            if (step == a.nsteps - 1) a.energy[0] = sum + cmp;
        }
        __syncthreads();
    }
    for (int q = tid; q < n3; q += nt) {
        if (!a.eval_only) {
            a.mom[q] = mom[q] + 0.5 * dt * (F[q] + Fp[q]);
            a.pos[q] = pos[q];
        }
        a.force[q] = F[q];
    }
    if (tid == 0) {
        if (a.eval_only) {
            // the caller cleared acc; plain stores (acc may be mapped host
            // memory, where a read-modify-write costs a bus round trip)
            a.acc[0] = status[0];
            a.acc[1] = a.nsteps;
        } else {
            a.acc[0] |= status[0];
            a.acc[1] += a.nsteps;
        }
    }
    if (box) {
        // every thread's outputs are visible to the host before the answer
        __threadfence_system();
        __syncthreads();
        if (tid == 0) box->ack = served;
    }
    }  // rounds
    if (box && tid == 0) {
        __threadfence_system();
        box->exited = 1;
    }
}

// Shared-memory layout of the item-parallel form; SIZE_MAX if it does not fit.
size_t tiny_md_layout(const DevModel& m, int N, TinyArgs* a) {
    if (N < 1 || N > kSmallMolecule || m.nlayers > 8) return SIZE_MAX;
    const size_t n = (size_t)N, ecap = n * (n - 1), pcap = N >= 3 ? n * (n - 1) * (n - 2) / 2 : 0;
    const size_t nsf = (size_t)m.nsf_max, g2w = m.g2max > 0 ? m.g2max : 1, g4w = m.gmax > 0 ? m.gmax : 1;
    size_t row = 0;
    int maxw = 1;
    for (int l = 0; l < m.nlayers; ++l) {
        row += 2 * (size_t)m.width[l + 1];
        maxw = m.width[l + 1] > maxw ? m.width[l + 1] : maxw;
    }
    const size_t dbuf = (size_t)(nsf > (size_t)maxw ? nsf : maxw);  // deltas, up to the input width
    const size_t mlp = n * (row + 2 * dbuf);
    const size_t bytes[tSlots] = {
        24 * n, 24 * n, 24 * n, 24 * n, 8 * n, 8 * n, 8 * n * nsf, 8 * n * nsf,  // pos .. W
        48 * ecap, 8 * ecap * g2w, 24 * ecap,                                    // EG ERC Gent
        40 * pcap, 8 * pcap * g4w, 8 * pcap * g4w, 48 * pcap,                    // PS PE PT PG
        8 * mlp, 8 * n,                                                          // Mlp Mask
        4 * n, 4 * (n + 1), 4 * (n + 1), 4 * ecap, 4 * ecap, 4 * ecap, 4 * pcap, 4 * pcap,
        4 * (size_t)m.nel * nsf, 4 * (size_t)kMaxEl * kMaxEl, 16};
    size_t off = 0;
    for (int k = 0; k < tSlots; ++k) {
        if (a) a->slot[k] = (int)off;
        off += align16z(bytes[k] > 0 ? bytes[k] : 16);
    }
    if (off > 226 * 1024) return SIZE_MAX;
    if (a) {
        a->g2w = (int)g2w;
        a->g4w = (int)g4w;
        a->maxw = (int)dbuf;
    }
    return off;
}

}  // namespace

size_t small_md_smem_bytes(const DevModel& m, int natoms) {
    const size_t t = tiny_md_layout(m, natoms, nullptr);
    return t != SIZE_MAX ? t : small_md_layout(m, natoms, nullptr);
}

bool small_md_tiny(const DevModel& m, int natoms) { return tiny_md_layout(m, natoms, nullptr) != SIZE_MAX; }

int launch_small_resident(const DevModel& m, int natoms, ResidentBox* box, cudaStream_t s) {
    TinyArgs ta{};
    const size_t tsm = tiny_md_layout(m, natoms, &ta);
    if (tsm == SIZE_MAX) return 0;
    ta.natoms = natoms;
    ta.nsteps = 1;
    ta.dt = 0.0;
    ta.rc2 = m.max_rc * m.max_rc;
    ta.pos = box->pos;
    ta.force = box->force;
    ta.energy = &box->energy;
    ta.acc = box->acc;
    ta.elem = box->elem;
    ta.eval_only = 1;
    ta.box = box;
    cudaFuncSetAttribute(k_tiny_md, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm);
    k_tiny_md<<<1, kThreads, tsm, s>>>(m, ta);
    return 1;
}

int launch_small_md(const Batch& b, const DevModel& m, const SmallMdArgs& x, cudaStream_t s) {
    TinyArgs ta{};
    const size_t tsm = tiny_md_layout(m, x.natoms, &ta);
    if (tsm != SIZE_MAX) {
        ta.natoms = x.natoms;
        ta.nsteps = x.nsteps;
        ta.dt = x.dt;
        ta.rc2 = m.max_rc * m.max_rc;
        ta.pos = x.pos;
        ta.mom = x.mom;
        ta.mass = x.mass;
        ta.force = x.force;
        ta.energy = x.energy;
        ta.hist = x.hist;
        ta.acc = x.acc;
        ta.elem = b.elem;
        ta.eval_only = x.eval_only;
        if (x.inline_pos && x.inline_elem && x.natoms <= kSmallMolecule) {
            ta.inline_in = 1;
            for (int q = 0; q < 3 * x.natoms; ++q) ta.in_pos[q] = x.inline_pos[q];
            for (int i = 0; i < x.natoms; ++i) ta.in_elem[i] = x.inline_elem[i];
        }
        // the shared-memory limit is raised once per device and size (the
        // attribute call costs about a microsecond)
        {
            constexpr int kMaxDev = 64;
            static std::atomic<size_t> raised[kMaxDev];
            int dev = 0;
            cudaGetDevice(&dev);
            if (dev < 0 || dev >= kMaxDev || raised[dev].load(std::memory_order_relaxed) < tsm) {
                cudaFuncSetAttribute(k_tiny_md, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm);
                if (dev >= 0 && dev < kMaxDev) {
                    size_t cur = raised[dev].load(std::memory_order_relaxed);
                    while (cur < tsm && !raised[dev].compare_exchange_weak(cur, tsm)) {
                    }
                }
            }
        }
        k_tiny_md<<<1, kThreads, tsm, s>>>(m, ta);
        return 1;
    }
    FusedArgs a{};
    const size_t smem = small_md_layout(m, x.natoms, &a);
    a.natoms = x.natoms;
    a.nsteps = x.nsteps;
    a.dt = x.dt;
    a.rc2 = m.max_rc * m.max_rc;
    a.pos = x.pos;
    a.mom = x.mom;
    a.mass = x.mass;
    a.force = x.force;
    a.energy = x.energy;
    a.hist = x.hist;
    a.acc = x.acc;
    a.eval_only = x.eval_only;
    auto run = [&](auto kernel) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kernel<<<1, kThreads, smem, s>>>(b, m, a);
    };
    if (m.gmax <= 4)
        run(k_small_md<4>);
    else if (m.gmax <= 8)
        run(k_small_md<8>);
    else if (m.gmax <= 16)
        run(k_small_md<16>);
    else
        run(k_small_md<32>);
    return 1;
}

}  // namespace hdnnp

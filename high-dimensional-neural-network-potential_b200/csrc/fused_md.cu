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
        mom[q] = a.mom[q];
        F[q] = a.force[q];
    }
    for (int i = tid; i < N; i += blockDim.x) {
        mass[i] = a.mass[i];
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
        a.mom[q] = mom[q] + 0.5 * dt * (F[q] + Fp[q]);
        a.pos[q] = pos[q];
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

}  // namespace

size_t small_md_smem_bytes(const DevModel& m, int natoms) { return small_md_layout(m, natoms, nullptr); }

int launch_small_md(const Batch& b, const DevModel& m, const SmallMdArgs& x, cudaStream_t s) {
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

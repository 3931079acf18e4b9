// fused_md.cu -- velocity-Verlet MD of one small molecule in ONE kernel launch.
//
// The reference's example runs MD of an 8-atom molecule, one
// hdnnpEnergyAndForces call per step (src/potentials/hdnnpExample.f90:58-64).
// Through the general pipeline such a step is ~26 tiny kernels, so its time is
// launch and pipeline latency, not work.  Here one thread block runs every
// stage of every step of a launch -- drift, neighbour lists, symmetry
// functions, networks, gradients, forces, kick -- separated by block
// barriers, with the per-atom routines of the generic kernels
// (symfn_generic.cuh, mlp_tile.cuh).  Molecules only (no images), FP64.
//
// Neighbour lists are built by direct search in atom-index order (the
// reference walks its cell grid; for a molecule both give the same set, the
// sums differ only in rounding).  All intermediates live in a scratch area
// that the plan allocates once.
#include "engine.h"
#include "mlp_tile.cuh"
#include "symfn_generic.cuh"

namespace hdnnp {

namespace {

struct FusedArgs {
    int natoms, nsteps, mm, maxw;
    double dt, rc2;
    size_t warp_bytes;              // symmetry-function shared memory per warp
    double* pos;
    double* mom;
    const double* mass;
    double* force;
    double* fprev;
    double* energy;
    double* hist;                   // [nsteps] or null
    int* acc;                       // [2]: OR of status flags, evaluations
    int el_start[kMaxEl + 1];       // element groups of el_atoms
};

template <int GM>
__global__ void __launch_bounds__(kThreads, 1) k_small_md(Batch b, DevModel m, FusedArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int cnt[kSmallMolecule + 1];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    const int N = a.natoms;
    const double dt = a.dt;
    if (tid == 0) b.status[0] = 0;
    __syncthreads();
    for (int step = 0; step < a.nsteps; ++step) {
        // drift (hdnnpExample.f90:61-62)
        for (int q = tid; q < 3 * N; q += blockDim.x) {
            const double mi = a.mass[q / 3];
            const double x = a.pos[q] + (a.mom[q] / mi * dt + 0.5 * a.force[q] / mi * dt * dt);
            if (!isfinite(x)) atomicOr(b.status, 8);  // same flag as the list build's check
            a.pos[q] = x;
            a.fprev[q] = a.force[q];
        }
        __syncthreads();
        // neighbour lists: every j != i with |d|^2 < rc^2, in index order
        for (int i = tid; i < N; i += blockDim.x) {
            int n = 0;
            for (int j = 0; j < N; ++j) {
                const double dx = a.pos[3 * i] - a.pos[3 * j], dy = a.pos[3 * i + 1] - a.pos[3 * j + 1],
                             dz = a.pos[3 * i + 2] - a.pos[3 * j + 2];
                n += (j != i && dx * dx + dy * dy + dz * dz < a.rc2);
            }
            cnt[i] = n;
        }
        __syncthreads();
        if (tid == 0) {
            int acc = 0;
            for (int i = 0; i < N; ++i) {
                b.nei_off[i] = acc;
                acc += cnt[i];
            }
            b.nei_off[N] = acc;
        }
        __syncthreads();
        for (int i = tid; i < N; i += blockDim.x) {
            int o = b.nei_off[i];
            for (int j = 0; j < N; ++j) {
                const double dx = a.pos[3 * i] - a.pos[3 * j], dy = a.pos[3 * i + 1] - a.pos[3 * j + 1],
                             dz = a.pos[3 * i + 2] - a.pos[3 * j + 2];
                if (j != i && dx * dx + dy * dy + dz * dz < a.rc2) {
                    b.nei_j[o] = j;
                    b.nei_s[o] = 0;
                    ++o;
                }
            }
        }
        __syncthreads();
        // reverse entries: (i -> j) pairs with (j -> i)
        for (int i = tid; i < N; i += blockDim.x)
            for (int e = b.nei_off[i]; e < b.nei_off[i + 1]; ++e) {
                const int j = b.nei_j[e];
                int r = e;
                for (int f = b.nei_off[j]; f < b.nei_off[j + 1]; ++f)
                    if (b.nei_j[f] == i) {
                        r = f;
                        break;
                    }
                b.nei_rev[e] = r;
            }
        __syncthreads();
        // symmetry functions (one warp per atom)
        {
            Smem<double> s = carve<double>(smem + w * a.warp_bytes, a.mm, m.nsf_max, false);
            for (int i = w; i < N; i += nw) sfv_atom<GM>(b, m, a.mm, s, i, lane);
        }
        __syncthreads();
        // networks: element tiles
        for (int e = 0; e < m.nel; ++e)
            for (int t0 = a.el_start[e]; t0 < a.el_start[e + 1]; t0 += kTile) {
                const int c = a.el_start[e + 1] - t0 < kTile ? a.el_start[e + 1] - t0 : kTile;
                mlp_tile<double>(b, m, a.maxw, e, t0, c, smem);
                __syncthreads();
            }
        // dE/dG-weighted gradients
        {
            Smem<double> s = carve<double>(smem + w * a.warp_bytes, a.mm, m.nsf_max, true);
            for (int i = w; i < N; i += nw) sfg_atom(b, m, a.mm, s, i, lane);
        }
        __syncthreads();
        // forces: F_a = -(g_self(a) + sum over the reverse entries)
        for (int i = tid; i < N; i += blockDim.x) {
            double fx = b.gself[3 * i], fy = b.gself[3 * i + 1], fz = b.gself[3 * i + 2];
            for (int e = b.nei_off[i]; e < b.nei_off[i + 1]; ++e) {
                const int r = b.nei_rev[e];
                fx += b.gent[3 * r];
                fy += b.gent[3 * r + 1];
                fz += b.gent[3 * r + 2];
            }
            a.force[3 * i] = -fx;
            a.force[3 * i + 1] = -fy;
            a.force[3 * i + 2] = -fz;
        }
        if (tid == 0) {
            // compensated (Neumaier) sum of the atomic energies
            double sum = 0.0, c = 0.0;
            for (int i = 0; i < N; ++i) {
                const double x = b.atE[i], t = sum + x;
                c += fabs(sum) >= fabs(x) ? (sum - t) + x : (x - t) + sum;
                sum = t;
            }
            a.energy[0] = sum + c;
            if (a.hist) a.hist[step] = sum + c;
        }
        __syncthreads();
        // kick (hdnnpExample.f90:64)
        for (int q = tid; q < 3 * N; q += blockDim.x) a.mom[q] += 0.5 * dt * (a.force[q] + a.fprev[q]);
        __syncthreads();
    }
    if (tid == 0) {
        a.acc[0] |= b.status[0];
        a.acc[1] += a.nsteps;
    }
}

}  // namespace

size_t small_md_smem_bytes(const DevModel& m, int mm) {
    const size_t sf = warp_bytes<double>(mm, m.nsf_max, true) * (kThreads / 32);
    const size_t nn = mlp_smem_bytes(m, sizeof(double));
    return sf > nn ? sf : nn;
}

int launch_small_md(const Batch& b, const DevModel& m, const SmallMdArgs& x, cudaStream_t s) {
    FusedArgs a{};
    a.natoms = x.natoms;
    a.nsteps = x.nsteps;
    a.mm = ((x.natoms - 1 + 31) / 32) * 32;
    if (a.mm < 32) a.mm = 32;
    a.dt = x.dt;
    a.rc2 = m.max_rc * m.max_rc;
    a.warp_bytes = warp_bytes<double>(a.mm, m.nsf_max, true);
    a.pos = x.pos;
    a.mom = x.mom;
    a.mass = x.mass;
    a.force = x.force;
    a.fprev = x.fprev;
    a.energy = x.energy;
    a.hist = x.hist;
    a.acc = x.acc;
    int maxw = 1;
    for (int l = 0; l < m.nlayers; ++l) maxw = m.width[l + 1] > maxw ? m.width[l + 1] : maxw;
    a.maxw = maxw;
    for (int e = 0; e <= m.nel; ++e) a.el_start[e] = x.el_start[e];
    const size_t smem = small_md_smem_bytes(m, a.mm);
    auto run = [&](auto kernel) {
        if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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

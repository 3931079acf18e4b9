// mlp.cu -- K5: per-element atomic networks, forward pass and dE/dG (FP64
// on the FP64 tensor cores, FP32 on the CUDA cores).
//
// Same arithmetic as nn_forward / nn_backward(gradOut = 1) per atom
// (neuralNetworks.f90:94-158, 220-313; called from hdnnps.f90:523-531):
//   c_l = W_l y_{l-1} + b_l,  y_l = act_l(c_l);   E_atom = y_L + atom_energy
//   delta_L = act'(c_L);  delta_{l-1} = (W_l^T delta_l) * act'(c_{l-1});
//   dE/dG = W_1^T delta_1
// Atoms are grouped by element (a grouped GEMM: one weight set per element);
// one CTA evaluates a tile of 32 atoms of one element with the activations
// kept in shared memory and the weights read through L1 (W^T for the forward
// pass so that consecutive threads read consecutive outputs, W for dE/dG).
#include "engine.h"
#include "mlp_tile.cuh"

namespace hdnnp {

namespace {

// Counts and slots per element with warp-aggregated atomics: the lanes of
// one element in a warp add their number once (a handful of counters would
// otherwise take one atomic per atom).  The order inside an element group is
// that of the atomics; each atom's network output does not depend on it.
__global__ void k_count_elements(Batch b, int nel) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = i < b.natoms ? b.elem[i] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, e);
    if (e >= 0 && (peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0) atomicAdd(&b.el_count[e], __popc(peers));
}

__global__ void k_element_starts(Batch b, int nel) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int acc = 0;
        for (int e = 0; e < nel; ++e) {
            b.el_start[e] = acc;
            acc += b.el_count[e];
            b.el_count[e] = 0;  // reused as the fill cursor
        }
        b.el_start[nel] = acc;
    }
}

__global__ void k_fill_elements(Batch b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int e = i < b.natoms ? b.elem[i] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, e);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (e >= 0 && lane == leader) base = atomicAdd(&b.el_count[e], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (e >= 0) b.el_atoms[b.el_start[e] + base + __popc(peers & ((1u << lane) - 1u))] = i;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_mlp(Batch b, DevModel m, int maxw) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    // locate (element, tile) of this block
    int tile = blockIdx.x, e = -1, t0 = 0, cnt = 0;
    for (int x = 0; x < m.nel; ++x) {
        int n = b.el_start[x + 1] - b.el_start[x];
        int nt = (n + kTile - 1) / kTile;
        if (tile < nt) {
            e = x;
            t0 = b.el_start[x] + tile * kTile;
            cnt = min(kTile, n - tile * kTile);
            break;
        }
        tile -= nt;
    }
    if (e < 0) return;
    mlp_tile<T>(b, m, maxw, e, t0, cnt, sm_raw);
}

// ---------------------------------------------------------------- FP64 tensor cores
// The FP64 networks on the FP64 tensor cores: mma.sync m8n8k4 f64 (tcgen05
// has no FP64 kind), a warp per 8 atoms of one element.  The first layer's
// GEMM (8 x nin) x (nin x 32) and the input gradient dE/dG = delta_1 W_1,
// (8 x 32) x (32 x nin), carry ~90 % of the multiply-adds; the hidden and
// output layers (widths <= 32) run on the lanes from shared memory.  Same
// formulas as mlp_tile (neuralNetworks.f90:94-158); the sums of the two
// GEMMs run in the tensor cores' order.
//   fragments (thread t): A[t/4][t%4], B[k = t%4][n = t/4],
//   C[t/4][2 (t%4) + v], v = 0, 1
__device__ __forceinline__ void dmma(double (&c)[2], double a, double bb) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(bb));
}

constexpr int kDW = 4;   // warps per block
constexpr int kDH = 32;  // widest layer the kernel takes
constexpr int kDR = 8;   // atoms per warp

// Row stride of the per-warp activation rows: the widest layer + 1, odd.
__host__ __device__ inline int dmma_stride(int maxw) { return (maxw + 1) | 1; }
// per warp: act'(c_l) of every layer and two rotating rows (activations in
// the forward pass, deltas in the backward pass), [8][stride] each
__host__ __device__ inline int dmma_warp_doubles(int L, int stride) { return (L + 2) * kDR * stride; }

__global__ void __launch_bounds__(32 * kDW, 6) k_mlp_dmma(Batch b, DevModel m, int S) {
    extern __shared__ __align__(16) double dsm[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int L = m.nlayers;
    // locate (element, tile of 8 atoms) of this warp
    int tile = blockIdx.x * kDW + wib, e = -1, t0 = 0, cnt = 0;
    for (int x = 0; x < m.nel; ++x) {
        const int n = b.el_start[x + 1] - b.el_start[x];
        const int nt = (n + kDR - 1) / kDR;
        if (tile < nt) {
            e = x;
            t0 = b.el_start[x] + tile * kDR;
            cnt = min(kDR, n - tile * kDR);
            break;
        }
        tile -= nt;
    }
    if (e < 0) return;  // uniform per warp
    double* ws = dsm + (size_t)wib * dmma_warp_doubles(L, S);
    auto da = [&](int l) { return ws + l * kDR * S; };          // act'(c_l)
    auto yb = [&](int p) { return ws + (L + p) * kDR * S; };    // rotating rows
    const int r = lane >> 2, q = lane & 3;
    const int atom = r < cnt ? b.el_atoms[t0 + r] : -1;
    const int nin = m.nin_el[e], nsf = m.nsf_max, H1 = m.width[1];
    // layer 1: C[8 x 32] = G[8 x nin] W1^T on the tensor cores; the next
    // k-step's operands are loaded while this one multiplies
    double acc[4][2];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) acc[nt][0] = acc[nt][1] = 0.0;
    const double* grow = atom >= 0 ? b.G + (size_t)atom * nsf : nullptr;
    const double* F = m.dm_fwd + m.dm_off_f[e] + lane;  // [ks][nt][32]
    const int KS = (nin + 3) >> 2;
    // operands of k-step ks (zero A and no B load beyond the last step)
    auto load = [&](int ks, double& a, double (&bf)[4]) {
        const int k = 4 * ks + q;
        a = (grow && k < nin) ? __ldg(grow + k) : 0.0;
        if (ks < KS) {
            const double* f = F + (size_t)ks * 128;
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) bf[nt] = __ldg(f + nt * 32);
        }
    };
    // two k-steps in flight: the operands of ks + 2 are loaded while ks
    // multiplies (two register sets, the loop unrolled by two)
    double a0 = 0.0, a1 = 0.0, b0[4] = {0.0, 0.0, 0.0, 0.0}, b1[4] = {0.0, 0.0, 0.0, 0.0};
    load(0, a0, b0);
    load(1, a1, b1);
    for (int ks = 0; ks < KS; ks += 2) {
        {
            const double a = a0;
            double bb[4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) bb[nt] = b0[nt];
            if (ks + 2 < KS) load(ks + 2, a0, b0);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) dmma(acc[nt], a, bb[nt]);
        }
        if (ks + 1 < KS) {
            const double a = a1;
            double bb[4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) bb[nt] = b1[nt];
            if (ks + 3 < KS) load(ks + 3, a1, b1);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) dmma(acc[nt], a, bb[nt]);
        }
    }
    {
        const double* b1 = m.b + m.b_off[e * L];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                const int col = nt * 8 + 2 * q + v;
                if (col < H1) {
                    const double cv = acc[nt][v] + b1[col];
                    const double yv = act_f(m.act[0], cv);
                    yb(0)[r * S + col] = yv;
                    da(0)[r * S + col] = act_d(m.act[0], cv, yv);
                }
            }
    }
    __syncwarp();
    // hidden and output layers: lane = output neuron, the warp's 8 atoms
    for (int l = 1; l < L; ++l) {
        const int win = m.width[l], wout = m.width[l + 1];
        // transposed weights [win][wout]: the lanes' loads of one input are
        // one coalesced row
        const double* WT = m.wt + m.w_off[e * L + l];
        const double* bl = m.b + m.b_off[e * L + l];
        const double* yin = yb((l - 1) & 1);
        double* yout = yb(l & 1);
        if (lane < wout) {
            double sacc[kDR];
#pragma unroll
            for (int rr = 0; rr < kDR; ++rr) sacc[rr] = 0.0;
            // unrolled so that several weight loads are in flight (they come
            // from L2: the shared memory of 6 blocks leaves no L1)
#pragma unroll 5
            for (int i = 0; i < win; ++i) {
                const double w = __ldg(WT + (size_t)i * wout + lane);
#pragma unroll
                for (int rr = 0; rr < kDR; ++rr) sacc[rr] += w * yin[rr * S + i];
            }
#pragma unroll
            for (int rr = 0; rr < kDR; ++rr) {
                const double cv = sacc[rr] + bl[lane];
                const double yv = act_f(m.act[l], cv);
                yout[rr * S + lane] = yv;
                da(l)[rr * S + lane] = act_d(m.act[l], cv, yv);
            }
        }
        __syncwarp();
    }
    // atomic energies, then the rotating rows carry the deltas
    if (lane < cnt) b.atE[b.el_atoms[t0 + lane]] = yb((L - 1) & 1)[lane * S] + m.atom_energy[e];
    __syncwarp();
    double* dcur = yb(0);
    double* dnext = yb(1);
    {
        const int w = m.width[L];  // gradOut = 1
        if (lane < w)
#pragma unroll
            for (int rr = 0; rr < kDR; ++rr) dcur[rr * S + lane] = da(L - 1)[rr * S + lane];
    }
    __syncwarp();
    for (int l = L - 1; l >= 1; --l) {
        const int wout = m.width[l + 1], wi = m.width[l];
        const double* W = m.w + m.w_off[e * L + l];  // [wout][wi]
        if (lane < wi) {
            // each weight loaded once for the warp's 8 atoms (same sum order)
            double sv[kDR];
#pragma unroll
            for (int rr = 0; rr < kDR; ++rr) sv[rr] = 0.0;
#pragma unroll 5
            for (int o = 0; o < wout; ++o) {
                const double w = __ldg(W + (size_t)o * wi + lane);
#pragma unroll
                for (int rr = 0; rr < kDR; ++rr) sv[rr] += dcur[rr * S + o] * w;
            }
#pragma unroll
            for (int rr = 0; rr < kDR; ++rr) dnext[rr * S + lane] = sv[rr] * da(l - 1)[rr * S + lane];
        }
        __syncwarp();
        double* t = dcur;
        dcur = dnext;
        dnext = t;
    }
    // dE/dG = delta_1 W1: C[8 x nin] = A[8 x 32] B[32 x nin] on the tensor cores
    double afr[kDH / 4];
#pragma unroll
    for (int ks = 0; ks < kDH / 4; ++ks) afr[ks] = (4 * ks + q < H1) ? dcur[r * S + 4 * ks + q] : 0.0;
    // two n-tiles per iteration (independent accumulator chains)
    const double* Bw = m.dm_bwd + m.dm_off_b[e] + lane;  // [nb][ks][32]
    const int KB = (H1 + 3) >> 2, NB = (nin + 7) >> 3;
    for (int nb = 0; nb < NB; nb += 2) {
        const bool two = nb + 1 < NB;  // uniform
        const double* b0 = Bw + (size_t)nb * KB * 32;
        const double* b1 = b0 + KB * 32;
        double c0[2] = {0.0, 0.0}, c1[2] = {0.0, 0.0};
#pragma unroll
        for (int ks = 0; ks < kDH / 4; ++ks) {
            if (ks < KB) {
                dmma(c0, afr[ks], __ldg(b0 + ks * 32));
                if (two) dmma(c1, afr[ks], __ldg(b1 + ks * 32));
            }
        }
        if (atom >= 0) {
            double* drow = b.dEdG + (size_t)atom * nsf;
#pragma unroll
            for (int v = 0; v < 2; ++v) {
                const int col = nb * 8 + 2 * q + v;
                if (col < nin) drow[col] = c0[v];
                if (two && col + 8 < nin) drow[col + 8] = c1[v];
            }
        }
    }
}

}  // namespace

int launch_element_groups(const Batch& b, const DevModel& m, cudaStream_t s) {
    const int g = (b.natoms + 255) / 256;
    cudaMemsetAsync(b.el_count, 0, sizeof(int) * (m.nel + 1), s);
    k_count_elements<<<g, 256, 0, s>>>(b, m.nel);
    k_element_starts<<<1, 32, 0, s>>>(b, m.nel);
    k_fill_elements<<<g, 256, 0, s>>>(b);
    return 3;
}

size_t mlp_smem_bytes(const DevModel& m, size_t elem) {
    int nin = 0, maxw = 1;
    for (int e = 0; e < m.nel; ++e) nin = nin > m.nin_el[e] ? nin : m.nin_el[e];
    size_t n = (size_t)kTile * nin;
    for (int l = 0; l < m.nlayers; ++l) {
        n += 2 * (size_t)kTile * m.width[l + 1];
        if (m.width[l + 1] > maxw) maxw = m.width[l + 1];
    }
    n += 2 * (size_t)kTile * maxw;  // deltas of the hidden/output layers
    return n * elem;
}

template <typename T>
void run_mlp(const Batch& b, const DevModel& m, cudaStream_t s) {
    int nin = 0, maxw = 1;
    for (int e = 0; e < m.nel; ++e) nin = nin > m.nin_el[e] ? nin : m.nin_el[e];
    for (int l = 0; l < m.nlayers; ++l)
        if (m.width[l + 1] > maxw) maxw = m.width[l + 1];
    size_t smem = mlp_smem_bytes(m, sizeof(T));
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_mlp<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int tiles = b.natoms / kTile + m.nel + 1;
    k_mlp<T><<<tiles, kThreads, smem, s>>>(b, m, maxw);
}

// The tensor-core form takes networks whose layers are at most kDH wide,
// with one output and at most 8 layers (dm_ok, set with the fragments at
// model upload).
int launch_mlp(const Batch& b, const DevModel& m, cudaStream_t s) {
    if (!m.dm_ok) {
        run_mlp<double>(b, m, s);
        return 1;
    }
    int maxw = 1;
    for (int l = 1; l <= m.nlayers; ++l) maxw = maxw > m.width[l] ? maxw : m.width[l];
    const int S = dmma_stride(maxw);
    const size_t smem = (size_t)dmma_warp_doubles(m.nlayers, S) * sizeof(double) * kDW;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_mlp_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long long warps = b.natoms / kDR + m.nel + 1;  // >= the tiles of all elements
    k_mlp_dmma<<<(unsigned)((warps + kDW - 1) / kDW), 32 * kDW, smem, s>>>(b, m, S);
    return 1;
}

int launch_mlp_fp32(const Batch& b, const DevModel& m, cudaStream_t s) {
    run_mlp<float>(b, m, s);
    return 1;
}

}  // namespace hdnnp

// mlp.cu -- K5: per-element atomic networks, forward pass and dE/dG (FP64).
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

int launch_mlp(const Batch& b, const DevModel& m, cudaStream_t s) {
    run_mlp<double>(b, m, s);
    return 1;
}

int launch_mlp_fp32(const Batch& b, const DevModel& m, cudaStream_t s) {
    run_mlp<float>(b, m, s);
    return 1;
}

}  // namespace hdnnp

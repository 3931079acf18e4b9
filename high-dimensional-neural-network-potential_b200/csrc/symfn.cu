// symfn.cu -- K4 (symmetry-function values) and K6 (dE/dG-weighted gradients).
//
// Math of calcAllSymmetryFunctions (symmetryFunctions.f90:158-308) with the
// tanh^3 cutoff of :310-327 and the scaling of hdnnpCalcSymfunctions
// (hdnnps.f90:471-481):
//   G2_s = sum_j exp(-eta (r_ij - Rs)^2) fc(r_ij)                 (j of element el1)
//   G4_s = sum_{j<k} 2^(1-zeta) (1 + lambda cos)^zeta
//                    exp(-eta (r_ij^2 + r_ik^2 + r_jk^2)) fc_ij fc_ik fc_jk
//   G'_s = (G_s - mean_s) / (max_s - min_s)
// Pairs with r_jk >= rc contribute exact zeros in the reference (fc_jk = dfc_jk
// = 0) and are skipped here.
//
// Design (one warp per centre atom):
//  * the atom's neighbour entries are staged in shared memory, sorted by
//    element (stable, so entry order is kept inside an element): relative
//    vector d = r_centre - r_neighbour, |d|, fc, dfc/r;
//  * radial SFs: lane = SF, loop over the neighbours of its element;
//  * angular SFs: for each unordered element pair (a,b) the candidate pairs
//    are tested for r_jk < rc in chunks of 32 lanes and compacted into a
//    shared queue; full chunks of contributing pairs are evaluated with one
//    pair per lane; pass 1 keeps up to GM SF sums per lane in registers and
//    reduces them across the warp with a recursive-halving shuffle
//    reduce-scatter; pass 2 folds the SF sum into three scalars per pair,
//       A = sum_s w_s pf_s cp_s ex_s,  B = sum_s w_s pf_s cp_s ex_s eta_s,
//       C = sum_s w_s pf_s tmp2_s lambda_s zeta_s ex_s      (w_s = dE/dG_s),
//    so that the two 3-vectors dE/dr_j, dE/dr_k are assembled once per pair
//    instead of once per (pair, SF) as the reference's dsf arrays are; dsf is
//    never materialised.
//  * pass 2 writes, for every neighbour entry e of atom i, g_e = dE_i/dr_e
//    (3 doubles), the centre term g_self = -sum_e g_e and the atom virial
//    W_i = -sum_e g_e (x) d_e, which the force gather and the structure
//    reduction consume.
#include <atomic>
#include <cstdio>

#include "engine.h"
#include "symfn_generic.cuh"

namespace hdnnp {

namespace {

template <int GM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_sf_values(Batch b, DevModel m, int mm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    Smem<double> s = carve<double>(smem_raw + wib * warp_bytes<double>(mm, m.nsf_max, false), mm, m.nsf_max, false);
    for (int i = blockIdx.x * kWarpsPerBlock + wib; i < b.natoms; i += gridDim.x * kWarpsPerBlock) {
        sfv_atom<GM>(b, m, mm, s, i, lane);
    }
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_sf_gradients(Batch b, DevModel m, int mm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    Smem<double> s = carve<double>(smem_raw + wib * warp_bytes<double>(mm, m.nsf_max, true), mm, m.nsf_max, true);
    for (int i = blockIdx.x * kWarpsPerBlock + wib; i < b.natoms; i += gridDim.x * kWarpsPerBlock) {
        sfg_atom(b, m, mm, s, i, lane);
    }
}

int num_sms() { return device_sm_count(); }

template <int GM>
void launch_values_gm(const Batch& b, const DevModel& m, int mm, cudaStream_t st) {
    size_t smem = warp_bytes<double>(mm, m.nsf_max, false) * kWarpsPerBlock;
    // set on every launch: the attribute is per device, and calls come from several threads
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_sf_values<GM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int blocks = (b.natoms + kWarpsPerBlock - 1) / kWarpsPerBlock;
    int cap = num_sms() * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_sf_values<GM><<<blocks, 32 * kWarpsPerBlock, smem, st>>>(b, m, mm);
}

}  // namespace

size_t sf_smem_per_warp(int mm, bool grad) { return warp_bytes<double>(mm, 512, grad); }

int launch_sf_values(const Batch& b, const DevModel& m, cudaStream_t st) {
    const int mm = ((b.mmax + 31) / 32) * 32 > 0 ? ((b.mmax + 31) / 32) * 32 : 32;
    if (m.gmax <= 4)
        launch_values_gm<4>(b, m, mm, st);
    else if (m.gmax <= 8)
        launch_values_gm<8>(b, m, mm, st);
    else if (m.gmax <= 16)
        launch_values_gm<16>(b, m, mm, st);
    else
        launch_values_gm<32>(b, m, mm, st);
    return 1;
}

int launch_sf_gradients(const Batch& b, const DevModel& m, cudaStream_t st) {
    const int mm = ((b.mmax + 31) / 32) * 32 > 0 ? ((b.mmax + 31) / 32) * 32 : 32;
    size_t smem = warp_bytes<double>(mm, m.nsf_max, true) * kWarpsPerBlock;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_sf_gradients, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int blocks = (b.natoms + kWarpsPerBlock - 1) / kWarpsPerBlock;
    int cap = num_sms() * 16;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_sf_gradients<<<blocks, 32 * kWarpsPerBlock, smem, st>>>(b, m, mm);
    return 1;
}

// Multiprocessor count of the current device, cached per device ordinal
// (contexts on several devices and several host threads call this).
int device_sm_count() {
    constexpr int kMaxDev = 64;
    static std::atomic<int> cache[kMaxDev];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    if (dev >= 0 && dev < kMaxDev) {
        const int c = cache[dev].load(std::memory_order_relaxed);
        if (c > 0) return c;
    }
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    if (dev >= 0 && dev < kMaxDev) cache[dev].store(n, std::memory_order_relaxed);
    return n;
}

}  // namespace hdnnp

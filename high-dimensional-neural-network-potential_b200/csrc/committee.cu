// committee.cu -- committee of potentials on shared neighbour lists and
// symmetry functions.
//
// Follows globalHdnnpEnergyAndForces (src/potentials/globalHdnnps.f90:31-70):
// the neighbour lists and the symmetry functions (with their scaling) come
// from the first member (:47, :51); every member's networks run on them
// (:55-57); energy, forces and dE/dh are the member means (:60-64) and std is
// the population standard deviation of the member energies (:66-68).
//
// The force and lattice-derivative contraction is linear in dE/dG, so the
// members' dE/dG are averaged (fixed member order) before one contraction
// instead of contracting K times and averaging the forces; the results agree
// within rounding.  Member energies are compensated per-structure sums.
#include <cmath>

#include "engine.h"

namespace hdnnp {

namespace {

constexpr int kThreads = 256;

template <typename T>
__global__ void k_cm_accumulate(T* __restrict__ acc, const T* __restrict__ x, long long n, int first) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    acc[i] = first ? x[i] : acc[i] + x[i];
}

template <typename T>
__global__ void k_cm_mean(T* __restrict__ out, const T* __restrict__ acc, long long n, int k) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = acc[i] / (T)k;
}

// energy[s] = sum_k E_k(s) / K ; std[s] = sqrt(sum_k (E_k(s) - energy[s])^2 / K)
__global__ void k_cm_finish(const double* __restrict__ Ek, int k, int nstruct, double* __restrict__ energy,
                            double* __restrict__ std_dev) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nstruct) return;
    double sum = 0.0;
    for (int q = 0; q < k; ++q) sum += Ek[(size_t)q * nstruct + s];
    const double mean = sum / k;
    double v = 0.0;
    for (int q = 0; q < k; ++q) {
        const double d = Ek[(size_t)q * nstruct + s] - mean;
        v += d * d;
    }
    energy[s] = mean;
    if (std_dev) std_dev[s] = sqrt(v / k);
}

inline unsigned blocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

}  // namespace

int launch_committee_networks(const Batch& b, const Committee& cm, bool mixed, bool use_tc, void* acc, double* Ek,
                              cudaStream_t s) {
    int L = 0;
    const long long n = (long long)b.natoms * cm.members[0]->nsf_max;
    for (int q = 0; q < cm.k; ++q) {
        const DevModel& M = *cm.members[q];
        if (mixed && use_tc && M.tc_ok)
            L += launch_mlp_tc(b, M, s);
        else
            L += mixed ? launch_mlp_fp32(b, M, s) : launch_mlp(b, M, s);
        L += launch_struct_energies(b, mixed, Ek + (size_t)q * b.nstruct, s);
        if (mixed)
            k_cm_accumulate<float><<<blocks(n), kThreads, 0, s>>>((float*)acc, b.dEdGf, n, q == 0);
        else
            k_cm_accumulate<double><<<blocks(n), kThreads, 0, s>>>((double*)acc, b.dEdG, n, q == 0);
        ++L;
    }
    if (mixed)
        k_cm_mean<float><<<blocks(n), kThreads, 0, s>>>(b.dEdGf, (const float*)acc, n, cm.k);
    else
        k_cm_mean<double><<<blocks(n), kThreads, 0, s>>>(b.dEdG, (const double*)acc, n, cm.k);
    return L + 1;
}

int launch_committee_finish(const Batch& b, const Committee& cm, const double* Ek, cudaStream_t s) {
    k_cm_finish<<<(b.nstruct + 127) / 128, 128, 0, s>>>(Ek, cm.k, b.nstruct, b.energy, cm.std_dev);
    return 1;
}

}  // namespace hdnnp

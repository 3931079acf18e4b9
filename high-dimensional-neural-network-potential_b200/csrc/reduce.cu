// reduce.cu -- K7 force gather and K8 per-structure energy / virial reduction.
//
// The reference accumulates forces with an OpenMP array reduction
// (hdnnps.f90:514-538): force(:, ineis(n)) -= dEdSf(s) * dsf(:, n).  Here
// every neighbour entry e = (i -> j, S) carries g_e = dE_i/dr_e from the
// gradient pass and its reverse entry rev(e) = (j -> i, -S), so that
//     F_a = -( g_self(a) + sum_{e in list(a)} g_rev(e) )
// is a gather in a fixed order: no floating-point atomics, identical results
// for a structure alone and inside any batch.
// Energy: energy = sum(atEns) (hdnnps.f90:557) as a compensated (Neumaier)
// sum per structure.  dEdLat: the reference sums dEdSf dsf (h^-1 r_n)
// (hdnnps.f90:539-552); with sum_n g_n = 0 per centre this equals
// W h^-T with W = -sum_i sum_n g_n (x) d_n, reduced here in FP64.
#include "engine.h"

namespace hdnnp {

namespace {

// One warp per atom: lane l sums the reverse-entry gradients of entries
// e0 + l, e0 + l + 32, ... in order (coalesced index loads), a butterfly
// combines the lanes and lane 0 adds g_self.  The order depends only on the
// atom's own list, so a structure gets the same forces alone and in a batch.
template <typename T>
__global__ void k_force_gather(Batch b, const T* gself, const T* gent) {
    const int a = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (a >= b.natoms) return;  // uniform per warp
    double fx = 0.0, fy = 0.0, fz = 0.0;
    const int e0 = b.nei_off[a], e1 = b.nei_off[a + 1];
    for (int e = e0 + lane; e < e1; e += 32) {
        const size_t r = (size_t)b.nei_rev[e];
        fx += gent[3 * r];
        fy += gent[3 * r + 1];
        fz += gent[3 * r + 2];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (lane == 0) {
        b.force[3 * (size_t)a] = -((double)gself[3 * (size_t)a] + fx);
        b.force[3 * (size_t)a + 1] = -((double)gself[3 * (size_t)a + 1] + fy);
        b.force[3 * (size_t)a + 2] = -((double)gself[3 * (size_t)a + 2] + fz);
    }
}

// Neumaier running sum
struct KSum {
    double s, c;
    __device__ void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    }
    __device__ void merge(const KSum& o) {
        add(o.s);
        c += o.c;
    }
};

constexpr int kRedThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_struct_reduce(Batch b, int want_dEdLat, const T* atE, const T* vir) {
    __shared__ double se[kRedThreads], sc[kRedThreads];
    __shared__ double sv[9][kRedThreads];
    const int st = blockIdx.x;
    const StructInfo& S = b.info[st];
    const int a0 = S.atom_off, n = S.nat;
    KSum k{0.0, 0.0};
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += kRedThreads) {
        k.add((double)atE[a0 + i]);
        if (want_dEdLat)
#pragma unroll
            for (int u = 0; u < 9; ++u) v[u] += (double)vir[9 * (size_t)(a0 + i) + u];
    }
    se[threadIdx.x] = k.s;
    sc[threadIdx.x] = k.c;
#pragma unroll
    for (int u = 0; u < 9; ++u) sv[u][threadIdx.x] = v[u];
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            KSum a{se[threadIdx.x], sc[threadIdx.x]};
            KSum o{se[threadIdx.x + w], sc[threadIdx.x + w]};
            a.merge(o);
            se[threadIdx.x] = a.s;
            sc[threadIdx.x] = a.c;
#pragma unroll
            for (int u = 0; u < 9; ++u) sv[u][threadIdx.x] += sv[u][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        b.energy[st] = se[0] + sc[0];
        if (want_dEdLat && b.dEdLat) {
            double* out = b.dEdLat + 9 * (size_t)st;
            if (S.periodic) {
                // dEdLat(a,bb) = sum_c W(a,c) hinv(bb,c)   (column-major storage)
                for (int a = 0; a < 3; ++a)
                    for (int bb = 0; bb < 3; ++bb) {
                        double s = 0.0;
                        for (int c = 0; c < 3; ++c) s += sv[a + 3 * c][0] * S.hinv[bb + 3 * c];
                        out[a + 3 * bb] = s;
                    }
            } else {
                for (int u = 0; u < 9; ++u) out[u] = 0.0;
            }
        }
    }
}

// Compensated per-structure sum of the atomic energies only (committee members).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_struct_energy(Batch b, const T* atE, double* out) {
    __shared__ double se[kRedThreads], sc[kRedThreads];
    const StructInfo& S = b.info[blockIdx.x];
    KSum k{0.0, 0.0};
    for (int i = threadIdx.x; i < S.nat; i += kRedThreads) k.add((double)atE[S.atom_off + i]);
    se[threadIdx.x] = k.s;
    sc[threadIdx.x] = k.c;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            KSum a{se[threadIdx.x], sc[threadIdx.x]};
            KSum o{se[threadIdx.x + w], sc[threadIdx.x + w]};
            a.merge(o);
            se[threadIdx.x] = a.s;
            sc[threadIdx.x] = a.c;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = se[0] + sc[0];
}

}  // namespace

int launch_struct_energies(const Batch& b, bool fp32, double* out, cudaStream_t s) {
    if (fp32)
        k_struct_energy<float><<<b.nstruct, kRedThreads, 0, s>>>(b, b.atEf, out);
    else
        k_struct_energy<double><<<b.nstruct, kRedThreads, 0, s>>>(b, b.atE, out);
    return 1;
}

int launch_forces_and_reduce(const Batch& b, const DevModel& m, int want_dEdLat, cudaStream_t s) {
    (void)m;
    k_force_gather<double><<<(unsigned)((32LL * b.natoms + 255) / 256), 256, 0, s>>>(b, b.gself, b.gent);
    k_struct_reduce<double><<<b.nstruct, kRedThreads, 0, s>>>(b, want_dEdLat, b.atE, b.vir);
    return 2;
}

// mixed-precision form: FP32 intermediates, FP64 accumulation and outputs
int launch_forces_and_reduce_fp32(const Batch& b, const DevModel& m, int want_dEdLat, cudaStream_t s) {
    (void)m;
    k_force_gather<float><<<(unsigned)((32LL * b.natoms + 255) / 256), 256, 0, s>>>(b, b.gselff, b.gentf);
    k_struct_reduce<float><<<b.nstruct, kRedThreads, 0, s>>>(b, want_dEdLat, b.atEf, b.virf);
    return 2;
}

}  // namespace hdnnp

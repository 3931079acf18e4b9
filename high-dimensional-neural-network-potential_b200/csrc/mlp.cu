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

namespace hdnnp {

namespace {

constexpr int kTile = 32;
constexpr int kThreads = 256;

__device__ __forceinline__ double act_f(char a, double x) {
    switch (a) {
        case 't': return tanh(x);
        case 'p': return log(1.0 + exp(x));
        case 'r': return x > 0.0 ? x : 0.0;
        default: return x;
    }
}
__device__ __forceinline__ float act_f(char a, float x) {
    switch (a) {
        case 't': return tanhf(x);
        case 'p': return log1pf(expf(x));
        case 'r': return x > 0.0f ? x : 0.0f;
        default: return x;
    }
}
// derivative from the pre-activation c and the activation y = act(c)
template <typename T>
__device__ __forceinline__ T act_d(char a, T c, T y) {
    switch (a) {
        case 't': return (T)1 - y * y;
        case 'p': return (T)1 / ((T)1 + (T)exp((double)-c));
        case 'r': return c > (T)0 ? (T)1 : (T)0;
        default: return (T)1;
    }
}

template <typename T> struct MB;
template <> struct MB<double> {
    static __device__ const double* G(const Batch& b) { return b.G; }
    static __device__ double* dEdG(const Batch& b) { return b.dEdG; }
    static __device__ double* atE(const Batch& b) { return b.atE; }
    static __device__ const double* w(const DevModel& m) { return m.w; }
    static __device__ const double* wt(const DevModel& m) { return m.wt; }
    static __device__ const double* bias(const DevModel& m) { return m.b; }
};
template <> struct MB<float> {
    static __device__ const float* G(const Batch& b) { return b.Gf; }
    static __device__ float* dEdG(const Batch& b) { return b.dEdGf; }
    static __device__ float* atE(const Batch& b) { return b.atEf; }
    static __device__ const float* w(const DevModel& m) { return m.wf; }
    static __device__ const float* wt(const DevModel& m) { return m.wtf; }
    static __device__ const float* bias(const DevModel& m) { return m.bf; }
};

__global__ void k_count_elements(Batch b, int nel) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < b.natoms) {
        int e = b.elem[i];
        if (e >= 0) atomicAdd(&b.el_count[e], 1);
    }
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
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < b.natoms) {
        int e = b.elem[i];
        if (e >= 0) {
            int p = atomicAdd(&b.el_count[e], 1);
            b.el_atoms[b.el_start[e] + p] = i;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_mlp(Batch b, DevModel m, int maxw) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T* sm = (T*)sm_raw;
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
    const int nin = m.nin_el[e];
    const int L = m.nlayers;
    // shared layout: x[kTile][nin] | per layer c_l, y_l [kTile][w_l] | two delta buffers [kTile][maxw]
    T* x = sm;
    T* cbuf[8];
    T* ybuf[8];
    T* p = x + kTile * nin;
    for (int l = 0; l < L; ++l) {
        cbuf[l] = p;
        p += kTile * m.width[l + 1];
        ybuf[l] = p;
        p += kTile * m.width[l + 1];
    }
    T* d0 = p;
    T* d1 = p + kTile * maxw;
    const int tid = threadIdx.x;
    const T* Gin = MB<T>::G(b);
    for (int idx = tid; idx < kTile * nin; idx += kThreads) {
        int a = idx / nin, i = idx % nin;
        x[idx] = a < cnt ? Gin[(size_t)b.el_atoms[t0 + a] * m.nsf_max + i] : (T)0;
    }
    __syncthreads();
    // forward
    const T* in = x;
    int win = nin;
    for (int l = 0; l < L; ++l) {
        const int wout = m.width[l + 1];
        const T* WT = MB<T>::wt(m) + m.w_off[e * L + l];
        const T* bb = MB<T>::bias(m) + m.b_off[e * L + l];
        const char act = m.act[l];
        for (int idx = tid; idx < kTile * wout; idx += kThreads) {
            int a = idx / wout, o = idx % wout;
            T s = (T)0;
            const T* xa = in + a * win;
            for (int i = 0; i < win; ++i) s += WT[(size_t)i * wout + o] * xa[i];
            T c = s + bb[o];
            cbuf[l][idx] = c;
            ybuf[l][idx] = act_f(act, c);
        }
        __syncthreads();
        in = ybuf[l];
        win = wout;
    }
    // energy
    for (int a = tid; a < cnt; a += kThreads)
        MB<T>::atE(b)[b.el_atoms[t0 + a]] = (T)((double)ybuf[L - 1][a * m.width[L]] + m.atom_energy[e]);
    // backward: delta of the output layer (gradOut = 1)
    {
        const int w = m.width[L];
        for (int idx = tid; idx < kTile * w; idx += kThreads)
            d0[idx] = act_d(m.act[L - 1], cbuf[L - 1][idx], ybuf[L - 1][idx]);
    }
    __syncthreads();
    T* dcur = d0;
    T* dnext = d1;
    for (int l = L - 1; l >= 0; --l) {
        const int wout = m.width[l + 1];
        const int wi = (l == 0) ? nin : m.width[l];
        const T* W = MB<T>::w(m) + m.w_off[e * L + l];
        for (int idx = tid; idx < kTile * wi; idx += kThreads) {
            int a = idx / wi, i = idx % wi;
            T s = (T)0;
            const T* da = dcur + a * wout;
            for (int o = 0; o < wout; ++o) s += da[o] * W[(size_t)o * wi + i];
            if (l == 0) {
                if (a < cnt) MB<T>::dEdG(b)[(size_t)b.el_atoms[t0 + a] * m.nsf_max + i] = s;
            } else {
                dnext[idx] = s * act_d(m.act[l - 1], cbuf[l - 1][idx], ybuf[l - 1][idx]);
            }
        }
        __syncthreads();
        T* tmp = dcur;
        dcur = dnext;
        dnext = tmp;
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

int launch_mlp(const Batch& b, const DevModel& m, cudaStream_t s) {
    run_mlp<double>(b, m, s);
    return 1;
}

int launch_mlp_fp32(const Batch& b, const DevModel& m, cudaStream_t s) {
    run_mlp<float>(b, m, s);
    return 1;
}

}  // namespace hdnnp

// mlp_tile.cuh -- activations and one element tile of the per-element
// networks (forward pass and dE/dG), shared by the batched network kernel
// (mlp.cu) and the single-block MD kernel for small molecules (fused_md.cu).
#pragma once

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

// One tile of up to kTile atoms of element e (atoms el_atoms[t0 .. t0+cnt)),
// evaluated by the whole block (blockDim.x == kThreads) with the activations
// in the shared memory at sm_raw (mlp_smem_bytes).
template <typename T>
__device__ __forceinline__ void mlp_tile(const Batch& b, const DevModel& m, int maxw, int e, int t0, int cnt,
                                         unsigned char* sm_raw) {
    T* sm = (T*)sm_raw;
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

}  // namespace hdnnp

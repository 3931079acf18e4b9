// mlp_tc.cu -- K5 of the mixed-precision form: per-element atomic networks
// with the first layer on the 5th-generation tensor cores (tcgen05).
//
// Same mathematics as nn_forward / nn_backward(gradOut = 1)
// (neuralNetworks.f90:94-158, 220-313; called per atom from
// hdnnps.f90:523-531).  One CTA evaluates a tile of 128 atoms of one element;
// thread m owns atom m, which is also TMEM lane m.
//   forward layer 1:  C1[128 x H] = G'[128 x K] W1^T        (tcgen05.mma, M=128)
//   layers 2..L:      per thread in FP32 registers (widths <= 32)
//   input gradient:   dE/dG'[128 x N] = delta1[128 x H] W1   (tcgen05.mma, N split
//                     into chunks of <= 256 columns)
// Both GEMMs run in FP16 with FP32 accumulation and a hi + lo split of both
// operands (x = hi + lo, both FP16): A B = Ahi Bhi + Ahi Blo + Alo Bhi, which
// carries about 22 significant bits, so the input gradient that sets the
// forces keeps FP32-level accuracy.  Weights are pre-scaled by a power of two
// (so that their lo parts stay normal FP16 numbers) and pre-packed at model
// upload in the K-major, no-swizzle core-matrix layout the MMA descriptors
// describe: 8 rows x 16 bytes per core matrix, rows 16 B apart, row groups
// (SBO) 128 B apart, K chunks of 8 elements (LBO) one row-group column apart.
// Operands are staged into shared memory with plain loads (the activations
// are converted FP32 -> FP16 hi/lo on the way), MMAs are issued by one
// thread, completion is signalled through an mbarrier by tcgen05.commit, and
// results are read back with tcgen05.ld.  Every mbarrier wait is bounded;
// on expiry the kernel raises status bit 16 and frees its TMEM.
#include <cuda_fp16.h>

#include "engine.h"

namespace hdnnp {

namespace {

constexpr int kM = 128;        // atoms per tile (TMEM lanes, MMA M)
constexpr int kThr = 512;      // threads per CTA: 16 warps; warp w serves TMEM lanes (rows)
                               // 32 (w % 4) .. +31 and quarter w / 4 of each layer's neurons
constexpr int kQ = kThr / kM;  // threads per row (4)
constexpr int kHq = 32 / kQ;   // neurons of a padded layer per thread (8)
constexpr int kX = 36;         // row stride (floats) of the activation exchange: 144 B rows,
                               // float4 accesses of a warp free of bank conflicts
constexpr int kH = 32;         // padded hidden width (N of GEMM 1, K of GEMM 2)
constexpr int kTmemCols = 512;
constexpr long long kWaitIters = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start, leading (K) and stride (M/N) byte
// offsets in 16-byte units, version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: FP16 x FP16 -> FP32, both operands K-major
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N) {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (long long it = 0; it < kWaitIters; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// byte offset of element (row, k) in a K-major core-matrix tile with `rows` rows
__device__ __forceinline__ uint32_t cm_off(int row, int k, int rows) {
    return (uint32_t)((k >> 3) * (rows >> 3) * 128 + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void split_h(float x, __half& hi, __half& lo) {
    hi = __float2half_rn(x);
    lo = __float2half_rn(x - __half2float(hi));
}

__device__ __forceinline__ float act_fw(char a, float x) {
    switch (a) {
        case 't': return tanhf(x);
        case 'p': return log1pf(expf(x));
        case 'r': return x > 0.f ? x : 0.f;
        default: return x;
    }
}
__device__ __forceinline__ float act_dv(char a, float c, float y) {
    switch (a) {
        case 't': return 1.f - y * y;
        case 'p': return 1.f / (1.f + expf(-c));
        case 'r': return c > 0.f ? 1.f : 0.f;
        default: return 1.f;
    }
}

// Shared-memory plan (bytes):
//   [0, szA)            A_fwd hi | lo  (128 x Kp each); reused for B_bwd hi|lo and A_bwd hi|lo
//   [szA, szA+szBf)     B_fwd hi | lo  (32 x Kp each)
//   then FP32 small weights of layers 2..L (b1 and each layer's W [32][32]
//   and bias [32], zero-padded: rows read as float4), the mbarrier, the TMEM slot
struct TCPlan {
    int Kp, Np, nch, chN;
    size_t szA, szBf, szBb, szAb, szW, total;
};

__host__ __device__ inline TCPlan tc_plan(const DevModel& m) {
    TCPlan p{};
    p.Kp = m.tc_kp;
    p.Np = m.tc_np;
    p.nch = m.tc_nch;
    p.chN = m.tc_chn;
    p.szA = (size_t)2 * kM * p.Kp * 2;
    p.szBf = (size_t)2 * kH * p.Kp * 2;
    p.szBb = (size_t)2 * p.Np * kH * 2;
    p.szAb = (size_t)2 * kM * kH * 2;
    const size_t w = kH + (size_t)(m.nlayers - 1) * (kH * kH + kH);  // b1, then W_l and b_l padded
    p.szW = ((w * 4) + 15) & ~size_t(15);
    // the A_fwd region after GEMM 1: B_bwd | A_bwd, then the activation
    // exchange of the hidden layers (two [kM][kH] FP32 buffers)
    size_t reuse = p.szBb + p.szAb + (size_t)2 * kM * kX * 4;
    p.total = (p.szA > reuse ? p.szA : reuse) + p.szBf + p.szW + 64;
    return p;
}

template <int NL>
__global__ void __launch_bounds__(kThr, 1) k_mlp_tc(Batch b, DevModel m) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const TCPlan P = tc_plan(m);
    const int tid = threadIdx.x, warp = tid >> 5;
    // locate (element, tile)
    int tile = blockIdx.x, e = -1, t0 = 0, cnt = 0;
    for (int x = 0; x < m.nel; ++x) {
        const int n = b.el_start[x + 1] - b.el_start[x];
        const int nt = (n + kM - 1) / kM;
        if (tile < nt) {
            e = x;
            t0 = b.el_start[x] + tile * kM;
            cnt = min(kM, n - tile * kM);
            break;
        }
        tile -= nt;
    }
    if (e < 0) return;
    const int nin = m.nin_el[e];
    const int H = m.width[1];
    constexpr int L = NL;
    unsigned char* sA = sm;
    const size_t reuse = P.szBb + P.szAb + (size_t)2 * kM * kX * 4;  // B_bwd | A_bwd | exchange
    unsigned char* sBf = sm + (P.szA > reuse ? P.szA : reuse);
    float* sW = (float*)(sBf + P.szBf);
    uint64_t* mbar = (uint64_t*)((unsigned char*)sW + P.szW);
    uint32_t* tslot = (uint32_t*)(mbar + 1);
    const uint32_t mb = smem_u32(mbar);

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }

    // ---- stage B_fwd (pre-packed hi|lo) and the small FP32 weights
    {
        const uint4* src = (const uint4*)(m.tc_fwd + (size_t)e * (P.szBf / 2));
        uint4* dst = (uint4*)sBf;
        for (int i = tid; i < (int)(P.szBf / 16); i += kThr) dst[i] = src[i];
        int o = 0;
        const float* b1 = m.bf + m.b_off[e * L + 0];
        for (int i = tid; i < kH; i += kThr) sW[i] = i < H ? b1[i] : 0.f;
        o += kH;
        for (int l = 1; l < L; ++l) {
            const int wi = m.width[l], wo = m.width[l + 1];
            const float* W = m.wf + m.w_off[e * L + l];
            const float* bb = m.bf + m.b_off[e * L + l];
            for (int i = tid; i < kH * kH; i += kThr) {
                const int r = i / kH, q = i % kH;
                sW[o + i] = (r < wo && q < wi) ? W[r * wi + q] : 0.f;
            }
            o += kH * kH;
            for (int i = tid; i < kH; i += kThr) sW[o + i] = i < wo ? bb[i] : 0.f;
            o += kH;
        }
    }
    // ---- stage A_fwd: thread (row, quarter q); its row of G' (FP32) -> FP16
    // hi | lo in groups of 4 k (one 8-byte store per part), zero padding; the
    // quarter takes every kQ-th block of 32 k.  32 values are loaded before
    // any is stored, so each thread keeps 8 vector loads in flight.
    const int row = (warp & 3) * 32 + (tid & 31), quarter = warp >> 2;
    {
        __half* Ahi = (__half*)sA;
        __half* Alo = (__half*)(sA + P.szA / 2);
        const int kp = P.Kp;
        const int r = row;
        const int at = r < cnt ? b.el_atoms[t0 + r] : -1;
        const float* grow = at >= 0 ? b.Gf + (size_t)at * m.nsf_max : nullptr;
        const bool vec = (m.nsf_max & 3) == 0;
        for (int k0 = 32 * quarter; k0 < kp; k0 += 32 * kQ) {
            float x[32];
            if (vec && at >= 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int k = k0 + 4 * q;
                    float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (k + 3 < nin) f = *(const float4*)(grow + k);
                    else {
                        if (k < nin) f.x = grow[k];
                        if (k + 1 < nin) f.y = grow[k + 1];
                        if (k + 2 < nin) f.z = grow[k + 2];
                    }
                    x[4 * q] = f.x; x[4 * q + 1] = f.y; x[4 * q + 2] = f.z; x[4 * q + 3] = f.w;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 32; ++q) x[q] = (at >= 0 && k0 + q < nin) ? grow[k0 + q] : 0.f;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = k0 + 4 * q;
                if (k < kp) {
                    __half h[4], l[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) split_h(x[4 * q + u], h[u], l[u]);
                    const uint32_t off = cm_off(r, k, kM);
                    auto pk = [](const __half (&v)[4]) {
                        return make_uint2((uint32_t)__half_as_ushort(v[0]) | ((uint32_t)__half_as_ushort(v[1]) << 16),
                                          (uint32_t)__half_as_ushort(v[2]) | ((uint32_t)__half_as_ushort(v[3]) << 16));
                    };
                    *(uint2*)((unsigned char*)Ahi + off) = pk(h);
                    *(uint2*)((unsigned char*)Alo + off) = pk(l);
                }
            }
        }
    }
    fence_async_smem();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    bool ok = true;

    // ---- GEMM 1: C1[128 x 32] = A_fwd * B_fwd^T  (K = Kp in steps of 16)
    if (tid == 0) {
        const uint32_t aH = smem_u32(sA), aL = aH + (uint32_t)(P.szA / 2);
        const uint32_t bH = smem_u32(sBf), bL = bH + (uint32_t)(P.szBf / 2);
        const uint32_t lboA = (kM / 8) * 128, lboB = (kH / 8) * 128;
        const uint32_t id = idesc_f16(kM, kH);
        for (int s = 0; s < P.Kp / 16; ++s) {
            const uint32_t oa = (uint32_t)(2 * s) * lboA, ob = (uint32_t)(2 * s) * lboB;
            mma_f16(tbase, umma_desc(aH + oa, lboA, 128), umma_desc(bH + ob, lboB, 128), id, s > 0);
            mma_f16(tbase, umma_desc(aH + oa, lboA, 128), umma_desc(bL + ob, lboB, 128), id, 1);
            mma_f16(tbase, umma_desc(aL + oa, lboA, 128), umma_desc(bH + ob, lboB, 128), id, 1);
        }
        mma_commit(mb);
    }
    ok = mbar_wait(mb, 0);
    tc_fence_after();
    ok = __syncthreads_and(ok ? 1 : 0) != 0;  // A_fwd is free from here on

    const bool live = row < cnt;
    const int atom = live ? b.el_atoms[t0 + row] : 0;
    // activation exchange: two [kM][kX] buffers after B_bwd | A_bwd in the A_fwd region
    float* xa = (float*)(sA + P.szBb + P.szAb);
    float* xb = xa + kM * kX;
    const int o0 = quarter * kHq;  // this thread's neurons o0 .. o0 + kHq - 1
    if (ok) {
        constexpr int kWB = kH * kH + kH;
        auto woff = [](int l) { return kH + (l - 1) * kWB; };
        auto boff = [](int l) { return kH + (l - 1) * kWB + kH * kH; };
        float v[32];
        tmem_ld32(tbase + ((uint32_t)((warp & 3) * 32) << 16), v);
        const float inv = m.tc_inv_s1[e];
        float dact[NL][kHq];  // act'(c) of this thread's neurons of every layer
        // own eight values of a row of the exchange buffer, as two float4
        auto put8 = [&](float* buf, const float (&x)[kHq]) {
            float4* d4 = (float4*)(buf + row * kX + o0);
            d4[0] = make_float4(x[0], x[1], x[2], x[3]);
            d4[1] = make_float4(x[4], x[5], x[6], x[7]);
        };
        // first hidden layer: own neurons, activations to the exchange buffer
        {
            float y8[kHq];
#pragma unroll
            for (int u = 0; u < kHq; ++u) {
                const int o = o0 + u;
                float c = 0.f, yv = 0.f, dv = 0.f;
#pragma unroll
                for (int qq = 0; qq < kQ; ++qq)  // v[o] with a compile-time index
                    if (qq == quarter) c = v[qq * kHq + u];
                if (o < H) {
                    c = c * inv + sW[o];
                    yv = act_fw(m.act[0], c);
                    dv = act_dv(m.act[0], c, yv);
                }
                y8[u] = yv;
                dact[0][u] = dv;
            }
            put8(xa, y8);
        }
        __syncthreads();
        // Layers 2..L: each thread its neurons from the whole previous layer
        // (read back from the exchange buffer); padded rows read as float4
        // (broadcast), neurons beyond the layer's width skipped by a branch
        // uniform over the CTA.  Padding adds only zero terms, in the same
        // order as the unpadded sums.
        float* cur = xa;
        float* nxt = xb;
        float yout = 0.f;  // output neuron (quarter 0)
#pragma unroll
        for (int l = 1; l < NL; ++l) {
            const int wo = m.width[l + 1];
            const float4* W4 = (const float4*)(sW + woff(l));
            const float* bb = sW + boff(l);
            const char al = m.act[l];
            float yp[kH], y8[kHq];
#pragma unroll
            for (int q = 0; q < kH / 4; ++q) {
                const float4 t = *(const float4*)(cur + row * kX + 4 * q);
                yp[4 * q] = t.x; yp[4 * q + 1] = t.y; yp[4 * q + 2] = t.z; yp[4 * q + 3] = t.w;
            }
#pragma unroll
            for (int u = 0; u < kHq; ++u) {
                const int o = o0 + u;
                float c = 0.f, yv = 0.f, dv = 0.f;
                if (o < wo) {
                    c = bb[o];
#pragma unroll
                    for (int q = 0; q < kH / 4; ++q) {
                        const float4 w = W4[o * (kH / 4) + q];
                        c += w.x * yp[4 * q];
                        c += w.y * yp[4 * q + 1];
                        c += w.z * yp[4 * q + 2];
                        c += w.w * yp[4 * q + 3];
                    }
                    yv = act_fw(al, c);
                    dv = act_dv(al, c, yv);
                }
                y8[u] = yv;
                dact[l][u] = dv;
                if (l == NL - 1 && o == 0) yout = yv;
            }
            put8(nxt, y8);
            __syncthreads();
            float* t = cur;
            cur = nxt;
            nxt = t;
        }
        if (live && quarter == 0) b.atEf[atom] = (float)((double)yout + m.atom_energy[e]);
        // backward (gradOut = 1) down to the first hidden layer: deltas of
        // this thread's neurons; the whole delta vector of a layer through
        // the exchange buffer
        put8(cur, dact[NL - 1]);
        __syncthreads();
        float d[kHq];
#pragma unroll
        for (int l = NL - 1; l >= 1; --l) {
            const int wo = m.width[l + 1];
            const float4* W4 = (const float4*)(sW + woff(l));
            float dl[kH];
#pragma unroll
            for (int q = 0; q < kH / 4; ++q) {
                const float4 t = *(const float4*)(cur + row * kX + 4 * q);
                dl[4 * q] = t.x; dl[4 * q + 1] = t.y; dl[4 * q + 2] = t.z; dl[4 * q + 3] = t.w;
            }
            float g[kHq];
#pragma unroll
            for (int u = 0; u < kHq; ++u) g[u] = 0.f;
            // g_i = sum over o (ascending) of W[o][i] d_o, for this thread's i
#pragma unroll
            for (int o = 0; o < kH; ++o) {
                if (o < wo) {
#pragma unroll
                    for (int q = 0; q < kHq / 4; ++q) {
                        const float4 w = W4[o * (kH / 4) + quarter * (kHq / 4) + q];
                        g[4 * q] += w.x * dl[o];
                        g[4 * q + 1] += w.y * dl[o];
                        g[4 * q + 2] += w.z * dl[o];
                        g[4 * q + 3] += w.w * dl[o];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kHq; ++u) d[u] = g[u] * dact[l - 1][u];
            if (l > 1) {
                put8(nxt, d);
                __syncthreads();
                float* t = cur;
                cur = nxt;
                nxt = t;
            }
        }
        if (NL == 1) {
#pragma unroll
            for (int u = 0; u < kHq; ++u) d[u] = dact[0][u];
        }
        // ---- stage A_bwd (delta1 scaled, hi | lo: this thread's k) and B_bwd
        // in the A_fwd region
        __half* Bhi = (__half*)sA;
        __half* Ahi = (__half*)(sA + P.szBb);
        __half* Alo = (__half*)(sA + P.szBb + P.szAb / 2);
        const float sd = m.tc_sdelta;
#pragma unroll
        for (int u = 0; u < kHq; ++u) {
            __half h, lo;
            split_h(live ? d[u] * sd : 0.f, h, lo);
            const uint32_t o2 = cm_off(row, o0 + u, kM) >> 1;
            Ahi[o2] = h;
            Alo[o2] = lo;
        }
        const uint4* src = (const uint4*)(m.tc_bwd + (size_t)e * (P.szBb / 2));
        uint4* dst = (uint4*)Bhi;
        for (int i = tid; i < (int)(P.szBb / 16); i += kThr) dst[i] = src[i];
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const int okall = __syncthreads_and(ok ? 1 : 0);

    // ---- GEMM 2: dE/dG'[128 x Np] = A_bwd * B_bwd^T (K = 32, N in chunks)
    if (okall) {
        if (tid == 0) {
            const uint32_t bH = smem_u32(sA), bL = bH + (uint32_t)(P.szBb / 2);
            const uint32_t aH = smem_u32(sA) + (uint32_t)P.szBb, aL = aH + (uint32_t)(P.szAb / 2);
            const uint32_t lboA = (kM / 8) * 128, lboB = (uint32_t)(P.Np / 8) * 128;
            const uint32_t id = idesc_f16(kM, P.chN);
            for (int c = 0; c < P.nch; ++c) {
                const uint32_t dcol = tbase + kH + (uint32_t)(c * P.chN);
                const uint32_t boff = (uint32_t)(c * P.chN / 8) * 128;
                for (int s = 0; s < kH / 16; ++s) {
                    const uint32_t oa = (uint32_t)(2 * s) * lboA, ob = (uint32_t)(2 * s) * lboB + boff;
                    mma_f16(dcol, umma_desc(aH + oa, lboA, 128), umma_desc(bH + ob, lboB, 128), id, s > 0);
                    mma_f16(dcol, umma_desc(aH + oa, lboA, 128), umma_desc(bL + ob, lboB, 128), id, 1);
                    mma_f16(dcol, umma_desc(aL + oa, lboA, 128), umma_desc(bH + ob, lboB, 128), id, 1);
                }
            }
            mma_commit(mb);
        }
        ok = mbar_wait(mb, 1);
        tc_fence_after();
        if (ok) {
            const float inv = m.tc_inv_s1[e] / m.tc_sdelta;
            float* out = b.dEdGf + (size_t)atom * m.nsf_max;
            for (int c0 = 32 * quarter; c0 < P.nch * P.chN; c0 += 32 * kQ) {
                float v[32];
                tmem_ld32(tbase + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(kH + c0), v);
                if (live) {
                    if ((m.nsf_max & 3) == 0 && c0 + 32 <= nin) {
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            *(float4*)(out + c0 + 4 * q) = make_float4(v[4 * q] * inv, v[4 * q + 1] * inv,
                                                                       v[4 * q + 2] * inv, v[4 * q + 3] * inv);
                    } else {
#pragma unroll
                        for (int i = 0; i < 32; ++i)
                            if (c0 + i < nin) out[c0 + i] = v[i] * inv;
                    }
                }
            }
        }
    }
    if (!ok && tid == 0) atomicOr(&b.status[0], 16);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTmemCols) : "memory");
    }
}

}  // namespace

size_t mlp_tc_smem_bytes(const DevModel& m) { return tc_plan(m).total; }

template <int NL>
void run_tc(const Batch& b, const DevModel& m, cudaStream_t s) {
    const size_t smem = tc_plan(m).total;
    cudaFuncSetAttribute(k_mlp_tc<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int tiles = b.natoms / kM + m.nel + 1;
    k_mlp_tc<NL><<<tiles, kThr, smem, s>>>(b, m);
}

int launch_mlp_tc(const Batch& b, const DevModel& m, cudaStream_t s) {
    switch (m.nlayers) {
        case 2: run_tc<2>(b, m, s); break;
        case 3: run_tc<3>(b, m, s); break;
        case 4: run_tc<4>(b, m, s); break;
        default: return 0;
    }
    return 1;
}

}  // namespace hdnnp

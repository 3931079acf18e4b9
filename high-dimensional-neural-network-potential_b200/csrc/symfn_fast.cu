// symfn_fast.cu -- K4/K6 symmetry-function kernels on the potential's
// lambda x zeta x eta grid ("product space"), FP64 or FP32.
//
// Same mathematics as symfn.cu (calcAllSymmetryFunctions,
// symmetryFunctions.f90:158-308; scaling hdnnps.f90:471-481), organised so
// that the per-(pair, SF) work is one fused multiply-add:
//   * per pair: X_l = 1 + lambda_l cos, one square chain X, X^2, X^4, ...
//     shared by every zeta, T_lz = X_l^zeta_z (and X_l^(zeta_z - 1) for the
//     gradient), and one exponential Y_e = exp(-eta_e (r_ij^2+r_ik^2+r_jk^2))
//     per distinct eta;
//   * pass 1 accumulates acc[l,z,e] += T_lz Y_e fcp in registers and maps the
//     product entries to SF indices at the end of each element-pair block
//     (G_s = 2^(1-zeta) acc[l,z,e]);
//   * pass 2 stages per block the weight tensors WA[l,z,e] = w_s 2^(1-zeta)
//     and WC = WA lambda zeta (w_s = dE/dG_s / (max_s - min_s)) and contracts
//     A = sum WA T Y, B = sum eta WA T Y, C = sum WC T' Y per pair, from which
//     dE/dr_j and dE/dr_k are assembled as in symfn.cu.
// Per-neighbour 1/r is precomputed, so a pair needs one sqrt, one tanh and
// one exp per distinct eta.  Warp per centre atom; neighbours staged in
// shared memory sorted by element; candidate pairs compacted through a shared
// queue; chunks of 32 contributing pairs, one per lane.
#include <algorithm>

#include "engine.h"
#include "fastmath.cuh"

namespace hdnnp {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;
// Resident blocks per SM the FP32 kernels are compiled for (registers): 7 x 4
// warps for the value pass, 8 x 4 for the gradient pass (a few bytes of
// spill), which the shared memory of a launch sized for 64 neighbours also
// allows.  The FP64 kernels keep their registers (4 blocks).

template <typename T>
struct alignas(4 * sizeof(T)) V4 {
    T x, y, z, w;
};

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) & ~size_t(15); }

template <typename T>
struct FSmem {
    V4<T>* nb;      // dx, dy, dz, r        (centre - neighbour)
    double4* dd;    // FP32 value pass: the FP64 relative vector (x, y, z, -) for the pair cutoff
    V4<T>* ax;      // fc, dfc/r, 1/r, -
    T* gx;          // gradient accumulators (pass 2), one array per component:
    T* gy;          // a slot's x, y, z in one 16- or 32-byte record put random
    T* gz;          // slots on 4 (FP64) or 8 (FP32) bank groups only
    int* ent;       // entry index of a slot (pass 2)
    unsigned char* el;
    unsigned* queue;
    int* est;
    int* cur;
    T* w2;          // dE/dG / width of the centre's radial SFs (pass 2)
    T* WA;          // [nblk][P] (pass 2)
    T* WC;
    T* red;         // [32][P+1] (pass 1)
};

template <typename T>
__host__ __device__ inline size_t fast_warp_bytes(int mm, int g2max, int nblk, int P, bool grad) {
    size_t b = a16(sizeof(V4<T>) * mm) * 2;
    if (sizeof(T) == 4 && !grad) b += a16(sizeof(double4) * mm);
    if (grad) b += 3 * a16(sizeof(T) * mm) + a16(sizeof(int) * mm) + a16(sizeof(T) * g2max) + 2 * a16(sizeof(T) * nblk * P);
    else b += a16(sizeof(T) * 32 * (P + 1));
    b += a16(mm) + 64 * sizeof(unsigned) + a16(sizeof(int) * (kMaxEl + 1)) + a16(sizeof(int) * kMaxEl);
    return b;
}

template <typename T>
__device__ inline FSmem<T> fcarve(unsigned char* p, int mm, int g2max, int nblk, int P, bool grad) {
    FSmem<T> s{};
    auto take = [&](size_t bytes) {
        unsigned char* q = p;
        p += a16(bytes);
        return q;
    };
    s.nb = (V4<T>*)take(sizeof(V4<T>) * mm);
    s.dd = (sizeof(T) == 4 && !grad) ? (double4*)take(sizeof(double4) * mm) : nullptr;
    s.ax = (V4<T>*)take(sizeof(V4<T>) * mm);
    if (grad) {
        s.gx = (T*)take(sizeof(T) * mm);
        s.gy = (T*)take(sizeof(T) * mm);
        s.gz = (T*)take(sizeof(T) * mm);
        s.ent = (int*)take(sizeof(int) * mm);
        s.w2 = (T*)take(sizeof(T) * g2max);
        s.WA = (T*)take(sizeof(T) * nblk * P);
        s.WC = (T*)take(sizeof(T) * nblk * P);
    } else {
        s.red = (T*)take(sizeof(T) * 32 * (P + 1));
    }
    s.el = (unsigned char*)take(mm);
    s.queue = (unsigned*)take(64 * sizeof(unsigned));
    s.est = (int*)take(sizeof(int) * (kMaxEl + 1));
    s.cur = (int*)take(sizeof(int) * kMaxEl);
    return s;
}

// P consecutive weights of one block from shared memory in 16-byte loads
// (P is a multiple of 4; each block's tensor starts on a 16-byte boundary).
template <int P>
__device__ __forceinline__ void ldvec(const float* p, float (&w)[P]) {
#pragma unroll
    for (int q = 0; q < P / 4; ++q) {
        const float4 v = reinterpret_cast<const float4*>(p)[q];
        w[4 * q] = v.x;
        w[4 * q + 1] = v.y;
        w[4 * q + 2] = v.z;
        w[4 * q + 3] = v.w;
    }
}
template <int P>
__device__ __forceinline__ void ldvec(const double* p, double (&w)[P]) {
#pragma unroll
    for (int q = 0; q < P / 2; ++q) {
        const double2 v = reinterpret_cast<const double2*>(p)[q];
        w[2 * q] = v.x;
        w[2 * q + 1] = v.y;
    }
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// precision-dispatched math.  FP64: the branch-free forms of fastmath.cuh
// for the bounded arguments of these kernels (exp of -eta r^2, tanh of
// u = 1 - r/rc in [0, 1], square roots of squared distances).
__device__ __forceinline__ double xsqrt(double x) {
    double r, ir;
    sqrt_rsqrt(x, r, ir);
    return r;
}
__device__ __forceinline__ float xsqrt(float x) { return sqrtf(x); }
// r and 1/r from r^2 > 0: FP64 by the refined reciprocal square root of
// fastmath.cuh, FP32 by rsqrtf (2 ulp) and a product
__device__ __forceinline__ void dist_inv(double r2, double& r, double& ir) { sqrt_rsqrt(r2, r, ir); }
__device__ __forceinline__ void dist_inv(float r2, float& r, float& ir) {
    ir = rsqrtf(r2);
    r = r2 * ir;
}
// a / b: FP64 by division; FP32 by the fast reciprocal-based form (2 ulp,
// b between 2^-126 and 2^126)
__device__ __forceinline__ double xdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double xexp(double x) { return exp_clamped(x); }
// FP32 form: the exp2-based intrinsic (max error 2 + floor(1.173 |x|) ulp;
// the angular arguments stay below ~5, where it is within 8 ulp)
__device__ __forceinline__ float xexp(float x) { return __expf(x); }
// tanh of a cutoff argument u = 1 - r/rc in [0, 1]
__device__ __forceinline__ double xtanh(double x) { return tanh01(x); }
__device__ __forceinline__ float xtanh(float x) { return tanhf(x); }
__device__ __forceinline__ double xpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float xpow(float x, float y) { return powf(x, y); }

// Y[e] = exp(-eta_e R) for the distinct etas of the grid (zero beyond ne).
// kPowers (FP64 with integer eta ratios k_e = eta_e / eta_0,
// DevModel::eta_k): one exponential and Y[e] = Y[0]^k_e by squaring
// (relative error about k_e ulp, far below the FP64 tolerances); otherwise
// one exponential per eta.  With the branch-free FP64 exponential the value
// pass is faster with one exponential per eta (19.29 against 19.80 ms per C4
// step: independent sequences instead of a dependent chain of products), the
// gradient pass with the powers (18.20 against 18.60: it spills at 96
// registers otherwise).
template <int NE, bool kPowers, typename T>
__device__ __forceinline__ void eta_exps(const DevModel& m, int ne, T R, T (&Y)[NE]) {
    if (kPowers && sizeof(T) == 8 && NE > 1 && m.eta_k[0] == 1) {
        const T y0 = xexp(-(T)m.eta4[0] * R);
        Y[0] = y0;
#pragma unroll
        for (int e = 1; e < NE; ++e) {
            T r = (T)1, base = y0;
            int k = e < ne ? m.eta_k[e] : 0;
            if (e >= ne) r = (T)0;
#pragma unroll
            for (int bit = 0; bit < 7; ++bit) {
                if (k & 1) r *= base;
                k >>= 1;
                if (!k) break;
                base *= base;
            }
            Y[e] = r;
        }
        return;
    }
#pragma unroll
    for (int e = 0; e < NE; ++e) Y[e] = e < ne ? xexp(-(T)m.eta4[e] * R) : (T)0;
}

template <typename T> struct Buf;
template <> struct Buf<double> {
    static __device__ double* G(const Batch& b) { return b.G; }
    static __device__ const double* dEdG(const Batch& b) { return b.dEdG; }
    static __device__ double* gent(const Batch& b) { return b.gent; }
    static __device__ double* gself(const Batch& b) { return b.gself; }
    static __device__ double* vir(const Batch& b) { return b.vir; }
};
template <> struct Buf<float> {
    static __device__ float* G(const Batch& b) { return b.Gf; }
    static __device__ const float* dEdG(const Batch& b) { return b.dEdGf; }
    static __device__ float* gent(const Batch& b) { return b.gentf; }
    static __device__ float* gself(const Batch& b) { return b.gselff; }
    static __device__ float* vir(const Batch& b) { return b.virf; }
};

// Relative vector centre - image of neighbour entry (j, packed shift), FP64.
__device__ __forceinline__ void entry_vec(const Batch& b, const StructInfo& S, double xi, double yi, double zi, int j,
                                          int sh, double& dx, double& dy, double& dz) {
    int sx, sy, sz;
    unpack_shift(sh, sx, sy, sz);
    const double* h = S.h;
    double lx = 0, ly = 0, lz = 0;
    if (sz) { lx += h[6] * sz; ly += h[7] * sz; lz += h[8] * sz; }
    if (sy) { lx += h[3] * sy; ly += h[4] * sy; lz += h[5] * sy; }
    if (sx) { lx += h[0] * sx; ly += h[1] * sx; lz += h[2] * sx; }
    dx = xi - (b.wpos[3 * j] + lx);
    dy = yi - (b.wpos[3 * j + 1] + ly);
    dz = zi - (b.wpos[3 * j + 2] + lz);
}

// Stage the neighbour entries of atom i sorted by element (stable).  The
// relative vectors are formed in FP64 from the wrapped positions and image
// shifts and then rounded to T.  With a Verlet-skin list (list cutoff above
// rc) only entries with r < rc are staged; the gradient pass writes zero
// gradients for the others.  Returns the number of staged entries.
template <typename T, bool kGrad>
__device__ int fstage(const Batch& b, const DevModel& m, int i, int c, FSmem<T>& s, int lane, int M) {
    const int e0 = b.nei_off[i];
    const int nel = m.nel;
    const double xi = b.wpos[3 * i], yi = b.wpos[3 * i + 1], zi = b.wpos[3 * i + 2];
    const StructInfo& S = b.info[b.sid[i]];
    const double rc = m.rc[c];
    const bool filt = b.rc_list > rc;
    const double rc2 = rc * rc;
    if (lane < nel) s.cur[lane] = 0;
    __syncwarp();
    for (int base = 0; base < M; base += 32) {
        const int q = base + lane;
        bool keep = q < M;
        int el = 0;
        if (keep) {
            const int j = b.nei_j[e0 + q];
            el = b.elem[j];
            if (filt) {
                double dx, dy, dz;
                entry_vec(b, S, xi, yi, zi, j, b.nei_s[e0 + q], dx, dy, dz);
                keep = dx * dx + dy * dy + dz * dz < rc2;
            }
        }
        const unsigned act = __ballot_sync(kFull, keep);
        if (keep) {
            const unsigned peers = __match_any_sync(act, el);
            if ((peers & lanemask_lt()) == 0) s.cur[el] += __popc(peers);
        }
        __syncwarp();
    }
    if (lane == 0) {
        int acc = 0;
        for (int x = 0; x < nel; ++x) {
            s.est[x] = acc;
            acc += s.cur[x];
        }
        s.est[nel] = acc;
    }
    __syncwarp();
    if (lane < nel) s.cur[lane] = s.est[lane];
    __syncwarp();
    for (int base = 0; base < M; base += 32) {
        const int q = base + lane;
        int slot = 0, el = 0, j = 0, sh = 0;
        double dx = 0, dy = 0, dz = 0;
        bool keep = q < M;
        if (keep) {
            j = b.nei_j[e0 + q];
            sh = b.nei_s[e0 + q];
            el = b.elem[j];
            entry_vec(b, S, xi, yi, zi, j, sh, dx, dy, dz);
            if (filt && !(dx * dx + dy * dy + dz * dz < rc2)) {
                keep = false;
                if (kGrad) {
                    T* gent = Buf<T>::gent(b);
                    const size_t e = (size_t)(e0 + q);
                    gent[3 * e] = (T)0;
                    gent[3 * e + 1] = (T)0;
                    gent[3 * e + 2] = (T)0;
                }
            }
        }
        const unsigned act = __ballot_sync(kFull, keep);
        if (keep) {
            const unsigned peers = __match_any_sync(act, el);
            slot = s.cur[el] + __popc(peers & lanemask_lt());
            __syncwarp(act);
            if ((peers & lanemask_lt()) == 0) s.cur[el] += __popc(peers);
        }
        __syncwarp();
        if (keep) {
            // distance and cutoff in FP64
            double r, ir;
            sqrt_rsqrt(dx * dx + dy * dy + dz * dz, r, ir);
            const double irc = 1.0 / rc;
            double fc = 0.0, dfc = 0.0;
            if (r < rc) {
                const double t = tanh01(1.0 - r * irc), tt = t * t;
                fc = tt * t;
                dfc = -3.0 * irc * ir * (tt - tt * tt);
            }
            s.nb[slot] = V4<T>{(T)dx, (T)dy, (T)dz, (T)r};
            if (sizeof(T) == 4 && s.dd)
                s.dd[slot] = make_double4(dx, dy, dz, 0.0);
            s.ax[slot] = V4<T>{(T)fc, (T)dfc, (T)ir, (T)0};
            s.el[slot] = (unsigned char)el;
            if (kGrad) {
                s.gx[slot] = s.gy[slot] = s.gz[slot] = (T)0;
                s.ent[slot] = e0 + q;
            }
        }
    }
    __syncwarp();
    return s.est[nel];
}

// Candidate c of block (a,b) -> slots (j,k) without divisions: rectangular
// blocks use a float reciprocal of nb (exact for these sizes), triangular
// blocks a float square root with integer fix-ups.
__device__ __forceinline__ void fpair(int c, int sa, int na, int sb, int nb, bool same, float inv_nb, int& j, int& k) {
    if (!same) {
        int jj = (int)(((float)c + 0.5f) * inv_nb);
        int kk = c - jj * nb;
        if (kk < 0) { --jj; kk += nb; }
        else if (kk >= nb) { ++jj; kk -= nb; }
        j = sa + jj;
        k = sb + kk;
    } else {
        const float t = (float)(2 * na - 1);
        int jj = (int)((t - sqrtf(fmaxf(t * t - 8.0f * (float)c, 0.0f))) * 0.5f);
        if (jj < 0) jj = 0;
        auto off = [&](int x) { return x * (2 * na - x - 1) / 2; };
        while (jj > 0 && off(jj) > c) --jj;
        while (off(jj + 1) <= c) ++jj;
        j = sa + jj;
        k = sa + jj + 1 + (c - off(jj));
    }
}

// u = 1 - r_jk/rc for the pair cutoff.  In the FP32 form the difference
// cancels near rc; it is formed as (rc^2 - r_jk^2) / (rc (rc + r_jk)) with
// rc^2 - r_jk^2 taken in FP64.  The value pass takes it from the FP64
// relative vectors, so G stays accurate to FP32 rounding even for pairs just
// inside rc (whose SFs can have tiny scaling ranges and therefore large
// weights).  The gradient pass takes it from the FP32 vectors: its terms of
// such pairs scale with u^2, so the absolute error stays at FP32 rounding,
// and leaving the FP64 vectors out of its shared memory lets 8 blocks of it
// reside per SM instead of 7 (13.7 -> 11.3 ms per C4 step).
template <typename T>
__device__ __forceinline__ T pair_u(const FSmem<T>& s, int j, int k, double rc2d, T rc, T inv_rc, T rjk) {
    if (sizeof(T) == 8) {
        // FP64: 1 - r_jk / rc directly (r_jk < rc by the candidate test); its
        // absolute error is a few ulp, which near rc only touches terms of
        // order u^3
        const T u = (T)1 - rjk * inv_rc;
        return u > (T)0 ? u : (T)0;
    }
    double cx, cy, cz;
    if (sizeof(T) == 4 && s.dd) {
        // the FP64 relative vectors staged beside the FP32 ones (value pass)
        const double4 a = s.dd[j], b = s.dd[k];
        cx = b.x - a.x;
        cy = b.y - a.y;
        cz = b.z - a.z;
    } else {
        const V4<T> a = s.nb[j], b = s.nb[k];
        cx = (double)b.x - (double)a.x;
        cy = (double)b.y - (double)a.y;
        cz = (double)b.z - (double)a.z;
    }
    const double D = rc2d - (cx * cx + cy * cy + cz * cz);
    return D > 0.0 ? xdiv((T)D, rc * (rc + rjk)) : (T)0;
}

// ---------------------------------------------------------------- grid specs
// Spec<NL, NZ, NE, Z0..Z3>: compiled shape of the lambda x zeta x eta grid.
// With Z0 > 0 the zeta values are compile-time constants (the power chain and
// every product are straight-line code); with Z0 == 0 they are read from the
// model (uniform branches).
template <int NL_, int NZ_, int NE_, int Z0 = 0, int Z1 = 0, int Z2 = 0, int Z3 = 0>
struct Spec {
    static constexpr int NL = NL_, NZ = NZ_, NE = NE_, P = NL_ * NZ_ * NE_;
    static constexpr bool kFixed = Z0 > 0;
    __host__ __device__ static constexpr int zeta(int z) { return z == 0 ? Z0 : z == 1 ? Z1 : z == 2 ? Z2 : Z3; }
    __host__ __device__ static constexpr int maxbit() {
        int mz = 1;
        for (int z = 0; z < NZ_; ++z) mz = zeta(z) > mz ? zeta(z) : mz;
        int b = 0;
        while ((1 << (b + 1)) <= mz) ++b;
        return b;
    }
};

// X^E from the square chain ch[b] = X^(2^b); E is a compile-time constant
// after unrolling, so the bit tests fold away.
template <int E, typename T>
__device__ __forceinline__ T cpow(const T (&ch)[5]) {
    T r = (T)1;
#pragma unroll
    for (int bit = 0; bit < 5; ++bit)
        if ((E >> bit) & 1) r = r * ch[bit];
    return r;
}

template <typename T>
__device__ __forceinline__ T rpow(const T (&ch)[5], int e) {
    T r = (T)1;
#pragma unroll
    for (int bit = 0; bit < 5; ++bit)
        if ((e >> bit) & 1) r *= ch[bit];
    return r;
}

// Tz[z] = X^zeta_z and (kDeriv) Tp[z] = X^(zeta_z - 1) for one lambda.
template <class S, bool kDeriv, typename T>
__device__ __forceinline__ void powers(const DevModel& m, T X, T (&Tz)[S::NZ], T (&Tp)[S::NZ]) {
    T ch[5];
    ch[0] = X;
    if constexpr (S::kFixed) {
        constexpr int mb = S::maxbit();
#pragma unroll
        for (int b = 1; b < 5; ++b) ch[b] = b <= mb ? ch[b - 1] * ch[b - 1] : (T)0;
#pragma unroll
        for (int z = 0; z < S::NZ; ++z) {
            if constexpr (kDeriv) {
                // X^(zeta-1) from the chain, X^zeta = X^(zeta-1) * X
                T p = (T)1;
#pragma unroll
                for (int bit = 0; bit < 5; ++bit)
                    if (((S::zeta(z) - 1) >> bit) & 1) p = p * ch[bit];
                Tp[z] = p;
                Tz[z] = p * X;
            } else {
                T p = (T)1;
#pragma unroll
                for (int bit = 0; bit < 5; ++bit)
                    if ((S::zeta(z) >> bit) & 1) p = p * ch[bit];
                Tz[z] = p;
            }
        }
    } else {
#pragma unroll
        for (int b = 1; b < 5; ++b) ch[b] = b <= m.zmaxbit ? ch[b - 1] * ch[b - 1] : (T)0;
#pragma unroll
        for (int z = 0; z < S::NZ; ++z) {
            T p = (T)0, q = (T)0;
            if (z < m.fz) {
                const int ez = m.zint[z];
                if (kDeriv) {
                    p = ez >= 0 ? rpow(ch, ez) : xpow(X, (T)m.zet[z] - (T)1);
                    q = p * X;
                } else {
                    q = ez >= 0 ? rpow(ch, ez + 1) : xpow(X, (T)m.zet[z]);
                }
            }
            Tz[z] = q;
            if (kDeriv) Tp[z] = p;
        }
    }
}

// Packed FP32 form of powers() for NL == 2: both lambdas of a pair in one
// float2, X = (1 + lambda_0 cos, 1 + lambda_1 cos), squared and multiplied by
// the paired f32x2 instructions of sm_100 (fma.rn.f32x2 / mul.rn.f32x2; each
// half rounds exactly like the scalar instruction, so the results are those
// of powers<S, kDeriv, float>).
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

template <class S, bool kDeriv>
__device__ __forceinline__ void powers2(const DevModel& m, float2 X, float2 (&Tz)[S::NZ], float2 (&Tp)[S::NZ]) {
    float2 ch[5];
    ch[0] = X;
    if constexpr (S::kFixed) {
        constexpr int mb = S::maxbit();
#pragma unroll
        for (int b = 1; b < 5; ++b) ch[b] = b <= mb ? __fmul2_rn(ch[b - 1], ch[b - 1]) : f2(0.0f);
#pragma unroll
        for (int z = 0; z < S::NZ; ++z) {
            const int e = kDeriv ? S::zeta(z) - 1 : S::zeta(z);
            float2 p = f2(1.0f);
            bool first = true;
#pragma unroll
            for (int bit = 0; bit < 5; ++bit)
                if ((e >> bit) & 1) {
                    p = first ? ch[bit] : __fmul2_rn(p, ch[bit]);
                    first = false;
                }
            if constexpr (kDeriv) {
                Tp[z] = p;
                Tz[z] = __fmul2_rn(p, X);
            } else {
                Tz[z] = p;
            }
        }
    } else {
#pragma unroll
        for (int b = 1; b < 5; ++b) ch[b] = b <= m.zmaxbit ? __fmul2_rn(ch[b - 1], ch[b - 1]) : f2(0.0f);
#pragma unroll
        for (int z = 0; z < S::NZ; ++z) {
            float2 p = f2(0.0f), q = f2(0.0f);
            if (z < m.fz) {
                const int ez = m.zint[z];
                const int e = kDeriv ? ez : ez + 1;
                if (ez >= 0) {
                    float2 r = f2(1.0f);
#pragma unroll
                    for (int bit = 0; bit < 5; ++bit)
                        if ((e >> bit) & 1) r = __fmul2_rn(r, ch[bit]);
                    if (kDeriv) {
                        p = r;
                        q = __fmul2_rn(r, X);
                    } else {
                        q = r;
                    }
                } else if (kDeriv) {
                    const float zm = (float)m.zet[z] - 1.0f;
                    p = make_float2(powf(X.x, zm), powf(X.y, zm));
                    q = __fmul2_rn(p, X);
                } else {
                    const float zz = (float)m.zet[z];
                    q = make_float2(powf(X.x, zz), powf(X.y, zz));
                }
            }
            Tz[z] = q;
            if (kDeriv) Tp[z] = p;
        }
    }
}

template <class S>
__device__ __forceinline__ int n_eta(const DevModel& m) {
    return S::kFixed ? S::NE : m.fe;
}

// ---------------------------------------------------------------- pass 1
template <typename T, class S>
__global__ void __launch_bounds__(32 * kWarps, sizeof(T) == 4 ? 7 : 4) k_sfv_fast(Batch b, DevModel m, int mm, int mlo, int last) {
    constexpr int NL = S::NL, NZ = S::NZ, NE = S::NE, P = S::P;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    FSmem<T> s = fcarve<T>(smem_raw + wib * fast_warp_bytes<T>(mm, m.g2max, m.nblk, P, false), mm, m.g2max,
                           m.nblk, P, false);
    const int nel = m.nel;
    T* Gout = Buf<T>::G(b);
    const int ne = n_eta<S>(m);
    // work counters of this warp's atoms (profiling), added to b.stats once at the end
    unsigned long long st_ent = 0, st_cand = 0, st_pairs = 0, st_g2 = 0;
    for (int i = blockIdx.x * kWarps + wib; i < b.natoms; i += gridDim.x * kWarps) {
        const int c = b.elem[i];
        if (c < 0) continue;
        const int M = b.nei_off[i + 1] - b.nei_off[i];
        // this launch takes the atoms with mlo < M <= mm (see run_spec)
        if (M > mm) {
            if (last && lane == 0) atomicOr(&b.status[0], 4);
            continue;
        }
        if (M <= mlo) continue;
        const int Ms = fstage<T, false>(b, m, i, c, s, lane, M);
        const T rc = (T)m.rc[c], inv_rc = (T)(1.0 / m.rc[c]), rc2 = rc * rc;
        const double rc2d = m.rc[c] * m.rc[c];
        T* Gi = Gout + (size_t)i * m.nsf_max;
        const double* mean = m.smean + (size_t)c * m.nsf_max;
        const double* iwidth = m.sinvw + (size_t)c * m.nsf_max;

        // radial SFs: lane = SF, its neighbour element's staged neighbours in
        // order.  (A lane per (neighbour, SF) with shuffle sums was measured
        // slower in both precisions: 25.4 against 20.8 ms per C4 step in
        // FP64, 14.9 against 12.8 in FP32.  Groups of lanes per neighbour
        // element, each lane a function and a share of the neighbours, with a
        // butterfly over the groups, gained nothing.)
        const int r0 = m.g2_off[c * nel], r1 = m.g2_off[c * nel + nel];
        for (int f = r0 + lane; f < r1; f += 32) {
            const SF2 q = m.g2[f];
            const T eta = (T)q.eta, rs = (T)q.rs;
            T acc = (T)0;
            for (int t = s.est[q.nel]; t < s.est[q.nel + 1]; ++t) {
                const T x = s.nb[t].w - rs;
                acc += xexp(-eta * x * x) * s.ax[t].x;
            }
            Gi[q.sf] = (T)(((double)acc - mean[q.sf]) * iwidth[q.sf]);
        }

        unsigned long long n_cand = 0, n_pairs = 0;
        // Contributing pairs of all element-pair blocks go through one queue
        // (entries j | k << 10 | block << 20, enumeration order), so a chunk of
        // 32 pairs may hold the end of one block and the start of the next:
        // the lanes of the older block add their terms, every lane writes its
        // sums of that block for the reduction (the newer block's lanes the
        // sums they held before this chunk), and then the newer block's lanes
        // start their sums with their terms.  The queue holds at most two
        // blocks, and a block's remainder is carried into the next block's
        // chunks instead of being flushed as a partly filled chunk.
        // FP32 with two lambdas: the accumulators packed over lambda,
        // acc2[z * NE + e] = (acc[0, z, e], acc[1, z, e]).  FP64 with two
        // lambdas: the lambdas split over a lane pair (lane, lane ^ 1), each
        // lane adding lambda_(lane & 1) of both pairs' terms, acc[z * NE + e]
        // (half the accumulators and half the reduction per lane).
        constexpr bool kPk = sizeof(T) == 4 && NL == 2;
        constexpr bool kSp = sizeof(T) == 8 && NL == 2;
        constexpr int NA = kSp ? P / 2 : P;
        T acc[NA];
        float2 acc2[kPk ? NZ * NE : 1];
        auto zero_acc = [&]() {
#pragma unroll
            for (int p = 0; p < NA; ++p) acc[p] = (T)0;
#pragma unroll
            for (int p = 0; p < (kPk ? NZ * NE : 1); ++p) acc2[p] = f2(0.0f);
        };
        // terms of one pair: cos(theta) and Y[e] = exp(-eta_e R) fc_ij fc_ik fc_jk
        auto pair_terms = [&](unsigned pk, T& cth, T (&Y)[NE]) {
            const int pj = pk & 0x3ff, pq = (pk >> 10) & 0x3ff;
            const V4<T> a = s.nb[pj], bq = s.nb[pq];
            const V4<T> xa = s.ax[pj], xb = s.ax[pq];
            const T cx = bq.x - a.x, cy = bq.y - a.y, cz = bq.z - a.z;
            const T rjk2 = cx * cx + cy * cy + cz * cz;
            const T rjk = xsqrt(rjk2);
            const T tj = xtanh(pair_u(s, pj, pq, rc2d, rc, inv_rc, rjk));
            const T fjk = tj * tj * tj;
            const T t1 = -xa.z * xb.z;  // -1/(rj rk)
            cth = (T)0.5 * (rjk2 - a.w * a.w - bq.w * bq.w) * t1;
            const T fcp = xa.x * xb.x * fjk;
            const T R = a.w * a.w + bq.w * bq.w + rjk2;
            eta_exps<NE, false>(m, ne, R, Y);
#pragma unroll
            for (int e = 0; e < NE; ++e) Y[e] *= fcp;
        };
        // acc[l, z, e] += (1 + lambda_l cos)^zeta_z Y[e]
        auto accumulate = [&](T cth, const T (&Y)[NE]) {
            if constexpr (kPk) {
                const float2 X = __ffma2_rn(make_float2((float)m.lam[0], (float)m.lam[1]), f2((float)cth), f2(1.0f));
                float2 Tz[NZ], Tp[NZ];
                powers2<S, false>(m, X, Tz, Tp);
#pragma unroll
                for (int z = 0; z < NZ; ++z)
#pragma unroll
                    for (int e = 0; e < NE; ++e) acc2[z * NE + e] = __ffma2_rn(Tz[z], f2((float)Y[e]), acc2[z * NE + e]);
            } else if constexpr (kSp) {
                const T lam = (lane & 1) ? (T)m.lam[1] : (T)m.lam[0];
                T Tz[NZ], Tp[NZ];
                powers<S, false>(m, (T)1 + lam * cth, Tz, Tp);
#pragma unroll
                for (int z = 0; z < NZ; ++z)
#pragma unroll
                    for (int e = 0; e < NE; ++e) acc[z * NE + e] += Tz[z] * Y[e];
            } else {
#pragma unroll
                for (int l = 0; l < NL; ++l) {
                    T Tz[NZ], Tp[NZ];
                    powers<S, false>(m, (T)1 + (T)m.lam[l] * cth, Tz, Tp);
#pragma unroll
                    for (int z = 0; z < NZ; ++z)
#pragma unroll
                        for (int e = 0; e < NE; ++e) acc[(l * NZ + z) * NE + e] += Tz[z] * Y[e];
                }
            }
        };
        // every lane's sums of block t -> G of block t (warp reduction through
        // shared memory: rows of P + 1, or of P/2 + 1 with the lambda split);
        // called by all lanes
        auto emit = [&](int t) {
            if constexpr (kSp) {
                // rows of P/2: lane L holds lambda_(L & 1); output p = (l, z, e)
                // sums the 16 rows of parity l, 32/P helper lanes per output
                T* row = s.red + lane * (P / 2 + 1);
#pragma unroll
                for (int q = 0; q < P / 2; ++q) row[q] = acc[q];
                __syncwarp();
                constexpr int NH = 32 / P > 0 ? 32 / P : 1;
                static_assert(16 % NH == 0, "helpers per output");
                const int p = lane % P, hh = lane / P;
                const int l = p / (NZ * NE), q = p % (NZ * NE);
                T sum = (T)0;
                if (hh < NH)
#pragma unroll
                    for (int r = 0; r < 16 / NH; ++r) sum += s.red[(2 * (hh + r * NH) + l) * (P / 2 + 1) + q];
#pragma unroll
                for (int off = P; off < 32; off <<= 1) sum += __shfl_xor_sync(kFull, sum, off);
                __syncwarp();
                if (lane < P) {
                    const int sf = m.pmap[((size_t)c * m.nblk + t) * P + lane];
                    if (sf >= 0) {
                        const int z = (lane / NE) % NZ;
                        Gi[sf] = (T)(((double)((T)m.pfz[z] * sum) - mean[sf]) * iwidth[sf]);
                    }
                }
                return;
            }
            {
                T* row = s.red + lane * (P + 1);
                if constexpr (kPk) {
#pragma unroll
                    for (int q = 0; q < NZ * NE; ++q) {
                        row[q] = (T)acc2[q].x;            // l = 0
                        row[NZ * NE + q] = (T)acc2[q].y;  // l = 1
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < P; ++p) row[p] = acc[p];
                }
            }
            __syncwarp();
            constexpr int NH = 32 / P > 0 ? 32 / P : 1;
            const int p = lane % P, h = lane / P;
            T sum = (T)0;
            if (h < NH)
#pragma unroll
                for (int r = 0; r < 32 / NH; ++r) sum += s.red[(h + r * NH) * (P + 1) + p];
#pragma unroll
            for (int off = P; off < 32; off <<= 1) sum += __shfl_xor_sync(kFull, sum, off);
            __syncwarp();
            if (lane < P) {
                const int sf = m.pmap[((size_t)c * m.nblk + t) * P + lane];
                if (sf >= 0) {
                    const int z = (lane / NE) % NZ;
                    Gi[sf] = (T)(((double)((T)m.pfz[z] * sum) - mean[sf]) * iwidth[sf]);
                }
            }
        };
        int qlen = 0;   // pending queue entries
        int cur = -1;   // block whose sums the accumulators hold
        zero_acc();
        // process the first n queue entries (all lanes call)
        auto flush = [&](int n) {
            const unsigned pk = lane < n ? s.queue[lane] : 0u;
            const int tg = lane < n ? (int)(pk >> 20) : cur;
            T cth = (T)0, Y[NE];
#pragma unroll
            for (int e = 0; e < NE; ++e) Y[e] = (T)0;
            if (lane < n) pair_terms(pk, cth, Y);
            // a chunk that ends block cur and starts the next one (the last
            // lane's): cur's lanes add their terms, cur is reduced, then the
            // next block's lanes start their sums
            const bool straddle = __any_sync(kFull, tg != cur);
            const int nxt = straddle ? __shfl_sync(kFull, tg, n - 1) : cur;
            if constexpr (sizeof(T) == 8) {
                // FP64: one call site of the accumulation, in two passes
                // around the reduction (smaller code: the value pass was
                // instruction-fetch bound; 24.7 against 25.4 ms on the C4
                // batch).  With the lambda split this lane also takes its
                // partner's (lane ^ 1) pair, whose terms come by shuffle.
                T cth_o = (T)0, Y_o[NE];
                int tg_o = cur;
                const bool live_o = kSp && (lane ^ 1) < n;
                if constexpr (kSp) {
                    cth_o = __shfl_xor_sync(kFull, cth, 1);
#pragma unroll
                    for (int e = 0; e < NE; ++e) Y_o[e] = __shfl_xor_sync(kFull, Y[e], 1);
                    tg_o = __shfl_xor_sync(kFull, tg, 1);
                }
                for (int pass = 0; pass < (straddle ? 2 : 1); ++pass) {
                    if (pass == 1) {
                        emit(cur);
                        zero_acc();
                        cur = nxt;
                    }
                    for (int w2 = 0; w2 < (kSp ? 2 : 1); ++w2) {
                        const bool own = w2 == 0;
                        if (own ? (lane < n && tg == cur) : (live_o && tg_o == cur)) {
                            T Yw[NE];
#pragma unroll
                            for (int e = 0; e < NE; ++e) Yw[e] = own ? Y[e] : Y_o[e];
                            accumulate(own ? cth : cth_o, Yw);
                        }
                    }
                }
            } else if (!straddle) {
                // FP32 at 72 registers: the two-pass loop spills (70.4 against 73.0 ms)
                if (lane < n) accumulate(cth, Y);
            } else {
                if (lane < n && tg == cur) accumulate(cth, Y);
                emit(cur);
                zero_acc();
                if (lane < n && tg == nxt) accumulate(cth, Y);
                cur = nxt;
            }
            __syncwarp();
            const int rem = qlen - n;
            unsigned v = 0;
            if (lane < rem) v = s.queue[n + lane];
            __syncwarp();
            if (lane < rem) s.queue[lane] = v;
            __syncwarp();
            qlen = rem;
        };
        for (int t = 0; t < m.nblk; ++t) {
            const int gb = m.g4_off[c * m.nblk + t], ge = m.g4_off[c * m.nblk + t + 1];
            if (ge == gb) continue;
            if (cur < 0) cur = t;
            const int ea = m.blk_a[t], eb = m.blk_b[t];
            const int sa = s.est[ea], na = s.est[ea + 1] - sa;
            const int sb = s.est[eb], nb = s.est[eb + 1] - sb;
            const bool same = (ea == eb);
            const int ncand = same ? na * (na - 1) / 2 : na * nb;
            const float inv_nb = nb > 0 ? 1.0f / (float)nb : 0.0f;
            n_cand += ncand;
            for (int cb = 0; cb < ncand; cb += 32) {
                const int cidx = cb + lane;
                bool ok = cidx < ncand;
                int j = 0, k = 0;
                if (ok) {
                    fpair(cidx, sa, na, sb, nb, same, inv_nb, j, k);
                    const V4<T> a = s.nb[j], bb = s.nb[k];
                    const T ex = bb.x - a.x, ey = bb.y - a.y, ez = bb.z - a.z;
                    ok = ex * ex + ey * ey + ez * ez < rc2;
                }
                const unsigned bal = __ballot_sync(kFull, ok);
                const unsigned ent = (unsigned)j | ((unsigned)k << 10) | ((unsigned)t << 20);
                if (ok) s.queue[qlen + __popc(bal & lanemask_lt())] = ent;
                if (ok && b.pairs) {
                    // contributing-pair list for the gradient pass (enumeration order)
                    const long long slot = (long long)n_pairs + __popc(bal & lanemask_lt());
                    if (slot < b.pcap) b.pairs[(size_t)i * b.pcap + slot] = ent;
                }
                qlen += __popc(bal);
                n_pairs += __popc(bal);
                __syncwarp();
                while (qlen >= 32) flush(32);
            }
            // block t is screened.  An older block still pending in the queue
            // (its remainder followed by t's pairs, fewer than 32 together) is
            // finished now, and then t with it.
            if (cur != t) {
                if (qlen > 0) flush(qlen);
                if (cur != t) {  // t had no contributing pairs
                    emit(cur);
                    zero_acc();
                    cur = t;
                }
                if (qlen > 0) flush(qlen);
                emit(t);
                zero_acc();
                cur = -1;
            } else if (qlen == 0) {
                emit(t);
                zero_acc();
                cur = -1;
            }
        }
        if (cur >= 0) {
            if (qlen > 0) flush(qlen);
            emit(cur);
            zero_acc();
        }
        if (b.pairs && lane == 0) b.npairs[i] = n_pairs > (unsigned long long)INT32_MAX ? INT32_MAX : (int)n_pairs;
        if (b.stats) {
            // radial terms: staged neighbours of each element x the centre's radial SFs for it
            for (int el = 0; el < nel; ++el)
                st_g2 += (unsigned long long)(s.est[el + 1] - s.est[el]) *
                         (unsigned long long)(m.g2_off[c * nel + el + 1] - m.g2_off[c * nel + el]);
            st_ent += (unsigned long long)M;
            st_cand += n_cand;
            st_pairs += n_pairs;
        }
        __syncwarp();
    }
    if (b.stats && lane == 0 && st_ent) {
        atomicAdd(&b.stats[2], st_ent);
        atomicAdd(&b.stats[3], st_cand);
        atomicAdd(&b.stats[4], st_pairs);
        atomicAdd(&b.stats[5], st_pairs * (unsigned long long)P);
        atomicAdd(&b.stats[6], st_g2);
    }
}

// ---------------------------------------------------------------- pass 2
// (x, y, z) of every lane with `live` set added to gradient slot `slot`.  The
// lanes naming one slot form a group (__match_any_sync); its lowest lane adds
// the other members' values in ascending lane order (indexed shuffles, as many
// rounds as the largest group has members) and writes the slot with one plain
// read-modify-write, so no two lanes write one slot and the result does not
// depend on timing.  (Shared-memory FP64 atomicAdd measured 5.6 ms of the 21 ms
// FP64 gradient pass on the 4096-structure batch, against 0.3 ms for plain
// read-modify-writes; rounds of an integer atomicMin that elect one lane per
// slot cost as much as the atomics.)  Called by all lanes.
template <typename T>
__device__ __forceinline__ void group_add(const FSmem<T>& s, bool live, int slot, T x, T y, T z, int lane) {
    const unsigned grp = __match_any_sync(kFull, live ? slot : -1 - lane);
    const int most = __reduce_max_sync(kFull, __popc(grp));
    const bool lead = live && (grp & lanemask_lt()) == 0;
    unsigned rest = grp & ~(1u << lane);
    T sx = x, sy = y, sz = z;
    for (int r = 1; r < most; ++r) {
        const int src = rest ? __ffs(rest) - 1 : lane;
        const T ox = __shfl_sync(kFull, x, src);
        const T oy = __shfl_sync(kFull, y, src);
        const T oz = __shfl_sync(kFull, z, src);
        if (rest) {
            rest &= rest - 1;
            sx += ox;
            sy += oy;
            sz += oz;
        }
    }
    if (lead) {
        s.gx[slot] += sx;
        s.gy[slot] += sy;
        s.gz[slot] += sz;
    }
}

// Gradient contributions of up to 32 contributing pairs (one per lane; pk =
// j | k << 10 | block << 20, live for lane < n): dE/dr_k added to slot k,
// dE/dr_j summed over runs of equal j (lanes hold pairs in enumeration order,
// so equal j are contiguous) and added once per run.  Called by all lanes.
template <typename T, class S>
__device__ __forceinline__ void grad_pairs(const FSmem<T>& s, const DevModel& m, int ne, T rc, T inv_rc, double rc2d,
                                           unsigned pk_in, int n, int lane) {
    constexpr int NL = S::NL, NZ = S::NZ, NE = S::NE, P = S::P;
        // dE/dr_j of this lane's pair (summed over runs of equal j below) and
        // dE/dr_k
        int pj = -1 - lane, pq = -1 - lane;
        T gjx = (T)0, gjy = (T)0, gjz = (T)0, gkx = (T)0, gky = (T)0, gkz = (T)0;
        if (lane < n) {
            const unsigned pk = pk_in;
            pj = pk & 0x3ff;
            pq = (pk >> 10) & 0x3ff;
            const int pt = pk >> 20;
            const V4<T> a = s.nb[pj], bq = s.nb[pq];
            const V4<T> xa = s.ax[pj], xb = s.ax[pq];
            const T fj = xa.x, fk = xb.x, dfj = xa.y, dfk = xb.y;
            const T cx = bq.x - a.x, cy = bq.y - a.y, cz = bq.z - a.z;  // djk = r_j - r_k
            const T rjk2 = cx * cx + cy * cy + cz * cz;
            T rjk, irjk;
            dist_inv(rjk2, rjk, irjk);
            const T tj = xtanh(pair_u(s, pj, pq, rc2d, rc, inv_rc, rjk)), tt = tj * tj;
            const T fjk = tt * tj;
            const T dfjk = (T)(-3) * inv_rc * irjk * (tt - tt * tt);
            const T irj = xa.z, irk = xb.z;
            const T t1 = -irj * irk;
            const T cth = (T)0.5 * (rjk2 - a.w * a.w - bq.w * bq.w) * t1;
            const T dot = a.x * bq.x + a.y * bq.y + a.z * bq.z;
            const T cj = dot * irj * irj * irj * irk, ck = dot * irk * irk * irk * irj;
            const T fcp = fj * fk * fjk;
            const T R = a.w * a.w + bq.w * bq.w + rjk2;
            T Y[NE];
            eta_exps<NE, true>(m, ne, R, Y);
            T SA[NE], SC[NE];
#pragma unroll
            for (int e = 0; e < NE; ++e) SA[e] = SC[e] = (T)0;
            T wa[P], wc[P];
            ldvec<P>(s.WA + pt * P, wa);
            ldvec<P>(s.WC + pt * P, wc);
            if constexpr (sizeof(T) == 4 && NL == 2) {
                // packed over lambda: the weights are staged as (l = 0, l = 1)
                // pairs, wa[2 (z NE + e) + l] (see the staging in k_sfg_fast)
                const float2 X = __ffma2_rn(make_float2((float)m.lam[0], (float)m.lam[1]), f2((float)cth), f2(1.0f));
                float2 Tz[NZ], Tp[NZ];
                powers2<S, true>(m, X, Tz, Tp);
                float2 SA2[NE], SC2[NE];
#pragma unroll
                for (int e = 0; e < NE; ++e) SA2[e] = SC2[e] = f2(0.0f);
#pragma unroll
                for (int z = 0; z < NZ; ++z)
#pragma unroll
                    for (int e = 0; e < NE; ++e) {
                        const int q = 2 * (z * NE + e);
                        SA2[e] = __ffma2_rn(make_float2(wa[q], wa[q + 1]), Tz[z], SA2[e]);
                        SC2[e] = __ffma2_rn(make_float2(wc[q], wc[q + 1]), Tp[z], SC2[e]);
                    }
#pragma unroll
                for (int e = 0; e < NE; ++e) {
                    SA[e] = SA2[e].x + SA2[e].y;
                    SC[e] = SC2[e].x + SC2[e].y;
                }
            } else {
#pragma unroll
                for (int l = 0; l < NL; ++l) {
                    T Tz[NZ], Tp[NZ];
                    powers<S, true>(m, (T)1 + (T)m.lam[l] * cth, Tz, Tp);
#pragma unroll
                    for (int z = 0; z < NZ; ++z)
#pragma unroll
                        for (int e = 0; e < NE; ++e) {
                            SA[e] += wa[(l * NZ + z) * NE + e] * Tz[z];
                            SC[e] += wc[(l * NZ + z) * NE + e] * Tp[z];
                        }
                }
            }
            T A = (T)0, B = (T)0, C = (T)0;
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                A += Y[e] * SA[e];
                B += (T)m.eta4[e] * Y[e] * SA[e];
                C += Y[e] * SC[e];
            }
            const T B2 = (T)2 * B * fcp, Cf = C * fcp;
            const T pj1 = A * fk * fj * dfjk, pj2 = A * fk * dfj * fjk;
            const T pk1 = A * fj * fk * dfjk, pk2 = A * fj * dfk * fjk;
            gjx = pj1 * cx - pj2 * a.x + B2 * (a.x - cx) + Cf * (t1 * bq.x + a.x * cj);
            gjy = pj1 * cy - pj2 * a.y + B2 * (a.y - cy) + Cf * (t1 * bq.y + a.y * cj);
            gjz = pj1 * cz - pj2 * a.z + B2 * (a.z - cz) + Cf * (t1 * bq.z + a.z * cj);
            gkx = -pk1 * cx - pk2 * bq.x + B2 * (bq.x + cx) + Cf * (t1 * a.x + bq.x * ck);
            gky = -pk1 * cy - pk2 * bq.y + B2 * (bq.y + cy) + Cf * (t1 * a.y + bq.y * ck);
            gkz = -pk1 * cz - pk2 * bq.z + B2 * (bq.z + cz) + Cf * (t1 * a.z + bq.z * ck);
        }
        group_add(s, lane < n, pq, gkx, gky, gkz, lane);
        __syncwarp();
        // Queue order is enumeration order, so pairs sharing j sit in
        // contiguous lanes: a segmented suffix sum (fixed shuffle order)
        // leaves each run's total in its first lane, which alone
        // updates slot j -- instead of one conflicting atomic per lane.
        {
            // every lane executes the shuffle (no short-circuit around it)
            const int prev_j = __shfl_up_sync(kFull, pj, 1);
            const bool head = lane == 0 || prev_j != pj;
            const unsigned heads = __ballot_sync(kFull, head);
            const unsigned after = heads & ~((2u << lane) - 1u);  // heads above this lane
            const int last = after ? __ffs(after) - 2 : 31;        // last lane of my run
            // doubling steps up to the longest run of the chunk (later steps
            // would add nothing)
            const int longest = __reduce_max_sync(kFull, head ? last - lane + 1 : 1);
            for (int d = 1; d < longest; d <<= 1) {
                const T ox = __shfl_down_sync(kFull, gjx, d);
                const T oy = __shfl_down_sync(kFull, gjy, d);
                const T oz = __shfl_down_sync(kFull, gjz, d);
                if (lane + d <= last) {
                    gjx += ox;
                    gjy += oy;
                    gjz += oz;
                }
            }
            // run totals into their slots (one block's runs name distinct
            // slots; a chunk that spans two blocks can name one twice)
            group_add(s, head && lane < n, pj, gjx, gjy, gjz, lane);
        }
}

template <typename T, class S>
// FP64: 5 blocks per SM at 96 registers (a few spills) beat 4 at 120 (23.1
// against 23.9 ms on the C4 batch); the value pass loses at 5 (27.4 against 24.6)
__global__ void __launch_bounds__(32 * kWarps, sizeof(T) == 4 ? 8 : 5) k_sfg_fast(Batch b, DevModel m, int mm, int mlo, int last) {
    constexpr int NL = S::NL, NZ = S::NZ, NE = S::NE, P = S::P;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    FSmem<T> s = fcarve<T>(smem_raw + wib * fast_warp_bytes<T>(mm, m.g2max, m.nblk, P, true), mm, m.g2max,
                           m.nblk, P, true);
    const int nel = m.nel;
    const T* dEdG = Buf<T>::dEdG(b);
    const int ne = n_eta<S>(m);
    for (int i = blockIdx.x * kWarps + wib; i < b.natoms; i += gridDim.x * kWarps) {
        const int c = b.elem[i];
        if (c < 0) continue;
        const int M = b.nei_off[i + 1] - b.nei_off[i];
        // this launch takes the atoms with mlo < M <= mm (see run_spec)
        if (M > mm) {
            if (last && lane == 0) atomicOr(&b.status[0], 4);
            continue;
        }
        if (M <= mlo) continue;
        const int Ms = fstage<T, true>(b, m, i, c, s, lane, M);
        const T rc = (T)m.rc[c], inv_rc = (T)(1.0 / m.rc[c]), rc2 = rc * rc;
        const double rc2d = m.rc[c] * m.rc[c];
        // w_s = dE/dG_s / width_s: radial SFs staged per slot of g2, angular
        // ones folded into the product-space weight tensors of each block
        const T* dEdGi = dEdG + (size_t)i * m.nsf_max;
        const double* iwc = m.sinvw + (size_t)c * m.nsf_max;
        const int r0 = m.g2_off[c * nel], r1 = m.g2_off[c * nel + nel];
        for (int f = r0 + lane; f < r1; f += 32) {
            const int sf = m.g2[f].sf;
            s.w2[f - r0] = (T)((double)dEdGi[sf] * iwc[sf]);
        }
        for (int q = lane; q < m.nblk * P; q += 32) {
            const int t = q / P, p = q % P;
            const int sf = m.pmap[((size_t)c * m.nblk + t) * P + p];
            T wa = (T)0, wc = (T)0;
            const int l = p / (NZ * NE), z = (p / NE) % NZ;
            if (sf >= 0) {
                wa = (T)((double)dEdGi[sf] * iwc[sf]) * (T)m.pfz[z];
                wc = wa * (T)m.lam[l] * (T)m.zet[z];
            }
            // FP32 with two lambdas: (l = 0, l = 1) pairs for the packed contraction
            const int dst = (sizeof(T) == 4 && NL == 2) ? t * P + 2 * (p % (NZ * NE)) + l : q;
            s.WA[dst] = wa;
            s.WC[dst] = wc;
        }
        __syncwarp();

        // radial: lane = neighbour slot
        for (int t = lane; t < Ms; t += 32) {
            const int el = s.el[t];
            const int f0 = m.g2_off[c * nel + el], f1 = m.g2_off[c * nel + el + 1];
            const V4<T> d = s.nb[t];
            const V4<T> x = s.ax[t];
            T coef = (T)0;
            for (int f = f0; f < f1; ++f) {
                const SF2 q = m.g2[f];
                const T eta = (T)q.eta, xr = d.w - (T)q.rs;
                const T e = xexp(-eta * xr * xr);
                coef += s.w2[f - r0] * (-e * x.y + (T)2 * eta * xr * x.z * e * x.x);
            }
            s.gx[t] += coef * d.x;
            s.gy[t] += coef * d.y;
            s.gz[t] += coef * d.z;
        }
        __syncwarp();

        // angular: the contributing pairs listed by the value pass, or (list
        // missing or over capacity) screened again; the queue spans element-pair
        // blocks (entries carry the block)
        const int np = b.pairs ? b.npairs[i] : -1;
        if (np >= 0 && np <= b.pcap) {
            const unsigned* pl = b.pairs + (size_t)i * b.pcap;
            // the next chunk's entries are loaded while this chunk computes
            unsigned nxt = lane < np ? __ldg(pl + lane) : 0u;
            for (int base = 0; base < np; base += 32) {
                const int n = np - base < 32 ? np - base : 32;
                const unsigned pk = nxt;
                if (base + 32 < np) nxt = base + 32 + lane < np ? __ldg(pl + base + 32 + lane) : 0u;
                grad_pairs<T, S>(s, m, ne, rc, inv_rc, rc2d, lane < n ? pk : 0u, n, lane);
                __syncwarp();
            }
        } else {
        int qlen = 0;
        for (int t = 0; t < m.nblk; ++t) {
            const int gb = m.g4_off[c * m.nblk + t], ge = m.g4_off[c * m.nblk + t + 1];
            const bool has = ge > gb;
            const int ea = m.blk_a[t], eb = m.blk_b[t];
            const int sa = s.est[ea], na = s.est[ea + 1] - sa;
            const int sb = s.est[eb], nb = s.est[eb + 1] - sb;
            const bool same = (ea == eb);
            const int ncand = has ? (same ? na * (na - 1) / 2 : na * nb) : 0;
            const float inv_nb = nb > 0 ? 1.0f / (float)nb : 0.0f;
            const bool last_blk = (t == m.nblk - 1);
            for (int cb = 0; cb < ncand || (last_blk && cb == 0); cb += 32) {
                const int cidx = cb + lane;
                bool ok = cidx < ncand;
                int j = 0, k = 0;
                if (ok) {
                    fpair(cidx, sa, na, sb, nb, same, inv_nb, j, k);
                    const V4<T> a = s.nb[j], bb = s.nb[k];
                    const T ex = bb.x - a.x, ey = bb.y - a.y, ez = bb.z - a.z;
                    ok = ex * ex + ey * ey + ez * ez < rc2;
                }
                const unsigned bal = __ballot_sync(kFull, ok);
                if (ok) s.queue[qlen + __popc(bal & lanemask_lt())] = (unsigned)j | ((unsigned)k << 10) | ((unsigned)t << 20);
                qlen += __popc(bal);
                __syncwarp();
                const bool flush_all = last_blk && cb + 32 >= ncand;
                while (qlen >= 32 || (flush_all && qlen > 0)) {
                    const int n = qlen < 32 ? qlen : 32;
                    grad_pairs<T, S>(s, m, ne, rc, inv_rc, rc2d, lane < n ? s.queue[lane] : 0u, n, lane);
                    __syncwarp();
                    const int rem = qlen - n;
                    unsigned v = 0;
                    if (lane < rem) v = s.queue[n + lane];
                    __syncwarp();
                    if (lane < rem) s.queue[lane] = v;
                    __syncwarp();
                    qlen = rem;
                }
            }
        }
        }
        __syncwarp();
        T* gent = Buf<T>::gent(b);
        T sx = 0, sy = 0, sz = 0;
        T v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int t = lane; t < Ms; t += 32) {
            const V4<T> g{s.gx[t], s.gy[t], s.gz[t], (T)0};
            const V4<T> d = s.nb[t];
            const size_t e = (size_t)s.ent[t];
            gent[3 * e] = g.x;
            gent[3 * e + 1] = g.y;
            gent[3 * e + 2] = g.z;
            sx -= g.x;
            sy -= g.y;
            sz -= g.z;
            v[0] -= g.x * d.x; v[1] -= g.y * d.x; v[2] -= g.z * d.x;
            v[3] -= g.x * d.y; v[4] -= g.y * d.y; v[5] -= g.z * d.y;
            v[6] -= g.x * d.z; v[7] -= g.y * d.z; v[8] -= g.z * d.z;
        }
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(kFull, sx, o);
            sy += __shfl_xor_sync(kFull, sy, o);
            sz += __shfl_xor_sync(kFull, sz, o);
#pragma unroll
            for (int u = 0; u < 9; ++u) v[u] += __shfl_xor_sync(kFull, v[u], o);
        }
        if (lane == 0) {
            T* gs = Buf<T>::gself(b);
            T* vr = Buf<T>::vir(b);
            gs[3 * (size_t)i] = sx;
            gs[3 * (size_t)i + 1] = sy;
            gs[3 * (size_t)i + 2] = sz;
#pragma unroll
            for (int u = 0; u < 9; ++u) vr[9 * (size_t)i + u] = v[u];
        }
        __syncwarp();
    }
}

int nsm() { return device_sm_count(); }

template <typename K>
void set_smem(K kernel, size_t smem) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// Shared memory per warp grows with the largest neighbour count of the
// batch, and it sets how many warps an SM holds.  Atoms with at most `split`
// neighbours (64 by default: about 98 % in the dense workloads) run in a
// launch sized for that count; the rest follow in a second launch sized for
// the batch maximum.  Each atom is evaluated once, by the same code.  The
// split and the persistent grid (blocks per SM) are the knobs of the plans'
// autotuner (Batch::sf_split, Batch::sf_blocks_per_sm).
constexpr int kSplitCount = 64;
constexpr int kBlocksPerSm = 32;

template <typename T, class S>
int run_spec(const Batch& b, const DevModel& m, bool grad, cudaStream_t st) {
    const int mfull = b.mmax > 0 ? ((b.mmax + 31) / 32) * 32 : 32;
    int split = b.sf_split > 0 ? b.sf_split : b.sf_split < 0 ? mfull : kSplitCount;
    const int per_sm = b.sf_blocks_per_sm > 0 ? b.sf_blocks_per_sm : kBlocksPerSm;
    if (b.sf_split == 0 && mfull > split) {
        // a batch whose warps all fit on the GPU at the full size needs no
        // second launch (same code per atom: same results)
        const size_t blk = fast_warp_bytes<T>(mfull, m.g2max, m.nblk, S::P, grad) * kWarps;
        const int fit = std::min<int>(sizeof(T) == 4 ? (grad ? 8 : 7) : 4, (int)((227u * 1024u) / blk));
        if ((long long)b.natoms <= (long long)nsm() * fit * kWarps) split = mfull;
    }
    int L = 0;
    auto go = [&](int mm, int mlo, int last) {
        const size_t smem = fast_warp_bytes<T>(mm, m.g2max, m.nblk, S::P, grad) * kWarps;
        int blocks = (b.natoms + kWarps - 1) / kWarps;
        const int cap = nsm() * per_sm;
        if (blocks > cap) blocks = cap;
        if (blocks < 1) blocks = 1;
        if (grad) {
            set_smem(k_sfg_fast<T, S>, smem);
            k_sfg_fast<T, S><<<blocks, 32 * kWarps, smem, st>>>(b, m, mm, mlo, last);
        } else {
            set_smem(k_sfv_fast<T, S>, smem);
            k_sfv_fast<T, S><<<blocks, 32 * kWarps, smem, st>>>(b, m, mm, mlo, last);
        }
        ++L;
    };
    if (mfull > split) {
        go(split, -1, 0);
        go(mfull, split, 1);
    } else {
        go(mfull, -1, 1);
    }
    return L;
}

template <typename T>
int run_any(const Batch& b, const DevModel& m, bool grad, cudaStream_t st) {
    switch (m.fast) {
        case 1: return run_spec<T, Spec<2, 2, 1>>(b, m, grad, st);
        case 2: return run_spec<T, Spec<2, 4, 2>>(b, m, grad, st);
        case 3: return run_spec<T, Spec<2, 4, 4>>(b, m, grad, st);
        case 4: return run_spec<T, Spec<2, 8, 2>>(b, m, grad, st);
        case 5: return run_spec<T, Spec<2, 2, 1, 1, 4>>(b, m, grad, st);
        case 6: return run_spec<T, Spec<2, 4, 2, 1, 2, 4, 16>>(b, m, grad, st);
        default: return 0;
    }
}

}  // namespace

size_t sf_fast_smem_per_warp(int mmax, int g2max, int nblk, int P, bool grad, bool fp32) {
    const int mm = mmax > 0 ? ((mmax + 31) / 32) * 32 : 32;
    return fp32 ? fast_warp_bytes<float>(mm, g2max, nblk, P, grad) : fast_warp_bytes<double>(mm, g2max, nblk, P, grad);
}

int launch_sf_values_fast(const Batch& b, const DevModel& m, bool fp32, cudaStream_t st) {
    return fp32 ? run_any<float>(b, m, false, st) : run_any<double>(b, m, false, st);
}

int launch_sf_gradients_fast(const Batch& b, const DevModel& m, bool fp32, cudaStream_t st) {
    return fp32 ? run_any<float>(b, m, true, st) : run_any<double>(b, m, true, st);
}

}  // namespace hdnnp

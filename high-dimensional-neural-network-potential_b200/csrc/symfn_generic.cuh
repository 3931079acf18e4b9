// symfn_generic.cuh -- per-atom device routines of the generic (one record
// per symmetry function) kernels: neighbour staging, the values of one centre
// atom (sfv_atom) and its dE/dG-weighted gradients (sfg_atom), one warp per
// centre.  Shared by the batched kernels (symfn.cu) and the single-block MD
// kernel for small molecules (fused_md.cu); the mathematics and the design
// are described at the top of symfn.cu.
#pragma once

#include "engine.h"

namespace hdnnp {

namespace {


constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;

template <typename T>
struct Smem {
    T* dx;
    T* dy;
    T* dz;
    T* r;
    T* fc;
    T* dfc;
    T* gx;
    T* gy;
    T* gz;
    T* w;          // dE/dG_s / width_s of the centre (pass 2)
    int* ent;      // entry index of a slot
    unsigned char* el;
    unsigned* queue;   // 64 packed (j | k << 16)
    int* est;          // element start per slot range [kMaxEl+1]
    int* cur;          // cursors [kMaxEl]
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

template <typename T>
__host__ __device__ inline size_t warp_bytes(int mm, int nsf, bool grad) {
    size_t b = 0;
    b += align16(sizeof(T) * mm) * (grad ? 9 : 5);  // dx dy dz r fc [dfc gx gy gz]
    b += align16(sizeof(T) * (grad ? nsf : 0));
    b += align16(sizeof(int) * mm);
    b += align16(mm);
    b += 64 * sizeof(unsigned);
    b += align16(sizeof(int) * (kMaxEl + 1)) + align16(sizeof(int) * kMaxEl);
    return b;
}

template <typename T>
__device__ inline Smem<T> carve(unsigned char* p, int mm, int nsf, bool grad) {
    Smem<T> s;
    auto take = [&](size_t bytes) {
        unsigned char* q = p;
        p += align16(bytes);
        return q;
    };
    s.dx = (T*)take(sizeof(T) * mm);
    s.dy = (T*)take(sizeof(T) * mm);
    s.dz = (T*)take(sizeof(T) * mm);
    s.r = (T*)take(sizeof(T) * mm);
    s.fc = (T*)take(sizeof(T) * mm);
    if (grad) {
        s.dfc = (T*)take(sizeof(T) * mm);
        s.gx = (T*)take(sizeof(T) * mm);
        s.gy = (T*)take(sizeof(T) * mm);
        s.gz = (T*)take(sizeof(T) * mm);
        s.w = (T*)take(sizeof(T) * nsf);
    } else {
        s.dfc = s.gx = s.gy = s.gz = s.w = nullptr;
    }
    s.ent = (int*)take(sizeof(int) * mm);
    s.el = (unsigned char*)take(mm);
    s.queue = (unsigned*)take(64 * sizeof(unsigned));
    s.est = (int*)take(sizeof(int) * (kMaxEl + 1));
    s.cur = (int*)take(sizeof(int) * kMaxEl);
    return s;
}

// tanh^3 cutoff; dfc is (dfc/dr)/r as in the reference.
__device__ __forceinline__ void cutoff(double r, double rc, double& fc, double& dfc) {
    if (r < rc) {
        double t = tanh(1.0 - r / rc);
        double tt = t * t;
        fc = tt * t;
        dfc = -3.0 / (rc * r) * (tt - tt * tt);
    } else {
        fc = 0.0;
        dfc = 0.0;
    }
}

// x^n for integer n >= 0 by binary exponentiation
__device__ __forceinline__ double ipow(double x, int n) {
    double r = 1.0;
    while (n > 0) {
        if (n & 1) r *= x;
        x *= x;
        n >>= 1;
    }
    return r;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Stage the neighbour entries of atom i, sorted by element (stable).
// Returns the number of entries M.  Requires M <= mm.
template <bool kGrad>
__device__ int stage_neighbours(const Batch& b, const DevModel& m, int i, int c, Smem<double>& s, int lane) {
    const int e0 = b.nei_off[i];
    const int M = b.nei_off[i + 1] - e0;
    const int nel = m.nel;
    if (lane < nel) s.cur[lane] = 0;
    __syncwarp();
    // count per element
    for (int base = 0; base < M; base += 32) {
        int q = base + lane;
        int el = 255;
        if (q < M) el = b.elem[b.nei_j[e0 + q]];
        unsigned act = __ballot_sync(kFull, q < M);
        if (q < M) {
            unsigned peers = __match_any_sync(act, el);
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
    const double xi = b.wpos[3 * i], yi = b.wpos[3 * i + 1], zi = b.wpos[3 * i + 2];
    const StructInfo& S = b.info[b.sid[i]];
    const double rc = m.rc[c];
    for (int base = 0; base < M; base += 32) {
        int q = base + lane;
        unsigned act = __ballot_sync(kFull, q < M);
        int slot = 0, el = 255, j = 0, sh = 0;
        if (q < M) {
            j = b.nei_j[e0 + q];
            sh = b.nei_s[e0 + q];
            el = b.elem[j];
            unsigned peers = __match_any_sync(act, el);
            slot = s.cur[el] + __popc(peers & lanemask_lt());
            __syncwarp(act);
            if ((peers & lanemask_lt()) == 0) s.cur[el] += __popc(peers);
        }
        __syncwarp();
        if (q < M) {
            int sx, sy, sz;
            unpack_shift(sh, sx, sy, sz);
            double lx = 0, ly = 0, lz = 0;
            const double* h = S.h;
            if (sz) { lx += h[6] * sz; ly += h[7] * sz; lz += h[8] * sz; }
            if (sy) { lx += h[3] * sy; ly += h[4] * sy; lz += h[5] * sy; }
            if (sx) { lx += h[0] * sx; ly += h[1] * sx; lz += h[2] * sx; }
            double px = b.wpos[3 * j] + lx, py = b.wpos[3 * j + 1] + ly, pz = b.wpos[3 * j + 2] + lz;
            double dx = xi - px, dy = yi - py, dz = zi - pz;
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            double fc, dfc;
            cutoff(r, rc, fc, dfc);
            s.dx[slot] = dx;
            s.dy[slot] = dy;
            s.dz[slot] = dz;
            s.r[slot] = r;
            s.fc[slot] = fc;
            if (kGrad) {
                s.dfc[slot] = dfc;
                s.gx[slot] = 0;
                s.gy[slot] = 0;
                s.gz[slot] = 0;
            }
            s.el[slot] = (unsigned char)el;
            s.ent[slot] = e0 + q;
        }
    }
    __syncwarp();
    return M;
}

// (j,k) of candidate c inside the block (a,b); j, k are slots.
__device__ __forceinline__ void pair_of(int c, int sa, int na, int sb, int nb, bool same, int& j, int& k) {
    if (!same) {
        j = sa + c / nb;
        k = sb + c % nb;
    } else {
        // upper triangle of na x na, row-major: row j has na-1-j entries
        double t = (double)(2 * na - 1);
        int jj = (int)((t - sqrt(t * t - 8.0 * c)) * 0.5);
        if (jj < 0) jj = 0;
        auto off = [&](int x) { return x * (2 * na - x - 1) / 2; };
        while (jj > 0 && off(jj) > c) --jj;
        while (off(jj + 1) <= c) ++jj;
        j = sa + jj;
        k = sa + jj + 1 + (c - off(jj));
    }
}

// recursive-halving reduce-scatter of GM values over 32 lanes; afterwards the
// lane holds the warp sum of value index (lane >> (5 - log2 GM)).
template <int GM>
__device__ __forceinline__ double reduce_scatter(double (&v)[GM], int lane) {
    int cnt = GM;
    int off = 16;
#pragma unroll
    for (int step = 0; step < 5; ++step) {
        if (cnt > 1) {
            const int half = cnt >> 1;
            const bool up = (lane & off) != 0;
#pragma unroll
            for (int k = 0; k < GM / 2; ++k) {
                if (k < half) {
                    double send = up ? v[k] : v[k + half];
                    double keep = up ? v[k + half] : v[k];
                    v[k] = keep + __shfl_xor_sync(kFull, send, off);
                }
            }
            cnt = half;
        } else {
            v[0] += __shfl_xor_sync(kFull, v[0], off);
        }
        off >>= 1;
    }
    return v[0];
}

template <int GM>
struct Log2 {
    static constexpr int v = GM >= 32 ? 5 : GM >= 16 ? 4 : GM >= 8 ? 3 : GM >= 4 ? 2 : GM >= 2 ? 1 : 0;
};

// ---------------------------------------------------------------- pass 1
template <int GM>
__device__ __forceinline__ void sfv_atom(const Batch& b, const DevModel& m, int mm, Smem<double>& s, int i, int lane) {
    const int nel = m.nel;
    const int c = b.elem[i];
    if (c < 0) return;
    const int M = b.nei_off[i + 1] - b.nei_off[i];
    if (M > mm) {
        if (lane == 0) atomicOr(&b.status[0], 4);
        return;
    }
    stage_neighbours<false>(b, m, i, c, s, lane);
    const double mrc = m.rc[c], rc2 = mrc * mrc;
    double* Gi = b.G + (size_t)i * m.nsf_max;
    const double* mean = m.smean + (size_t)c * m.nsf_max;
    const double* width = m.swidth + (size_t)c * m.nsf_max;

    // radial: lane = SF
    const int r0 = m.g2_off[c * nel], r1 = m.g2_off[c * nel + nel];
    for (int f = r0 + lane; f < r1; f += 32) {
        const SF2 q = m.g2[f];
        double acc = 0.0;
        for (int t = s.est[q.nel]; t < s.est[q.nel + 1]; ++t) {
            double x = s.r[t] - q.rs;
            acc += exp(-q.eta * x * x) * s.fc[t];
        }
        Gi[q.sf] = (acc - mean[q.sf]) / width[q.sf];
    }

    unsigned long long n_cand = 0, n_pairs = 0, n_terms = 0;
    // angular: per element pair
    for (int t = 0; t < m.nblk; ++t) {
        const int gb = m.g4_off[c * m.nblk + t], ge = m.g4_off[c * m.nblk + t + 1];
        const int gcount = ge - gb;
        if (gcount == 0) continue;
        const int ea = m.blk_a[t], eb = m.blk_b[t];
        const int sa = s.est[ea], na = s.est[ea + 1] - sa;
        const int sb = s.est[eb], nb = s.est[eb + 1] - sb;
        const bool same = (ea == eb);
        const int ncand = same ? na * (na - 1) / 2 : na * nb;
        n_cand += ncand;
        for (int q0 = 0; q0 < gcount; q0 += GM) {
            double acc[GM];
#pragma unroll
            for (int u = 0; u < GM; ++u) acc[u] = 0.0;
            int qlen = 0;
            for (int cb = 0; cb < ncand; cb += 32) {
                const int cidx = cb + lane;
                bool ok = cidx < ncand;
                int j = 0, k = 0;
                if (ok) {
                    pair_of(cidx, sa, na, sb, nb, same, j, k);
                    double ex = s.dx[k] - s.dx[j], ey = s.dy[k] - s.dy[j], ez = s.dz[k] - s.dz[j];
                    ok = ex * ex + ey * ey + ez * ez < rc2;
                }
                const unsigned bal = __ballot_sync(kFull, ok);
                if (ok) s.queue[qlen + __popc(bal & lanemask_lt())] = (unsigned)j | ((unsigned)k << 16);
                qlen += __popc(bal);
                if (q0 == 0) {
                    n_pairs += __popc(bal);
                    n_terms += (unsigned long long)__popc(bal) * gcount;
                }
                __syncwarp();
                const bool last = cb + 32 >= ncand;
                while (qlen >= 32 || (last && qlen > 0)) {
                    const int n = qlen < 32 ? qlen : 32;
                    if (lane < n) {
                        const unsigned pk = s.queue[lane];
                        const int pj = pk & 0xffff, pk2 = pk >> 16;
                        const double ajx = s.dx[pj], ajy = s.dy[pj], ajz = s.dz[pj];
                        const double akx = s.dx[pk2], aky = s.dy[pk2], akz = s.dz[pk2];
                        const double rj = s.r[pj], rk = s.r[pk2];
                        const double cx = akx - ajx, cy = aky - ajy, cz = akz - ajz;
                        const double rjk2 = cx * cx + cy * cy + cz * cz;
                        const double rjk = sqrt(rjk2);
                        double fjk, dfjk;
                        cutoff(rjk, mrc, fjk, dfjk);
                        const double t1 = -1.0 / (rj * rk);
                        const double cth = 0.5 * (rjk * rjk - rj * rj - rk * rk) * t1;
                        const double fcp = s.fc[pj] * s.fc[pk2] * fjk;
                        const double rsum = rj * rj + rk * rk + rjk * rjk;
                        double last_eta = -1.0, ex = 0.0;
#pragma unroll
                        for (int u = 0; u < GM; ++u) {
                            if (q0 + u < gcount) {
                                const SF4 f = m.g4[gb + q0 + u];
                                if (f.eta != last_eta) {
                                    ex = exp(-f.eta * rsum);
                                    last_eta = f.eta;
                                }
                                const double base = 1.0 + f.lambda * cth;
                                const double t2 = f.izeta >= 0 ? ipow(base, f.izeta - 1) : pow(base, f.zeta - 1.0);
                                acc[u] += f.pf * (t2 * base) * ex * fcp;
                            }
                        }
                    }
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
            const double tot = reduce_scatter<GM>(acc, lane);
            const int idx = lane >> (5 - Log2<GM>::v);
            if ((lane & ((32 / GM) - 1)) == 0 && q0 + idx < gcount) {
                const int sf = m.g4[gb + q0 + idx].sf;
                Gi[sf] = (tot - mean[sf]) / width[sf];
            }
        }
    }
    if (b.stats && lane == 0) {
        unsigned long long n2 = 0;
        for (int f = r0; f < r1; ++f) {
            const SF2 q = m.g2[f];
            n2 += s.est[q.nel + 1] - s.est[q.nel];
        }
        atomicAdd(&b.stats[2], (unsigned long long)M);
        atomicAdd(&b.stats[3], n_cand);
        atomicAdd(&b.stats[4], n_pairs);
        atomicAdd(&b.stats[5], n_terms);
        atomicAdd(&b.stats[6], n2);
    }
    __syncwarp();
}

// ---------------------------------------------------------------- pass 2
__device__ __forceinline__ void sfg_atom(const Batch& b, const DevModel& m, int mm, Smem<double>& s, int i, int lane) {
    const int nel = m.nel;
    const int c = b.elem[i];
    if (c < 0) return;
    const int M = b.nei_off[i + 1] - b.nei_off[i];
    if (M > mm) {
        if (lane == 0) atomicOr(&b.status[0], 4);
        return;
    }
    stage_neighbours<true>(b, m, i, c, s, lane);
    const double mrc = m.rc[c], rc2 = mrc * mrc;
    const int nsf = m.nsf[c];
    for (int q = lane; q < nsf; q += 32)
        s.w[q] = b.dEdG[(size_t)i * m.nsf_max + q] / m.swidth[(size_t)c * m.nsf_max + q];
    __syncwarp();

    // radial: lane = neighbour slot
    for (int t = lane; t < M; t += 32) {
        const int el = s.el[t];
        const int f0 = m.g2_off[c * nel + el], f1 = m.g2_off[c * nel + el + 1];
        const double r = s.r[t], fc = s.fc[t], dfc = s.dfc[t];
        double coef = 0.0;
        for (int f = f0; f < f1; ++f) {
            const SF2 q = m.g2[f];
            const double x = r - q.rs;
            const double e = exp(-q.eta * x * x);
            coef += s.w[q.sf] * (-e * dfc + 2.0 * q.eta * x / r * e * fc);
        }
        s.gx[t] += coef * s.dx[t];
        s.gy[t] += coef * s.dy[t];
        s.gz[t] += coef * s.dz[t];
    }
    __syncwarp();

    for (int t = 0; t < m.nblk; ++t) {
        const int gb = m.g4_off[c * m.nblk + t], ge = m.g4_off[c * m.nblk + t + 1];
        if (ge == gb) continue;
        const int ea = m.blk_a[t], eb = m.blk_b[t];
        const int sa = s.est[ea], na = s.est[ea + 1] - sa;
        const int sb = s.est[eb], nb = s.est[eb + 1] - sb;
        const bool same = (ea == eb);
        const int ncand = same ? na * (na - 1) / 2 : na * nb;
        int qlen = 0;
        for (int cb = 0; cb < ncand; cb += 32) {
            const int cidx = cb + lane;
            bool ok = cidx < ncand;
            int j = 0, k = 0;
            if (ok) {
                pair_of(cidx, sa, na, sb, nb, same, j, k);
                double ex = s.dx[k] - s.dx[j], ey = s.dy[k] - s.dy[j], ez = s.dz[k] - s.dz[j];
                ok = ex * ex + ey * ey + ez * ez < rc2;
            }
            const unsigned bal = __ballot_sync(kFull, ok);
            if (ok) s.queue[qlen + __popc(bal & lanemask_lt())] = (unsigned)j | ((unsigned)k << 16);
            qlen += __popc(bal);
            __syncwarp();
            const bool last = cb + 32 >= ncand;
            while (qlen >= 32 || (last && qlen > 0)) {
                const int n = qlen < 32 ? qlen : 32;
                if (lane < n) {
                    const unsigned pk = s.queue[lane];
                    const int pj = pk & 0xffff, pk2 = pk >> 16;
                    const double ajx = s.dx[pj], ajy = s.dy[pj], ajz = s.dz[pj];
                    const double akx = s.dx[pk2], aky = s.dy[pk2], akz = s.dz[pk2];
                    const double rj = s.r[pj], rk = s.r[pk2];
                    const double fj = s.fc[pj], fk = s.fc[pk2], dfj = s.dfc[pj], dfk = s.dfc[pk2];
                    const double cx = akx - ajx, cy = aky - ajy, cz = akz - ajz;  // djk = r_j - r_k
                    const double rjk2 = cx * cx + cy * cy + cz * cz;
                    const double rjk = sqrt(rjk2);
                    double fjk, dfjk;
                    cutoff(rjk, mrc, fjk, dfjk);
                    const double t1 = -1.0 / (rj * rk);
                    const double cth = 0.5 * (rjk * rjk - rj * rj - rk * rk) * t1;
                    const double dot = ajx * akx + ajy * aky + ajz * akz;
                    const double cj = dot / (rj * rj * rj * rk), ck = dot / (rk * rk * rk * rj);
                    const double fcp = fj * fk * fjk;
                    const double rsum = rj * rj + rk * rk + rjk * rjk;
                    double A = 0.0, B = 0.0, C = 0.0;
                    double last_eta = -1.0, ex = 0.0;
                    for (int g = gb; g < ge; ++g) {
                        const SF4 f = m.g4[g];
                        if (f.eta != last_eta) {
                            ex = exp(-f.eta * rsum);
                            last_eta = f.eta;
                        }
                        const double base = 1.0 + f.lambda * cth;
                        const double t2 = f.izeta >= 0 ? ipow(base, f.izeta - 1) : pow(base, f.zeta - 1.0);
                        const double wpe = s.w[f.sf] * f.pf * ex;
                        const double cp = t2 * base;
                        A += wpe * cp;
                        B += wpe * cp * f.eta;
                        C += wpe * t2 * f.lambda * f.zeta;
                    }
                    // dfcpart, dexppart and dcos pieces of dsf (symmetryFunctions.f90:246-297)
                    const double B2 = 2.0 * B * fcp, Cf = C * fcp;
                    const double gjx = A * fk * (dfjk * cx * fj - dfj * ajx * fjk) + B2 * (ajx - cx) + Cf * (t1 * akx + ajx * cj);
                    const double gjy = A * fk * (dfjk * cy * fj - dfj * ajy * fjk) + B2 * (ajy - cy) + Cf * (t1 * aky + ajy * cj);
                    const double gjz = A * fk * (dfjk * cz * fj - dfj * ajz * fjk) + B2 * (ajz - cz) + Cf * (t1 * akz + ajz * cj);
                    const double gkx = -A * fj * (dfjk * cx * fk + dfk * akx * fjk) + B2 * (akx + cx) + Cf * (t1 * ajx + akx * ck);
                    const double gky = -A * fj * (dfjk * cy * fk + dfk * aky * fjk) + B2 * (aky + cy) + Cf * (t1 * ajy + aky * ck);
                    const double gkz = -A * fj * (dfjk * cz * fk + dfk * akz * fjk) + B2 * (akz + cz) + Cf * (t1 * ajz + akz * ck);
                    atomicAdd(&s.gx[pj], gjx);
                    atomicAdd(&s.gy[pj], gjy);
                    atomicAdd(&s.gz[pj], gjz);
                    atomicAdd(&s.gx[pk2], gkx);
                    atomicAdd(&s.gy[pk2], gky);
                    atomicAdd(&s.gz[pk2], gkz);
                }
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
    __syncwarp();
    // outputs: per entry gradient, centre term, atom virial
    double sx = 0, sy = 0, sz = 0;
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = lane; t < M; t += 32) {
        const double gx = s.gx[t], gy = s.gy[t], gz = s.gz[t];
        const int e = s.ent[t];
        b.gent[3 * (size_t)e] = gx;
        b.gent[3 * (size_t)e + 1] = gy;
        b.gent[3 * (size_t)e + 2] = gz;
        sx -= gx;
        sy -= gy;
        sz -= gz;
        const double dx = s.dx[t], dy = s.dy[t], dz = s.dz[t];
        // W[a][c] = -sum g[a] d[c]  (column-major v[a + 3c])
        v[0] -= gx * dx; v[1] -= gy * dx; v[2] -= gz * dx;
        v[3] -= gx * dy; v[4] -= gy * dy; v[5] -= gz * dy;
        v[6] -= gx * dz; v[7] -= gy * dz; v[8] -= gz * dz;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(kFull, sx, o);
        sy += __shfl_xor_sync(kFull, sy, o);
        sz += __shfl_xor_sync(kFull, sz, o);
#pragma unroll
        for (int u = 0; u < 9; ++u) v[u] += __shfl_xor_sync(kFull, v[u], o);
    }
    if (lane == 0) {
        b.gself[3 * (size_t)i] = sx;
        b.gself[3 * (size_t)i + 1] = sy;
        b.gself[3 * (size_t)i + 2] = sz;
#pragma unroll
        for (int u = 0; u < 9; ++u) b.vir[9 * (size_t)i + u] = v[u];
    }
    __syncwarp();
}

}  // namespace

}  // namespace hdnnp

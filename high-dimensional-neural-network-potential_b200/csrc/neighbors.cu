// neighbors.cu -- K1..K3: fractional wrap, cell lists and CSR neighbour lists.
//
// Semantics follow hdnnpCalcNeighborLists / buildNeighborListGrid
// (hdnnps.f90:373-388, neighborLists.f90:104-230): periodic atoms are wrapped
// with s = h^-1 r, s -= floor(s); the grid has int(|a_d| / (0.6 rc)) + 1 cells
// per lattice direction; every atom searches getNcells(grid, rc) cells each
// way in the order jx (outer), jy, jz (inner), wrapping z, then y, then x into
// the cell with an image shift; inside a cell atoms come in increasing index;
// an entry is kept when |d|^2 < rc^2 (strict) and it is not the atom itself
// without a shift.  Molecules use the artificial box and never wrap.
// The atom itself is not stored (the reference keeps it as entry 1); the
// symmetry-function kernels treat it implicitly.
//
// HBM-bound integer/FP64 work: one thread per atom (wrap, count, fill, force
// gather), one thread per entry (reverse index), one thread per cell (sort).
#include "engine.h"

namespace hdnnp {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void matvec(const double* a, double x, double y, double z, double& ox, double& oy,
                                       double& oz) {
    ox = a[0] * x + a[3] * y + a[6] * z;
    oy = a[1] * x + a[4] * y + a[7] * z;
    oz = a[2] * x + a[5] * y + a[8] * z;
}

__global__ void k_atom_struct(const StructInfo* info, int nstruct, int* sid) {
    int s = blockIdx.x;
    if (s >= nstruct) return;
    const int a0 = info[s].atom_off, n = info[s].nat;
    for (int i = threadIdx.x; i < n; i += blockDim.x) sid[a0 + i] = s;
}

// K1: wrap into the cell, element index, cell id, per-cell counts.
__global__ void k_wrap_bin(Batch b, DevModel m) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.natoms) return;
    const StructInfo& S = b.info[b.sid[i]];
    int z = b.Z[i];
    int e = (z >= 1 && z <= 118) ? m.z2e[z] : -1;
    b.elem[i] = e;
    if (e < 0) atomicOr(&b.status[0], 1);  // unknown element (validated on the host too)
    double x = b.pos[3 * i] - S.org[0], y = b.pos[3 * i + 1] - S.org[1], zz = b.pos[3 * i + 2] - S.org[2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(zz)) {  // device-resident input: flag, keep indices valid
        atomicOr(&b.status[0], 8);
        atomicMax(&b.status[2], b.sid[i] + 1);  // last structure with such an atom
        x = y = zz = 0.0;
    }
    double s0, s1, s2;
    matvec(S.hinv, x, y, zz, s0, s1, s2);
    s0 -= floor(s0);
    s1 -= floor(s1);
    s2 -= floor(s2);
    double wx, wy, wz;
    matvec(S.h, s0, s1, s2, wx, wy, wz);
    b.wpos[3 * i] = wx;
    b.wpos[3 * i + 1] = wy;
    b.wpos[3 * i + 2] = wz;
    // cell from the fractional coordinates of the wrapped position
    double f0, f1, f2;
    matvec(S.hinv, wx, wy, wz, f0, f1, f2);
    int c0 = min(max((int)(f0 * S.ngrid[0]), 0), S.ngrid[0] - 1);
    int c1 = min(max((int)(f1 * S.ngrid[1]), 0), S.ngrid[1] - 1);
    int c2 = min(max((int)(f2 * S.ngrid[2]), 0), S.ngrid[2] - 1);
    int cid = S.cell_off + (c0 * S.ngrid[1] + c1) * S.ngrid[2] + c2;
    b.cell_of[i] = cid;
    atomicAdd(&b.cell_cnt[cid], 1);
}

__global__ void k_fill_cells(Batch b, int* cursor) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.natoms) return;
    int c = b.cell_of[i];
    int p = atomicAdd(&cursor[c], 1);
    b.cell_atoms[b.cell_start[c] + p] = i;
}

// deterministic order inside a cell: increasing atom index
__global__ void k_sort_cells(Batch b) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= b.ncells) return;
    int s = b.cell_start[c], e = b.cell_start[c + 1];
    for (int p = s + 1; p < e; ++p) {
        int v = b.cell_atoms[p];
        int q = p - 1;
        while (q >= s && b.cell_atoms[q] > v) {
            b.cell_atoms[q + 1] = b.cell_atoms[q];
            --q;
        }
        b.cell_atoms[q + 1] = v;
    }
}

// K3 enumeration shared by the count and the fill pass.
template <bool kFill>
__global__ void k_neighbours(Batch b, DevModel m) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.natoms) return;
    const StructInfo& S = b.info[b.sid[i]];
    const double rc = m.max_rc, rc2 = rc * rc;
    const double xi = b.wpos[3 * i], yi = b.wpos[3 * i + 1], zi = b.wpos[3 * i + 2];
    const int c = b.cell_of[i] - S.cell_off;
    const int ix = c / (S.ngrid[1] * S.ngrid[2]);
    const int iy = (c / S.ngrid[2]) % S.ngrid[1];
    const int iz = c % S.ngrid[2];
    const double* h = S.h;
    int n = 0;
    int out = kFill ? b.nei_off[i] : 0;
    for (int jx = -S.nsearch[0]; jx <= S.nsearch[0]; ++jx) {
        for (int jy = -S.nsearch[1]; jy <= S.nsearch[1]; ++jy) {
            for (int jz = -S.nsearch[2]; jz <= S.nsearch[2]; ++jz) {
                int cx = ix + jx, cy = iy + jy, cz = iz + jz;
                int dx = 0, dy = 0, dz = 0;
                if (cz < 0 || cz >= S.ngrid[2]) {
                    if (!S.periodic) continue;
                    dz = (int)floor((double)cz / S.ngrid[2]);
                    cz -= S.ngrid[2] * dz;
                }
                if (cy < 0 || cy >= S.ngrid[1]) {
                    if (!S.periodic) continue;
                    dy = (int)floor((double)cy / S.ngrid[1]);
                    cy -= S.ngrid[1] * dy;
                }
                if (cx < 0 || cx >= S.ngrid[0]) {
                    if (!S.periodic) continue;
                    dx = (int)floor((double)cx / S.ngrid[0]);
                    cx -= S.ngrid[0] * dx;
                }
                // image shift, summed z, y, x like the reference
                double lx = 0, ly = 0, lz = 0;
                if (dz) { lx += h[6] * dz; ly += h[7] * dz; lz += h[8] * dz; }
                if (dy) { lx += h[3] * dy; ly += h[4] * dy; lz += h[5] * dy; }
                if (dx) { lx += h[0] * dx; ly += h[1] * dx; lz += h[2] * dx; }
                const bool home = (jx == 0 && jy == 0 && jz == 0);
                const int cell = S.cell_off + (cx * S.ngrid[1] + cy) * S.ngrid[2] + cz;
                const int p0 = b.cell_start[cell], p1 = b.cell_start[cell + 1];
                for (int p = p0; p < p1; ++p) {
                    const int j = b.cell_atoms[p];
                    if (j == i && home) continue;
                    double px = b.wpos[3 * j] + lx, py = b.wpos[3 * j + 1] + ly, pz = b.wpos[3 * j + 2] + lz;
                    double ddx = xi - px, ddy = yi - py, ddz = zi - pz;
                    if (ddx * ddx + ddy * ddy + ddz * ddz < rc2) {
                        if (kFill) {
                            b.nei_j[out] = j;
                            b.nei_s[out] = pack_shift(dx, dy, dz);
                            ++out;
                        } else {
                            ++n;
                        }
                    }
                }
            }
        }
    }
    if (!kFill) b.nei_cnt[i] = n;
}

// reverse entry: entry e = (a -> j, S) maps to the entry (j -> a, -S)
__global__ void k_reverse(Batch b) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= b.natoms) return;
    for (int e = b.nei_off[a]; e < b.nei_off[a + 1]; ++e) {
        const int j = b.nei_j[e];
        int sx, sy, sz;
        unpack_shift(b.nei_s[e], sx, sy, sz);
        const int want = pack_shift(-sx, -sy, -sz);
        int r = -1;
        for (int f = b.nei_off[j]; f < b.nei_off[j + 1]; ++f) {
            if (b.nei_j[f] == a && b.nei_s[f] == want) {
                r = f;
                break;
            }
        }
        if (r < 0) atomicOr(&b.status[0], 2);  // asymmetric list (should not happen)
        b.nei_rev[e] = r < 0 ? e : r;
    }
}

__global__ void k_max_count(const int* cnt, int n, int* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int v = i < n ? cnt[i] : 0;
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, v);
}

// ---------------------------------------------------------------- scan
// Exclusive scan of n ints in place (data[n] receives the total).  Two-level:
// per-block scan of 1024 values, scan of block sums (recursive), add.
__global__ void k_scan_block(int* d, int n, int* sums) {
    __shared__ int wsum[32];
    int base = blockIdx.x * 1024;
    int t = threadIdx.x;  // 1024 threads
    int i = base + t;
    int v = i < n ? d[i] : 0;
    int lane = t & 31, w = t >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    int incl = x + (w > 0 ? wsum[w - 1] : 0);
    if (i < n) d[i] = incl - v;
    if (t == 1023) sums[blockIdx.x] = incl;
}

__global__ void k_scan_add(int* d, int n, const int* sums) {
    int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n && blockIdx.x > 0) d[i] += sums[blockIdx.x];
}

}  // namespace

int launch_scan(int* data, int n, int* tmp, int* total_unused, cudaStream_t s) {
    (void)total_unused;
    int launches = 0;
    int nb = (n + 1023) / 1024;
    if (nb <= 0) nb = 1;
    // tmp must hold nb + 1 ints, plus space for the recursion
    k_scan_block<<<nb, 1024, 0, s>>>(data, n, tmp);
    ++launches;
    if (nb > 1) {
        launches += launch_scan(tmp, nb, tmp + nb + 1, nullptr, s);  // tmp[nb] = grand total
        k_scan_add<<<nb, 1024, 0, s>>>(data, n, tmp);
        ++launches;
        // data[n] = total
        cudaMemcpyAsync(data + n, tmp + nb, sizeof(int), cudaMemcpyDeviceToDevice, s);
    } else {
        cudaMemcpyAsync(data + n, tmp, sizeof(int), cudaMemcpyDeviceToDevice, s);
    }
    return launches;
}

int launch_neighbour_build_a(const Batch& b, const DevModel& m, cudaStream_t s) {
    int L = 0;
    const int gA = (b.natoms + kThreads - 1) / kThreads;
    k_atom_struct<<<b.nstruct, 128, 0, s>>>(b.info, b.nstruct, b.sid);
    ++L;
    cudaMemsetAsync(b.cell_cnt, 0, sizeof(int) * (b.ncells + 1), s);
    k_wrap_bin<<<gA, kThreads, 0, s>>>(b, m);
    ++L;
    cudaMemcpyAsync(b.cell_start, b.cell_cnt, sizeof(int) * (b.ncells + 1), cudaMemcpyDeviceToDevice, s);
    L += launch_scan(b.cell_start, b.ncells, b.scan_tmp, nullptr, s);
    cudaMemsetAsync(b.cell_cnt, 0, sizeof(int) * (b.ncells + 1), s);
    k_fill_cells<<<gA, kThreads, 0, s>>>(b, b.cell_cnt);
    ++L;
    k_sort_cells<<<(b.ncells + kThreads - 1) / kThreads, kThreads, 0, s>>>(b);
    ++L;
    k_neighbours<false><<<gA, kThreads, 0, s>>>(b, m);
    ++L;
    cudaMemcpyAsync(b.nei_off, b.nei_cnt, sizeof(int) * b.natoms, cudaMemcpyDeviceToDevice, s);
    L += launch_scan(b.nei_off, b.natoms, b.scan_tmp, nullptr, s);
    // status[1] = max count
    cudaMemsetAsync(b.status + 1, 0, sizeof(int), s);
    k_max_count<<<gA, kThreads, 0, s>>>(b.nei_cnt, b.natoms, b.status + 1);
    ++L;
    return L;
}

int launch_neighbour_build_b(const Batch& b, const DevModel& m, cudaStream_t s) {
    const int gA = (b.natoms + kThreads - 1) / kThreads;
    k_neighbours<true><<<gA, kThreads, 0, s>>>(b, m);
    k_reverse<<<gA, kThreads, 0, s>>>(b);
    return 2;
}

}  // namespace hdnnp

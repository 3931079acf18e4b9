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
// HBM-bound integer/FP64 work: a thread per atom (wrap), a thread or a warp
// per atom (count, fill), one or more warps per atom (reverse index), a warp
// per cell (sort) and per atom (skin-list compaction).
#include <algorithm>
#include <cmath>

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

// Verlet-skin reuse: the list of the last build stays valid this evaluation.
__device__ __forceinline__ bool keep_list(const Batch& b) { return b.rebuild && !*b.rebuild; }

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
    if (keep_list(b)) {
        // same translation as at the last build: distances to the listed images stay consistent
        for (int d = 0; d < 3; ++d) {
            const double x = b.pos[3 * i + d];
            if (!isfinite(x)) {
                atomicOr(&b.status[0], 8);
                atomicMax(&b.status[2], b.sid[i] + 1);
            }
            b.wpos[3 * i + d] = isfinite(x) ? x + b.wshift[3 * i + d] : b.pos_ref[3 * i + d] + b.wshift[3 * i + d];
        }
        return;
    }
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
    if (b.wshift) {
        b.wshift[3 * i] = wx - b.pos[3 * i];
        b.wshift[3 * i + 1] = wy - b.pos[3 * i + 1];
        b.wshift[3 * i + 2] = wz - b.pos[3 * i + 2];
        b.pos_ref[3 * i] = b.pos[3 * i];
        b.pos_ref[3 * i + 1] = b.pos[3 * i + 1];
        b.pos_ref[3 * i + 2] = b.pos[3 * i + 2];
    }
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
    if (i >= b.natoms || keep_list(b)) return;
    int c = b.cell_of[i];
    int p = atomicAdd(&cursor[c], 1);
    b.cell_atoms[b.cell_start[c] + p] = i;
}

// Deterministic order inside a cell: increasing atom index.  One warp per
// cell: the cell's atoms are copied to shared memory and each goes to its
// rank (the number of smaller indices; indices are distinct).  Cells above
// kSortCap atoms are sorted by one lane in place (insertion sort).
constexpr int kSortCap = 256;
constexpr int kSortWarps = kThreads / 32;
__global__ void k_sort_cells(Batch b) {
    __shared__ int buf[kSortWarps][kSortCap];
    const int c = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (c >= b.ncells || keep_list(b)) return;  // uniform per warp
    const int s = b.cell_start[c], e = b.cell_start[c + 1], n = e - s;
    if (n <= 1) return;
    if (n > kSortCap) {
        if (lane == 0)
            for (int p = s + 1; p < e; ++p) {
                const int v = b.cell_atoms[p];
                int q = p - 1;
                while (q >= s && b.cell_atoms[q] > v) {
                    b.cell_atoms[q + 1] = b.cell_atoms[q];
                    --q;
                }
                b.cell_atoms[q + 1] = v;
            }
        return;
    }
    int* t = buf[w];
    for (int p = lane; p < n; p += 32) t[p] = b.cell_atoms[s + p];
    __syncwarp();
    for (int p = lane; p < n; p += 32) {
        const int v = t[p];
        int r = 0;
        for (int q = 0; q < n; ++q) r += t[q] < v;
        b.cell_atoms[s + r] = v;
    }
}

// Cell-ordered copy of the wrapped positions: the neighbour search reads one
// 32-byte record per candidate instead of an index and then the position.
__global__ void k_cell_positions(Batch b) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= b.natoms || keep_list(b)) return;
    const int j = b.cell_atoms[p];
    b.posc[p] = make_double4(b.wpos[3 * j], b.wpos[3 * j + 1], b.wpos[3 * j + 2], __longlong_as_double((long long)j));
}

// Candidate p of the cell lists: atom index and wrapped position.
__device__ __forceinline__ int cand(const Batch& b, int p, double& x, double& y, double& z) {
    if (b.posc) {
        const double4 q = b.posc[p];
        x = q.x;
        y = q.y;
        z = q.z;
        return (int)__double_as_longlong(q.w);
    }
    const int j = b.cell_atoms[p];
    x = b.wpos[3 * j];
    y = b.wpos[3 * j + 1];
    z = b.wpos[3 * j + 2];
    return j;
}

// floor(a / n) for n > 0, in integers (the same value as the floating-point
// floor of the exact quotient)
__device__ __forceinline__ int floor_div(int a, int n) { return a >= 0 ? a / n : -((n - 1 - a) / n); }

// Wrap a cell coordinate c into [0, n) and return the image count floor(c / n):
// the search offsets reach at most nsearch cells beyond the grid, so this is
// one step for grids of at least nsearch cells and a few for tiny cells --
// the same result as floor_div without an integer division.
__device__ __forceinline__ int wrap_cell(int& c, int n) {
    int d = 0;
    while (c < 0) {
        c += n;
        --d;
    }
    while (c >= n) {
        c -= n;
        ++d;
    }
    return d;
}

// K3 enumeration shared by the passes.  kMode 0: count; 1: fill the CSR
// lists at nei_off; 2 (plans): count and fill the atom's padded row of
// pad_cap entries in one pass (entries beyond pad_cap are counted only; the
// capacity check then empties the lists), copied into the CSR arrays by
// k_rows_to_lists after the scan.
template <int kMode>
__global__ void k_neighbours(Batch b, DevModel m) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.natoms || keep_list(b)) return;
    if (kMode == 1 && b.status[3]) return;  // planned capacity exceeded: the lists stay empty
    const StructInfo& S = b.info[b.sid[i]];
    const double rc = b.rc_list > 0.0 ? b.rc_list : m.max_rc, rc2 = rc * rc;
    const double xi = b.wpos[3 * i], yi = b.wpos[3 * i + 1], zi = b.wpos[3 * i + 2];
    const int c = b.cell_of[i] - S.cell_off;
    const int ix = c / (S.ngrid[1] * S.ngrid[2]);
    const int iy = (c / S.ngrid[2]) % S.ngrid[1];
    const int iz = c % S.ngrid[2];
    const double* h = S.h;
    int n = 0;
    int out = kMode == 1 ? b.nei_off[i] : 0;
    int2* row = kMode == 2 ? b.pad + (size_t)i * b.pad_cap : nullptr;
    // slab prefixes of the padded row (see Batch::slab)
    const int nslab = (2 * S.nsearch[0] + 1) * (2 * S.nsearch[1] + 1);
    unsigned short* tab = (kMode == 2 && b.slab && nslab <= kMaxSlabs) ? b.slab + (size_t)i * kSlabStride : nullptr;
    int slab = 0;
    for (int jx = -S.nsearch[0]; jx <= S.nsearch[0]; ++jx) {
        // x and y of the virtual cell are wrapped once per column, z per cell
        int cx = ix + jx;
        const bool xin = cx >= 0 && cx < S.ngrid[0];
        const int dx = xin ? 0 : wrap_cell(cx, S.ngrid[0]);
        for (int jy = -S.nsearch[1]; jy <= S.nsearch[1]; ++jy, ++slab) {
            if (tab) tab[slab] = (unsigned short)min(n, 0xffff);
            int cy = iy + jy;
            const bool yin = cy >= 0 && cy < S.ngrid[1];
            const int dy = yin ? 0 : wrap_cell(cy, S.ngrid[1]);
            if (!S.periodic && !(xin && yin)) continue;  // a molecule: no cells beyond its grid
            for (int jz = -S.nsearch[2]; jz <= S.nsearch[2]; ++jz) {
                int cz = iz + jz;
                int dz = 0;
                if (cz < 0 || cz >= S.ngrid[2]) {
                    if (!S.periodic) continue;
                    dz = wrap_cell(cz, S.ngrid[2]);
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
                    double px, py, pz;
                    const int j = cand(b, p, px, py, pz);
                    if (j == i && home) continue;
                    px += lx;
                    py += ly;
                    pz += lz;
                    double ddx = xi - px, ddy = yi - py, ddz = zi - pz;
                    if (ddx * ddx + ddy * ddy + ddz * ddz < rc2) {
                        if (kMode == 1) {
                            b.nei_j[out] = j;
                            b.nei_s[out] = pack_shift(dx, dy, dz);
                            ++out;
                        } else {
                            if (kMode == 2 && n < b.pad_cap)
                                row[n] = make_int2(j, pack_shift(dx, dy, dz) | (tab ? slab << 24 : 0));
                            ++n;
                        }
                    }
                }
            }
        }
    }
    if (tab) tab[nslab] = (unsigned short)min(n, 0xffff);
    if (kMode != 1) b.nei_cnt[i] = n;
}

// The same enumeration with one warp per atom: the virtual cells, in the
// reference's order (jx outer, jz inner), are dealt to the lanes 32 at a time;
// each lane walks its cell's atoms in cell order, and the fill pass places a
// round's accepted atoms by an ordered prefix sum over the lanes -- so the
// list is the same, entry for entry.  For batches too small to fill the GPU
// with a thread per atom (a single cell of a few hundred atoms has thousands
// of candidates per atom, walked serially by one thread).
template <int kMode>
__global__ void k_neighbours_warp(Batch b, DevModel m) {
    const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= b.natoms || keep_list(b)) return;  // uniform per warp
    if (kMode == 1 && b.status[3]) return;
    const StructInfo& S = b.info[b.sid[i]];
    const double rc = b.rc_list > 0.0 ? b.rc_list : m.max_rc, rc2 = rc * rc;
    const double xi = b.wpos[3 * i], yi = b.wpos[3 * i + 1], zi = b.wpos[3 * i + 2];
    const int c = b.cell_of[i] - S.cell_off;
    const int ix = c / (S.ngrid[1] * S.ngrid[2]);
    const int iy = (c / S.ngrid[2]) % S.ngrid[1];
    const int iz = c % S.ngrid[2];
    const double* h = S.h;
    const int ny = 2 * S.nsearch[1] + 1, nz = 2 * S.nsearch[2] + 1;
    const int nv = (2 * S.nsearch[0] + 1) * ny * nz;
    int n = 0;
    int out = kMode == 1 ? b.nei_off[i] : 0;
    int2* row = kMode == 2 ? b.pad + (size_t)i * b.pad_cap : nullptr;
    // slab prefixes of the padded row (see Batch::slab): slab = v / nz
    const int nslab = (2 * S.nsearch[0] + 1) * ny;
    unsigned short* tab = (kMode == 2 && b.slab && nslab <= kMaxSlabs) ? b.slab + (size_t)i * kSlabStride : nullptr;
    for (int v0 = 0; v0 < nv; v0 += 32) {
        const int v = v0 + lane;
        int p0 = 0, p1 = 0, dx = 0, dy = 0, dz = 0;
        double lx = 0, ly = 0, lz = 0;
        bool home = false;
        if (v < nv) {
            const int jx = v / (ny * nz) - S.nsearch[0];
            const int jy = (v / nz) % ny - S.nsearch[1];
            const int jz = v % nz - S.nsearch[2];
            int cx = ix + jx, cy = iy + jy, cz = iz + jz;
            bool inside = true;
            if (cz < 0 || cz >= S.ngrid[2]) {
                inside = S.periodic;
                dz = wrap_cell(cz, S.ngrid[2]);
            }
            if (cy < 0 || cy >= S.ngrid[1]) {
                inside = inside && S.periodic;
                dy = wrap_cell(cy, S.ngrid[1]);
            }
            if (cx < 0 || cx >= S.ngrid[0]) {
                inside = inside && S.periodic;
                dx = wrap_cell(cx, S.ngrid[0]);
            }
            if (inside) {
                if (dz) { lx += h[6] * dz; ly += h[7] * dz; lz += h[8] * dz; }
                if (dy) { lx += h[3] * dy; ly += h[4] * dy; lz += h[5] * dy; }
                if (dx) { lx += h[0] * dx; ly += h[1] * dx; lz += h[2] * dx; }
                home = (jx == 0 && jy == 0 && jz == 0);
                const int cell = S.cell_off + (cx * S.ngrid[1] + cy) * S.ngrid[2] + cz;
                p0 = b.cell_start[cell];
                p1 = b.cell_start[cell + 1];
            }
        }
        // this lane's accepted atoms of its virtual cell
        int cnt = 0;
        for (int p = p0; p < p1; ++p) {
            double px, py, pz;
            const int j = cand(b, p, px, py, pz);
            if (j == i && home) continue;
            px += lx;
            py += ly;
            pz += lz;
            double ddx = xi - px, ddy = yi - py, ddz = zi - pz;
            cnt += ddx * ddx + ddy * ddy + ddz * ddz < rc2;
        }
        int incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        if (tab && v < nv && v % nz == 0) tab[v / nz] = (unsigned short)min(n + incl - cnt, 0xffff);
        if (kMode != 0 && cnt > 0) {
            int o = (kMode == 1 ? out : n) + incl - cnt;
            const int sh = pack_shift(dx, dy, dz) | (tab ? (v / nz) << 24 : 0);
            for (int p = p0; p < p1; ++p) {
                double px, py, pz;
                const int j = cand(b, p, px, py, pz);
                if (j == i && home) continue;
                px += lx;
                py += ly;
                pz += lz;
                double ddx = xi - px, ddy = yi - py, ddz = zi - pz;
                if (ddx * ddx + ddy * ddy + ddz * ddz < rc2) {
                    if (kMode == 1) {
                        b.nei_j[o] = j;
                        b.nei_s[o] = sh;
                    } else if (o < b.pad_cap) {
                        row[o] = make_int2(j, sh);
                    }
                    ++o;
                }
            }
        }
        out += total;
        n += total;
    }
    if (tab && lane == 0) tab[nslab] = (unsigned short)min(n, 0xffff);
    if (kMode != 1 && lane == 0) b.nei_cnt[i] = n;
}

// Padded rows -> CSR lists (plans, eager calls after the first), one warp
// per atom, lanes over its entries; with the slab table it also writes the
// reverse index: the entry (j -> i, -S) of (i -> j, S) found in slab s lies
// in slab K - 1 - s of j's row (the mirrored (jx, jy) column, because j's
// search offsets mirror i's), a scan of a few entries.  Without the table
// (more than kMaxSlabs columns) the whole row of j is scanned.  After an
// overflow the capacity check has emptied the lists (nei_off all 0), so
// nothing is copied.
__global__ void k_rows_to_lists(Batch b) {
    const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= b.natoms || keep_list(b)) return;  // uniform per warp
    const int e0 = b.nei_off[i], n = min(b.nei_off[i + 1] - e0, b.pad_cap);
    const int2* row = b.pad + (size_t)i * b.pad_cap;
    int nslab = 0;
    if (b.slab) {
        const StructInfo& S = b.info[b.sid[i]];
        nslab = (2 * S.nsearch[0] + 1) * (2 * S.nsearch[1] + 1);
        if (nslab > kMaxSlabs) nslab = 0;
    }
    for (int q = lane; q < n; q += 32) {
        const int2 v = row[q];
        const int j = v.x, sh = v.y & 0xffffff;
        b.nei_j[e0 + q] = j;
        b.nei_s[e0 + q] = sh;
        if (!b.slab) continue;
        int sx, sy, sz;
        unpack_shift(sh, sx, sy, sz);
        const int want = pack_shift(-sx, -sy, -sz);
        const int2* rj = b.pad + (size_t)j * b.pad_cap;
        const int nj = min(b.nei_off[j + 1] - b.nei_off[j], b.pad_cap);
        int lo = 0, hi = nj;
        if (nslab) {
            const int m = nslab - 1 - (int)((unsigned)v.y >> 24);
            const unsigned short* tj = b.slab + (size_t)j * kSlabStride;
            lo = min((int)tj[m], nj);
            hi = min((int)tj[m + 1], nj);
        }
        int r = -1;
        for (int p = lo; p < hi && r < 0; ++p) {
            const int2 u = rj[p];
            if (u.x == i && (u.y & 0xffffff) == want) r = p;
        }
        for (int p = 0; p < nj && r < 0; ++p) {  // not in its slab (should not happen): the whole row
            const int2 u = rj[p];
            if (u.x == i && (u.y & 0xffffff) == want) r = p;
        }
        if (r < 0) atomicOr(&b.status[0], 2);  // asymmetric list (should not happen)
        b.nei_rev[e0 + q] = r < 0 ? e0 + q : b.nei_off[j] + r;
    }
}

// Batches below this many atoms list neighbours with a warp per atom
// (measured on B200, count + fill: the 768-atom cell 0.14 against 0.47 ms, the
// 49,152-atom cell 0.60 against 0.73 ms; the 758,676-atom batch of 4096 cells
// 7.4 against 6.2 ms, where threads already fill the GPU).
constexpr int kWarpListAtoms = 131072;
inline bool warp_lists(const Batch& b) {
    return b.nei_warp > 0 || (b.nei_warp == 0 && b.natoms < kWarpListAtoms);
}

// Reverse-entry index: for entry e = (a -> j, shift s) the entry (j -> a, -s)
// of j's list.  `parts` warps per atom a, each taking every parts-th group
// of four entries; one search per group of 8 lanes, which scan j's list in
// coalesced 8-entry chunks, the ballot picking the first match.  Small
// batches use several warps per atom so that enough searches are in flight.
// kPad: the lists' padded rows are still in place (plans, eager calls after
// the first): the search reads (j, shift) pairs as one 8-byte load from j's
// row instead of two arrays; indices stay those of the CSR lists.
template <bool kMulti, bool kPad>
__global__ void k_reverse(Batch b, int parts) {
    const long long w = (long long)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    if (!kMulti) parts = 1;
    const int a = kMulti ? (int)(w / parts) : (int)w, part = kMulti ? (int)(w % parts) : 0;
    const int lane = threadIdx.x & 31;
    if (a >= b.natoms || keep_list(b)) return;  // uniform per warp
    // four entries of atom a at a time, one per group of 8 lanes, so that the
    // dependent loads of four searches overlap
    const int grp = lane >> 3, gl = lane & 7;
    const int ea = b.nei_off[a], e1 = b.nei_off[a + 1];
    for (int e0 = ea + 4 * part; e0 < e1; e0 += 4 * parts) {
        const int e = e0 + grp;
        const bool live = e < e1;
        int want = 0, f0 = 0, f1 = 0;
        const int2* row = nullptr;
        if (live) {
            int j, sh;
            if (kPad) {
                const int2 v = b.pad[(size_t)a * b.pad_cap + (e - ea)];
                j = v.x;
                sh = v.y & 0xffffff;
            } else {
                j = b.nei_j[e];
                sh = b.nei_s[e];
            }
            int sx, sy, sz;
            unpack_shift(sh, sx, sy, sz);
            want = pack_shift(-sx, -sy, -sz);
            f0 = b.nei_off[j];
            f1 = b.nei_off[j + 1];
            if (kPad) row = b.pad + (size_t)j * b.pad_cap;
        }
        int r = -1;
        // every iteration advances each open search by 8 entries of its list,
        // so the loop ends after (longest list) / 8 iterations
        for (int fb = 0;; fb += 8) {
            const int f = f0 + fb + gl;
            const bool open = live && r < 0 && f0 + fb < f1;
            bool hit = false;
            if (open && f < f1) {
                if (kPad) {
                    const int2 v = row[fb + gl];
                    hit = v.x == a && (v.y & 0xffffff) == want;
                } else {
                    hit = b.nei_j[f] == a && b.nei_s[f] == want;
                }
            }
            const unsigned gm = (__ballot_sync(0xffffffffu, hit) >> (8 * grp)) & 0xffu;
            if (open && gm) r = f0 + fb + __ffs(gm) - 1;
            if (!__any_sync(0xffffffffu, live && r < 0 && f0 + fb + 8 < f1)) break;
        }
        if (live && gl == 0) {
            if (r < 0) atomicOr(&b.status[0], 2);  // asymmetric list (should not happen)
            b.nei_rev[e] = r < 0 ? e : r;
        }
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
// src may equal d (in place); a single block also writes the total to d[n].
__global__ void k_scan_block(const int* src, int* d, int n, int* sums) {
    __shared__ int wsum[32];
    int base = blockIdx.x * 1024;
    int t = threadIdx.x;  // 1024 threads
    int i = base + t;
    int v = i < n ? src[i] : 0;
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
    if (t == 1023) {
        sums[blockIdx.x] = incl;
        if (gridDim.x == 1) d[n] = incl;
    }
}

// sums[gridDim.x] holds the grand total (the recursive scan of the block sums)
__global__ void k_scan_add(int* d, int n, const int* sums) {
    int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n && blockIdx.x > 0) d[i] += sums[blockIdx.x];
    if (blockIdx.x == 0 && threadIdx.x == 0) d[n] = sums[gridDim.x];
}

}  // namespace

int launch_scan_from(const int* src, int* data, int n, int* tmp, cudaStream_t s) {
    int launches = 0;
    int nb = (n + 1023) / 1024;
    if (nb <= 0) nb = 1;
    // tmp must hold nb + 1 ints, plus space for the recursion
    k_scan_block<<<nb, 1024, 0, s>>>(src, data, n, tmp);
    ++launches;
    if (nb > 1) {
        launches += launch_scan(tmp, nb, tmp + nb + 1, nullptr, s);  // tmp[nb] = grand total
        k_scan_add<<<nb, 1024, 0, s>>>(data, n, tmp);                // also data[n] = total
        ++launches;
    }
    return launches;
}

int launch_scan(int* data, int n, int* tmp, int* total_unused, cudaStream_t s) {
    (void)total_unused;
    return launch_scan_from(data, data, n, tmp, s);
}

int launch_neighbour_build_a(const Batch& b, const DevModel& m, cudaStream_t s, bool sid_valid) {
    int L = 0;
    const int gA = (b.natoms + kThreads - 1) / kThreads;
    if (!sid_valid) {
        k_atom_struct<<<b.nstruct, 128, 0, s>>>(b.info, b.nstruct, b.sid);
        ++L;
    }
    cudaMemsetAsync(b.cell_cnt, 0, sizeof(int) * (b.ncells + 1), s);
    k_wrap_bin<<<gA, kThreads, 0, s>>>(b, m);
    ++L;
    L += launch_scan_from(b.cell_cnt, b.cell_start, b.ncells, b.scan_tmp, s);
    cudaMemsetAsync(b.cell_cnt, 0, sizeof(int) * (b.ncells + 1), s);
    k_fill_cells<<<gA, kThreads, 0, s>>>(b, b.cell_cnt);
    ++L;
    k_sort_cells<<<(unsigned)((32LL * b.ncells + kThreads - 1) / kThreads), kThreads, 0, s>>>(b);
    ++L;
    if (b.posc) {
        k_cell_positions<<<gA, kThreads, 0, s>>>(b);
        ++L;
    }
    const unsigned gW = (unsigned)((32LL * b.natoms + kThreads - 1) / kThreads);
    if (b.pad_cap > 0) {  // plans: one search pass into padded rows
        if (warp_lists(b))
            k_neighbours_warp<2><<<gW, kThreads, 0, s>>>(b, m);
        else
            k_neighbours<2><<<gA, kThreads, 0, s>>>(b, m);
    } else if (warp_lists(b)) {
        k_neighbours_warp<0><<<gW, kThreads, 0, s>>>(b, m);
    } else {
        k_neighbours<0><<<gA, kThreads, 0, s>>>(b, m);
    }
    ++L;
    L += launch_scan_from(b.nei_cnt, b.nei_off, b.natoms, b.scan_tmp, s);
    // status[1] = max count
    cudaMemsetAsync(b.status + 1, 0, sizeof(int), s);
    k_max_count<<<gA, kThreads, 0, s>>>(b.nei_cnt, b.natoms, b.status + 1);
    ++L;
    return L;
}

int launch_neighbour_build_b(const Batch& b, const DevModel& m, cudaStream_t s) {
    const int gA = (b.natoms + kThreads - 1) / kThreads;
    const long long warps_threads = 32LL * b.natoms;
    if (b.pad_cap > 0 && b.slab) {
        // copy and reverse index in one pass
        k_rows_to_lists<<<(unsigned)((warps_threads + kThreads - 1) / kThreads), kThreads, 0, s>>>(b);
        return 1;
    }
    if (b.pad_cap > 0)
        k_rows_to_lists<<<(unsigned)((warps_threads + kThreads - 1) / kThreads), kThreads, 0, s>>>(b);
    else if (warp_lists(b))
        k_neighbours_warp<1><<<(unsigned)((warps_threads + kThreads - 1) / kThreads), kThreads, 0, s>>>(b, m);
    else
        k_neighbours<1><<<gA, kThreads, 0, s>>>(b, m);
    // warps per atom: up to 8, until ~64 warps per SM of a B200 are in flight
    const int parts = (int)std::min<long long>(8, std::max<long long>(1, (148LL * 64 + b.natoms - 1) / std::max(b.natoms, 1)));
    const unsigned gR = (unsigned)((warps_threads * parts + kThreads - 1) / kThreads);
    if (b.pad_cap > 0) {
        if (parts > 1)
            k_reverse<true, true><<<gR, kThreads, 0, s>>>(b, parts);
        else
            k_reverse<false, true><<<gR, kThreads, 0, s>>>(b, 1);
    } else if (parts > 1) {
        k_reverse<true, false><<<gR, kThreads, 0, s>>>(b, parts);
    } else {
        k_reverse<false, false><<<gR, kThreads, 0, s>>>(b, 1);
    }
    return 2;
}

// ---------------------------------------------------------------- skin lists
// A Verlet-skin list (cutoff max_rc + skin) holds about (1 + skin/rc)^3 times
// the entries that contribute.  Every evaluation copies the entries closer
// than max_rc into a second CSR list, in list order, and remaps the reverse
// index onto it; the symmetry-function and force stages then read only that
// list.  The test computes d = (x_a - x_j) - L(S) in FP64 with every step
// negated exactly for the reverse entry (x_j - x_a) - L(-S) (round to nearest
// is symmetric), so an entry and its reverse are kept or dropped together.
namespace {

__device__ __forceinline__ bool entry_inside(const Batch& b, const StructInfo& S, double xa, double ya, double za,
                                             int j, int sh, double rc2) {
    int sx, sy, sz;
    unpack_shift(sh, sx, sy, sz);
    const double* h = S.h;
    double lx = 0, ly = 0, lz = 0;
    if (sz) { lx += h[6] * sz; ly += h[7] * sz; lz += h[8] * sz; }
    if (sy) { lx += h[3] * sy; ly += h[4] * sy; lz += h[5] * sy; }
    if (sx) { lx += h[0] * sx; ly += h[1] * sx; lz += h[2] * sx; }
    const double dx = (xa - b.wpos[3 * j]) - lx, dy = (ya - b.wpos[3 * j + 1]) - ly, dz = (za - b.wpos[3 * j + 2]) - lz;
    return dx * dx + dy * dy + dz * dz < rc2;
}

// One warp per atom: kFill = false counts the kept entries (ccnt, and coff
// for the scan); kFill = true writes them at coff and maps every entry of
// the full list to its compacted index (-1: dropped).
template <bool kFill>
__global__ void k_compact(Batch b, double rc2, int* ccnt, int* coff, int* cj, int* cs, int* cmap) {
    const int a = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (a >= b.natoms) return;  // uniform per warp
    const int e0 = b.nei_off[a], e1 = b.nei_off[a + 1];
    const StructInfo& S = b.info[b.sid[a]];
    const double xa = b.wpos[3 * a], ya = b.wpos[3 * a + 1], za = b.wpos[3 * a + 2];
    int n = kFill ? coff[a] : 0;
    for (int base = e0; base < e1; base += 32) {
        const int e = base + lane;
        int j = 0, sh = 0;
        bool in = false;
        if (e < e1) {
            j = b.nei_j[e];
            sh = b.nei_s[e];
            in = entry_inside(b, S, xa, ya, za, j, sh, rc2);
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (kFill && e < e1) {
            const int o = n + __popc(m & ((1u << lane) - 1u));
            if (in) {
                cj[o] = j;
                cs[o] = sh;
            }
            cmap[e] = in ? o : -1;
        }
        n += __popc(m);
    }
    if (!kFill && lane == 0) {
        ccnt[a] = n;
        coff[a] = n;
    }
}

// Reverse index of the compacted list, one thread per entry of the full list.
__global__ void k_compact_rev(Batch b, const int* cmap, int* crev) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= b.nei_off[b.natoms]) return;
    const int o = cmap[e];
    if (o < 0) return;
    const int r = cmap[b.nei_rev[e]];
    if (r < 0) atomicOr(&b.status[0], 2);  // asymmetric list (should not happen)
    crev[o] = r < 0 ? o : r;
}

}  // namespace

int launch_compact_lists(const Batch& b, double rc, const CompactLists& c, cudaStream_t s) {
    const unsigned gW = (unsigned)((32LL * b.natoms + kThreads - 1) / kThreads);
    const double rc2 = rc * rc;
    k_compact<false><<<gW, kThreads, 0, s>>>(b, rc2, c.cnt, c.off, nullptr, nullptr, nullptr);
    int L = 1 + launch_scan(c.off, b.natoms, b.scan_tmp, nullptr, s);
    k_compact<true><<<gW, kThreads, 0, s>>>(b, rc2, c.cnt, c.off, c.nj, c.ns, c.map);
    k_compact_rev<<<(unsigned)(((long long)b.nentries + kThreads - 1) / kThreads), kThreads, 0, s>>>(b, c.map, c.rev);
    return L + 2;
}

// ---------------------------------------------------------------- planned capacities
namespace {

// After the count pass of an evaluation without a host read: entries or the
// largest per-atom count above the planned capacity set flag 32 and status[3],
// and the lists are emptied so that no later kernel indexes past its arrays.
__global__ void k_caps_check(Batch b, long long e_cap, int m_cap) {
    if (blockIdx.x || threadIdx.x) return;
    const int total = b.nei_off[b.natoms];
    if (total < 0 || (long long)total > e_cap || b.status[1] > m_cap) {
        atomicOr(&b.status[0], 32);
        b.status[3] = 1;
    }
}

__global__ void k_caps_clear(Batch b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= b.natoms && b.status[3]) b.nei_off[i] = 0;
}

// Device copies of the host set-up arithmetic (struct_setup, n_cells and inv3
// in capi.cu) with every operation rounded on its own (no contraction), so the
// device-built box of a molecule equals the host-built one bit for bit.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }

__device__ void d_cross(const double* a, const double* b, double* c) {
    c[0] = sub(mul(a[1], b[2]), mul(a[2], b[1]));
    c[1] = sub(mul(a[2], b[0]), mul(a[0], b[2]));
    c[2] = sub(mul(a[0], b[1]), mul(a[1], b[0]));
}

__device__ void d_n_cells(const double* lat, double cut, int* n) {
    double axb[3], axc[3], bxc[3];
    d_cross(lat, lat + 3, axb);
    d_cross(lat, lat + 6, axc);
    d_cross(lat + 3, lat + 6, bxc);
    double* vs[3] = {axb, axc, bxc};
    for (double* v : vs) {
        const double s = __dsqrt_rn(add(add(mul(v[0], v[0]), mul(v[1], v[1])), mul(v[2], v[2])));
        for (int k = 0; k < 3; ++k) v[k] = dv(v[k], s);
    }
    const double p0 = add(add(mul(lat[0], bxc[0]), mul(lat[1], bxc[1])), mul(lat[2], bxc[2]));
    const double p1 = add(add(mul(lat[3], axc[0]), mul(lat[4], axc[1])), mul(lat[5], axc[2]));
    const double p2 = add(add(mul(lat[6], axb[0]), mul(lat[7], axb[1])), mul(lat[8], axb[2]));
    n[0] = (int)ceil(dv(cut, fabs(p0)));
    n[1] = (int)ceil(dv(cut, fabs(p1)));
    n[2] = (int)ceil(dv(cut, fabs(p2)));
}

__device__ void d_inv3(const double* a, double* b) {
    auto A = [&](int r, int c) { return a[r + 3 * c]; };
    const double d = sub(sub(sub(add(add(mul(mul(a[0], a[4]), a[8]), mul(mul(a[3], a[7]), a[2])),
                                     mul(mul(a[6], a[1]), a[5])),
                                 mul(mul(a[0], a[7]), a[5])),
                             mul(mul(a[3], a[1]), a[8])),
                         mul(mul(a[6], a[4]), a[2]));
    const double r0[3] = {A(0, 0), A(0, 1), A(0, 2)}, r1[3] = {A(1, 0), A(1, 1), A(1, 2)},
                 r2[3] = {A(2, 0), A(2, 1), A(2, 2)};
    const double c0[3] = {sub(mul(r1[1], r2[2]), mul(r1[2], r2[1])), sub(mul(r0[2], r2[1]), mul(r0[1], r2[2])),
                          sub(mul(r0[1], r1[2]), mul(r0[2], r1[1]))};
    const double c1[3] = {sub(mul(r1[2], r2[0]), mul(r1[0], r2[2])), sub(mul(r0[0], r2[2]), mul(r0[2], r2[0])),
                          sub(mul(r0[2], r1[0]), mul(r0[0], r1[2]))};
    const double c2[3] = {sub(mul(r1[0], r2[1]), mul(r1[1], r2[0])), sub(mul(r0[1], r2[0]), mul(r0[0], r2[1])),
                          sub(mul(r0[0], r1[1]), mul(r0[1], r1[0]))};
    for (int k = 0; k < 3; ++k) {
        b[0 + 3 * k] = dv(c0[k], d);
        b[1 + 3 * k] = dv(c1[k], d);
        b[2 + 3 * k] = dv(c2[k], d);
    }
}

// Artificial box of each molecule from its current positions (the reference's
// non-periodic branch, neighborLists.f90:129-169): origin min - 1e-4, edge
// extent + 1e-4, grid of >= 0.6 rc cells coarsened like the host set-up, and
// the search range.  One block per structure; periodic structures keep their
// set-up.  Cells were reserved for the largest grid the coarsening allows.
__global__ void k_molecule_boxes(Batch b, double rc) {
    StructInfo& S = const_cast<StructInfo*>(b.info)[blockIdx.x];
    if (S.periodic || keep_list(b)) return;
    __shared__ double red[6][32];
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    const double* p = b.pos + 3 * (size_t)S.atom_off;
    for (int i = threadIdx.x; i < S.nat; i += blockDim.x)
        for (int d = 0; d < 3; ++d) {
            mn[d] = fmin(mn[d], p[3 * i + d]);
            mx[d] = fmax(mx[d], p[3 * i + d]);
        }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int d = 0; d < 3; ++d)
        for (int o = 16; o; o >>= 1) {
            mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    if (lane == 0)
        for (int d = 0; d < 3; ++d) {
            red[d][w] = mn[d];
            red[3 + d][w] = mx[d];
        }
    __syncthreads();
    if (threadIdx.x) return;
    for (int k = 1; k < nw; ++k)
        for (int d = 0; d < 3; ++d) {
            red[d][0] = fmin(red[d][0], red[d][k]);
            red[3 + d][0] = fmax(red[3 + d][0], red[3 + d][k]);
        }
    if (!(isfinite(red[0][0]) && isfinite(red[1][0]) && isfinite(red[2][0]) && isfinite(red[3][0]) &&
          isfinite(red[4][0]) && isfinite(red[5][0]))) {
        // non-finite positions: keep the previous box; the wrap kernel flags the atoms
        return;
    }
    for (int k = 0; k < 9; ++k) S.h[k] = 0.0;
    for (int d = 0; d < 3; ++d) {
        S.org[d] = sub(red[d][0], 1.e-4);
        // max(x - org) = max(x) - org: subtraction by a constant is monotone
        S.h[d + 3 * d] = add(sub(red[3 + d][0], S.org[d]), 1.e-4);
    }
    d_inv3(S.h, S.hinv);
    const double target = mul(rc, 0.6);
    long long ncell = 1;
    for (int d = 0; d < 3; ++d) {
        const double len = __dsqrt_rn(add(add(mul(S.h[3 * d], S.h[3 * d]), mul(S.h[3 * d + 1], S.h[3 * d + 1])),
                                          mul(S.h[3 * d + 2], S.h[3 * d + 2])));
        S.ngrid[d] = (int)dv(len, target) + 1;
        ncell *= S.ngrid[d];
    }
    const long long limit = 64LL * S.nat + 4096;
    while (ncell > limit) {
        ncell = 1;
        for (int d = 0; d < 3; ++d) {
            S.ngrid[d] = max(1, S.ngrid[d] / 2);
            ncell *= S.ngrid[d];
        }
    }
    double grid[9];
    for (int d = 0; d < 3; ++d)
        for (int r = 0; r < 3; ++r) grid[r + 3 * d] = dv(S.h[r + 3 * d], (double)S.ngrid[d]);
    d_n_cells(grid, rc, S.nsearch);
    // cells beyond the molecule's grid are empty (see the host set-up)
    for (int d = 0; d < 3; ++d) S.nsearch[d] = min(S.nsearch[d], S.ngrid[d] - 1);
    for (int d = 0; d < 3; ++d)
        if (S.nsearch[d] > 64) {
            atomicOr(&b.status[0], 32);  // reported as a capacity error
            S.nsearch[d] = 64;
        }
}

}  // namespace

int launch_capacity_guard(const Batch& b, long long e_cap, int m_cap, cudaStream_t s) {
    k_caps_check<<<1, 32, 0, s>>>(b, e_cap, m_cap);
    k_caps_clear<<<(b.natoms + 1 + kThreads - 1) / kThreads, kThreads, 0, s>>>(b);
    return 2;
}

int launch_molecule_boxes(const Batch& b, double rc, cudaStream_t s) {
    k_molecule_boxes<<<b.nstruct, 128, 0, s>>>(b, rc);
    return 1;
}

}  // namespace hdnnp

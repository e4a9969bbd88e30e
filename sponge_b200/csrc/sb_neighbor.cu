// Neighbor list for the nonbonded hot path — replaces SPONGE's NEIGHBOR_LIST
// (SPONGE/neighbor_list/neighbor_list.cu). B200 design:
//
//   1. k_prepare   one pass over atoms: periodic wrap in place (Crd_Periodic_Map semantics,
//                  common.cu:299-352), old_crd copy, fixed-point conversion (Crd_To_Uint_Crd
//                  with 0.25*2^32/L, common.cu:264-287), xy-column index computed exactly in
//                  integers from the fixed-point coordinate, column histogram.
//   2. k_colscan   padded exclusive scan: every column starts on a multiple of 8 slots.
//   3. k_scatter   (z << 32 | atom) keys into their column.
//   4. k_colsort   per-column bitonic sort in shared memory -> deterministic slot order
//                  (z, atom id); writes slot_atom / atom_slot / slot-order coordinates and a
//                  per-column index of 128 z bins.
//   5. k_search    one warp per 8-atom cluster walks the columns around it (half shell in
//                  slot order), takes the z window from the z-bin index, and tests every candidate pair
//                  with the pinned FP32 criterion; surviving j become entries (j | mask << 24).
//
// The pair set represented is exactly the reference's half list: pairs within (rc+skin) under
// minimum image, each unordered pair once, exclusions removed ({a<b} removed iff b is in a's
// CSR exclusion list, neighbor_list.cu:461-511). The reference's list order (atomic appends)
// is non-deterministic; this one is fully determined by the coordinates.

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "sb_internal.cuh"

struct SbAtomGroup {  // layout of SPONGE's ATOM_GROUP (common.cuh:106-110)
    int atom_numbers;
    int* atom_serial;
};

// ---------------------------------------------------------------------------------------------
// pinned FP32 pair criterion (identical to the oracle's pair_r2_f32)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float pair_r2_rn(uint32_t ui, uint32_t vi, uint32_t wi, uint32_t uj,
                                            uint32_t vj, uint32_t wj, float sx, float sy,
                                            float sz) {
    float dx = __fmul_rn(__int2float_rn((int)(uj - ui)), sx);
    float dy = __fmul_rn(__int2float_rn((int)(vj - vi)), sy);
    float dz = __fmul_rn(__int2float_rn((int)(wj - wi)), sz);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// ---------------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------------
__global__ void k_prepare(int n, float* __restrict__ crd, float* __restrict__ old_crd,
                          uint32_t* __restrict__ ucrd, float bx, float by, float bz, float cofx,
                          float cofy, float cofz, int ncx, int ncy, int* __restrict__ col_of,
                          int* __restrict__ col_rank, int* __restrict__ col_count,
                          const int* __restrict__ refresh_flag) {
    if (refresh_flag && refresh_flag[0] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = crd[3 * i], y = crd[3 * i + 1], z = crd[3 * i + 2];
    // Crd_Periodic_Map: a single shift into [0, L)
    if (x >= 0) { if (!(x < bx)) x = x - bx; } else x = x + bx;
    if (y >= 0) { if (!(y < by)) y = y - by; } else y = y + by;
    if (z >= 0) { if (!(z < bz)) z = z - bz; } else z = z + bz;
    crd[3 * i] = x; crd[3 * i + 1] = y; crd[3 * i + 2] = z;
    old_crd[3 * i] = x; old_crd[3 * i + 1] = y; old_crd[3 * i + 2] = z;
    uint32_t ux = ((uint32_t)(int)__fmul_rn(x, cofx)) << 2;
    uint32_t uy = ((uint32_t)(int)__fmul_rn(y, cofy)) << 2;
    uint32_t uz = ((uint32_t)(int)__fmul_rn(z, cofz)) << 2;
    ucrd[3 * i] = ux; ucrd[3 * i + 1] = uy; ucrd[3 * i + 2] = uz;
    int cx = (int)(((unsigned long long)ux * (unsigned)ncx) >> 32);
    int cy = (int)(((unsigned long long)uy * (unsigned)ncy) >> 32);
    int col = cy * ncx + cx;
    col_of[i] = col;
    col_rank[i] = atomicAdd(&col_count[col], 1);
}

// single block: padded exclusive scan of column counts; meta[0] = clusters, meta[3] = slots
__global__ void k_colscan(int ncol, const int* __restrict__ col_count, int* __restrict__ col_start,
                          int* __restrict__ meta, int slot_cap, const int* __restrict__ refresh_flag) {
    if (refresh_flag && refresh_flag[0] == 0) return;
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ncol; base += blockDim.x) {
        int c = base + threadIdx.x;
        int v = c < ncol ? ((col_count[c] + 7) & ~7) : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) >= o) x += t;
        }
        if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            int nw = blockDim.x >> 5;
            int w = threadIdx.x < nw ? warp_sums[threadIdx.x] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= o) w += t;
            }
            warp_sums[threadIdx.x] = w;
        }
        __syncthreads();
        int wid = threadIdx.x >> 5;
        int excl = x - v + (wid > 0 ? warp_sums[wid - 1] : 0) + carry;
        if (c < ncol) col_start[c] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        col_start[ncol] = carry;
        int total = carry > slot_cap ? slot_cap : carry;
        meta[0] = total / SB_CLUSTER;
        meta[3] = total;
    }
}

__global__ void k_scatter(int n, const uint32_t* __restrict__ ucrd, const int* __restrict__ col_of,
                          const int* __restrict__ col_rank, const int* __restrict__ col_start,
                          unsigned long long* __restrict__ tmp, int slot_cap,
                          const int* __restrict__ refresh_flag) {
    if (refresh_flag && refresh_flag[0] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int p = col_start[col_of[i]] + col_rank[i];
    if (p < slot_cap) tmp[p] = ((unsigned long long)ucrd[3 * i + 2] << 32) | (unsigned)i;
}

// one block per column: bitonic sort of (z, atom) keys, then slot bookkeeping
__global__ void k_colsort(int ncol, const int* __restrict__ col_count,
                          const int* __restrict__ col_start,
                          const unsigned long long* __restrict__ tmp,
                          const uint32_t* __restrict__ ucrd, int* __restrict__ slot_atom,
                          int* __restrict__ atom_slot, uint32_t* __restrict__ slot_u,
                          int slot_cap, int* __restrict__ meta, int* __restrict__ zbin,
                          const int* __restrict__ refresh_flag) {
    if (refresh_flag && refresh_flag[0] == 0) return;
    extern __shared__ unsigned long long keys[];
    int col = blockIdx.x;
    int cnt = col_count[col];
    int start = col_start[col];
    int padded = (cnt + 7) & ~7;
    if (start + padded > slot_cap) {
        if (threadIdx.x == 0) atomicOr(&meta[1], SB_STATUS_LIST_OVERFLOW);
        return;
    }
    if (cnt > SB_COLUMN_SORT_CAP) {
        if (threadIdx.x == 0) atomicOr(&meta[1], SB_STATUS_COLUMN_OVERFLOW);
        cnt = SB_COLUMN_SORT_CAP;
    }
    int m = 1;
    while (m < cnt) m <<= 1;
    for (int t = threadIdx.x; t < m; t += blockDim.x)
        keys[t] = t < cnt ? tmp[start + t] : ~0ull;
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < m; t += blockDim.x) {
                int p = t ^ j;
                if (p > t) {
                    unsigned long long a = keys[t], b = keys[p];
                    bool up = (t & k) == 0;
                    if ((a > b) == up) {
                        keys[t] = b;
                        keys[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    // z-bin index of the sorted column: zbin[b] = first slot whose z >= b 2^SB_ZBIN_SHIFT
    for (int b = threadIdx.x; b <= SB_ZBINS; b += blockDim.x) {
        const unsigned long long zb = (unsigned long long)b << SB_ZBIN_SHIFT;
        int lo = 0, hi = cnt;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((keys[mid] >> 32) < zb) lo = mid + 1;
            else hi = mid;
        }
        zbin[(size_t)col * (SB_ZBINS + 1) + b] = start + lo;
    }
    int sz = slot_cap;
    for (int t = threadIdx.x; t < padded; t += blockDim.x) {
        int s = start + t;
        if (t < cnt) {
            int a = (int)(keys[t] & 0xffffffffu);
            slot_atom[s] = a;
            atom_slot[a] = s;
            slot_u[s] = ucrd[3 * a];
            slot_u[sz + s] = ucrd[3 * a + 1];
            slot_u[2 * sz + s] = ucrd[3 * a + 2];
        } else {
            slot_atom[s] = -1;
            slot_u[s] = 0;
            slot_u[sz + s] = 0;
            slot_u[2 * sz + s] = 0;
        }
    }
}

__global__ void k_excl_range(int n, const int* __restrict__ es, const int* __restrict__ en,
                             const int* __restrict__ el, int* __restrict__ lo,
                             int* __restrict__ hi, const int* __restrict__ refresh_flag) {
    if (refresh_flag && refresh_flag[0] == 0) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = INT_MAX, b = -1;
    if (en) {
        int s = es[i], e = s + en[i];
        for (int k = s; k < e; k++) {
            int v = el[k];
            a = min(a, v);
            b = max(b, v);
        }
    }
    lo[i] = a;
    hi[i] = b;
}

// {a, b} excluded: the pair's lower id p carries the other id q in its CSR list; [lo, hi] is the
// id range of p's list (the caller holds it for both atoms), so most pairs need no list walk
__device__ __forceinline__ bool excluded_pair(int a, int b, int lo_a, int hi_a, int lo_b,
                                              int hi_b, const int* __restrict__ es,
                                              const int* __restrict__ en,
                                              const int* __restrict__ el) {
    const bool a_low = a < b;
    const int p = a_low ? a : b, q = a_low ? b : a;
    const int lo = a_low ? lo_a : lo_b, hi = a_low ? hi_a : hi_b;
    if (q < lo || q > hi) return false;
    const int s = es[p], e = s + en[p];
    for (int k = s; k < e; k++)
        if (el[k] == q) return true;
    return false;
}

struct SearchParams {
    int ncx, ncy, nxr, nyr, fullx, fully;
    float sx, sy, sz, cs2, colwx, colwy, cs, lx, ly, lz;
    float colw;            // the wider column width
    int max_ranges;        // 2 x columns of the half-shell walk (two z windows per column)
    float zscale;          // fixed-point units per A along z (2^32 / Lz)
    int slot_cap, ent_cap;
};

// inclusive z windows [zmin - rz, zmax + rz] with periodic wrap (one or two ranges)
__device__ __forceinline__ int z_windows(uint32_t zmin, uint32_t zmax, unsigned long long rz,
                                         uint32_t (&wa)[2], uint32_t (&wb)[2]) {
    const long long zlo = (long long)zmin - (long long)rz;
    const long long zhi = (long long)zmax + (long long)rz;
    if (zhi - zlo >= 4294967296ll) {
        wa[0] = 0; wb[0] = 0xffffffffu;
        return 1;
    }
    if (zlo < 0) {
        wa[0] = 0; wb[0] = (uint32_t)zhi; wa[1] = (uint32_t)(zlo + 4294967296ll); wb[1] = 0xffffffffu;
        return 2;
    }
    if (zhi > 0xffffffffll) {
        wa[0] = 0; wb[0] = (uint32_t)(zhi - 4294967296ll); wa[1] = (uint32_t)zlo; wb[1] = 0xffffffffu;
        return 2;
    }
    wa[0] = (uint32_t)zlo; wb[0] = (uint32_t)zhi;
    return 1;
}

// One warp per cluster; lanes take candidate j slots, each lane tests its j against the 8 i
// atoms. The decision per (i, j) is the pinned FP32 criterion (pair_r2_rn < cs^2). It is
// evaluated exactly only where it could go either way: every candidate is first placed in the
// cluster's relative float frame (one conversion per coordinate per j). Both that r^2 and the
// pinned one are within a few ulp per coordinate of the exact value: with R a bound on the
// frame coordinates of any candidate (cluster extent + 2 cs + 2 column widths), the two differ
// by at most 2 sqrt(3) cs (R 2^-21) + cs^2 2^-20 near cs^2; outside ten times that band the
// frame's answer is the pinned answer. Clusters flagged exact (the frame may not be the minimum
// image) use the pinned test on every pair. The z window of each column shrinks with the xy gap
// between the cluster's column and that column.
#define SB_SEARCH_WARPS 4
__global__ void __launch_bounds__(32 * SB_SEARCH_WARPS) k_search(
    SearchParams P, const int* __restrict__ col_start, const int* __restrict__ col_count,
    const uint32_t* __restrict__ slot_u, const int* __restrict__ slot_atom,
    const int* __restrict__ excl_lo, const int* __restrict__ excl_hi,
    const int* __restrict__ es, const int* __restrict__ en, const int* __restrict__ el,
    const int* __restrict__ zbin,
    int* __restrict__ cl_count, uint32_t* __restrict__ cl_ent, int* __restrict__ meta,
    const int* __restrict__ refresh_flag) {
    // per-warp copy of the cluster's atoms for the rarely taken per-slot paths (dynamic index)
    __shared__ int s_ia[SB_SEARCH_WARPS][SB_CLUSTER], s_lo[SB_SEARCH_WARPS][SB_CLUSTER],
        s_hi[SB_SEARCH_WARPS][SB_CLUSTER];
    __shared__ uint32_t s_u[SB_SEARCH_WARPS][SB_CLUSTER], s_v[SB_SEARCH_WARPS][SB_CLUSTER],
        s_w[SB_SEARCH_WARPS][SB_CLUSTER];
    extern __shared__ int s_ranges[];  // per warp: max_ranges starts, max_ranges + 1 prefixes
    if (refresh_flag && refresh_flag[0] == 0) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= meta[0]) return;
    const uint32_t* __restrict__ UX = slot_u;
    const uint32_t* __restrict__ UY = slot_u + P.slot_cap;
    const uint32_t* __restrict__ UZ = slot_u + 2 * P.slot_cap;
    const int base = c * SB_CLUSTER;
    // cluster atoms: lanes 0..7 load; register copies of the relative frame for all lanes
    const int my_atom = lane < SB_CLUSTER ? slot_atom[base + lane] : -1;
    const uint32_t my_u = lane < SB_CLUSTER ? UX[base + lane] : 0;
    const uint32_t my_v = lane < SB_CLUSTER ? UY[base + lane] : 0;
    const uint32_t my_w = lane < SB_CLUSTER ? UZ[base + lane] : 0;
    if (lane < SB_CLUSTER) {
        s_ia[wid][lane] = my_atom;
        s_lo[wid][lane] = my_atom >= 0 ? excl_lo[my_atom] : INT_MAX;
        s_hi[wid][lane] = my_atom >= 0 ? excl_hi[my_atom] : -1;
        s_u[wid][lane] = my_u;
        s_v[wid][lane] = my_v;
        s_w[wid][lane] = my_w;
    }
    __syncwarp();
    const uint32_t u0 = __shfl_sync(0xffffffffu, my_u, 0);
    const uint32_t v0 = __shfl_sync(0xffffffffu, my_v, 0);
    const uint32_t w0 = __shfl_sync(0xffffffffu, my_w, 0);
    // z extent of the real atoms (sorted ascending in z inside the cluster)
    const unsigned real = __ballot_sync(0xffffffffu, my_atom >= 0) & 0xffu;
    const uint32_t zmin = w0;
    const uint32_t zmax = __shfl_sync(0xffffffffu, my_w, 31 - __clz(real));
    // relative float frame of the cluster (origin: its first atom)
    const float mxr = __int2float_rn((int)(my_u - u0)) * P.sx;
    const float myr = __int2float_rn((int)(my_v - v0)) * P.sy;
    const float mzr = __int2float_rn((int)(my_w - w0)) * P.sz;
    float ex = (lane < SB_CLUSTER && my_atom >= 0) ? fmaxf(fabsf(mxr), 0.f) : 0.f;
    float ey = (lane < SB_CLUSTER && my_atom >= 0) ? fabsf(myr) : 0.f;
    float ez = (lane < SB_CLUSTER && my_atom >= 0) ? fabsf(mzr) : 0.f;
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1) {
        ex = fmaxf(ex, __shfl_xor_sync(0xffffffffu, ex, o));
        ey = fmaxf(ey, __shfl_xor_sync(0xffffffffu, ey, o));
        ez = fmaxf(ez, __shfl_xor_sync(0xffffffffu, ez, o));
    }
    ex = __shfl_sync(0xffffffffu, ex, 0);
    ey = __shfl_sync(0xffffffffu, ey, 0);
    ez = __shfl_sync(0xffffffffu, ez, 0);
    // the cluster's relative coordinates, negated, as slot pairs (2p, 2p+1) in every lane: the
    // candidate tests run on packed FP32x2 arithmetic (each half rounds as the scalar operation)
    float2 nrx[SB_CLUSTER / 2], nry[SB_CLUSTER / 2], nrz[SB_CLUSTER / 2];
#pragma unroll
    for (int p = 0; p < SB_CLUSTER / 2; p++) {
        nrx[p] = make_float2(-__shfl_sync(0xffffffffu, mxr, 2 * p),
                             -__shfl_sync(0xffffffffu, mxr, 2 * p + 1));
        nry[p] = make_float2(-__shfl_sync(0xffffffffu, myr, 2 * p),
                             -__shfl_sync(0xffffffffu, myr, 2 * p + 1));
        nrz[p] = make_float2(-__shfl_sync(0xffffffffu, mzr, 2 * p),
                             -__shfl_sync(0xffffffffu, mzr, 2 * p + 1));
    }
    __syncwarp();
    // exact-path flag: the cluster-relative float frame of the pair kernel is a faithful
    // minimum image only while cs + (extent of the cluster from its first atom) < L/2
    const int exact = (ex + P.cs >= 0.49f * P.lx) || (ey + P.cs >= 0.49f * P.ly) ||
                      (ez + P.cs >= 0.49f * P.lz);
    const float R = fmaxf(ex, fmaxf(ey, ez)) + 2.f * P.cs + 2.f * P.colw;
    const float band = 10.f * (3.5f * P.cs * R * 4.8e-7f + P.cs2 * 9.6e-7f);
    const float cs2_lo = P.cs2 - band, cs2_hi = P.cs2 + band;
    // own column from the first atom
    const int cx = (int)(((unsigned long long)u0 * (unsigned)P.ncx) >> 32);
    const int cy = (int)(((unsigned long long)v0 * (unsigned)P.ncy) >> 32);
    const int col = cy * P.ncx + cx;
    // candidate ranges: the lanes take the (dy, dx) columns of the half shell in parallel, each
    // giving up to two slot ranges (its z window, wrapped); r = 2 (column index) + window keeps
    // the order of a sequential walk (dy outer, dx inner, window), so the entries come out in
    // that order. rs[r] = first slot, rp[r] = exclusive prefix of the range lengths.
    const int dy0 = P.fully ? 0 : -P.nyr, dy1 = P.fully ? P.ncy - 1 : P.nyr;
    const int dx0 = P.fullx ? 0 : -P.nxr, dx1 = P.fullx ? P.ncx - 1 : P.nxr;
    const int nxw = dx1 - dx0 + 1;
    const int ncols = (dy1 - dy0 + 1) * nxw;
    int* rs = s_ranges + wid * (2 * P.max_ranges + 1);
    int* rp = rs + P.max_ranges;  // max_ranges + 1 entries
    const int nr = 2 * ncols;
    int carry = 0;
    for (int q0 = 0; q0 < ncols; q0 += 16) {
        // 16 columns per round: lane l handles column q0 + l/2, window l&1
        const int q = q0 + (lane >> 1), w = lane & 1;
        int ra = 0, len = 0;
        if (q < ncols) {
            const int dy = dy0 + q / nxw, dx = dx0 + q % nxw;
            int cy2, ady, cx2, adx;
            if (P.fully) {
                cy2 = dy;
                const int d = abs(cy2 - cy);
                ady = min(d, P.ncy - d);
            } else {
                cy2 = cy + dy;
                if (cy2 < 0) cy2 += P.ncy;
                if (cy2 >= P.ncy) cy2 -= P.ncy;
                ady = abs(dy);
            }
            if (P.fullx) {
                cx2 = dx;
                const int d = abs(cx2 - cx);
                adx = min(d, P.ncx - d);
            } else {
                cx2 = cx + dx;
                if (cx2 < 0) cx2 += P.ncx;
                if (cx2 >= P.ncx) cx2 -= P.ncx;
                adx = abs(dx);
            }
            const int col2 = cy2 * P.ncx + cx2;
            const float gy = fmaxf(0.f, (float)(ady - 1)) * P.colwy;
            const float gx = fmaxf(0.f, (float)(adx - 1)) * P.colwx;
            const float g2 = gx * gx + gy * gy;
            // earlier columns precede this cluster in slot order; columns beyond cs are skipped
            if (col2 >= col && g2 < P.cs2) {
                // z reach in this column: sqrt(cs^2 - (xy gap)^2), widened for rounding
                const float rzA = sqrtf(P.cs2 - g2) * 1.001f + 1e-3f;
                const unsigned long long rz =
                    (unsigned long long)((double)rzA * (double)P.zscale) + 1024ull;
                uint32_t wa[2], wb[2];
                const int nwin = z_windows(zmin, zmax, rz, wa, wb);
                if (w < nwin) {
                    const int s0 = col_start[col2];
                    const int s1 = s0 + col_count[col2];
                    // a superset of the z window (whole bins); the pair test filters
                    const int* zb = zbin + (size_t)col2 * (SB_ZBINS + 1);
                    int lo = max(zb[(w ? wa[1] : wa[0]) >> SB_ZBIN_SHIFT], s0);
                    const int hi = min(zb[((w ? wb[1] : wb[0]) >> SB_ZBIN_SHIFT) + 1], s1);
                    if (col2 == col) lo = max(lo, base + 1);
                    ra = lo;
                    len = max(hi - lo, 0);
                }
            }
        }
        // exclusive scan of the lengths over the warp, continuing the running carry
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int r = 2 * q0 + lane;
        if (r < nr) {
            rs[r] = ra;
            rp[r] = carry + incl - len;
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) rp[nr] = carry;
    __syncwarp();
    const int total = carry;
    int count = 0;
    uint32_t* out = cl_ent + (size_t)c * P.ent_cap;
    int r = 0;  // this lane's current range (advances monotonically)
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        unsigned mask = 0;
        if (t < total) {
            while (rp[r + 1] <= t) r++;
            const int j = rs[r] + (t - rp[r]);
            const uint32_t ju = UX[j], jv = UY[j], jw = UZ[j];
            unsigned near = 0, border = 0xffu;
            if (!exact) {
                const float xj = __int2float_rn((int)(ju - u0)) * P.sx;
                const float yj = __int2float_rn((int)(jv - v0)) * P.sy;
                const float zj = __int2float_rn((int)(jw - w0)) * P.sz;
                unsigned notfar = 0;
                const float2 xj2 = make_float2(xj, xj), yj2 = make_float2(yj, yj),
                             zj2 = make_float2(zj, zj);
#pragma unroll
                for (int p = 0; p < SB_CLUSTER / 2; p++) {
                    // xj + (-r) rounds as xj - r
                    const float2 ddx = __fadd2_rn(xj2, nrx[p]), ddy = __fadd2_rn(yj2, nry[p]),
                                 ddz = __fadd2_rn(zj2, nrz[p]);
                    const float2 r2a =
                        __ffma2_rn(ddx, ddx, __ffma2_rn(ddy, ddy, __fmul2_rn(ddz, ddz)));
                    near |= ((r2a.x < cs2_lo ? 1u : 0u) | (r2a.y < cs2_lo ? 2u : 0u)) << (2 * p);
                    notfar |= ((r2a.x <= cs2_hi ? 1u : 0u) | (r2a.y <= cs2_hi ? 2u : 0u))
                              << (2 * p);
                }
                border = notfar & ~near;
            }
            // slots the frame cannot decide: the pinned test itself
            while (border) {
                const int k = __ffs(border) - 1;
                border &= border - 1u;
                if (pair_r2_rn(s_u[wid][k], s_v[wid][k], s_w[wid][k], ju, jv, jw, P.sx, P.sy,
                               P.sz) < P.cs2)
                    near |= 1u << k;
            }
            // slots in range: padding, slot order and exclusions
            if (near) {
                const int ja = slot_atom[j];
                const int jlo = ja >= 0 ? excl_lo[ja] : INT_MAX;
                const int jhi = ja >= 0 ? excl_hi[ja] : -1;
                while (near) {
                    const int k = __ffs(near) - 1;
                    near &= near - 1u;
                    const int ak = s_ia[wid][k];
                    if (ak >= 0 && base + k < j &&
                        !excluded_pair(ak, ja, s_lo[wid][k], s_hi[wid][k], jlo, jhi, es, en,
                                       el))
                        mask |= 1u << k;
                }
            }
            if (mask != 0) mask |= (unsigned)j << 8;  // carry j for the store below
        }
        const unsigned bal = __ballot_sync(0xffffffffu, mask != 0);
        const int pos = count + __popc(bal & ((1u << lane) - 1u));
        if (mask != 0) {
            if (pos < P.ent_cap)
                out[pos] = (mask >> 8) | ((mask & 0xffu) << 24);
            else
                atomicOr(&meta[1], SB_STATUS_LIST_OVERFLOW);
        }
        count += __popc(bal);
    }
    if (lane == 0) cl_count[c] = min(count, P.ent_cap) | (exact ? SB_CL_EXACT : 0);
}

__global__ void k_refresh_check(int n, const float* __restrict__ crd,
                                const float* __restrict__ old_crd, float bx, float by, float bz,
                                float thr, int* __restrict__ flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // Is_need_refresh_neighbor_list_cuda (neighbor_list.cu:444-459)
    float dx = crd[3 * i] - old_crd[3 * i];
    float dy = crd[3 * i + 1] - old_crd[3 * i + 1];
    float dz = crd[3 * i + 2] - old_crd[3 * i + 2];
    dx = dx - floorf(dx / bx + 0.5f) * bx;
    dy = dy - floorf(dy / by + 0.5f) * by;
    dz = dz - floorf(dz / bz + 0.5f) * bz;
    if (dx * dx + dy * dy + dz * dz > thr) atomicExch(flag, 1);
}

__global__ void k_count_pairs(const int* __restrict__ meta, const int* __restrict__ cl_count,
                              const uint32_t* __restrict__ cl_ent, int ent_cap,
                              unsigned long long* __restrict__ total) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = 0;
    if (c < meta[0]) {
        const uint32_t* e = cl_ent + (size_t)c * ent_cap;
        int cnt = min(cl_count[c] & SB_CL_COUNT_MASK, ent_cap);
        for (int k = 0; k < cnt; k++) v += __popc(e[k] >> 24);
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(total, v);
}

__global__ void k_export_pairs(int n, const int* __restrict__ meta, const int* __restrict__ cl_count,
                               const uint32_t* __restrict__ cl_ent, int ent_cap,
                               const int* __restrict__ slot_atom,
                               unsigned long long* __restrict__ cursor,
                               long long* __restrict__ keys, long long cap) {
    int c = blockIdx.x;
    if (c >= meta[0]) return;
    const uint32_t* e = cl_ent + (size_t)c * ent_cap;
    int cnt = min(cl_count[c] & SB_CL_COUNT_MASK, ent_cap);
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        uint32_t v = e[t];
        int j = (int)(v & 0xffffffu);
        unsigned m = v >> 24;
        int b = slot_atom[j];
        for (int k = 0; k < SB_CLUSTER; k++)
            if (m & (1u << k)) {
                int a = slot_atom[c * SB_CLUSTER + k];
                long long lo = min(a, b), hi = max(a, b);
                unsigned long long p = atomicAdd(cursor, 1ull);
                if ((long long)p < cap) keys[p] = lo * (long long)n + hi;
            }
    }
}

__global__ void k_ag_reset(int n, SbAtomGroup* __restrict__ ag, int* __restrict__ serial,
                           int maxnb, int set_ptr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ag[i].atom_numbers = 0;
    if (set_ptr) ag[i].atom_serial = serial + (size_t)i * maxnb;
}

__global__ void k_ag_fill(const int* __restrict__ meta, const int* __restrict__ cl_count,
                          const uint32_t* __restrict__ cl_ent, int ent_cap,
                          const int* __restrict__ slot_atom, SbAtomGroup* __restrict__ ag,
                          int* __restrict__ serial, int maxnb, int* __restrict__ meta_w) {
    int c = blockIdx.x;
    if (c >= meta[0]) return;
    const uint32_t* e = cl_ent + (size_t)c * ent_cap;
    int cnt = min(cl_count[c] & SB_CL_COUNT_MASK, ent_cap);
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        uint32_t v = e[t];
        int j = (int)(v & 0xffffffu);
        unsigned m = v >> 24;
        int b = slot_atom[j];
        for (int k = 0; k < SB_CLUSTER; k++)
            if (m & (1u << k)) {
                int a = slot_atom[c * SB_CLUSTER + k];
                int lo = min(a, b), hi = max(a, b);
                int p = atomicAdd(&ag[lo].atom_numbers, 1);
                if (p < maxnb)
                    serial[(size_t)lo * maxnb + p] = hi;
                else
                    atomicOr(&meta_w[1], SB_STATUS_ATOMGROUP_OVERFLOW);
            }
    }
}

__global__ void k_ag_clamp(int n, SbAtomGroup* __restrict__ ag, int maxnb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && ag[i].atom_numbers > maxnb) ag[i].atom_numbers = maxnb;
}

// slot-order coordinates, charges and types for the pair kernels; with a pruned list
// (xq_prune given) also the displacement test against the coordinates of the last prune: an atom
// that moved more than half the prune buffer requests a new prune (prune_req = meta + 6)
__global__ void k_pack(const int* __restrict__ meta, const int* __restrict__ slot_atom,
                       const uint32_t* __restrict__ uc, const float* __restrict__ q,
                       const int* __restrict__ type, uint4* __restrict__ xq,
                       int* __restrict__ stype, const uint4* __restrict__ xq_prune, float sx,
                       float sy, float sz, float move2, int* __restrict__ prune_req,
                       int slot_cap) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slot_cap) return;
    const int a = slot_atom[s];
    const uint4 o = xq_prune ? xq_prune[s] : make_uint4(0u, 0u, 0u, 0u);
    if (s < meta[3])
        sb_pack_slot(s, a, o, uc, q, type, xq, stype, xq_prune != nullptr, sx, sy, sz, move2,
                     prune_req);
}

// fixed-point forces to the caller's float array (slot order -> atom order), clearing the
// accumulator; also retires a prune request that the pair launch before it served (meta[6..7])
__global__ void k_finalize(int* __restrict__ meta, const int* __restrict__ slot_atom,
                           long long* __restrict__ fix, int slot_cap, float* __restrict__ frc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) sb_retire_prune(meta);
    if (s >= slot_cap) return;
    const int a = slot_atom[s];
    const long long fx = fix[s], fy = fix[slot_cap + s], fz = fix[2 * slot_cap + s];
    if (s < meta[3]) sb_finalize_slot(s, a, fx, fy, fz, fix, slot_cap, frc);
}

__global__ void k_crd_to_uint(int n, const float* __restrict__ crd, float cx, float cy, float cz,
                              uint32_t* __restrict__ uc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uc[3 * i] = ((uint32_t)(int)__fmul_rn(crd[3 * i], cx)) << 2;
    uc[3 * i + 1] = ((uint32_t)(int)__fmul_rn(crd[3 * i + 1], cy)) << 2;
    uc[3 * i + 2] = ((uint32_t)(int)__fmul_rn(crd[3 * i + 2], cz)) << 2;
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
static void nl_grid(sb_neighbor_list* nl) {
    double V = (double)nl->box[0] * nl->box[1] * nl->box[2];
    double rho = nl->n / V;
    double w = cbrt((double)SB_CLUSTER / (rho > 0 ? rho : 1e-3));
    nl->ncx = std::max(1, (int)floor(nl->box[0] / w));
    nl->ncy = std::max(1, (int)floor(nl->box[1] / w));
    nl->ncol = nl->ncx * nl->ncy;
    double cwx = (double)nl->box[0] / nl->ncx, cwy = (double)nl->box[1] / nl->ncy;
    nl->nxr = (int)ceil(nl->cs / cwx);
    nl->nyr = (int)ceil(nl->cs / cwy);
    nl->slot_cap = nl->n + SB_CLUSTER * nl->ncol;
    nl->clu_cap = nl->slot_cap / SB_CLUSTER;
    // entry capacity: all atoms within cs of a cluster box (a half shell in slot order can be a
    // full shell for the first columns), with 50% margin
    double h = SB_CLUSTER / (rho * cwx * cwy);
    double ax = cwx, ay = cwy, az = std::min(h, (double)nl->box[2]);
    double R = nl->cs;
    double vm = ax * ay * az + 2 * R * (ax * ay + ay * az + ax * az) +
                M_PI * R * R * (ax + ay + az) + 4.0 / 3.0 * M_PI * R * R * R;
    vm = std::min(vm, V);
    int cap = (int)(1.5 * rho * vm) + 64;
    cap = std::min(cap, nl->n + 32);
    nl->ent_cap = std::max(64, (cap + 31) & ~31);
}

static int nl_alloc(sb_neighbor_list* nl) {
    int n = nl->n;
    SB_TRY(sb_malloc((void**)&nl->old_crd, sizeof(float) * 3 * n, "old_crd"));
    SB_TRY(sb_malloc((void**)&nl->ucrd, sizeof(uint32_t) * 3 * n, "uint_crd"));
    SB_TRY(sb_malloc((void**)&nl->col_of, sizeof(int) * n, "col_of"));
    SB_TRY(sb_malloc((void**)&nl->col_rank, sizeof(int) * n, "col_rank"));
    SB_TRY(sb_malloc((void**)&nl->col_count, sizeof(int) * nl->ncol, "col_count"));
    SB_TRY(sb_malloc((void**)&nl->col_start, sizeof(int) * (nl->ncol + 1), "col_start"));
    SB_TRY(sb_malloc((void**)&nl->sort_tmp, sizeof(unsigned long long) * nl->slot_cap, "sort"));
    SB_TRY(sb_malloc((void**)&nl->slot_atom, sizeof(int) * nl->slot_cap, "slot_atom"));
    SB_TRY(sb_malloc((void**)&nl->atom_slot, sizeof(int) * n, "atom_slot"));
    SB_TRY(sb_malloc((void**)&nl->slot_u, sizeof(uint32_t) * 3 * nl->slot_cap, "slot_u"));
    SB_TRY(sb_malloc((void**)&nl->excl_lo, sizeof(int) * n, "excl_lo"));
    SB_TRY(sb_malloc((void**)&nl->excl_hi, sizeof(int) * n, "excl_hi"));
    SB_TRY(sb_malloc((void**)&nl->cl_count, sizeof(int) * nl->clu_cap, "cl_count"));
    SB_TRY(sb_malloc((void**)&nl->zbin, sizeof(int) * (size_t)nl->ncol * (SB_ZBINS + 1),
                     "z bins"));
    SB_TRY(sb_malloc((void**)&nl->cl_ent, sizeof(uint32_t) * (size_t)nl->clu_cap * nl->ent_cap,
                     "cluster list"));
    SB_TRY(sb_malloc((void**)&nl->meta, sizeof(int) * 8, "meta"));
    SB_TRY(sb_malloc((void**)&nl->xq, sizeof(uint4) * nl->slot_cap, "xq"));
    SB_TRY(sb_malloc((void**)&nl->stype, sizeof(int) * nl->slot_cap, "stype"));
    SB_TRY(sb_malloc((void**)&nl->fix, sizeof(long long) * 3 * nl->slot_cap, "force fix"));
    SB_CHECK_CUDA(cudaMemset(nl->meta, 0, sizeof(int) * 8));  // no prune requested
    SB_CHECK_CUDA(cudaMemset(nl->fix, 0, sizeof(long long) * 3 * nl->slot_cap));
    SB_CHECK_CUDA(cudaMemset(nl->cl_count, 0, sizeof(int) * nl->clu_cap));
    SB_CHECK_CUDA(cudaMemset(nl->slot_atom, 0xff, sizeof(int) * nl->slot_cap));
    return SB_OK;
}

static void nl_free(sb_neighbor_list* nl) {
    void* ps[] = {nl->old_crd, nl->ucrd, nl->col_of, nl->col_rank, nl->col_count, nl->col_start,
                  nl->sort_tmp, nl->slot_atom, nl->atom_slot, nl->slot_u, nl->excl_lo,
                  nl->excl_hi, nl->cl_count, nl->cl_ent, nl->meta, nl->xq, nl->stype, nl->fix,
                  nl->ag, nl->ag_serial, nl->zbin, nl->cl_count_in, nl->cl_ent_in,
                  nl->cl_ent_tmp, nl->xq_prune};
    for (void* p : ps) sb_free(p);
}

extern "C" int sb_nl_create(int atom_numbers, const float box_length[3], float cutoff,
                            float skin, int refresh_interval, float skin_permit,
                            int max_neighbor_numbers, int form, sb_neighbor_list** out) {
    if (!out || atom_numbers <= 0 || !box_length || cutoff <= 0 || skin < 0) {
        sb_set_error("sb_nl_create: invalid argument");
        return SB_ERR_ARG;
    }
    if (atom_numbers >= SB_MAX_SLOTS) {
        sb_set_error("sb_nl_create: at most %d atoms supported", SB_MAX_SLOTS - 1);
        return SB_ERR_ARG;
    }
    sb_neighbor_list* nl = new sb_neighbor_list();
    nl->n = atom_numbers;
    for (int d = 0; d < 3; d++) nl->box[d] = box_length[d];
    nl->cutoff = cutoff;
    nl->skin = skin;
    nl->cs = cutoff + skin;  // float, as cutoff_with_skin (neighbor_list.cu:723)
    nl->cs2 = nl->cs * nl->cs;
    nl->refresh_interval = refresh_interval;
    nl->skin_permit = 2.0f * (skin_permit > 0 ? skin_permit : 0.5f);
    nl->half_skin_square = 0.25f * skin * skin;
    nl->form = form;
    nl->max_neighbor_numbers = max_neighbor_numbers > 0 ? max_neighbor_numbers : 800;
    nl_grid(nl);
    if (nl->slot_cap >= SB_MAX_SLOTS) {
        delete nl;
        sb_set_error("sb_nl_create: too many slots");
        return SB_ERR_ARG;
    }
    int st = nl_alloc(nl);
    if (st != SB_OK) {
        nl_free(nl);
        delete nl;
        return st;
    }
    *out = nl;
    return SB_OK;
}

extern "C" int sb_nl_destroy(sb_neighbor_list* nl) {
    if (!nl) return SB_OK;
    cudaDeviceSynchronize();
    nl_free(nl);
    delete nl;
    return SB_OK;
}

static int nl_rebuild(sb_neighbor_list* nl, float* d_crd, const int* es, const int* el,
                      const int* en, const int* dflag, cudaStream_t s) {
    int n = nl->n;
    int tb = 256;
    float cof[3], sc[3];
    for (int d = 0; d < 3; d++) {
        cof[d] = (0.25f * 4294967296.0f) / nl->box[d];
        sc[d] = (1.0f / 4294967296.0f) * nl->box[d];
    }
    SB_CHECK_CUDA(cudaMemsetAsync(nl->col_count, 0, sizeof(int) * nl->ncol, s));
    k_prepare<<<(n + tb - 1) / tb, tb, 0, s>>>(n, d_crd, nl->old_crd, nl->ucrd, nl->box[0],
                                               nl->box[1], nl->box[2], cof[0], cof[1], cof[2],
                                               nl->ncx, nl->ncy, nl->col_of, nl->col_rank,
                                               nl->col_count, dflag);
    SB_CHECK_LAUNCH();
    k_colscan<<<1, 1024, 0, s>>>(nl->ncol, nl->col_count, nl->col_start, nl->meta, nl->slot_cap,
                                 dflag);
    SB_CHECK_LAUNCH();
    k_scatter<<<(n + tb - 1) / tb, tb, 0, s>>>(n, nl->ucrd, nl->col_of, nl->col_rank,
                                               nl->col_start, nl->sort_tmp, nl->slot_cap, dflag);
    SB_CHECK_LAUNCH();
    // sort capacity: largest power of two needed is bounded by SB_COLUMN_SORT_CAP
    k_colsort<<<nl->ncol, 256, SB_COLUMN_SORT_CAP * sizeof(unsigned long long), s>>>(
        nl->ncol, nl->col_count, nl->col_start, nl->sort_tmp, nl->ucrd, nl->slot_atom,
        nl->atom_slot, nl->slot_u, nl->slot_cap, nl->meta, nl->zbin, dflag);
    SB_CHECK_LAUNCH();
    k_excl_range<<<(n + tb - 1) / tb, tb, 0, s>>>(n, es, en, el, nl->excl_lo, nl->excl_hi, dflag);
    SB_CHECK_LAUNCH();
    SearchParams P;
    P.ncx = nl->ncx;
    P.ncy = nl->ncy;
    P.nxr = nl->nxr;
    P.nyr = nl->nyr;
    P.fullx = (2 * nl->nxr + 1 >= nl->ncx);
    P.fully = (2 * nl->nyr + 1 >= nl->ncy);
    P.sx = sc[0];
    P.sy = sc[1];
    P.sz = sc[2];
    P.cs2 = nl->cs2;
    P.cs = nl->cs;
    P.lx = nl->box[0];
    P.ly = nl->box[1];
    P.lz = nl->box[2];
    P.colwx = nl->box[0] / nl->ncx;
    P.colwy = nl->box[1] / nl->ncy;
    // fixed-point units per A along z (the z windows are sized per column in the kernel)
    P.zscale = (float)(4294967296.0 / (double)nl->box[2]);
    P.colw = std::max(P.colwx, P.colwy);
    P.slot_cap = nl->slot_cap;
    P.ent_cap = nl->ent_cap;
    {
        const int nyw = P.fully ? P.ncy : 2 * P.nyr + 1, nxw = P.fullx ? P.ncx : 2 * P.nxr + 1;
        P.max_ranges = 2 * nyw * nxw;
    }
    const size_t search_smem = sizeof(int) * SB_SEARCH_WARPS * (2 * (size_t)P.max_ranges + 1);
    if (search_smem > 200 * 1024) {
        sb_set_error("neighbor search: %d column ranges per cluster exceed shared memory",
                     P.max_ranges);
        return SB_ERR_ARG;
    }
    if (search_smem > 48 * 1024)
        cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)search_smem);
    const int warps_per_block = SB_SEARCH_WARPS;
    const int blocks = (nl->clu_cap + warps_per_block - 1) / warps_per_block;
    k_search<<<blocks, 32 * warps_per_block, search_smem, s>>>(
        P, nl->col_start, nl->col_count, nl->slot_u, nl->slot_atom, nl->excl_lo, nl->excl_hi,
        es, en, el, nl->zbin, nl->cl_count, nl->cl_ent, nl->meta, dflag);
    SB_CHECK_LAUNCH();
    if (nl->prune_buffer > 0.f) {
        // the slots changed: the pruned list is rebuilt by the next pair launch
        SB_CHECK_CUDA(cudaMemsetAsync(nl->meta + 6, 1, sizeof(int), s));
        nl->prune_count = 0;
    }
    nl->ag_valid = 0;
    nl->build_id++;
    return SB_OK;
}

extern "C" int sb_nl_update(sb_neighbor_list* nl, float* d_crd, const int* es, const int* el,
                            const int* en, int forced_update, int forced_check, void* stream) {
    if (!nl || !d_crd) {
        sb_set_error("sb_nl_update: null argument");
        return SB_ERR_ARG;
    }
    if ((es == nullptr) != (en == nullptr)) {
        sb_set_error("sb_nl_update: exclusion start/numbers must both be given or both NULL");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    int rebuild = 0;
    if (forced_update) {
        rebuild = 1;
    } else if (nl->refresh_interval > 0 && !forced_check) {
        rebuild = (nl->refresh_count % nl->refresh_interval) == 0 || !nl->built ||
                  nl->needs_rebuild;
        nl->refresh_count += 1;
    } else if (!nl->built || nl->needs_rebuild) {
        rebuild = 1;
    } else {
        // skin check on the device; the host reads the flag (one small copy)
        int* flag = nl->meta + 2;
        SB_CHECK_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
        int tb = 128;
        // with a pruned list the outer list must hold every pair within cutoff + prune buffer,
        // so the skin left for motion is skin - prune_buffer
        const float hs = 0.5f * (nl->skin - nl->prune_buffer);
        k_refresh_check<<<(nl->n + tb - 1) / tb, tb, 0, s>>>(
            nl->n, d_crd, nl->old_crd, nl->box[0], nl->box[1], nl->box[2],
            nl->skin_permit * nl->skin_permit * hs * hs, flag);
        SB_CHECK_LAUNCH();
        int h = 0;
        SB_CHECK_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
        SB_CHECK_CUDA(cudaStreamSynchronize(s));
        rebuild = h;
    }
    if (rebuild) {
        SB_TRY(nl_rebuild(nl, d_crd, es, el, en, nullptr, s));
        nl->built = 1;
        nl->needs_rebuild = 0;
    } else if (nl->prune_buffer > 0.f && nl->prune_interval > 0 &&
               ++nl->prune_count >= nl->prune_interval) {
        SB_CHECK_CUDA(cudaMemsetAsync(nl->meta + 6, 1, sizeof(int), s));
        nl->prune_count = 0;
    }
    return SB_OK;
}

extern "C" int sb_nl_set_prune(sb_neighbor_list* nl, float prune_buffer, int prune_interval) {
    if (!nl || !(prune_buffer >= 0.f) || prune_buffer > nl->skin || prune_interval < 0) {
        sb_set_error("sb_nl_set_prune: buffer must be in [0, skin] and the interval >= 0");
        return SB_ERR_ARG;
    }
    cudaDeviceSynchronize();
    if (prune_buffer > 0.f) {
        if (!nl->cl_count_in) {
            SB_TRY(sb_malloc((void**)&nl->cl_count_in, sizeof(int) * nl->clu_cap,
                             "pruned counts"));
            SB_CHECK_CUDA(cudaMemset(nl->cl_count_in, 0, sizeof(int) * nl->clu_cap));
        }
        if (!nl->cl_ent_in)
            SB_TRY(sb_malloc((void**)&nl->cl_ent_in,
                             sizeof(uint32_t) * (size_t)nl->clu_cap * nl->ent_cap, "pruned list"));
        if (!nl->cl_ent_tmp)
            SB_TRY(sb_malloc((void**)&nl->cl_ent_tmp,
                             sizeof(uint32_t) * (size_t)nl->clu_cap * nl->ent_cap,
                             "prune scratch"));
        if (!nl->xq_prune) {
            SB_TRY(sb_malloc((void**)&nl->xq_prune, sizeof(uint4) * nl->slot_cap,
                             "prune coordinates"));
            SB_CHECK_CUDA(cudaMemset(nl->xq_prune, 0, sizeof(uint4) * nl->slot_cap));
        }
    }
    nl->prune_buffer = prune_buffer;
    nl->prune_interval = prune_interval;
    nl->prune_count = 0;
    // meta[6] = prune requested (the first pair launch builds the pruned list), meta[7] = 0
    SB_CHECK_CUDA(cudaMemset(nl->meta + 6, 0, 2 * sizeof(int)));
    if (prune_buffer > 0.f) SB_CHECK_CUDA(cudaMemset(nl->meta + 6, 1, 1));
    return SB_OK;
}

extern "C" int sb_nl_update_volume(sb_neighbor_list* nl, const float box_length[3]) {
    if (!nl || !box_length) {
        sb_set_error("sb_nl_update_volume: null argument");
        return SB_ERR_ARG;
    }
    for (int d = 0; d < 3; d++) {
        if (!(box_length[d] > 0.f)) {
            sb_set_error("sb_nl_update_volume: box lengths must be positive");
            return SB_ERR_ARG;
        }
    }
    for (int d = 0; d < 3; d++) nl->box[d] = box_length[d];
    // the column grid keeps its counts (as the reference keeps its cell counts); the widths
    // change, so the number of columns the search window spans is recomputed (a shrinking box
    // needs more of them). The capacities keep their sizes; an overflow at the new density sets
    // the status flags like any other.
    const double cwx = (double)nl->box[0] / nl->ncx, cwy = (double)nl->box[1] / nl->ncy;
    nl->nxr = (int)ceil(nl->cs / cwx);
    nl->nyr = (int)ceil(nl->cs / cwy);
    nl->needs_rebuild = 1;
    return SB_OK;
}

int sb_nl_ensure_built(sb_neighbor_list* nl) {
    if (!nl || !nl->built) {
        sb_set_error("neighbor list used before its first update");
        return SB_ERR_STATE;
    }
    return SB_OK;
}

int sb_nl_pack(sb_neighbor_list* nl, const uint32_t* d_uint_crd, const float* d_charge,
               const int* d_type, cudaStream_t s) {
    int tb = 256;
    const bool pr = nl->prune_buffer > 0.f;
    const float half = 0.5f * nl->prune_buffer;
    k_pack<<<(nl->slot_cap + tb - 1) / tb, tb, 0, s>>>(
        nl->meta, nl->slot_atom, d_uint_crd, d_charge, d_type, nl->xq, nl->stype,
        pr ? nl->xq_prune : nullptr, (1.0f / 4294967296.0f) * nl->box[0],
        (1.0f / 4294967296.0f) * nl->box[1], (1.0f / 4294967296.0f) * nl->box[2], half * half,
        nl->meta + 6, nl->slot_cap);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

__global__ void k_retire_prune(int* __restrict__ meta) {
    if (meta[7]) {
        meta[6] = 0;
        meta[7] = 0;
    }
}

// retires a prune request served by a pair launch that no k_finalize follows (timing runs)
int sb_nl_retire_prune(sb_neighbor_list* nl, cudaStream_t s) {
    if (nl->prune_buffer <= 0.f) return SB_OK;
    k_retire_prune<<<1, 1, 0, s>>>(nl->meta);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

int sb_nl_finalize_forces(sb_neighbor_list* nl, float* d_frc, cudaStream_t s) {
    int tb = 256;
    k_finalize<<<(nl->slot_cap + tb - 1) / tb, tb, 0, s>>>(nl->meta, nl->slot_atom, nl->fix,
                                                           nl->slot_cap, d_frc);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

int sb_nl_build_atom_group(sb_neighbor_list* nl, cudaStream_t s) {
    SB_TRY(sb_nl_ensure_built(nl));
    int n = nl->n;
    int set_ptr = 0;
    if (!nl->ag) {
        SB_TRY(sb_malloc(&nl->ag, sizeof(SbAtomGroup) * n, "ATOM_GROUP"));
        SB_TRY(sb_malloc((void**)&nl->ag_serial,
                         sizeof(int) * (size_t)n * nl->max_neighbor_numbers, "ATOM_GROUP serial"));
        set_ptr = 1;
    }
    if (nl->ag_valid) return SB_OK;
    int tb = 256;
    k_ag_reset<<<(n + tb - 1) / tb, tb, 0, s>>>(n, (SbAtomGroup*)nl->ag, nl->ag_serial,
                                                nl->max_neighbor_numbers, set_ptr);
    SB_CHECK_LAUNCH();
    k_ag_fill<<<nl->clu_cap, 128, 0, s>>>(nl->meta, nl->cl_count, nl->cl_ent, nl->ent_cap,
                                          nl->slot_atom, (SbAtomGroup*)nl->ag, nl->ag_serial,
                                          nl->max_neighbor_numbers, nl->meta);
    SB_CHECK_LAUNCH();
    k_ag_clamp<<<(n + tb - 1) / tb, tb, 0, s>>>(n, (SbAtomGroup*)nl->ag,
                                                nl->max_neighbor_numbers);
    SB_CHECK_LAUNCH();
    nl->ag_valid = 1;
    return SB_OK;
}

extern "C" int sb_nl_atom_group(sb_neighbor_list* nl, void** d_atom_group, void* stream) {
    if (!nl || !d_atom_group) {
        sb_set_error("sb_nl_atom_group: null argument");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_build_atom_group(nl, sb_stream(stream)));
    *d_atom_group = nl->ag;
    return SB_OK;
}

extern "C" int sb_nl_pair_count(sb_neighbor_list* nl, int64_t* h_count, void* stream) {
    if (!nl || !h_count) {
        sb_set_error("sb_nl_pair_count: null argument");
        return SB_ERR_ARG;
    }
    SB_TRY(sb_nl_ensure_built(nl));
    cudaStream_t s = sb_stream(stream);
    unsigned long long* d = (unsigned long long*)(nl->meta + 4);
    SB_CHECK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s));
    int tb = 256;
    k_count_pairs<<<(nl->clu_cap + tb - 1) / tb, tb, 0, s>>>(nl->meta, nl->cl_count, nl->cl_ent,
                                                             nl->ent_cap, d);
    SB_CHECK_LAUNCH();
    unsigned long long h = 0;
    SB_CHECK_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
    SB_CHECK_CUDA(cudaStreamSynchronize(s));
    *h_count = (int64_t)h;
    return SB_OK;
}

extern "C" int sb_nl_export_pairs(sb_neighbor_list* nl, int64_t* h_keys, int64_t cap,
                                  int64_t* h_count, void* stream) {
    if (!nl || !h_count) {
        sb_set_error("sb_nl_export_pairs: null argument");
        return SB_ERR_ARG;
    }
    int64_t cnt = 0;
    SB_TRY(sb_nl_pair_count(nl, &cnt, stream));
    *h_count = cnt;
    if (cnt > cap || (cnt > 0 && !h_keys)) {
        sb_set_error("sb_nl_export_pairs: capacity %lld < %lld pairs", (long long)cap,
                     (long long)cnt);
        return SB_ERR_OVERFLOW;
    }
    if (cnt == 0) return SB_OK;
    cudaStream_t s = sb_stream(stream);
    long long* d_keys = nullptr;
    SB_TRY(sb_malloc((void**)&d_keys, sizeof(long long) * cnt, "pair export"));
    unsigned long long* cur = (unsigned long long*)(nl->meta + 4);
    SB_CHECK_CUDA(cudaMemsetAsync(cur, 0, sizeof(unsigned long long), s));
    k_export_pairs<<<nl->clu_cap, 128, 0, s>>>(nl->n, nl->meta, nl->cl_count, nl->cl_ent,
                                               nl->ent_cap, nl->slot_atom, cur, d_keys, cnt);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_keys, d_keys, sizeof(long long) * cnt, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    sb_free(d_keys);
    if (e != cudaSuccess) {
        sb_set_error("sb_nl_export_pairs: %s", cudaGetErrorString(e));
        return SB_ERR_CUDA;
    }
    std::sort(h_keys, h_keys + cnt);
    return SB_OK;
}

extern "C" int sb_nl_status(sb_neighbor_list* nl, int* h_flags, void* stream) {
    if (!nl || !h_flags) {
        sb_set_error("sb_nl_status: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    int h = 0;
    SB_CHECK_CUDA(cudaMemcpyAsync(&h, nl->meta + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    SB_CHECK_CUDA(cudaMemsetAsync(nl->meta + 1, 0, sizeof(int), s));
    SB_CHECK_CUDA(cudaStreamSynchronize(s));
    *h_flags = h;
    return SB_OK;
}

extern "C" int sb_nl_uint_crd(sb_neighbor_list* nl, const uint32_t** d_uint_crd) {
    if (!nl || !d_uint_crd) {
        sb_set_error("sb_nl_uint_crd: null argument");
        return SB_ERR_ARG;
    }
    *d_uint_crd = nl->ucrd;
    return SB_OK;
}

extern "C" int sb_crd_to_uint_crd(int atom_numbers, const float box_length[3], const float* d_crd,
                                  uint32_t* d_uint_crd, void* stream) {
    if (atom_numbers <= 0 || !box_length || !d_crd || !d_uint_crd) {
        sb_set_error("sb_crd_to_uint_crd: invalid argument");
        return SB_ERR_ARG;
    }
    float c[3];
    for (int d = 0; d < 3; d++) c[d] = (0.25f * 4294967296.0f) / box_length[d];
    int tb = 256;
    k_crd_to_uint<<<(atom_numbers + tb - 1) / tb, tb, 0, sb_stream(stream)>>>(
        atom_numbers, d_crd, c[0], c[1], c[2], d_uint_crd);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

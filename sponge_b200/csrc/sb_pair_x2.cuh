// Fixed-point cluster pair kernel on packed FP32x2 arithmetic (chosen form) — included by
// sb_pair.cu after sb_pair_fixed.cuh.
//
// Same work decomposition as the eight-atoms-per-lane kernel (one warp per 8-atom i-cluster, one
// lane per list entry, j force out through three 64-bit fixed-point atomics, i forces reduced
// over the warp once per cluster), but the eight (i, j) slots of an entry are evaluated as four
// pairs of slots (i atoms 2p and 2p+1) on the sm_100 FP32x2 instructions (fma/mul/add .f32x2),
// which do two single-precision operations per issue slot. Per component each operation rounds
// exactly like its scalar counterpart; only the order of the j-force sum changes (even and odd
// i atoms summed separately, then added).
//
// The LJ coefficients of a slot pair come from a per-cluster table in shared memory built when
// the warp takes its cluster: row tj holds, for every i pair p, the float4 (-A(t_2p, tj),
// -A(t_2p+1, tj), B(t_2p, tj), B(t_2p+1, tj)), so one 16-byte load yields both slots' packed
// operands.
#pragma once

__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

__device__ __forceinline__ float sb_rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// -beta^3 G(z) on a pair of slots by the (5,4) rational of sb_ewald_G_rational (valid for
// z <= 9); gp holds the numerator coefficients pre-multiplied by beta^3, highest degree first
__device__ __forceinline__ float2 ewald_nG2(float2 z, const float* gp) {
    float2 p = f2(-gp[0]);
    p = f2fma(p, z, f2(-gp[1]));
    p = f2fma(p, z, f2(-gp[2]));
    p = f2fma(p, z, f2(-gp[3]));
    p = f2fma(p, z, f2(-gp[4]));
    p = f2fma(p, z, f2(-gp[5]));
    float2 q = f2(7.681388070e-04f);
    q = f2fma(q, z, f2(1.258269309e-02f));
    q = f2fma(q, z, f2(1.063599183e-01f));
    q = f2fma(q, z, f2(4.911114809e-01f));
    q = f2fma(q, z, f2(1.0f));
    return f2mul(p, make_float2(sb_rcp(q.x), sb_rcp(q.y)));
}

// Slot-pair patterns of a pruned entry: bit p is set when slot pair p (i atoms 2p and 2p + 1)
// has an active slot within the prune radius. A prune sorts each cluster's entries by the rank
// of their pattern, in the order below, so that entries needing the same slot pairs share the
// walk's batches of 32 and a batch more often has slot pairs that none of its entries needs,
// which the whole warp then skips. The order was found by a search over the patterns of the
// 96,000-atom solvated box's clusters (rc 10 A, prune radius 10.5 A): sorted, its batches
// evaluate 80.5 % of the slot pairs that unsorted batches do.
//   rank:    0  1  2  3  4  5  6   7   8   9  10  11  12  13  14
//   pattern: 1  3  2  6  7  5  9  13  15  11  10  14  12   4   8
// Nibble k of SB_PAT_RANK is the rank of pattern k (pattern 0, never kept, has rank 15).
#define SB_PAT_RANK 0x8b7c9a6e435d120full
#define SB_PAT_COUNTS 16
__device__ __forceinline__ int pat_rank(uint32_t mask8) {
    const uint32_t a = (mask8 | (mask8 >> 1)) & 0x55u;
    const uint32_t k = (a & 1u) | ((a >> 1) & 2u) | ((a >> 2) & 4u) | ((a >> 3) & 8u);
    return (int)((SB_PAT_RANK >> (4 * k)) & 15ull);
}

// Pruning pass over the full list of one cluster: keeps the entries with an active slot (mask
// bit set) whose r^2 — computed exactly as pair_walk_x2 computes it — is below
// (rc + prune buffer)^2, with the mask reduced to those slots, and writes them to `out` sorted by
// pattern rank (a counting sort: the kept entries go to `tmp` in list order while `rcnt`, 16 ints
// of the block's shared memory, counts the ranks; then they are scattered to their rank's range
// in list order, so the sorted list does not depend on the order of the counting atomics). Every slot the walk would find inside the cut-off before the next prune keeps its bit
// (an atom that moves more than half the buffer requests a prune), and the forces are
// fixed-point sums, so neither the dropped slots nor the order changes a bit. Returns the number
// kept.
template <bool EXACT>
__device__ __forceinline__ int prune_walk_x2(
    const PairParams& P, const int cnt, const uint32_t* __restrict__ ents,
    uint32_t* __restrict__ out, uint32_t* __restrict__ tmp, int* rcnt,
    const uint4* __restrict__ xq, const int base, const int lane, const uint32_t rx,
    const uint32_t ry, const uint32_t rz, const float2 (&nx)[4], const float2 (&ny)[4],
    const float2 (&nz)[4]) {
    const float2 rb2 = f2(P.rb2);
    const unsigned lt = (1u << lane) - 1u;
    if (lane < SB_PAT_COUNTS) rcnt[lane] = 0;
    __syncwarp();
    int kept = 0;
    // four batches of 32 entries per step, with the next step's entries loaded while this step's
    // j coordinates arrive: the test itself is short, so more loads are kept in flight than in
    // the walk (past the end an entry reads as 0: mask 0, never kept)
    constexpr int G = 4;
    uint32_t vn[G];
#pragma unroll
    for (int g = 0; g < G; g++) vn[g] = lane + 32 * g < cnt ? ents[lane + 32 * g] : 0u;
    for (int e0 = 0; e0 < cnt; e0 += 32 * G) {
        uint32_t v[G];
        uint4 xj[G];
#pragma unroll
        for (int g = 0; g < G; g++) {
            v[g] = vn[g];
            xj[g] = xq[v[g] & 0xffffffu];
        }
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int e = e0 + 32 * (G + g) + lane;
            vn[g] = e < cnt ? ents[e] : 0u;
        }
#pragma unroll
        for (int g = 0; g < G; g++) {
            const float2 xj2 = f2(__int2float_rn((int)(xj[g].x - rx)) * P.sx);
            const float2 yj2 = f2(__int2float_rn((int)(xj[g].y - ry)) * P.sy);
            const float2 zj2 = f2(__int2float_rn((int)(xj[g].z - rz)) * P.sz);
            uint32_t near = 0u;
#pragma unroll
            for (int p = 0; p < 4; p++) {
                float2 dx, dy, dz;
                if (EXACT) {
                    const uint4 xa = xq[base + 2 * p], xb = xq[base + 2 * p + 1];
                    dx = make_float2(__int2float_rn((int)(xj[g].x - xa.x)) * P.sx,
                                     __int2float_rn((int)(xj[g].x - xb.x)) * P.sx);
                    dy = make_float2(__int2float_rn((int)(xj[g].y - xa.y)) * P.sy,
                                     __int2float_rn((int)(xj[g].y - xb.y)) * P.sy);
                    dz = make_float2(__int2float_rn((int)(xj[g].z - xa.z)) * P.sz,
                                     __int2float_rn((int)(xj[g].z - xb.z)) * P.sz);
                } else {
                    dx = f2add(xj2, nx[p]);
                    dy = f2add(yj2, ny[p]);
                    dz = f2add(zj2, nz[p]);
                }
                const float2 r2 = f2fma(dx, dx, f2fma(dy, dy, f2mul(dz, dz)));
                near |= (r2.x < rb2.x ? 1u << (2 * p) : 0u) | (r2.y < rb2.y ? 2u << (2 * p) : 0u);
            }
            const uint32_t act = near & (v[g] >> 24);
            const bool keep = act != 0u;
            const unsigned b = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                tmp[kept + __popc(b & lt)] = (v[g] & 0xffffffu) | (act << 24);
                atomicAdd(&rcnt[pat_rank(act)], 1);
            }
            kept += __popc(b);
        }
    }
    __syncwarp();
    // each rank's first position, then the scatter (the entries of one rank keep their order);
    // the kept entries are read eight batches at a time, so that their loads overlap
    const int c = lane < SB_PAT_COUNTS ? rcnt[lane] : 0;
    int incl = c;
#pragma unroll
    for (int o = 1; o < SB_PAT_COUNTS; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    __syncwarp();
    if (lane < SB_PAT_COUNTS) rcnt[lane] = incl - c;
    __syncwarp();
    constexpr int S = 8;
    for (int e0 = 0; e0 < kept; e0 += 32 * S) {
        uint32_t vs[S];
#pragma unroll
        for (int g = 0; g < S; g++) {
            const int e = e0 + 32 * g + lane;
            vs[g] = e < kept ? __ldcg(tmp + e) : 0u;  // a kept entry is never 0 (mask != 0)
        }
#pragma unroll
        for (int g = 0; g < S; g++) {
            if (e0 + 32 * g >= kept) break;
            const bool valid = vs[g] != 0u;
            const int r = valid ? pat_rank(vs[g] >> 24) : SB_PAT_COUNTS;
            const unsigned grp = __match_any_sync(0xffffffffu, r);
            const int pos = valid ? rcnt[r] + __popc(grp & lt) : 0;
            __syncwarp();
            if (valid) {
                out[pos] = vs[g];
                if ((grp & lt) == 0u) rcnt[r] += __popc(grp);
            }
            __syncwarp();
        }
    }
    return kept;
}

template <int EV, bool EXACT>
__device__ __forceinline__ void pair_walk_x2(
    const PairParams& P, const int cnt, const uint32_t* __restrict__ ents,
    const uint4* __restrict__ xq, const int* __restrict__ stype, const float4* ctab,
    long long* __restrict__ fix, const int base, const int lane, const uint32_t rx,
    const uint32_t ry, const uint32_t rz, const float2 (&nx)[4], const float2 (&ny)[4],
    const float2 (&nz)[4], const float2 (&nq)[4], float2 (&fx)[4], float2 (&fy)[4],
    float2 (&fz)[4], float (&ei)[8], float (&vi)[8], float (&di)[8], uint32_t v1, uint32_t v2) {
    const float2 rc2 = f2(P.rc2);
    const float2 b2 = f2(P.beta2);
    // two-deep software pipeline as in the scalar kernel: entries two batches ahead (the first
    // two batches, v1 and v2, are loaded by the caller), j data one. Entries are read through L2
    // (ld.global.cg): a pruning launch reads the list it has just written.
    uint4 xj1 = xq[v1 & 0xffffffu];
    int tj1 = stype[v1 & 0xffffffu];
    for (int e0 = 0; e0 < cnt; e0 += 32) {
        const int e = e0 + lane;
        const bool valid = e < cnt;
        const uint32_t v = v1;
        const uint4 xj = xj1;
        const int tj = tj1;
        v1 = v2;
        v2 = e + 64 < cnt ? __ldcg(ents + e + 64) : 0u;
        xj1 = xq[v1 & 0xffffffu];
        tj1 = stype[v1 & 0xffffffu];
        const int j = (int)(v & 0xffffffu);
        const uint32_t m = v >> 24;
        // the slots that some entry of this batch uses
        const uint32_t mu = __reduce_or_sync(0xffffffffu, m);
        const float2 xj2 = f2(__int2float_rn((int)(xj.x - rx)) * P.sx);
        const float2 yj2 = f2(__int2float_rn((int)(xj.y - ry)) * P.sy);
        const float2 zj2 = f2(__int2float_rn((int)(xj.z - rz)) * P.sz);
        const float2 qj2 = f2(__uint_as_float(xj.w));
        const float4* trow = ctab + tj * 4;
        float2 gx = f2(0.f), gy = f2(0.f), gz = f2(0.f);
        // slot pair p of this lane's entry (a skipped pair would add exactly zero)
        auto slot_pair = [&](const int p) {
            float2 dx, dy, dz;
            if (EXACT) {
                const uint4 xa = xq[base + 2 * p], xb = xq[base + 2 * p + 1];
                dx = make_float2(__int2float_rn((int)(xj.x - xa.x)) * P.sx,
                                 __int2float_rn((int)(xj.x - xb.x)) * P.sx);
                dy = make_float2(__int2float_rn((int)(xj.y - xa.y)) * P.sy,
                                 __int2float_rn((int)(xj.y - xb.y)) * P.sy);
                dz = make_float2(__int2float_rn((int)(xj.z - xa.z)) * P.sz,
                                 __int2float_rn((int)(xj.z - xb.z)) * P.sz);
            } else {
                dx = f2add(xj2, nx[p]);
                dy = f2add(yj2, ny[p]);
                dz = f2add(zj2, nz[p]);
            }
            const float2 r2 = f2fma(dx, dx, f2fma(dy, dy, f2mul(dz, dz)));
            const bool a0 = (m & (1u << (2 * p))) != 0u && r2.x < rc2.x;
            const bool a1 = (m & (2u << (2 * p))) != 0u && r2.y < rc2.y;
            // evaluated on every slot and discarded by a select where inactive
            const float2 ri = make_float2(sb_rsqrt(r2.x), sb_rsqrt(r2.y));
            const float2 ri2 = f2mul(ri, ri);
            const float2 ri6 = f2mul(f2mul(ri2, ri2), ri2);
            const float4 t = trow[p];
            const float2 l = f2fma(make_float2(t.x, t.y), ri6, make_float2(t.z, t.w));
            const float2 flj = f2mul(l, f2mul(ri6, ri2));
            const float2 nqq = f2mul(nq[p], qj2);
            const float2 ngb = ewald_nG2(f2mul(b2, r2), P.gp);
            const float2 fs2 = f2fma(nqq, f2add(f2mul(ri, ri2), ngb), flj);
            const float2 fs = make_float2(a0 ? fs2.x : 0.f, a1 ? fs2.y : 0.f);
            fx[p] = f2fma(fs, dx, fx[p]);
            fy[p] = f2fma(fs, dy, fy[p]);
            fz[p] = f2fma(fs, dz, fz[p]);
            gx = f2fma(fs, dx, gx);
            gy = f2fma(fs, dy, gy);
            gz = f2fma(fs, dz, gz);
            if (EV) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const bool act = h ? a1 : a0;
                    if (act) {
                        const int k = 2 * p + h;
                        const float rr2 = h ? r2.y : r2.x, rri = h ? ri.y : ri.x;
                        const float rri6 = h ? ri6.y : ri6.x;
                        const float A = -(h ? t.y : t.x), B = h ? t.w : t.z;
                        const float qq = -(h ? nqq.y : nqq.x);
                        const float ec = qq * erfcf(P.beta * rr2 * rri) * rri;
                        if (EV & SB_EV_ENERGY)
                            ei[k] += (0.083333333f * A * rri6 - 0.166666667f * B) * rri6 + ec;
                        if (EV & SB_EV_VIRIAL) vi[k] -= (h ? flj.y : flj.x) * rr2;
                        di[k] += ec;
                    }
                }
            }
        };
        // a batch that uses every slot pair runs the four interleaved; otherwise the warp takes
        // only the pairs some entry uses (the prune sorts the entries to make such batches)
        const uint32_t need = (mu | (mu >> 1)) & 0x55u;
        if (need == 0x55u) {
#pragma unroll
            for (int p = 0; p < 4; p++) slot_pair(p);
        } else {
#pragma unroll
            for (int p = 0; p < 4; p++)
                if (need & (1u << (2 * p))) slot_pair(p);
        }
        if (valid) {
            add_fix(&fix[j], -(gx.x + gx.y));
            add_fix(&fix[P.slot_cap + j], -(gy.x + gy.y));
            add_fix(&fix[2 * P.slot_cap + j], -(gz.x + gz.y));
        }
    }
}

// one cluster c (the body of k_pair_x2)
template <int EV>
__device__ __forceinline__ void x2_cluster(
    const PairParams& P, const int c, const int lane, float4* ctab,
    const int* __restrict__ cl_count, const uint32_t* __restrict__ cl_ent,
    const uint4* __restrict__ xq, const int* __restrict__ stype, const float2* __restrict__ AB,
    const int* __restrict__ slot_atom, long long* __restrict__ fix,
    float* __restrict__ atom_energy, float* __restrict__ atom_virial,
    float* __restrict__ atom_direct) {
    const int base = c * SB_CLUSTER;
    // the loads that start a cluster are issued together: list counts (full and pruned), the
    // prune request, the cluster's atoms; then the first two batches of entries, which arrive
    // while the LJ table is built
    const bool pruned = P.rb2 > 0.f;
    const int req = pruned ? P.prune[0] : 0;
    int cntf = cl_count[c];
    const int cntf_in = pruned ? P.cl_count_in[c] : 0;
    const uint4 my = lane < SB_CLUSTER ? xq[base + lane] : make_uint4(0, 0, 0, 0);
    const int myt = lane < SB_CLUSTER ? stype[base + lane] : 0;
    const uint32_t* ents = cl_ent + (size_t)c * P.ent_cap;
    uint32_t* in_ents = pruned ? P.cl_ent_in + (size_t)c * P.ent_cap : nullptr;
    if (pruned && !req) {
        cntf = cntf_in;
        ents = in_ents;
    }
    int cnt = min(cntf & SB_CL_COUNT_MASK, P.ent_cap);
    uint32_t v1 = 0u, v2 = 0u;
    if (!req) {
        v1 = lane < cnt ? __ldcg(ents + lane) : 0u;
        v2 = lane + 32 < cnt ? __ldcg(ents + lane + 32) : 0u;
    }
    // cluster LJ table: entry (tj, p) = (-A(t_2p,tj), -A(t_2p+1,tj), B(t_2p,tj), B(t_2p+1,tj))
    const int nt = P.nt;
    {
        // lane l always serves pair p = l & 3, so its two i types are fetched once
        const int p = lane & 3;
        const int ta = __shfl_sync(0xffffffffu, myt, 2 * p) * nt;
        const int tb = __shfl_sync(0xffffffffu, myt, 2 * p + 1) * nt;
        for (int t = lane; t < 4 * nt; t += 32) {
            const int tj = t >> 2;
            const float2 a = AB[ta + tj], b = AB[tb + tj];
            ctab[t] = make_float4(-a.x, -b.x, a.y, b.y);
        }
    }
    const uint32_t rx = __shfl_sync(0xffffffffu, my.x, 0);
    const uint32_t ry = __shfl_sync(0xffffffffu, my.y, 0);
    const uint32_t rz = __shfl_sync(0xffffffffu, my.z, 0);
    const float mxr = __int2float_rn((int)(my.x - rx)) * P.sx;
    const float myr = __int2float_rn((int)(my.y - ry)) * P.sy;
    const float mzr = __int2float_rn((int)(my.z - rz)) * P.sz;
    const float mq = __uint_as_float(my.w);
    float2 nx[4], ny[4], nz[4], nq[4], fx[4], fy[4], fz[4];
    float ei[8], vi[8], di[8];
#pragma unroll
    for (int p = 0; p < 4; p++) {
        nx[p] = make_float2(-__shfl_sync(0xffffffffu, mxr, 2 * p),
                            -__shfl_sync(0xffffffffu, mxr, 2 * p + 1));
        ny[p] = make_float2(-__shfl_sync(0xffffffffu, myr, 2 * p),
                            -__shfl_sync(0xffffffffu, myr, 2 * p + 1));
        nz[p] = make_float2(-__shfl_sync(0xffffffffu, mzr, 2 * p),
                            -__shfl_sync(0xffffffffu, mzr, 2 * p + 1));
        nq[p] = make_float2(-__shfl_sync(0xffffffffu, mq, 2 * p),
                            -__shfl_sync(0xffffffffu, mq, 2 * p + 1));
        fx[p] = fy[p] = fz[p] = f2(0.f);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) ei[k] = vi[k] = di[k] = 0.f;
    __syncwarp();

    if (req) {
        // pruned list: rebuilt from the full list on request, then walked as in the other
        // launches, so the forces do not depend on whether this launch pruned
        uint32_t* tmp = P.cl_ent_tmp + (size_t)c * P.ent_cap;
        int* rcnt = (int*)(ctab + 4 * nt);
        cnt = (cntf & SB_CL_EXACT)
                  ? prune_walk_x2<true>(P, cnt, ents, in_ents, tmp, rcnt, xq, base, lane, rx, ry,
                                        rz, nx, ny, nz)
                  : prune_walk_x2<false>(P, cnt, ents, in_ents, tmp, rcnt, xq, base, lane, rx, ry,
                                         rz, nx, ny, nz);
        if (lane == 0) {
            P.cl_count_in[c] = cnt | (cntf & ~SB_CL_COUNT_MASK);
            if (c == 0) P.prune[1] = 1;  // k_finalize retires the request
        }
        if (lane < SB_CLUSTER) P.xq_prune[base + lane] = my;
        __syncwarp();
        ents = in_ents;
        v1 = lane < cnt ? __ldcg(ents + lane) : 0u;
        v2 = lane + 32 < cnt ? __ldcg(ents + lane + 32) : 0u;
    }
    if (cntf & SB_CL_EXACT)
        pair_walk_x2<EV, true>(P, cnt, ents, xq, stype, ctab, fix, base, lane, rx, ry, rz, nx, ny,
                               nz, nq, fx, fy, fz, ei, vi, di, v1, v2);
    else
        pair_walk_x2<EV, false>(P, cnt, ents, xq, stype, ctab, fix, base, lane, rx, ry, rz, nx,
                                ny, nz, nq, fx, fy, fz, ei, vi, di, v1, v2);

    // i forces: transpose-reduce the 24 per-lane sums (x, y, z of 8 atoms, padded to 32) over the
    // warp; each of the 5 steps halves the values a lane holds, after which lane l holds the
    // total of value l (component l / 8 of cluster slot l % 8): 31 shuffles instead of 120
    float v[32];
#pragma unroll
    for (int p = 0; p < 4; p++) {
        v[2 * p] = fx[p].x, v[2 * p + 1] = fx[p].y;
        v[8 + 2 * p] = fy[p].x, v[9 + 2 * p] = fy[p].y;
        v[16 + 2 * p] = fz[p].x, v[17 + 2 * p] = fz[p].y;
    }
#pragma unroll
    for (int k = 24; k < 32; k++) v[k] = 0.f;
#pragma unroll
    for (int o = 16, n = 16; o >= 1; o >>= 1, n >>= 1) {
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < n; k++) {
            const float send = upper ? v[k] : v[k + n];
            const float keep = upper ? v[k + n] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    if (lane < 24) {
        const int k = lane & 7, comp = lane >> 3;
        if (slot_atom[base + k] >= 0) red_fix(&fix[(size_t)comp * P.slot_cap + base + k], v[0]);
    }
    if (EV) {
        // energy and virial terms (energy/virial steps only): butterfly sums, lane 0 writes
#pragma unroll
        for (int k = 0; k < 8; k++) {
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) {
                ei[k] += __shfl_xor_sync(0xffffffffu, ei[k], o);
                vi[k] += __shfl_xor_sync(0xffffffffu, vi[k], o);
                di[k] += __shfl_xor_sync(0xffffffffu, di[k], o);
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int a = slot_atom[base + k];
                if (a >= 0) {
                    if (EV & SB_EV_ENERGY) atom_energy[a] += ei[k];
                    if (EV & SB_EV_VIRIAL) {
                        atom_virial[a] += vi[k];
                        atom_direct[a] = di[k];
                    }
                }
            }
        }
    }
}

// One-warp blocks; a block takes clusters blockIdx.x, blockIdx.x + gridDim.x, ... (one each when
// the grid has a block per cluster). The force-only form is held to 80 registers (24 blocks per
// SM): 85 us against 88 us at 128 registers on the 96k-atom box, for a few spilled bytes outside
// the pair loop. Every cluster's forces go to fixed-point accumulators and
// its energies to its own atoms, so the assignment does not change a bit. Dynamic shared memory:
// the cluster's LJ table, 4 nt float4, then the prune's SB_PAT_COUNTS rank counts.
template <int EV>
__global__ void __launch_bounds__(32, EV ? 12 : 24) k_pair_x2(
    PairParams P, const int* __restrict__ meta, const int* __restrict__ cl_count,
    const uint32_t* __restrict__ cl_ent, const uint4* __restrict__ xq,
    const int* __restrict__ stype, const float2* __restrict__ AB,
    const int* __restrict__ slot_atom, long long* __restrict__ fix,
    float* __restrict__ atom_energy, float* __restrict__ atom_virial,
    float* __restrict__ atom_direct) {
    extern __shared__ float4 ctab[];
    const int lane = threadIdx.x & 31;
    const int ncl = meta[0];
    for (int c = blockIdx.x; c < ncl; c += gridDim.x) {
        x2_cluster<EV>(P, c, lane, ctab, cl_count, cl_ent, xq, stype, AB, slot_atom, fix,
                       atom_energy, atom_virial, atom_direct);
        __syncwarp();  // the next cluster rewrites the LJ table
    }
}


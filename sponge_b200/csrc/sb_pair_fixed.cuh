// Fixed-point cluster pair kernel (chosen form) — included by sb_pair.cu.
//
// One warp per 8-atom i-cluster. LPE = 8 / IPL lanes share one list entry (a j atom plus the
// 8-bit mask of i atoms it pairs with); lane h of the LPE handles i atoms [h*IPL, h*IPL+IPL),
// held in registers for the whole list walk. IPL = 8 keeps one lane per entry; IPL = 4 halves
// the per-lane register state (two lanes per entry, roughly twice the resident warps) at the
// cost of converting each j twice and one shuffle per force component per entry. Positions
// are relative to the cluster's first atom (exact integer difference, one float conversion
// per j). The j force is complete after the i loop and leaves as three 64-bit fixed-point
// atomics; i forces are reduced across the warp once per cluster.
#pragma once

template <int IPL>
struct PairLane {
    static constexpr int LPE = SB_CLUSTER / IPL;  // lanes per entry
    static constexpr int EPW = 32 / LPE;          // entries per warp iteration
};

template <int EV, bool EXACT, int IPL, bool WIDE>
__device__ __forceinline__ void pair_walk(
    const PairParams& P, const int cnt, const uint32_t* __restrict__ ents,
    const uint4* __restrict__ xq, const int* __restrict__ stype, const float2* sAB,
    long long* __restrict__ fix, const int base, const int h, const int eslot,
    const uint32_t rx, const uint32_t ry, const uint32_t rz, const float (&xi)[IPL],
    const float (&yi)[IPL], const float (&zi)[IPL], const float (&qi)[IPL],
    const int (&ti)[IPL], float (&fxi)[IPL], float (&fyi)[IPL], float (&fzi)[IPL],
    float (&ei)[IPL], float (&vi)[IPL], float (&di)[IPL]) {
    constexpr int LPE = PairLane<IPL>::LPE;
    constexpr int EPW = PairLane<IPL>::EPW;
    // two-deep software pipeline: list entries are loaded two batches ahead (a DRAM stream) and
    // the j coordinates/types one batch ahead (L1/L2 gathers), so their latency overlaps the
    // current batch's arithmetic. Past the end v = 0: j = 0 (a valid slot) and an empty mask.
    uint32_t v1 = eslot < cnt ? ents[eslot] : 0u;
    uint32_t v2 = eslot + EPW < cnt ? ents[eslot + EPW] : 0u;
    uint4 xj1 = xq[v1 & 0xffffffu];
    int tj1 = stype[v1 & 0xffffffu];
    // warp-uniform trip count so that the lanes of one entry stay converged for the shuffles
    for (int e0 = 0; e0 < cnt; e0 += EPW) {
        const int e = e0 + eslot;
        const bool valid = e < cnt;
        const uint32_t v = v1;
        const uint4 xj = xj1;
        const int tj = tj1;
        v1 = v2;
        v2 = e + 2 * EPW < cnt ? ents[e + 2 * EPW] : 0u;
        xj1 = xq[v1 & 0xffffffu];
        tj1 = stype[v1 & 0xffffffu];
        const int j = (int)(v & 0xffffffu);
        const uint32_t m = (v >> 24) >> (h * IPL);
        const float xjr = __int2float_rn((int)(xj.x - rx)) * P.sx;
        const float yjr = __int2float_rn((int)(xj.y - ry)) * P.sy;
        const float zjr = __int2float_rn((int)(xj.z - rz)) * P.sz;
        const float qj = __uint_as_float(xj.w);
        float fjx = 0.f, fjy = 0.f, fjz = 0.f;
#pragma unroll
        for (int k = 0; k < IPL; k++) {
            float dx, dy, dz;
            if (EXACT) {
                const uint4 xk = xq[base + h * IPL + k];
                dx = __int2float_rn((int)(xj.x - xk.x)) * P.sx;
                dy = __int2float_rn((int)(xj.y - xk.y)) * P.sy;
                dz = __int2float_rn((int)(xj.z - xk.z)) * P.sz;
            } else {
                dx = xjr - xi[k];
                dy = yjr - yi[k];
                dz = zjr - zi[k];
            }
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool act = ((m >> k) & 1u) && r2 < P.rc2;
            // evaluated for every lane and discarded by a select where inactive (r2 may be 0
            // there, so a select, not a multiply, removes the non-finite values)
            const float ri = sb_rsqrt(r2);
            const float ri2 = ri * ri;
            const float ri6 = ri2 * ri2 * ri2;
            const float2 ab = sAB[ti[k] + tj];
            const float flj = (ab.y - ab.x * ri6) * (ri6 * ri2);
            const float qq = qi[k] * qj;
            const float bg = WIDE ? sb_ewald_G_scaled(P.beta2 * r2, P.gp)
                                  : sb_ewald_G_rational(P.beta2 * r2, P.gp);
            const float fc = qq * (ri * ri2 - bg);
            const float fs = act ? flj - fc : 0.f;
            fxi[k] = fmaf(fs, dx, fxi[k]);
            fyi[k] = fmaf(fs, dy, fyi[k]);
            fzi[k] = fmaf(fs, dz, fzi[k]);
            fjx = fmaf(-fs, dx, fjx);
            fjy = fmaf(-fs, dy, fjy);
            fjz = fmaf(-fs, dz, fjz);
            if (EV && act) {
                const float ec = qq * erfcf(P.beta * r2 * ri) * ri;
                if (EV & SB_EV_ENERGY)
                    ei[k] += (0.083333333f * ab.x * ri6 - 0.166666667f * ab.y) * ri6 + ec;
                if (EV & SB_EV_VIRIAL) vi[k] -= flj * r2;
                di[k] += ec;
            }
        }
        if (LPE == 2) {
            fjx += __shfl_xor_sync(0xffffffffu, fjx, 1);
            fjy += __shfl_xor_sync(0xffffffffu, fjy, 1);
            fjz += __shfl_xor_sync(0xffffffffu, fjz, 1);
        }
        if (valid && h == 0) {
            add_fix(&fix[j], fjx);
            add_fix(&fix[P.slot_cap + j], fjy);
            add_fix(&fix[2 * P.slot_cap + j], fjz);
        }
    }
}

// One-warp blocks: a block's slot frees as soon as its cluster is done (no waiting on a slower
// sibling warp), which also lets the reciprocal kernels of the side stream interleave. Force-only
// launches are capped at 96 registers (20 warps per SM; the few spills cost less than the
// occupancy gains), energy/virial launches at 128 (16 warps).
template <int EV, int IPL>
__global__ void __launch_bounds__(32, EV ? 16 : 20) k_pair_fixed(
    PairParams P, const int* __restrict__ meta, const int* __restrict__ cl_count,
    const uint32_t* __restrict__ cl_ent, const uint4* __restrict__ xq,
    const int* __restrict__ stype, const float2* __restrict__ AB,
    const int* __restrict__ slot_atom, long long* __restrict__ fix,
    float* __restrict__ atom_energy, float* __restrict__ atom_virial,
    float* __restrict__ atom_direct) {
    constexpr int LPE = PairLane<IPL>::LPE;
    extern __shared__ float2 sAB[];
    const int ntt = P.nt * P.nt;
    for (int t = threadIdx.x; t < ntt; t += blockDim.x) sAB[t] = AB[t];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= meta[0]) return;
    const int base = c * SB_CLUSTER;
    const int h = lane % LPE, eslot = lane / LPE;

    const uint4 my = lane < SB_CLUSTER ? xq[base + lane] : make_uint4(0, 0, 0, 0);
    const int myt = lane < SB_CLUSTER ? stype[base + lane] : 0;
    const uint32_t rx = __shfl_sync(0xffffffffu, my.x, 0);
    const uint32_t ry = __shfl_sync(0xffffffffu, my.y, 0);
    const uint32_t rz = __shfl_sync(0xffffffffu, my.z, 0);
    const float mxr = __int2float_rn((int)(my.x - rx)) * P.sx;
    const float myr = __int2float_rn((int)(my.y - ry)) * P.sy;
    const float mzr = __int2float_rn((int)(my.z - rz)) * P.sz;

    float xi[IPL], yi[IPL], zi[IPL], qi[IPL];
    int ti[IPL];
    float fxi[IPL], fyi[IPL], fzi[IPL], ei[IPL], vi[IPL], di[IPL];
#pragma unroll
    for (int k = 0; k < IPL; k++) {
        const int src = h * IPL + k;
        xi[k] = __shfl_sync(0xffffffffu, mxr, src);
        yi[k] = __shfl_sync(0xffffffffu, myr, src);
        zi[k] = __shfl_sync(0xffffffffu, mzr, src);
        qi[k] = __uint_as_float(__shfl_sync(0xffffffffu, my.w, src));
        ti[k] = __shfl_sync(0xffffffffu, myt, src) * P.nt;
        fxi[k] = fyi[k] = fzi[k] = 0.f;
        ei[k] = vi[k] = di[k] = 0.f;
    }

    const int cntf = cl_count[c];
    const int cnt = min(cntf & SB_CL_COUNT_MASK, P.ent_cap);
    const uint32_t* ents = cl_ent + (size_t)c * P.ent_cap;
    // (beta rc)^2 > 12 ("wide") needs the exact Ewald expression beyond the fitted range; the
    // common case runs the branch-free rational so the IPL pair chains interleave
    if (P.wide) {
        if (cntf & SB_CL_EXACT)
            pair_walk<EV, true, IPL, true>(P, cnt, ents, xq, stype, sAB, fix, base, h, eslot, rx,
                                           ry, rz, xi, yi, zi, qi, ti, fxi, fyi, fzi, ei, vi, di);
        else
            pair_walk<EV, false, IPL, true>(P, cnt, ents, xq, stype, sAB, fix, base, h, eslot, rx,
                                            ry, rz, xi, yi, zi, qi, ti, fxi, fyi, fzi, ei, vi, di);
    } else {
        if (cntf & SB_CL_EXACT)
            pair_walk<EV, true, IPL, false>(P, cnt, ents, xq, stype, sAB, fix, base, h, eslot, rx,
                                            ry, rz, xi, yi, zi, qi, ti, fxi, fyi, fzi, ei, vi, di);
        else
            pair_walk<EV, false, IPL, false>(P, cnt, ents, xq, stype, sAB, fix, base, h, eslot,
                                             rx, ry, rz, xi, yi, zi, qi, ti, fxi, fyi, fzi, ei, vi,
                                             di);
    }

    // reduce over the lanes that hold the same i atoms (same h); lanes 0..LPE-1 end with totals
#pragma unroll
    for (int k = 0; k < IPL; k++) {
#pragma unroll
        for (int o = 16; o >= LPE; o >>= 1) {
            fxi[k] += __shfl_xor_sync(0xffffffffu, fxi[k], o);
            fyi[k] += __shfl_xor_sync(0xffffffffu, fyi[k], o);
            fzi[k] += __shfl_xor_sync(0xffffffffu, fzi[k], o);
            if (EV) {
                ei[k] += __shfl_xor_sync(0xffffffffu, ei[k], o);
                vi[k] += __shfl_xor_sync(0xffffffffu, vi[k], o);
                di[k] += __shfl_xor_sync(0xffffffffu, di[k], o);
            }
        }
    }
    if (lane < LPE) {
#pragma unroll
        for (int k = 0; k < IPL; k++) {
            const int s = base + h * IPL + k;
            const int a = slot_atom[s];
            if (a >= 0) {
                red_fix(&fix[s], fxi[k]);
                red_fix(&fix[P.slot_cap + s], fyi[k]);
                red_fix(&fix[2 * P.slot_cap + s], fzi[k]);
                if (EV & SB_EV_ENERGY) atom_energy[a] += ei[k];
                if (EV & SB_EV_VIRIAL) {
                    atom_virial[a] += vi[k];
                    atom_direct[a] = di[k];
                }
            }
        }
    }
}

// Compacted cluster pair kernel (chosen form) — included by sb_pair.cu after sb_pair_fixed.cuh.
//
// One warp per 8-atom i-cluster, one lane per list entry (j atom + 8-bit i mask), batches of 32
// entries. The list holds pairs within rc + skin, so only ~40% of the 8 x 32 (i, j) slots of a
// batch are inside rc; evaluating the full LJ + Ewald expression on every slot (the IPL kernels)
// wastes most of the issue slots. Here each batch runs three phases over per-warp shared memory:
//   A  filter: every lane tests its 8 slots (relative-frame distance, in-cutoff test) and stages
//      {dx, dy, dz, r^2} of the in-cutoff ones at position k*32 + lane (consecutive lanes hit
//      consecutive shared-memory words); a warp prefix sum of the per-lane counts gives a dense
//      map of the staged pairs;
//   B  evaluate: all 32 lanes walk the dense map, one pair per lane, and overwrite r^2 with the
//      force factor F/r (energies and virial into side arrays on energy/virial steps);
//   C  accumulate: every lane sums its own entry's pairs in k order into the j force (three
//      64-bit fixed-point atomics) and into per-lane i-force registers, reduced over the warp
//      once per cluster.
// Every sum runs in an order fixed by the list, so forces stay bit-identical run to run.
#pragma once

#define SB_CP_WARPS 4
#define SB_CP_SLOTS (32 * SB_CLUSTER)

template <int EV>
struct CompactSmem {
    float4 stage[SB_CP_WARPS][SB_CP_SLOTS];
    unsigned char pmap[SB_CP_WARPS][SB_CP_SLOTS];
    float qj[SB_CP_WARPS][32];
    int tj[SB_CP_WARPS][32];
    float qi[SB_CP_WARPS][SB_CLUSTER];
    int ti[SB_CP_WARPS][SB_CLUSTER];
    float e[EV ? SB_CP_WARPS : 1][EV ? SB_CP_SLOTS : 1];
    float v[EV ? SB_CP_WARPS : 1][EV ? SB_CP_SLOTS : 1];
    float d[EV ? SB_CP_WARPS : 1][EV ? SB_CP_SLOTS : 1];
};

template <int EV, bool EXACT, bool WIDE>
__device__ __forceinline__ void compact_walk(
    const PairParams& P, const int cnt, const uint32_t* __restrict__ ents,
    const uint4* __restrict__ xq, const int* __restrict__ stype, const float2* sAB,
    long long* __restrict__ fix, const int base, const int lane, const uint32_t rx,
    const uint32_t ry, const uint32_t rz, const float (&xi)[SB_CLUSTER],
    const float (&yi)[SB_CLUSTER], const float (&zi)[SB_CLUSTER], CompactSmem<EV>& S,
    const int w, float (&fxi)[SB_CLUSTER], float (&fyi)[SB_CLUSTER], float (&fzi)[SB_CLUSTER],
    float (&ei)[SB_CLUSTER], float (&vi)[SB_CLUSTER], float (&di)[SB_CLUSTER]) {
    float4* stage = S.stage[w];
    unsigned char* pmap = S.pmap[w];
    for (int e0 = 0; e0 < cnt; e0 += 32) {
        // ---- A: filter and stage ----
        const int e = e0 + lane;
        const bool valid = e < cnt;
        const uint32_t v = valid ? ents[e] : 0u;
        const int j = (int)(v & 0xffffffu);
        const uint32_t m = v >> 24;
        const uint4 xj = xq[j];
        S.qj[w][lane] = __uint_as_float(xj.w);
        S.tj[w][lane] = stype[j];
        const float xjr = __int2float_rn((int)(xj.x - rx)) * P.sx;
        const float yjr = __int2float_rn((int)(xj.y - ry)) * P.sy;
        const float zjr = __int2float_rn((int)(xj.z - rz)) * P.sz;
        uint32_t am = 0;
#pragma unroll
        for (int k = 0; k < SB_CLUSTER; k++) {
            float dx, dy, dz;
            if (EXACT) {
                const uint4 xk = xq[base + k];
                dx = __int2float_rn((int)(xj.x - xk.x)) * P.sx;
                dy = __int2float_rn((int)(xj.y - xk.y)) * P.sy;
                dz = __int2float_rn((int)(xj.z - xk.z)) * P.sz;
            } else {
                dx = xjr - xi[k];
                dy = yjr - yi[k];
                dz = zjr - zi[k];
            }
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (((m >> k) & 1u) && r2 < P.rc2) {
                stage[k * 32 + lane] = make_float4(dx, dy, dz, r2);
                am |= 1u << k;
            }
        }
        const int c = __popc(am);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int n = __shfl_sync(0xffffffffu, incl, 31);
        {
            uint32_t mm = am;
            int r = incl - c;
            while (mm) {
                const int k = __ffs(mm) - 1;
                pmap[r++] = (unsigned char)(k * 32 + lane);
                mm &= mm - 1u;
            }
        }
        __syncwarp();
        // ---- B: one in-cutoff pair per lane ----
        for (int p = lane; p < n; p += 32) {
            const int code = pmap[p];
            const int l = code & 31, k = code >> 5;
            const float4 d = stage[code];
            const float r2 = d.w;
            const float ri = rsqrtf(r2);
            const float ri2 = ri * ri;
            const float ri6 = ri2 * ri2 * ri2;
            const float2 ab = sAB[S.ti[w][k] + S.tj[w][l]];
            const float flj = (ab.y - ab.x * ri6) * (ri6 * ri2);
            const float qq = S.qi[w][k] * S.qj[w][l];
            const float bg = WIDE ? sb_ewald_G_scaled(P.beta2 * r2, P.gp)
                                  : sb_ewald_G_rational(P.beta2 * r2, P.gp);
            const float fc = qq * (ri * ri2 - bg);
            reinterpret_cast<float*>(stage)[4 * code + 3] = flj - fc;
            if (EV) {
                const float ec = qq * erfcf(P.beta * r2 * ri) * ri;
                S.e[w][code] = (0.083333333f * ab.x * ri6 - 0.166666667f * ab.y) * ri6 + ec;
                S.v[w][code] = -flj * r2;
                S.d[w][code] = ec;
            }
        }
        __syncwarp();
        // ---- C: accumulate this lane's entry in k order ----
        if (am) {
            float fjx = 0.f, fjy = 0.f, fjz = 0.f;
#pragma unroll
            for (int k = 0; k < SB_CLUSTER; k++) {
                if ((am >> k) & 1u) {
                    const int code = k * 32 + lane;
                    const float4 t = stage[code];
                    const float fs = t.w;
                    fxi[k] = fmaf(fs, t.x, fxi[k]);
                    fyi[k] = fmaf(fs, t.y, fyi[k]);
                    fzi[k] = fmaf(fs, t.z, fzi[k]);
                    fjx = fmaf(-fs, t.x, fjx);
                    fjy = fmaf(-fs, t.y, fjy);
                    fjz = fmaf(-fs, t.z, fjz);
                    if (EV & SB_EV_ENERGY) ei[k] += S.e[w][code];
                    if (EV & SB_EV_VIRIAL) vi[k] += S.v[w][code];
                    if (EV) di[k] += S.d[w][code];
                }
            }
            red_fix(&fix[j], fjx);
            red_fix(&fix[P.slot_cap + j], fjy);
            red_fix(&fix[2 * P.slot_cap + j], fjz);
        }
        __syncwarp();
    }
}

template <int EV>
__global__ void __launch_bounds__(32 * SB_CP_WARPS) k_pair_compact(
    PairParams P, const int* __restrict__ meta, const int* __restrict__ cl_count,
    const uint32_t* __restrict__ cl_ent, const uint4* __restrict__ xq,
    const int* __restrict__ stype, const float2* __restrict__ AB,
    const int* __restrict__ slot_atom, long long* __restrict__ fix,
    float* __restrict__ atom_energy, float* __restrict__ atom_virial,
    float* __restrict__ atom_direct) {
    extern __shared__ float2 sAB[];
    __shared__ CompactSmem<EV> S;
    const int ntt = P.nt * P.nt;
    for (int t = threadIdx.x; t < ntt; t += blockDim.x) sAB[t] = AB[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int c = blockIdx.x * SB_CP_WARPS + w;
    if (c >= meta[0]) return;
    const int base = c * SB_CLUSTER;
    const uint4 my = lane < SB_CLUSTER ? xq[base + lane] : make_uint4(0, 0, 0, 0);
    const int myt = lane < SB_CLUSTER ? stype[base + lane] : 0;
    if (lane < SB_CLUSTER) {
        S.qi[w][lane] = __uint_as_float(my.w);
        S.ti[w][lane] = myt * P.nt;
    }
    const uint32_t rx = __shfl_sync(0xffffffffu, my.x, 0);
    const uint32_t ry = __shfl_sync(0xffffffffu, my.y, 0);
    const uint32_t rz = __shfl_sync(0xffffffffu, my.z, 0);
    const float mxr = __int2float_rn((int)(my.x - rx)) * P.sx;
    const float myr = __int2float_rn((int)(my.y - ry)) * P.sy;
    const float mzr = __int2float_rn((int)(my.z - rz)) * P.sz;
    float xi[SB_CLUSTER], yi[SB_CLUSTER], zi[SB_CLUSTER];
    float fxi[SB_CLUSTER], fyi[SB_CLUSTER], fzi[SB_CLUSTER];
    float ei[SB_CLUSTER], vi[SB_CLUSTER], di[SB_CLUSTER];
#pragma unroll
    for (int k = 0; k < SB_CLUSTER; k++) {
        xi[k] = __shfl_sync(0xffffffffu, mxr, k);
        yi[k] = __shfl_sync(0xffffffffu, myr, k);
        zi[k] = __shfl_sync(0xffffffffu, mzr, k);
        fxi[k] = fyi[k] = fzi[k] = 0.f;
        ei[k] = vi[k] = di[k] = 0.f;
    }
    __syncwarp();
    const int cntf = cl_count[c];
    const int cnt = min(cntf & SB_CL_COUNT_MASK, P.ent_cap);
    const uint32_t* ents = cl_ent + (size_t)c * P.ent_cap;
    if (P.wide) {
        if (cntf & SB_CL_EXACT)
            compact_walk<EV, true, true>(P, cnt, ents, xq, stype, sAB, fix, base, lane, rx, ry,
                                         rz, xi, yi, zi, S, w, fxi, fyi, fzi, ei, vi, di);
        else
            compact_walk<EV, false, true>(P, cnt, ents, xq, stype, sAB, fix, base, lane, rx, ry,
                                          rz, xi, yi, zi, S, w, fxi, fyi, fzi, ei, vi, di);
    } else {
        if (cntf & SB_CL_EXACT)
            compact_walk<EV, true, false>(P, cnt, ents, xq, stype, sAB, fix, base, lane, rx, ry,
                                          rz, xi, yi, zi, S, w, fxi, fyi, fzi, ei, vi, di);
        else
            compact_walk<EV, false, false>(P, cnt, ents, xq, stype, sAB, fix, base, lane, rx, ry,
                                           rz, xi, yi, zi, S, w, fxi, fyi, fzi, ei, vi, di);
    }
    // i forces: butterfly over the warp (every lane ends with the totals); lane k writes atom k
#pragma unroll
    for (int k = 0; k < SB_CLUSTER; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            fxi[k] += __shfl_xor_sync(0xffffffffu, fxi[k], o);
            fyi[k] += __shfl_xor_sync(0xffffffffu, fyi[k], o);
            fzi[k] += __shfl_xor_sync(0xffffffffu, fzi[k], o);
            if (EV) {
                ei[k] += __shfl_xor_sync(0xffffffffu, ei[k], o);
                vi[k] += __shfl_xor_sync(0xffffffffu, vi[k], o);
                di[k] += __shfl_xor_sync(0xffffffffu, di[k], o);
            }
        }
        if (lane == k) {
            const int s = base + k;
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

// Integrator + rigid-water constraints behind the force graph: the NVE leap-frog of
// MD_INFORMATION (SPONGE/MD_core/MD_core.cu:13-32, :1535-1547) and SETTLE
// (SPONGE/constrain/SETTLE.cu), in the order Main_Iteration runs them (SPONGE/main.cu:283-325:
// Remember_Last_Coordinates, Leap_Frog, Do_SETTLE).
//
// B200 design: every atom is written by exactly one thread, so the step needs no atomics and
// is deterministic. The fused step is one launch: threads [0, T) each take a rigid triangle
// (remember its edge vectors from the fixed-point coordinates of the step start, leap-frog its
// three atoms, SETTLE them), threads [T, T+P) a rigid pair, the rest one unconstrained atom
// (leap-frog only). The separate calls (remember / leap-frog / apply) keep the reference's
// module boundaries and give the same bits. The constraint virial is reduced in FP64 in a fixed
// order.

#include <algorithm>
#include <cmath>
#include <vector>

#include "sb_internal.cuh"

struct SbTri {
    int A, B, C;
    float ra, rb, rc, rd, re;
};
struct SbCPair {
    int i, j;
    float r, k;  // k = 1 / (m_i + m_j)
};

struct sb_settle {
    int n = 0, ntri = 0, npair = 0, nfree = 0, nrest = 0;
    float dt = 0.f, v_factor = 1.f, x_factor = 1.f;
    SbTri* d_tri = nullptr;
    SbCPair* d_pair = nullptr;
    int* d_free = nullptr;         // atoms in no triangle and no pair
    float3* d_last = nullptr;      // [2 ntri] triangle B-A, C-A; [npair] pair B-A
    float* d_vir = nullptr;        // [ntri + npair] scalar virial of each constraint
    double* d_red = nullptr;
    std::vector<int> rest_i, rest_j;  // constrained pairs left to another scheme
    std::vector<float> rest_r;
};

// ---------------------------------------------------------------------------------------------
// host: triangle geometry and the search for rigid triangles and pairs (SETTLE::Initial)
// ---------------------------------------------------------------------------------------------
// Get_Rabcde_From_SSS (SETTLE.cu:7-41): the rigid triangle with its centre of mass at the origin,
// A at (0, ra, 0), B at (rc, rb, 0), C at (rd, re, 0); FP32 as the reference computes it
static void rabcde_from_sss(float rAB, float rAC, float rBC, float mA, float mB, float mC,
                            float& ra, float& rb, float& rc, float& rd, float& re) {
    const float mT = mA + mB + mC;
    float Ax = 0, Ay = 0, Bx = -rAB, By = 0;
    float c = (rBC * rBC - rAC * rAC - rAB * rAB) / (2 * rAC * rAB);
    float Cx = rAC * c;
    float sn = sqrtf(1.0f - c * c);
    float Cy = rAC * sn;
    const float Ox = (Bx * mB + Cx * mC) / mT, Oy = Cy * mC / mT;
    Ax -= Ox;
    Ay -= Oy;
    Bx -= Ox;
    By -= Oy;
    Cx -= Ox;
    Cy -= Oy;
    c = 1.0f / sqrtf(1.0f + Ax * Ax / Ay / Ay);
    sn = c * Ax / Ay;
    ra = Ax * sn + Ay * c;
    rc = Bx * c - By * sn;
    rb = Bx * sn + By * c;
    rd = Cx * c - Cy * sn;
    re = Cx * sn + Cy * c;
    if (ra < 0) {
        ra = -ra;
        rb = -rb;
        re = -re;
    }
}

// ---------------------------------------------------------------------------------------------
// device
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 ld3(const float* p, int i) { return f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void st3(float* p, int i, float3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
// Get_Periodic_Displacement of fixed-point coordinates (common.cu:89-97): a - b
__device__ __forceinline__ float3 udisp(const uint32_t* uc, int a, int b, float3 s) {
    return f3((float)(int)(uc[3 * a] - uc[3 * b]) * s.x, (float)(int)(uc[3 * a + 1] - uc[3 * b + 1]) * s.y,
              (float)(int)(uc[3 * a + 2] - uc[3 * b + 2]) * s.z);
}
// Get_Periodic_Displacement of float coordinates (common.cu:99-107): a - b, nearest image
__device__ __forceinline__ float3 fdisp(float3 a, float3 b, float3 L) {
    float3 d = a - b;
    d.x = d.x - floorf(d.x / L.x + 0.5f) * L.x;
    d.y = d.y - floorf(d.y / L.y + 0.5f) * L.y;
    d.z = d.z - floorf(d.z / L.z + 0.5f) * L.z;
    return d;
}

// MD_Iteration_Leap_Frog (MD_core.cu:13-32) on values in registers: a = F/m; v += dt a;
// x += dt v
__device__ __forceinline__ void leap_frog_regs(float im, float3 f, float3& v, float3& x,
                                               float3& a, float dt) {
    a = f3(im * f.x, im * f.y, im * f.z);
    v = f3(v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z);
    x = f3(x.x + dt * v.x, x.y + dt * v.y, x.z + dt * v.z);
}

// the same on atom i in memory
__device__ __forceinline__ void leap_frog_atom(int i, const float* __restrict__ inv_mass,
                                               const float* __restrict__ frc, float* __restrict__ vel,
                                               float* __restrict__ crd, float* __restrict__ acc,
                                               float dt) {
    float3 v = ld3(vel, i), x = ld3(crd, i), a;
    leap_frog_regs(inv_mass[i], ld3(frc, i), v, x, a, dt);
    if (acc) st3(acc, i, a);
    st3(vel, i, v);
    st3(crd, i, x);
}

// SETTLE_DO_TRIANGLE (SETTLE.cu:93-176): positions relative to the centre of mass
__device__ __forceinline__ void settle_do_triangle(float3 rB0, float3 rC0, float3& rA, float3& rB,
                                                   float3& rC, const SbTri& T, float mB, float mC,
                                                   float dt, float xf, float vf, float3& vA,
                                                   float3& vB, float3& vC, float& vir) {
    const float3 rA1 = rA, rB1 = rB, rC1 = rC;
    float3 bz = cross3(rB0, rC0);
    float3 bx = cross3(rA1, bz);
    float3 by = cross3(bz, bx);
    bx = rnorm3df(bx.x, bx.y, bx.z) * bx;
    by = rnorm3df(by.x, by.y, by.z) * by;
    bz = rnorm3df(bz.x, bz.y, bz.z) * bz;
    const float3 rB0d = f3(dot3(bx, rB0), dot3(by, rB0), 0.f);
    const float3 rC0d = f3(dot3(bx, rC0), dot3(by, rC0), 0.f);
    const float3 rA1d = f3(0.f, 0.f, dot3(bz, rA1));
    const float3 rB1d = f3(dot3(bx, rB1), dot3(by, rB1), dot3(bz, rB1));
    const float3 rC1d = f3(dot3(bx, rC1), dot3(by, rC1), dot3(bz, rC1));
    const float sinphi = rA1d.z / T.ra;
    const float cosphi = sqrtf(1.0f - sinphi * sinphi);
    const float sinpsi = (rB1d.z - rC1d.z - (T.rb - T.re) * sinphi) / ((T.rd - T.rc) * cosphi);
    const float cospsi = sqrtf(1.0f - sinpsi * sinpsi);
    const float3 rA2d = f3(0.0f, T.ra * cosphi, rA1d.z);
    const float3 rB2d = f3(T.rc * cospsi, T.rb * cosphi + T.rc * sinpsi * sinphi, rB1d.z);
    const float3 rC2d = f3(T.rd * cospsi, T.re * cosphi + T.rd * sinpsi * sinphi, rC1d.z);
    const float alpha = rB2d.x * rB0d.x + rC2d.x * rC0d.x + rB2d.y * rB0d.y + rC2d.y * rC0d.y;
    const float beta = -rB2d.x * rB0d.y - rC2d.x * rC0d.y + rB2d.y * rB0d.x + rC2d.y * rC0d.x;
    const float gamma = rB1d.y * rB0d.x - rB1d.x * rB0d.y + rC1d.y * rC0d.x - rC1d.x * rC0d.y;
    const float ab = alpha * alpha + beta * beta;
    const float sintheta = (alpha * gamma - beta * sqrtf(ab - gamma * gamma)) / ab;
    const float costheta = sqrtf(1.0f - sintheta * sintheta);
    const float3 rA3d = f3(-rA2d.y * sintheta, rA2d.y * costheta, rA2d.z);
    const float3 rB3d = f3(rB2d.x * costheta - rB2d.y * sintheta,
                           rB2d.x * sintheta + rB2d.y * costheta, rB2d.z);
    const float3 rC3d = f3(rC2d.x * costheta - rC2d.y * sintheta,
                           rC2d.x * sintheta + rC2d.y * costheta, rC2d.z);
    auto back = [&](float3 d) {
        return f3(d.x * bx.x + d.y * by.x + d.z * bz.x, d.x * bx.y + d.y * by.y + d.z * bz.y,
                  d.x * bx.z + d.y * by.z + d.z * bz.z);
    };
    rA = back(rA3d);
    rB = back(rB3d);
    rC = back(rC3d);
    const float kv = vf / dt / xf;
    vA = vA + kv * (rA - rA1);
    vB = vB + kv * (rB - rB1);
    vC = vC + kv * (rC - rC1);
    const float kf = 1.0f / dt / dt / xf;
    const float3 FB = (kf * mB) * (rB - rB1), FC = (kf * mC) * (rC - rC1);
    vir = (FB.x * rB0.x + FC.x * rC0.x) + (FB.y * rB0.y + FC.y * rC0.y) + (FB.z * rB0.z + FC.z * rC0.z);
}

// settle_triangle (SETTLE.cu:349-380) on one triangle whose edge vectors at the step start are
// BA, CA, on positions and velocities in registers (updated in place)
__device__ __forceinline__ void settle_triangle_regs(const SbTri& T, float3 BA, float3 CA,
                                                     float mA, float mB, float mC, float3& xA,
                                                     float3& xB, float3& xC, float3& vA,
                                                     float3& vB, float3& vC, float3 L, float dt,
                                                     float vf, float xf, float& vir) {
    float3 rA = xA;
    float3 rB = fdisp(xB, rA, L);
    float3 rC = fdisp(xC, rA, L);
    const float3 rO = (1.0f / (mA + mB + mC)) * (mB * rB + mC * rC) + rA;
    rA = rA - rO;
    rB = rB + rA;
    rC = rC + rA;
    settle_do_triangle(BA, CA, rA, rB, rC, T, mB, mC, dt, xf, vf, vA, vB, vC, vir);
    xA = rA + rO;
    xB = rB + rO;
    xC = rC + rO;
}

// the same on a triangle in memory
__device__ __forceinline__ void settle_triangle_one(const SbTri& T, float3 BA, float3 CA,
                                                    const float* __restrict__ mass,
                                                    float* __restrict__ crd, float* __restrict__ vel,
                                                    float3 L, float dt, float vf, float xf,
                                                    float& vir) {
    float3 xA = ld3(crd, T.A), xB = ld3(crd, T.B), xC = ld3(crd, T.C);
    float3 vA = ld3(vel, T.A), vB = ld3(vel, T.B), vC = ld3(vel, T.C);
    settle_triangle_regs(T, BA, CA, mass[T.A], mass[T.B], mass[T.C], xA, xB, xC, vA, vB, vC, L,
                         dt, vf, xf, vir);
    st3(crd, T.A, xA);
    st3(crd, T.B, xB);
    st3(crd, T.C, xC);
    st3(vel, T.A, vA);
    st3(vel, T.B, vB);
    st3(vel, T.C, vC);
}

// settle_pair (SETTLE.cu:381-414) on one rigid pair whose vector at the step start is AB
__device__ __forceinline__ void settle_pair_one(const SbCPair& P, float3 r2,
                                                const float* __restrict__ mass,
                                                float* __restrict__ crd, float* __restrict__ vel,
                                                float3 L, float dt, float vf, float xf, float& vir) {
    float3 r1 = fdisp(ld3(crd, P.j), ld3(crd, P.i), L);
    const float mA = mass[P.i], mB = mass[P.j];
    const float r0r0 = P.r * P.r, r1r1 = dot3(r1, r1), r1r2 = dot3(r1, r2), r2r2 = dot3(r2, r2);
    float k = (sqrtf(r1r2 * r1r2 - r1r1 * r2r2 + r2r2 * r0r0) - r1r2) / r2r2;
    float3 kr2 = k * r2;
    r1 = (-mB * P.k) * kr2;
    kr2 = (mA * P.k) * kr2;
    st3(crd, P.i, ld3(crd, P.i) + r1);
    st3(crd, P.j, ld3(crd, P.j) + kr2);
    k = vf / dt / xf;
    st3(vel, P.i, ld3(vel, P.i) + k * r1);
    st3(vel, P.j, ld3(vel, P.j) + k * kr2);
    r1 = (k * mB / dt / vf) * kr2;
    vir = r1.x * r2.x + r1.y * r2.y + r1.z * r2.z;
}

__global__ void k_settle_remember(int ntri, int npair, const SbTri* __restrict__ tri,
                                  const SbCPair* __restrict__ pr, const uint32_t* __restrict__ uc,
                                  float3 s, float3* __restrict__ last) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntri) {
        const SbTri T = tri[t];
        last[2 * t] = udisp(uc, T.B, T.A, s);
        last[2 * t + 1] = udisp(uc, T.C, T.A, s);
    } else if (t < ntri + npair) {
        const SbCPair P = pr[t - ntri];
        last[2 * ntri + (t - ntri)] = udisp(uc, P.j, P.i, s);
    }
}

__global__ void k_leap_frog(int n, const float* __restrict__ inv_mass, const float* __restrict__ frc,
                            float* __restrict__ vel, float* __restrict__ crd, float* __restrict__ acc,
                            float dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) leap_frog_atom(i, inv_mass, frc, vel, crd, acc, dt);
}

__global__ void k_settle_apply(int ntri, int npair, const SbTri* __restrict__ tri,
                               const SbCPair* __restrict__ pr, const float3* __restrict__ last,
                               const float* __restrict__ mass, float* __restrict__ crd,
                               float* __restrict__ vel, float3 L, float dt, float vf, float xf,
                               float* __restrict__ vir) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float v = 0.f;
    if (t < ntri) {
        settle_triangle_one(tri[t], last[2 * t], last[2 * t + 1], mass, crd, vel, L, dt, vf, xf, v);
        vir[t] = v;
    } else if (t < ntri + npair) {
        const int p = t - ntri;
        settle_pair_one(pr[p], last[2 * ntri + p], mass, crd, vel, L, dt, vf, xf, v);
        vir[t] = v;
    }
}

// the three calls in one launch: triangles, pairs, then the unconstrained atoms
__global__ void k_md_step(int ntri, int npair, int nfree, const SbTri* __restrict__ tri,
                          const SbCPair* __restrict__ pr, const int* __restrict__ free_atoms,
                          const uint32_t* __restrict__ uc, float3 s,
                          const float* __restrict__ inv_mass, const float* __restrict__ mass,
                          const float* __restrict__ frc, float* __restrict__ vel,
                          float* __restrict__ crd, float* __restrict__ acc, float3 L, float dt,
                          float vf, float xf, float* __restrict__ vir) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float v = 0.f;
    if (t < ntri) {
        // every load of the triangle is issued before the arithmetic, which then runs on
        // registers (the same operations as the separate calls)
        const SbTri T = tri[t];
        const float3 BA = udisp(uc, T.B, T.A, s), CA = udisp(uc, T.C, T.A, s);
        float3 xA = ld3(crd, T.A), xB = ld3(crd, T.B), xC = ld3(crd, T.C);
        float3 vA = ld3(vel, T.A), vB = ld3(vel, T.B), vC = ld3(vel, T.C);
        const float3 fA = ld3(frc, T.A), fB = ld3(frc, T.B), fC = ld3(frc, T.C);
        const float iA = inv_mass[T.A], iB = inv_mass[T.B], iC = inv_mass[T.C];
        const float mA = mass[T.A], mB = mass[T.B], mC = mass[T.C];
        float3 aA, aB, aC;
        leap_frog_regs(iA, fA, vA, xA, aA, dt);
        leap_frog_regs(iB, fB, vB, xB, aB, dt);
        leap_frog_regs(iC, fC, vC, xC, aC, dt);
        if (acc) {
            st3(acc, T.A, aA);
            st3(acc, T.B, aB);
            st3(acc, T.C, aC);
        }
        settle_triangle_regs(T, BA, CA, mA, mB, mC, xA, xB, xC, vA, vB, vC, L, dt, vf, xf, v);
        st3(crd, T.A, xA);
        st3(crd, T.B, xB);
        st3(crd, T.C, xC);
        st3(vel, T.A, vA);
        st3(vel, T.B, vB);
        st3(vel, T.C, vC);
        vir[t] = v;
    } else if (t < ntri + npair) {
        const SbCPair P = pr[t - ntri];
        const float3 AB = udisp(uc, P.j, P.i, s);
        leap_frog_atom(P.i, inv_mass, frc, vel, crd, acc, dt);
        leap_frog_atom(P.j, inv_mass, frc, vel, crd, acc, dt);
        settle_pair_one(P, AB, mass, crd, vel, L, dt, vf, xf, v);
        vir[t] = v;
    } else if (t < ntri + npair + nfree) {
        leap_frog_atom(free_atoms[t - ntri - npair], inv_mass, frc, vel, crd, acc, dt);
    }
}

__global__ void k_pressure_add(const double* __restrict__ sum, double factor,
                               float* __restrict__ pressure) {
    pressure[0] += (float)(sum[0] * factor);
}

// ---------------------------------------------------------------------------------------------
// host API
// ---------------------------------------------------------------------------------------------
extern "C" int sb_settle_create(int atom_numbers, int constrain_pair_numbers, const int* h_pair_i,
                                const int* h_pair_j, const float* h_pair_r, const float* h_mass,
                                float dt, float exp_gamma, sb_settle** out) {
    if (!out || atom_numbers <= 0 || constrain_pair_numbers < 0 || !h_mass || dt <= 0.f ||
        (constrain_pair_numbers > 0 && (!h_pair_i || !h_pair_j || !h_pair_r))) {
        sb_set_error("sb_settle_create: invalid arguments");
        return SB_ERR_ARG;
    }
    const int n = atom_numbers;
    for (int p = 0; p < constrain_pair_numbers; p++)
        if (h_pair_i[p] < 0 || h_pair_i[p] >= n || h_pair_j[p] < 0 || h_pair_j[p] >= n ||
            h_pair_i[p] == h_pair_j[p]) {
            sb_set_error("sb_settle_create: constraint pair %d is not two atoms of [0, %d)", p, n);
            return SB_ERR_ARG;
        }
    // SETTLE::Initial (SETTLE.cu:194-305): atoms with two constraints closing a triangle become
    // rigid triangles, isolated constrained pairs rigid pairs, everything else stays with the
    // other constraint schemes
    std::vector<int> num(n, 0), link(2 * (size_t)n, -1);
    std::vector<float> lr(3 * (size_t)n, 0.f);
    for (int p = 0; p < constrain_pair_numbers; p++) {
        const int a = h_pair_i[p], b = h_pair_j[p];
        if (num[a] < 2 && num[b] < 2) {
            link[2 * a + num[a]] = b;
            link[2 * b + num[b]] = a;
            lr[3 * a + num[a]] = h_pair_r[p];
            lr[3 * b + num[b]] = h_pair_r[p];
            num[a]++;
            num[b]++;
        } else {
            num[a] = 3;
            num[b] = 3;
        }
    }
    for (int i = 0; i < n; i++) {
        if (num[i] == 2) {
            const int a = link[2 * i], b = link[2 * i + 1];
            if (num[a] == 2 && num[b] == 2 &&
                ((link[2 * a] == i && link[2 * a + 1] == b) || (link[2 * a + 1] == i && link[2 * a] == b))) {
                num[a] = -2;
                num[b] = -2;
                lr[3 * i + 2] = link[2 * a + 1] == b ? lr[3 * a + 1] : lr[3 * a];
            } else {
                num[i] = 3;
                num[a] = 3;
                num[b] = 3;
            }
        } else if (num[i] == 1) {
            const int a = link[2 * i];
            if (num[a] == 1) {
                num[a] = -1;
            } else {
                num[i] = 3;
                num[a] = 3;
            }
        }
    }
    sb_settle* m = new sb_settle();
    m->n = n;
    m->dt = dt;
    m->v_factor = exp_gamma;                 // CONSTRAIN::Initial_Constrain (constrain.cu:11-12)
    m->x_factor = 0.5f * (1.0f + exp_gamma);
    std::vector<SbTri> tri;
    std::vector<SbCPair> prs;
    std::vector<char> used(n, 0);
    for (int i = 0; i < n; i++) {
        if (num[i] == 2) {
            const int a = link[2 * i], b = link[2 * i + 1];
            SbTri T;
            T.A = i;
            T.B = a;
            T.C = b;
            rabcde_from_sss(lr[3 * i], lr[3 * i + 1], lr[3 * i + 2], h_mass[i], h_mass[a],
                            h_mass[b], T.ra, T.rb, T.rc, T.rd, T.re);
            tri.push_back(T);
            used[i] = used[a] = used[b] = 1;
            num[i] = -2;
        }
        if (num[i] == 1) {
            const int j = link[2 * i];
            SbCPair P;
            P.i = i;
            P.j = j;
            P.r = lr[3 * i];
            P.k = 1.0f / (h_mass[i] + h_mass[j]);
            prs.push_back(P);
            used[i] = used[j] = 1;
            num[i] = -1;
        }
    }
    for (int p = 0; p < constrain_pair_numbers; p++)
        if (num[h_pair_i[p]] > 0) {
            m->rest_i.push_back(h_pair_i[p]);
            m->rest_j.push_back(h_pair_j[p]);
            m->rest_r.push_back(h_pair_r[p]);
        }
    std::vector<int> fr;
    for (int i = 0; i < n; i++)
        if (!used[i]) fr.push_back(i);
    m->ntri = (int)tri.size();
    m->npair = (int)prs.size();
    m->nfree = (int)fr.size();
    m->nrest = (int)m->rest_i.size();
    const size_t nc = std::max<size_t>(1, tri.size() + prs.size());
    int st = SB_OK;
    if ((st = sb_malloc((void**)&m->d_tri, sizeof(SbTri) * std::max<size_t>(1, tri.size()), "triangles")) ||
        (st = sb_malloc((void**)&m->d_pair, sizeof(SbCPair) * std::max<size_t>(1, prs.size()), "pairs")) ||
        (st = sb_malloc((void**)&m->d_free, sizeof(int) * std::max<size_t>(1, fr.size()), "free atoms")) ||
        (st = sb_malloc((void**)&m->d_last, sizeof(float3) * (2 * tri.size() + prs.size() + 1), "last vectors")) ||
        (st = sb_malloc((void**)&m->d_vir, sizeof(float) * nc, "constraint virial")) ||
        (st = sb_malloc((void**)&m->d_red, sizeof(double), "virial sum"))) {
        sb_settle_destroy(m);
        return st;
    }
    if (!tri.empty()) cudaMemcpy(m->d_tri, tri.data(), sizeof(SbTri) * tri.size(), cudaMemcpyHostToDevice);
    if (!prs.empty()) cudaMemcpy(m->d_pair, prs.data(), sizeof(SbCPair) * prs.size(), cudaMemcpyHostToDevice);
    if (!fr.empty()) cudaMemcpy(m->d_free, fr.data(), sizeof(int) * fr.size(), cudaMemcpyHostToDevice);
    if (cudaGetLastError() != cudaSuccess) {
        sb_set_error("sb_settle_create: device copy failed");
        sb_settle_destroy(m);
        return SB_ERR_CUDA;
    }
    *out = m;
    return SB_OK;
}

extern "C" int sb_settle_destroy(sb_settle* m) {
    if (!m) return SB_OK;
    void* ps[] = {m->d_tri, m->d_pair, m->d_free, m->d_last, m->d_vir, m->d_red};
    for (void* p : ps) sb_free(p);
    delete m;
    return SB_OK;
}

extern "C" int sb_settle_info(sb_settle* m, int* h_triangles, int* h_pairs, int* h_remaining) {
    if (!m) {
        sb_set_error("sb_settle_info: null handle");
        return SB_ERR_ARG;
    }
    if (h_triangles) *h_triangles = m->ntri;
    if (h_pairs) *h_pairs = m->npair;
    if (h_remaining) *h_remaining = m->nrest;
    return SB_OK;
}

extern "C" int sb_settle_remember(sb_settle* m, const uint32_t* d_uint_crd, const float scaler[3],
                                  void* stream) {
    if (!m || !d_uint_crd || !scaler) {
        sb_set_error("sb_settle_remember: null argument");
        return SB_ERR_ARG;
    }
    const int nt = m->ntri + m->npair;
    if (nt == 0) return SB_OK;
    k_settle_remember<<<(nt + 127) / 128, 128, 0, sb_stream(stream)>>>(
        m->ntri, m->npair, m->d_tri, m->d_pair, d_uint_crd,
        make_float3(scaler[0], scaler[1], scaler[2]), m->d_last);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

static int add_pressure(sb_settle* m, const float box[3], float* d_pressure, cudaStream_t s) {
    const int nc = m->ntri + m->npair;
    if (nc == 0) return SB_OK;
    SB_TRY(sb_reduce_sum_f32(m->d_vir, nc, m->d_red, s));
    // Sum_Of_Virial_Vector_To_Pressure's factor (SETTLE.cu:425-433, :448)
    const double factor = (double)(0.33333f / box[0] / box[1] / box[2]);
    k_pressure_add<<<1, 1, 0, s>>>(m->d_red, factor, d_pressure);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

extern "C" int sb_settle_apply(sb_settle* m, const float* d_mass, float* d_crd,
                               const float box[3], float* d_vel, int need_pressure,
                               float* d_pressure, void* stream) {
    if (!m || !d_mass || !d_crd || !box || !d_vel || (need_pressure && !d_pressure)) {
        sb_set_error("sb_settle_apply: null argument");
        return SB_ERR_ARG;
    }
    cudaStream_t s = sb_stream(stream);
    const int nc = m->ntri + m->npair;
    if (nc == 0) return SB_OK;
    k_settle_apply<<<(nc + 127) / 128, 128, 0, s>>>(
        m->ntri, m->npair, m->d_tri, m->d_pair, m->d_last, d_mass, d_crd, d_vel,
        make_float3(box[0], box[1], box[2]), m->dt, m->v_factor, m->x_factor, m->d_vir);
    SB_CHECK_LAUNCH();
    if (need_pressure) SB_TRY(add_pressure(m, box, d_pressure, s));
    return SB_OK;
}

extern "C" int sb_md_leap_frog(int atom_numbers, const float* d_inverse_mass, const float* d_frc,
                               float* d_vel, float* d_crd, float* d_acc, float dt, void* stream) {
    if (atom_numbers < 0 || !d_inverse_mass || !d_frc || !d_vel || !d_crd) {
        sb_set_error("sb_md_leap_frog: null argument");
        return SB_ERR_ARG;
    }
    if (atom_numbers == 0) return SB_OK;
    k_leap_frog<<<(atom_numbers + 127) / 128, 128, 0, sb_stream(stream)>>>(
        atom_numbers, d_inverse_mass, d_frc, d_vel, d_crd, d_acc, dt);
    SB_CHECK_LAUNCH();
    return SB_OK;
}

extern "C" int sb_md_nve_settle_step(sb_settle* m, const uint32_t* d_uint_crd,
                                     const float scaler[3], const float* d_inverse_mass,
                                     const float* d_mass, const float* d_frc, float* d_vel,
                                     float* d_crd, float* d_acc, const float box[3],
                                     int need_pressure, float* d_pressure, void* stream) {
    if (!m || !d_uint_crd || !scaler || !d_inverse_mass || !d_mass || !d_frc || !d_vel ||
        !d_crd || !box || (need_pressure && !d_pressure)) {
        sb_set_error("sb_md_nve_settle_step: null argument");
        return SB_ERR_ARG;
    }
    if (m->nrest > 0) {
        sb_set_error("sb_md_nve_settle_step: %d constrained pairs need another constraint scheme",
                     m->nrest);
        return SB_ERR_STATE;
    }
    cudaStream_t s = sb_stream(stream);
    const int nt = m->ntri + m->npair + m->nfree;
    if (nt > 0) {
        k_md_step<<<(nt + 127) / 128, 128, 0, s>>>(
            m->ntri, m->npair, m->nfree, m->d_tri, m->d_pair, m->d_free, d_uint_crd,
            make_float3(scaler[0], scaler[1], scaler[2]), d_inverse_mass, d_mass, d_frc, d_vel,
            d_crd, d_acc, make_float3(box[0], box[1], box[2]), m->dt, m->v_factor, m->x_factor,
            m->d_vir);
        SB_CHECK_LAUNCH();
    }
    if (need_pressure) SB_TRY(add_pressure(m, box, d_pressure, s));
    return SB_OK;
}

// FP64 CPU oracle for SPONGE's nonbonded hot path.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links or calls this file; it is
// loaded by the tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, where it
// is the checker and the timed CPU comparison, never the thing that is measured as the product.
//
// It restates, in double precision, the algorithm of the reference (paths relative to the
// SPONGE project root):
//   * fixed-point coordinates        SPONGE/common.cu:264-287 (Crd_To_Uint_Crd),
//                                    SPONGE/neighbor_list/neighbor_list.cu:730 (0.25*2^32/L)
//   * periodic wrap                  SPONGE/common.cu:299-352 (Crd_Periodic_Map)
//   * minimum-image displacement     SPONGE/common.cu:89-97
//   * neighbor-list pair set          SPONGE/neighbor_list/neighbor_list.cu:331-391 (j>i,
//                                    dr^2 < (rc+skin)^2) and :461-511 (exclusions removed)
//   * LJ + Ewald direct pair force    SPONGE/Lennard_Jones_force/Lennard_Jones_force.cu:47-158,
//                                    energies/virial :424-562, pair-type index :106-112
//   * long-range LJ correction       SPONGE/Lennard_Jones_force/Lennard_Jones_force.cu:1042-1130,
//                                    :1178-1191
//   * exclusion correction           SPONGE/PME_force/PME_force.cu:620-695
//   * SPME                           SPONGE/PME_force/PME_force.cu:8-14 (B-spline weights),
//                                    :45-67 (moduli), :71-100 (Get_Beta), :253-286 (BC table),
//                                    :367-550 (grid points, spread, gather), :553-566 + :753-771
//                                    (reciprocal and self energies)
//   * FFT grid size                  SPONGE/common.cu:467-534 (Get_Fft_Patameter)
//   * 1-4 pairs                      SPONGE/nb14/nb14.cu:92-170 (force, energy, virial),
//                                    :5-91 (energies), :203-217 (per-pair A, B)
//   * NVE leap-frog + SETTLE         SPONGE/MD_core/MD_core.cu:13-32, SPONGE/constrain/SETTLE.cu
//                                    :7-41 (triangle geometry), :93-176 (triangle), :183-305
//                                    (rigid triangles and pairs), :349-414 (kernels)
//   * virtual atoms                  SPONGE/virtual_atoms/virtual_atoms.cu:2-73 (positions),
//                                    :75-180 (force redistribution), :246-290 + :495-530
//                                    (levels and their order)
//
// Pair-set criterion. The reference decides list membership with an FP32 expression whose
// evaluation order (and FMA contraction) is chosen by its compiler. This build pins ONE order:
//   dx = fmul_rn((float)(int)(u_j - u_i), L*2^-32); r2 = fadd(fadd(dx*dx, dy*dy), dz*dz)
// with every operation rounded to nearest and no contraction, member iff r2 < (rc+skin)^2
// (threshold squared in float as the reference does, neighbor_list.cu:723-725). The GPU list
// kernels evaluate the identical expression, so pair sets compare bit-exactly. The in-cutoff
// decision of the force kernels (r2 < rc^2) uses the same expression.
//
// This file is compiled with -ffp-contract=off so that the FP32 criterion above is exact.

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <vector>
#include <thread>
#include <vector>

typedef std::complex<double> cplx;

static int g_threads = 0;

static int nthreads_eff(int requested) {
    int hw = (int)std::thread::hardware_concurrency();
    if (hw <= 0) hw = 1;
    int t = requested > 0 ? requested : (g_threads > 0 ? g_threads : hw);
    return std::max(1, std::min(t, 256));
}

static void parallel_for(long n, int nthreads, const std::function<void(long, long, int)>& fn) {
    int t = nthreads_eff(nthreads);
    if (t == 1 || n < 2) {
        fn(0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    long chunk = (n + t - 1) / t;
    for (int k = 0; k < t; k++) {
        long b = k * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        th.emplace_back(fn, b, e, k);
    }
    for (auto& x : th) x.join();
}

// ------------------------------------------------------------------------------------------
// fixed point and small helpers
// ------------------------------------------------------------------------------------------

static inline float pair_r2_f32(uint32_t ui, uint32_t uj, uint32_t vi, uint32_t vj, uint32_t wi,
                                uint32_t wj, const float s[3]) {
    // exact restatement of the pinned FP32 criterion (see header)
    volatile float dx = (float)(int32_t)(uj - ui) * s[0];
    volatile float dy = (float)(int32_t)(vj - vi) * s[1];
    volatile float dz = (float)(int32_t)(wj - wi) * s[2];
    volatile float xx = dx * dx;
    volatile float yy = dy * dy;
    volatile float zz = dz * dz;
    volatile float a = xx + yy;
    volatile float r2 = a + zz;
    return r2;
}

static inline void scaler_of(const float* box, float s[3]) {
    // uint_dr_to_dr_cof = 1.0f / 2^32 * L  (neighbor_list.cu:731): an exact power-of-two scaling
    for (int d = 0; d < 3; d++) s[d] = (1.0f / 4294967296.0f) * box[d];
}

static inline void dr_f64(const uint32_t* a, const uint32_t* b, const float s[3], double dr[3]) {
    // displacement b - a in FP64; the int difference is exact, its product with s is one rounding
    for (int d = 0; d < 3; d++) dr[d] = (double)(int32_t)(b[d] - a[d]) * (double)s[d];
}

extern "C" {

int orc_version() { return 3; }

void orc_set_threads(int n) { g_threads = n; }

int orc_threads() { return nthreads_eff(0); }

// Crd_Periodic_Map: one shift into [0, L).
void orc_periodic_map(int n, float* crd, const float* box) {
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            float& x = crd[3 * i + d];
            if (x >= 0) {
                if (!(x < box[d])) x = x - box[d];
            } else {
                x = x + box[d];
            }
        }
}

// Crd_To_Uint_Crd with the quarter coefficient 0.25f*2^32/L computed in float.
void orc_crd_to_uint(int n, const float* crd, const float* box, uint32_t* uc) {
    float cof[3];
    for (int d = 0; d < 3; d++) cof[d] = (0.25f * 4294967296.0f) / box[d];
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            volatile float t = crd[3 * i + d] * cof[d];
            int ti = (int)t;
            uc[3 * i + d] = ((uint32_t)ti) << 2;
        }
}

// Get_Beta: bisection on erfc(beta*rc)/rc = tol with the reference's float/double mix.
float orc_get_beta(float cutoff, float tolerance) {
    float beta = 0, low, high, tempf;
    int ilow, ihigh;
    high = 1.0f;
    ihigh = 1;
    while (1) {
        float hc = high * cutoff;
        tempf = (float)(erfc((double)hc) / (double)cutoff);
        if (tempf <= tolerance) break;
        high *= 2;
        ihigh++;
    }
    ihigh += 50;
    low = 0.0f;
    for (ilow = 1; ilow < ihigh; ilow++) {
        beta = (low + high) / 2;
        float bc = beta * cutoff;
        tempf = (float)(erfc((double)bc) / (double)cutoff);
        if (tempf >= tolerance)
            low = beta;
        else
            high = beta;
    }
    return beta;
}

static int check_2357(int number) {
    const int primes[4] = {2, 3, 5, 7};
    for (int p : primes) {
        while (number > 0) {
            if (number == 1) return 1;
            int t = number / p;
            if (t * p != number) break;
            number = t;
        }
    }
    return number == 1;
}

// Get_Fft_Patameter
int orc_fft_size(float length) {
    int t = ((int)ceil((double)length + 3)) >> 2 << 2;
    if (t >= 60 && t <= 68) t = 64;
    else if (t >= 120 && t <= 136) t = 128;
    else if (t >= 240 && t <= 272) t = 256;
    else if (t >= 480 && t <= 544) t = 512;
    else if (t >= 960 && t <= 1088) t = 1024;
    while (1) {
        if (check_2357(t)) return t;
        t += 4;
    }
}

// |b(k)|^2 for 4th-order cardinal B-splines: 1/|sum_{j=0}^{2} M4(j+1) e^{2 pi i jk/K}|^2
void orc_bspline_moduli(int K, double* out) {
    const double M4[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
    for (int k = 0; k < K; k++) {
        cplx s(0, 0);
        for (int j = 0; j < 3; j++) s += M4[j] * std::polar(1.0, 2 * M_PI * j * (double)k / K);
        out[k] = 1.0 / std::norm(s);
    }
}

// ------------------------------------------------------------------------------------------
// pair sets
// ------------------------------------------------------------------------------------------

static inline bool is_excluded(int a, int b, const int* es, const int* en, const int* el) {
    // pair {a<b} is removed from the list iff b appears in a's own exclusion list
    // (neighbor_list.cu:461-511 only scans nl[a], which holds j > a)
    int s = es[a], e = s + en[a];
    for (int k = s; k < e; k++)
        if (el[k] == b) return true;
    return false;
}

// Brute-force O(N^2) half pair set. Writes keys i*n+j (i<j) sorted ascending. Returns count.
long orc_pairs_bruteforce(int n, const uint32_t* uc, const float* box, float cutoff, float skin,
                          const int* es, const int* en, const int* el, int64_t* out, long cap,
                          int nthreads) {
    float s[3];
    scaler_of(box, s);
    float cs = cutoff + skin;
    float thr = cs * cs;
    int t = nthreads_eff(nthreads);
    std::vector<std::vector<int64_t>> parts(t);
    parallel_for(n, t, [&](long b, long e, int k) {
        auto& v = parts[k];
        for (long i = b; i < e; i++) {
            const uint32_t* a = uc + 3 * i;
            for (long j = i + 1; j < n; j++) {
                const uint32_t* c = uc + 3 * j;
                float r2 = pair_r2_f32(a[0], c[0], a[1], c[1], a[2], c[2], s);
                if (r2 < thr && !is_excluded((int)i, (int)j, es, en, el))
                    v.push_back((int64_t)i * n + j);
            }
        }
    });
    long total = 0;
    for (auto& v : parts) {
        for (auto x : v) {
            if (total < cap) out[total] = x;
            total++;
        }
    }
    if (total <= cap) std::sort(out, out + total);
    return total;
}

// Cell-based O(N) half pair set with the same criterion (reference cell rule:
// Nx = floor(L / ((rc+skin)/2)), 5x5x5 stencil, neighbor_list.cu:111-258). Same output.
long orc_pairs_cells(int n, const uint32_t* uc, const float* box, float cutoff, float skin,
                     const int* es, const int* en, const int* el, int64_t* out, long cap,
                     int nthreads) {
    float s[3];
    scaler_of(box, s);
    float cs = cutoff + skin;
    float thr = cs * cs;
    int N[3];
    for (int d = 0; d < 3; d++) {
        N[d] = (int)floor((double)box[d] / (0.5 * cs));
        if (N[d] < 1) N[d] = 1;
    }
    long ncell = (long)N[0] * N[1] * N[2];
    std::vector<int> cell(n), cnt(ncell + 1, 0);
    for (int i = 0; i < n; i++) {
        int c[3];
        for (int d = 0; d < 3; d++) c[d] = (int)(((uint64_t)uc[3 * i + d] * (uint64_t)N[d]) >> 32);
        cell[i] = (c[2] * N[1] + c[1]) * N[0] + c[0];
        cnt[cell[i] + 1]++;
    }
    for (long c = 0; c < ncell; c++) cnt[c + 1] += cnt[c];
    std::vector<int> idx(n), fill(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < n; i++) idx[fill[cell[i]]++] = i;  // ascending atom id per cell
    // neighbor cell offsets: all cells within +-2, de-duplicated for small grids
    int t = nthreads_eff(nthreads);
    std::vector<std::vector<int64_t>> parts(t);
    parallel_for(n, t, [&](long b, long e, int k) {
        auto& v = parts[k];
        std::vector<int> nb;
        for (long i = b; i < e; i++) {
            int ci = cell[i];
            int cz = ci / (N[0] * N[1]), cy = (ci / N[0]) % N[1], cx = ci % N[0];
            nb.clear();
            for (int dz = -2; dz <= 2; dz++)
                for (int dy = -2; dy <= 2; dy++)
                    for (int dx = -2; dx <= 2; dx++) {
                        int x = ((cx + dx) % N[0] + N[0]) % N[0];
                        int y = ((cy + dy) % N[1] + N[1]) % N[1];
                        int z = ((cz + dz) % N[2] + N[2]) % N[2];
                        nb.push_back((z * N[1] + y) * N[0] + x);
                    }
            std::sort(nb.begin(), nb.end());
            nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
            const uint32_t* a = uc + 3 * i;
            for (int c : nb)
                for (int p = cnt[c]; p < cnt[c + 1]; p++) {
                    int j = idx[p];
                    if (j <= i) continue;
                    const uint32_t* q = uc + 3 * (long)j;
                    float r2 = pair_r2_f32(a[0], q[0], a[1], q[1], a[2], q[2], s);
                    if (r2 < thr && !is_excluded((int)i, j, es, en, el))
                        v.push_back((int64_t)i * n + j);
                }
        }
    });
    long total = 0;
    for (auto& v : parts)
        for (auto x : v) {
            if (total < cap) out[total] = x;
            total++;
        }
    if (total <= cap) std::sort(out, out + total);
    return total;
}

// ------------------------------------------------------------------------------------------
// LJ + Ewald direct space over a pair list
// ------------------------------------------------------------------------------------------

static inline int pair_type(int a, int b) {
    int M = a > b ? a : b, m = a > b ? b : a;
    return M * (M + 1) / 2 + m;
}

// out[0] = E_LJ, out[1] = E_direct_coulomb, out[2] = LJ virial (sum r.F), out[3] = in-cutoff
// pairs. frc (3n) and atom_energy (n) are accumulated (+=) in FP64; per-atom energy of a pair is
// attributed to its lower atom id as the reference's half list does.
void orc_direct(int n, const uint32_t* uc, const float* q, const int* type, const float* A12,
                const float* B6, const float* box, float cutoff, double beta,
                const int64_t* pairs, long npairs, double* frc, double* atom_energy,
                double* out, int nthreads) {
    float s[3];
    scaler_of(box, s);
    float rc2 = cutoff * cutoff;
    int t = nthreads_eff(nthreads);
    std::vector<std::vector<double>> fb(t, std::vector<double>());
    std::vector<std::vector<double>> eb(t, std::vector<double>());
    std::vector<double> acc(4 * t, 0.0);
    const double two_over_sqrt_pi = 2.0 / std::sqrt(M_PI);
    parallel_for(npairs, t, [&](long b, long e, int k) {
        auto& f = fb[k];
        auto& en = eb[k];
        f.assign(3 * (size_t)n, 0.0);
        en.assign((size_t)n, 0.0);
        double elj = 0, edir = 0, vir = 0, cnt = 0;
        for (long p = b; p < e; p++) {
            int i = (int)(pairs[p] / n), j = (int)(pairs[p] % n);
            const uint32_t* a = uc + 3 * (long)i;
            const uint32_t* c = uc + 3 * (long)j;
            float r2f = pair_r2_f32(a[0], c[0], a[1], c[1], a[2], c[2], s);
            if (!(r2f < rc2)) continue;
            double dr[3];
            dr_f64(a, c, s, dr);  // r_j - r_i
            double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            double r = std::sqrt(r2);
            double ri = 1.0 / r, ri2 = ri * ri, ri6 = ri2 * ri2 * ri2;
            int pt = pair_type(type[i], type[j]);
            double A = A12[pt], B = B6[pt];
            double flj = (-A * ri6 + B) * ri6 * ri2;  // (dE/dr)/r
            double br = beta * r;
            double qq = (double)q[i] * (double)q[j];
            double ec = std::erfc(br);
            double fcf = qq * (br * two_over_sqrt_pi * std::exp(-br * br) + ec) * ri2 * ri;
            double fs = flj - fcf;  // force on i = fs * (r_j - r_i)
            for (int d = 0; d < 3; d++) {
                f[3 * (size_t)i + d] += fs * dr[d];
                f[3 * (size_t)j + d] -= fs * dr[d];
            }
            double e_lj = (A / 12.0 * ri6 - B / 6.0) * ri6;
            double e_c = qq * ec * ri;
            en[i] += e_lj + e_c;
            elj += e_lj;
            edir += e_c;
            vir += -flj * r2;
            cnt += 1;
        }
        acc[4 * k + 0] = elj;
        acc[4 * k + 1] = edir;
        acc[4 * k + 2] = vir;
        acc[4 * k + 3] = cnt;
    });
    for (int k = 0; k < t; k++) {
        if (fb[k].empty()) continue;
        for (size_t x = 0; x < 3 * (size_t)n; x++) frc[x] += fb[k][x];
        if (atom_energy)
            for (size_t x = 0; x < (size_t)n; x++) atom_energy[x] += eb[k][x];
    }
    for (int m = 0; m < 4; m++) {
        double v = 0;
        for (int k = 0; k < t; k++) v += acc[4 * k + m];
        out[m] = v;
    }
}

// LJ long-range correction factor (Lennard_Jones_force.cu:1119-1130 with the N^2 type-pair sum
// of Total_C6_Get done exactly through type counts): f = -(2pi/3)/rc^3 * sum_{i,j} B6_ij / 6.
// E_lrc = f / V, virial_lrc = 6 f / V.
double orc_lrc_factor(int n, const int* type, int ntypes, const float* B6, float cutoff) {
    std::vector<double> cnt(ntypes, 0.0);
    for (int i = 0; i < n; i++) cnt[type[i]] += 1.0;
    double sum = 0;
    for (int a = 0; a < ntypes; a++)
        for (int b = 0; b < ntypes; b++) sum += cnt[a] * cnt[b] * (double)B6[pair_type(a, b)];
    double rc = cutoff;
    return sum * (-2.0 / 3.0 * M_PI / (rc * rc * rc) / 6.0);
}

// Exclusion correction (PME_force.cu:620-695): for every CSR entry (i, j):
//   F_i += -qq[(erfc(br) + 2br/sqrt(pi) e^{-b^2r^2}) - 1]/r^3 * (r_j - r_i);  E -= qq erf(br)/r
void orc_excluded(int n, const uint32_t* uc, const float* q, const float* box, double beta,
                  const int* es, const int* en, const int* el, double* frc, double* atom_energy,
                  double* out) {
    float s[3];
    scaler_of(box, s);
    const double two_over_sqrt_pi = 2.0 / std::sqrt(M_PI);
    double etot = 0;
    for (int i = 0; i < n; i++) {
        for (int k = es[i]; k < es[i] + en[i]; k++) {
            int j = el[k];
            double dr[3];
            dr_f64(uc + 3 * (long)i, uc + 3 * (long)j, s, dr);
            double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            double r = std::sqrt(r2);
            double br = beta * r;
            double qq = (double)q[i] * (double)q[j];
            double fa = br * two_over_sqrt_pi * std::exp(-br * br) + std::erfc(br);
            fa = -qq * (fa - 1.0) / r2 / r;
            for (int d = 0; d < 3; d++) {
                frc[3 * (size_t)i + d] += fa * dr[d];
                frc[3 * (size_t)j + d] -= fa * dr[d];
            }
            double e = -qq * std::erf(br) / r;
            if (atom_energy) atom_energy[i] += e;
            etot += e;
        }
    }
    out[0] = etot;
}

// self + neutralising energy (PME_force.cu:758-762, :169)
double orc_self_energy(int n, const float* q, double beta, double volume) {
    double s2 = 0, s1 = 0;
    for (int i = 0; i < n; i++) {
        s2 += (double)q[i] * q[i];
        s1 += q[i];
    }
    return -beta / std::sqrt(M_PI) * s2 - 0.5 * M_PI / (beta * beta * volume) * s1 * s1;
}

// ------------------------------------------------------------------------------------------
// FFT (mixed radix, FP64) and SPME
// ------------------------------------------------------------------------------------------

struct FftPlan {
    int n;
    std::vector<cplx> w;  // e^{sign 2 pi i j / n}
};

static int smallest_factor(int n) {
    for (int p = 2; p * p <= n; p++)
        if (n % p == 0) return p;
    return n;
}

static void fft_rec(const cplx* in, cplx* out, int n, long istride, const FftPlan& P, int wstep) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    int p = smallest_factor(n);
    int m = n / p;
    for (int r = 0; r < p; r++) fft_rec(in + r * istride, out + r * m, m, istride * p, P, wstep * p);
    cplx tmp[64];
    std::vector<cplx> big;
    cplx* t = tmp;
    if (p > 64) {
        big.resize(p);
        t = big.data();
    }
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) t[r] = out[r * m + k] * P.w[((long)r * k * wstep) % P.n];
        for (int qq = 0; qq < p; qq++) {
            cplx acc(0, 0);
            for (int r = 0; r < p; r++) acc += t[r] * P.w[((long)r * qq * m * wstep) % P.n];
            out[k + m * qq] = acc;
        }
    }
}

static FftPlan make_plan(int n, int sign) {
    FftPlan P;
    P.n = n;
    P.w.resize(n);
    for (int j = 0; j < n; j++) P.w[j] = std::polar(1.0, sign * 2 * M_PI * (double)j / n);
    return P;
}

// In-place unnormalised 3D FFT of a [K0][K1][K2] complex grid (sign -1 forward, +1 inverse).
static void fft3(cplx* g, const int* K, int sign, int nthreads) {
    for (int axis = 2; axis >= 0; axis--) {
        int n = K[axis];
        FftPlan P = make_plan(n, sign);
        long stride = axis == 2 ? 1 : (axis == 1 ? K[2] : (long)K[1] * K[2]);
        long nlines = (long)K[0] * K[1] * K[2] / n;
        parallel_for(nlines, nthreads, [&](long b, long e, int) {
            std::vector<cplx> in(n), out(n);
            for (long l = b; l < e; l++) {
                long base;
                if (axis == 2) base = l * n;
                else if (axis == 1) base = (l / K[2]) * ((long)K[1] * K[2]) + (l % K[2]);
                else base = l;
                for (int x = 0; x < n; x++) in[x] = g[base + x * stride];
                fft_rec(in.data(), out.data(), n, 1, P, 1);
                for (int x = 0; x < n; x++) g[base + x * stride] = out[x];
            }
        });
    }
}

// exposed for tests: forward (sign=-1) / inverse (sign=+1) unnormalised 3D FFT, interleaved re/im
void orc_fft3(double* data, const int* K, int sign, int nthreads) {
    fft3(reinterpret_cast<cplx*>(data), K, sign, nthreads);
}

static inline void bspline4(double fr, double w[4], double dw[4]) {
    // weight of grid point (base - k) for fractional offset fr, k = 0..3 (PME_force.cu:8-14)
    double f2 = fr * fr, f3 = f2 * fr;
    w[0] = f3 / 6.0;
    w[1] = -0.5 * f3 + 0.5 * f2 + 0.5 * fr + 1.0 / 6.0;
    w[2] = 0.5 * f3 - f2 + 2.0 / 3.0;
    w[3] = -f3 / 6.0 + 0.5 * f2 - 0.5 * fr + 1.0 / 6.0;
    dw[0] = 0.5 * f2;
    dw[1] = -1.5 * f2 + fr + 0.5;
    dw[2] = 1.5 * f2 - 2.0 * fr;
    dw[3] = -0.5 * f2 + fr - 0.5;
}

// BC(m) = B1 B2 B3 exp(-pi^2 m^2/beta^2)/(pi m^2 V), BC(0)=0 (PME_force.cu:253-286), full grid
static void bc_table(const int* K, const float* box, double beta, std::vector<double>& bc) {
    std::vector<double> B[3];
    for (int d = 0; d < 3; d++) {
        B[d].resize(K[d]);
        orc_bspline_moduli(K[d], B[d].data());
    }
    double V = (double)box[0] * box[1] * box[2];
    bc.assign((size_t)K[0] * K[1] * K[2], 0.0);
    for (int x = 0; x < K[0]; x++) {
        int mx = x > K[0] / 2 ? K[0] - x : x;
        for (int y = 0; y < K[1]; y++) {
            int my = y > K[1] / 2 ? K[1] - y : y;
            for (int z = 0; z < K[2]; z++) {
                int mz = z > K[2] / 2 ? K[2] - z : z;
                if (x + y + z == 0) continue;
                double m2 = (double)mx * mx / ((double)box[0] * box[0]) +
                            (double)my * my / ((double)box[1] * box[1]) +
                            (double)mz * mz / ((double)box[2] * box[2]);
                bc[((size_t)x * K[1] + y) * K[2] + z] =
                    B[0][x] * B[1][y] * B[2][z] * std::exp(-M_PI * M_PI * m2 / (beta * beta)) /
                    (M_PI * m2 * V);
            }
        }
    }
}

// Grid coordinate of an atom: u = uint * K / 2^32 (exact in double), base = floor(u).
static inline void grid_coord(uint32_t u, int K, int& base, double& fr) {
    uint64_t p = (uint64_t)u * (uint64_t)K;
    base = (int)(p >> 32);
    fr = (double)(p & 0xffffffffull) * (1.0 / 4294967296.0);
}

// SPME reciprocal force and energy. out[0] = E_rec. frc (3n) is accumulated. If qgrid_out is
// non-null it receives the spread charge grid Q[K0][K1][K2].
void orc_pme(int n, const uint32_t* uc, const float* q, const float* box, const int* K,
             double beta, double* frc, double* out, double* qgrid_out, int nthreads) {
    size_t G = (size_t)K[0] * K[1] * K[2];
    std::vector<cplx> Q(G, cplx(0, 0));
    std::vector<int> bases(3 * (size_t)n);
    std::vector<double> frs(3 * (size_t)n);
    for (int i = 0; i < n; i++) {
        int b[3];
        double fr[3];
        for (int d = 0; d < 3; d++) {
            grid_coord(uc[3 * (size_t)i + d], K[d], b[d], fr[d]);
            bases[3 * (size_t)i + d] = b[d];
            frs[3 * (size_t)i + d] = fr[d];
        }
        double w[3][4], dw[3][4];
        for (int d = 0; d < 3; d++) bspline4(fr[d], w[d], dw[d]);
        for (int kx = 0; kx < 4; kx++) {
            int gx = ((b[0] - kx) % K[0] + K[0]) % K[0];
            for (int ky = 0; ky < 4; ky++) {
                int gy = ((b[1] - ky) % K[1] + K[1]) % K[1];
                for (int kz = 0; kz < 4; kz++) {
                    int gz = ((b[2] - kz) % K[2] + K[2]) % K[2];
                    Q[((size_t)gx * K[1] + gy) * K[2] + gz] +=
                        (double)q[i] * w[0][kx] * w[1][ky] * w[2][kz];
                }
            }
        }
    }
    std::vector<double> Qr(G);
    for (size_t g = 0; g < G; g++) Qr[g] = Q[g].real();
    if (qgrid_out) std::memcpy(qgrid_out, Qr.data(), G * sizeof(double));
    fft3(Q.data(), K, -1, nthreads);
    std::vector<double> bc;
    bc_table(K, box, beta, bc);
    double erec = 0;
    for (size_t g = 0; g < G; g++) {
        erec += bc[g] * std::norm(Q[g]);
        Q[g] *= bc[g];
    }
    erec *= 0.5;
    fft3(Q.data(), K, +1, nthreads);
    double inv[3] = {K[0] / (double)box[0], K[1] / (double)box[1], K[2] / (double)box[2]};
    parallel_for(n, nthreads, [&](long bgn, long end, int) {
        for (long i = bgn; i < end; i++) {
            double w[3][4], dw[3][4];
            int b[3];
            for (int d = 0; d < 3; d++) {
                b[d] = bases[3 * i + d];
                bspline4(frs[3 * i + d], w[d], dw[d]);
            }
            double f[3] = {0, 0, 0};
            for (int kx = 0; kx < 4; kx++) {
                int gx = ((b[0] - kx) % K[0] + K[0]) % K[0];
                for (int ky = 0; ky < 4; ky++) {
                    int gy = ((b[1] - ky) % K[1] + K[1]) % K[1];
                    for (int kz = 0; kz < 4; kz++) {
                        int gz = ((b[2] - kz) % K[2] + K[2]) % K[2];
                        double th = Q[((size_t)gx * K[1] + gy) * K[2] + gz].real();
                        double dq = -th * (double)q[i];
                        f[0] += dq * dw[0][kx] * w[1][ky] * w[2][kz] * inv[0];
                        f[1] += dq * w[0][kx] * dw[1][ky] * w[2][kz] * inv[1];
                        f[2] += dq * w[0][kx] * w[1][ky] * dw[2][kz] * inv[2];
                    }
                }
            }
            for (int d = 0; d < 3; d++) frc[3 * i + d] += f[d];
        }
    });
    out[0] = erec;
}

// Classic Ewald reciprocal sum (no grid) for small systems: the converged reference for the
// SPME method error. Positions from the fixed-point coordinates. out[0] = E_rec.
void orc_ewald_recip(int n, const uint32_t* uc, const float* q, const float* box, double beta,
                     int kmax, double* frc, double* out, int nthreads) {
    double L[3] = {box[0], box[1], box[2]};
    double V = L[0] * L[1] * L[2];
    std::vector<double> pos(3 * (size_t)n);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++)
            pos[3 * (size_t)i + d] = (double)uc[3 * (size_t)i + d] * (L[d] / 4294967296.0);
    std::vector<std::array<int, 3>> ks;
    for (int a = -kmax; a <= kmax; a++)
        for (int b = -kmax; b <= kmax; b++)
            for (int c = 0; c <= kmax; c++) {
                if (c == 0 && (b < 0 || (b == 0 && a <= 0))) continue;  // half space, k != 0
                ks.push_back({a, b, c});
            }
    int t = nthreads_eff(nthreads);
    std::vector<std::vector<double>> fb(t);
    std::vector<double> eb(t, 0.0);
    parallel_for((long)ks.size(), t, [&](long bgn, long end, int k) {
        auto& f = fb[k];
        f.assign(3 * (size_t)n, 0.0);
        std::vector<double> cs(n), sn(n);
        for (long m = bgn; m < end; m++) {
            double kv[3] = {2 * M_PI * ks[m][0] / L[0], 2 * M_PI * ks[m][1] / L[1],
                            2 * M_PI * ks[m][2] / L[2]};
            double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
            // half space k > 0 counts each +-k pair once: E = sum_half 4 pi/(V k^2) e^{-k^2/4b^2} |S|^2
            double pref = 4 * M_PI / V * std::exp(-k2 / (4 * beta * beta)) / k2;
            double S_re = 0, S_im = 0;
            for (int i = 0; i < n; i++) {
                double ph = kv[0] * pos[3 * i] + kv[1] * pos[3 * i + 1] + kv[2] * pos[3 * i + 2];
                cs[i] = std::cos(ph);
                sn[i] = std::sin(ph);
                S_re += q[i] * cs[i];
                S_im += q[i] * sn[i];
            }
            eb[k] += pref * (S_re * S_re + S_im * S_im);
            for (int i = 0; i < n; i++) {
                double g = 2 * pref * q[i] * (sn[i] * S_re - cs[i] * S_im);
                for (int d = 0; d < 3; d++) f[3 * (size_t)i + d] += g * kv[d];
            }
        }
    });
    for (int k = 0; k < t; k++) {
        if (fb[k].empty()) continue;
        for (size_t x = 0; x < 3 * (size_t)n; x++) frc[x] += fb[k][x];
    }
    double e = 0;
    for (int k = 0; k < t; k++) e += eb[k];
    out[0] = e;
}

// Whole nonbonded evaluation for the CPU baseline: cell list + direct + exclusions + SPME.
// out[0..6] = E_lj, E_direct, E_corr, E_rec, E_self, LJ virial, in-cutoff pairs.
// Returns the number of pairs in the list (or -1 on allocation failure).
long orc_nonbonded(int n, const uint32_t* uc, const float* q, const int* type, const float* A12,
                   const float* B6, const float* box, float cutoff, float skin, double beta,
                   const int* K, const int* es, const int* en, const int* el, double* frc,
                   double* out, int nthreads) {
    long cap = (long)n * 1024;
    std::vector<int64_t> pairs;
    try {
        pairs.resize(cap);
    } catch (...) {
        return -1;
    }
    long np = orc_pairs_cells(n, uc, box, cutoff, skin, es, en, el, pairs.data(), cap, nthreads);
    if (np > cap) return -1;
    double d4[4], c1[1], r1[1];
    std::memset(frc, 0, sizeof(double) * 3 * (size_t)n);
    orc_direct(n, uc, q, type, A12, B6, box, cutoff, beta, pairs.data(), np, frc, nullptr, d4,
               nthreads);
    orc_excluded(n, uc, q, box, beta, es, en, el, frc, nullptr, c1);
    orc_pme(n, uc, q, box, K, beta, frc, r1, nullptr, nthreads);
    out[0] = d4[0];
    out[1] = d4[1];
    out[2] = c1[0];
    out[3] = r1[0];
    out[4] = orc_self_energy(n, q, beta, (double)box[0] * box[1] * box[2]);
    out[5] = d4[2];
    out[6] = d4[3];
    return np;
}

// ------------------------------------------------------------------------------------------
// FEP / TI: soft-core LJ + direct Coulomb (LJ_soft_core.cu:159-317 forces, :320-664 energies,
// :1137-1283 dH/dlambda) and the TI cross terms of PME (TI_core.cu:670-730)
// ------------------------------------------------------------------------------------------

// Over a half pair list, at coupling lambda: forces (accumulated into frc) and
// out[0] = E_LJ, out[1] = E_direct_coulomb, out[2] = dH/dlambda (LJ), out[3] = dH/dlambda
// (direct Coulomb, including the charge change dq = q_B - q_A at fixed geometry).
// q holds the charges at lambda. Tables are lower-triangular and scaled (x12, x6): AA/AB of
// the A state indexed by A types, BA/BB of the B state indexed by B types. A pair is soft-core
// when its two atoms differ in mask or when exactly one end state has LJ; then
//   r_A^6 = r^6 + alpha lambda^p sigma_A^6,  r_B^6 = r^6 + alpha (1-lambda)^p sigma_B^6,
//   E = (1-l) [AA/12 r_A^-12 - AB/6 r_A^-6 + qq erfc(b r_A)/r_A] + l [same with B and r_B],
// sigma^6 = max(AA/(2 AB), sigma_min^6) (sigma^6 if either coefficient vanishes); otherwise the
// tables are mixed linearly in lambda and r is not softened. dH/dlambda is the exact derivative
// of that energy (the soft-cored radii depend on lambda).
void orc_softcore(int n, const uint32_t* uc, const float* q, const float* dq, const int* ta,
                  const int* tb, const int* mask, const float* AA, const float* AB,
                  const float* BA, const float* BB, const float* box, float cutoff, double beta,
                  double lambda, double alpha, double p, double sigma6, double sigma6_min,
                  const int64_t* pairs, long npairs, double* frc, double* out) {
    float s[3];
    scaler_of(box, s);
    const float rc2 = cutoff * cutoff;
    const double tsp = 2.0 / std::sqrt(M_PI);
    const double l = lambda, l_ = 1.0 - lambda;
    const double cA0 = alpha * std::pow(l, p), cB0 = alpha * std::pow(l_, p);
    const double dcA0 = alpha * p * std::pow(l, p - 1.0), dcB0 = -alpha * p * std::pow(l_, p - 1.0);
    double elj = 0, edir = 0, hlj = 0, hdir = 0;
    for (long k = 0; k < npairs; k++) {
        const int i = (int)(pairs[k] / n), j = (int)(pairs[k] % n);
        const uint32_t* a = uc + 3 * (long)i;
        const uint32_t* c = uc + 3 * (long)j;
        if (!(pair_r2_f32(a[0], c[0], a[1], c[1], a[2], c[2], s) < rc2)) continue;
        double dr[3];
        dr_f64(a, c, s, dr);  // r_j - r_i
        const double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        const double r = std::sqrt(r2);
        const int pa = pair_type(ta[i], ta[j]), pb = pair_type(tb[i], tb[j]);
        const double Aa = AA[pa], Ab = AB[pa], Ba = BA[pb], Bb = BB[pb];
        const double qq = (double)q[i] * q[j];
        const double dqq = (double)dq[j] * q[i] + (double)q[j] * dq[i];
        const bool soft = mask[i] != mask[j] || (Ba > 1e-6 && Aa < 1e-6) || (Ba < 1e-6 && Aa > 1e-6);
        double fs;
        if (!soft) {
            const double ri2 = 1.0 / r2, ri6 = ri2 * ri2 * ri2;
            const double Am = l_ * Aa + l * Ba, Bm = l_ * Ab + l * Bb;
            const double flj = (-Am * ri6 + Bm) * ri6 * ri2;
            const double br = beta * r, ec = std::erfc(br);
            const double fc = qq * (br * tsp * std::exp(-br * br) + ec) * ri2 / r;
            fs = flj - fc;
            elj += (Am / 12.0 * ri6 - Bm / 6.0) * ri6;
            edir += qq * ec / r;
            hlj += ((Ba - Aa) / 12.0 * ri6 - (Bb - Ab) / 6.0) * ri6;
            hdir += dqq * ec / r;
        } else {
            const double r4 = r2 * r2, r6 = r4 * r2;
            const double sgA = (Aa < 1e-6 || Ab < 1e-6) ? sigma6 : std::max(0.5 * Aa / Ab, sigma6_min);
            const double sgB = (Ba < 1e-6 || Bb < 1e-6) ? sigma6 : std::max(0.5 * Ba / Bb, sigma6_min);
            const double sA = 1.0 / (r6 + cA0 * sgA), sB = 1.0 / (r6 + cB0 * sgB);
            const double rA = std::pow(r6 + cA0 * sgA, 1.0 / 6.0), rB = std::pow(r6 + cB0 * sgB, 1.0 / 6.0);
            const double flj = r4 * (l_ * (Ab - Aa * sA) * sA * sA + l * (Bb - Ba * sB) * sB * sB);
            const double gA = beta * tsp * std::exp(-beta * beta * rA * rA);
            const double gB = beta * tsp * std::exp(-beta * beta * rB * rB);
            const double phA = std::erfc(beta * rA) / rA, phB = std::erfc(beta * rB) / rB;
            const double fc = qq * r4 * (l_ * (gA + phA) * sA + l * (gB + phB) * sB);
            fs = flj - fc;
            const double EA = Aa / 12.0 * sA * sA - Ab / 6.0 * sA;
            const double EB = Ba / 12.0 * sB * sB - Bb / 6.0 * sB;
            elj += l_ * EA + l * EB;
            edir += qq * (l_ * phA + l * phB);
            const double dEA = (Aa / 6.0 * sA - Ab / 6.0) * (-sA * sA * dcA0 * sgA);
            const double dEB = (Ba / 6.0 * sB - Bb / 6.0) * (-sB * sB * dcB0 * sgB);
            hlj += EB - EA + l_ * dEA + l * dEB;
            const double dphA = -(gA + phA) * sA / 6.0 * dcA0 * sgA;
            const double dphB = -(gB + phB) * sB / 6.0 * dcB0 * sgB;
            hdir += qq * (phB - phA + l_ * dphA + l * dphB) + dqq * (l_ * phA + l * phB);
        }
        for (int d = 0; d < 3; d++) {
            frc[3 * (size_t)i + d] += fs * dr[d];
            frc[3 * (size_t)j + d] -= fs * dr[d];
        }
    }
    out[0] = elj;
    out[1] = edir;
    out[2] = hlj;
    out[3] = hdir;
}

// TI cross terms of PME for charges q (at lambda) changing by dq per unit lambda:
// out[0] = sum_i dq_i phi_i (reciprocal; phi the SPME potential of q at atom i),
// out[1] = d/dlambda of the self + neutralising energy, out[2] = d/dlambda of the exclusion
// correction energy at fixed geometry.
void orc_ti_cross(int n, const uint32_t* uc, const float* q, const float* dq, const float* box,
                  const int* K, double beta, const int* es, const int* en, const int* el,
                  double* out) {
    const size_t G = (size_t)K[0] * K[1] * K[2];
    std::vector<cplx> Q(G, cplx(0, 0));
    for (int i = 0; i < n; i++) {
        int b[3];
        double fr[3], w[3][4], dw[3][4];
        for (int d = 0; d < 3; d++) {
            grid_coord(uc[3 * (size_t)i + d], K[d], b[d], fr[d]);
            bspline4(fr[d], w[d], dw[d]);
        }
        for (int kx = 0; kx < 4; kx++)
            for (int ky = 0; ky < 4; ky++)
                for (int kz = 0; kz < 4; kz++) {
                    const int gx = ((b[0] - kx) % K[0] + K[0]) % K[0];
                    const int gy = ((b[1] - ky) % K[1] + K[1]) % K[1];
                    const int gz = ((b[2] - kz) % K[2] + K[2]) % K[2];
                    Q[((size_t)gx * K[1] + gy) * K[2] + gz] +=
                        (double)q[i] * w[0][kx] * w[1][ky] * w[2][kz];
                }
    }
    fft3(Q.data(), K, -1, 0);
    std::vector<double> bc;
    bc_table(K, box, beta, bc);
    for (size_t g = 0; g < G; g++) Q[g] *= bc[g];
    fft3(Q.data(), K, +1, 0);
    double rec = 0;
    for (int i = 0; i < n; i++) {
        int b[3];
        double fr[3], w[3][4], dw[3][4];
        for (int d = 0; d < 3; d++) {
            grid_coord(uc[3 * (size_t)i + d], K[d], b[d], fr[d]);
            bspline4(fr[d], w[d], dw[d]);
        }
        double phi = 0;
        for (int kx = 0; kx < 4; kx++)
            for (int ky = 0; ky < 4; ky++)
                for (int kz = 0; kz < 4; kz++) {
                    const int gx = ((b[0] - kx) % K[0] + K[0]) % K[0];
                    const int gy = ((b[1] - ky) % K[1] + K[1]) % K[1];
                    const int gz = ((b[2] - kz) % K[2] + K[2]) % K[2];
                    phi += w[0][kx] * w[1][ky] * w[2][kz] * Q[((size_t)gx * K[1] + gy) * K[2] + gz].real();
                }
        rec += (double)dq[i] * phi;
    }
    double sqq = 0, sq = 0, sdq = 0;
    for (int i = 0; i < n; i++) {
        sqq += (double)q[i] * dq[i];
        sq += q[i];
        sdq += dq[i];
    }
    const double V = (double)box[0] * box[1] * box[2];
    const double nf = -0.5 * M_PI / (beta * beta * V);
    float s[3];
    scaler_of(box, s);
    double corr = 0;
    for (int i = 0; i < n; i++)
        for (int k = es[i]; k < es[i] + en[i]; k++) {
            const int j = el[k];
            double dr[3];
            dr_f64(uc + 3 * (long)i, uc + 3 * (long)j, s, dr);
            const double r = std::sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
            corr -= ((double)q[i] * dq[j] + (double)dq[i] * q[j]) * std::erf(beta * r) / r;
        }
    out[0] = rec;
    out[1] = -2.0 * beta / std::sqrt(M_PI) * sqq + 2.0 * nf * sq * sdq;
    out[2] = corr;
}

// 1-4 pairs in FP64 (nb14.cu:92-170): dr = r_b - r_a (minimum image); F/r = -A r^-14 + B r^-8
// - cf q_a q_b r^-3 with charges below 1e-10 clamped to 1e-10 (nb14.cu:77-82); F r_hat added to
// a and subtracted from b; E = cf q_a q_b / r + A/12 r^-12 - B/6 r^-6 and the virial -F.dr to
// atom a. out[0] = sum of the LJ parts, out[1] = sum of the Coulomb parts.
void orc_nb14(int n, int n14, const uint32_t* uc, const float* q, const float* box,
              const int* a14, const int* b14, const float* A, const float* B, const float* cf,
              double* frc, double* atom_energy, double* atom_virial, double* out) {
    float s[3];
    scaler_of(box, s);
    double elj = 0.0, ecf = 0.0;
    for (int p = 0; p < n14; p++) {
        const int i = a14[p], j = b14[p];
        double dr[3];
        dr_f64(uc + 3 * (size_t)i, uc + 3 * (size_t)j, s, dr);
        const double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        const double ri2 = 1.0 / r2, ri = std::sqrt(ri2);
        double qi = q[i], qj = q[j];
        if (std::fabs(qi) < 1e-10) qi = (double)1e-10f;
        if (std::fabs(qj) < 1e-10) qj = (double)1e-10f;
        const double ri6 = ri2 * ri2 * ri2;
        const double fs = -(double)A[p] * ri6 * ri6 * ri2 + (double)B[p] * ri6 * ri2 -
                          (double)cf[p] * qi * qj * ri2 * ri;
        for (int d = 0; d < 3; d++) {
            frc[3 * (size_t)i + d] += fs * dr[d];
            frc[3 * (size_t)j + d] -= fs * dr[d];
        }
        const double el = (double)A[p] / 12.0 * ri6 * ri6 - (double)B[p] / 6.0 * ri6;
        const double ec = (double)cf[p] * qi * qj * ri;
        atom_energy[i] += el + ec;
        atom_virial[i] -= fs * r2;
        elj += el;
        ecf += ec;
    }
    out[0] = elj;
    out[1] = ecf;
}

// Virtual atoms in FP64. Records: type[v], atoms[4v..4v+3] = {virtual, from_1, from_2, from_3},
// param[2v..2v+1] as the input line gives them (type 0: h; 1: a; 2: a, b; 3: d, k); level[]
// gives each record's level (1 = built from real atoms only). Displacements are the minimum-image
// ones of the fixed-point coordinates, positions are the parent's position plus the displacement
// (virtual_atoms.cu:2-73). mode 0: refresh crd (lowest level first); mode 1: move each virtual
// atom's force to its parents and zero it (highest level first, virtual_atoms.cu:75-180).
static void vs_dr(const uint32_t* uc, int from, int to, const float s[3], double d[3]) {
    dr_f64(uc + 3 * (size_t)from, uc + 3 * (size_t)to, s, d);
}

void orc_vsite(int nv, const int* type, const int* atoms, const float* param, const int* level,
               int maxlevel, const uint32_t* uc, const float* box, int mode, double* crd,
               double* frc) {
    float s[3];
    scaler_of(box, s);
    for (int li = 0; li < maxlevel; li++) {
        const int L = mode == 0 ? li + 1 : maxlevel - li;
        for (int r = 0; r < nv; r++) {
            if (level[r] != L) continue;
            const int t = type[r];
            const int v = atoms[4 * r], f1 = atoms[4 * r + 1], f2 = atoms[4 * r + 2],
                      f3 = atoms[4 * r + 3];
            const double p0 = param[2 * r], p1 = param[2 * r + 1];
            if (mode == 0) {
                double x[3] = {crd[3 * (size_t)f1], crd[3 * (size_t)f1 + 1], crd[3 * (size_t)f1 + 2]};
                if (t == 0) {
                    x[2] = 2.0 * p0 - x[2];  // mirror in the plane z = h
                } else if (t == 1) {
                    double d[3];
                    vs_dr(uc, f1, f2, s, d);
                    for (int k = 0; k < 3; k++) x[k] += p0 * d[k];
                } else if (t == 2) {
                    double d1[3], d2[3];
                    vs_dr(uc, f1, f2, s, d1);
                    vs_dr(uc, f1, f3, s, d2);
                    for (int k = 0; k < 3; k++) x[k] += p0 * d1[k] + p1 * d2[k];
                } else {
                    double r21[3], r32[3], tt[3];
                    vs_dr(uc, f1, f2, s, r21);
                    vs_dr(uc, f2, f3, s, r32);
                    for (int k = 0; k < 3; k++) tt[k] = r21[k] + p1 * r32[k];
                    const double f = p0 / std::sqrt(tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2]);
                    for (int k = 0; k < 3; k++) x[k] += f * tt[k];
                }
                for (int k = 0; k < 3; k++) crd[3 * (size_t)v + k] = x[k];
            } else {
                double fv[3] = {frc[3 * (size_t)v], frc[3 * (size_t)v + 1], frc[3 * (size_t)v + 2]};
                if (t == 0) {
                    frc[3 * (size_t)f1] += fv[0];
                    frc[3 * (size_t)f1 + 1] += fv[1];
                    frc[3 * (size_t)f1 + 2] -= fv[2];
                } else if (t == 1) {
                    for (int k = 0; k < 3; k++) {
                        frc[3 * (size_t)f1 + k] += p0 * fv[k];
                        frc[3 * (size_t)f2 + k] += (1.0 - p0) * fv[k];
                    }
                } else if (t == 2) {
                    for (int k = 0; k < 3; k++) {
                        frc[3 * (size_t)f1 + k] += (1.0 - p0 - p1) * fv[k];
                        frc[3 * (size_t)f2 + k] += p0 * fv[k];
                        frc[3 * (size_t)f3 + k] += p1 * fv[k];
                    }
                } else {
                    double r21[3], r32[3], rv1[3], tt[3];
                    vs_dr(uc, f1, f2, s, r21);
                    vs_dr(uc, f2, f3, s, r32);
                    vs_dr(uc, f1, v, s, rv1);
                    for (int k = 0; k < 3; k++) tt[k] = r21[k] + p1 * r32[k];
                    const double factor =
                        p0 / std::sqrt(tt[0] * tt[0] + tt[1] * tt[1] + tt[2] * tt[2]);
                    const double proj = (rv1[0] * fv[0] + rv1[1] * fv[1] + rv1[2] * fv[2]) /
                                        (rv1[0] * rv1[0] + rv1[1] * rv1[1] + rv1[2] * rv1[2]);
                    for (int k = 0; k < 3; k++) {
                        const double tk = factor * (fv[k] - proj * rv1[k]);
                        frc[3 * (size_t)f1 + k] += fv[k] - tk;
                        frc[3 * (size_t)f2 + k] += (1.0 - p1) * tk;
                        frc[3 * (size_t)f3 + k] += p1 * tk;
                    }
                }
                for (int k = 0; k < 3; k++) frc[3 * (size_t)v + k] = 0.0;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// NVE leap-frog + SETTLE in FP64 (one step): crd, vel updated in place; acc written; the
// constraint virial sum returned in out[0]. Constraint pairs (i, j, r) in CONSTRAIN's order.
// ---------------------------------------------------------------------------------------------
struct OTri { int A, B, C; double ra, rb, rc, rd, re; };
struct OPair { int i, j; double r, k; };

static void o_rabcde(double rAB, double rAC, double rBC, double mA, double mB, double mC,
                     double& ra, double& rb, double& rc, double& rd, double& re) {
    const double mT = mA + mB + mC;
    double Ax = 0, Ay = 0, Bx = -rAB, By = 0;
    double c = (rBC * rBC - rAC * rAC - rAB * rAB) / (2 * rAC * rAB);
    double Cx = rAC * c, Cy = rAC * std::sqrt(1.0 - c * c);
    const double Ox = (Bx * mB + Cx * mC) / mT, Oy = Cy * mC / mT;
    Ax -= Ox; Ay -= Oy; Bx -= Ox; By -= Oy; Cx -= Ox; Cy -= Oy;
    c = 1.0 / std::sqrt(1.0 + Ax * Ax / Ay / Ay);
    const double sn = c * Ax / Ay;
    ra = Ax * sn + Ay * c;
    rc = Bx * c - By * sn;
    rb = Bx * sn + By * c;
    rd = Cx * c - Cy * sn;
    re = Cx * sn + Cy * c;
    if (ra < 0) { ra = -ra; rb = -rb; re = -re; }
}

static inline void o_fdisp(const double* a, const double* b, const double* L, double d[3]) {
    for (int k = 0; k < 3; k++) {
        d[k] = a[k] - b[k];
        d[k] -= std::floor(d[k] / L[k] + 0.5) * L[k];
    }
}
static inline void o_cross(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double o_dot(const double* a, const double* b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline void o_unit(double* a) {
    const double r = 1.0 / std::sqrt(o_dot(a, a));
    for (int k = 0; k < 3; k++) a[k] *= r;
}

int orc_nve_settle(int n, int np, const int* pi, const int* pj, const float* pr,
                   const float* mass, const uint32_t* uc, const float* box, double dt,
                   double exp_gamma, const double* frc, double* crd, double* vel, double* acc,
                   double* out) {
    // SETTLE::Initial (SETTLE.cu:194-305)
    std::vector<int> num(n, 0), link(2 * (size_t)n, -1);
    std::vector<double> lr(3 * (size_t)n, 0.0);
    for (int p = 0; p < np; p++) {
        const int a = pi[p], b = pj[p];
        if (num[a] < 2 && num[b] < 2) {
            link[2 * a + num[a]] = b; link[2 * b + num[b]] = a;
            lr[3 * a + num[a]] = pr[p]; lr[3 * b + num[b]] = pr[p];
            num[a]++; num[b]++;
        } else { num[a] = 3; num[b] = 3; }
    }
    for (int i = 0; i < n; i++) {
        if (num[i] == 2) {
            const int a = link[2 * i], b = link[2 * i + 1];
            if (num[a] == 2 && num[b] == 2 &&
                ((link[2 * a] == i && link[2 * a + 1] == b) || (link[2 * a + 1] == i && link[2 * a] == b))) {
                num[a] = -2; num[b] = -2;
                lr[3 * i + 2] = link[2 * a + 1] == b ? lr[3 * a + 1] : lr[3 * a];
            } else { num[i] = 3; num[a] = 3; num[b] = 3; }
        } else if (num[i] == 1) {
            const int a = link[2 * i];
            if (num[a] == 1) num[a] = -1;
            else { num[i] = 3; num[a] = 3; }
        }
    }
    std::vector<OTri> tri;
    std::vector<OPair> prs;
    for (int i = 0; i < n; i++) {
        if (num[i] == 2) {
            OTri T;
            T.A = i; T.B = link[2 * i]; T.C = link[2 * i + 1];
            o_rabcde(lr[3 * i], lr[3 * i + 1], lr[3 * i + 2], mass[T.A], mass[T.B], mass[T.C],
                     T.ra, T.rb, T.rc, T.rd, T.re);
            tri.push_back(T);
            num[i] = -2;
        }
        if (num[i] == 1) {
            OPair P;
            P.i = i; P.j = link[2 * i]; P.r = lr[3 * i];
            P.k = 1.0 / ((double)mass[P.i] + (double)mass[P.j]);
            prs.push_back(P);
            num[i] = -1;
        }
    }
    float s[3];
    scaler_of(box, s);
    const double L[3] = {box[0], box[1], box[2]};
    // Remember_Last_Coordinates (SETTLE.cu:355-395)
    std::vector<double> last(6 * tri.size() + 3 * prs.size());
    for (size_t t = 0; t < tri.size(); t++) {
        dr_f64(uc + 3 * (size_t)tri[t].A, uc + 3 * (size_t)tri[t].B, s, &last[6 * t]);
        dr_f64(uc + 3 * (size_t)tri[t].A, uc + 3 * (size_t)tri[t].C, s, &last[6 * t + 3]);
    }
    for (size_t p = 0; p < prs.size(); p++)
        dr_f64(uc + 3 * (size_t)prs[p].i, uc + 3 * (size_t)prs[p].j, s, &last[6 * tri.size() + 3 * p]);
    // leap-frog (MD_core.cu:13-32)
    for (int i = 0; i < n; i++) {
        const double im = mass[i] > 0 ? 1.0 / (double)mass[i] : 0.0;
        for (int k = 0; k < 3; k++) {
            const double a = im * frc[3 * (size_t)i + k];
            acc[3 * (size_t)i + k] = a;
            vel[3 * (size_t)i + k] += dt * a;
            crd[3 * (size_t)i + k] += dt * vel[3 * (size_t)i + k];
        }
    }
    const double vf = exp_gamma, xf = 0.5 * (1.0 + exp_gamma);
    double vir = 0.0;
    // settle_pair (SETTLE.cu:381-414)
    for (size_t p = 0; p < prs.size(); p++) {
        const OPair& P = prs[p];
        const double* r2 = &last[6 * tri.size() + 3 * p];
        double r1[3];
        o_fdisp(&crd[3 * (size_t)P.j], &crd[3 * (size_t)P.i], L, r1);
        const double mA = mass[P.i], mB = mass[P.j];
        const double r0r0 = P.r * P.r, r1r1 = o_dot(r1, r1), r1r2 = o_dot(r1, r2), r2r2 = o_dot(r2, r2);
        const double k = (std::sqrt(r1r2 * r1r2 - r1r1 * r2r2 + r2r2 * r0r0) - r1r2) / r2r2;
        const double kv = vf / dt / xf;
        for (int d = 0; d < 3; d++) {
            const double kr2 = k * r2[d];
            const double di = -mB * P.k * kr2, dj = mA * P.k * kr2;
            crd[3 * (size_t)P.i + d] += di;
            crd[3 * (size_t)P.j + d] += dj;
            vel[3 * (size_t)P.i + d] += kv * di;
            vel[3 * (size_t)P.j + d] += kv * dj;
            vir += (kv * mB / dt / vf * dj) * r2[d];
        }
    }
    // settle_triangle (SETTLE.cu:349-380) + SETTLE_DO_TRIANGLE (:93-176)
    for (size_t t = 0; t < tri.size(); t++) {
        const OTri& T = tri[t];
        const double* rB0 = &last[6 * t];
        const double* rC0 = &last[6 * t + 3];
        double rA[3], rB[3], rC[3], rO[3];
        for (int d = 0; d < 3; d++) rA[d] = crd[3 * (size_t)T.A + d];
        o_fdisp(&crd[3 * (size_t)T.B], rA, L, rB);
        o_fdisp(&crd[3 * (size_t)T.C], rA, L, rC);
        const double mA = mass[T.A], mB = mass[T.B], mC = mass[T.C];
        for (int d = 0; d < 3; d++) {
            rO[d] = (mB * rB[d] + mC * rC[d]) / (mA + mB + mC) + rA[d];
            rA[d] -= rO[d];
            rB[d] += rA[d];
            rC[d] += rA[d];
        }
        double bz[3], bx[3], by[3];
        o_cross(rB0, rC0, bz);
        o_cross(rA, bz, bx);
        o_cross(bz, bx, by);
        o_unit(bx); o_unit(by); o_unit(bz);
        const double B0x = o_dot(bx, rB0), B0y = o_dot(by, rB0);
        const double C0x = o_dot(bx, rC0), C0y = o_dot(by, rC0);
        const double A1z = o_dot(bz, rA);
        const double B1x = o_dot(bx, rB), B1y = o_dot(by, rB), B1z = o_dot(bz, rB);
        const double C1x = o_dot(bx, rC), C1y = o_dot(by, rC), C1z = o_dot(bz, rC);
        const double sinphi = A1z / T.ra, cosphi = std::sqrt(1.0 - sinphi * sinphi);
        const double sinpsi = (B1z - C1z - (T.rb - T.re) * sinphi) / ((T.rd - T.rc) * cosphi);
        const double cospsi = std::sqrt(1.0 - sinpsi * sinpsi);
        const double A2y = T.ra * cosphi;
        const double B2x = T.rc * cospsi, B2y = T.rb * cosphi + T.rc * sinpsi * sinphi;
        const double C2x = T.rd * cospsi, C2y = T.re * cosphi + T.rd * sinpsi * sinphi;
        const double alpha = B2x * B0x + C2x * C0x + B2y * B0y + C2y * C0y;
        const double beta = -B2x * B0y - C2x * C0y + B2y * B0x + C2y * C0x;
        const double gamma = B1y * B0x - B1x * B0y + C1y * C0x - C1x * C0y;
        const double ab = alpha * alpha + beta * beta;
        const double st = (alpha * gamma - beta * std::sqrt(ab - gamma * gamma)) / ab;
        const double ct = std::sqrt(1.0 - st * st);
        const double A3[3] = {-A2y * st, A2y * ct, A1z};
        const double B3[3] = {B2x * ct - B2y * st, B2x * st + B2y * ct, B1z};
        const double C3[3] = {C2x * ct - C2y * st, C2x * st + C2y * ct, C1z};
        double nA[3], nB[3], nC[3];
        for (int d = 0; d < 3; d++) {
            nA[d] = A3[0] * bx[d] + A3[1] * by[d] + A3[2] * bz[d];
            nB[d] = B3[0] * bx[d] + B3[1] * by[d] + B3[2] * bz[d];
            nC[d] = C3[0] * bx[d] + C3[1] * by[d] + C3[2] * bz[d];
        }
        const double kv = vf / dt / xf, kf = 1.0 / dt / dt / xf;
        for (int d = 0; d < 3; d++) {
            vel[3 * (size_t)T.A + d] += kv * (nA[d] - rA[d]);
            vel[3 * (size_t)T.B + d] += kv * (nB[d] - rB[d]);
            vel[3 * (size_t)T.C + d] += kv * (nC[d] - rC[d]);
            vir += kf * mB * (nB[d] - rB[d]) * rB0[d] + kf * mC * (nC[d] - rC[d]) * rC0[d];
            crd[3 * (size_t)T.A + d] = nA[d] + rO[d];
            crd[3 * (size_t)T.B + d] = nB[d] + rO[d];
            crd[3 * (size_t)T.C + d] = nC[d] + rO[d];
        }
    }
    out[0] = vir;
    out[1] = (double)tri.size();
    out[2] = (double)prs.size();
    return 0;
}

}  // extern "C"

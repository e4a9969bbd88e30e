// Register-resident line FFTs for the PME passes — included by sb_fft.cu.
//
// A line of N = N1 * N2 points is transformed in two passes through shared memory ("four
// step"): in pass 1, thread n2 of the line holds the N1 points n2 + N2 n1 in registers, runs an
// N1-point DFT, multiplies by W_N^(n2 k1) and writes the results back to the same positions; in
// pass 2, thread k1 holds the N2 points N2 k1 + n2, runs an N2-point DFT and writes X[k1 + N1 k2].
// The small DFTs are fully unrolled (mixed radix 2/3/4/5/7, decimation in time, every index a
// compile-time constant) with twiddles from a constant-memory table, so a point costs a few tens
// of instructions instead of the generic stage loops' index arithmetic and per-stage shared-memory
// round trips. Input and output are in natural order. Transforms are unnormalised.
#pragma once

// e^{-2 pi i k / n} for 2 <= n <= SB_SMALL_N, k < n, at offset n (n - 1) / 2 - 1
#define SB_SMALL_N 20
#define SB_SMALL_TW (SB_SMALL_N * (SB_SMALL_N + 1) / 2 - 1)
__constant__ float2 c_small_tw[SB_SMALL_TW];

template <int N, bool INV>
__device__ __forceinline__ float2 stw(int k) {
    const float2 w = c_small_tw[N * (N - 1) / 2 - 1 + (k % N)];
    return INV ? make_float2(w.x, -w.y) : w;
}

__host__ __device__ constexpr int sb_spf(int n) {
    return n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n % 5 == 0 ? 5 : n % 7 == 0 ? 7 : n;
}

// Every product that meets a sum is written out as an explicit fused multiply-add or an unfused
// multiply (__fmul_rn), so the compiler has no contraction to choose: the plane kernel and the
// pass-by-pass kernels, which inline these helpers in different surroundings, round alike.
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -__fmul_rn(a.y, b.y)), fmaf(a.x, b.y, __fmul_rn(a.y, b.x)));
}

// in-place N-point DFT of x (natural order in and out)
template <int N, bool INV>
__device__ __forceinline__ void rdft(float2 (&x)[N]) {
    if constexpr (N == 1) {
    } else if constexpr (N == 2) {
        const float2 a = x[0], b = x[1];
        x[0] = make_float2(a.x + b.x, a.y + b.y);
        x[1] = make_float2(a.x - b.x, a.y - b.y);
    } else if constexpr (N == 4) {
        const float2 a = x[0], b = x[1], c = x[2], d = x[3];
        const float2 s0 = make_float2(a.x + c.x, a.y + c.y), s1 = make_float2(a.x - c.x, a.y - c.y);
        const float2 s2 = make_float2(b.x + d.x, b.y + d.y), s3 = make_float2(b.x - d.x, b.y - d.y);
        // -i s3 forward, +i s3 inverse
        const float2 j3 = INV ? make_float2(-s3.y, s3.x) : make_float2(s3.y, -s3.x);
        x[0] = make_float2(s0.x + s2.x, s0.y + s2.y);
        x[2] = make_float2(s0.x - s2.x, s0.y - s2.y);
        x[1] = make_float2(s1.x + j3.x, s1.y + j3.y);
        x[3] = make_float2(s1.x - j3.x, s1.y - j3.y);
    } else if constexpr (N == 3) {
        const float c = -0.5f, s = INV ? -0.86602540378443865f : 0.86602540378443865f;
        const float2 a = x[0], b = x[1], d = x[2];
        const float2 t1 = make_float2(b.x + d.x, b.y + d.y), t2 = make_float2(b.x - d.x, b.y - d.y);
        const float2 m = make_float2(fmaf(c, t1.x, a.x), fmaf(c, t1.y, a.y));
        const float2 st = make_float2(__fmul_rn(s, t2.y), __fmul_rn(-s, t2.x));
        x[0] = make_float2(a.x + t1.x, a.y + t1.y);
        x[1] = make_float2(m.x + st.x, m.y + st.y);
        x[2] = make_float2(m.x - st.x, m.y - st.y);
    } else if constexpr (N == 5 || N == 7) {
        // prime: direct sum with table twiddles (symmetric pairs share the real parts)
        float2 y[N];
#pragma unroll
        for (int q = 0; q < N; q++) {
            float2 acc = x[0];
#pragma unroll
            for (int j = 1; j < N; j++) {
                const float2 t = c_mul(x[j], stw<N, INV>(j * q));
                acc.x += t.x;
                acc.y += t.y;
            }
            y[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < N; q++) x[q] = y[q];
    } else {
        constexpr int P = sb_spf(N), M = N / P;
        float2 y[P][M];
#pragma unroll
        for (int p = 0; p < P; p++)
#pragma unroll
            for (int m = 0; m < M; m++) y[p][m] = x[m * P + p];
#pragma unroll
        for (int p = 0; p < P; p++) rdft<M, INV>(y[p]);
#pragma unroll
        for (int k = 0; k < M; k++) {
            float2 z[P];
#pragma unroll
            for (int p = 0; p < P; p++) z[p] = (p * k) % N == 0 ? y[p][k] : c_mul(y[p][k], stw<N, INV>(p * k));
            rdft<P, INV>(z);
#pragma unroll
            for (int q = 0; q < P; q++) x[k + M * q] = z[q];
        }
    }
}

// NL lines of N1*N2 points in shared memory, point e of line l at buf[l * ls + e * es]; twN holds
// W_N^k (forward sign), k < N. All threads of the block take part; one barrier inside and one at
// the end.
template <int N1, int N2, int NL, bool INV>
__device__ __forceinline__ void line_fft4(float2* buf, int ls, int es, const float2* twN) {
    constexpr int N = N1 * N2;
    // pass 1: (line, n2) items
    for (int t = threadIdx.x; t < NL * N2; t += blockDim.x) {
        const int l = t % NL, n2 = t / NL;
        float2* p = buf + l * ls + n2 * es;
        float2 x[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) x[n1] = p[n1 * N2 * es];
        rdft<N1, INV>(x);
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) {
            float2 w = twN[(n2 * k1) % N];
            if (INV) w.y = -w.y;
            p[k1 * N2 * es] = k1 == 0 ? x[0] : c_mul(x[k1], w);
        }
    }
    __syncthreads();
    // pass 2: one (line, k1) item per thread (the launch gives at least NL * N1 threads); every
    // item reads its points before any item writes, since the written set differs
    const int t = threadIdx.x;
    const bool live = t < NL * N1;
    const int l = t % NL, k1 = t / NL;
    float2 y[N2];
    if (live) {
        const float2* p = buf + l * ls + k1 * N2 * es;
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) y[n2] = p[n2 * es];
        rdft<N2, INV>(y);
    }
    __syncthreads();
    if (live) {
        float2* p = buf + l * ls + k1 * es;
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) p[k2 * N1 * es] = y[k2];
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// passes built on line_fft4 (natural order throughout; same data layout as the generic passes)
// ---------------------------------------------------------------------------------------------
#define SB_F4_NL 16  // lines per block of the y and x passes
#define SB_F4_ZR 32  // rows per block of the z passes

template <int N1, int N2>
struct F4 {
    static constexpr int N = N1 * N2;
    static constexpr int T = N1 > N2 ? N1 : N2;  // threads per line
};

// Global loads and stores of the passes run as unrolled loops with a compile-time trip count
// (the tile divides evenly among the threads), so that a thread issues all of its loads before
// the first use and one memory latency covers the tile.

template <int N1, int N2, bool INV>
__global__ void __launch_bounds__(SB_F4_NL * F4<N1, N2>::T) k_ypass4(
    const float2* __restrict__ twy, float2* __restrict__ spec, int K0, int H,
    const SbFftBatchIo* __restrict__ bio) {
    constexpr int K1 = N1 * N2, NL = SB_F4_NL, NT = NL * F4<N1, N2>::T, IT = K1 * NL / NT;
    static_assert(K1 * NL % NT == 0, "tile must divide among the threads");
    if (bio) spec = bio[blockIdx.y].spec;
    __shared__ float2 tw[K1];
    __shared__ float2 D[K1 * NL];
    __shared__ long long cbase[NL];
    const int nlines = K0 * H;
    const int l0 = blockIdx.x * NL;
    for (int t = threadIdx.x; t < K1; t += NT) tw[t] = twy[t];
    if (threadIdx.x < NL) {
        const int l = l0 + threadIdx.x;
        const int x = l / H, kz = l - x * H;
        cbase[threadIdx.x] = l < nlines ? (long long)x * K1 * H + kz : -1;
    }
    __syncthreads();
    {
        float2 r[IT];
#pragma unroll
        for (int i = 0; i < IT; i++) {
            const int t = threadIdx.x + i * NT;
            const int p = t / NL, c = t - p * NL;
            const long long cb = cbase[c];
            r[i] = cb >= 0 ? spec[cb + (size_t)p * H] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < IT; i++) D[threadIdx.x + i * NT] = r[i];
    }
    __syncthreads();
    line_fft4<N1, N2, NL, INV>(D, 1, NL, tw);
#pragma unroll
    for (int i = 0; i < IT; i++) {
        const int t = threadIdx.x + i * NT;
        const int p = t / NL, c = t - p * NL;
        const long long cb = cbase[c];
        if (cb >= 0) spec[cb + (size_t)p * H] = D[t];
    }
}

template <int N1, int N2>
__global__ void __launch_bounds__(SB_F4_NL * F4<N1, N2>::T) k_xconv4(
    const float2* __restrict__ twx, float2* __restrict__ spec, const float* __restrict__ bc,
    double* __restrict__ epart, int K1, int H, int K2, const SbFftBatchIo* __restrict__ bio) {
    constexpr int K0 = N1 * N2, NL = SB_F4_NL, NT = NL * F4<N1, N2>::T, IT = K0 * NL / NT;
    static_assert(K0 * NL % NT == 0, "tile must divide among the threads");
    if (bio) {
        spec = bio[blockIdx.y].spec;
        bc = bio[blockIdx.y].bc;
        epart = bio[blockIdx.y].epart;
    }
    __shared__ float2 tw[K0];
    __shared__ float2 D[K0 * NL];
    __shared__ int cbase[NL], ckz[NL];
    __shared__ double red[NT];
    const int nlines = K1 * H;
    const int l0 = blockIdx.x * NL;
    for (int t = threadIdx.x; t < K0; t += NT) tw[t] = twx[t];
    if (threadIdx.x < NL) {
        const int l = l0 + threadIdx.x;
        const int y = l / H, kz = l - y * H;
        cbase[threadIdx.x] = l < nlines ? y * H + kz : -1;
        ckz[threadIdx.x] = kz;
    }
    __syncthreads();
    const size_t pstride = (size_t)K1 * H;
    // the Green's function values of this thread's points, loaded with the spectrum
    float g[IT];
    {
        float2 r[IT];
#pragma unroll
        for (int i = 0; i < IT; i++) {
            const int t = threadIdx.x + i * NT;
            const int p = t / NL, c = t - p * NL;
            const int cb = cbase[c];
            r[i] = cb >= 0 ? spec[(size_t)p * pstride + cb] : make_float2(0.f, 0.f);
            g[i] = cb >= 0 ? bc[(size_t)p * pstride + cb] : 0.f;
        }
#pragma unroll
        for (int i = 0; i < IT; i++) D[threadIdx.x + i * NT] = r[i];
    }
    __syncthreads();
    line_fft4<N1, N2, NL, false>(D, 1, NL, tw);
    double e = 0.0;
#pragma unroll
    for (int i = 0; i < IT; i++) {
        const int t = threadIdx.x + i * NT;
        const int c = t % NL;
        if (cbase[c] >= 0) {
            const float2 v = D[t];
            if (epart) {
                const int kz = ckz[c];
                const double w = (kz == 0 || 2 * kz == K2) ? 1.0 : 2.0;
                e += w * (double)g[i] * ((double)v.x * v.x + (double)v.y * v.y);
            }
            D[t] = make_float2(v.x * g[i], v.y * g[i]);
        }
    }
    __syncthreads();
    line_fft4<N1, N2, NL, true>(D, 1, NL, tw);
#pragma unroll
    for (int i = 0; i < IT; i++) {
        const int t = threadIdx.x + i * NT;
        const int p = t / NL, c = t - p * NL;
        const int cb = cbase[c];
        if (cb >= 0) spec[(size_t)p * pstride + cb] = D[t];
    }
    if (epart) {
        // deterministic block reduction (fixed tree over a power-of-two prefix)
        red[threadIdx.x] = e;
        __syncthreads();
        int m = 1;
        while (m * 2 <= NT) m *= 2;
        if (threadIdx.x >= m) red[threadIdx.x - m] += red[threadIdx.x];
        __syncthreads();
        for (int o = m / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) epart[blockIdx.x] = 0.5 * red[0];
    }
}

// real-to-complex along z: int64 grid rows (cleared behind) -> half-spectrum rows; with TR the
// spectrum is stored plane by plane ([kz][row], for k_plane4) instead of row by row ([row][kz])
template <int N1, int N2, bool TR>
__global__ void __launch_bounds__(SB_F4_ZR * F4<N1, N2>::T) k_zfwd4(
    const float2* __restrict__ twz, const float2* __restrict__ post,
    long long* __restrict__ qfix, float2* __restrict__ spec, int nrows,
    const SbFftBatchIo* __restrict__ bio) {
    constexpr int M = N1 * N2, K2 = 2 * M, H = M + 1, NL = SB_F4_ZR;
    constexpr int NT = NL * F4<N1, N2>::T, IT = NL * K2 / NT, ITO = (NL * H + NT - 1) / NT;
    static_assert(NL * K2 % NT == 0, "tile must divide among the threads");
    if (bio) {
        qfix = bio[blockIdx.y].qfix;
        spec = bio[blockIdx.y].spec;
    }
    __shared__ float2 tw[M], ps[M];
    __shared__ float2 D[NL * H];
    float* Df = reinterpret_cast<float*>(D);
    for (int t = threadIdx.x; t < M; t += NT) {
        tw[t] = twz[t];
        ps[t] = post[t];
    }
    const int r0 = blockIdx.x * NL;
    const int nr = min(NL, nrows - r0);
    long long* q = qfix + (size_t)r0 * K2;
    {
        long long v[IT];
#pragma unroll
        for (int i = 0; i < IT; i++) {
            const int t = threadIdx.x + i * NT;
            v[i] = t < nr * K2 ? q[t] : 0ll;
        }
#pragma unroll
        for (int i = 0; i < IT; i++) {
            const int t = threadIdx.x + i * NT;
            const int r = t / K2, col = t - r * K2;
            if (v[i]) q[t] = 0;  // the grid is left zero for the next spread
            Df[2 * r * H + col] = (float)v[i] * SB_GRID_UNSCALE;
        }
    }
    __syncthreads();
    line_fft4<N1, N2, NL, false>(D, H, 1, tw);
    // X[k] = E[k] + W_K2^k O[k], k = 0..M, from Z = FFT_M(x_even + i x_odd)
    constexpr int half = M / 2;
    for (int t = threadIdx.x; t < NL * (half + 1); t += NT) {
        const int k = t / NL, r = t - k * NL;
        float2* row = D + r * H;
        if (k == 0) {
            const float2 z0 = row[0];
            row[0] = make_float2(z0.x + z0.y, 0.f);
            row[M] = make_float2(z0.x - z0.y, 0.f);
        } else {
            const int k2 = M - k;
            const float2 a = row[k], b = row[k2];
            const float2 Ek = make_float2(__fmul_rn(0.5f, a.x + b.x), __fmul_rn(0.5f, a.y - b.y));
            const float2 Ok = make_float2(__fmul_rn(0.5f, a.y + b.y), __fmul_rn(-0.5f, a.x - b.x));
            const float2 pk = ps[k];
            const float2 pO = c_mul(pk, Ok);
            const float2 Xk = make_float2(Ek.x + pO.x, Ek.y + pO.y);
            if (k2 != k) {
                const float2 w2 = make_float2(-pk.x, pk.y);
                const float2 cE = make_float2(Ek.x, -Ek.y), cO = make_float2(Ok.x, -Ok.y);
                const float2 wO = c_mul(w2, cO);
                row[k2] = make_float2(cE.x + wO.x, cE.y + wO.y);
            }
            row[k] = Xk;
        }
    }
    __syncthreads();
    if (TR) {
        // consecutive threads take consecutive rows of one kz plane (coalesced)
#pragma unroll
        for (int i = 0; i < ITO; i++) {
            const int t = threadIdx.x + i * NT;
            const int kz = t / NL, r = t - kz * NL;
            if (t < NL * H && r < nr) spec[(size_t)kz * nrows + r0 + r] = D[r * H + kz];
        }
    } else {
        float2* out = spec + (size_t)r0 * H;
#pragma unroll
        for (int i = 0; i < ITO; i++) {
            const int t = threadIdx.x + i * NT;
            if (t < nr * H) out[t] = D[t];
        }
    }
}

// complex-to-real along z: half-spectrum rows -> real rows (TR: spectrum stored plane by plane)
template <int N1, int N2, bool TR>
__global__ void __launch_bounds__(SB_F4_ZR * F4<N1, N2>::T) k_zinv4(
    const float2* __restrict__ twz, const float2* __restrict__ post,
    const float2* __restrict__ spec, float* __restrict__ real, int nrows,
    const SbFftBatchIo* __restrict__ bio) {
    constexpr int M = N1 * N2, K2 = 2 * M, H = M + 1, NL = SB_F4_ZR;
    constexpr int NT = NL * F4<N1, N2>::T, ITI = (NL * H + NT - 1) / NT, IT = NL * K2 / NT;
    static_assert(NL * K2 % NT == 0, "tile must divide among the threads");
    if (bio) {
        spec = bio[blockIdx.y].spec;
        real = bio[blockIdx.y].real;
    }
    __shared__ float2 tw[M], ps[M];
    __shared__ float2 D[NL * H];
    const float* Df = reinterpret_cast<const float*>(D);
    for (int t = threadIdx.x; t < M; t += NT) {
        tw[t] = twz[t];
        ps[t] = post[t];
    }
    const int r0 = blockIdx.x * NL;
    const int nr = min(NL, nrows - r0);
    if (TR) {
        float2 r[ITI];
#pragma unroll
        for (int i = 0; i < ITI; i++) {
            const int t = threadIdx.x + i * NT;
            const int kz = t / NL, rr = t - kz * NL;
            r[i] = t < NL * H && rr < nr ? spec[(size_t)kz * nrows + r0 + rr]
                                         : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < ITI; i++) {
            const int t = threadIdx.x + i * NT;
            const int kz = t / NL, rr = t - kz * NL;
            if (t < NL * H) D[rr * H + kz] = r[i];
        }
    } else {
        const float2* in = spec + (size_t)r0 * H;
        float2 r[ITI];
#pragma unroll
        for (int i = 0; i < ITI; i++) {
            const int t = threadIdx.x + i * NT;
            r[i] = t < nr * H ? in[t] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < ITI; i++) {
            const int t = threadIdx.x + i * NT;
            if (t < NL * H) D[t] = r[i];
        }
    }
    __syncthreads();
    // Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) W_K2^{-k}, k = 0..M-1
    constexpr int half = M / 2;
    for (int t = threadIdx.x; t < NL * (half + 1); t += NT) {
        const int k = t / NL, r = t - k * NL;
        float2* row = D + r * H;
        const int k2 = M - k;
        const float2 a = row[k], b = row[k2];
        const float2 wk = make_float2(ps[k].x, -ps[k].y);
        const float2 E = make_float2(a.x + b.x, a.y - b.y);
        const float2 dd = make_float2(a.x - b.x, a.y + b.y);
        const float2 O = c_mul(dd, wk);
        const float2 Zk = make_float2(E.x - O.y, E.y + O.x);
        if (k != 0 && k2 != k) {
            const float2 w2 = make_float2(-wk.x, wk.y);
            const float2 E2 = make_float2(b.x + a.x, b.y - a.y);
            const float2 d2 = make_float2(b.x - a.x, b.y + a.y);
            const float2 O2 = c_mul(d2, w2);
            row[k2] = make_float2(E2.x - O2.y, E2.y + O2.x);
        }
        row[k] = Zk;
    }
    __syncthreads();
    line_fft4<N1, N2, NL, true>(D, H, 1, tw);
    float* o = real + (size_t)r0 * K2;
#pragma unroll
    for (int i = 0; i < IT; i++) {
        const int t = threadIdx.x + i * NT;
        const int r = t / K2, col = t - r * K2;
        if (t < nr * K2) o[t] = Df[2 * r * H + col];
    }
}

// The y forward, x forward, Green's function, x inverse and y inverse passes of one kz plane in
// one block, for square planes (K0 = K1 = K = N1 N2) whose K x K complex points fit in shared
// memory: the spectrum is stored plane by plane ([kz][x][y], written so by k_zfwd4<TR>), the
// block loads its plane once, runs the same line transforms as k_ypass4 / k_xconv4 (so the same
// bits), and stores it once. One block per kz: few blocks, each long, which leaves most SMs to
// the pair kernel that runs beside the reciprocal chain. Dynamic shared memory: the twiddles (K)
// and the plane with a row pitch of K + 1 (conflict-free for lines in both directions).
template <int N1, int N2, int NL>
__global__ void __launch_bounds__(NL * F4<N1, N2>::T) k_plane4(
    const float2* __restrict__ tw_in, float2* __restrict__ spec, const float* __restrict__ bc,
    double* __restrict__ epart, int H, int K2, const SbFftBatchIo* __restrict__ bio) {
    constexpr int K = N1 * N2, P = K + 1, NT = NL * F4<N1, N2>::T, IT = K * K / NT;
    static_assert(K * K % NT == 0 && K % NL == 0, "plane must divide among the threads");
    if (bio) {
        spec = bio[blockIdx.y].spec;
        bc = bio[blockIdx.y].bc;
        epart = bio[blockIdx.y].epart;
    }
    extern __shared__ float2 smem_plane[];
    float2* tw = smem_plane;
    float2* D = smem_plane + K;
    __shared__ double red[NT];
    const int kz = blockIdx.x;
    float2* plane = spec + (size_t)kz * K * K;
    for (int t = threadIdx.x; t < K; t += NT) tw[t] = tw_in[t];
    {
        float2 r[IT];
#pragma unroll
        for (int i = 0; i < IT; i++) r[i] = plane[threadIdx.x + i * NT];
#pragma unroll
        for (int i = 0; i < IT; i++) {
            const int t = threadIdx.x + i * NT;
            const int x = t / K, y = t - x * K;
            D[x * P + y] = r[i];
        }
    }
    __syncthreads();
    for (int l0 = 0; l0 < K; l0 += NL) line_fft4<N1, N2, NL, false>(D + l0 * P, P, 1, tw);
    for (int l0 = 0; l0 < K; l0 += NL) line_fft4<N1, N2, NL, false>(D + l0, 1, P, tw);
    const double wkz = (kz == 0 || 2 * kz == K2) ? 1.0 : 2.0;
    double e = 0.0;
    {
        float g[IT];
#pragma unroll
        for (int i = 0; i < IT; i++) {
            const int t = threadIdx.x + i * NT;
            const int x = t / K, y = t - x * K;
            g[i] = bc[((size_t)x * K + y) * H + kz];
        }
#pragma unroll
        for (int i = 0; i < IT; i++) {
            const int t = threadIdx.x + i * NT;
            const int x = t / K, y = t - x * K;
            const float2 v = D[x * P + y];
            if (epart) e += wkz * (double)g[i] * ((double)v.x * v.x + (double)v.y * v.y);
            D[x * P + y] = make_float2(v.x * g[i], v.y * g[i]);
        }
    }
    __syncthreads();
    for (int l0 = 0; l0 < K; l0 += NL) line_fft4<N1, N2, NL, true>(D + l0, 1, P, tw);
    for (int l0 = 0; l0 < K; l0 += NL) line_fft4<N1, N2, NL, true>(D + l0 * P, P, 1, tw);
#pragma unroll
    for (int i = 0; i < IT; i++) {
        const int t = threadIdx.x + i * NT;
        const int x = t / K, y = t - x * K;
        plane[t] = D[x * P + y];
    }
    if (epart) {
        // deterministic block reduction (fixed tree over a power-of-two prefix)
        red[threadIdx.x] = e;
        __syncthreads();
        int m = 1;
        while (m * 2 <= NT) m *= 2;
        if (threadIdx.x >= m) red[threadIdx.x - m] += red[threadIdx.x];
        __syncthreads();
        for (int o = m / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) epart[kz] = 0.5 * red[0];
    }
}

// square plane sizes fused by k_plane4: X(K, N1, N2, NL) (the even 2-3-5-smooth sizes of about
// 1 A grids on 30-64 A boxes, and 80, 96, 128)
#define SB_FFT4_PLANE_SIZES(X)                                                                   \
    X(30, 5, 6, 30) X(32, 4, 8, 32) X(36, 6, 6, 36) X(40, 5, 8, 40) X(48, 6, 8, 16)             \
    X(50, 5, 10, 50) X(54, 6, 9, 54) X(60, 6, 10, 60) X(64, 8, 8, 64) X(80, 8, 10, 16)          \
    X(96, 8, 12, 48) X(128, 8, 16, 64)

// sizes with a register line transform: X(N, N1, N2). The z passes (half length M = K2 / 2)
// take the sizes whose 32-row tile fits the static shared-memory limit.
#define SB_FFT4_ZSIZES(X)                                                                        \
    X(8, 2, 4) X(12, 3, 4) X(15, 3, 5) X(16, 4, 4) X(18, 3, 6) X(20, 4, 5) X(24, 4, 6)           \
    X(25, 5, 5) X(27, 3, 9) X(30, 5, 6) X(32, 4, 8) X(36, 6, 6) X(40, 5, 8) X(45, 5, 9)          \
    X(48, 6, 8) X(50, 5, 10) X(54, 6, 9) X(60, 6, 10) X(64, 8, 8) X(72, 8, 9) X(80, 8, 10)       \
    X(90, 9, 10) X(96, 8, 12) X(100, 10, 10) X(108, 9, 12) X(120, 10, 12)
#define SB_FFT4_SIZES(X)                                                                         \
    SB_FFT4_ZSIZES(X) X(128, 8, 16) X(144, 12, 12) X(160, 10, 16) X(180, 12, 15)                 \
    X(192, 12, 16) X(216, 12, 18) X(240, 15, 16) X(256, 16, 16)

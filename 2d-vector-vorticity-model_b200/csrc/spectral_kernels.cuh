// Exact preconditioner of the cal_w operator by Fourier modes in x.
//
// The operator (PoissonSolver::InitPoissonMatrix, src/PoissonSolver.cpp:760-796,
// in the symmetric form S of poisson_kernels.cuh) has coefficients that depend
// on the row k only and is periodic in x, so the discrete Fourier transform
// along each row diagonalises its x part: mode m of every row sees
//   (cx_k mu_m + ru_k + rd_k) w_k - ru_k w_{k+1} - rd_k w_{k-1} = f_k,
//   mu_m = 2 - 2 cos(2 pi m / NX),
// a real tridiagonal system in z per mode. S^{-1} r is then: a forward FFT of
// every row, one tridiagonal solve per mode (real and imaginary parts alike),
// and an inverse FFT. It is S^{-1} up to round-off: the solver applies it to
// the right-hand side directly and checks the FP64 residual, with CG
// iterations only if that check fails. NX must be a power of two.
//
// Row transforms run in shared memory, one block per pair of rows: the two
// real rows are the real and imaginary parts of one complex row, whose FFT
// separates into the two row spectra by Hermitian symmetry (and, backwards,
// two Hermitian spectra combine into one complex row whose inverse FFT gives
// both real rows). Spectra are stored [NK][mpitch] as separate real and
// imaginary arrays, modes m = 0..NX/2 contiguous, so the per-mode solve reads
// them coalesced with one thread per mode.
#pragma once

#include "vvm_common.cuh"

namespace vvm {

// The z solve of each mode uses the twisted (two-sided) factorisation: rows
// 0..mid are eliminated downwards (y_k = (f_k + rd_k y_{k-1}) inv_k, leaving
// w_k + cp_k w_{k+1} = y_k), rows NK-1..mid+1 upwards (z_k = (f_k + ru_k
// z_{k+1}) inv_k, leaving w_k + cp_k w_{k-1} = z_k); the two middle rows give
// w_mid = (y_mid - cp_mid z_{mid+1}) den and w_{mid+1} = z_{mid+1} -
// cp_{mid+1} w_mid, den = 1 / (1 - cp_mid cp_{mid+1}); both halves then
// back-substitute outwards. inv and cp hold the factors of each row's half.
template <typename P>
struct SpecArgs {
    int NX, logN, NK, pitch, mpitch, mid;
    const P *twr, *twi;      // exp(-2 pi i j / NX), j < NX/2
    const P *inv, *cp;       // per-mode factors, [NK][mpitch]
    const P* den;            // per-mode meeting factor, [mpitch]
    const P *rd, *ru;        // couplings of each row to the rows below / above, [NK]
    P *sre, *sim;            // spectra, [NK][mpitch]
};

// Shared-memory slot of point i of a row: i with its low four bits XORed with
// bits 2-5 and 8-11 (a permutation of 0..N-1). Eight-byte words fall in 16
// bank pairs; unswizzled, the bit-reversed stores and the first two double
// passes of fft_shared put 4 to 16 of a half-warp's words in one pair (1.6 M
// bank conflicts a launch at NX = 2048). With the swizzle every access
// pattern of these kernels averages about 1.1 wavefronts a half-warp at NX =
// 2048 and 8192. Only the slot changes, so the arithmetic is the same.
__device__ __forceinline__ int sw(int i) { return i ^ (((i >> 2) ^ (i >> 8)) & 15); }
// The twiddle table's slot of entry j (a permutation of 0..N/2-1): the passes
// read entries j * N / 2^s of up to 16 distinct j a half-warp, which all fall
// in one bank pair unswizzled; XORing the low four bits with bits 4-7 and
// 8-11 spreads them.
__device__ __forceinline__ int twz(int j) { return j ^ (((j >> 4) ^ (j >> 8)) & 15); }

// The twiddles exp(-2 pi i j / N), j < N/2, copied into shared memory (tw:
// N values, real parts then imaginary, entry j at slot twz(j)) before the
// first barrier of a kernel.
template <typename P>
__device__ __forceinline__ void load_twiddles(P* tw, const SpecArgs<P>& a) {
    for (int j = threadIdx.x; j < a.NX / 2; j += blockDim.x) {
        tw[twz(j)] = a.twr[j];
        tw[a.NX / 2 + twz(j)] = a.twi[j];
    }
}

// One radix-2 butterfly of the DIT FFT: (u, x) -> (u + w x, u - w x).
template <typename P>
__device__ __forceinline__ void fft_bfly(P& ur, P& ui, P& xr, P& xi, P wr, P wi) {
    const P vr = xr * wr - xi * wi, vi = xr * wi + xi * wr;
    const P r0 = ur + vr, i0 = ui + vi;
    xr = ur - vr;
    xi = ui - vi;
    ur = r0;
    ui = i0;
}

// In-place radix-2 DIT FFT of N = 2^logN points held bit-reversed in (re,
// im); sign -1 forward, +1 inverse (unnormalised). All threads of the block
// call it. Twiddles come from shared memory (load_twiddles). Stages go two at
// a time: for stages s, s+1 (h = 2^(s-1)) a thread holds the four points
// base + {0, h, 2h, 3h} of one group in registers, does stage s's two
// butterflies (same twiddle) and stage s+1's two, each exactly as the
// one-stage form does it (same operations, same table twiddles: the result
// is bit for bit that of eleven single stages), with half the passes through
// shared memory and half the barriers; an odd last stage runs alone.
template <typename P>
__device__ __forceinline__ void fft_shared(P* re, P* im, const P* tw, const SpecArgs<P>& a, bool inverse) {
    const int N = a.NX;
    const P* twr = tw;
    const P* twi = tw + N / 2;
    const P sg = inverse ? P(-1) : P(1);
    int s = 1;
    for (; s + 1 <= a.logN; s += 2) {
        const int h = 1 << (s - 1);
        const int ts1 = N >> s, ts2 = N >> (s + 1);
        for (int t = threadIdx.x; t < N / 4; t += blockDim.x) {
            const int j = t & (h - 1);
            const int b0 = ((t >> (s - 1)) << (s + 1)) + j;
            P r0 = re[sw(b0)], i0 = im[sw(b0)], r1 = re[sw(b0 + h)], i1 = im[sw(b0 + h)];
            P r2 = re[sw(b0 + 2 * h)], i2 = im[sw(b0 + 2 * h)], r3 = re[sw(b0 + 3 * h)], i3 = im[sw(b0 + 3 * h)];
            const P w1r = twr[twz(j * ts1)], w1i = sg * twi[twz(j * ts1)];
            fft_bfly(r0, i0, r1, i1, w1r, w1i);   // stage s: (b0, b0+h), (b0+2h, b0+3h)
            fft_bfly(r2, i2, r3, i3, w1r, w1i);
            const P w2r = twr[twz(j * ts2)], w2i = sg * twi[twz(j * ts2)];
            const P w3r = twr[twz((j + h) * ts2)], w3i = sg * twi[twz((j + h) * ts2)];
            fft_bfly(r0, i0, r2, i2, w2r, w2i);   // stage s+1: (b0, b0+2h), (b0+h, b0+3h)
            fft_bfly(r1, i1, r3, i3, w3r, w3i);
            re[sw(b0)] = r0;
            im[sw(b0)] = i0;
            re[sw(b0 + h)] = r1;
            im[sw(b0 + h)] = i1;
            re[sw(b0 + 2 * h)] = r2;
            im[sw(b0 + 2 * h)] = i2;
            re[sw(b0 + 3 * h)] = r3;
            im[sw(b0 + 3 * h)] = i3;
        }
        __syncthreads();
    }
    if (s == a.logN) {   // the last stage alone
        const int half = 1 << (s - 1);
        const int tstride = N >> s;
        for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
            const int j = t & (half - 1);
            const int i0 = ((t >> (s - 1)) << s) + j, i1 = i0 + half;
            P ur = re[sw(i0)], ui = im[sw(i0)], xr = re[sw(i1)], xi = im[sw(i1)];
            fft_bfly(ur, ui, xr, xi, twr[twz(j * tstride)], sg * twi[twz(j * tstride)]);
            re[sw(i0)] = ur;
            im[sw(i0)] = ui;
            re[sw(i1)] = xr;
            im[sw(i1)] = xi;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int bitrev(int j, int logN) { return (int)(__brev((unsigned)j) >> (32 - logN)); }

// Spectra of rows 2b and 2b+1 of r ([NK][pitch]).
template <typename P>
__device__ __forceinline__ void k_spec_forward_body(const SpecArgs<P>& a, const P* r) {
    extern __shared__ unsigned char smem_raw[];
    P* re = reinterpret_cast<P*>(smem_raw);
    P* im = re + a.NX;
    P* tw = im + a.NX;
    const int k0 = 2 * blockIdx.x, k1 = k0 + 1;
    const bool two = k1 < a.NK;
    load_twiddles(tw, a);
    for (int j = threadIdx.x; j < a.NX; j += blockDim.x) {
        const int jr = sw(bitrev(j, a.logN));
        re[jr] = r[(size_t)k0 * a.pitch + j];
        im[jr] = two ? r[(size_t)k1 * a.pitch + j] : P(0);
    }
    __syncthreads();
    fft_shared(re, im, tw, a, false);
    const int N = a.NX;
    for (int m = threadIdx.x; m <= N / 2; m += blockDim.x) {
        const int mn = (N - m) & (N - 1);
        const P zr = re[sw(m)], zi = im[sw(m)], nr = re[sw(mn)], ni = im[sw(mn)];
        // X0 = (Z[m] + conj Z[N-m]) / 2,  X1 = (Z[m] - conj Z[N-m]) / 2i
        a.sre[(size_t)k0 * a.mpitch + m] = P(0.5) * (zr + nr);
        a.sim[(size_t)k0 * a.mpitch + m] = P(0.5) * (zi - ni);
        if (two) {
            a.sre[(size_t)k1 * a.mpitch + m] = P(0.5) * (zi + ni);
            a.sim[(size_t)k1 * a.mpitch + m] = P(0.5) * (nr - zr);
        }
    }
}
template <typename P>
__global__ void k_spec_forward(SpecArgs<P> a, const P* r) { k_spec_forward_body<P>(a, r); }

// The z solve of every mode m = 0..NX/2 in place on the spectra, by the
// twisted factorisation precomputed per mode (inv, cp, den): rows 0..mid are
// eliminated from the bottom up (coupling rd), rows NK-1..mid+1 from the top
// down (coupling ru), the two meet at rows mid, mid+1, and both halves
// back-substitute outwards. Each half's chains are cut into kModeSegs
// segments: a block takes 32 consecutive modes (lane = mode, so every load is coalesced)
// with 2 * kModeSegs warps, warp (h, s) owning segment s of half h (about
// NK / (2 kModeSegs) rows). Both the elimination y_k = (f_k + c_k y_prev)
// inv_k and the back-substitution w_k = y_k - cp_k w_next are first-order
// affine recurrences: each warp composes its segment's map (A, B), the maps
// meet in shared memory, each warp takes its carry-in by chaining the maps
// of the segments before it, and applies its rows. The serial chain drops from NK/2 rows to about
// 2 NK / (2 kModeSegs) + kModeSegs steps.
constexpr int kModeSegs = 16;

template <typename P>
__device__ __forceinline__ void k_spec_modes_seg_body(const SpecArgs<P>& a) {
    __shared__ P shA[2][kModeSegs][32][3];   // (A re, A im, B) per half, segment, lane
    __shared__ P shY[2][32][2];              // the halves' last rows after elimination
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int h = warp / kModeSegs, sg = warp % kModeSegs;
    const int m = blockIdx.x * 32 + lane;
    const bool on = m <= a.NX / 2;
    const int NK = a.NK, mid = a.mid;
    const size_t mp = a.mpitch;
    P* __restrict__ sre = a.sre;
    P* __restrict__ sim = a.sim;
    const P* __restrict__ inv = a.inv;
    const P* __restrict__ cpv = a.cp;
    const P* __restrict__ lc = h ? a.ru : a.rd;
    // this half's rows in elimination order: k(j) = k0 + dir j, j < n
    const int n = h ? NK - 1 - mid : mid + 1;
    const int dir = h ? -1 : 1, k0 = h ? NK - 1 : 0;
    const int L = (n + kModeSegs - 1) / kModeSegs;
    const int j0 = min(n, sg * L), j1 = min(n, j0 + L);
    auto at = [&](int j) { return (size_t)(k0 + dir * j) * mp + m; };

    // elimination: local map over rows j0..j1-1
    P Ar = P(0), Ai = P(0), Bm = P(1);
    if (on) {
        for (int j = j0; j < j1; j++) {
            const size_t e = at(j);
            const P iv = inv[e], c = lc[k0 + dir * j] * iv;
            Ar = sre[e] * iv + c * Ar;
            Ai = sim[e] * iv + c * Ai;
            Bm = c * Bm;
        }
    }
    shA[h][sg][lane][0] = Ar;
    shA[h][sg][lane][1] = Ai;
    shA[h][sg][lane][2] = Bm;
    if (threadIdx.x < 64) (&shY[0][0][0])[threadIdx.x * 2] = (&shY[0][0][0])[threadIdx.x * 2 + 1] = P(0);   // an empty half: 0
    __syncthreads();
    P yr = P(0), yi = P(0);
    for (int t = 0; t < sg; t++) {
        const P b = shA[h][t][lane][2];
        yr = shA[h][t][lane][0] + b * yr;
        yi = shA[h][t][lane][1] + b * yi;
    }
    if (on) {
        for (int j = j0; j < j1; j++) {
            const size_t e = at(j);
            const P iv = inv[e], c = lc[k0 + dir * j];
            yr = (sre[e] + c * yr) * iv;
            yi = (sim[e] + c * yi) * iv;
            sre[e] = yr;
            sim[e] = yi;
        }
    }
    if (j0 < j1 && j1 == n) {
        shY[h][lane][0] = yr;
        shY[h][lane][1] = yi;
    }
    __syncthreads();
    // the meeting rows mid (half 0) and mid + 1 (half 1)
    P wmr = P(0), wmi = P(0);
    if (on) {
        const P cpm = cpv[(size_t)mid * mp + m], dn = a.den[m];
        const P cqm = (mid + 1 < NK) ? cpv[(size_t)(mid + 1) * mp + m] : P(0);
        const P ymr = shY[0][lane][0], ymi = shY[0][lane][1], zr = shY[1][lane][0], zi = shY[1][lane][1];
        const P w0r = (ymr - cpm * zr) * dn, w0i = (ymi - cpm * zi) * dn;
        if (h == 0) {
            wmr = w0r;
            wmi = w0i;
        } else {
            wmr = zr - cqm * w0r;
            wmi = zi - cqm * w0i;
        }
    }
    // back-substitution outwards over rows j = n-2 .. 0; segment sg takes
    // min(j1, n-1) - 1 down to j0
    const int jt = min(j1, n - 1);
    Ar = P(0);
    Ai = P(0);
    Bm = P(1);
    if (on) {
        for (int j = jt - 1; j >= j0; j--) {
            const size_t e = at(j);
            const P c = -cpv[e];
            Ar = sre[e] + c * Ar;
            Ai = sim[e] + c * Ai;
            Bm = c * Bm;
        }
    }
    __syncthreads();   // every warp has read shY and finished the first maps
    shA[h][sg][lane][0] = Ar;
    shA[h][sg][lane][1] = Ai;
    shA[h][sg][lane][2] = Bm;
    __syncthreads();
    P wr = wmr, wi = wmi;
    for (int t = kModeSegs - 1; t > sg; t--) {
        const P b = shA[h][t][lane][2];
        wr = shA[h][t][lane][0] + b * wr;
        wi = shA[h][t][lane][1] + b * wi;
    }
    if (on) {
        if (j0 < j1 && j1 == n) {   // the meeting row
            sre[at(n - 1)] = wmr;
            sim[at(n - 1)] = wmi;
        }
        for (int j = jt - 1; j >= j0; j--) {
            const size_t e = at(j);
            wr = sre[e] - cpv[e] * wr;
            wi = sim[e] - cpv[e] * wi;
            sre[e] = wr;
            sim[e] = wi;
        }
    }
}
template <typename P>
__global__ void __launch_bounds__(64 * kModeSegs) k_spec_modes_seg(SpecArgs<P> a) { k_spec_modes_seg_body<P>(a); }

// Rows 2b and 2b+1 of out ([NK][pitch]) from their spectra, scaled by 1/NX.
template <typename P>
__device__ __forceinline__ void k_spec_inverse_body(const SpecArgs<P>& a, P* out) {
    extern __shared__ unsigned char smem_raw[];
    P* re = reinterpret_cast<P*>(smem_raw);
    P* im = re + a.NX;
    P* tw = im + a.NX;
    const int k0 = 2 * blockIdx.x, k1 = k0 + 1;
    const bool two = k1 < a.NK;
    const int N = a.NX;
    load_twiddles(tw, a);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        // Hermitian extension: X[N-m] = conj X[m]
        const bool lo = j <= N / 2;
        const int m = lo ? j : N - j;
        const P sg = lo ? P(1) : P(-1);
        const P ar = a.sre[(size_t)k0 * a.mpitch + m], ai = sg * a.sim[(size_t)k0 * a.mpitch + m];
        P br = P(0), bi = P(0);
        if (two) {
            br = a.sre[(size_t)k1 * a.mpitch + m];
            bi = sg * a.sim[(size_t)k1 * a.mpitch + m];
        }
        const int jr = sw(bitrev(j, a.logN));
        re[jr] = ar - bi;   // Z = X0 + i X1
        im[jr] = ai + br;
    }
    __syncthreads();
    fft_shared(re, im, tw, a, true);
    const P scale = P(1) / P(N);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        out[(size_t)k0 * a.pitch + j] = re[sw(j)] * scale;
        if (two) out[(size_t)k1 * a.pitch + j] = im[sw(j)] * scale;
    }
}
template <typename P>
__global__ void k_spec_inverse(SpecArgs<P> a, P* out) { k_spec_inverse_body<P>(a, out); }

}  // namespace vvm

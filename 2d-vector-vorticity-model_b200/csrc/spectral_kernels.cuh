// Exact preconditioner of the cal_w operator by Fourier modes in x.
//
// The operator (PoissonSolver::InitPoissonMatrix, src/PoissonSolver.cpp:760-796,
// in the symmetric form S of poisson_kernels.cuh) has coefficients that depend
// on the row k only and is periodic in x, so the discrete Fourier transform
// along each row diagonalises its x part: mode m of every row sees
//   (cx_k mu_m + ru_k + rd_k) w_k - ru_k w_{k+1} - rd_k w_{k-1} = f_k,
//   mu_m = 2 - 2 cos(2 pi m / NX),
// a real tridiagonal system in z per mode. S^{-1} r is then: a forward FFT of
// every row, one Thomas solve per mode (real and imaginary parts alike), and
// an inverse FFT. In PCG this preconditioner is S^{-1} up to round-off, so
// one iteration reaches the FP64 residual floor. NX must be a power of two.
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

template <typename P>
struct SpecArgs {
    int NX, logN, NK, pitch, mpitch;
    const P *twr, *twi;      // exp(-2 pi i j / NX), j < NX/2
    const P *inv, *cp;       // per-mode Thomas factors, [NK][mpitch]
    const P* rd;             // lower coupling of each row, [NK]
    P *sre, *sim;            // spectra, [NK][mpitch]
};

// In-place radix-2 FFT of N = 2^logN points held bit-reversed in (re, im);
// sign -1 forward, +1 inverse (unnormalised). All threads of the block call it.
template <typename P>
__device__ __forceinline__ void fft_shared(P* re, P* im, const SpecArgs<P>& a, bool inverse) {
    const int N = a.NX;
    for (int s = 1; s <= a.logN; s++) {
        const int half = 1 << (s - 1);
        const int tstride = N >> s;
        for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
            const int j = t & (half - 1);
            const int i0 = ((t >> (s - 1)) << s) + j;
            const int i1 = i0 + half;
            const P wr = __ldg(a.twr + j * tstride);
            const P wi = inverse ? -__ldg(a.twi + j * tstride) : __ldg(a.twi + j * tstride);
            const P xr = re[i1], xi = im[i1];
            const P vr = xr * wr - xi * wi, vi = xr * wi + xi * wr;
            const P ur = re[i0], ui = im[i0];
            re[i0] = ur + vr;
            im[i0] = ui + vi;
            re[i1] = ur - vr;
            im[i1] = ui - vi;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int bitrev(int j, int logN) { return (int)(__brev((unsigned)j) >> (32 - logN)); }

// Spectra of rows 2b and 2b+1 of r ([NK][pitch]).
template <typename P>
__global__ void k_spec_forward(SpecArgs<P> a, const P* r) {
    extern __shared__ unsigned char smem_raw[];
    P* re = reinterpret_cast<P*>(smem_raw);
    P* im = re + a.NX;
    const int k0 = 2 * blockIdx.x, k1 = k0 + 1;
    const bool two = k1 < a.NK;
    for (int j = threadIdx.x; j < a.NX; j += blockDim.x) {
        const int jr = bitrev(j, a.logN);
        re[jr] = r[(size_t)k0 * a.pitch + j];
        im[jr] = two ? r[(size_t)k1 * a.pitch + j] : P(0);
    }
    __syncthreads();
    fft_shared(re, im, a, false);
    const int N = a.NX;
    for (int m = threadIdx.x; m <= N / 2; m += blockDim.x) {
        const int mn = (N - m) & (N - 1);
        const P zr = re[m], zi = im[m], nr = re[mn], ni = im[mn];
        // X0 = (Z[m] + conj Z[N-m]) / 2,  X1 = (Z[m] - conj Z[N-m]) / 2i
        a.sre[(size_t)k0 * a.mpitch + m] = P(0.5) * (zr + nr);
        a.sim[(size_t)k0 * a.mpitch + m] = P(0.5) * (zi - ni);
        if (two) {
            a.sre[(size_t)k1 * a.mpitch + m] = P(0.5) * (zi + ni);
            a.sim[(size_t)k1 * a.mpitch + m] = P(0.5) * (nr - zr);
        }
    }
}

// The z solve of every mode m = 0..NX/2 in place on the spectra (one thread
// per mode; real and imaginary parts share the factors). The recurrence is
// serial in k, so rows are taken kModeBatch at a time: the batch's loads are
// issued together and the chain then runs from registers, one memory round
// trip per batch instead of one per row.
constexpr int kModeBatch = 16;

template <typename P>
__global__ void __launch_bounds__(64) k_spec_modes(SpecArgs<P> a) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m > a.NX / 2) return;
    const size_t mp = a.mpitch;
    P* __restrict__ sre = a.sre;
    P* __restrict__ sim = a.sim;
    const P* __restrict__ inv = a.inv;
    const P* __restrict__ cpv = a.cp;
    const P* __restrict__ rdv = a.rd;
    const int NK = a.NK;
    P yr = P(0), yi = P(0);
    for (int k0 = 0; k0 < NK; k0 += kModeBatch) {
        P fr[kModeBatch], fi[kModeBatch], iv[kModeBatch], rd[kModeBatch];
#pragma unroll
        for (int j = 0; j < kModeBatch; j++) {
            const int kk = k0 + j;
            if (kk < NK) {
                const size_t e = (size_t)kk * mp + m;
                fr[j] = sre[e];
                fi[j] = sim[e];
                iv[j] = inv[e];
                rd[j] = rdv[kk];
            }
        }
#pragma unroll
        for (int j = 0; j < kModeBatch; j++) {
            const int kk = k0 + j;
            if (kk < NK) {
                yr = (fr[j] + rd[j] * yr) * iv[j];
                yi = (fi[j] + rd[j] * yi) * iv[j];
                const size_t e = (size_t)kk * mp + m;
                sre[e] = yr;
                sim[e] = yi;
            }
        }
    }
    // yr, yi hold row NK-1, which is final; back-substitute rows NK-2 .. 0
    for (int k1 = NK - 2; k1 >= 0; k1 -= kModeBatch) {
        P fr[kModeBatch], fi[kModeBatch], c[kModeBatch];
#pragma unroll
        for (int j = 0; j < kModeBatch; j++) {
            const int kk = k1 - j;
            if (kk >= 0) {
                const size_t e = (size_t)kk * mp + m;
                fr[j] = sre[e];
                fi[j] = sim[e];
                c[j] = cpv[e];
            }
        }
#pragma unroll
        for (int j = 0; j < kModeBatch; j++) {
            const int kk = k1 - j;
            if (kk >= 0) {
                yr = fr[j] - c[j] * yr;
                yi = fi[j] - c[j] * yi;
                const size_t e = (size_t)kk * mp + m;
                sre[e] = yr;
                sim[e] = yi;
            }
        }
    }
}

// Rows 2b and 2b+1 of out ([NK][pitch]) from their spectra, scaled by 1/NX.
template <typename P>
__global__ void k_spec_inverse(SpecArgs<P> a, P* out) {
    extern __shared__ unsigned char smem_raw[];
    P* re = reinterpret_cast<P*>(smem_raw);
    P* im = re + a.NX;
    const int k0 = 2 * blockIdx.x, k1 = k0 + 1;
    const bool two = k1 < a.NK;
    const int N = a.NX;
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
        const int jr = bitrev(j, a.logN);
        re[jr] = ar - bi;   // Z = X0 + i X1
        im[jr] = ai + br;
    }
    __syncthreads();
    fft_shared(re, im, a, true);
    const P scale = P(1) / P(N);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        out[(size_t)k0 * a.pitch + j] = re[j] * scale;
        if (two) out[(size_t)k1 * a.pitch + j] = im[j] * scale;
    }
}

}  // namespace vvm

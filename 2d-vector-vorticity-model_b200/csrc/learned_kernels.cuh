// Kernels of the learned preconditioner: a linear multi-level 3x3
// convolutional network on the cal_w residual, BF16 activations and weights
// with FP32 accumulation.
//
// Activations are stored chunk-major, [H][4][W][8]: the 32 channels of a
// pixel are 4 chunks of 8 (16 bytes), and chunk q of row y is a contiguous
// run of W pixels (act_at). A row's chunk is then one 16 W-byte run, which
// TMA reads in 128-byte lines. Rows are periodic in x (the cal_w operator
// is) and zero-padded in y (W = 0 outside the rows).
//
// The 32 -> 32 convolutions run on the tensor cores (tcgen05): one CTA of 128
// threads computes 128 consecutive pixels of one row as D[128 x 32] =
// sum over the 9 taps and 2 K-steps of 16 channels of A_tap[128 x 16] x
// B_tap[16 x 32]. A_tap is the input tile shifted by the tap: the CTA stages
// rows y-1..y+1, pixels x0-1..x0+128, in shared memory in the canonical
// K-major no-swizzle layout (for each group of 8 channels, the pixels
// 16 bytes apart), so a shift of one pixel is a shift of 16 bytes of the
// operand's start address and no im2col copy is made. The accumulator lives
// in 32 TMEM columns; each warp reads back its 32 lanes (pixels).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "vvm_common.cuh"

namespace vvm {

constexpr int kNetC = 32;        // channels

// Element index of channel 8 q of pixel (y, x) in a level of width W.
__device__ __forceinline__ size_t act_at(int y, int q, int x, int W) {
    return (((size_t)y * 4 + q) * W + x) * 8;
}
constexpr int kConvTile = 128;   // pixels of a CTA (the MMA's M)
constexpr int kConvSpan = kConvTile + 2;
constexpr int kNetErrWait = 2;   // device error word: an MMA completion wait gave up
constexpr int kMmaSpinLimit = 1 << 22;

// Shared-memory matrix descriptor of tcgen05 (K-major, no swizzle): start
// address, the byte offset between the two 8-element K chunks (LBO) and
// between groups of 8 rows (SBO), all in 16-byte units; version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                  // version
    return d;                                // base offset 0, legacy LBO mode, layout SWIZZLE_NONE
}

// Instruction descriptor of kind::f16: D in FP32, A and B in BF16, both
// K-major, N = 32, M = 128.
constexpr uint32_t kConvIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kNetC >> 3) << 17) |
                                ((uint32_t)(kConvTile >> 4) << 24);

struct ConvArgs {
    const __nv_bfloat16* in;   // [H][W][32]
    __nv_bfloat16* out;        // [H][W][32]
    const uint4* w;            // packed B operand: [9 taps][4 chunks][32 out] of 8 inputs
    int H, W;
    int* err;                  // device error word
};

// out = conv3x3(in, w), 32 -> 32 channels; grid = H * ceil(W / 128) CTAs of
// 128 threads.
__global__ void __launch_bounds__(kConvTile) k_conv32_tc(ConvArgs a) {
    __shared__ __align__(128) uint4 sA[3][4][kConvSpan];   // [row][channel chunk][pixel]
    __shared__ __align__(128) uint4 sB[9][4][kNetC];       // [tap][channel chunk][out channel]
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tiles = (a.W + kConvTile - 1) / kConvTile;
    const int y = blockIdx.x / tiles, x0 = (blockIdx.x % tiles) * kConvTile;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(32)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // input tile: rows y-1..y+1 (zero outside), pixels x0-1..x0+128 (periodic)
    for (int j = tid; j < 3 * kConvSpan * 4; j += kConvTile) {
        const int kc = j & 3, p = (j >> 2) % kConvSpan, dy = (j >> 2) / kConvSpan;
        const int yy = y + dy - 1;
        int xx = (x0 + p - 1) % a.W;
        if (xx < 0) xx += a.W;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (yy >= 0 && yy < a.H)
            v = *reinterpret_cast<const uint4*>(a.in + act_at(yy, kc, xx, a.W));
        sA[dy][kc][p] = v;
    }
    for (int j = tid; j < 9 * 4 * kNetC; j += kConvTile) (&sB[0][0][0])[j] = a.w[j];
    // make the generic-proxy shared stores visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (tid == 0) {
        uint32_t acc = 0;
        for (int dy = 0; dy < 3; dy++)
            for (int dx = 0; dx < 3; dx++)
                for (int ks = 0; ks < 2; ks++) {
                    const uint64_t ad = umma_desc(smem_u32(&sA[dy][2 * ks][dx]), kConvSpan * 16, 128);
                    const uint64_t bd = umma_desc(smem_u32(&sB[dy * 3 + dx][2 * ks][0]), kNetC * 16, 128);
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
                        "l"(ad), "l"(bd), "r"(kConvIdesc), "r"(acc), "r"(0u)
                        : "memory");
                    acc = 1;
                }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
    }
    // wait for the MMAs (bounded; on give-up, record it and wait once more so
    // no MMA is in flight when TMEM is freed)
    bool done = false;
    for (int pass = 0; pass < 2 && !done; pass++) {
        for (int it = 0; it < kMmaSpinLimit; it++) {
            uint32_t ok;
            asm volatile(
                "{\n\t.reg .pred P1;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, P1;\n\t}\n"
                : "=r"(ok)
                : "r"(smem_u32(&mbar)), "r"(0u)
                : "memory");
            if (ok) {
                done = true;
                break;
            }
        }
        if (!done && pass == 0 && tid == 0 && a.err) atomicOr(a.err, kNetErrWait);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (__all_sync(0xffffffffu, done)) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int x = x0 + tid;   // TMEM lane = pixel of the tile
        if (x < a.W) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                __nv_bfloat162 h0 = __floats2bfloat162_rn(__uint_as_float(r[8 * q + 0]), __uint_as_float(r[8 * q + 1]));
                __nv_bfloat162 h1 = __floats2bfloat162_rn(__uint_as_float(r[8 * q + 2]), __uint_as_float(r[8 * q + 3]));
                __nv_bfloat162 h2 = __floats2bfloat162_rn(__uint_as_float(r[8 * q + 4]), __uint_as_float(r[8 * q + 5]));
                __nv_bfloat162 h3 = __floats2bfloat162_rn(__uint_as_float(r[8 * q + 6]), __uint_as_float(r[8 * q + 7]));
                uint4 v;
                v.x = *reinterpret_cast<uint32_t*>(&h0);
                v.y = *reinterpret_cast<uint32_t*>(&h1);
                v.z = *reinterpret_cast<uint32_t*>(&h2);
                v.w = *reinterpret_cast<uint32_t*>(&h3);
                *reinterpret_cast<uint4*>(a.out + act_at(y, q, x, a.W)) = v;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32) : "memory");
}

// ---------------------------------------------------------------------------
// The same convolution for rows of at least kCBox pixels, streamed: a CTA
// owns a strip of 128 pixels of R consecutive output rows and keeps the
// input rows it needs in a ring of kCSlots shared-memory slots, so every
// input row is read from global memory once per strip and the packed weights
// once per CTA (against three rows and all weights per 128 output pixels in
// k_conv32_tc).
//
// Loads are TMA (cp.async.bulk.tensor, no multicast) from a 3D tensor map of
// the chunk-major activations, dims {64 elements (8 pixels x 8 channels,
// 128 bytes), W / 8 pixel blocks, 4 H chunk rows}: one box {64, 18, 1} per
// 8-channel chunk (18 lines of 128 bytes) lands as that chunk's canonical
// K-major rows (pixel p at 16 p bytes) for pixels x0-8 .. x0+135, so tap dx
// of output pixel x0+m reads box pixel 7+dx+m. The box is zero outside the
// tensor, which gives the zero rows y = -1 and y = H; the periodic pixels
// x0-1 = W-1 (first strip) and x0+128 = W (last strip) come from a second
// map with one-line boxes and are copied into place in shared memory.
// Needs W a multiple of 8.
//
// Warp-specialised: lane 0 of warp 4 issues the loads and the MMAs; warps
// 0-3 read the accumulators back (warp w owns TMEM lanes 32w..32w+31, the
// tile's pixels) and store them. Input row j goes to slot j % kCSlots; it is
// read by output rows j-2..j, so the slot of row r-2 is refilled with row
// r-2+kCSlots once output r-2's MMAs are done, which never holds up the
// issue of row r. kCAcc TMEM accumulators (32 columns each) let the MMA warp
// run kCAcc rows ahead of the write-back. Barriers: full[slot] (TMA bytes of
// an input row), done[b] (MMAs of the row in accumulator b, by
// tcgen05.commit), empty[b] (accumulator b read back, one arrive per
// epilogue warp), one for the weights. Every wait is bounded; a wait that
// gives up sets kNetErrWait and an abort flag that ends the CTA's remaining
// work, after a bounded wait for the copies and MMAs in flight.
constexpr int kCSlots = 8;                        // ring of input rows
constexpr int kCAcc = 4;                          // TMEM accumulators
constexpr int kCThreads = 160;                    // 4 epilogue warps + 1 producer warp
constexpr int kCBox = 144;
constexpr int kCRowBytes = kCBox * 16;            // one 8-channel chunk of a row
constexpr int kCSlotBytes = 4 * kCRowBytes;       // 9216
constexpr int kCWBytes = 9 * 4 * kNetC * 16;      // packed weights, 18432
constexpr int kCWrapBytes = 2 * 4 * 8 * 16;       // [side][chunk][8 pixels], 1024 a slot
constexpr int kCBars = kCSlots + 2 * kCAcc + 1;   // full[], done[], empty[], weights
constexpr int kConvStreamSmem = 128 + kCWBytes + kCSlots * (kCSlotBytes + kCWrapBytes) + 8 * kCBars + 16;

struct ConvStreamArgs {
    const __nv_bfloat16* in;   // [H][W][32] (the tensor maps' tensor)
    __nv_bfloat16* out;        // [H][W][32]
    const uint4* w;            // packed B operand, as for k_conv32_tc
    int H, W, R;               // R: output rows per CTA
    int* err;
};

// Bounded wait on one phase of an mbarrier; gives up early when *abort is set.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
    for (int it = 0; it < kMmaSpinLimit; it++) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255) == 255 && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(kCThreads) k_conv32_stream(const __grid_constant__ CUtensorMap trow,
                                                              const __grid_constant__ CUtensorMap twrap,
                                                              ConvStreamArgs a) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t* base = smem_raw + (((raw + 127) & ~127u) - raw);
    uint8_t* sB = base;
    uint8_t* sA = sB + kCWBytes;                                   // [slot][chunk][144 pixels]
    uint8_t* sW = sA + kCSlots * kCSlotBytes;                      // [slot][side][chunk][8 pixels]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sW + kCSlots * kCWrapBytes);
    volatile int* abort = reinterpret_cast<volatile int*>(bars + kCBars);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kCBars) + 1;
    const uint32_t full0 = smem_u32(bars), done0 = full0 + 8 * kCSlots, empty0 = done0 + 8 * kCAcc,
                   wbar = empty0 + 8 * kCAcc;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int strips = (a.W + kConvTile - 1) / kConvTile;
    const int x0 = (blockIdx.x % strips) * kConvTile;
    const int y0 = (blockIdx.x / strips) * a.R;
    const int R = min(a.R, a.H - y0);
    const int nin = R + 2;                       // input rows y0-1 .. y0+R
    const bool left = x0 == 0, right = x0 + kConvTile >= a.W;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(32 * kCAcc)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < kCBars; i++) {
            const bool is_empty = i >= kCSlots + kCAcc && i < kCSlots + 2 * kCAcc;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(full0 + 8 * i), "r"(is_empty ? 4u : 1u)
                         : "memory");
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 4) {
        if (lane == 0) {
            int issued = 0, consumed = 0, committed = 0;
            bool wdone = false;
            auto load_row = [&](int j) {
                const int sl = j % kCSlots, y = y0 - 1 + j;
                const uint32_t bar = full0 + 8 * sl;
                const uint32_t bytes = kCSlotBytes + (left ? 512u : 0u) + (right ? 512u : 0u);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
                for (int kc = 0; kc < 4; kc++) {
                    // map coordinates: (element in an 8-pixel line, 8-pixel block, chunk row 4 y + kc)
                    tma_load_3d(smem_u32(sA + sl * kCSlotBytes + kc * kCRowBytes), &trow, 0, (x0 - 8) / 8, 4 * y + kc, bar);
                    if (left) tma_load_3d(smem_u32(sW + sl * kCWrapBytes + kc * 128), &twrap, 0, a.W / 8 - 1, 4 * y + kc, bar);
                    if (right) tma_load_3d(smem_u32(sW + sl * kCWrapBytes + 512 + kc * 128), &twrap, 0, 0, 4 * y + kc, bar);
                }
                issued = j + 1;
            };
            auto take_row = [&](int j) -> bool {   // wait for input row j, then put its periodic pixels in place
                const int sl = j % kCSlots;
                if (!mbar_wait(full0 + 8 * sl, (uint32_t)((j / kCSlots) & 1), abort)) return false;
                consumed = j + 1;
                uint4* A = reinterpret_cast<uint4*>(sA + sl * kCSlotBytes);
                const uint4* Wr = reinterpret_cast<const uint4*>(sW + sl * kCWrapBytes);
                for (int kc = 0; kc < 4; kc++) {
                    if (left) A[kc * kCBox + 7] = Wr[kc * 8 + 7];
                    if (right) A[kc * kCBox + (a.W - x0 + 8)] = Wr[32 + kc * 8];
                }
                return true;
            };
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(wbar), "r"(kCWBytes) : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             smem_u32(sB)),
                         "l"(reinterpret_cast<uint64_t>(a.w)), "r"(kCWBytes), "r"(wbar)
                         : "memory");
            for (int j = 0; j < min(kCSlots, nin); j++) load_row(j);
            bool ok = true;
            for (int r = 0; r < R && ok; r++) {
                if (r == 0) {
                    ok = mbar_wait(wbar, 0, abort);
                    wdone = ok;
                    for (int j = 0; j < 3 && ok; j++) ok = take_row(j);
                } else {
                    ok = take_row(r + 2);
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the copied pixels, for the MMAs
                const int b = r % kCAcc;
                if (ok && r >= kCAcc) ok = mbar_wait(empty0 + 8 * b, (uint32_t)(((r - kCAcc) / kCAcc) & 1), abort);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                uint32_t acc = 0;
                for (int dy = 0; dy < 3; dy++) {
                    const uint8_t* row = sA + ((r + dy) % kCSlots) * kCSlotBytes;
                    for (int dx = 0; dx < 3; dx++)
                        for (int ks = 0; ks < 2; ks++) {
                            const uint64_t ad = umma_desc(smem_u32(row + (2 * ks) * kCRowBytes + (7 + dx) * 16), kCRowBytes, 128);
                            const uint64_t bd = umma_desc(smem_u32(sB + ((dy * 3 + dx) * 4 + 2 * ks) * kNetC * 16), kNetC * 16, 128);
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(
                                    tmem + 32u * b),
                                "l"(ad), "l"(bd), "r"(kConvIdesc), "r"(acc), "r"(0u)
                                : "memory");
                            acc = 1;
                        }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 done0 + 8 * b)
                             : "memory");
                committed = r + 1;
                // input row r-2+kCSlots reuses the slot of row r-2, free once
                // output r-2's MMAs are done
                const int jn = r - 2 + kCSlots;
                if (r >= 2 && jn < nin) {
                    const int q = r - 2;
                    ok = mbar_wait(done0 + 8 * (q % kCAcc), (uint32_t)((q / kCAcc) & 1), abort);
                    if (ok) load_row(jn);
                }
            }
            if (!ok) {
                if (a.err) atomicOr(a.err, kNetErrWait);
                *abort = 1;
                // wait (bounded) for the copies and MMAs in flight before the
                // shared memory and TMEM go away
                volatile int never = 0;
                if (!wdone) mbar_wait(wbar, 0, &never);
                for (int j = consumed; j < issued; j++)
                    mbar_wait(full0 + 8 * (j % kCSlots), (uint32_t)((j / kCSlots) & 1), &never);
                if (committed > 0) {
                    const int q = committed - 1;
                    mbar_wait(done0 + 8 * (q % kCAcc), (uint32_t)((q / kCAcc) & 1), &never);
                }
            }
        }
    } else {
        // epilogue warps: write out output rows as their MMAs complete
        for (int q = 0; q < R; q++) {
            const int b = q % kCAcc;
            bool got = !*abort && mbar_wait(done0 + 8 * b, (uint32_t)((q / kCAcc) & 1), abort);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            got = __all_sync(0xffffffffu, got);
            if (!got) {   // give up; the producer's cleanup waits for what is in flight
                if (lane == 0 && !*abort) {
                    if (a.err) atomicOr(a.err, kNetErrWait);
                    *abort = 1;
                }
                break;
            }
            uint32_t v[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + 32u * b)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(empty0 + 8 * b) : "memory");
            const int x = x0 + tid;
            if (x < a.W) {
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    __nv_bfloat162 h0 = __floats2bfloat162_rn(__uint_as_float(v[8 * c + 0]), __uint_as_float(v[8 * c + 1]));
                    __nv_bfloat162 h1 = __floats2bfloat162_rn(__uint_as_float(v[8 * c + 2]), __uint_as_float(v[8 * c + 3]));
                    __nv_bfloat162 h2 = __floats2bfloat162_rn(__uint_as_float(v[8 * c + 4]), __uint_as_float(v[8 * c + 5]));
                    __nv_bfloat162 h3 = __floats2bfloat162_rn(__uint_as_float(v[8 * c + 6]), __uint_as_float(v[8 * c + 7]));
                    uint4 o;
                    o.x = *reinterpret_cast<uint32_t*>(&h0);
                    o.y = *reinterpret_cast<uint32_t*>(&h1);
                    o.z = *reinterpret_cast<uint32_t*>(&h2);
                    o.w = *reinterpret_cast<uint32_t*>(&h3);
                    *reinterpret_cast<uint4*>(a.out + act_at(y0 + q, c, x, a.W)) = o;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32 * kCAcc) : "memory");
}

// Packs FP32 weights w[tap][in][out] into the B operand of k_conv32_tc:
// [tap][in / 8][out] of 8 consecutive inputs in BF16. With flip, the packed
// operand is that of the adjoint convolution: tap 8 - t, in and out swapped.
__global__ void k_pack_conv32(const float* w, uint4* packed, int flip) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;   // (tap, chunk, out)
    if (j >= 9 * 4 * kNetC) return;
    const int co = j % kNetC, kc = (j / kNetC) % 4, t = j / (4 * kNetC);
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const int ci = kc * 8 + e;
        v[e] = flip ? w[((8 - t) * kNetC + co) * kNetC + ci] : w[(t * kNetC + ci) * kNetC + co];
    }
    __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
    uint4 o;
    o.x = *reinterpret_cast<uint32_t*>(&h0);
    o.y = *reinterpret_cast<uint32_t*>(&h1);
    o.z = *reinterpret_cast<uint32_t*>(&h2);
    o.w = *reinterpret_cast<uint32_t*>(&h3);
    packed[j] = o;
}

// ---------------------------------------------------------------------------
// The rest of the network on the CUDA cores. Pixels of level l form an
// [H][W] grid (H, W of level 0 multiples of 8; level l+1 halves both); a
// thread handles one pixel, or one pixel's chunk of 8 channels (16 bytes).

__device__ __forceinline__ void bf16x8_load(const __nv_bfloat16* p, float (&v)[8]) {
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float2 f = __bfloat1622float2(h[q]);
        v[2 * q] = f.x;
        v[2 * q + 1] = f.y;
    }
}

__device__ __forceinline__ void bf16x8_store(__nv_bfloat16* p, const float (&v)[8]) {
    uint4 u;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    *reinterpret_cast<uint4*>(p) = u;
}

__device__ __forceinline__ int wrapx(int x, int W) { return x < 0 ? x + W : (x >= W ? x - W : x); }

// h[p][c] = sum_t wl[t][c] x[p + off(t)]  (1 -> 32 channels; x FP32 [H][W]).
// The 288 weights are staged in shared memory (read as broadcasts).
// A thread computes one pixel's chunk of 8 channels; consecutive threads
// take consecutive pixels of one chunk plane, so a warp stores 512 contiguous
// bytes and reads the same weights.
__global__ void k_net_lift(const float* x, const float* wl, __nv_bfloat16* h, int H, int W) {
    __shared__ float sw[9 * kNetC];
    for (int j = threadIdx.x; j < 9 * kNetC; j += blockDim.x) sw[j] = wl[j];
    __syncthreads();
    const long j = blockIdx.x * (long)blockDim.x + threadIdx.x;   // (chunk, pixel): pixels fastest
    if (j >= 4L * H * W) return;
    const int q = (int)(j / ((long)H * W)), p = (int)(j - (long)q * H * W);
    const int y = p / W, xx = p - y * W;
    float xv[9];
#pragma unroll
    for (int t = 0; t < 9; t++) {
        const int yy = y + t / 3 - 1, xs = wrapx(xx + t % 3 - 1, W);
        xv[t] = (yy >= 0 && yy < H) ? x[(size_t)yy * W + xs] : 0.f;
    }
    float o[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        float acc = 0.f;
#pragma unroll
        for (int t = 0; t < 9; t++) acc += sw[t * kNetC + 8 * q + e] * xv[t];
        o[e] = acc;
    }
    bf16x8_store(h + act_at(y, q, xx, W), o);
}

// z[p] = scale * sum_t sum_c wp[t][c] g[p + off(t)][c] for rows < hvalid, else 0
// (32 -> 1 channel; z FP32 [H][W]).
// Four consecutive threads share a pixel, one 8-channel chunk each (a warp's
// loads of a tap are 512 contiguous bytes), and add their partial sums by
// shuffles. blockDim.x is a multiple of 32.
__global__ void k_net_proj(const __nv_bfloat16* g, const float* wp, float* z, int H, int W, int hvalid,
                           float scale) {
    __shared__ float sw[9 * kNetC];
    for (int j = threadIdx.x; j < 9 * kNetC; j += blockDim.x) sw[j] = wp[j];
    __syncthreads();
    const long j = blockIdx.x * (long)blockDim.x + threadIdx.x;   // (pixel, chunk)
    const bool in = j < 4L * H * W;
    const int q = (int)(j & 3), p = in ? (int)(j >> 2) : 0;
    const int y = p / W, xx = p - y * W;
    float acc = 0.f;
    if (in && y < hvalid) {
#pragma unroll
        for (int t = 0; t < 9; t++) {
            const int yy = y + t / 3 - 1, xs = wrapx(xx + t % 3 - 1, W);
            if (yy < 0 || yy >= H) continue;
            float v[8];
            bf16x8_load(g + act_at(yy, q, xs, W), v);
#pragma unroll
            for (int e = 0; e < 8; e++) acc += sw[t * kNetC + 8 * q + e] * v[e];
        }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (in && q == 0) z[p] = acc * scale;
}

// Adjoint of k_net_proj (scale 1): dg[q][c] = sum_t wp[t][c] dz[q - off(t)].
__global__ void k_net_proj_adj(const float* dz, const float* wp, __nv_bfloat16* dg, int H, int W) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= H * W) return;
    const int y = p / W, xx = p - y * W;
    float dv[9];
#pragma unroll
    for (int t = 0; t < 9; t++) {
        const int yy = y - (t / 3 - 1), xs = wrapx(xx - (t % 3 - 1), W);
        dv[t] = (yy >= 0 && yy < H) ? dz[(size_t)yy * W + xs] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float o[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            float acc = 0.f;
#pragma unroll
            for (int t = 0; t < 9; t++) acc += __ldg(wp + t * kNetC + 8 * q + e) * dv[t];
            o[e] = acc;
        }
        bf16x8_store(dg + act_at(y, q, xx, W), o);
    }
}

// out[y][x] = mult * sum of the 2x2 block of in at (2y, 2x); Ho x Wo coarse
// pixels (mult 1/4: average pooling; 1: adjoint of nearest upsampling).
__global__ void k_net_sum4(const __nv_bfloat16* in, __nv_bfloat16* out, int Ho, int Wo, float mult) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;   // (coarse pixel, chunk)
    if (j >= Ho * Wo * 4) return;
    const int q = j / (Ho * Wo), p = j - q * (Ho * Wo), y = p / Wo, x = p - y * Wo;   // pixels fastest
    const int Wf = 2 * Wo;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++) {
            float v[8];
            bf16x8_load(in + act_at(2 * y + a, q, 2 * x + b, Wf), v);
#pragma unroll
            for (int e = 0; e < 8; e++) s[e] += v[e];
        }
#pragma unroll
    for (int e = 0; e < 8; e++) s[e] *= mult;
    bf16x8_store(out + act_at(y, q, x, Wo), s);
}

// out[y][x] = mult * lo[y/2][x/2] + skip[y][x] (out may be skip); H x W fine
// pixels (mult 1: nearest upsampling plus the skip connection; 1/4: adjoint
// of average pooling, accumulated).
__global__ void k_net_up_add(const __nv_bfloat16* lo, const __nv_bfloat16* skip, __nv_bfloat16* out, int H, int W,
                             float mult) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= H * W * 4) return;
    const int q = j / (H * W), p = j - q * (H * W), y = p / W, x = p - y * W;   // pixels fastest
    float a[8], b[8];
    bf16x8_load(lo + act_at(y >> 1, q, x >> 1, W >> 1), a);
    bf16x8_load(skip + act_at(y, q, x, W), b);
#pragma unroll
    for (int e = 0; e < 8; e++) a[e] = mult * a[e] + b[e];
    bf16x8_store(out + act_at(y, q, x, W), a);
}

// dW[t][ci][co] += sum_p X[p + off(t)][ci] dY[p][co] over one tile of 128
// pixels of a row (grid = H * ceil(W / 128), 256 threads; 36 weights a thread).
__global__ void __launch_bounds__(256) k_net_wgrad32(const __nv_bfloat16* X, const __nv_bfloat16* dY, float* dW,
                                                     int H, int W) {
    __shared__ __nv_bfloat16 sx[3][kConvSpan][kNetC];
    __shared__ __nv_bfloat16 sy[kConvTile][kNetC];
    const int tiles = (W + kConvTile - 1) / kConvTile;
    const int y = blockIdx.x / tiles, x0 = (blockIdx.x % tiles) * kConvTile;
    const int n = min(kConvTile, W - x0);
    for (int j = threadIdx.x; j < 3 * kConvSpan * 4; j += blockDim.x) {
        const int q = j & 3, p = (j >> 2) % kConvSpan, dy = (j >> 2) / kConvSpan;
        const int yy = y + dy - 1, xx = ((x0 + p - 1) % W + W) % W;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (yy >= 0 && yy < H) v = *reinterpret_cast<const uint4*>(X + act_at(yy, q, xx, W));
        *reinterpret_cast<uint4*>(&sx[dy][p][8 * q]) = v;
    }
    for (int j = threadIdx.x; j < kConvTile * 4; j += blockDim.x) {
        const int q = j & 3, m = j >> 2;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (m < n) v = *reinterpret_cast<const uint4*>(dY + act_at(y, q, x0 + m, W));
        *reinterpret_cast<uint4*>(&sy[m][8 * q]) = v;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 9 * kNetC * kNetC; j += blockDim.x) {
        const int co = j % kNetC, ci = (j / kNetC) % kNetC, t = j / (kNetC * kNetC);
        const int dy = t / 3, dx = t % 3;
        float acc = 0.f;
        for (int m = 0; m < n; m++) acc += __bfloat162float(sx[dy][m + dx][ci]) * __bfloat162float(sy[m][co]);
        atomicAdd(dW + j, acc);
    }
}

// dw[t][c] += sum_p s[p + off(t)] d[p][c]: the weight gradient of the lift
// (s = its FP32 input, d = the gradient of its output) and, with the roles
// read the other way, of the projection (s = dz at p, d = g at p + off(t)).
// mode 0: lift, s shifted; mode 1: projection, d shifted. One block of 288
// threads (one weight each) per row.
__global__ void k_net_wgrad_edge(const float* s, const __nv_bfloat16* d, float* dw, int H, int W, int mode) {
    const int y = blockIdx.x;
    const int j = threadIdx.x;   // (t, c)
    if (j >= 9 * kNetC) return;
    const int t = j / kNetC, c = j % kNetC, dy = t / 3 - 1, dx = t % 3 - 1;
    const int yy = y + dy;
    if (yy < 0 || yy >= H) return;
    float acc = 0.f;
    for (int x = 0; x < W; x++) {
        const int xs = wrapx(x + dx, W);
        if (mode == 0) acc += s[(size_t)yy * W + xs] * __bfloat162float(d[act_at(y, c >> 3, x, W) + (c & 7)]);
        else acc += s[(size_t)y * W + x] * __bfloat162float(d[act_at(yy, c >> 3, xs, W) + (c & 7)]);
    }
    atomicAdd(dw + j, acc);
}

// Loss of one pair: the S-norm error that the preconditioner's Galerkin step
// leaves, S the operator the network works in (the cal_w operator in
// symmetric form, diagonally scaled: see LearnedNet::set_operator),
//   (S a)[k][i] = dg_k a - cx_k (a[i-1] + a[i+1]) - ru_k a[k+1] - rd_k a[k-1]
// on rows k < NK (periodic in i, zero beyond the rows):
//   L = min_g ||t - g z||_S^2 / ||t||_S^2 = 1 - a^2 / (b c),
//   a = (z, S t), b = (z, S z), c = (t, S t),
// independent of the scale of z, as the step is. Partials of a, b, c per block
// in FP64; S z and S t are kept for the gradient
//   dL/dz = 2 a / (b c) (g S z - S t), g = a / b.
// op rows: cx, ru, rd, diagonal ([4][H]), the operator the network works in.
__device__ __forceinline__ double s_apply_net(const float* a, const float* op, int H, int W, int NK, int k, int i) {
    const double cx = op[k], ru = op[H + k], rd = op[2 * H + k], dg = op[3 * H + k];
    const size_t row = (size_t)k * W;
    const int il = i == 0 ? W - 1 : i - 1, ir = i == W - 1 ? 0 : i + 1;
    double y = dg * a[row + i] - cx * ((double)a[row + il] + (double)a[row + ir]);
    if (k + 1 < NK) y -= ru * a[row + W + i];
    if (k > 0) y -= rd * a[row - W + i];
    return y;
}

__global__ void k_net_loss_partial(const float* z, const float* t, const float* op, int H, int W, int NK, float* sz,
                                   float* st, double* part) {
    __shared__ double sh[96];
    double v[3] = {0, 0, 0};
    const size_t n = (size_t)H * W;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(p / W), i = (int)(p - (size_t)k * W);
        double a = 0.0, b = 0.0;
        if (k < NK) {
            a = s_apply_net(z, op, H, W, NK, k, i);
            b = s_apply_net(t, op, H, W, NK, k, i);
            v[0] += (double)z[p] * b;
            v[1] += (double)z[p] * a;
            v[2] += (double)t[p] * b;
        }
        sz[p] = (float)a;
        st[p] = (float)b;
    }
    block_sum(v, sh);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = v[0];
        part[3 * blockIdx.x + 1] = v[1];
        part[3 * blockIdx.x + 2] = v[2];
    }
}

__global__ void k_net_loss_final(const double* part, int nb, double* out) {   // out: [L, a, b, c]
    __shared__ double sh[96];
    double v[3] = {0, 0, 0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        v[0] += part[3 * b];
        v[1] += part[3 * b + 1];
        v[2] += part[3 * b + 2];
    }
    block_sum(v, sh);
    if (threadIdx.x == 0) {
        out[1] = v[0];
        out[2] = v[1];
        out[3] = v[2];
        out[0] = (v[1] > 0 && v[2] > 0) ? 1.0 - v[0] * v[0] / (v[1] * v[2]) : 1.0;
    }
}

__global__ void k_net_loss_grad(const float* sz, const float* st, size_t n, const double* lt, float* dz, float mult) {
    const double a = lt[1], b = lt[2], c = lt[3];
    const bool ok = b > 0 && c > 0;
    const double f = ok ? mult * 2.0 * a / (b * c) : 0.0, g = ok ? a / b : 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dz[i] = (float)(f * (g * (double)sz[i] - (double)st[i]));
}

// Adam on FP32 master weights (gradients already averaged over the batch).
__global__ void k_net_adam(float* w, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                           float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// [H][W][32] FP32 (host order) <-> chunk-major BF16 activations.
__global__ void k_nhwc_to_act(const float* x, __nv_bfloat16* y, int H, int W) {
    const size_t n = (size_t)H * W * kNetC;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % kNetC);
        const size_t p = i / kNetC;
        const int yy = (int)(p / W), xx = (int)(p - (size_t)yy * W);
        y[act_at(yy, c >> 3, xx, W) + (c & 7)] = __float2bfloat16(x[i]);
    }
}
__global__ void k_act_to_nhwc(const __nv_bfloat16* x, float* y, int H, int W) {
    const size_t n = (size_t)H * W * kNetC;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % kNetC);
        const size_t p = i / kNetC;
        const int yy = (int)(p / W), xx = (int)(p - (size_t)yy * W);
        y[i] = __bfloat162float(x[act_at(yy, c >> 3, xx, W) + (c & 7)]);
    }
}

}  // namespace vvm

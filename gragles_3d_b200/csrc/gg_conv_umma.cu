// gg_conv_umma.cu -- mixed-path Gaussian convolution on the tcgen05 tensor cores.
//
// The convolution of box.cpp:685-795 is three applications of the real symmetric
// circulant C_n (gg_conv_tc.cuh), one per axis.  One pass contracts the contiguous
// axis of a box T[a][b][c] and writes the result rotated,
//     U[c'][a][b] = sum_c C_n[c'][c] T[a][b][c],
// so three identical passes take [z][y][x] -> [x'][z][y] -> [y'][x'][z] -> [z'][y'][x'].
// In one pass a box is an (n^2 x n) row-major matrix times C_n: a GEMM with M = n^2
// rows and K = N = n, cut into 128-row tiles (M = 128 = the TMEM lanes).  A 128-row
// tile is one contiguous span of the box.  One persistent CTA per SM takes a
// contiguous range of tiles with warp-specialised roles:
//   TMA (1 thread): cp.async.bulk of each tile span into a ring of staging buffers,
//     and of C_n (pre-split hi/lo in HBM) when the side changes;
//   split (8 warps): re-layout of a staged tile into the no-swizzle K-major
//     core-matrix layout of the MMA operand (8 rows x 16 B per core matrix, K padding
//     and rows past n^2 zero), scaled by 2^8 and split into FP16 hi + lo (22
//     significant bits; a*c ~ ah*ch + al*ch + ah*cl, about FP32 accuracy; C_n is
//     scaled by 2^8 as well and the product by 2^-16 in the epilogue, all exact);
//   MMA (1 thread): 3 * K/16 tcgen05.mma kind::f16 per tile into one of four FP32 TMEM
//     accumulators; tcgen05.commit frees the operand stage and hands the accumulator on;
//   epilogue (8 warps, two tiles at a time): tcgen05.ld of one tile row per thread, column c' stored to
//     U[c'][row]; lanes hold consecutive rows, so each store writes 128 contiguous bytes.
// Every wait is bounded: a timeout flags ERR_TIMEOUT and raises a CTA abort flag that
// ends the other roles' waits too.  Before the CTA exits, on every path, the TMA thread
// waits (bounded, whatever the abort flag says) for the last bulk copy it issued into
// each shared-memory buffer, and the MMA thread commits and waits for its last MMAs,
// so that no asynchronous write to this CTA's shared memory or TMEM is still in flight
// when TMEM is freed and the CTA's shared memory is released.
#include <cstring>
#include <cuda_fp16.h>

#include "gg_common.cuh"
#include "gg_conv_tc.cuh"

namespace gg {

namespace {

constexpr int kRows = kUmmaRows;     // MMA M and TMEM lanes
constexpr int kSplitWarps = 8;
constexpr int kEpiWarps = 8;                         // two groups of four (one per TMEM lane quarter)
constexpr int kAcc = 4;                              // TMEM accumulators
constexpr int kThreadsU = (kSplitWarps + kEpiWarps + 2) * 32;  // split, epilogue, MMA, TMA warps
constexpr int kMaxR = 4, kMaxS = 4;                  // staged tiles, operand stages
constexpr int kBars = 2 * kMaxR + 2 * kMaxS + 2 * kAcc + 2 + 2 + 1;
constexpr uint32_t kAccCols = 64;   // one accumulator: N <= round16(kUmmaMaxSide) columns
constexpr uint32_t kTmemCols = kAcc * kAccCols;
constexpr long long kWaitCycles = 1LL << 31;  // ~1 s at the B200 clock
constexpr int kSuspendNs = 1000;              // suspend-time hint of one mbarrier try_wait
constexpr float kScale = 256.f;               // operands are scaled by 2^8 before the FP16 split
constexpr float kUnscale = 1.f / 65536.f;     // the product by 2^-16

__host__ __device__ constexpr int round_k(int n) { return (n + 15) & ~15; } // K per MMA = 16 (f16)
__host__ __device__ constexpr int round_n(int n) { return (n + 15) & ~15; } // N multiple of 16 at M = 128

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// The waiting thread sleeps until the phase completes or ~kSuspendNs elapse.
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "n"(kSuspendNs)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor: no swizzle, K-major core matrices of 8 rows x 16 B,
// K-adjacent core matrices 128 B apart (LBO), 8-row groups sbo bytes apart (SBO).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           ((uint64_t)1 << 46);
}
// Instruction descriptor, kind::f16: D f32, A/B f16, both K-major, M = 128, N = np.
__device__ __forceinline__ uint32_t instr_desc(int np) {
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
// 16 consecutive 32-bit TMEM columns of this thread's lane; complete after tmem_wait().
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// FP16 hi + lo of v * 2^8 (round to nearest even, both parts).
__host__ __device__ __forceinline__ void split_f16(float v, __half& h, __half& l) {
    const float x = v * kScale;
    h = __float2half_rn(x);
    l = __float2half_rn(x - __half2float(h));
}

// The same split for a pair, with the hi part rounded in FP32 arithmetic (Veltkamp's
// splitting of x at 11 significant bits: c = (2^13 + 1) x, hi = c - (c - x)), so that
// only the two packed conversions touch the conversion unit.  hi is exact in FP16
// above the FP16 subnormal range and x - hi is exact in FP32.
__device__ __forceinline__ void split_f16x2(float v0, float v1, __half2& h, __half2& l) {
    const float x0 = __fmul_rn(v0, kScale), x1 = __fmul_rn(v1, kScale);
    const float c0 = __fmul_rn(x0, 8193.f), c1 = __fmul_rn(x1, 8193.f);
    const float h0 = __fsub_rn(c0, __fsub_rn(c0, x0)), h1 = __fsub_rn(c1, __fsub_rn(c1, x1));
    h = __floats2half2_rn(h0, h1);
    l = __floats2half2_rn(__fsub_rn(x0, h0), __fsub_rn(x1, h1));
}

// Walks the tile range of a CTA in order: grain, tile within the grain, side.
struct Cursor {
    int g, local, ntiles, n;
    const UmmaPassArgs* a;
    __device__ void load(int gg) {
        g = gg;
        ntiles = a->toff[g + 1] - a->toff[g];
        const int* b = a->box + 6 * g;
        n = b[1] - b[0];
    }
    __device__ void init(const UmmaPassArgs* args, int t) {
        a = args;
        load(tile_grain(a->toff, a->G, t));
        local = t - a->toff[g];
    }
    __device__ void advance() {
        if (++local < ntiles) return;
        local = 0;
        while (g < a->G) {  // next grain with tiles; stays in [1, G]
            load(g + 1);
            if (ntiles > 0) return;
        }
    }
    __device__ int r0() const { return local * kRows; }
    __device__ int rows() const { return min(kRows, n * n - local * kRows); }
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(bar),
                 "r"(bytes)
                 : "memory");
}
// One-dimensional bulk copy global -> shared on the TMA engine, completing on `bar`.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Bounded wait for the phase of `bar` with the given parity.  Gives up (false) when the
// CTA's abort flag is raised or after kWaitCycles, raising the flag and ERR_TIMEOUT, so
// that no role of the CTA waits for one that has stopped.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err) {
    const long long t0 = clock64();
    for (int it = 0; it < (1 << 24); it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
        if (clock64() - t0 > kWaitCycles) break;
    }
    *abort_flag = 1;
    atomicOr(err, ERR_TIMEOUT);
    return false;
}

// Bounded wait at exit for asynchronous work this thread issued (a bulk copy's
// complete_tx, or a tcgen05.commit): it ignores the abort flag, since the point is to
// let that work land before the CTA's shared memory and TMEM are released.
__device__ __forceinline__ void drain_bar(uint32_t bar, uint32_t parity, int* err) {
    const long long t0 = clock64();
    for (int it = 0; it < (1 << 24); it++) {
        if (mbar_try_wait(bar, parity)) return;
        if (clock64() - t0 > kWaitCycles) break;
    }
    atomicOr(err, ERR_TIMEOUT);
}

// Re-layout one staged tile (rows x n floats, row-major) into the MMA's K-major
// core-matrix layout, split into FP16 hi and lo.  Core matrix q = mg KC + kc holds
// rows 8 mg .. 8 mg + 7, columns 8 kc .. 8 kc + 7 as 8 rows of 16 B at byte 128 q;
// a thread writes one such row (lane % 8 = row, lane / 8 picks one of four
// consecutive core matrices), so each 8-lane phase stores one whole core matrix.
// Padding rows and columns become zero.
__device__ __forceinline__ void split_tile(const float* raw, __half* hi, __half* lo, int n, int rows, int stid) {
    const int KC = round_k(n) >> 3;
    const int w = stid >> 5, lane = stid & 31;
    const int r = lane & 7, j = lane >> 3;
    const bool vec = (n & 3) == 0;  // rows start on 16-byte boundaries
    for (int q = 4 * w + j; q < 16 * KC; q += 4 * kSplitWarps) {
        const int mg = q / KC, kc = q - mg * KC;
        const int m = 8 * mg + r, k0 = 8 * kc;
        float v[8];
        if (m < rows && vec && k0 + 8 <= n) {
            const float4 a = *reinterpret_cast<const float4*>(raw + m * n + k0);
            const float4 b = *reinterpret_cast<const float4*>(raw + m * n + k0 + 4);
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
            v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        } else {
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = (m < rows && k0 + e < n) ? raw[m * n + k0 + e] : 0.f;
        }
        __align__(16) __half2 hv[4], lv[4];
#pragma unroll
        for (int e = 0; e < 4; e++) split_f16x2(v[2 * e], v[2 * e + 1], hv[e], lv[e]);
        const int off = q * 64 + r * 8;  // halves
        *reinterpret_cast<uint4*>(hi + off) = *reinterpret_cast<const uint4*>(hv);
        *reinterpret_cast<uint4*>(lo + off) = *reinterpret_cast<const uint4*>(lv);
    }
}

// Warp roles: 0-7 split (staged tile -> hi/lo operands), 8-15 epilogue (TMEM -> HBM,
// two groups taking alternate tiles), 16 MMA issue, 17 TMA loads (one thread each).
// Rings: R staged tiles, S hi/lo operand stages, four TMEM accumulators, two C_n
// buffers switched when the side changes along the CTA's tile range.
__global__ void __launch_bounds__(kThreadsU, 1)
    conv_umma_kernel(UmmaPassArgs a, int kp_max, int np_max, int R, int S) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[kBars];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile_floats = kRows * kp_max;                  // one staged tile (fp32)
    const int tile_halves = kRows * kp_max;                  // one operand part (fp16)
    float* raw_base = reinterpret_cast<float*>(smem_raw);
    __half* op_base = reinterpret_cast<__half*>(raw_base + R * tile_floats);  // S x (hi, lo)
    __half* b_base = op_base + S * 2 * tile_halves;                          // 2 x (hi, lo) C_n
    const int b_halves = 2 * np_max * kp_max;
    auto bar = [&](int i) { return smem_u32(&bars[i]); };
    constexpr int RFULL = 0, REMPTY = kMaxR, FULL = 2 * kMaxR, EMPTY = FULL + kMaxS, TFULL = EMPTY + kMaxS,
                  TEMPTY = TFULL + kAcc, BFULL = TEMPTY + kAcc, BFREE = BFULL + 2, DRAIN = BFREE + 2;

    const int total = a.toff[a.G + 1];
    const int t_begin = (int)((long long)total * blockIdx.x / gridDim.x);
    const int t_end = (int)((long long)total * (blockIdx.x + 1) / gridDim.x);
    if (t_begin >= t_end) return;
    const int count = t_end - t_begin;

    if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), kTmemCols);
    if (tid == 0) {
        for (int r = 0; r < R; r++) {
            mbar_init(bar(RFULL + r), 1);
            mbar_init(bar(REMPTY + r), kSplitWarps);  // one arrive per warp
        }
        for (int s = 0; s < S; s++) {
            mbar_init(bar(FULL + s), kSplitWarps);
            mbar_init(bar(EMPTY + s), 1);
        }
        for (int b = 0; b < kAcc; b++) {
            mbar_init(bar(TFULL + b), 1);
            mbar_init(bar(TEMPTY + b), 4);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(bar(BFULL + b), 1);
            mbar_init(bar(BFREE + b), 1);
        }
        mbar_init(bar(DRAIN), 1);
        abort_flag = 0;
    }
    // a side beyond the launch's shared-memory sizing would overrun the buffers
    bool sized = true;
    if (warp == 0)
        for (int t = t_begin + lane; t < t_end; t += 32) {
            const int* bx = a.box + 6 * tile_grain(a.toff, a.G, t);
            const int n = bx[1] - bx[0];
            if (n < 1 || round_k(n) > kp_max || round_n(n) > np_max || n > kUmmaMaxSide) sized = false;
        }
    tc_fence_before();
    sized = __syncthreads_and(sized);
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    if (!sized && tid == 0) atomicOr(a.err, ERR_BOX);
    volatile int* ab = &abort_flag;

    if (!sized) {
    } else if (warp < kSplitWarps) {
        // ---------------- split ----------------
        Cursor c;
        c.init(&a, t_begin);
        for (int i = 0; i < count; i++, c.advance()) {
            const int r = i % R, s = i % S;
            if (!wait_bar(bar(RFULL + r), (i / R) & 1, ab, a.err)) break;
            if (i >= S && !wait_bar(bar(EMPTY + s), (i / S - 1) & 1, ab, a.err)) break;
            __half* hi = op_base + s * 2 * tile_halves;
            split_tile(raw_base + r * tile_floats, hi, hi + tile_halves, c.n, c.rows(), tid);
            // every lane's stores visible to the tensor core, then one arrive per warp
            // (arrives on one barrier serialise, so 256 of them would cost microseconds)
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(bar(REMPTY + r));
                mbar_arrive(bar(FULL + s));
            }
        }
    } else if (warp < kSplitWarps + kEpiWarps) {
        // ---------------- epilogue: group e drains tiles i = e mod 2 ----------------
        const int q = warp & 3;  // TMEM lane quarter of this warp
        const int e = (warp - kSplitWarps) >> 2;
        Cursor c;
        c.init(&a, t_begin);
        if (e) c.advance();
        for (int i = e; i < count; i += 2, c.advance(), c.advance()) {
            const int b = i % kAcc;
            if (!wait_bar(bar(TFULL + b), (i / kAcc) & 1, ab, a.err)) break;
            tc_fence_after();
            const int n = c.n, np = round_n(n);
            const int row = q * 32 + lane;
            const long long n2 = (long long)n * n;
            float* dst = a.dst + a.dst_off[c.g] + c.r0() + row;
            const bool live = row < c.rows();
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kAccCols);
            float v[kAccCols];
#pragma unroll
            for (int c0 = 0; c0 < (int)kAccCols; c0 += 16)
                if (c0 < np) tmem_ld16(trow + (uint32_t)c0, v + c0);
            tmem_wait();
            // the accumulator is in registers: hand it back before the stores, so that the
            // arrive's release does not wait for them
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(TEMPTY + b));
            if (live) {
                float* p = dst;
#pragma unroll
                for (int cc = 0; cc < (int)kAccCols; cc++, p += n2)
                    if (cc < n) *p = v[cc] * kUnscale;
            }
        }
    } else if (warp == kSplitWarps + kEpiWarps && lane == 0) {
        // ---------------- MMA issue ----------------
        Cursor c;
        c.init(&a, t_begin);
        int cur_n = -1, nsw = 0, kb = 0;
        bool issued = false;
        for (int i = 0; i < count; i++, c.advance()) {
            const int s = i % S, b = i % kAcc;
            if (!wait_bar(bar(FULL + s), (i / S) & 1, ab, a.err)) break;
            if (c.n != cur_n) {
                kb = nsw & 1;
                if (nsw >= 1) mma_commit(bar(BFREE + (kb ^ 1)));  // after every MMA on the old C_n
                if (!wait_bar(bar(BFULL + kb), (nsw >> 1) & 1, ab, a.err)) break;
                cur_n = c.n;
                nsw++;
            }
            if (i >= kAcc && !wait_bar(bar(TEMPTY + b), (i / kAcc - 1) & 1, ab, a.err)) break;
            tc_fence_after();
            const int kp = round_k(c.n), np = round_n(c.n);
            const uint32_t sbo = 16u * kp;  // 8 rows x kp halves
            const __half* hi = op_base + s * 2 * tile_halves;
            const uint32_t a_hi = smem_u32(hi), a_lo = smem_u32(hi + tile_halves);
            const __half* bk = b_base + kb * b_halves;
            const uint32_t b_hi = smem_u32(bk), b_lo = smem_u32(bk + np * kp);
            const uint32_t idesc = instr_desc(np);
            const uint32_t d = tmem + (uint32_t)(b * kAccCols);
            for (int j = 0; j < kp / 16; j++) {
                const uint32_t o = 256u * j;  // two 128-B core matrices along K
                mma_f16(d, smem_desc(a_lo + o, sbo), smem_desc(b_hi + o, sbo), idesc, j > 0);
                mma_f16(d, smem_desc(a_hi + o, sbo), smem_desc(b_lo + o, sbo), idesc, 1);
                mma_f16(d, smem_desc(a_hi + o, sbo), smem_desc(b_hi + o, sbo), idesc, 1);
            }
            issued = true;
            mma_commit(bar(EMPTY + s));
            mma_commit(bar(TFULL + b));
        }
        if (issued) {  // every MMA issued above has completed before TMEM is freed
            mma_commit(bar(DRAIN));
            drain_bar(bar(DRAIN), 0, a.err);
        }
    } else if (warp == kSplitWarps + kEpiWarps + 1 && lane == 0) {
        // ---------------- TMA loads ----------------
        Cursor c;
        c.init(&a, t_begin);
        int cur_n = -1, nsw = 0;
        int last_tile[kMaxR] = {-1, -1, -1, -1}, last_b[2] = {-1, -1};  // last copy into each buffer
        for (int i = 0; i < count; i++, c.advance()) {
            const int r = i % R;
            if (i >= R && !wait_bar(bar(REMPTY + r), (i / R - 1) & 1, ab, a.err)) break;
            if (c.n != cur_n) {
                const int kb = nsw & 1;
                if (nsw >= 2 && !wait_bar(bar(BFREE + kb), ((nsw - 2) >> 1) & 1, ab, a.err)) break;
                const uint32_t bytes = 2u * round_n(c.n) * round_k(c.n) * 2u;
                mbar_expect_tx(bar(BFULL + kb), bytes);
                bulk_load(smem_u32(b_base + kb * b_halves), a.bmat + a.boff[c.n], bytes, bar(BFULL + kb));
                last_b[kb] = nsw;
                cur_n = c.n;
                nsw++;
            }
            // rows x n contiguous floats; 16-byte aligned start, length rounded up to 16 B
            const uint32_t bytes = ((uint32_t)(c.rows() * c.n) * 4u + 15u) & ~15u;
            mbar_expect_tx(bar(RFULL + r), bytes);
            bulk_load(smem_u32(raw_base + r * tile_floats), a.src + a.src_off[c.g] + (long long)c.r0() * c.n, bytes,
                      bar(RFULL + r));
            last_tile[r] = i;
        }
        // the copies land before the CTA exits, also when a role gave up early
        for (int r = 0; r < R && r < kMaxR; r++)
            if (last_tile[r] >= 0) drain_bar(bar(RFULL + r), (last_tile[r] / R) & 1, a.err);
        for (int kb = 0; kb < 2; kb++)
            if (last_b[kb] >= 0) drain_bar(bar(BFULL + kb), (last_b[kb] >> 1) & 1, a.err);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

struct UmmaShape {
    int kp, np, R, S;
    size_t smem;
};

UmmaShape umma_shape(int side_max) {
    UmmaShape sh{round_k(side_max), round_n(side_max), 0, 0, 0};
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (optin <= 0) optin = 227 * 1024;
    const size_t room = (size_t)optin - 2048;
    const size_t tile = (size_t)kRows * sh.kp * sizeof(float);    // staged fp32 tile
    const size_t part = (size_t)kRows * sh.kp * sizeof(__half);   // one fp16 operand part
    const size_t bbytes = 2 * 2 * (size_t)sh.np * sh.kp * sizeof(__half);
    // deepest rings that fit, staged tiles at least as deep as operand stages
    const int order[][2] = {{4, 4}, {4, 3}, {3, 3}, {3, 2}, {2, 2}, {2, 1}};
    for (const auto& rs : order) {
        const size_t need = rs[0] * tile + 2 * rs[1] * part + bbytes;
        if (need <= room) {
            sh.R = rs[0];
            sh.S = rs[1];
            sh.smem = need;
            return sh;
        }
    }
    return sh;
}

}  // namespace

int umma_side_limit() { return kUmmaMaxSide; }

bool umma_supported(int side_max) { return side_max >= 1 && side_max <= kUmmaMaxSide && umma_shape(side_max).R >= 2; }

void umma_tables(int N, double time_step, int nmax, std::vector<uint16_t>& bmat, std::vector<long long>& boff) {
    boff.assign(nmax + 2, 0);
    for (int n = 1; n <= nmax; n++) {
        std::vector<float> C;
        circulant_matrix(n, N, time_step, C);
        const int kp = round_k(n), np = round_n(n), KC = kp / 8;
        const size_t base = bmat.size();
        boff[n] = (long long)base;
        bmat.resize(base + 2 * (size_t)np * kp, 0);
        for (int r = 0; r < n; r++)
            for (int k = 0; k < n; k++) {
                // B[k][r] = C[r][k] as the N x K K-major operand (row r = output column)
                __half h, l;
                split_f16(C[(size_t)r * n + k], h, l);
                const size_t pos = ((size_t)(r / 8) * KC + k / 8) * 64 + (r % 8) * 8 + (k % 8);
                bmat[base + pos] = __half_as_ushort(h);
                bmat[base + (size_t)np * kp + pos] = __half_as_ushort(l);
            }
    }
}

void launch_conv_umma(const UmmaConvArgs& c, int num_sms, int side_max, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(conv_umma_kernel);
    });
    const UmmaShape sh = umma_shape(side_max);
    UmmaPassArgs p{};
    p.G = c.G;
    p.toff = c.toff;
    p.box = c.box;
    p.bmat = c.bmat;
    p.boff = c.boff;
    p.err = c.err;
    p.side_max = side_max;
    // [z][y][x] -> [x'][z][y] -> [y'][x'][z] -> [z'][y'][x']
    const float* srcs[3] = {c.in, c.out, c.scratch};
    const long long* src_offs[3] = {c.in_off, c.out_off, c.out_off};
    float* dsts[3] = {c.out, c.scratch, c.out};
    for (int pass = 0; pass < 3; pass++) {
        p.src = srcs[pass];
        p.src_off = src_offs[pass];
        p.dst = dsts[pass];
        p.dst_off = c.out_off;
        conv_umma_kernel<<<num_sms, kThreadsU, sh.smem, s>>>(p, sh.kp, sh.np, sh.R, sh.S);
    }
}

}  // namespace gg

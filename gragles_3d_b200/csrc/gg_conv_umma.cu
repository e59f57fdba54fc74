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
//     and rows past n^2 zero), split into TF32 hi and lo (3xTF32: a*b ~ ah*bh + al*bh
//     + ah*bl, about FP32 accuracy);
//   MMA (1 thread): 3 * K/8 tcgen05.mma kind::tf32 per tile into one of two FP32 TMEM
//     accumulators; tcgen05.commit frees the operand stage and hands the accumulator on;
//   epilogue (4 warps): tcgen05.ld of one tile row per thread, column c' stored to
//     U[c'][row]; lanes hold consecutive rows, so each store writes 128 contiguous bytes.
// Every wait is bounded: a timeout flags ERR_TIMEOUT and raises a CTA abort flag that
// ends the other roles' waits too; TMEM is freed on every exit path.
#include <cstring>

#include "gg_common.cuh"
#include "gg_conv_tc.cuh"

namespace gg {

namespace {

constexpr int kRows = kUmmaRows;     // MMA M and TMEM lanes
constexpr int kSplitWarps = 8;
constexpr int kThreadsU = (kSplitWarps + 6) * 32;  // split, 4 epilogue, MMA, TMA warps
constexpr int kBars = 20;
constexpr uint32_t kAccCols = 64;   // one accumulator: N <= round16(kUmmaMaxSide) columns
constexpr uint32_t kTmemCols = 128; // two accumulators
constexpr long long kWaitCycles = 1LL << 31;  // ~1 s at the B200 clock

__host__ __device__ constexpr int round_k(int n) { return (n + 7) & ~7; }   // K per MMA = 8 (tf32)
__host__ __device__ constexpr int round_n(int n) { return (n + 15) & ~15; } // N multiple of 16 at M = 128

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
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
// Instruction descriptor, kind::tf32: D f32, A/B tf32, both K-major, M = 128, N = np.
__device__ __forceinline__ uint32_t instr_desc(int np) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// TF32 part of v: round to nearest (ties away) at 10 explicit mantissa bits.
__host__ __device__ __forceinline__ float tf32_hi(float v) {
    uint32_t u;
#ifdef __CUDA_ARCH__
    u = __float_as_uint(v);
#else
    std::memcpy(&u, &v, 4);
#endif
    u = (u + 0x1000u) & 0xFFFFE000u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float r;
    std::memcpy(&r, &u, 4);
    return r;
#endif
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
    for (int it = 0; it < (1 << 30); it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 15) == 15) {
            if (*abort_flag) return false;
            if (clock64() - t0 > kWaitCycles) break;
        }
    }
    *abort_flag = 1;
    atomicOr(err, ERR_TIMEOUT);
    return false;
}

// Re-layout one staged tile (rows x n floats, row-major) into the MMA's K-major
// core-matrix layout, split into TF32 hi and lo.  Canonical element p = tid + 256 j is
// core matrix cm = p / 32 (8-row group mg = cm / KC, K chunk kc = cm % KC), row
// 8 mg + lane / 4, column 4 kc + lane % 4; padding rows and columns become zero.
__device__ __forceinline__ void split_tile(const float* raw, float* hi, float* lo, int n, int rows, int stid) {
    const int kp = round_k(n), KC = kp >> 2;
    const int w = stid >> 5, lane = stid & 31;
    const int mlo = lane >> 2, klo = lane & 3;
    int mg = w / KC, kc = w - (w / KC) * KC;
    for (int cm = w; cm < 16 * KC; cm += kSplitWarps) {
        const int m = 8 * mg + mlo, k = 4 * kc + klo;
        const float v = (m < rows && k < n) ? raw[m * n + k] : 0.f;
        const float h = tf32_hi(v);
        const int p = 32 * cm + lane;
        hi[p] = h;
        lo[p] = tf32_hi(v - h);
        kc += kSplitWarps;
        while (kc >= KC) {
            kc -= KC;
            mg++;
        }
    }
}

// Warp roles: 0-7 split (staged tile -> hi/lo operands), 8-11 epilogue (TMEM -> HBM),
// 12 MMA issue, 13 TMA loads (one thread each).  Rings: R staged tiles, S hi/lo
// operand stages, two TMEM accumulators, two C_n buffers switched when the side
// changes along the CTA's tile range.
__global__ void __launch_bounds__(kThreadsU, 1)
    conv_umma_kernel(UmmaPassArgs a, int kp_max, int np_max, int R, int S) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[kBars];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile_floats = kRows * kp_max;
    float* raw_base = reinterpret_cast<float*>(smem_raw);
    float* op_base = raw_base + R * tile_floats;            // S x (hi, lo)
    float* b_base = op_base + S * 2 * tile_floats;           // 2 x (hi, lo) C_n
    const int b_floats = 2 * np_max * kp_max;
    auto bar = [&](int i) { return smem_u32(&bars[i]); };
    constexpr int RFULL = 0, REMPTY = 4, FULL = 8, EMPTY = 10, TFULL = 12, TEMPTY = 14, BFULL = 16, BFREE = 18;

    const int total = a.toff[a.G + 1];
    const int t_begin = (int)((long long)total * blockIdx.x / gridDim.x);
    const int t_end = (int)((long long)total * (blockIdx.x + 1) / gridDim.x);
    if (t_begin >= t_end) return;
    const int count = t_end - t_begin;

    if (warp == 0) tmem_alloc(smem_u32(&tmem_slot), kTmemCols);
    if (tid == 0) {
        for (int r = 0; r < R; r++) {
            mbar_init(bar(RFULL + r), 1);
            mbar_init(bar(REMPTY + r), kSplitWarps * 32);
        }
        for (int s = 0; s < S; s++) {
            mbar_init(bar(FULL + s), kSplitWarps * 32);
            mbar_init(bar(EMPTY + s), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(bar(TFULL + b), 1);
            mbar_init(bar(TEMPTY + b), 128);
            mbar_init(bar(BFULL + b), 1);
            mbar_init(bar(BFREE + b), 1);
        }
        abort_flag = 0;
    }
    // a side beyond the launch's shared-memory sizing would overrun the buffers
    bool sized = true;
    {
        Cursor c;
        c.init(&a, t_begin);
        for (int i = 0; i < count; i++, c.advance())
            if (c.n < 1 || round_k(c.n) > kp_max || round_n(c.n) > np_max || c.n > kUmmaMaxSide) sized = false;
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
            float* hi = op_base + s * 2 * tile_floats;
            split_tile(raw_base + r * tile_floats, hi, hi + tile_floats, c.n, c.rows(), tid);
            fence_proxy_async();
            mbar_arrive(bar(REMPTY + r));
            mbar_arrive(bar(FULL + s));
        }
    } else if (warp < kSplitWarps + 4) {
        // ---------------- epilogue ----------------
        const int q = warp & 3;  // TMEM lane quarter of this warp
        Cursor c;
        c.init(&a, t_begin);
        for (int i = 0; i < count; i++, c.advance()) {
            const int b = i & 1;
            if (!wait_bar(bar(TFULL + b), (i >> 1) & 1, ab, a.err)) break;
            tc_fence_after();
            const int n = c.n, np = round_n(n);
            const int row = q * 32 + lane;
            const long long n2 = (long long)n * n;
            float* dst = a.dst + a.dst_off[c.g] + c.r0() + row;
            const bool live = row < c.rows();
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kAccCols);
            for (int c0 = 0; c0 < np; c0 += 16) {
                float v[16];
                tmem_ld16(trow + (uint32_t)c0, v);
                if (live) {
#pragma unroll
                    for (int cc = 0; cc < 16; cc++)
                        if (c0 + cc < n) dst[(long long)(c0 + cc) * n2] = v[cc];
                }
            }
            tc_fence_before();
            mbar_arrive(bar(TEMPTY + b));
        }
    } else if (warp == kSplitWarps + 4 && lane == 0) {
        // ---------------- MMA issue ----------------
        Cursor c;
        c.init(&a, t_begin);
        int cur_n = -1, nsw = 0, kb = 0;
        for (int i = 0; i < count; i++, c.advance()) {
            const int s = i % S, b = i & 1;
            if (!wait_bar(bar(FULL + s), (i / S) & 1, ab, a.err)) break;
            if (c.n != cur_n) {
                kb = nsw & 1;
                if (nsw >= 1) mma_commit(bar(BFREE + (kb ^ 1)));  // after every MMA on the old C_n
                if (!wait_bar(bar(BFULL + kb), (nsw >> 1) & 1, ab, a.err)) break;
                cur_n = c.n;
                nsw++;
            }
            if (i >= 2 && !wait_bar(bar(TEMPTY + b), ((i >> 1) - 1) & 1, ab, a.err)) break;
            tc_fence_after();
            const int kp = round_k(c.n), np = round_n(c.n);
            const uint32_t sbo = 32u * kp;  // 8 rows x kp floats
            const float* hi = op_base + s * 2 * tile_floats;
            const uint32_t a_hi = smem_u32(hi), a_lo = smem_u32(hi + tile_floats);
            const float* bk = b_base + kb * b_floats;
            const uint32_t b_hi = smem_u32(bk), b_lo = smem_u32(bk + np * kp);
            const uint32_t idesc = instr_desc(np);
            const uint32_t d = tmem + (uint32_t)(b * kAccCols);
            for (int j = 0; j < kp / 8; j++) {
                const uint32_t o = 256u * j;  // two 128-B core matrices along K
                mma_tf32(d, smem_desc(a_lo + o, sbo), smem_desc(b_hi + o, sbo), idesc, j > 0);
                mma_tf32(d, smem_desc(a_hi + o, sbo), smem_desc(b_lo + o, sbo), idesc, 1);
                mma_tf32(d, smem_desc(a_hi + o, sbo), smem_desc(b_hi + o, sbo), idesc, 1);
            }
            mma_commit(bar(EMPTY + s));
            mma_commit(bar(TFULL + b));
        }
    } else if (warp == kSplitWarps + 5 && lane == 0) {
        // ---------------- TMA loads ----------------
        Cursor c;
        c.init(&a, t_begin);
        int cur_n = -1, nsw = 0;
        for (int i = 0; i < count; i++, c.advance()) {
            const int r = i % R;
            if (i >= R && !wait_bar(bar(REMPTY + r), (i / R - 1) & 1, ab, a.err)) break;
            if (c.n != cur_n) {
                const int kb = nsw & 1;
                if (nsw >= 2 && !wait_bar(bar(BFREE + kb), ((nsw - 2) >> 1) & 1, ab, a.err)) break;
                const uint32_t bytes = 2u * round_n(c.n) * round_k(c.n) * 4u;
                mbar_expect_tx(bar(BFULL + kb), bytes);
                bulk_load(smem_u32(b_base + kb * b_floats), a.bmat + a.boff[c.n], bytes, bar(BFULL + kb));
                cur_n = c.n;
                nsw++;
            }
            // rows x n contiguous floats; 16-byte aligned start, length rounded up to 16 B
            const uint32_t bytes = ((uint32_t)(c.rows() * c.n) * 4u + 15u) & ~15u;
            mbar_expect_tx(bar(RFULL + r), bytes);
            bulk_load(smem_u32(raw_base + r * tile_floats), a.src + a.src_off[c.g] + (long long)c.r0() * c.n, bytes,
                      bar(RFULL + r));
        }
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
    const size_t tile = (size_t)kRows * sh.kp * sizeof(float);
    const size_t bbytes = 2 * 2 * (size_t)sh.np * sh.kp * sizeof(float);
    for (int S = 2; S >= 1; S--)
        for (int R = 4; R >= 2; R--) {
            const size_t need = R * tile + 2 * S * tile + bbytes;
            if (need <= room) {
                sh.R = R;
                sh.S = S;
                sh.smem = need;
                return sh;
            }
        }
    return sh;
}

}  // namespace

int umma_side_limit() { return kUmmaMaxSide; }

bool umma_supported(int side_max) { return side_max >= 1 && side_max <= kUmmaMaxSide && umma_shape(side_max).R >= 2; }

void umma_tables(int N, double time_step, int nmax, std::vector<float>& bmat, std::vector<long long>& boff) {
    boff.assign(nmax + 2, 0);
    for (int n = 1; n <= nmax; n++) {
        std::vector<float> C;
        circulant_matrix(n, N, time_step, C);
        const int kp = round_k(n), np = round_n(n);
        const size_t base = bmat.size();
        boff[n] = (long long)base;
        bmat.resize(base + 2 * (size_t)np * kp, 0.f);
        for (int r = 0; r < n; r++)
            for (int k = 0; k < n; k++) {
                // B[k][r] = C[r][k] as the N x K K-major operand (row r = output column)
                const float v = C[(size_t)r * n + k];
                const float hi = tf32_hi(v);
                const size_t pos = (size_t)(r / 8) * 8 * kp + (size_t)(k / 4) * 32 + (r % 8) * 4 + (k % 4);
                bmat[base + pos] = hi;
                bmat[base + (size_t)np * kp + pos] = tf32_hi(v - hi);
            }
    }
}

void launch_conv_umma(const UmmaConvArgs& c, int num_sms, int side_max, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        allow_max_dynamic_smem(conv_umma_kernel);
        configured = true;
    }
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

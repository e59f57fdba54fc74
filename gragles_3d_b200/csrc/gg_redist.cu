// gg_redist.cu -- directional-sweep redistancing of every grain.
//
// Stands in for LSbox::executeRedistancing (box.cpp:2322-2586).  The reference
// clears the new (resized) output box to -1, then for every z-slice of the in/out
// intersection except the last runs four sweeps (x forward, x backward, y forward,
// y backward), then sweeps z forward and backward over all columns, and clamps to
// +-delta.  Every sweep is a recurrence along one line and the lines of a sweep are
// independent, so a thread runs one line, and a CTA runs one to five units side by side
// (all of one grain; the count is fixed per box-size class so that 120-128 lanes have a
// line):
//   kernel xy: a unit is (grain, output z-slice); the slice of the output sits in shared
//              memory, threads run rows for the x sweeps and columns for the y sweeps;
//   kernel z:  a unit is (grain, output y-row); the [z][x] plane of the row sits in shared
//              memory and threads run the z recurrences of one column each (x-adjacent
//              threads touch adjacent words).
// A unit's buffers are small (two n x n planes).  Its input values on the in/out
// intersection are staged next to it with coalesced loads over one flat range (a
// recurrence that read HBM step by step would wait on every load).  Along a line the
// value that the next step updates is carried in a register, so a step costs its
// arithmetic and shared-memory loads that do not depend on the chain.  The arithmetic
// is the reference's, statement by statement (no contraction), and the lines of a sweep
// run in the reference's order, so the FP64 result is bit-identical.
#include "gg_kernels.cuh"

namespace gg {

namespace {

constexpr int kMaxThreads = 128;  // one thread per line up to side 128, then lines loop

struct Intersect {
    int xmin, xmax, ymin, ymax, zmin, zmax;
    __device__ Intersect(const Box& ib, const Box& ob) {
        xmin = ib.x0 < ob.x0 ? ob.x0 : ib.x0;
        ymin = ib.y0 < ob.y0 ? ob.y0 : ib.y0;
        zmin = ib.z0 < ob.z0 ? ob.z0 : ib.z0;
        xmax = ib.x1 < ob.x1 ? ib.x1 : ob.x1;
        ymax = ib.y1 < ob.y1 ? ib.y1 : ob.y1;
        zmax = ib.z1 < ob.z1 ? ib.z1 : ob.z1;
    }
};

// q / d for 0 <= q < 2^12 and 1 <= d <= 64, from d's FP32 reciprocal: (q + 1/2) / d lies
// at least 1/(2d) from an integer and the product's rounding error is below 2^-10.
// S = 0 (the runtime-pitch kernels, any side): the integer division.
template <int S>
__device__ __forceinline__ int div_small(int q, int d, float rd) {
    if (S) return __float2int_rz(((float)q + 0.5f) * rd);
    return q / d;
}

// 4- or 8-byte asynchronous copy to a shared-memory address given as a 32-bit offset.
template <typename T>
__device__ __forceinline__ void cp_async_to(uint32_t dst, const T* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(src), "n"(sizeof(T)) : "memory");
}

// isgn(s) * h of the reference: h, -h or +0 (isgn is 0 for +-0 and NaN), as a sign copy.
__device__ __forceinline__ float copysign_t(float h, float s) { return copysignf(h, s); }
__device__ __forceinline__ double copysign_t(double h, double s) { return copysign(h, s); }
template <typename T>
__device__ __forceinline__ T sgn_h(T s, T h) {
    return fabs(s) > T(0) ? copysign_t(h, s) : T(0);
}

// The propagation step: out_next takes out_here + isgn(src) * h when that is closer to 0.
template <typename T>
__device__ __forceinline__ void step_prop(T src, T out_here, T& out_next, T h) {
    const T candidate = out_here + sgn_h(src, h);
    if (fabs(candidate) < fabs(out_next)) out_next = candidate;
}

// The interpolation step at a sign change between a (here) and b (next), then the
// candidate propagated to next; box.cpp:2370-2391 and the y/z twins.
template <typename T>
__device__ __forceinline__ void step_in(T a, T b, T& out_here, T& out_next, T h) {
    if (a * b <= T(0)) {
        const T i_slope = (b - a) / h;
        const T distToZero = -a / i_slope;
        if (fabs(out_here) > fabs(distToZero)) out_here = -distToZero * isgn(i_slope);
    }
    step_prop(b, out_here, out_next, h);
}

// `count` steps along one line from op = &o[p] (cur = o[p]), moving s elements a step
// (s < 0 backwards); the input value at a position sits d elements after the output's.
// Each step stores o[p] and carries the updated o[p + s].  MODE 0 propagates with the
// sign of o[p + s] itself, MODE 1 with the sign of in[p + s], MODE 2 is step_in between
// in[p] and in[p + s].  Steps run four at a time with their loads issued first; in
// MODE 2 a group without a sign change in the input (nearly all of them) takes the
// propagation alone, which is what step_in does there, with one sign for the group.
// s and d are compile-time constants for the fixed-pitch classes, so every address is a
// register plus an offset.
template <typename T, int MODE>
__device__ __forceinline__ T* line_steps(T* op, T& cur, int count, int s, int d, T h) {
    int k = 0;
    if constexpr (MODE == 2) {
        if (count <= 0) return op;
        T a = op[d];
        for (; k + 4 <= count; k += 4, op += 4 * s) {
            T nx[4], b[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                nx[j] = op[(j + 1) * s];
                b[j] = op[d + (j + 1) * s];
            }
            const bool change = (a * b[0] <= T(0)) | (b[0] * b[1] <= T(0)) | (b[1] * b[2] <= T(0)) |
                                (b[2] * b[3] <= T(0));
            if (change) {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    step_in(j ? b[j - 1] : a, b[j], cur, nx[j], h);
                    op[j * s] = cur;
                    cur = nx[j];
                }
            } else {
                // a * b > 0 at every step: a and the four b share one sign and none is
                // 0, so isgn(b) * h is the same for the four steps
                const T inc = copysign_t(h, a);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const T candidate = cur + inc;
                    if (fabs(candidate) < fabs(nx[j])) nx[j] = candidate;
                    op[j * s] = cur;
                    cur = nx[j];
                }
            }
            a = b[3];
        }
        for (; k < count; k++, op += s) {
            T nx = op[s];
            const T b = op[d + s];
            step_in(a, b, cur, nx, h);
            *op = cur;
            cur = nx;
            a = b;
        }
        return op;
    } else {
        for (; k + 4 <= count; k += 4, op += 4 * s) {
            T nx[4], src[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                nx[j] = op[(j + 1) * s];
                src[j] = MODE == 1 ? op[d + (j + 1) * s] : nx[j];
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                step_prop(src[j], cur, nx[j], h);
                op[j * s] = cur;
                cur = nx[j];
            }
        }
        for (; k < count; k++, op += s) {
            T nx = op[s];
            step_prop(MODE == 1 ? op[d + s] : nx, cur, nx, h);
            *op = cur;
            cur = nx;
        }
        return op;
    }
}

// Forward sweep over positions p0 .. p_end - 1 of a line with stride so, the input d
// elements after the output.  The reference's x/y/z forward loops (box.cpp:2367-2401,
// 2437-2472, 2501-2538) take step_in while p < p_in_end - 1 (and inside), else the
// propagation with the output's own sign: a prefix, so the loop is split in two.
template <typename T>
__device__ __forceinline__ void sweep_forward(T* o, int so, int d, int p0, int p_end, int p_in_end, bool inside,
                                              T h) {
    if (p0 >= p_end - 1) return;
    T* op = o + p0 * so;
    T cur = *op;
    const int pin = inside ? min(p_in_end - 1, p_end - 1) : p0;
    const int nin = pin > p0 ? pin - p0 : 0;
    op = line_steps<T, 2>(op, cur, nin, so, d, h);
    op = line_steps<T, 0>(op, cur, p_end - 1 - p0 - nin, so, d, h);
    *op = cur;
}

// Backward propagation from p_start down to p_lo + 1 (box.cpp:2403-2435, 2474-2496):
// the sign of in(p - 1) while p > p_in_lo (and inside), else of the output itself.
// out(p_start) is never modified (storing it back leaves it as it was).
template <typename T>
__device__ __forceinline__ void sweep_backward_prop(T* o, int so, int d, int p_start, int p_lo, int p_in_lo,
                                                    bool inside, T h) {
    if (p_start <= p_lo) return;
    T* op = o + p_start * so;
    T cur = *op;
    const int plim = max(p_in_lo, p_lo);
    const int nin = inside && p_start > plim ? p_start - plim : 0;
    op = line_steps<T, 1>(op, cur, nin, -so, d, h);
    op = line_steps<T, 0>(op, cur, p_start - nin - p_lo, -so, d, h);
    *op = cur;
}

// Backward sweep with interpolation (the z backward loop, box.cpp:2539-2576): step_in
// while p > p_in_lo (and inside), else the propagation with the output's own sign.
template <typename T>
__device__ __forceinline__ void sweep_backward_in(T* o, int so, int d, int p_start, int p_lo, int p_in_lo,
                                                  bool inside, T h) {
    if (p_start <= p_lo) return;
    T* op = o + p_start * so;
    T cur = *op;
    const int plim = max(p_in_lo, p_lo);
    const int nin = inside && p_start > plim ? p_start - plim : 0;
    op = line_steps<T, 2>(op, cur, nin, -so, d, h);
    op = line_steps<T, 0>(op, cur, p_start - nin - p_lo, -so, d, h);
    *op = cur;
}

// Shared-memory layout of a fixed-pitch class of largest side S (even, a multiple of 8):
// one unit's output plane and input plane of S rows of pitch S + 1 (xy) or S x S (z),
// units spaced so that lane t of the CTA, unit t / S, line t % S, reads bank t mod 32 in
// every sweep (the unit stride is congruent to S modulo 32, as S (S + 1) is).
__host__ __device__ constexpr int xy_unit_stride(int S) { return 2 * S * (S + 1) + (32 - S % 32) % 32; }
static_assert(xy_unit_stride(24) % 4 == 0 && xy_unit_stride(40) % 4 == 0 && xy_unit_stride(56) % 4 == 0,
              "unit planes start on 16 bytes");
__host__ __device__ constexpr int z_unit_stride(int S) { return 2 * S * S + S % 32; }
__host__ __device__ constexpr int class_threads(int S, int U) { return S ? (U * S + 31) / 32 * 32 : kMaxThreads; }

// Kernel xy: a CTA per (grain, U consecutive output z-slices); unit u of the CTA owns
// slice ob.z0 + U * tile + u, its threads run its rows for the x sweeps and its columns
// for the y sweeps.  S = 0: one unit of runtime pitch (sides above the fixed classes).
template <typename T, int S, int U>
__global__ void __launch_bounds__(kMaxThreads) redist_xy_kernel(RedistArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int u = S ? tid / S : 0;
    const int line = S ? tid - u * S : tid;
    const int lstride = S ? S : blockDim.x;
    const T h = (T)a.geo.h;
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        const Box ob = a.out.grain_box(g);
        const Box ib = a.in.grain_box(g);
        const int k = ob.z0 + w.local * U + u;
        const bool unit = u < U && k < ob.z1;
        const Intersect I(ib, ob);
        const int nx = ob.nx(), ny = ob.ny();
        const int P = S ? S + 1 : (nx | 1);
        const int PL = S ? S * (S + 1) : ny * P;  // the input plane follows the output plane
        T* O = reinterpret_cast<T*>(smem_raw) + (S ? u * xy_unit_stride(S) : 0);
        T* In = O + PL;
        T* outg = a.out.grain_ptr(g) + (long long)(k - ob.z0) * nx * ny;
        const bool sweeps = unit && k >= I.zmin && k < I.zmax - 1;
        if (unit && !sweeps)  // no xy sweep reaches this slice
            for (int q = line; q < nx * ny; q += lstride) outg[q] = T(-1);
        if (sweeps) {
            // O (16-byte aligned: every unit stride is a multiple of 4 elements) to -1,
            // 16 bytes a store
            constexpr int kPer = 16 / (int)sizeof(T);
            const uint4 m1 = sizeof(T) == 4 ? make_uint4(0xBF800000u, 0xBF800000u, 0xBF800000u, 0xBF800000u)
                                            : make_uint4(0u, 0xBFF00000u, 0u, 0xBFF00000u);
            const int n4 = ny * P / kPer;
            for (int q = line; q < n4; q += lstride) reinterpret_cast<uint4*>(O)[q] = m1;
            for (int q = n4 * kPer + line; q < ny * P; q += lstride) O[q] = T(-1);
            // the rows of the intersection as one flat range, x-adjacent threads on
            // x-adjacent words: element q is row q / wd, column q % wd
            const int wd = I.xmax - I.xmin, n = (I.ymax - I.ymin) * wd, inx = ib.nx();
            const float rwd = 1.f / (float)wd;
            const T* src = a.in.grain_ptr(g) + ib.at(I.ymin, I.xmin, k);
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(In + (I.ymin - ob.y0) * P + (I.xmin - ob.x0));
            for (int q = line; q < n; q += lstride) {
                const int r = div_small<S>(q, wd, rwd), c = q - r * wd;
                cp_async_to(dst + (uint32_t)(sizeof(T) * (r * P + c)), src + (r * inx + c));
            }
        }
        cp_async_wait_all();
        __syncthreads();
        T* O0 = O - (long long)ob.y0 * P - ob.x0;  // O0[i * P + j] = OUT(i, j), IN(i, j) PL further
        if (sweeps)
            for (int i = I.ymin + line; i < ob.y1; i += lstride)  // x forward, box.cpp:2367-2401
                sweep_forward(O0 + (long long)i * P, 1, PL, I.xmin, ob.x1, I.xmax, i < I.ymax, h);
        __syncthreads();
        if (sweeps)
            for (int i = I.ymin + line; i < ob.y1; i += lstride)  // x backward, box.cpp:2403-2435
                sweep_backward_prop(O0 + (long long)i * P, 1, PL, I.xmax - 1, ob.x0, I.xmin, i < I.ymax, h);
        __syncthreads();
        if (sweeps)
            for (int j = I.xmin + line; j < ob.x1; j += lstride)  // y forward, box.cpp:2437-2472
                sweep_forward(O0 + j, P, PL, I.ymin, ob.y1, I.ymax, j < I.xmax, h);
        __syncthreads();
        if (sweeps) {
            for (int j = I.xmin + line; j < ob.x1; j += lstride)  // y backward, box.cpp:2474-2496
                sweep_backward_prop(O0 + j, P, PL, I.ymax - 1, ob.y0, I.ymin, j < I.xmax, h);
        }
        __syncthreads();
        if (sweeps) {
            const float rnx = 1.f / (float)nx;
            for (int q = line; q < nx * ny; q += lstride) {
                const int r = div_small<S>(q, nx, rnx);
                outg[q] = O[r * P + (q - r * nx)];
            }
        }
        __syncthreads();
    }
}

// Kernel z: a CTA per (grain, U consecutive output y-rows); unit u owns row
// ob.y0 + U * tile + u, whose [z][x] plane sits in shared memory, and its threads run
// the z recurrences of one column each (x-adjacent threads touch adjacent words).
template <typename T, int S, int U>
__global__ void __launch_bounds__(kMaxThreads) redist_z_kernel(RedistArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int u = S ? tid / S : 0;
    const int line = S ? tid - u * S : tid;
    const int lstride = S ? S : blockDim.x;
    const T h = (T)a.geo.h;
    const T delta = (T)a.geo.delta;
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        const Box ob = a.out.grain_box(g);
        const Box ib = a.in.grain_box(g);
        const int i = ob.y0 + w.local * U + u;
        const bool unit = u < U && i < ob.y1;
        const Intersect I(ib, ob);
        const int nx = ob.nx(), nz = ob.nz();
        const int PZ = S ? S : nx;                // z stride in shared memory
        const int PLZ = S ? S * S : nx * nz;      // the input plane follows the output plane
        const long long zs = (long long)nx * ob.ny();  // z stride of the output box
        T* Z = reinterpret_cast<T*>(smem_raw) + (S ? u * z_unit_stride(S) : 0);
        T* Zin = Z + PLZ;
        T* outr = a.out.grain_ptr(g) + (long long)(i - ob.y0) * nx;  // OUT(i, x0, z0)
        const float rnx = 1.f / (float)nx;
        if (unit) {
            // the row's [z][x] plane and its input on the intersection, each as one flat
            // range (element q: z q / width, x q % width), x-adjacent threads on x-adjacent words
            const uint32_t zd = (uint32_t)__cvta_generic_to_shared(Z);
            for (int q = line; q < nz * nx; q += lstride) {
                const int r = div_small<S>(q, nx, rnx), c = q - r * nx;
                cp_async_to(zd + (uint32_t)(sizeof(T) * (r * PZ + c)), outr + (r * zs + c));
            }
            if (i >= I.ymin && i < I.ymax) {
                const int wd = I.xmax - I.xmin, n = (I.zmax - I.zmin) * wd;
                const float rwd = 1.f / (float)wd;
                const long long izs = (long long)ib.nx() * ib.ny();
                const T* src = a.in.grain_ptr(g) + ib.at(i, I.xmin, I.zmin);
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(Zin + (I.zmin - ob.z0) * PZ + (I.xmin - ob.x0));
                for (int q = line; q < n; q += lstride) {
                    const int r = div_small<S>(q, wd, rwd), c = q - r * wd;
                    cp_async_to(dst + (uint32_t)(sizeof(T) * (r * PZ + c)), src + (r * izs + c));
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
        if (unit && i >= I.ymin) {
            T* Z0 = Z - (long long)ob.z0 * PZ - ob.x0;  // Z0[k * PZ + j] = OUT(i, j, k), IN PLZ further
            for (int j = I.xmin + line; j < ob.x1; j += lstride) {
                const bool inside = i < I.ymax && j < I.xmax;
                // z forward, box.cpp:2501-2538
                sweep_forward(Z0 + j, PZ, PLZ, I.zmin, ob.z1, I.zmax, inside, h);
                // z backward, box.cpp:2539-2576
                sweep_backward_in(Z0 + j, PZ, PLZ, I.zmax - 1, ob.z0, I.zmin, inside, h);
            }
        }
        __syncthreads();
        // clampValues(-delta, delta), dimensionalBufferReal.h:44-57
        if (unit)
            for (int q = line; q < nz * nx; q += lstride) {
                const int r = div_small<S>(q, nx, rnx), c = q - r * nx;
                T v = Z[r * PZ + c];
                if (v < -delta) v = -delta;
                else if (v > delta) v = delta;
                outr[r * zs + c] = v;
            }
        __syncthreads();
    }
}

}  // namespace

// Shared memory of one unit: output and input slices with odd pitch, or [z][x] planes.
size_t redist_smem_bytes(int nmax, bool fp64) {
    const size_t e = fp64 ? 8 : 4;
    const size_t xy = (size_t)nmax * (nmax | 1);
    const size_t z = (size_t)nmax * nmax;
    return 2 * (xy > z ? xy : z) * e;
}

namespace {
// Per class c, the exclusive scan over grains of ceil(n / redist_units(c)) (n the output
// box side) for the grains of toff_all (n tiles each) whose n is in class c; one CTA over
// chunks of 1024 consecutive grains, each grain's box read once.
__global__ void __launch_bounds__(1024) redist_class_kernel(int G, const int* toff_all, const int* box,
                                                            int* class_toff) {
    __shared__ int warp_tot[32][kRedistClasses];
    __shared__ int carry[kRedistClasses];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int stride = G + 2;
    const bool none = toff_all[G + 1] == 0;  // the plan overflowed: no tiles at all
    if (threadIdx.x < kRedistClasses) carry[threadIdx.x] = 0;
    __syncthreads();
    for (int g0 = 0; g0 <= G; g0 += blockDim.x) {
        const int g = g0 + threadIdx.x;
        int cls = -1, tiles = 0;
        if (!none && g >= 1 && g <= G && toff_all[g + 1] - toff_all[g] > 0) {
            const Box b = load_box(box + 6 * g);  // cubes; the largest side bounds every stride
            const int n = max(b.nx(), max(b.ny(), b.nz()));
#pragma unroll
            for (int c = 0; c < kRedistClasses; c++) {
                const int lo = c == 0 ? 0 : redist_side(c - 1);
                if (n > lo && n <= redist_side(c)) {
                    cls = c;
                    tiles = (n + redist_units(c) - 1) / redist_units(c);
                }
            }
        }
        int incl[kRedistClasses];
#pragma unroll
        for (int c = 0; c < kRedistClasses; c++) {
            incl[c] = cls == c ? tiles : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl[c], o);
                if (lane >= o) incl[c] += u;
            }
            if (lane == 31) warp_tot[warp][c] = incl[c];
        }
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int c = 0; c < kRedistClasses; c++) {
                int wi = warp_tot[lane][c];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, wi, o);
                    if (lane >= o) wi += u;
                }
                warp_tot[lane][c] = wi;  // inclusive over warps
            }
        }
        __syncthreads();
        if (g <= G) {
#pragma unroll
            for (int c = 0; c < kRedistClasses; c++)
                class_toff[(long long)c * stride + g] =
                    carry[c] + (warp > 0 ? warp_tot[warp - 1][c] : 0) + incl[c] - (cls == c ? tiles : 0);
        }
        __syncthreads();
        if (threadIdx.x < kRedistClasses) carry[threadIdx.x] += warp_tot[31][threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x < kRedistClasses) class_toff[(long long)threadIdx.x * stride + G + 1] = carry[threadIdx.x];
}

// CTAs of kernel k with `threads` threads and `smem` bytes that fit the device at once.
template <typename K>
int resident_ctas(K kernel, int threads, size_t smem) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    return sms * (per_sm > 0 ? per_sm : 1);
}
}  // namespace

void launch_redist_classes(int G, const int* toff_all, const int* box, int* class_toff, cudaStream_t s) {
    redist_class_kernel<<<1, 1024, 0, s>>>(G, toff_all, box, class_toff);
}

namespace {
template <typename T, int S, int U>
void launch_class(const RedistArgs<T>& a, int n, cudaStream_t s) {
    static_assert(S % 8 == 0 && U * S <= kMaxThreads, "fixed-pitch classes: sides a multiple of 8");
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(redist_xy_kernel<T, S, U>);
        allow_max_dynamic_smem(redist_z_kernel<T, S, U>);
    });
    const int threads = S ? class_threads(S, U) : std::min((n + 31) / 32 * 32, kMaxThreads);
    const size_t e = sizeof(T);
    const size_t sxy = S ? (size_t)U * xy_unit_stride(S) * e : redist_smem_bytes(n, e == 8);
    const size_t sz = S ? (size_t)U * z_unit_stride(S) * e : redist_smem_bytes(n, e == 8);
    redist_xy_kernel<T, S, U><<<resident_ctas(redist_xy_kernel<T, S, U>, threads, sxy), threads, sxy, s>>>(a);
    redist_z_kernel<T, S, U><<<resident_ctas(redist_z_kernel<T, S, U>, threads, sz), threads, sz, s>>>(a);
}
}  // namespace

template <typename T>
void launch_redistance(const RedistArgs<T>& a, int grid, int side, const int* class_toff, cudaStream_t s) {
    if (!class_toff) {  // one unit per CTA of runtime pitch, over a.toff (n tiles a grain)
        static PerDevice configured;
        configured.once([] {
            allow_max_dynamic_smem(redist_xy_kernel<T, 0, 1>);
            allow_max_dynamic_smem(redist_z_kernel<T, 0, 1>);
        });
        const size_t smem = redist_smem_bytes(side, sizeof(T) == 8);
        int threads = (side + 31) / 32 * 32;
        threads = threads > kMaxThreads ? kMaxThreads : threads;
        redist_xy_kernel<T, 0, 1><<<grid * 2, threads, smem, s>>>(a);
        redist_z_kernel<T, 0, 1><<<grid * 2, threads, smem, s>>>(a);
        return;
    }
    // one pair of launches per size class up to the largest side, each filling the
    // device with its own CTAs
    for (int c = 0; c < kRedistClasses; c++) {
        const int lo = c == 0 ? 0 : redist_side(c - 1);
        if (lo >= side) break;
        RedistArgs<T> ac = a;
        ac.toff = class_toff + (long long)c * (a.G + 2);
        switch (c) {
            case 0: launch_class<T, redist_side(0), redist_units(0)>(ac, 0, s); break;
            case 1: launch_class<T, redist_side(1), redist_units(1)>(ac, 0, s); break;
            case 2: launch_class<T, redist_side(2), redist_units(2)>(ac, 0, s); break;
            case 3: launch_class<T, redist_side(3), redist_units(3)>(ac, 0, s); break;
            case 4: launch_class<T, redist_side(4), redist_units(4)>(ac, 0, s); break;
            case 5: launch_class<T, redist_side(5), redist_units(5)>(ac, 0, s); break;
            default: launch_class<T, 0, 1>(ac, side, s); break;
        }
    }
}

template void launch_redistance<double>(const RedistArgs<double>&, int, int, const int*, cudaStream_t);
template void launch_redistance<float>(const RedistArgs<float>&, int, int, const int*, cudaStream_t);

}  // namespace gg

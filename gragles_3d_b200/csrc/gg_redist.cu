// gg_redist.cu -- directional-sweep redistancing of every grain.
//
// Stands in for LSbox::executeRedistancing (box.cpp:2322-2586).  The reference
// clears the new (resized) output box to -1, then for every z-slice of the in/out
// intersection except the last runs four sweeps (x forward, x backward, y forward,
// y backward), then sweeps z forward and backward over all columns, and clamps to
// +-delta.  Every sweep is a recurrence along one line and the lines of a sweep are
// independent, so a small CTA (one thread per line: 32 or 64 threads for the usual
// sides) owns one unit of work at a time:
//   kernel xy: a CTA per (grain, output z-slice); the slice of the output sits in
//              shared memory, threads run rows for the x sweeps and columns for the
//              y sweeps;
//   kernel z:  a CTA per (grain, output y-row); the [z][x] plane of the row sits in
//              shared memory and threads run the z recurrences of one column each
//              (x-adjacent threads touch adjacent words).
// One unit's buffers are small (two n x n planes), so many CTAs share an SM.
// The unit's input values on the in/out intersection are staged next to it with
// coalesced loads (a recurrence that read HBM step by step would wait on every load).
// Along a line the value that the next step updates is carried in a register, so a
// step costs its arithmetic and shared-memory loads that do not depend on the chain.  The
// arithmetic is the reference's, statement by statement (no contraction), and the
// lines of a sweep run in the reference's order, so the FP64 result is bit-identical.
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

// x + isgn(s) * h of the reference, without the int -> T conversion and product:
// isgn(s) * h is exactly h, -h or +0.
template <typename T>
__device__ __forceinline__ T add_sgn(T x, T s, T h) {
    return x + (s > T(0) ? h : (s < T(0) ? -h : T(0)));  // x - h is x + (-h) in IEEE arithmetic
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
    const T candidate = add_sgn(out_here, b, h);
    if (fabs(candidate) < fabs(out_next)) out_next = candidate;
}
template <typename T>
__device__ __forceinline__ void step_prop(T sgn_src, T out_here, T& out_next, T h) {
    const T candidate = add_sgn(out_here, sgn_src, h);
    if (fabs(candidate) < fabs(out_next)) out_next = candidate;
}

// Forward sweep over positions p0 .. p_end - 1 of a line: o[p * so] is the output at
// p, in[p * si] the input, valid for p in [p0, p_in_end) when `inside`.  The
// reference's x/y/z forward loops (box.cpp:2367-2401, 2437-2472, 2501-2538) take
// step_in while p < p_in_end - 1 (and inside), else step_prop: a prefix, so the loop
// is split in two.
template <typename T>
__device__ __forceinline__ void sweep_forward(T* o, int so, const T* in, int si, int p0, int p_end, int p_in_end,
                                              bool inside, T h) {
    if (p0 >= p_end - 1) return;
    T* op = o + p0 * so;
    T cur = *op;
    int p = p0;
    const int pin = inside ? min(p_in_end - 1, p_end - 1) : p0;
    if (p < pin) {
        const T* ip = in + p0 * si;
        T icur = *ip;
#pragma unroll 4
        for (; p < pin; p++, op += so, ip += si) {
            T nxt = op[so];
            const T inx = ip[si];
            step_in(icur, inx, cur, nxt, h);
            *op = cur;
            cur = nxt;
            icur = inx;
        }
    }
#pragma unroll 4
    for (; p < p_end - 1; p++, op += so) {
        T nxt = op[so];
        step_prop(nxt, cur, nxt, h);
        *op = cur;
        cur = nxt;
    }
    *op = cur;
}

// Backward propagation from p_start down to p_lo + 1 (box.cpp:2403-2435, 2474-2496):
// step_prop with the sign of in(p - 1) while p > p_in_lo (and inside), else of the
// output itself.  out_here is never modified.
template <typename T>
__device__ __forceinline__ void sweep_backward_prop(T* o, int so, const T* in, int si, int p_start, int p_lo,
                                                    int p_in_lo, bool inside, T h) {
    if (p_start <= p_lo) return;
    T* op = o + p_start * so;
    T cur = *op;
    int p = p_start;
    if (inside) {
        const int plim = max(p_in_lo, p_lo);
        const T* ip = in + (p_start - 1) * si;
#pragma unroll 4
        for (; p > plim; p--, op -= so, ip -= si) {
            T nxt = op[-so];
            step_prop(*ip, cur, nxt, h);
            op[-so] = nxt;
            cur = nxt;
        }
    }
#pragma unroll 4
    for (; p > p_lo; p--, op -= so) {
        T nxt = op[-so];
        step_prop(nxt, cur, nxt, h);
        op[-so] = nxt;
        cur = nxt;
    }
}

// Backward sweep with interpolation (the z backward loop, box.cpp:2539-2576): step_in
// while p > p_in_lo (and inside), else step_prop; step_in may change o(p) as well.
template <typename T>
__device__ __forceinline__ void sweep_backward_in(T* o, int so, const T* in, int si, int p_start, int p_lo,
                                                  int p_in_lo, bool inside, T h) {
    if (p_start <= p_lo) return;
    T* op = o + p_start * so;
    T cur = *op;
    int p = p_start;
    const int plim = max(p_in_lo, p_lo);
    if (inside && p > plim) {
        const T* ip = in + p_start * si;
        T icur = *ip;
#pragma unroll 4
        for (; p > plim; p--, op -= so, ip -= si) {
            T nxt = op[-so];
            const T inx = ip[-si];
            step_in(icur, inx, cur, nxt, h);
            *op = cur;
            cur = nxt;
            icur = inx;
        }
    }
#pragma unroll 4
    for (; p > p_lo; p--, op -= so) {
        T nxt = op[-so];
        step_prop(nxt, cur, nxt, h);
        *op = cur;
        cur = nxt;
    }
    *op = cur;
}

template <typename T>
__global__ void __launch_bounds__(kMaxThreads) redist_xy_kernel(RedistArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x, nt = blockDim.x;
    T* O = reinterpret_cast<T*>(smem_raw);  // out slice, [y][x] with pitch P, then in values
    const T h = (T)a.geo.h;
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        const Box ob = a.out.grain_box(g);
        const Box ib = a.in.grain_box(g);
        const int k = ob.z0 + w.local;
        const Intersect I(ib, ob);
        const int nx = ob.nx(), ny = ob.ny();
        T* outg = a.out.grain_ptr(g) + (long long)(k - ob.z0) * nx * ny;
        if (!(k >= I.zmin && k < I.zmax - 1)) {  // no xy sweep reaches this slice
            for (int q = tid; q < nx * ny; q += nt) outg[q] = T(-1);
            continue;  // uniform across the CTA
        }
        const int P = nx | 1;
        T* In = O + ny * P;  // IN(i, j) at the same position as OUT(i, j), on the intersection
        for (int q = tid; q < ny * P; q += nt) O[q] = T(-1);
        {
            // rows of the intersection, x-adjacent threads on x-adjacent words
            const int w = I.xmax - I.xmin;
            const T* src = a.in.grain_ptr(g) + ib.at(I.ymin, I.xmin, k);
            T* dst = In + (I.ymin - ob.y0) * P + (I.xmin - ob.x0);
            for (int yy = 0; yy < I.ymax - I.ymin; yy++, src += ib.nx(), dst += P)
                for (int xx = tid; xx < w; xx += nt) cp_async_elem(dst + xx, src + xx);
        }
        cp_async_wait_all();
        __syncthreads();
        T* O0 = O - (long long)ob.y0 * P - ob.x0;  // O0[i * P + j] = OUT(i, j)
        const T* in_k = In - (long long)ob.y0 * P - ob.x0;  // in_k[i * P + j] = IN(i, j)
        const int inx = P;
        for (int i = I.ymin + tid; i < ob.y1; i += nt)  // x forward, box.cpp:2367-2401
            sweep_forward(O0 + (long long)i * P, 1, in_k + (long long)i * inx, 1, I.xmin, ob.x1, I.xmax, i < I.ymax, h);
        __syncthreads();
        for (int i = I.ymin + tid; i < ob.y1; i += nt)  // x backward, box.cpp:2403-2435
            sweep_backward_prop(O0 + (long long)i * P, 1, in_k + (long long)i * inx, 1, I.xmax - 1, ob.x0, I.xmin,
                                i < I.ymax, h);
        __syncthreads();
        for (int j = I.xmin + tid; j < ob.x1; j += nt)  // y forward, box.cpp:2437-2472
            sweep_forward(O0 + j, P, in_k + j, inx, I.ymin, ob.y1, I.ymax, j < I.xmax, h);
        __syncthreads();
        for (int j = I.xmin + tid; j < ob.x1; j += nt)  // y backward, box.cpp:2474-2496
            sweep_backward_prop(O0 + j, P, in_k + j, inx, I.ymax - 1, ob.y0, I.ymin, j < I.xmax, h);
        __syncthreads();
        for (int yy = 0; yy < ny; yy++)
            for (int xx = tid; xx < nx; xx += nt) outg[yy * nx + xx] = O[yy * P + xx];
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(kMaxThreads) redist_z_kernel(RedistArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x, nt = blockDim.x;
    T* Z = reinterpret_cast<T*>(smem_raw);  // [k][x] of this row, then the in values
    const T h = (T)a.geo.h;
    const T delta = (T)a.geo.delta;
    for (TileWalk w(a.toff, a.G, blockIdx.x, gridDim.x); w.valid(); w.next()) {
        const int g = w.g;
        const Box ob = a.out.grain_box(g);
        const Box ib = a.in.grain_box(g);
        const int i = ob.y0 + w.local;
        const Intersect I(ib, ob);
        const int nx = ob.nx(), nz = ob.nz();
        const long long zs = (long long)nx * ob.ny();  // z stride of the output box
        T* outr = a.out.grain_ptr(g) + (long long)(i - ob.y0) * nx;  // OUT(i, x0, z0)
        T* Zin = Z + nx * nz;  // IN(i, j, k) at the position of OUT(i, j, k), on the intersection
        for (int kk = 0; kk < nz; kk++)
            for (int xx = tid; xx < nx; xx += nt) cp_async_elem(Z + kk * nx + xx, outr + kk * zs + xx);
        if (i >= I.ymin && i < I.ymax) {
            const int w = I.xmax - I.xmin;
            const long long izs = (long long)ib.nx() * ib.ny();
            const T* src = a.in.grain_ptr(g) + ib.at(i, I.xmin, I.zmin);
            T* dst = Zin + (I.zmin - ob.z0) * nx + (I.xmin - ob.x0);
            for (int k = I.zmin; k < I.zmax; k++, src += izs, dst += nx)
                for (int xx = tid; xx < w; xx += nt) cp_async_elem(dst + xx, src + xx);
        }
        cp_async_wait_all();
        __syncthreads();
        if (i >= I.ymin) {
            const int izs = nx;
            T* Z0 = Z - (long long)ob.z0 * nx - ob.x0;  // Z0[k * nx + j] = OUT(i, j, k)
            const T* in_i = Zin - (long long)ob.z0 * nx - ob.x0;  // in_i[k * nx + j] = IN(i, j, k)
            for (int j = I.xmin + tid; j < ob.x1; j += nt) {
                const bool inside = i < I.ymax && j < I.xmax;
                // z forward, box.cpp:2501-2538
                sweep_forward(Z0 + j, nx, in_i + j, izs, I.zmin, ob.z1, I.zmax, inside, h);
                // z backward, box.cpp:2539-2576
                sweep_backward_in(Z0 + j, nx, in_i + j, izs, I.zmax - 1, ob.z0, I.zmin, inside, h);
            }
        }
        __syncthreads();
        // clampValues(-delta, delta), dimensionalBufferReal.h:44-57
        for (int kk = 0; kk < nz; kk++)
            for (int xx = tid; xx < nx; xx += nt) {
                T v = Z[kk * nx + xx];
                if (v < -delta) v = -delta;
                else if (v > delta) v = delta;
                outr[kk * zs + xx] = v;
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
// Per class c, the exclusive scan over grains of n (the output box side) for the grains
// of toff_all (n tiles each) whose n is in class c; one CTA, as plan_kernel.
__global__ void __launch_bounds__(1024) redist_class_kernel(int G, const int* toff_all, const int* box,
                                                            int* class_toff) {
    __shared__ int warp_tot[32][kRedistClasses];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int stride = G + 2;
    const bool none = toff_all[G + 1] == 0;  // the plan overflowed: no tiles at all
    const int per = (G + blockDim.x) / blockDim.x;  // grains 0..G
    const int g0 = threadIdx.x * per, g1 = min(G + 1, g0 + per);
    auto count = [&](int g, int c) {
        if (none || g < 1 || g > G || toff_all[g + 1] - toff_all[g] <= 0) return 0;
        const int n = load_box(box + 6 * g).nx();
        const int lo = c == 0 ? 0 : redist_side(c - 1);
        return (n > lo && n <= redist_side(c)) ? n : 0;
    };
    int mine[kRedistClasses], incl[kRedistClasses];
#pragma unroll
    for (int c = 0; c < kRedistClasses; c++) {
        mine[c] = 0;
        for (int g = g0; g < g1; g++) mine[c] += count(g, c);
        incl[c] = mine[c];
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
            const int w = warp_tot[lane][c];
            int wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += u;
            }
            warp_tot[lane][c] = wi;  // inclusive over warps
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kRedistClasses; c++) {
        int run = (warp > 0 ? warp_tot[warp - 1][c] : 0) + incl[c] - mine[c];
        int* t = class_toff + (long long)c * stride;
        for (int g = g0; g < g1; g++) {
            t[g] = run;
            run += count(g, c);
        }
        if (threadIdx.x == blockDim.x - 1) t[G + 1] = warp_tot[31][c];
    }
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

template <typename T>
void launch_redistance(const RedistArgs<T>& a, int grid, int side, const int* class_toff, cudaStream_t s) {
    static PerDevice configured;
    configured.once([] {
        allow_max_dynamic_smem(redist_xy_kernel<T>);
        allow_max_dynamic_smem(redist_z_kernel<T>);
    });
    if (!class_toff) {
        const size_t smem = redist_smem_bytes(side, sizeof(T) == 8);
        int threads = (side + 31) / 32 * 32;
        threads = threads > kMaxThreads ? kMaxThreads : threads;
        redist_xy_kernel<T><<<grid * 2, threads, smem, s>>>(a);
        redist_z_kernel<T><<<grid * 2, threads, smem, s>>>(a);
        return;
    }
    // one pair of launches per size class up to the largest side, each sized for its
    // class's largest side and filling the device with its own CTAs
    for (int c = 0; c < kRedistClasses; c++) {
        const int lo = c == 0 ? 0 : redist_side(c - 1);
        if (lo >= side) break;
        const int n = std::min(redist_side(c), side);
        const size_t smem = redist_smem_bytes(n, sizeof(T) == 8);
        const int threads = std::min((n + 31) / 32 * 32, kMaxThreads);
        RedistArgs<T> ac = a;
        ac.toff = class_toff + (long long)c * (a.G + 2);
        redist_xy_kernel<T><<<resident_ctas(redist_xy_kernel<T>, threads, smem), threads, smem, s>>>(ac);
        redist_z_kernel<T><<<resident_ctas(redist_z_kernel<T>, threads, smem), threads, smem, s>>>(ac);
    }
}

template void launch_redistance<double>(const RedistArgs<double>&, int, int, const int*, cudaStream_t);
template void launch_redistance<float>(const RedistArgs<float>&, int, int, const int*, cudaStream_t);

}  // namespace gg

// cg_tma.cuh — the two CG passes of the pressure and heat solves as
// plane-marching kernels whose tiles arrive by TMA (cp.async.bulk.tensor) into
// a shared-memory ring, included by k_cg.cu (uses its Red, the operators and
// the scalar slots).
//
// One CTA owns a tile of TJ x TK cells in the (j, k) plane and marches along i
// over a chunk of planes. For every plane q the ring holds, as TMA boxes of
// the plane:
//   MODE 0 (direction): r and p_old with a one-cell halo in j and k
//                       (the box starts 4 floats before the tile so that its
//                       x coordinate stays 16-byte aligned), and the
//                       neighbour bytes of the tile;
//   MODE 1 (update):    p with the same halo, x, r and the neighbour bytes.
// The CTA turns the box into the plane's stencil operand once, in a window of
// four planes (MODE 0: p = r + beta p_old, the direction vector, computed once
// per cell instead of once per stencil tap; MODE 1: p copied), and applies the
// 7-point row of plane q-1 from the window planes q-2, q-1, q. The operands
// and their arithmetic order are those of k_cg_v4 (PressOp/HeatOp::apply), so
// the vectors it writes are the same bit for bit; only the FP64 dot product
// adds its terms in another order. Loads run NS-1 planes ahead of the stencil.
//
// Requirements checked by the host: FP32 vectors, NZ a multiple of 16 (the
// neighbour-byte box's row stride), every vector 16-byte aligned. The tensor
// maps cover this GPU's own arrays only and no load uses cluster multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

namespace {

#ifndef TT_NS0
#define TT_NS0 3
#endif
#ifndef TT_CTAS0
#define TT_CTAS0 4
#endif
#ifndef TT_NS1
#define TT_NS1 2
#endif
#ifndef TT_CTAS1
#define TT_CTAS1 4
#endif
constexpr int TT_K = 64;              // tile cells along k (16 float4 groups)
constexpr int TT_J = 16;              // tile rows along j
constexpr int TT_THREADS = TT_J * (TT_K / 4);   // one thread per float4 group: 256
constexpr int TT_HK = TT_K + 8;       // halo box along k: k0-4 .. k0+TK+3 (72 floats)
constexpr int TT_HJ = TT_J + 2;       // halo box along j: j0-1 .. j0+TJ (18 rows)
// ring stages and resident CTAs per SM. Both passes are bound by issue
// latency at the occupancy shared memory allows, so more resident warps beat
// deeper prefetch: the direction pass keeps two planes in flight with 4 CTAs
// of 54 KB per SM (faster than three planes with 3 CTAs of 65 KB, and than
// one plane with 5 CTAs of 43 KB); the update pass, whose stages are larger,
// keeps one plane in flight with 4 CTAs of 49 KB (faster than two planes with
// 3 CTAs of 63 KB)
template <int MODE> __host__ __device__ constexpr int tt_ns() { return MODE == 0 ? TT_NS0 : TT_NS1; }
template <int MODE> __host__ __device__ constexpr int tt_ctas() { return MODE == 0 ? TT_CTAS0 : TT_CTAS1; }
constexpr int TT_NW = 4;              // window planes
constexpr uint32_t TT_HALO_BYTES = TT_HK * TT_HJ * 4;        // 5184
constexpr uint32_t TT_HALO_PAD = (TT_HALO_BYTES + 127) / 128 * 128;   // 5248
constexpr uint32_t TT_TILE_BYTES = TT_K * TT_J * 4;          // 4096
constexpr uint32_t TT_NB_BYTES = TT_K * TT_J;                // 1024
// stage layout (byte offsets, each 128-byte aligned)
//   MODE 0: [halo r][halo p_old][nb]        MODE 1: [halo p][x][r][nb]
constexpr uint32_t TT_STAGE0 = 2 * TT_HALO_PAD + TT_NB_BYTES;
constexpr uint32_t TT_STAGE1 = TT_HALO_PAD + 2 * TT_TILE_BYTES + TT_NB_BYTES;
constexpr uint32_t TT_WIN_BYTES = TT_NW * TT_HALO_BYTES;
template <int MODE> __host__ __device__ constexpr uint32_t tt_stage_bytes() { return MODE == 0 ? TT_STAGE0 : TT_STAGE1; }
template <int MODE> __host__ __device__ constexpr uint32_t tt_smem_bytes() {
    return tt_ns<MODE>() * tt_stage_bytes<MODE>() + TT_WIN_BYTES + tt_ns<MODE>() * 8 + 128;   // + barriers, alignment
}
// a wait on a TMA barrier gives up after this long (ns) and reports MP_ERR_TIMEOUT
constexpr unsigned long long TT_WAIT_NS = 1000000000ull;

__device__ __forceinline__ uint32_t tt_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long tt_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void tt_bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tt_smem(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void tt_bar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tt_smem(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool tt_bar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(tt_smem(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// waits for the barrier's phase `parity` to complete; false after TT_WAIT_NS
// (the clock is read once every 256 polls: a poll already suspends the warp
// for a while, and reading the clock on every poll costs issue slots)
__device__ __forceinline__ bool tt_bar_wait(uint64_t* bar, uint32_t parity) {
    unsigned long long t0 = 0;
    for (uint32_t i = 1;; ++i) {
        if (tt_bar_test(bar, parity)) return true;
        if ((i & 255u) == 0) {
            const unsigned long long t = tt_clock_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > TT_WAIT_NS) return false;
        }
    }
}
__device__ __forceinline__ void tt_load(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(tt_smem(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(tt_smem(bar))
        : "memory");
}

// the FP64 sum of one value per thread over all blocks of a 3-D grid of
// TT_THREADS-thread blocks: block partials, then the last block to finish adds
// them in a fixed order (deterministic); true in thread 0 of that block
__device__ __forceinline__ bool tt_finish(const Red& R, double mine, double* tot) {
    __shared__ double ws[TT_THREADS / 32];
    __shared__ bool last;
    const int tid = threadIdx.x;
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    double v = mine;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) ws[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int w = 0; w < TT_THREADS / 32; w++) s += ws[w];
        R.part[bid] = s;
        __threadfence();
        unsigned int t = atomicAdd(R.count, 1u);
        last = (t == nblk - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double a = 0;
    for (unsigned int b = tid; b < nblk; b += TT_THREADS) a += __ldcg(R.part + b);
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    __syncthreads();
    if ((tid & 31) == 0) ws[tid >> 5] = a;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int w = 0; w < TT_THREADS / 32; w++) s += ws[w];
        *tot = s; *R.count = 0;
    }
    return tid == 0;
}

// launch with programmatic stream serialization (the kernel waits with
// griddepcontrol.wait before it reads the previous launch's results)
template <typename... KArgs, typename... Args>
inline cudaError_t tt_launch(void (*kern)(KArgs...), dim3 grid, int block, size_t smem, cudaStream_t s,
                             Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid; cfg.blockDim = dim3(block); cfg.dynamicSmemBytes = smem; cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr; cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

struct TtMaps {
    CUtensorMap a;     // MODE 0: r (halo box)       MODE 1: p (halo box)
    CUtensorMap b;     // MODE 0: p_old (halo box)   MODE 1: x (tile box)
    CUtensorMap c;     //                            MODE 1: r (tile box)
    CUtensorMap nb;    // neighbour bytes (tile box)
};

// MODE 0: p_new = r + beta p_old (first: r); z = A p_new; p_new . z
// MODE 1: z = A p; x += alpha p, r -= alpha z; r . r; stop test
template <class Op, int MODE>
__global__ void __launch_bounds__(TT_THREADS, tt_ctas<MODE>())
    k_cg_tma(Op op, const __grid_constant__ TtMaps maps, float* __restrict__ pout, float* __restrict__ x,
             float* __restrict__ r, Red Rd, int chunk, int first, int it, int maxiter, int skip_dot) {
    // launched with programmatic stream serialization: the previous launch on
    // the stream (the other pass) may still be finishing; its results (the
    // vectors, the scalars, the stop flag) are visible after this wait
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (Rd.flag[F_DONE] != DONE_RUN) return;
    extern __shared__ unsigned char tt_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tt_raw) + 127) & ~uintptr_t(127));
    constexpr uint32_t SB = tt_stage_bytes<MODE>();
    constexpr int TT_NS = tt_ns<MODE>();
    float* win = reinterpret_cast<float*>(sm + TT_NS * SB);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + TT_NS * SB + TT_WIN_BYTES);
    __shared__ int tt_fail;

    const Grid& g = op.g;
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tg = tid & 15;
    const int k0 = blockIdx.x * TT_K, j0 = blockIdx.y * TT_J;
    const int i0 = blockIdx.z * chunk, i1 = min(i0 + chunk, g.NX);
    const int kk = k0 + 4 * tg, jj = j0 + ty;
    const bool inb = kk < g.NZ && jj < g.NY;
    const float bf = (MODE == 0 && !first) ? (float)Rd.scal[S_BETA] : 0.0f;
    const float af = MODE == 1 ? (float)Rd.scal[S_ALPHA] : 0.0f;
    const bool load_b = MODE == 1 || !first;
    const uint32_t tx = MODE == 0 ? (load_b ? 2 * TT_HALO_BYTES : TT_HALO_BYTES) + TT_NB_BYTES
                                  : TT_HALO_BYTES + 2 * TT_TILE_BYTES + TT_NB_BYTES;
    // planes q = i0-1 .. i1 pass through the ring; plane q uses stage (q - i0 + 1) % NS
    const int q0 = i0 - 1, nplanes = i1 - i0 + 2;

    auto issue = [&](int t) {   // plane q0 + t into stage t % NS (thread 0)
        unsigned char* st = sm + (t % TT_NS) * SB;
        uint64_t* b = bar + (t % TT_NS);
        const int q = q0 + t;
        tt_bar_expect(b, tx);
        if (MODE == 0) {
            tt_load(st, &maps.a, b, k0 - 4, j0 - 1, q);
            if (load_b) tt_load(st + TT_HALO_PAD, &maps.b, b, k0 - 4, j0 - 1, q);
            tt_load(st + 2 * TT_HALO_PAD, &maps.nb, b, k0, j0, q);
        } else {
            tt_load(st, &maps.a, b, k0 - 4, j0 - 1, q);
            tt_load(st + TT_HALO_PAD, &maps.b, b, k0, j0, q);
            tt_load(st + TT_HALO_PAD + TT_TILE_BYTES, &maps.c, b, k0, j0, q);
            tt_load(st + TT_HALO_PAD + 2 * TT_TILE_BYTES, &maps.nb, b, k0, j0, q);
        }
    };
    if (tid == 0) {
        tt_fail = 0;
        for (int s = 0; s < TT_NS; s++) tt_bar_init(bar + s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int t = 0; t < TT_NS && t < nplanes; t++) issue(t);
    }
    __syncthreads();

    double acc = 0;
    // this thread's group of the previous plane: neighbour bytes, x, r
    uint32_t m_prev = 0;
    float4 x_prev = make_float4(0, 0, 0, 0), r_prev = x_prev;
    int t = 0;
    for (; t < nplanes; t++) {
        const int q = q0 + t;
        unsigned char* st = sm + (t % TT_NS) * SB;
        // every thread waits for the stage itself; a wait that runs out is
        // seen by all threads after the barrier below
        const bool ok = tt_bar_wait(bar + (t % TT_NS), (uint32_t)((t / TT_NS) & 1));
        if (!ok) atomicExch(&tt_fail, 1);
        // the window plane of q from the stage
        float4* w = reinterpret_cast<float4*>(win + (t % TT_NW) * (TT_HK * TT_HJ));
        const float4* sa = reinterpret_cast<const float4*>(st);
        const float4* sb = reinterpret_cast<const float4*>(st + TT_HALO_PAD);
        for (int e = tid; ok && e < TT_HK * TT_HJ / 4; e += TT_THREADS) {
            float4 a = sa[e];
            if (MODE == 0 && !first) {
                const float4 b = sb[e];
                a = make_float4(a.x + bf * b.x, a.y + bf * b.y, a.z + bf * b.z, a.w + bf * b.w);
            }
            w[e] = a;
        }
        // this thread's own group of plane q
        uint32_t m_cur;
        float4 x_cur = make_float4(0, 0, 0, 0), r_cur = x_cur;
        if (MODE == 0) {
            m_cur = reinterpret_cast<const uint32_t*>(st + 2 * TT_HALO_PAD)[tid];
        } else {
            x_cur = reinterpret_cast<const float4*>(st + TT_HALO_PAD)[tid];
            r_cur = reinterpret_cast<const float4*>(st + TT_HALO_PAD + TT_TILE_BYTES)[tid];
            m_cur = reinterpret_cast<const uint32_t*>(st + TT_HALO_PAD + 2 * TT_TILE_BYTES)[tid];
        }
        // every thread has read stage t: order those reads before the TMA
        // writes that refill it, and publish the window plane
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tt_fail) break;
        if (tid == 0 && t + TT_NS < nplanes) issue(t + TT_NS);
        // the row of plane q-1 from window planes q-2, q-1, q
        const int ic = q - 1;
        if (t >= 2 && inb && (m_prev & 0x80808080u)) {
            const float* wm = win + ((t - 2) % TT_NW) * (TT_HK * TT_HJ);
            const float* wc = win + ((t - 1) % TT_NW) * (TT_HK * TT_HJ);
            const float* wp = win + (t % TT_NW) * (TT_HK * TT_HJ);
            const int o = (ty + 1) * TT_HK + 4 + 4 * tg;
            const float4 c = *reinterpret_cast<const float4*>(wc + o);
            const float4 xp = *reinterpret_cast<const float4*>(wp + o);
            const float4 xm = *reinterpret_cast<const float4*>(wm + o);
            const float4 yp = *reinterpret_cast<const float4*>(wc + o + TT_HK);
            const float4 ym = *reinterpret_cast<const float4*>(wc + o - TT_HK);
            const float zm = wc[o - 1], zp = wc[o + 4];
            const float cv[6] = {zm, c.x, c.y, c.z, c.w, zp};
            const float xpv[4] = {xp.x, xp.y, xp.z, xp.w}, xmv[4] = {xm.x, xm.y, xm.z, xm.w};
            const float ypv[4] = {yp.x, yp.y, yp.z, yp.w}, ymv[4] = {ym.x, ym.y, ym.z, ym.w};
            float xov[4] = {x_prev.x, x_prev.y, x_prev.z, x_prev.w}, rov[4] = {r_prev.x, r_prev.y, r_prev.z, r_prev.w};
            float po[4];
            const int cidx = (ic * g.NY + jj) * g.NZ + kk;
            #pragma unroll
            for (int e = 0; e < 4; e++) {
                const uint32_t m = (m_prev >> (8 * e)) & 0xffu;
                const float cur = cv[e + 1];
                po[e] = (m & 0x80) ? cur : 0.0f;
                if (m & 0x80) {
                    float s = op.template start<float>(cidx + e, cur);
                    s = op.template comb<float>(s, (m & 1) ? cur : xpv[e]);
                    s = op.template comb<float>(s, (m & 2) ? cur : ypv[e]);
                    s = op.template comb<float>(s, (m & 4) ? cur : cv[e + 2]);
                    s = op.template comb<float>(s, (m & 8) ? cur : xmv[e]);
                    s = op.template comb<float>(s, (m & 16) ? cur : ymv[e]);
                    s = op.template comb<float>(s, (m & 32) ? cur : cv[e]);
                    const float z = op.template finish<float>(s);
                    if (MODE == 0) {
                        acc += (double)z * (double)cur;
                    } else {
                        xov[e] = xov[e] + af * cur;
                        rov[e] = rov[e] + (-af) * z;
                        acc += (double)rov[e] * (double)rov[e];
                    }
                }
            }
            if (MODE == 0) {
                reinterpret_cast<float4*>(pout)[cidx >> 2] = make_float4(po[0], po[1], po[2], po[3]);
            } else {
                reinterpret_cast<float4*>(x)[cidx >> 2] = make_float4(xov[0], xov[1], xov[2], xov[3]);
                reinterpret_cast<float4*>(r)[cidx >> 2] = make_float4(rov[0], rov[1], rov[2], rov[3]);
            }
        }
        m_prev = m_cur; x_prev = x_cur; r_prev = r_cur;
    }
    // the next pass may be launched now; it waits for this grid's completion
    // before it reads anything this grid writes
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (tt_fail) {
        // a TMA wait ran out: wait (bounded) for the loads still in flight
        // into this CTA's ring, report the timeout and leave without joining
        // the sum (the host clears the block counter before the next solve)
        if (tid == 0) {
            for (int u = t; u < nplanes && u < t + TT_NS; u++) tt_bar_wait(bar + (u % TT_NS), (uint32_t)((u / TT_NS) & 1));
            Rd.flag[F_DONE] = DONE_TIMEOUT;
        }
        return;
    }
    if (MODE == 1 && skip_dot) return;
    double tot;
    if (tt_finish(Rd, acc, &tot)) {
        if (MODE == 0) {
            Rd.scal[S_ZP] = tot;
            if (tot == 0) Rd.flag[F_DONE] = DONE_ZP0;
            else Rd.scal[S_ALPHA] = Rd.scal[S_A] / tot;
        } else {
            Rd.scal[S_RR] = tot;
            Rd.flag[F_ITERS] = it + 1;
            if (tot < Rd.scal[S_EPS]) Rd.flag[F_DONE] = DONE_CONV;
            else if (it + 1 >= maxiter) Rd.flag[F_DONE] = DONE_CAP;
            else { Rd.scal[S_BETA] = tot / Rd.scal[S_A]; Rd.scal[S_A] = tot; }
        }
    }
}

// Encodes a 3-D tensor map over an NX x NY x NZ array of `esize`-byte
// elements (k innermost) with box bx x by x 1; out-of-range elements of a box
// read as zero.
using TtEncodeFn = PFN_cuTensorMapEncodeTiled_v12000;
inline TtEncodeFn tt_encoder() {
    static TtEncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<TtEncodeFn>(p);
    }
    return fn;
}
inline bool tt_encode(CUtensorMap* m, const void* base, const Grid& g, int esize, int bx, int by) {
    TtEncodeFn enc = tt_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)g.NZ, (cuuint64_t)g.NY, (cuuint64_t)g.NX};
    const cuuint64_t strides[2] = {(cuuint64_t)g.NZ * esize, (cuuint64_t)g.NZ * g.NY * esize};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult rc = enc(m, esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 3,
                      const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return rc == CUDA_SUCCESS;
}

}  // namespace

/*
 * kernels.cu -- the sm_100a encode core: one warp per macroblock.
 *
 * A launch covers a flat list of (session, MB) work items, one frame-step
 * of any number of sessions of mixed size.  The grid is one wave of
 * resident CTAs; each warp owns a contiguous run of work items (consecutive
 * MBs of mostly one session) and, for each MB, runs the phases the launch
 * asks for while the next MB's inputs are already on their way:
 *
 *   stage   16-byte cp.async copies of the 46x48 luma search window (rows
 *           mb_y-15 .. +30, columns mb_x-16 .. +31) and of the source MB
 *           into one of two per-warp shared-memory buffers, issued one MB
 *           ahead.
 *   ME      - reference mode: SAD over the 11x11 coarse grid of
 *             megpu_kernels.cuh:27-166, then the 7x7 refinement of :307-446
 *             around its winner; full mode: every vector of [-15,15]^2;
 *           four packed pixels per step (__vabsdiffu4 + __dp4a on funnel-
 *           shifted words), two candidates interleaved per lane with split
 *           accumulators.  The reference picks a winner with a 2-D tree of
 *           strict '<' comparisons in the order self, right, below, diagonal
 *           (:95-154); that tree returns the minimum cost and, among equal
 *           costs, the cell with the smallest Z-order index (x bits on even
 *           positions).  Each lane therefore folds (cost << 10 | zorder) into
 *           one 32-bit key and a single redux.sync min picks the same winner.
 *           Then the three 16x16 SATD costs of :617-987 (inter, inter with
 *           the 3x3 interior filter, intra).
 *   MD      the decision of h261_moded.c:53-95.
 *   ENCDEC  per 8x8 block, one lane per row then per column: prediction
 *           with the H.261 loop filter, the reference's float/double AAN
 *           FDCT (mbgpu_kernels.cuh:337-442) with every rounding step
 *           spelled out by intrinsics, denoise against the session's
 *           offsets (:506-636), quantisation (:644-724), dequantisation
 *           (:731-815), the AAN IDCT (:827-931) and reconstruction
 *           (:988-1277) into the session's output picture.
 *
 * Denoise statistics are summed per warp over its run of MBs of one session
 * and published when the session changes; the warp whose publication
 * completes a session's frame (a ticket counting MBs) turns the statistics
 * into the next frame's offsets (:478-503).  No warp waits on another.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "h261b_device.h"

namespace {

constexpr int WIN_ROWS = 46;        /* rows mb_y-15 .. mb_y+30; columns mb_x-16 .. mb_x+31 */
/* A warp's two buffers (this MB, next MB) share 46 rows of 36 words.
 * Buffer k starts at word 16k of the array and holds, relative to that:
 *   words 0-11 of row r      window row r (12 words, 48 pixels)
 *   words 12-15 of row i     source luma row i (i < 16)
 *   words 12-13 of row 16+j  source chroma row j (Cb j < 8, Cr j >= 8)
 * so one base pointer addresses all of an MB's inputs.  Rows are 144 B, so
 * every row and source row is 16-byte aligned for the 16-byte copies, and
 * with a 36-word pitch the search's lanes, which read rows up to three
 * apart at up to 13 word columns, meet no bank twice. */
constexpr int WIN_PITCH_W = 36;
constexpr int SRC_COL_W = 12;
constexpr uint32_t FULL = 0xffffffffu;

struct __align__(16) WarpSmem {
    uint32_t buf[WIN_ROWS * WIN_PITCH_W]; /* both buffers, interleaved      */
    uint64_t bar[2];                      /* per buffer: the barrier its bulk
                                             row copies complete on (bulk
                                             staging only)                   */
    float t[4][72];                       /* transpose buffer: row stride 9,
                                             block stride 72 words, so both
                                             row and column accesses of the
                                             four blocks are conflict-free   */
};

/* one MB's staged inputs: buffer k of the warp's shared memory */
struct StageBuf {
    const uint32_t *p;
    /* window row r from word c */
    __device__ __forceinline__ const uint32_t *win(int r, int c) const { return p + r * WIN_PITCH_W + c; }
    /* source luma row i from word c */
    __device__ __forceinline__ const uint32_t *cur(int i, int c) const { return p + i * WIN_PITCH_W + SRC_COL_W + c; }
    /* source chroma row j (Cb rows 0-7, Cr rows 8-15), two words */
    __device__ __forceinline__ const uint32_t *curc(int j) const { return p + (16 + j) * WIN_PITCH_W + SRC_COL_W; }
};

__device__ __forceinline__ StageBuf stage_view(const uint32_t *wbuf, int k) { return StageBuf{ wbuf + 16 * k }; }

/* shared memory of one warp: both staging buffers, plus the transpose
 * buffer for kernels that encode (the search-only kernel has none) */
constexpr size_t kSearchWarpBytes = sizeof(uint32_t) * WIN_ROWS * WIN_PITCH_W + 2 * sizeof(uint64_t);
static_assert(kSearchWarpBytes % 16 == 0 && offsetof(WarpSmem, t) == kSearchWarpBytes, "warp shared layout");

/* what a launch of the step kernel does per MB */
enum StepKind {
    KIND_FUSED = 0,    /* the phases the launch asks for, in one pass       */
    KIND_SEARCH = 1,   /* search, costs and mode decision (into md_out)     */
    KIND_ENCODE = 2,   /* MC ... reconstruction from md_in, after a search
                          launch (programmatic dependent launch: waits for
                          that grid before it reads anything)               */
    KIND_FULL = 3,     /* KIND_FUSED with every phase (search, mode decision,
                          encode): the engine's and the no-allocation
                          entry point's launch, compiled without the paths
                          of partial launches                               */
};

/* the coarse grid's offsets { -14, -11, -8, -5, -2, 0, 2, 5, 8, 11, 14 }
 * (megpu_kernels.cuh:27-166), by arithmetic: lanes index it at 11 places
 * at once, which a constant-memory table would serve one address at a time */
__device__ __forceinline__ int stage1_offset(int t)
{
    return 3 * t - 14 - (t == 5 ? 1 : 0) - (t > 5 ? 2 : 0);
}
/* float tables initialised from double literals like the reference's */
__constant__ float c_fwd_post[8] = { 1.0, 0.720960, 0.765367, 0.850430, 1.0, 1.272759, 1.847759, 3.624510 };
__constant__ float c_inv_pre[8] = { 1.0, 1.387040, 1.306563, 1.175876, 1.0, 0.785695, 0.541196, 0.275899 };
__constant__ float c_inv_quant[32];

/* ------------------------------------------------ debug bounds checks
 *
 * Built with -DH261B_DEBUG_CHECKS (make check: lib/libh261b_check.so),
 * every global access whose address depends on a vector, a work item or a
 * picture size, and the shared-memory window reads of the motion
 * compensation, first test their index: a failing test is counted and its
 * site and index recorded (h261b_debug_check_status), and the access is
 * skipped or its index clamped into the buffer.  In the normal build the
 * checks compile to nothing. */
enum CheckSite {
    CHK_WORK_ITEM = 1,      /* MB index of a work item inside its picture     */
    CHK_STAGE_WINDOW = 2,   /* a staged window chunk inside the reference     */
    CHK_STAGE_SOURCE = 3,   /* a staged source row inside the picture         */
    CHK_MC_WINDOW = 4,      /* luma prediction rows inside the staged window  */
    CHK_MC_CHROMA = 5,      /* chroma prediction rows inside the reference    */
    CHK_RECON = 6,          /* reconstruction row inside the output picture   */
};

#ifdef H261B_DEBUG_CHECKS
__device__ unsigned long long g_check_count;
__device__ int g_check_first[2];

__device__ __noinline__ void check_fail(int site, int value)
{
    if (atomicAdd(&g_check_count, 1ull) == 0) {
        g_check_first[0] = site;
        g_check_first[1] = value;
    }
}
#define H261B_CHECK(cond, site, value) ((cond) ? true : (check_fail((site), (int)(value)), false))
#else
#define H261B_CHECK(cond, site, value) true
#endif

/* ------------------------------------------------------------ helpers */

__device__ __forceinline__ uint32_t spread8(uint32_t v)
{
    v &= 0xFFu;
    v = (v | (v << 4)) & 0x0F0Fu;
    v = (v | (v << 2)) & 0x3333u;
    v = (v | (v << 1)) & 0x5555u;
    return v;
}

__device__ __forceinline__ uint32_t compact8(uint32_t v)
{
    v &= 0x5555u;
    v = (v | (v >> 1)) & 0x3333u;
    v = (v | (v >> 2)) & 0x0F0Fu;
    v = (v | (v >> 4)) & 0x00FFu;
    return v;
}

__device__ __forceinline__ uint32_t zorder(uint32_t x, uint32_t y) { return spread8(x) | (spread8(y) << 1); }

/* eight window bytes of row `row` from byte column `col` (any alignment):
 * three word loads, two funnel shifts; 0 <= col <= 43 keeps the loads
 * inside the row (bytes past column 47, which are the source words or the
 * other buffer, are never used) */
__device__ __forceinline__ uint2 win8(const StageBuf s, int row, int col)
{
    const uint32_t *p = s.win(row, col >> 2);
    const uint32_t sh = (uint32_t)(col & 3) * 8u;
    const uint32_t a = p[0], b = p[1], c = p[2];
    return make_uint2(__funnelshift_r(a, b, sh), __funnelshift_r(b, c, sh));
}

/* eight bytes from global memory at any alignment; reads only the words
 * that hold one of those bytes */
__device__ __forceinline__ uint2 glob8(const uint8_t *ptr)
{
    const uint32_t *p = reinterpret_cast<const uint32_t *>((uintptr_t)ptr & ~(uintptr_t)3);
    const uint32_t sh = (uint32_t)((uintptr_t)ptr & 3) * 8u;
    const uint32_t a = p[0], b = p[1], c = sh ? p[2] : 0u;
    return make_uint2(__funnelshift_r(a, b, sh), __funnelshift_r(b, c, sh));
}

__device__ __forceinline__ int byte8(uint2 v, int i)
{
    return (int)(((i < 4 ? v.x : v.y) >> (8 * (i & 3))) & 0xFFu);
}

/* asynchronous global -> shared copies; a 16-byte window chunk outside the
 * picture is not read (src-size 0) and its bytes are zero-filled.  Window
 * chunks are cached in L1 too: neighbouring MBs of a warp share two thirds
 * of them. */
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16z(void *dst, const void *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

/* bulk copies (the async proxy) completed on a shared-memory barrier: the
 * alternative staging of the search window, one copy per window row.  The
 * source is always this GPU's own memory, and no copy is multicast. */
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
/* the one arrival of a phase, announcing the bytes its copies will bring */
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
/* this thread's earlier generic accesses of shared memory before its later
 * async-proxy writes (a buffer is refilled after the warp read it) */
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

/* bulk staging waits that gave up (bounded, so that nothing can hang);
 * reported by h261b_stage_status, always 0 in a correct run */
__device__ unsigned int g_stage_timeouts;

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

/* wait for a buffer's phase for at most 100 ms of the global timer (a row
 * copy takes about a microsecond): a copy that never completes is counted,
 * not waited for forever, and the warp stops waiting from then on */
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int lane)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 64; i++)
            if (mbar_try_wait(bar, parity))
                return true;
        if (global_ns() - t0 > 100000000ull)
            break;
    }
    if (lane == 0)
        atomicAdd(&g_stage_timeouts, 1u);
    return false;
}

/* sum of |a_i - b_i| over the four bytes, added to acc: per-byte absolute
 * difference, then a dot product with 1,1,1,1 (measured on B200 faster
 * than __vsadu4) */
__device__ __forceinline__ uint32_t sad4(uint32_t a, uint32_t b, uint32_t acc)
{
    return __dp4a(__vabsdiffu4(a, b), 0x01010101u, acc);
}

/* SADs of the source MB against the window blocks at two vectors, computed
 * together: four accumulators keep the dependency chains short */
__device__ __forceinline__ void sad16x16_pair(const StageBuf s, int vx0, int vy0, int vx1, int vy1, uint32_t &s0,
                                              uint32_t &s1)
{
    const int b0 = 16 + vx0, b1 = 16 + vx1;
    const uint32_t *p0 = s.win(15 + vy0, b0 >> 2);
    const uint32_t *p1 = s.win(15 + vy1, b1 >> 2);
    const uint32_t sh0 = (uint32_t)(b0 & 3) * 8u, sh1 = (uint32_t)(b1 & 3) * 8u;
    uint32_t a0 = 0, a1 = 0, c0 = 0, c1 = 0;
#pragma unroll 4
    for (int r = 0; r < 16; r++) {
        const uint4 c = *reinterpret_cast<const uint4 *>(s.cur(r, 0));
        const uint32_t x0 = p0[0], x1 = p0[1], x2 = p0[2], x3 = p0[3], x4 = p0[4];
        const uint32_t y0 = p1[0], y1 = p1[1], y2 = p1[2], y3 = p1[3], y4 = p1[4];
        a0 = sad4(c.x, __funnelshift_r(x0, x1, sh0), a0);
        c0 = sad4(c.x, __funnelshift_r(y0, y1, sh1), c0);
        a1 = sad4(c.y, __funnelshift_r(x1, x2, sh0), a1);
        c1 = sad4(c.y, __funnelshift_r(y1, y2, sh1), c1);
        a0 = sad4(c.z, __funnelshift_r(x2, x3, sh0), a0);
        c0 = sad4(c.z, __funnelshift_r(y2, y3, sh1), c0);
        a1 = sad4(c.w, __funnelshift_r(x3, x4, sh0), a1);
        c1 = sad4(c.w, __funnelshift_r(y3, y4, sh1), c1);
        p0 += WIN_PITCH_W;
        p1 += WIN_PITCH_W;
    }
    s0 = a0 + a1;
    s1 = c0 + c1;
}

/* SADs of the source MB against N window blocks stacked one row apart:
 * the vectors (vx, vy0 + k), k < N, with vx in [-15, 15] and vy0 in
 * [-15, 16 - N].  Window row R serves candidate k with source row R - k,
 * so each of the 15 + N window rows is loaded and aligned once for all N
 * candidates (the pair above loads and aligns 16 rows per candidate).
 * Rows R < N - 1 and R > 15 reach only some candidates; they are unrolled
 * apart from the steady rows in between. */
template <int N>
__device__ __forceinline__ void sad16x16_column(const StageBuf s, int vx, int vy0, uint32_t sad[N])
{
    const int b = 16 + vx;
    const uint32_t *p = s.win(15 + vy0, b >> 2);
    const uint32_t sh = (uint32_t)(b & 3) * 8u;
    uint32_t lo[N], hi[N];   /* two accumulators per candidate: shorter chains */
#pragma unroll
    for (int k = 0; k < N; k++)
        lo[k] = hi[k] = 0u;
    auto row = [&](const uint32_t *q, uint32_t w[4]) {
        const uint32_t x0 = q[0], x1 = q[1], x2 = q[2], x3 = q[3], x4 = q[4];
        w[0] = __funnelshift_r(x0, x1, sh);
        w[1] = __funnelshift_r(x1, x2, sh);
        w[2] = __funnelshift_r(x2, x3, sh);
        w[3] = __funnelshift_r(x3, x4, sh);
    };
    auto add = [&](int k, int r, const uint32_t w[4]) {
        const uint4 c = *reinterpret_cast<const uint4 *>(s.cur(r, 0));
        lo[k] = sad4(c.x, w[0], lo[k]);
        hi[k] = sad4(c.y, w[1], hi[k]);
        lo[k] = sad4(c.z, w[2], lo[k]);
        hi[k] = sad4(c.w, w[3], hi[k]);
    };
    /* rows 0 .. N-2: candidates k <= R */
#pragma unroll
    for (int R = 0; R < N - 1; R++) {
        uint32_t w[4];
        row(p + R * WIN_PITCH_W, w);
#pragma unroll
        for (int k = 0; k <= R; k++)
            add(k, R - k, w);
    }
    /* rows N-1 .. 15: every candidate */
#pragma unroll 1
    for (int R = N - 1; R < 16; R++) {
        uint32_t w[4];
        row(p + R * WIN_PITCH_W, w);
#pragma unroll
        for (int k = 0; k < N; k++)
            add(k, R - k, w);
    }
    /* rows 16 .. 14+N: candidates k >= R - 15 */
#pragma unroll
    for (int R = 16; R < 15 + N; R++) {
        uint32_t w[4];
        row(p + R * WIN_PITCH_W, w);
#pragma unroll
        for (int k = R - 15; k < N; k++)
            add(k, R - k, w);
    }
#pragma unroll
    for (int k = 0; k < N; k++)
        sad[k] = lo[k] + hi[k];
}

/* 4x4 Hadamard SATD, megpu_kernels.cuh:467-500 */
__device__ __forceinline__ int32_t satd4x4(const int32_t d[16])
{
    int32_t t[16];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int32_t a1 = d[4 * i] + d[4 * i + 1], a2 = d[4 * i] - d[4 * i + 1];
        const int32_t a3 = d[4 * i + 2] + d[4 * i + 3], a4 = d[4 * i + 2] - d[4 * i + 3];
        t[4 * i + 0] = a1 + a3;
        t[4 * i + 1] = a2 + a4;
        t[4 * i + 2] = a1 - a3;
        t[4 * i + 3] = a2 - a4;
    }
    int32_t satd = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int32_t a1 = t[i] + t[4 + i], a2 = t[i] - t[4 + i];
        const int32_t a3 = t[8 + i] + t[12 + i], a4 = t[8 + i] - t[12 + i];
        satd += abs(a1 + a3) + abs(a2 + a4) + abs(a1 - a3) + abs(a2 - a4);
    }
    return satd;
}

/* ---------------------------------------------- exact float/double math */

/* `float *= double`: double product rounded to float */
__device__ __forceinline__ float dmulf(float x, double k)
{
    return __double2float_rn(__dmul_rn((double)x, k));
}

/* `float = float * double + float`: fused (one rounding) or not */
template <int FMAD>
__device__ __forceinline__ float dmadf(float a, double k, float c)
{
    if (FMAD)
        return __double2float_rn(__fma_rn((double)a, k, (double)c));
    return __double2float_rn(__dadd_rn(__dmul_rn((double)a, k), (double)c));
}

/* the AAN forward butterfly shared by both passes (mbgpu_kernels.cuh:359-388) */
template <int FMAD>
__device__ __forceinline__ void fdct_butterfly(float tmp0, float tmp1, float tmp2, float tmp3, float tmp4,
                                               float tmp5, float tmp6, float tmp7, float o[8])
{
    const float tmp10 = tmp0 + tmp3, tmp13 = tmp0 - tmp3, tmp11 = tmp1 + tmp2, tmp12 = tmp1 - tmp2;
    o[0] = tmp10 + tmp11;
    o[4] = tmp10 - tmp11;
    const float z1 = dmulf(tmp12 + tmp13, 0.707107);
    o[2] = tmp13 + z1;
    o[6] = tmp13 - z1;
    tmp4 = tmp4 + tmp5;
    tmp5 = tmp5 + tmp6;
    tmp6 = tmp6 + tmp7;
    const float z5 = dmulf(tmp4 - tmp6, 0.382683);
    const float z2 = dmadf<FMAD>(tmp4, 0.541196, z5);
    const float z4 = dmadf<FMAD>(tmp6, 1.306563, z5);
    const float z3 = dmulf(tmp5, 0.707107);
    const float z11 = tmp7 + z3, z13 = tmp7 - z3;
    o[5] = z13 + z2;
    o[3] = z13 - z2;
    o[1] = z11 + z4;
    o[7] = z11 - z4;
}

/* floorf( cs * post * v + 0.49999 ) as the reference writes it
 * (mbgpu_kernels.cuh:413-437): a float product, the sum with the double
 * literal rounded to double, then to float, then the floor.  For every
 * finite float p, floorf((float)((double)p + 0.49999)) equals
 * floorf(p + 0.49999f) with the float literal (the float nearest to
 * 0.49999) -- checked for all 2.5e9 floats of magnitude below 2^24 by
 * tests/rounding_check.c; above it both leave p unchanged -- so the sum is
 * taken in float and floored by the conversion itself: no conversion to or
 * from double. */
__device__ __forceinline__ int32_t fdct_round(float cs, float post, float v)
{
    const float prod = __fmul_rn(__fmul_rn(cs, post), v);
    return __float2int_rd(__fadd_rn(prod, 0.49999f));
}

/* the AAN inverse butterfly after its first level of adds (mbgpu_kernels.cuh
 * :851-887 for columns, :892-919 for rows); the caller forms the first level
 * (tmp12 = p2 - p6, tmp13 = p2 + p6, tmp10 = p0 + p4, tmp11 = p0 - p4,
 * z11 = p1 + p7, z12 = p1 - p7, z13 = p5 + p3, z10 = p5 - p3) */
template <int FMAD>
__device__ __forceinline__ void idct_rest(float tmp12, float tmp13, float tmp10, float tmp11, float z11,
                                          float z12, float z13, float z10, float o[8])
{
    tmp12 = dmulf(tmp12, 1.414214);
    tmp12 = tmp12 - tmp13;
    const float tmp0 = tmp10 + tmp13, tmp1 = tmp11 + tmp12, tmp2 = tmp11 - tmp12, tmp3 = tmp10 - tmp13;
    tmp13 = z11 + z13;
    tmp11 = dmulf(z11 - z13, 1.414214);
    const float z5 = dmulf(z12 + z10, 1.84776);
    tmp10 = dmadf<FMAD>(z12, 1.082392, -z5);
    tmp12 = dmadf<FMAD>(z10, -2.613126, z5);
    tmp12 = tmp12 - tmp13;
    tmp11 = tmp11 - tmp12;
    tmp10 = tmp10 + tmp11;
    o[0] = tmp0 + tmp13;
    o[1] = tmp1 + tmp12;
    o[2] = tmp2 + tmp11;
    o[3] = tmp3 - tmp10;
    o[4] = tmp3 + tmp10;
    o[5] = tmp2 - tmp11;
    o[6] = tmp1 - tmp12;
    o[7] = tmp0 - tmp13;
}

/* first level of the column pass on prescaled products t = P * cs: the
 * reference built with nvcc defaults fuses the left-hand product of each
 * add into one FFMA (its product rounds once, with the sum) */
template <int FMAD>
__device__ __forceinline__ float first_add(float Pa, float csa, float ta, float tb)
{
    return FMAD ? __fmaf_rn(Pa, csa, tb) : __fadd_rn(ta, tb);
}
template <int FMAD>
__device__ __forceinline__ float first_sub(float Pa, float csa, float ta, float tb)
{
    return FMAD ? __fmaf_rn(Pa, csa, -tb) : __fsub_rn(ta, tb);
}

/* CLAMP_255( (Int32) floor( v + 0.49999 ) ) with v widened to double */
__device__ __forceinline__ int32_t idct_round(float v)
{
    const int32_t r = (int32_t)floor(__dadd_rn((double)v, 0.49999));
    return min(255, max(-256, r));
}

/* ---------------------------------------------------------- per MB */

struct MbDecision {
    int32_t type, flags, mvx, mvy, cost;
};

/* start the asynchronous copies of one MB's inputs into buffer k.  The
 * window is 46 rows of three 16-byte chunks; picture widths are multiples
 * of 16 and luma planes 16-byte aligned, so a chunk lies wholly inside or
 * wholly outside the picture, and one outside is zero-filled.  Lanes 0-29
 * take (row, chunk) = (lane / 3 + 10 i, lane % 3). */
__device__ __forceinline__ void stage_mb(uint32_t *wbuf, int k, const h261b_session_dev_t &S, int mbx, int mby,
                                         int lane, int row_lo = 0, int row_n = WIN_ROWS, uint64_t *bar = nullptr,
                                         uint32_t extra_bytes = 0)
{
    const int H = S.mbh * 16;
    const int x0 = mbx * 16, y0 = mby * 16;
    uint32_t *base = wbuf + 16 * k;
    if (bar) {
        /* bulk staging: one copy per window row inside the picture, of its
         * 16-byte chunks inside the picture (48 bytes, or 32 at a left or
         * right picture edge), into the same pitched rows; chunks outside
         * the picture are zeroed by plain stores.  Lane 0 arrives on the
         * buffer's barrier announcing the bytes of all the copies. */
        const int c_lo = mbx > 0 ? 0 : 1, c_hi = mbx < S.mbw - 1 ? 3 : 2;
        const uint32_t row_bytes = 16u * (uint32_t)(c_hi - c_lo);
        const int y_first = max(y0 - 15 + row_lo, 0), y_last = min(y0 - 15 + row_lo + row_n, H);
        const uint32_t bytes = y_last > y_first ? row_bytes * (uint32_t)(y_last - y_first) : 0u;
        fence_proxy_async();
        if (lane == 0)
            mbar_arrive_expect(bar, bytes + extra_bytes);
        for (int r = row_lo + lane; r < row_lo + row_n; r += 32) {
            const int y = y0 - 15 + r;
            uint32_t *dst = base + r * WIN_PITCH_W;
            if (y >= 0 && y < H && H261B_CHECK(x0 - 16 + 16 * c_lo >= 0 && x0 - 16 + 16 * c_hi <= S.mbw * 16,
                                               CHK_STAGE_WINDOW, x0))
                bulk_copy(dst + 4 * c_lo, S.ref_y + (size_t)y * S.pitch_y + x0 - 16 + 16 * c_lo, row_bytes, bar);
            const uint4 z = make_uint4(0u, 0u, 0u, 0u);
            for (int j = 0; j < 3; j++)
                if (y < 0 || y >= H || j < c_lo || j >= c_hi)
                    *reinterpret_cast<uint4 *>(dst + 4 * j) = z;
        }
    } else if (lane < 30) {
        const int j = lane % 3, r0 = lane / 3;
        const bool xok = j == 1 || (j == 0 ? mbx > 0 : mbx < S.mbw - 1);
        const int x = x0 - 16 + 16 * j;
        uint32_t *dst = base + 4 * j;
        for (int r = row_lo + r0; r < row_lo + row_n; r += 10) {
            const int y = y0 - 15 + r;
            bool ok = xok && y >= 0 && y < H;
            ok = ok && H261B_CHECK(x >= 0 && x + 16 <= S.mbw * 16, CHK_STAGE_WINDOW, x);
            cp_async16z(dst + r * WIN_PITCH_W, ok ? S.ref_y + (size_t)y * S.pitch_y + x : S.ref_y, ok);
        }
    }
    if (lane < 16) {
        if (H261B_CHECK(y0 + lane < H && x0 + 16 <= S.mbw * 16, CHK_STAGE_SOURCE, y0 + lane))
            cp_async16(base + lane * WIN_PITCH_W + SRC_COL_W, S.cur_y + (size_t)(y0 + lane) * S.pitch_y + x0);
    } else {
        const int q = lane - 16, pl = q >> 3, r = q & 7;
        const uint8_t *src = pl ? S.cur_cr : S.cur_cb;
        if (H261B_CHECK(mby * 8 + r < S.mbh * 8 && mbx * 8 + 8 <= S.mbw * 8, CHK_STAGE_SOURCE, mby * 8 + r))
            cp_async8(base + (16 + q) * WIN_PITCH_W + SRC_COL_W,
                      src + (size_t)(mby * 8 + r) * S.pitch_c + mbx * 8);
    }
}

/* motion search + SATD costs; results are warp-uniform.  FULL: the
 * exhaustive search, else the reference's grid and refinement (a launch
 * compiles only the one it runs: a smaller body misses the instruction
 * cache less) */
template <bool FULL_SEARCH>
__device__ __forceinline__ void motion_estimate(const StageBuf s, const h261b_session_dev_t &S, int mbx, int mby,
                                                int lane, me_gpu_mb_t &res, int8_t &s1x, int8_t &s1y)
{
    const int bx = mbx * 16, by = mby * 16;
    /* per-MB limits, gpu_device.cu:226-265 */
    const int lminx = max(-15, -bx), lmaxx = min(15, (S.mbw - 1) * 16 - bx);
    const int lminy = max(-15, -by), lmaxy = min(15, (S.mbh - 1) * 16 - by);
    int vx, vy;
    /* every lane computes two SADs per iteration; a vector outside the
     * limits is replaced by (0, 0) so no address leaves the window, and its
     * cost discarded (65535, as the reference marks skipped candidates) */
    if (FULL_SEARCH) {
        /* columns of four vertically adjacent vectors: 31 columns x 8
         * groups, the last group (vy 13..15) started at vy 12, which the
         * group before holds too (a repeated key changes no minimum) */
        uint32_t best = FULL;
        for (int t = lane; t < 31 * 8; t += 32) {
            const int gy = t / 31, tx = t - gy * 31;
            const int x = tx - 15, y0 = min(-15 + 4 * gy, 12);
            uint32_t sad[4];
            sad16x16_column<4>(s, x, y0, sad);
            const bool ox = x >= lminx && x <= lmaxx;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int y = y0 + k;
                const bool ok = ox && y >= lminy && y <= lmaxy;
                best = min(best, ((ok ? sad[k] : 65535u) << 10) | zorder(tx, y + 15));
            }
        }
        best = __reduce_min_sync(FULL, best) & 1023u; /* Z-order index only */
        vx = (int)compact8(best) - 15;
        vy = (int)compact8(best >> 1) - 15;
        s1x = s1y = 0;
    } else {
        uint32_t best = FULL;
        for (int c = lane; c < 121; c += 64) {
            const int c1 = c + 32;
            const bool has1 = c1 < 121;
            const int ty0 = c / 11, tx0 = c - ty0 * 11, ty1 = (has1 ? c1 : c) / 11, tx1 = (has1 ? c1 : c) - ty1 * 11;
            const int x0 = stage1_offset(tx0), y0 = stage1_offset(ty0), x1 = stage1_offset(tx1), y1 = stage1_offset(ty1);
            const bool o0 = x0 >= lminx && x0 <= lmaxx && y0 >= lminy && y0 <= lmaxy;
            const bool o1 = has1 && x1 >= lminx && x1 <= lmaxx && y1 >= lminy && y1 <= lmaxy;
            uint32_t s0, s1;
            sad16x16_pair(s, o0 ? x0 : 0, o0 ? y0 : 0, o1 ? x1 : 0, o1 ? y1 : 0, s0, s1);
            best = min(best, ((o0 ? s0 : 65535u) << 10) | zorder(tx0, ty0));
            if (has1)
                best = min(best, ((o1 ? s1 : 65535u) << 10) | zorder(tx1, ty1));
        }
        best = __reduce_min_sync(FULL, best) & 1023u; /* Z-order index only */
        const int v1x = stage1_offset((int)compact8(best)), v1y = stage1_offset((int)compact8(best >> 1));
        s1x = (int8_t)v1x;
        s1y = (int8_t)v1y;
        /* the 7x7 refinement as 28 vertical pairs, lanes 0-27: column tx,
         * rows 2gy and 2gy+1 (row 7 of the last pair is past the grid).  A
         * pair reaching past +-15 is computed from the nearest in-window
         * rows and each vector takes its SAD from there; vectors outside
         * the limits are discarded as before */
        best = FULL;
        if (lane < 28) {
            const int gy = lane / 7, tx = lane - gy * 7;
            const int x = v1x + tx - 3, y0 = v1y + 2 * gy - 3;
            const int base = min(max(y0, -15), 14);
            uint32_t sad[2];
            sad16x16_column<2>(s, min(max(x, -15), 15), base, sad);
            const bool ox = x >= lminx && x <= lmaxx;
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int y = y0 + k, ty = 2 * gy + k;
                const bool ok = ox && ty < 7 && y >= lminy && y <= lmaxy;
                const uint32_t v = (y - base) == 0 ? sad[0] : sad[1];
                if (ty < 7)
                    best = min(best, ((ok ? v : 65535u) << 10) | zorder(tx, ty));
            }
        }
        best = __reduce_min_sync(FULL, best) & 1023u;
        vx = v1x + (int)compact8(best) - 3;
        vy = v1y + (int)compact8(best >> 1) - 3;
    }

    /* costs at the final vector: lanes 0-15 inter, 16-31 filtered inter,
     * one 4x4 sub-block each; then intra on lanes 0-15.  Each lane reads
     * six window rows around its sub-block (clamped to the window: a
     * clamped row is one the sub-block never needs) from one column left of
     * it, so pixel (iy, ix) is byte ix + 1 of row iy + 1 */
    const int sb = lane & 15, sx = sb & 3, sy = sb >> 2;
    const bool filt = lane >= 16;
    const int wr0 = 15 + vy + sy * 4, wc0 = 16 + vx + sx * 4;
    uint2 rr[6];
#pragma unroll
    for (int k = 0; k < 6; k++)
        rr[k] = win8(s, min(max(wr0 - 1 + k, 0), WIN_ROWS - 1), wc0 - 1);
    /* the 3x3 filter, separable: horizontal [1 2 1] sums of rows R = 0..5
     * at columns C = 1..4, then vertical [1 2 1] over them.  Pixel (ix, iy)
     * of the sub-block sits at (lx, ly) = ((sx & 1) * 4 + ix, (sy & 1) * 4
     * + iy) of its 8x8 block; only the block's interior (1..6) is filtered */
    int32_t hs[6][4];
#pragma unroll
    for (int R = 0; R < 6; R++) {
#pragma unroll
        for (int C = 1; C <= 4; C++)
            hs[R][C - 1] = byte8(rr[R], C - 1) + 2 * byte8(rr[R], C) + byte8(rr[R], C + 1);
    }
    const uint32_t xin = (sx & 1) ? 0x7u : 0xEu, yin = (sy & 1) ? 0x7u : 0xEu; /* interior ix / iy bits */
    int32_t d[16], di[16];
#pragma unroll
    for (int iy = 0; iy < 4; iy++) {
        const uint32_t cw = *s.cur(sy * 4 + iy, sx);
#pragma unroll
        for (int ix = 0; ix < 4; ix++) {
            const int c = (int)((cw >> (8 * ix)) & 0xFFu);
            const int f = (hs[iy][ix] + 2 * hs[iy + 1][ix] + hs[iy + 2][ix] + 8) >> 4;
            const bool use_f = filt && ((xin >> ix) & (yin >> iy) & 1u);
            const int p = use_f ? f : byte8(rr[iy + 1], ix + 1);
            d[iy * 4 + ix] = c - p;
            di[iy * 4 + ix] = c;
        }
    }
    const int32_t satd = satd4x4(d), satd_i = satd4x4(di);
    res.i_16x16_cost = (int32_t)__reduce_add_sync(FULL, filt ? 0u : (uint32_t)satd);
    res.i_16x16_filter_cost = (int32_t)__reduce_add_sync(FULL, filt ? (uint32_t)satd : 0u);
    res.i_intra_cost = (int32_t)__reduce_add_sync(FULL, filt ? 0u : (uint32_t)satd_i);
    res.i_zero_cost = 0;
    res.s_16x16_mv.i8_mx = (int8_t)vx;
    res.s_16x16_mv.i8_my = (int8_t)vy;
}

/* h261_moded.c:53-95 */
__device__ __forceinline__ MbDecision mode_decide(const me_gpu_mb_t &g, int frame_type)
{
    MbDecision m;
    if (frame_type == H261B_FRAME_TYPE_INTRA ||
        (g.i_intra_cost <= g.i_16x16_cost && g.i_intra_cost <= g.i_16x16_filter_cost)) {
        m.type = H261B_MB_TYPE_INTRA;
        m.cost = g.i_intra_cost;
        m.flags = 0;
        m.mvx = m.mvy = 0;
    } else {
        m.type = H261B_MB_TYPE_INTER;
        if (g.i_16x16_filter_cost < g.i_16x16_cost) {
            m.flags = H261B_MB_MC | H261B_MB_FILTER;
            m.cost = g.i_16x16_filter_cost;
        } else {
            m.flags = 0;
            m.cost = g.i_16x16_cost;
        }
        m.mvx = g.s_16x16_mv.i8_mx;
        m.mvy = g.s_16x16_mv.i8_my;
        if (m.mvx != 0 || m.mvy != 0)
            m.flags |= H261B_MB_MC;
    }
    return m;
}

/* H.261 loop-filter tap pair, horizontal [1 2 1] with x4 edge columns
 * (mbgpu_kernels.cuh:88-103) on one 8-pixel row */
__device__ __forceinline__ int hfilt(uint2 v, int c)
{
    if (c == 0)
        return byte8(v, 0) * 4;
    if (c == 7)
        return byte8(v, 7) * 4;
    return byte8(v, c - 1) + byte8(v, c) * 2 + byte8(v, c + 1);
}

/* one pass over up to four blocks of the MB: lane = slot * 8 + row (then
 * column).  Adds the block-summed |coefficient| of column (lane & 7) to
 * colsum[v] and returns this pass's CBP bits. */
template <int FMAD, bool ABI>
__device__ __forceinline__ uint32_t encdec_pass(float (*tb)[72], const StageBuf s, const h261b_session_dev_t &S,
                                                int mb, int mbx, int mby, const MbDecision &m, int quant,
                                                bool luma_pass, int lane, int32_t colsum[8], uint32_t &ssd)
{
    const bool active = luma_pass || lane < 16;
    const int slot = lane >> 3, r = lane & 7;
    const int b = luma_pass ? slot : 4 + (slot & 1);
    const bool intra = m.type == H261B_MB_TYPE_INTRA;
    const bool filter = (m.flags & H261B_MB_FILTER) != 0;
    const int t = intra ? 0 : 1;

    /* ---- prediction and residual of row r (mbgpu_kernels.cuh:59-166):
     * the source row and up to three reference rows as 8-byte vectors */
    const int bx8 = luma_pass ? (b & 1) * 8 : 0, by8 = luma_pass ? (b >> 1) * 8 : 0;
    int32_t res[8];
    uint32_t pred_lo = 0, pred_hi = 0;   /* the row's prediction, one byte a pixel */
    if (active) {
        const uint2 cw = luma_pass ? *reinterpret_cast<const uint2 *>(s.cur(by8 + r, bx8 >> 2))
                                   : *reinterpret_cast<const uint2 *>(s.curc(8 * (b - 4) + r));
        if (intra) {
#pragma unroll
            for (int i = 0; i < 8; i++)
                res[i] = byte8(cw, i);
        } else {
            /* rows r-1, r, r+1 of the prediction block, clamped inside it
             * (the edge rows of the loop filter use row r only) */
            const int ra_i = max(r - 1, 0), rc_i = min(r + 1, 7);
            uint2 ra, rb, rc;
            if (luma_pass) {
                int wr = 15 + m.mvy + by8, wc = 16 + m.mvx + bx8;
                /* rows wr..wr+7 of the 46-row window, byte columns wc..wc+7
                 * with win8's three words inside the 12-word row */
                if (!H261B_CHECK(wr >= 0 && wr + 7 < WIN_ROWS && wc >= 0 && wc <= 40, CHK_MC_WINDOW,
                                 wr * 64 + wc)) {
                    wr = min(max(wr, 0), WIN_ROWS - 8);
                    wc = min(max(wc, 0), 40);
                }
                rb = win8(s, wr + r, wc);
                ra = filter ? win8(s, wr + ra_i, wc) : rb;
                rc = filter ? win8(s, wr + rc_i, wc) : rb;
            } else {
                int cmx = m.mvx / 2, cmy = m.mvy / 2; /* truncation toward zero */
#ifdef H261B_DEBUG_CHECKS
                /* rows inside the chroma plane; glob8's words (12 bytes from
                 * the word boundary when unaligned) inside the row */
                {
                    const int cx = mbx * 8 + cmx, cy = mby * 8 + cmy, wc8 = S.mbw * 8;
                    if (!H261B_CHECK(cy >= 0 && cy + 8 <= S.mbh * 8 && cx >= 0 &&
                                         (cx & ~3) + ((cx & 3) ? 12 : 8) <= wc8,
                                     CHK_MC_CHROMA, cy * 4096 + cx))
                        cmx = cmy = 0;
                }
#endif
                const uint8_t *g = ((b == 4) ? S.ref_cb : S.ref_cr) + (size_t)(mby * 8 + cmy) * S.pitch_c +
                                   (mbx * 8 + cmx);
                rb = glob8(g + (size_t)r * S.pitch_c);
                ra = filter ? glob8(g + (size_t)ra_i * S.pitch_c) : rb;
                rc = filter ? glob8(g + (size_t)rc_i * S.pitch_c) : rb;
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                int p;
                if (filter) {
                    if (r == 0 || r == 7)
                        p = (hfilt(rb, i) + 2) >> 2;
                    else
                        p = (hfilt(ra, i) + hfilt(rb, i) * 2 + hfilt(rc, i) + 8) >> 4;
                } else {
                    p = byte8(rb, i);
                }
                if (i < 4)
                    pred_lo |= (uint32_t)p << (8 * i);
                else
                    pred_hi |= (uint32_t)p << (8 * (i - 4));
                res[i] = byte8(cw, i) - p;
            }
        }
        /* ---- FDCT pass 1 on row r */
        float o[8];
        fdct_butterfly<FMAD>((float)(res[0] + res[7]), (float)(res[1] + res[6]), (float)(res[2] + res[5]),
                             (float)(res[3] + res[4]), (float)(res[3] - res[4]), (float)(res[2] - res[5]),
                             (float)(res[1] - res[6]), (float)(res[0] - res[7]), o);
#pragma unroll
        for (int k = 0; k < 8; k++)
            tb[slot][r * 9 + k] = o[k];
    }
    __syncwarp();

    /* ---- FDCT pass 2 on column c = r: coefficients (v, c), v = 0..7 */
    const int c = r;
    int32_t lev[8], nz[8];
    int32_t acc = 0;
#pragma unroll
    for (int v = 0; v < 8; v++) {
        lev[v] = 0;
        nz[v] = 0;
    }
    if (active) {
        float q[8], o[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            q[k] = tb[slot][k * 9 + c];
        fdct_butterfly<FMAD>(q[0] + q[7], q[1] + q[6], q[2] + q[5], q[3] + q[4], q[3] - q[4], q[2] - q[5],
                             q[1] - q[6], q[0] - q[7], o);
        const float cs = __fmul_rn(c_fwd_post[c], 0.125f); /* = dmulf(.., 0.125): a power-of-two scaling is exact */
        const float inv = c_inv_quant[quant];
        /* this column's eight offsets, UInt16, one 16-byte load */
        const uint4 ow = *reinterpret_cast<const uint4 *>(&S.dn->offset[t][c][0]);
        const uint32_t offw[4] = { ow.x, ow.y, ow.z, ow.w };
#pragma unroll
        for (int v = 0; v < 8; v++) {
            int32_t lv = fdct_round(cs, c_fwd_post[v], o[v]);
            /* denoise (mbgpu_kernels.cuh:586-604) */
            const int32_t sign = lv >> 31;
            lv = (lv ^ sign) - sign;
            nz[v] = lv;
            const int32_t off = (int32_t)((offw[v >> 1] >> (16 * (v & 1))) & 0xFFFFu);
            lv = max(lv - off, 0);
            lv = (lv ^ sign) - sign;
            /* quant (mbgpu_kernels.cuh:689-716) */
            if (intra && v == 0 && c == 0) {
                int32_t dc = lv / 8;
                dc = max(dc, 1);
                dc = min(dc, 254);
                if (dc == 128)
                    dc = 255;
                lev[0] = dc;
                acc += 100;
            } else {
                const int32_t l = min(127, max(-127, __float2int_rz(__fmul_rn(__int2float_rn(lv), inv))));
                lev[v] = l;
                const int32_t al = abs(l);
                acc += al > 1 ? 100 : al;
            }
        }
    }
    /* block sums over the 8 lanes of a block */
    acc += __shfl_xor_sync(FULL, acc, 1);
    acc += __shfl_xor_sync(FULL, acc, 2);
    acc += __shfl_xor_sync(FULL, acc, 4);
    const bool coded = active && acc > 2;
    const uint32_t cbp = __reduce_or_sync(FULL, coded ? (uint32_t)H261B_CBP_BIT(b) : 0u);

    /* denoise statistics: sum the same coefficient position over blocks */
#pragma unroll
    for (int v = 0; v < 8; v++) {
        int32_t x = nz[v];
        x += __shfl_xor_sync(FULL, x, 8);
        x += __shfl_xor_sync(FULL, x, 16);
        colsum[v] += x;
    }

    /* ---- levels out */
    if (active) {
        if (ABI && S.abi_out) {
            int32_t *tc = S.abi_out[mb].rgi_tcoeff[b];
#pragma unroll
            for (int v = 0; v < 8; v++)
                tc[v * 8 + c] = lev[v];
        }
        if (S.level_out) {
            /* column-major: this lane's eight levels are contiguous */
            uint32_t lo = 0, hi = 0;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                lo |= ((uint32_t)lev[v] & 0xFFu) << (8 * v);
                hi |= ((uint32_t)lev[v + 4] & 0xFFu) << (8 * v);
            }
            *reinterpret_cast<uint2 *>(S.level_out + (size_t)mb * 384 + b * 64 + c * 8) = make_uint2(lo, hi);
        }
    }

    /* ---- dequant (mbgpu_kernels.cuh:763-814) and IDCT pass 1 on column c */
    __syncwarp(); /* pass-2 reads of the transpose buffer are done */
    if (active) {
        const int32_t qa = coded ? ((quant - 1) | 1) : 0, qm = coded ? quant * 2 : 0;
        float col[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            int32_t dq;
            if (intra && k == 0 && c == 0) {
                dq = lev[0] == 255 ? 1024 : lev[0] * 8;
            } else {
                int32_t l = lev[k] * qm;
                if (l > 0)
                    l += qa;
                else if (l < 0)
                    l -= qa;
                dq = min(2047, max(-2048, l));
            }
            col[k] = (float)dq;
        }
        if (coded) {
            /* prescale: t = (coef * pre[col]) * (pre[row] * 0.125) */
            float P[8], cs[8], tt[8], o[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                cs[k] = __fmul_rn(c_inv_pre[k], 0.125f); /* exact, as dmulf(.., 0.125) */
                P[k] = __fmul_rn(col[k], c_inv_pre[c]);
                tt[k] = __fmul_rn(P[k], cs[k]);
            }
            idct_rest<FMAD>(first_sub<FMAD>(P[2], cs[2], tt[2], tt[6]), first_add<FMAD>(P[2], cs[2], tt[2], tt[6]),
                            first_add<FMAD>(P[0], cs[0], tt[0], tt[4]), first_sub<FMAD>(P[0], cs[0], tt[0], tt[4]),
                            first_add<FMAD>(P[1], cs[1], tt[1], tt[7]), first_sub<FMAD>(P[1], cs[1], tt[1], tt[7]),
                            first_add<FMAD>(P[5], cs[5], tt[5], tt[3]), first_sub<FMAD>(P[5], cs[5], tt[5], tt[3]), o);
#pragma unroll
            for (int k = 0; k < 8; k++)
                tb[slot][k * 9 + c] = o[k];
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++)
                tb[slot][k * 9 + c] = col[k];
        }
    }
    __syncwarp();

    /* ---- IDCT pass 2 on row r and reconstruction (mbgpu_kernels.cuh:988-1096) */
    if (active) {
        const float *p = tb[slot] + r * 9;
        int32_t out[8];
        if (coded) {
            float o[8];
            idct_rest<FMAD>(p[2] - p[6], p[2] + p[6], p[0] + p[4], p[0] - p[4], p[1] + p[7], p[1] - p[7],
                            p[5] + p[3], p[5] - p[3], o);
#pragma unroll
            for (int i = 0; i < 8; i++)
                out[i] = idct_round(o[i]);
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++)
                out[i] = (int32_t)p[i];
        }
        uint32_t lo = 0, hi = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int32_t pi = (int32_t)(((i < 4 ? pred_lo : pred_hi) >> (8 * (i & 3))) & 0xFFu);
            const int32_t v = min(255, max(0, out[i] + pi));
            if (i < 4)
                lo |= (uint32_t)v << (8 * i);
            else
                hi |= (uint32_t)v << (8 * (i - 4));
        }
        uint8_t *dst;
        if (luma_pass)
            dst = S.rec_y + (size_t)(mby * 16 + by8 + r) * S.pitch_y + mbx * 16 + bx8;
        else
            dst = ((b == 4) ? S.rec_cb : S.rec_cr) + (size_t)(mby * 8 + r) * S.pitch_c + mbx * 8;
        if (H261B_CHECK(luma_pass ? (mby * 16 + by8 + r < S.mbh * 16 && mbx * 16 + bx8 + 8 <= S.mbw * 16)
                                  : (mby * 8 + r < S.mbh * 8 && mbx * 8 + 8 <= S.mbw * 8),
                        CHK_RECON, mby * 4096 + mbx))
            *reinterpret_cast<uint2 *>(dst) = make_uint2(lo, hi);
        if (S.ssd_out) {
            /* squared error of this row against the source, for the
             * picture's PSNR (h261_main.c:38-91) */
            const uint2 cw = luma_pass ? *reinterpret_cast<const uint2 *>(s.cur(by8 + r, bx8 >> 2))
                                       : *reinterpret_cast<const uint2 *>(s.curc(8 * (b - 4) + r));
            const uint2 rw = make_uint2(lo, hi);
            uint32_t e = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int d = byte8(cw, i) - byte8(rw, i);
                e += (uint32_t)(d * d);
            }
            ssd = e;
        }
    }
    __syncwarp();
    return cbp;
}

/* frame-end denoise update by the session's last warp (mbgpu_kernels.cuh:478-503) */
__device__ __forceinline__ void denoise_frame_end(h261b_denoise_dev_t *dn, int lane)
{
    int32_t cnt0 = 0, cnt1 = 0;
    if (lane == 0) {
        cnt0 = atomicExch(&dn->count[0], 0);
        cnt1 = atomicExch(&dn->count[1], 0);
    }
    cnt0 = __shfl_sync(FULL, cnt0, 0);
    cnt1 = __shfl_sync(FULL, cnt1, 0);
    for (int p = lane; p < 64; p += 32) {
        const int32_t n1 = atomicExch(&dn->noise[1][p], 0);
        const int32_t n0 = atomicExch(&dn->noise[0][p], 0);
        const int u = p & 7, v = p >> 3;
        /* the reference keeps Int32 offsets and loads them as UInt16 */
        dn->offset[1][u][v] = (uint16_t)((cnt1 * dn->denoise + n1 / 2) / (n1 + 1));
        dn->offset[0][u][v] = (uint16_t)((cnt0 * dn->denoise + n0 / 2) / (n0 + 1));
    }
    __threadfence();
    if (lane == 0)
        atomicExch(&dn->ticket, 0u);
}

/* publish a warp's statistics for a run of n MBs of one session and type;
 * the publication that completes the session's frame updates the offsets */
__device__ __forceinline__ void publish_run(const h261b_session_dev_t &S, int t, int n, const int32_t colsum[8],
                                            int lane)
{
    h261b_denoise_dev_t *dn = S.dn;
    if (lane < 8) {
#pragma unroll
        for (int v = 0; v < 8; v++)
            if (colsum[v])
                atomicAdd(&dn->noise[t][v * 8 + lane], colsum[v]);
    }
    if (lane == 0)
        atomicAdd(&dn->count[t], 6 * n);
    __threadfence();
    __syncwarp();
    uint32_t last = 0;
    if (lane == 0) {
        last = atomicAdd(&dn->ticket, (uint32_t)n) + (uint32_t)n == (uint32_t)(S.mbw * S.mbh) ? 1u : 0u;
        /* the run's levels and records are written and fenced: count its
         * MBs for the codes kernel */
        atomicAdd(const_cast<int32_t *>(&S.mbs_done), n);
    }
    last = __shfl_sync(FULL, last, 0);
    if (last) {
        __threadfence();
        denoise_frame_end(dn, lane);
    }
}

/* resident CTAs of 256 threads the register allocation must allow per SM */
#ifndef H261B_STEP_MIN_BLOCKS
#define H261B_STEP_MIN_BLOCKS 2
#endif
/* the search-only kernel keeps neither the transforms' registers nor the
 * transpose buffer, so more of its CTAs fit an SM */
#ifndef H261B_SEARCH_MIN_BLOCKS
#define H261B_SEARCH_MIN_BLOCKS 3
#endif

/* Work items are handed out in two parts.  Warp w first takes the static
 * run [w * chunk, (w + 1) * chunk) of the first total_warps * chunk items
 * (consecutive MBs of mostly one session: neighbouring windows hit in L1
 * and the denoise statistics publish once per run).  With a scheduler
 * (sched != nullptr, two zeroed counters) the remaining items are then
 * drawn one at a time from sched[0], so that warps which met cheaper MBs
 * take more of the tail; every warp makes exactly one fetch past the end,
 * and the last warp to finish (sched[1]) zeroes both counters for the next
 * launch.  Without a scheduler the static runs cover every item. */
/* FMAD: the arithmetic of the reference's default build; KIND: what the
 * launch does per MB; FULL_SEARCH: the exhaustive search instead of the
 * reference's; ABI: the launch may write the reference-layout outputs
 * (h261_macroblock_t records, ME results, stage-1 vectors) that only the
 * gpu_device.h boundary asks for.  Each launch runs the instantiation for
 * its flags (h261b_launch_step), so no launch carries code it never runs. */
template <int FMAD, int KIND, bool FULL_SEARCH, bool ABI>
__global__ void __launch_bounds__(256, KIND == KIND_SEARCH ? H261B_SEARCH_MIN_BLOCKS : H261B_STEP_MIN_BLOCKS)
    step_kernel(const h261b_session_dev_t *__restrict__ sessions, const uint32_t *__restrict__ work, int32_t n_work,
                int32_t chunk, int32_t phases_arg, int32_t *sched)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    /* the kernel after this one (the encode launch after a search launch,
     * or the bitstream kernel) may launch now; it waits for the whole grid
     * before it reads anything (griddepcontrol.wait) */
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    /* an encode launch reads the mode decisions of the search launch before
     * it: wait for that grid and its writes (a no-op when launched without
     * the programmatic dependency) */
    if (KIND == KIND_ENCODE)
        asm volatile("griddepcontrol.wait;" ::: "memory");
    const int phases = KIND == KIND_SEARCH   ? (H261B_PHASE_ME | H261B_PHASE_MD)
                       : KIND == KIND_ENCODE ? H261B_PHASE_ENCDEC
                       : KIND == KIND_FULL   ? (H261B_PHASE_ME | H261B_PHASE_MD | H261B_PHASE_ENCDEC)
                                             : phases_arg;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t warp_bytes = KIND == KIND_SEARCH ? kSearchWarpBytes : sizeof(WarpSmem);
    unsigned char *mine = smem_raw + warp * warp_bytes;
    uint32_t *wbuf = reinterpret_cast<uint32_t *>(mine);
    float(*tb)[72] = reinterpret_cast<WarpSmem *>(mine)->t;   /* not used by KIND_SEARCH */
    /* bulk staging: the two buffers' barriers; per buffer, the parity of
     * its next phase, whether its current staging used the barrier, and
     * whether a wait on it gave up.  A barrier whose wait gave up is not
     * armed again (its phase may never complete): that buffer falls back to
     * cp.async staging, and at the end the warp waits once more, bounded,
     * for the copies of the phase that gave up. */
    uint64_t *bars = (phases_arg & H261B_STAGE_BULK) ? reinterpret_cast<WarpSmem *>(mine)->bar : nullptr;
    uint32_t parity = 0, bulk_used = 0, stuck = 0;
#ifdef H261B_DEBUG_CHECKS
    /* checking build only: the warp's first bulk staging announces 16 bytes
     * more than its copies bring, so that its wait runs out (the test of the
     * bounded wait and of h261b_stage_status) */
    uint32_t short_first = (phases_arg & H261B_STAGE_SHORT) ? 16u : 0u;
#else
    const uint32_t short_first = 0u;
#endif
    if (bars) {
        if (lane == 0) {
            mbar_init(&bars[0]);
            mbar_init(&bars[1]);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
        __syncwarp();
    }
    const int warps = blockDim.x >> 5;
    const int total_warps = gridDim.x * warps;
    const int n_static = sched ? min(n_work, total_warps * chunk) : n_work;
    int static_next = (blockIdx.x * warps + warp) * chunk;
    const int static_end = min(static_next + chunk, n_static);
    /* the warp's next work item (n_work when it has none left): a static
     * index, or a draw from the scheduler while the static run lasts */
    auto next_item = [&]() -> int {
        if (static_next < static_end)
            return static_next++;
        if (!sched)
            return n_work;
        int v = 0;
        if (lane == 0)
            v = n_static + atomicAdd(&sched[0], 1);
        return min(__shfl_sync(FULL, v, 0), n_work);
    };
    const bool want_enc = (phases & H261B_PHASE_ENCDEC) != 0;
    /* start the copies of a work item's inputs into buffer k: the whole
     * search window, or for an encode launch only the 16 window rows its
     * prediction block covers (none for an intra MB) */
    auto stage_item = [&](int k, uint32_t it) {
        const h261b_session_dev_t &N = sessions[it >> 12];
        const int nmb = (int)(it & 0xFFFu), nmby = nmb / N.mbw;
        uint64_t *bar = (bars && !((stuck >> k) & 1u)) ? &bars[k] : nullptr;
        const uint32_t extra = bar ? short_first : 0u;
        if (bar) {
            bulk_used |= 1u << k;
#ifdef H261B_DEBUG_CHECKS
            short_first = 0u;
#endif
        } else {
            bulk_used &= ~(1u << k);
        }
        if (KIND == KIND_ENCODE) {
            const h261_mb_mode_decision_t &d = N.md_in[nmb];
            const bool inter = d.i_mb_type != H261B_MB_TYPE_INTRA;
            stage_mb(wbuf, k, N, nmb - nmby * N.mbw, nmby, lane, 15 + d.i_mv_y, inter ? 16 : 0, bar, extra);
        } else {
            stage_mb(wbuf, k, N, nmb - nmby * N.mbw, nmby, lane, 0, WIN_ROWS, bar, extra);
        }
    };

    int g = next_item();
    uint32_t item = g < n_work ? work[g] : 0u;
    if (g < n_work) {
        stage_item(0, item);
        cp_async_commit();
    }
    /* the item after g, known one MB ahead of its staging */
    int gn = g < n_work ? next_item() : n_work;
    uint32_t nitem = gn < n_work ? work[gn] : 0u;

    int run_s = -1, run_t = 0, run_n = 0;
    int32_t colsum[8];
#pragma unroll
    for (int v = 0; v < 8; v++)
        colsum[v] = 0;

    for (int cur = 0; g < n_work; cur ^= 1) {
        const int gnn = gn < n_work ? next_item() : n_work;
        const uint32_t nnitem = gnn < n_work ? work[gnn] : 0u;
        if (gn < n_work) {
            stage_item(cur ^ 1, nitem);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        if ((bulk_used >> cur) & 1u) {
            /* a wait that gives up is counted; the buffer's barrier is not
             * used again, so no arrival meets a phase that never ended */
            if (!__all_sync(FULL, mbar_wait_bounded(&bars[cur], (parity >> cur) & 1u, lane)))
                stuck |= 1u << cur;
            else
                parity ^= 1u << cur;
        }
        __syncwarp();

        const int sidx = (int)(item >> 12);
        const h261b_session_dev_t &S = sessions[sidx];
        const int mb = (int)(item & 0xFFFu);
        if (!H261B_CHECK(mb < S.mbw * S.mbh, CHK_WORK_ITEM, (int)item)) {
            /* an item past its picture: nothing of it is read or written */
            __syncwarp();
            g = gn;
            item = nitem;
            gn = gnn;
            nitem = nnitem;
            continue;
        }
        const int mby = mb / S.mbw, mbx = mb - mby * S.mbw;
        const StageBuf b = stage_view(wbuf, cur);
        const bool do_me = (phases & H261B_PHASE_ME) && !S.skip_search;

        me_gpu_mb_t me;
        me.i_intra_cost = me.i_zero_cost = me.i_16x16_cost = me.i_16x16_filter_cost = 0;
        me.s_16x16_mv.i8_mx = me.s_16x16_mv.i8_my = 0;
        int8_t s1x = 0, s1y = 0;
        if (do_me) {
            /* the launch's search mode is the session's (checking build) */
            (void)H261B_CHECK(S.me_mode == (FULL_SEARCH ? 1 : 0), CHK_WORK_ITEM, S.me_mode);
            motion_estimate<FULL_SEARCH>(b, S, mbx, mby, lane, me, s1x, s1y);
            if (ABI && lane == 0) {
                if (S.me_out)
                    S.me_out[mb] = me;
                if (S.stage1_out) {
                    S.stage1_out[mb].i8_mx = s1x;
                    S.stage1_out[mb].i8_my = s1y;
                }
            }
        }

        MbDecision m;
        if (phases & H261B_PHASE_MD) {
            if (!do_me) {
                /* intra picture without search: only the intra cost matters */
                int32_t d[16];
                const int sb = lane & 15;
#pragma unroll
                for (int iy = 0; iy < 4; iy++) {
                    const uint32_t cw = *b.cur((sb >> 2) * 4 + iy, sb & 3);
#pragma unroll
                    for (int ix = 0; ix < 4; ix++)
                        d[iy * 4 + ix] = (int32_t)((cw >> (8 * ix)) & 0xFFu);
                }
                const int32_t v = satd4x4(d);
                me.i_intra_cost = (int32_t)__reduce_add_sync(FULL, lane < 16 ? (uint32_t)v : 0u);
            }
            m = mode_decide(me, S.frame_type);
            if (lane == 0 && S.rc)
                atomicAdd(&S.rc->cost_sum, m.cost);   /* the rate control's picture cost */
            if (lane == 0 && S.md_out) {
                h261_mb_mode_decision_t o;
                o.i_cost = m.cost;
                o.i_quantiser_adjust = 0;
                o.i_mb_type = m.type;
                o.i_mb_flags = m.flags;
                o.i_mv_x = m.mvx;
                o.i_mv_y = m.mvy;
                S.md_out[mb] = o;
            }
        } else if (S.md_in) {
            const h261_mb_mode_decision_t &d = S.md_in[mb];
            m.type = d.i_mb_type;
            m.flags = d.i_mb_flags;
            m.mvx = d.i_mv_x;
            m.mvy = d.i_mv_y;
            m.cost = d.i_cost;
        } else {
            m.type = H261B_MB_TYPE_INTRA;
            m.flags = m.mvx = m.mvy = m.cost = 0;
        }

        /* a rate-controlled session is encoded by a second launch, once its
         * picture QUANT is known */
        if (want_enc && !(S.rc && (phases & H261B_PHASE_MD))) {
            const int t = m.type == H261B_MB_TYPE_INTRA ? 0 : 1;
            if (run_n > 0 && (sidx != run_s || t != run_t)) {
                publish_run(sessions[run_s], run_t, run_n, colsum, lane);
                run_n = 0;
#pragma unroll
                for (int v = 0; v < 8; v++)
                    colsum[v] = 0;
            }
            run_s = sidx;
            run_t = t;
            int quant = S.rc ? S.rc->picture_quant : S.quant;
            if (S.md_in && !(phases & H261B_PHASE_MD))
                quant += S.md_in[mb].i_quantiser_adjust;
            quant = min(31, max(1, quant)); /* gpu_device.cu:625-627 */
            /* the luma pass, then the chroma pass: one copy of the pass's
             * code run twice (two inlined copies miss the instruction cache
             * more) */
            uint32_t ssd_l = 0, ssd_c = 0, cbp = 0;
#pragma unroll 1
            for (int pass = 0; pass < 2; pass++) {
                uint32_t e = 0;
                cbp |= encdec_pass<FMAD, ABI>(tb, b, S, mb, mbx, mby, m, quant, pass == 0, lane, colsum, e);
                if (pass == 0)
                    ssd_l = e;
                else
                    ssd_c = e;
            }
            if (S.ssd_out) {
                const uint32_t ey = __reduce_add_sync(FULL, ssd_l);
                const uint32_t ecb = __reduce_add_sync(FULL, lane < 8 ? ssd_c : 0u);
                const uint32_t ecr = __reduce_add_sync(FULL, lane >= 8 && lane < 16 ? ssd_c : 0u);
                if (lane == 0) {
                    atomicAdd(&S.ssd_out[0], (unsigned long long)ey);
                    atomicAdd(&S.ssd_out[1], (unsigned long long)ecb);
                    atomicAdd(&S.ssd_out[2], (unsigned long long)ecr);
                }
            }
            run_n++;

            const int flags = m.flags | (cbp ? H261B_MB_COEFF : 0);
            if (lane == 0) {
                if (ABI && S.abi_out) {
                    h261_macroblock_t *o = &S.abi_out[mb];
                    o->i_macroblock_address = 0;
                    o->i_macroblock_type = m.type;
                    o->i_macroblock_type_flags = flags;
                    o->i_macroblock_quant = quant;
                    o->rgi_mv[0] = m.mvx;
                    o->rgi_mv[1] = m.mvy;
                    o->i_coded_block_pattern = (int32_t)cbp;
                    o->i_mb_x = mbx * 16;
                    o->i_mb_y = mby * 16;
                }
                if (S.info_out) {
                    h261b_mb_info_t inf;
                    inf.type = (int16_t)m.type;
                    inf.flags = (int16_t)flags;
                    inf.quant = (int8_t)quant;
                    inf.cbp = (int8_t)cbp;
                    inf.mvx = (int8_t)m.mvx;
                    inf.mvy = (int8_t)m.mvy;
                    inf.cost = m.cost;
                    inf.coef_bits = 0;   /* the bitstream kernels fill it in */
                    S.info_out[mb] = inf;
                }
            }
        }
        __syncwarp(); /* this buffer may be refilled from the next iteration on */
        g = gn;
        item = nitem;
        gn = gnn;
        nitem = nnitem;
    }
    if (want_enc && run_n > 0)
        publish_run(sessions[run_s], run_t, run_n, colsum, lane);
    if (bars) {
        for (int k = 0; k < 2; k++) {
            /* the copies of a phase whose wait gave up may still be landing:
             * wait for them once more, bounded, before the CTA's shared
             * memory goes; a barrier left in a phase is not invalidated */
            bool done = true;
            if ((stuck >> k) & 1u)
                done = __all_sync(FULL, mbar_wait_bounded(&bars[k], (parity >> k) & 1u, lane));
            if (done && lane == 0)
                mbar_inval(&bars[k]);
        }
    }
    if (sched && lane == 0) {
        __threadfence();
        if (atomicAdd(&sched[1], 1) == total_warps - 1) {
            atomicExch(&sched[0], 0);
            atomicExch(&sched[1], 0);
        }
    }
}

} // namespace

extern "C" int h261b_debug_check_status(int32_t *enabled, int64_t *violations, int32_t *first_site,
                                        int32_t *first_value)
{
    if (!enabled || !violations || !first_site || !first_value)
        return H261B_ERR_ARG;
    *violations = 0;
    *first_site = *first_value = 0;
#ifdef H261B_DEBUG_CHECKS
    *enabled = 1;
    unsigned long long n = 0;
    int first[2] = { 0, 0 };
    const unsigned long long zero = 0;
    if (cudaMemcpyFromSymbol(&n, g_check_count, sizeof(n)) != cudaSuccess ||
        cudaMemcpyFromSymbol(first, g_check_first, sizeof(first)) != cudaSuccess ||
        cudaMemcpyToSymbol(g_check_count, &zero, sizeof(zero)) != cudaSuccess)
        return H261B_ERR_CUDA;
    *violations = (int64_t)n;
    *first_site = first[0];
    *first_value = first[1];
#else
    *enabled = 0;
#endif
    return H261B_OK;
}

extern "C" int h261b_stage_status(int64_t *timeouts)
{
    if (!timeouts)
        return H261B_ERR_ARG;
    unsigned int n = 0;
    const unsigned int zero = 0;
    if (cudaMemcpyFromSymbol(&n, g_stage_timeouts, sizeof(n)) != cudaSuccess ||
        cudaMemcpyToSymbol(g_stage_timeouts, &zero, sizeof(zero)) != cudaSuccess)
        return H261B_ERR_CUDA;
    *timeouts = (int64_t)n;
    return H261B_OK;
}

extern "C" int h261b_set_quant_table(void)
{
    /* f_inv_quant = 1.0 / ( float ) ( i_quant * 2 ) (mbgpu_kernels.cuh:685),
     * evaluated on the host in IEEE double and rounded to float */
    float tab[32];
    tab[0] = 0.0f;
    for (int q = 1; q < 32; q++)
        tab[q] = (float)(1.0 / (double)(float)(q * 2));
    return (int)cudaMemcpyToSymbol(c_inv_quant, tab, sizeof(tab));
}

namespace {

using StepFn = void (*)(const h261b_session_dev_t *, const uint32_t *, int32_t, int32_t, int32_t, int32_t *);

/* the instantiation of a launch's flags: the encode kind has no search and
 * writes no reference-layout output, the search kind no encode output */
template <int FMAD>
StepFn step_fn_of(int kind, int full, int abi)
{
    if (kind == KIND_ENCODE)
        return step_kernel<FMAD, KIND_ENCODE, false, false>;
    if (kind == KIND_SEARCH)
        return full ? step_kernel<FMAD, KIND_SEARCH, true, false> : step_kernel<FMAD, KIND_SEARCH, false, false>;
    if (abi)
        return full ? step_kernel<FMAD, KIND_FUSED, true, true> : step_kernel<FMAD, KIND_FUSED, false, true>;
    if (kind == KIND_FULL)
        return full ? step_kernel<FMAD, KIND_FULL, true, false> : step_kernel<FMAD, KIND_FULL, false, false>;
    return full ? step_kernel<FMAD, KIND_FUSED, true, false> : step_kernel<FMAD, KIND_FUSED, false, false>;
}

StepFn step_fn(int fmad, int kind, int full, int abi)
{
    return fmad ? step_fn_of<1>(kind, full, abi) : step_fn_of<0>(kind, full, abi);
}

} // namespace

extern "C" int h261b_launch_step(const h261b_session_dev_t *sessions_dev, const uint32_t *work_dev,
                                 int32_t n_work, int32_t phases, int32_t warps_per_cta, int32_t max_ctas,
                                 int32_t *sched_dev, void *stream)
{
    if (n_work <= 0)
        return 0;
    if (warps_per_cta < 1 || warps_per_cta > 8)
        return (int)cudaErrorInvalidValue;
    const int fmad = (phases >> 8) & 1;
    int kind = (phases >> H261B_KIND_SHIFT) & 3;
    /* a fused launch of every phase runs the kernel compiled for exactly that */
    const int all_phases = H261B_PHASE_ME | H261B_PHASE_MD | H261B_PHASE_ENCDEC;
    if (kind == KIND_FUSED && (phases & all_phases) == all_phases)
        kind = KIND_FULL;
    const int full = (phases & H261B_LAUNCH_ME_FULL) ? 1 : 0, abi = (phases & H261B_ABI_OUT) ? 1 : 0;
    const bool pdl = (phases & H261B_LAUNCH_PDL) != 0;
    const int tail_code = (phases >> H261B_TAIL_SHIFT) & 15;
    if (kind > KIND_FULL)
        return (int)cudaErrorInvalidValue;
    const int ph = phases & (0xFF | H261B_STAGE_BULK | H261B_STAGE_SHORT);
    const int threads = warps_per_cta * 32;
    const size_t warp_bytes = kind == KIND_SEARCH ? kSearchWarpBytes : sizeof(WarpSmem);
    const size_t smem = warp_bytes * (size_t)warps_per_cta;
    const StepFn fn = step_fn(fmad, kind, full, abi);
    static std::mutex mu;
    static int sms[64], resident[64][2][4][2][2][9];
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess || dev < 0 || dev >= 64)
        return (int)(err != cudaSuccess ? err : cudaErrorInvalidDevice);
    int per_sm = 0, nsm = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!sms[dev]) {
            if ((err = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
                return (int)err;
            const int max_smem = (int)(sizeof(WarpSmem) * 8);
            for (int f = 0; f < 2; f++)
                for (int k = 0; k < 4; k++)
                    for (int x = 0; x < 4; x++)
                        if ((err = cudaFuncSetAttribute(step_fn(f, k, x & 1, x >> 1),
                                                        cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem)) !=
                            cudaSuccess)
                            return (int)err;
        }
        int &r = resident[dev][fmad][kind][full][abi][warps_per_cta];
        if (!r) {
            err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, fn, threads, smem);
            if (err != cudaSuccess)
                return (int)err;
            r = r < 1 ? 1 : r;
        }
        per_sm = r;
        nsm = sms[dev];
    }
    /* one wave of resident CTAs */
    int ctas = max_ctas > 0 ? max_ctas : nsm * per_sm;
    int chunk;
    if (sched_dev) {
        /* static runs of all but about `tail` items per warp, the rest drawn
         * from the scheduler (tail_code: tail + 1, 0 for the default 2) */
        const int tail = tail_code ? tail_code - 1 : 2;
        ctas = (int)std::min<long long>(ctas, (n_work + warps_per_cta - 1) / warps_per_cta);
        const long long total_warps = (long long)ctas * warps_per_cta;
        chunk = (int)std::max<long long>(0, n_work / total_warps - tail);
    } else {
        /* contiguous runs covering every item */
        const long long total_warps = (long long)ctas * warps_per_cta;
        chunk = (int)((n_work + total_warps - 1) / total_warps);
        ctas = (n_work + chunk * warps_per_cta - 1) / (chunk * warps_per_cta);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return (int)cudaLaunchKernelEx(&cfg, fn, sessions_dev, work_dev, n_work, chunk, ph, sched_dev);
}

/* ------------------------------------------------ SAD primitive peak */

namespace {

/* the motion search's inner step, on registers: one funnel shift and one
 * 4-pixel SAD per word, eight independent chains per thread */
__global__ void __launch_bounds__(256) sad_peak_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                       int iters)
{
    uint32_t c[8], r[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        c[i] = in[(threadIdx.x + i) & 255];
        r[i] = in[(threadIdx.x * 7 + i) & 255];
    }
    uint32_t acc = 0;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            acc = sad4(c[i], r[i], acc);
            r[i] = __funnelshift_r(r[i], r[(i + 1) & 7], 8);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

} // namespace

extern "C" int h261b_measure_sad_peak(int32_t device, double *absdiff_per_s)
{
    if (!absdiff_per_s)
        return -1;
    int sms = 0;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return -2;
    const int blocks = sms * 8, threads = 256, iters = 2048;
    uint32_t *in = nullptr, *out = nullptr;
    uint32_t h[256];
    for (int i = 0; i < 256; i++)
        h[i] = (uint32_t)i * 2654435761u;
    cudaEvent_t a, b;
    float ms = 0.f;
    int rc = -2;
    if (cudaMalloc(&in, sizeof(h)) == cudaSuccess && cudaMalloc(&out, sizeof(uint32_t) * blocks * threads) == cudaSuccess &&
        cudaMemcpy(in, h, sizeof(h), cudaMemcpyHostToDevice) == cudaSuccess && cudaEventCreate(&a) == cudaSuccess &&
        cudaEventCreate(&b) == cudaSuccess) {
        sad_peak_kernel<<<blocks, threads>>>(in, out, 64);
        cudaEventRecord(a);
        sad_peak_kernel<<<blocks, threads>>>(in, out, iters);
        cudaEventRecord(b);
        if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess && ms > 0.f) {
            *absdiff_per_s = (double)blocks * threads * iters * 8 * 4 / (ms * 1e-3);
            rc = 0;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    cudaFree(in);
    cudaFree(out);
    return rc;
}

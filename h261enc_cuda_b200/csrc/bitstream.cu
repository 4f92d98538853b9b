/*
 * bitstream.cu -- H.261 bitstream writer on the device.
 *
 * Writes each picture in the syntax of the reference's host writers
 * (src/h261_picture.c:115-148, src/h261_gob.c:6-199,
 * src/h261_macroblock.c:5-262), byte for byte: picture header, GOBs in the
 * QCIF / CIF order, macroblocks with MBA, MTYPE, MQUANT, MVD, CBP, TCOEFF
 * and EOB, the last byte zero-padded (src/h261_bitstream.c:64-76).
 *
 * Three launches; the macroblock-parallel ones take contiguous ranges of the
 * step's work list, one warp per macroblock, so that every SM takes part
 * whatever the mix of picture sizes.  Kernel boundaries order layout and
 * pack; codes starts on a picture as soon as the encode launch has counted
 * all of its MBs done:
 *
 *   codes   the macroblock's coded blocks, four at a time with eight lanes
 *           per block (lane j holds positions 8j..8j+7 of the transmission
 *           order): runs from the block's nonzero mask, TCOEFF / escape /
 *           DC / EOB codes, a scan for their offsets, assembled in shared
 *           memory and stored as the MB's coefficient bit string.
 *   layout  one CTA per picture, a warp per GOB with a lane per macroblock:
 *           the address increments, quantiser in force and vector
 *           predictors come from ballots over the GOB's coded / COEFF / MC
 *           flags; MB sizes, a scan over the GOB and one over the GOBs give
 *           every macroblock's position; the picture is cleared and gets its
 *           picture and GOB headers.
 *   pack    every coded macroblock (one per half-warp) writes its header and
 *           shifts its bit string into place; a macroblock's first and last
 *           word can be shared with its neighbours and are ORed in with
 *           atomics.  Half-warps count the MBs they finish per picture; the
 *           CTA whose count completes a picture copies it into the host
 *           arena (mapped pinned memory) at the offset layout drew with one
 *           atomic, and writes its record.
 *
 * All three are programmatic dependent launches: the kernel before each
 * one (the encode kernel, codes, layout) lets it launch as soon as its own
 * CTAs are running, so each launch's latency overlaps the kernel before it.
 * Layout and pack wait (griddepcontrol.wait) for the whole previous grid
 * and its memory before they read what it wrote.  Codes instead waits per
 * picture, bounded, on the count the encode warps release after their
 * writes (session_dev_t.mbs_done), so that it codes the pictures finished
 * early while the encode launch's last MBs still run on other SMs; it
 * starts only once every encode CTA is running, and no encode CTA waits on
 * it.  The events that mark the
 * encode kernel's end are recorded on a side stream, so that nothing sits
 * between the encode kernel and codes in the stream.
 */
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "h261b_device.h"

namespace {

/* programmatic dependent launch: allow the next kernel in the stream to
 * launch now / wait until the previous kernel has completed and its
 * writes are visible (both no-ops for a kernel launched without the
 * attribute) */
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

} // namespace
#include "ratectrl_dev.h"
#include "vlc_coder.h"

namespace h261b {
namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr int VLC_WARPS = 8;
constexpr int VLC_THREADS = VLC_WARPS * 32;
constexpr int MB_WORDS = H261B_VLC_MB_WORDS;
/* header bits of one macroblock at most: MBA 11, MTYPE 10, MQUANT 5,
 * MVD 2 x 11, CBP 9 */
constexpr int MB_HDR_MAX = 57;

struct CodesSmem {
    alignas(16) int8_t blk[VLC_WARPS][4][64];   /* column-major levels of the blocks in flight */
    alignas(16) uint32_t stage[VLC_WARPS][MB_WORDS];
    uint16_t tc[27][16];
};

__device__ __forceinline__ uint32_t bswap(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

/* the same on a picture in device memory, whose words hold the stream's
 * bytes in order (byte-swapped) */
__device__ __forceinline__ void put_bits_pic(uint32_t *w, int64_t words, int64_t pos, uint32_t code, int len,
                                             int &oob)
{
    if (len <= 0)
        return;
    if (pos < 0 || pos + len > words * 32) {
        oob = 1;
        return;
    }
    const int64_t word = pos >> 5;
    const int end = (int)(pos & 31) + len;
    if (end <= 32) {
        atomicOr(&w[word], bswap(code << (32 - end)));
    } else {
        atomicOr(&w[word], bswap(code >> (end - 32)));
        atomicOr(&w[word + 1], bswap(code << (64 - end)));
    }
}

__device__ __forceinline__ int wrap_mvd(int d) { return ((d + 16) & 31) - 16; }

__device__ __forceinline__ void mvd_code(int w, uint32_t &code, int &len)
{
    const uint16_t e = c_vlc_mvd[w < 0 ? -w : w];
    len = e >> 8;
    code = (uint32_t)(e & 0xFF) - (w > 0 ? 1u : 0u);
}

/* MTYPE of a coded macroblock (src/h261_macroblock.c:94-194); -1 for a
 * combination the syntax has no code for */
__device__ __forceinline__ int mtype_of(int type, int flags, int mq)
{
    if (type == H261B_MB_TYPE_INTRA)
        return mq ? MT_INTRA_MQ : MT_INTRA;
    switch (flags) {
    case 1: return mq ? -1 : MT_MC;
    case 3: return mq ? -1 : MT_MC_FIL;
    case 4: return mq ? MT_INTER_MQ : MT_INTER;
    case 5: return mq ? MT_MC_CBP_MQ : MT_MC_CBP;
    case 7: return mq ? MT_MC_FIL_CBP_MQ : MT_MC_FIL_CBP;
    default: return -1;
    }
}

/* header plan: address increment, MTYPE, MQUANT flag, wrapped MVDs */
__device__ __forceinline__ uint32_t plan_pack(int addr, int mtype, int mq, int dx, int dy)
{
    return (uint32_t)addr | ((uint32_t)mtype << 6) | ((uint32_t)mq << 10) | ((uint32_t)(dx + 16) << 11) |
           ((uint32_t)(dy + 16) << 16);
}

/* coded blocks of a record: all six of an intra MB, the CBP of an inter MB
 * with COEFF, else none; bit (5 - b) = block b */
__device__ __forceinline__ int coded_blocks(const h261b_mb_info_t &r)
{
    if (r.type == H261B_MB_TYPE_INTRA)
        return 63;
    return (r.flags & H261B_MB_COEFF) ? (r.cbp & 63) : 0;
}

/* header of one macroblock from its record and its GOB neighbours' state:
 * plan and size in bits; bad when the syntax has no code for it */
struct MbHeader {
    uint32_t plan;
    int bits;
    bool bad;
};

__device__ __forceinline__ MbHeader mb_header(const h261b_mb_info_t &r, int addr, int q_state, bool mv_ok, int pmx,
                                              int pmy)
{
    const bool intra = r.type == H261B_MB_TYPE_INTRA;
    const int mq = intra ? (r.quant != q_state) : (r.quant != q_state && (r.flags & H261B_MB_COEFF));
    const int mt = mtype_of(r.type, r.flags, mq);
    const int dx = wrap_mvd(r.mvx - (mv_ok ? pmx : 0)), dy = wrap_mvd(r.mvy - (mv_ok ? pmy : 0));
    int h = (c_vlc_mba[addr] >> 8) + (mt >= 0 ? c_vlc_mtype_len[mt] : 0) + (mq ? 5 : 0);
    if (!intra && (r.flags & H261B_MB_MC))
        h += (c_vlc_mvd[dx < 0 ? -dx : dx] >> 8) + (c_vlc_mvd[dy < 0 ? -dy : dy] >> 8);
    const int cbp = coded_blocks(r);
    if (!intra && cbp)
        h += c_vlc_cbp[cbp] >> 8;
    MbHeader o;
    o.plan = plan_pack(addr, mt < 0 ? 0 : mt, mq, dx, dy);
    o.bits = h;
    o.bad = mt < 0 || (!intra && (r.flags & H261B_MB_COEFF) && cbp == 0);
    return o;
}

/* the range of the work list a warp takes: contiguous, so that its
 * macroblocks mostly share a picture */
__device__ __forceinline__ void warp_range(int32_t n_work, int &lo, int &hi)
{
    const int nwarps = gridDim.x * VLC_WARPS;
    const int w = blockIdx.x * VLC_WARPS + (threadIdx.x >> 5);
    const int chunk = (n_work + nwarps - 1) / nwarps;
    lo = min(w * chunk, n_work);
    hi = min(lo + chunk, n_work);
}

/* Waits (lane 0) until an encoding launch has finished every MB of a
 * picture: an acquire load of the count the encode warps add to after
 * fencing their levels and records.  The codes kernel is a programmatic
 * dependent of that launch, so it starts once every encode CTA is running,
 * and no encode CTA waits on it: the count completes.  The wait is bounded
 * all the same (bound_ns of globaltimer, or 2^22 polls); false when it
 * gives up. */
__device__ __forceinline__ bool wait_picture_encoded(const int32_t *done, int32_t nmb, uint64_t bound_ns)
{
    uint64_t t0 = 0;
    for (int it = 0; it < (1 << 22); it++) {
        int32_t v;
        asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(done) : "memory");
        if (v >= nmb)
            return true;
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (it == 0)
            t0 = t;
        else if (t - t0 > bound_ns)
            return false;
        __nanosleep(200);
    }
    return false;
}

/* work items a codes warp takes per draw: an intra MB codes six blocks, a
 * skipped inter MB none, so a static split leaves SMs idle at the end */
constexpr int CODES_DRAW = 2;

/* ---- codes: each macroblock's coefficient bit string */
/* extra > 0 (the checking build's test of the bounded wait): wait for
 * that many MBs more than a picture has, for 2 ms at most */
__global__ void __launch_bounds__(VLC_THREADS) codes_kernel(const h261b_session_dev_t *sessions,
                                                            const uint32_t *work, int32_t n_work,
                                                            h261b_step_dev_t *step, int32_t extra)
{
    __shared__ CodesSmem sm;
    pdl_launch_dependents();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    load_tcoeff_table(sm.tc, tid, VLC_THREADS);
    uint32_t zz0, zz1;
    zigzag_lane(lane, zz0, zz1);
    uint32_t *stage = sm.stage[warp];
    for (int i = lane; i < MB_WORDS; i += 32)
        stage[i] = 0u;
    /* no wait for the whole encode grid: each picture is coded once its
     * MBs are (the encode launch's tail overlaps this kernel) */
    __syncthreads();

    const int slot = lane >> 3, j = lane & 7;
    /* the warp draws CODES_DRAW items at a time from the step's counter
     * (zeroed by the step's descriptor upload) until the list is done */
    int lo = 0, hi = 0;
    int ready = -1;         /* the last session seen complete             */
    bool failed = false;    /* a wait gave up: code nothing more          */
    for (int w = 0;; w++) {
        if (w >= hi) {
            int d = 0;
            if (lane == 0)
                d = (int)atomicAdd(&step->codes_next, (uint32_t)CODES_DRAW);
            lo = __shfl_sync(FULL, d, 0);
            if (lo >= n_work)
                break;
            hi = min(lo + CODES_DRAW, n_work);
            w = lo;
        }
        const uint32_t item = work[w];
        const int sidx = (int)(item >> 12);
        const h261b_session_dev_t &S = sessions[sidx];
        if (!S.bits_out || failed)
            continue;
        if (sidx != ready) {
            int ok = 0;
            if (lane == 0)
                ok = wait_picture_encoded(&S.mbs_done, S.mbw * S.mbh + extra,
                                          extra ? 2000000ull : 200000000ull) ? 1 : 0;
            __syncwarp();   /* orders lane 0's acquire before every lane's reads */
            if (!__shfl_sync(FULL, ok, 0)) {
                if (lane == 0)
                    atomicExch(&step->codes_failed, 1u);
                failed = true;
                continue;
            }
            ready = sidx;
        }
        const int mb = (int)(item & 4095u);
        h261b_mb_info_t &rec = S.info_out[mb];
        const int cbp = coded_blocks(rec);
        const bool intra = rec.type == H261B_MB_TYPE_INTRA;
        /* block b is coded when bit b of `order` is set */
        const uint32_t order = __brev((uint32_t)cbp) >> 26;
        const int nb = __popc(order);

        int pos = 0, oob = 0;
        const int8_t *lv = S.level_out + (size_t)mb * 384;
        for (int r0 = 0; r0 < nb; r0 += 4) {
            const bool here = r0 + slot < nb;
            const int b = here ? (int)__fns(order, 0, r0 + slot + 1) : 0;
            if (here)
                *reinterpret_cast<uint2 *>(&sm.blk[warp][slot][j * 8]) =
                    *reinterpret_cast<const uint2 *>(lv + b * 64 + j * 8);
            __syncwarp();
            pos += code_block_group(sm.blk[warp][slot], here, intra, zz0, zz1, sm.tc, stage, MB_WORDS, pos, lane,
                                    oob);
            __syncwarp();
        }
        const int bits = store_mb_string(stage, S.vlc_scratch + (size_t)mb * MB_WORDS, pos, oob, lane);
        if (lane == 0)
            rec.coef_bits = bits;
    }
}

/* ---- layout: one CTA per picture, a warp per GOB (12 warps: all of a CIF
 * picture's GOBs at once); it also draws the picture's place in the host
 * arena, so that whichever CTA finishes the picture can copy it */
constexpr int LAYOUT_THREADS = 12 * 32;

__global__ void __launch_bounds__(LAYOUT_THREADS) layout_kernel(const h261b_session_dev_t *sessions,
                                                                h261b_step_dev_t *step, int64_t host_cap)
{
    pdl_launch_dependents();
    const h261b_session_dev_t &S = sessions[blockIdx.x];
    if (!S.bits_out)
        return;
    pdl_wait();   /* the codes kernel's MB sizes */
    __shared__ int32_t rel[396];       /* MB position within its GOB */
    __shared__ int32_t gob_bits[12];
    __shared__ int64_t gob_start[13];
    __shared__ int bad;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool cif = S.mbw == 22;
    const int ngob = cif ? 12 : 3, nmb = S.mbw * S.mbh;
    const int gq = S.rc ? S.rc->picture_quant : S.quant;
    const h261b_mb_info_t *info = S.info_out;
    if (tid == 0)
        bad = step->codes_failed ? 1 : 0;   /* some picture's strings are missing */
    __syncthreads();

    const int nwarps = blockDim.x >> 5;
    for (int g = warp; g < ngob; g += nwarps) {
        const int x0 = cif ? (g & 1) * 11 : 0, y0 = (cif ? g >> 1 : g) * 3;
        const int mi = (y0 + lane / 11) * S.mbw + x0 + lane % 11;
        const int m32 = (y0 + 2) * S.mbw + x0 + 10;
        const h261b_mb_info_t r = info[mi];
        const h261b_mb_info_t r32 = info[m32];
        const uint32_t C = __ballot_sync(FULL, r.flags != 0);
        const uint32_t K = __ballot_sync(FULL, (r.flags & H261B_MB_COEFF) != 0);
        const uint32_t M = __ballot_sync(FULL, (r.flags & H261B_MB_MC) != 0);
        const int pmx = __shfl_up_sync(FULL, (int)r.mvx, 1), pmy = __shfl_up_sync(FULL, (int)r.mvy, 1);
        const uint32_t below = (1u << lane) - 1u, kb = K & below, cb = C & below;
        /* quantiser in force: the last COEFF macroblock before, else GQUANT */
        const int qv = __shfl_sync(FULL, (int)r.quant, kb ? 31 - __clz((int)kb) : lane);
        const int qv32 = __shfl_sync(FULL, (int)r.quant, K ? 31 - __clz((int)K) : 0);
        const int mvx31 = __shfl_sync(FULL, (int)r.mvx, 31), mvy31 = __shfl_sync(FULL, (int)r.mvy, 31);

        int bits = 0, bits32 = 0, b = 0;
        if (r.flags != 0) {
            const int addr = cb ? lane - (31 - __clz((int)cb)) : lane + 1;
            /* the predictor: the previous MB of the same MB row, coded with MC */
            const bool ok = lane > 0 && lane % 11 != 0 && ((M >> (lane - 1)) & 1u);
            const MbHeader hd = mb_header(r, addr, kb ? qv : gq, ok, pmx, pmy);
            b |= hd.bad || r.coef_bits < 0 || r.coef_bits > MB_WORDS * 32;
            bits = hd.bits + r.coef_bits;
            S.vlc_plan[mi] = hd.plan;
        }
        if (r32.flags != 0) {
            /* the 33rd macroblock, by every lane */
            const int addr = C ? 32 - (31 - __clz((int)C)) : 33;
            const MbHeader hd = mb_header(r32, addr, K ? qv32 : gq, (M >> 31) & 1u, mvx31, mvy31);
            b |= hd.bad || r32.coef_bits < 0 || r32.coef_bits > MB_WORDS * 32;
            bits32 = hd.bits + r32.coef_bits;
            if (lane == 0)
                S.vlc_plan[m32] = hd.plan;
        }
        int incl = bits;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o)
                incl += t;
        }
        const int sum32 = __shfl_sync(FULL, incl, 31);
        rel[mi] = 26 + incl - bits;
        if (lane == 0) {
            rel[m32] = 26 + sum32;
            gob_bits[g] = 26 + sum32 + bits32;
        }
        if (__any_sync(FULL, b) && lane == 0)
            bad = 1;
    }
    __syncthreads();
    if (tid == 0) {
        int64_t at = 32;                    /* after PSC, TR, PTYPE, PEI */
        for (int g = 0; g < ngob; g++) {
            gob_start[g] = at;
            at += gob_bits[g];
        }
        gob_start[ngob] = at;
    }
    __syncthreads();
    const int64_t total = gob_start[ngob];
    const int64_t words = ((total + 127) / 128) * 4;   /* whole 16-byte units */
    const int status = bad ? H261B_BITS_BAD_RECORD : (words * 4 > S.bits_cap ? H261B_BITS_OVERFLOW : 0);
    if (status == 0) {
        for (int i = tid; i < nmb; i += (int)blockDim.x) {
            const int mbx = i % S.mbw, mby = i / S.mbw;
            const int g = cif ? (mby / 3) * 2 + mbx / 11 : mby / 3;
            S.vlc_pos[i] = (int32_t)(gob_start[g] + rel[i]);
        }
        for (int64_t i = tid; i < words; i += (int)blockDim.x)
            S.bits_out[i] = 0u;
    }
    __syncthreads();
    int oob = 0;
    if (status == 0) {
        if (tid == 0) {
            /* PSC, TR, PTYPE (split 0, document camera 0, freeze release 1,
             * source format, HI_RES bit 1, spare 1), PEI 0 */
            const uint32_t ptype = (1u << 3) | ((cif ? 1u : 0u) << 2) | (1u << 1) | 1u;
            S.bits_out[0] = bswap((16u << 12) | ((uint32_t)(S.frame_num & 31) << 7) | (ptype << 1));
        }
        if (tid < ngob) {
            /* GOB header: GBSC, GN, GQUANT, GEI */
            const uint32_t number = cif ? (uint32_t)tid + 1u : 2u * (uint32_t)tid + 1u;
            put_bits_pic(S.bits_out, words, gob_start[tid], (1u << 10) | (number << 6) | ((uint32_t)gq << 1), 26,
                         oob);
        }
    }
    const int any_oob = __syncthreads_or(oob);
    if (tid == 0) {
        S.vlc_total[0] = (int32_t)total;
        S.vlc_total[1] = status != 0 ? status : (any_oob ? H261B_BITS_MISMATCH : 0);
        /* the picture's place in the host arena */
        int32_t off = -1;
        if (S.vlc_total[1] == 0 && host_cap > 0) {
            const uint32_t padded = (uint32_t)((((total + 7) >> 3) + 15) & ~15);
            const uint32_t a = atomicAdd(&step->host_used, padded);
            if ((int64_t)a + padded <= host_cap)
                off = (int32_t)a;
        }
        S.vlc_total[2] = off;
        S.vlc_total[3] = 0;   /* MBs the pack kernel has finished */
        /* the rate control learns the picture's size */
        if (S.rc && S.vlc_total[1] == 0)
            rc_update(*S.rc, S.frame_type, (int32_t)((total + 7) >> 3));
    }
}

/* ---- pack: headers and coefficient strings into the picture; the CTA
 * that finishes a picture's last MB then copies it into the host arena */
constexpr int PACK_DONE_MAX = 64;   /* pictures a CTA copies together at its end */

/* a finished picture into the host arena by threads t0, t0 + nt, ..., and
 * its record (bytes, offset, status, QUANT) by thread t0 */
__device__ __forceinline__ void copy_picture(const h261b_session_dev_t &S, uint8_t *host_arena, int t0, int nt)
{
    const int total = S.vlc_total[0];
    const int64_t words = ((int64_t)(total + 127) / 128) * 4;
    const int st = (total < 0 || words * 4 > S.bits_cap) ? H261B_BITS_OVERFLOW : S.vlc_total[1];
    const int off = st == 0 ? S.vlc_total[2] : -1;
    const int bytes = (total + 7) >> 3;
    const int units = ((bytes + 15) & ~15) / 16;
    if (t0 == 0)
        *S.pic_out = h261b_pic_info_t{ st == 0 ? bytes : 0, off, st, S.rc ? S.rc->picture_quant : S.quant };
    if (off < 0 || !host_arena)
        return;
    /* other SMs wrote the words: read them from L2 */
    const uint4 *s4 = reinterpret_cast<const uint4 *>(S.bits_out);
    uint4 *d4 = reinterpret_cast<uint4 *>(host_arena + off);
    for (int i = t0; i < units; i += nt)
        d4[i] = __ldcg(s4 + i);
}

__global__ void __launch_bounds__(VLC_THREADS) pack_kernel(const h261b_session_dev_t *sessions,
                                                           const uint32_t *work, int32_t n_work,
                                                           uint8_t *host_arena)
{
    __shared__ int done[PACK_DONE_MAX];
    __shared__ int n_done;
    pdl_launch_dependents();
    /* each half-warp packs every other MB of the warp's range, so that the
     * two MBs' chains of dependent loads overlap */
    const int lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
    const unsigned hmask = 0xFFFFu << (16 * half);
    if (threadIdx.x == 0)
        n_done = 0;
    __syncthreads();
    int lo, hi;
    warp_range(n_work, lo, hi);
    pdl_wait();   /* the layout kernel's positions */
    int run_s = -1, run_n = 0;
    /* the half-warp's finished MBs of picture run_s: published once it
     * moves on; the publication that completes the picture queues its copy */
    auto publish = [&]() {
        if (run_n == 0)
            return;
        const h261b_session_dev_t &P = sessions[run_s];
        __threadfence();   /* this lane's words before the count */
        __syncwarp(hmask);
        int k = -1;
        if (hl == 0 && atomicAdd(&P.vlc_total[3], run_n) + run_n == P.mbw * P.mbh) {
            k = atomicAdd(&n_done, 1);
            if (k < PACK_DONE_MAX)
                done[k] = run_s;
        }
        k = __shfl_sync(hmask, k, 16 * half);
        if (k >= PACK_DONE_MAX) {
            /* the CTA's list is full: this half-warp copies the picture now */
            __threadfence();
            copy_picture(P, host_arena, hl, 16);
        }
        run_n = 0;
    };
    for (int w = lo + half; w < hi; w += 2) {
        const uint32_t item = work[w];
        const int sidx = (int)(item >> 12);
        const h261b_session_dev_t &S = sessions[sidx];
        if (!S.bits_out)
            continue;
        if (sidx != run_s) {
            publish();
            run_s = sidx;
        }
        run_n++;
        const int mb = (int)(item & 4095u);
        const h261b_mb_info_t r = S.info_out[mb];
        if (r.flags == 0)
            continue;
        const int total = S.vlc_total[0];
        const int64_t words = ((int64_t)(total + 127) / 128) * 4;
        /* a layout that does not fit the slot is refused, whatever wrote it */
        if (S.vlc_total[1] != 0 || total < 0 || words * 4 > S.bits_cap)
            continue;
        int oob = 0;
        const int64_t pos = S.vlc_pos[mb];
        const uint32_t plan = S.vlc_plan[mb];
        const int addr = plan & 63, mt = (plan >> 6) & 15, mq = (plan >> 10) & 1;
        const int dx = (int)((plan >> 11) & 31) - 16, dy = (int)((plan >> 16) & 31) - 16;
        const bool intra = r.type == H261B_MB_TYPE_INTRA;
        const int cbp = coded_blocks(r);
        /* the header as one MSB-first value of at most 57 bits */
        uint64_t hv;
        int hbits;
        {
            const uint16_t e = c_vlc_mba[addr];
            hv = e & 0xFF;
            hbits = e >> 8;
            const int ml = c_vlc_mtype_len[mt];
            hv = (hv << ml) | 1u;
            hbits += ml;
            if (mq) {
                hv = (hv << 5) | (uint32_t)r.quant;
                hbits += 5;
            }
            if (!intra && (r.flags & H261B_MB_MC)) {
                uint32_t cx, cy;
                int lx, ly;
                mvd_code(dx, cx, lx);
                mvd_code(dy, cy, ly);
                hv = (((hv << lx) | cx) << ly) | cy;
                hbits += lx + ly;
            }
            if (!intra && cbp) {
                const uint16_t e2 = c_vlc_cbp[cbp];
                hv = (hv << (e2 >> 8)) | (e2 & 0xFF);
                hbits += e2 >> 8;
            }
        }
        if (hl == 0) {
            if (hbits > 32) {
                put_bits_pic(S.bits_out, words, pos, (uint32_t)(hv >> 32), hbits - 32, oob);
                put_bits_pic(S.bits_out, words, pos + (hbits - 32), (uint32_t)hv, 32, oob);
            } else {
                put_bits_pic(S.bits_out, words, pos, (uint32_t)hv, hbits, oob);
            }
        }
        /* the coefficient bits, shifted into place */
        const int nbits = r.coef_bits;
        if (nbits > 0) {
            const int64_t q = pos + hbits;
            const int sh = (int)(q & 31);
            const int64_t w0 = q >> 5;
            const int nout = (sh + nbits + 31) >> 5, nin = (nbits + 31) >> 5;
            const uint32_t *src = S.vlc_scratch + (size_t)mb * MB_WORDS;
            if (w0 < 0 || w0 + nout > words || nin > MB_WORDS) {
                oob = 1;
            } else {
                for (int i = hl; i < nout; i += 16) {
                    const uint32_t hi = i < nin ? src[i] : 0u;
                    const uint32_t lo = i > 0 ? src[i - 1] : 0u;
                    const uint32_t x = sh ? ((hi >> sh) | (lo << (32 - sh))) : hi;
                    uint32_t *d = S.bits_out + w0 + i;
                    if (i == 0 || i == nout - 1)
                        atomicOr(d, bswap(x));
                    else
                        *d = bswap(x);
                }
            }
        }
        if (__any_sync(hmask, oob) && hl == 0)
            atomicExch(&S.vlc_total[1], H261B_BITS_MISMATCH);
    }
    publish();
    __syncthreads();
    const int nd = min(n_done, PACK_DONE_MAX);
    for (int i = 0; i < nd; i++) {
        __threadfence();   /* the other CTAs' words, published before their counts */
        copy_picture(sessions[done[i]], host_arena, (int)threadIdx.x, VLC_THREADS);
    }
}

} // namespace
} // namespace h261b

using namespace h261b;

extern "C" h261b_bits_layout_t h261b_bits_layout(int32_t w, int32_t h)
{
    h261b_bits_layout_t l = { 0, 0, 0, 0, 0, 0 };
    const bool cif = w == 352 && h == 288, qcif = w == 176 && h == 144;
    if (!cif && !qcif)
        return l;
    const int64_t nmb = (int64_t)(w / 16) * (h / 16), ngob = cif ? 12 : 3;
    const int64_t pic_bits = 32 + 26 * ngob + nmb * (MB_HDR_MAX + MB_WORDS * 32);
    auto al = [](int64_t x) { return (x + 255) / 256 * 256; };
    l.picture = 0;
    l.scratch = al(((pic_bits + 127) / 128) * 16);
    l.pos = l.scratch + al(nmb * MB_WORDS * 4);
    l.plan = l.pos + al(nmb * 4);
    l.total = l.plan + al(nmb * 4);
    l.bytes = l.total + 256;
    return l;
}

extern "C" int64_t h261b_bits_slot_bytes(int32_t w, int32_t h) { return h261b_bits_layout(w, h).bytes; }

/* CTAs of the codes and pack kernels resident per SM, per device */
static cudaError_t resident_ctas(const void *codes, const void *pack, int *codes_res, int *pack_res)
{
    static std::mutex mu;
    static int cached[64][2];
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess)
        return err;
    if (dev < 0 || dev >= 64)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    int *c = cached[dev];
    if (!c[0]) {
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c[0], codes, VLC_THREADS, 0)) != cudaSuccess ||
            (err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c[1], pack, VLC_THREADS, 0)) != cudaSuccess)
            return err;
        c[0] = std::max(c[0], 1);
        c[1] = std::max(c[1], 1);
    }
    *codes_res = c[0];
    *pack_res = c[1];
    return cudaSuccess;
}

/* a launch that may begin while the kernel before it in the stream runs */
template <typename... Params, typename... Args>
static cudaError_t launch_dependent(void (*kernel)(Params...), dim3 grid, dim3 block, cudaStream_t st,
                                    Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

extern "C" int h261b_launch_bitstream(h261b_session_dev_t *sessions_dev, int32_t n_sessions, const uint32_t *work_dev,
                                      int32_t n_work, h261b_step_dev_t *step, uint8_t *host_arena_dev,
                                      int64_t host_cap, int32_t sm_count, void *stream, void *layout_done_event,
                                      int32_t test_extra_wait)
{
    if (n_work <= 0 || n_sessions <= 0)
        return 0;
    /* at least two MBs per warp, and no more CTAs than are resident at once
     * (latency-bound kernels want every warp slot they can get, but a
     * second, partial wave would only add a tail) */
    int codes_res = 0, pack_res = 0;
    cudaError_t err = resident_ctas((const void *)codes_kernel, (const void *)pack_kernel, &codes_res, &pack_res);
    if (err != cudaSuccess)
        return (int)err;
    const int64_t want = (n_work + 2 * VLC_WARPS - 1) / (2 * VLC_WARPS);
    const int codes_ctas = (int)std::min<int64_t>(want, (int64_t)sm_count * codes_res);
    const int ctas = (int)std::min<int64_t>(want, (int64_t)sm_count * pack_res);
    cudaStream_t st = (cudaStream_t)stream;
    err = launch_dependent(codes_kernel, dim3(codes_ctas), dim3(VLC_THREADS), st,
                           (const h261b_session_dev_t *)sessions_dev, work_dev, n_work, step, test_extra_wait);
    if (err != cudaSuccess)
        return (int)err;
    err = launch_dependent(layout_kernel, dim3(n_sessions), dim3(LAYOUT_THREADS), st,
                                       (const h261b_session_dev_t *)sessions_dev, step,
                                       (int64_t)(host_arena_dev ? host_cap : 0));
    if (err != cudaSuccess)
        return (int)err;
    if (layout_done_event) {
        /* the next step's rate control reads what the layout updated */
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaError_t err = cudaStreamIsCapturing(st, &cs);
        if (err == cudaSuccess)
            err = cudaEventRecordWithFlags((cudaEvent_t)layout_done_event, st,
                                           cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                               : cudaEventRecordDefault);
        if (err != cudaSuccess)
            return (int)err;
    }
    err = launch_dependent(pack_kernel, dim3(ctas), dim3(VLC_THREADS), st, (const h261b_session_dev_t *)sessions_dev,
                           work_dev, n_work, host_arena_dev);
    if (err != cudaSuccess)
        return (int)err;
    return (int)cudaGetLastError();
}

/*
 * bitstream.cu -- H.261 bitstream writer on the device.
 *
 * Writes each picture in the syntax of the reference's host writers
 * (src/h261_picture.c:115-148, src/h261_gob.c:6-199,
 * src/h261_macroblock.c:5-262), byte for byte: picture header, GOBs in the
 * QCIF / CIF order, macroblocks with MBA, MTYPE, MQUANT, MVD, CBP, TCOEFF
 * and EOB, the last byte zero-padded (src/h261_bitstream.c:64-76).
 *
 * One CTA per picture:
 *   A  every GOB is one warp, one lane per macroblock (the 33rd by all
 *      lanes): the address increment, quantiser in force and vector
 *      predictor of a macroblock depend only on earlier records of its GOB,
 *      so ballots over the GOB's coded / COEFF / MC flags give them all at
 *      once.  Header bits plus the coefficient bits the encode kernel
 *      counted (h261b_mb_info_t.coef_bits) give every macroblock's size; a
 *      warp scan gives its offset in the GOB.
 *   B  one thread scans the GOB sizes; the picture's words are cleared.
 *   C  warps take macroblocks: each assembles its macroblock in a shared
 *      staging buffer (lane 0 the header; eight lanes per block, each lane
 *      eight consecutive coefficients of the transmission order, a scan for
 *      the code offsets) and stores it; only a macroblock's first and last
 *      word can be shared with a neighbour and are ORed in with atomics.
 *   D  the picture is copied to the host arena (mapped pinned memory) at an
 *      offset drawn with one atomic, so no separate copy is issued for it.
 */
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "h261b_device.h"
#include "vlc_tables.h"

namespace h261b {
namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr int BS_WARPS = 8;
constexpr int BS_THREADS = BS_WARPS * 32;
constexpr int MAX_MB = 396;          /* CIF */
/* one macroblock: header <= 57 bits, six blocks <= 6 * (8 + 63 * 20 + 2);
 * plus up to 31 bits of offset into the first word */
constexpr int MB_MAX_BITS = 57 + 6 * (64 * 20 + 2);
constexpr int STAGE_WORDS = (MB_MAX_BITS + 31 + 31) / 32 + 1;

struct BsSmem {
    /* vector-accessed arrays first, on 16-byte boundaries */
    alignas(16) int8_t blk[BS_WARPS][4][64];   /* column-major levels of the blocks in flight */
    alignas(16) uint32_t stage[BS_WARPS][STAGE_WORDS];
    uint16_t tc[27][16];
    uint8_t zz_cm[64];               /* column-major index of the k-th coefficient sent */
    int32_t mb_off[MAX_MB];          /* bit offset of the MB within its GOB */
    int32_t mb_len[MAX_MB];          /* its size in bits, 0 = not coded */
    uint32_t mb_plan[MAX_MB];        /* header fields, see plan_* */
    int32_t gob_bits[12];
    int32_t gob_off[12];
    int32_t total_bits;
    int32_t status;
    int32_t host_off;
};
static_assert(offsetof(BsSmem, blk) % 16 == 0 && offsetof(BsSmem, stage) % 16 == 0, "vector alignment");

/* header plan of a macroblock: address increment, MTYPE, MQUANT flag and
 * the two wrapped vector differences */
__device__ __forceinline__ uint32_t plan_pack(int addr, int mtype, int mq, int dx, int dy)
{
    return (uint32_t)addr | ((uint32_t)mtype << 6) | ((uint32_t)mq << 10) | ((uint32_t)(dx + 16) << 11) |
           ((uint32_t)(dy + 16) << 16);
}

__device__ __forceinline__ int wrap_mvd(int d) { return ((d + 16) & 31) - 16; }

__device__ __forceinline__ void mvd_code(int w, uint32_t &code, int &len)
{
    const int a = w < 0 ? -w : w;
    const uint16_t e = c_vlc_mvd[a];
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

/* OR a code of len <= 32 bits into the MSB-first staging words at bit
 * position pos; a position outside the buffer is not written and counts
 * as an error */
__device__ __forceinline__ void put_bits(uint32_t *w, int pos, uint32_t code, int len, int &oob)
{
    if (len <= 0)
        return;
    if (pos < 0 || pos + len > STAGE_WORDS * 32) {
        oob = 1;
        return;
    }
    const int word = pos >> 5, off = pos & 31;
    const int end = off + len;
    if (end <= 32) {
        atomicOr(&w[word], code << (32 - end));
    } else {
        atomicOr(&w[word], code >> (end - 32));
        atomicOr(&w[word + 1], code << (64 - end));
    }
}

__device__ __forceinline__ uint32_t bswap(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

/* same, on the picture's words in device memory (stored byte-swapped, so
 * that their bytes are the stream's bytes) */
__device__ __forceinline__ void put_bits_global(uint32_t *w, int64_t pos, uint32_t code, int len)
{
    const int64_t word = pos >> 5;
    const int off = (int)(pos & 31), end = off + len;
    if (end <= 32) {
        atomicOr(&w[word], bswap(code << (32 - end)));
    } else {
        atomicOr(&w[word], bswap(code >> (end - 32)));
        atomicOr(&w[word + 1], bswap(code << (64 - end)));
    }
}

__global__ void __launch_bounds__(BS_THREADS) bitstream_kernel(const h261b_session_dev_t *sessions,
                                                               h261b_step_dev_t *step, uint8_t *host_arena,
                                                               int64_t host_cap)
{
    const h261b_session_dev_t &S = sessions[blockIdx.x];
    if (!S.bits_out)
        return;
    __shared__ BsSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool cif = S.mbw == 22;
    const int ngob = cif ? 12 : 3, nmb = S.mbw * S.mbh;
    const int gq = S.quant;
    const h261b_mb_info_t *info = S.info_out;

    for (int i = tid; i < 27 * 16; i += BS_THREADS)
        (&sm.tc[0][0])[i] = (&c_vlc_tcoeff[0][0])[i];
    if (tid < 64) {
        /* column-major index of zig-zag position tid */
        for (int v = 0; v < 8; v++)
            for (int u = 0; u < 8; u++)
                if (zigzag_index(v, u) == tid)
                    sm.zz_cm[tid] = (uint8_t)(u * 8 + v);
    }
    if (tid == 0)
        sm.status = 0;
    __syncthreads();

    /* ---- A: macroblock headers and sizes, one warp per GOB */
    for (int g = warp; g < ngob; g += BS_WARPS) {
        const int x0 = cif ? (g & 1) * 11 : 0, y0 = (cif ? g >> 1 : g) * 3;
        const int mi = (y0 + lane / 11) * S.mbw + x0 + lane % 11;
        const int m32 = (y0 + 2) * S.mbw + x0 + 10;
        const h261b_mb_info_t r = info[mi];
        const h261b_mb_info_t r32 = info[m32];
        const uint32_t C = __ballot_sync(FULL, r.flags != 0);
        const uint32_t K = __ballot_sync(FULL, (r.flags & H261B_MB_COEFF) != 0);
        const uint32_t M = __ballot_sync(FULL, (r.flags & H261B_MB_MC) != 0);
        const int prev_mvx = __shfl_up_sync(FULL, (int)r.mvx, 1), prev_mvy = __shfl_up_sync(FULL, (int)r.mvy, 1);
        const uint32_t below = (1u << lane) - 1u;
        /* quantiser in force: the last COEFF macroblock before, else GQUANT */
        const uint32_t kb = K & below;
        const int qv = __shfl_sync(FULL, (int)r.quant, kb ? 31 - __clz((int)kb) : lane);
        const int qv32 = __shfl_sync(FULL, (int)r.quant, K ? 31 - __clz((int)K) : 0);
        const int mvx31 = __shfl_sync(FULL, (int)r.mvx, 31), mvy31 = __shfl_sync(FULL, (int)r.mvy, 31);

        int bits = 0, bits32 = 0, bad = 0;
        /* lane's macroblock */
        if (r.flags != 0) {
            const uint32_t cb = C & below;
            const int addr = cb ? lane - (31 - __clz((int)cb)) : lane + 1;
            const int qs = kb ? qv : gq;
            const bool intra = r.type == H261B_MB_TYPE_INTRA;
            const int mq = intra ? (r.quant != qs) : (r.quant != qs && (r.flags & H261B_MB_COEFF));
            const int mt = mtype_of(r.type, r.flags, mq);
            const bool ok = lane > 0 && lane % 11 != 0 && ((M >> (lane - 1)) & 1u);
            const int dx = wrap_mvd(r.mvx - (ok ? prev_mvx : 0)), dy = wrap_mvd(r.mvy - (ok ? prev_mvy : 0));
            int h = (c_vlc_mba[addr] >> 8) + (mt >= 0 ? c_vlc_mtype_len[mt] : 0) + (mq ? 5 : 0);
            if (!intra && (r.flags & H261B_MB_MC))
                h += (c_vlc_mvd[dx < 0 ? -dx : dx] >> 8) + (c_vlc_mvd[dy < 0 ? -dy : dy] >> 8);
            if (!intra && (r.flags & H261B_MB_COEFF))
                h += c_vlc_cbp[r.cbp & 63] >> 8;
            bad = mt < 0 || (!intra && (r.flags & H261B_MB_COEFF) && (r.cbp & 63) == 0);
            bits = h + r.coef_bits;
            sm.mb_plan[mi] = plan_pack(addr, mt < 0 ? 0 : mt, mq, dx, dy);
        }
        /* the 33rd macroblock, by every lane */
        if (r32.flags != 0) {
            const int addr = C ? 32 - (31 - __clz((int)C)) : 33;
            const int qs = K ? qv32 : gq;
            const bool intra = r32.type == H261B_MB_TYPE_INTRA;
            const int mq = intra ? (r32.quant != qs) : (r32.quant != qs && (r32.flags & H261B_MB_COEFF));
            const int mt = mtype_of(r32.type, r32.flags, mq);
            const bool ok = (M >> 31) & 1u;
            const int dx = wrap_mvd(r32.mvx - (ok ? mvx31 : 0)), dy = wrap_mvd(r32.mvy - (ok ? mvy31 : 0));
            int h = (c_vlc_mba[addr] >> 8) + (mt >= 0 ? c_vlc_mtype_len[mt] : 0) + (mq ? 5 : 0);
            if (!intra && (r32.flags & H261B_MB_MC))
                h += (c_vlc_mvd[dx < 0 ? -dx : dx] >> 8) + (c_vlc_mvd[dy < 0 ? -dy : dy] >> 8);
            if (!intra && (r32.flags & H261B_MB_COEFF))
                h += c_vlc_cbp[r32.cbp & 63] >> 8;
            bad |= mt < 0 || (!intra && (r32.flags & H261B_MB_COEFF) && (r32.cbp & 63) == 0);
            bits32 = h + r32.coef_bits;
            if (lane == 0)
                sm.mb_plan[m32] = plan_pack(addr, mt < 0 ? 0 : mt, mq, dx, dy);
        }
        /* offsets within the GOB, after its 26-bit header */
        int incl = bits;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o)
                incl += t;
        }
        const int sum32 = __shfl_sync(FULL, incl, 31);
        sm.mb_off[mi] = 26 + incl - bits;
        sm.mb_len[mi] = bits;
        if (lane == 0) {
            sm.mb_off[m32] = 26 + sum32;
            sm.mb_len[m32] = bits32;
            sm.gob_bits[g] = 26 + sum32 + bits32;
        }
        /* a size beyond the syntax's maximum would overrun the staging
         * buffer: only a wrong count can produce one */
        bad |= bits < 0 || bits > MB_MAX_BITS || bits32 < 0 || bits32 > MB_MAX_BITS;
        if (__any_sync(FULL, bad) && lane == 0)
            atomicExch(&sm.status, H261B_BITS_BAD_RECORD);
    }
    __syncthreads();

    /* ---- B: GOB offsets after the 32-bit picture header */
    if (tid == 0) {
        int o = 32;
        for (int g = 0; g < ngob; g++) {
            sm.gob_off[g] = o;
            o += sm.gob_bits[g];
        }
        sm.total_bits = o;
        if ((int64_t)((o + 127) / 128) * 16 > S.bits_cap)
            sm.status = H261B_BITS_OVERFLOW;
    }
    __syncthreads();
    const int total = sm.total_bits;
    if (sm.status != 0) {
        if (tid == 0)
            *S.pic_out = h261b_pic_info_t{ 0, -1, sm.status, gq };
        return;
    }
    const int words = ((total + 127) / 128) * 4;   /* whole 16-byte units */
    for (int i = tid; i < words; i += BS_THREADS)
        S.bits_out[i] = 0u;
    __syncthreads();

    /* ---- C: headers and macroblocks */
    if (tid == 0) {
        /* PSC, TR, PTYPE (split 0, document camera 0, freeze release 1,
         * source format, HI_RES bit 1, spare 1), PEI 0 */
        const uint32_t ptype = (1u << 3) | ((cif ? 1u : 0u) << 2) | (1u << 1) | 1u;
        S.bits_out[0] = bswap((16u << 12) | ((uint32_t)(S.frame_num & 31) << 7) | (ptype << 1));
    }
    if (tid < ngob) {
        const uint32_t number = cif ? (uint32_t)tid + 1u : 2u * (uint32_t)tid + 1u;
        put_bits_global(S.bits_out, sm.gob_off[tid], (1u << 10) | (number << 6) | ((uint32_t)gq << 1), 26);
    }

    uint32_t *stage = sm.stage[warp];
    int oob = 0;
    for (int mb = warp; mb < nmb; mb += BS_WARPS) {
        const int len = sm.mb_len[mb];
        if (len == 0)
            continue;
        const int mbx = mb % S.mbw, mby = mb / S.mbw;
        const int g = cif ? (mby / 3) * 2 + mbx / 11 : mby / 3;
        const int64_t pos = (int64_t)sm.gob_off[g] + sm.mb_off[mb];
        const int base = (int)(pos & 31);
        const int nw = (base + len + 31) >> 5;
        for (int i = lane; i < nw; i += 32)
            stage[i] = 0u;
        const h261b_mb_info_t r = info[mb];
        const bool intra = r.type == H261B_MB_TYPE_INTRA;
        const int cbp = intra ? 63 : ((r.flags & H261B_MB_COEFF) ? (r.cbp & 63) : 0);
        __syncwarp();

        /* header, lane 0 */
        const uint32_t plan = sm.mb_plan[mb];
        const int addr = plan & 63, mt = (plan >> 6) & 15, mq = (plan >> 10) & 1;
        const int dx = (int)((plan >> 11) & 31) - 16, dy = (int)((plan >> 16) & 31) - 16;
        int hpos = base;
        {
            const uint16_t e = c_vlc_mba[addr];
            hpos += e >> 8;
            if (lane == 0)
                put_bits(stage, hpos - (e >> 8), e & 0xFF, e >> 8, oob);
            const int ml = c_vlc_mtype_len[mt];
            if (lane == 0)
                put_bits(stage, hpos, 1u, ml, oob);
            hpos += ml;
            if (mq) {
                if (lane == 0)
                    put_bits(stage, hpos, (uint32_t)r.quant, 5, oob);
                hpos += 5;
            }
            if (!intra && (r.flags & H261B_MB_MC)) {
                uint32_t cx, cy;
                int lx, ly;
                mvd_code(dx, cx, lx);
                mvd_code(dy, cy, ly);
                if (lane == 0) {
                    put_bits(stage, hpos, cx, lx, oob);
                    put_bits(stage, hpos + lx, cy, ly, oob);
                }
                hpos += lx + ly;
            }
            if (!intra && cbp) {
                const uint16_t e2 = c_vlc_cbp[cbp];
                if (lane == 0)
                    put_bits(stage, hpos, e2 & 0xFF, e2 >> 8, oob);
                hpos += e2 >> 8;
            }
        }

        /* blocks: luma 0-3 in one round, chroma 4-5 in the next; eight
         * lanes per block, lane j of a block holds positions 8j..8j+7 of
         * the transmission order */
        const int slot = lane >> 3, j = lane & 7;
        const int8_t *lv = S.level_out + (size_t)mb * 384;
        for (int round = 0; round < 2; round++) {
            const int b = round * 4 + slot;
            const bool here = b < 6 && ((cbp >> (5 - b)) & 1);
            if (b < 6)
                *reinterpret_cast<uint2 *>(&sm.blk[warp][slot][j * 8]) =
                    *reinterpret_cast<const uint2 *>(lv + b * 64 + j * 8);
            __syncwarp();
            int c[8];
            uint32_t m8 = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int8_t x = sm.blk[warp][slot][sm.zz_cm[8 * j + i]];
                c[i] = (intra && j == 0 && i == 0) ? (int)(uint8_t)x : (int)x;
                m8 |= (here && c[i] != 0) ? (1u << i) : 0u;
            }
            /* the block's nonzero mask in transmission order */
            uint32_t mlo = j < 4 ? m8 << (8 * j) : 0u, mhi = j >= 4 ? m8 << (8 * (j - 4)) : 0u;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                mlo |= __shfl_xor_sync(FULL, mlo, o);
                mhi |= __shfl_xor_sync(FULL, mhi, o);
            }
            const uint64_t mask = ((uint64_t)mhi << 32) | mlo;
            const uint64_t bl = j ? mask & ((1ull << (8 * j)) - 1ull) : 0ull;
            int prev = bl ? 63 - __clzll((long long)bl) : -1;
            uint32_t code[8];
            int clen[8], mine = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int k = 8 * j + i;
                clen[i] = 0;
                code[i] = 0;
                if (!((m8 >> i) & 1u))
                    continue;
                const int v = c[i];
                if (k == 0 && intra) {
                    code[i] = (uint32_t)v & 0xFFu;
                    clen[i] = 8;
                } else if (k == 0 && (v == 1 || v == -1)) {
                    code[i] = v < 0 ? 3u : 2u;
                    clen[i] = 2;
                } else {
                    const int run = k - prev - 1;
                    const int a = v < 0 ? -v : v;
                    const uint16_t e = (run <= 26 && a <= 15) ? sm.tc[run][a] : (uint16_t)0;
                    if (e) {
                        code[i] = ((uint32_t)(e & 0xFF) << 1) | (v < 0 ? 1u : 0u);
                        clen[i] = (e >> 8) + 1;
                    } else {
                        code[i] = (1u << 14) | ((uint32_t)run << 8) | ((uint32_t)v & 0xFFu);
                        clen[i] = 20;
                    }
                }
                prev = k;
                mine += clen[i];
            }
            /* offsets of this lane's codes within the block */
            int incl = mine;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, o, 8);
                if (j >= o)
                    incl += t;
            }
            const int last = __shfl_sync(FULL, incl, (slot << 3) | 7);
            const int btotal = here ? last + 2 : 0;
            /* start of each block of the round after the earlier ones */
            int bstart = hpos, rtotal = 0;
#pragma unroll
            for (int s2 = 0; s2 < 4; s2++) {
                const int t = __shfl_sync(FULL, btotal, s2 << 3);
                if (s2 < slot)
                    bstart += t;
                rtotal += t;
            }
            if (here) {
                int p = bstart + incl - mine;
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    put_bits(stage, p, code[i], clen[i], oob);
                    p += clen[i];
                }
                if (j == 7)
                    put_bits(stage, bstart + btotal - 2, 2u, 2, oob);   /* EOB */
            }
            hpos += rtotal;
            __syncwarp();
        }
        const bool wrong = __any_sync(FULL, oob) || hpos - base != len || (pos >> 5) + nw > words;
        if (wrong) {
            if (lane == 0)
                atomicExch(&sm.status, H261B_BITS_MISMATCH);
            __syncwarp();
            continue;
        }

        /* store; the first and the last word may be shared with the
         * neighbouring macroblocks */
        uint32_t *dst = S.bits_out + (pos >> 5);
        for (int i = lane; i < nw; i += 32) {
            const uint32_t x = bswap(stage[i]);
            if (i == 0 || i == nw - 1)
                atomicOr(&dst[i], x);
            else
                dst[i] = x;
        }
        __syncwarp();
    }
    __syncthreads();

    /* ---- D: to the host arena */
    const int bytes = (total + 7) >> 3;
    const int padded = (bytes + 15) & ~15;
    if (tid == 0) {
        int off = -1;
        if (sm.status != 0) {
            *S.pic_out = h261b_pic_info_t{ 0, -1, sm.status, gq };
            sm.host_off = -1;
        } else {
        if (host_arena) {
            const uint32_t o = atomicAdd(&step->host_used, (uint32_t)padded);
            if ((int64_t)o + padded <= host_cap)
                off = (int)o;
        }
        sm.host_off = off;
        *S.pic_out = h261b_pic_info_t{ bytes, off, 0, gq };
        }
    }
    __syncthreads();
    if (sm.host_off >= 0) {
        const uint4 *src = reinterpret_cast<const uint4 *>(S.bits_out);
        uint4 *dst = reinterpret_cast<uint4 *>(host_arena + sm.host_off);
        for (int i = tid; i < padded / 16; i += BS_THREADS)
            dst[i] = src[i];
    }
}

} // namespace
} // namespace h261b

using namespace h261b;

extern "C" int64_t h261b_bits_slot_bytes(int32_t w, int32_t h)
{
    const bool cif = w == 352 && h == 288, qcif = w == 176 && h == 144;
    if (!cif && !qcif)
        return 0;
    const int64_t nmb = (w / 16) * (h / 16), ngob = cif ? 12 : 3;
    const int64_t bits = 32 + 26 * ngob + nmb * MB_MAX_BITS;
    return ((bits + 127) / 128) * 16;
}

extern "C" int h261b_launch_bitstream(const h261b_session_dev_t *sessions_dev, int32_t n_sessions,
                                      h261b_step_dev_t *step, uint8_t *host_arena_dev, int64_t host_cap,
                                      void *stream)
{
    if (n_sessions <= 0)
        return 0;
    bitstream_kernel<<<n_sessions, BS_THREADS, 0, (cudaStream_t)stream>>>(sessions_dev, step, host_arena_dev,
                                                                          host_cap);
    return (int)cudaGetLastError();
}

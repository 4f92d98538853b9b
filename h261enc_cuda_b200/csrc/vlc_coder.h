/* The coefficient part of an H.261 macroblock on the device: each coded
 * block's TCOEFF codes in transmission (zig-zag) order and its EOB, as the
 * reference's host writer sends them (src/h261_macroblock.c:196-262):
 *
 *   - an intra block's DC level as its 8-bit value;
 *   - an inter block's first coefficient, when it is +-1, as the short code
 *     1s (s the sign);
 *   - every other nonzero level after `run` zeros as the table code plus a
 *     sign bit, or the 20-bit escape (000001, 6-bit run, 8-bit level) where
 *     the table has no entry;
 *   - EOB (10) after the block.
 *
 * A warp codes up to four blocks at once: lane (slot, j), slot = lane / 8,
 * holds transmission positions 8j .. 8j+7 of its slot's block.  The codes
 * are ORed into a zeroed word buffer, MSB first.  The bitstream's codes
 * kernel runs them on each MB's levels after the encode kernel. */
#pragma once

#include <cstdint>

#include "vlc_tables.h"

namespace h261b {

/* MB string words: six blocks of an 8-bit DC or a first code, 63 escapes of
 * 20 bits and an EOB */
constexpr int VLC_MB_WORDS = H261B_VLC_MB_WORDS;

/* OR a code of len <= 32 bits into MSB-first words at bit position pos of
 * a buffer of `words` words; a position outside it is not written and
 * counts as an error */
__device__ __forceinline__ void put_bits(uint32_t *w, int words, int pos, uint32_t code, int len, int &oob)
{
    if (len <= 0)
        return;
    if (pos < 0 || pos + len > words * 32) {
        oob = 1;
        return;
    }
    const int word = pos >> 5, end = (pos & 31) + len;
    if (end <= 32) {
        atomicOr(&w[word], code << (32 - end));
    } else {
        atomicOr(&w[word], code >> (end - 32));
        atomicOr(&w[word + 1], code << (64 - end));
    }
}

/* this lane's eight column-major indices of transmission positions
 * 8j .. 8j+7 (j = lane % 8), packed one byte each into two words */
__device__ __forceinline__ void zigzag_lane(int lane, uint32_t &zz0, uint32_t &zz1)
{
    const int j = lane & 7;
    zz0 = zz1 = 0u;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        zz0 |= (uint32_t)c_zigzag_cm.cm[8 * j + i] << (8 * i);
        zz1 |= (uint32_t)c_zigzag_cm.cm[8 * j + 4 + i] << (8 * i);
    }
}

/* the TCOEFF table into shared memory (27 x 16 entries), by the threads of
 * a CTA; the caller synchronises before the first lookup */
__device__ __forceinline__ void load_tcoeff_table(uint16_t (*tc)[16], int tid, int nthreads)
{
    for (int i = tid; i < 27 * 16; i += nthreads)
        (&tc[0][0])[i] = (&c_vlc_tcoeff[0][0])[i];
}

/* One group of up to four coded blocks.  Lane (slot, j) codes positions
 * 8j .. 8j+7 of `blk` (the slot's block: 64 levels, column-major, an intra
 * DC stored as uint8) when `here`.  The group's codes go into `stage` from
 * bit `pos` on, the blocks one after another in slot order; returns the
 * group's bits (the same on every lane).  Every lane of the warp calls it. */
__device__ __forceinline__ int code_block_group(const int8_t *blk, bool here, bool intra, uint32_t zz0, uint32_t zz1,
                                                const uint16_t (*tc)[16], uint32_t *stage, int words, int pos,
                                                int lane, int &oob)
{
    constexpr unsigned FULLMASK = 0xFFFFFFFFu;
    const int slot = lane >> 3, j = lane & 7;
    int c[8];
    uint32_t m8 = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int idx = (int)(((i < 4 ? zz0 : zz1) >> (8 * (i & 3))) & 0xFFu);
        const int8_t x = here ? blk[idx] : (int8_t)0;
        c[i] = (intra && j == 0 && i == 0) ? (int)(uint8_t)x : (int)x;
        m8 |= (c[i] != 0) ? (1u << i) : 0u;
    }
    /* the block's nonzero mask in transmission order */
    uint32_t mlo = j < 4 ? m8 << (8 * j) : 0u, mhi = j >= 4 ? m8 << (8 * (j - 4)) : 0u;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        mlo |= __shfl_xor_sync(FULLMASK, mlo, o);
        mhi |= __shfl_xor_sync(FULLMASK, mhi, o);
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
            code[i] = (uint32_t)v & 0xFFu;       /* the DC level as it is */
            clen[i] = 8;
        } else if (k == 0 && (v == 1 || v == -1)) {
            code[i] = v < 0 ? 3u : 2u;            /* first inter coefficient +-1 */
            clen[i] = 2;
        } else {
            const int run = k - prev - 1;
            const int a = v < 0 ? -v : v;
            const uint16_t e = (run <= 26 && a <= 15) ? tc[run][a] : (uint16_t)0;
            if (e) {
                code[i] = ((uint32_t)(e & 0xFF) << 1) | (v < 0 ? 1u : 0u);
                clen[i] = (e >> 8) + 1;
            } else {
                /* escape 0000 01, 6-bit run, 8-bit level */
                code[i] = (1u << 14) | ((uint32_t)run << 8) | ((uint32_t)v & 0xFFu);
                clen[i] = 20;
            }
        }
        prev = k;
        mine += clen[i];
    }
    /* offsets of this lane's codes within its block */
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        const int t = __shfl_up_sync(FULLMASK, incl, o, 8);
        if (j >= o)
            incl += t;
    }
    const int last = __shfl_sync(FULLMASK, incl, (slot << 3) | 7);
    const int btotal = here ? last + 2 : 0;
    int bstart = pos, rtotal = 0;
#pragma unroll
    for (int s2 = 0; s2 < 4; s2++) {
        const int t = __shfl_sync(FULLMASK, btotal, s2 << 3);
        if (s2 < slot)
            bstart += t;
        rtotal += t;
    }
    if (here) {
        int p = bstart + incl - mine;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            put_bits(stage, words, p, code[i], clen[i], oob);
            p += clen[i];
        }
        if (j == 7)
            put_bits(stage, words, bstart + btotal - 2, 2u, 2, oob);   /* EOB */
    }
    return rtotal;
}

/* after an MB's groups: its string from the staging words into dst (the
 * MB's VLC_MB_WORDS words), the staging words cleared for the next MB;
 * returns the string's bits, or -1 if a code fell outside the words (which
 * makes the layout refuse the picture).  Every lane calls it. */
__device__ __forceinline__ int store_mb_string(uint32_t *stage, uint32_t *dst, int pos, int oob, int lane)
{
    oob = __any_sync(0xFFFFFFFFu, oob);
    const int nw = min((pos + 31) >> 5, VLC_MB_WORDS);
    for (int i = lane; i < nw; i += 32) {
        dst[i] = stage[i];
        stage[i] = 0u;
    }
    __syncwarp();
    return oob ? -1 : pos;
}

} // namespace h261b

/*
 * h261_decoder.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A conformance decoder for the bitstreams this project writes: it parses
 * the H.261 syntax (ITU-T H.261 sections 4.2.1-4.2.4: picture, GOB and
 * macroblock layers, the VLC tables 1-5 and the TCOEFF escape) back into
 * macroblock records and reconstructs the picture from them with the
 * oracle's restatement of the reference's reconstruction
 * (orc_decode_frame: dequantisation, IDCT, motion compensation with the
 * loop filter).  A stream decoded here must reproduce the encoder's own
 * reconstructions bit for bit, and its records must be the encoder's.
 *
 * The syntax elements the encoder never emits (PEI/GEI extension bytes,
 * MBA stuffing) are still parsed.
 */
#include "h261_oracle.h"

#include <string.h>

typedef struct {
    const uint8_t *buf;
    int64_t nbits;
    int64_t pos;
    int err;
} bitr_t;

static uint32_t peek(bitr_t *r, int n)
{
    uint32_t v = 0;
    for (int i = 0; i < n; i++) {
        const int64_t p = r->pos + i;
        const uint32_t bit = p < r->nbits ? (r->buf[p >> 3] >> (7 - (p & 7))) & 1u : 0u;
        v = (v << 1) | bit;
    }
    return v;
}

static uint32_t peek_bit(bitr_t *r, int at)
{
    const int64_t p = r->pos + at;
    return p < r->nbits ? (r->buf[p >> 3] >> (7 - (p & 7))) & 1u : 0u;
}

static uint32_t get(bitr_t *r, int n)
{
    if (r->pos + n > r->nbits)
        r->err = 1;
    const uint32_t v = peek(r, n);
    r->pos += n;
    return v;
}

/* ---- VLC tables (the standard's, as in h261_writer.c) */

static const uint8_t d_mba[34][2] = {
    { 0, 0 },
    { 1, 1 },   { 3, 3 },   { 2, 3 },   { 3, 4 },   { 2, 4 },   { 3, 5 },   { 2, 5 },
    { 7, 7 },   { 6, 7 },   { 11, 8 },  { 10, 8 },  { 9, 8 },   { 8, 8 },   { 7, 8 },
    { 6, 8 },   { 23, 10 }, { 22, 10 }, { 21, 10 }, { 20, 10 }, { 19, 10 }, { 18, 10 },
    { 35, 11 }, { 34, 11 }, { 33, 11 }, { 32, 11 }, { 31, 11 }, { 30, 11 }, { 29, 11 },
    { 28, 11 }, { 27, 11 }, { 26, 11 }, { 25, 11 }, { 24, 11 },
};
#define MBA_STUFFING_CODE 15   /* 0000 0001 111, 11 bits */

static const uint8_t d_mtype_len[10] = { 4, 7, 1, 5, 9, 8, 10, 3, 2, 6 };
/* per MTYPE: intra, MQUANT, MC, CBP (coded blocks), FILTER */
static const uint8_t d_mtype_has[10][5] = {
    { 1, 0, 0, 0, 0 }, { 1, 1, 0, 0, 0 }, { 0, 0, 0, 1, 0 }, { 0, 1, 0, 1, 0 }, { 0, 0, 1, 0, 0 },
    { 0, 0, 1, 1, 0 }, { 0, 1, 1, 1, 0 }, { 0, 0, 1, 0, 1 }, { 0, 0, 1, 1, 1 }, { 0, 1, 1, 1, 1 },
};

static const uint8_t d_mvd_mag[17][2] = {
    { 1, 1 },   { 3, 3 },   { 3, 4 },   { 3, 5 },   { 7, 7 },   { 11, 8 },  { 9, 8 },
    { 7, 8 },   { 23, 10 }, { 21, 10 }, { 19, 10 }, { 35, 11 }, { 33, 11 }, { 31, 11 },
    { 29, 11 }, { 27, 11 }, { 25, 11 },
};

static const uint8_t d_cbp[64][2] = {
    { 0, 0 },   { 11, 5 },  { 9, 5 },   { 13, 6 },  { 13, 4 },  { 23, 7 },  { 19, 7 },  { 31, 8 },
    { 12, 4 },  { 22, 7 },  { 18, 7 },  { 30, 8 },  { 19, 5 },  { 27, 8 },  { 23, 8 },  { 19, 8 },
    { 11, 4 },  { 21, 7 },  { 17, 7 },  { 29, 8 },  { 17, 5 },  { 25, 8 },  { 21, 8 },  { 17, 8 },
    { 15, 6 },  { 15, 8 },  { 13, 8 },  { 3, 9 },   { 15, 5 },  { 11, 8 },  { 7, 8 },   { 7, 9 },
    { 10, 4 },  { 20, 7 },  { 16, 7 },  { 28, 8 },  { 14, 6 },  { 14, 8 },  { 12, 8 },  { 2, 9 },
    { 16, 5 },  { 24, 8 },  { 20, 8 },  { 16, 8 },  { 14, 5 },  { 10, 8 },  { 6, 8 },   { 6, 9 },
    { 18, 5 },  { 26, 8 },  { 22, 8 },  { 18, 8 },  { 13, 5 },  { 9, 8 },   { 5, 8 },   { 5, 9 },
    { 12, 5 },  { 8, 8 },   { 4, 8 },   { 4, 9 },   { 7, 3 },   { 10, 5 },  { 8, 5 },   { 12, 6 },
};

/* TCOEFF (run, level) -> code without sign */
typedef struct {
    uint8_t run, level, code, len;
} tc_entry_t;

static const tc_entry_t d_tc[] = {
    { 0, 1, 3, 2 },    { 0, 2, 4, 4 },    { 0, 3, 5, 5 },    { 0, 4, 6, 7 },    { 0, 5, 38, 8 },
    { 0, 6, 33, 8 },   { 0, 7, 10, 10 },  { 0, 8, 29, 12 },  { 0, 9, 24, 12 },  { 0, 10, 19, 12 },
    { 0, 11, 16, 12 }, { 0, 12, 26, 13 }, { 0, 13, 25, 13 }, { 0, 14, 24, 13 }, { 0, 15, 23, 13 },
    { 1, 1, 3, 3 },    { 1, 2, 6, 6 },    { 1, 3, 37, 8 },   { 1, 4, 12, 10 },  { 1, 5, 27, 12 },
    { 1, 6, 22, 13 },  { 1, 7, 21, 13 },  { 2, 1, 5, 4 },    { 2, 2, 4, 7 },    { 2, 3, 11, 10 },
    { 2, 4, 20, 12 },  { 2, 5, 20, 13 },  { 3, 1, 7, 5 },    { 3, 2, 36, 8 },   { 3, 3, 28, 12 },
    { 3, 4, 19, 13 },  { 4, 1, 6, 5 },    { 4, 2, 15, 10 },  { 4, 3, 18, 12 },  { 5, 1, 7, 6 },
    { 5, 2, 9, 10 },   { 5, 3, 18, 13 },  { 6, 1, 5, 6 },    { 6, 2, 30, 12 },  { 7, 1, 4, 6 },
    { 7, 2, 21, 12 },  { 8, 1, 7, 7 },    { 8, 2, 17, 12 },  { 9, 1, 5, 7 },    { 9, 2, 17, 13 },
    { 10, 1, 39, 8 },  { 10, 2, 16, 13 }, { 11, 1, 35, 8 },  { 12, 1, 34, 8 },  { 13, 1, 32, 8 },
    { 14, 1, 14, 10 }, { 15, 1, 13, 10 }, { 16, 1, 8, 10 },  { 17, 1, 31, 12 }, { 18, 1, 26, 12 },
    { 19, 1, 25, 12 }, { 20, 1, 23, 12 }, { 21, 1, 22, 12 }, { 22, 1, 31, 13 }, { 23, 1, 30, 13 },
    { 24, 1, 29, 13 }, { 25, 1, 28, 13 }, { 26, 1, 27, 13 },
};

static const uint8_t d_zigzag[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63,
};

/* match the next bits against a (code, length) table; -1 when nothing fits */
static int match(bitr_t *r, const uint8_t (*tab)[2], int n, int first)
{
    for (int i = first; i < n; i++) {
        const int len = tab[i][1];
        if (len && peek(r, len) == tab[i][0]) {
            r->pos += len;
            return i;
        }
    }
    return -1;
}

static int read_mvd(bitr_t *r)
{
    if (peek(r, 1) == 1) {
        r->pos += 1;
        return 0;
    }
    for (int m = 1; m <= 16; m++) {
        const int len = d_mvd_mag[m][1];
        const uint32_t v = peek(r, len);
        if (v == d_mvd_mag[m][0]) {
            r->pos += len;
            return -m;
        }
        if (m < 16 && v == d_mvd_mag[m][0] - 1u) {
            r->pos += len;
            return m;
        }
    }
    r->err = 1;
    return 0;
}

/* one block's coefficients in raster order; 0 or -1 on a syntax error */
static int read_block(bitr_t *r, int32_t *c, int intra)
{
    memset(c, 0, 64 * sizeof(int32_t));
    int k = 0;
    if (intra) {
        c[0] = (int32_t)get(r, 8);
        k = 1;
    } else if (peek(r, 1) == 1) {
        /* first coefficient: "1s" is run 0, level +-1 */
        r->pos += 1;
        c[0] = get(r, 1) ? -1 : 1;
        k = 1;
    }
    for (;;) {
        if (r->err || r->pos >= r->nbits)
            return -1;
        if (k > 0 && peek(r, 2) == 2) {
            r->pos += 2;                      /* EOB */
            return 0;
        }
        int run, level;
        if (peek(r, 6) == 1) {
            r->pos += 6;                      /* escape */
            run = (int)get(r, 6);
            level = (int)(int8_t)get(r, 8);
            if (level == 0 || level == -128)
                return -1;
        } else {
            int found = -1;
            for (size_t i = 0; i < sizeof(d_tc) / sizeof(d_tc[0]); i++)
                if (peek(r, d_tc[i].len) == d_tc[i].code) {
                    found = (int)i;
                    break;
                }
            if (found < 0)
                return -1;
            r->pos += d_tc[found].len;
            run = d_tc[found].run;
            level = get(r, 1) ? -(int)d_tc[found].level : (int)d_tc[found].level;
        }
        k += run;
        if (k > 63)
            return -1;
        c[d_zigzag[k]] = level;
        k++;
    }
}

/* Parse one picture starting at bit `pos` of `bits` (nbytes long): fills
 * mbs (the reference's records, raster MB order), the picture's format,
 * temporal reference and GQUANT of its first GOB, and returns the bit
 * position after the picture (its last byte padded), or -1. */
int64_t orc_parse_picture(const uint8_t *bits, int64_t nbytes, int64_t pos, int32_t *w, int32_t *h,
                          int32_t *tr, h261_macroblock_t *mbs, int32_t mbs_cap)
{
    bitr_t r = { bits, nbytes * 8, pos, 0 };
    if (get(&r, 20) != 16)
        return -1;
    *tr = (int32_t)get(&r, 5);
    const uint32_t ptype = get(&r, 6);
    const int cif = (ptype >> 2) & 1;
    while (get(&r, 1))
        get(&r, 8);                           /* PSPARE */
    *w = cif ? 352 : 176;
    *h = cif ? 288 : 144;
    const int mbw = *w / 16, nmb = mbw * (*h / 16), ngob = cif ? 12 : 3;
    if (nmb > mbs_cap)
        return -1;
    memset(mbs, 0, sizeof(h261_macroblock_t) * (size_t)nmb);
    for (int i = 0; i < nmb; i++) {
        mbs[i].i_macroblock_type = H261B_MB_TYPE_INTER;
        mbs[i].i_mb_x = (i % mbw) * 16;
        mbs[i].i_mb_y = (i / mbw) * 16;
    }
    for (int gob = 0; gob < ngob; gob++) {
        if (get(&r, 16) != 1)
            return -1;
        const int gn = (int)get(&r, 4);
        const int expect = cif ? gob + 1 : 2 * gob + 1;
        if (gn != expect)
            return -1;
        int quant = (int)get(&r, 5);
        while (get(&r, 1))
            get(&r, 8);                       /* GSPARE */
        const int x0 = cif ? (gn - 1) % 2 * 11 : 0, y0 = (cif ? (gn - 1) / 2 : gob) * 3;
        /* MBs the GOB skips keep GQUANT, as the encoder's records do */
        for (int i = 0; i < 33; i++)
            mbs[(y0 + i / 11) * mbw + x0 + i % 11].i_macroblock_quant = quant;
        int addr = 0, mv_ok = 0, pmx = 0, pmy = 0;
        for (;;) {
            /* 15 or more zeros: a start code follows (the next GOB, or the
             * next picture after the last byte's padding), or the data
             * ends; no macroblock-layer code has more than 7 */
            int zeros = 0;
            while (zeros < 24 && r.pos + zeros < r.nbits && peek_bit(&r, zeros) == 0)
                zeros++;
            if (zeros >= 15 || r.pos + zeros >= r.nbits)
                break;
            if (peek(&r, 11) == MBA_STUFFING_CODE) {
                r.pos += 11;
                continue;
            }
            const int inc = match(&r, d_mba, 34, 1);
            if (inc < 0)
                return -1;
            const int prev_addr = addr;
            addr += inc;
            if (addr > 33)
                return -1;
            /* skipped MBs break the vector prediction chain */
            if (inc > 1)
                mv_ok = 0;
            const int i = addr - 1;
            if (i % 11 == 0)
                mv_ok = 0;
            (void)prev_addr;
            h261_macroblock_t *m = &mbs[(y0 + i / 11) * mbw + x0 + i % 11];
            int mt = -1;
            for (int t = 0; t < 10; t++)
                if (peek(&r, d_mtype_len[t]) == 1u) {
                    /* the shortest code that matches: codes are a 1 after zeros */
                    if (mt < 0 || d_mtype_len[t] < d_mtype_len[mt])
                        mt = t;
                }
            if (mt < 0)
                return -1;
            r.pos += d_mtype_len[mt];
            const uint8_t *has = d_mtype_has[mt];
            if (has[1])
                quant = (int)get(&r, 5);
            m->i_macroblock_type = has[0] ? H261B_MB_TYPE_INTRA : H261B_MB_TYPE_INTER;
            m->i_macroblock_quant = quant;
            int flags = has[0] ? H261B_MB_COEFF : 0;
            if (has[2]) {
                int mx = read_mvd(&r) + (mv_ok ? pmx : 0);
                int my = read_mvd(&r) + (mv_ok ? pmy : 0);
                /* the vector lies in [-15, 15]: differences are modulo 32 */
                if (mx > 15)
                    mx -= 32;
                else if (mx < -15)
                    mx += 32;
                if (my > 15)
                    my -= 32;
                else if (my < -15)
                    my += 32;
                m->rgi_mv[0] = mx;
                m->rgi_mv[1] = my;
                flags |= H261B_MB_MC;
                pmx = mx;
                pmy = my;
                mv_ok = 1;
            } else {
                mv_ok = 0;
            }
            if (has[4])
                flags |= H261B_MB_FILTER;
            int cbp = has[0] ? 63 : 0;
            if (has[3]) {
                cbp = match(&r, d_cbp, 64, 1);
                if (cbp < 0)
                    return -1;
                flags |= H261B_MB_COEFF;
            }
            m->i_macroblock_type_flags = flags;
            m->i_coded_block_pattern = cbp;
            for (int b = 0; b < 6; b++)
                if (cbp & H261B_CBP_BIT(b))
                    if (read_block(&r, m->rgi_tcoeff[b], has[0]))
                        return -1;
            if (r.err)
                return -1;
        }
    }
    if (r.err)
        return -1;
    return (r.pos + 7) & ~(int64_t)7;
}

int64_t orc_decode_stream(const uint8_t *bits, int64_t nbytes, int32_t fmad, uint8_t *recon_out, int32_t max_frames,
                          h261_macroblock_t *mbs_out, int32_t *frames, int32_t *width, int32_t *height)
{
    static h261_macroblock_t mbs[396];
    int64_t pos = 0;
    int32_t n = 0, w0 = 0, h0 = 0;
    uint8_t *ref = NULL;
    while (pos + 32 <= nbytes * 8 && n < max_frames) {
        int32_t w, h, tr;
        const int64_t next = orc_parse_picture(bits, nbytes, pos, &w, &h, &tr, mbs, 396);
        if (next < 0)
            return -1 - n;
        if (n == 0) {
            w0 = w;
            h0 = h;
        } else if (w != w0 || h != h0) {
            return -1 - n;
        }
        const size_t fs = (size_t)w * h * 3 / 2, ny = (size_t)w * h, nc = ny / 4;
        uint8_t *out = recon_out + (size_t)n * fs;
        /* the first reference is black (h261_main.c:155-157) */
        static uint8_t black[352 * 288 * 3 / 2];
        const uint8_t *rp = n == 0 ? black : ref;
        orc_frame_t rf = { rp, rp + ny, rp + ny + nc };
        orc_frame_out_t of = { out, out + ny, out + ny + nc };
        orc_decode_frame(&rf, w, h, mbs, fmad, &of);
        if (mbs_out)
            memcpy(mbs_out + (size_t)n * (w / 16) * (h / 16), mbs, sizeof(h261_macroblock_t) * (size_t)(w / 16) * (h / 16));
        ref = out;
        pos = next;
        n++;
    }
    *frames = n;
    *width = w0;
    *height = h0;
    return pos >> 3;
}

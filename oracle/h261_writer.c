/*
 * h261_writer.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference encoder's bitstream syntax and rate
 * control, the checker for the device bitstream writer and the device rate
 * control of libh261b.so:
 *
 *   picture layer     src/h261_picture.c:83-148   (PSC, TR, PTYPE, PEI)
 *   GOB layer         src/h261_gob.c:6-199        (GOB order, MBA, MV
 *                                                  predictor, GQUANT state)
 *   macroblock layer  src/h261_macroblock.c:5-262 (MTYPE, MQUANT, MVD,
 *                                                  CBP, TCOEFF, EOB)
 *   bit writer        src/h261_bitstream.c:28-76  (MSB first, last byte
 *                                                  zero-padded)
 *   rate control      src/h261_ratectrl.c:4-245   (6-bit fixed point)
 *
 * The variable-length code tables are those of ITU-T H.261 (Tables 1-5 of
 * the standard), which src/h261_tables.c also holds; they have to be the
 * same bit for bit, so the values below are the standard's.  The TCOEFF
 * table holds exactly the standard's run/level pairs: a pair outside it is
 * sent with the 20-bit escape, as src/h261_macroblock.c:55-70 does.
 */
#include "h261_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ bit writer */

typedef struct {
    uint8_t *buf;
    int64_t cap_bits;
    int64_t pos;
    int overflow;
} bitw_t;

static void put(bitw_t *b, uint32_t code, int32_t len)
{
    for (int32_t i = len - 1; i >= 0; i--) {
        if (b->pos >= b->cap_bits) {
            b->overflow = 1;
            return;
        }
        if ((code >> i) & 1u)
            b->buf[b->pos >> 3] |= (uint8_t)(0x80u >> (b->pos & 7));
        b->pos++;
    }
}

/* ---------------------------------------------------------------- tables */

/* MBA, address increment 1..33: (code, length) */
static const uint8_t k_mba[34][2] = {
    { 0, 0 },
    { 1, 1 },   { 3, 3 },   { 2, 3 },   { 3, 4 },   { 2, 4 },   { 3, 5 },   { 2, 5 },
    { 7, 7 },   { 6, 7 },   { 11, 8 },  { 10, 8 },  { 9, 8 },   { 8, 8 },   { 7, 8 },
    { 6, 8 },   { 23, 10 }, { 22, 10 }, { 21, 10 }, { 20, 10 }, { 19, 10 }, { 18, 10 },
    { 35, 11 }, { 34, 11 }, { 33, 11 }, { 32, 11 }, { 31, 11 }, { 30, 11 }, { 29, 11 },
    { 28, 11 }, { 27, 11 }, { 26, 11 }, { 25, 11 }, { 24, 11 },
};

/* MTYPE: every code is a 1 after (length - 1) zeros; index = the reference's
 * macroblock type numbering (src/h261_types.h:15-24) */
enum {
    MT_INTRA = 0, MT_INTRA_MQ, MT_INTER, MT_INTER_MQ, MT_MC, MT_MC_CBP, MT_MC_CBP_MQ,
    MT_MC_FIL, MT_MC_FIL_CBP, MT_MC_FIL_CBP_MQ
};
static const uint8_t k_mtype_len[10] = { 4, 7, 1, 5, 9, 8, 10, 3, 2, 6 };

/* MVD by magnitude 1..16 of the (wrapped) difference: code of the negative
 * value and length; the positive value's code is one less */
static const uint8_t k_mvd_mag[17][2] = {
    { 1, 1 },   { 3, 3 },   { 3, 4 },   { 3, 5 },   { 7, 7 },   { 11, 8 },  { 9, 8 },
    { 7, 8 },   { 23, 10 }, { 21, 10 }, { 19, 10 }, { 35, 11 }, { 33, 11 }, { 31, 11 },
    { 29, 11 }, { 27, 11 }, { 25, 11 },
};

/* CBP 1..63: (code, length) */
static const uint8_t k_cbp[64][2] = {
    { 0, 0 },   { 11, 5 },  { 9, 5 },   { 13, 6 },  { 13, 4 },  { 23, 7 },  { 19, 7 },  { 31, 8 },
    { 12, 4 },  { 22, 7 },  { 18, 7 },  { 30, 8 },  { 19, 5 },  { 27, 8 },  { 23, 8 },  { 19, 8 },
    { 11, 4 },  { 21, 7 },  { 17, 7 },  { 29, 8 },  { 17, 5 },  { 25, 8 },  { 21, 8 },  { 17, 8 },
    { 15, 6 },  { 15, 8 },  { 13, 8 },  { 3, 9 },   { 15, 5 },  { 11, 8 },  { 7, 8 },   { 7, 9 },
    { 10, 4 },  { 20, 7 },  { 16, 7 },  { 28, 8 },  { 14, 6 },  { 14, 8 },  { 12, 8 },  { 2, 9 },
    { 16, 5 },  { 24, 8 },  { 20, 8 },  { 16, 8 },  { 14, 5 },  { 10, 8 },  { 6, 8 },   { 6, 9 },
    { 18, 5 },  { 26, 8 },  { 22, 8 },  { 18, 8 },  { 13, 5 },  { 9, 8 },   { 5, 8 },   { 5, 9 },
    { 12, 5 },  { 8, 8 },   { 4, 8 },   { 4, 9 },   { 7, 3 },   { 10, 5 },  { 8, 5 },   { 12, 6 },
};

/* TCOEFF: (code, length) without the sign bit for run 0..26, level 1..15;
 * length 0 = not in the table (escape) */
static uint8_t k_tc[27][16][2];
static int k_tc_ready;

static void tc_init(void)
{
    /* per run: the codes of levels 1, 2, ... */
    static const uint8_t r0[15][2] = { { 3, 2 }, { 4, 4 }, { 5, 5 }, { 6, 7 }, { 38, 8 }, { 33, 8 }, { 10, 10 },
                                       { 29, 12 }, { 24, 12 }, { 19, 12 }, { 16, 12 }, { 26, 13 },
                                       { 25, 13 }, { 24, 13 }, { 23, 13 } };
    static const uint8_t r1[7][2] = { { 3, 3 }, { 6, 6 }, { 37, 8 }, { 12, 10 }, { 27, 12 }, { 22, 13 }, { 21, 13 } };
    static const uint8_t r2[5][2] = { { 5, 4 }, { 4, 7 }, { 11, 10 }, { 20, 12 }, { 20, 13 } };
    static const uint8_t r3[4][2] = { { 7, 5 }, { 36, 8 }, { 28, 12 }, { 19, 13 } };
    static const uint8_t r4[3][2] = { { 6, 5 }, { 15, 10 }, { 18, 12 } };
    static const uint8_t r5[3][2] = { { 7, 6 }, { 9, 10 }, { 18, 13 } };
    static const uint8_t r6_10[5][2][2] = { { { 5, 6 }, { 30, 12 } }, { { 4, 6 }, { 21, 12 } },
                                             { { 7, 7 }, { 17, 12 } }, { { 5, 7 }, { 17, 13 } },
                                             { { 39, 8 }, { 16, 13 } } };
    /* runs 11..26, level 1 */
    static const uint8_t r11_26[16][2] = { { 35, 8 }, { 34, 8 }, { 32, 8 }, { 14, 10 }, { 13, 10 }, { 8, 10 },
                                           { 31, 12 }, { 26, 12 }, { 25, 12 }, { 23, 12 }, { 22, 12 },
                                           { 31, 13 }, { 30, 13 }, { 29, 13 }, { 28, 13 }, { 27, 13 } };
    memset(k_tc, 0, sizeof(k_tc));
    for (int l = 0; l < 15; l++)
        memcpy(k_tc[0][l + 1], r0[l], 2);
    for (int l = 0; l < 7; l++)
        memcpy(k_tc[1][l + 1], r1[l], 2);
    for (int l = 0; l < 5; l++)
        memcpy(k_tc[2][l + 1], r2[l], 2);
    for (int l = 0; l < 4; l++)
        memcpy(k_tc[3][l + 1], r3[l], 2);
    for (int l = 0; l < 3; l++) {
        memcpy(k_tc[4][l + 1], r4[l], 2);
        memcpy(k_tc[5][l + 1], r5[l], 2);
    }
    for (int r = 6; r <= 10; r++)
        for (int l = 0; l < 2; l++)
            memcpy(k_tc[r][l + 1], r6_10[r - 6][l], 2);
    for (int r = 11; r <= 26; r++)
        memcpy(k_tc[r][1], r11_26[r - 11], 2);
    k_tc_ready = 1;
}

/* transmission (zig-zag) order as raster indices, row = vertical frequency */
static const uint8_t k_zigzag[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
    12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
    35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
    58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63,
};

const uint8_t *orc_zigzag(void) { return k_zigzag; }

/* ------------------------------------------------------------ the layers */

static void put_level(bitw_t *b, int32_t run, int32_t level)
{
    const int32_t mag = level < 0 ? -level : level;
    if (run <= 26 && mag <= 15 && k_tc[run][mag][1]) {
        put(b, k_tc[run][mag][0], k_tc[run][mag][1]);
        put(b, level < 0 ? 1u : 0u, 1);
    } else {
        put(b, 1, 6);                      /* escape 0000 01 */
        put(b, (uint32_t)run, 6);
        put(b, (uint32_t)level & 0xffu, 8);
    }
}

/* one block (src/h261_macroblock.c:5-92): coefficients in raster order */
static int put_block(bitw_t *b, const int32_t *c, int intra)
{
    int32_t k = 1, run = 0;
    if (intra) {
        put(b, (uint32_t)c[0], 8);         /* the quantised DC as it is */
    } else if (c[0] == 1 || c[0] == -1) {
        put(b, 1, 1);                      /* first coefficient +-1: "1s" */
        put(b, c[0] < 0 ? 1u : 0u, 1);
    } else if (c[0] != 0) {
        k = 0;
    } else {
        run = 1;
    }
    for (; k < 64; k++) {
        const int32_t v = c[k_zigzag[k]];
        if (v) {
            put_level(b, run, v);
            run = 0;
        } else {
            run++;
        }
    }
    put(b, 2, 2);                          /* EOB */
    return run == 64 ? -1 : 0;             /* a coded inter block of zeros */
}

static void put_mvd(bitw_t *b, int32_t d)
{
    /* differences wrap modulo 32 into -16..15 */
    int32_t w = ((d + 16) & 31) - 16;
    if (w < 0)
        put(b, k_mvd_mag[-w][0], k_mvd_mag[-w][1]);
    else
        put(b, w ? k_mvd_mag[w][0] - 1u : 1u, k_mvd_mag[w][1]);
}

typedef struct {
    int32_t quant;     /* quantiser in force: GQUANT or the last MQUANT */
    int32_t mv_ok;     /* the previous MB's vector predicts this one     */
    int32_t mvx, mvy;
} gob_state_t;

static int put_macroblock(bitw_t *b, const h261_macroblock_t *m, int32_t addr, gob_state_t *s)
{
    put(b, k_mba[addr][0], k_mba[addr][1]);
    const int32_t fl = m->i_macroblock_type_flags;
    if (m->i_macroblock_type == H261B_MB_TYPE_INTRA) {
        const int mq = m->i_macroblock_quant != s->quant;
        put(b, 1, k_mtype_len[mq ? MT_INTRA_MQ : MT_INTRA]);
        if (mq)
            put(b, (uint32_t)m->i_macroblock_quant, 5);
        for (int k = 0; k < 6; k++)
            put_block(b, m->rgi_tcoeff[k], 1);
        return 0;
    }
    const int mq = m->i_macroblock_quant != s->quant && (fl & H261B_MB_COEFF);
    int mt;
    switch (fl) {
    case 1: mt = MT_MC; break;
    case 3: mt = MT_MC_FIL; break;
    case 4: mt = mq ? MT_INTER_MQ : MT_INTER; break;
    case 5: mt = mq ? MT_MC_CBP_MQ : MT_MC_CBP; break;
    case 7: mt = mq ? MT_MC_FIL_CBP_MQ : MT_MC_FIL_CBP; break;
    default: return -1;                    /* not a valid inter combination */
    }
    if (mq && (fl == 1 || fl == 3))
        return -1;
    put(b, 1, k_mtype_len[mt]);
    if (mq)
        put(b, (uint32_t)m->i_macroblock_quant, 5);
    if (fl & H261B_MB_MC) {
        put_mvd(b, m->rgi_mv[0] - (s->mv_ok ? s->mvx : 0));
        put_mvd(b, m->rgi_mv[1] - (s->mv_ok ? s->mvy : 0));
    }
    if (fl & H261B_MB_COEFF) {
        const int32_t cbp = m->i_coded_block_pattern;
        if (cbp <= 0 || cbp > 63)
            return -1;
        put(b, k_cbp[cbp][0], k_cbp[cbp][1]);
        for (int k = 0; k < 6; k++)
            if (cbp & H261B_CBP_BIT(k))
                if (put_block(b, m->rgi_tcoeff[k], 0))
                    return -1;
    }
    return 0;
}

int32_t orc_write_picture(int32_t w, int32_t h, int32_t frame_num, int32_t frame_type, int32_t quant,
                          const h261_macroblock_t *mbs, uint8_t *out, int32_t out_cap)
{
    (void)frame_type;
    if (!k_tc_ready)
        tc_init();
    const int cif = w == 352 && h == 288;
    if (!cif && !(w == 176 && h == 144))
        return -2;
    quant = quant < 1 ? 1 : quant > 31 ? 31 : quant;    /* src/h261_picture.c:102-110 */
    memset(out, 0, (size_t)out_cap);
    bitw_t b = { out, (int64_t)out_cap * 8, 0, 0 };

    /* picture header: PSC, TR, PTYPE (split screen 0, document camera 0,
     * freeze release 1, source format, HI_RES bit 1, spare 1), PEI 0 */
    put(&b, 16, 20);
    put(&b, (uint32_t)(frame_num & 31), 5);
    put(&b, 0, 1);
    put(&b, 0, 1);
    put(&b, 1, 1);
    put(&b, cif ? 1u : 0u, 1);
    put(&b, 1, 1);
    put(&b, 1, 1);
    put(&b, 0, 1);

    const int32_t ngob = cif ? 12 : 3, mbw = w / 16;
    for (int32_t g = 0; g < ngob; g++) {
        /* CIF: GOBs 1..12, two per band of 48 lines; QCIF: GOBs 1, 3, 5 */
        const int32_t number = cif ? g + 1 : 2 * g + 1;
        const int32_t x0 = cif ? (g & 1) * 11 : 0, y0 = (cif ? g >> 1 : g) * 3;
        put(&b, 1, 16);                    /* GBSC */
        put(&b, (uint32_t)number, 4);
        put(&b, (uint32_t)quant, 5);       /* GQUANT = picture QUANT */
        put(&b, 0, 1);                     /* GEI */
        gob_state_t s = { quant, 0, 0, 0 };
        int32_t addr = 0;
        for (int32_t i = 0; i < 33; i++) {
            const h261_macroblock_t *m = &mbs[(y0 + i / 11) * mbw + x0 + i % 11];
            addr++;
            if (i % 11 == 0)
                s.mv_ok = 0;               /* start of each MB row of the GOB */
            if (!m->i_macroblock_type_flags) {
                s.mv_ok = 0;
                continue;
            }
            if (put_macroblock(&b, m, addr, &s))
                return -3;
            addr = 0;
            if (m->i_macroblock_type_flags & H261B_MB_COEFF)
                s.quant = m->i_macroblock_quant;
            if (m->i_macroblock_type_flags & H261B_MB_MC) {
                s.mv_ok = 1;
                s.mvx = m->rgi_mv[0];
                s.mvy = m->rgi_mv[1];
            } else {
                s.mv_ok = 0;
            }
        }
    }
    if (b.overflow)
        return -1;
    return (int32_t)((b.pos + 7) >> 3);
}

/* ---------------------------------------------------------- rate control */

#define RC_BITS 6
#define RC_ONE (1 << RC_BITS)
#define RC_HALF (1 << (RC_BITS - 1))
#define RC_TIME_SCALE 1918                 /* 29.97 Hz in 6-bit fixed point */

/* round(64 * 2^(f/5)) for f = -31..31, as src/h261_ratectrl.c:11-19 */
static const int32_t k_qscale[63] = {
    0,    1,    1,    1,    1,    1,    2,    2,    2,    3,    3,    4,    4,    5,    6,    6,
    8,    9,    10,   12,   13,   16,   18,   21,   24,   27,   32,   36,   42,   48,   55,   64,
    73,   84,   97,   111,  128,  147,  168,  194,  222,  256,  294,  337,  388,  445,  512,  588,
    675,  776,  891,  1024, 1176, 1351, 1552, 1782, 2048, 2352, 2702, 3104, 3565, 4096, 4705,
};

static int32_t rc_mul(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * (int64_t)b) >> RC_BITS); }
static int32_t rc_div(int32_t a, int32_t b) { return (int32_t)((((int64_t)a) << RC_BITS) / b); }
static int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }
static int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }

static int32_t qscale_of(int32_t q) { return k_qscale[imin(imax(q, 0), 31) + 31]; }

/* nearest table entry by binary search, ties to the upper one
 * (src/h261_ratectrl.c:63-104) */
static int32_t quant_delta_of(int32_t qs)
{
    int32_t pos = 31;
    for (int32_t step = 16; step; step >>= 1)
        pos += k_qscale[pos] < qs ? step : -step;
    int32_t lo, hi;
    if (k_qscale[pos] < qs) {
        lo = pos;
        hi = imin(pos + 1, 62);
    } else {
        lo = imax(0, pos - 1);
        hi = pos;
    }
    return (qs - k_qscale[lo] < k_qscale[hi] - qs ? lo : hi) - 31;
}

void orc_rc_init(orc_rc_t *rc, int32_t quant, int32_t bitrate, int32_t vbv_size)
{
    memset(rc, 0, sizeof(*rc));
    rc->current_quant = quant;
    for (int k = 0; k < 2; k++) {
        rc->prediction_cost[k] = 100;
        rc->prediction_size[k] = 1;
    }
    rc->bitrate = bitrate / 8;
    rc->vbv_size = vbv_size / 8;
    rc->vbv_fill = rc->vbv_size;
}

int32_t orc_rc_picture_quant(orc_rc_t *rc, int32_t frame_type, int32_t picture_cost, int32_t num_mb)
{
    /* src/h261_ratectrl.c:225-245: the picture cost, at least 100 per MB */
    rc->current_picture_cost = imax(picture_cost, num_mb * 100);

    /* src/h261_ratectrl.c:144-195 */
    rc->vbv_fill = imin(rc->vbv_fill + rc_div(rc->bitrate, RC_TIME_SCALE), rc->vbv_size);
    const int32_t cost_scale = rc_div(rc->current_picture_cost, rc->prediction_cost[frame_type]);
    const int32_t predicted = rc_div(rc_mul(cost_scale, rc->prediction_size[frame_type]),
                                     qscale_of(rc->current_quant));
    int32_t target = rc_div(rc->bitrate, RC_TIME_SCALE);
    if (frame_type == H261B_FRAME_TYPE_INTRA)
        target *= 20;
    const int32_t up = rc_div(rc->vbv_fill, rc->vbv_size);
    const int32_t lower = target - rc_mul(target, RC_ONE - up);
    /* the reference clamps the prediction into [lower, upper] and then
     * overwrites the result with max(lower, 10) */
    target = imax(lower, 10);
    int32_t scale = rc_div(predicted, target);
    if (scale < RC_ONE)
        scale = rc_mul(RC_ONE - up, RC_ONE) + rc_mul(up, scale);
    rc->current_quant = imin(imax(rc->current_quant + quant_delta_of(scale), 1), 31);
    const int32_t q = rc->current_quant + ((RC_ONE - up) * 4 >> RC_BITS);
    return q < 1 ? 1 : q > 31 ? 31 : q;   /* h261_init_picture's clamp */
}

void orc_rc_update(orc_rc_t *rc, int32_t frame_type, int32_t quant, int32_t bytes)
{
    /* src/h261_ratectrl.c:198-222 */
    rc->prediction_cost[frame_type] = rc_mul(rc->prediction_cost[frame_type], RC_HALF) + rc->current_picture_cost;
    rc->prediction_size[frame_type] = rc_mul(rc->prediction_size[frame_type], RC_HALF) +
                                      rc_mul(bytes, qscale_of(quant));
    rc->vbv_fill -= bytes;
}

/* ------------------------------------------------------------ the stream */

/* one stream's state between pictures: the reference picture, denoise
 * offsets, rate control and picture counter (what h261_main.c keeps across
 * its frame loop, :173-271) */
struct orc_stream {
    int32_t w, h, nmb, quant, bitrate, intra_period, fmad, me_mode, frame;
    size_t fs, ny, nc;
    uint8_t *ref, *rec, *pic;
    me_gpu_mb_t *me;
    h261_mb_mode_decision_t *md;
    h261_macroblock_t *mbs;
    h261_dct_denoise_t dn;
    orc_rc_t rc;
};

/* one picture is at most 32 + 12 * 26 + 396 * 7749 bits */
#define ORC_PIC_CAP (400 * 1024)

orc_stream_t *orc_stream_open(int32_t w, int32_t h, int32_t quant, int32_t bitrate, int32_t intra_period,
                              int32_t denoise, int32_t fmad, int32_t me_mode)
{
    if (!((w == 176 && h == 144) || (w == 352 && h == 288)) || quant > 31)
        return NULL;
    orc_stream_t *s = (orc_stream_t *)calloc(1, sizeof(orc_stream_t));
    if (!s)
        return NULL;
    s->w = w;
    s->h = h;
    s->nmb = (w / 16) * (h / 16);
    s->quant = quant;
    s->bitrate = bitrate;
    s->intra_period = intra_period;
    s->fmad = fmad;
    s->me_mode = me_mode;
    s->fs = (size_t)w * h * 3 / 2;
    s->ny = (size_t)w * h;
    s->nc = s->ny / 4;
    s->ref = (uint8_t *)calloc(s->fs, 1);   /* the first reference is black */
    s->rec = (uint8_t *)calloc(s->fs, 1);
    s->pic = (uint8_t *)malloc(ORC_PIC_CAP);
    s->me = (me_gpu_mb_t *)calloc((size_t)s->nmb, sizeof(me_gpu_mb_t));
    s->md = (h261_mb_mode_decision_t *)calloc((size_t)s->nmb, sizeof(h261_mb_mode_decision_t));
    s->mbs = (h261_macroblock_t *)calloc((size_t)s->nmb, sizeof(h261_macroblock_t));
    if (!s->ref || !s->rec || !s->pic || !s->me || !s->md || !s->mbs) {
        orc_stream_close(s);
        return NULL;
    }
    orc_denoise_init(&s->dn, denoise);
    orc_rc_init(&s->rc, 10, bitrate, bitrate);
    for (int32_t i = 0; i < s->nmb; i++) {
        s->mbs[i].i_mb_x = (i % (w / 16)) * 16;
        s->mbs[i].i_mb_y = (i / (w / 16)) * 16;
    }
    return s;
}

void orc_stream_close(orc_stream_t *s)
{
    if (!s)
        return;
    free(s->ref);
    free(s->rec);
    free(s->pic);
    free(s->me);
    free(s->md);
    free(s->mbs);
    free(s);
}

int32_t orc_stream_encode(orc_stream_t *s, const uint8_t *cur, uint8_t *out, int32_t out_cap, int32_t *quant_out,
                          uint8_t *recon_out)
{
    const int32_t w = s->w, h = s->h, nmb = s->nmb, f = s->frame;
    orc_me_frame(cur, s->ref, w, h, s->me_mode, s->me, NULL);
    const int32_t ft = (f == 0 || (s->intra_period > 0 && f % s->intra_period == 0)) ? H261B_FRAME_TYPE_INTRA
                                                                                   : H261B_FRAME_TYPE_INTER;
    orc_mode_decision(s->me, nmb, ft, s->md);
    int32_t q = s->quant;
    if (s->quant <= 0) {
        int32_t cost = 0;
        for (int32_t i = 0; i < nmb; i++)
            cost += s->md[i].i_cost;
        q = orc_rc_picture_quant(&s->rc, ft, cost, nmb);
    }
    orc_frame_t c = { cur, cur + s->ny, cur + s->ny + s->nc }, r = { s->ref, s->ref + s->ny, s->ref + s->ny + s->nc };
    orc_encode_frame(&c, &r, w, h, s->md, q, &s->dn, s->fmad, s->mbs);
    const int32_t nb = orc_write_picture(w, h, f, ft, q, s->mbs, s->pic, ORC_PIC_CAP);
    if (nb < 0)
        return nb;
    if (nb > out_cap)
        return -1;
    memcpy(out, s->pic, (size_t)nb);
    if (quant_out)
        *quant_out = q;
    if (s->quant <= 0)
        orc_rc_update(&s->rc, ft, q, nb);
    orc_frame_out_t o = { s->rec, s->rec + s->ny, s->rec + s->ny + s->nc };
    orc_decode_frame(&r, w, h, s->mbs, s->fmad, &o);
    uint8_t *t = s->ref;
    s->ref = s->rec;
    s->rec = t;
    if (recon_out)
        memcpy(recon_out, s->ref, s->fs);
    s->frame++;
    return nb;
}

int64_t orc_encode_stream(const uint8_t *yuv, int32_t w, int32_t h, int32_t nframes, int32_t quant,
                          int32_t bitrate, int32_t intra_period, int32_t denoise, int32_t fmad,
                          int32_t me_mode, uint8_t *bits, int64_t bits_cap, int32_t *frame_bytes,
                          int32_t *frame_quant, uint8_t *recon_out)
{
    orc_stream_t *s = orc_stream_open(w, h, quant, bitrate, intra_period, denoise, fmad, me_mode);
    if (!s)
        return -2;
    int64_t total = 0;
    for (int32_t f = 0; f < nframes; f++) {
        const int64_t room = bits_cap - total;
        int32_t q = 0;
        const int32_t nb = orc_stream_encode(s, yuv + (size_t)f * s->fs, bits + total,
                                             room > ORC_PIC_CAP ? ORC_PIC_CAP : (int32_t)room, &q,
                                             recon_out ? recon_out + (size_t)f * s->fs : NULL);
        if (nb < 0) {
            total = nb;
            break;
        }
        total += nb;
        if (frame_bytes)
            frame_bytes[f] = nb;
        if (frame_quant)
            frame_quant[f] = q;
    }
    orc_stream_close(s);
    return total;
}

/* ------------------------------------------------------------------ PSNR */

/* per-plane PSNR of a reconstruction, as src/h261_main.c:38-91 computes it */
void orc_psnr(const uint8_t *orig, const uint8_t *recon, int32_t w, int32_t h, uint64_t ssd[3], double psnr[3])
{
    const size_t ny = (size_t)w * h, nc = ny / 4;
    const size_t off[3] = { 0, ny, ny + nc }, n[3] = { ny, nc, nc };
    for (int c = 0; c < 3; c++) {
        uint64_t e = 0;
        for (size_t i = 0; i < n[c]; i++) {
            const uint32_t d = (uint32_t)orig[off[c] + i] - (uint32_t)recon[off[c] + i];
            e += (uint64_t)(d * d);
        }
        const int32_t px = c == 0 ? w : w / 2, py = c == 0 ? h : h / 2;
        ssd[c] = e;
        psnr[c] = e == 0 ? 100.0 : 10 * log10(255.0 * 255.0 * (px * py) / (double)e);
    }
}

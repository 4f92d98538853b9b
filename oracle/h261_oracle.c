/*
 * h261_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU restatement of the
 * reference's device path.  See h261_oracle.h for its role and limits.
 *
 * Build with -ffp-contract=off (oracle/Makefile does): every float and
 * double operation below must round exactly where the C source rounds.
 * Citations are file:line inside rwillenbacher/h261enc_cuda.
 */
#include "h261_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MIN(a, b) ((a) < (b) ? (a) : (b))
#define MAX(a, b) ((a) > (b) ? (a) : (b))

/* ------------------------------------------------------------------ ME */

void orc_mv_limits(int32_t mbw, int32_t mbh, int8_t *lim)
{
    /* gpu_device.cu:226-265: keep the 16x16 block inside the frame and the
     * vector within +-15 */
    const int32_t gmax_x = (mbw - 1) * 16, gmax_y = (mbh - 1) * 16;
    for (int32_t y = 0; y < mbh; y++)
        for (int32_t x = 0; x < mbw; x++) {
            int32_t bx = x * 16, by = y * 16;
            int8_t *l = lim + (size_t)(x + y * mbw) * 4;
            l[0] = (int8_t)(MAX(bx - 15, 0) - bx);
            l[1] = (int8_t)(MIN(bx + 15, gmax_x) - bx);
            l[2] = (int8_t)(MAX(by - 15, 0) - by);
            l[3] = (int8_t)(MIN(by + 15, gmax_y) - by);
        }
}

int32_t orc_sad16(const uint8_t *cur, const uint8_t *ref, int32_t stride,
                  int32_t cx, int32_t cy, int32_t rx, int32_t ry)
{
    /* megpu_kernels.cuh:3-21 */
    int32_t sad = 0;
    for (int32_t j = 0; j < 16; j++)
        for (int32_t i = 0; i < 16; i++) {
            int32_t d = (int32_t)cur[(cy + j) * stride + cx + i] - (int32_t)ref[(ry + j) * stride + rx + i];
            sad += d < 0 ? -d : d;
        }
    return sad;
}

void orc_tree_reduce(int32_t D, uint32_t *cost, int8_t *vx, int8_t *vy)
{
    /* megpu_kernels.cuh:95-154 (stage 1) and :375-434 (stage 2): every cell
     * in parallel takes the best of itself, right, below and diagonal at the
     * current stride, strict '<' in that order; strides 1, 2, 4, ... < D */
    uint32_t *nc = (uint32_t *)malloc(sizeof(uint32_t) * D * D);
    int8_t *nx = (int8_t *)malloc((size_t)D * D), *ny = (int8_t *)malloc((size_t)D * D);
    for (int32_t s = 1; s < D; s *= 2) {
        for (int32_t ty = 0; ty < D; ty++)
            for (int32_t tx = 0; tx < D; tx++) {
                int32_t i = ty * D + tx;
                uint32_t best = cost[i];
                int8_t bx = vx[i], by = vy[i];
                const int32_t cand[3][2] = { { tx + s, ty }, { tx, ty + s }, { tx + s, ty + s } };
                for (int k = 0; k < 3; k++) {
                    int32_t cx = cand[k][0], cy = cand[k][1];
                    if (cx < D && cy < D) {
                        int32_t j = cy * D + cx;
                        if (cost[j] < best) {
                            best = cost[j];
                            bx = vx[j];
                            by = vy[j];
                        }
                    }
                }
                nc[i] = best;
                nx[i] = bx;
                ny[i] = by;
            }
        memcpy(cost, nc, sizeof(uint32_t) * D * D);
        memcpy(vx, nx, (size_t)D * D);
        memcpy(vy, ny, (size_t)D * D);
    }
    free(nc);
    free(nx);
    free(ny);
}

int32_t orc_satd4x4(const int16_t d[16])
{
    /* megpu_kernels.cuh:467-500: unnormalised Hadamard, sum of |.| */
    int32_t t[4][4], satd = 0;
    for (int i = 0; i < 4; i++) {
        const int16_t *r = d + 4 * i;
        int32_t a1 = r[0] + r[1], a2 = r[0] - r[1], a3 = r[2] + r[3], a4 = r[2] - r[3];
        t[i][0] = a1 + a3;
        t[i][1] = a2 + a4;
        t[i][2] = a1 - a3;
        t[i][3] = a2 - a4;
    }
    for (int i = 0; i < 4; i++) {
        int32_t a1 = t[0][i] + t[1][i], a2 = t[0][i] - t[1][i];
        int32_t a3 = t[2][i] + t[3][i], a4 = t[2][i] - t[3][i];
        satd += abs(a1 + a3) + abs(a2 + a4) + abs(a1 - a3) + abs(a2 - a4);
    }
    return satd;
}

static const int8_t k_stage1[11] = { -14, -11, -8, -5, -2, 0, 2, 5, 8, 11, 14 };
static const int8_t k_stage2[7] = { -3, -2, -1, 0, 1, 2, 3 };

static int in_limits(const int8_t *l, int32_t x, int32_t y)
{
    /* the skip test of megpu_kernels.cuh:67-83 */
    return !(x < l[0] || x > l[1] || y < l[2] || y > l[3]);
}

static void grid_search(const uint8_t *cur, const uint8_t *ref, int32_t w, int32_t bx, int32_t by,
                        const int8_t *lim, int32_t D, const int8_t *tv, int32_t ox, int32_t oy,
                        int8_t *rx, int8_t *ry)
{
    uint32_t *cost = (uint32_t *)malloc(sizeof(uint32_t) * D * D);
    int8_t *vx = (int8_t *)malloc((size_t)D * D), *vy = (int8_t *)malloc((size_t)D * D);
    for (int32_t ty = 0; ty < D; ty++)
        for (int32_t tx = 0; tx < D; tx++) {
            int32_t x = tv[tx] + ox, y = tv[ty] + oy, i = ty * D + tx;
            vx[i] = (int8_t)x;
            vy[i] = (int8_t)y;
            /* UInt16 cost, 65535 for a skipped candidate */
            cost[i] = in_limits(lim, x, y) ? (uint16_t)orc_sad16(cur, ref, w, bx, by, bx + x, by + y) : 65535u;
        }
    orc_tree_reduce(D, cost, vx, vy);
    *rx = vx[0];
    *ry = vy[0];
    free(cost);
    free(vx);
    free(vy);
}

static int32_t eval_cost(const uint8_t *cur, const uint8_t *ref, int32_t w, int32_t bx, int32_t by,
                         int32_t mvx, int32_t mvy, int32_t kind)
{
    /* kind 0: inter (megpu_kernels.cuh:617-721); 1: inter with the 3x3
     * interior filter (:724-905); 2: intra (:907-987) */
    int32_t total = 0;
    for (int32_t sy = 0; sy < 4; sy++)
        for (int32_t sx = 0; sx < 4; sx++) {
            int16_t d[16];
            for (int32_t iy = 0; iy < 4; iy++)
                for (int32_t ix = 0; ix < 4; ix++) {
                    int32_t px = bx + sx * 4 + ix, py = by + sy * 4 + iy;
                    int32_t c = cur[py * w + px];
                    if (kind == 2) {
                        d[iy * 4 + ix] = (int16_t)c;
                        continue;
                    }
                    int32_t rx = px + mvx, ry = py + mvy, p;
                    /* the filtered positions are the 6x6 interior of each
                     * 8x8 block (threadIdx parity test, :833-853) */
                    int32_t lx = (sx & 1) * 4 + ix, ly = (sy & 1) * 4 + iy;
                    if (kind == 1 && lx >= 1 && lx <= 6 && ly >= 1 && ly <= 6) {
                        const uint8_t *r0 = ref + (ry - 1) * w + rx;
                        const uint8_t *r1 = r0 + w, *r2 = r1 + w;
                        p = (r0[-1] + 2 * r0[0] + r0[1] + 2 * r1[-1] + 4 * r1[0] + 2 * r1[1] +
                             r2[-1] + 2 * r2[0] + r2[1] + 8) / 16;
                    } else {
                        p = ref[ry * w + rx];
                    }
                    d[iy * 4 + ix] = (int16_t)(c - p);
                }
            total += orc_satd4x4(d);
        }
    return total;
}

void orc_me_frame(const uint8_t *cur_y, const uint8_t *ref_y, int32_t w, int32_t h,
                  int32_t mode, me_gpu_mb_t *out, me_gpu_mv_t *stage1)
{
    const int32_t mbw = w / 16, mbh = h / 16;
    int8_t *lim = (int8_t *)malloc((size_t)mbw * mbh * 4);
    orc_mv_limits(mbw, mbh, lim);
    for (int32_t my = 0; my < mbh; my++)
        for (int32_t mx = 0; mx < mbw; mx++) {
            int32_t idx = my * mbw + mx, bx = mx * 16, by = my * 16;
            const int8_t *l = lim + (size_t)idx * 4;
            int8_t vx, vy;
            if (mode == ORC_ME_FULL) {
                int8_t tv[31];
                for (int k = 0; k < 31; k++)
                    tv[k] = (int8_t)(k - 15);
                grid_search(cur_y, ref_y, w, bx, by, l, 31, tv, 0, 0, &vx, &vy);
            } else {
                int8_t v1x, v1y;
                grid_search(cur_y, ref_y, w, bx, by, l, 11, k_stage1, 0, 0, &v1x, &v1y);
                if (stage1) {
                    stage1[idx].i8_mx = v1x;
                    stage1[idx].i8_my = v1y;
                }
                grid_search(cur_y, ref_y, w, bx, by, l, 7, k_stage2, v1x, v1y, &vx, &vy);
            }
            me_gpu_mb_t *o = &out[idx];
            o->i_intra_cost = eval_cost(cur_y, ref_y, w, bx, by, 0, 0, 2);
            o->i_zero_cost = 0;
            o->i_16x16_cost = eval_cost(cur_y, ref_y, w, bx, by, vx, vy, 0);
            o->i_16x16_filter_cost = eval_cost(cur_y, ref_y, w, bx, by, vx, vy, 1);
            o->s_16x16_mv.i8_mx = vx;
            o->s_16x16_mv.i8_my = vy;
        }
    free(lim);
}

/* ------------------------------------------------------- mode decision */

void orc_mode_decision(const me_gpu_mb_t *me, int32_t nmb, int32_t frame_type,
                       h261_mb_mode_decision_t *md)
{
    /* h261_moded.c:42-100 (the quant-adjust block at :106-122 is commented
     * out in the reference, so i_quantiser_adjust stays as initialised: 0) */
    for (int32_t i = 0; i < nmb; i++) {
        const me_gpu_mb_t *g = &me[i];
        h261_mb_mode_decision_t *m = &md[i];
        int intra = frame_type == H261B_FRAME_TYPE_INTRA ||
                    (g->i_intra_cost <= g->i_16x16_cost && g->i_intra_cost <= g->i_16x16_filter_cost);
        m->i_quantiser_adjust = 0;
        if (intra) {
            m->i_mb_type = H261B_MB_TYPE_INTRA;
            m->i_cost = g->i_intra_cost;
            m->i_mb_flags = 0;
            m->i_mv_x = m->i_mv_y = 0;
        } else {
            m->i_mb_type = H261B_MB_TYPE_INTER;
            if (g->i_16x16_filter_cost < g->i_16x16_cost) {
                m->i_mb_flags = H261B_MB_MC | H261B_MB_FILTER;
                m->i_cost = g->i_16x16_filter_cost;
            } else {
                m->i_mb_flags = 0;
                m->i_cost = g->i_16x16_cost;
            }
            m->i_mv_x = g->s_16x16_mv.i8_mx;
            m->i_mv_y = g->s_16x16_mv.i8_my;
            if (m->i_mv_x != 0 || m->i_mv_y != 0)
                m->i_mb_flags |= H261B_MB_MC;
        }
    }
}

/* ------------------------------------------------------------ transforms */

/* float tables initialised from double literals, as the reference's
 * __constant__ arrays are (mbgpu_kernels.cuh:335, :823) */
static const float k_fwd_post[8] = { 1.0, 0.720960, 0.765367, 0.850430, 1.0, 1.272759, 1.847759, 3.624510 };
static const float k_inv_pre[8] = { 1.0, 1.387040, 1.306563, 1.175876, 1.0, 0.785695, 0.541196, 0.275899 };

/* a double multiply feeding a double add: one rounding when fused */
static double mul_add(double a, double b, double c, int32_t fmad)
{
    if (fmad)
        return fma(a, b, c);
    double p = a * b;
    return p + c;
}

static float dmulf(float x, double k)
{
    /* `float *= double literal`: product in double, rounded to float */
    return (float)((double)x * k);
}

static int32_t fdct_out(float cs, float post, float v)
{
    /* floorf( (cs * post * v) + 0.49999 ): the float product is widened,
     * the double sum is rounded back to float by floorf's float argument */
    float prod = (cs * post) * v;
    double s = (double)prod + 0.49999;
    return (int32_t)floorf((float)s);
}

void orc_fdct8x8(const int32_t in[64], int32_t out[64], int32_t fmad)
{
    /* mbgpu_kernels.cuh:337-442 (AAN forward DCT) */
    float T[64];
    for (int r = 0; r < 8; r++) {
        const int32_t *s = in + 8 * r;
        float tmp0 = (float)(s[0] + s[7]), tmp1 = (float)(s[1] + s[6]);
        float tmp2 = (float)(s[2] + s[5]), tmp3 = (float)(s[3] + s[4]);
        float tmp4 = (float)(s[3] - s[4]), tmp5 = (float)(s[2] - s[5]);
        float tmp6 = (float)(s[1] - s[6]), tmp7 = (float)(s[0] - s[7]);
        float tmp10 = tmp0 + tmp3, tmp13 = tmp0 - tmp3, tmp11 = tmp1 + tmp2, tmp12 = tmp1 - tmp2;
        float *o = T + 8 * r;
        o[0] = tmp10 + tmp11;
        o[4] = tmp10 - tmp11;
        float z1 = tmp12 + tmp13;
        z1 = dmulf(z1, 0.707107);
        o[2] = tmp13 + z1;
        o[6] = tmp13 - z1;
        tmp4 = tmp4 + tmp5;
        tmp5 = tmp5 + tmp6;
        tmp6 = tmp6 + tmp7;
        float z5 = dmulf(tmp4 - tmp6, 0.382683);
        float z2 = (float)mul_add((double)tmp4, 0.541196, (double)z5, fmad);
        float z4 = (float)mul_add((double)tmp6, 1.306563, (double)z5, fmad);
        float z3 = dmulf(tmp5, 0.707107);
        float z11 = tmp7 + z3, z13 = tmp7 - z3;
        o[5] = z13 + z2;
        o[3] = z13 - z2;
        o[1] = z11 + z4;
        o[7] = z11 - z4;
    }
    for (int c = 0; c < 8; c++) {
        const float *p = T + c;
        float cs = dmulf(k_fwd_post[c], 0.125);
        float tmp0 = p[0] + p[56], tmp1 = p[8] + p[48], tmp2 = p[16] + p[40], tmp3 = p[24] + p[32];
        float tmp4 = p[24] - p[32], tmp5 = p[16] - p[40], tmp6 = p[8] - p[48], tmp7 = p[0] - p[56];
        float tmp10 = tmp0 + tmp3, tmp13 = tmp0 - tmp3, tmp11 = tmp1 + tmp2, tmp12 = tmp1 - tmp2;
        out[0 * 8 + c] = fdct_out(cs, k_fwd_post[0], tmp10 + tmp11);
        out[4 * 8 + c] = fdct_out(cs, k_fwd_post[4], tmp10 - tmp11);
        float z1 = dmulf(tmp12 + tmp13, 0.707107);
        out[2 * 8 + c] = fdct_out(cs, k_fwd_post[2], tmp13 + z1);
        out[6 * 8 + c] = fdct_out(cs, k_fwd_post[6], tmp13 - z1);
        tmp4 = tmp4 + tmp5;
        tmp5 = tmp5 + tmp6;
        tmp6 = tmp6 + tmp7;
        float z5 = dmulf(tmp4 - tmp6, 0.382683);
        float z2 = (float)mul_add((double)tmp4, 0.541196, (double)z5, fmad);
        float z4 = (float)mul_add((double)tmp6, 1.306563, (double)z5, fmad);
        float z3 = dmulf(tmp5, 0.707107);
        float z11 = tmp7 + z3, z13 = tmp7 - z3;
        out[5 * 8 + c] = fdct_out(cs, k_fwd_post[5], z13 + z2);
        out[3 * 8 + c] = fdct_out(cs, k_fwd_post[3], z13 - z2);
        out[1 * 8 + c] = fdct_out(cs, k_fwd_post[1], z11 + z4);
        out[7 * 8 + c] = fdct_out(cs, k_fwd_post[7], z11 - z4);
    }
}

static int32_t idct_out(float v)
{
    /* CLAMP_255( (Int32) floor( v + 0.49999 ) ), v a float sum widened */
    int32_t r = (int32_t)floor((double)v + 0.49999);
    return MIN(255, MAX(-256, r));
}

void orc_idct8x8(const int32_t in[64], int32_t out[64], int32_t fmad)
{
    /* mbgpu_kernels.cuh:827-931 (AAN inverse DCT).  Prescale products
     * t = (c * pre[col]) * (pre[row] * 0.125) feed the first adds of the
     * column pass.  nvcc's default -fmad=true fuses the left-hand product of
     * each of those adds into one FFMA (the product rounds once, with the
     * sum); pinned against the reference's own B200 build, whose
     * reconstructions differ from its -fmad=false build exactly there. */
    float W[64], P[64], cs[8];
    for (int r = 0; r < 8; r++) {
        cs[r] = dmulf(k_inv_pre[r], 0.125);
        for (int j = 0; j < 8; j++) {
            P[r * 8 + j] = (float)in[r * 8 + j] * k_inv_pre[j];
            W[r * 8 + j] = P[r * 8 + j] * cs[r];
        }
    }
    for (int u = 0; u < 8; u++) {
        float *p = W + u;
        const float *q = P + u;
        /* x + y with x = q[8a] * cs[a], y = p[8b] */
#define FIRST(a, b, sgn) (fmad ? fmaf(q[8 * (a)], cs[a], (sgn)*p[8 * (b)]) : p[8 * (a)] + (sgn)*p[8 * (b)])
        float tmp12 = FIRST(2, 6, -1.0f), tmp13 = FIRST(2, 6, 1.0f);
        tmp12 = dmulf(tmp12, 1.414214);
        tmp12 = tmp12 - tmp13;
        float tmp10 = FIRST(0, 4, 1.0f), tmp11 = FIRST(0, 4, -1.0f);
        float tmp0 = tmp10 + tmp13, tmp1 = tmp11 + tmp12, tmp2 = tmp11 - tmp12, tmp3 = tmp10 - tmp13;
        float z11 = FIRST(1, 7, 1.0f), z12 = FIRST(1, 7, -1.0f), z13 = FIRST(5, 3, 1.0f), z10 = FIRST(5, 3, -1.0f);
#undef FIRST
        tmp13 = z11 + z13;
        tmp11 = dmulf(z11 - z13, 1.414214);
        float z5 = dmulf(z12 + z10, 1.84776);
        tmp10 = (float)mul_add((double)z12, 1.082392, -(double)z5, fmad);
        tmp12 = (float)mul_add((double)z10, -2.613126, (double)z5, fmad);
        tmp12 = tmp12 - tmp13;
        tmp11 = tmp11 - tmp12;
        tmp10 = tmp10 + tmp11;
        p[0] = tmp0 + tmp13;
        p[8] = tmp1 + tmp12;
        p[16] = tmp2 + tmp11;
        p[24] = tmp3 - tmp10;
        p[32] = tmp3 + tmp10;
        p[40] = tmp2 - tmp11;
        p[48] = tmp1 - tmp12;
        p[56] = tmp0 - tmp13;
    }
    for (int r = 0; r < 8; r++) {
        const float *p = W + 8 * r;
        int32_t *o = out + 8 * r;
        float tmp13 = p[2] + p[6], tmp12 = p[2] - p[6];
        tmp12 = dmulf(tmp12, 1.414214);
        tmp12 = tmp12 - tmp13;
        float tmp10 = p[0] + p[4], tmp11 = p[0] - p[4];
        float tmp0 = tmp10 + tmp13, tmp1 = tmp11 + tmp12, tmp2 = tmp11 - tmp12, tmp3 = tmp10 - tmp13;
        float z11 = p[1] + p[7], z12 = p[1] - p[7], z13 = p[5] + p[3], z10 = p[5] - p[3];
        tmp13 = z11 + z13;
        tmp11 = dmulf(z11 - z13, 1.414214);
        float z5 = dmulf(z12 + z10, 1.84776);
        tmp10 = (float)mul_add((double)z12, 1.082392, -(double)z5, fmad);
        tmp12 = (float)mul_add((double)z10, -2.613126, (double)z5, fmad);
        tmp12 = tmp12 - tmp13;
        tmp11 = tmp11 - tmp12;
        tmp10 = tmp10 + tmp11;
        o[0] = idct_out(tmp0 + tmp13);
        o[1] = idct_out(tmp1 + tmp12);
        o[2] = idct_out(tmp2 + tmp11);
        o[3] = idct_out(tmp3 - tmp10);
        o[4] = idct_out(tmp3 + tmp10);
        o[5] = idct_out(tmp2 - tmp11);
        o[6] = idct_out(tmp1 - tmp12);
        o[7] = idct_out(tmp0 - tmp13);
    }
}

/* --------------------------------------------------------- loop filter */

void orc_loop_filter_hv(const uint8_t *p, int32_t stride, int32_t x, int32_t y, int32_t out[64])
{
    /* mbgpu_kernels.cuh:84-149: horizontal [1 2 1] (edge columns x4), then
     * vertical with (s+2)>>2 on the edge rows and (s+8)>>4 inside */
    int32_t t[64];
    for (int j = 0; j < 8; j++) {
        const uint8_t *r = p + (size_t)(y + j) * stride + x;
        t[j * 8 + 0] = r[0] * 4;
        for (int i = 1; i < 7; i++)
            t[j * 8 + i] = r[i - 1] + r[i] * 2 + r[i + 1];
        t[j * 8 + 7] = r[7] * 4;
    }
    for (int i = 0; i < 8; i++) {
        out[0 * 8 + i] = (t[0 * 8 + i] + 2) >> 2;
        for (int j = 1; j < 7; j++)
            out[j * 8 + i] = (t[(j - 1) * 8 + i] + t[j * 8 + i] * 2 + t[(j + 1) * 8 + i] + 8) >> 4;
        out[7 * 8 + i] = (t[7 * 8 + i] + 2) >> 2;
    }
}

void orc_loop_filter_vh(const uint8_t *p, int32_t stride, int32_t x, int32_t y, int32_t out[64])
{
    /* mbgpu_kernels.cuh:1015-1080: vertical first, then horizontal */
    int32_t t[64];
    for (int i = 0; i < 8; i++) {
        const uint8_t *c = p + (size_t)y * stride + x + i;
        t[0 * 8 + i] = c[0] * 4;
        for (int j = 1; j < 7; j++)
            t[j * 8 + i] = c[(j - 1) * stride] + c[j * stride] * 2 + c[(j + 1) * stride];
        t[7 * 8 + i] = c[7 * stride] * 4;
    }
    for (int j = 0; j < 8; j++) {
        out[j * 8 + 0] = (t[j * 8 + 0] + 2) >> 2;
        for (int i = 1; i < 7; i++)
            out[j * 8 + i] = (t[j * 8 + i - 1] + t[j * 8 + i] * 2 + t[j * 8 + i + 1] + 8) >> 4;
        out[j * 8 + 7] = (t[j * 8 + 7] + 2) >> 2;
    }
}

/* -------------------------------------------------------------- encode */

float orc_inv_quant(int32_t quant)
{
    /* f_inv_quant = 1.0 / ( float ) ( i_quant * 2 ): double division,
     * rounded to float on assignment */
    return (float)(1.0 / (double)(float)(quant * 2));
}

void orc_denoise_init(h261_dct_denoise_t *dn, int32_t denoise)
{
    memset(dn, 0, sizeof(*dn));
    dn->i_denoise = denoise;
}

/* block b of a MB: plane, stride, position and (luma or halved) vector */
static void block_geometry(int32_t b, int32_t w, int32_t mb_x, int32_t mb_y, int32_t mvx, int32_t mvy,
                           int32_t *stride, int32_t *px, int32_t *py, int32_t *bmx, int32_t *bmy)
{
    if (b < 4) {
        /* mbgpu_kernels.cuh:216-219 */
        *stride = w;
        *px = mb_x + (b & 1) * 8;
        *py = mb_y + ((b & 2) >> 1) * 8;
        *bmx = mvx;
        *bmy = mvy;
    } else {
        /* mbgpu_kernels.cuh:266-269: C division truncates toward zero */
        *stride = w / 2;
        *px = mb_x / 2;
        *py = mb_y / 2;
        *bmx = mvx / 2;
        *bmy = mvy / 2;
    }
}

static const uint8_t *plane_of(const orc_frame_t *f, int32_t b)
{
    return b < 4 ? f->y : b == 4 ? f->cb : f->cr;
}

void orc_encode_frame(const orc_frame_t *cur, const orc_frame_t *ref, int32_t w, int32_t h,
                      const h261_mb_mode_decision_t *md, int32_t pic_quant,
                      h261_dct_denoise_t *dn, int32_t fmad, h261_macroblock_t *mbs)
{
    const int32_t nmb = (w / 16) * (h / 16);
    /* offsets of this frame, as the denoise kernel loads them: UInt16
     * (mbgpu_kernels.cuh:513, :525-529) */
    uint16_t off[2][64];
    for (int i = 0; i < 64; i++) {
        off[0][i] = (uint16_t)dn->rgi_intra_signal_offset[i];
        off[1][i] = (uint16_t)dn->rgi_inter_signal_offset[i];
    }
    for (int32_t m = 0; m < nmb; m++) {
        const h261_mb_mode_decision_t *d = &md[m];
        h261_macroblock_t *mb = &mbs[m];
        /* gpu_device.cu:614-629 and mbgpu_kernels.cuh:205-212 */
        int32_t q = pic_quant + d->i_quantiser_adjust;
        q = MIN(31, MAX(1, q));
        mb->i_macroblock_type = d->i_mb_type;
        mb->i_macroblock_type_flags = d->i_mb_flags;
        mb->i_macroblock_quant = q;
        mb->rgi_mv[0] = d->i_mv_x;
        mb->rgi_mv[1] = d->i_mv_y;
        mb->i_coded_block_pattern = 0; /* the intended semantics of :676-679 */
        const int intra = d->i_mb_type == H261B_MB_TYPE_INTRA;
        const float inv = orc_inv_quant(q);
        for (int32_t b = 0; b < 6; b++) {
            int32_t stride, px, py, bmx, bmy;
            block_geometry(b, w, mb->i_mb_x, mb->i_mb_y, d->i_mv_x, d->i_mv_y, &stride, &px, &py, &bmx, &bmy);
            const uint8_t *cp = plane_of(cur, b), *rp = plane_of(ref, b);
            int32_t res[64], coef[64];
            /* setup: mbgpu_kernels.cuh:59-166 */
            if (intra) {
                for (int j = 0; j < 8; j++)
                    for (int i = 0; i < 8; i++)
                        res[j * 8 + i] = cp[(py + j) * stride + px + i];
            } else if (d->i_mb_type == H261B_MB_TYPE_INTER) {
                int32_t pred[64];
                if (d->i_mb_flags & H261B_MB_FILTER) {
                    orc_loop_filter_hv(rp, stride, px + bmx, py + bmy, pred);
                } else {
                    for (int j = 0; j < 8; j++)
                        for (int i = 0; i < 8; i++)
                            pred[j * 8 + i] = rp[(py + bmy + j) * stride + px + bmx + i];
                }
                for (int j = 0; j < 8; j++)
                    for (int i = 0; i < 8; i++)
                        res[j * 8 + i] = cp[(py + j) * stride + px + i] - pred[j * 8 + i];
            } else {
                memset(res, 0, sizeof(res));
            }
            orc_fdct8x8(res, coef, fmad);

            /* denoise: mbgpu_kernels.cuh:538-636 -- statistics of the
             * unshrunk magnitudes, shrink by this frame's offsets */
            int32_t t = intra ? 0 : 1;
            if (intra)
                dn->i_intra_count += 1;
            else
                dn->i_inter_count += 1;
            for (int i = 0; i < 64; i++) {
                int32_t lv = coef[i], sign = lv >> 31;
                lv = (lv ^ sign) - sign;
                if (intra)
                    dn->rgi_intra_noise[i] += lv;
                else
                    dn->rgi_inter_noise[i] += lv;
                lv -= off[t][i];
                lv = MAX(lv, 0);
                coef[i] = (lv ^ sign) - sign;
            }

            /* quant: mbgpu_kernels.cuh:685-722 */
            int32_t *lev = mb->rgi_tcoeff[b], acc = 0, start = 0;
            if (intra) {
                int32_t dc = coef[0] / 8;
                dc = MAX(dc, 1);
                dc = MIN(dc, 254);
                if (dc == 128)
                    dc = 255;
                lev[0] = dc;
                acc = 100;
                start = 1;
            }
            for (int i = start; i < 64; i++) {
                float f = (float)coef[i] * inv;
                int32_t l = MIN(127, MAX(-127, (int32_t)f));
                lev[i] = l;
                l = abs(l);
                acc += l > 1 ? 100 : l;
            }
            if (acc > 2) {
                mb->i_coded_block_pattern |= H261B_CBP_BIT(b);
                mb->i_macroblock_type_flags |= H261B_MB_COEFF;
            }
        }
    }
    /* update for the next frame: mbgpu_kernels.cuh:478-503 */
    for (int i = 0; i < 64; i++) {
        dn->rgi_inter_signal_offset[i] =
            (dn->i_inter_count * dn->i_denoise + dn->rgi_inter_noise[i] / 2) / (dn->rgi_inter_noise[i] + 1);
        dn->rgi_intra_signal_offset[i] =
            (dn->i_intra_count * dn->i_denoise + dn->rgi_intra_noise[i] / 2) / (dn->rgi_intra_noise[i] + 1);
        dn->rgi_inter_noise[i] = 0;
        dn->rgi_intra_noise[i] = 0;
    }
    dn->i_inter_count = 0;
    dn->i_intra_count = 0;
}

/* -------------------------------------------------------------- decode */

void orc_decode_frame(const orc_frame_t *ref, int32_t w, int32_t h,
                      const h261_macroblock_t *mbs, int32_t fmad, orc_frame_out_t *recon)
{
    const int32_t nmb = (w / 16) * (h / 16);
    for (int32_t m = 0; m < nmb; m++) {
        const h261_macroblock_t *mb = &mbs[m];
        const int intra = mb->i_macroblock_type == H261B_MB_TYPE_INTRA;
        for (int32_t b = 0; b < 6; b++) {
            /* dequant: mbgpu_kernels.cuh:763-814 */
            int32_t q = mb->i_macroblock_quant, add = (q - 1) | 1, mul = q * 2;
            const int coded = (mb->i_coded_block_pattern & H261B_CBP_BIT(b)) != 0;
            if (!coded)
                add = mul = 0;
            int32_t deq[64], res[64], start = 0;
            const int32_t *lev = mb->rgi_tcoeff[b];
            if (intra) {
                deq[0] = lev[0] == 255 ? 1024 : lev[0] * 8;
                start = 1;
            }
            for (int i = start; i < 64; i++) {
                int32_t l = lev[i] * mul;
                if (l > 0)
                    l += add;
                else if (l < 0)
                    l -= add;
                deq[i] = MIN(2047, MAX(-2048, l));
            }
            /* idct only for coded blocks (mbgpu_kernels.cuh:966-978) */
            if (coded)
                orc_idct8x8(deq, res, fmad);
            else
                memcpy(res, deq, sizeof(res));

            /* reconstruct: mbgpu_kernels.cuh:988-1096, 1130-1157, 1194-1218 */
            int32_t stride, px, py, bmx, bmy;
            block_geometry(b, w, mb->i_mb_x, mb->i_mb_y, mb->rgi_mv[0], mb->rgi_mv[1], &stride, &px, &py, &bmx, &bmy);
            uint8_t *dst = b < 4 ? recon->y : b == 4 ? recon->cb : recon->cr;
            const uint8_t *rp = b < 4 ? ref->y : b == 4 ? ref->cb : ref->cr;
            int32_t pred[64];
            if (intra) {
                memset(pred, 0, sizeof(pred));
            } else if (mb->i_macroblock_type_flags & H261B_MB_FILTER) {
                orc_loop_filter_vh(rp, stride, px + bmx, py + bmy, pred);
            } else {
                for (int j = 0; j < 8; j++)
                    for (int i = 0; i < 8; i++)
                        pred[j * 8 + i] = rp[(py + bmy + j) * stride + px + bmx + i];
            }
            if (!intra && mb->i_macroblock_type != H261B_MB_TYPE_INTER)
                continue;
            for (int j = 0; j < 8; j++)
                for (int i = 0; i < 8; i++) {
                    int32_t v = res[j * 8 + i] + pred[j * 8 + i];
                    dst[(py + j) * stride + px + i] = (uint8_t)MIN(255, MAX(0, v));
                }
        }
    }
}

/* ------------------------------------------------------------ sequence */

int32_t orc_encode_sequence(const uint8_t *yuv, int32_t w, int32_t h, int32_t nframes, int32_t quant,
                            int32_t intra_period, int32_t denoise, int32_t fmad, int32_t me_mode,
                            uint8_t *recon_out, h261_macroblock_t *mbs_out, me_gpu_mb_t *me_out,
                            h261_mb_mode_decision_t *md_out)
{
    /* the per-frame order of the reference's main (src/h261_main.c:302-400)
     * with a fixed QUANT: the first reference picture is black, only the
     * device-side steps, no bitstream */
    if (w < 16 || h < 16 || (w & 15) || (h & 15) || quant < 1 || quant > 31)
        return -1;
    const int32_t nmb = (w / 16) * (h / 16);
    const size_t fs = (size_t)w * h * 3 / 2, ny = (size_t)w * h, nc = ny / 4;
    uint8_t *ref = (uint8_t *)calloc(fs, 1), *rec = (uint8_t *)calloc(fs, 1);
    me_gpu_mb_t *me = (me_gpu_mb_t *)calloc((size_t)nmb, sizeof(me_gpu_mb_t));
    h261_mb_mode_decision_t *md = (h261_mb_mode_decision_t *)calloc((size_t)nmb, sizeof(*md));
    h261_macroblock_t *mbs = (h261_macroblock_t *)calloc((size_t)nmb, sizeof(h261_macroblock_t));
    h261_dct_denoise_t dn;
    orc_denoise_init(&dn, denoise);
    for (int32_t i = 0; i < nmb; i++) {
        mbs[i].i_mb_x = (i % (w / 16)) * 16;
        mbs[i].i_mb_y = (i / (w / 16)) * 16;
    }
    for (int32_t f = 0; f < nframes; f++) {
        const uint8_t *cur = yuv + (size_t)f * fs;
        orc_me_frame(cur, ref, w, h, me_mode, me, NULL);
        const int32_t ft = (f == 0 || (intra_period > 0 && f % intra_period == 0)) ? H261B_FRAME_TYPE_INTRA
                                                                                 : H261B_FRAME_TYPE_INTER;
        orc_mode_decision(me, nmb, ft, md);
        orc_frame_t c = { cur, cur + ny, cur + ny + nc }, r = { ref, ref + ny, ref + ny + nc };
        orc_encode_frame(&c, &r, w, h, md, quant, &dn, fmad, mbs);
        orc_frame_out_t o = { rec, rec + ny, rec + ny + nc };
        orc_decode_frame(&r, w, h, mbs, fmad, &o);
        memcpy(ref, rec, fs);
        if (recon_out)
            memcpy(recon_out + (size_t)f * fs, rec, fs);
        if (mbs_out)
            memcpy(mbs_out + (size_t)f * nmb, mbs, sizeof(h261_macroblock_t) * nmb);
        if (me_out)
            memcpy(me_out + (size_t)f * nmb, me, sizeof(me_gpu_mb_t) * nmb);
        if (md_out)
            memcpy(md_out + (size_t)f * nmb, md, sizeof(*md) * nmb);
    }
    free(ref);
    free(rec);
    free(me);
    free(md);
    free(mbs);
    return nmb * nframes;
}

/*
 * oracle_abi.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The sixteen gpu_device.h entry points (src/gpu_device.h:7-32) implemented
 * on the CPU over the oracle, with the reference's process-global,
 * single-encoder state model (src/gpu_device.cu:26-42).  Linked into the
 * oracle flavour of the frame-loop driver so that the reference's unchanged
 * host code can produce an oracle bitstream.
 *
 * Environment: H261_ORACLE_FMAD=0|1 (default 1) selects fused or separately
 * rounded double multiply-adds in the transforms; H261_ORACLE_ME=full
 * selects the exhaustive search extension.
 */
#include "h261_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static struct {
    int32_t w, h;
    uint8_t *cur[3], *ref[3];
    int32_t fmad, me_mode;
} g;

void h261_gpu_init(void)
{
    const char *f = getenv("H261_ORACLE_FMAD");
    const char *m = getenv("H261_ORACLE_ME");
    g.fmad = f ? atoi(f) : 1;
    g.me_mode = (m && strcmp(m, "full") == 0) ? ORC_ME_FULL : ORC_ME_REFERENCE;
}

void h261_gpu_device_init_textures(int32_t w, int32_t h)
{
    g.w = w;
    g.h = h;
    for (int p = 0; p < 3; p++) {
        size_t n = p ? (size_t)(w / 2) * (h / 2) : (size_t)w * h;
        g.cur[p] = (uint8_t *)calloc(n, 1);
        g.ref[p] = (uint8_t *)calloc(n, 1);
    }
}

void h261_gpu_device_deinit_textures(void)
{
    for (int p = 0; p < 3; p++) {
        free(g.cur[p]);
        free(g.ref[p]);
        g.cur[p] = g.ref[p] = NULL;
    }
}

static void put(uint8_t *dst, const uint8_t *src, int32_t w, int32_t h)
{
    memcpy(dst, src, (size_t)w * h);
}

void h261_gpu_device_set_current(uint8_t *d, int32_t w, int32_t h) { put(g.cur[0], d, w, h); }
void h261_gpu_device_set_current_chroma_cb(uint8_t *d, int32_t w, int32_t h) { put(g.cur[1], d, w, h); }
void h261_gpu_device_set_current_chroma_cr(uint8_t *d, int32_t w, int32_t h) { put(g.cur[2], d, w, h); }
void h261_gpu_device_set_reference(uint8_t *d, int32_t w, int32_t h) { put(g.ref[0], d, w, h); }
void h261_gpu_device_set_reference_chroma_cb(uint8_t *d, int32_t w, int32_t h) { put(g.ref[1], d, w, h); }
void h261_gpu_device_set_reference_chroma_cr(uint8_t *d, int32_t w, int32_t h) { put(g.ref[2], d, w, h); }

void h261_gpu_device_init_me(me_gpu_t **pps, int32_t w, int32_t h)
{
    me_gpu_t *s = (me_gpu_t *)calloc(1, sizeof(*s));
    s->i_mb_width = w / 16;
    s->i_mb_height = h / 16;
    s->i_num_mb = s->i_mb_width * s->i_mb_height;
    s->prgs_macroblocks_result = (me_gpu_mb_t *)calloc(s->i_num_mb, sizeof(me_gpu_mb_t));
    s->ps_starting_vector_host = (me_gpu_mv_t *)calloc(s->i_num_mb, sizeof(me_gpu_mv_t));
    s->ps_candidate_vector_host = (me_gpu_mv_t *)calloc(s->i_num_mb, sizeof(me_gpu_mv_t));
    s->pi8_motion_vector_limits_host = (int8_t *)calloc(s->i_num_mb, 4);
    orc_mv_limits(s->i_mb_width, s->i_mb_height, s->pi8_motion_vector_limits_host);
    *pps = s;
}

void h261_gpu_device_deinit_me(me_gpu_t **pps)
{
    me_gpu_t *s = *pps;
    free(s->prgs_macroblocks_result);
    free(s->ps_starting_vector_host);
    free(s->ps_candidate_vector_host);
    free(s->pi8_motion_vector_limits_host);
    free(s);
    *pps = NULL;
}

void h261_gpu_device_me(me_gpu_t *s)
{
    orc_me_frame(g.cur[0], g.ref[0], g.w, g.h, g.me_mode, s->prgs_macroblocks_result,
                 g.me_mode == ORC_ME_REFERENCE ? s->ps_starting_vector_host : NULL);
}

void h261_init_macroblocks(h261_macroblocks_t **pps, int32_t w, int32_t h, int32_t denoise)
{
    h261_macroblocks_t *s = (h261_macroblocks_t *)calloc(1, sizeof(*s));
    s->i_mb_width = w / 16;
    s->i_mb_height = h / 16;
    s->i_num_mb = s->i_mb_width * s->i_mb_height;
    s->ps_macroblocks = (h261_macroblock_t *)calloc(s->i_num_mb, sizeof(h261_macroblock_t));
    for (int32_t y = 0; y < s->i_mb_height; y++)
        for (int32_t x = 0; x < s->i_mb_width; x++) {
            s->ps_macroblocks[y * s->i_mb_width + x].i_mb_x = x * 16;
            s->ps_macroblocks[y * s->i_mb_width + x].i_mb_y = y * 16;
        }
    s->ps_denoise_host = (h261_dct_denoise_t *)calloc(1, sizeof(h261_dct_denoise_t));
    orc_denoise_init(s->ps_denoise_host, denoise);
    s->pui8_reconstructed_Y_host = (uint8_t *)calloc((size_t)s->i_num_mb, 256);
    s->pui8_reconstructed_Cb_host = (uint8_t *)calloc((size_t)s->i_num_mb, 256);
    s->pui8_reconstructed_Cr_host = (uint8_t *)calloc((size_t)s->i_num_mb, 256);
    *pps = s;
}

void h261_deinit_macroblocks(h261_macroblocks_t *s)
{
    free(s->ps_macroblocks);
    free(s->ps_denoise_host);
    free(s->pui8_reconstructed_Y_host);
    free(s->pui8_reconstructed_Cb_host);
    free(s->pui8_reconstructed_Cr_host);
    free(s);
}

void h261_gpu_device_encode_macroblocks(h261_context_t *ctx)
{
    h261_macroblocks_t *s = ctx->ps_macroblocks;
    orc_frame_t cur = { g.cur[0], g.cur[1], g.cur[2] }, ref = { g.ref[0], g.ref[1], g.ref[2] };
    orc_encode_frame(&cur, &ref, g.w, g.h, ctx->ps_mode_decision->prgs_mb, ctx->s_picture.i_quantiser,
                     s->ps_denoise_host, g.fmad, s->ps_macroblocks);
}

void h261_gpu_device_decode_macroblocks(h261_context_t *ctx)
{
    h261_macroblocks_t *s = ctx->ps_macroblocks;
    orc_frame_t ref = { g.ref[0], g.ref[1], g.ref[2] };
    orc_frame_out_t rec = { s->pui8_reconstructed_Y_host, s->pui8_reconstructed_Cb_host,
                            s->pui8_reconstructed_Cr_host };
    orc_decode_frame(&ref, g.w, g.h, s->ps_macroblocks, g.fmad, &rec);
}

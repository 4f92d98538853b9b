/*
 * ref_writer.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Lets a test turn one frame of macroblock results (levels, CBP, types,
 * vectors, as produced by any encode core) into H.261 bytes with the
 * reference's own, unchanged picture / GOB / macroblock writers
 * (src/h261_picture.c:6-71, src/h261_gob.c:6-199, src/h261_macroblock.c).
 * Built with those sources into _ref/libh261ref_writer.so.
 */
#include "h261_decl.h"

#include <string.h>

static h261_context_t g_ctx;
static h261_macroblocks_t g_mbs;
static int g_ready;

/* Returns the number of bytes written to out, or -1 if out is too small. */
Int32 ref_write_picture(Int32 w, Int32 h, Int32 frame_num, Int32 frame_type, Int32 quant,
                        h261_macroblock_t *mbs, UInt8 *out, Int32 out_cap)
{
    if (!g_ready) {
        h261_bitstream_init(&g_ctx.s_bitstream, 0x100000);
        g_ready = 1;
    }
    h261_picture_parameters_t pp;
    memset(&pp, 0, sizeof(pp));
    g_ctx.i_source_format = w == 352 ? H261_SOURCE_FORMAT_CIF : H261_SOURCE_FORMAT_QCIF;
    pp.i_frame_num = frame_num;
    pp.i_source_format = g_ctx.i_source_format;
    pp.i_frame_type = frame_type;
    pp.i_quantiser = quant;
    h261_init_picture(&g_ctx, &pp);
    g_mbs.i_mb_width = w / 16;
    g_mbs.i_mb_height = h / 16;
    g_mbs.i_num_mb = g_mbs.i_mb_width * g_mbs.i_mb_height;
    g_mbs.ps_macroblocks = mbs;
    g_ctx.ps_macroblocks = &g_mbs;
    h261_bitstream_reset(&g_ctx.s_bitstream);
    h261_write_picture_header(&g_ctx);
    h261_write_gobs(&g_ctx);
    UInt8 *bytes;
    UInt32 len;
    h261_bitstream_get(&g_ctx.s_bitstream, &bytes, &len);
    if ((Int32)len > out_cap)
        return -1;
    memcpy(out, bytes, len);
    return (Int32)len;
}

/*
 * ref_driver.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A frame-loop driver written for this project that runs the reference
 * encoder's own, unchanged host code (src/h261_moded.c, h261_ratectrl.c,
 * h261_picture.c, h261_gob.c, h261_macroblock.c, h261_bitstream.c,
 * h261_tables.c, compiled from the reference sources by oracle/Makefile)
 * on top of one of three implementations of the gpu_device.h boundary:
 *
 *   h261_drive_oracle   the CPU oracle (oracle_abi.c)
 *   h261_drive_refgpu   the reference's own src/gpu_device.cu, sm_100a
 *   h261_drive_ours     libh261b.so, the B200 core of this project
 *
 * It follows the per-frame call order of the reference's main
 * (src/h261_main.c:302-400) and adds what that main lacks: QCIF, a fixed
 * QUANT, an intra period and a per-frame dump of every value that crosses
 * the boundary, so that the three builds can be compared byte for byte.
 *
 * usage: h261_drive in=<yuv> w=<W> h=<H> frames=<N> bits=<out.h261>
 *                   recon=<out.yuv> dump=<out.bin>
 *                   [quant=<1..31> | bitrate=<bit/s>] [intra=<period>]
 *                   [denoise=<d>] [timing=<out.txt>]
 *
 * timing= writes the milliseconds each picture took from its upload to its
 * reconstruction (the boundary calls and the host mode decision, rate
 * control and writers, not the file reads and dumps), one line per picture.
 *
 * Dump record per frame (little endian):
 *   "H261FRM1", int32 frame, frame_type, picture_quant, num_mb, bytes,
 *   me_gpu_mb_t[num_mb] (i_zero_cost written as 0: the reference never
 *   computes it), h261_mb_mode_decision_t[num_mb], h261_macroblock_t[num_mb]
 */
#include "h261_decl.h"

#include <string.h>
#include <time.h>

double h261_get_time()
{
    /* POSIX stand-in for the reference's Win32 timer (src/sys_win32.c:6-26) */
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec * 1000.0 + (double)ts.tv_nsec / 1.0e6;
}

static const char *arg(int argc, char **argv, const char *key, const char *def)
{
    size_t n = strlen(key);
    for (int i = 1; i < argc; i++)
        if (strncmp(argv[i], key, n) == 0 && argv[i][n] == '=')
            return argv[i] + n + 1;
    return def;
}

static void alloc_frame(h261_frame_t *f, Int32 w, Int32 h)
{
    f->i_width = w;
    f->i_height = h;
    f->i_stride_y = w;
    f->i_stride_c = w / 2;
    f->pui8_Y = calloc((size_t)w * h, 1);
    f->pui8_Cb = calloc((size_t)w * h / 4, 1);
    f->pui8_Cr = calloc((size_t)w * h / 4, 1);
}

int main(int argc, char **argv)
{
    const char *in_path = arg(argc, argv, "in", NULL);
    const char *bits_path = arg(argc, argv, "bits", NULL);
    const char *recon_path = arg(argc, argv, "recon", NULL);
    const char *dump_path = arg(argc, argv, "dump", NULL);
    Int32 w = atoi(arg(argc, argv, "w", "176"));
    Int32 h = atoi(arg(argc, argv, "h", "144"));
    Int32 frames = atoi(arg(argc, argv, "frames", "1"));
    Int32 quant = atoi(arg(argc, argv, "quant", "0"));
    Int32 bitrate = atoi(arg(argc, argv, "bitrate", "384000"));
    Int32 intra_period = atoi(arg(argc, argv, "intra", "0"));
    Int32 denoise = atoi(arg(argc, argv, "denoise", "5"));
    const char *timing_path = arg(argc, argv, "timing", NULL);
    FILE *ftime = timing_path ? fopen(timing_path, "w") : NULL;
    if (!in_path || !bits_path || !recon_path || !dump_path ||
        !((w == 176 && h == 144) || (w == 352 && h == 288))) {
        fprintf(stderr, "usage: h261_drive in= w= h= frames= bits= recon= dump= [quant=|bitrate=] [intra=] [denoise=]\n");
        return 2;
    }
    FILE *fin = fopen(in_path, "rb"), *fbits = fopen(bits_path, "wb");
    FILE *frec = fopen(recon_path, "wb"), *fdump = fopen(dump_path, "wb");
    if (!fin || !fbits || !frec || !fdump) {
        fprintf(stderr, "h261_drive: cannot open files\n");
        return 3;
    }

    h261_context_t *ctx = calloc(1, sizeof(h261_context_t));
    ctx->i_source_format = w == 352 ? H261_SOURCE_FORMAT_CIF : H261_SOURCE_FORMAT_QCIF;
    alloc_frame(&ctx->s_current_frame, w, h);
    alloc_frame(&ctx->s_reference_frame, w, h);
    h261_bitstream_init(&ctx->s_bitstream, 0x100000);

    me_gpu_t *me;
    h261_mode_decision_t *md;
    h261_macroblocks_t *mbs;
    h261_gpu_init();
    h261_gpu_device_init_textures(w, h);
    h261_init_macroblocks(&mbs, w, h, denoise);
    h261_gpu_device_init_me(&me, w, h);
    h261_init_mode_decision(&md, me->i_mb_width, me->i_mb_height);
    if (quant <= 0)
        h261_init_ratectrl(ctx, 10, bitrate, bitrate, H261_RATECTRL_MODE_CBR);

    const Int32 fsize = w * h, nmb = me->i_num_mb;
    h261_frame_t *src = &ctx->s_current_frame, *ref = &ctx->s_reference_frame;
    int status = 0;
    for (Int32 f = 0; f < frames; f++) {
        if (fread(src->pui8_Y, fsize, 1, fin) != 1 || fread(src->pui8_Cb, fsize / 4, 1, fin) != 1 ||
            fread(src->pui8_Cr, fsize / 4, 1, fin) != 1) {
            fprintf(stderr, "h261_drive: short input at frame %d\n", f);
            status = 4;
            break;
        }
        const double t0 = h261_get_time();
        h261_gpu_device_set_current(src->pui8_Y, w, h);
        h261_gpu_device_set_current_chroma_cb(src->pui8_Cb, w / 2, h / 2);
        h261_gpu_device_set_current_chroma_cr(src->pui8_Cr, w / 2, h / 2);
        h261_gpu_device_set_reference(ref->pui8_Y, w, h);
        h261_gpu_device_set_reference_chroma_cb(ref->pui8_Cb, w / 2, h / 2);
        h261_gpu_device_set_reference_chroma_cr(ref->pui8_Cr, w / 2, h / 2);

        h261_gpu_device_me(me);

        h261_picture_parameters_t pp;
        memset(&pp, 0, sizeof(pp));
        pp.i_frame_num = f;
        pp.i_source_format = ctx->i_source_format;
        pp.i_frame_type = (f == 0 || (intra_period > 0 && f % intra_period == 0)) ? H261_FRAME_TYPE_INTRA
                                                                                  : H261_FRAME_TYPE_INTER;
        h261_mode_decision(md, me, &pp);
        ctx->ps_mode_decision = md;
        if (quant <= 0) {
            h261_ratectrl_collect_picture_stats(ctx, &pp);
            h261_ratectrl_init_picture(ctx, &pp);
        } else {
            pp.i_quantiser = quant;
        }
        h261_init_picture(ctx, &pp);
        ctx->ps_macroblocks = mbs;
        h261_gpu_device_encode_macroblocks(ctx);

        h261_bitstream_reset(&ctx->s_bitstream);
        h261_write_picture_header(ctx);
        h261_write_gobs(ctx);

        h261_gpu_device_decode_macroblocks(ctx);

        UInt8 *bytes;
        UInt32 len;
        h261_bitstream_get(&ctx->s_bitstream, &bytes, &len);
        fwrite(bytes, len, 1, fbits);
        if (quant <= 0)
            h261_ratectrl_update_picture(ctx, (Int32)len);

        memcpy(ref->pui8_Y, mbs->pui8_reconstructed_Y_host, fsize);
        memcpy(ref->pui8_Cb, mbs->pui8_reconstructed_Cb_host, fsize / 4);
        memcpy(ref->pui8_Cr, mbs->pui8_reconstructed_Cr_host, fsize / 4);
        if (ftime)
            fprintf(ftime, "%.4f\n", h261_get_time() - t0);
        fwrite(ref->pui8_Y, fsize, 1, frec);
        fwrite(ref->pui8_Cb, fsize / 4, 1, frec);
        fwrite(ref->pui8_Cr, fsize / 4, 1, frec);

        Int32 hdr[5] = { f, pp.i_frame_type, ctx->s_picture.i_quantiser, nmb, (Int32)len };
        fwrite("H261FRM1", 8, 1, fdump);
        fwrite(hdr, sizeof(hdr), 1, fdump);
        for (Int32 i = 0; i < nmb; i++) {
            const me_gpu_mb_t *g = &me->prgs_macroblocks_result[i];
            me_gpu_mb_t r;
            memset(&r, 0, sizeof(r)); /* padding bytes too */
            r.i_intra_cost = g->i_intra_cost;
            r.i_16x16_cost = g->i_16x16_cost;
            r.i_16x16_filter_cost = g->i_16x16_filter_cost;
            r.s_16x16_mv = g->s_16x16_mv;
            fwrite(&r, sizeof(r), 1, fdump);
        }
        fwrite(md->prgs_mb, sizeof(h261_mb_mode_decision_t), nmb, fdump);
        fwrite(mbs->ps_macroblocks, sizeof(h261_macroblock_t), nmb, fdump);
        fflush(stdout);
    }
    fclose(fin);
    fclose(fbits);
    fclose(frec);
    fclose(fdump);
    if (ftime)
        fclose(ftime);
    return status;
}

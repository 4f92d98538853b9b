/*
 * h261_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement, on the CPU, of the reference encoder's device
 * path (rwillenbacher/h261enc_cuda: src/megpu_kernels.cuh,
 * src/mbgpu_kernels.cuh, src/gpu_device.cu, src/h261_moded.c).  It is the
 * checker that the CUDA core is compared against, and the CPU baseline that
 * the benchmark times beside it.  Only the tests, the smoke check and the
 * benchmark's CPU-baseline leg may load it; the encoder library never links
 * it and has no CPU fallback.
 *
 * Parity pins: the oracle is checked against outputs of the reference's
 * own CUDA code, built for sm_100a from the reference sources by
 * oracle/Makefile and run on a B200 (fixtures under tests/golden/).
 *
 * Float semantics: the reference's DCT and IDCT mix float temporaries with
 * double constants.  The oracle is compiled with -ffp-contract=off and
 * spells every double-rounding step out; `fmad` selects whether the two
 * double multiply-adds per 1-D pass are fused (one rounding, what nvcc's
 * default -fmad=true does) or rounded twice.
 */
#ifndef H261_ORACLE_H
#define H261_ORACLE_H

#include "../include/h261b_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_ME_REFERENCE 0   /* 11x11 coarse grid + 7x7 refinement        */
#define ORC_ME_FULL      1   /* every vector in [-15,15]^2 within limits  */

typedef struct {
    const uint8_t *y, *cb, *cr;  /* packed planes: stride W and W/2       */
} orc_frame_t;

typedef struct {
    uint8_t *y, *cb, *cr;
} orc_frame_out_t;

/* per-MB search limits [min_x, max_x, min_y, max_y] (gpu_device.cu:226-265) */
void orc_mv_limits(int32_t mbw, int32_t mbh, int8_t *lim);

/* 16x16 SAD (megpu_kernels.cuh:3-21) */
int32_t orc_sad16(const uint8_t *cur, const uint8_t *ref, int32_t stride,
                  int32_t cx, int32_t cy, int32_t rx, int32_t ry);

/* the 2-D tie-break tree of megpu_kernels.cuh:95-154; D x D cells, cell
 * (x, y) at index y * D + x; the winner ends in cell 0 */
void orc_tree_reduce(int32_t D, uint32_t *cost, int8_t *vx, int8_t *vy);

/* 4x4 Hadamard SATD (megpu_kernels.cuh:467-500) */
int32_t orc_satd4x4(const int16_t d[16]);

/* motion estimation of one frame: results per MB, plus the stage-1 vector
 * when stage1 != NULL (ORC_ME_REFERENCE only) */
void orc_me_frame(const uint8_t *cur_y, const uint8_t *ref_y, int32_t w, int32_t h,
                  int32_t mode, me_gpu_mb_t *out, me_gpu_mv_t *stage1);

/* h261_moded.c:31-123 */
void orc_mode_decision(const me_gpu_mb_t *me, int32_t nmb, int32_t frame_type,
                       h261_mb_mode_decision_t *md);

/* 8x8 transforms of mbgpu_kernels.cuh:337-442 and :827-931; in/out raster
 * (row = vertical frequency) */
void orc_fdct8x8(const int32_t in[64], int32_t out[64], int32_t fmad);
void orc_idct8x8(const int32_t in[64], int32_t out[64], int32_t fmad);

/* H.261 loop filter of an 8x8 block at (x, y), in the two orders the
 * reference uses (mbgpu_kernels.cuh:84-149 and :1015-1080) */
void orc_loop_filter_hv(const uint8_t *p, int32_t stride, int32_t x, int32_t y, int32_t out[64]);
void orc_loop_filter_vh(const uint8_t *p, int32_t stride, int32_t x, int32_t y, int32_t out[64]);

/* 1 / (2q) as float, computed the reference's way (mbgpu_kernels.cuh:685) */
float orc_inv_quant(int32_t quant);

/* encode one frame (mbgpu_kernels.cuh setup / dct / denoise / update /
 * quant, gpu_device.cu:614-629 packing).  mbs[] must carry i_mb_x/i_mb_y;
 * denoise state dn is updated for the next frame. */
void orc_encode_frame(const orc_frame_t *cur, const orc_frame_t *ref, int32_t w, int32_t h,
                      const h261_mb_mode_decision_t *md, int32_t pic_quant,
                      h261_dct_denoise_t *dn, int32_t fmad, h261_macroblock_t *mbs);

/* decode one frame (dequant / idct / reconstruct) into packed planes */
void orc_decode_frame(const orc_frame_t *ref, int32_t w, int32_t h,
                      const h261_macroblock_t *mbs, int32_t fmad, orc_frame_out_t *recon);

/* denoise state at stream start (gpu_device.cu:495-508) */
void orc_denoise_init(h261_dct_denoise_t *dn, int32_t denoise);

/* whole fixed-QUANT sequence (packed frames, W*H*3/2 bytes each), per-frame
 * outputs optional; returns the number of MBs encoded or -1 */
int32_t orc_encode_sequence(const uint8_t *yuv, int32_t w, int32_t h, int32_t nframes, int32_t quant,
                            int32_t intra_period, int32_t denoise, int32_t fmad, int32_t me_mode,
                            uint8_t *recon_out, h261_macroblock_t *mbs_out, me_gpu_mb_t *me_out,
                            h261_mb_mode_decision_t *md_out);

/* ---- bitstream syntax and rate control (h261_writer.c) ---- */

/* one picture in H.261 syntax from its macroblock records (QCIF or CIF):
 * src/h261_picture.c:115-148, src/h261_gob.c:6-199,
 * src/h261_macroblock.c:5-262.  Returns the byte count, -1 if out_cap is
 * too small, -2 for another picture size, -3 for records the reference
 * writer cannot write (it dereferences NULL on those). */
int32_t orc_write_picture(int32_t w, int32_t h, int32_t frame_num, int32_t frame_type, int32_t quant,
                          const h261_macroblock_t *mbs, uint8_t *out, int32_t out_cap);
/* transmission order: raster index of the k-th coefficient sent */
const uint8_t *orc_zigzag(void);

/* src/h261_ratectrl.c state (h261_ratectrl_t without the mode field) */
typedef struct {
    int32_t current_quant;
    int32_t prediction_cost[2];
    int32_t prediction_size[2];
    int32_t bitrate;              /* bytes per second   */
    int32_t vbv_size;             /* bytes              */
    int32_t vbv_fill;
    int32_t current_picture_cost;
} orc_rc_t;

void orc_rc_init(orc_rc_t *rc, int32_t quant, int32_t bitrate, int32_t vbv_size);
/* picture QUANT from the mode-decision cost sum (collect_picture_stats +
 * init_picture + h261_init_picture's clamp) */
int32_t orc_rc_picture_quant(orc_rc_t *rc, int32_t frame_type, int32_t picture_cost, int32_t num_mb);
/* after the picture: its QUANT and its size in bytes */
void orc_rc_update(orc_rc_t *rc, int32_t frame_type, int32_t quant, int32_t bytes);

/* one encode stream of the reference's frame loop (h261_main.c:173-271
 * plus an intra period), a picture at a time: fixed QUANT when quant > 0,
 * else CBR rate control started at QUANT 10 with VBV = bitrate.  The state
 * between pictures is the reference picture, denoise offsets, rate control
 * and picture counter.  orc_stream_encode writes one picture's bytes to out
 * and returns their count (-1: out_cap too small, other negatives as
 * orc_write_picture); quant_out and recon_out optional.  Streams are
 * independent: different streams may be encoded on different threads. */
typedef struct orc_stream orc_stream_t;
orc_stream_t *orc_stream_open(int32_t w, int32_t h, int32_t quant, int32_t bitrate, int32_t intra_period,
                              int32_t denoise, int32_t fmad, int32_t me_mode);
int32_t orc_stream_encode(orc_stream_t *s, const uint8_t *picture, uint8_t *out, int32_t out_cap,
                          int32_t *quant_out, uint8_t *recon_out);
void orc_stream_close(orc_stream_t *s);

/* the reference encoder's whole frame loop (h261_main.c:178-275 plus an
 * intra period): fixed QUANT when quant > 0, else CBR rate control started
 * at QUANT 10 with VBV = bitrate.  Writes the concatenated pictures to bits
 * (capacity bits_cap) and per picture its byte count and QUANT; recon_out
 * optional.  Returns the total byte count, or a negative status. */
int64_t orc_encode_stream(const uint8_t *yuv, int32_t w, int32_t h, int32_t nframes, int32_t quant,
                          int32_t bitrate, int32_t intra_period, int32_t denoise, int32_t fmad,
                          int32_t me_mode, uint8_t *bits, int64_t bits_cap, int32_t *frame_bytes,
                          int32_t *frame_quant, uint8_t *recon_out);

/* per-plane squared error and PSNR of a reconstruction (packed planes), as
 * src/h261_main.c:38-91 computes them */
void orc_psnr(const uint8_t *orig, const uint8_t *recon, int32_t w, int32_t h, uint64_t ssd[3], double psnr[3]);

/* ---- conformance decoder (h261_decoder.c) ---- */

/* parse one picture from bit `pos`: its records (raster MB order), format,
 * temporal reference; returns the byte-aligned bit position after it or -1 */
int64_t orc_parse_picture(const uint8_t *bits, int64_t nbytes, int64_t pos, int32_t *w, int32_t *h,
                          int32_t *tr, h261_macroblock_t *mbs, int32_t mbs_cap);
/* decode a whole stream (black first reference, pictures of one format) into
 * packed reconstructions; records optional.  Returns the bytes consumed or
 * -1 - (index of the picture that failed).  Not reentrant. */
int64_t orc_decode_stream(const uint8_t *bits, int64_t nbytes, int32_t fmad, uint8_t *recon_out, int32_t max_frames,
                          h261_macroblock_t *mbs_out, int32_t *frames, int32_t *width, int32_t *height);

#ifdef __cplusplus
}
#endif
#endif

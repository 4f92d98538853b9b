/*
 * h261b_abi.h -- the drop-in device boundary of the H.261 encode core.
 *
 * This header declares, in this project's own words, the exact binary
 * interface that the reference encoder's host code (picture / GOB /
 * macroblock writers, rate control, mode decision, frame loop) links
 * against.  A program built against the reference's `gpu_device.h` and
 * `h261_types.h` runs unchanged on top of libh261b.so: the sixteen entry
 * points below keep the reference's names, argument meaning and (void)
 * return convention, and every struct that crosses the boundary keeps the
 * reference's field order, types and therefore its layout on LP64.
 *
 * Reference interface replaced (paths inside the reference project):
 *   src/gpu_device.h:7-32      the entry points
 *   src/h261_types.h:46-292    the shared structs
 *
 * The layouts are pinned by static assertions at the end of this file; the
 * sizes are the ones gcc x86-64 gives for the reference's own header.
 *
 * Errors: like the reference, the entry points return nothing.  A failure
 * is printed to stderr and recorded; h261b_last_error() (declared in
 * h261b.h) returns the last recorded status.
 */
#ifndef H261B_ABI_H
#define H261B_ABI_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- constants shared with the reference host code (src/h261_types.h:2-37) */
#define H261B_FRAME_TYPE_INTRA 0
#define H261B_FRAME_TYPE_INTER 1

#define H261B_SOURCE_FORMAT_QCIF 0
#define H261B_SOURCE_FORMAT_CIF  1

#define H261B_MB_TYPE_INTRA 0
#define H261B_MB_TYPE_INTER 2

#define H261B_MB_MC     1
#define H261B_MB_FILTER 2
#define H261B_MB_COEFF  4

/* coded-block-pattern bit of block b (0..3 luma, 4 Cb, 5 Cr) is 32 >> b */
#define H261B_CBP_BIT(b) (32 >> (b))

/* SoA coefficient scratch geometry of the reference (src/h261_types.h:181-184) */
#define H261B_COEFF_BLOCK_WIDTH 16
#define H261B_COEFF_BLOCK_SIZE  (16 * 8 * 8)

/* ---- motion estimation (src/h261_types.h:46-79) ----------------------- */
typedef struct {
    int8_t i8_mx;
    int8_t i8_my;
} me_gpu_mv_t;

typedef struct {
    int32_t i_intra_cost;        /* SATD of the source MB                      */
    int32_t i_zero_cost;         /* never computed by the reference; 0 here    */
    int32_t i_16x16_cost;        /* SATD of the residual at the final vector   */
    int32_t i_16x16_filter_cost; /* same with the 3x3 interior filter          */
    me_gpu_mv_t s_16x16_mv;      /* final integer-pel vector                   */
} me_gpu_mb_t;

typedef struct me_gpu_s {
    int32_t i_mb_width;
    int32_t i_mb_height;
    int32_t i_num_mb;

    me_gpu_mb_t *prgs_macroblocks_device;
    me_gpu_mb_t *prgs_macroblocks_result;   /* host-visible results        */

    me_gpu_mv_t *ps_candidate_vector_device;
    me_gpu_mv_t *ps_candidate_vector_host;

    me_gpu_mv_t *ps_starting_vector_device;
    me_gpu_mv_t *ps_starting_vector_host;

    int8_t *pi8_motion_vector_limits_device;
    int8_t *pi8_motion_vector_limits_host;

    void *p_cuda;                            /* library-private state       */
} me_gpu_t;

/* ---- mode decision (src/h261_types.h:84-96) -------------------------- */
typedef struct {
    int32_t i_cost;
    int32_t i_quantiser_adjust;
    int32_t i_mb_type;
    int32_t i_mb_flags;
    int32_t i_mv_x, i_mv_y;
} h261_mb_mode_decision_t;

typedef struct {
    int32_t i_mb_width;
    int32_t i_mb_height;
    h261_mb_mode_decision_t *prgs_mb;
} h261_mode_decision_t;

/* ---- encoder structures (src/h261_types.h:100-292) --------------------- */
typedef struct {
    int32_t i_width;
    int32_t i_height;
    int32_t i_stride_y;
    int32_t i_stride_c;
    uint8_t *pui8_Y;
    uint8_t *pui8_Cr;
    uint8_t *pui8_Cb;
} h261_frame_t;

typedef struct {
    uint8_t *pui8_bitstream;
    int32_t i_length;
    int32_t i_byte_count;
    int32_t i_next_bit;
} h261_bitstream_t;

typedef struct {
    int32_t i_denoise;
    int32_t i_intra_count;
    int32_t rgi_intra_noise[64];
    int32_t rgi_intra_signal_offset[64];
    int32_t i_inter_count;
    int32_t rgi_inter_noise[64];
    int32_t rgi_inter_signal_offset[64];
} h261_dct_denoise_t;

typedef struct h261_macroblock_s {
    int32_t i_macroblock_address;
    int32_t i_macroblock_type;
    int32_t i_macroblock_type_flags;
    int32_t i_macroblock_quant;
    int32_t rgi_mv[2];
    int32_t i_coded_block_pattern;
    int32_t rgi_tcoeff[6][64];     /* raster order, row = vertical frequency */
    int32_t i_mb_x;                /* pel coordinates of the MB              */
    int32_t i_mb_y;
} h261_macroblock_t;

typedef struct {
    int32_t i_mb_width;
    int32_t i_mb_height;
    int32_t i_num_mb;

    h261_macroblock_t *ps_macroblocks;         /* host-visible results      */
    h261_macroblock_t *ps_macroblocks_device;

    h261_dct_denoise_t *ps_denoise_host;
    h261_dct_denoise_t *ps_denoise_device;

    int32_t *pi_mb_types_host;
    int32_t *pi_mb_types_device;
    int32_t *pi_mb_flags_host;
    int32_t *pi_mb_flags_device;
    int32_t *pi_mb_quant_host;
    int32_t *pi_mb_quant_device;
    int32_t *pi_mb_mv_x_host;
    int32_t *pi_mb_mv_x_device;
    int32_t *pi_mb_mv_y_host;
    int32_t *pi_mb_mv_y_device;

    uint8_t *pui8_reconstructed_Y_device;
    uint8_t *pui8_reconstructed_Y_host;
    uint8_t *pui8_reconstructed_Cr_device;
    uint8_t *pui8_reconstructed_Cr_host;
    uint8_t *pui8_reconstructed_Cb_device;
    uint8_t *pui8_reconstructed_Cb_host;

    int32_t i_num_blocks;
    int32_t i_num_coeff_blocks;
    int32_t *pi_coeff_blocks_device;
    int32_t *pi_coeff_blocks_host;

    void *p_cuda;                              /* library-private state     */
} h261_macroblocks_t;

typedef struct {
    int32_t i_quantiser;
    int32_t i_last_mv_valid;
    int32_t i_last_mv_x;
    int32_t i_last_mv_y;
} h261_mb_coding_vars_t;

typedef struct {
    int32_t i_group_of_blocks_start_code;
    int32_t i_group_number;
    int32_t i_quantiser;
    int32_t i_num_extra_insertion_information;
    h261_mb_coding_vars_t s_coding_vars;
} h261_gob_t;

typedef struct {
    int32_t i_picture_start_code;
    int32_t i_temporal_reference;
    int32_t i_split_screen_indicator;
    int32_t i_document_camera_indicator;
    int32_t i_freeze_picture_release;
    int32_t i_source_format;
    int32_t i_highres_mode;
    int32_t i_spare_bit;
    int32_t i_num_extra_insertion_information;
    uint8_t rgui8_extra_insertion_information[1];
    h261_gob_t s_groups_of_blocks;
    int32_t i_quantiser;                       /* read by encode            */
    int32_t i_frame_type;
} h261_picture_t;

typedef struct {
    int32_t i_ratectrl_mode;
    int32_t i_current_quant;
    int32_t i_current_picture_cost;
    int32_t i_prediction_cost[2];
    int32_t i_prediction_size[2];
    int32_t i_bitrate;
    int32_t i_vbv_size;
    int32_t i_vbv_fill;
} h261_ratectrl_t;

typedef struct {
    int32_t i_source_format;
    int32_t i_frame_counter;
    h261_frame_t s_current_frame;
    h261_frame_t s_reference_frame;
    h261_picture_t s_picture;
    h261_bitstream_t s_bitstream;
    h261_mode_decision_t *ps_mode_decision;    /* read by encode            */
    h261_ratectrl_t s_ratectrl;
    h261_macroblocks_t *ps_macroblocks;        /* read by encode / decode   */
} h261_context_t;

typedef struct {
    int32_t i_frame_num;
    int32_t i_source_format;
    int32_t i_quantiser;
    int32_t i_frame_type;
} h261_picture_parameters_t;

/* ---- the sixteen entry points (src/gpu_device.h:7-32) ------------------ */

/* src/gpu_device.h:7 -- select device 0 and set it up. */
void h261_gpu_init(void);

/* src/gpu_device.h:10-11 -- allocate / free the current and reference
 * frame planes of the default session (W x H luma, W/2 x H/2 chroma). */
void h261_gpu_device_init_textures(int32_t i_width, int32_t i_height);
void h261_gpu_device_deinit_textures(void);

/* src/gpu_device.h:13-19 -- upload one packed plane (stride = width) of the
 * current (source) picture or of the reference (previous reconstruction). */
void h261_gpu_device_set_current(uint8_t *pui8_frame_data, int32_t i_width, int32_t i_height);
void h261_gpu_device_set_current_chroma_cb(uint8_t *pui8_frame_data, int32_t i_width, int32_t i_height);
void h261_gpu_device_set_current_chroma_cr(uint8_t *pui8_frame_data, int32_t i_width, int32_t i_height);
void h261_gpu_device_set_reference(uint8_t *pui8_frame_data, int32_t i_width, int32_t i_height);
void h261_gpu_device_set_reference_chroma_cb(uint8_t *pui8_frame_data, int32_t i_width, int32_t i_height);
void h261_gpu_device_set_reference_chroma_cr(uint8_t *pui8_frame_data, int32_t i_width, int32_t i_height);

/* src/gpu_device.h:23-25 -- motion estimation.  init allocates the
 * me_gpu_t (pinned) and returns it; h261_gpu_device_me fills
 * prgs_macroblocks_result[] for every MB and returns when it is valid. */
void h261_gpu_device_init_me(me_gpu_t **pps_me_gpu, int32_t i_width, int32_t i_height);
void h261_gpu_device_deinit_me(me_gpu_t **pps_me_gpu);
void h261_gpu_device_me(me_gpu_t *ps_me_gpu);

/* src/gpu_device.h:28-29 -- macroblock coder state (pinned struct, host
 * result arrays, denoise state with strength i_denoise). */
void h261_init_macroblocks(h261_macroblocks_t **pps_mbs, int32_t i_width, int32_t i_height, int32_t i_denoise);
void h261_deinit_macroblocks(h261_macroblocks_t *ps_mbs);

/* src/gpu_device.h:31-32 -- encode: reads ps_ctx->s_picture.i_quantiser,
 * ps_ctx->ps_mode_decision and ps_ctx->ps_macroblocks and fills
 * ps_macroblocks->ps_macroblocks[] (levels, CBP, flags).  decode: fills the
 * pui8_reconstructed_{Y,Cb,Cr}_host planes with the reconstruction. */
void h261_gpu_device_encode_macroblocks(h261_context_t *ps_ctx);
void h261_gpu_device_decode_macroblocks(h261_context_t *ps_ctx);

#ifdef __cplusplus
}
#endif

/* ---- layout pins (sizes of the reference structs, gcc x86-64) ---------- */
#if defined(__cplusplus)
#define H261B_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define H261B_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
H261B_STATIC_ASSERT(sizeof(me_gpu_mv_t) == 2, "me_gpu_mv_t layout");
H261B_STATIC_ASSERT(sizeof(me_gpu_mb_t) == 20, "me_gpu_mb_t layout");
H261B_STATIC_ASSERT(sizeof(me_gpu_t) == 88, "me_gpu_t layout");
H261B_STATIC_ASSERT(sizeof(h261_mb_mode_decision_t) == 24, "mode decision layout");
H261B_STATIC_ASSERT(sizeof(h261_dct_denoise_t) == 1036, "denoise layout");
H261B_STATIC_ASSERT(sizeof(h261_macroblock_t) == 1572, "macroblock layout");
H261B_STATIC_ASSERT(offsetof(h261_macroblock_t, rgi_tcoeff) == 28, "tcoeff offset");
H261B_STATIC_ASSERT(sizeof(h261_macroblocks_t) == 208, "macroblocks layout");
H261B_STATIC_ASSERT(offsetof(h261_macroblocks_t, p_cuda) == 200, "macroblocks p_cuda");
H261B_STATIC_ASSERT(sizeof(h261_picture_t) == 80, "picture layout");
H261B_STATIC_ASSERT(offsetof(h261_picture_t, i_quantiser) == 72, "picture quant");
H261B_STATIC_ASSERT(sizeof(h261_context_t) == 248, "context layout");
H261B_STATIC_ASSERT(offsetof(h261_context_t, ps_mode_decision) == 192, "ctx md");
H261B_STATIC_ASSERT(offsetof(h261_context_t, ps_macroblocks) == 240, "ctx mbs");

#endif /* H261B_ABI_H */

/*
 * h261b_device.h -- descriptors shared by the host engine and the kernels.
 *
 * Device memory model (all in HBM, nothing re-uploaded per frame):
 *   picture   three planes; luma pitch = W, chroma pitch = W/2 rounded up
 *             to 16 bytes, every plane 256-byte aligned;
 *   session   one encode stream: a source picture per in-flight frame, two
 *             reconstruction pictures that alternate as reference / output,
 *             and its denoise state;
 *   step      one picture of every participating session; a flat list of
 *             (session, MB) work items covers the step.
 */
#ifndef H261B_DEVICE_H
#define H261B_DEVICE_H

#include <stdint.h>
#include "../../include/h261b.h"

#define H261B_MAX_MB_PER_SESSION 4096

/* per-session denoise state: the reference's h261_dct_denoise_t
 * (src/h261_types.h:122-132) split into the shrink offsets of the current
 * frame and the accumulators of the frame being coded, plus the frame-end
 * ticket.  The offsets are kept the way the reference's kernel uses them,
 * as UInt16 (mbgpu_kernels.cuh:513, :525-529), column-major so that a lane
 * holding one coefficient column reads its eight offsets with one load. */
typedef struct {
    int32_t denoise;
    uint32_t ticket;              /* MBs of the current frame published      */
    int32_t count[2];             /* blocks coded this frame: [0] intra [1] inter */
    int32_t noise[2][64];         /* sum of |coefficient| before shrinking,
                                     raster position v * 8 + u               */
    uint16_t offset[2][8][8];     /* [type][column u][row v]                */
    uint8_t reserved[256];        /* keeps the state at 1040 bytes          */
} h261b_denoise_dev_t;

/* compact per-MB result of the batched path (16 bytes) */
typedef struct {
    int16_t type;             /* H261B_MB_TYPE_INTRA / _INTER                */
    int16_t flags;            /* MC | FILTER | COEFF                          */
    int8_t quant;
    int8_t cbp;
    int8_t mvx, mvy;
    int32_t cost;             /* mode-decision cost (rate control input)     */
    int32_t coef_bits;        /* bits of its blocks in the bitstream (0 when
                                 the session writes none)                   */
} h261b_mb_info_t;

/* CBR rate control of one session (src/h261_ratectrl.c h261_ratectrl_t,
 * 6-bit fixed point), in HBM between pictures */
typedef struct {
    int32_t current_quant;
    int32_t prediction_cost[2];   /* [intra, inter]                         */
    int32_t prediction_size[2];
    int32_t bitrate;              /* bytes per second                       */
    int32_t vbv_size;             /* bytes                                  */
    int32_t vbv_fill;
    int32_t current_picture_cost;
    int32_t picture_quant;        /* QUANT of the picture in flight         */
    int32_t cost_sum;             /* its summed mode-decision costs         */
    int32_t reserved[5];
} h261b_rc_dev_t;

/* per-picture result of the bitstream writer (16 bytes) */
typedef struct {
    int32_t bytes;            /* picture size in bytes                       */
    int32_t host_off;         /* offset in the host bitstream arena, -1 when
                                 the arena was full (bytes stay in bits_out) */
    int32_t status;           /* 0, or H261B_BITS_* below                    */
    int32_t quant;            /* picture QUANT                               */
} h261b_pic_info_t;

#define H261B_BITS_BAD_RECORD  -3 /* a record the syntax cannot express      */
#define H261B_BITS_OVERFLOW    -4 /* larger than the device slot             */
#define H261B_BITS_MISMATCH    -5 /* a macroblock's size differs from the
                                     encode kernel's count (an internal error) */

/* step-wide state of the bitstream writer, in the descriptor arena (the
 * descriptor upload zeroes it every step) */
typedef struct {
    uint32_t host_used;       /* bytes of the host arena handed out          */
    uint32_t codes_next;      /* work items the codes kernel has handed out  */
    uint32_t codes_failed;    /* nonzero: a codes warp gave up waiting for a
                                 picture's MBs (the layout refuses every
                                 picture of the step)                        */
    uint32_t pad[61];
} h261b_step_dev_t;

typedef struct {
    /* pictures */
    const uint8_t *cur_y, *cur_cb, *cur_cr;
    const uint8_t *ref_y, *ref_cb, *ref_cr;
    uint8_t *rec_y, *rec_cb, *rec_cr;
    int32_t pitch_y, pitch_c;
    int32_t mbw, mbh;
    /* picture parameters */
    int32_t frame_type;       /* H261B_FRAME_TYPE_INTRA / _INTER             */
    int32_t quant;            /* picture QUANT, 1..31                         */
    int32_t me_mode;          /* 0 reference two-stage search, 1 full search */
    int32_t skip_search;      /* 1: intra picture, leave ME results unset    */
    h261b_denoise_dev_t *dn;
    /* inputs of the encode-only phase (ABI path): host mode decision */
    const h261_mb_mode_decision_t *md_in;
    /* outputs, any may be NULL */
    me_gpu_mb_t *me_out;          /* ME results per MB                      */
    me_gpu_mv_t *stage1_out;      /* stage-1 vector per MB                  */
    h261_mb_mode_decision_t *md_out;
    h261_macroblock_t *abi_out;   /* reference layout, int32 levels         */
    h261b_mb_info_t *info_out;    /* compact layout                         */
    int8_t *level_out;            /* [nmb][6][64], per block column-major
                                     ([u][v]); an intra DC stored as uint8   */
    /* bitstream of the picture (QCIF / CIF sessions that write one) */
    uint32_t *bits_out;           /* picture bytes, 16-byte aligned; NULL = no
                                     bitstream                               */
    int32_t bits_cap;             /* bytes in bits_out                       */
    int32_t frame_num;            /* temporal reference = frame_num & 31     */
    h261b_pic_info_t *pic_out;
    uint32_t *vlc_scratch;        /* per MB: its coefficient bits, MSB first,
                                     H261B_VLC_MB_WORDS words apart          */
    int32_t *vlc_pos;             /* per MB: bit position in the picture     */
    uint32_t *vlc_plan;           /* per MB: header fields                   */
    int32_t *vlc_total;           /* [0] picture bits, [1] status, [2] host
                                     arena offset, [3] MBs packed            */
    /* CBR sessions: the step's first encode launch runs search and mode
     * decision (into md_out, costs summed into rc), the rate control picks
     * the picture QUANT, a second launch encodes (md_in = md_out) */
    h261b_rc_dev_t *rc;
    /* sums of squared errors of the picture's Y, Cb, Cr reconstruction
     * (sessions that measure PSNR), zeroed before the step */
    unsigned long long *ssd_out;
    /* MBs of the picture an encoding launch has finished, zero before the
     * step: each warp adds a run's MBs after a fence, so that the codes
     * kernel (a programmatic dependent of the encode launch) may code a
     * picture as soon as its count is complete, while the encode launch
     * still works on other pictures */
    int32_t mbs_done;
} h261b_session_dev_t;

/* coefficient bits of one MB at most: six blocks of an 8-bit DC or a first
 * code, 63 escapes of 20 bits and an EOB */
#define H261B_VLC_MB_WORDS 240

/* phases a launch runs for each MB */
#define H261B_PHASE_ME      1     /* search + cost evaluation               */
#define H261B_PHASE_MD      2     /* device mode decision                   */
#define H261B_PHASE_ENCDEC  4     /* MC, FDCT, denoise, quant, IDCT, recon  */

/* the rest of h261b_launch_step's phases word:
 *   bit 8        the reference's default-build (fused) arithmetic
 *   bits 9-10    kernel kind: 0 fused (the phases above in one pass),
 *                1 search (ME + MD into md_out), 2 encode (ENCDEC from md_in)
 *   bit 11       programmatic dependent launch on the kernel before it in
 *                the stream (an encode launch right after its search launch)
 *   bits 12-15   tail items per warp drawn from the scheduler, plus one
 *                (0: the default, 2)
 */
#define H261B_FMAD_BIT      0x100
#define H261B_KIND_SHIFT    9
#define H261B_KIND_SEARCH   (1 << H261B_KIND_SHIFT)
#define H261B_KIND_ENCODE   (2 << H261B_KIND_SHIFT)
#define H261B_LAUNCH_PDL    0x800
#define H261B_TAIL_SHIFT    12
/*   bit 16       stage the search window with one bulk copy per row
 *                (cp.async.bulk, completed on a shared-memory barrier)
 *                instead of 16-byte cp.async copies */
#define H261B_STAGE_BULK    0x10000
/*   bit 17       checking build only: each warp's first bulk staging
 *                announces 16 bytes more than it copies, so that its bounded
 *                wait runs out (the test of h261b_stage_status) */
#define H261B_STAGE_SHORT   0x20000
/*   bit 18       the exhaustive +-15 search (the sessions' me_mode 1)
 *   bit 19       the launch may write the reference-layout outputs
 *                (abi_out, me_out, stage1_out: the gpu_device.h boundary) */
#define H261B_LAUNCH_ME_FULL 0x40000
#define H261B_ABI_OUT       0x80000

#ifdef __cplusplus
extern "C" {
#endif
/* host-side launchers (kernels.cu); return a cudaError_t value.
 * h261b_launch_step: sched_dev, when not null, is two int32 counters, zero
 * before the first launch and left zero by each, that balance the launch's
 * tail; one launch at a time may use them (null: static runs only). */
int h261b_launch_step(const h261b_session_dev_t *sessions_dev, const uint32_t *work_dev,
                      int32_t n_work, int32_t phases, int32_t warps_per_cta, int32_t max_ctas,
                      int32_t *sched_dev, void *stream);
int h261b_set_quant_table(void);
/* the picture QUANT of every session with rc (one thread per session) */
int h261b_launch_ratectrl(h261b_session_dev_t *sessions_dev, int32_t n_sessions, void *stream);

/* the bitstream of every work item's session that has bits_out: three
 * launches (coefficient codes and packing over the step's work list, the
 * layout per session; the CTA that packs a picture's last MBs copies it);
 * the picture ends in bits_out and in the host arena (device-mapped pinned
 * memory, host_cap bytes) at an offset drawn from step->host_used.
 * test_extra_wait > 0 (tests of the checking build only): the codes kernel
 * waits for that many MBs more than each picture has, for 2 ms, so that its
 * bounded wait runs out and the step's pictures are refused */
int h261b_launch_bitstream(h261b_session_dev_t *sessions_dev, int32_t n_sessions, const uint32_t *work_dev,
                           int32_t n_work, h261b_step_dev_t *step, uint8_t *host_arena_dev, int64_t host_cap,
                           int32_t sm_count, void *stream, void *layout_done_event, int32_t test_extra_wait);
/* device bytes per step slot a w x h session's bitstream needs: picture
 * bytes, MB scratch and offsets (0: no bitstream for this size), and where
 * each part starts in that block */
int64_t h261b_bits_slot_bytes(int32_t w, int32_t h);
typedef struct {
    int64_t picture, scratch, pos, plan, total, bytes;
} h261b_bits_layout_t;
h261b_bits_layout_t h261b_bits_layout(int32_t w, int32_t h);
#ifdef __cplusplus
}
#endif

#endif

/*
 * h261b_synth.h -- seeded synthetic YUV 4:2:0 sources for the encoder.
 *
 * The reference project ships no test material, so every workload the
 * encoder is measured or checked on is generated here from a 64-bit seed.
 * After a 4096-entry sine table is filled once (libm sin), everything is
 * integer arithmetic, so a given parameter set yields the same bytes on
 * every run of the same build.
 *
 * Content model (one stream):
 *   background  128 + sum of 8 plane waves (period 4..64 px, amplitude
 *               0..40, random orientation and phase), sampled at the
 *               accumulated pan offset;
 *   objects     N rectangles of uniform-random texture moving with
 *               integer velocities, wrapping at the frame edges;
 *   block motion (alternative model) every 16x16 block of frame t is the
 *               clean frame t-1 displaced by a per-block integer offset,
 *               clamped so the source block stays inside the frame;
 *   noise       approximately Gaussian (sum of 12 uniforms), added to the
 *               output only, so it does not accumulate;
 *   chroma      2x2 box average of the output luma, re-centred as
 *               128 + (avg - 128) / 2.
 */
#ifndef H261B_SYNTH_H
#define H261B_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define H261B_SYNTH_PAN_OBJECTS  0
#define H261B_SYNTH_BLOCK_MOTION 1

typedef struct {
    int32_t width, height;      /* 176x144 (QCIF) or 352x288 (CIF)            */
    int32_t kind;               /* H261B_SYNTH_PAN_OBJECTS / _BLOCK_MOTION     */
    uint64_t seed;
    int32_t n_objects;          /* textured rectangles                         */
    int32_t obj_min, obj_max;   /* side length range in pixels (inclusive)     */
    int32_t obj_vmax;           /* velocities uniform in [-vmax, vmax]         */
    int32_t pan_dx, pan_dy;     /* pan per frame when pan_period == 0          */
    int32_t pan_period;         /* >0: redraw the pan every pan_period frames  */
    int32_t pan_rand;           /*     uniformly from [-pan_rand, pan_rand]^2  */
    int32_t scene_cut;          /* >0: reseed the content at this frame        */
    int32_t noise_sigma16;      /* noise standard deviation in 1/16 pel        */
    int32_t block_motion_max;   /* block-motion offsets in [-max, max]         */
} h261b_synth_params_t;

typedef struct h261b_synth_s h261b_synth_t;

/* Fill *p with the preset of a named workload:
 *   0  QCIF, pan (+2,-1), 2 objects 32x32, v in [-6,6], sigma 2
 *   1  CIF, pan redrawn every 30 frames in [-8,8], 6 objects 16..64,
 *      v in [-15,15], scene cut at 150, sigma 3
 *   2  per-stream variant of 0 at the given size, pan speed in [-4,4]
 *      drawn from the seed
 *   3  QCIF block motion, offsets in [-15,15], sigma 4
 * Returns 0, or -1 for an unknown preset. */
int h261b_synth_preset(int32_t preset, int32_t width, int32_t height, uint64_t seed,
                       h261b_synth_params_t *p);

/* Create a generator; returns 0 or a negative error (bad size, no memory). */
int h261b_synth_create(const h261b_synth_params_t *p, h261b_synth_t **out);

/* Produce the next frame into packed planes (Y stride = width, chroma
 * stride = width / 2).  Returns the index of the frame produced. */
int h261b_synth_next(h261b_synth_t *s, uint8_t *y, uint8_t *cb, uint8_t *cr);

void h261b_synth_destroy(h261b_synth_t *s);

#ifdef __cplusplus
}
#endif
#endif

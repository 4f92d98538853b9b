/*
 * synth.c -- seeded synthetic 4:2:0 sources (see include/h261b_synth.h).
 *
 * Everything after the sine table is integer arithmetic with a splitmix64
 * generator, so a parameter set maps to one byte sequence.  Separate
 * generator streams drive the content layout, the pan draws, the block
 * motion and the noise, so changing one knob does not reshuffle the rest.
 */
#include "h261b_synth.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define N_WAVES 8
#define MAX_OBJECTS 16
#define LUT_BITS 12
#define LUT_SIZE (1 << LUT_BITS)

typedef struct {
    int32_t amp;        /* 0..40                                           */
    int64_t dphx, dphy; /* phase step per pixel, 2^32 = one cycle          */
    uint32_t phase0;
} wave_t;

typedef struct {
    int32_t w, h, x0, y0, vx, vy;
    uint8_t *tex;
} object_t;

struct h261b_synth_s {
    h261b_synth_params_t p;
    int32_t t;                 /* index of the next frame                   */
    int32_t t_scene;           /* first frame of the current scene          */
    int64_t pan_x, pan_y;      /* accumulated pan offset                    */
    int32_t pan_vx, pan_vy;
    uint64_t rng_noise, rng_pan, rng_motion;
    wave_t waves[N_WAVES];
    object_t obj[MAX_OBJECTS];
    int32_t n_obj;
    uint8_t *clean;            /* clean luma of the previous frame          */
    uint8_t *work;
};

static int32_t g_lut[LUT_SIZE];
static int g_lut_ready;

static uint64_t sm64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static int32_t urange(uint64_t *s, int32_t lo, int32_t hi)
{
    return lo + (int32_t)(sm64(s) % (uint64_t)(hi - lo + 1));
}

static void lut_init(void)
{
    if (g_lut_ready)
        return;
    for (int k = 0; k < LUT_SIZE; k++)
        g_lut[k] = (int32_t)floor(sin(6.283185307179586 * k / LUT_SIZE) * 65536.0 + 0.5);
    g_lut_ready = 1;
}

static int32_t wrap(int64_t v, int32_t m)
{
    int64_t r = v % m;
    return (int32_t)(r < 0 ? r + m : r);
}

static void free_objects(struct h261b_synth_s *s)
{
    for (int i = 0; i < s->n_obj; i++)
        free(s->obj[i].tex);
    s->n_obj = 0;
}

/* Draw the background waves and the objects of one scene. */
static int build_scene(struct h261b_synth_s *s, uint64_t seed)
{
    uint64_t r = seed ^ 0xC0FFEE1234567ULL;
    for (int k = 0; k < N_WAVES; k++) {
        wave_t *w = &s->waves[k];
        int32_t period = urange(&r, 4, 64);
        int32_t theta = urange(&r, 0, LUT_SIZE - 1);
        int32_t c = g_lut[(theta + LUT_SIZE / 4) & (LUT_SIZE - 1)];
        int32_t sn = g_lut[theta];
        w->amp = urange(&r, 0, 40);
        w->dphx = ((int64_t)c * 65536) / period;
        w->dphy = ((int64_t)sn * 65536) / period;
        w->phase0 = (uint32_t)sm64(&r);
    }
    free_objects(s);
    int32_t n = s->p.n_objects < MAX_OBJECTS ? s->p.n_objects : MAX_OBJECTS;
    for (int i = 0; i < n; i++) {
        object_t *o = &s->obj[i];
        o->w = urange(&r, s->p.obj_min, s->p.obj_max);
        o->h = urange(&r, s->p.obj_min, s->p.obj_max);
        o->x0 = urange(&r, 0, s->p.width - 1);
        o->y0 = urange(&r, 0, s->p.height - 1);
        o->vx = urange(&r, -s->p.obj_vmax, s->p.obj_vmax);
        o->vy = urange(&r, -s->p.obj_vmax, s->p.obj_vmax);
        o->tex = (uint8_t *)malloc((size_t)o->w * o->h);
        if (!o->tex)
            return -1;
        for (int j = 0; j < o->w * o->h; j++)
            o->tex[j] = (uint8_t)(sm64(&r) >> 56);
        s->n_obj = i + 1;
    }
    return 0;
}

static void render_scene(struct h261b_synth_s *s, uint8_t *dst)
{
    const int32_t W = s->p.width, H = s->p.height;
    for (int32_t y = 0; y < H; y++) {
        uint32_t ph[N_WAVES];
        int64_t sy = (int64_t)y + s->pan_y;
        int64_t sx0 = s->pan_x;
        for (int k = 0; k < N_WAVES; k++)
            ph[k] = s->waves[k].phase0 + (uint32_t)(sx0 * s->waves[k].dphx + sy * s->waves[k].dphy);
        for (int32_t x = 0; x < W; x++) {
            int32_t acc = 0;
            for (int k = 0; k < N_WAVES; k++) {
                acc += s->waves[k].amp * g_lut[ph[k] >> (32 - LUT_BITS)];
                ph[k] += (uint32_t)s->waves[k].dphx;
            }
            int32_t v = 128 + ((acc + 32768) >> 16);
            dst[y * W + x] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
    int32_t dt = s->t - s->t_scene;
    for (int i = 0; i < s->n_obj; i++) {
        const object_t *o = &s->obj[i];
        int32_t ox = wrap((int64_t)o->x0 + (int64_t)o->vx * dt, W);
        int32_t oy = wrap((int64_t)o->y0 + (int64_t)o->vy * dt, H);
        for (int32_t j = 0; j < o->h; j++) {
            uint8_t *row = dst + (size_t)((oy + j) % H) * W;
            for (int32_t i2 = 0; i2 < o->w; i2++)
                row[(ox + i2) % W] = o->tex[j * o->w + i2];
        }
    }
}

static void block_motion(struct h261b_synth_s *s)
{
    const int32_t W = s->p.width, H = s->p.height, m = s->p.block_motion_max;
    for (int32_t by = 0; by < H / 16; by++)
        for (int32_t bx = 0; bx < W / 16; bx++) {
            int32_t dx = urange(&s->rng_motion, -m, m);
            int32_t dy = urange(&s->rng_motion, -m, m);
            int32_t sx = bx * 16 + dx, sy = by * 16 + dy;
            sx = sx < 0 ? 0 : sx > W - 16 ? W - 16 : sx;
            sy = sy < 0 ? 0 : sy > H - 16 ? H - 16 : sy;
            for (int32_t j = 0; j < 16; j++)
                memcpy(s->work + (size_t)(by * 16 + j) * W + bx * 16,
                       s->clean + (size_t)(sy + j) * W + sx, 16);
        }
    uint8_t *t = s->clean;
    s->clean = s->work;
    s->work = t;
}

int h261b_synth_preset(int32_t preset, int32_t width, int32_t height, uint64_t seed,
                       h261b_synth_params_t *p)
{
    memset(p, 0, sizeof(*p));
    p->width = width;
    p->height = height;
    p->seed = seed;
    p->kind = H261B_SYNTH_PAN_OBJECTS;
    switch (preset) {
    case 0:
        p->n_objects = 2; p->obj_min = 32; p->obj_max = 32; p->obj_vmax = 6;
        p->pan_dx = 2; p->pan_dy = -1; p->noise_sigma16 = 32;
        return 0;
    case 1:
        p->n_objects = 6; p->obj_min = 16; p->obj_max = 64; p->obj_vmax = 15;
        p->pan_period = 30; p->pan_rand = 8; p->scene_cut = 150; p->noise_sigma16 = 48;
        return 0;
    case 2: {
        uint64_t r = seed ^ 0xBADC0DEULL;
        p->n_objects = 2; p->obj_min = 32; p->obj_max = 32; p->obj_vmax = 6;
        p->pan_dx = urange(&r, -4, 4); p->pan_dy = urange(&r, -4, 4); p->noise_sigma16 = 32;
        return 0;
    }
    case 3:
        p->kind = H261B_SYNTH_BLOCK_MOTION;
        p->n_objects = 2; p->obj_min = 32; p->obj_max = 32; p->obj_vmax = 6;
        p->pan_dx = 2; p->pan_dy = -1; p->noise_sigma16 = 64; p->block_motion_max = 15;
        return 0;
    default:
        return -1;
    }
}

int h261b_synth_create(const h261b_synth_params_t *p, h261b_synth_t **out)
{
    *out = NULL;
    if (p->width < 16 || p->height < 16 || (p->width & 15) || (p->height & 15) ||
        p->obj_min < 1 || p->obj_max < p->obj_min || p->obj_max > p->width || p->obj_max > p->height)
        return -1;
    lut_init();
    struct h261b_synth_s *s = (struct h261b_synth_s *)calloc(1, sizeof(*s));
    if (!s)
        return -2;
    s->p = *p;
    s->rng_noise = p->seed ^ 0x4E4F495345ULL;
    s->rng_pan = p->seed ^ 0x50414EULL;
    s->rng_motion = p->seed ^ 0x4D4F54ULL;
    s->pan_vx = p->pan_dx;
    s->pan_vy = p->pan_dy;
    s->clean = (uint8_t *)malloc((size_t)p->width * p->height);
    s->work = (uint8_t *)malloc((size_t)p->width * p->height);
    if (!s->clean || !s->work || build_scene(s, p->seed) != 0) {
        h261b_synth_destroy(s);
        return -2;
    }
    *out = s;
    return 0;
}

int h261b_synth_next(h261b_synth_t *s, uint8_t *y, uint8_t *cb, uint8_t *cr)
{
    const int32_t W = s->p.width, H = s->p.height;
    if (s->p.scene_cut > 0 && s->t == s->p.scene_cut) {
        build_scene(s, s->p.seed * 0x9E3779B97F4A7C15ULL + 0x5CE7E);
        s->t_scene = s->t;
    }
    if (s->p.pan_period > 0 && s->t % s->p.pan_period == 0) {
        s->pan_vx = urange(&s->rng_pan, -s->p.pan_rand, s->p.pan_rand);
        s->pan_vy = urange(&s->rng_pan, -s->p.pan_rand, s->p.pan_rand);
    }
    if (s->p.kind == H261B_SYNTH_BLOCK_MOTION && s->t > 0)
        block_motion(s);
    else
        render_scene(s, s->clean);

    /* noise on the output only: sum of 12 16-bit uniforms has mean 393210
     * and standard deviation ~65536, scaled by sigma/16 and rounded down. */
    for (int32_t i = 0; i < W * H; i++) {
        uint64_t a = sm64(&s->rng_noise), b = sm64(&s->rng_noise), c = sm64(&s->rng_noise);
        int64_t sum = 0;
        for (int k = 0; k < 4; k++) {
            sum += (int64_t)((a >> (16 * k)) & 0xFFFF);
            sum += (int64_t)((b >> (16 * k)) & 0xFFFF);
            sum += (int64_t)((c >> (16 * k)) & 0xFFFF);
        }
        int64_t nv = ((sum - 393210) * s->p.noise_sigma16 + 524288) >> 20;
        int64_t v = (int64_t)s->clean[i] + nv;
        y[i] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
    }
    const int32_t CW = W / 2, CH = H / 2;
    for (int32_t j = 0; j < CH; j++)
        for (int32_t i = 0; i < CW; i++) {
            const uint8_t *p0 = y + (size_t)(2 * j) * W + 2 * i;
            int32_t avg = (p0[0] + p0[1] + p0[W] + p0[W + 1] + 2) >> 2;
            cb[j * CW + i] = (uint8_t)(128 + (avg - 128) / 2);
            cr[j * CW + i] = (uint8_t)(128 - (avg - 128) / 2);
        }
    s->pan_x += s->pan_vx;
    s->pan_y += s->pan_vy;
    return s->t++;
}

void h261b_synth_destroy(h261b_synth_t *s)
{
    if (!s)
        return;
    free_objects(s);
    free(s->clean);
    free(s->work);
    free(s);
}

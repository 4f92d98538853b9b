/* Rate control on the device: the reference's 6-bit fixed-point CBR rate
 * control (src/h261_ratectrl.c:4-245), one thread per session.
 *
 *   picture QUANT  collect_picture_stats (:225-245), init_picture
 *                  (:144-195) and h261_init_picture's clamp
 *                  (src/h261_picture.c:102-110), from the picture's summed
 *                  mode-decision costs;
 *   update         update_picture (:198-222), from the picture's size in
 *                  bytes, which the bitstream writer knows.
 *
 * Integer arithmetic only; the oracle restates the same steps
 * (oracle/h261_writer.c) and both are pinned to the reference's stream. */
#pragma once

#include <stdint.h>

#include "h261b_device.h"

namespace h261b {

/* round(64 * 2^(f/5)) for f = -31..31 (src/h261_ratectrl.c:11-19) */
static __device__ __constant__ int32_t c_rc_qscale[63] = {
    0,    1,    1,    1,    1,    1,    2,    2,    2,    3,    3,    4,    4,    5,    6,    6,
    8,    9,    10,   12,   13,   16,   18,   21,   24,   27,   32,   36,   42,   48,   55,   64,
    73,   84,   97,   111,  128,  147,  168,  194,  222,  256,  294,  337,  388,  445,  512,  588,
    675,  776,  891,  1024, 1176, 1351, 1552, 1782, 2048, 2352, 2702, 3104, 3565, 4096, 4705,
};

constexpr int RC_BITS = 6;
constexpr int32_t RC_ONE = 1 << RC_BITS;
constexpr int32_t RC_HALF = 1 << (RC_BITS - 1);
constexpr int32_t RC_TIME_SCALE = 1918;   /* 29.97 Hz in 6-bit fixed point */

__device__ __forceinline__ int32_t rc_mul(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * b) >> RC_BITS); }
__device__ __forceinline__ int32_t rc_div(int32_t a, int32_t b) { return (int32_t)(((int64_t)a * RC_ONE) / b); }
__device__ __forceinline__ int32_t rc_qscale(int32_t q) { return c_rc_qscale[min(max(q, 0), 31) + 31]; }

/* nearest qscale entry by binary search, ties to the upper one */
__device__ __forceinline__ int32_t rc_quant_delta(int32_t qs)
{
    int32_t pos = 31;
    for (int32_t step = 16; step; step >>= 1)
        pos += c_rc_qscale[pos] < qs ? step : -step;
    int32_t lo, hi;
    if (c_rc_qscale[pos] < qs) {
        lo = pos;
        hi = min(pos + 1, 62);
    } else {
        lo = max(0, pos - 1);
        hi = pos;
    }
    return (qs - c_rc_qscale[lo] < c_rc_qscale[hi] - qs ? lo : hi) - 31;
}

/* QUANT of the picture in flight from its cost sum; resets the sum */
__device__ __forceinline__ void rc_picture_quant(h261b_rc_dev_t &rc, int32_t frame_type, int32_t num_mb)
{
    rc.current_picture_cost = max(rc.cost_sum, num_mb * 100);
    rc.cost_sum = 0;
    rc.vbv_fill = min(rc.vbv_fill + rc_div(rc.bitrate, RC_TIME_SCALE), rc.vbv_size);
    const int32_t cost_scale = rc_div(rc.current_picture_cost, rc.prediction_cost[frame_type]);
    const int32_t predicted = rc_div(rc_mul(cost_scale, rc.prediction_size[frame_type]), rc_qscale(rc.current_quant));
    int32_t target = rc_div(rc.bitrate, RC_TIME_SCALE);
    if (frame_type == H261B_FRAME_TYPE_INTRA)
        target *= 20;
    const int32_t up = rc_div(rc.vbv_fill, rc.vbv_size);
    /* the reference clamps the prediction into [lower, upper] and then
     * replaces the result with max(lower, 10) */
    target = max(target - rc_mul(target, RC_ONE - up), 10);
    int32_t scale = rc_div(predicted, target);
    if (scale < RC_ONE)
        scale = rc_mul(RC_ONE - up, RC_ONE) + rc_mul(up, scale);
    rc.current_quant = min(max(rc.current_quant + rc_quant_delta(scale), 1), 31);
    const int32_t q = rc.current_quant + (((RC_ONE - up) * 4) >> RC_BITS);
    rc.picture_quant = min(max(q, 1), 31);
}

/* after the picture: its size in bytes */
__device__ __forceinline__ void rc_update(h261b_rc_dev_t &rc, int32_t frame_type, int32_t bytes)
{
    rc.prediction_cost[frame_type] = rc_mul(rc.prediction_cost[frame_type], RC_HALF) + rc.current_picture_cost;
    rc.prediction_size[frame_type] =
        rc_mul(rc.prediction_size[frame_type], RC_HALF) + rc_mul(bytes, rc_qscale(rc.picture_quant));
    rc.vbv_fill -= bytes;
}

} // namespace h261b

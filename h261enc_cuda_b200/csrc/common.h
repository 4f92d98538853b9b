/*
 * common.h -- host-side helpers shared by the engine and the
 * reference-compatible boundary: status recording and CUDA checks.
 */
#ifndef H261B_COMMON_H
#define H261B_COMMON_H

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/h261b.h"

/* NVTX (header-only nvtx3): ranges cost a function-pointer check when no
 * profiler is attached */
#include <nvtx3/nvToolsExt.h>

namespace h261b {

/* a named NVTX range over a scope: the engine marks every frame-step's host
 * work (descriptors, uploads, launches), every wait for a step and every
 * batch of picture copies, so that a timeline shows where host time goes */
class NvtxRange {
  public:
    explicit NvtxRange(const char *fmt, ...)
    {
        char buf[96];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        nvtxRangePushA(buf);
    }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

void set_error(const char *fmt, ...);
void clear_error();

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

/* byte offsets of the three planes of a packed picture (256-byte aligned) */
struct PictureLayout {
    size_t off_y, off_cb, off_cr, bytes;
    int32_t pitch_y, pitch_c;
    static PictureLayout of(int32_t w, int32_t h)
    {
        PictureLayout l;
        l.pitch_y = w;
        l.pitch_c = w / 2;
        l.off_y = 0;
        l.off_cb = align_up((size_t)w * h, 256);
        l.off_cr = l.off_cb + align_up((size_t)(w / 2) * (h / 2), 256);
        l.bytes = l.off_cr + align_up((size_t)(w / 2) * (h / 2), 256);
        return l;
    }
};

} // namespace h261b

#define H261B_CUDA_TRY(expr)                                                                    \
    do {                                                                                        \
        cudaError_t err__ = (expr);                                                             \
        if (err__ != cudaSuccess) {                                                             \
            h261b::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(err__), __FILE__, \
                             __LINE__);                                                         \
            return H261B_ERR_CUDA;                                                              \
        }                                                                                       \
    } while (0)

#endif

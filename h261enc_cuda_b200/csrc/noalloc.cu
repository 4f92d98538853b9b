/*
 * noalloc.cu -- encode one picture without allocating anything.
 *
 * Who needs this: callers that cannot call cudaMalloc -- a host program
 * whose device memory is owned by another allocator (a framework's caching
 * allocator, a pool sized once at start-up), code that runs where a
 * device allocation would synchronise or fail (inside a latency-critical
 * loop, on a device whose memory a larger job has reserved), or a plugin
 * that may only touch buffers it is handed.  Such a caller owns its input,
 * output and per-stream state buffers; it cannot give the engine the small
 * descriptor and work list the step kernel needs, which the engine
 * normally cudaMallocs.
 *
 * Here that scratch -- one session descriptor and the macroblock work list
 * -- lives in g_noalloc_scratch, a file-scope static __device__ array of a
 * fixed size (about 16.6 KB: room for pictures of at most
 * H261B_NOALLOC_MAX_MB macroblocks).  Every GPU that loads the library
 * holds it until the process exits.  Host code cannot use the array's name
 * as a device address, so on the first call on a device, with that device
 * current, its address is looked up with cudaGetSymbolAddress (return code
 * checked) and the constant work list is written; later calls on that
 * device reuse the address.  Because of that set-up, the first call on a
 * device should come before any stream capture.
 *
 * Every call shares the array and leaves its descriptor there; nothing in
 * it has to start at zero (the descriptor is rewritten in full, the work
 * list never changes).  Calls whose work overlaps on the GPU race on the
 * descriptor: issue them on one stream, or wait for one before the next.
 */
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <mutex>

#include "common.h"
#include "h261b_device.h"

using namespace h261b;

namespace {

constexpr size_t kDescBytes = (sizeof(h261b_session_dev_t) + 255) / 256 * 256;
constexpr size_t kScratchWords = kDescBytes / 4 + H261B_NOALLOC_MAX_MB;
static_assert(sizeof(h261b_denoise_dev_t) == H261B_NOALLOC_STATE_BYTES, "state size");
static_assert(sizeof(h261b_mb_info_t) == sizeof(h261b_mb_result_t), "result record size");
static_assert(offsetof(h261b_denoise_dev_t, denoise) == 0, "the strength is the state's first word");

static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t *g_addr[kMaxDevices];

/* Per-device set-up with the device current: the scratch address and the
 * work list 0 .. H261B_NOALLOC_MAX_MB-1 (session 0, every MB). */
int scratch_for_device(int dev, uint32_t **out)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *addr = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
        if (err != cudaSuccess) {
            set_error("h261b_encode_picture_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(err));
            return H261B_ERR_CUDA;
        }
        static uint32_t work[H261B_NOALLOC_MAX_MB];
        for (uint32_t i = 0; i < H261B_NOALLOC_MAX_MB; i++)
            work[i] = i;
        err = cudaMemcpy((uint8_t *)addr + kDescBytes, work, sizeof(work), cudaMemcpyHostToDevice);
        if (err != cudaSuccess || h261b_set_quant_table() != 0) {
            set_error("h261b_encode_picture_noalloc: device set-up failed: %s",
                      cudaGetErrorString(err != cudaSuccess ? err : cudaGetLastError()));
            return H261B_ERR_CUDA;
        }
        g_addr[dev] = (uint32_t *)addr;
    }
    *out = g_addr[dev];
    return H261B_OK;
}

/* Writes the call's descriptor into the scratch and, for the first picture
 * of a stream, clears the caller's denoise state and sets its strength (the
 * reference's starting state, gpu_device.cu:495-508): offsets,
 * accumulators and frame-end ticket zero. */
__global__ void noalloc_prepare(h261b_session_dev_t d, h261b_session_dev_t *slot, uint32_t *state, int32_t reset,
                                int32_t strength)
{
    if (reset) {
        /* word 0 of h261b_denoise_dev_t is the strength */
        for (int i = threadIdx.x; i < H261B_NOALLOC_STATE_BYTES / 4; i += blockDim.x)
            state[i] = i == 0 ? (uint32_t)strength : 0u;
    }
    if (threadIdx.x == 0)
        *slot = d;
}

} // namespace

extern "C" int h261b_encode_picture_noalloc(const h261b_noalloc_picture_t *p, void *stream)
{
    clear_error();
    if (!p || !p->cur_y || !p->cur_cb || !p->cur_cr || !p->ref_y || !p->ref_cb || !p->ref_cr || !p->rec_y ||
        !p->rec_cb || !p->rec_cr || !p->state || !p->mbs || !p->levels) {
        set_error("h261b_encode_picture_noalloc: a buffer pointer is NULL");
        return H261B_ERR_ARG;
    }
    if (p->width < 16 || p->height < 16 || (p->width & 15) || (p->height & 15)) {
        set_error("h261b_encode_picture_noalloc: %dx%d is not a positive multiple of 16", p->width, p->height);
        return H261B_ERR_ARG;
    }
    const int32_t mbw = p->width / 16, mbh = p->height / 16, nmb = mbw * mbh;
    if (nmb > H261B_NOALLOC_MAX_MB) {
        set_error("h261b_encode_picture_noalloc: %dx%d has %d macroblocks, more than the %d this entry point's "
                  "fixed scratch holds",
                  p->width, p->height, nmb, H261B_NOALLOC_MAX_MB);
        return H261B_ERR_ARG;
    }
    if (p->quant < 1 || p->quant > 31 || (p->frame_type != H261B_FRAME_TYPE_INTRA &&
                                          p->frame_type != H261B_FRAME_TYPE_INTER) ||
        (p->me_mode != H261B_ME_REFERENCE && p->me_mode != H261B_ME_FULL) || p->denoise < 0) {
        set_error("h261b_encode_picture_noalloc: QUANT, picture type, search mode or denoise out of range");
        return H261B_ERR_ARG;
    }
    const uintptr_t a16 = (uintptr_t)p->cur_y | (uintptr_t)p->ref_y | (uintptr_t)p->rec_y | (uintptr_t)p->state |
                          (uintptr_t)p->mbs;
    const uintptr_t a8 = (uintptr_t)p->cur_cb | (uintptr_t)p->cur_cr | (uintptr_t)p->ref_cb | (uintptr_t)p->ref_cr |
                         (uintptr_t)p->rec_cb | (uintptr_t)p->rec_cr | (uintptr_t)p->levels;
    if ((a16 & 15) || (a8 & 7)) {
        set_error("h261b_encode_picture_noalloc: luma planes, state and results must be 16-byte, chroma planes and "
                  "levels 8-byte aligned");
        return H261B_ERR_ARG;
    }
    int dev = 0;
    H261B_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("h261b_encode_picture_noalloc: device %d out of range", dev);
        return H261B_ERR_ARG;
    }
    uint32_t *scratch = nullptr;
    int rc = scratch_for_device(dev, &scratch);
    if (rc)
        return rc;
    cudaStream_t st = (cudaStream_t)stream;

    h261b_session_dev_t d;
    memset(&d, 0, sizeof(d));
    d.cur_y = p->cur_y;
    d.cur_cb = p->cur_cb;
    d.cur_cr = p->cur_cr;
    d.ref_y = p->ref_y;
    d.ref_cb = p->ref_cb;
    d.ref_cr = p->ref_cr;
    d.rec_y = p->rec_y;
    d.rec_cb = p->rec_cb;
    d.rec_cr = p->rec_cr;
    d.pitch_y = p->width;
    d.pitch_c = p->width / 2;
    d.mbw = mbw;
    d.mbh = mbh;
    d.frame_type = p->frame_type;
    d.quant = p->quant;
    d.me_mode = p->me_mode;
    d.skip_search = p->frame_type == H261B_FRAME_TYPE_INTRA;
    d.dn = (h261b_denoise_dev_t *)p->state;
    d.info_out = (h261b_mb_info_t *)p->mbs;
    d.level_out = p->levels;
    /* the descriptor (and, for a new stream, the cleared state with its
     * strength) goes to the device as kernel arguments: no host buffer has
     * to outlive the call */
    noalloc_prepare<<<1, 256, 0, st>>>(d, (h261b_session_dev_t *)scratch, (uint32_t *)p->state,
                                       p->reset_state ? 1 : 0, p->denoise);
    H261B_CUDA_TRY(cudaGetLastError());
    const int phases = H261B_PHASE_ME | H261B_PHASE_MD | H261B_PHASE_ENCDEC | (p->fmad ? H261B_FMAD_BIT : 0) |
                       (p->me_mode == H261B_ME_FULL ? H261B_LAUNCH_ME_FULL : 0);
    const int lr = h261b_launch_step((const h261b_session_dev_t *)scratch,
                                     (const uint32_t *)((const uint8_t *)scratch + kDescBytes), nmb, phases, 4, 0,
                                     nullptr, st);
    if (lr != 0) {
        set_error("h261b_encode_picture_noalloc: launch failed: %s", cudaGetErrorString((cudaError_t)lr));
        return H261B_ERR_CUDA;
    }
    return H261B_OK;
}

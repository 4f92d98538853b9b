/*
 * compat.cu -- the reference's device boundary (src/gpu_device.h:7-32) on
 * the sm_100a core.
 *
 * Same contract as src/gpu_device.cu: one process-global encoder, every
 * call synchronous on return, results in pinned host arrays owned by the
 * library, void returns.  What differs inside:
 *   - pictures live in plain device memory (packed planes) instead of
 *     cudaArray textures; every fetch of the reference is in bounds, so
 *     plain loads read the same pixels (gpu_device.cu:90-145);
 *   - h261_gpu_device_me is one launch (search, refinement and the three
 *     SATD costs per MB), not five;
 *   - h261_gpu_device_encode_macroblocks is one launch that also
 *     reconstructs; h261_gpu_device_decode_macroblocks returns that
 *     reconstruction.  Both reference kernels decode from their own device
 *     copy of the levels, never the host one, so the output is the same;
 *   - a failure is printed to stderr and kept for h261b_abi_last_status()
 *     (the reference prints cudaGetLastError after each call).
 * Environment: H261B_DEVICE (default 0), H261B_FMAD=0 for separately
 * rounded double multiply-adds, H261B_ME=full for the exhaustive search.
 */
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>

#include "common.h"
#include "h261b_device.h"

using namespace h261b;

namespace {

struct Compat {
    bool ready = false;
    int device = 0;
    int fmad = 1, me_mode = 0;
    cudaStream_t stream = nullptr;
    int32_t w = 0, h = 0;
    PictureLayout lay;
    uint8_t *cur = nullptr, *ref = nullptr, *rec = nullptr;
    h261b_session_dev_t *desc_dev = nullptr;
    uint32_t *work_dev = nullptr;
    int32_t work_n = 0;
    h261b_denoise_dev_t *dn_dev = nullptr;
    h261_mb_mode_decision_t *md_dev = nullptr;
    int status = H261B_OK;
};

Compat g;

void fail(const char *where, cudaError_t err)
{
    g.status = H261B_ERR_CUDA;
    set_error("%s: %s", where, cudaGetErrorString(err));
    fprintf(stderr, "h261b: %s: %s\n", where, cudaGetErrorString(err));
}

void fail_arg(const char *where, const char *what)
{
    g.status = H261B_ERR_ARG;
    set_error("%s: %s", where, what);
    fprintf(stderr, "h261b: %s: %s\n", where, what);
}

#define CK(where, expr)                    \
    do {                                   \
        cudaError_t e__ = (expr);          \
        if (e__ != cudaSuccess) {          \
            fail(where, e__);              \
            return;                        \
        }                                  \
    } while (0)

bool ensure_ready(const char *where)
{
    if (!g.ready) {
        fail_arg(where, "h261_gpu_init has not been called");
        return false;
    }
    return true;
}

/* one work list covering every MB of the picture */
bool ensure_work(const char *where, int32_t nmb)
{
    if (g.work_dev && g.work_n == nmb)
        return true;
    if (g.work_dev)
        cudaFree(g.work_dev);
    g.work_dev = nullptr;
    uint32_t *host = (uint32_t *)malloc(sizeof(uint32_t) * nmb);
    for (int32_t i = 0; i < nmb; i++)
        host[i] = (uint32_t)i;
    cudaError_t e1 = cudaMalloc(&g.work_dev, sizeof(uint32_t) * nmb);
    cudaError_t e2 = e1 == cudaSuccess ? cudaMemcpy(g.work_dev, host, sizeof(uint32_t) * nmb, cudaMemcpyHostToDevice)
                                       : e1;
    free(host);
    if (e2 != cudaSuccess) {
        fail(where, e2);
        return false;
    }
    g.work_n = nmb;
    return true;
}

void base_desc(h261b_session_dev_t &d)
{
    memset(&d, 0, sizeof(d));
    d.cur_y = g.cur + g.lay.off_y;
    d.cur_cb = g.cur + g.lay.off_cb;
    d.cur_cr = g.cur + g.lay.off_cr;
    d.ref_y = g.ref + g.lay.off_y;
    d.ref_cb = g.ref + g.lay.off_cb;
    d.ref_cr = g.ref + g.lay.off_cr;
    d.rec_y = g.rec + g.lay.off_y;
    d.rec_cb = g.rec + g.lay.off_cb;
    d.rec_cr = g.rec + g.lay.off_cr;
    d.pitch_y = g.lay.pitch_y;
    d.pitch_c = g.lay.pitch_c;
    d.mbw = g.w / 16;
    d.mbh = g.h / 16;
    d.me_mode = g.me_mode;
}

void upload(const char *where, uint8_t *pic, size_t off, const uint8_t *data, int32_t w, int32_t h,
            int32_t ew, int32_t eh)
{
    if (!ensure_ready(where))
        return;
    if (!pic) {
        fail_arg(where, "h261_gpu_device_init_textures has not been called");
        return;
    }
    if (!data || w != ew || h != eh) {
        fail_arg(where, "plane size does not match the initialised picture");
        return;
    }
    CK(where, cudaMemcpy(pic + off, data, (size_t)w * h, cudaMemcpyHostToDevice));
}

} // namespace

extern "C" int h261b_abi_last_status(void) { return g.status; }

extern "C" void h261_gpu_init(void)
{
    const char *dv = getenv("H261B_DEVICE");
    const char *fm = getenv("H261B_FMAD");
    const char *me = getenv("H261B_ME");
    g.device = dv ? atoi(dv) : 0;
    g.fmad = fm ? atoi(fm) != 0 : 1;
    g.me_mode = (me && strcmp(me, "full") == 0) ? 1 : 0;
    g.status = H261B_OK;
    CK("h261_gpu_init", cudaSetDevice(g.device));
    if (!g.stream)
        CK("h261_gpu_init", cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    if (h261b_set_quant_table() != 0) {
        fail("h261_gpu_init", cudaGetLastError());
        return;
    }
    if (!g.desc_dev)
        CK("h261_gpu_init", cudaMalloc(&g.desc_dev, sizeof(h261b_session_dev_t)));
    g.ready = true;
}

extern "C" void h261_gpu_device_init_textures(int32_t w, int32_t h)
{
    const char *where = "h261_gpu_device_init_textures";
    if (!ensure_ready(where))
        return;
    if (w < 16 || h < 16 || (w & 15) || (h & 15) || (w / 16) * (h / 16) > H261B_MAX_MB_PER_SESSION) {
        fail_arg(where, "unsupported picture size");
        return;
    }
    h261_gpu_device_deinit_textures();
    g.w = w;
    g.h = h;
    g.lay = PictureLayout::of(w, h);
    CK(where, cudaMalloc(&g.cur, g.lay.bytes));
    CK(where, cudaMalloc(&g.ref, g.lay.bytes));
    CK(where, cudaMalloc(&g.rec, g.lay.bytes));
    CK(where, cudaMemset(g.cur, 0, g.lay.bytes));
    CK(where, cudaMemset(g.ref, 0, g.lay.bytes));
    CK(where, cudaMemset(g.rec, 0, g.lay.bytes));
}

extern "C" void h261_gpu_device_deinit_textures(void)
{
    cudaFree(g.cur);
    cudaFree(g.ref);
    cudaFree(g.rec);
    g.cur = g.ref = g.rec = nullptr;
}

extern "C" void h261_gpu_device_set_current(uint8_t *d, int32_t w, int32_t h)
{
    upload("h261_gpu_device_set_current", g.cur, g.lay.off_y, d, w, h, g.w, g.h);
}
extern "C" void h261_gpu_device_set_current_chroma_cb(uint8_t *d, int32_t w, int32_t h)
{
    upload("h261_gpu_device_set_current_chroma_cb", g.cur, g.lay.off_cb, d, w, h, g.w / 2, g.h / 2);
}
extern "C" void h261_gpu_device_set_current_chroma_cr(uint8_t *d, int32_t w, int32_t h)
{
    upload("h261_gpu_device_set_current_chroma_cr", g.cur, g.lay.off_cr, d, w, h, g.w / 2, g.h / 2);
}
extern "C" void h261_gpu_device_set_reference(uint8_t *d, int32_t w, int32_t h)
{
    upload("h261_gpu_device_set_reference", g.ref, g.lay.off_y, d, w, h, g.w, g.h);
}
extern "C" void h261_gpu_device_set_reference_chroma_cb(uint8_t *d, int32_t w, int32_t h)
{
    upload("h261_gpu_device_set_reference_chroma_cb", g.ref, g.lay.off_cb, d, w, h, g.w / 2, g.h / 2);
}
extern "C" void h261_gpu_device_set_reference_chroma_cr(uint8_t *d, int32_t w, int32_t h)
{
    upload("h261_gpu_device_set_reference_chroma_cr", g.ref, g.lay.off_cr, d, w, h, g.w / 2, g.h / 2);
}

extern "C" void h261_gpu_device_init_me(me_gpu_t **pps, int32_t w, int32_t h)
{
    const char *where = "h261_gpu_device_init_me";
    if (!pps) {
        fail_arg(where, "null output pointer");
        return;
    }
    *pps = nullptr;
    if (!ensure_ready(where))
        return;
    if (w < 16 || h < 16 || (w & 15) || (h & 15)) {
        fail_arg(where, "unsupported picture size");
        return;
    }
    me_gpu_t *s = nullptr;
    CK(where, cudaMallocHost(&s, sizeof(me_gpu_t)));
    memset(s, 0, sizeof(*s));
    s->i_mb_width = w / 16;
    s->i_mb_height = h / 16;
    s->i_num_mb = s->i_mb_width * s->i_mb_height;
    const size_t n = (size_t)s->i_num_mb;
    CK(where, cudaMalloc(&s->prgs_macroblocks_device, sizeof(me_gpu_mb_t) * n));
    CK(where, cudaMallocHost(&s->prgs_macroblocks_result, sizeof(me_gpu_mb_t) * n));
    CK(where, cudaMalloc(&s->ps_candidate_vector_device, sizeof(me_gpu_mv_t) * n));
    CK(where, cudaMallocHost(&s->ps_candidate_vector_host, sizeof(me_gpu_mv_t) * n));
    CK(where, cudaMalloc(&s->ps_starting_vector_device, sizeof(me_gpu_mv_t) * n));
    CK(where, cudaMallocHost(&s->ps_starting_vector_host, sizeof(me_gpu_mv_t) * n));
    CK(where, cudaMalloc(&s->pi8_motion_vector_limits_device, 4 * n));
    CK(where, cudaMallocHost(&s->pi8_motion_vector_limits_host, 4 * n));
    memset(s->prgs_macroblocks_result, 0, sizeof(me_gpu_mb_t) * n);
    memset(s->ps_candidate_vector_host, 0, sizeof(me_gpu_mv_t) * n);
    memset(s->ps_starting_vector_host, 0, sizeof(me_gpu_mv_t) * n);
    /* the per-MB limits of gpu_device.cu:226-265, kept for callers that read
     * them (the kernel derives the same limits from the MB position) */
    for (int32_t y = 0; y < s->i_mb_height; y++)
        for (int32_t x = 0; x < s->i_mb_width; x++) {
            const int32_t bx = x * 16, by = y * 16, gx = (s->i_mb_width - 1) * 16, gy = (s->i_mb_height - 1) * 16;
            int8_t *l = s->pi8_motion_vector_limits_host + (size_t)(x + y * s->i_mb_width) * 4;
            l[0] = (int8_t)((bx - 15 > 0 ? bx - 15 : 0) - bx);
            l[1] = (int8_t)((bx + 15 < gx ? bx + 15 : gx) - bx);
            l[2] = (int8_t)((by - 15 > 0 ? by - 15 : 0) - by);
            l[3] = (int8_t)((by + 15 < gy ? by + 15 : gy) - by);
        }
    CK(where, cudaMemcpy(s->pi8_motion_vector_limits_device, s->pi8_motion_vector_limits_host, 4 * n,
                         cudaMemcpyHostToDevice));
    CK(where, cudaMemset(s->ps_candidate_vector_device, 0, sizeof(me_gpu_mv_t) * n));
    CK(where, cudaMemset(s->prgs_macroblocks_device, 0, sizeof(me_gpu_mb_t) * n));
    *pps = s;
}

extern "C" void h261_gpu_device_deinit_me(me_gpu_t **pps)
{
    if (!pps || !*pps)
        return;
    me_gpu_t *s = *pps;
    cudaFree(s->prgs_macroblocks_device);
    cudaFreeHost(s->prgs_macroblocks_result);
    cudaFree(s->ps_candidate_vector_device);
    cudaFreeHost(s->ps_candidate_vector_host);
    cudaFree(s->ps_starting_vector_device);
    cudaFreeHost(s->ps_starting_vector_host);
    cudaFree(s->pi8_motion_vector_limits_device);
    cudaFreeHost(s->pi8_motion_vector_limits_host);
    cudaFreeHost(s);
    *pps = nullptr;
}

extern "C" void h261_gpu_device_me(me_gpu_t *s)
{
    const char *where = "h261_gpu_device_me";
    if (!ensure_ready(where))
        return;
    if (!s || !g.cur || s->i_mb_width != g.w / 16 || s->i_mb_height != g.h / 16) {
        fail_arg(where, "ME state does not match the initialised picture");
        return;
    }
    const int32_t n = s->i_num_mb;
    if (!ensure_work(where, n))
        return;
    h261b_session_dev_t d;
    base_desc(d);
    d.frame_type = H261B_FRAME_TYPE_INTER;
    d.me_out = s->prgs_macroblocks_device;
    CK(where, cudaMemcpyAsync(g.desc_dev, &d, sizeof(d), cudaMemcpyHostToDevice, g.stream));
    int rc = h261b_launch_step(g.desc_dev, g.work_dev, n,
                               H261B_PHASE_ME | H261B_ABI_OUT | (g.me_mode ? H261B_LAUNCH_ME_FULL : 0) |
                                   (g.fmad ? H261B_FMAD_BIT : 0),
                               4, 0, nullptr, g.stream);
    if (rc) {
        fail(where, (cudaError_t)rc);
        return;
    }
    CK(where, cudaMemcpyAsync(s->prgs_macroblocks_result, s->prgs_macroblocks_device, sizeof(me_gpu_mb_t) * n,
                              cudaMemcpyDeviceToHost, g.stream));
    CK(where, cudaStreamSynchronize(g.stream));
    /* the reference leaves the final vector in the starting-vector arrays
     * and copies it to the candidate ones (gpu_device.cu:403-422) */
    for (int32_t i = 0; i < n; i++)
        s->ps_starting_vector_host[i] = s->prgs_macroblocks_result[i].s_16x16_mv;
    CK(where, cudaMemcpyAsync(s->ps_starting_vector_device, s->ps_starting_vector_host, sizeof(me_gpu_mv_t) * n,
                              cudaMemcpyHostToDevice, g.stream));
    CK(where, cudaMemcpyAsync(s->ps_candidate_vector_device, s->ps_starting_vector_device,
                              sizeof(me_gpu_mv_t) * n, cudaMemcpyDeviceToDevice, g.stream));
    CK(where, cudaStreamSynchronize(g.stream));
}

extern "C" void h261_init_macroblocks(h261_macroblocks_t **pps, int32_t w, int32_t h, int32_t denoise)
{
    const char *where = "h261_init_macroblocks";
    if (!pps) {
        fail_arg(where, "null output pointer");
        return;
    }
    *pps = nullptr;
    if (!ensure_ready(where))
        return;
    if (w < 16 || h < 16 || (w & 15) || (h & 15) || !g.rec || w != g.w || h != g.h) {
        fail_arg(where, "size does not match the initialised picture");
        return;
    }
    h261_macroblocks_t *s = nullptr;
    CK(where, cudaMallocHost(&s, sizeof(*s)));
    memset(s, 0, sizeof(*s));
    s->i_mb_width = w / 16;
    s->i_mb_height = h / 16;
    s->i_num_mb = s->i_mb_width * s->i_mb_height;
    const size_t n = (size_t)s->i_num_mb;
    CK(where, cudaMallocHost(&s->ps_macroblocks, sizeof(h261_macroblock_t) * n));
    memset(s->ps_macroblocks, 0, sizeof(h261_macroblock_t) * n);
    for (int32_t y = 0; y < s->i_mb_height; y++)
        for (int32_t x = 0; x < s->i_mb_width; x++) {
            s->ps_macroblocks[y * s->i_mb_width + x].i_mb_x = x * 16;
            s->ps_macroblocks[y * s->i_mb_width + x].i_mb_y = y * 16;
        }
    CK(where, cudaMalloc(&s->ps_macroblocks_device, sizeof(h261_macroblock_t) * n));
    CK(where, cudaMemcpy(s->ps_macroblocks_device, s->ps_macroblocks, sizeof(h261_macroblock_t) * n,
                         cudaMemcpyHostToDevice));
    int32_t **arrs[5][2] = { { &s->pi_mb_types_host, &s->pi_mb_types_device },
                             { &s->pi_mb_flags_host, &s->pi_mb_flags_device },
                             { &s->pi_mb_quant_host, &s->pi_mb_quant_device },
                             { &s->pi_mb_mv_x_host, &s->pi_mb_mv_x_device },
                             { &s->pi_mb_mv_y_host, &s->pi_mb_mv_y_device } };
    for (auto &a : arrs) {
        CK(where, cudaMallocHost(a[0], sizeof(int32_t) * n));
        CK(where, cudaMalloc(a[1], sizeof(int32_t) * n));
    }
    /* denoise: the reference layout on the host side, the engine's on the
     * device (same starting values, gpu_device.cu:495-508) */
    CK(where, cudaMallocHost(&s->ps_denoise_host, sizeof(h261_dct_denoise_t)));
    memset(s->ps_denoise_host, 0, sizeof(h261_dct_denoise_t));
    s->ps_denoise_host->i_denoise = denoise;
    h261b_denoise_dev_t dn0;
    memset(&dn0, 0, sizeof(dn0));
    dn0.denoise = denoise;
    if (g.dn_dev)
        cudaFree(g.dn_dev);
    CK(where, cudaMalloc(&g.dn_dev, sizeof(dn0)));
    CK(where, cudaMemcpy(g.dn_dev, &dn0, sizeof(dn0), cudaMemcpyHostToDevice));
    s->ps_denoise_device = (h261_dct_denoise_t *)g.dn_dev;
    if (g.md_dev)
        cudaFree(g.md_dev);
    CK(where, cudaMalloc(&g.md_dev, sizeof(h261_mb_mode_decision_t) * n));
    /* reconstruction: device planes are the core's output picture; the host
     * arrays have the reference's size (num_mb * 256 bytes each) */
    s->pui8_reconstructed_Y_device = g.rec + g.lay.off_y;
    s->pui8_reconstructed_Cb_device = g.rec + g.lay.off_cb;
    s->pui8_reconstructed_Cr_device = g.rec + g.lay.off_cr;
    CK(where, cudaMallocHost(&s->pui8_reconstructed_Y_host, n * 256));
    CK(where, cudaMallocHost(&s->pui8_reconstructed_Cb_host, n * 256));
    CK(where, cudaMallocHost(&s->pui8_reconstructed_Cr_host, n * 256));
    memset(s->pui8_reconstructed_Y_host, 0, n * 256);
    memset(s->pui8_reconstructed_Cb_host, 0, n * 256);
    memset(s->pui8_reconstructed_Cr_host, 0, n * 256);
    /* no SoA coefficient scratch: transforms run in registers */
    s->i_num_blocks = (int32_t)((n * 6 + H261B_COEFF_BLOCK_WIDTH - 1) / H261B_COEFF_BLOCK_WIDTH);
    s->i_num_coeff_blocks = s->i_num_blocks * H261B_COEFF_BLOCK_WIDTH;
    s->pi_coeff_blocks_device = nullptr;
    s->pi_coeff_blocks_host = nullptr;
    s->p_cuda = nullptr;
    *pps = s;
}

extern "C" void h261_deinit_macroblocks(h261_macroblocks_t *s)
{
    if (!s)
        return;
    cudaFree(s->ps_macroblocks_device);
    cudaFreeHost(s->ps_macroblocks);
    cudaFreeHost(s->pi_mb_types_host);
    cudaFree(s->pi_mb_types_device);
    cudaFreeHost(s->pi_mb_flags_host);
    cudaFree(s->pi_mb_flags_device);
    cudaFreeHost(s->pi_mb_quant_host);
    cudaFree(s->pi_mb_quant_device);
    cudaFreeHost(s->pi_mb_mv_x_host);
    cudaFree(s->pi_mb_mv_x_device);
    cudaFreeHost(s->pi_mb_mv_y_host);
    cudaFree(s->pi_mb_mv_y_device);
    cudaFreeHost(s->ps_denoise_host);
    cudaFreeHost(s->pui8_reconstructed_Y_host);
    cudaFreeHost(s->pui8_reconstructed_Cb_host);
    cudaFreeHost(s->pui8_reconstructed_Cr_host);
    cudaFreeHost(s);
    cudaFree(g.dn_dev);
    cudaFree(g.md_dev);
    g.dn_dev = nullptr;
    g.md_dev = nullptr;
}

extern "C" void h261_gpu_device_encode_macroblocks(h261_context_t *ctx)
{
    const char *where = "h261_gpu_device_encode_macroblocks";
    if (!ensure_ready(where))
        return;
    if (!ctx || !ctx->ps_macroblocks || !ctx->ps_mode_decision || !ctx->ps_mode_decision->prgs_mb || !g.dn_dev) {
        fail_arg(where, "context is missing macroblocks or mode decision");
        return;
    }
    h261_macroblocks_t *s = ctx->ps_macroblocks;
    const h261_mode_decision_t *md = ctx->ps_mode_decision;
    const int32_t n = s->i_num_mb;
    if (s->i_mb_width != g.w / 16 || s->i_mb_height != g.h / 16 || md->i_mb_width != s->i_mb_width ||
        md->i_mb_height != s->i_mb_height) {
        fail_arg(where, "macroblock state does not match the initialised picture");
        return;
    }
    if (!ensure_work(where, n))
        return;
    /* a caller's mode decision must stay inside what the search could
     * return: the reference reads such blocks through clamping textures,
     * this core through the staged search window, so reject it loudly */
    const int32_t mbw = s->i_mb_width, mbh = s->i_mb_height;
    for (int32_t i = 0; i < n; i++) {
        const h261_mb_mode_decision_t &m = md->prgs_mb[i];
        const int32_t bx = (i % mbw) * 16, by = (i / mbw) * 16;
        const bool type_ok = m.i_mb_type == H261B_MB_TYPE_INTRA || m.i_mb_type == H261B_MB_TYPE_INTER;
        const bool mv_ok = m.i_mv_x >= -15 && m.i_mv_x <= 15 && m.i_mv_y >= -15 && m.i_mv_y <= 15 &&
                           bx + m.i_mv_x >= 0 && bx + m.i_mv_x <= (mbw - 1) * 16 && by + m.i_mv_y >= 0 &&
                           by + m.i_mv_y <= (mbh - 1) * 16;
        if (!type_ok || !mv_ok || (m.i_mb_flags & ~(H261B_MB_MC | H261B_MB_FILTER))) {
            fail_arg(where, "mode decision has a type, flag or vector the search cannot produce");
            return;
        }
    }
    /* the host packing of gpu_device.cu:614-629, kept for callers that read it */
    const int32_t pq = ctx->s_picture.i_quantiser;
    for (int32_t i = 0; i < n; i++) {
        const h261_mb_mode_decision_t &m = md->prgs_mb[i];
        int32_t q = pq + m.i_quantiser_adjust;
        s->pi_mb_types_host[i] = m.i_mb_type;
        s->pi_mb_flags_host[i] = m.i_mb_flags;
        s->pi_mb_mv_x_host[i] = m.i_mv_x;
        s->pi_mb_mv_y_host[i] = m.i_mv_y;
        s->pi_mb_quant_host[i] = q < 1 ? 1 : q > 31 ? 31 : q;
    }
    CK(where, cudaMemcpyAsync(g.md_dev, md->prgs_mb, sizeof(h261_mb_mode_decision_t) * n, cudaMemcpyHostToDevice,
                              g.stream));
    h261b_session_dev_t d;
    base_desc(d);
    d.quant = pq;
    d.dn = g.dn_dev;
    d.md_in = g.md_dev;
    d.abi_out = s->ps_macroblocks_device;
    d.frame_type = ctx->s_picture.i_frame_type;
    CK(where, cudaMemcpyAsync(g.desc_dev, &d, sizeof(d), cudaMemcpyHostToDevice, g.stream));
    int rc = h261b_launch_step(g.desc_dev, g.work_dev, n,
                               H261B_PHASE_ENCDEC | H261B_ABI_OUT | (g.me_mode ? H261B_LAUNCH_ME_FULL : 0) |
                                   (g.fmad ? H261B_FMAD_BIT : 0),
                               4, 0, nullptr, g.stream);
    if (rc) {
        fail(where, (cudaError_t)rc);
        return;
    }
    CK(where, cudaMemcpyAsync(s->ps_macroblocks, s->ps_macroblocks_device, sizeof(h261_macroblock_t) * n,
                              cudaMemcpyDeviceToHost, g.stream));
    CK(where, cudaStreamSynchronize(g.stream));
}

extern "C" void h261_gpu_device_decode_macroblocks(h261_context_t *ctx)
{
    const char *where = "h261_gpu_device_decode_macroblocks";
    if (!ensure_ready(where))
        return;
    if (!ctx || !ctx->ps_macroblocks) {
        fail_arg(where, "context is missing macroblocks");
        return;
    }
    h261_macroblocks_t *s = ctx->ps_macroblocks;
    const size_t ny = (size_t)g.w * g.h, nc = ny / 4;
    CK(where, cudaMemcpyAsync(s->pui8_reconstructed_Y_host, g.rec + g.lay.off_y, ny, cudaMemcpyDeviceToHost,
                              g.stream));
    CK(where, cudaMemcpyAsync(s->pui8_reconstructed_Cb_host, g.rec + g.lay.off_cb, nc, cudaMemcpyDeviceToHost,
                              g.stream));
    CK(where, cudaMemcpyAsync(s->pui8_reconstructed_Cr_host, g.rec + g.lay.off_cr, nc, cudaMemcpyDeviceToHost,
                              g.stream));
    CK(where, cudaStreamSynchronize(g.stream));
}

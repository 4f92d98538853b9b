/* ratectrl.cu -- the picture QUANT of rate-controlled sessions, on the
 * device, between the step's search/mode-decision launch and its encode
 * launch (the arithmetic is in ratectrl_dev.h). */
#include <cuda_runtime.h>

#include "h261b_device.h"
#include "ratectrl_dev.h"

namespace h261b {
namespace {

__global__ void ratectrl_kernel(h261b_session_dev_t *sessions, int32_t n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    h261b_session_dev_t &S = sessions[i];
    if (!S.rc)
        return;
    rc_picture_quant(*S.rc, S.frame_type, S.mbw * S.mbh);
}

} // namespace
} // namespace h261b

extern "C" int h261b_launch_ratectrl(h261b_session_dev_t *sessions_dev, int32_t n_sessions, void *stream)
{
    if (n_sessions <= 0)
        return 0;
    h261b::ratectrl_kernel<<<(n_sessions + 127) / 128, 128, 0, (cudaStream_t)stream>>>(sessions_dev, n_sessions);
    return (int)cudaGetLastError();
}

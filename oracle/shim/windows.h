/* Empty stand-in for the Win32 header that the reference's
 * src/gpu_device.cu includes but does not use on this path; lets the
 * reference's CUDA source compile unchanged on Linux.  Test build only. */

// bd_common.cu -- status strings, version and device selection.
#include <cstdio>

#include "bd_internal.h"

namespace bd {

namespace {
int g_device = 0;
thread_local char g_last_cuda_error[256] = "";
}  // namespace

bd_status cuda_fail(cudaError_t err, const char *what, const char *file, int line)
{
    snprintf(g_last_cuda_error, sizeof g_last_cuda_error, "%s: %s (%s:%d)", what,
             cudaGetErrorString(err), file, line);
    if (err == cudaErrorMemoryAllocation) { return BD_ERR_OOM; }
    return BD_ERR_CUDA;
}

int current_device() { return g_device; }

bd_status ensure_device()
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= g_device) {
        cudaGetLastError();
        return BD_ERR_NODEV;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, g_device) != cudaSuccess) { return BD_ERR_NODEV; }
    // The kernels are built for sm_100a only.
    if (prop.major != 10) { return BD_ERR_NODEV; }
    if (cudaSetDevice(g_device) != cudaSuccess) { return BD_ERR_NODEV; }
    return BD_OK;
}

}  // namespace bd

extern "C" {

const char *bd_status_string(bd_status s)
{
    switch (s) {
        case BD_OK: return "ok";
        case BD_ERR_INVALID: return "invalid argument";
        case BD_ERR_IO: return "file cannot be opened, read or written";
        case BD_ERR_FORMAT: return "edge list or CSR rejected";
        case BD_ERR_OOM: return "out of memory";
        case BD_ERR_CUDA: return bd::g_last_cuda_error[0] ? bd::g_last_cuda_error : "CUDA error";
        case BD_ERR_TIMEOUT: return "device-side wait timed out";
        case BD_ERR_RANGE: return "vertex id out of range";
        case BD_ERR_STATE: return "call out of order";
        case BD_ERR_NODEV: return "no usable CUDA device (sm_100 required)";
        case BD_ERR_LIMIT: return "size beyond a supported limit";
        default: return "unknown status";
    }
}

const char *bd_version(void) { return "beedrill-b200 0.1.0 (sm_100a)"; }

bd_status bd_set_device(int device)
{
    if (device < 0) { return BD_ERR_INVALID; }
    bd::g_device = device;
    return BD_OK;
}

}  // extern "C"

// rpl_output.cu -- output during a run without stalling the time stepping: the snapshot export behind
// Oceananigans' fetch_output(::ProductField) = interior(field) (src/OceananigansIntegration.jl:7-9),
// per-step diagnostics into device memory, and pinned host buffers for both.
//
// A snapshot converts the current action from the device layout into the caller's layout (x fastest)
// in a staging buffer in HBM on the handle's stream, then copies the staging buffer to the caller's
// host buffer on a second stream. The steps that follow run while that copy crosses to the host; the
// next snapshot waits for it before reusing the staging buffer.
#include <cuda_runtime.h>

#include <string>

#include "rpl_internal.h"

namespace {

using rpl::Handle;

int ofail(int code, const std::string& msg) {
    rpl::set_last_error(msg);
    return code;
}

int ocuda(cudaError_t e, const char* what) {
    cudaGetLastError();
    return ofail(e == cudaErrorMemoryAllocation ? RPL_ERR_OOM : RPL_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

int ready(rpl_handle* hh, Handle** out) {
    if (!hh) return ofail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return ocuda(e, "cudaSetDevice");
    *out = h;
    return RPL_OK;
}

}  // namespace

namespace rpl {

void free_output(Handle* h) {
    if (h->snap_stream) {
        cudaStreamSynchronize(h->snap_stream);
        cudaStreamDestroy(h->snap_stream);
    }
    if (h->snap_ready) cudaEventDestroy(h->snap_ready);
    if (h->snap_done) cudaEventDestroy(h->snap_done);
    if (h->d_snap) {
        cudaFree(h->d_snap);
        h->bytes -= h->snap_bytes;
    }
    h->snap_stream = nullptr;
    h->snap_ready = h->snap_done = nullptr;
    h->d_snap = nullptr;
    h->snap_bytes = 0;
    h->snap_pending = false;
}

}  // namespace rpl

extern "C" {

int rpl_host_alloc(int64_t bytes, void** ptr) {
    if (!ptr || bytes < 0) return ofail(RPL_ERR_ARGUMENT, "rpl_host_alloc needs bytes >= 0 and an output pointer");
    *ptr = nullptr;
    cudaError_t e = cudaHostAlloc(ptr, bytes ? (size_t)bytes : 1, cudaHostAllocPortable);
    if (e != cudaSuccess) return ocuda(e, "cudaHostAlloc");
    return RPL_OK;
}

int rpl_host_free(void* ptr) {
    if (!ptr) return RPL_OK;
    cudaError_t e = cudaFreeHost(ptr);
    if (e != cudaSuccess) return ocuda(e, "cudaFreeHost");
    return RPL_OK;
}

int rpl_snapshot_async(rpl_handle* hh, void* host, int32_t dtype) {
    Handle* h = nullptr;
    int st = ready(hh, &h);
    if (st) return st;
    if (!host) return ofail(RPL_ERR_ARGUMENT, "null snapshot buffer");
    if (dtype != RPL_F64 && dtype != RPL_F32) return ofail(RPL_ERR_ARGUMENT, "unknown dtype");
    const int64_t bytes = h->units * (dtype == RPL_F64 ? 8 : 4);
    cudaError_t e;
    if (!h->snap_stream) {
        e = cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->snap_ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            rpl::free_output(h);
            return ocuda(e, "rpl_snapshot_async");
        }
    }
    if (h->snap_bytes < bytes) {
        // a larger staging buffer: the previous copy out of the old one must finish first
        e = cudaStreamSynchronize(h->snap_stream);
        if (e != cudaSuccess) return ocuda(e, "rpl_snapshot_async");
        if (h->d_snap) {
            cudaFree(h->d_snap);
            h->bytes -= h->snap_bytes;
            h->d_snap = nullptr;
            h->snap_bytes = 0;
        }
        if (h->desc.memory_limit_bytes > 0 && h->bytes + bytes > h->desc.memory_limit_bytes)
            return ofail(RPL_ERR_OOM, "the snapshot staging buffer (" + std::to_string(bytes) +
                                          " bytes) would exceed the memory limit");
        e = cudaMalloc(&h->d_snap, bytes);
        if (e != cudaSuccess) {
            h->d_snap = nullptr;
            return ocuda(e, "snapshot staging buffer");
        }
        h->snap_bytes = bytes;
        h->bytes += bytes;
    }
    cudaStream_t s = h->stream;
    if (h->snap_pending) {
        e = cudaStreamWaitEvent(s, h->snap_done, 0);
        if (e != cudaSuccess) return ocuda(e, "rpl_snapshot_async");
    }
    const int src = h->precision == RPL_FP64 ? RPL_F64 : RPL_F32;
    e = rpl::launch_from_device_layout(*h, h->N, src, h->d_snap, dtype, 0, h->desc.Np, 0, h->desc.Nk, s);
    if (e == cudaSuccess) e = cudaEventRecord(h->snap_ready, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->snap_stream, h->snap_ready, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, h->d_snap, bytes, cudaMemcpyDeviceToHost, h->snap_stream);
    if (e == cudaSuccess) e = cudaEventRecord(h->snap_done, h->snap_stream);
    if (e != cudaSuccess) return ocuda(e, "rpl_snapshot_async");
    h->snap_pending = true;
    return RPL_OK;
}

int rpl_snapshot_wait(rpl_handle* hh) {
    Handle* h = nullptr;
    int st = ready(hh, &h);
    if (st) return st;
    if (!h->snap_pending) return RPL_OK;
    cudaError_t e = cudaEventSynchronize(h->snap_done);
    if (e != cudaSuccess) return ocuda(e, "rpl_snapshot_wait");
    h->snap_pending = false;
    return RPL_OK;
}

int rpl_diagnostics_device(rpl_handle* hh, double* m0, double* hs, double* krms, double* mean_dir,
                           double* total_action) {
    Handle* h = nullptr;
    int st = ready(hh, &h);
    if (st) return st;
    cudaStream_t s = h->stream;
    const int64_t P = h->cells;
    cudaError_t e = rpl::launch_diagnostics(*h, h->N, s, hs || krms || mean_dir);
    double* outs[4] = {m0, hs, krms, mean_dir};
    for (int k = 0; k < 4 && e == cudaSuccess; ++k)
        if (outs[k]) e = cudaMemcpyAsync(outs[k], h->d_diag + k * P, P * 8, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && total_action)
        e = cudaMemcpyAsync(total_action, h->d_diag + 4 * P, 8, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return ocuda(e, "rpl_diagnostics_device");
    return RPL_OK;
}

}  // extern "C"

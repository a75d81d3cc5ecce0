// rpl_halo.cu -- row copies of the state buffers for a y-slab domain decomposition: a rank copies its
// boundary rows out of a stage's input buffer, exchanges them with its neighbours, and copies the
// received rows into its halo rows before launching that stage (rpl_stage_async). The reference runs
// one domain per architecture and has no counterpart.
//
// In the device layout (kappa fastest, then x, then y, then direction) the rows j0 .. j0+nrows-1 of one
// direction are one contiguous block of nrows*Nx*Nk words, so a copy is one strided 2-D copy over the
// Np directions into a packed (Np, nrows, Nx, Nk) buffer, stream-ordered on the handle's stream.
#include <cuda_runtime.h>

#include <string>

#include "rpl_internal.h"

namespace {

using rpl::Handle;

int hfail(int code, const std::string& msg) {
    rpl::set_last_error(msg);
    return code;
}

int rows_copy(rpl_handle* hh, int32_t which, int64_t row0, int64_t nrows, void* packed, bool out,
              cudaStream_t stream, bool own_stream) {
    if (!hh) return hfail(RPL_ERR_ARGUMENT, "null handle");
    Handle* h = reinterpret_cast<Handle*>(hh);
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return hfail(RPL_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    if (which < 0 || which > 2) return hfail(RPL_ERR_ARGUMENT, "buffer must be 0 (N), 1 (A) or 2 (B)");
    const rpl_desc& d = h->desc;
    if (!packed || row0 < 0 || nrows < 1 || row0 + nrows > d.Ny)
        return hfail(RPL_ERR_ARGUMENT, "rows out of range or null buffer");
    char* state = (char*)(which == 0 ? h->N : (which == 1 ? h->A : h->B));
    const size_t row_bytes = (size_t)(d.Nx * d.Nk) * h->elem;
    const size_t width = (size_t)nrows * row_bytes, pitch = (size_t)d.Ny * row_bytes;
    char* rows = state + (size_t)row0 * row_bytes;
    if (own_stream) stream = h->stream;
    e = out ? cudaMemcpy2DAsync(packed, width, rows, pitch, width, (size_t)d.Np, cudaMemcpyDeviceToDevice, stream)
            : cudaMemcpy2DAsync(rows, pitch, packed, width, width, (size_t)d.Np, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return hfail(RPL_ERR_CUDA, std::string(out ? "rpl_rows_get: " : "rpl_rows_set: ") + cudaGetErrorString(e));
    }
    return RPL_OK;
}

}  // namespace

extern "C" {

int rpl_rows_get(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, void* dst) {
    return rows_copy(h, which, row0, nrows, dst, true, nullptr, true);
}

int rpl_rows_set(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, const void* src) {
    return rows_copy(h, which, row0, nrows, const_cast<void*>(src), false, nullptr, true);
}

int rpl_rows_get_on(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, void* dst, void* stream) {
    return rows_copy(h, which, row0, nrows, dst, true, (cudaStream_t)stream, false);
}

int rpl_rows_set_on(rpl_handle* h, int32_t which, int64_t row0, int64_t nrows, const void* src, void* stream) {
    return rows_copy(h, which, row0, nrows, const_cast<void*>(src), false, (cudaStream_t)stream, false);
}

}  // extern "C"

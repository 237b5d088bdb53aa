// pe_noalloc.cu -- hairpin-stem objective for device-resident solutions without
// any device allocation.
//
// Who needs this: callers that may not call cudaMalloc/cudaFree -- code embedded
// in a host application whose memory manager has already reserved the GPU's
// memory (a caching allocator holding the whole device, a plugin that is handed
// buffers but may not allocate), and latency-critical loops that cannot pay the
// device-wide synchronisation of cudaMalloc/cudaFree.  They pass device pointers
// for inputs and outputs; the scratch the scan needs (nucleotide bit planes,
// per-CDS partial results, per-solution completion counters) lives in one
// fixed-size file-scope device array instead of being allocated.
//
// When the array's memory is taken: CUDA loads this file's device code, and with
// it the array, on each device the first time the code is used there (lazy module
// loading, the default since CUDA 12.2), so the first call on a device reserves
// the 8 MiB -- a call with n_solutions = 0 does only that set-up.  Make that call
// while setting up, before the host application's memory manager takes the
// device's memory and before any stream capture; with CUDA_MODULE_LOADING=EAGER
// the array is reserved when the CUDA context is created instead.  Afterwards the
// array stays reserved until the process exits, and no call allocates.  Every call
// uses the same array and finds it holding the previous call's data, so each call
// clears the parts that must start at zero itself; calls that overlap on the GPU
// (different streams, or a call issued while the previous one still runs
// elsewhere) race on it.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "pe_internal.h"

namespace pe {
namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;  // 8 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};

// nucleotide codes (one byte each, 0..3) -> (lo, hi) bit planes; outputs preset to
// NaN and -1 so a solution whose scan did not finish shows it in all three outputs
__global__ void k_pack_nt(const uint8_t *__restrict__ nt, int items, int n, int W, int Wp, uint2 *planes,
                          int nsol, float *value, int32_t *pql)
{
    size_t total = (size_t)items * Wp;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        size_t item = e / Wp;
        int w = (int)(e - item * Wp);
        uint32_t lo = 0, hi = 0;
        if (w < W) {
            const uint8_t *row = nt + item * n;
            int lim = min(32, n - 32 * w);
            for (int i = 0; i < lim; i++) {
                uint32_t code = row[32 * w + i] & 3u;
                lo |= (code & 1u) << i;
                hi |= (code >> 1) << i;
            }
        }
        planes[e] = make_uint2(lo, hi);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsol; i += gridDim.x * blockDim.x) {
        value[i] = __int_as_float(0x7fc00000);
        pql[3 * i] = pql[3 * i + 1] = pql[3 * i + 2] = -1;
    }
}

__global__ void k_clear_counters(int32_t *counter, int nsol, int32_t *status)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsol; i += gridDim.x * blockDim.x) counter[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *status = 0;
}

// the stem's CDS, or -1 where the scan did not finish (value still NaN)
__global__ void k_copy_cds(const int8_t *objidx, const float *value, int nsol, int8_t *cds)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsol; i += gridDim.x * blockDim.x)
        cds[i] = isnan(value[i]) ? (int8_t)-1 : objidx[2 * i];
}

// device address of the scratch array for the current device (looked up once per device)
int scratch_for_current_device(unsigned char **out, const char **err)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *err = "no usable current CUDA device";
        return PE_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            *err = cudaGetErrorString(e);
            return PE_ERR_CUDA;
        }
        g_scratch_ptr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_ptr[dev];
    return PE_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace pe

using namespace pe;

extern "C" int pe_hairpin_noalloc(const uint8_t *d_nt, int32_t n_solutions, int32_t m, int32_t L, float *d_value,
                                  int32_t *d_pql, int8_t *d_cds, void *cuda_stream)
{
    if (n_solutions < 0) {
        set_error_text("pe_hairpin_noalloc: negative count");
        return PE_ERR_ARG;
    }
    if (n_solutions == 0) {
        // set-up only: load this file's device code on the current device, which
        // reserves the scratch array, and look its address up
        unsigned char *base = nullptr;
        const char *err = nullptr;
        int rc = scratch_for_current_device(&base, &err);
        if (rc != PE_OK) set_error_text(err);
        return rc;
    }
    if (!d_nt || !d_value || !d_pql || !d_cds) {
        set_error_text("pe_hairpin_noalloc: null pointer");
        return PE_ERR_ARG;
    }
    if (m < 1 || m > kMaxCds || L < 3) {
        set_error_text("pe_hairpin_noalloc: need 1 <= m <= 64 CDSs and L >= 3 positions");
        return PE_ERR_ARG;
    }
    Shape s{};
    s.L = L;
    s.Lp = (L + 15) & ~15;
    s.m = m;
    s.N = n_solutions;
    s.M = 1;
    s.n = 3 * L;
    s.W = (s.n + 31) / 32;
    s.Wp = (s.W + 2) & ~1;
    s.K = (s.n - 4) / 2;
    for (int k = 0; k < 6; k++) s.slot[k] = -1;
    s.slot[K_SL] = 0;
    const size_t items = (size_t)n_solutions * m;
    const size_t off_status = 0;
    const size_t off_counter = 256;
    const size_t off_part = align256(off_counter + sizeof(int32_t) * (size_t)n_solutions);
    const size_t off_objidx = align256(off_part + sizeof(int2) * items);
    const size_t off_planes = align256(off_objidx + 2 * (size_t)n_solutions);
    const size_t need = off_planes + sizeof(uint2) * items * (size_t)s.Wp;
    if (need > kScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "pe_hairpin_noalloc: %d solutions x %d CDSs of %d positions need %zu bytes of scratch; the fixed "
                 "scratch holds %zu bytes",
                 n_solutions, m, L, need, kScratchBytes);
        set_error_text(msg);
        return PE_ERR_ARG;
    }
    int dev = 0;
    int smem_optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        set_error_text("pe_hairpin_noalloc: no usable CUDA device");
        return PE_ERR_NO_DEVICE;
    }
    if (sl_smem_bytes(s) > (size_t)smem_optin) {
        set_error_text("pe_hairpin_noalloc: CDS too long for the shared-memory scan");
        return PE_ERR_ARG;
    }
    unsigned char *base = nullptr;
    const char *err = nullptr;
    int rc = scratch_for_current_device(&base, &err);
    if (rc != PE_OK) {
        set_error_text(err);
        return rc;
    }
    cudaStream_t st = (cudaStream_t)cuda_stream;
    int32_t *status = (int32_t *)(base + off_status);
    int32_t *counter = (int32_t *)(base + off_counter);
    int2 *part = (int2 *)(base + off_part);
    int8_t *objidx = (int8_t *)(base + off_objidx);
    uint2 *planes = (uint2 *)(base + off_planes);
    k_clear_counters<<<(n_solutions + 255) / 256, 256, 0, st>>>(counter, n_solutions, status);
    size_t words = items * s.Wp;
    int blocks = (int)std::min<size_t>((words + 255) / 256, 4096);
    k_pack_nt<<<blocks, 256, 0, st>>>(d_nt, (int)items, s.n, s.W, s.Wp, planes, n_solutions, d_value, d_pql);
    PopBuf buf{};
    buf.planes = planes;
    buf.obj = d_value;
    buf.objidx = objidx;
    buf.pql = d_pql;
    cudaError_t e = launch_sl(s, buf, 0, n_solutions, part, counter, status, st);
    if (e == cudaSuccess) {
        k_copy_cds<<<(n_solutions + 255) / 256, 256, 0, st>>>(objidx, d_value, n_solutions, d_cds);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_error_text(cudaGetErrorString(e));
        return PE_ERR_CUDA;
    }
    return PE_OK;
}

// noalloc.cu -- parity verification that allocates no device memory.
//
// Who needs this: callers that cannot call cudaMalloc when they verify
// parity.  Typical cases are a storage or serving process that reserved its
// whole HBM budget at start-up and only lends the library the shard buffers,
// and latency-critical paths where a cudaMalloc is not acceptable because it
// can synchronise the device and can fail under fragmentation.  The regular
// rsgpu_check_some_shards needs a context (whose creation allocates a stream,
// a flag and grows a scratch buffer); this entry point needs neither.
//
// Its only scratch memory is g_noalloc_scratch below, a file-scope device
// array of kNoAllocScratchBytes (8 MiB).  It holds the mismatch flag and,
// when there are more inputs than one kernel launch takes (32), the partial
// parity rows; calls whose partial rows would not fit are rejected.
//
// Device memory is also taken when code is loaded: with lazy module loading
// (the CUDA default) a module is loaded, and its memory allocated, when one
// of its symbols is first used.  So the first call on a device does all of
// that up front: it looks up the array's device address (which loads this
// file's module, array included) and loads every kernel this entry point can
// launch (a fixed set of table kernels, the same for every geometry).  From
// then on, calls on that device allocate nothing.  Callers should make one
// call at start-up, before any stream capture; every GPU that has run it
// holds the array and the loaded code until the process exits.
#include <cstring>
#include <mutex>

#include "rsgpu_internal.h"

namespace rsgpu {
namespace {

constexpr size_t kNoAllocScratchBytes = 8u << 20;  // per device
constexpr size_t kFlagBytes = 256;                 // mismatch flag, padded to keep rows aligned
constexpr int kMaxDevices = 64;

__device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
uint8_t *g_scratch_addr[kMaxDevices];
DeviceInfo g_info[kMaxDevices];
bool g_ready[kMaxDevices];

// Once per device, with that device current: the device address of the
// array (in host code the symbol itself is only a host-side stand-in), the
// SM count used to size grids, and every kernel the calls launch loaded.
int device_scratch(uint8_t **scratch, DeviceInfo *info) {
    int dev = 0;
    RS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return RS_ERR_INVALID_INPUT;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_ready[dev]) {
        void *p = nullptr;
        RS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        int sms = 0;
        RS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        RS_CUDA(preload_static_kernels());
        g_scratch_addr[dev] = (uint8_t *)p;
        g_info[dev].device = dev;
        g_info[dev].sm_count = sms;
        g_ready[dev] = true;
    }
    *scratch = g_scratch_addr[dev];
    *info = g_info[dev];
    return RS_OK;
}

}  // namespace
}  // namespace rsgpu

using namespace rsgpu;

extern "C" int rsgpu_check_some_shards_noalloc(const uint8_t *rows, int n_in, int n_out,
                                               const uint8_t *const *in,
                                               const uint8_t *const *to_check, size_t nbytes,
                                               void *stream, int *ok) {
    if (!ok || !rows || !in || !to_check || n_in <= 0 || n_out < 0) return RS_ERR_INVALID_INPUT;
    *ok = 0;
    if (n_out == 0 || nbytes == 0) {
        *ok = 1;
        return RS_OK;
    }
    const size_t pitch = (nbytes + 255) & ~(size_t)255;
    if (n_in > kMaxIn && (size_t)n_out * pitch > kNoAllocScratchBytes - kFlagBytes) {
        set_error("rsgpu_check_some_shards_noalloc: more than 32 inputs needs n_out * shard bytes "
                  "(rounded up to 256) <= 8 MiB - 256 of static scratch");
        return RS_ERR_INVALID_INPUT;
    }
    uint8_t *scratch = nullptr;
    DeviceInfo info;
    int rc = device_scratch(&scratch, &info);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int *d_flag = reinterpret_cast<int *>(scratch);
    // The array keeps the previous call's contents: the flag must start at 0.
    RS_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), st));
    if (n_in <= kMaxIn) {
        RS_CUDA(launch_gf8_matmul_static(st, info, rows, n_in, n_out, in,
                                         const_cast<uint8_t *const *>(to_check), nbytes, kModeVerify, d_flag));
    } else {
        uint8_t *tmp[kMaxOut];
        for (int o0 = 0; o0 < n_out; o0 += kMaxOut) {
            // partial rows fit by the check above; outputs are processed in
            // groups of kMaxOut so the rows pointer array stays on the stack
            const int no = n_out - o0 < kMaxOut ? n_out - o0 : kMaxOut;
            for (int o = 0; o < no; o++) tmp[o] = scratch + kFlagBytes + pitch * (size_t)(o0 + o);
            RS_CUDA(launch_gf8_matmul_static(st, info, rows + (size_t)o0 * n_in, n_in, no, in, tmp, nbytes,
                                             kModeWrite, d_flag));
            const uint8_t one = 1;
            for (int o = 0; o < no; o++) {
                const uint8_t *src = tmp[o];
                uint8_t *chk = const_cast<uint8_t *>(to_check[o0 + o]);
                RS_CUDA(launch_gf8_matmul_static(st, info, &one, 1, 1, &src, &chk, nbytes, kModeVerify, d_flag));
            }
        }
    }
    int h_flag = 0;
    RS_CUDA(cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    RS_CUDA(cudaStreamSynchronize(st));
    *ok = (h_flag == 0);
    return RS_OK;
}

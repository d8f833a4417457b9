// kernels_gf8_bitslice.cu -- host launcher of the bit-sliced run-time-
// coefficient GF(2^8) kernel (gf8_rt.cuh).
//
// Shape: one CTA per SM (grid = SM count, or fewer for small shards), up to
// 16 warps per CTA; every warp keeps a ring of n_in + ahead 1 KiB slots in
// dynamic shared memory, so wide input counts get fewer warps (RS(10,4):
// 13 KiB per warp, 16 warps; 32 inputs: 35 KiB, 6 warps).  Algorithmic bytes per
// launch: (n_in + n_out) * nbytes (+ n_out * nbytes read in xor / verify
// modes).
#include <algorithm>
#include <mutex>

#include "gf8_rt.cuh"

namespace rsgpu {
namespace {

constexpr int kMaxWarps = 16;  // the kernel is compiled for at most 512 threads per CTA
constexpr int kAhead = 3;  // next-chunk inputs issued before the last pass starts
constexpr int kMaxDevices = 64;

std::mutex g_mu;
int g_smem_optin[kMaxDevices];  // 0 = not set up on that device

// Opts the kernel in to the device's full per-block shared memory, once per
// device; returns the usable bytes.
int smem_limit(int device) {
    if (device < 0 || device >= kMaxDevices) return 48 << 10;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_smem_optin[device] == 0) {
        int optin = 0;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
            optin < (48 << 10))
            optin = 48 << 10;
        if (cudaFuncSetAttribute((const void *)gf8rt::gf8_bitslice_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess)
            optin = 48 << 10;
        g_smem_optin[device] = optin;
    }
    return g_smem_optin[device];
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

cudaError_t launch_bitslice(cudaStream_t st, const DeviceInfo &dev, const GfMatArgs &a, int mode,
                            long long *bytes_done) {
    *bytes_done = 0;
    const long long nchunk = a.nbytes / gf8rt::kChunk;
    if (nchunk == 0 || a.n_in < 1 || a.n_in > kMaxIn || a.n_out < 1 || a.n_out > kMaxOut) return cudaSuccess;
    for (int i = 0; i < a.n_in; i++)
        if (!aligned16(a.in[i])) return cudaSuccess;
    for (int o = 0; o < a.n_out; o++)
        if (!aligned16(a.out[o])) return cudaSuccess;
    const int ahead = std::min(a.n_in, kAhead);
    const int per_warp = (a.n_in + ahead) * gf8rt::kChunk;
    int warps = std::min(kMaxWarps, smem_limit(dev.device) / per_warp);
    if (warps < 1) return cudaSuccess;
    // fewer warps per CTA while that leaves SMs idle (small shards)
    while (warps > 1 && nchunk < (long long)dev.sm_count * warps) warps >>= 1;
    const int threads = 32 * warps;
    const size_t smem = (size_t)warps * per_warp;
    const long long want = (nchunk + warps - 1) / warps;
    const int grid = (int)std::max(1LL, std::min(want, (long long)dev.sm_count));
    gf8rt::gf8_bitslice_kernel<<<grid, threads, smem, st>>>(a, nchunk, mode, ahead);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) *bytes_done = nchunk * gf8rt::kChunk;
    return e;
}

}  // namespace rsgpu

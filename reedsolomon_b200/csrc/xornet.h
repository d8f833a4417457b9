// xornet.h -- run-time generated bit-sliced XOR-network kernels (xornet.cpp).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "kernels.h"

namespace rsgpu {

constexpr int kXornetChunk = 1024;   // bytes of every shard per warp step
constexpr int kXornetMaxOut = 16;
constexpr int kXornetCacheCap = 512; // matrices kept per process; the least recently used idle one is evicted
constexpr size_t kXornetDefaultMin = 256 << 10;  // untuned default from this many bytes per shard

// Threads per CTA of a tile's kernel: 512 (a 128-register cap, 16 warps per
// SM) up to 6 outputs; 256 beyond, where the accumulators need more registers.
int xornet_threads(int n_out);
// Preferred inputs per factoring pass: 3 up to 6 outputs, 2 beyond (wider
// tiles need the registers for their accumulators); the compile falls back
// to smaller groups when ptxas spills.
int xornet_group(int n_out);
// True when NVRTC could be loaded (the XOR-network variant exists).
bool xornet_available();
// Compiles (now) the kernel for a's coefficients; false when it cannot exist.
bool xornet_prepare(const GfMatArgs &a, int mode);
// NVRTC compilations run by this process (kernels read from the on-disk
// cache, RSGPU_KERNEL_CACHE, do not count).
int xornet_compile_count();
// Waits for queued background compiles; returns the number of compiled kernels.
int xornet_wait_idle();
// Drops queued background compiles and waits (bounded) for those running.
void xornet_drain();
// Runs the XOR-network kernel over the whole 1 KiB chunks of a (16-byte
// aligned shards only).  *bytes_done is 0 when it did not run: no NVRTC, an
// unaligned pointer, a tile too large, or (sync == false) a matrix whose
// background compile has not finished; the caller covers the rest.
cudaError_t xornet_launch(cudaStream_t st, const DeviceInfo &dev, const GfMatArgs &a, int mode, bool sync,
                          long long *bytes_done);
// Generated text for one mode (GfMode): the kernel source; the same schedule
// as a plain C function rs_xornet_host(in, out, nchunk, flag) over host
// arrays (for checking the generator on the CPU); and the shared body.
// group: inputs per factoring pass (0: xornet_group(n_out)).
std::string xornet_source(const uint8_t *coef, int stride, int n_in, int n_out, int mode, int group);
std::string xornet_host_source(const uint8_t *coef, int stride, int n_in, int n_out, int mode, int group);
std::string xornet_body(const uint8_t *coef, int stride, int n_in, int n_out, int mode, int group);

}  // namespace rsgpu

// kernels.h -- launch interfaces of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace rsgpu {

// Limits of one GF(2^8) matrix launch; larger matrices are tiled by the host
// the way codeSomeShardsAVXP tiles into 10x10 plans (reedsolomon.go:1073-1153).
constexpr int kMaxIn = 32;   // inputs per launch
constexpr int kMaxOut = 16;  // outputs per launch (4 groups of 4 packed bytes)

enum GfMode : int { kModeWrite = 0, kModeXor = 1, kModeVerify = 2 };

struct DeviceInfo {
    int device = 0;
    int sm_count = 148;
};

// Kernel parameter block (passed by value, < 1 KB).
struct GfMatArgs {
    const uint8_t *in[kMaxIn];
    uint8_t *out[kMaxOut];
    uint8_t coef[kMaxOut][kMaxIn];
    long long nbytes;  // bytes of every shard to process, from the given pointers
    int n_in, n_out;
    int *flag;         // verify: set to 1 on any mismatch
    // Nibble-address multipliers for the mul.hi address variant (runtime
    // values, so the compiler cannot turn the multiplies back into shifts).
    uint32_t mul[8];
};

// Nibble address generation variants of the GF(2^8) kernel (all compute the
// same bytes; the autotuner picks one per geometry and size bucket).
enum GfVariant : int {
    kVariantShift = 0,  // shift + mask/or on the ALU pipe
    kVariantMulHi = 1,  // shifts as mul.hi on the FMA pipe, mask/or on the ALU pipe
    kVariantPrmt = 2,   // nibble*4 bytes, PRMT merges them into the table base
    kVariantFixed = 3,  // PRMT addressing, input loop unrolled for the exact input count
    kVariantFixed2 = 4, // as kVariantFixed, registers capped for 2 resident CTAs per SM
    kVariantFixed3 = 5, // as kVariantFixed, registers capped for 3 resident CTAs per SM
    kVariantFixed4 = 6, // as kVariantFixed, registers capped for 4 resident CTAs per SM
    kVariantXorNet = 7, // bit-sliced XOR network generated for the tile's coefficients (xornet.cpp)
    kVariantBitslice = 8, // bit-sliced, coefficients read at run time (gf8_rt.cuh): no compile per matrix
    kNumVariants = 9,
};

// Force a variant for every launch (-1 restores the tuned / default choice).
void set_forced_variant(int v);
int forced_variant();
int choose_variant(int n_in, int n_out, int mode, size_t nbytes);
void record_variant(int n_in, int n_out, int mode, size_t nbytes, int v);  // v < 0 erases
// Fill a parameter block for one tile (n_in <= kMaxIn, n_out <= kMaxOut).
void fill_args(GfMatArgs &a, const uint8_t *rows, int row_stride, int n_in, int n_out,
               const uint8_t *const *in, uint8_t *const *out, size_t nbytes, int *d_flag);
// Launch exactly one tile with the given variant.
cudaError_t launch_gf8_tile(cudaStream_t st, const DeviceInfo &dev, const GfMatArgs &a, int mode,
                            int variant);

// out[o] (^)= sum_i coef[o][i] * in[i] over nbytes.  Host tiles n_in > kMaxIn
// and n_out > kMaxOut.  rows is n_out x n_in row-major on the host.  For
// kModeVerify the sum is compared with out[] and *d_flag is set on mismatch
// (requires n_in <= kMaxIn; larger verifies are composed by the caller).
// allow_generated = false keeps every tile on the table kernels: no run-time
// compiled XOR-network module is loaded (a device allocation) or queued.
cudaError_t launch_gf8_matmul(cudaStream_t st, const DeviceInfo &dev, const uint8_t *rows, int n_in,
                              int n_out, const uint8_t *const *in, uint8_t *const *out,
                              size_t nbytes, int mode, int *d_flag, bool allow_generated = true);

// Runs the bit-sliced run-time-coefficient kernel (kernels_gf8_bitslice.cu)
// over the whole 1 KiB chunks of a (16-byte aligned shards, n_in <= 32,
// n_out <= 16); *bytes_done is 0 when it did not run (unaligned pointers or
// no whole chunk); the caller covers the rest.
cudaError_t launch_bitslice(cudaStream_t st, const DeviceInfo &dev, const GfMatArgs &a, int mode,
                            long long *bytes_done);

// launch_gf8_matmul restricted to a fixed set of table kernels (one per
// output-group count and mode, plus the byte kernel for tails), chosen
// without the tuner and without occupancy queries.  After
// preload_static_kernels() has run on a device, launches of this set load no
// code there (with lazy module loading a kernel's first launch loads its
// module, which allocates device memory).
cudaError_t launch_gf8_matmul_static(cudaStream_t st, const DeviceInfo &dev, const uint8_t *rows, int n_in,
                                     int n_out, const uint8_t *const *in, uint8_t *const *out, size_t nbytes,
                                     int mode, int *d_flag);
// Loads every kernel launch_gf8_matmul_static can launch on the current device.
cudaError_t preload_static_kernels();

// Fill an 8-byte aligned buffer with uniform pseudo-random bytes (tuning inputs).
cudaError_t launch_fill_random(cudaStream_t st, const DeviceInfo &dev, uint8_t *p, size_t nbytes,
                               uint64_t seed);

// out ^= in (sliceXor)
cudaError_t launch_xor(cudaStream_t st, const DeviceInfo &dev, const uint8_t *in, uint8_t *out,
                       size_t nbytes);

}  // namespace rsgpu

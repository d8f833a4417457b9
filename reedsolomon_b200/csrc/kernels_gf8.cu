// kernels_gf8.cu -- GF(2^8) matrix x shards contraction for sm_100a.
//
// Replaces the reference's generated SIMD kernels behind codeSomeShards
// (mulAvxTwo_IxO / mulGFNI_IxO_64 / galMulAVX2*, galois_gen_switch_amd64.go:
// 46-2104; algorithm in _gen/gen.go:339-1312) with one kernel family:
//
//   * Every CTA expands the coefficient block (<= 16 outputs x 32 inputs) into
//     packed nibble-product tables in shared memory: for input i, nibble half
//     h and output group g, 16 u32 words whose byte o is coef[4g+o][i]*(e<<4h).
//     A 16-word table spans 16 banks, so a warp's lookups never conflict.
//   * Each thread streams 16-byte vectors of every input once (coalesced,
//     evict-first, four inputs in flight) and accumulates ALL outputs in
//     registers: per input byte, two shared-memory lookups produce four
//     output bytes at once.
//   * Accumulators are 4x4 byte-transposed with PRMT and stored as 16-byte
//     vectors; verify mode compares instead of storing (fused checkSomeShards).
//
// The byte work is bound by integer issue (nibble address generation, PRMT /
// LOP3 on the ALU pipe) and shared-memory lookups next to HBM; the address
// generation variants trade ALU for FMA/PRMT work, an input-count-specialised
// kernel removes the loop overhead, and the tuner keeps the fastest.  Algorithmic bytes: (n_in + n_out) * nbytes
// (+ n_out * nbytes read in xor / verify modes).
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "gf8_device.cuh"
#include "gf8_fixed.cuh"
#include "kernels.h"
#include "xornet.h"

namespace rsgpu {
namespace {

using namespace gf8dev;

// Loads batch b (inputs 4b..4b+3) of vector v; inputs past n_in are skipped.
__device__ __forceinline__ void load_batch(const GfMatArgs &a, long long v, int b, uint4 (&x)[4]) {
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (4 * b + j < a.n_in) x[j] = ld_in(a.in[4 * b + j], v);
}

template <int G, int MODE, int V>
__global__ void __launch_bounds__(kThreads) gf8_matmul_vec(const __grid_constant__ GfMatArgs a) {
    extern __shared__ __align__(128) uint32_t smem_raw[];
    uint32_t *tab = aligned_tables(smem_raw);
    const long long nvec = a.nbytes >> 4;
    const long long stride = (long long)gridDim.x * kThreads;
    long long v = (long long)blockIdx.x * kThreads + threadIdx.x;
    // Software pipeline: the next batch of four 16-byte input vectors is
    // always in flight while the current batch is multiplied; the first
    // batch is issued before the table build.
    uint4 nx[4] = {};
    if (v < nvec) load_batch(a, v, 0, nx);
    build_tables<G>(tab, a);
    Mul mu;
#pragma unroll
    for (int j = 0; j < 8; j++) mu.m[j] = a.mul[j];
    __syncthreads();
    const uint32_t tab_s = (uint32_t)__cvta_generic_to_shared(tab);
    const int n_in = a.n_in;
    const int nb = (n_in + 3) >> 2;
    uint32_t mism = 0;
    for (; v < nvec; v += stride) {
        uint32_t acc[G][16];
#pragma unroll
        for (int g = 0; g < G; g++)
#pragma unroll
            for (int b = 0; b < 16; b++) acc[g][b] = 0;
        for (int b = 0; b < nb; b++) {
            uint4 cur[4];
#pragma unroll
            for (int j = 0; j < 4; j++) cur[j] = nx[j];
            const bool last = (b + 1 == nb);
            const long long nv = last ? v + stride : v;
            if (nv < nvec) load_batch(a, nv, last ? 0 : b + 1, nx);
            const uint32_t base = tab_s + 4 * b * kInStride;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (4 * b + j < n_in) mac_vec<G, V>(cur[j], base + j * kInStride, mu, acc);
        }
#pragma unroll
        for (int g = 0; g < G; g++) {
            uint4 w[4];
            transpose4x4(acc[g][0], acc[g][1], acc[g][2], acc[g][3], w[0].x, w[1].x, w[2].x, w[3].x);
            transpose4x4(acc[g][4], acc[g][5], acc[g][6], acc[g][7], w[0].y, w[1].y, w[2].y, w[3].y);
            transpose4x4(acc[g][8], acc[g][9], acc[g][10], acc[g][11], w[0].z, w[1].z, w[2].z, w[3].z);
            transpose4x4(acc[g][12], acc[g][13], acc[g][14], acc[g][15], w[0].w, w[1].w, w[2].w, w[3].w);
#pragma unroll
            for (int o = 0; o < 4; o++) {
                const int oo = 4 * g + o;
                if (oo >= a.n_out) break;
                uint4 *dst = reinterpret_cast<uint4 *>(a.out[oo]) + v;
                if (MODE == kModeWrite) {
                    __stcs(dst, w[o]);
                } else if (MODE == kModeXor) {
                    uint4 old = __ldcs(dst);
                    old.x ^= w[o].x; old.y ^= w[o].y; old.z ^= w[o].z; old.w ^= w[o].w;
                    __stcs(dst, old);
                } else {
                    const uint4 chk = __ldcs(dst);
                    mism |= (chk.x ^ w[o].x) | (chk.y ^ w[o].y) | (chk.z ^ w[o].z) | (chk.w ^ w[o].w);
                }
            }
        }
    }
    if (MODE == kModeVerify && mism) *reinterpret_cast<volatile int *>(a.flag) = 1;
}

// One byte position per thread: tails and misaligned pointers.
template <int G, int MODE>
__global__ void __launch_bounds__(kThreads) gf8_matmul_bytes(const __grid_constant__ GfMatArgs a,
                                                             long long first) {
    extern __shared__ __align__(128) uint32_t smem_raw[];
    uint32_t *tab = aligned_tables(smem_raw);
    build_tables<G>(tab, a);
    __syncthreads();
    uint32_t mism = 0;
    for (long long pos = first + (long long)blockIdx.x * kThreads + threadIdx.x; pos < a.nbytes;
         pos += (long long)gridDim.x * kThreads) {
        uint32_t acc[G];
#pragma unroll
        for (int g = 0; g < G; g++) acc[g] = 0;
        for (int i = 0; i < a.n_in; i++) {
            const uint32_t x = a.in[i][pos];
            const uint32_t *t = tab + i * (kInStride / 4);
#pragma unroll
            for (int g = 0; g < G; g++)
                acc[g] ^= t[g * 16 + (x & 15)] ^ t[kHalfStride / 4 + g * 16 + (x >> 4)];
        }
#pragma unroll
        for (int g = 0; g < G; g++)
#pragma unroll
            for (int o = 0; o < 4; o++) {
                const int oo = 4 * g + o;
                if (oo >= a.n_out) break;
                const uint8_t r = (uint8_t)(acc[g] >> (8 * o));
                if (MODE == kModeWrite) a.out[oo][pos] = r;
                else if (MODE == kModeXor) a.out[oo][pos] ^= r;
                else mism |= (uint32_t)(a.out[oo][pos] ^ r);
            }
    }
    if (MODE == kModeVerify && mism) *reinterpret_cast<volatile int *>(a.flag) = 1;
}

__global__ void __launch_bounds__(kThreads) xor_vec(const uint4 *__restrict__ in, uint4 *out, long long nvec) {
    for (long long v = (long long)blockIdx.x * kThreads + threadIdx.x; v < nvec;
         v += (long long)gridDim.x * kThreads) {
        const uint4 x = __ldcs(in + v);
        uint4 y = __ldcs(out + v);
        y.x ^= x.x; y.y ^= x.y; y.z ^= x.z; y.w ^= x.w;
        __stcs(out + v, y);
    }
}

__global__ void __launch_bounds__(kThreads) xor_bytes(const uint8_t *__restrict__ in, uint8_t *out,
                                                      long long first, long long n) {
    for (long long p = first + (long long)blockIdx.x * kThreads + threadIdx.x; p < n;
         p += (long long)gridDim.x * kThreads)
        out[p] ^= in[p];
}

// Uniform pseudo-random bytes (splitmix64 of the word index and a seed), so
// tuning runs see lookups spread like real shard data.
__global__ void __launch_bounds__(kThreads) fill_random(uint64_t *p, long long nwords, uint64_t seed) {
    for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < nwords;
         i += (long long)gridDim.x * kThreads) {
        uint64_t z = seed + (uint64_t)i * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        p[i] = z ^ (z >> 31);
    }
}

typedef void (*ByteKernel)(GfMatArgs, long long);

template <int G, int MODE>
VecKernel pick_variant(int v) {
    if (v == kVariantShift) return gf8_matmul_vec<G, MODE, kVariantShift>;
    if (v == kVariantMulHi) return gf8_matmul_vec<G, MODE, kVariantMulHi>;
    return gf8_matmul_vec<G, MODE, kVariantPrmt>;
}
template <int G>
VecKernel pick_vec(int mode, int v) {
    if (mode == kModeWrite) return pick_variant<G, kModeWrite>(v);
    if (mode == kModeXor) return pick_variant<G, kModeXor>(v);
    return pick_variant<G, kModeVerify>(v);
}
template <int G>
ByteKernel pick_bytes(int mode) {
    if (mode == kModeWrite) return gf8_matmul_bytes<G, kModeWrite>;
    if (mode == kModeXor) return gf8_matmul_bytes<G, kModeXor>;
    return gf8_matmul_bytes<G, kModeVerify>;
}

// nullptr when no specialisation exists for (n_in, G).
VecKernel fixed_kernel(int n_in, int G, int mode, int variant) {
    if (variant == kVariantFixed2) return fixed_kernel_minb2(n_in, G, mode);
    if (variant == kVariantFixed3) return fixed_kernel_minb3(n_in, G, mode);
    if (variant == kVariantFixed4) return fixed_kernel_minb4(n_in, G, mode);
    return fixed_kernel_minb1(n_in, G, mode);
}

VecKernel vec_kernel(int G, int mode, int v) {
    switch (G) {
    case 1: return pick_vec<1>(mode, v);
    case 2: return pick_vec<2>(mode, v);
    case 3: return pick_vec<3>(mode, v);
    default: return pick_vec<4>(mode, v);
    }
}
ByteKernel byte_kernel(int G, int mode) {
    switch (G) {
    case 1: return pick_bytes<1>(mode);
    case 2: return pick_bytes<2>(mode);
    case 3: return pick_bytes<3>(mode);
    default: return pick_bytes<4>(mode);
    }
}

std::mutex g_mu;

// Resident CTAs per SM of a kernel at a shared-memory size (cached).
int blocks_per_sm(VecKernel k, size_t smem) {
    static std::map<std::pair<const void *, size_t>, int> cache;
    std::lock_guard<std::mutex> lk(g_mu);
    int &c = cache[std::make_pair((const void *)k, smem)];
    if (c == 0) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void *)k, kThreads, smem) != cudaSuccess ||
            nb < 1)
            nb = 1;
        c = nb;
    }
    return c;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int g_forced = -1;
std::map<std::tuple<int, int, int, int>, int> g_tuned;

int size_bucket(size_t nbytes) {
    int b = 0;
    while (b < 48 && ((size_t)1 << (b + 1)) <= nbytes) b++;
    return b;
}

}  // namespace

void set_forced_variant(int v) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_forced = (v >= 0 && v < kNumVariants) ? v : -1;
}

int forced_variant() {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_forced;
}

namespace {
// The untuned table-kernel choice (see choose_variant).
int table_variant(int n_out, int mode) {
    if (n_out > 4) return kVariantFixed2;
    return mode == kModeWrite ? kVariantFixed4 : kVariantFixed3;
}
}  // namespace

int choose_variant(int n_in, int n_out, int mode, size_t nbytes) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_forced >= 0) return g_forced;
    auto it = g_tuned.find(std::make_tuple(n_in, (n_out + 3) / 4, mode, size_bucket(nbytes)));
    if (it != g_tuned.end()) return it->second;
    // Untuned default from 256 KiB per shard: the generated XOR network when
    // NVRTC is present (faster than every table kernel at 16 MiB and above in
    // all measured geometries, and at 1 MiB with enough SMs covered); while a
    // new matrix's network compiles, the table kernel below runs instead.
    // Otherwise the unrolled table kernel with the most resident warps that
    // does not spill (up to 4 outputs: 4 CTAs per SM when writing, 3 when the
    // outputs are also read, which holds them in registers; 2 for 5-8
    // outputs); input counts without a specialisation fall back to
    // kVariantPrmt.  The bit-sliced run-time-coefficient kernel (variant 8)
    // is slower than the table kernel for every measured geometry but
    // single-output ones, so it runs only where the tuner picked it.
    if (nbytes >= kXornetDefaultMin && xornet_available()) return kVariantXorNet;
    return table_variant(n_out, mode);
}

void record_variant(int n_in, int n_out, int mode, size_t nbytes, int v) {
    std::lock_guard<std::mutex> lk(g_mu);
    const auto key = std::make_tuple(n_in, (n_out + 3) / 4, mode, size_bucket(nbytes));
    if (v < 0) g_tuned.erase(key);
    else g_tuned[key] = v;
}

void fill_args(GfMatArgs &a, const uint8_t *rows, int row_stride, int ni, int no,
               const uint8_t *const *in, uint8_t *const *out, size_t nbytes, int *d_flag) {
    for (int i = 0; i < kMaxIn; i++) a.in[i] = i < ni ? in[i] : nullptr;
    for (int o = 0; o < kMaxOut; o++) a.out[o] = o < no ? out[o] : nullptr;
    for (int o = 0; o < kMaxOut; o++)
        for (int i = 0; i < kMaxIn; i++)
            a.coef[o][i] = (o < no && i < ni) ? rows[(size_t)o * row_stride + i] : 0;
    a.nbytes = (long long)nbytes;
    a.n_in = ni;
    a.n_out = no;
    a.flag = d_flag;
    // lo nibble of byte j needs x >> (8j-2) (j=0: x << 2), hi nibble x >> (8j+2).
    const uint32_t mul[8] = {4u, 1u << 26, 1u << 18, 1u << 10, 1u << 30, 1u << 22, 1u << 14, 1u << 6};
    for (int j = 0; j < 8; j++) a.mul[j] = mul[j];
}

cudaError_t launch_gf8_tile(cudaStream_t st, const DeviceInfo &dev, const GfMatArgs &a, int mode,
                            int variant) {
    const int G = (a.n_out + 3) / 4;
    const size_t smem = (size_t)a.n_in * kInStride + kTableAlign;
    bool vec_ok = true;
    for (int i = 0; i < a.n_in; i++) vec_ok &= aligned16(a.in[i]);
    for (int o = 0; o < a.n_out; o++) vec_ok &= aligned16(a.out[o]);
    long long done = 0;
    if (variant == kVariantXorNet || variant == kVariantBitslice) {
        // Whole 1 KiB chunks through the generated network (compiled on the
        // spot when forced, else in the background; while it is not ready the
        // default table kernel covers everything) or through the bit-sliced
        // run-time-coefficient kernel; the tail through the table kernel.
        cudaError_t e = variant == kVariantXorNet
                            ? xornet_launch(st, dev, a, mode, forced_variant() == kVariantXorNet, &done)
                            : launch_bitslice(st, dev, a, mode, &done);
        if (e != cudaSuccess) return e;
        variant = table_variant(a.n_out, mode);
        if (done == a.nbytes) return cudaGetLastError();
        if (done > 0) {
            GfMatArgs t = a;
            for (int i = 0; i < a.n_in; i++) t.in[i] = a.in[i] + done;
            for (int o = 0; o < a.n_out; o++) t.out[o] = a.out[o] + done;
            t.nbytes = a.nbytes - done;
            return launch_gf8_tile(st, dev, t, mode, variant);
        }
    }
    if (vec_ok) {
        const long long nvec = a.nbytes >> 4;
        if (nvec > 0) {
            VecKernel kern = nullptr;
            const bool fixed = variant >= kVariantFixed;
            if (fixed) kern = fixed_kernel(a.n_in, G, mode, variant);
            if (!kern) kern = vec_kernel(G, mode, fixed ? kVariantPrmt : variant);
            const long long want = (nvec + kThreads - 1) / kThreads;
            const long long cap = (long long)dev.sm_count * blocks_per_sm(kern, smem);
            const int grid = (int)std::max(1LL, std::min(want, cap));
            kern<<<grid, kThreads, smem, st>>>(a);
            done = nvec << 4;
        }
    }
    if (done < a.nbytes) {
        const long long rem = a.nbytes - done;
        const long long want = (rem + kThreads - 1) / kThreads;
        const int grid = (int)std::max(1LL, std::min(want, (long long)dev.sm_count * 8));
        byte_kernel(G, mode)<<<grid, kThreads, smem, st>>>(a, done);
    }
    return cudaGetLastError();
}

cudaError_t launch_gf8_matmul(cudaStream_t st, const DeviceInfo &dev, const uint8_t *rows, int n_in,
                              int n_out, const uint8_t *const *in, uint8_t *const *out,
                              size_t nbytes, int mode, int *d_flag, bool allow_generated) {
    if (n_in <= 0 || n_out <= 0 || nbytes == 0) return cudaSuccess;
    for (int o0 = 0; o0 < n_out; o0 += kMaxOut) {
        const int no = std::min(kMaxOut, n_out - o0);
        for (int i0 = 0; i0 < n_in; i0 += kMaxIn) {
            const int ni = std::min(kMaxIn, n_in - i0);
            GfMatArgs a;
            fill_args(a, rows + (size_t)o0 * n_in + i0, n_in, ni, no, in + i0, out + o0, nbytes, d_flag);
            // Only the first input tile may overwrite; later tiles accumulate.
            const int m = (mode == kModeWrite && i0 > 0) ? kModeXor : mode;
            int v = choose_variant(ni, no, m, nbytes);
            if (!allow_generated && v == kVariantXorNet) v = table_variant(no, m);
            cudaError_t e = launch_gf8_tile(st, dev, a, m, v);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

// The fixed kernel set of launch_gf8_matmul_static: the PRMT-addressed
// table kernel (input loop not unrolled, so one kernel serves every input
// count) and the byte kernel, per output-group count and mode.
namespace {
constexpr int kStaticBlocksPerSm = 4;  // grid cap; the kernels loop over what is left

void static_kernels(int G, int mode, VecKernel *vk, ByteKernel *bk) {
    *vk = vec_kernel(G, mode, kVariantPrmt);
    *bk = byte_kernel(G, mode);
}
}  // namespace

cudaError_t preload_static_kernels() {
    for (int G = 1; G <= 4; G++)
        for (int mode = kModeWrite; mode <= kModeVerify; mode++) {
            VecKernel vk;
            ByteKernel bk;
            static_kernels(G, mode, &vk, &bk);
            cudaFuncAttributes fa;
            cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)vk);
            if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)bk);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

cudaError_t launch_gf8_matmul_static(cudaStream_t st, const DeviceInfo &dev, const uint8_t *rows, int n_in,
                                     int n_out, const uint8_t *const *in, uint8_t *const *out, size_t nbytes,
                                     int mode, int *d_flag) {
    if (n_in <= 0 || n_out <= 0 || nbytes == 0) return cudaSuccess;
    for (int o0 = 0; o0 < n_out; o0 += kMaxOut) {
        const int no = std::min(kMaxOut, n_out - o0);
        for (int i0 = 0; i0 < n_in; i0 += kMaxIn) {
            const int ni = std::min(kMaxIn, n_in - i0);
            GfMatArgs a;
            fill_args(a, rows + (size_t)o0 * n_in + i0, n_in, ni, no, in + i0, out + o0, nbytes, d_flag);
            const int m = (mode == kModeWrite && i0 > 0) ? kModeXor : mode;
            const int G = (no + 3) / 4;
            const size_t smem = (size_t)ni * kInStride + kTableAlign;
            VecKernel vk;
            ByteKernel bk;
            static_kernels(G, m, &vk, &bk);
            bool vec_ok = true;
            for (int i = 0; i < ni; i++) vec_ok &= aligned16(a.in[i]);
            for (int o = 0; o < no; o++) vec_ok &= aligned16(a.out[o]);
            long long done = 0;
            const long long cap = (long long)dev.sm_count * kStaticBlocksPerSm;
            if (vec_ok && (a.nbytes >> 4) > 0) {
                const long long nvec = a.nbytes >> 4;
                const int grid = (int)std::max(1LL, std::min((nvec + kThreads - 1) / kThreads, cap));
                vk<<<grid, kThreads, smem, st>>>(a);
                done = nvec << 4;
            }
            if (done < a.nbytes) {
                const long long rem = a.nbytes - done;
                const int grid = (int)std::max(1LL, std::min((rem + kThreads - 1) / kThreads, cap));
                bk<<<grid, kThreads, smem, st>>>(a, done);
            }
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_fill_random(cudaStream_t st, const DeviceInfo &dev, uint8_t *p, size_t nbytes,
                               uint64_t seed) {
    const long long nwords = (long long)(nbytes / 8);
    if (nwords == 0) return cudaSuccess;
    const int grid = (int)std::min<long long>((nwords + kThreads - 1) / kThreads, (long long)dev.sm_count * 8);
    fill_random<<<grid, kThreads, 0, st>>>(reinterpret_cast<uint64_t *>(p), nwords, seed);
    return cudaGetLastError();
}

cudaError_t launch_xor(cudaStream_t st, const DeviceInfo &dev, const uint8_t *in, uint8_t *out,
                       size_t nbytes) {
    if (nbytes == 0) return cudaSuccess;
    long long done = 0;
    if (aligned16(in) && aligned16(out)) {
        const long long nvec = (long long)(nbytes >> 4);
        if (nvec) {
            const long long want = (nvec + kThreads - 1) / kThreads;
            const int grid = (int)std::max(1LL, std::min(want, (long long)dev.sm_count * 8));
            xor_vec<<<grid, kThreads, 0, st>>>(reinterpret_cast<const uint4 *>(in),
                                               reinterpret_cast<uint4 *>(out), nvec);
            done = nvec << 4;
        }
    }
    if (done < (long long)nbytes) {
        const long long rem = (long long)nbytes - done;
        const int grid = (int)std::max(1LL, std::min((rem + kThreads - 1) / kThreads, (long long)dev.sm_count * 8));
        xor_bytes<<<grid, kThreads, 0, st>>>(in, out, done, (long long)nbytes);
    }
    return cudaGetLastError();
}

}  // namespace rsgpu

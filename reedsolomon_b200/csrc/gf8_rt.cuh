// gf8_rt.cuh -- bit-sliced GF(2^8) contraction with run-time coefficients.
//
// Multiplication by a constant c in GF(2^8) is linear over GF(2): bit b of
// c*x is the XOR of the bits a of x for which bit b of c*2^a is set (the 8x8
// bit matrices of the reference's GFNI path, genGFNIMatrix, galois.go:
// 1004-1016).  On bit-planes (bit a of 32 bytes in one 32-bit word) a product
// is therefore a fixed XOR pattern of whole words.  The run-time generated
// XOR network (xornet.cpp) bakes one matrix's coefficients into straight-line
// code and needs an NVRTC compile per matrix; this kernel is compiled once,
// ahead of time:
//
//   * all 256 "accumulate c*x" bodies exist in the binary, one per constant,
//     each a straight line of at most eight LOP3s;
//   * the coefficient of (output j, input i) is read at run time (kernel
//     parameter space, warp-uniform) and one indirect jump lands on its body:
//     every lane of a warp takes the same branch, so there is no divergence,
//     only the jump itself per (j, i) pair;
//   * a warp owns 1 KiB of every shard per step (lane l holds 16-byte vectors
//     l and l+32), transposes each input's eight words into bit-planes (three
//     delta-swap stages), forms the XORs of all subsets of its low and high
//     four planes (so each row of a body is one three-input XOR), keeps
//     4 x 8 accumulator planes in registers per pass over the inputs, and
//     transposes them back.
//
// Register arrays cannot be indexed by a run-time input number, and inlining
// the 256 bodies once per (output, input) pair makes the code, and ptxas's
// time (quadratic in the copies), explode.  So a warp's inputs are staged raw
// in a ring of 1 KiB slots in shared memory with cp.async: each lane owns its
// own 16-byte slots (no synchronisation, no bank conflicts), the input loop
// stays rolled, and the kernel holds exactly four copies of the bodies (one
// per accumulated output).  The next chunk's inputs are copied into the
// slots as this chunk consumes them, so loads overlap the arithmetic.
//
// Any matrix (a decode matrix of Reconstruct, ReconstructData, ReconstructSome,
// DecodeIdx, or a batched job's) runs this bit-sliced path with no compile and
// no module load.  Measured on B200 it is slower than the nibble-table kernel
// except for single-output tiles (RS(10,4) x 64 MiB encode: 0.232 ms against
// 0.204 ms; 10+1: 0.150 against 0.193 ms): each indirect jump costs about
// eight instructions of dispatch and an instruction-fetch redirect (warps
// wait on instruction fetch for ~17 % of their cycles), so it runs where the
// autotuner picks it, not by default.
#pragma once

#include <cstdint>

#include "gf8_rt_dispatch.inc"
#include "kernels.h"

namespace rsgpu {
namespace gf8rt {

constexpr int kChunk = 1024;  // bytes of every shard per warp step
constexpr int kPass = 4;      // outputs accumulated in registers per pass over the inputs

// The XORs of every non-empty subset of x's planes 0-3 (t[m-1] = lo[m]) and
// of planes 4-7 (t[14+m] = hi[m]), m = 1..15: 22 XORs per input, shared by
// all the outputs it feeds.
__device__ __forceinline__ void subset_xors(const uint32_t (&x)[8], uint32_t (&t)[30]) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
        uint32_t *T = t + 15 * h;  // T[m-1]
        const uint32_t *w = x + 4 * h;
        T[0] = w[0];
        T[1] = w[1];
        T[2] = w[0] ^ w[1];
        T[3] = w[2];
        T[4] = w[2] ^ w[0];
        T[5] = w[2] ^ w[1];
        T[6] = w[2] ^ T[2];
        T[7] = w[3];
#pragma unroll
        for (int m = 1; m < 8; m++) T[7 + m] = w[3] ^ T[m - 1];
    }
}

// y ^= c * x on bit-planes for a warp-uniform run-time coefficient c
// (0..255), given x's subset XORs t.  One indirect jump (PTX brx.idx over a
// list of 256 labels) lands on the body for c: row b of c*x XORs the planes
// of a fixed mask, i.e. lo[mask & 15] ^ hi[mask >> 4], so a body is at most
// eight three-input XORs (none for c = 0).  The bodies are generated at build
// time (gen_rt_dispatch.py); a C++ switch over the same cases compiles to a
// binary compare tree of about nine levels instead of one jump.
__device__ __forceinline__ void mul_acc_rt(uint32_t c, uint32_t (&y)[8], const uint32_t (&t)[30]) {
    asm(RSGPU_RT_DISPATCH_ASM
        : "+r"(y[0]), "+r"(y[1]), "+r"(y[2]), "+r"(y[3]), "+r"(y[4]), "+r"(y[5]), "+r"(y[6]), "+r"(y[7])
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]), "r"(t[8]),
          "r"(t[9]), "r"(t[10]), "r"(t[11]), "r"(t[12]), "r"(t[13]), "r"(t[14]), "r"(t[15]), "r"(t[16]),
          "r"(t[17]), "r"(t[18]), "r"(t[19]), "r"(t[20]), "r"(t[21]), "r"(t[22]), "r"(t[23]), "r"(t[24]),
          "r"(t[25]), "r"(t[26]), "r"(t[27]), "r"(t[28]), "r"(t[29]), "r"(c & 0xFFu));
}

// Exchanges bits (m << s) of x with bits m of y (one delta swap).
__device__ __forceinline__ void dswap(uint32_t &x, uint32_t &y, uint32_t m, int s) {
    const uint32_t xs = x >> s, ys = y << s;
    x = (x & ~(m << s)) | (ys & (m << s));
    y = (y & ~m) | (xs & m);
}

// 8x8 bit transpose of every byte lane of w[0..7] (an involution): word a
// becomes bit-plane a of the 32 bytes the eight words hold.
__device__ __forceinline__ void t8(uint32_t (&w)[8]) {
    dswap(w[0], w[4], 0x0F0F0F0Fu, 4); dswap(w[1], w[5], 0x0F0F0F0Fu, 4);
    dswap(w[2], w[6], 0x0F0F0F0Fu, 4); dswap(w[3], w[7], 0x0F0F0F0Fu, 4);
    dswap(w[0], w[2], 0x33333333u, 2); dswap(w[1], w[3], 0x33333333u, 2);
    dswap(w[4], w[6], 0x33333333u, 2); dswap(w[5], w[7], 0x33333333u, 2);
    dswap(w[0], w[1], 0x55555555u, 1); dswap(w[2], w[3], 0x55555555u, 1);
    dswap(w[4], w[5], 0x55555555u, 1); dswap(w[6], w[7], 0x55555555u, 1);
}

__device__ __forceinline__ void cp_async16(uint32_t smem_addr, const void *gptr) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr), "l"(gptr) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A lane's 32 bytes of one ring slot: 16-byte pieces at sa and sa + 512.
__device__ __forceinline__ void lds2(uint32_t sa, uint32_t (&x)[8]) {
    asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]) : "r"(sa));
    asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(x[4]), "=r"(x[5]), "=r"(x[6]), "=r"(x[7])
                 : "r"(sa + 512));
}
__device__ __forceinline__ void sts2(uint32_t sa, const uint32_t (&x)[8]) {
    asm volatile("st.shared.v4.u32 [%0], {%1,%2,%3,%4};" ::"r"(sa), "r"(x[0]), "r"(x[1]), "r"(x[2]), "r"(x[3])
                 : "memory");
    asm volatile("st.shared.v4.u32 [%0], {%1,%2,%3,%4};" ::"r"(sa + 512), "r"(x[4]), "r"(x[5]), "r"(x[6]),
                 "r"(x[7])
                 : "memory");
}

// The result of one output (eight planes, transposed back here) goes to
// 16-byte vectors v0 and v0+32 of dst: stored, XORed in, or compared.
__device__ __forceinline__ void finish_output(uint32_t (&y)[8], uint4 *dst, long long v0, int mode, uint32_t &diff) {
    t8(y);
    const uint4 r0 = make_uint4(y[0], y[1], y[2], y[3]);
    const uint4 r1 = make_uint4(y[4], y[5], y[6], y[7]);
    if (mode == kModeWrite) {
        __stcs(dst + v0, r0);
        __stcs(dst + v0 + 32, r1);
        return;
    }
    const uint4 e0 = __ldcs(dst + v0), e1 = __ldcs(dst + v0 + 32);
    if (mode == kModeXor) {
        __stcs(dst + v0, make_uint4(r0.x ^ e0.x, r0.y ^ e0.y, r0.z ^ e0.z, r0.w ^ e0.w));
        __stcs(dst + v0 + 32, make_uint4(r1.x ^ e1.x, r1.y ^ e1.y, r1.z ^ e1.z, r1.w ^ e1.w));
    } else {
        diff |= (r0.x ^ e0.x) | (r0.y ^ e0.y) | (r0.z ^ e0.z) | (r0.w ^ e0.w) | (r1.x ^ e1.x) | (r1.y ^ e1.y) |
                (r1.z ^ e1.z) | (r1.w ^ e1.w);
    }
}

// One pass over the inputs for outputs j0..j0+3 (all four exist when kFull;
// otherwise outputs from n_out on are skipped).  See bitslice_step.
template <bool kFull, typename CoefFn, typename NextFn>
__device__ __forceinline__ void bitslice_pass(uint32_t (&y)[kPass][8], uint32_t ring_s, int base, int ring, int lane,
                                              int n_in, int n_out, int j0, bool first, bool last, int ahead,
                                              CoefFn coef, NextFn issue_next) {
    int slot = base;
    for (int i = 0; i < n_in; i++) {
        const uint32_t sa = ring_s + (uint32_t)(slot * kChunk + lane * 16);
        uint32_t x[8];
        lds2(sa, x);
        if (first) {
            t8(x);
            if (!last) sts2(sa, x);
        }
        uint32_t t[30];
        subset_xors(x, t);
        mul_acc_rt(coef(j0, i), y[0], t);
        if (kFull || j0 + 1 < n_out) mul_acc_rt(coef(j0 + 1, i), y[1], t);
        if (kFull || j0 + 2 < n_out) mul_acc_rt(coef(j0 + 2, i), y[2], t);
        if (kFull || j0 + 3 < n_out) mul_acc_rt(coef(j0 + 3, i), y[3], t);
        // x has been consumed (the products depend on it), so the slot may
        // be overwritten by the next chunk's copy.
        if (last && i + ahead < n_in) issue_next(i + ahead, sa);
        slot = slot + 1 == ring ? 0 : slot + 1;
    }
}

// One warp's step over chunk c (1 KiB of every shard) whose raw input vectors
// have landed in the warp's ring (slot of input i: (base + i) mod ring).
// Outputs are produced kPass at a time; with more than one pass the first
// writes the transposed planes back into the ring so later passes skip the
// transpose.  During the last pass, once input i's slot has been consumed,
// issue_next(i + ahead, slot address) refills it with the next chunk's input.
template <typename CoefFn, typename OutFn, typename NextFn>
__device__ __forceinline__ void bitslice_step(uint32_t ring_s, int base, int ring, int lane, int n_in, int n_out,
                                              int ahead, int mode, long long v0, CoefFn coef, OutFn out,
                                              NextFn issue_next, uint32_t &diff) {
    const int npass = (n_out + kPass - 1) / kPass;
    for (int pass = 0; pass < npass; pass++) {
        const bool last = pass + 1 == npass;
        const int j0 = pass * kPass;
        uint32_t y[kPass][8];
#pragma unroll
        for (int j = 0; j < kPass; j++)
#pragma unroll
            for (int b = 0; b < 8; b++) y[j][b] = 0;
        if (j0 + kPass <= n_out)
            bitslice_pass<true>(y, ring_s, base, ring, lane, n_in, n_out, j0, pass == 0, last, ahead, coef, issue_next);
        else
            bitslice_pass<false>(y, ring_s, base, ring, lane, n_in, n_out, j0, pass == 0, last, ahead, coef, issue_next);
        finish_output(y[0], out(j0), v0, mode, diff);
        if (j0 + 1 < n_out) finish_output(y[1], out(j0 + 1), v0, mode, diff);
        if (j0 + 2 < n_out) finish_output(y[2], out(j0 + 2), v0, mode, diff);
        if (j0 + 3 < n_out) finish_output(y[3], out(j0 + 3), v0, mode, diff);
    }
}

// out[j] (^)= sum_i coef[j][i] * in[i] over the first nchunk KiB of every
// shard (16-byte aligned pointers), n_in <= 32 and n_out <= 16.  Each warp
// owns a ring of n_in + ahead 1 KiB slots of dynamic shared memory.
__global__ void __launch_bounds__(512, 1) gf8_bitslice_kernel(const __grid_constant__ GfMatArgs a, long long nchunk,
                                                               int mode, int ahead) {
    extern __shared__ __align__(16) uint8_t rt_smem[];
    const int lane = threadIdx.x & 31;
    const int n_in = a.n_in, n_out = a.n_out;
    const int ring = n_in + ahead;
    const uint32_t ring_s =
        (uint32_t)__cvta_generic_to_shared(rt_smem) + (uint32_t)((threadIdx.x >> 5) * ring * kChunk);
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    auto issue = [&](long long chunk, int i, uint32_t sa) {
        const uint4 *p = reinterpret_cast<const uint4 *>(a.in[i]) + chunk * (kChunk / 16) + lane;
        cp_async16(sa, p);
        cp_async16(sa + 512, p + 32);
    };
    int base = 0;
    if (c < nchunk)
        for (int i = 0; i < n_in; i++) issue(c, i, ring_s + (uint32_t)(i * kChunk + lane * 16));
    uint32_t diff = 0;
    for (; c < nchunk; c += nwarps) {
        cp_async_wait_all();  // everything in flight belongs to chunk c
        const long long cn = c + nwarps;
        const bool has_next = cn < nchunk;
        int nb = base + n_in;  // the next chunk's slot of input 0
        if (nb >= ring) nb -= ring;
        if (has_next) {  // its first `ahead` inputs go to the free slots now
            int s = nb;
            for (int i = 0; i < ahead; i++) {
                issue(cn, i, ring_s + (uint32_t)(s * kChunk + lane * 16));
                s = s + 1 == ring ? 0 : s + 1;
            }
        }
        bitslice_step(
            ring_s, base, ring, lane, n_in, n_out, ahead, mode, c * (kChunk / 16) + lane,
            [&](int j, int i) -> uint32_t { return a.coef[j][i]; },
            [&](int j) { return reinterpret_cast<uint4 *>(a.out[j]); },
            [&](int i, uint32_t sa) {
                if (has_next) issue(cn, i, sa);
            },
            diff);
        base = nb;
    }
    cp_async_wait_all();
    if (mode == kModeVerify && diff) *reinterpret_cast<volatile int *>(a.flag) = 1;
}

}  // namespace gf8rt
}  // namespace rsgpu

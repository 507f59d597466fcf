// surrogate.cuh — the BF16 surrogate MLP on the 5th-generation tensor cores.
//
// Network (the surrogate configuration): 5 -> 256 -> 256 -> 256 -> 256 -> 4,
// SiLU after each hidden layer, BF16 weights and activations, FP32
// accumulation, FP32 biases. One CTA of 256 threads owns one SM and walks
// 128-row tiles of the input:
//
//   * B operands (weights, N x K) sit in shared memory, K-major, in the
//     no-swizzle core-matrix layout of the UMMA shared-memory descriptor:
//     element (row, k) at byte (row % 8) * 16 + (row / 8) * SBO + (k / 8) * 128
//     + (k % 8) * 2, SBO = (K / 8) * 128.
//   * The FP32 accumulator and the BF16 activations (the A operand of layers
//     2-5) live in tensor memory; layer 1 reads its 16-wide padded input from
//     shared memory: each feature as two BF16 terms (hi, lo) against W1
//     repeated in two column groups, so the inputs keep 16 significant bits
//     (pack_input_row). One thread issues tcgen05.mma (M = 128, N = 128 or 16,
//     K = 16 per instruction) and commits each N-half to its own mbarrier.
//   * The 128 KB weight images of layers 2-4 stream from global memory by a
//     bulk TMA copy (cp.async.bulk, no tensor map, no multicast) into one
//     buffer, each issued as soon as the previous layer's MMAs have drained it,
//     so the copy overlaps the epilogue. Layer 1 (K 2 x 5 padded to 16) and layer 5
//     (N padded 4 -> 16) weights and all biases stay resident.
//   * Epilogue: 8 warps read the accumulator with tcgen05.ld, add the bias,
//     apply SiLU x (1 + tanh(x / 2)) / 2 (one MUFU op), round to BF16 and write
//     the next layer's A operand with tcgen05.st; half 0 of a layer converts
//     while the tensor core still works on half 1.
//
// Every mbarrier wait is bounded by the device clock; on a timeout the block
// agrees (a block-wide vote) to stop, records an error flag, waits (bounded)
// for its copy in flight and frees its TMEM.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "tcgen05.cuh"

namespace sirius {
namespace surrogate {

constexpr int kIn = 5, kInPad = 16, kHid = 256, kOut = 4, kOutPad = 16, kTileM = 128, kThreads = 256;
// packed weight image (bytes): W2 | W3 | W4 | W1 | W5 | b1 b2 b3 b4 (256 f32 each) | b5 (16 f32)
constexpr int kBigBytes = kHid * kHid * 2;            // 131072
constexpr int kW1Bytes = kHid * kInPad * 2;           // 8192
constexpr int kW5Bytes = kOutPad * kHid * 2;          // 8192
constexpr int kBiasBytes = (4 * kHid + kOutPad) * 4;  // 4160
constexpr int kOffW1 = 3 * kBigBytes, kOffW5 = kOffW1 + kW1Bytes, kOffBias = kOffW5 + kW5Bytes;
constexpr int kImageBytes = kOffBias + kBiasBytes;
// host parameter vector (PyTorch nn.Linear order, out x in): W1 b1 W2 b2 W3 b3 W4 b4 W5 b5
constexpr long long kParams = (long long)kHid * kIn + kHid + 3LL * (kHid * kHid + kHid) + kOut * kHid + kOut;

using namespace ::sirius::tc;

#ifdef __CUDACC__
// ---------------------------------------------------------------------------
// The MLP kernel, with its activations in tensor memory.
//
// TMEM (512 columns, one CTA per SM): columns [0, 256) the FP32 accumulator,
// [256, 384) and [384, 512) two BF16 activation buffers (row m in lane m,
// element k in column k / 2, even k in the low half), used in turn as the A
// operand of tcgen05.mma (the form that reads A from tensor memory) and as the
// epilogue's destination. Each layer's MMAs run as two N-halves committed to
// separate mbarriers, so the epilogue of half 0 (TMEM -> bias -> SiLU -> BF16
// -> tcgen05.st) overlaps the tensor core's work on half 1. Layer 1 reads its
// 16-wide (padded) input from shared memory.
// ---------------------------------------------------------------------------
constexpr int kTsSmWbuf = 0, kTsSmW1 = kBigBytes, kTsSmW5 = kTsSmW1 + kW1Bytes, kTsSmX = kTsSmW5 + kW5Bytes,
              kTsSmBias = kTsSmX + kTileM * kInPad * 2, kTsSmBar = kTsSmBias + kBiasBytes,
              kTsSmTmemSlot = kTsSmBar + 32, kTsSmBytes = kTsSmTmemSlot + 16;
static_assert(kTsSmBytes <= 227 * 1024, "the MLP kernel's shared memory fits one SM");
static_assert(kTsSmBar % 8 == 0, "mbarriers are 8-byte aligned");
constexpr uint32_t kTmemAcc = 0, kTmemA0 = 256, kTmemA1 = 384, kTmemCols = 512;

// Epilogue of accumulator half H (columns 128 H ..): bias + SiLU -> BF16 pairs
// into the activation buffer at TMEM column a_next. Warp w: lanes 32 (w % 4)..,
// columns 128 H + 64 (w / 4)...
__device__ __forceinline__ void epilogue_half_ts(uint32_t tmem, int H, const float* bias, uint32_t a_next) {
    const int warp = threadIdx.x >> 5;
    const uint32_t lanes = uint32_t((warp & 3) * 32) << 16;
    // both 32-column loads in flight before one wait
    const int col0 = 128 * H + 64 * (warp >> 2);
    float v[64];
    tmem_ld32_nowait(tmem + kTmemAcc + lanes + uint32_t(col0), v);
    tmem_ld32_nowait(tmem + kTmemAcc + lanes + uint32_t(col0 + 32), v + 32);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        uint32_t r[16];
#pragma unroll
        for (int i = 0; i < 16; ++i)
            r[i] = pack_bf16x2(silu(v[32 * c + 2 * i] + bias[col0 + 32 * c + 2 * i]),
                               silu(v[32 * c + 2 * i + 1] + bias[col0 + 32 * c + 2 * i + 1]));
        tmem_st16(tmem + a_next + lanes + uint32_t((col0 + 32 * c) / 2), r);
    }
}

__global__ void __launch_bounds__(kThreads, 1)
    mlp_kernel_ts(const unsigned char* __restrict__ wimg, const float* __restrict__ feat, long long n,
                  float* __restrict__ out, int* err, unsigned long long* tile_counter,
                  unsigned long long wait_limit_ns, const unsigned* __restrict__ rows) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* Wbuf = sm + kTsSmWbuf;
    unsigned char* W1s = sm + kTsSmW1;
    unsigned char* W5s = sm + kTsSmW5;
    unsigned char* Xs = sm + kTsSmX;
    float* bias = reinterpret_cast<float*>(sm + kTsSmBias);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kTsSmTmemSlot);
    long long* next_s = reinterpret_cast<long long*>(sm + kTsSmTmemSlot + 8);  // the next tile to take
    const uint32_t bar_a = smem_u32(sm + kTsSmBar), bar_b = smem_u32(sm + kTsSmBar + 8),
                   bar_tma = smem_u32(sm + kTsSmBar + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long ntiles = (n + kTileM - 1) / kTileM;

    if (tid == 0) {
        mbar_init(bar_a, 1);
        mbar_init(bar_b, 1);
        mbar_init(bar_tma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // tiles come from a counter, so a CTA that starts late (its SM still busy
    // with another kernel's blocks) takes fewer of them
    if (tid == 32) *next_s = (long long)atomicAdd(tile_counter, 1ull);
    {  // resident operands: W1 | W5 (contiguous in the image and in shared memory) and the biases
        const uint4* src1 = reinterpret_cast<const uint4*>(wimg + kOffW1);
        uint4* dst1 = reinterpret_cast<uint4*>(W1s);
        for (int i = tid; i < (kW1Bytes + kW5Bytes) / 16; i += kThreads) dst1[i] = src1[i];
        const float4* srcb = reinterpret_cast<const float4*>(wimg + kOffBias);
        float4* dstb = reinterpret_cast<float4*>(bias);
        for (int i = tid; i < kBiasBytes / 16; i += kThreads) dstb[i] = srcb[i];
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    uint32_t ph_a = 0, ph_b = 0, ph_tma = 0;
    bool tma_pending = false, ok = true;
    long long tile = *next_s;
    // this thread's input row (tid / 2) of the tile to come, gathered a tile ahead
    // so that the gather's latency (row index, then the row) overlaps the current
    // tile's layers; rows past n read as zeros, which pack to zero operands
    const int in_r = tid >> 1, in_chunk = tid & 1;
    float xin[kIn];
    auto fetch_row = [&](long long t) {
        const long long gr = t * kTileM + in_r;
        const bool live = t < ntiles && gr < n;
        const float* f = feat + (live ? (rows ? (long long)rows[gr] : gr) : 0LL) * kIn;
#pragma unroll
        for (int k = 0; k < kIn; ++k) xin[k] = live ? f[k] : 0.f;
    };
    fetch_row(tile);
    if (tid == 0 && tile < ntiles) bulk_load(smem_u32(Wbuf), wimg, kBigBytes, bar_tma);
    tma_pending = tile < ntiles;
    const uint32_t idesc128 = instr_desc(128), idesc16 = instr_desc(kOutPad);

    while (tile < ntiles) {
        const long long row0 = tile * kTileM;
        __syncthreads();  // every thread has read *next_s
        if (tid == 32) *next_s = (long long)atomicAdd(tile_counter, 1ull);
        {  // input tile: 128 rows x 16 BF16 (features 0..4 as two BF16 terms, zero padding)
            uint4 c0, c1;
            pack_input_row(xin, c0, c1);
            *reinterpret_cast<uint4*>(Xs + packed_offset(in_r, in_chunk * 8, kInPad)) = in_chunk == 0 ? c0 : c1;
        }
        fence_async_smem();
        __syncthreads();
        const long long next = *next_s;
        fetch_row(next);  // in flight during this tile's layers
        // layer 1 (A from shared memory, K = 16): two N-halves
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sbo = (kInPad / 8) * 128;
            mma_bf16(tmem + kTmemAcc, smem_desc(smem_u32(Xs), sbo), smem_desc(smem_u32(W1s), sbo), idesc128, 0u);
            mma_commit(bar_a);
            mma_bf16(tmem + kTmemAcc + 128, smem_desc(smem_u32(Xs), sbo), smem_desc(smem_u32(W1s) + 16 * sbo, sbo),
                     idesc128, 0u);
            mma_commit(bar_b);
        }
        uint32_t a_cur = kTmemA0, a_nxt = kTmemA1;
        // epilogue of layer 1 into a_cur
        ok = mbar_wait(bar_a, ph_a, wait_limit_ns);
        ph_a ^= 1;
        ok = __syncthreads_and(ok);
        if (!ok) break;
        tc_fence_after();
        epilogue_half_ts(tmem, 0, bias, a_cur);
        ok = mbar_wait(bar_b, ph_b, wait_limit_ns);
        ph_b ^= 1;
        ok = __syncthreads_and(ok);
        if (!ok) break;
        tc_fence_after();
        epilogue_half_ts(tmem, 1, bias, a_cur);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        // layers 2..4 (A from tensor memory, K = 256): weights streamed into Wbuf
        for (int L = 0; L < 3 && ok; ++L) {
            ok = mbar_wait(bar_tma, ph_tma, wait_limit_ns);
            ok = __syncthreads_and(ok);
            if (!ok) break;
            ph_tma ^= 1;
            tma_pending = false;
            if (tid == 0) {
                tc_fence_after();
                const uint32_t sbo = (kHid / 8) * 128;
#pragma unroll 1
                for (int hh = 0; hh < 2; ++hh) {
#pragma unroll 1
                    for (int s = 0; s < kHid / 16; ++s)
                        mma_bf16_ts(tmem + kTmemAcc + 128 * hh, tmem + a_cur + 8 * s,
                                    smem_desc(smem_u32(Wbuf) + hh * (kBigBytes / 2) + s * 256, sbo), idesc128,
                                    s > 0);
                    mma_commit(hh == 0 ? bar_a : bar_b);
                }
            }
            const float* b = bias + (L + 1) * kHid;
            ok = mbar_wait(bar_a, ph_a, wait_limit_ns);
            ph_a ^= 1;
            ok = __syncthreads_and(ok);
            if (!ok) break;
            tc_fence_after();
            epilogue_half_ts(tmem, 0, b, a_nxt);
            ok = mbar_wait(bar_b, ph_b, wait_limit_ns);
            ph_b ^= 1;
            ok = __syncthreads_and(ok);
            if (!ok) break;
            // Wbuf is drained: bring the next layer's weights (or layer 2's for the next tile)
            if (L < 2 || next < ntiles) {
                if (tid == 0) bulk_load(smem_u32(Wbuf), wimg + size_t(L < 2 ? L + 1 : 0) * kBigBytes, kBigBytes, bar_tma);
                tma_pending = true;
            }
            tc_fence_after();
            epilogue_half_ts(tmem, 1, b, a_nxt);
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            __syncthreads();
            const uint32_t t = a_cur;
            a_cur = a_nxt;
            a_nxt = t;
        }
        if (!ok) break;
        // layer 5: N = 16 (4 outputs used), A from tensor memory
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sbo = (kHid / 8) * 128;
#pragma unroll 1
            for (int s = 0; s < kHid / 16; ++s)
                mma_bf16_ts(tmem + kTmemAcc, tmem + a_cur + 8 * s, smem_desc(smem_u32(W5s) + s * 256, sbo), idesc16,
                            s > 0);
            mma_commit(bar_a);
        }
        ok = mbar_wait(bar_a, ph_a, wait_limit_ns);
        ph_a ^= 1;
        ok = __syncthreads_and(ok);
        if (!ok) break;
        tc_fence_after();
        if (warp < 4) {
            float v[16];
            tmem_ld16(tmem + kTmemAcc + (uint32_t(warp * 32) << 16), v);
            const long long gr = row0 + warp * 32 + lane;
            if (gr < n) {
                const float* b5 = bias + 4 * kHid;
                *reinterpret_cast<float4*>(out + (rows ? (long long)rows[gr] : gr) * kOut) =
                    make_float4(v[0] + b5[0], v[1] + b5[1], v[2] + b5[2], v[3] + b5[3]);
            }
        }
        tc_fence_before();
        __syncthreads();
        tile = next;
    }
    if (!ok) {
        if (tid == 0) atomicOr(err, 1);
        mbar_wait(bar_a, ph_a, wait_limit_ns);
        mbar_wait(bar_b, ph_b, wait_limit_ns);
    }
    if (tma_pending) {
        const bool landed = mbar_wait(bar_tma, ph_tma, wait_limit_ns);
        if (!landed && tid == 0) atomicOr(err, 2);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}
#endif  // __CUDACC__

// Host: pack the parameter vector (W1 b1 ... W5 b5, nn.Linear order) into the
// kernel's weight image (BF16 core-matrix layouts, FP32 biases).
inline void pack_weights(const float* p, unsigned char* img) {
    auto bf16 = [](float x) -> uint16_t {
        uint32_t u;
        __builtin_memcpy(&u, &x, 4);
        if ((u & 0x7f800000u) == 0x7f800000u) return uint16_t(u >> 16);  // inf / nan
        const uint32_t r = 0x7fffu + ((u >> 16) & 1u);                  // round to nearest even
        return uint16_t((u + r) >> 16);
    };
    for (int i = 0; i < kImageBytes; ++i) img[i] = 0;
    auto put = [&](int off, int rows, int K, int kin, const float* W) {
        for (int r = 0; r < rows; ++r)
            for (int k = 0; k < kin; ++k) {
                const uint16_t h = bf16(W[r * kin + k]);
                __builtin_memcpy(img + off + packed_offset(r, k, K), &h, 2);
            }
    };
    const float* W1 = p;
    const float* b1 = W1 + kHid * kIn;
    const float* W2 = b1 + kHid;
    const float* b2 = W2 + kHid * kHid;
    const float* W3 = b2 + kHid;
    const float* b3 = W3 + kHid * kHid;
    const float* W4 = b3 + kHid;
    const float* b4 = W4 + kHid * kHid;
    const float* W5 = b4 + kHid;
    const float* b5 = W5 + kOut * kHid;
    put(0, kHid, kHid, kHid, W2);
    put(kBigBytes, kHid, kHid, kHid, W3);
    put(2 * kBigBytes, kHid, kHid, kHid, W4);
    put(kOffW1, kHid, kInPad, kIn, W1);
    for (int r = 0; r < kHid; ++r)  // columns kIn..2 kIn - 1 repeat W1 for the inputs' low BF16 terms
        for (int k = 0; k < kIn; ++k) {
            const uint16_t h = bf16(W1[r * kIn + k]);
            __builtin_memcpy(img + kOffW1 + packed_offset(r, kIn + k, kInPad), &h, 2);
        }
    put(kOffW5, kOut, kHid, kHid, W5);
    float* bias = reinterpret_cast<float*>(img + kOffBias);
    for (int i = 0; i < kHid; ++i) {
        bias[i] = b1[i];
        bias[kHid + i] = b2[i];
        bias[2 * kHid + i] = b3[i];
        bias[3 * kHid + i] = b4[i];
    }
    for (int i = 0; i < kOut; ++i) bias[4 * kHid + i] = b5[i];
}

}  // namespace surrogate
}  // namespace sirius

// train.cuh — training of the surrogate MLP on the tensor cores.
//
// One training step on a batch of B rows (B a multiple of 128) is a fixed
// sequence of launches, captured once in a CUDA graph and replayed:
//
//   gather      rows of the device-resident training set, picked by a keyed
//               Feistel permutation of [0, n) per epoch, into a BF16 input
//               tile X0 (B x 16, features 0..4 as two BF16 terms, zero padding) and FP32
//               targets / weights; zeroes the loss sums
//   forward     Z_l = H_{l-1} W_l^T + b_l, H_l = BF16(SiLU(Z_l)) for l = 1..4
//               and Y = H_4 W_5^T + b_5 (tcgen05 GEMMs, epilogue fused)
//   loss        batch sums, then dL/dY (BF16, 16 wide) and the b_5 gradient
//   backward    dW_5^T = H_4^T dY, dH_4 = dY W_5, and for l = 4..1
//               dZ_l = dH_l * SiLU'(Z_l) (fused into the dH GEMM's epilogue,
//               with the bias gradient as column sums), dW_l = dZ_l^T H_{l-1},
//               dH_{l-1} = dZ_l W_l
//   adam        FP32 master weights, first and second moments; writes the
//               BF16 copies the GEMMs read, clears the gradient, and the last
//               block advances the device step counter (which drives the
//               batch position, the epoch's permutation and the learning rate,
//               so the captured graph replays unchanged)
//
// The GEMM: D (M x N, FP32 in tensor memory) = sum_k A(m, k) B(n, k), one CTA
// of 128 threads per 128 x BN tile (BN = 256 or 16), K in chunks of 64 through
// two shared-memory stages. Operands are BF16 in global memory in either
// orientation: a K-major source (A(m, k) at p[m * ld + k]) is copied 16 bytes
// at a time straight into the K-major core-matrix layout; an M-major source
// (A(m, k) at p[k * ld + m], as for dW = dZ^T H) is read as 8 x 8 blocks and
// transposed in registers (byte permutes), so the tensor core always sees the
// K-major layout of tcgen05.cuh. One thread issues tcgen05.mma (M 128, N BN,
// K 16) per 16 columns of the chunk and commits the chunk to its stage's
// mbarrier; each thread fetches its share of the next chunk into registers
// before those MMAs are issued, so the loads overlap them. The weight
// gradients split K (the batch) over CTAs and add their partial tiles with
// FP32 vector atomics. Every mbarrier wait is bounded by the device clock.
//
// Forward arithmetic is the inference kernel's: BF16 operands, FP32 sums and
// biases, SiLU x (1 + tanh(x / 2)) / 2 with the hardware tanh, BF16 hidden
// activations. The gradient is that of this rounded network with respect to
// the FP32 master weights (straight-through the roundings); dL/dY and dZ are
// rounded to BF16 as GEMM operands, the bias gradients are FP32 sums.
#pragma once

#include <cuda.h>  // CUtensorMap (a plain 128-byte descriptor type; nothing from the driver library is linked)
#include <cuda_bf16.h>
#include <cstdint>

#include "surrogate.cuh"
#include "tcgen05.cuh"

namespace sirius {
namespace train {

using namespace ::sirius::tc;
using surrogate::kHid;
using surrogate::kIn;
using surrogate::kInPad;
using surrogate::kOut;
using surrogate::kOutPad;
using surrogate::kParams;

// offsets in the parameter vector (nn.Linear order: W1 b1 W2 b2 W3 b3 W4 b4 W5 b5)
constexpr long long kOffW[5] = {0, kHid * kIn + kHid, kHid * kIn + 2 * kHid + kHid * kHid,
                                kHid * kIn + 3 * kHid + 2LL * kHid * kHid, kHid * kIn + 4 * kHid + 3LL * kHid * kHid};
constexpr long long kOffB[5] = {kOffW[0] + kHid * kIn, kOffW[1] + kHid * kHid, kOffW[2] + kHid * kHid,
                                kOffW[3] + kHid * kHid, kOffW[4] + kOut * kHid};
static_assert(kOffB[4] + kOut == kParams && kOffW[1] == kOffB[0] + kHid && kOffW[4] == kOffB[3] + kHid,
              "parameter layout");
// BF16 weight copies read by the GEMMs (row-major, out x in): W1 256 x 16 (in padded),
// W2..W4 256 x 256, W5 16 x 256 (out padded); element offsets in one buffer
constexpr long long kBfW1 = 0, kBfW2 = kBfW1 + kHid * kInPad, kBfW3 = kBfW2 + kHid * kHid,
                    kBfW4 = kBfW3 + kHid * kHid, kBfW5 = kBfW4 + kHid * kHid, kBfTotal = kBfW5 + kOutPad * kHid;

constexpr int kBM = 128, kBK = 64, kGemmThreads = 128, kStages = 2;

struct Operand {
    const __nv_bfloat16* p;  // A(row, k) at p[row * ld + k] (kmajor) or p[k * ld + row]
    long long ld;
    int kmajor;
    int rows;                // rows present (a multiple of 8 for an M-major source); rows beyond read as zero
};

enum Epi : int { kEpiHidden = 0, kEpiOutput = 1, kEpiDHidden = 2, kEpiDWeight = 3, kEpiDWeightT = 4 };

struct EpiArgs {
    const float* bias;      // Hidden, Output: per-column FP32 bias
    float* z;               // Hidden: pre-activations out; DHidden: pre-activations in (FP32, ld ldz)
    long long ldz;
    __nv_bfloat16* h;       // Hidden: activations out; DHidden: dZ out (BF16, ld ldh)
    long long ldh;
    float* y;               // Output: first ny columns, ld ldy
    long long ldy;
    int ny;
    float* grad;            // DHidden: per-column sums; DWeight: grad[m * ldg + n]; DWeightT: grad[n * ldg + m]
    long long ldg;
    int ng;                 // DWeight / DWeightT: columns n < ng are accumulated
    int fold;               // DWeight with BN 16: > 0 adds column n into column n % fold
};

struct GemmArgs {
    Operand a, b;
    int M, N, K;            // K a multiple of 16
    int k_per_cta;          // K rows per CTA along gridDim.z (a multiple of 64, or K itself)
    EpiArgs e;
    int* err;
    unsigned long long wait_limit_ns;
    // Operands may come by TMA with the 128-byte swizzle (tma_a / tma_b: 0 = staged
    // through registers into the no-swizzle K-major core-matrix layout; 1 = K-major,
    // one box of rows x 64 K per chunk; 2 = MN-major, rows / 64 boxes of 64 MN x 64 K
    // per chunk, read by the tensor core as MN-major without a transpose)
    int tma_a, tma_b;
    CUtensorMap ta, tb;
};

template <int BN>
struct GemmSmem {
    static constexpr int A = kBM * kBK * 2;
    static constexpr int B = BN * kBK * 2;
    static constexpr int Stage = A + B;
    static constexpr int Bar = kStages * Stage;
    static constexpr int Slot = Bar + 8 * (2 * kStages + 1);  // per stage: MMAs done; TMA landed; accumulator
    static constexpr int Bytes = Slot + 16;
    static constexpr uint32_t Cols = BN < 32 ? 32 : BN;
};
static_assert(GemmSmem<256>::Stage % 1024 == 0 && GemmSmem<16>::Stage % 1024 == 0, "stage alignment");
static_assert(GemmSmem<256>::Bar >= (kGemmThreads / 32) * 32 * 33 * 4, "the epilogue's transposition tiles fit the stages");
static_assert(GemmSmem<256>::Bytes <= 113 * 1024, "two 256-wide GEMM CTAs fit one SM (and its 512 TMEM columns)");

#ifdef __CUDACC__
__device__ __forceinline__ uint4 ldg16(const __nv_bfloat16* p) {
    return __ldg(reinterpret_cast<const uint4*>(p));
}

__device__ __forceinline__ uint32_t word_of(const uint4& v, int w) {
    return w == 0 ? v.x : w == 1 ? v.y : w == 2 ? v.z : v.w;
}

// An operand chunk (R rows x kw columns, kw a multiple of 16, at most 64) goes
// into the K-major core-matrix layout of a 64-column stage (SBO 1024 bytes).
// The copy comes in two parts, for software pipelining: fetch_operand loads
// this thread's share of a chunk into registers (N uint4: K-major pieces,
// or N / 8 eight-row blocks of an M-major source), stash_operand writes them
// to shared memory. The next chunk's loads are then in flight while the
// tensor core works on the current one.
template <int N>
__device__ __forceinline__ void fetch_operand(uint4 (&buf)[N], const Operand& op, int row0, int R, int k0, int kw) {
    const uint4 zero = make_uint4(0, 0, 0, 0);
    if (op.kmajor) {
        const int per_row = kw / 8, n = R * per_row;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            const int q = threadIdx.x + kGemmThreads * j;
            buf[j] = zero;
            if (q < n) {
                const int r = q / per_row, kg = q - r * per_row;
                if (row0 + r < op.rows) buf[j] = ldg16(op.p + (long long)(row0 + r) * op.ld + k0 + kg * 8);
            }
        }
    } else {
        const int rg_n = R / 8, n = rg_n * (kw / 8);
#pragma unroll
        for (int j = 0; j < N / 8; ++j) {
            const int u = threadIdx.x + kGemmThreads * j;
            const int kg = u / rg_n, gr = row0 + (u - kg * rg_n) * 8;
            const bool live = u < n && gr < op.rows;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                buf[8 * j + i] = live ? ldg16(op.p + (long long)(k0 + kg * 8 + i) * op.ld + gr) : zero;
        }
    }
}

template <int N>
__device__ __forceinline__ void stash_operand(unsigned char* dst, const uint4 (&buf)[N], const Operand& op, int R,
                                              int kw) {
    if (op.kmajor) {
        const int per_row = kw / 8, n = R * per_row;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            const int q = threadIdx.x + kGemmThreads * j;
            if (q < n) {
                const int r = q / per_row, kg = q - r * per_row;
                *reinterpret_cast<uint4*>(dst + packed_offset(r, kg * 8, kBK)) = buf[j];
            }
        }
    } else {
        const int rg_n = R / 8, n = rg_n * (kw / 8);
#pragma unroll
        for (int j = 0; j < N / 8; ++j) {
            const int u = threadIdx.x + kGemmThreads * j;
            if (u >= n) continue;
            const int kg = u / rg_n, rg = u - kg * rg_n;
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {  // core-matrix row jj: element jj of each of the 8 K rows
                const int w = jj >> 1;
                const uint32_t sel = (jj & 1) ? 0x7632u : 0x5410u;
                uint4 o;
                o.x = __byte_perm(word_of(buf[8 * j + 0], w), word_of(buf[8 * j + 1], w), sel);
                o.y = __byte_perm(word_of(buf[8 * j + 2], w), word_of(buf[8 * j + 3], w), sel);
                o.z = __byte_perm(word_of(buf[8 * j + 4], w), word_of(buf[8 * j + 5], w), sel);
                o.w = __byte_perm(word_of(buf[8 * j + 6], w), word_of(buf[8 * j + 7], w), sel);
                *reinterpret_cast<uint4*>(dst + packed_offset(rg * 8 + jj, kg * 8, kBK)) = o;
            }
        }
    }
}

// SiLU'(z) = s (1 + z (1 - s)), s = (1 + tanh(z / 2)) / 2
__device__ __forceinline__ float dsilu(float z) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
    const float s = 0.5f * (1.f + t);
    return s * (1.f + z * (1.f - s));
}

// Sum of v[c] over the warp's 32 lanes for each c < 32; lane l returns the sum for column l.
__device__ __forceinline__ float transpose_sum32(float v[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int j = 0; j < o; ++j) {
            const float send = upper ? v[j] : v[j + o];
            const float keep = upper ? v[j + o] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
}

// A warp's 32 x 32 block of FP32 values (block row r held by lane r) to global
// memory through the warp's shared tile (32 x 33 floats, conflict-free): each
// store instruction then writes four 128-byte row segments, where a lane per
// row would write 32 scattered 16-byte pieces. Rows at or beyond rows_end are
// left alone.
__device__ __forceinline__ void warp_rows_f32_out(float* t, const float v[32], float* dst, long long ld,
                                                  long long row0, long long rows_end) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 32; ++j) t[lane * 33 + j] = v[j];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = 4 * i + (lane >> 3), c = (lane & 7) * 4;
        if (row0 + r < rows_end) {
            const float* q = t + r * 33 + c;
            *reinterpret_cast<float4*>(dst + (row0 + r) * ld + c) = make_float4(q[0], q[1], q[2], q[3]);
        }
    }
    __syncwarp();
}

// The same for BF16 values (eight 64-byte row segments per store instruction).
__device__ __forceinline__ void warp_rows_bf16_out(float* t, const float v[32], __nv_bfloat16* dst, long long ld,
                                                   long long row0, long long rows_end) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 32; ++j) t[lane * 33 + j] = v[j];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = 8 * i + (lane >> 2), c = (lane & 3) * 8;
        if (row0 + r < rows_end) {
            const float* q = t + r * 33 + c;
            *reinterpret_cast<uint4*>(dst + (row0 + r) * ld + c) =
                make_uint4(pack_bf16x2(q[0], q[1]), pack_bf16x2(q[2], q[3]), pack_bf16x2(q[4], q[5]),
                           pack_bf16x2(q[6], q[7]));
        }
    }
    __syncwarp();
}

// A warp's 32 x 32 FP32 block from global memory (coalesced, as above); lane r
// returns block row r (zeros for rows at or beyond rows_end).
__device__ __forceinline__ void warp_rows_f32_in(float* t, float v[32], const float* src, long long ld,
                                                 long long row0, long long rows_end) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = 4 * i + (lane >> 3), c = (lane & 7) * 4;
        const float4 z = row0 + r < rows_end ? *reinterpret_cast<const float4*>(src + (row0 + r) * ld + c)
                                             : make_float4(0.f, 0.f, 0.f, 0.f);
        float* q = t + r * 33 + c;
        q[0] = z.x;
        q[1] = z.y;
        q[2] = z.z;
        q[3] = z.w;
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = t[lane * 33 + j];
    __syncwarp();
}

// tile: shared memory for the warps' 32 x 33 transposition tiles (the drained stages)
template <int BN, int E>
__device__ __forceinline__ void gemm_epilogue(const GemmArgs& g, uint32_t tmem, int m0, int n0, float* tile) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tl = tmem + (uint32_t(warp * 32) << 16);
    const long long row = (long long)m0 + warp * 32 + lane;
    const bool live = row < g.M;
    if constexpr (BN == 16) {
        float v[16];
        tmem_ld16(tl, v);
        if (!live) return;
        // (unrolled over the 16 columns so that v stays in registers)
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            if constexpr (E == kEpiOutput) {
                if (j < g.e.ny) g.e.y[row * g.e.ldy + j] = v[j] + g.e.bias[j];
            } else if constexpr (E == kEpiDWeight) {
                // fold > 0: columns c and c + fold hold the same weight (W1's two input terms)
                const int c = n0 + j, cf = g.e.fold > 0 ? c % g.e.fold : c;
                if (j < g.e.ng && c < g.N) atomicAdd(g.e.grad + row * g.e.ldg + cf, v[j]);
            } else if constexpr (E == kEpiDWeightT) {
                if (j < g.e.ng && n0 + j < g.N) atomicAdd(g.e.grad + (long long)(n0 + j) * g.e.ldg + row, v[j]);
            }
        }
    } else {
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            float v[32];
            tmem_ld32(tl + uint32_t(c0), v);
            const int n = n0 + c0;
            float* t = tile + warp * (32 * 33);
            const long long row0 = (long long)m0 + warp * 32;
            if constexpr (E == kEpiHidden) {
                // Z = acc + bias (FP32, kept for the backward pass), H = SiLU(Z) (BF16)
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] += g.e.bias[n + i];
                warp_rows_f32_out(t, v, g.e.z + n, g.e.ldz, row0, g.M);
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] = silu(v[i]);
                warp_rows_bf16_out(t, v, g.e.h + n, g.e.ldh, row0, g.M);
            } else if constexpr (E == kEpiDHidden) {
                // dZ = dH SiLU'(Z) (BF16) and the bias gradient (column sums)
                float z[32];
                warp_rows_f32_in(t, z, g.e.z + n, g.e.ldz, row0, g.M);
#pragma unroll
                for (int i = 0; i < 32; ++i) v[i] = live ? v[i] * dsilu(z[i]) : 0.f;
                warp_rows_bf16_out(t, v, g.e.h + n, g.e.ldh, row0, g.M);
                const float s = transpose_sum32(v);
                atomicAdd(g.e.grad + n + lane, s);
            } else if constexpr (E == kEpiDWeight) {
                if (live) {
                    float* gr = g.e.grad + row * g.e.ldg + n;
                    if (n + 32 <= g.e.ng) {
#pragma unroll
                        for (int i = 0; i < 8; ++i)
                            atomicAdd(reinterpret_cast<float4*>(gr) + i,
                                      make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
                    } else {
#pragma unroll
                        for (int i = 0; i < 32; ++i)
                            if (n + i < g.e.ng) atomicAdd(gr + i, v[i]);
                    }
                }
            }
        }
    }
}

// TMA: compiled with the TMA operand path (the launch has an operand in g.ta or
// g.tb); without it the register path alone, as compact as before.
template <int BN, int E, bool TMA>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(const __grid_constant__ GemmArgs g) {
    using S = GemmSmem<BN>;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const int kbeg = blockIdx.z * g.k_per_cta, kend = min(g.K, kbeg + g.k_per_cta);
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + S::Slot);
    const uint32_t bar0 = smem_u32(sm + S::Bar), bar_acc = bar0 + 8 * kStages, bar_full0 = bar0 + 8 * (kStages + 1);
    if (tid == 0) {
        for (int s = 0; s < 2 * kStages + 1; ++s) mbar_init(bar0 + 8 * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                     "r"(S::Cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    const uint32_t idesc = instr_desc(BN);
    const bool ta = TMA && g.tma_a != 0, tb = TMA && g.tma_b != 0;
    const bool ta_mn = ta && g.tma_a == 2, tb_mn = tb && g.tma_b == 2;
    const uint32_t idesc_t = idesc | (ta_mn ? 1u << 15 : 0u) | (tb_mn ? 1u << 16 : 0u);
    const uint32_t tx_bytes = (ta ? uint32_t(S::A) : 0u) + (tb ? uint32_t(S::B) : 0u);
    uint32_t ph = 0, pending = 0;   // per stage: MMA-barrier wait parity, a commit not yet waited for
    uint32_t ph_full = 0, in_flight = 0;  // per stage: TMA-barrier wait parity, a copy not yet waited for (thread 0)
    bool ok = true;
    int chunk = 0;
    constexpr int NA = 8, NB = BN >= 256 ? 16 : 8;  // this thread's share of a chunk (uint4)
    uint4 ra[NA], rb[NB];
    if (kbeg < kend) {
        if (!ta) fetch_operand(ra, g.a, m0, kBM, kbeg, min(kBK, kend - kbeg));
        if (!tb) fetch_operand(rb, g.b, n0, BN, kbeg, min(kBK, kend - kbeg));
    }
    for (int k0 = kbeg; k0 < kend; k0 += kBK, ++chunk) {
        const int s = chunk % kStages;
        const int kw = min(kBK, kend - k0);
        if (pending & (1u << s)) {  // the MMAs of chunk - kStages have released this stage
            ok = mbar_wait(bar0 + 8 * s, (ph >> s) & 1u, g.wait_limit_ns);
            ph ^= 1u << s;
            pending &= ~(1u << s);
            ok = __syncthreads_and(ok);
            if (!ok) break;
        }
        unsigned char* As = sm + s * S::Stage;
        unsigned char* Bs = As + S::A;
        if (tx_bytes && tid == 0) {  // this chunk's TMA operands
            mbar_expect_tx(bar_full0 + 8 * s, tx_bytes);
            if (ta) {
                if (ta_mn)
                    for (int j = 0; j < kBM / 64; ++j) tma_load_2d(smem_u32(As) + j * 8192, &g.ta, m0 + 64 * j, k0, bar_full0 + 8 * s);
                else
                    tma_load_2d(smem_u32(As), &g.ta, k0, m0, bar_full0 + 8 * s);
            }
            if (tb) {
                if (tb_mn)
                    for (int j = 0; j < BN / 64; ++j) tma_load_2d(smem_u32(Bs) + j * 8192, &g.tb, n0 + 64 * j, k0, bar_full0 + 8 * s);
                else
                    tma_load_2d(smem_u32(Bs), &g.tb, k0, n0, bar_full0 + 8 * s);
            }
        }
        if (tx_bytes) in_flight |= 1u << s;
        if (!ta) stash_operand(As, ra, g.a, kBM, kw);
        if (!tb) stash_operand(Bs, rb, g.b, BN, kw);
        if (k0 + kBK < kend) {  // the next chunk's register loads fly while this one multiplies
            if (!ta) fetch_operand(ra, g.a, m0, kBM, k0 + kBK, min(kBK, kend - k0 - kBK));
            if (!tb) fetch_operand(rb, g.b, n0, BN, k0 + kBK, min(kBK, kend - k0 - kBK));
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            if (tx_bytes) {
                ok = mbar_wait(bar_full0 + 8 * s, (ph_full >> s) & 1u, g.wait_limit_ns);
                ph_full ^= 1u << s;
                in_flight &= ~(1u << s);
            }
            if (ok) {
                tc_fence_after();
                for (int t = 0; t < kw / 16; ++t) {
                    const uint64_t ad = ta_mn ? smem_desc_sw128_mn(smem_u32(As) + t * 2048)
                                        : ta  ? smem_desc_sw128(smem_u32(As) + t * 32)
                                              : smem_desc(smem_u32(As) + t * 256, 1024);
                    const uint64_t bd = tb_mn ? smem_desc_sw128_mn(smem_u32(Bs) + t * 2048)
                                        : tb  ? smem_desc_sw128(smem_u32(Bs) + t * 32)
                                              : smem_desc(smem_u32(Bs) + t * 256, 1024);
                    mma_bf16(tmem, ad, bd, idesc_t, (chunk > 0 || t > 0) ? 1u : 0u);
                }
                mma_commit(bar0 + 8 * s);
            }
        }
        if (tx_bytes) {  // thread 0's wait for the copies may have run out
            ok = __syncthreads_and(ok);
            if (!ok) break;
        }
        pending |= 1u << s;
    }
    if (tid == 0) mma_commit(bar_acc);  // completes once every MMA issued above has finished
    bool drained = mbar_wait(bar_acc, 0, g.wait_limit_ns);
    for (int s = 0; s < kStages; ++s)  // and the stage barriers' last arrivals have landed
        if (pending & (1u << s)) drained = mbar_wait(bar0 + 8 * s, (ph >> s) & 1u, g.wait_limit_ns) && drained;
    if (tid == 0)  // no copy may land after the CTA has left
        for (int s = 0; s < kStages; ++s)
            if (in_flight & (1u << s)) drained = mbar_wait(bar_full0 + 8 * s, (ph_full >> s) & 1u, g.wait_limit_ns) && drained;
    ok = __syncthreads_and(ok && drained);
    tc_fence_after();
    if (ok && chunk > 0) {
        gemm_epilogue<BN, E>(g, tmem, m0, n0, reinterpret_cast<float*>(sm));
    } else if (!ok && tid == 0) {
        atomicOr(g.err, 4);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::Cols));
}

// ---------------------------------------------------------------------------
// Batch selection: a keyed Feistel permutation of [0, 4^half), cycle-walked
// into [0, n), so every epoch visits each training row once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t mix32(uint32_t x, uint32_t key) {
    x ^= key;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ uint64_t feistel(uint64_t i, int half_bits, uint32_t key) {
    const uint64_t mask = (1ull << half_bits) - 1;
    uint64_t l = i >> half_bits, r = i & mask;
#pragma unroll
    for (int round = 0; round < 4; ++round) {
        const uint64_t f = mix32(uint32_t(r), key + 0x9E3779B9u * uint32_t(round + 1)) & mask;
        const uint64_t t = l ^ f;
        l = r;
        r = t;
    }
    return (l << half_bits) | r;
}

__device__ __forceinline__ long long permute_row(long long i, long long n, uint32_t key) {
    int half = 1;
    while ((1ll << (2 * half)) < n) ++half;
    uint64_t x = uint64_t(i);
    for (int it = 0; it < 4096; ++it) {  // expected < 4 walks (the domain is below 4n)
        x = feistel(x, half, key);
        if (x < uint64_t(n)) return (long long)x;
    }
    return i % n;
}

struct StepState {
    long long step;          // optimiser steps taken
    unsigned done_blocks;    // Adam kernel's last-block ticket
    int pad;
    float sums[8];           // S_w, S_hw, loss parts (bce, r, g, higher) of the current batch
};

// the batch's rows: training order (permuted per epoch) or rows offset.. in order
__global__ void gather_kernel(const float* __restrict__ feat, const float* __restrict__ targets,
                              const float* __restrict__ weights, long long n_rows, int batch, int steps_per_epoch,
                              unsigned seed, int ordered, long long offset, StepState* st, __nv_bfloat16* x0,
                              float* t, float* w) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < 8) st->sums[threadIdx.x] = 0.f;
    if (b >= batch) return;
    long long idx;
    if (ordered) {
        idx = offset + b;
    } else {
        const long long step = st->step;
        const long long epoch = step / steps_per_epoch, pos = step % steps_per_epoch;
        idx = permute_row(pos * batch + b, n_rows, seed * 0x85EBCA6Bu + uint32_t(epoch) * 0xC2B2AE35u + 1u);
    }
    uint4* xr = reinterpret_cast<uint4*>(x0 + (long long)b * kInPad);
    pack_input_row(feat + idx * kIn, xr[0], xr[1]);  // the inference kernel's two-term inputs
    reinterpret_cast<float4*>(t)[b] = reinterpret_cast<const float4*>(targets)[idx];
    w[b] = weights[idx];
}

__device__ __forceinline__ float block_sum(float v, float* red) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    float s = 0.f;
    if (threadIdx.x == 0)
        for (int i = 0; i < int(blockDim.x >> 5); ++i) s += red[i];
    return s;  // valid in thread 0
}

// S_w = sum w, S_hw = sum hit * w
__global__ void loss_sums_kernel(const float* __restrict__ t, const float* __restrict__ w, int batch, StepState* st) {
    __shared__ float red[32];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float sw = 0.f, shw = 0.f;
    if (b < batch) {
        sw = w[b];
        shw = t[4 * b] * w[b];
    }
    const float a = block_sum(sw, red);
    const float c = block_sum(shw, red);
    if (threadIdx.x == 0) {
        atomicAdd(&st->sums[0], a);
        atomicAdd(&st->sums[1], c);
    }
}

// Loss L = BCE(o0, hit) + 100 (l_r + l_g) + 10 l_h with
//   l_r = sum hit w (o1 - t1)^2 / max(S_hw, 1e-12 B), l_g likewise on o2,
//   l_h = sum w (o3 - t3)^2 / S_w;
// writes dL/dY (BF16, 16 wide), adds the b_5 gradient (grad_b5 may be null)
// and the loss parts.
__global__ void loss_grad_kernel(const float* __restrict__ y, const float* __restrict__ t, const float* __restrict__ w,
                                 int batch, StepState* st, __nv_bfloat16* dy, float* grad_b5) {
    __shared__ float red[32];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const float inv_b = 1.f / float(batch);
    const float shw = fmaxf(st->sums[1], 1e-12f * float(batch)), sw = fmaxf(st->sums[0], 1e-30f);
    float d[4] = {0.f, 0.f, 0.f, 0.f}, part[4] = {0.f, 0.f, 0.f, 0.f};
    if (b < batch) {
        const float4 o = reinterpret_cast<const float4*>(y)[b];
        const float4 tt = reinterpret_cast<const float4*>(t)[b];
        const float wb = w[b], hit = tt.x;
        const float p = 1.f / (1.f + __expf(-o.x));
        part[0] = (fmaxf(o.x, 0.f) - hit * o.x + log1pf(__expf(-fabsf(o.x)))) * inv_b;
        d[0] = (p - hit) * inv_b;
        const float e1 = o.y - tt.y, e2 = o.z - tt.z, e3 = o.w - tt.w;
        part[1] = hit * wb * e1 * e1 / shw;
        part[2] = hit * wb * e2 * e2 / shw;
        part[3] = wb * e3 * e3 / sw;
        d[1] = 200.f * hit * wb * e1 / shw;
        d[2] = 200.f * hit * wb * e2 / shw;
        d[3] = 20.f * wb * e3 / sw;
        uint4* dr = reinterpret_cast<uint4*>(dy + (long long)b * kOutPad);
        dr[0] = make_uint4(pack_bf16x2(d[0], d[1]), pack_bf16x2(d[2], d[3]), 0u, 0u);
        dr[1] = make_uint4(0, 0, 0, 0);
    }
    for (int j = 0; j < 4; ++j) {
        const float s = block_sum(part[j], red);
        if (threadIdx.x == 0) atomicAdd(&st->sums[2 + j], s);
    }
    if (grad_b5)
        for (int j = 0; j < 4; ++j) {
            const float s = block_sum(d[j], red);
            if (threadIdx.x == 0) atomicAdd(grad_b5 + j, s);
        }
}

struct AdamConfig {
    float max_lr, warmup_fraction, beta1, beta2, eps, weight_decay;
    long long total_steps;
};

// learning rate at optimiser step t: linear warm-up from max/25, then a cosine
// to max * 4e-6
__device__ __forceinline__ float learning_rate(const AdamConfig& c, long long t) {
    const double warm = fmax(1.0, double(c.warmup_fraction) * double(c.total_steps));
    const double lo = 0.04 * c.max_lr, fin = 4e-6 * c.max_lr;
    if (double(t) < warm) return float(lo + (c.max_lr - lo) * double(t) / warm);
    const double span = fmax(1.0, double(c.total_steps) - warm);
    const double u = fmin(1.0, (double(t) - warm) / span);
    return float(fin + 0.5 * (c.max_lr - fin) * (1.0 + cos(3.141592653589793 * u)));
}

// parameter index -> element of the BF16 weight copies, or -1 for a bias
__device__ __forceinline__ long long bf16_slot(long long i) {
    constexpr long long w2 = kOffW[1], w3 = kOffW[2], w4 = kOffW[3], w5 = kOffW[4];
    constexpr long long b1 = kOffB[0], b2 = kOffB[1], b3 = kOffB[2], b4 = kOffB[3], b5 = kOffB[4];
    if (i < b1) return kBfW1 + (i / kIn) * kInPad + (i % kIn);
    if (i >= w2 && i < b2) return kBfW2 + (i - w2);
    if (i >= w3 && i < b3) return kBfW3 + (i - w3);
    if (i >= w4 && i < b4) return kBfW4 + (i - w4);
    if (i >= w5 && i < b5) return kBfW5 + (i - w5);
    return -1;
}

__global__ void adam_kernel(float* __restrict__ params, float* __restrict__ grad, float* __restrict__ m1,
                            float* __restrict__ m2, __nv_bfloat16* __restrict__ wbf, StepState* st, AdamConfig c) {
    const long long t = st->step;
    const float lr = learning_rate(c, t);
    const float bc1 = 1.f - powf(c.beta1, float(t + 1)), bc2 = 1.f - powf(c.beta2, float(t + 1));
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < kParams;
         i += (long long)gridDim.x * blockDim.x) {
        const float g = grad[i];
        float p = params[i];
        const float a = c.beta1 * m1[i] + (1.f - c.beta1) * g;
        const float b = c.beta2 * m2[i] + (1.f - c.beta2) * g * g;
        m1[i] = a;
        m2[i] = b;
        p -= lr * (c.weight_decay * p + (a / bc1) / (sqrtf(b / bc2) + c.eps));
        params[i] = p;
        grad[i] = 0.f;
        const long long k = bf16_slot(i);
        if (k >= 0) wbf[k] = __float2bfloat16_rn(p);
        if (i < kHid * kIn) wbf[k + kIn] = __float2bfloat16_rn(p);  // W1 again, for the inputs' low terms
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        if (atomicAdd(&st->done_blocks, 1u) == gridDim.x - 1) {  // every block has read st->step
            st->done_blocks = 0;
            st->step = t + 1;
        }
    }
}

// BF16 copies of the master weights (padding stays zero), after a load
__global__ void weights_to_bf16_kernel(const float* __restrict__ params, __nv_bfloat16* __restrict__ wbf) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < kParams;
         i += (long long)gridDim.x * blockDim.x) {
        const long long k = bf16_slot(i);
        if (k >= 0) wbf[k] = __float2bfloat16_rn(params[i]);
        if (i < kHid * kIn) wbf[k + kIn] = __float2bfloat16_rn(params[i]);
    }
}
#endif  // __CUDACC__

}  // namespace train
}  // namespace sirius

// Learned warm start: a per-cell MLP that predicts the converged conserved
// state of a case from geometry and free-stream parameters, trained on
// converged fields of this solver.
//
// Network: 8 inputs (centroid x, y, z, wall distance, Mach, sin AoA, cos AoA,
// 1) -> 128 -> 128 -> 128 (SiLU) -> 5 outputs (rho, rho u, rho v, rho w,
// rho E), no other bias than the constant input.  GEMMs run on the 5th
// generation tensor cores (tcgen05.mma, bf16 operands in shared memory, f32
// accumulators in TMEM); the master weights and Adam moments stay f32.
//
// Training kernel: a persistent CTA per SM takes tiles of 128 samples (one
// sample per TMEM lane; the four warps of each lane quarter split each
// epilogue's columns).  Per tile it runs the
// forward pass (pre-activations in TMEM, bf16 activations in shared memory),
// the loss gradient, and the backward pass, recomputing each pre-activation
// from the stored input of its layer instead of keeping it.  The weight
// gradients of the two 128x128 layers accumulate in TMEM over all tiles of
// the launch; the two thin layers' weight gradients are read back per tile
// into registers.  Each CTA writes its gradient once per step into its own
// slot, and the Adam kernel sums the slots in a fixed order, so training is
// deterministic.  One training step = train kernel + Adam kernel + step-end
// kernel, replayed from a CUDA graph.
//
// Inputs are scaled with a fixed squashing map u / sqrt(1 + u^2) of the
// offset from the wall's centre in units of the wall's extent; outputs are
// (q - q_freestream) / s with s the root-mean-square of the training targets
// per component.
#include <cuda_bf16.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <random>
#include <vector>

#include "gb_device.cuh"
#include "gb_internal.h"
#include "umma.cuh"

namespace gb {
namespace {

constexpr int kTile = 128;                 // samples per tile = TMEM lanes
// Threads per CTA: four warps per TMEM lane quarter, each taking 32 of an
// epilogue's 128 columns (bit-identical to two warps per quarter and 5 %
// faster in training: more warps hide the TMEM loads and the SiLU chains).
#ifndef GB_MLP_THREADS
#define GB_MLP_THREADS 512
#endif
constexpr int kThreads = GB_MLP_THREADS;    // kGroups warps per TMEM lane quarter
constexpr int kGroups = kThreads / 128;      // column groups of an epilogue
constexpr int kChunks = 4 / kGroups;         // 32-column TMEM chunks per group and epilogue
static_assert(kThreads == 256 || kThreads == 512, "two or four warps per TMEM lane quarter");
constexpr int kFeatures = 8;
constexpr int kOutputs = 5;
constexpr int kIn = 16;                    // padded input width (K of layer 1)
constexpr int kHid = 128;
constexpr int kOutPad = 16;                // padded output width (N of layer 4)

// parameters, master order: W1[128][16], W2[128][128], W3[128][128], W4[16][128]
constexpr int kOffW1 = 0;
constexpr int kOffW2 = kOffW1 + kHid * kIn;
constexpr int kOffW3 = kOffW2 + kHid * kHid;
constexpr int kOffW4 = kOffW3 + kHid * kHid;
constexpr int kParams = kOffW4 + kOutPad * kHid;   // 36864

// bf16 weight image (the shared-memory operand layout), byte offsets
constexpr uint32_t kImgW1 = 0;
constexpr uint32_t kImgW2 = kImgW1 + kHid * kIn * 2;
constexpr uint32_t kImgW3 = kImgW2 + kHid * kHid * 2;
constexpr uint32_t kImgW4 = kImgW3 + kHid * kHid * 2;
constexpr uint32_t kImgBytes = kImgW4 + kOutPad * kHid * 2;   // 73728

// shared memory map
constexpr uint32_t kSmX = kImgBytes;                  // [128][16]  bf16
constexpr uint32_t kSmA1 = kSmX + kTile * kIn * 2;    // [128][128] bf16 (A1, later dZ1)
constexpr uint32_t kSmA2 = kSmA1 + kTile * kHid * 2;  // (A2, later dZ2)
constexpr uint32_t kSmA3 = kSmA2 + kTile * kHid * 2;  // (A3, later dZ3)
constexpr uint32_t kSmDY = kSmA3 + kTile * kHid * 2;  // [128][16]
constexpr uint32_t kSmBytes = kSmDY + kTile * kOutPad * 2;   // 180224

// TMEM columns (512 allocated)
constexpr uint32_t kTmDW2 = 0, kTmDW3 = 128, kTmS1 = 256, kTmS2 = 384;
constexpr uint32_t kTmCols = 512;

constexpr long long kWaitCycles = 4000000000ll;   // ~2 s at 2 GHz

__host__ __device__ inline uint32_t core_off(int r, int c, int cols) {
    return (uint32_t)((r >> 3) * cols * 16 + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

__host__ __device__ inline uint32_t image_offset(int p) {
    if (p < kOffW2) return kImgW1 + core_off(p / kIn, p % kIn, kIn);
    if (p < kOffW3) { const int q = p - kOffW2; return kImgW2 + core_off(q / kHid, q % kHid, kHid); }
    if (p < kOffW4) { const int q = p - kOffW3; return kImgW3 + core_off(q / kHid, q % kHid, kHid); }
    const int q = p - kOffW4;
    return kImgW4 + core_off(q / kHid, q % kHid, kHid);
}

// parameters that multiply a padding column / produce a padding output
__host__ __device__ inline bool padded_param(int p) {
    if (p < kOffW2) return (p % kIn) >= kFeatures;
    if (p >= kOffW4) return (p - kOffW4) / kHid >= kOutputs;
    return false;
}

struct TrainCtl {
    unsigned long long step;
    double b1t, b2t;          // beta1^(step+1), beta2^(step+1)
    int error;                // stage of a wait that gave up (0 none)
    long long wait_cycles;    // bound of each stage's wait for its MMAs
};

// Where a tile's samples come from.
struct Samples {
    // dataset: tile -> (field, 128 consecutive cells)
    const float4* geo;        // [N] (x', y', z', d')
    const float4* par;        // [F] (Mach, sin AoA, cos AoA, 1)
    const float* target;      // [F][N][5] q - q_freestream
    int64_t n_cells;
    int64_t tiles_per_field;
    int64_t n_tiles;
    // explicit samples (x != nullptr): x[n][8], t[n][5] (already scaled)
    const float* x;
    const float* t;
    int64_t n;
    float inv_scale[kOutputs];
};

struct TrainArgs {
    const uint4* img;         // bf16 weight image
    Samples s;
    TrainCtl* ctl;
    float* partials;          // [grid][kParams]
    double* loss_partials;    // [grid]
    int tiles_per_cta;
    int permute;              // permute tiles per epoch (dataset)
    uint64_t seed;
    int64_t total_slots;
    float dy_scale;           // d loss / d y = dy_scale * (y - t)
};

struct ForwardArgs {
    const uint4* img;
    Samples s;                // dataset with one field (par[0]) or explicit x
    TrainCtl* ctl;
    float* y;                 // explicit mode: y[n][5] (scaled outputs)
    // dataset mode: state buffers (device order), both copies
    float* rho0; float* rho1;
    float4* rhou0; float4* rhou1;
    float* rhoe0; float* rhoe1;
    float qinf[kOutputs];
    float scale[kOutputs];
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// 8 values -> bf16 chunk c8 of row r of a buffer with `cols` columns
__device__ __forceinline__ void put8(uint8_t* buf, int cols, int r, int c8, const float* v) {
    uint4 u;
    u.x = pack_bf16(v[0], v[1]);
    u.y = pack_bf16(v[2], v[3]);
    u.z = pack_bf16(v[4], v[5]);
    u.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(buf + (r >> 3) * cols * 16 + c8 * 128 + (r & 7) * 16) = u;
}

__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigm(float z) { return fmaf(0.5f, tanh_fast(0.5f * z), 0.5f); }

// 32-bit integer hash (the "lowbias32" mixer of C. Wellons, public domain)
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Bijection of [0, n): a 4-round Feistel network on the smallest even power
// of two >= n, cycle-walked back into range.
__device__ int64_t permute_index(int64_t i, int64_t n, uint64_t key) {
    int bits = 2;
    while ((1ll << bits) < n) bits += 2;
    const int h = bits / 2;
    const uint32_t mask = (h >= 32) ? 0xFFFFFFFFu : ((1u << h) - 1u);
    uint64_t x = (uint64_t)i;
    for (int walk = 0; walk < 4096; ++walk) {
        uint32_t L = (uint32_t)(x >> h) & mask, R = (uint32_t)x & mask;
        for (int r = 0; r < 4; ++r) {
            const uint32_t f = mix32(R ^ (uint32_t)(key >> (16 * r)) ^ (0x9e3779b9u * (uint32_t)(r + 1))) & mask;
            const uint32_t nl = R;
            R = L ^ f;
            L = nl;
        }
        x = ((uint64_t)L << h) | R;
        if ((int64_t)x < n) return (int64_t)x;
    }
    return i;
}

// D (+)= A * B over K, the operands given as shared-memory buffers (see umma.cuh)
__device__ __forceinline__ void gemm(uint32_t d, uint32_t a, int a_cols, bool a_mn, uint32_t b, int b_cols, bool b_mn,
                                     int M, int N, int K, bool accumulate) {
    const uint32_t id = umma::idesc_bf16(M, N, a_mn, b_mn);
    for (int kk = 0; kk < K / 16; ++kk) {
        const uint64_t da = a_mn ? umma::mnmajor(a + (uint32_t)kk * 32u * a_cols, a_cols)
                                 : umma::kmajor(a + (uint32_t)kk * 256u, a_cols);
        const uint64_t db = b_mn ? umma::mnmajor(b + (uint32_t)kk * 32u * b_cols, b_cols)
                                 : umma::kmajor(b + (uint32_t)kk * 256u, b_cols);
        umma::mma(d, da, db, id, (kk > 0 || accumulate) ? 1u : 0u);
    }
}

// Shared state of one CTA of the MLP kernels.  Thread t works on row (sample
// or hidden unit) `row` = its TMEM lane: warp w reads lane quarter w % 4;
// the kGroups warps of a quarter split the 128 columns of an epilogue
// (`group` g takes columns 128 g / kGroups onwards).
struct Cta {
    uint8_t* sm;              // generic pointer to the dynamic shared memory
    uint32_t sa;              // its shared address
    uint32_t tm;              // TMEM base
    uint32_t lane;            // this warp's TMEM lane offset (bits 16..)
    int row;                  // TMEM lane = tile row of this thread
    int group;                // column group; group 0 also does the per-row work
    uint64_t* bar;
    uint32_t phase;
    long long wait;           // SM cycles a stage waits for its MMAs before giving up
};

// Ends a stage: publishes shared-memory writes to the tensor core, lets thread
// 0 issue the next MMAs (the callable), and waits for them.  Returns false
// (on every thread) if the wait gave up.
template <typename Issue>
__device__ __forceinline__ bool stage(Cta& c, Issue issue) {
    umma::fence_smem_async();
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        umma::fence_after_sync();
        issue();
        umma::commit(c.bar);
    }
    const bool ok = umma::bar_wait(c.bar, c.phase, c.wait);
    c.phase ^= 1u;
    const bool any_fail = __syncthreads_or(!ok);
    umma::fence_after_sync();
    return !any_fail;
}

// S (128 fp32 columns of this thread's row) -> silu -> bf16 row of buf
__device__ __forceinline__ void epi_silu(const Cta& c, uint32_t s_col, uint8_t* buf) {
    const int r = c.row;
#pragma unroll 1
    for (int q = kChunks * c.group; q < kChunks * (c.group + 1); ++q) {
        float z[32];
        umma::ld32(c.tm + c.lane + s_col + 32u * q, z);
#pragma unroll
        for (int k = 0; k < 32; ++k) z[k] = z[k] * sigm(z[k]);
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) put8(buf, kHid, r, 4 * q + cc, z + 8 * cc);
    }
}

// dZ = dA * silu'(Z) with dA in S1, Z in S2 -> bf16 row of buf
__device__ __forceinline__ void epi_dsilu(const Cta& c, uint8_t* buf) {
    const int r = c.row;
#pragma unroll 1
    for (int q = kChunks * c.group; q < kChunks * (c.group + 1); ++q) {
        float da[32], z[32];
        umma::ld32x2(c.tm + c.lane + kTmS1 + 32u * q, c.tm + c.lane + kTmS2 + 32u * q, da, z);
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            const float s = sigm(z[k]);
            da[k] *= s * fmaf(z[k], 1.0f - s, 1.0f);
        }
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) put8(buf, kHid, r, 4 * q + cc, da + 8 * cc);
    }
}

// sample of this thread in tile `tile`: features f[8], targets tg[5]; false = padding row
__device__ __forceinline__ bool load_sample(const Samples& s, int64_t tile, int field_fixed, int r, float* f,
                                            float* tg) {
    if (s.x) {
        const int64_t i = tile * kTile + r;
        if (i >= s.n) return false;
#pragma unroll
        for (int k = 0; k < kFeatures; ++k) f[k] = s.x[i * kFeatures + k];
        if (s.t)
#pragma unroll
            for (int k = 0; k < kOutputs; ++k) tg[k] = s.t[i * kOutputs + k];
        return true;
    }
    int64_t field, cell;
    if (field_fixed >= 0) {
        field = field_fixed;
        cell = tile * kTile + r;
    } else {
        field = tile / s.tiles_per_field;
        cell = (tile % s.tiles_per_field) * kTile + r;
    }
    if (cell >= s.n_cells) return false;
    const float4 g = s.geo[cell];
    const float4 p = s.par[field];
    f[0] = g.x; f[1] = g.y; f[2] = g.z; f[3] = g.w;
    f[4] = p.x; f[5] = p.y; f[6] = p.z; f[7] = p.w;
    if (s.target) {
        const float* t = s.target + (field * s.n_cells + cell) * kOutputs;
#pragma unroll
        for (int k = 0; k < kOutputs; ++k) tg[k] = t[k] * s.inv_scale[k];
    }
    return true;
}

__device__ __forceinline__ void put_x(uint8_t* sm, int r, bool valid, const float* f) {
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = valid ? f[k] : 0.0f;
    put8(sm + kSmX, kIn, r, 0, v);
    const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    put8(sm + kSmX, kIn, r, 1, zero);
}

__device__ __forceinline__ void cta_setup(Cta& c, uint8_t* sm, const uint4* img, uint64_t* bar, uint32_t* slot,
                                          const TrainCtl* ctl) {
    c.sm = sm;
    c.sa = umma::smem_addr(sm);
    c.bar = bar;
    c.phase = 0;
    c.wait = ctl->wait_cycles > 0 ? ctl->wait_cycles : kWaitCycles;
    for (int k = threadIdx.x; k < (int)(kImgBytes / 16); k += blockDim.x) reinterpret_cast<uint4*>(sm)[k] = img[k];
    if (threadIdx.x == 0) umma::bar_init(bar, 1);
    if (threadIdx.x < 32) umma::tmem_alloc(slot, kTmCols);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    c.tm = *slot;
    c.lane = (uint32_t)(((threadIdx.x >> 5) & 3) * 32) << 16;
    c.row = (int)(((threadIdx.x >> 5) & 3) * 32 + (threadIdx.x & 31));
    c.group = (int)(threadIdx.x >> 7);
}

__device__ __forceinline__ void cta_teardown(Cta& c, TrainCtl* ctl, bool ok, int where) {
    if (!ok) {
        if (threadIdx.x == 0) atomicCAS(&ctl->error, 0, where);
        // let any MMA still in flight finish (bounded by the full default,
        // whatever the stage bound was) before giving TMEM back
        if (threadIdx.x == 0) {
            umma::commit(c.bar);
            umma::bar_wait(c.bar, c.phase, kWaitCycles);
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::fence_after_sync();
        umma::tmem_free(c.tm, kTmCols);
    }
}

// forward through layers 1-3 (A1..A3 in shared memory) and layer 4 into S2
__device__ __forceinline__ bool forward(Cta& c) {
    const uint32_t X = c.sa + kSmX, A1 = c.sa + kSmA1, A2 = c.sa + kSmA2, A3 = c.sa + kSmA3;
    const uint32_t W1 = c.sa + kImgW1, W2 = c.sa + kImgW2, W3 = c.sa + kImgW3, W4 = c.sa + kImgW4;
    const uint32_t S1 = c.tm + kTmS1, S2 = c.tm + kTmS2;
    if (!stage(c, [&] { gemm(S1, X, kIn, false, W1, kIn, false, 128, kHid, kIn, false); })) return false;
    epi_silu(c, kTmS1, c.sm + kSmA1);
    if (!stage(c, [&] { gemm(S1, A1, kHid, false, W2, kHid, false, 128, kHid, kHid, false); })) return false;
    epi_silu(c, kTmS1, c.sm + kSmA2);
    if (!stage(c, [&] { gemm(S1, A2, kHid, false, W3, kHid, false, 128, kHid, kHid, false); })) return false;
    epi_silu(c, kTmS1, c.sm + kSmA3);
    return stage(c, [&] { gemm(S2, A3, kHid, false, W4, kHid, false, 128, kOutPad, kHid, false); });
}

__global__ void __launch_bounds__(kThreads, 1) k_mlp_train(const TrainArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    Cta c;
    cta_setup(c, sm, a.img, &bar, &slot, a.ctl);
    const int r = c.row;
    const bool rowwork = c.group == 0;   // the per-row work (sample, loss, thin layers) is done by group 0
    const uint32_t X = c.sa + kSmX, A1 = c.sa + kSmA1, A2 = c.sa + kSmA2, A3 = c.sa + kSmA3, DY = c.sa + kSmDY;
    const uint32_t W1 = c.sa + kImgW1, W2 = c.sa + kImgW2, W3 = c.sa + kImgW3, W4 = c.sa + kImgW4;
    const uint32_t S1 = c.tm + kTmS1, S2 = c.tm + kTmS2, DW2 = c.tm + kTmDW2, DW3 = c.tm + kTmDW3;
    float acc1[16], acc4[16];      // this thread's hidden unit: dW1[r][:], dW4[:][r]
#pragma unroll
    for (int k = 0; k < 16; ++k) acc1[k] = acc4[k] = 0.0f;
    double loss = 0.0;
    bool first = true, ok = true;
    int where = 0;
    const unsigned long long step = a.ctl->step;
    for (int j = 0; j < a.tiles_per_cta && ok; ++j) {
        const int64_t slot_id = (int64_t)step * gridDim.x * a.tiles_per_cta + (int64_t)blockIdx.x * a.tiles_per_cta + j;
        if (slot_id >= a.total_slots) break;
        int64_t tile = slot_id;
        if (a.permute) {
            const int64_t epoch = slot_id / a.s.n_tiles;
            tile = permute_index(slot_id % a.s.n_tiles, a.s.n_tiles, a.seed ^ (0x9E3779B97F4A7C15ull * (epoch + 1)));
        }
        float f[8], tg[5] = {0, 0, 0, 0, 0};
        bool valid = false;
        if (rowwork) {
            valid = load_sample(a.s, tile, -1, r, f, tg);
            put_x(c.sm, r, valid, f);
        }
        where = 1;
        if (!(ok = forward(c))) break;
        // loss gradient: dY = dy_scale * (y - t) on valid rows
        if (rowwork) {
            float y[16];
            umma::ld16(S2 + c.lane, y);
            float dy[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) dy[k] = 0.0f;
            if (valid) {
#pragma unroll
                for (int k = 0; k < kOutputs; ++k) {
                    const float e = y[k] - tg[k];
                    loss += (double)e * e;
                    dy[k] = a.dy_scale * e;
                }
            }
            put8(c.sm + kSmDY, kOutPad, r, 0, dy);
            put8(c.sm + kSmDY, kOutPad, r, 1, dy + 8);
        }
        where = 2;
        // dW4^T (this tile) = A3^T dY -> S2
        if (!(ok = stage(c, [&] { gemm(S2, A3, kHid, true, DY, kOutPad, true, 128, kOutPad, kTile, false); }))) break;
        if (rowwork) {
            float v[16];
            umma::ld16(S2 + c.lane, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) acc4[k] += v[k];
        }
        where = 3;
        // dA3 = dY W4 -> S1; Z3 = A2 W3^T -> S2
        if (!(ok = stage(c, [&] {
                  gemm(S1, DY, kOutPad, false, W4, kHid, true, 128, kHid, kOutPad, false);
                  gemm(S2, A2, kHid, false, W3, kHid, false, 128, kHid, kHid, false);
              })))
            break;
        epi_dsilu(c, c.sm + kSmA3);            // dZ3 over A3
        where = 4;
        // dA2 = dZ3 W3 -> S1; dW3 += dZ3^T A2; Z2 = A1 W2^T -> S2
        if (!(ok = stage(c, [&] {
                  gemm(S1, A3, kHid, false, W3, kHid, true, 128, kHid, kHid, false);
                  gemm(DW3, A3, kHid, true, A2, kHid, true, 128, kHid, kTile, !first);
                  gemm(S2, A1, kHid, false, W2, kHid, false, 128, kHid, kHid, false);
              })))
            break;
        epi_dsilu(c, c.sm + kSmA2);            // dZ2 over A2
        where = 5;
        // dA1 = dZ2 W2 -> S1; dW2 += dZ2^T A1; Z1 = X W1^T -> S2
        if (!(ok = stage(c, [&] {
                  gemm(S1, A2, kHid, false, W2, kHid, true, 128, kHid, kHid, false);
                  gemm(DW2, A2, kHid, true, A1, kHid, true, 128, kHid, kTile, !first);
                  gemm(S2, X, kIn, false, W1, kIn, false, 128, kHid, kIn, false);
              })))
            break;
        first = false;
        epi_dsilu(c, c.sm + kSmA1);            // dZ1 over A1
        where = 6;
        // dW1 (this tile) = dZ1^T X -> S1
        if (!(ok = stage(c, [&] { gemm(S1, A1, kHid, true, X, kIn, true, 128, kIn, kTile, false); }))) break;
        if (rowwork) {
            float v[16];
            umma::ld16(S1 + c.lane, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) acc1[k] += v[k];
        }
    }
    if (ok) {
        float* P = a.partials + (size_t)blockIdx.x * kParams;
        // the first half of the groups drains dW2, the second dW3 (row r =
        // output unit), each group its share of the 32-column chunks
        const bool second = c.group >= kGroups / 2;
        const uint32_t DW = second ? DW3 : DW2;
        float* Pw = P + (second ? kOffW3 : kOffW2) + r * kHid;
        const int q0 = (c.group % (kGroups / 2)) * (8 / kGroups);
#pragma unroll 1
        for (int q = q0; q < q0 + 8 / kGroups; ++q) {
            float v2[32];
            if (first) {
#pragma unroll
                for (int k = 0; k < 32; ++k) v2[k] = 0.0f;
            } else {
                umma::ld32(DW + c.lane + 32u * q, v2);
            }
            float4* p2 = reinterpret_cast<float4*>(Pw + 32 * q);
#pragma unroll
            for (int k = 0; k < 8; ++k) p2[k] = make_float4(v2[4 * k], v2[4 * k + 1], v2[4 * k + 2], v2[4 * k + 3]);
        }
        if (rowwork) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                P[kOffW1 + r * kIn + k] = acc1[k];
                P[kOffW4 + k * kHid + r] = acc4[k];
            }
        }
        // loss partial (fixed order)
        __shared__ double red[kThreads];
        red[threadIdx.x] = loss;
        __syncthreads();
        if (r == 0) {
            double s = 0.0;
            for (int k = 0; k < kThreads; ++k) s += red[k];
            a.loss_partials[blockIdx.x] = s;
        }
    }
    cta_teardown(c, a.ctl, ok, where);
}

// Adam over the summed gradient partials; writes f32 master weights and the
// bf16 image.  Bias-corrected with beta^(step+1) from the control block.
__global__ void k_mlp_adam(const float* __restrict__ partials, int n_parts, float* w, float* m, float* v,
                           uint16_t* img, const TrainCtl* ctl, float lr, float b1, float b2, float eps) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    if (padded_param(p)) return;
    float g = 0.0f;
    for (int k = 0; k < n_parts; ++k) g += partials[(size_t)k * kParams + p];
    const float mm = b1 * m[p] + (1.0f - b1) * g;
    const float vv = b2 * v[p] + (1.0f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float mh = mm / (float)(1.0 - ctl->b1t);
    const float vh = vv / (float)(1.0 - ctl->b2t);
    const float nw = w[p] - lr * mh / (sqrtf(vh) + eps);
    w[p] = nw;
    __nv_bfloat16 h = __float2bfloat16_rn(nw);
    img[image_offset(p) / 2] = *reinterpret_cast<uint16_t*>(&h);
}

__global__ void k_mlp_step_end(TrainCtl* ctl, const double* loss_partials, int n_parts, double* history,
                               int64_t history_len, double loss_norm, float b1, float b2) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int k = 0; k < n_parts; ++k) s += loss_partials[k];
    const unsigned long long st = ctl->step;
    if (history && (int64_t)st < history_len) history[st] = s * loss_norm;
    ctl->step = st + 1;
    ctl->b1t *= b1;
    ctl->b2t *= b2;
}

// f32 master weights -> bf16 image
__global__ void k_mlp_pack(const float* __restrict__ w, uint16_t* img) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    __nv_bfloat16 h = __float2bfloat16_rn(padded_param(p) ? 0.0f : w[p]);
    img[image_offset(p) / 2] = *reinterpret_cast<uint16_t*>(&h);
}

__global__ void k_grad_sum(const float* __restrict__ partials, int n_parts, float* g) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float s = 0.0f;
    for (int k = 0; k < n_parts; ++k) s += partials[(size_t)k * kParams + p];
    g[p] = s;
}

// forward pass: scaled outputs (explicit samples) or the predicted state
__global__ void __launch_bounds__(kThreads, 1) k_mlp_forward(const ForwardArgs a, int64_t n_tiles) {
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    Cta c;
    cta_setup(c, sm, a.img, &bar, &slot, a.ctl);
    bool ok = true;
    for (int64_t tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        float f[8], tg[5];
        bool valid = false;
        if (c.group == 0) {
            valid = load_sample(a.s, tile, 0, c.row, f, tg);
            put_x(c.sm, c.row, valid, f);
        }
        if (!(ok = forward(c))) break;
        if (c.group != 0) continue;
        float y[16];
        umma::ld16(c.tm + kTmS2 + c.lane, y);
        if (!valid) continue;
        const int64_t i = tile * kTile + c.row;
        if (a.y) {
#pragma unroll
            for (int k = 0; k < kOutputs; ++k) a.y[i * kOutputs + k] = y[k];
        } else {
            float q[kOutputs];
#pragma unroll
            for (int k = 0; k < kOutputs; ++k) q[k] = fmaf(a.scale[k], y[k], a.qinf[k]);
            const float4 ru = make_float4(q[1], q[2], q[3], 0.0f);
            a.rho0[i] = q[0]; a.rho1[i] = q[0];
            a.rhou0[i] = ru; a.rhou1[i] = ru;
            a.rhoe0[i] = q[4]; a.rhoe1[i] = q[4];
        }
    }
    cta_teardown(c, a.ctl, ok, 9);
}

// ---- features ----
// closest point of a triangle to p: the region test of Ericson, Real-Time
// Collision Detection (2005), sec. 5.1.5; returns the squared distance
__device__ float tri_dist2(float3 p, float3 a, float3 b, float3 c) {
    auto sub = [](float3 u, float3 v) { return make_float3(u.x - v.x, u.y - v.y, u.z - v.z); };
    auto dot3 = [](float3 u, float3 v) { return u.x * v.x + u.y * v.y + u.z * v.z; };
    auto at = [](float3 o, float3 u, float s, float3 v, float t) {
        return make_float3(o.x + s * u.x + t * v.x, o.y + s * u.y + t * v.y, o.z + s * u.z + t * v.z);
    };
    const float3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    float3 q;
    const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    const float3 bp = sub(p, b);
    const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    const float3 cp = sub(p, c);
    const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
    if (d1 <= 0.f && d2 <= 0.f) q = a;
    else if (d3 >= 0.f && d4 <= d3) q = b;
    else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) q = at(a, ab, d1 / (d1 - d3), ac, 0.f);
    else if (d6 >= 0.f && d5 <= d6) q = c;
    else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) q = at(a, ab, 0.f, ac, d2 / (d2 - d6));
    else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        q = make_float3(b.x + w * (c.x - b.x), b.y + w * (c.y - b.y), b.z + w * (c.z - b.z));
    } else {
        const float den = 1.f / (va + vb + vc);
        q = at(a, ab, vb * den, ac, vc * den);
    }
    const float3 e = sub(p, q);
    return dot3(e, e);
}

__device__ __forceinline__ float squash(float u) { return u * rsqrtf(1.0f + u * u); }

// geo[i] = (squash((x - c) / L), ..., squash(d / L)) with d the distance to
// the nearest wall triangle
__global__ void k_geo_features(const float4* __restrict__ cell_geo, int64_t N, const float4* __restrict__ tris,
                               int n_tris, float3 centre, float inv_len, float4* geo) {
    __shared__ float4 st[3 * 128];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const float4 cg = i < N ? cell_geo[i] : make_float4(0, 0, 0, 0);
    const float3 p = make_float3(cg.x, cg.y, cg.z);
    float best = 3.0e38f;
    for (int t0 = 0; t0 < n_tris; t0 += 128) {
        const int nt = min(128, n_tris - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < 3 * nt; k += blockDim.x) st[k] = tris[3 * t0 + k];
        __syncthreads();
        for (int t = 0; t < nt; ++t) {
            const float4 a = st[3 * t], b = st[3 * t + 1], cc = st[3 * t + 2];
            best = fminf(best, tri_dist2(p, make_float3(a.x, a.y, a.z), make_float3(b.x, b.y, b.z),
                                         make_float3(cc.x, cc.y, cc.z)));
        }
    }
    if (i >= N) return;
    const float d = n_tris ? sqrtf(best) : 0.0f;
    geo[i] = make_float4(squash((p.x - centre.x) * inv_len), squash((p.y - centre.y) * inv_len),
                         squash((p.z - centre.z) * inv_len), squash(d * inv_len));
}

// training target of one field: q - q_freestream, interior cells
__global__ void k_add_field(int64_t N, const float* __restrict__ rho, const float4* __restrict__ rhou,
                            const float* __restrict__ rhoe, float q0, float q1, float q2, float q3, float q4,
                            float* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 ru = rhou[i];
    float* o = out + i * kOutputs;
    o[0] = rho[i] - q0;
    o[1] = ru.x - q1;
    o[2] = ru.y - q2;
    o[3] = ru.z - q3;
    o[4] = rhoe[i] - q4;
}

// per-block sums of squares of the targets (5 doubles per block)
__global__ void k_target_moments(const float* __restrict__ t, int64_t n, double* partials) {
    __shared__ double red[5][256];
    double s[5] = {0, 0, 0, 0, 0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < 5; ++k) {
            const double v = t[i * 5 + k];
            s[k] += v * v;
        }
    for (int k = 0; k < 5; ++k) red[k][threadIdx.x] = s[k];
    __syncthreads();
    if (threadIdx.x < 5) {
        double a = 0.0;
        for (int k = 0; k < (int)blockDim.x; ++k) a += red[threadIdx.x][k];
        partials[blockIdx.x * 5 + threadIdx.x] = a;
    }
}

}  // namespace
}  // namespace gb

struct gbWarmStartImpl {
    cuMesh* mesh = nullptr;
    gb::MeshAccess acc{};
    int64_t N = 0;
    float4* d_geo = nullptr;
    float centre[3] = {0, 0, 0};
    float length = 1.0f;
    std::vector<float4> par;           // per training field
    float* d_target = nullptr;         // [cap][N][5]
    int cap_fields = 0;
    float scale[5] = {1, 1, 1, 1, 1};
    bool scale_set = false;
    float* d_w = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    uint16_t* d_img = nullptr;
    gb::TrainCtl* d_ctl = nullptr;
    long long wait_cycles = 0;         // 0: the kernels' default bound
    float4* d_par = nullptr;
    int n_par_alloc = 0;
    uint64_t seed = 0;
};

namespace gb {
namespace {

using WS = ::gbWarmStartImpl;

bool ok_(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

int n_sms() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

bool set_smem_attrs() {
    static bool done = false;
    if (done) return true;
    if (!ok_(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmBytes),
             "warm start kernel attributes") ||
        !ok_(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmBytes),
             "warm start kernel attributes"))
        return false;
    done = true;
    return true;
}

void freestream(gb_vector mach, float p, float T, float* q, float4* par) {
    // euler_init, src/models/euler.cu:401-404
    const float r = p / T;
    const float c = sqrtf(1.4f * p / r);
    const float u = mach.x * c, v = mach.y * c, w = mach.z * c;
    q[0] = r;
    q[1] = r * u;
    q[2] = r * v;
    q[3] = r * w;
    q[4] = p / 0.4f + 0.5f * r * (u * u + v * v + w * w);
    const float M = sqrtf(mach.x * mach.x + mach.y * mach.y + mach.z * mach.z);
    // angle of attack in the x-z plane
    const float sa = M > 0.f ? mach.z / M : 0.f, ca = M > 0.f ? mach.x / M : 1.f;
    if (par) *par = make_float4(M, sa, ca, 1.0f);
}

bool check_ctl(WS* w, const char* what) {
    TrainCtl h{};
    if (!ok_(cudaMemcpy(&h, w->d_ctl, sizeof(h), cudaMemcpyDeviceToHost), what)) return false;
    if (h.error) {
        set_error(std::string(what) + ": a tensor-core wait gave up (stage " + std::to_string(h.error) + ")");
        return false;
    }
    return true;
}

bool reset_ctl(WS* w, cudaStream_t s) {
    const TrainCtl h{0ull, 0.9, 0.999, 0, w->wait_cycles};
    return ok_(cudaMemcpyAsync(w->d_ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s), "warm start control");
}

bool upload_weights(WS* w, const float* host) {
    cudaStream_t s = (cudaStream_t)gbGetStream();
    if (!ok_(cudaMemcpyAsync(w->d_w, host, kParams * sizeof(float), cudaMemcpyHostToDevice, s), "warm start weights") ||
        !ok_(cudaMemsetAsync(w->d_m, 0, kParams * sizeof(float), s), "warm start weights") ||
        !ok_(cudaMemsetAsync(w->d_v, 0, kParams * sizeof(float), s), "warm start weights"))
        return false;
    k_mlp_pack<<<(kParams + 255) / 256, 256, 0, s>>>(w->d_w, w->d_img);
    count_launch();
    return ok_(cudaStreamSynchronize(s), "warm start weights");
}

// explicit samples on the device (scaled inputs and targets)
struct DevSamples {
    float* x = nullptr;
    float* t = nullptr;
    ~DevSamples() {
        if (x) cudaFree(x);
        if (t) cudaFree(t);
    }
};

Samples explicit_samples(const DevSamples& d, int64_t n) {
    Samples s{};
    s.x = d.x;
    s.t = d.t;
    s.n = n;
    for (int k = 0; k < kOutputs; ++k) s.inv_scale[k] = 1.0f;
    return s;
}

bool forward_launch(WS* w, const ForwardArgs& fa, int64_t n_tiles, cudaStream_t s) {
    if (n_tiles <= 0) return true;
    if (!set_smem_attrs()) return false;
    const int grid = (int)std::min<int64_t>(n_tiles, n_sms());
    k_mlp_forward<<<grid, kThreads, kSmBytes, s>>>(fa, n_tiles);
    count_launch();
    return ok_(cudaGetLastError(), "warm start forward");
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int64_t gbWarmStartParamCount(void) { return kParams; }

gbWarmStart* gbWarmStartCreate(cuMesh* mesh, unsigned wall_region, uint64_t seed) {
    clear_error();
    WS* w = new WS();
    w->seed = seed;
    bool ok = ok_(cudaMalloc((void**)&w->d_w, kParams * sizeof(float)), "gbWarmStartCreate") &&
              ok_(cudaMalloc((void**)&w->d_m, kParams * sizeof(float)), "gbWarmStartCreate") &&
              ok_(cudaMalloc((void**)&w->d_v, kParams * sizeof(float)), "gbWarmStartCreate") &&
              ok_(cudaMalloc((void**)&w->d_img, kImgBytes), "gbWarmStartCreate") &&
              ok_(cudaMemset(w->d_img, 0, kImgBytes), "gbWarmStartCreate") &&
              ok_(cudaMalloc((void**)&w->d_ctl, sizeof(TrainCtl)), "gbWarmStartCreate") &&
              ok_(cudaMemset(w->d_ctl, 0, sizeof(TrainCtl)), "gbWarmStartCreate");
    // PyTorch-style uniform init, bound 1/sqrt(fan in); the output layer
    // starts small so that the first prediction is close to free stream
    if (ok) {
        std::mt19937_64 rng(seed);
        std::vector<float> h(kParams, 0.0f);
        auto fill = [&](int off, int rows, int cols, int used_rows, int used_cols, float bound) {
            std::uniform_real_distribution<float> U(-bound, bound);
            for (int i = 0; i < rows; ++i)
                for (int j = 0; j < cols; ++j) h[off + i * cols + j] = (i < used_rows && j < used_cols) ? U(rng) : 0.0f;
        };
        fill(kOffW1, kHid, kIn, kHid, kFeatures, 1.0f / sqrtf((float)kFeatures));
        fill(kOffW2, kHid, kHid, kHid, kHid, 1.0f / sqrtf((float)kHid));
        fill(kOffW3, kHid, kHid, kHid, kHid, 1.0f / sqrtf((float)kHid));
        fill(kOffW4, kOutPad, kHid, kOutputs, kHid, 0.1f / sqrtf((float)kHid));
        ok = upload_weights(w, h.data());
    }
    if (ok && mesh) {
        w->mesh = mesh;
        ok = mesh_access(mesh, &w->acc);
        if (ok && (int)wall_region >= w->acc.n_regions) {
            set_error("gbWarmStartCreate: unknown wall region");
            ok = false;
        }
        if (ok) {
            const Topology& T = *w->acc.topo;
            const Numbering& U = *w->acc.num;
            w->N = w->acc.N;
            // wall triangles (fan of each wall face) and their extent
            std::vector<float4> tris;
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, cen[3] = {0, 0, 0};
            int64_t nf = 0;
            for (uint32_t g = U.region_start[wall_region]; g < U.region_start[wall_region + 1]; ++g) {
                const uint32_t f = U.face_old[U.ghost_face[g - w->N]];
                const uint32_t b = T.fns[f], e = T.fns[f + 1];
                auto node = [&](uint32_t k) {
                    const double* x = &T.nodes[3 * (size_t)T.fn[k]];
                    return make_float4((float)x[0], (float)x[1], (float)x[2], 0.f);
                };
                for (uint32_t k = b; k < e; ++k)
                    for (int d = 0; d < 3; ++d) {
                        const double x = T.nodes[3 * (size_t)T.fn[k] + d];
                        lo[d] = std::min(lo[d], x);
                        hi[d] = std::max(hi[d], x);
                        cen[d] += x / (double)(e - b);
                    }
                ++nf;
                for (uint32_t k = b + 1; k + 1 < e; ++k) {
                    tris.push_back(node(b));
                    tris.push_back(node(k));
                    tris.push_back(node(k + 1));
                }
            }
            double len = 0.0;
            for (int d = 0; d < 3; ++d) {
                w->centre[d] = nf ? (float)(cen[d] / nf) : 0.f;
                if (nf) len = std::max(len, hi[d] - lo[d]);
            }
            w->length = len > 0.0 ? (float)len : 1.0f;
            float4* d_tris = nullptr;
            ok = ok_(cudaMalloc((void**)&d_tris, std::max<size_t>(tris.size(), 1) * sizeof(float4)), "gbWarmStartCreate") &&
                 ok_(cudaMemcpy(d_tris, tris.data(), tris.size() * sizeof(float4), cudaMemcpyHostToDevice),
                     "gbWarmStartCreate") &&
                 ok_(cudaMalloc((void**)&w->d_geo, std::max<int64_t>(w->N, 1) * sizeof(float4)), "gbWarmStartCreate");
            if (ok && w->N) {
                k_geo_features<<<(unsigned)((w->N + 255) / 256), 256>>>(
                    w->acc.dev->cell_geo, w->N, d_tris, (int)(tris.size() / 3),
                    make_float3(w->centre[0], w->centre[1], w->centre[2]), 1.0f / w->length, w->d_geo);
                count_launch();
                ok = ok_(cudaDeviceSynchronize(), "gbWarmStartCreate");
            }
            if (d_tris) cudaFree(d_tris);
        }
    }
    if (!ok) {
        gbWarmStartFree(w);
        return nullptr;
    }
    return w;
}

void gbWarmStartFree(gbWarmStart* w) {
    if (!w) return;
    for (void* p : {(void*)w->d_geo, (void*)w->d_target, (void*)w->d_w, (void*)w->d_m, (void*)w->d_v,
                    (void*)w->d_img, (void*)w->d_ctl, (void*)w->d_par})
        if (p) cudaFree(p);
    delete w;
}

int gbWarmStartGetWeights(gbWarmStart* w, float* out) {
    clear_error();
    if (!w || !out) { set_error("gbWarmStartGetWeights: bad arguments"); return 1; }
    cudaStream_t s = (cudaStream_t)gbGetStream();
    return ok_(cudaMemcpyAsync(out, w->d_w, kParams * sizeof(float), cudaMemcpyDeviceToHost, s), "gbWarmStartGetWeights") &&
                   ok_(cudaStreamSynchronize(s), "gbWarmStartGetWeights")
               ? 0
               : 1;
}

int gbWarmStartSetWeights(gbWarmStart* w, const float* in) {
    clear_error();
    if (!w || !in) { set_error("gbWarmStartSetWeights: bad arguments"); return 1; }
    return upload_weights(w, in) ? 0 : 1;
}

int gbWarmStartGetScales(gbWarmStart* w, float* geometry, float* target) {
    clear_error();
    if (!w) { set_error("gbWarmStartGetScales: bad arguments"); return 1; }
    if (geometry) {
        geometry[0] = w->centre[0];
        geometry[1] = w->centre[1];
        geometry[2] = w->centre[2];
        geometry[3] = w->length;
    }
    if (target)
        for (int k = 0; k < kOutputs; ++k) target[k] = w->scale[k];
    return 0;
}

int gbWarmStartSetScales(gbWarmStart* w, const float* target) {
    clear_error();
    if (!w || !target) { set_error("gbWarmStartSetScales: bad arguments"); return 1; }
    for (int k = 0; k < kOutputs; ++k) {
        if (!(target[k] > 0.f)) { set_error("gbWarmStartSetScales: scales must be positive"); return 1; }
        w->scale[k] = target[k];
    }
    w->scale_set = true;
    return 0;
}

int gbWarmStartGetFeatures(gbWarmStart* w, float* geo) {
    clear_error();
    if (!w || !geo || !w->mesh) { set_error("gbWarmStartGetFeatures: bad arguments"); return 1; }
    std::vector<float4> h((size_t)w->N);
    if (!ok_(cudaMemcpy(h.data(), w->d_geo, h.size() * sizeof(float4), cudaMemcpyDeviceToHost), "gbWarmStartGetFeatures"))
        return 1;
    const Numbering& U = *w->acc.num;
    for (int64_t i = 0; i < w->N; ++i) {   // reference cell order
        const float4 g = h[U.cell_new[i]];
        geo[4 * i] = g.x;
        geo[4 * i + 1] = g.y;
        geo[4 * i + 2] = g.z;
        geo[4 * i + 3] = g.w;
    }
    return 0;
}

int64_t gbWarmStartFieldCount(gbWarmStart* w) { return w ? (int64_t)w->par.size() : -1; }

static int add_field(WS* w, const float* rho, const float4* rhou, const float* rhoe, gb_vector mach, float p, float T) {
    cudaStream_t s = (cudaStream_t)gbGetStream();
    const int n = (int)w->par.size();
    if (n == w->cap_fields) {
        const int cap = std::max(8, 2 * w->cap_fields);
        float* nt = nullptr;
        if (!ok_(cudaMalloc((void**)&nt, (size_t)cap * w->N * kOutputs * sizeof(float)), "gbWarmStartAddField")) return 1;
        if (w->d_target) {
            if (!ok_(cudaMemcpyAsync(nt, w->d_target, (size_t)n * w->N * kOutputs * sizeof(float),
                                     cudaMemcpyDeviceToDevice, s),
                     "gbWarmStartAddField") ||
                !ok_(cudaStreamSynchronize(s), "gbWarmStartAddField")) {
                cudaFree(nt);
                return 1;
            }
            cudaFree(w->d_target);
        }
        w->d_target = nt;
        w->cap_fields = cap;
    }
    float q[5];
    float4 par;
    freestream(mach, p, T, q, &par);
    k_add_field<<<(unsigned)((w->N + 255) / 256), 256, 0, s>>>(w->N, rho, rhou, rhoe, q[0], q[1], q[2], q[3], q[4],
                                                              w->d_target + (size_t)n * w->N * kOutputs);
    count_launch();
    if (!ok_(cudaGetLastError(), "gbWarmStartAddField")) return 1;
    w->par.push_back(par);
    return 0;
}

int gbWarmStartAddBatchField(gbWarmStart* w, gbBatch* b, int inst, gb_vector mach, gb_scalar pressure,
                             gb_scalar temperature) {
    clear_error();
    BatchInstanceAccess bi;
    if (!w || !w->mesh || !batch_instance(b, inst, &bi)) {
        if (!*gbGetLastError()) set_error("gbWarmStartAddBatchField: bad arguments");
        return 1;
    }
    if (bi.mesh != w->mesh) { set_error("gbWarmStartAddBatchField: instance is on another mesh"); return 1; }
    return add_field(w, bi.rho[bi.cur], bi.rhou[bi.cur], bi.rhoe[bi.cur], mach, pressure, temperature);
}

int gbWarmStartAddField(gbWarmStart* w, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach,
                        gb_scalar pressure, gb_scalar temperature) {
    clear_error();
    FieldAccess a, b, c;
    if (!w || !w->mesh) { set_error("gbWarmStartAddField: needs a warm start with a mesh"); return 1; }
    if (!field_access(rho, w->mesh, 1, &a) || !field_access(rhou, w->mesh, 3, &b) || !field_access(rhoe, w->mesh, 1, &c))
        return 1;
    return add_field(w, (const float*)a.val[a.cur], (const float4*)b.val[b.cur], (const float*)c.val[c.cur], mach,
                     pressure, temperature);
}

int64_t gbWarmStartTrain(gbWarmStart* w, int epochs, int tiles_per_cta, float lr, double* loss_history,
                         int64_t history_len) {
    clear_error();
    if (!w || !w->mesh || w->par.empty() || epochs <= 0 || tiles_per_cta <= 0 || !(lr > 0.f)) {
        set_error("gbWarmStartTrain: bad arguments (needs a mesh, training fields, epochs, tiles, lr)");
        return -1;
    }
    if (!set_smem_attrs()) return -1;
    cudaStream_t s = (cudaStream_t)gbGetStream();
    const int64_t nf = (int64_t)w->par.size();
    const int64_t tpf = (w->N + kTile - 1) / kTile;
    const int64_t n_tiles = nf * tpf;
    const int grid = n_sms();
    // target scales: root mean square of each component over the training set
    if (!w->scale_set) {
        const int blocks = 296;
        double* d_part = nullptr;
        std::vector<double> hp((size_t)blocks * 5);
        if (!ok_(cudaMalloc((void**)&d_part, hp.size() * sizeof(double)), "gbWarmStartTrain")) return -1;
        k_target_moments<<<blocks, 256, 0, s>>>(w->d_target, nf * w->N, d_part);
        count_launch();
        const bool ok = ok_(cudaMemcpyAsync(hp.data(), d_part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s),
                            "gbWarmStartTrain") &&
                        ok_(cudaStreamSynchronize(s), "gbWarmStartTrain");
        cudaFree(d_part);
        if (!ok) return -1;
        for (int k = 0; k < 5; ++k) {
            double a = 0.0;
            for (int b = 0; b < blocks; ++b) a += hp[(size_t)b * 5 + k];
            w->scale[k] = (float)std::max(std::sqrt(a / (double)(nf * w->N)), 1e-6);
        }
        w->scale_set = true;
    }
    if (w->n_par_alloc < (int)nf) {
        if (w->d_par) cudaFree(w->d_par);
        w->d_par = nullptr;
        if (!ok_(cudaMalloc((void**)&w->d_par, nf * sizeof(float4)), "gbWarmStartTrain")) return -1;
        w->n_par_alloc = (int)nf;
    }
    float* d_partials = nullptr;
    double* d_lossp = nullptr;
    double* d_hist = nullptr;
    const int64_t per_step = (int64_t)grid * tiles_per_cta;
    const int64_t total = (int64_t)epochs * n_tiles;
    const int64_t n_steps = (total + per_step - 1) / per_step;
    bool ok = ok_(cudaMemcpyAsync(w->d_par, w->par.data(), nf * sizeof(float4), cudaMemcpyHostToDevice, s),
                  "gbWarmStartTrain") &&
              ok_(cudaMalloc((void**)&d_partials, (size_t)grid * kParams * sizeof(float)), "gbWarmStartTrain") &&
              ok_(cudaMalloc((void**)&d_lossp, grid * sizeof(double)), "gbWarmStartTrain") &&
              ok_(cudaMemsetAsync(w->d_m, 0, kParams * sizeof(float), s), "gbWarmStartTrain") &&
              ok_(cudaMemsetAsync(w->d_v, 0, kParams * sizeof(float), s), "gbWarmStartTrain") && reset_ctl(w, s);
    if (ok && loss_history && history_len > 0)
        ok = ok_(cudaMalloc((void**)&d_hist, std::min(history_len, n_steps) * sizeof(double)), "gbWarmStartTrain");
    TrainArgs ta{};
    ta.img = reinterpret_cast<const uint4*>(w->d_img);
    ta.s.geo = w->d_geo;
    ta.s.par = w->d_par;
    ta.s.target = w->d_target;
    ta.s.n_cells = w->N;
    ta.s.tiles_per_field = tpf;
    ta.s.n_tiles = n_tiles;
    for (int k = 0; k < kOutputs; ++k) ta.s.inv_scale[k] = 1.0f / w->scale[k];
    ta.ctl = w->d_ctl;
    ta.partials = d_partials;
    ta.loss_partials = d_lossp;
    ta.tiles_per_cta = tiles_per_cta;
    ta.permute = 1;
    ta.seed = w->seed;
    ta.total_slots = total;
    ta.dy_scale = 2.0f / (float)(per_step * kTile * kOutputs);
    const double loss_norm = 1.0 / (double)(per_step * kTile * kOutputs);
    const int64_t hist_len = d_hist ? std::min(history_len, n_steps) : 0;
    auto enqueue_step = [&](cudaStream_t st) {
        k_mlp_train<<<grid, kThreads, kSmBytes, st>>>(ta);
        k_mlp_adam<<<(kParams + 255) / 256, 256, 0, st>>>(d_partials, grid, w->d_w, w->d_m, w->d_v, w->d_img,
                                                           w->d_ctl, lr, 0.9f, 0.999f, 1e-8f);
        k_mlp_step_end<<<1, 32, 0, st>>>(w->d_ctl, d_lossp, grid, d_hist, hist_len, loss_norm, 0.9f, 0.999f);
    };
    // the steps run as a replayed graph of up to 64 steps
    const int64_t chunk = std::min<int64_t>(64, n_steps);
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (ok) {
        ok = ok_(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "gbWarmStartTrain");
        cudaGraph_t graph = nullptr;
        ok = ok && ok_(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "gbWarmStartTrain");
        if (ok) {
            for (int64_t k = 0; k < chunk; ++k) enqueue_step(cap);
            ok = ok_(cudaStreamEndCapture(cap, &graph), "gbWarmStartTrain") &&
                 ok_(cudaGraphInstantiate(&exec, graph, 0), "gbWarmStartTrain");
        }
        if (graph) cudaGraphDestroy(graph);
    }
    int64_t done = 0;
    while (ok && done + chunk <= n_steps) {
        ok = ok_(cudaGraphLaunch(exec, s), "gbWarmStartTrain");
        count_launch(3 * (int)chunk);
        done += chunk;
        if (ok && (done / chunk) % 64 == 0) ok = ok_(cudaStreamSynchronize(s), "gbWarmStartTrain") && check_ctl(w, "gbWarmStartTrain");
    }
    while (ok && done < n_steps) {
        enqueue_step(s);
        count_launch(3);
        ++done;
        ok = ok_(cudaGetLastError(), "gbWarmStartTrain");
    }
    ok = ok && ok_(cudaStreamSynchronize(s), "gbWarmStartTrain") && check_ctl(w, "gbWarmStartTrain");
    if (ok && d_hist)
        ok = ok_(cudaMemcpy(loss_history, d_hist, hist_len * sizeof(double), cudaMemcpyDeviceToHost), "gbWarmStartTrain");
    if (exec) cudaGraphExecDestroy(exec);
    if (cap) cudaStreamDestroy(cap);
    for (void* p : {(void*)d_partials, (void*)d_lossp, (void*)d_hist})
        if (p) cudaFree(p);
    return ok ? n_steps : -1;
}

int gbWarmStartSetWaitLimit(gbWarmStart* w, long long cycles) {
    clear_error();
    if (!w) { set_error("gbWarmStartSetWaitLimit: null warm start"); return 1; }
    w->wait_cycles = cycles > 0 ? cycles : 0;
    return 0;
}

int gbWarmStartGradient(gbWarmStart* w, int64_t n, const float* x, const float* t, float* grad, double* loss) {
    clear_error();
    if (!w || n <= 0 || !x || !t || !grad) { set_error("gbWarmStartGradient: bad arguments"); return 1; }
    if (!set_smem_attrs()) return 1;
    cudaStream_t s = (cudaStream_t)gbGetStream();
    const int64_t n_tiles = (n + kTile - 1) / kTile;
    const int tiles_per_cta = 2;
    const int grid = (int)((n_tiles + tiles_per_cta - 1) / tiles_per_cta);
    DevSamples d;
    float* d_partials = nullptr;
    float* d_g = nullptr;
    double* d_lossp = nullptr;
    bool ok = ok_(cudaMalloc((void**)&d.x, n * kFeatures * sizeof(float)), "gbWarmStartGradient") &&
              ok_(cudaMalloc((void**)&d.t, n * kOutputs * sizeof(float)), "gbWarmStartGradient") &&
              ok_(cudaMemcpyAsync(d.x, x, n * kFeatures * sizeof(float), cudaMemcpyHostToDevice, s), "gbWarmStartGradient") &&
              ok_(cudaMemcpyAsync(d.t, t, n * kOutputs * sizeof(float), cudaMemcpyHostToDevice, s), "gbWarmStartGradient") &&
              ok_(cudaMalloc((void**)&d_partials, (size_t)grid * kParams * sizeof(float)), "gbWarmStartGradient") &&
              ok_(cudaMalloc((void**)&d_g, kParams * sizeof(float)), "gbWarmStartGradient") &&
              ok_(cudaMalloc((void**)&d_lossp, grid * sizeof(double)), "gbWarmStartGradient") && reset_ctl(w, s);
    if (ok) {
        TrainArgs ta{};
        ta.img = reinterpret_cast<const uint4*>(w->d_img);
        ta.s = explicit_samples(d, n);
        ta.ctl = w->d_ctl;
        ta.partials = d_partials;
        ta.loss_partials = d_lossp;
        ta.tiles_per_cta = tiles_per_cta;
        ta.permute = 0;
        ta.total_slots = n_tiles;
        ta.dy_scale = 2.0f / (float)(n * kOutputs);
        k_mlp_train<<<grid, kThreads, kSmBytes, s>>>(ta);
        k_grad_sum<<<(kParams + 255) / 256, 256, 0, s>>>(d_partials, grid, d_g);
        count_launch(2);
        std::vector<double> lp(grid);
        ok = ok_(cudaGetLastError(), "gbWarmStartGradient") &&
             ok_(cudaMemcpyAsync(grad, d_g, kParams * sizeof(float), cudaMemcpyDeviceToHost, s), "gbWarmStartGradient") &&
             ok_(cudaMemcpyAsync(lp.data(), d_lossp, grid * sizeof(double), cudaMemcpyDeviceToHost, s),
                 "gbWarmStartGradient") &&
             ok_(cudaStreamSynchronize(s), "gbWarmStartGradient") && check_ctl(w, "gbWarmStartGradient");
        if (ok && loss) {
            double a = 0.0;
            for (double v : lp) a += v;
            *loss = a / (double)(n * kOutputs);
        }
    }
    for (void* p : {(void*)d_partials, (void*)d_g, (void*)d_lossp})
        if (p) cudaFree(p);
    return ok ? 0 : 1;
}

int gbWarmStartForward(gbWarmStart* w, int64_t n, const float* x, float* y) {
    clear_error();
    if (!w || n <= 0 || !x || !y) { set_error("gbWarmStartForward: bad arguments"); return 1; }
    cudaStream_t s = (cudaStream_t)gbGetStream();
    DevSamples d;
    float* d_y = nullptr;
    bool ok = ok_(cudaMalloc((void**)&d.x, n * kFeatures * sizeof(float)), "gbWarmStartForward") &&
              ok_(cudaMemcpyAsync(d.x, x, n * kFeatures * sizeof(float), cudaMemcpyHostToDevice, s), "gbWarmStartForward") &&
              ok_(cudaMalloc((void**)&d_y, n * kOutputs * sizeof(float)), "gbWarmStartForward") && reset_ctl(w, s);
    if (ok) {
        ForwardArgs fa{};
        fa.img = reinterpret_cast<const uint4*>(w->d_img);
        fa.s = explicit_samples(d, n);
        fa.s.t = nullptr;
        fa.ctl = w->d_ctl;
        fa.y = d_y;
        ok = forward_launch(w, fa, (n + kTile - 1) / kTile, s) &&
             ok_(cudaMemcpyAsync(y, d_y, n * kOutputs * sizeof(float), cudaMemcpyDeviceToHost, s), "gbWarmStartForward") &&
             ok_(cudaStreamSynchronize(s), "gbWarmStartForward") && check_ctl(w, "gbWarmStartForward");
    }
    if (d_y) cudaFree(d_y);
    return ok ? 0 : 1;
}

static int predict(WS* w, float* rho[2], float4* rhou[2], float* rhoe[2], gb_vector mach, float p, float T) {
    cudaStream_t s = (cudaStream_t)gbGetStream();
    float q[5];
    float4 par;
    freestream(mach, p, T, q, &par);
    float4* d_par1 = nullptr;
    bool ok = ok_(cudaMalloc((void**)&d_par1, sizeof(float4)), "gbWarmStartPredict") &&
              ok_(cudaMemcpyAsync(d_par1, &par, sizeof(float4), cudaMemcpyHostToDevice, s), "gbWarmStartPredict") &&
              reset_ctl(w, s);
    if (ok) {
        ForwardArgs fa{};
        fa.img = reinterpret_cast<const uint4*>(w->d_img);
        fa.s.geo = w->d_geo;
        fa.s.par = d_par1;
        fa.s.n_cells = w->N;
        fa.s.tiles_per_field = (w->N + kTile - 1) / kTile;
        fa.s.n_tiles = fa.s.tiles_per_field;
        fa.ctl = w->d_ctl;
        fa.rho0 = rho[0]; fa.rho1 = rho[1];
        fa.rhou0 = rhou[0]; fa.rhou1 = rhou[1];
        fa.rhoe0 = rhoe[0]; fa.rhoe1 = rhoe[1];
        for (int k = 0; k < kOutputs; ++k) {
            fa.qinf[k] = q[k];
            fa.scale[k] = w->scale[k];
        }
        ok = forward_launch(w, fa, fa.s.n_tiles, s) && ok_(cudaStreamSynchronize(s), "gbWarmStartPredict") &&
             check_ctl(w, "gbWarmStartPredict");
    }
    if (d_par1) cudaFree(d_par1);
    return ok ? 0 : 1;
}

int gbWarmStartPredictBatch(gbWarmStart* w, gbBatch* b, int inst, gb_vector mach, gb_scalar pressure,
                            gb_scalar temperature) {
    clear_error();
    BatchInstanceAccess bi;
    if (!w || !w->mesh || !batch_instance(b, inst, &bi)) {
        if (!*gbGetLastError()) set_error("gbWarmStartPredictBatch: bad arguments");
        return 1;
    }
    if (bi.mesh != w->mesh) { set_error("gbWarmStartPredictBatch: instance is on another mesh"); return 1; }
    return predict(w, bi.rho, bi.rhou, bi.rhoe, mach, pressure, temperature);
}

int gbWarmStartPredict(gbWarmStart* w, FvmField* rho, FvmField* rhou, FvmField* rhoe, gb_vector mach,
                       gb_scalar pressure, gb_scalar temperature) {
    clear_error();
    FieldAccess a, b, c;
    if (!w || !w->mesh) { set_error("gbWarmStartPredict: needs a warm start with a mesh"); return 1; }
    if (!field_access(rho, w->mesh, 1, &a) || !field_access(rhou, w->mesh, 3, &b) || !field_access(rhoe, w->mesh, 1, &c))
        return 1;
    float* r[2] = {(float*)a.val[0], (float*)a.val[1]};
    float4* u[2] = {(float4*)b.val[0], (float4*)b.val[1]};
    float* e[2] = {(float*)c.val[0], (float*)c.val[1]};
    return predict(w, r, u, e, mach, pressure, temperature);
}

}  // extern "C"

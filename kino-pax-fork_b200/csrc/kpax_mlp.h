// kpax_mlp.h — layout of the learned proposal network, shared by its kernels and the planner.
//
// The network has no counterpart in the reference planner, which draws every control and
// duration uniformly (propagateAndCheck in statePropagatorSpatialHash.cu).  It only changes the
// distribution of those draws: every segment is still propagated and collision-checked exactly.
//
// 51 inputs (12D quadrotor state, goal - state, 27 occupancy bits of the 3x3x3 R1 workspace
// cells around the state) -> 256 -> 256 (SiLU) -> 88 outputs: 8 mixture components, each
// 1 logit + 5 means + 5 log-standard-deviations over the logits of the five draw uniforms
// (4 controls, duration).  FP32 master parameters live in one array; rows are padded (inputs to
// 64, outputs to 96) so every GEMM dimension is a multiple of 16.  The tensor-core copy is an
// image of BF16 weights in the shared-memory layout the MMA reads (K-major, 128-byte swizzle),
// followed by the FP32 biases.
#pragma once
#include <stddef.h>
#include <stdint.h>

namespace kpax {
namespace mlp {

constexpr int kIn = 51, kInPad = 64, kH = 256, kOut = 88, kOutPad = 96, kComp = 8, kDim = 5, kCompStride = 11;
constexpr size_t kOffW1 = 0;                        // [kH][kInPad]
constexpr size_t kOffB1 = kOffW1 + kH * kInPad;     // [kH]
constexpr size_t kOffW2 = kOffB1 + kH;              // [kH][kH]
constexpr size_t kOffB2 = kOffW2 + kH * kH;         // [kH]
constexpr size_t kOffW3 = kOffB2 + kH;              // [kOutPad][kH]
constexpr size_t kOffB3 = kOffW3 + kOutPad * kH;    // [kOutPad]
constexpr size_t kNumParams = kOffB3 + kOutPad;
constexpr uint64_t kFlopPerInference = 2ull * (kIn * kH + kH * kH + kH * kOut);  // 202 240

// Log-standard-deviation: s = kSigMid + kSigHalf * tanh(raw / kSigHalf), in (-7, 3).
constexpr float kSigMid = -2.0f, kSigHalf = 5.0f;
// Logit targets are clamped to +-kLogitClamp (u in [1e-4, 1 - 1e-4]).
constexpr float kLogitClamp = 9.21024f;

// Per-entry mixture record written by the proposal pass: the network's 88 outputs with biases,
// component k at [11k] (logit), [11k+1 .. 11k+5] (means), [11k+6 .. 11k+10] (raw log-sigmas).
constexpr int kMixFloats = kOut;

// BF16 image: slabs of 64 K-columns, each row 128 bytes, rows grouped by 8 into 1024-byte atoms,
// the 16-byte chunk j of row r stored at chunk position j ^ (r & 7).
constexpr uint32_t kSlabRowBytes = 128;
constexpr uint32_t kImgW1 = 0;                               // 256 rows x 64
constexpr uint32_t kImgW2 = kImgW1 + kH * kSlabRowBytes;     // 4 slabs of 256 rows
constexpr uint32_t kImgW3 = kImgW2 + 4 * kH * kSlabRowBytes; // 4 slabs of 96 rows
constexpr uint32_t kImgBias = kImgW3 + 4 * kOutPad * kSlabRowBytes;
constexpr uint32_t kImgBytes = kImgBias + (kH + kH + kOutPad) * 4;

__host__ __device__ inline uint32_t swz(uint32_t r, uint32_t k)  // byte offset of (row, k) in a slab
{
    return (r >> 3) * 1024u + (r & 7u) * 128u + ((((k >> 3) ^ (r & 7u)) & 7u) << 4) + ((k & 7u) << 1);
}

// Input scaling: positions and goal offsets / 100, velocities / 10, angles and rates unscaled.
__host__ __device__ inline float input_scale(int i)
{
    if(i >= 24) return 1.0f;  // occupancy bits
    const int d = i % 12;
    if(d < 3) return 0.01f;
    if(d >= 6 && d < 9) return 0.1f;
    return 1.0f;
}

}  // namespace mlp
}  // namespace kpax

// green_sg.h -- the surrogate's inference kernel for far panel pairs (green_sg.cu).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <vector>

#include "kernels.cuh"
#include "surrogate.h"

// One 128 x 128 FP16 operand in the tensor cores' canonical K-major layout
// without swizzle: 8 x 8 core matrices (8 rows of 16 bytes, 128 bytes
// contiguous), 16 along K 128 bytes apart, row groups of 8 rows 2048 bytes
// apart.  Byte offset of element (row, k):
__host__ __device__ constexpr int sg_core_off(int row, int k) {
  return (row >> 3) * 2048 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}
constexpr int kSgOperandBytes = 128 * 128 * 2;
// output layer: 16 rows (3 used) x 128
constexpr int kSgOutRows = 16;
constexpr int kSgOutBytes = kSgOutRows * 128 * 2;
// hidden layers 1..3 then the output layer
constexpr int kSgHalves = ((sg::kHidden - 1) * kSgOperandBytes + kSgOutBytes) / 2;
constexpr int kSgBias = sg::kHidden * sg::kWidth + 8;
// The biases of layers 1..3 and of the output layer enter through the tensor
// cores: one more K = 16 product per layer, a 128 x 16 block of ones (columns
// 0 and 1 one, the rest zero) times a bias block (row o: the layer's bias o
// split into two FP16 parts, hi = fp16(b), lo = fp16(b - hi), in columns 0
// and 1).  These small operands use the same core matrices with 8-row groups
// 256 bytes apart; byte offset of element (row, k < 16):
__host__ __device__ constexpr int sg_small_off(int row, int k) {
  return (row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}
constexpr int kSgOnesBytes = 128 * 16 * 2;
constexpr int kSgBiasBlkBytes = 128 * 16 * 2;        // hidden layers
constexpr int kSgBiasOutBytes = kSgOutRows * 16 * 2;  // output layer
constexpr int kSgOnesOff = kSgHalves * 2;             // byte offsets in the image
constexpr int kSgBiasBlkOff = kSgOnesOff + kSgOnesBytes;
// The first layer (4 inputs) is one K = 16 product as well, at FP32
// accuracy from FP16 parts: the pair's row is (f_hi[0..3], f_lo[0..3],
// f_hi[0..3], 1, 1, 0, 0) and output o's row (w_hi[0..3], w_hi[0..3],
// w_lo[0..3], b_hi, b_lo, 0, 0), x_hi = fp16(x), x_lo = fp16(x - x_hi), so
// that the product is w f + b up to the w_lo f_lo term (~2^-22 relative).
constexpr int kSgW0Off = kSgBiasBlkOff + (sg::kHidden - 1) * kSgBiasBlkBytes + kSgBiasOutBytes;
constexpr int kSgW0Bytes = 128 * 16 * 2;
// the whole image copied to shared memory: weights, ones, bias blocks, first layer
constexpr int kSgImageBytes = kSgW0Off + kSgW0Bytes;
static_assert(kSgImageBytes % 16 == 0, "image copied in 16-byte pieces");

// device copy of a trained network, in the kernel's layout
struct SgDev {
  const __half* wh;    // kSgImageBytes / 2: the weight image (weights, ones, bias blocks)
  const float* w0;     // first layer, 128 x 4 column-major
  const float* bias;   // kSgBias: layer l at l * 128, output layer at 4 * 128
  double mean[sg::kOut], scale[sg::kOut];
};

// Green functions of `count` far pairs (list of pair indices) from the
// network at dispersion parameter K = k0 h tanh(k0 h), the propagating mode
// from slot 1 of the frequency's mode tables; a tensor-core barrier wait that
// gives up sets bit 2 of *err.  Returns 0, or 1 on a launch error.
int launch_green_sg(cudaStream_t st, int sms, DevGeom g, WaveDev w, const SgDev& sp, const hams::ModeTab& mt, double K,
                    const uint32_t* pairs, long long count, const double* rs, const double* rd, double2* A,
                    double2* S, int* err);

// Trained parameters (surrogate.h layout) into the kernel's layout.
void pack_surrogate(const float* P, std::vector<__half>& wh, std::vector<float>& w0, std::vector<float>& bias);

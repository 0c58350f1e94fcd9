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
// hidden layers 1..3 then the output layer, as one image copied to shared memory
constexpr int kSgHalves = ((sg::kHidden - 1) * kSgOperandBytes + kSgOutBytes) / 2;
constexpr int kSgBias = sg::kHidden * sg::kWidth + 8;

// device copy of a trained network, in the kernel's layout
struct SgDev {
  const __half* wh;    // kSgHalves: the weight image
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

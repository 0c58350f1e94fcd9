// green_sg.h -- the surrogate's inference kernel for far panel pairs (green_sg.cu).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <vector>

#include "kernels.cuh"
#include "surrogate.h"

// padded row length (halves) of the weight rows in shared memory: 136 halves
// put the 8 rows a fragment load touches in distinct banks
constexpr int kSgPadK = 136;
// hidden layers 1..3 (128 rows each) and the output layer (8 rows, 3 used)
constexpr int kSgHalves = ((sg::kHidden - 1) * sg::kWidth + 8) * kSgPadK;
constexpr int kSgBias = sg::kHidden * sg::kWidth + 8;
constexpr int kSgSmem = kSgHalves * 2 + (sg::kWidth * sg::kIn + kSgBias) * 4;

// device copy of a trained network, in the kernel's layout
struct SgDev {
  const __half* wh;    // kSgHalves: rows [layer][out][kSgPadK]
  const float* w0;     // first layer, 128 x 4 column-major
  const float* bias;   // kSgBias: layer l at l * 128, output layer at 4 * 128
  double mean[sg::kOut], scale[sg::kOut];
};

// Green functions of `count` far pairs (list of pair indices) from the
// network at dispersion parameter K = k0 h tanh(k0 h), the propagating mode
// from slot 1 of the frequency's mode tables; returns 0 or 1 on a launch
// error.
int launch_green_sg(cudaStream_t st, int sms, DevGeom g, WaveDev w, const SgDev& sp, const hams::ModeTab& mt, double K,
                    const uint32_t* pairs, long long count, const double* rs, const double* rd, double2* A,
                    double2* S);

// Trained parameters (surrogate.h layout) into the kernel's layout.
void pack_surrogate(const float* P, std::vector<__half>& wh, std::vector<float>& w0, std::vector<float>& bias);

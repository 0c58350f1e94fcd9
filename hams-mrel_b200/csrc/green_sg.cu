// green_sg.cu -- far-field finite-depth Green functions from the MLP
// surrogate (surrogate.h), fused with the pair algebra of the assembly.
//
// One warp evaluates 16 panel pairs at a time.  The first layer (4 inputs)
// runs in FP32 on the CUDA cores; the three 128 x 128 hidden layers and the
// output layer run on the tensor cores as mma.sync m16n8k16 (FP16 operands,
// FP32 accumulation) with the pairs as the M dimension, so each layer's
// accumulator fragments, after bias and SiLU, are repacked in registers as
// the next layer's A fragments.  The weights of a block live in shared
// memory.  Lanes 0-15 then finish their pair in FP64: the exact propagating
// mode (FinGreen3D.f90:311-322), the surrogate's evanescent part, the point
// source terms by the near/far flag, and A, S as the series kernels store
// them.
#include <cuda_fp16.h>

#include "kernels.cuh"
#include "surrogate.h"
#include "green_sg.h"

namespace {

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

// SiLU as z (1 + tanh(z / 2)) / 2 with the hardware tanh approximation
// (relative error ~2^-11, below the FP16 rounding of the activations)
__device__ __forceinline__ float silu(float z) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
  return 0.5f * z * (1.0f + t);
}

// Four 8 x 8 FP16 matrices from shared memory (one row address per lane).
__device__ __forceinline__ void ldsm_x4(const __half* row, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  unsigned a = (unsigned)__cvta_generic_to_shared(row);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(a));
}

}  // namespace

__global__ void __launch_bounds__(128, 2) k_green_sg(DevGeom g, WaveDev w, SgDev sp, hams::ModeTab mt, double K,
                                                     const uint32_t* __restrict__ pairs, long long count,
                                                     const double* __restrict__ rs, const double* __restrict__ rd,
                                                     double2* __restrict__ A, double2* __restrict__ S) {
  extern __shared__ __align__(16) unsigned char smem[];
  __half* sW = reinterpret_cast<__half*>(smem);                        // kSgHalves
  float* sW0 = reinterpret_cast<float*>(smem + kSgHalves * 2);         // 128 x 4, column-major
  float* sB = sW0 + sg::kWidth * sg::kIn;                              // biases
  {
    const uint4* src = reinterpret_cast<const uint4*>(sp.wh);
    uint4* dst = reinterpret_cast<uint4*>(sW);
    for (int e = threadIdx.x; e < kSgHalves / 8; e += blockDim.x) dst[e] = src[e];
    for (int e = threadIdx.x; e < sg::kWidth * sg::kIn; e += blockDim.x) sW0[e] = sp.w0[e];
    for (int e = threadIdx.x; e < kSgBias; e += blockDim.x) sB[e] = sp.bias[e];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const double h = w.h;
  const long long ngroups = (count + 15) / 16;
  for (long long grp = (long long)blockIdx.x * 4 + warp; grp < ngroups; grp += (long long)gridDim.x * 4) {
    // pair of this lane (lanes 16-31 repeat lanes 0-15)
    const long long t = grp * 16 + (lane & 15);
    const bool live = t < count;
    size_t p = 0;
    int i = 0, j = 0;
    double xp = 0, yp = 0, zp = -0.25 * h, xq = 0.1 * h, yq = 0, zq = -0.25 * h;
    if (live) {
      p = pairs[t];
      i = (int)(p % (size_t)g.tn);
      j = (int)(p / (size_t)g.tn);
      xp = g.fxyz[i];
      yp = g.fxyz[i + g.tn];
      zp = g.fxyz[i + 2 * g.tn];
      xq = g.xq[j];
      yq = g.xq[j + g.n];
      zq = g.xq[j + 2 * g.n];
    }
    const double xpq = xq - xp, ypq = yq - yp;
    const double rr = sqrt(xpq * xpq + ypq * ypq);
    const double X = rr / h;
    float f[sg::kIn];
    sg::features(X, (zq + h) / h, (zp + h) / h, K, f);
    // inputs of rows gq and gq + 8 of the 16 x 4 input tile
    float fa[sg::kIn], fb[sg::kIn];
    for (int k = 0; k < sg::kIn; ++k) {
      fa[k] = __shfl_sync(0xffffffffu, f[k], gq);
      fb[k] = __shfl_sync(0xffffffffu, f[k], gq + 8);
    }
    // layer 0 in FP32, straight into A fragments
    uint32_t a[8][4];
#pragma unroll
    for (int kt = 0; kt < 8; ++kt) {
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int o = 16 * kt + 2 * tq + 8 * hh;
        float va0 = sB[o], va1 = sB[o + 1], vb0 = sB[o], vb1 = sB[o + 1];
#pragma unroll
        for (int k = 0; k < sg::kIn; ++k) {
          const float w0 = sW0[o + sg::kWidth * k], w1 = sW0[o + 1 + sg::kWidth * k];
          va0 = fmaf(w0, fa[k], va0);
          va1 = fmaf(w1, fa[k], va1);
          vb0 = fmaf(w0, fb[k], vb0);
          vb1 = fmaf(w1, fb[k], vb1);
        }
        a[kt][2 * hh] = pack2(silu(va0), silu(va1));
        a[kt][2 * hh + 1] = pack2(silu(vb0), silu(vb1));
      }
    }
    // hidden layers 1..3 on the tensor cores
#pragma unroll 1
    for (int l = 1; l < sg::kHidden; ++l) {
      const __half* Wl = sW + (size_t)(l - 1) * sg::kWidth * kSgPadK;
      float c[16][4];
#pragma unroll
      for (int nt = 0; nt < 16; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0f;
      // lane L addresses row L % 8 of matrix L / 8: (n-tile nt + m / 2, k half m % 2)
      const int lm = lane >> 3, lr = lane & 7;
#pragma unroll
      for (int kt = 0; kt < 8; ++kt) {
#pragma unroll
        for (int nt = 0; nt < 16; nt += 2) {
          uint32_t b00, b01, b10, b11;
          ldsm_x4(Wl + (size_t)(8 * (nt + (lm >> 1)) + lr) * kSgPadK + 16 * kt + 8 * (lm & 1), b00, b01, b10, b11);
          mma16816(c[nt], a[kt], b00, b01);
          mma16816(c[nt + 1], a[kt], b10, b11);
        }
      }
      const float* bl = sB + l * sg::kWidth;
#pragma unroll
      for (int nt = 0; nt < 16; ++nt) {
        const int o = 8 * nt + 2 * tq;
        const uint32_t lo = pack2(silu(c[nt][0] + bl[o]), silu(c[nt][1] + bl[o + 1]));
        const uint32_t hi = pack2(silu(c[nt][2] + bl[o]), silu(c[nt][3] + bl[o + 1]));
        a[nt / 2][(nt & 1) * 2] = lo;
        a[nt / 2][(nt & 1) * 2 + 1] = hi;
      }
    }
    // output layer: one n-tile, columns 0-2 used
    float co[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    {
      const __half* Wo = sW + (size_t)(sg::kHidden - 1) * sg::kWidth * kSgPadK;
#pragma unroll
      for (int kt = 0; kt < 8; ++kt) {
        const __half* row = Wo + (size_t)gq * kSgPadK + 16 * kt + 2 * tq;
        mma16816(co, a[kt], *reinterpret_cast<const uint32_t*>(row), *reinterpret_cast<const uint32_t*>(row + 8));
      }
    }
    // outputs of pair L (lane L < 16): row L % 8 of the tile, upper half for L >= 8
    const int src = 4 * (lane & 7);
    const float r0a = __shfl_sync(0xffffffffu, co[0], src), r0b = __shfl_sync(0xffffffffu, co[2], src);
    const float r1a = __shfl_sync(0xffffffffu, co[1], src), r1b = __shfl_sync(0xffffffffu, co[3], src);
    const float r2a = __shfl_sync(0xffffffffu, co[0], src + 1), r2b = __shfl_sync(0xffffffffu, co[2], src + 1);
    const bool up = (lane & 15) >= 8;
    const float* bo = sB + sg::kHidden * sg::kWidth;
    const double y0 = (double)((up ? r0b : r0a) + bo[0]), y1 = (double)((up ? r1b : r1a) + bo[1]),
                 y2 = (double)((up ? r2b : r2a) + bo[2]);
    if (lane < 16 && live) {
      const double t0 = sp.mean[0] + sp.scale[0] * y0, t1 = sp.mean[1] + sp.scale[1] * y1,
                   t2 = sp.mean[2] + sp.scale[2] * y2;
      // propagating mode (FinGreen3D.f90:311-322) from the per-frequency factors
      hams::cplx fg[3];
      double rk[3];
      {
        const double2 sc = mt.src[g.n + j];
        const double czp = mt.fld[g.tn + i], p0 = mt.pm[1] * sc.y * czp, dp0 = mt.pm[1] * sc.x * czp;
        double j0, j1, y0, y1;
        hams::jy01b(w.wk * rr, j0, j1, y0, y1);
        fg[0] = hams::cmk(-p0 * y0, p0 * j0);
        fg[1] = hams::cmk(w.wk * p0 * y1, -w.wk * p0 * j1);
        fg[2] = hams::cmk(-w.wk * dp0 * y0, w.wk * dp0 * j0);
      }
      sg::rankine_parts(rr, zq, zp, rk);
      fg[0].re += t0 / (X * h) + rk[0];
      fg[1].re += t1 / (X * X * h * h) + rk[1];
      fg[2].re += t2 / (X * X * h * h) + rk[2];
      const double zpq = zq + zp;
      const double r = sqrt(rr * rr + (zp - zq) * (zp - zq)), r1 = sqrt(rr * rr + zpq * zpq);
      const int flag = near_flag(g, i, j);
      grn4 G = hams::finish_green(fg, xpq, ypq, zq, zp, rr, r, r1, flag);
      store_pair(g, p, i, j, G, rs, rd, A, S);
    }
  }
}

int launch_green_sg(cudaStream_t st, int sms, DevGeom g, WaveDev w, const SgDev& sp, const hams::ModeTab& mt, double K,
                    const uint32_t* pairs,
                    long long count, const double* rs, const double* rd, double2* A, double2* S) {
  if (count <= 0) return 0;
  if (cudaFuncSetAttribute(k_green_sg, cudaFuncAttributeMaxDynamicSharedMemorySize, kSgSmem) != cudaSuccess) return 1;
  long long groups = (count + 15) / 16;
  long long blocks = std::min<long long>(2LL * sms, (groups + 3) / 4);
  k_green_sg<<<(unsigned)blocks, 128, kSgSmem, st>>>(g, w, sp, mt, K, pairs, count, rs, rd, A, S);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

void pack_surrogate(const float* P, std::vector<__half>& wh, std::vector<float>& w0, std::vector<float>& bias) {
  wh.assign(kSgHalves, __float2half(0.0f));
  for (int l = 1; l < sg::kLayers; ++l) {
    const int fi = sg::layer_in(l), fo = sg::layer_out(l);
    __half* dst = wh.data() + (size_t)(l - 1) * sg::kWidth * kSgPadK;
    for (int o = 0; o < fo; ++o)
      for (int k = 0; k < fi; ++k) dst[(size_t)o * kSgPadK + k] = __float2half(P[sg::w_off(l) + o + fo * k]);
  }
  w0.assign(P + sg::w_off(0), P + sg::w_off(0) + sg::kWidth * sg::kIn);
  bias.assign(kSgBias, 0.0f);
  for (int l = 0; l < sg::kLayers; ++l)
    for (int o = 0; o < sg::layer_out(l); ++o) bias[l * sg::kWidth + o] = P[sg::b_off(l) + o];
}

// green_sg.cu -- far-field finite-depth Green functions from the MLP
// surrogate (surrogate.h), fused with the pair algebra of the assembly, on
// the fifth-generation tensor cores.
//
// A CTA runs kWG warpgroups; each takes tiles of 128 panel pairs, one pair
// per thread.  Every layer runs as tcgen05.mma (FP16 operands, FP32
// accumulation, M = 128 pairs) issued by one thread of the warpgroup, with
// the activations of the tile and all weights in shared memory in the
// canonical K-major layout and the accumulator in tensor memory: the first
// layer (4 inputs and the bias) as one K = 16 product of the inputs and
// weights split into FP16 parts (FP32 accuracy, green_sg.h), the three
// 128 x 128 hidden layers and the output layer as eight K = 16 products
// plus one for the bias (a block of ones times the bias split in two).
// After each layer the warpgroup reads its 128 x 128 accumulator back with
// tcgen05.ld (thread t owns TMEM lane t = pair t), applies SiLU, and writes
// the FP16 activations over the tile for the next layer.  While one warpgroup runs its epilogue the
// other's MMAs run.  Each thread then finishes its pair in FP64: the exact
// propagating mode (FinGreen3D.f90:311-322), the surrogate's evanescent part,
// the point-source terms by the near/far flag, and A, S as the series kernels
// store them.
//
// Every wait on a tensor-core completion barrier is bounded; a wait that
// gives up sets bit 2 of the error word, the warpgroup stops, and the CTA
// frees its tensor memory before it returns.
#include <cuda_fp16.h>

#include "kernels.cuh"
#include "surrogate.h"
#include "green_sg.h"

namespace {

constexpr int kWG = 3;                 // warpgroups per CTA, one 128-pair tile in flight each
constexpr int kThreads = 128 * kWG;
constexpr int kCols = kWG <= 2 ? 256 : 512;  // TMEM columns (power of two): 128 f32 columns per warpgroup
constexpr int kOffAct = (kSgImageBytes + 1023) / 1024 * 1024;  // activation tiles, one per warpgroup
constexpr int kOffBar = kOffAct + kWG * kSgOperandBytes;  // one mbarrier per warpgroup
constexpr int kOffTmem = kOffBar + 8 * kWG;                          // TMEM base written by tcgen05.alloc
constexpr int kSmemBytes = kOffTmem + 16;
static_assert(kCols >= 128 * kWG, "tensor memory for the accumulators");
static_assert(kSmemBytes <= 227 * 1024, "shared memory per CTA");

// instruction descriptor of kind::f16: FP16 A and B, FP32 D, both K-major,
// M = 128, N = n
constexpr uint32_t idesc_f16(int n) { return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24); }
constexpr uint32_t kIdescHidden = idesc_f16(128), kIdescOut = idesc_f16(kSgOutRows);

// shared-memory matrix descriptor of a canonical K-major operand without
// swizzle (sg_core_off): K-direction core matrices 128 B apart (leading byte
// offset), 8-row groups 2048 B apart (stride byte offset), version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(2048 >> 4) << 32) |
         (1ull << 46);
}
// the same for the 16-column ones and bias blocks (sg_small_off): 8-row
// groups 256 B apart
__device__ __forceinline__ uint64_t sdesc_small(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
         (1ull << 46);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// bounded wait for the phase `parity` of the mbarrier to complete
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void wg_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
// OR of p over the 128 threads of a warpgroup (a barrier as well)
__device__ __forceinline__ bool wg_any(int id, bool p) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred q, s;\n\tsetp.ne.u32 q, %1, 0;\n\tbarrier.red.or.pred s, %2, 128, q;\n\t"
      "selp.u32 %0, 1, 0, s;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)p), "r"(id)
      : "memory");
  return r != 0;
}

// 16 consecutive f32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

// SiLU of z = 2h from the half pre-activation h (the weights and biases of
// the layers that feed a SiLU are stored halved, an exact power-of-two
// scaling): silu(z) = z (1 + tanh(z / 2)) / 2 = h + h tanh(h), one hardware
// tanh (relative error ~2^-11, below the FP16 rounding of the activations)
// and one fused multiply-add.
__device__ __forceinline__ float silu(float h) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
  return fmaf(h, t, h);
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 1) k_green_sg(DevGeom g, WaveDev w, SgDev sp, hams::ModeTab mt, double K,
                                                          const uint32_t* __restrict__ pairs, long long count,
                                                          const double* __restrict__ rs, const double* __restrict__ rd,
                                                          double2* __restrict__ A, double2* __restrict__ S, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kOffTmem);
  const int tid = threadIdx.x, warp = tid >> 5, wg = warp >> 2, t = tid & 127;
  {
    const uint4* src = reinterpret_cast<const uint4*>(sp.wh);
    uint4* dst = reinterpret_cast<uint4*>(smem);
    for (int e = tid; e < kSgImageBytes / 16; e += kThreads) dst[e] = src[e];
  }
  if (tid == 0) {
    for (int k = 0; k < kWG; ++k) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[k])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *reinterpret_cast<volatile uint32_t*>(tslot);
  const uint32_t tacc = tbase + (uint32_t)(128 * wg);                   // this warpgroup's accumulator
  const uint32_t tld = tacc + ((uint32_t)(32 * (warp & 3)) << 16);     // + this warp's 32 lanes
  unsigned char* act = smem + kOffAct + wg * kSgOperandBytes;
  const uint32_t act_sa = smem_u32(act), w_sa = smem_u32(smem), bar = smem_u32(&bars[wg]);
  const int bar_id = 1 + wg;
  uint32_t phase = 0;
  const double h = w.h;
  const long long ntiles = (count + 127) / 128;
  for (long long tile = (long long)blockIdx.x * kWG + wg; tile < ntiles; tile += (long long)gridDim.x * kWG) {
    const long long tp = tile * 128 + t;
    const bool live = tp < count;
    size_t p = 0;
    int i = 0, j = 0;
    double xp = 0, yp = 0, zp = -0.25 * h, xq = 0.1 * h, yq = 0, zq = -0.25 * h;
    // the pair's FP64 operands of the epilogue, loaded now so that their
    // latency passes under the network's layers
    double pf_rs = 0.0, pf_rd = 0.0, pf_ds = 0.0, pf_n1 = 0.0, pf_n2 = 0.0, pf_n3 = 0.0, pf_pn = 0.0, pf_fld = 0.0;
    double2 pf_src = make_double2(0.0, 0.0);
    if (live) {
      p = pairs[tp];
      i = (int)(p % (size_t)g.tn);
      j = (int)(p / (size_t)g.tn);
      xp = g.fxyz[i];
      yp = g.fxyz[i + g.tn];
      zp = g.fxyz[i + 2 * g.tn];
      xq = g.xq[j];
      yq = g.xq[j + g.n];
      zq = g.xq[j + 2 * g.n];
      pf_rs = rs[p];
      pf_rd = rd[p];
      pf_ds = g.ds[j];
      pf_n1 = g.nrm[j];
      pf_n2 = g.nrm[j + g.n];
      pf_n3 = g.nrm[j + 2 * g.n];
      pf_pn = g.pnsz[j];
      pf_src = mt.src[g.n + j];  // the propagating mode's vertical factors (mode-table slot 1)
      pf_fld = mt.fld[g.tn + i];
    }
    const double xpq = xq - xp, ypq = yq - yp;
    const double rr = sqrt(xpq * xpq + ypq * ypq);
    const double X = rr / h;
    float f[sg::kIn];
    sg::features(X, (zq + h) / h, (zp + h) / h, K, f);
    // the first layer's operand row (green_sg.h) into K columns 0..15 of the tile
    {
      uint32_t hv[8];
      __half fh[sg::kIn], fl[sg::kIn];
#pragma unroll
      for (int k = 0; k < sg::kIn; ++k) {
        fh[k] = __float2half_rn(f[k]);
        fl[k] = __float2half_rn(f[k] - __half2float(fh[k]));
      }
      auto pk = [](__half a, __half b) {
        __half2 v = __halves2half2(a, b);
        return *reinterpret_cast<uint32_t*>(&v);
      };
      const __half one = __float2half_rn(1.0f), zero = __float2half_rn(0.0f);
      hv[0] = pk(fh[0], fh[1]);
      hv[1] = pk(fh[2], fh[3]);
      hv[2] = pk(fl[0], fl[1]);
      hv[3] = pk(fl[2], fl[3]);
      hv[4] = pk(fh[0], fh[1]);
      hv[5] = pk(fh[2], fh[3]);
      hv[6] = pk(one, one);
      hv[7] = pk(zero, zero);
      *reinterpret_cast<uint4*>(act + sg_core_off(t, 0)) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
      *reinterpret_cast<uint4*>(act + sg_core_off(t, 8)) = make_uint4(hv[4], hv[5], hv[6], hv[7]);
    }
    // layer 0 (K = 16), layers 1..3 (N = 128) and the output layer (N = 16, three columns used)
    float y[3] = {0.0f, 0.0f, 0.0f};
    bool ok = true;
    for (int l = 0; l <= sg::kHidden; ++l) {
      proxy_fence();
      tc_fence_before();
      wg_sync(bar_id);
      if (t == 0) {
        tc_fence_after();
        if (l == 0) {
          umma_f16(tacc, sdesc(act_sa), sdesc_small(w_sa + kSgW0Off), kIdescHidden, 0);
        } else {
          const uint32_t wb = w_sa + (uint32_t)((l - 1) * kSgOperandBytes);
          const uint32_t id = l < sg::kHidden ? kIdescHidden : kIdescOut;
#pragma unroll
          for (int s = 0; s < 8; ++s) umma_f16(tacc, sdesc(act_sa + 256 * s), sdesc(wb + 256 * s), id, s > 0);
          // + the bias: ones (128 x 16) times the layer's bias block
          umma_f16(tacc, sdesc_small(w_sa + kSgOnesOff),
                   sdesc_small(w_sa + (uint32_t)(kSgBiasBlkOff + (l - 1) * kSgBiasBlkBytes)), id, 1);
        }
        umma_commit(bar);
      }
      const bool done = mbar_wait(bar, phase);
      phase ^= 1u;
      if (wg_any(bar_id, !done)) {
        ok = false;
        break;
      }
      tc_fence_after();
      if (l < sg::kHidden) {
#pragma unroll 1
        for (int c = 0; c < 128; c += 32) {
          uint32_t v0[16], v1[16];
          tmem_ld16(tld + c, v0);
          tmem_ld16(tld + c + 16, v1);
          tmem_wait_ld();
          uint32_t hv[16];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            hv[e] = pack2(silu(__uint_as_float(v0[2 * e])), silu(__uint_as_float(v0[2 * e + 1])));
            hv[8 + e] = pack2(silu(__uint_as_float(v1[2 * e])), silu(__uint_as_float(v1[2 * e + 1])));
          }
#pragma unroll
          for (int q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(act + sg_core_off(t, c + 8 * q)) =
                make_uint4(hv[4 * q], hv[4 * q + 1], hv[4 * q + 2], hv[4 * q + 3]);
        }
      } else {
        uint32_t v[4];
        tmem_ld4(tld, v);
        tmem_wait_ld();
        for (int k = 0; k < 3; ++k) y[k] = __uint_as_float(v[k]);
      }
    }
    if (!ok) {
      if (t == 0) atomicOr(err, 2);
      break;
    }
    if (live) {
      const double t0 = sp.mean[0] + sp.scale[0] * (double)y[0], t1 = sp.mean[1] + sp.scale[1] * (double)y[1],
                   t2 = sp.mean[2] + sp.scale[2] * (double)y[2];
      // propagating mode (FinGreen3D.f90:311-322) from the per-frequency factors
      hams::cplx fg[3];
      double rk[3];
      {
        const double2 sc = pf_src;
        const double czp = pf_fld, p0 = mt.pm[1] * sc.y * czp, dp0 = mt.pm[1] * sc.x * czp;
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
      // near_flag of the pair from the coordinates and size already loaded
      const double fx = xp - xq, fy = yp - yq, fz = zp - zq;
      const int flag = sqrt(fx * fx + fy * fy + fz * fz) <= 50.0 * pf_pn ? 1 : 0;
      grn4 G = hams::finish_green(fg, xpq, ypq, zq, zp, rr, r, r1, flag);
      store_pair_v(p, i, j, G, pf_ds, pf_n1, pf_n2, pf_n3, pf_rs, pf_rd, A, S);
    }
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kCols));
}

int launch_green_sg(cudaStream_t st, int sms, DevGeom g, WaveDev w, const SgDev& sp, const hams::ModeTab& mt, double K,
                    const uint32_t* pairs, long long count, const double* rs, const double* rd, double2* A,
                    double2* S, int* err) {
  if (count <= 0) return 0;
  if (cudaFuncSetAttribute(k_green_sg, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes) != cudaSuccess)
    return 1;
  const long long tiles = (count + 127) / 128;
  const long long blocks = std::min<long long>(sms, (tiles + kWG - 1) / kWG);  // persistent: one CTA per SM
  k_green_sg<<<(unsigned)blocks, kThreads, kSmemBytes, st>>>(g, w, sp, mt, K, pairs, count, rs, rd, A, S, err);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

void pack_surrogate(const float* P, std::vector<__half>& wh, std::vector<float>& w0, std::vector<float>& bias) {
  // layer l's weights as the B operand (N = outputs, K = inputs), rows past
  // the output layer's three left zero; the layers that feed a SiLU (all but
  // the output layer) halved, so that the kernel's accumulators are z / 2
  auto scale = [](int l) { return l < sg::kLayers - 1 ? 0.5f : 1.0f; };
  wh.assign(kSgImageBytes / 2, __float2half(0.0f));
  for (int l = 1; l < sg::kLayers; ++l) {
    const int fi = sg::layer_in(l), fo = sg::layer_out(l);
    __half* dst = wh.data() + (size_t)(l - 1) * (kSgOperandBytes / 2);
    for (int o = 0; o < fo; ++o)
      for (int k = 0; k < fi; ++k)
        dst[sg_core_off(o, k) / 2] = __float2half(scale(l) * P[sg::w_off(l) + o + fo * k]);
  }
  w0.resize(sg::kWidth * sg::kIn);
  for (int e = 0; e < sg::kWidth * sg::kIn; ++e) w0[e] = scale(0) * P[sg::w_off(0) + e];
  bias.assign(kSgBias, 0.0f);
  for (int l = 0; l < sg::kLayers; ++l)
    for (int o = 0; o < sg::layer_out(l); ++o) bias[l * sg::kWidth + o] = scale(l) * P[sg::b_off(l) + o];
  // the ones block and the bias blocks of layers 1..3 and the output layer
  for (int r = 0; r < 128; ++r)
    for (int k = 0; k < 2; ++k) wh[(kSgOnesOff + sg_small_off(r, k)) / 2] = __float2half(1.0f);
  auto split = [](float x, __half& hi, __half& lo) {
    hi = __float2half_rn(x);
    lo = __float2half_rn(x - __half2float(hi));
  };
  for (int o = 0; o < sg::kWidth; ++o) {  // the first layer's block (green_sg.h)
    __half* row[16];
    for (int k = 0; k < 16; ++k) row[k] = &wh[(kSgW0Off + sg_small_off(o, k)) / 2];
    for (int k = 0; k < sg::kIn; ++k) {
      __half hi, lo;
      split(w0[o + sg::kWidth * k], hi, lo);
      *row[k] = hi;
      *row[4 + k] = hi;
      *row[8 + k] = lo;
    }
    __half hi, lo;
    split(bias[o], hi, lo);
    *row[12] = hi;
    *row[13] = lo;
  }
  for (int l = 1; l < sg::kLayers; ++l) {
    const int off = kSgBiasBlkOff + (l - 1) * kSgBiasBlkBytes;
    for (int o = 0; o < sg::layer_out(l); ++o) {
      const float b = bias[l * sg::kWidth + o];
      const __half hi = __float2half_rn(b);
      const __half lo = __float2half_rn(b - __half2float(hi));
      wh[(off + sg_small_off(o, 0)) / 2] = hi;
      wh[(off + sg_small_off(o, 1)) / 2] = lo;
    }
  }
}

// Spectral neural operator (SNO) of libcfft_b200, sm_100a: a learned warm start for the
// SCFT driver.  The reference has no learned component; the network is this library's
// own design, built on its symmetry-reduced transforms:
//
// Every activation is a real field symmetric under the plan's space group, held on the
// stride-L subgrid (M-grid) like the SCFT fields.  A Fourier layer
//   z = W v + b + S(v),  v' = gelu(z)  (identity after the last layer)
// computes S(v) = KRFFT^-1[ W_spec(class(h)) KRFFT[v](h) ] on the spectral ASU: the
// library's forward transform of the 32 channels of every sample as one batch, a real
// 32 x 32 channel matrix per retained representative h (|h_c,i| <= 11; the class of
// the sorted absolute components, shared by all cubic groups), then the backward
// transform.  The 1 x 1 channel products (W v, the projection's first layer and their
// transposes in the backward pass) run on the tensor cores: tcgen05.mma kind::f16,
// BF16 operands staged from the FP32 fields into shared memory, FP32 accumulators in
// tensor memory, with the bias, the spectral branch, gelu and its derivative fused into
// the epilogue that reads the accumulators back.
//
// Gradients: grid sums over the subgrid equal the full-grid sums divided by prod(L) for
// symmetric fields, so every pointwise gradient is taken on the subgrid, and the
// gradient of a spectral matrix is (1 / (prod(L) N^3)) sum over representatives of
// mult(h) Re(G(h) conj V(h)^T), G and V the transforms of the layer's output gradient and
// input.  The spectral branch's input gradient is KRFFT^-1[W^T KRFFT[g]].
//
// Weights: FP32 master copy, Adam, BF16 working copies (the channel and spectral
// matrices; biases stay FP32).  Every wait on the tensor-core completion barrier is
// bounded by a global-timer limit: a wait that runs out records CFFT_ERR_TIMEOUT in the
// context's status word, waits once more (bounded), frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "exec.h"
#include "sno.h"

namespace cfft {
namespace {

using bf16 = __nv_bfloat16;
using LP = SnoLayout;
constexpr int W = kSnoWidth;
constexpr int kMaxSamples = 32;  // S x 32 threads per spectral-mixing CTA
constexpr unsigned long long kSnoWaitNs = 1000000000ull;

// BF16 working copies: lift [32][21]; per layer W [32 out][32 in], W^T [32 in][32 out],
// S [364][32][32]; projection W1 [64][32], W1^T [32][64], W2 [2][64].  Every offset is a
// multiple of 8 elements (16-byte rows for the tensor-core staging).
struct BL {
  static constexpr int64_t lift = 0;
  static constexpr int64_t layer0 = 672;  // 32 * 21 rounded up to a multiple of 8 (already one)
  static constexpr int64_t lW = 0, lWT = W * W, lS = 2 * W * W;
  static constexpr int64_t lsize = 2 * W * W + int64_t(kSnoClasses) * W * W;
  static constexpr int64_t p1 = layer0 + kSnoLayers * lsize;
  static constexpr int64_t p1T = p1 + kSnoHidden * W;
  static constexpr int64_t p2 = p1T + kSnoHidden * W;
  static constexpr int64_t total = p2 + 2 * kSnoHidden;
};
static_assert(BL::layer0 % 8 == 0 && BL::lsize % 8 == 0 && BL::p1 % 8 == 0, "16-byte rows");

struct SnoPrm {
  float chiN[kMaxSamples];
  float f[kMaxSamples];
};

// ------------------------------------------------------------------------- device helpers
__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ uint64_t gtime_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok)
               : "r"(su32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = gtime_ns();
  while (!mbar_try(bar, parity))
    if (gtime_ns() - t0 > limit_ns) return false;
  return true;
}

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8 rows x 16
// bytes stored contiguously; lbo = byte step between core matrices along K, sbo = byte
// step between 8-row groups; version field 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(su32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// 32 consecutive FP32 accumulator columns of this warp's 32 lanes (one row per thread).
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------------------- tensor-core channel product
enum Epi : int {
  kEpiGelu = 0,       // z = acc + b + add -> out0 = z, out1 = gelu(z)
  kEpiLinear = 1,     // out1 = acc + b + add
  kEpiProjTrain = 2,  // hp = acc + b -> out0 = hp; out1 = W2 gelu(hp) + b2 (2 channels)
  kEpiProjInfer = 3,  // as kEpiProjTrain, out1 = [w_A | w_B] = homogeneous + chiN * output
  kEpiBwdGelu = 4,    // out0 = (acc + add) * gelu'(zprev)
  kEpiBwdLinear = 5,  // out0 = acc + add (add may be null)
};

struct GemmArgs {
  const float* X;      // A source: S x K x P (FP32)
  const bf16* B;       // N x K, K contiguous (BF16)
  int P, S, tiles;     // P a multiple of 128; tiles = S * P / 128
  const float* bias;   // N (kEpiGelu, kEpiLinear, kEpiProj*)
  const float* add;    // S x N x P (kEpiGelu, kEpiLinear, kEpiBwd*)
  const float* zprev;  // S x N x P (kEpiBwdGelu)
  float* out0;
  float* out1;
  const bf16* w2;      // 2 x 64 BF16 (kEpiProj*)
  const float* b2;     // 2
  SnoPrm prm;
  int* status;
};

template <int K, int N>
struct GemmSmem {
  static constexpr int a_bytes = 128 * K * 2;
  static constexpr int b_bytes = N * K * 2;
  static constexpr int sbo = (K / 8) * 128;  // bytes between 8-row groups (A and B)
  static constexpr int bytes = a_bytes + b_bytes + 64;
};

template <int K, int N, int EPI>
__global__ void __launch_bounds__(128) k_sno_gemm(GemmArgs a) {
  static_assert(K % 16 == 0 && (N == 32 || N == 64), "tile shape");
  using SM = GemmSmem<K, N>;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + SM::a_bytes;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + SM::a_bytes + SM::b_bytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  int* abort_flag = reinterpret_cast<int*>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(su32(tslot)), "r"(N)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(su32(bar)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *abort_flag = 0;
  }
  // B operand: row n, 16-byte chunk kg of 8 K values -> core matrix (n / 8, kg)
  for (int c = tid; c < N * (K / 8); c += 128) {
    const int n = c / (K / 8), kg = c % (K / 8);
    const uint4 v = *reinterpret_cast<const uint4*>(a.B + static_cast<size_t>(n) * K + kg * 8);
    *reinterpret_cast<uint4*>(sB + (n >> 3) * SM::sbo + kg * 128 + (n & 7) * 16) = v;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t aaddr = su32(sA), baddr = su32(sB);
  constexpr uint32_t idesc = idesc_bf16(128, N);
  const int tiles_per_sample = a.P / 128;
  uint32_t phase = 0;

  for (int tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
    const int s = tile / tiles_per_sample;
    const int p0 = (tile % tiles_per_sample) * 128;
    // A operand: thread = row (point p0 + tid); 8 channels per 16-byte chunk
    const float* xs = a.X + static_cast<size_t>(s) * K * a.P + p0 + tid;
#pragma unroll
    for (int kg = 0; kg < K / 8; ++kg) {
      float v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = __ldg(xs + static_cast<size_t>(kg * 8 + j) * a.P);
      uint4 pk;
      __nv_bfloat162 h0 = __floats2bfloat162_rn(v[0], v[1]), h1 = __floats2bfloat162_rn(v[2], v[3]);
      __nv_bfloat162 h2 = __floats2bfloat162_rn(v[4], v[5]), h3 = __floats2bfloat162_rn(v[6], v[7]);
      pk.x = *reinterpret_cast<uint32_t*>(&h0);
      pk.y = *reinterpret_cast<uint32_t*>(&h1);
      pk.z = *reinterpret_cast<uint32_t*>(&h2);
      pk.w = *reinterpret_cast<uint32_t*>(&h3);
      *reinterpret_cast<uint4*>(sA + (tid >> 3) * SM::sbo + kg * 128 + (tid & 7) * 16) = pk;
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kk = 0; kk < K / 16; ++kk) {
        const uint64_t da = smem_desc(aaddr + kk * 256, 128, SM::sbo);
        const uint64_t db = smem_desc(baddr + kk * 256, 128, SM::sbo);
        tc_mma(tmem, da, db, idesc, kk > 0 ? 1u : 0u);
      }
      tc_commit(bar);
      if (!mbar_wait_ns(bar, phase, kSnoWaitNs)) {
        if (a.status) atomicExch(a.status, 5);
        mbar_wait_ns(bar, phase, kSnoWaitNs);
        *abort_flag = 1;
      }
    }
    __syncthreads();
    if (*abort_flag) break;
    mbar_try(bar, phase);  // every thread observes the completed phase
    phase ^= 1u;
    tc_fence_after();

    // epilogue: row p = p0 + 32 warp + lane reads its accumulators 32 columns at a time
    // (at most 32 accumulator registers live) and applies the fused operations
    const int p = p0 + warp * 32 + lane;
    const size_t base = static_cast<size_t>(s) * N * a.P + p;
    float o0 = 0.f, o1 = 0.f;
    if constexpr (EPI == kEpiProjTrain || EPI == kEpiProjInfer) {
      o0 = __ldg(a.b2);
      o1 = __ldg(a.b2 + 1);
    }
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 32) {
      float acc[32];
      tc_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, acc);
      if constexpr (EPI == kEpiGelu || EPI == kEpiLinear) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int c = c0 + i;
          const size_t o = base + static_cast<size_t>(c) * a.P;
          const float z = acc[i] + __ldg(a.bias + c) + __ldg(a.add + o);
          if constexpr (EPI == kEpiGelu) {
            a.out0[o] = z;
            a.out1[o] = gelu_f(z);
          } else {
            a.out1[o] = z;
          }
        }
      } else if constexpr (EPI == kEpiProjTrain || EPI == kEpiProjInfer) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int c = c0 + i;
          const float hp = acc[i] + __ldg(a.bias + c);
          if constexpr (EPI == kEpiProjTrain) a.out0[base + static_cast<size_t>(c) * a.P] = hp;
          const float h = gelu_f(hp);
          o0 = fmaf(__bfloat162float(a.w2[c]), h, o0);
          o1 = fmaf(__bfloat162float(a.w2[N + c]), h, o1);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const size_t o = base + static_cast<size_t>(c0 + i) * a.P;
          float g = acc[i] + (a.add ? __ldg(a.add + o) : 0.0f);
          if constexpr (EPI == kEpiBwdGelu) g *= gelu_grad_f(__ldg(a.zprev + o));
          a.out0[o] = g;
        }
      }
    }
    if constexpr (EPI == kEpiProjTrain || EPI == kEpiProjInfer) {
      const size_t ob = static_cast<size_t>(s) * 2 * a.P + p;
      if constexpr (EPI == kEpiProjTrain) {
        a.out1[ob] = o0;
        a.out1[ob + a.P] = o1;
      } else {
        const float chiN = a.prm.chiN[s], f = a.prm.f[s];
        a.out1[ob] = chiN * (1.0f - f) + chiN * o0;
        a.out1[ob + a.P] = chiN * f + chiN * o1;
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(N) : "memory");
  }
}

// ------------------------------------------------------------------------- other kernels
// Plane-wave features (cos, sin per reflection) on the M-grid: (1/|G|) sum_g of
// cos/sin(2 pi (h . (R_g x + t_g) / N + h . shift)), x = L o n, (R_g, t_g) the shifted
// operations in grid units (equal to the unshifted operations at x / N + shift).
__global__ void k_sno_features(const int* __restrict__ ops, int n_ops, int N, int L0, int L1, int L2, int M0, int M1,
                               int P, double s0, double s1, double s2, float* __restrict__ feat) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int n0 = p % M0, n1 = (p / M0) % M1, n2 = p / (M0 * M1);
  const long x0 = static_cast<long>(n0) * L0, x1 = static_cast<long>(n1) * L1, x2 = static_cast<long>(n2) * L2;
  const int H[kSnoRefl][3] = {{1, 0, 0}, {1, 1, 0}, {1, 1, 1}, {2, 0, 0}, {2, 1, 0}, {2, 1, 1}, {2, 2, 0}, {3, 1, 0}};
  for (int j = 0; j < kSnoRefl; ++j) {
    double c = 0.0, sn = 0.0;
    const double hs = H[j][0] * s0 + H[j][1] * s1 + H[j][2] * s2;
    for (int g = 0; g < n_ops; ++g) {
      const int* o = ops + 12 * g;
      const long y0 = o[0] * x0 + o[1] * x1 + o[2] * x2 + o[9];
      const long y1 = o[3] * x0 + o[4] * x1 + o[5] * x2 + o[10];
      const long y2 = o[6] * x0 + o[7] * x1 + o[8] * x2 + o[11];
      const long num = H[j][0] * y0 + H[j][1] * y1 + H[j][2] * y2;
      const long r = ((num % N) + N) % N;  // the phase is periodic in num with period N
      double sv, cv;
      sincospi(2.0 * (static_cast<double>(r) / N + hs), &sv, &cv);
      c += cv;
      sn += sv;
    }
    feat[static_cast<size_t>(2 * j) * P + p] = static_cast<float>(c / n_ops);
    feat[static_cast<size_t>(2 * j + 1) * P + p] = static_cast<float>(sn / n_ops);
  }
}

__device__ __forceinline__ void sample_consts(const SnoPrm& prm, int s, int slot, float* a) {
  a[0] = (prm.chiN[s] - 21.0f) / 9.0f;
  a[1] = (prm.f[s] - 0.4f) / 0.1f;
  a[2] = slot == 0 ? 1.0f : 0.0f;
  a[3] = slot == 1 ? 1.0f : 0.0f;
  a[4] = slot == 2 ? 1.0f : 0.0f;
}

// v0 = W_lift a + b_lift (thread per point and sample).
__global__ void __launch_bounds__(256) k_sno_lift(const float* __restrict__ feat, SnoPrm prm, int slot,
                                                  const bf16* __restrict__ Wl, const float* __restrict__ bl, int P,
                                                  int S, float* __restrict__ v0) {
  __shared__ float ws[W][kSnoCin];
  __shared__ float bs[W];
  for (int e = threadIdx.x; e < W * kSnoCin; e += blockDim.x) ws[e / kSnoCin][e % kSnoCin] = __bfloat162float(Wl[e]);
  for (int e = threadIdx.x; e < W; e += blockDim.x) bs[e] = bl[e];
  __syncthreads();
  const size_t total = static_cast<size_t>(S) * P;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int s = static_cast<int>(i / P), p = static_cast<int>(i % P);
    float a[kSnoCin];
    sample_consts(prm, s, slot, a);
#pragma unroll
    for (int j = 0; j < 2 * kSnoRefl; ++j) a[5 + j] = __ldg(feat + static_cast<size_t>(j) * P + p);
    float* out = v0 + static_cast<size_t>(s) * W * P + p;
#pragma unroll 4
    for (int o = 0; o < W; ++o) {
      float acc = bs[o];
#pragma unroll
      for (int j = 0; j < kSnoCin; ++j) acc = fmaf(ws[o][j], a[j], acc);
      out[static_cast<size_t>(o) * P] = acc;
    }
  }
}

// Spectral mixing at the retained representatives (one CTA per representative, thread
// (sample, channel)): Y(h) = W_spec[class] F(h); F(h) is also kept (Vret) for the
// gradient.  Non-retained entries of Y stay zero.
__global__ void k_sno_specmix_fwd(const float2* __restrict__ F, int n_spec, const int* __restrict__ ret_spec,
                                  const int* __restrict__ ret_cls, const bf16* __restrict__ Sw,
                                  float2* __restrict__ Y, float2* __restrict__ Vret) {
  __shared__ float ws[W][W + 1];
  __shared__ float2 fc[kMaxSamples * W];
  const int r = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const int spec = ret_spec[r], cls = ret_cls[r];
  for (int e = tid; e < W * W; e += nt) ws[e / W][e % W] = __bfloat162float(Sw[static_cast<size_t>(cls) * W * W + e]);
  const float2 v = F[static_cast<size_t>(tid) * n_spec + spec];
  fc[tid] = v;
  Vret[static_cast<size_t>(r) * nt + tid] = v;
  __syncthreads();
  const int s = tid / W, o = tid % W;
  float2 y = make_float2(0.f, 0.f);
#pragma unroll 8
  for (int i = 0; i < W; ++i) {
    const float w = ws[o][i];
    const float2 x = fc[s * W + i];
    y.x = fmaf(w, x.x, y.x);
    y.y = fmaf(w, x.y, y.y);
  }
  Y[static_cast<size_t>(s * W + o) * n_spec + spec] = y;
}

// Backward of the spectral mixing: Y(h) = W_spec[class]^T G(h), and
// dW_spec[class][o][i] += wt * sum_s Re(G_o conj V_i), wt = mult / (prod(L) N^3).
__global__ void k_sno_specmix_bwd(const float2* __restrict__ G, int n_spec, const int* __restrict__ ret_spec,
                                  const int* __restrict__ ret_cls, const float* __restrict__ ret_wt,
                                  const bf16* __restrict__ Sw, const float2* __restrict__ Vret,
                                  float2* __restrict__ Y, float* __restrict__ dS) {
  __shared__ float ws[W][W + 1];
  __shared__ float2 gc[kMaxSamples * W];
  __shared__ float2 vc[kMaxSamples * W];
  const int r = blockIdx.x, tid = threadIdx.x, nt = blockDim.x, S = nt / W;
  const int spec = ret_spec[r], cls = ret_cls[r];
  for (int e = tid; e < W * W; e += nt) ws[e / W][e % W] = __bfloat162float(Sw[static_cast<size_t>(cls) * W * W + e]);
  gc[tid] = G[static_cast<size_t>(tid) * n_spec + spec];
  vc[tid] = Vret[static_cast<size_t>(r) * nt + tid];
  __syncthreads();
  const int s = tid / W, i = tid % W;
  float2 y = make_float2(0.f, 0.f);
#pragma unroll 8
  for (int o = 0; o < W; ++o) {
    const float w = ws[o][i];
    const float2 g = gc[s * W + o];
    y.x = fmaf(w, g.x, y.x);
    y.y = fmaf(w, g.y, y.y);
  }
  Y[static_cast<size_t>(s * W + i) * n_spec + spec] = y;
  const float wt = ret_wt[r];
  for (int e = tid; e < W * W; e += nt) {
    const int o = e / W, ii = e % W;
    float acc = 0.f;
    for (int q = 0; q < S; ++q) {
      const float2 g = gc[q * W + o], v = vc[q * W + ii];
      acc = fmaf(g.x, v.x, fmaf(g.y, v.y, acc));
    }
    atomicAdd(dS + static_cast<size_t>(cls) * W * W + e, wt * acc);
  }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Loss and the first backward steps of the projection, thread per point and sample:
// t = (w_target - homogeneous) / chiN, e = out - t, loss += sum e^2 (FP64 partials),
// g = 2 e / (S 2 P); dW2 += g h^T, db2 += g (warp sums, then shared and global atomics);
// ghp = (W2^T g) * gelu'(hp).
__global__ void __launch_bounds__(256) k_sno_loss(const float* __restrict__ out, const float* __restrict__ wt,
                                                  const float* __restrict__ hp, SnoPrm prm,
                                                  const bf16* __restrict__ W2b, int P, int S,
                                                  float* __restrict__ ghp, float* __restrict__ dW2,
                                                  float* __restrict__ db2, double* __restrict__ loss_part) {
  __shared__ float w2[2][kSnoHidden];
  __shared__ float acc[2 * kSnoHidden + 2];
  __shared__ double lsum;
  const int tid = threadIdx.x;
  for (int e = tid; e < 2 * kSnoHidden; e += blockDim.x) w2[e / kSnoHidden][e % kSnoHidden] = __bfloat162float(W2b[e]);
  for (int e = tid; e < 2 * kSnoHidden + 2; e += blockDim.x) acc[e] = 0.f;
  if (tid == 0) lsum = 0.0;
  __syncthreads();
  const float scale = 2.0f / (static_cast<float>(S) * 2.0f * static_cast<float>(P));
  const size_t total = static_cast<size_t>(S) * P;  // a multiple of 128: every warp is full
  double lacc = 0.0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + tid; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int s = static_cast<int>(i / P), p = static_cast<int>(i % P);
    const float chiN = prm.chiN[s], f = prm.f[s];
    const size_t ob = static_cast<size_t>(s) * 2 * P + p;
    const float t0 = (wt[ob] - chiN * (1.0f - f)) / chiN, t1 = (wt[ob + P] - chiN * f) / chiN;
    const float e0 = out[ob] - t0, e1 = out[ob + P] - t1;
    lacc += static_cast<double>(e0) * e0 + static_cast<double>(e1) * e1;
    const float g0 = scale * e0, g1 = scale * e1;
    const float s0 = warp_sum(g0), s1 = warp_sum(g1);
    if ((tid & 31) == 0) {
      atomicAdd(&acc[2 * kSnoHidden], s0);
      atomicAdd(&acc[2 * kSnoHidden + 1], s1);
    }
    const size_t hb = static_cast<size_t>(s) * kSnoHidden * P + p;
    for (int j = 0; j < kSnoHidden; ++j) {
      const float x = hp[hb + static_cast<size_t>(j) * P];
      const float h = gelu_f(x);
      const float a0 = warp_sum(g0 * h), a1 = warp_sum(g1 * h);
      if ((tid & 31) == 0) {
        atomicAdd(&acc[j], a0);
        atomicAdd(&acc[kSnoHidden + j], a1);
      }
      ghp[hb + static_cast<size_t>(j) * P] = (w2[0][j] * g0 + w2[1][j] * g1) * gelu_grad_f(x);
    }
  }
  atomicAdd(&lsum, lacc);
  __syncthreads();
  for (int e = tid; e < 2 * kSnoHidden; e += blockDim.x) atomicAdd(dW2 + e, acc[e]);
  if (tid < 2) atomicAdd(db2 + tid, acc[2 * kSnoHidden + tid]);
  if (tid == 0) loss_part[blockIdx.x] = lsum;
}

// dW[o][i] += sum_{s,p} G[s][o][p] X[s][i][p] (X sample stride xs, 0 for shared
// features) and gsum[s][o] += sum_p G[s][o][p].  256 threads as 16 x 16, each owning an
// (CO/16) x (CI/16) block; tiles of 64 points of one sample staged in shared memory.
template <int CO, int CI>
__global__ void __launch_bounds__(256) k_sno_wgrad(const float* __restrict__ G, const float* __restrict__ X,
                                                   size_t xs, int P, int S, float* __restrict__ dW,
                                                   float* __restrict__ gsum) {
  constexpr int TP = 64, BO = CO / 16, BI = CI / 16;
  __shared__ float gt[CO][TP + 1];
  __shared__ float xt[CI][TP + 1];
  const int tid = threadIdx.x, to = tid / 16, ti = tid % 16;
  float acc[BO][BI] = {};
  const int tps = P / TP;
  for (int tile = blockIdx.x; tile < S * tps; tile += gridDim.x) {
    const int s = tile / tps, p0 = (tile % tps) * TP;
    for (int e = tid; e < CO * TP; e += 256)
      gt[e / TP][e % TP] = G[(static_cast<size_t>(s) * CO + e / TP) * P + p0 + e % TP];
    for (int e = tid; e < CI * TP; e += 256)
      xt[e / TP][e % TP] = X[s * xs + static_cast<size_t>(e / TP) * P + p0 + e % TP];
    __syncthreads();
    if (gsum && tid < CO) {
      float t = 0.f;
      for (int q = 0; q < TP; ++q) t += gt[tid][q];
      atomicAdd(gsum + static_cast<size_t>(s) * CO + tid, t);
    }
#pragma unroll 4
    for (int q = 0; q < TP; ++q) {
      float gv[BO], xv[BI];
#pragma unroll
      for (int a = 0; a < BO; ++a) gv[a] = gt[to + 16 * a][q];
#pragma unroll
      for (int b = 0; b < BI; ++b) xv[b] = xt[ti + 16 * b][q];
#pragma unroll
      for (int a = 0; a < BO; ++a)
#pragma unroll
        for (int b = 0; b < BI; ++b) acc[a][b] = fmaf(gv[a], xv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < BO; ++a)
#pragma unroll
    for (int b = 0; b < BI; ++b) atomicAdd(dW + (to + 16 * a) * CI + ti + 16 * b, acc[a][b]);
}

// Bias gradients from the per-sample channel sums, and the lift's constant channels:
// db[o] = sum_s gsum[s][o]; lift: dW_lift[o][j] = sum_s a_j(s) gsum[s][o], j < 5.
__global__ void k_sno_bias_grads(const float* __restrict__ gsum, int S, int CO, float* __restrict__ db,
                                 float* __restrict__ dW_lift_const, SnoPrm prm, int slot) {
  const int o = threadIdx.x;
  if (o >= CO) return;
  float b = 0.f, c[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int s = 0; s < S; ++s) {
    const float g = gsum[static_cast<size_t>(s) * CO + o];
    b += g;
    if (dW_lift_const) {
      float a[5];
      sample_consts(prm, s, slot, a);
      for (int j = 0; j < 5; ++j) c[j] += a[j] * g;
    }
  }
  db[o] += b;
  if (dW_lift_const)
    for (int j = 0; j < 5; ++j) dW_lift_const[o * kSnoCin + j] += c[j];
}

__global__ void k_sno_sum(const double* __restrict__ part, int n, double* __restrict__ out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) v += part[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) *out = v;
}

// Adam (decoupled weight decay) on the FP32 master copy.
__global__ void k_sno_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float wd,
                           float c1, float c2) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * w[i]);
  }
}

// Master index of BF16 working-copy element j (transposes included).
__device__ __forceinline__ int64_t bf_source(int64_t j) {
  if (j < BL::layer0) return LP::lift_W + j;
  if (j < BL::p1) {
    const int64_t l = (j - BL::layer0) / BL::lsize, r = (j - BL::layer0) % BL::lsize;
    const int64_t base = LP::layer0 + l * LP::layer_size;
    if (r < BL::lWT) return base + LP::layer_W + r;
    if (r < BL::lS) {
      const int64_t q = r - BL::lWT, i = q / W, o = q % W;  // W^T[i][o] = W[o][i]
      return base + LP::layer_W + o * W + i;
    }
    return base + LP::layer_S + (r - BL::lS);
  }
  if (j < BL::p1T) return LP::p1_W + (j - BL::p1);
  if (j < BL::p2) {
    const int64_t q = j - BL::p1T, i = q / kSnoHidden, h = q % kSnoHidden;  // W1^T[i][h] = W1[h][i]
    return LP::p1_W + h * W + i;
  }
  return LP::p2_W + (j - BL::p2);
}

__global__ void k_sno_to_bf16(const float* __restrict__ w, bf16* __restrict__ wb) {
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < BL::total;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x)
    wb[j] = __float2bfloat16_rn(w[bf_source(j)]);
}

// dW_lift[o][5 + j] += dfeat[o][j] (the feature block of the lift gradient).
__global__ void k_sno_scatter_lift(const float* __restrict__ dfeat, float* __restrict__ dW_lift) {
  const int e = threadIdx.x;
  if (e >= W * 2 * kSnoRefl) return;
  const int o = e / (2 * kSnoRefl), j = e % (2 * kSnoRefl);
  dW_lift[o * kSnoCin + 5 + j] += dfeat[e];
}

#define SNO_CUDA(expr, what)                                                   \
  do {                                                                         \
    cudaError_t e_ = (expr);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      *err = std::string(what) + ": " + cudaGetErrorString(e_);               \
      return e_ == cudaErrorMemoryAllocation ? Status::kAlloc : Status::kCuda; \
    }                                                                          \
  } while (0)

int grid_for(size_t n, int threads, int cap = 148 * 8) {
  return static_cast<int>(std::max<size_t>(1, std::min<size_t>((n + threads - 1) / threads, cap)));
}

// splitmix64 uniform in [0, 1)
double uniform01(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

struct SnoModel {
  SnoConfig cfg;
  float* w = nullptr;  // FP32 master
  float* g = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  bf16* wb = nullptr;
  int64_t t = 0;  // Adam steps taken
};

struct SnoCtx {
  SnoModel* model = nullptr;
  Plan* plan = nullptr;
  int slot = 0, S = 0, P = 0, n_spec = 0, n_ret = 0;
  int* ret_spec = nullptr;
  int* ret_cls = nullptr;
  float* ret_wt = nullptr;
  float* feat = nullptr;
  float* v[kSnoLayers + 1] = {};
  float* z[kSnoLayers - 1] = {};
  float* sbuf = nullptr;
  float* hp = nullptr;
  float* out = nullptr;
  float* gz[2] = {};
  float* ghp = nullptr;
  float2* F = nullptr;
  float2* Y = nullptr;
  float2* Vret = nullptr;  // layers x n_ret x S * 32
  float* gsum = nullptr;   // S x 64
  float* dfeat = nullptr;  // 32 x 16: feature block of the lift gradient
  double* loss_part = nullptr;
  double* loss = nullptr;
  int* status = nullptr;
  std::vector<void*> owned;
};

Status sno_model_create(const SnoConfig& cfg, SnoModel** out, std::string* err) {
  auto* m = new SnoModel();
  m->cfg = cfg;
  const size_t nb = LP::total * sizeof(float);
  cudaError_t e = cudaMalloc(&m->w, nb);
  if (e == cudaSuccess) e = cudaMalloc(&m->g, nb);
  if (e == cudaSuccess) e = cudaMalloc(&m->m, nb);
  if (e == cudaSuccess) e = cudaMalloc(&m->v, nb);
  if (e == cudaSuccess) e = cudaMalloc(&m->wb, BL::total * sizeof(bf16));
  if (e == cudaSuccess) e = cudaMemset(m->g, 0, nb);
  if (e == cudaSuccess) e = cudaMemset(m->m, 0, nb);
  if (e == cudaSuccess) e = cudaMemset(m->v, 0, nb);
  if (e != cudaSuccess) {
    *err = std::string("SNO model allocation: ") + cudaGetErrorString(e);
    sno_model_destroy(m);
    return e == cudaErrorMemoryAllocation ? Status::kAlloc : Status::kCuda;
  }
  // seeded initial weights: channel maps uniform in +-1/sqrt(fan_in), spectral matrices
  // uniform in [0, 4 / 32^2)
  std::vector<float> h(LP::total);
  uint64_t st = 0x5EED5EEDull;
  auto lin = [&](int64_t off_w, int64_t off_b, int o, int i) {
    const double b = 1.0 / std::sqrt(static_cast<double>(i));
    for (int64_t k = 0; k < int64_t(o) * i; ++k) h[off_w + k] = static_cast<float>((2.0 * uniform01(&st) - 1.0) * b);
    for (int k = 0; k < o; ++k) h[off_b + k] = static_cast<float>((2.0 * uniform01(&st) - 1.0) * b);
  };
  lin(LP::lift_W, LP::lift_b, W, kSnoCin);
  for (int l = 0; l < kSnoLayers; ++l) {
    const int64_t base = LP::layer0 + l * LP::layer_size;
    lin(base + LP::layer_W, base + LP::layer_b, W, W);
    for (int64_t k = 0; k < int64_t(kSnoClasses) * W * W; ++k)
      h[base + LP::layer_S + k] = static_cast<float>(uniform01(&st) * 4.0 / (W * W));
  }
  lin(LP::p1_W, LP::p1_b, kSnoHidden, W);
  lin(LP::p2_W, LP::p2_b, 2, kSnoHidden);
  *out = m;
  return sno_set_params(m, h.data(), err);
}

void sno_model_destroy(SnoModel* m) {
  if (!m) return;
  cudaFree(m->w);
  cudaFree(m->g);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->wb);
  delete m;
}

Status sno_set_params(SnoModel* m, const float* host, std::string* err) {
  SNO_CUDA(cudaMemcpy(m->w, host, LP::total * sizeof(float), cudaMemcpyHostToDevice), "SNO parameter upload");
  k_sno_to_bf16<<<grid_for(BL::total, 256), 256>>>(m->w, m->wb);
  add_launches(1);
  SNO_CUDA(cudaGetLastError(), "SNO weight conversion launch");
  SNO_CUDA(cudaDeviceSynchronize(), "SNO weight conversion");
  return Status::kOk;
}

Status sno_get_params(const SnoModel* m, float* host, std::string* err) {
  SNO_CUDA(cudaMemcpy(host, m->w, LP::total * sizeof(float), cudaMemcpyDeviceToHost), "SNO parameter download");
  return Status::kOk;
}

Status sno_get_grads(const SnoModel* m, float* host, std::string* err) {
  SNO_CUDA(cudaMemcpy(host, m->g, LP::total * sizeof(float), cudaMemcpyDeviceToHost), "SNO gradient download");
  return Status::kOk;
}

void sno_unbind(SnoCtx* c) {
  if (!c) return;
  for (void* p : c->owned) cudaFree(p);
  delete c;
}

Status sno_bind(SnoModel* m, Plan* p, int group_slot, const double* shift, int max_samples, SnoCtx** out,
                std::string* err) {
  const PlanTables& T = p->T;
  if (!p->d_geom) { *err = "the SNO needs a device plan"; return Status::kInvalid; }
  if (p->precision != 4) { *err = "the SNO runs on FP32 plans"; return Status::kUnsupported; }
  if (T.dim != 3 || T.N[0] != T.N[1] || T.N[0] != T.N[2]) { *err = "the SNO needs a cubic 3-D grid"; return Status::kUnsupported; }
  if (group_slot < 0 || group_slot >= kSnoGroups) { *err = "group_slot must be 0, 1 or 2"; return Status::kInvalid; }
  if (max_samples < 1 || max_samples > kMaxSamples) { *err = "max_samples must be 1..32"; return Status::kInvalid; }
  if (p->max_batch < W * max_samples) { *err = "the plan's max_batch must be at least 32 * max_samples"; return Status::kInvalid; }
  const int P = T.M[0] * T.M[1] * T.M[2];
  if (P % 128 != 0) { *err = "the SNO needs M1 M2 M3 to be a multiple of 128"; return Status::kUnsupported; }
  auto* c = new SnoCtx();
  c->model = m;
  c->plan = p;
  c->slot = group_slot;
  c->S = max_samples;
  c->P = P;
  c->n_spec = static_cast<int>(T.spec.size());
  // retained representatives and their classes
  int tab[kSnoModes][kSnoModes][kSnoModes];
  int k = 0;
  for (int a = 0; a < kSnoModes; ++a)
    for (int b = 0; b <= a; ++b)
      for (int cc = 0; cc <= b; ++cc) tab[a][b][cc] = k++;
  std::vector<int> rs, rc;
  std::vector<float> rw;
  const double N3 = static_cast<double>(T.N[0]) * T.N[1] * T.N[2];
  for (int i = 0; i < c->n_spec; ++i) {
    int hc[3];
    get_k_vector(T.spec[i], T.N, hc);
    int s3[3] = {std::abs(hc[0]), std::abs(hc[1]), std::abs(hc[2])};
    std::sort(s3, s3 + 3, [](int x, int y) { return x > y; });
    if (s3[0] >= kSnoModes) continue;
    rs.push_back(i);
    rc.push_back(tab[s3[0]][s3[1]][s3[2]]);
    rw.push_back(static_cast<float>(T.spec[i].mult / (static_cast<double>(T.d) * N3)));
  }
  c->n_ret = static_cast<int>(rs.size());
  const size_t S = static_cast<size_t>(max_samples), Pz = static_cast<size_t>(P);
  auto alloc = [&](void** ptr, size_t bytes) -> bool {
    if (cudaMalloc(ptr, std::max<size_t>(bytes, 16)) != cudaSuccess) return false;
    c->owned.push_back(*ptr);
    return true;
  };
  bool ok = alloc(reinterpret_cast<void**>(&c->ret_spec), rs.size() * 4) &&
            alloc(reinterpret_cast<void**>(&c->ret_cls), rs.size() * 4) &&
            alloc(reinterpret_cast<void**>(&c->ret_wt), rs.size() * 4) &&
            alloc(reinterpret_cast<void**>(&c->feat), 2 * kSnoRefl * Pz * 4);
  for (int l = 0; ok && l <= kSnoLayers; ++l) ok = alloc(reinterpret_cast<void**>(&c->v[l]), S * W * Pz * 4);
  for (int l = 0; ok && l < kSnoLayers - 1; ++l) ok = alloc(reinterpret_cast<void**>(&c->z[l]), S * W * Pz * 4);
  ok = ok && alloc(reinterpret_cast<void**>(&c->sbuf), S * W * Pz * 4) &&
       alloc(reinterpret_cast<void**>(&c->hp), S * kSnoHidden * Pz * 4) &&
       alloc(reinterpret_cast<void**>(&c->out), S * 2 * Pz * 4) &&
       alloc(reinterpret_cast<void**>(&c->gz[0]), S * W * Pz * 4) &&
       alloc(reinterpret_cast<void**>(&c->gz[1]), S * W * Pz * 4) &&
       alloc(reinterpret_cast<void**>(&c->ghp), S * kSnoHidden * Pz * 4) &&
       alloc(reinterpret_cast<void**>(&c->F), S * W * c->n_spec * sizeof(float2)) &&
       alloc(reinterpret_cast<void**>(&c->Y), S * W * c->n_spec * sizeof(float2)) &&
       alloc(reinterpret_cast<void**>(&c->Vret), kSnoLayers * rs.size() * S * W * sizeof(float2)) &&
       alloc(reinterpret_cast<void**>(&c->gsum), S * kSnoHidden * 4) &&
       alloc(reinterpret_cast<void**>(&c->dfeat), W * 2 * kSnoRefl * 4) &&
       alloc(reinterpret_cast<void**>(&c->loss_part), 148 * 8 * sizeof(double)) &&
       alloc(reinterpret_cast<void**>(&c->loss), sizeof(double)) &&
       alloc(reinterpret_cast<void**>(&c->status), sizeof(int));
  if (!ok) {
    *err = "SNO context allocation failed";
    sno_unbind(c);
    return Status::kAlloc;
  }
  cudaError_t e = cudaMemcpy(c->ret_spec, rs.data(), rs.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->ret_cls, rc.data(), rc.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->ret_wt, rw.data(), rw.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->Y, 0, S * W * c->n_spec * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemset(c->status, 0, sizeof(int));
  // features from the shifted operations
  std::vector<int> ops(12 * T.ops.size());
  for (size_t g = 0; g < T.ops.size(); ++g) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) ops[12 * g + 3 * i + j] = T.ops[g].R[i][j];
    for (int i = 0; i < 3; ++i) ops[12 * g + 9 + i] = T.ops[g].t[i];
  }
  int* d_ops = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&d_ops, ops.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(d_ops, ops.data(), ops.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_sno_features<<<(P + 127) / 128, 128>>>(d_ops, static_cast<int>(T.ops.size()), T.N[0], T.L[0], T.L[1], T.L[2],
                                             T.M[0], T.M[1], P, shift[0], shift[1], shift[2], c->feat);
    add_launches(1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (d_ops) cudaFree(d_ops);
  if (e != cudaSuccess) {
    *err = std::string("SNO bind: ") + cudaGetErrorString(e);
    sno_unbind(c);
    return Status::kCuda;
  }
  *out = c;
  return Status::kOk;
}

namespace {

template <int K, int N, int EPI>
Status launch_gemm(const GemmArgs& a0, cudaStream_t st, std::string* err) {
  GemmArgs a = a0;
  a.tiles = a.S * (a.P / 128);
  const int smem = GemmSmem<K, N>::bytes;
  const int per_sm = N == 64 ? 8 : 16;  // tensor-memory columns: 512 per SM
  const int grid = std::max(1, std::min(a.tiles, 148 * per_sm));
  k_sno_gemm<K, N, EPI><<<grid, 128, smem, st>>>(a);
  add_launches(1);
  SNO_CUDA(cudaGetLastError(), "SNO tensor-core product launch");
  return Status::kOk;
}

Status forward_t(SnoCtx* c, const SnoPrm& prm, int S, bool train, void* w_out, cudaStream_t st, std::string* err) {
  SnoModel* m = c->model;
  const int P = c->P;
  Status s;
  k_sno_lift<<<grid_for(static_cast<size_t>(S) * P, 256), 256, 0, st>>>(c->feat, prm, c->slot, m->wb + BL::lift,
                                                                          m->w + LP::lift_b, P, S, c->v[0]);
  add_launches(1);
  SNO_CUDA(cudaGetLastError(), "SNO lift launch");
  for (int l = 0; l < kSnoLayers; ++l) {
    if ((s = exec_forward(c->plan, c->v[l], c->F, S * W, st, err)) != Status::kOk) return s;
    if (c->n_ret > 0) {
      k_sno_specmix_fwd<<<c->n_ret, S * W, 0, st>>>(c->F, c->n_spec, c->ret_spec, c->ret_cls,
                                                    m->wb + BL::layer0 + l * BL::lsize + BL::lS, c->Y,
                                                    c->Vret + static_cast<size_t>(l) * c->n_ret * S * W);
      add_launches(1);
      SNO_CUDA(cudaGetLastError(), "SNO spectral mixing launch");
    }
    if ((s = exec_backward(c->plan, c->Y, c->sbuf, S * W, st, err)) != Status::kOk) return s;
    GemmArgs a{};
    a.X = c->v[l];
    a.B = m->wb + BL::layer0 + l * BL::lsize + BL::lW;
    a.P = P;
    a.S = S;
    a.bias = m->w + LP::layer0 + l * LP::layer_size + LP::layer_b;
    a.add = c->sbuf;
    a.status = c->status;
    if (l < kSnoLayers - 1) {
      a.out0 = c->z[l];
      a.out1 = c->v[l + 1];
      s = launch_gemm<32, 32, kEpiGelu>(a, st, err);
    } else {
      a.out1 = c->v[l + 1];
      s = launch_gemm<32, 32, kEpiLinear>(a, st, err);
    }
    if (s != Status::kOk) return s;
  }
  GemmArgs a{};
  a.X = c->v[kSnoLayers];
  a.B = m->wb + BL::p1;
  a.P = P;
  a.S = S;
  a.bias = m->w + LP::p1_b;
  a.w2 = m->wb + BL::p2;
  a.b2 = m->w + LP::p2_b;
  a.prm = prm;
  a.status = c->status;
  if (train) {
    a.out0 = c->hp;
    a.out1 = c->out;
    return launch_gemm<32, 64, kEpiProjTrain>(a, st, err);
  }
  a.out1 = static_cast<float*>(w_out);
  return launch_gemm<32, 64, kEpiProjInfer>(a, st, err);
}

Status backward_t(SnoCtx* c, const SnoPrm& prm, int S, const float* wt, cudaStream_t st, std::string* err) {
  SnoModel* m = c->model;
  const int P = c->P;
  const size_t Pz = static_cast<size_t>(P);
  Status s;
  SNO_CUDA(cudaMemsetAsync(m->g, 0, LP::total * sizeof(float), st), "SNO gradient clear");
  // loss, dW2 / db2 and the hidden-layer gradient
  const int lg = grid_for(static_cast<size_t>(S) * P, 256, 148 * 4);
  k_sno_loss<<<lg, 256, 0, st>>>(c->out, wt, c->hp, prm, m->wb + BL::p2, P, S, c->ghp, m->g + LP::p2_W,
                                 m->g + LP::p2_b, c->loss_part);
  k_sno_sum<<<1, 32, 0, st>>>(c->loss_part, lg, c->loss);
  add_launches(2);
  SNO_CUDA(cudaGetLastError(), "SNO loss launch");
  // dW1, db1, then g_v4 = W1^T ghp (tensor cores)
  SNO_CUDA(cudaMemsetAsync(c->gsum, 0, static_cast<size_t>(S) * kSnoHidden * sizeof(float), st), "SNO sums clear");
  const int wg = grid_for(static_cast<size_t>(S) * (P / 64), 1, 148 * 4);
  k_sno_wgrad<kSnoHidden, W><<<wg, 256, 0, st>>>(c->ghp, c->v[kSnoLayers], static_cast<size_t>(W) * Pz, P, S,
                                                  m->g + LP::p1_W, c->gsum);
  k_sno_bias_grads<<<1, kSnoHidden, 0, st>>>(c->gsum, S, kSnoHidden, m->g + LP::p1_b, nullptr, prm, c->slot);
  add_launches(2);
  SNO_CUDA(cudaGetLastError(), "SNO projection gradient launch");
  GemmArgs a{};
  a.X = c->ghp;
  a.B = m->wb + BL::p1T;
  a.P = P;
  a.S = S;
  a.add = nullptr;
  a.out0 = c->gz[0];
  a.status = c->status;
  if ((s = launch_gemm<kSnoHidden, 32, kEpiBwdLinear>(a, st, err)) != Status::kOk) return s;
  int cur = 0;
  for (int l = kSnoLayers - 1; l >= 0; --l) {
    float* g = c->gz[cur];
    float* gn = c->gz[cur ^ 1];
    const int64_t lb = LP::layer0 + l * LP::layer_size;
    SNO_CUDA(cudaMemsetAsync(c->gsum, 0, static_cast<size_t>(S) * W * sizeof(float), st), "SNO sums clear");
    k_sno_wgrad<W, W><<<wg, 256, 0, st>>>(g, c->v[l], static_cast<size_t>(W) * Pz, P, S, m->g + lb + LP::layer_W,
                                          c->gsum);
    k_sno_bias_grads<<<1, W, 0, st>>>(c->gsum, S, W, m->g + lb + LP::layer_b, nullptr, prm, c->slot);
    add_launches(2);
    SNO_CUDA(cudaGetLastError(), "SNO layer gradient launch");
    if ((s = exec_forward(c->plan, g, c->F, S * W, st, err)) != Status::kOk) return s;
    if (c->n_ret > 0) {
      k_sno_specmix_bwd<<<c->n_ret, S * W, 0, st>>>(c->F, c->n_spec, c->ret_spec, c->ret_cls, c->ret_wt,
                                                    m->wb + BL::layer0 + l * BL::lsize + BL::lS,
                                                    c->Vret + static_cast<size_t>(l) * c->n_ret * S * W, c->Y,
                                                    m->g + lb + LP::layer_S);
      add_launches(1);
      SNO_CUDA(cudaGetLastError(), "SNO spectral gradient launch");
    }
    if ((s = exec_backward(c->plan, c->Y, c->sbuf, S * W, st, err)) != Status::kOk) return s;
    GemmArgs b{};
    b.X = g;
    b.B = m->wb + BL::layer0 + l * BL::lsize + BL::lWT;
    b.P = P;
    b.S = S;
    b.add = c->sbuf;
    b.out0 = gn;
    b.status = c->status;
    if (l > 0) {
      b.zprev = c->z[l - 1];
      s = launch_gemm<32, 32, kEpiBwdGelu>(b, st, err);
    } else {
      s = launch_gemm<32, 32, kEpiBwdLinear>(b, st, err);
    }
    if (s != Status::kOk) return s;
    cur ^= 1;
  }
  // lift: feature channels by the product kernel, constant channels and bias from the sums
  SNO_CUDA(cudaMemsetAsync(c->gsum, 0, static_cast<size_t>(S) * W * sizeof(float), st), "SNO sums clear");
  float* dfeat = c->dfeat;  // the feature block of dW_lift ([32][5 + j]) is scattered in afterwards
  SNO_CUDA(cudaMemsetAsync(dfeat, 0, W * 2 * kSnoRefl * sizeof(float), st), "SNO lift scratch clear");
  k_sno_wgrad<W, 2 * kSnoRefl><<<wg, 256, 0, st>>>(c->gz[cur], c->feat, 0, P, S, dfeat, c->gsum);
  k_sno_bias_grads<<<1, W, 0, st>>>(c->gsum, S, W, m->g + LP::lift_b, m->g + LP::lift_W, prm, c->slot);
  k_sno_scatter_lift<<<1, W * 2 * kSnoRefl, 0, st>>>(dfeat, m->g + LP::lift_W);
  add_launches(3);
  SNO_CUDA(cudaGetLastError(), "SNO lift gradient launch");
  return Status::kOk;
}

SnoPrm make_prm(const double* params, int S) {
  SnoPrm prm{};
  for (int s = 0; s < S; ++s) {
    prm.chiN[s] = static_cast<float>(params[2 * s]);
    prm.f[s] = static_cast<float>(params[2 * s + 1]);
  }
  return prm;
}

Status check_status_word(SnoCtx* c, cudaStream_t st, std::string* err) {
  int h = 0;
  SNO_CUDA(cudaMemcpyAsync(&h, c->status, sizeof(int), cudaMemcpyDeviceToHost, st), "SNO status read");
  SNO_CUDA(cudaStreamSynchronize(st), "SNO synchronise");
  if (h != 0) {
    cudaMemsetAsync(c->status, 0, sizeof(int), st);  // reported once; the next call starts clean
    *err = "a tensor-core completion wait of the SNO ran out of time";
    return Status::kTimeout;
  }
  return Status::kOk;
}

// One Adam step from the model's gradient buffer, then the BF16 working copies.
Status adam_step(SnoModel* m, double lr, cudaStream_t st, std::string* err) {
  m->t += 1;
  const SnoConfig& k = m->cfg;
  const float c1 = static_cast<float>(1.0 - std::pow(k.beta1, static_cast<double>(m->t)));
  const float c2 = static_cast<float>(1.0 - std::pow(k.beta2, static_cast<double>(m->t)));
  k_sno_adam<<<grid_for(LP::total, 256), 256, 0, st>>>(m->w, m->g, m->m, m->v, LP::total, static_cast<float>(lr),
                                                       static_cast<float>(k.beta1), static_cast<float>(k.beta2),
                                                       static_cast<float>(k.eps), static_cast<float>(k.weight_decay),
                                                       c1, c2);
  k_sno_to_bf16<<<grid_for(BL::total, 256), 256, 0, st>>>(m->w, m->wb);
  add_launches(2);
  SNO_CUDA(cudaGetLastError(), "SNO optimiser launch");
  return Status::kOk;
}

}  // namespace

Status sno_grads_device(const SnoModel* m, void* dst, void* stream, std::string* err) {
  SNO_CUDA(cudaMemcpyAsync(dst, m->g, LP::total * sizeof(float), cudaMemcpyDeviceToDevice,
                           static_cast<cudaStream_t>(stream)),
           "SNO gradient copy");
  return Status::kOk;
}

Status sno_apply_grads(SnoModel* m, const void* grads, double lr, void* stream, std::string* err) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (grads && grads != m->g)
    SNO_CUDA(cudaMemcpyAsync(m->g, grads, LP::total * sizeof(float), cudaMemcpyDeviceToDevice, st),
             "SNO gradient upload");
  Status s = adam_step(m, lr, st, err);
  if (s != Status::kOk) return s;
  SNO_CUDA(cudaStreamSynchronize(st), "SNO optimiser");
  return Status::kOk;
}

Status sno_predict(SnoCtx* c, const double* params, int S, void* w_out, void* stream, std::string* err) {
  if (!c || !params || !w_out || S < 1 || S > c->S) { *err = "invalid SNO predict arguments"; return Status::kInvalid; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const SnoPrm prm = make_prm(params, S);
  Status s = forward_t(c, prm, S, false, w_out, st, err);
  if (s != Status::kOk) return s;
  return check_status_word(c, st, err);
}

Status sno_train(SnoCtx* c, const double* params, int S, const void* w_target, double lr, int step, double* loss,
                 void* stream, std::string* err) {
  if (!c || !params || !w_target || S < 1 || S > c->S) { *err = "invalid SNO train arguments"; return Status::kInvalid; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const SnoPrm prm = make_prm(params, S);
  Status s = forward_t(c, prm, S, true, nullptr, st, err);
  if (s != Status::kOk) return s;
  if ((s = backward_t(c, prm, S, static_cast<const float*>(w_target), st, err)) != Status::kOk) return s;
  SnoModel* m = c->model;
  if (step && (s = adam_step(m, lr, st, err)) != Status::kOk) return s;
  if (loss) {
    double h = 0.0;
    SNO_CUDA(cudaMemcpyAsync(&h, c->loss, sizeof(double), cudaMemcpyDeviceToHost, st), "SNO loss read");
    s = check_status_word(c, st, err);
    *loss = h / (static_cast<double>(S) * 2.0 * c->P);
    return s;
  }
  return check_status_word(c, st, err);
}

}  // namespace cfft

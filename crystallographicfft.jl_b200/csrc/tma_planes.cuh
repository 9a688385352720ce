// Persistent plane kernels with bulk-copy (TMA) staging, sm_100a.  Included by
// fast_kernels.cuh for the plane-stage translation units.
//
// The forward plane stage reads, for one task (workspace slot s, channel z-plane iz),
// the two f0 z-planes iz and iz + H of both fields of the slot: four contiguous M x M
// planes.  The backward plane stage reads the slot's nch channel planes W[s][c][iz],
// contiguous H x H complex each.  Both are regular, 16-byte aligned boxes, so one
// thread per group moves them with `cp.async.bulk` into a shared-memory stage and
// signals an mbarrier; no register holds a byte in flight.  A CTA runs NG independent
// groups of GT threads, each owning one stage and one padded FFT buffer, and walks
// tasks t = group, group + groups, ... (persistent): a group issues the copy of its next
// task as soon as it has consumed the stage, so the copy overlaps the group's own FFT
// phases and the other groups' work.
//
// Every wait on an mbarrier is bounded (timeout_ns of %globaltimer).  A wait that runs
// out writes CFFT_ERR_TIMEOUT (5) to *status, waits once more (bounded) for the group's
// copy in flight, and the group stops taking tasks.
//
// Included inside namespace cfft::(anonymous) of fast_kernels.cuh, after the plane
// helpers it uses (fold_emit, group_rows, y_lines_to_workspace, unfold_plane).
#pragma once

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Global -> shared bulk copy completing on `bar` (addresses 16-byte aligned, bytes a
// multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Named barrier of one group (ids 1..15; id 0 is __syncthreads).
__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}

// Bounded wait for phase `parity` of `bar`: true when it completed, false after
// timeout_ns of global time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > timeout_ns) return false;
  }
  return true;
}

constexpr uint64_t kWaitGraceNs = 1000000000ull;  // second bounded wait after a timeout

// Wait of a whole group for the stage's copy: the leader waits (bounded) and shares
// the verdict through shared memory, so every thread of the group takes the same
// branch and no named barrier is left short.  On success each thread observes the
// completed phase itself (an immediate try_wait), which orders its reads of the
// staged data after the copy.  On a timeout the leader records CFFT_ERR_TIMEOUT in
// *status and waits once more (bounded) for the copy still in flight, and the whole
// group returns false.
__device__ __forceinline__ bool group_wait(uint64_t* bar, uint32_t parity, uint64_t timeout_ns, int* abort_flag,
                                           int* status, int tid, int grp, int nthreads,
                                           uint64_t grace_ns = kWaitGraceNs) {
  if (tid == 0) *abort_flag = mbar_wait_bounded(bar, parity, timeout_ns) ? 0 : 1;
  group_sync(1 + grp, nthreads);
  if (*abort_flag) {
    if (tid == 0) {
      if (status) atomicExch(status, 5);
      mbar_wait_bounded(bar, parity, grace_ns);
    }
    return false;
  }
  mbar_try_wait(bar, parity);
  return true;
}

// Shared-memory layout of one group: [stage | FFT buffer], each 128-byte aligned.
template <typename T, int H, int CT, bool USE_E>
struct FwdTmaShape {
  using C = typename Cx<T>::type;
  static constexpr int M = 2 * H;
  static constexpr int nch = Cent<CT>::n;
  static constexpr size_t plane = static_cast<size_t>(M) * M * sizeof(T);  // one f0 z-plane
  static constexpr size_t stage = (USE_E ? 8 : 4) * plane;                // [E?][field][kz] planes
  static constexpr size_t buf = static_cast<size_t>(nch) * H * (H + 1) * sizeof(C);
  static constexpr size_t group = ((stage + 127) / 128) * 128 + ((buf + 127) / 128) * 128;
  static constexpr int threads = (nch * H + 31) / 32 * 32 < 128 ? 128 : (nch * H + 31) / 32 * 32;
};
template <typename T, int H, int CT>
struct BwdTmaShape {
  using C = typename Cx<T>::type;
  static constexpr int nch = Cent<CT>::n;
  static constexpr size_t plane = static_cast<size_t>(H) * H * sizeof(C);  // one channel plane of W
  static constexpr size_t stage = nch * plane;
  static constexpr size_t buf = static_cast<size_t>(nch) * H * (H + 1) * sizeof(C);
  static constexpr size_t group = ((stage + 127) / 128) * 128 + ((buf + 127) / 128) * 128;
  static constexpr int threads = (nch * H + 31) / 32 * 32 < 128 ? 128 : (nch * H + 31) / 32 * 32;
};
constexpr size_t kTmaSmemCap = 227 * 1024 - 256;  // dynamic shared memory per CTA, less the barriers' slack
template <typename Shape> constexpr int tma_groups() {
  return kTmaSmemCap / Shape::group >= 3 ? 3 : static_cast<int>(kTmaSmemCap / Shape::group);
}

// Fold of the slot's two fields at channel z-plane iz from the staged planes
// stage[e][f][kz][y][x] (e = 1: interaction factors) into the padded planes at buf.
template <typename T, int H, int CT, bool USE_E>
__device__ __forceinline__ void fold_from_stage(const T* stage, bool has_b, const typename Cx<T>::type* ftx,
                                                typename Cx<T>::type ftz, typename Cx<T>::type* buf, int tid, int nth) {
  constexpr int M = 2 * H;
  constexpr int VW = 16 / static_cast<int>(sizeof(T));
  constexpr int PLN = M * M;
  const T zero = static_cast<T>(0);
  for (int e = tid; e < H * H / VW; e += nth) {
    const int ix0 = (e % (H / VW)) * VW, iy = e / (H / VW);
    T va[8][VW], vb[8][VW];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int idx = ((k >> 2) & 1) * PLN + (iy + ((k >> 1) & 1) * H) * M + ix0 + (k & 1) * H;
      vload<T>(va[k], stage + idx);
      if (has_b) vload<T>(vb[k], stage + 2 * PLN + idx);
      else {
#pragma unroll
        for (int l = 0; l < VW; ++l) vb[k][l] = zero;
      }
      if constexpr (USE_E) {
        T ea[VW];
        vload<T>(ea, stage + 4 * PLN + idx);
#pragma unroll
        for (int l = 0; l < VW; ++l) va[k][l] *= ea[l];
        if (has_b) {
          vload<T>(ea, stage + 6 * PLN + idx);
#pragma unroll
          for (int l = 0; l < VW; ++l) vb[k][l] *= ea[l];
        }
      }
    }
    fold_emit<T, H, CT, VW>(va, vb, ix0, iy, ftx, ftz, buf);
  }
}

// Forward plane stage, persistent: per task (slot, iz) fold (WHT8 + twiddle, optional
// interaction factors E) of the staged planes + x FFT + y FFT -> W[slot][c][iz][y][x].
// Launched with NG * Shape::threads threads and NG * Shape::group bytes of dynamic
// shared memory; ntasks = slots * H.
template <typename T, int H, int CT, int NG, bool USE_E>
__global__ void __launch_bounds__(NG * FwdTmaShape<T, H, CT, USE_E>::threads)
k_plane_fwd_tma(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                const T* __restrict__ f0, const T* __restrict__ E, typename Cx<T>::type* __restrict__ W, int nfields,
                int ntasks, uint64_t timeout_ns, int* status) {
  using C = typename Cx<T>::type;
  using SH = FwdTmaShape<T, H, CT, USE_E>;
  constexpr int M = SH::M, GT = SH::threads, HV = H * H * H, nch = SH::nch;
  constexpr uint32_t PB = static_cast<uint32_t>(SH::plane);
  extern __shared__ __align__(128) unsigned char smem_tma[];
  __shared__ __align__(8) uint64_t bars[NG];
  __shared__ int aborts[NG];
  const int grp = threadIdx.x / GT, tid = threadIdx.x % GT;
  T* stage = reinterpret_cast<T*>(smem_tma + grp * SH::group);
  C* buf = reinterpret_cast<C*>(smem_tma + grp * SH::group + ((SH::stage + 127) / 128) * 128);
  uint64_t* bar = &bars[grp];
  if (tid == 0) mbar_init(bar, 1);
  fence_mbar_init();
  __syncthreads();
  pdl_enter();
  const size_t mvol = static_cast<size_t>(M) * M * M;
  const int groups = gridDim.x * NG;
  const C* ftx = tables + g->ftw_off[0];
  // Issue the copies of task t into this group's stage (group leader only).
  auto issue = [&](int t) {
    const int slot = t / H, iz = t % H, fa = 2 * slot;
    const bool hb = fa + 1 < nfields;
    const uint32_t nplanes = (hb ? 4u : 2u) * (USE_E ? 2u : 1u);
    mbar_expect_tx(bar, nplanes * PB);
#pragma unroll
    for (int e = 0; e < (USE_E ? 2 : 1); ++e) {
      const T* base = (e ? E : f0) + static_cast<size_t>(fa) * mvol;
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        if (f == 1 && !hb) break;
#pragma unroll
        for (int kz = 0; kz < 2; ++kz)
          bulk_g2s(stage + (e * 4 + f * 2 + kz) * (M * M), base + f * mvol + static_cast<size_t>(iz + kz * H) * M * M,
                   PB, bar);
      }
    }
  };
  int t = blockIdx.x * NG + grp;
  if (tid == 0 && t < ntasks) issue(t);
  uint32_t phase = 0;
  for (; t < ntasks; t += groups) {
    if (!group_wait(bar, phase, timeout_ns, &aborts[grp], status, tid, grp, GT)) return;
    phase ^= 1u;
    const int slot = t / H, iz = t % H, fa = 2 * slot;
    const bool hb = fa + 1 < nfields;
    fold_from_stage<T, H, CT, USE_E>(stage, hb, ftx, tables[g->ftw_off[2] + iz], buf, tid, GT);
    group_sync(1 + grp, GT);  // stage consumed, buf complete
    if (tid == 0 && t + groups < ntasks) issue(t + groups);
    group_rows<C, false, H>(buf, nch * H, tid, GT);  // x lines
    group_sync(1 + grp, GT);
    y_lines_to_workspace<C, H, nch>(buf, W + static_cast<size_t>(slot) * nch * HV + iz * H * H, tid, GT);
    group_sync(1 + grp, GT);  // buf free for the next fold
  }
}

// Backward plane stage, persistent: per task (slot, iz) the nch channel planes
// W[slot][c][iz] are staged, inverse y FFT (stage -> padded buffer), inverse x FFT,
// unfold (conjugate twiddle, inverse WHT8 / 8, optional E) -> f0 as 16-byte stores.
template <typename T, int H, int CT, int NG>
__global__ void __launch_bounds__(NG * BwdTmaShape<T, H, CT>::threads)
k_plane_bwd_tma(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                const typename Cx<T>::type* __restrict__ W, const T* __restrict__ E, T* __restrict__ f0, int nfields,
                int ntasks, uint64_t timeout_ns, int* status) {
  using C = typename Cx<T>::type;
  using SH = BwdTmaShape<T, H, CT>;
  constexpr int GT = SH::threads, HV = H * H * H, nch = SH::nch, S = H + 1, PL = H * S;
  constexpr uint32_t PB = static_cast<uint32_t>(SH::plane);
  extern __shared__ __align__(128) unsigned char smem_tma[];
  __shared__ __align__(8) uint64_t bars[NG];
  __shared__ int aborts[NG];
  const int grp = threadIdx.x / GT, tid = threadIdx.x % GT;
  C* stage = reinterpret_cast<C*>(smem_tma + grp * SH::group);
  C* buf = reinterpret_cast<C*>(smem_tma + grp * SH::group + ((SH::stage + 127) / 128) * 128);
  uint64_t* bar = &bars[grp];
  if (tid == 0) mbar_init(bar, 1);
  fence_mbar_init();
  __syncthreads();
  pdl_enter();
  const size_t mvol = static_cast<size_t>(8) * HV;
  const int groups = gridDim.x * NG;
  auto issue = [&](int t) {
    const int slot = t / H, iz = t % H;
    mbar_expect_tx(bar, nch * PB);
#pragma unroll
    for (int c = 0; c < nch; ++c)
      bulk_g2s(stage + c * H * H, W + (static_cast<size_t>(slot) * nch + c) * HV + static_cast<size_t>(iz) * H * H, PB,
               bar);
  };
  int t = blockIdx.x * NG + grp;
  if (tid == 0 && t < ntasks) issue(t);
  uint32_t phase = 0;
  for (; t < ntasks; t += groups) {
    if (!group_wait(bar, phase, timeout_ns, &aborts[grp], status, tid, grp, GT)) return;
    phase ^= 1u;
    const int slot = t / H, iz = t % H, fa = 2 * slot;
    const bool hb = fa + 1 < nfields;
    // The staged channel planes are the last read of these workspace lines: drop them
    // from L2 without a write-back (planes are whole 128-byte lines for H % 4 == 0).
    if constexpr (SH::plane % 128 == 0) {
      constexpr int LPP = static_cast<int>(SH::plane / 128);
      for (int i = tid; i < nch * LPP; i += GT)
        discard_l2_line(reinterpret_cast<const char*>(W + (static_cast<size_t>(slot) * nch + i / LPP) * HV +
                                                      static_cast<size_t>(iz) * H * H) + (i % LPP) * 128);
    }
    // inverse y FFT: column (c, x) of the staged plane -> padded buffer
    for (int l = tid; l < nch * H; l += GT) {
      const int c = l / H, x = l % H;
      const C* q = stage + c * H * H + x;
      C v[H];
#pragma unroll
      for (int i = 0; i < H; ++i) v[i] = q[i * H];
      reg_fft<C, true, H>(v);
      C* p = buf + c * PL + x;
#pragma unroll
      for (int i = 0; i < H; ++i) p[i * S] = v[i];
    }
    group_sync(1 + grp, GT);  // stage consumed, buf complete
    if (tid == 0 && t + groups < ntasks) issue(t + groups);
    group_rows<C, true, H>(buf, nch * H, tid, GT);
    group_sync(1 + grp, GT);
    T* dsta = f0 + static_cast<size_t>(fa) * mvol;
    const bool use_e = E != nullptr;
    const T* Ea = use_e ? E + static_cast<size_t>(fa) * mvol : nullptr;
    unfold_plane<T, H, CT, true>(g, tables, buf, dsta, dsta + mvol, Ea, use_e ? Ea + mvol : nullptr, hb, use_e, iz,
                                 tid, GT);
    group_sync(1 + grp, GT);  // buf free for the next y FFT
  }
}

// Self-test of the bounded wait (no reference counterpart): one group of 128 threads
// expects 16 bytes on its mbarrier that no copy ever delivers, so group_wait must run
// out after timeout_ns, record CFFT_ERR_TIMEOUT in *status and return; no copy is in
// flight, so the grace wait is short.  *status is left alone if the wait completes.
__global__ void __launch_bounds__(128) k_wait_selftest(uint64_t timeout_ns, int* status) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  fence_mbar_init();
  __syncthreads();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);
  group_wait(&bar, 0, timeout_ns, &abort_flag, status, threadIdx.x, 0, 128, 1000);
}

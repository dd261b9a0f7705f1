// Device helpers shared by the solver kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace cfd {

constexpr int kMaxNGP = 27;

// Quadrature and shape-function tables for hex27 velocity / hex8 pressure
// elements at the Gauss points (blascoCodinaHuerta.cpp:2166-2488), laid out
// for the device: Sv[k][j], dSv[d][k][j], Sp[k][m], dSp[d][k][m].
struct Basis {
  int ngp;
  int pad;
  double w[kMaxNGP];
  double Sv[kMaxNGP][27];
  double dSv[3][kMaxNGP][27];
  double Sp[kMaxNGP][8];
  double dSp[3][kMaxNGP][8];
};

#if defined(__CUDACC__)
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Sum over aligned groups of G lanes (G a power of two <= 32); every lane of
// the group receives the group sum.
template <int G, class T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum of NV values (blockDim.x a multiple of 32, <= 1024).  The
// result is valid in thread 0.  Fixed reduction tree: deterministic.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++) sh[warp][k] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      double t = lane < nw ? sh[lane][k] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_add_release_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) {
  return *reinterpret_cast<const volatile int*>(p);
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier for a cooperative (co-resident) launch.  bar[0] counts
// arrivals, bar[1] is the generation.  Every wait is bounded: after
// timeout_ns a waiting block raises *err and returns false; blocks that see
// *err set also return false.  The host clears bar and err before a launch.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err, unsigned long long timeout_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned gen = ld_acquire_u32(bar + 1);
    __threadfence();
    unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned long long t0 = global_ns();
      while (ld_acquire_u32(bar + 1) == gen) {
        if (ld_volatile_i32(err)) { ok = 0; break; }
        if (global_ns() - t0 > timeout_ns) {
          atomicExch(err, 1);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    if (ok && ld_volatile_i32(err)) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Programmatic dependent launch (sm_90 and newer).  A kernel launched with
// launch_k(pdl = true, ...) may start while the kernel before it on the
// stream is still running: pdl_wait() returns once that kernel has finished
// and its writes are visible (at once for a launch without the attribute),
// and pdl_trigger() lets the kernel after this one launch as soon as every
// block of this one has reached it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// Read-only 32-byte load of a double4 node value (two 16-byte loads of the
// same aligned sector).
__device__ __forceinline__ double4 ldg4(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// Read-only load of a gathered velocity value: the float4 copy or the double4
// state.
__device__ __forceinline__ float4 ldgv(const float4* p) { return __ldg(p); }
__device__ __forceinline__ double4 ldgv(const double4* p) { return ldg4(p); }
__device__ __forceinline__ float4 to_f4(const double4& v) {
  return make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
}

// ---- bulk asynchronous copies (global -> shared) completed on an mbarrier ----
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* m, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}
// One bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(m))
               : "memory");
}
// L2 eviction policies (createpolicy): streams read once go first, data
// re-read by every iteration of a solve stays
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_evict_last() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// bulk_g2s with an L2 cache policy
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes, unsigned long long* m,
                                              unsigned long long policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(m)), "l"(policy)
      : "memory");
}
// read-only 16-byte load with an L2 cache policy
__device__ __forceinline__ uint4 ldg_hint(const uint4* p, unsigned long long policy) {
  uint4 v;
  asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p), "l"(policy));
  return v;
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* m, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity; false after timeout_ns.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* m, unsigned parity,
                                                  unsigned long long timeout_ns) {
  if (mbar_try_wait(m, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(m, parity)) {
    if (global_ns() - t0 > timeout_ns) return false;
  }
  return true;
}

// Position of key in the sorted range col[b, e); -1 when absent.
__device__ __forceinline__ int bsearch_slot(const int* __restrict__ col, int b, int e, int key) {
  int lo = b, hi = e - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int c = __ldg(col + mid);
    if (c == key) return mid;
    if (c < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// Kernel launch, with the programmatic-stream-serialisation attribute when
// pdl is set (the kernel must then call pdl_wait() before it reads what the
// previous kernel wrote).
template <typename... Params, typename... Args>
inline cudaError_t launch_k(bool pdl, void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem,
                            cudaStream_t s, Args... args) {
  if (!pdl) {
    kernel<<<grid, block, smem, s>>>(args...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

#endif  // __CUDACC__

}  // namespace cfd

// Shared device helpers for libpolar (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "polar.h"

#define POLAR_HD __host__ __device__ __forceinline__
#define POLAR_D __device__ __forceinline__

namespace polar {

// ---------------------------------------------------------------------------------------
// Vector access: V consecutive elements of T through one 4/8/16-byte load or store.
template <typename T, int V> struct VecType;
template <> struct VecType<float, 1> { using type = float; };
template <> struct VecType<float, 2> { using type = float2; };
template <> struct VecType<float, 4> { using type = float4; };
template <> struct VecType<double, 1> { using type = double; };
template <> struct VecType<double, 2> { using type = double2; };

template <typename T, int V>
union VecU {
  typename VecType<T, V>::type v;
  T a[V];
};

// Widest single access for V elements (at most 16 bytes); V elements are read as V / VW
// such accesses when V * sizeof(T) exceeds 16 bytes.
template <typename T, int V>
struct VecWidth {
  static constexpr int value = (V * (int)sizeof(T) <= 16) ? V : 16 / (int)sizeof(T);
};

template <typename T, int V>
POLAR_D void vload(T (&out)[V], const T* p) {
  constexpr int VW = VecWidth<T, V>::value;
#pragma unroll
  for (int c = 0; c < V / VW; ++c) {
    VecU<T, VW> u;
    u.v = *reinterpret_cast<const typename VecType<T, VW>::type*>(p + c * VW);
#pragma unroll
    for (int i = 0; i < VW; ++i) out[c * VW + i] = u.a[i];
  }
}

// L2-only load for data that other CTAs of the same persistent launch rewrite.
template <typename T, int V>
POLAR_D void vload_cg(T (&out)[V], const T* p) {
  constexpr int VW = VecWidth<T, V>::value;
#pragma unroll
  for (int c = 0; c < V / VW; ++c) {
    VecU<T, VW> u;
    u.v = __ldcg(reinterpret_cast<const typename VecType<T, VW>::type*>(p + c * VW));
#pragma unroll
    for (int i = 0; i < VW; ++i) out[c * VW + i] = u.a[i];
  }
}

template <typename T, int V>
POLAR_D void vstore(T* p, const T (&in)[V]) {
  constexpr int VW = VecWidth<T, V>::value;
#pragma unroll
  for (int c = 0; c < V / VW; ++c) {
    VecU<T, VW> u;
#pragma unroll
    for (int i = 0; i < VW; ++i) u.a[i] = in[c * VW + i];
    *reinterpret_cast<typename VecType<T, VW>::type*>(p + c * VW) = u.v;
  }
}

// Evict-first (streaming) store, for data that is not read again soon.
template <typename T, int V>
POLAR_D void vstore_cs(T* p, const T (&in)[V]) {
  constexpr int VW = VecWidth<T, V>::value;
#pragma unroll
  for (int c = 0; c < V / VW; ++c) {
    VecU<T, VW> u;
#pragma unroll
    for (int i = 0; i < VW; ++i) u.a[i] = in[c * VW + i];
    __stcs(reinterpret_cast<typename VecType<T, VW>::type*>(p + c * VW), u.v);
  }
}

// ---------------------------------------------------------------------------------------
// L2 eviction priority per access (createpolicy + .L2::cache_hint, sm_80+).  The SpMM's
// gathers are skewed: on degree-ordered graphs a prefix of rows takes most of them, so
// those rows are loaded (and, by the direction update, stored) with evict_last, while
// data read or written once per pass (neighbour indices, v) goes with evict_first and
// cannot push the prefix out of L2.  The hints change caching only, never results.
POLAR_D uint64_t l2_policy(int kind) {  // 0 normal, 1 evict_last, 2 evict_first
  uint64_t p;
  if (kind == 1)
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  else if (kind == 2)
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  else
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}

POLAR_D void ld_hint(float4& v, const void* p, uint64_t pol) {
  asm volatile("ld.global.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(pol));
}
POLAR_D void ld_hint(float2& v, const void* p, uint64_t pol) {
  asm volatile("ld.global.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
}
POLAR_D void ld_hint(float& v, const void* p, uint64_t pol) {
  asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
}
POLAR_D void ld_hint(double2& v, const void* p, uint64_t pol) {
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
}
POLAR_D void ld_hint(double& v, const void* p, uint64_t pol) {
  asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
}
POLAR_D int ld_hint_i32(const int* p, uint64_t pol) {
  int v;
  asm volatile("ld.global.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
POLAR_D void st_hint(void* p, const float4& v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1,%2,%3,%4}, %5;"
               ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol) : "memory");
}
POLAR_D void st_hint(void* p, const float2& v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1,%2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(pol) : "memory");
}
POLAR_D void st_hint(void* p, const float& v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}
POLAR_D void st_hint(void* p, const double2& v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1,%2}, %3;" ::"l"(p), "d"(v.x), "d"(v.y), "l"(pol) : "memory");
}
POLAR_D void st_hint(void* p, const double& v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}

template <typename T, int V>
POLAR_D void vload_hint(T (&out)[V], const T* p, uint64_t pol) {
  constexpr int VW = VecWidth<T, V>::value;
#pragma unroll
  for (int c = 0; c < V / VW; ++c) {
    VecU<T, VW> u;
    ld_hint(u.v, p + c * VW, pol);
#pragma unroll
    for (int i = 0; i < VW; ++i) out[c * VW + i] = u.a[i];
  }
}

template <typename T, int V>
POLAR_D void vstore_hint(T* p, const T (&in)[V], uint64_t pol) {
  constexpr int VW = VecWidth<T, V>::value;
#pragma unroll
  for (int c = 0; c < V / VW; ++c) {
    VecU<T, VW> u;
#pragma unroll
    for (int i = 0; i < VW; ++i) u.a[i] = in[c * VW + i];
    st_hint(p + c * VW, u.v, pol);
  }
}

// ---------------------------------------------------------------------------------------
// Programmatic dependent launch (sm_90+).  A kernel launched with programmatic stream
// serialization may start while its predecessor is still running; pdl_wait blocks until
// the predecessor grid has completed and its memory is visible (a no-op for an ordinary
// launch).  pdl_launch lets the successor be scheduled once every CTA of this grid has
// called it, so the successor's CTAs take SM slots as this grid's CTAs retire.
POLAR_D void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
POLAR_D void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

POLAR_D uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

POLAR_D unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

POLAR_D void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

POLAR_D int ld_volatile_i32(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// ---------------------------------------------------------------------------------------
// Grid barrier for a cooperative (co-resident) launch.  Arrival: every CTA fences its
// writes and bumps `count`; the last CTA to arrive may run serial work (a reduction of
// per-CTA partials) before it releases the others by advancing `gen`.  Waiting CTAs
// poll `gen` with a time limit; on expiry they record POLAR_ERR_TIMEOUT in `err` and
// every CTA leaves the kernel at its next barrier.  No wait is unbounded.  `nblk` is the
// number of CTAs that take part: the whole grid, or one problem's share of the CTAs of a
// batched launch (each share has its own count/gen words).
struct GridSync {
  unsigned* count;
  unsigned* gen;
  int* err;
  int* where;
  uint64_t timeout_ns;
  unsigned nblk;
};

// Returns true in every thread of the last-arriving CTA.  `my_gen` receives the
// generation to wait on.  Caller must later call grid_release (last CTA) or
// grid_wait (others).
POLAR_D bool grid_arrive(const GridSync& s, unsigned& my_gen) {
  __shared__ unsigned sh_last, sh_gen;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned g = ld_acquire_u32(s.gen);
    __threadfence();
    unsigned old = atomicAdd(s.count, 1u);
    sh_last = (old == s.nblk - 1) ? 1u : 0u;
    sh_gen = g;
    if (sh_last) __threadfence();
  }
  __syncthreads();
  my_gen = sh_gen;
  return sh_last != 0;
}

// Releases the waiting CTAs.  Returns true (uniformly across the CTA) when no error has
// been recorded.
POLAR_D bool grid_release(const GridSync& s, unsigned my_gen) {
  __shared__ int sh_ok2;
  __syncthreads();
  if (threadIdx.x == 0) {
    *s.count = 0u;
    __threadfence();
    st_release_u32(s.gen, my_gen + 1u);
    sh_ok2 = ld_volatile_i32(s.err) == 0;
  }
  __syncthreads();
  return sh_ok2 != 0;
}

// Returns false (in all threads of the CTA) when the kernel must stop: a wait timed out
// here or an error was recorded elsewhere.
POLAR_D bool grid_wait(const GridSync& s, unsigned my_gen, int where) {
  __shared__ int sh_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    uint64_t t0 = globaltimer_ns();
    while (ld_acquire_u32(s.gen) == my_gen) {
      if (ld_volatile_i32(s.err) != 0) { ok = 0; break; }
      if (globaltimer_ns() - t0 > s.timeout_ns) {
        atomicCAS(s.err, 0, (int)POLAR_ERR_TIMEOUT);
        atomicCAS(s.where, 0, where);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    if (ld_volatile_i32(s.err) != 0) ok = 0;
    sh_ok = ok;
  }
  __syncthreads();
  return sh_ok != 0;
}

// Plain barrier (no serial section).
POLAR_D bool grid_sync(const GridSync& s, int where) {
  unsigned g;
  if (grid_arrive(s, g)) return grid_release(s, g);
  return grid_wait(s, g, where);
}

POLAR_HD int next_pow2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace polar

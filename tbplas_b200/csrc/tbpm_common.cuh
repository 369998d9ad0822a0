// Shared device-side types for the TBPM kernels (sm_100a).
//
// State vectors are stored "row-interleaved": a block of B states over N
// orbitals is one array of N rows x ld complex numbers (ld = B, or 3B / 2B when
// several vector families are propagated together), so the gather of
// neighbour row c in the SpMV reads ld*sizeof(complex) contiguous bytes.
// Each thread owns V consecutive complex columns of a row, loaded as one 16-byte
// vector (double2 for FP64, float4 for FP32 pairs) or one 8-byte float2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tbpm {

template <typename R>
struct Cx;
template <>
struct Cx<double> {
  using t = double2;
};
template <>
struct Cx<float> {
  using t = float2;
};

// V complex numbers of precision R moved as one vector access.
template <typename R, int V>
struct alignas(2 * V * sizeof(R)) Pack {
  R v[2 * V];
};

__device__ __forceinline__ Pack<double, 1> ldg_pack(const Pack<double, 1>* p) {
  const double2 d = __ldg(reinterpret_cast<const double2*>(p));
  Pack<double, 1> r;
  r.v[0] = d.x;
  r.v[1] = d.y;
  return r;
}
__device__ __forceinline__ Pack<float, 2> ldg_pack(const Pack<float, 2>* p) {
  const float4 d = __ldg(reinterpret_cast<const float4*>(p));
  Pack<float, 2> r;
  r.v[0] = d.x;
  r.v[1] = d.y;
  r.v[2] = d.z;
  r.v[3] = d.w;
  return r;
}
__device__ __forceinline__ Pack<float, 1> ldg_pack(const Pack<float, 1>* p) {
  const float2 d = __ldg(reinterpret_cast<const float2*>(p));
  Pack<float, 1> r;
  r.v[0] = d.x;
  r.v[1] = d.y;
  return r;
}

// Two complex128 values per thread: one 256-bit access (ld/st .v4.f64, sm_100).
__device__ __forceinline__ Pack<double, 2> ldg_pack(const Pack<double, 2>* p) {
  Pack<double, 2> r;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3])
      : "l"(p));
  return r;
}

// Four complex64 values per thread: one 256-bit access (ld/st .v8.f32, sm_100).
__device__ __forceinline__ Pack<float, 4> ldg_pack(const Pack<float, 4>* p) {
  Pack<float, 4> r;
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]),
        "=f"(r.v[6]), "=f"(r.v[7])
      : "l"(p));
  return r;
}

// Streaming (evict-first) access for vectors read or written once per kernel,
// so they do not push the gathered vector out of L2.
__device__ __forceinline__ Pack<double, 1> ldcs_pack(const Pack<double, 1>* p) {
  const double2 d = __ldcs(reinterpret_cast<const double2*>(p));
  Pack<double, 1> r;
  r.v[0] = d.x;
  r.v[1] = d.y;
  return r;
}
__device__ __forceinline__ Pack<float, 2> ldcs_pack(const Pack<float, 2>* p) {
  const float4 d = __ldcs(reinterpret_cast<const float4*>(p));
  Pack<float, 2> r;
  r.v[0] = d.x;
  r.v[1] = d.y;
  r.v[2] = d.z;
  r.v[3] = d.w;
  return r;
}
__device__ __forceinline__ Pack<float, 1> ldcs_pack(const Pack<float, 1>* p) {
  const float2 d = __ldcs(reinterpret_cast<const float2*>(p));
  Pack<float, 1> r;
  r.v[0] = d.x;
  r.v[1] = d.y;
  return r;
}
__device__ __forceinline__ Pack<double, 2> ldcs_pack(const Pack<double, 2>* p) {
  Pack<double, 2> r;
  asm volatile("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3])
               : "l"(p)
               : "memory");
  return r;
}
__device__ __forceinline__ void stcs_pack(Pack<double, 2>* p, const Pack<double, 2>& v) {
  asm volatile("st.global.cs.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v.v[0]), "d"(v.v[1]),
               "d"(v.v[2]), "d"(v.v[3])
               : "memory");
}
__device__ __forceinline__ Pack<float, 4> ldcs_pack(const Pack<float, 4>* p) {
  Pack<float, 4> r;
  asm volatile("ld.global.cs.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]),
                 "=f"(r.v[5]), "=f"(r.v[6]), "=f"(r.v[7])
               : "l"(p)
               : "memory");
  return r;
}
__device__ __forceinline__ void stcs_pack(Pack<float, 4>* p, const Pack<float, 4>& v) {
  asm volatile("st.global.cs.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p),
               "f"(v.v[0]), "f"(v.v[1]), "f"(v.v[2]), "f"(v.v[3]), "f"(v.v[4]), "f"(v.v[5]),
               "f"(v.v[6]), "f"(v.v[7])
               : "memory");
}
__device__ __forceinline__ void stcs_pack(Pack<double, 1>* p, const Pack<double, 1>& v) {
  __stcs(reinterpret_cast<double2*>(p), make_double2(v.v[0], v.v[1]));
}
__device__ __forceinline__ void stcs_pack(Pack<float, 2>* p, const Pack<float, 2>& v) {
  __stcs(reinterpret_cast<float4*>(p), make_float4(v.v[0], v.v[1], v.v[2], v.v[3]));
}
__device__ __forceinline__ void stcs_pack(Pack<float, 1>* p, const Pack<float, 1>& v) {
  __stcs(reinterpret_cast<float2*>(p), make_float2(v.v[0], v.v[1]));
}

__device__ __forceinline__ double2 ldg_c(const double2* p) { return __ldg(p); }
__device__ __forceinline__ float2 ldg_c(const float2* p) { return __ldg(p); }

// Loads of values written earlier in the same launch by other blocks: cached
// in L2 only (ld.global.cg), never in the non-coherent L1/texture path.  The
// asm statements are volatile with a memory clobber so the compiler keeps
// them after the synchronisation that makes the values visible.
__device__ __forceinline__ Pack<double, 1> ldcg_pack(const Pack<double, 1>* p) {
  Pack<double, 1> r;
  asm volatile("ld.global.cg.v2.f64 {%0, %1}, [%2];" : "=d"(r.v[0]), "=d"(r.v[1]) : "l"(p)
               : "memory");
  return r;
}
__device__ __forceinline__ Pack<double, 2> ldcg_pack(const Pack<double, 2>* p) {
  Pack<double, 2> r;
  asm volatile("ld.global.cg.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(r.v[0]), "=d"(r.v[1]), "=d"(r.v[2]), "=d"(r.v[3])
               : "l"(p)
               : "memory");
  return r;
}
__device__ __forceinline__ Pack<float, 1> ldcg_pack(const Pack<float, 1>* p) {
  Pack<float, 1> r;
  asm volatile("ld.global.cg.v2.f32 {%0, %1}, [%2];" : "=f"(r.v[0]), "=f"(r.v[1]) : "l"(p)
               : "memory");
  return r;
}
__device__ __forceinline__ Pack<float, 2> ldcg_pack(const Pack<float, 2>* p) {
  Pack<float, 2> r;
  asm volatile("ld.global.cg.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3])
               : "l"(p)
               : "memory");
  return r;
}
__device__ __forceinline__ Pack<float, 4> ldcg_pack(const Pack<float, 4>* p) {
  Pack<float, 4> r;
  asm volatile("ld.global.cg.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]),
                 "=f"(r.v[5]), "=f"(r.v[6]), "=f"(r.v[7])
               : "l"(p)
               : "memory");
  return r;
}

// Stores with the default (write-back, evict-normal) policy, for values that
// are read again from L2 shortly after, within the same launch.
__device__ __forceinline__ void stwb_pack(Pack<double, 1>* p, const Pack<double, 1>& v) {
  asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.v[0]), "d"(v.v[1]) : "memory");
}
__device__ __forceinline__ void stwb_pack(Pack<double, 2>* p, const Pack<double, 2>& v) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v.v[0]), "d"(v.v[1]),
               "d"(v.v[2]), "d"(v.v[3])
               : "memory");
}
__device__ __forceinline__ void stwb_pack(Pack<float, 1>* p, const Pack<float, 1>& v) {
  asm volatile("st.global.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v.v[0]), "f"(v.v[1]) : "memory");
}
__device__ __forceinline__ void stwb_pack(Pack<float, 2>* p, const Pack<float, 2>& v) {
  asm volatile("st.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.v[0]), "f"(v.v[1]),
               "f"(v.v[2]), "f"(v.v[3])
               : "memory");
}
__device__ __forceinline__ void stwb_pack(Pack<float, 4>* p, const Pack<float, 4>& v) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p),
               "f"(v.v[0]), "f"(v.v[1]), "f"(v.v[2]), "f"(v.v[3]), "f"(v.v[4]), "f"(v.v[5]),
               "f"(v.v[6]), "f"(v.v[7])
               : "memory");
}

// Fixed-order tree reduction over the `rows` row slots of a block.  Values are
// laid out as smem[slot * width + k]; after the call slot 0 holds the sums.
// Every thread of the block must call it (it synchronises).
__device__ __forceinline__ void tree_reduce_slots(double* smem, int rows, int width, int slot,
                                                  int lane_lo, int lane_step) {
  int s = 1;
  while (s * 2 < rows) s *= 2;
  for (; s > 0; s >>= 1) {
    if (slot < s && slot + s < rows) {
      for (int k = lane_lo; k < width; k += lane_step)
        smem[slot * width + k] += smem[(slot + s) * width + k];
    }
    __syncthreads();
  }
}

}  // namespace tbpm

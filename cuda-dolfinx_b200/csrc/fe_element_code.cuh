// GENERATED by gen_element_code.py -- do not edit.
#pragma once

namespace fe {

// int_ref phi_i (reference volume 1/6)
__device__ __forceinline__ double p2_basis_integral(int i) {
  return i < 4 ? -0x1.1111111111111p-7 : 0x1.1111111111111p-5;
}

// int_ref phi_i of the equispaced P3 element (vertices, edge pairs, faces)
__device__ __forceinline__ double p3_basis_integral(int i) {
  return i < 4 ? 0x1.1111111111111p-8 : (i < 16 ? 0x0.0p+0 : 0x1.3333333333333p-5);
}

// P3 stiffness with a cellwise-constant coefficient: g[s] = k * Ghat_s;
// emit(i, j, value) for the 210 unique entries i <= j.
template <typename T, typename Emit>
__device__ __forceinline__ void p3_stiffness_const(const T* g, Emit&& emit) {
  if constexpr (sizeof(T) == 8) {
    emit(0, 0, (fma(g[4], T(0x1.e79e79e79e79ep-4), fma(g[2], T(0x1.e79e79e79e79ep-5), g[0] * T(0x1.e79e79e79e79ep-5))) + fma(g[5], T(0x1.e79e79e79e79ep-4), fma(g[3], T(0x1.e79e79e79e79ep-4), g[1] * T(0x1.e79e79e79e79ep-5)))));
    emit(0, 1, (fma(g[4], T(-0x1.7297297297297p-7), g[0] * T(-0x1.7297297297297p-7)) + g[3] * T(-0x1.7297297297297p-7)));
    emit(0, 2, (fma(g[5], T(-0x1.7297297297297p-7), g[1] * T(-0x1.7297297297297p-7)) + g[3] * T(-0x1.7297297297297p-7)));
    emit(0, 3, (fma(g[5], T(-0x1.7297297297297p-7), g[2] * T(-0x1.7297297297297p-7)) + g[4] * T(-0x1.7297297297297p-7)));
    emit(0, 4, (fma(g[5], T(-0x1.b6db6db6db6dbp-6), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[2] * T(-0x1.b6db6db6db6dbp-7))));
    emit(0, 5, (fma(g[5], T(-0x1.b6db6db6db6dbp-6), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[2] * T(-0x1.b6db6db6db6dbp-7))));
    emit(0, 6, (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-6), g[2] * T(-0x1.b6db6db6db6dbp-7))));
    emit(0, 7, (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-6), g[2] * T(-0x1.b6db6db6db6dbp-7))));
    emit(0, 8, (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-6), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))));
    emit(0, 9, (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-6), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))));
    emit(0, 10, (fma(g[4], T(-0x1.0cccccccccccdp-3), fma(g[2], T(-0x1.8af8af8af8af9p-4), g[0] * T(-0x1.1d41d41d41d42p-5))) + fma(g[5], T(-0x1.0cccccccccccdp-3), fma(g[3], T(-0x1.1d41d41d41d42p-4), g[1] * T(-0x1.1d41d41d41d42p-5)))));
    emit(0, 11, (fma(g[4], T(0x1.f8af8af8af8b0p-5), fma(g[2], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.b6db6db6db6dbp-7))) + fma(g[5], T(0x1.f8af8af8af8b0p-5), fma(g[3], T(0x1.b6db6db6db6dbp-6), g[1] * T(0x1.b6db6db6db6dbp-7)))));
    emit(0, 12, (fma(g[4], T(-0x1.1d41d41d41d42p-4), fma(g[2], T(-0x1.1d41d41d41d42p-5), g[0] * T(-0x1.1d41d41d41d42p-5))) + fma(g[5], T(-0x1.0cccccccccccdp-3), fma(g[3], T(-0x1.0cccccccccccdp-3), g[1] * T(-0x1.8af8af8af8af9p-4)))));
    emit(0, 13, (fma(g[4], T(0x1.b6db6db6db6dbp-6), fma(g[2], T(0x1.b6db6db6db6dbp-7), g[0] * T(0x1.b6db6db6db6dbp-7))) + fma(g[5], T(0x1.f8af8af8af8b0p-5), fma(g[3], T(0x1.f8af8af8af8b0p-5), g[1] * T(0x1.8af8af8af8af9p-5)))));
    emit(0, 14, (fma(g[4], T(-0x1.0cccccccccccdp-3), fma(g[2], T(-0x1.1d41d41d41d42p-5), g[0] * T(-0x1.8af8af8af8af9p-4))) + fma(g[5], T(-0x1.1d41d41d41d42p-4), fma(g[3], T(-0x1.0cccccccccccdp-3), g[1] * T(-0x1.1d41d41d41d42p-5)))));
    emit(0, 15, (fma(g[4], T(0x1.f8af8af8af8b0p-5), fma(g[2], T(0x1.b6db6db6db6dbp-7), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[5], T(0x1.b6db6db6db6dbp-6), fma(g[3], T(0x1.f8af8af8af8b0p-5), g[1] * T(0x1.b6db6db6db6dbp-7)))));
    emit(0, 16, (fma(g[4], T(-0x1.0750750750750p-4), fma(g[2], T(-0x1.0750750750750p-5), g[0] * T(-0x1.0750750750750p-5))) + fma(g[5], T(-0x1.0750750750750p-4), fma(g[3], T(-0x1.0750750750750p-4), g[1] * T(-0x1.0750750750750p-5)))));
    emit(0, 17, (fma(g[4], T(0x1.4924924924925p-4), fma(g[2], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.0750750750750p-5))) + fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.4924924924925p-4), g[1] * T(0x1.8af8af8af8af9p-5)))));
    emit(0, 18, (fma(g[4], T(0x1.8af8af8af8af9p-4), fma(g[2], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[5], T(0x1.4924924924925p-4), fma(g[3], T(0x1.4924924924925p-4), g[1] * T(0x1.0750750750750p-5)))));
    emit(0, 19, (fma(g[4], T(0x1.4924924924925p-4), fma(g[2], T(0x1.0750750750750p-5), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[5], T(0x1.4924924924925p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-5)))));
    emit(1, 1, g[0] * T(0x1.e79e79e79e79ep-5));
    emit(1, 2, g[3] * T(0x1.7297297297297p-7));
    emit(1, 3, g[4] * T(0x1.7297297297297p-7));
    emit(1, 4, (g[3] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(0x1.b6db6db6db6dbp-7)));
    emit(1, 5, (g[3] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(0x1.b6db6db6db6dbp-7)));
    emit(1, 6, (g[0] * T(-0x1.1d41d41d41d42p-5) + g[4] * T(0x1.f8af8af8af8b0p-5)));
    emit(1, 7, (g[0] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.1d41d41d41d42p-5)));
    emit(1, 8, (g[0] * T(-0x1.1d41d41d41d42p-5) + g[3] * T(0x1.f8af8af8af8b0p-5)));
    emit(1, 9, (g[0] * T(0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.1d41d41d41d42p-5)));
    emit(1, 10, (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)));
    emit(1, 11, (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)));
    emit(1, 12, (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)));
    emit(1, 13, (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)));
    emit(1, 14, (fma(g[4], T(0x1.1d41d41d41d42p-5), g[0] * T(0x1.8af8af8af8af9p-5)) + g[3] * T(0x1.1d41d41d41d42p-5)));
    emit(1, 15, (fma(g[4], T(-0x1.f8af8af8af8b0p-5), g[0] * T(-0x1.8af8af8af8af9p-4)) + g[3] * T(-0x1.f8af8af8af8b0p-5)));
    emit(1, 16, (fma(g[4], T(-0x1.0750750750750p-6), g[0] * T(0x1.0750750750750p-5)) + g[3] * T(-0x1.0750750750750p-6)));
    emit(1, 17, g[0] * T(-0x1.0750750750750p-5));
    emit(1, 18, (g[0] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.0750750750750p-6)));
    emit(1, 19, (g[0] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.0750750750750p-6)));
    emit(2, 2, g[1] * T(0x1.e79e79e79e79ep-5));
    emit(2, 3, g[5] * T(0x1.7297297297297p-7));
    emit(2, 4, (g[1] * T(-0x1.1d41d41d41d42p-5) + g[5] * T(0x1.f8af8af8af8b0p-5)));
    emit(2, 5, (g[1] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.1d41d41d41d42p-5)));
    emit(2, 6, (g[3] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)));
    emit(2, 7, (g[3] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)));
    emit(2, 8, (g[1] * T(0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.1d41d41d41d42p-5)));
    emit(2, 9, (g[1] * T(-0x1.1d41d41d41d42p-5) + g[3] * T(0x1.f8af8af8af8b0p-5)));
    emit(2, 10, (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)));
    emit(2, 11, (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)));
    emit(2, 12, (fma(g[5], T(0x1.1d41d41d41d42p-5), g[1] * T(0x1.8af8af8af8af9p-5)) + g[3] * T(0x1.1d41d41d41d42p-5)));
    emit(2, 13, (fma(g[5], T(-0x1.f8af8af8af8b0p-5), g[1] * T(-0x1.8af8af8af8af9p-4)) + g[3] * T(-0x1.f8af8af8af8b0p-5)));
    emit(2, 14, (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)));
    emit(2, 15, (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)));
    emit(2, 16, (fma(g[5], T(-0x1.0750750750750p-6), g[1] * T(0x1.0750750750750p-5)) + g[3] * T(-0x1.0750750750750p-6)));
    emit(2, 17, (g[1] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.0750750750750p-6)));
    emit(2, 18, g[1] * T(-0x1.0750750750750p-5));
    emit(2, 19, (g[1] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.0750750750750p-6)));
    emit(3, 3, g[2] * T(0x1.e79e79e79e79ep-5));
    emit(3, 4, (g[2] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.1d41d41d41d42p-5)));
    emit(3, 5, (g[2] * T(-0x1.1d41d41d41d42p-5) + g[5] * T(0x1.f8af8af8af8b0p-5)));
    emit(3, 6, (g[2] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.1d41d41d41d42p-5)));
    emit(3, 7, (g[2] * T(-0x1.1d41d41d41d42p-5) + g[4] * T(0x1.f8af8af8af8b0p-5)));
    emit(3, 8, (g[4] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)));
    emit(3, 9, (g[4] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)));
    emit(3, 10, (fma(g[5], T(0x1.1d41d41d41d42p-5), g[2] * T(0x1.8af8af8af8af9p-5)) + g[4] * T(0x1.1d41d41d41d42p-5)));
    emit(3, 11, (fma(g[5], T(-0x1.f8af8af8af8b0p-5), g[2] * T(-0x1.8af8af8af8af9p-4)) + g[4] * T(-0x1.f8af8af8af8b0p-5)));
    emit(3, 12, (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)));
    emit(3, 13, (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)));
    emit(3, 14, (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)));
    emit(3, 15, (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)));
    emit(3, 16, (fma(g[5], T(-0x1.0750750750750p-6), g[2] * T(0x1.0750750750750p-5)) + g[4] * T(-0x1.0750750750750p-6)));
    emit(3, 17, (g[2] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.0750750750750p-6)));
    emit(3, 18, (g[2] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.0750750750750p-6)));
    emit(3, 19, g[2] * T(-0x1.0750750750750p-5));
    emit(4, 4, (fma(g[5], T(0x1.8af8af8af8af9p-3), g[1] * T(0x1.edb6db6db6db7p-3)) + g[2] * T(0x1.8af8af8af8af9p-3)));
    emit(4, 5, (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(-0x1.283a83a83a83bp-4)) + g[2] * T(-0x1.283a83a83a83bp-4)));
    emit(4, 6, (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-5))));
    emit(4, 7, (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.283a83a83a83bp-4))));
    emit(4, 8, (fma(g[4], T(-0x1.283a83a83a83bp-4), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-5))));
    emit(4, 9, (fma(g[4], T(0x1.8af8af8af8af9p-3), g[1] * T(0x1.edb6db6db6db7p-4)) + fma(g[5], T(0x1.8af8af8af8af9p-4), g[3] * T(0x1.8af8af8af8af9p-4))));
    emit(4, 10, (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-5))));
    emit(4, 11, (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.283a83a83a83bp-4))));
    emit(4, 12, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(0x1.283a83a83a83bp-4), g[2] * T(0x1.283a83a83a83bp-4))));
    emit(4, 13, (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(-0x1.8af8af8af8af9p-3))));
    emit(4, 14, (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(4, 15, (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(4, 16, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[1] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))));
    emit(4, 17, (fma(g[4], T(-0x1.8af8af8af8af9p-4), g[1] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.edb6db6db6db7p-3))));
    emit(4, 18, (g[1] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.8af8af8af8af9p-5)));
    emit(4, 19, (fma(g[5], T(-0x1.edb6db6db6db7p-3), g[1] * T(-0x1.283a83a83a83bp-3)) + g[2] * T(-0x1.8af8af8af8af9p-4)));
    emit(5, 5, (fma(g[5], T(0x1.8af8af8af8af9p-3), g[1] * T(0x1.8af8af8af8af9p-3)) + g[2] * T(0x1.edb6db6db6db7p-3)));
    emit(5, 6, (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.283a83a83a83bp-4))));
    emit(5, 7, (fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.edb6db6db6db7p-4)) + fma(g[5], T(0x1.8af8af8af8af9p-4), g[3] * T(0x1.8af8af8af8af9p-3))));
    emit(5, 8, (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-6))));
    emit(5, 9, (fma(g[4], T(-0x1.283a83a83a83bp-4), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.8af8af8af8af9p-6))));
    emit(5, 10, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.283a83a83a83bp-4), g[1] * T(0x1.283a83a83a83bp-4))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-6))));
    emit(5, 11, (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-6))));
    emit(5, 12, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-6))));
    emit(5, 13, (fma(g[4], T(0x1.283a83a83a83bp-4), g[2] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-6))));
    emit(5, 14, (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(5, 15, (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(5, 16, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[2] * T(-0x1.8af8af8af8af9p-5))));
    emit(5, 17, (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[2] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.8af8af8af8af9p-4))));
    emit(5, 18, (fma(g[5], T(-0x1.edb6db6db6db7p-3), g[1] * T(-0x1.8af8af8af8af9p-4)) + g[2] * T(-0x1.283a83a83a83bp-3)));
    emit(5, 19, (g[2] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.8af8af8af8af9p-5)));
    emit(6, 6, (fma(g[4], T(0x1.8af8af8af8af9p-3), g[0] * T(0x1.edb6db6db6db7p-3)) + g[2] * T(0x1.8af8af8af8af9p-3)));
    emit(6, 7, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-4)) + g[2] * T(-0x1.283a83a83a83bp-4)));
    emit(6, 8, (fma(g[4], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.edb6db6db6db7p-4)) + fma(g[5], T(0x1.8af8af8af8af9p-3), g[3] * T(0x1.8af8af8af8af9p-4))));
    emit(6, 9, (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.283a83a83a83bp-4), g[3] * T(-0x1.8af8af8af8af9p-5))));
    emit(6, 10, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.8af8af8af8af9p-5))));
    emit(6, 11, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.283a83a83a83bp-4))));
    emit(6, 12, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(6, 13, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(6, 14, (fma(g[5], T(0x1.283a83a83a83bp-4), fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.283a83a83a83bp-4))));
    emit(6, 15, (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(-0x1.8af8af8af8af9p-3))));
    emit(6, 16, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))));
    emit(6, 17, (g[0] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.8af8af8af8af9p-5)));
    emit(6, 18, (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.8af8af8af8af9p-4), g[3] * T(-0x1.edb6db6db6db7p-3))));
    emit(6, 19, (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-3)) + g[2] * T(-0x1.8af8af8af8af9p-4)));
    emit(7, 7, (fma(g[4], T(0x1.8af8af8af8af9p-3), g[0] * T(0x1.8af8af8af8af9p-3)) + g[2] * T(0x1.edb6db6db6db7p-3)));
    emit(7, 8, (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.283a83a83a83bp-4), g[3] * T(-0x1.8af8af8af8af9p-6))));
    emit(7, 9, (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.8af8af8af8af9p-6))));
    emit(7, 10, (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.283a83a83a83bp-4), g[0] * T(0x1.283a83a83a83bp-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-6))));
    emit(7, 11, (fma(g[5], T(-0x1.8af8af8af8af9p-4), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.8af8af8af8af9p-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(0x1.8af8af8af8af9p-6))));
    emit(7, 12, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(7, 13, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)));
    emit(7, 14, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-6))));
    emit(7, 15, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.283a83a83a83bp-4), g[3] * T(0x1.8af8af8af8af9p-6))));
    emit(7, 16, (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(-0x1.8af8af8af8af9p-5))));
    emit(7, 17, (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-4)) + g[2] * T(-0x1.283a83a83a83bp-3)));
    emit(7, 18, (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[2] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.8af8af8af8af9p-4))));
    emit(7, 19, (g[2] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.8af8af8af8af9p-5)));
    emit(8, 8, (fma(g[3], T(0x1.8af8af8af8af9p-3), g[0] * T(0x1.edb6db6db6db7p-3)) + g[1] * T(0x1.8af8af8af8af9p-3)));
    emit(8, 9, (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-4)) + g[1] * T(-0x1.283a83a83a83bp-4)));
    emit(8, 10, (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)));
    emit(8, 11, (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)));
    emit(8, 12, (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.8af8af8af8af9p-5))));
    emit(8, 13, (fma(g[4], T(0x1.283a83a83a83bp-4), g[0] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.8af8af8af8af9p-5))));
    emit(8, 14, (fma(g[5], T(0x1.283a83a83a83bp-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.283a83a83a83bp-4))));
    emit(8, 15, (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(-0x1.8af8af8af8af9p-4), g[1] * T(-0x1.8af8af8af8af9p-3))));
    emit(8, 16, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[1] * T(0x1.8af8af8af8af9p-4))));
    emit(8, 17, (g[0] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.8af8af8af8af9p-5)));
    emit(8, 18, (fma(g[3], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-3)) + g[1] * T(-0x1.8af8af8af8af9p-4)));
    emit(8, 19, (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.8af8af8af8af9p-4), g[3] * T(-0x1.edb6db6db6db7p-3))));
    emit(9, 9, (fma(g[3], T(0x1.8af8af8af8af9p-3), g[0] * T(0x1.8af8af8af8af9p-3)) + g[1] * T(0x1.edb6db6db6db7p-3)));
    emit(9, 10, (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)));
    emit(9, 11, (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)));
    emit(9, 12, (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.283a83a83a83bp-4))) + fma(g[4], T(0x1.283a83a83a83bp-4), g[1] * T(0x1.8af8af8af8af9p-6))));
    emit(9, 13, (fma(g[5], T(-0x1.8af8af8af8af9p-4), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.8af8af8af8af9p-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[1] * T(0x1.8af8af8af8af9p-6))));
    emit(9, 14, (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-5))));
    emit(9, 15, (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.283a83a83a83bp-4), g[3] * T(0x1.8af8af8af8af9p-5))));
    emit(9, 16, (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[1] * T(-0x1.8af8af8af8af9p-5))));
    emit(9, 17, (fma(g[3], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-4)) + g[1] * T(-0x1.283a83a83a83bp-3)));
    emit(9, 18, (g[1] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.8af8af8af8af9p-5)));
    emit(9, 19, (fma(g[4], T(-0x1.8af8af8af8af9p-4), g[1] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.edb6db6db6db7p-3))));
    emit(10, 10, (fma(g[4], T(0x1.283a83a83a83bp-2), fma(g[2], T(0x1.edb6db6db6db7p-3), g[0] * T(0x1.edb6db6db6db7p-3))) + fma(g[5], T(0x1.283a83a83a83bp-2), fma(g[3], T(0x1.edb6db6db6db7p-2), g[1] * T(0x1.edb6db6db6db7p-3)))));
    emit(10, 11, (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.283a83a83a83bp-4))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.283a83a83a83bp-3), g[1] * T(-0x1.283a83a83a83bp-4)))));
    emit(10, 12, (fma(g[4], T(0x1.283a83a83a83bp-3), fma(g[2], T(0x1.8af8af8af8af9p-6), g[0] * T(0x1.edb6db6db6db7p-4))) + fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.283a83a83a83bp-3), g[1] * T(0x1.8af8af8af8af9p-6)))));
    emit(10, 13, (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6))));
    emit(10, 14, (fma(g[4], T(0x1.edb6db6db6db7p-3), fma(g[2], T(0x1.8af8af8af8af9p-6), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[5], T(0x1.283a83a83a83bp-3), fma(g[3], T(0x1.283a83a83a83bp-3), g[1] * T(0x1.edb6db6db6db7p-4)))));
    emit(10, 15, (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[1] * T(-0x1.8af8af8af8af9p-6))));
    emit(10, 16, (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-5))));
    emit(10, 17, (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.283a83a83a83bp-2)))));
    emit(10, 18, (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-2))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.8af8af8af8af9p-5)))));
    emit(10, 19, (fma(g[5], T(-0x1.8af8af8af8af9p-5), fma(g[3], T(-0x1.283a83a83a83bp-2), g[0] * T(-0x1.283a83a83a83bp-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.283a83a83a83bp-3))));
    emit(11, 11, (fma(g[4], T(0x1.8af8af8af8af9p-3), fma(g[2], T(0x1.edb6db6db6db7p-3), g[0] * T(0x1.8af8af8af8af9p-3))) + fma(g[5], T(0x1.8af8af8af8af9p-3), fma(g[3], T(0x1.8af8af8af8af9p-2), g[1] * T(0x1.8af8af8af8af9p-3)))));
    emit(11, 12, (fma(g[3], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-6))));
    emit(11, 13, (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.8af8af8af8af9p-6))));
    emit(11, 14, (fma(g[3], T(-0x1.8af8af8af8af9p-6), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[4], T(-0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-6))));
    emit(11, 15, (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-6))));
    emit(11, 16, (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-4))));
    emit(11, 17, (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(-0x1.8af8af8af8af9p-5))));
    emit(11, 18, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[2] * T(-0x1.8af8af8af8af9p-5))));
    emit(11, 19, (g[4] * T(-0x1.8af8af8af8af9p-5) + g[5] * T(-0x1.8af8af8af8af9p-5)));
    emit(12, 12, (fma(g[4], T(0x1.edb6db6db6db7p-2), fma(g[2], T(0x1.edb6db6db6db7p-3), g[0] * T(0x1.edb6db6db6db7p-3))) + fma(g[5], T(0x1.283a83a83a83bp-2), fma(g[3], T(0x1.283a83a83a83bp-2), g[1] * T(0x1.edb6db6db6db7p-3)))));
    emit(12, 13, (fma(g[4], T(-0x1.283a83a83a83bp-3), fma(g[2], T(-0x1.283a83a83a83bp-4), g[0] * T(-0x1.283a83a83a83bp-4))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-3)))));
    emit(12, 14, (fma(g[4], T(0x1.283a83a83a83bp-3), fma(g[2], T(0x1.edb6db6db6db7p-4), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[5], T(0x1.283a83a83a83bp-3), fma(g[3], T(0x1.edb6db6db6db7p-3), g[1] * T(0x1.8af8af8af8af9p-6)))));
    emit(12, 15, (fma(g[3], T(-0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6))));
    emit(12, 16, (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-5))));
    emit(12, 17, (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.283a83a83a83bp-2), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-5)))));
    emit(12, 18, (fma(g[5], T(-0x1.8af8af8af8af9p-5), fma(g[3], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-3))) + fma(g[4], T(-0x1.283a83a83a83bp-2), g[2] * T(-0x1.283a83a83a83bp-3))));
    emit(12, 19, (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-2))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.8af8af8af8af9p-5)))));
    emit(13, 13, (fma(g[4], T(0x1.8af8af8af8af9p-2), fma(g[2], T(0x1.8af8af8af8af9p-3), g[0] * T(0x1.8af8af8af8af9p-3))) + fma(g[5], T(0x1.8af8af8af8af9p-3), fma(g[3], T(0x1.8af8af8af8af9p-3), g[1] * T(0x1.edb6db6db6db7p-3)))));
    emit(13, 14, (fma(g[3], T(-0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6))));
    emit(13, 15, (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-5))));
    emit(13, 16, (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-4))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(-0x1.8af8af8af8af9p-4))));
    emit(13, 17, (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[1] * T(-0x1.8af8af8af8af9p-5))));
    emit(13, 18, (g[3] * T(-0x1.8af8af8af8af9p-5) + g[5] * T(-0x1.8af8af8af8af9p-5)));
    emit(13, 19, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[1] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))));
    emit(14, 14, (fma(g[4], T(0x1.283a83a83a83bp-2), fma(g[2], T(0x1.edb6db6db6db7p-3), g[0] * T(0x1.edb6db6db6db7p-3))) + fma(g[5], T(0x1.edb6db6db6db7p-2), fma(g[3], T(0x1.283a83a83a83bp-2), g[1] * T(0x1.edb6db6db6db7p-3)))));
    emit(14, 15, (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.283a83a83a83bp-4), g[0] * T(-0x1.8af8af8af8af9p-3))) + fma(g[5], T(-0x1.283a83a83a83bp-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.283a83a83a83bp-4)))));
    emit(14, 16, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-5))));
    emit(14, 17, (fma(g[5], T(-0x1.283a83a83a83bp-2), fma(g[3], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.283a83a83a83bp-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-5), g[2] * T(-0x1.283a83a83a83bp-3))));
    emit(14, 18, (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.283a83a83a83bp-2), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-5)))));
    emit(14, 19, (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.283a83a83a83bp-2)))));
    emit(15, 15, (fma(g[4], T(0x1.8af8af8af8af9p-3), fma(g[2], T(0x1.8af8af8af8af9p-3), g[0] * T(0x1.edb6db6db6db7p-3))) + fma(g[5], T(0x1.8af8af8af8af9p-2), fma(g[3], T(0x1.8af8af8af8af9p-3), g[1] * T(0x1.8af8af8af8af9p-3)))));
    emit(15, 16, (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(-0x1.8af8af8af8af9p-4))));
    emit(15, 17, (g[3] * T(-0x1.8af8af8af8af9p-5) + g[4] * T(-0x1.8af8af8af8af9p-5)));
    emit(15, 18, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[1] * T(0x1.8af8af8af8af9p-4))));
    emit(15, 19, (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))));
    emit(16, 16, (fma(g[4], T(0x1.283a83a83a83bp-1), fma(g[2], T(0x1.283a83a83a83bp-1), g[0] * T(0x1.283a83a83a83bp-1))) + fma(g[5], T(0x1.283a83a83a83bp-1), fma(g[3], T(0x1.283a83a83a83bp-1), g[1] * T(0x1.283a83a83a83bp-1)))));
    emit(16, 17, (fma(g[4], T(-0x1.283a83a83a83bp-1), g[0] * T(-0x1.283a83a83a83bp-1)) + fma(g[5], T(-0x1.283a83a83a83bp-2), g[3] * T(-0x1.283a83a83a83bp-1))));
    emit(16, 18, (fma(g[4], T(-0x1.283a83a83a83bp-2), g[1] * T(-0x1.283a83a83a83bp-1)) + fma(g[5], T(-0x1.283a83a83a83bp-1), g[3] * T(-0x1.283a83a83a83bp-1))));
    emit(16, 19, (fma(g[4], T(-0x1.283a83a83a83bp-1), g[2] * T(-0x1.283a83a83a83bp-1)) + fma(g[5], T(-0x1.283a83a83a83bp-1), g[3] * T(-0x1.283a83a83a83bp-2))));
    emit(17, 17, (fma(g[4], T(0x1.283a83a83a83bp-1), fma(g[2], T(0x1.283a83a83a83bp-1), g[0] * T(0x1.283a83a83a83bp-1))) + fma(g[5], T(0x1.283a83a83a83bp-1), fma(g[3], T(0x1.283a83a83a83bp-1), g[1] * T(0x1.283a83a83a83bp-1)))));
    emit(17, 18, (fma(g[4], T(0x1.283a83a83a83bp-2), g[2] * T(0x1.283a83a83a83bp-2)) + fma(g[5], T(0x1.283a83a83a83bp-2), g[3] * T(0x1.283a83a83a83bp-1))));
    emit(17, 19, (fma(g[4], T(0x1.283a83a83a83bp-1), g[1] * T(0x1.283a83a83a83bp-2)) + fma(g[5], T(0x1.283a83a83a83bp-2), g[3] * T(0x1.283a83a83a83bp-2))));
    emit(18, 18, (fma(g[4], T(0x1.283a83a83a83bp-1), fma(g[2], T(0x1.283a83a83a83bp-1), g[0] * T(0x1.283a83a83a83bp-1))) + fma(g[5], T(0x1.283a83a83a83bp-1), fma(g[3], T(0x1.283a83a83a83bp-1), g[1] * T(0x1.283a83a83a83bp-1)))));
    emit(18, 19, (fma(g[4], T(0x1.283a83a83a83bp-2), g[0] * T(0x1.283a83a83a83bp-2)) + fma(g[5], T(0x1.283a83a83a83bp-1), g[3] * T(0x1.283a83a83a83bp-2))));
    emit(19, 19, (fma(g[4], T(0x1.283a83a83a83bp-1), fma(g[2], T(0x1.283a83a83a83bp-1), g[0] * T(0x1.283a83a83a83bp-1))) + fma(g[5], T(0x1.283a83a83a83bp-1), fma(g[3], T(0x1.283a83a83a83bp-1), g[1] * T(0x1.283a83a83a83bp-1)))));
  } else {
    double rs[20] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    { const T v = (fma(g[4], T(-0x1.7297297297297p-7), g[0] * T(-0x1.7297297297297p-7)) + g[3] * T(-0x1.7297297297297p-7)); rs[0] += (double)v; rs[1] += (double)v; emit(0, 1, v); }
    { const T v = (fma(g[5], T(-0x1.7297297297297p-7), g[1] * T(-0x1.7297297297297p-7)) + g[3] * T(-0x1.7297297297297p-7)); rs[0] += (double)v; rs[2] += (double)v; emit(0, 2, v); }
    { const T v = (fma(g[5], T(-0x1.7297297297297p-7), g[2] * T(-0x1.7297297297297p-7)) + g[4] * T(-0x1.7297297297297p-7)); rs[0] += (double)v; rs[3] += (double)v; emit(0, 3, v); }
    { const T v = (fma(g[5], T(-0x1.b6db6db6db6dbp-6), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[2] * T(-0x1.b6db6db6db6dbp-7))); rs[0] += (double)v; rs[4] += (double)v; emit(0, 4, v); }
    { const T v = (fma(g[5], T(-0x1.b6db6db6db6dbp-6), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[2] * T(-0x1.b6db6db6db6dbp-7))); rs[0] += (double)v; rs[5] += (double)v; emit(0, 5, v); }
    { const T v = (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-6), g[2] * T(-0x1.b6db6db6db6dbp-7))); rs[0] += (double)v; rs[6] += (double)v; emit(0, 6, v); }
    { const T v = (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-7), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-6), g[2] * T(-0x1.b6db6db6db6dbp-7))); rs[0] += (double)v; rs[7] += (double)v; emit(0, 7, v); }
    { const T v = (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-6), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))); rs[0] += (double)v; rs[8] += (double)v; emit(0, 8, v); }
    { const T v = (fma(g[5], T(-0x1.b6db6db6db6dbp-7), fma(g[3], T(-0x1.b6db6db6db6dbp-6), g[0] * T(-0x1.b6db6db6db6dbp-7))) + fma(g[4], T(-0x1.b6db6db6db6dbp-7), g[1] * T(-0x1.b6db6db6db6dbp-7))); rs[0] += (double)v; rs[9] += (double)v; emit(0, 9, v); }
    { const T v = (fma(g[4], T(-0x1.0cccccccccccdp-3), fma(g[2], T(-0x1.8af8af8af8af9p-4), g[0] * T(-0x1.1d41d41d41d42p-5))) + fma(g[5], T(-0x1.0cccccccccccdp-3), fma(g[3], T(-0x1.1d41d41d41d42p-4), g[1] * T(-0x1.1d41d41d41d42p-5)))); rs[0] += (double)v; rs[10] += (double)v; emit(0, 10, v); }
    { const T v = (fma(g[4], T(0x1.f8af8af8af8b0p-5), fma(g[2], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.b6db6db6db6dbp-7))) + fma(g[5], T(0x1.f8af8af8af8b0p-5), fma(g[3], T(0x1.b6db6db6db6dbp-6), g[1] * T(0x1.b6db6db6db6dbp-7)))); rs[0] += (double)v; rs[11] += (double)v; emit(0, 11, v); }
    { const T v = (fma(g[4], T(-0x1.1d41d41d41d42p-4), fma(g[2], T(-0x1.1d41d41d41d42p-5), g[0] * T(-0x1.1d41d41d41d42p-5))) + fma(g[5], T(-0x1.0cccccccccccdp-3), fma(g[3], T(-0x1.0cccccccccccdp-3), g[1] * T(-0x1.8af8af8af8af9p-4)))); rs[0] += (double)v; rs[12] += (double)v; emit(0, 12, v); }
    { const T v = (fma(g[4], T(0x1.b6db6db6db6dbp-6), fma(g[2], T(0x1.b6db6db6db6dbp-7), g[0] * T(0x1.b6db6db6db6dbp-7))) + fma(g[5], T(0x1.f8af8af8af8b0p-5), fma(g[3], T(0x1.f8af8af8af8b0p-5), g[1] * T(0x1.8af8af8af8af9p-5)))); rs[0] += (double)v; rs[13] += (double)v; emit(0, 13, v); }
    { const T v = (fma(g[4], T(-0x1.0cccccccccccdp-3), fma(g[2], T(-0x1.1d41d41d41d42p-5), g[0] * T(-0x1.8af8af8af8af9p-4))) + fma(g[5], T(-0x1.1d41d41d41d42p-4), fma(g[3], T(-0x1.0cccccccccccdp-3), g[1] * T(-0x1.1d41d41d41d42p-5)))); rs[0] += (double)v; rs[14] += (double)v; emit(0, 14, v); }
    { const T v = (fma(g[4], T(0x1.f8af8af8af8b0p-5), fma(g[2], T(0x1.b6db6db6db6dbp-7), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[5], T(0x1.b6db6db6db6dbp-6), fma(g[3], T(0x1.f8af8af8af8b0p-5), g[1] * T(0x1.b6db6db6db6dbp-7)))); rs[0] += (double)v; rs[15] += (double)v; emit(0, 15, v); }
    { const T v = (fma(g[4], T(-0x1.0750750750750p-4), fma(g[2], T(-0x1.0750750750750p-5), g[0] * T(-0x1.0750750750750p-5))) + fma(g[5], T(-0x1.0750750750750p-4), fma(g[3], T(-0x1.0750750750750p-4), g[1] * T(-0x1.0750750750750p-5)))); rs[0] += (double)v; rs[16] += (double)v; emit(0, 16, v); }
    { const T v = (fma(g[4], T(0x1.4924924924925p-4), fma(g[2], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.0750750750750p-5))) + fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.4924924924925p-4), g[1] * T(0x1.8af8af8af8af9p-5)))); rs[0] += (double)v; rs[17] += (double)v; emit(0, 17, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-4), fma(g[2], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[5], T(0x1.4924924924925p-4), fma(g[3], T(0x1.4924924924925p-4), g[1] * T(0x1.0750750750750p-5)))); rs[0] += (double)v; rs[18] += (double)v; emit(0, 18, v); }
    { const T v = (fma(g[4], T(0x1.4924924924925p-4), fma(g[2], T(0x1.0750750750750p-5), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[5], T(0x1.4924924924925p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-5)))); rs[0] += (double)v; rs[19] += (double)v; emit(0, 19, v); }
    { const T v = g[3] * T(0x1.7297297297297p-7); rs[1] += (double)v; rs[2] += (double)v; emit(1, 2, v); }
    { const T v = g[4] * T(0x1.7297297297297p-7); rs[1] += (double)v; rs[3] += (double)v; emit(1, 3, v); }
    { const T v = (g[3] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(0x1.b6db6db6db6dbp-7)); rs[1] += (double)v; rs[4] += (double)v; emit(1, 4, v); }
    { const T v = (g[3] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(0x1.b6db6db6db6dbp-7)); rs[1] += (double)v; rs[5] += (double)v; emit(1, 5, v); }
    { const T v = (g[0] * T(-0x1.1d41d41d41d42p-5) + g[4] * T(0x1.f8af8af8af8b0p-5)); rs[1] += (double)v; rs[6] += (double)v; emit(1, 6, v); }
    { const T v = (g[0] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.1d41d41d41d42p-5)); rs[1] += (double)v; rs[7] += (double)v; emit(1, 7, v); }
    { const T v = (g[0] * T(-0x1.1d41d41d41d42p-5) + g[3] * T(0x1.f8af8af8af8b0p-5)); rs[1] += (double)v; rs[8] += (double)v; emit(1, 8, v); }
    { const T v = (g[0] * T(0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.1d41d41d41d42p-5)); rs[1] += (double)v; rs[9] += (double)v; emit(1, 9, v); }
    { const T v = (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)); rs[1] += (double)v; rs[10] += (double)v; emit(1, 10, v); }
    { const T v = (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)); rs[1] += (double)v; rs[11] += (double)v; emit(1, 11, v); }
    { const T v = (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)); rs[1] += (double)v; rs[12] += (double)v; emit(1, 12, v); }
    { const T v = (g[0] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)); rs[1] += (double)v; rs[13] += (double)v; emit(1, 13, v); }
    { const T v = (fma(g[4], T(0x1.1d41d41d41d42p-5), g[0] * T(0x1.8af8af8af8af9p-5)) + g[3] * T(0x1.1d41d41d41d42p-5)); rs[1] += (double)v; rs[14] += (double)v; emit(1, 14, v); }
    { const T v = (fma(g[4], T(-0x1.f8af8af8af8b0p-5), g[0] * T(-0x1.8af8af8af8af9p-4)) + g[3] * T(-0x1.f8af8af8af8b0p-5)); rs[1] += (double)v; rs[15] += (double)v; emit(1, 15, v); }
    { const T v = (fma(g[4], T(-0x1.0750750750750p-6), g[0] * T(0x1.0750750750750p-5)) + g[3] * T(-0x1.0750750750750p-6)); rs[1] += (double)v; rs[16] += (double)v; emit(1, 16, v); }
    { const T v = g[0] * T(-0x1.0750750750750p-5); rs[1] += (double)v; rs[17] += (double)v; emit(1, 17, v); }
    { const T v = (g[0] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.0750750750750p-6)); rs[1] += (double)v; rs[18] += (double)v; emit(1, 18, v); }
    { const T v = (g[0] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.0750750750750p-6)); rs[1] += (double)v; rs[19] += (double)v; emit(1, 19, v); }
    { const T v = g[5] * T(0x1.7297297297297p-7); rs[2] += (double)v; rs[3] += (double)v; emit(2, 3, v); }
    { const T v = (g[1] * T(-0x1.1d41d41d41d42p-5) + g[5] * T(0x1.f8af8af8af8b0p-5)); rs[2] += (double)v; rs[4] += (double)v; emit(2, 4, v); }
    { const T v = (g[1] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.1d41d41d41d42p-5)); rs[2] += (double)v; rs[5] += (double)v; emit(2, 5, v); }
    { const T v = (g[3] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)); rs[2] += (double)v; rs[6] += (double)v; emit(2, 6, v); }
    { const T v = (g[3] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)); rs[2] += (double)v; rs[7] += (double)v; emit(2, 7, v); }
    { const T v = (g[1] * T(0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.1d41d41d41d42p-5)); rs[2] += (double)v; rs[8] += (double)v; emit(2, 8, v); }
    { const T v = (g[1] * T(-0x1.1d41d41d41d42p-5) + g[3] * T(0x1.f8af8af8af8b0p-5)); rs[2] += (double)v; rs[9] += (double)v; emit(2, 9, v); }
    { const T v = (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)); rs[2] += (double)v; rs[10] += (double)v; emit(2, 10, v); }
    { const T v = (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[3] * T(-0x1.b6db6db6db6dbp-7)); rs[2] += (double)v; rs[11] += (double)v; emit(2, 11, v); }
    { const T v = (fma(g[5], T(0x1.1d41d41d41d42p-5), g[1] * T(0x1.8af8af8af8af9p-5)) + g[3] * T(0x1.1d41d41d41d42p-5)); rs[2] += (double)v; rs[12] += (double)v; emit(2, 12, v); }
    { const T v = (fma(g[5], T(-0x1.f8af8af8af8b0p-5), g[1] * T(-0x1.8af8af8af8af9p-4)) + g[3] * T(-0x1.f8af8af8af8b0p-5)); rs[2] += (double)v; rs[13] += (double)v; emit(2, 13, v); }
    { const T v = (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)); rs[2] += (double)v; rs[14] += (double)v; emit(2, 14, v); }
    { const T v = (g[1] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)); rs[2] += (double)v; rs[15] += (double)v; emit(2, 15, v); }
    { const T v = (fma(g[5], T(-0x1.0750750750750p-6), g[1] * T(0x1.0750750750750p-5)) + g[3] * T(-0x1.0750750750750p-6)); rs[2] += (double)v; rs[16] += (double)v; emit(2, 16, v); }
    { const T v = (g[1] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.0750750750750p-6)); rs[2] += (double)v; rs[17] += (double)v; emit(2, 17, v); }
    { const T v = g[1] * T(-0x1.0750750750750p-5); rs[2] += (double)v; rs[18] += (double)v; emit(2, 18, v); }
    { const T v = (g[1] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.0750750750750p-6)); rs[2] += (double)v; rs[19] += (double)v; emit(2, 19, v); }
    { const T v = (g[2] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.1d41d41d41d42p-5)); rs[3] += (double)v; rs[4] += (double)v; emit(3, 4, v); }
    { const T v = (g[2] * T(-0x1.1d41d41d41d42p-5) + g[5] * T(0x1.f8af8af8af8b0p-5)); rs[3] += (double)v; rs[5] += (double)v; emit(3, 5, v); }
    { const T v = (g[2] * T(0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.1d41d41d41d42p-5)); rs[3] += (double)v; rs[6] += (double)v; emit(3, 6, v); }
    { const T v = (g[2] * T(-0x1.1d41d41d41d42p-5) + g[4] * T(0x1.f8af8af8af8b0p-5)); rs[3] += (double)v; rs[7] += (double)v; emit(3, 7, v); }
    { const T v = (g[4] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)); rs[3] += (double)v; rs[8] += (double)v; emit(3, 8, v); }
    { const T v = (g[4] * T(0x1.b6db6db6db6dbp-7) + g[5] * T(0x1.b6db6db6db6dbp-7)); rs[3] += (double)v; rs[9] += (double)v; emit(3, 9, v); }
    { const T v = (fma(g[5], T(0x1.1d41d41d41d42p-5), g[2] * T(0x1.8af8af8af8af9p-5)) + g[4] * T(0x1.1d41d41d41d42p-5)); rs[3] += (double)v; rs[10] += (double)v; emit(3, 10, v); }
    { const T v = (fma(g[5], T(-0x1.f8af8af8af8b0p-5), g[2] * T(-0x1.8af8af8af8af9p-4)) + g[4] * T(-0x1.f8af8af8af8b0p-5)); rs[3] += (double)v; rs[11] += (double)v; emit(3, 11, v); }
    { const T v = (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)); rs[3] += (double)v; rs[12] += (double)v; emit(3, 12, v); }
    { const T v = (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[4] * T(-0x1.b6db6db6db6dbp-7)); rs[3] += (double)v; rs[13] += (double)v; emit(3, 13, v); }
    { const T v = (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)); rs[3] += (double)v; rs[14] += (double)v; emit(3, 14, v); }
    { const T v = (g[2] * T(-0x1.b6db6db6db6dbp-7) + g[5] * T(-0x1.b6db6db6db6dbp-7)); rs[3] += (double)v; rs[15] += (double)v; emit(3, 15, v); }
    { const T v = (fma(g[5], T(-0x1.0750750750750p-6), g[2] * T(0x1.0750750750750p-5)) + g[4] * T(-0x1.0750750750750p-6)); rs[3] += (double)v; rs[16] += (double)v; emit(3, 16, v); }
    { const T v = (g[2] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.0750750750750p-6)); rs[3] += (double)v; rs[17] += (double)v; emit(3, 17, v); }
    { const T v = (g[2] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.0750750750750p-6)); rs[3] += (double)v; rs[18] += (double)v; emit(3, 18, v); }
    { const T v = g[2] * T(-0x1.0750750750750p-5); rs[3] += (double)v; rs[19] += (double)v; emit(3, 19, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(-0x1.283a83a83a83bp-4)) + g[2] * T(-0x1.283a83a83a83bp-4)); rs[4] += (double)v; rs[5] += (double)v; emit(4, 5, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-5))); rs[4] += (double)v; rs[6] += (double)v; emit(4, 6, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.283a83a83a83bp-4))); rs[4] += (double)v; rs[7] += (double)v; emit(4, 7, v); }
    { const T v = (fma(g[4], T(-0x1.283a83a83a83bp-4), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-5))); rs[4] += (double)v; rs[8] += (double)v; emit(4, 8, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-3), g[1] * T(0x1.edb6db6db6db7p-4)) + fma(g[5], T(0x1.8af8af8af8af9p-4), g[3] * T(0x1.8af8af8af8af9p-4))); rs[4] += (double)v; rs[9] += (double)v; emit(4, 9, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-5))); rs[4] += (double)v; rs[10] += (double)v; emit(4, 10, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.283a83a83a83bp-4))); rs[4] += (double)v; rs[11] += (double)v; emit(4, 11, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(0x1.283a83a83a83bp-4), g[2] * T(0x1.283a83a83a83bp-4))); rs[4] += (double)v; rs[12] += (double)v; emit(4, 12, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(-0x1.8af8af8af8af9p-3))); rs[4] += (double)v; rs[13] += (double)v; emit(4, 13, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[4] += (double)v; rs[14] += (double)v; emit(4, 14, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[4] += (double)v; rs[15] += (double)v; emit(4, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[1] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))); rs[4] += (double)v; rs[16] += (double)v; emit(4, 16, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-4), g[1] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.edb6db6db6db7p-3))); rs[4] += (double)v; rs[17] += (double)v; emit(4, 17, v); }
    { const T v = (g[1] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.8af8af8af8af9p-5)); rs[4] += (double)v; rs[18] += (double)v; emit(4, 18, v); }
    { const T v = (fma(g[5], T(-0x1.edb6db6db6db7p-3), g[1] * T(-0x1.283a83a83a83bp-3)) + g[2] * T(-0x1.8af8af8af8af9p-4)); rs[4] += (double)v; rs[19] += (double)v; emit(4, 19, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.283a83a83a83bp-4))); rs[5] += (double)v; rs[6] += (double)v; emit(5, 6, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.edb6db6db6db7p-4)) + fma(g[5], T(0x1.8af8af8af8af9p-4), g[3] * T(0x1.8af8af8af8af9p-3))); rs[5] += (double)v; rs[7] += (double)v; emit(5, 7, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-6))); rs[5] += (double)v; rs[8] += (double)v; emit(5, 8, v); }
    { const T v = (fma(g[4], T(-0x1.283a83a83a83bp-4), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.8af8af8af8af9p-6))); rs[5] += (double)v; rs[9] += (double)v; emit(5, 9, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.283a83a83a83bp-4), g[1] * T(0x1.283a83a83a83bp-4))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-6))); rs[5] += (double)v; rs[10] += (double)v; emit(5, 10, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-6))); rs[5] += (double)v; rs[11] += (double)v; emit(5, 11, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-6))); rs[5] += (double)v; rs[12] += (double)v; emit(5, 12, v); }
    { const T v = (fma(g[4], T(0x1.283a83a83a83bp-4), g[2] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-6))); rs[5] += (double)v; rs[13] += (double)v; emit(5, 13, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[5] += (double)v; rs[14] += (double)v; emit(5, 14, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[5] += (double)v; rs[15] += (double)v; emit(5, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[2] * T(-0x1.8af8af8af8af9p-5))); rs[5] += (double)v; rs[16] += (double)v; emit(5, 16, v); }
    { const T v = (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[2] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.8af8af8af8af9p-4))); rs[5] += (double)v; rs[17] += (double)v; emit(5, 17, v); }
    { const T v = (fma(g[5], T(-0x1.edb6db6db6db7p-3), g[1] * T(-0x1.8af8af8af8af9p-4)) + g[2] * T(-0x1.283a83a83a83bp-3)); rs[5] += (double)v; rs[18] += (double)v; emit(5, 18, v); }
    { const T v = (g[2] * T(0x1.8af8af8af8af9p-5) + g[5] * T(0x1.8af8af8af8af9p-5)); rs[5] += (double)v; rs[19] += (double)v; emit(5, 19, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-4)) + g[2] * T(-0x1.283a83a83a83bp-4)); rs[6] += (double)v; rs[7] += (double)v; emit(6, 7, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.edb6db6db6db7p-4)) + fma(g[5], T(0x1.8af8af8af8af9p-3), g[3] * T(0x1.8af8af8af8af9p-4))); rs[6] += (double)v; rs[8] += (double)v; emit(6, 8, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.283a83a83a83bp-4), g[3] * T(-0x1.8af8af8af8af9p-5))); rs[6] += (double)v; rs[9] += (double)v; emit(6, 9, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.8af8af8af8af9p-5))); rs[6] += (double)v; rs[10] += (double)v; emit(6, 10, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.283a83a83a83bp-4))); rs[6] += (double)v; rs[11] += (double)v; emit(6, 11, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[6] += (double)v; rs[12] += (double)v; emit(6, 12, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[6] += (double)v; rs[13] += (double)v; emit(6, 13, v); }
    { const T v = (fma(g[5], T(0x1.283a83a83a83bp-4), fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.283a83a83a83bp-4))); rs[6] += (double)v; rs[14] += (double)v; emit(6, 14, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(-0x1.8af8af8af8af9p-3))); rs[6] += (double)v; rs[15] += (double)v; emit(6, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))); rs[6] += (double)v; rs[16] += (double)v; emit(6, 16, v); }
    { const T v = (g[0] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.8af8af8af8af9p-5)); rs[6] += (double)v; rs[17] += (double)v; emit(6, 17, v); }
    { const T v = (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.8af8af8af8af9p-4), g[3] * T(-0x1.edb6db6db6db7p-3))); rs[6] += (double)v; rs[18] += (double)v; emit(6, 18, v); }
    { const T v = (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-3)) + g[2] * T(-0x1.8af8af8af8af9p-4)); rs[6] += (double)v; rs[19] += (double)v; emit(6, 19, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.283a83a83a83bp-4), g[3] * T(-0x1.8af8af8af8af9p-6))); rs[7] += (double)v; rs[8] += (double)v; emit(7, 8, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.8af8af8af8af9p-6))); rs[7] += (double)v; rs[9] += (double)v; emit(7, 9, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.283a83a83a83bp-4), g[0] * T(0x1.283a83a83a83bp-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-6))); rs[7] += (double)v; rs[10] += (double)v; emit(7, 10, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-4), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.8af8af8af8af9p-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(0x1.8af8af8af8af9p-6))); rs[7] += (double)v; rs[11] += (double)v; emit(7, 11, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[7] += (double)v; rs[12] += (double)v; emit(7, 12, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[2] * T(0x1.8af8af8af8af9p-6)); rs[7] += (double)v; rs[13] += (double)v; emit(7, 13, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-6))); rs[7] += (double)v; rs[14] += (double)v; emit(7, 14, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.283a83a83a83bp-4), g[3] * T(0x1.8af8af8af8af9p-6))); rs[7] += (double)v; rs[15] += (double)v; emit(7, 15, v); }
    { const T v = (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(-0x1.8af8af8af8af9p-5))); rs[7] += (double)v; rs[16] += (double)v; emit(7, 16, v); }
    { const T v = (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-4)) + g[2] * T(-0x1.283a83a83a83bp-3)); rs[7] += (double)v; rs[17] += (double)v; emit(7, 17, v); }
    { const T v = (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[2] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.8af8af8af8af9p-4))); rs[7] += (double)v; rs[18] += (double)v; emit(7, 18, v); }
    { const T v = (g[2] * T(0x1.8af8af8af8af9p-5) + g[4] * T(0x1.8af8af8af8af9p-5)); rs[7] += (double)v; rs[19] += (double)v; emit(7, 19, v); }
    { const T v = (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-4)) + g[1] * T(-0x1.283a83a83a83bp-4)); rs[8] += (double)v; rs[9] += (double)v; emit(8, 9, v); }
    { const T v = (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)); rs[8] += (double)v; rs[10] += (double)v; emit(8, 10, v); }
    { const T v = (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)); rs[8] += (double)v; rs[11] += (double)v; emit(8, 11, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.8af8af8af8af9p-5))); rs[8] += (double)v; rs[12] += (double)v; emit(8, 12, v); }
    { const T v = (fma(g[4], T(0x1.283a83a83a83bp-4), g[0] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.8af8af8af8af9p-6), g[3] * T(0x1.8af8af8af8af9p-5))); rs[8] += (double)v; rs[13] += (double)v; emit(8, 13, v); }
    { const T v = (fma(g[5], T(0x1.283a83a83a83bp-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.283a83a83a83bp-4))); rs[8] += (double)v; rs[14] += (double)v; emit(8, 14, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[4], T(-0x1.8af8af8af8af9p-4), g[1] * T(-0x1.8af8af8af8af9p-3))); rs[8] += (double)v; rs[15] += (double)v; emit(8, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[1] * T(0x1.8af8af8af8af9p-4))); rs[8] += (double)v; rs[16] += (double)v; emit(8, 16, v); }
    { const T v = (g[0] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.8af8af8af8af9p-5)); rs[8] += (double)v; rs[17] += (double)v; emit(8, 17, v); }
    { const T v = (fma(g[3], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-3)) + g[1] * T(-0x1.8af8af8af8af9p-4)); rs[8] += (double)v; rs[18] += (double)v; emit(8, 18, v); }
    { const T v = (fma(g[4], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.8af8af8af8af9p-4), g[3] * T(-0x1.edb6db6db6db7p-3))); rs[8] += (double)v; rs[19] += (double)v; emit(8, 19, v); }
    { const T v = (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)); rs[9] += (double)v; rs[10] += (double)v; emit(9, 10, v); }
    { const T v = (fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + g[1] * T(0x1.8af8af8af8af9p-6)); rs[9] += (double)v; rs[11] += (double)v; emit(9, 11, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.283a83a83a83bp-4))) + fma(g[4], T(0x1.283a83a83a83bp-4), g[1] * T(0x1.8af8af8af8af9p-6))); rs[9] += (double)v; rs[12] += (double)v; emit(9, 12, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-4), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.8af8af8af8af9p-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[1] * T(0x1.8af8af8af8af9p-6))); rs[9] += (double)v; rs[13] += (double)v; emit(9, 13, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.8af8af8af8af9p-5)) + fma(g[5], T(0x1.8af8af8af8af9p-5), g[3] * T(0x1.8af8af8af8af9p-5))); rs[9] += (double)v; rs[14] += (double)v; emit(9, 14, v); }
    { const T v = (fma(g[4], T(0x1.8af8af8af8af9p-6), g[1] * T(0x1.283a83a83a83bp-4)) + fma(g[5], T(0x1.283a83a83a83bp-4), g[3] * T(0x1.8af8af8af8af9p-5))); rs[9] += (double)v; rs[15] += (double)v; emit(9, 15, v); }
    { const T v = (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[1] * T(-0x1.8af8af8af8af9p-5))); rs[9] += (double)v; rs[16] += (double)v; emit(9, 16, v); }
    { const T v = (fma(g[3], T(-0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-4)) + g[1] * T(-0x1.283a83a83a83bp-3)); rs[9] += (double)v; rs[17] += (double)v; emit(9, 17, v); }
    { const T v = (g[1] * T(0x1.8af8af8af8af9p-5) + g[3] * T(0x1.8af8af8af8af9p-5)); rs[9] += (double)v; rs[18] += (double)v; emit(9, 18, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-4), g[1] * T(-0x1.283a83a83a83bp-2)) + fma(g[5], T(-0x1.edb6db6db6db7p-3), g[3] * T(-0x1.edb6db6db6db7p-3))); rs[9] += (double)v; rs[19] += (double)v; emit(9, 19, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.283a83a83a83bp-4))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.283a83a83a83bp-3), g[1] * T(-0x1.283a83a83a83bp-4)))); rs[10] += (double)v; rs[11] += (double)v; emit(10, 11, v); }
    { const T v = (fma(g[4], T(0x1.283a83a83a83bp-3), fma(g[2], T(0x1.8af8af8af8af9p-6), g[0] * T(0x1.edb6db6db6db7p-4))) + fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.283a83a83a83bp-3), g[1] * T(0x1.8af8af8af8af9p-6)))); rs[10] += (double)v; rs[12] += (double)v; emit(10, 12, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6))); rs[10] += (double)v; rs[13] += (double)v; emit(10, 13, v); }
    { const T v = (fma(g[4], T(0x1.edb6db6db6db7p-3), fma(g[2], T(0x1.8af8af8af8af9p-6), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[5], T(0x1.283a83a83a83bp-3), fma(g[3], T(0x1.283a83a83a83bp-3), g[1] * T(0x1.edb6db6db6db7p-4)))); rs[10] += (double)v; rs[14] += (double)v; emit(10, 14, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[1] * T(-0x1.8af8af8af8af9p-6))); rs[10] += (double)v; rs[15] += (double)v; emit(10, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-5))); rs[10] += (double)v; rs[16] += (double)v; emit(10, 16, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.283a83a83a83bp-2)))); rs[10] += (double)v; rs[17] += (double)v; emit(10, 17, v); }
    { const T v = (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-2))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.8af8af8af8af9p-5)))); rs[10] += (double)v; rs[18] += (double)v; emit(10, 18, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-5), fma(g[3], T(-0x1.283a83a83a83bp-2), g[0] * T(-0x1.283a83a83a83bp-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.283a83a83a83bp-3))); rs[10] += (double)v; rs[19] += (double)v; emit(10, 19, v); }
    { const T v = (fma(g[3], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-6))); rs[11] += (double)v; rs[12] += (double)v; emit(11, 12, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[0] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-5), g[3] * T(-0x1.8af8af8af8af9p-6))); rs[11] += (double)v; rs[13] += (double)v; emit(11, 13, v); }
    { const T v = (fma(g[3], T(-0x1.8af8af8af8af9p-6), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[4], T(-0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-6))); rs[11] += (double)v; rs[14] += (double)v; emit(11, 14, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-6))); rs[11] += (double)v; rs[15] += (double)v; emit(11, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[0] * T(-0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-4))); rs[11] += (double)v; rs[16] += (double)v; emit(11, 16, v); }
    { const T v = (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(-0x1.8af8af8af8af9p-5))); rs[11] += (double)v; rs[17] += (double)v; emit(11, 17, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[1] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[2] * T(-0x1.8af8af8af8af9p-5))); rs[11] += (double)v; rs[18] += (double)v; emit(11, 18, v); }
    { const T v = (g[4] * T(-0x1.8af8af8af8af9p-5) + g[5] * T(-0x1.8af8af8af8af9p-5)); rs[11] += (double)v; rs[19] += (double)v; emit(11, 19, v); }
    { const T v = (fma(g[4], T(-0x1.283a83a83a83bp-3), fma(g[2], T(-0x1.283a83a83a83bp-4), g[0] * T(-0x1.283a83a83a83bp-4))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-3)))); rs[12] += (double)v; rs[13] += (double)v; emit(12, 13, v); }
    { const T v = (fma(g[4], T(0x1.283a83a83a83bp-3), fma(g[2], T(0x1.edb6db6db6db7p-4), g[0] * T(0x1.8af8af8af8af9p-6))) + fma(g[5], T(0x1.283a83a83a83bp-3), fma(g[3], T(0x1.edb6db6db6db7p-3), g[1] * T(0x1.8af8af8af8af9p-6)))); rs[12] += (double)v; rs[14] += (double)v; emit(12, 14, v); }
    { const T v = (fma(g[3], T(-0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6))); rs[12] += (double)v; rs[15] += (double)v; emit(12, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-5))); rs[12] += (double)v; rs[16] += (double)v; emit(12, 16, v); }
    { const T v = (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.283a83a83a83bp-2), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-5)))); rs[12] += (double)v; rs[17] += (double)v; emit(12, 17, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-5), fma(g[3], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-3))) + fma(g[4], T(-0x1.283a83a83a83bp-2), g[2] * T(-0x1.283a83a83a83bp-3))); rs[12] += (double)v; rs[18] += (double)v; emit(12, 18, v); }
    { const T v = (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.283a83a83a83bp-2))) + fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.8af8af8af8af9p-5)))); rs[12] += (double)v; rs[19] += (double)v; emit(12, 19, v); }
    { const T v = (fma(g[3], T(-0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-6)) + fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6))); rs[13] += (double)v; rs[14] += (double)v; emit(13, 14, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-6), g[2] * T(-0x1.8af8af8af8af9p-6)) + fma(g[5], T(-0x1.8af8af8af8af9p-6), g[3] * T(-0x1.8af8af8af8af9p-5))); rs[13] += (double)v; rs[15] += (double)v; emit(13, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-5), fma(g[3], T(0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-4))) + fma(g[4], T(-0x1.8af8af8af8af9p-3), g[2] * T(-0x1.8af8af8af8af9p-4))); rs[13] += (double)v; rs[16] += (double)v; emit(13, 16, v); }
    { const T v = (fma(g[5], T(0x1.edb6db6db6db7p-3), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[1] * T(-0x1.8af8af8af8af9p-5))); rs[13] += (double)v; rs[17] += (double)v; emit(13, 17, v); }
    { const T v = (g[3] * T(-0x1.8af8af8af8af9p-5) + g[5] * T(-0x1.8af8af8af8af9p-5)); rs[13] += (double)v; rs[18] += (double)v; emit(13, 18, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[1] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))); rs[13] += (double)v; rs[19] += (double)v; emit(13, 19, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.283a83a83a83bp-4), g[0] * T(-0x1.8af8af8af8af9p-3))) + fma(g[5], T(-0x1.283a83a83a83bp-3), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.283a83a83a83bp-4)))); rs[14] += (double)v; rs[15] += (double)v; emit(14, 15, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-5), g[1] * T(0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(0x1.8af8af8af8af9p-5))); rs[14] += (double)v; rs[16] += (double)v; emit(14, 16, v); }
    { const T v = (fma(g[5], T(-0x1.283a83a83a83bp-2), fma(g[3], T(-0x1.8af8af8af8af9p-5), g[1] * T(-0x1.283a83a83a83bp-3))) + fma(g[4], T(-0x1.8af8af8af8af9p-5), g[2] * T(-0x1.283a83a83a83bp-3))); rs[14] += (double)v; rs[17] += (double)v; emit(14, 17, v); }
    { const T v = (fma(g[4], T(-0x1.599999999999ap-2), fma(g[2], T(-0x1.283a83a83a83bp-2), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.8af8af8af8af9p-3), g[1] * T(-0x1.8af8af8af8af9p-5)))); rs[14] += (double)v; rs[18] += (double)v; emit(14, 18, v); }
    { const T v = (fma(g[4], T(-0x1.8af8af8af8af9p-3), fma(g[2], T(-0x1.8af8af8af8af9p-5), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[5], T(-0x1.599999999999ap-2), fma(g[3], T(-0x1.599999999999ap-2), g[1] * T(-0x1.283a83a83a83bp-2)))); rs[14] += (double)v; rs[19] += (double)v; emit(14, 19, v); }
    { const T v = (fma(g[5], T(-0x1.8af8af8af8af9p-3), fma(g[3], T(0x1.8af8af8af8af9p-5), g[1] * T(-0x1.8af8af8af8af9p-4))) + fma(g[4], T(0x1.8af8af8af8af9p-5), g[2] * T(-0x1.8af8af8af8af9p-4))); rs[15] += (double)v; rs[16] += (double)v; emit(15, 16, v); }
    { const T v = (g[3] * T(-0x1.8af8af8af8af9p-5) + g[4] * T(-0x1.8af8af8af8af9p-5)); rs[15] += (double)v; rs[17] += (double)v; emit(15, 17, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.8af8af8af8af9p-4), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.edb6db6db6db7p-3), g[1] * T(0x1.8af8af8af8af9p-4))); rs[15] += (double)v; rs[18] += (double)v; emit(15, 18, v); }
    { const T v = (fma(g[5], T(0x1.8af8af8af8af9p-4), fma(g[3], T(0x1.edb6db6db6db7p-3), g[0] * T(-0x1.8af8af8af8af9p-5))) + fma(g[4], T(0x1.8af8af8af8af9p-4), g[2] * T(0x1.8af8af8af8af9p-4))); rs[15] += (double)v; rs[19] += (double)v; emit(15, 19, v); }
    { const T v = (fma(g[4], T(-0x1.283a83a83a83bp-1), g[0] * T(-0x1.283a83a83a83bp-1)) + fma(g[5], T(-0x1.283a83a83a83bp-2), g[3] * T(-0x1.283a83a83a83bp-1))); rs[16] += (double)v; rs[17] += (double)v; emit(16, 17, v); }
    { const T v = (fma(g[4], T(-0x1.283a83a83a83bp-2), g[1] * T(-0x1.283a83a83a83bp-1)) + fma(g[5], T(-0x1.283a83a83a83bp-1), g[3] * T(-0x1.283a83a83a83bp-1))); rs[16] += (double)v; rs[18] += (double)v; emit(16, 18, v); }
    { const T v = (fma(g[4], T(-0x1.283a83a83a83bp-1), g[2] * T(-0x1.283a83a83a83bp-1)) + fma(g[5], T(-0x1.283a83a83a83bp-1), g[3] * T(-0x1.283a83a83a83bp-2))); rs[16] += (double)v; rs[19] += (double)v; emit(16, 19, v); }
    { const T v = (fma(g[4], T(0x1.283a83a83a83bp-2), g[2] * T(0x1.283a83a83a83bp-2)) + fma(g[5], T(0x1.283a83a83a83bp-2), g[3] * T(0x1.283a83a83a83bp-1))); rs[17] += (double)v; rs[18] += (double)v; emit(17, 18, v); }
    { const T v = (fma(g[4], T(0x1.283a83a83a83bp-1), g[1] * T(0x1.283a83a83a83bp-2)) + fma(g[5], T(0x1.283a83a83a83bp-2), g[3] * T(0x1.283a83a83a83bp-2))); rs[17] += (double)v; rs[19] += (double)v; emit(17, 19, v); }
    { const T v = (fma(g[4], T(0x1.283a83a83a83bp-2), g[0] * T(0x1.283a83a83a83bp-2)) + fma(g[5], T(0x1.283a83a83a83bp-1), g[3] * T(0x1.283a83a83a83bp-2))); rs[18] += (double)v; rs[19] += (double)v; emit(18, 19, v); }
    emit(0, 0, -rs[0]);
    emit(1, 1, -rs[1]);
    emit(2, 2, -rs[2]);
    emit(3, 3, -rs[3]);
    emit(4, 4, -rs[4]);
    emit(5, 5, -rs[5]);
    emit(6, 6, -rs[6]);
    emit(7, 7, -rs[7]);
    emit(8, 8, -rs[8]);
    emit(9, 9, -rs[9]);
    emit(10, 10, -rs[10]);
    emit(11, 11, -rs[11]);
    emit(12, 12, -rs[12]);
    emit(13, 13, -rs[13]);
    emit(14, 14, -rs[14]);
    emit(15, 15, -rs[15]);
    emit(16, 16, -rs[16]);
    emit(17, 17, -rs[17]);
    emit(18, 18, -rs[18]);
    emit(19, 19, -rs[19]);
  }
}
constexpr double kP3ConstTermMax = 0x1.283a83a83a83bp-1;

// P3 stiffness coefficients by geometry pair s: entry (i, j) = sum_s g[s] *
// kP3GradGradSym[s*400 + i*20 + j] (the terms of p3_stiffness_const).
__device__ const double kP3GradGradSym[2400] = {
    0x1.e79e79e79e79ep-5, -0x1.7297297297297p-7, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7,
    -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.0750750750750p-5, 0x1.0750750750750p-5,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.7297297297297p-7, 0x1.e79e79e79e79ep-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4,
    0x1.0750750750750p-5, -0x1.0750750750750p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    -0x1.283a83a83a83bp-2, -0x1.283a83a83a83bp-3, -0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6,
    0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, -0x1.283a83a83a83bp-2,
    -0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-4,
    0x0.0p+0, 0x0.0p+0, -0x1.1d41d41d41d42p-5, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2, -0x1.283a83a83a83bp-3, 0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    -0x1.1d41d41d41d42p-5, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6,
    0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    -0x1.283a83a83a83bp-3, -0x1.283a83a83a83bp-2, 0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0,
    0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x0.0p+0, -0x1.8af8af8af8af9p-3, 0x1.edb6db6db6db7p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.0750750750750p-5, 0x1.0750750750750p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    0x1.283a83a83a83bp-1, -0x1.283a83a83a83bp-1, 0x0.0p+0, 0x0.0p+0, 0x1.0750750750750p-5, -0x1.0750750750750p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4,
    0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.283a83a83a83bp-2, 0x0.0p+0, -0x1.283a83a83a83bp-3, 0x0.0p+0, -0x1.283a83a83a83bp-2, 0x0.0p+0,
    -0x1.283a83a83a83bp-3, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-2, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-3, 0x0.0p+0, -0x1.283a83a83a83bp-2, 0x0.0p+0,
    -0x1.283a83a83a83bp-3, 0x0.0p+0, -0x1.283a83a83a83bp-2, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x1.e79e79e79e79ep-5, 0x0.0p+0,
    -0x1.7297297297297p-7, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5,
    -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7, -0x1.0750750750750p-5, 0x1.8af8af8af8af9p-5, 0x1.0750750750750p-5, 0x1.8af8af8af8af9p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.7297297297297p-7, 0x0.0p+0, 0x1.e79e79e79e79ep-5, 0x0.0p+0,
    -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    0x1.0750750750750p-5, 0x1.8af8af8af8af9p-5, -0x1.0750750750750p-5, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, 0x0.0p+0, -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4,
    0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-4, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2,
    0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-3, -0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0,
    -0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, 0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2,
    -0x1.1d41d41d41d42p-5, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2,
    -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0,
    -0x1.8af8af8af8af9p-3, 0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5,
    0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.1d41d41d41d42p-5, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5,
    0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2, 0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0,
    -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x1.8af8af8af8af9p-4, 0x0.0p+0,
    -0x1.0750750750750p-5, 0x0.0p+0, 0x1.0750750750750p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x1.283a83a83a83bp-1, 0x0.0p+0,
    -0x1.283a83a83a83bp-1, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x0.0p+0,
    -0x1.283a83a83a83bp-2, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-3,
    -0x1.283a83a83a83bp-2, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, 0x0.0p+0,
    0x0.0p+0, 0x1.283a83a83a83bp-1, 0x0.0p+0, 0x1.283a83a83a83bp-2, 0x1.0750750750750p-5, 0x0.0p+0,
    -0x1.0750750750750p-5, 0x0.0p+0, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.283a83a83a83bp-1, 0x0.0p+0, 0x1.283a83a83a83bp-1, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.283a83a83a83bp-3, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-2, -0x1.283a83a83a83bp-3, 0x0.0p+0,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-2,
    0x0.0p+0, 0x1.283a83a83a83bp-1, 0x1.e79e79e79e79ep-5, 0x0.0p+0, 0x0.0p+0, -0x1.7297297297297p-7,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7,
    -0x1.0750750750750p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.0750750750750p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.7297297297297p-7, 0x0.0p+0, 0x0.0p+0, 0x1.e79e79e79e79ep-5,
    0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5, 0x1.b6db6db6db6dbp-7, -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    0x1.0750750750750p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.0750750750750p-5, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x1.8af8af8af8af9p-3, -0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-4,
    -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, -0x1.1d41d41d41d42p-5, -0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-3,
    -0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-4, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2,
    -0x1.283a83a83a83bp-3, 0x1.8af8af8af8af9p-5, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x1.b6db6db6db6dbp-7,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-3, -0x1.283a83a83a83bp-4, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-4, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x0.0p+0, -0x1.1d41d41d41d42p-5, -0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-4, -0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-3,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, -0x1.283a83a83a83bp-2, 0x1.8af8af8af8af9p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0,
    0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x0.0p+0, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-6, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-3, 0x1.edb6db6db6db7p-3,
    0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5,
    -0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7,
    0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-2, -0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-5, 0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4,
    -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.edb6db6db6db7p-4, -0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3,
    -0x1.283a83a83a83bp-2, -0x1.8af8af8af8af9p-5, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-4, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3,
    -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.0750750750750p-5, 0x0.0p+0,
    0x0.0p+0, 0x1.0750750750750p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x1.283a83a83a83bp-1, 0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-1,
    0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.283a83a83a83bp-2,
    0x0.0p+0, -0x1.283a83a83a83bp-3, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    -0x1.283a83a83a83bp-2, 0x0.0p+0, -0x1.283a83a83a83bp-3, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-1,
    0x1.283a83a83a83bp-2, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5,
    0x0.0p+0, -0x1.283a83a83a83bp-3, 0x0.0p+0, -0x1.283a83a83a83bp-2, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, 0x0.0p+0, -0x1.283a83a83a83bp-2, 0x0.0p+0,
    0x0.0p+0, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x0.0p+0, 0x1.0750750750750p-5, 0x0.0p+0,
    0x0.0p+0, -0x1.0750750750750p-5, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4,
    -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.283a83a83a83bp-1, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-1,
    0x1.e79e79e79e79ep-4, -0x1.7297297297297p-7, -0x1.7297297297297p-7, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-6, -0x1.b6db6db6db6dbp-6, -0x1.1d41d41d41d42p-4, 0x1.b6db6db6db6dbp-6,
    -0x1.0cccccccccccdp-3, 0x1.f8af8af8af8b0p-5, -0x1.0cccccccccccdp-3, 0x1.f8af8af8af8b0p-5, -0x1.0750750750750p-4, 0x1.4924924924925p-4,
    0x1.4924924924925p-4, 0x1.8af8af8af8af9p-4, -0x1.7297297297297p-7, 0x0.0p+0, 0x1.7297297297297p-7, 0x0.0p+0,
    0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x1.f8af8af8af8b0p-5, -0x1.1d41d41d41d42p-5,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x1.1d41d41d41d42p-5, -0x1.f8af8af8af8b0p-5,
    -0x1.0750750750750p-6, 0x0.0p+0, 0x1.0750750750750p-6, 0x0.0p+0, -0x1.7297297297297p-7, 0x1.7297297297297p-7,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7,
    -0x1.1d41d41d41d42p-5, 0x1.f8af8af8af8b0p-5, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x1.1d41d41d41d42p-5, -0x1.f8af8af8af8b0p-5,
    0x0.0p+0, 0x0.0p+0, -0x1.0750750750750p-6, 0x1.0750750750750p-6, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4,
    0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    0x1.edb6db6db6db7p-3, -0x1.edb6db6db6db7p-3, 0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-4,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3, 0x0.0p+0,
    -0x1.edb6db6db6db7p-3, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.b6db6db6db6dbp-6, 0x1.f8af8af8af8b0p-5,
    -0x1.1d41d41d41d42p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3, -0x1.edb6db6db6db7p-3,
    -0x1.b6db6db6db6dbp-6, -0x1.1d41d41d41d42p-5, 0x1.f8af8af8af8b0p-5, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-6,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3,
    0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3, -0x1.1d41d41d41d42p-4, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.edb6db6db6db7p-2, -0x1.283a83a83a83bp-3, 0x1.283a83a83a83bp-3, 0x0.0p+0, 0x1.283a83a83a83bp-3, 0x0.0p+0,
    0x1.8af8af8af8af9p-4, -0x1.599999999999ap-2, -0x1.599999999999ap-2, -0x1.283a83a83a83bp-2, 0x1.b6db6db6db6dbp-6, -0x1.b6db6db6db6dbp-7,
    -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-3, 0x1.8af8af8af8af9p-2, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, 0x0.0p+0,
    -0x1.0cccccccccccdp-3, 0x0.0p+0, 0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, 0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-6,
    0x1.283a83a83a83bp-2, -0x1.8af8af8af8af9p-3, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3,
    -0x1.8af8af8af8af9p-5, -0x1.599999999999ap-2, 0x1.f8af8af8af8b0p-5, 0x0.0p+0, -0x1.f8af8af8af8b0p-5, 0x0.0p+0,
    -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3,
    0x0.0p+0, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-3, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x1.edb6db6db6db7p-3, -0x1.0cccccccccccdp-3, 0x1.1d41d41d41d42p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5,
    0x1.283a83a83a83bp-2, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, -0x1.599999999999ap-2,
    0x1.f8af8af8af8b0p-5, -0x1.f8af8af8af8b0p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-6,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3, -0x1.0750750750750p-4, -0x1.0750750750750p-6, -0x1.0750750750750p-6, 0x0.0p+0,
    0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.283a83a83a83bp-1, -0x1.283a83a83a83bp-1, -0x1.283a83a83a83bp-1, -0x1.283a83a83a83bp-2, 0x1.4924924924925p-4, 0x0.0p+0,
    0x1.0750750750750p-6, 0x0.0p+0, -0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3, -0x1.599999999999ap-2, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-2,
    0x1.4924924924925p-4, 0x1.0750750750750p-6, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, -0x1.599999999999ap-2, 0x1.8af8af8af8af9p-4,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, -0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1,
    0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-2, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.edb6db6db6db7p-3, -0x1.edb6db6db6db7p-3,
    -0x1.283a83a83a83bp-2, 0x0.0p+0, -0x1.599999999999ap-2, 0x1.edb6db6db6db7p-3, -0x1.599999999999ap-2, 0x1.edb6db6db6db7p-3,
    -0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x1.e79e79e79e79ep-4, -0x1.7297297297297p-7,
    0x0.0p+0, -0x1.7297297297297p-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-6, -0x1.b6db6db6db6dbp-6,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.0cccccccccccdp-3, 0x1.f8af8af8af8b0p-5, -0x1.1d41d41d41d42p-4, 0x1.b6db6db6db6dbp-6,
    -0x1.0cccccccccccdp-3, 0x1.f8af8af8af8b0p-5, -0x1.0750750750750p-4, 0x1.4924924924925p-4, 0x1.8af8af8af8af9p-4, 0x1.4924924924925p-4,
    -0x1.7297297297297p-7, 0x0.0p+0, 0x0.0p+0, 0x1.7297297297297p-7, 0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7,
    0x1.f8af8af8af8b0p-5, -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x1.1d41d41d41d42p-5, -0x1.f8af8af8af8b0p-5, -0x1.0750750750750p-6, 0x0.0p+0,
    0x0.0p+0, 0x1.0750750750750p-6, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.7297297297297p-7, 0x1.7297297297297p-7,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1d41d41d41d42p-5, 0x1.f8af8af8af8b0p-5,
    0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x1.1d41d41d41d42p-5, -0x1.f8af8af8af8b0p-5, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    0x0.0p+0, 0x0.0p+0, -0x1.0750750750750p-6, 0x1.0750750750750p-6, 0x0.0p+0, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6,
    0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-4,
    0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x0.0p+0, 0x0.0p+0,
    0x1.edb6db6db6db7p-3, -0x1.edb6db6db6db7p-3, 0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-6, 0x1.f8af8af8af8b0p-5,
    0x0.0p+0, -0x1.1d41d41d41d42p-5, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3, -0x1.edb6db6db6db7p-3,
    -0x1.b6db6db6db6dbp-6, -0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x1.f8af8af8af8b0p-5, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-4,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-3, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3,
    -0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x1.b6db6db6db6dbp-7,
    -0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4,
    0x1.edb6db6db6db7p-3, 0x0.0p+0, 0x0.0p+0, -0x1.edb6db6db6db7p-3, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x1.8af8af8af8af9p-3, -0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-4,
    -0x1.0cccccccccccdp-3, 0x0.0p+0, 0x0.0p+0, 0x1.1d41d41d41d42p-5, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-2, -0x1.8af8af8af8af9p-3,
    0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-6, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3,
    -0x1.599999999999ap-2, -0x1.8af8af8af8af9p-5, 0x1.f8af8af8af8b0p-5, 0x0.0p+0, 0x0.0p+0, -0x1.f8af8af8af8b0p-5,
    0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-3, 0x0.0p+0, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5, -0x1.1d41d41d41d42p-4, -0x1.b6db6db6db6dbp-7,
    0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.283a83a83a83bp-3, 0x0.0p+0, 0x1.edb6db6db6db7p-2, -0x1.283a83a83a83bp-3,
    0x1.283a83a83a83bp-3, 0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.599999999999ap-2, -0x1.283a83a83a83bp-2, -0x1.599999999999ap-2,
    0x1.b6db6db6db6dbp-6, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    -0x1.283a83a83a83bp-3, 0x1.8af8af8af8af9p-2, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4,
    0x0.0p+0, 0x1.8af8af8af8af9p-4, -0x1.0cccccccccccdp-3, 0x1.1d41d41d41d42p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-6,
    0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-6, 0x1.283a83a83a83bp-2, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.599999999999ap-2, -0x1.8af8af8af8af9p-3, 0x1.f8af8af8af8b0p-5, -0x1.f8af8af8af8b0p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5,
    -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-6,
    -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, 0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-4,
    -0x1.0750750750750p-4, -0x1.0750750750750p-6, 0x0.0p+0, -0x1.0750750750750p-6, 0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3,
    0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-1, -0x1.283a83a83a83bp-1,
    -0x1.283a83a83a83bp-2, -0x1.283a83a83a83bp-1, 0x1.4924924924925p-4, 0x0.0p+0, 0x0.0p+0, 0x1.0750750750750p-6,
    -0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, -0x1.599999999999ap-2, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    -0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x1.8af8af8af8af9p-4, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.edb6db6db6db7p-3, -0x1.edb6db6db6db7p-3,
    0x0.0p+0, 0x0.0p+0, -0x1.599999999999ap-2, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-2, 0x0.0p+0,
    -0x1.599999999999ap-2, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-2,
    0x1.4924924924925p-4, 0x1.0750750750750p-6, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5,
    -0x1.599999999999ap-2, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, -0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1,
    0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x1.e79e79e79e79ep-4, 0x0.0p+0, -0x1.7297297297297p-7, -0x1.7297297297297p-7,
    -0x1.b6db6db6db6dbp-6, -0x1.b6db6db6db6dbp-6, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    -0x1.0cccccccccccdp-3, 0x1.f8af8af8af8b0p-5, -0x1.0cccccccccccdp-3, 0x1.f8af8af8af8b0p-5, -0x1.1d41d41d41d42p-4, 0x1.b6db6db6db6dbp-6,
    -0x1.0750750750750p-4, 0x1.8af8af8af8af9p-4, 0x1.4924924924925p-4, 0x1.4924924924925p-4, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.7297297297297p-7, 0x0.0p+0, 0x0.0p+0, 0x1.7297297297297p-7, 0x1.f8af8af8af8b0p-5, -0x1.1d41d41d41d42p-5,
    0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1d41d41d41d42p-5, -0x1.f8af8af8af8b0p-5, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, -0x1.0750750750750p-6, 0x0.0p+0,
    0x0.0p+0, 0x1.0750750750750p-6, -0x1.7297297297297p-7, 0x0.0p+0, 0x1.7297297297297p-7, 0x0.0p+0,
    -0x1.1d41d41d41d42p-5, 0x1.f8af8af8af8b0p-5, 0x0.0p+0, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x1.b6db6db6db6dbp-7,
    0x1.1d41d41d41d42p-5, -0x1.f8af8af8af8b0p-5, 0x0.0p+0, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    -0x1.0750750750750p-6, 0x0.0p+0, 0x1.0750750750750p-6, 0x0.0p+0, -0x1.b6db6db6db6dbp-6, 0x0.0p+0,
    0x1.f8af8af8af8b0p-5, -0x1.1d41d41d41d42p-5, 0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5,
    -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3,
    -0x1.b6db6db6db6dbp-6, 0x0.0p+0, -0x1.1d41d41d41d42p-5, 0x1.f8af8af8af8b0p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-3,
    -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3,
    -0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-3, -0x1.283a83a83a83bp-4,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.8af8af8af8af9p-4, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, 0x0.0p+0,
    0x1.b6db6db6db6dbp-7, 0x0.0p+0, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    -0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.edb6db6db6db7p-3, 0x0.0p+0, -0x1.edb6db6db6db7p-3, 0x0.0p+0,
    -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x1.b6db6db6db6dbp-7, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-3, -0x1.283a83a83a83bp-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-6, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, 0x0.0p+0,
    0x0.0p+0, -0x1.8af8af8af8af9p-4, -0x1.b6db6db6db6dbp-7, 0x0.0p+0, 0x0.0p+0, 0x1.b6db6db6db6dbp-7,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, -0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4,
    0x1.edb6db6db6db7p-3, 0x0.0p+0, 0x0.0p+0, -0x1.edb6db6db6db7p-3, -0x1.0cccccccccccdp-3, 0x0.0p+0,
    0x0.0p+0, 0x1.1d41d41d41d42p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5,
    0x0.0p+0, 0x0.0p+0, 0x1.283a83a83a83bp-2, -0x1.8af8af8af8af9p-3, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5,
    0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, -0x1.599999999999ap-2, -0x1.8af8af8af8af9p-3, -0x1.8af8af8af8af9p-5,
    0x1.f8af8af8af8b0p-5, 0x0.0p+0, 0x0.0p+0, -0x1.f8af8af8af8b0p-5, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3,
    0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-3,
    -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, 0x1.edb6db6db6db7p-3,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, -0x1.0cccccccccccdp-3, 0x0.0p+0, 0x1.1d41d41d41d42p-5, 0x0.0p+0,
    0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0, 0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5,
    0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-2, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-3, -0x1.8af8af8af8af9p-6,
    0x1.8af8af8af8af9p-5, -0x1.599999999999ap-2, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, 0x1.f8af8af8af8b0p-5, 0x0.0p+0,
    -0x1.f8af8af8af8b0p-5, 0x0.0p+0, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-3,
    0x0.0p+0, -0x1.8af8af8af8af9p-6, 0x1.8af8af8af8af9p-5, 0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-4,
    -0x1.1d41d41d41d42p-4, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-4, 0x1.8af8af8af8af9p-5, 0x1.283a83a83a83bp-3, 0x0.0p+0,
    0x1.283a83a83a83bp-3, 0x0.0p+0, 0x1.edb6db6db6db7p-2, -0x1.283a83a83a83bp-3, 0x1.8af8af8af8af9p-4, -0x1.283a83a83a83bp-2,
    -0x1.599999999999ap-2, -0x1.599999999999ap-2, 0x1.b6db6db6db6dbp-6, 0x0.0p+0, -0x1.b6db6db6db6dbp-7, -0x1.b6db6db6db6dbp-7,
    0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-4, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-4,
    -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.8af8af8af8af9p-6, -0x1.283a83a83a83bp-3, 0x1.8af8af8af8af9p-2,
    -0x1.8af8af8af8af9p-3, 0x0.0p+0, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, -0x1.0750750750750p-4, 0x0.0p+0,
    -0x1.0750750750750p-6, -0x1.0750750750750p-6, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, 0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3,
    0x1.8af8af8af8af9p-4, 0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5, 0x1.8af8af8af8af9p-5,
    0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-3, 0x1.283a83a83a83bp-1, -0x1.283a83a83a83bp-2, -0x1.283a83a83a83bp-1, -0x1.283a83a83a83bp-1,
    0x1.8af8af8af8af9p-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.edb6db6db6db7p-3, -0x1.edb6db6db6db7p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.599999999999ap-2, 0x1.edb6db6db6db7p-3,
    -0x1.599999999999ap-2, 0x1.edb6db6db6db7p-3, -0x1.283a83a83a83bp-2, 0x0.0p+0, -0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1,
    0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-2, 0x1.4924924924925p-4, 0x0.0p+0, 0x0.0p+0, 0x1.0750750750750p-6,
    0x1.8af8af8af8af9p-5, -0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.599999999999ap-2, 0x1.8af8af8af8af9p-4,
    -0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1, 0x1.4924924924925p-4, 0x0.0p+0,
    0x1.0750750750750p-6, 0x0.0p+0, -0x1.edb6db6db6db7p-3, 0x1.8af8af8af8af9p-5, 0x0.0p+0, 0x0.0p+0,
    -0x1.8af8af8af8af9p-4, -0x1.edb6db6db6db7p-3, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-5, -0x1.8af8af8af8af9p-3, 0x1.8af8af8af8af9p-4,
    -0x1.599999999999ap-2, 0x1.8af8af8af8af9p-4, -0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-2, 0x1.283a83a83a83bp-1, 0x1.283a83a83a83bp-1,
};

// P2 stiffness with a P1 coefficient: q[m*6+s] = k_m * Ghat_s,
// Ghat = |detJ| K K^T (s over (00,11,22,01,02,12)).  Calls emit(i, j, value)
// for the 55 unique entries i <= j (FP32: off-diagonal entries first, then
// the diagonal entries as minus their rows' FP64 sums; emit takes a double).
template <typename T, typename Emit>
__device__ __forceinline__ void p2_stiffness_p1coef(const T* q, Emit&& emit) {
  if constexpr (sizeof(T) == 8) {
    emit(0, 0, ((fma(q[20], T(0x1.3e93e93e93e94p-6), fma(q[16], T(0x1.3e93e93e93e94p-5), fma(q[12], T(0x1.3e93e93e93e94p-6), fma(q[8], T(0x1.3e93e93e93e94p-6), fma(q[4], T(0x1.5555555555555p-4), q[0] * T(0x1.5555555555555p-5)))))) + fma(q[21], T(0x1.3e93e93e93e94p-5), fma(q[17], T(0x1.3e93e93e93e94p-5), fma(q[13], T(0x1.3e93e93e93e94p-6), fma(q[9], T(0x1.3e93e93e93e94p-5), fma(q[5], T(0x1.5555555555555p-4), q[1] * T(0x1.5555555555555p-5))))))) + (fma(q[22], T(0x1.3e93e93e93e94p-5), fma(q[18], T(0x1.3e93e93e93e94p-6), fma(q[14], T(0x1.3e93e93e93e94p-6), fma(q[10], T(0x1.3e93e93e93e94p-5), fma(q[6], T(0x1.3e93e93e93e94p-6), q[2] * T(0x1.5555555555555p-5)))))) + fma(q[23], T(0x1.3e93e93e93e94p-5), fma(q[19], T(0x1.3e93e93e93e94p-6), fma(q[15], T(0x1.3e93e93e93e94p-5), fma(q[11], T(0x1.3e93e93e93e94p-5), fma(q[7], T(0x1.3e93e93e93e94p-6), q[3] * T(0x1.5555555555555p-4)))))))));
    emit(0, 1, ((fma(q[16], T(0x1.6c16c16c16c17p-9), fma(q[9], T(0x1.c71c71c71c71cp-7), q[0] * T(0x1.c71c71c71c71cp-7))) + fma(q[18], T(0x1.6c16c16c16c17p-9), fma(q[10], T(0x1.c71c71c71c71cp-7), q[3] * T(0x1.c71c71c71c71cp-7)))) + (fma(q[21], T(0x1.6c16c16c16c17p-9), fma(q[12], T(0x1.6c16c16c16c17p-9), q[4] * T(0x1.c71c71c71c71cp-7))) + fma(q[22], T(0x1.6c16c16c16c17p-9), fma(q[15], T(0x1.6c16c16c16c17p-9), q[6] * T(0x1.c71c71c71c71cp-7))))));
    emit(0, 2, ((fma(q[17], T(0x1.c71c71c71c71cp-7), fma(q[9], T(0x1.6c16c16c16c17p-9), q[1] * T(0x1.c71c71c71c71cp-7))) + fma(q[19], T(0x1.6c16c16c16c17p-9), fma(q[11], T(0x1.6c16c16c16c17p-9), q[3] * T(0x1.c71c71c71c71cp-7)))) + (fma(q[21], T(0x1.6c16c16c16c17p-9), fma(q[13], T(0x1.c71c71c71c71cp-7), q[5] * T(0x1.c71c71c71c71cp-7))) + fma(q[23], T(0x1.6c16c16c16c17p-9), fma(q[15], T(0x1.c71c71c71c71cp-7), q[7] * T(0x1.6c16c16c16c17p-9))))));
    emit(0, 3, ((fma(q[17], T(0x1.6c16c16c16c17p-9), fma(q[10], T(0x1.6c16c16c16c17p-9), q[2] * T(0x1.c71c71c71c71cp-7))) + fma(q[20], T(0x1.c71c71c71c71cp-7), fma(q[11], T(0x1.6c16c16c16c17p-9), q[4] * T(0x1.c71c71c71c71cp-7)))) + (fma(q[22], T(0x1.c71c71c71c71cp-7), fma(q[14], T(0x1.6c16c16c16c17p-9), q[5] * T(0x1.c71c71c71c71cp-7))) + fma(q[23], T(0x1.c71c71c71c71cp-7), fma(q[16], T(0x1.6c16c16c16c17p-9), q[8] * T(0x1.6c16c16c16c17p-9))))));
    emit(0, 4, ((fma(q[20], T(0x1.6c16c16c16c17p-7), fma(q[15], T(0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.6c16c16c16c17p-7), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-7), q[2] * T(-0x1.6c16c16c16c17p-7)))))) + (fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[17], T(0x1.1111111111111p-5), fma(q[13], T(0x1.6c16c16c16c17p-7), fma(q[8], T(0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[23], T(0x1.1111111111111p-5), fma(q[19], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-7))))))));
    emit(0, 5, ((fma(q[20], T(0x1.6c16c16c16c17p-7), fma(q[15], T(0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.1111111111111p-5), fma(q[5], T(-0x1.6c16c16c16c17p-7), q[0] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-6), fma(q[6], T(0x1.6c16c16c16c17p-7), q[2] * T(-0x1.6c16c16c16c17p-7)))))) + (fma(q[22], T(0x1.1111111111111p-5), fma(q[17], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-7), fma(q[8], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[18], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-7), fma(q[9], T(0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-6))))))));
    emit(0, 6, ((fma(q[19], T(0x1.6c16c16c16c17p-7), fma(q[15], T(0x1.1111111111111p-5), fma(q[10], T(0x1.6c16c16c16c17p-7), fma(q[5], T(-0x1.6c16c16c16c17p-7), q[0] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-6), fma(q[6], T(0x1.6c16c16c16c17p-7), q[1] * T(-0x1.6c16c16c16c17p-7)))))) + (fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[17], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[18], T(0x1.6c16c16c16c17p-7), fma(q[13], T(0x1.6c16c16c16c17p-7), fma(q[9], T(0x1.1111111111111p-5), q[4] * T(-0x1.6c16c16c16c17p-7))))))));
    emit(0, 7, ((fma(q[20], T(-0x1.1111111111111p-5), fma(q[16], T(-0x1.1111111111111p-5), fma(q[12], T(-0x1.6c16c16c16c17p-7), fma(q[8], T(-0x1.6c16c16c16c17p-6), fma(q[4], T(-0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.1111111111111p-5), fma(q[13], T(-0x1.6c16c16c16c17p-7), fma(q[9], T(-0x1.6c16c16c16c17p-6), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-7))))))) + (fma(q[22], T(-0x1.c71c71c71c71cp-5), fma(q[18], T(-0x1.6c16c16c16c17p-6), fma(q[14], T(-0x1.6c16c16c16c17p-6), fma(q[10], T(-0x1.1111111111111p-5), fma(q[6], T(-0x1.6c16c16c16c17p-7), q[2] * T(-0x1.c71c71c71c71cp-5)))))) + fma(q[23], T(-0x1.c71c71c71c71cp-5), fma(q[19], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-6), fma(q[11], T(-0x1.1111111111111p-5), fma(q[7], T(-0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-6)))))))));
    emit(0, 8, ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[12], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-7), fma(q[4], T(0x1.6c16c16c16c17p-6), q[0] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[21], T(-0x1.1111111111111p-5), fma(q[17], T(-0x1.c71c71c71c71cp-5), fma(q[13], T(-0x1.1111111111111p-5), fma(q[9], T(-0x1.1111111111111p-5), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[1] * T(-0x1.c71c71c71c71cp-5))))))) + (fma(q[22], T(-0x1.6c16c16c16c17p-6), fma(q[18], T(-0x1.6c16c16c16c17p-7), fma(q[14], T(-0x1.6c16c16c16c17p-6), fma(q[10], T(-0x1.6c16c16c16c17p-6), fma(q[6], T(-0x1.6c16c16c16c17p-7), q[2] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[23], T(-0x1.1111111111111p-5), fma(q[19], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.c71c71c71c71cp-5), fma(q[11], T(-0x1.1111111111111p-5), fma(q[7], T(-0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-5)))))))));
    emit(0, 9, ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[16], T(-0x1.1111111111111p-5), fma(q[12], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-6), fma(q[4], T(-0x1.6c16c16c16c17p-5), q[0] * T(-0x1.c71c71c71c71cp-5)))))) + fma(q[21], T(-0x1.1111111111111p-5), fma(q[17], T(-0x1.6c16c16c16c17p-6), fma(q[13], T(-0x1.6c16c16c16c17p-7), fma(q[9], T(-0x1.c71c71c71c71cp-5), fma(q[5], T(0x1.6c16c16c16c17p-6), q[1] * T(0x1.6c16c16c16c17p-7))))))) + (fma(q[22], T(-0x1.1111111111111p-5), fma(q[18], T(-0x1.6c16c16c16c17p-6), fma(q[14], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(-0x1.c71c71c71c71cp-5), fma(q[6], T(-0x1.1111111111111p-5), q[2] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[23], T(-0x1.6c16c16c16c17p-6), fma(q[19], T(-0x1.6c16c16c16c17p-7), fma(q[15], T(-0x1.1111111111111p-5), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[7], T(-0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-5)))))))));
    emit(1, 1, ((q[0] * T(0x1.3e93e93e93e94p-6) + q[6] * T(0x1.5555555555555p-5)) + (q[12] * T(0x1.3e93e93e93e94p-6) + q[18] * T(0x1.3e93e93e93e94p-6))));
    emit(1, 2, ((q[3] * T(-0x1.6c16c16c16c17p-9) + q[9] * T(-0x1.c71c71c71c71cp-7)) + (q[15] * T(-0x1.c71c71c71c71cp-7) + q[21] * T(-0x1.6c16c16c16c17p-9))));
    emit(1, 3, ((q[4] * T(-0x1.6c16c16c16c17p-9) + q[10] * T(-0x1.c71c71c71c71cp-7)) + (q[16] * T(-0x1.6c16c16c16c17p-9) + q[22] * T(-0x1.c71c71c71c71cp-7))));
    emit(1, 4, ((fma(q[15], T(-0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7)) + fma(q[16], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7))) + (fma(q[21], T(-0x1.6c16c16c16c17p-6), q[9] * T(0x1.6c16c16c16c17p-7)) + fma(q[22], T(-0x1.6c16c16c16c17p-7), q[10] * T(0x1.6c16c16c16c17p-7)))));
    emit(1, 5, ((fma(q[12], T(-0x1.6c16c16c16c17p-7), q[0] * T(-0x1.6c16c16c16c17p-7)) + fma(q[16], T(0x1.6c16c16c16c17p-7), q[4] * T(0x1.6c16c16c16c17p-7))) + (fma(q[18], T(-0x1.6c16c16c16c17p-6), q[6] * T(0x1.6c16c16c16c17p-7)) + fma(q[22], T(0x1.6c16c16c16c17p-7), q[10] * T(0x1.1111111111111p-4)))));
    emit(1, 6, ((fma(q[12], T(-0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-7)) + fma(q[15], T(0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-7))) + (fma(q[18], T(-0x1.6c16c16c16c17p-7), q[6] * T(0x1.6c16c16c16c17p-7)) + fma(q[21], T(0x1.6c16c16c16c17p-7), q[9] * T(0x1.1111111111111p-4)))));
    emit(1, 7, ((fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[9], T(-0x1.6c16c16c16c17p-7), q[0] * T(0x1.6c16c16c16c17p-7))) + fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-7)))) + (fma(q[15], T(0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-7)) + fma(q[18], T(0x1.6c16c16c16c17p-6), q[6] * T(-0x1.6c16c16c16c17p-7)))));
    emit(1, 8, ((fma(q[18], T(0x1.6c16c16c16c17p-7), fma(q[10], T(-0x1.6c16c16c16c17p-7), q[0] * T(0x1.6c16c16c16c17p-7))) + fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[15], T(0x1.6c16c16c16c17p-7), q[4] * T(0x1.6c16c16c16c17p-7)) + fma(q[16], T(0x1.6c16c16c16c17p-6), q[6] * T(-0x1.6c16c16c16c17p-7)))));
    emit(1, 9, ((fma(q[16], T(-0x1.6c16c16c16c17p-7), fma(q[9], T(-0x1.1111111111111p-4), q[0] * T(-0x1.1111111111111p-5))) + fma(q[18], T(-0x1.6c16c16c16c17p-6), fma(q[10], T(-0x1.1111111111111p-4), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[21], T(-0x1.6c16c16c16c17p-7), fma(q[12], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7))) + fma(q[22], T(-0x1.6c16c16c16c17p-7), fma(q[15], T(-0x1.6c16c16c16c17p-7), q[6] * T(-0x1.c71c71c71c71cp-5))))));
    emit(2, 2, ((q[1] * T(0x1.3e93e93e93e94p-6) + q[7] * T(0x1.3e93e93e93e94p-6)) + (q[13] * T(0x1.5555555555555p-5) + q[19] * T(0x1.3e93e93e93e94p-6))));
    emit(2, 3, ((q[5] * T(-0x1.6c16c16c16c17p-9) + q[11] * T(-0x1.6c16c16c16c17p-9)) + (q[17] * T(-0x1.c71c71c71c71cp-7) + q[23] * T(-0x1.c71c71c71c71cp-7))));
    emit(2, 4, ((fma(q[13], T(0x1.6c16c16c16c17p-7), q[1] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.1111111111111p-4), q[5] * T(0x1.6c16c16c16c17p-7))) + (fma(q[19], T(-0x1.6c16c16c16c17p-6), q[7] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(0x1.6c16c16c16c17p-7), q[11] * T(0x1.6c16c16c16c17p-7)))));
    emit(2, 5, ((fma(q[15], T(0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[5] * T(-0x1.6c16c16c16c17p-7))) + (fma(q[21], T(-0x1.6c16c16c16c17p-6), q[9] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(-0x1.6c16c16c16c17p-7), q[11] * T(-0x1.6c16c16c16c17p-6)))));
    emit(2, 6, ((fma(q[13], T(0x1.6c16c16c16c17p-7), q[1] * T(-0x1.6c16c16c16c17p-7)) + fma(q[15], T(0x1.1111111111111p-4), q[3] * T(0x1.6c16c16c16c17p-7))) + (fma(q[19], T(-0x1.6c16c16c16c17p-7), q[7] * T(-0x1.6c16c16c16c17p-6)) + fma(q[21], T(0x1.6c16c16c16c17p-7), q[9] * T(0x1.6c16c16c16c17p-7)))));
    emit(2, 7, ((fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-7), q[1] * T(0x1.6c16c16c16c17p-7))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[13], T(-0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-7)))) + (fma(q[15], T(-0x1.6c16c16c16c17p-7), q[5] * T(-0x1.6c16c16c16c17p-7)) + fma(q[19], T(0x1.6c16c16c16c17p-6), q[7] * T(0x1.6c16c16c16c17p-7)))));
    emit(2, 8, ((fma(q[17], T(-0x1.1111111111111p-4), fma(q[9], T(-0x1.6c16c16c16c17p-7), q[1] * T(-0x1.1111111111111p-5))) + fma(q[19], T(-0x1.6c16c16c16c17p-6), fma(q[11], T(-0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[21], T(-0x1.6c16c16c16c17p-7), fma(q[13], T(-0x1.c71c71c71c71cp-5), q[5] * T(-0x1.6c16c16c16c17p-7))) + fma(q[23], T(-0x1.6c16c16c16c17p-7), fma(q[15], T(-0x1.1111111111111p-4), q[7] * T(-0x1.6c16c16c16c17p-6))))));
    emit(2, 9, ((fma(q[19], T(0x1.6c16c16c16c17p-7), fma(q[9], T(0x1.6c16c16c16c17p-7), q[1] * T(0x1.6c16c16c16c17p-7))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[11], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[13], T(-0x1.6c16c16c16c17p-7), q[5] * T(0x1.6c16c16c16c17p-7)) + fma(q[17], T(-0x1.6c16c16c16c17p-7), q[7] * T(0x1.6c16c16c16c17p-6)))));
    emit(3, 3, ((q[2] * T(0x1.3e93e93e93e94p-6) + q[8] * T(0x1.3e93e93e93e94p-6)) + (q[14] * T(0x1.3e93e93e93e94p-6) + q[20] * T(0x1.5555555555555p-5))));
    emit(3, 4, ((fma(q[14], T(-0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[5] * T(0x1.6c16c16c16c17p-7))) + (fma(q[20], T(0x1.6c16c16c16c17p-7), q[8] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(0x1.1111111111111p-4), q[11] * T(0x1.6c16c16c16c17p-7)))));
    emit(3, 5, ((fma(q[14], T(-0x1.6c16c16c16c17p-7), q[2] * T(-0x1.6c16c16c16c17p-7)) + fma(q[16], T(0x1.6c16c16c16c17p-7), q[4] * T(0x1.6c16c16c16c17p-7))) + (fma(q[20], T(0x1.6c16c16c16c17p-7), q[8] * T(-0x1.6c16c16c16c17p-6)) + fma(q[22], T(0x1.1111111111111p-4), q[10] * T(0x1.6c16c16c16c17p-7)))));
    emit(3, 6, ((fma(q[16], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(-0x1.6c16c16c16c17p-7), q[5] * T(-0x1.6c16c16c16c17p-7))) + (fma(q[22], T(0x1.6c16c16c16c17p-7), q[10] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(0x1.6c16c16c16c17p-7), q[11] * T(-0x1.6c16c16c16c17p-6)))));
    emit(3, 7, ((fma(q[17], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(-0x1.6c16c16c16c17p-7), q[2] * T(-0x1.1111111111111p-5))) + fma(q[20], T(-0x1.c71c71c71c71cp-5), fma(q[11], T(-0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[22], T(-0x1.1111111111111p-4), fma(q[14], T(-0x1.6c16c16c16c17p-6), q[5] * T(-0x1.6c16c16c16c17p-7))) + fma(q[23], T(-0x1.1111111111111p-4), fma(q[16], T(-0x1.6c16c16c16c17p-7), q[8] * T(-0x1.6c16c16c16c17p-6))))));
    emit(3, 8, ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.6c16c16c16c17p-7), q[2] * T(0x1.6c16c16c16c17p-7))) + fma(q[22], T(-0x1.6c16c16c16c17p-7), fma(q[14], T(0x1.6c16c16c16c17p-6), q[4] * T(0x1.6c16c16c16c17p-7)))) + (fma(q[16], T(0x1.6c16c16c16c17p-6), q[5] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[8] * T(0x1.6c16c16c16c17p-7)))));
    emit(3, 9, ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.6c16c16c16c17p-7), q[2] * T(0x1.6c16c16c16c17p-7))) + fma(q[23], T(-0x1.6c16c16c16c17p-7), fma(q[11], T(0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[14], T(0x1.6c16c16c16c17p-7), q[5] * T(0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[8] * T(0x1.6c16c16c16c17p-6)))));
    emit(4, 4, ((fma(q[17], T(0x1.6c16c16c16c17p-4), fma(q[8], T(0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-5))) + fma(q[19], T(0x1.1111111111111p-3), fma(q[11], T(0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-5)))) + (fma(q[20], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-5), q[5] * T(0x1.6c16c16c16c17p-5))) + fma(q[23], T(0x1.6c16c16c16c17p-4), fma(q[14], T(0x1.1111111111111p-3), q[7] * T(0x1.6c16c16c16c17p-5))))));
    emit(4, 5, ((fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-5), fma(q[8], T(0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.1111111111111p-3), fma(q[15], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-5))))) + (fma(q[22], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.6c16c16c16c17p-6), q[4] * T(0x1.6c16c16c16c17p-6)))) + fma(q[23], T(0x1.6c16c16c16c17p-5), fma(q[17], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-5), q[5] * T(0x1.6c16c16c16c17p-6)))))));
    emit(4, 6, ((fma(q[19], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.6c16c16c16c17p-6), q[3] * T(0x1.6c16c16c16c17p-6))))) + (fma(q[22], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.1111111111111p-3), fma(q[10], T(0x1.6c16c16c16c17p-5), q[4] * T(0x1.6c16c16c16c17p-5)))) + fma(q[23], T(0x1.6c16c16c16c17p-6), fma(q[17], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.6c16c16c16c17p-5), q[5] * T(0x1.6c16c16c16c17p-6)))))));
    emit(4, 7, ((fma(q[22], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.1111111111111p-4), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-5))))) + fma(q[23], T(-0x1.1111111111111p-3), fma(q[19], T(-0x1.1111111111111p-3), fma(q[13], T(-0x1.6c16c16c16c17p-5), fma(q[7], T(-0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.6c16c16c16c17p-5), q[3] * T(-0x1.6c16c16c16c17p-5)))) + fma(q[21], T(-0x1.1111111111111p-3), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-6)))))));
    emit(4, 8, ((fma(q[22], T(-0x1.6c16c16c16c17p-5), fma(q[16], T(-0x1.1111111111111p-3), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[1] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(-0x1.1111111111111p-4), fma(q[17], T(-0x1.1111111111111p-3), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-5), q[2] * T(-0x1.6c16c16c16c17p-5)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-5), fma(q[14], T(-0x1.1111111111111p-3), fma(q[9], T(-0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.6c16c16c16c17p-5), q[4] * T(-0x1.6c16c16c16c17p-5)))))));
    emit(4, 9, ((fma(q[17], T(-0x1.1111111111111p-4), fma(q[10], T(-0x1.6c16c16c16c17p-6), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[1] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[19], T(-0x1.6c16c16c16c17p-5), fma(q[11], T(-0x1.6c16c16c16c17p-4), fma(q[7], T(-0x1.6c16c16c16c17p-5), q[2] * T(-0x1.6c16c16c16c17p-6))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-6)))) + fma(q[23], T(-0x1.1111111111111p-4), fma(q[14], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.6c16c16c16c17p-6), q[4] * T(0x1.6c16c16c16c17p-6)))))));
    emit(5, 5, ((fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[8], T(0x1.1111111111111p-3), q[0] * T(0x1.6c16c16c16c17p-5))) + fma(q[18], T(0x1.1111111111111p-3), fma(q[10], T(0x1.6c16c16c16c17p-4), q[2] * T(0x1.6c16c16c16c17p-5)))) + (fma(q[20], T(0x1.6c16c16c16c17p-5), fma(q[12], T(0x1.6c16c16c16c17p-5), q[4] * T(0x1.6c16c16c16c17p-5))) + fma(q[22], T(0x1.6c16c16c16c17p-4), fma(q[14], T(0x1.6c16c16c16c17p-5), q[6] * T(0x1.6c16c16c16c17p-5))))));
    emit(5, 6, ((fma(q[18], T(0x1.6c16c16c16c17p-5), fma(q[12], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-6))))) + (fma(q[22], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.6c16c16c16c17p-5), q[4] * T(0x1.6c16c16c16c17p-6)))) + fma(q[23], T(0x1.6c16c16c16c17p-5), fma(q[17], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.1111111111111p-3), q[5] * T(0x1.6c16c16c16c17p-5)))))));
    emit(5, 7, ((fma(q[22], T(-0x1.1111111111111p-3), fma(q[17], T(-0x1.6c16c16c16c17p-6), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-5))))) + fma(q[23], T(-0x1.6c16c16c16c17p-5), fma(q[18], T(-0x1.1111111111111p-3), fma(q[12], T(-0x1.6c16c16c16c17p-5), fma(q[6], T(-0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.6c16c16c16c17p-5), q[3] * T(-0x1.6c16c16c16c17p-5)))) + fma(q[21], T(-0x1.1111111111111p-3), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.1111111111111p-4), q[4] * T(-0x1.6c16c16c16c17p-6)))))));
    emit(5, 8, ((fma(q[17], T(-0x1.6c16c16c16c17p-6), fma(q[12], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[18], T(-0x1.6c16c16c16c17p-5), fma(q[14], T(-0x1.6c16c16c16c17p-5), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-6))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-6)))) + fma(q[22], T(-0x1.1111111111111p-4), fma(q[16], T(-0x1.6c16c16c16c17p-4), fma(q[10], T(-0x1.1111111111111p-4), q[4] * T(-0x1.6c16c16c16c17p-5)))))));
    emit(5, 9, ((fma(q[22], T(-0x1.1111111111111p-4), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.1111111111111p-3), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.6c16c16c16c17p-5), fma(q[11], T(-0x1.1111111111111p-3), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-5)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-5), fma(q[14], T(-0x1.6c16c16c16c17p-5), fma(q[8], T(-0x1.1111111111111p-3), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.6c16c16c16c17p-6), fma(q[9], T(-0x1.6c16c16c16c17p-5), q[4] * T(-0x1.6c16c16c16c17p-6)))))));
    emit(6, 6, ((fma(q[15], T(0x1.6c16c16c16c17p-4), fma(q[7], T(0x1.1111111111111p-3), q[0] * T(0x1.6c16c16c16c17p-5))) + fma(q[18], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.6c16c16c16c17p-4), q[1] * T(0x1.6c16c16c16c17p-5)))) + (fma(q[19], T(0x1.6c16c16c16c17p-5), fma(q[12], T(0x1.1111111111111p-3), q[3] * T(0x1.6c16c16c16c17p-5))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-5), q[6] * T(0x1.6c16c16c16c17p-5))))));
    emit(6, 7, ((fma(q[19], T(-0x1.6c16c16c16c17p-5), fma(q[12], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-4), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-6))))) + (fma(q[22], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.1111111111111p-4), fma(q[7], T(-0x1.6c16c16c16c17p-5), q[3] * T(-0x1.6c16c16c16c17p-5)))) + fma(q[23], T(-0x1.6c16c16c16c17p-6), fma(q[18], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.1111111111111p-4), q[4] * T(0x1.6c16c16c16c17p-6)))))));
    emit(6, 8, ((fma(q[22], T(-0x1.6c16c16c16c17p-5), fma(q[16], T(-0x1.1111111111111p-3), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-5))))) + fma(q[23], T(-0x1.6c16c16c16c17p-6), fma(q[17], T(-0x1.6c16c16c16c17p-5), fma(q[12], T(-0x1.1111111111111p-3), fma(q[6], T(-0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[18], T(-0x1.6c16c16c16c17p-5), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[9], T(-0x1.1111111111111p-4), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.1111111111111p-3), fma(q[10], T(-0x1.6c16c16c16c17p-5), q[4] * T(-0x1.6c16c16c16c17p-5)))))));
    emit(6, 9, ((fma(q[22], T(-0x1.6c16c16c16c17p-6), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.6c16c16c16c17p-5), fma(q[11], T(-0x1.1111111111111p-3), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-5)))))) + (fma(q[19], T(-0x1.6c16c16c16c17p-5), fma(q[13], T(-0x1.6c16c16c16c17p-5), fma(q[7], T(-0x1.1111111111111p-3), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.1111111111111p-4), fma(q[9], T(-0x1.1111111111111p-3), q[4] * T(-0x1.6c16c16c16c17p-6)))))));
    emit(7, 7, ((fma(q[22], T(0x1.6c16c16c16c17p-3), fma(q[18], T(0x1.1111111111111p-3), fma(q[14], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-5)))))) + fma(q[23], T(0x1.6c16c16c16c17p-3), fma(q[19], T(0x1.1111111111111p-3), fma(q[15], T(0x1.6c16c16c16c17p-4), fma(q[11], T(0x1.6c16c16c16c17p-5), fma(q[7], T(0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-5))))))) + (fma(q[20], T(0x1.6c16c16c16c17p-4), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[12], T(0x1.6c16c16c16c17p-5), fma(q[8], T(0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-4))))) + fma(q[21], T(0x1.1111111111111p-2), fma(q[17], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.6c16c16c16c17p-4), q[3] * T(0x1.6c16c16c16c17p-4))))))));
    emit(7, 8, ((fma(q[22], T(0x1.1111111111111p-4), fma(q[17], T(0x1.1111111111111p-4), fma(q[12], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.1111111111111p-4), fma(q[18], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[15], T(0x1.1111111111111p-4), fma(q[10], T(0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.6c16c16c16c17p-5), q[5] * T(0x1.6c16c16c16c17p-4)))))));
    emit(7, 9, ((fma(q[22], T(0x1.1111111111111p-4), fma(q[17], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.1111111111111p-4), fma(q[19], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[15], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.1111111111111p-4), q[2] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.1111111111111p-4), q[4] * T(0x1.6c16c16c16c17p-4)))))));
    emit(8, 8, ((fma(q[22], T(0x1.6c16c16c16c17p-4), fma(q[18], T(0x1.6c16c16c16c17p-5), fma(q[14], T(0x1.1111111111111p-3), fma(q[10], T(0x1.6c16c16c16c17p-4), fma(q[6], T(0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-5)))))) + fma(q[23], T(0x1.6c16c16c16c17p-5), fma(q[19], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.6c16c16c16c17p-3), fma(q[11], T(0x1.6c16c16c16c17p-5), fma(q[7], T(0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-4))))))) + (fma(q[20], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.1111111111111p-2), fma(q[12], T(0x1.1111111111111p-3), fma(q[8], T(0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-5))))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[17], T(0x1.6c16c16c16c17p-3), fma(q[13], T(0x1.6c16c16c16c17p-4), fma(q[9], T(0x1.6c16c16c16c17p-5), q[4] * T(0x1.6c16c16c16c17p-4))))))));
    emit(8, 9, ((fma(q[22], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.6c16c16c16c17p-6), fma(q[17], T(0x1.1111111111111p-4), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[8], T(0x1.6c16c16c16c17p-5), q[1] * T(-0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.1111111111111p-4), q[2] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.1111111111111p-4), fma(q[10], T(0x1.1111111111111p-4), q[3] * T(0x1.6c16c16c16c17p-4)))))));
    emit(9, 9, ((fma(q[22], T(0x1.6c16c16c16c17p-5), fma(q[18], T(0x1.6c16c16c16c17p-5), fma(q[14], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.6c16c16c16c17p-3), fma(q[6], T(0x1.6c16c16c16c17p-4), q[0] * T(0x1.6c16c16c16c17p-4)))))) + fma(q[23], T(0x1.6c16c16c16c17p-4), fma(q[19], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.1111111111111p-2), fma(q[7], T(0x1.1111111111111p-3), q[1] * T(0x1.6c16c16c16c17p-5))))))) + (fma(q[20], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[12], T(0x1.6c16c16c16c17p-5), fma(q[8], T(0x1.1111111111111p-3), q[2] * T(0x1.6c16c16c16c17p-5))))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[17], T(0x1.6c16c16c16c17p-4), fma(q[13], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.6c16c16c16c17p-3), q[5] * T(0x1.6c16c16c16c17p-4))))))));
  } else {
    double rs[10] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    { const T v = ((fma(q[16], T(0x1.6c16c16c16c17p-9), fma(q[9], T(0x1.c71c71c71c71cp-7), q[0] * T(0x1.c71c71c71c71cp-7))) + fma(q[18], T(0x1.6c16c16c16c17p-9), fma(q[10], T(0x1.c71c71c71c71cp-7), q[3] * T(0x1.c71c71c71c71cp-7)))) + (fma(q[21], T(0x1.6c16c16c16c17p-9), fma(q[12], T(0x1.6c16c16c16c17p-9), q[4] * T(0x1.c71c71c71c71cp-7))) + fma(q[22], T(0x1.6c16c16c16c17p-9), fma(q[15], T(0x1.6c16c16c16c17p-9), q[6] * T(0x1.c71c71c71c71cp-7))))); rs[0] += (double)v; rs[1] += (double)v; emit(0, 1, v); }
    { const T v = ((fma(q[17], T(0x1.c71c71c71c71cp-7), fma(q[9], T(0x1.6c16c16c16c17p-9), q[1] * T(0x1.c71c71c71c71cp-7))) + fma(q[19], T(0x1.6c16c16c16c17p-9), fma(q[11], T(0x1.6c16c16c16c17p-9), q[3] * T(0x1.c71c71c71c71cp-7)))) + (fma(q[21], T(0x1.6c16c16c16c17p-9), fma(q[13], T(0x1.c71c71c71c71cp-7), q[5] * T(0x1.c71c71c71c71cp-7))) + fma(q[23], T(0x1.6c16c16c16c17p-9), fma(q[15], T(0x1.c71c71c71c71cp-7), q[7] * T(0x1.6c16c16c16c17p-9))))); rs[0] += (double)v; rs[2] += (double)v; emit(0, 2, v); }
    { const T v = ((fma(q[17], T(0x1.6c16c16c16c17p-9), fma(q[10], T(0x1.6c16c16c16c17p-9), q[2] * T(0x1.c71c71c71c71cp-7))) + fma(q[20], T(0x1.c71c71c71c71cp-7), fma(q[11], T(0x1.6c16c16c16c17p-9), q[4] * T(0x1.c71c71c71c71cp-7)))) + (fma(q[22], T(0x1.c71c71c71c71cp-7), fma(q[14], T(0x1.6c16c16c16c17p-9), q[5] * T(0x1.c71c71c71c71cp-7))) + fma(q[23], T(0x1.c71c71c71c71cp-7), fma(q[16], T(0x1.6c16c16c16c17p-9), q[8] * T(0x1.6c16c16c16c17p-9))))); rs[0] += (double)v; rs[3] += (double)v; emit(0, 3, v); }
    { const T v = ((fma(q[20], T(0x1.6c16c16c16c17p-7), fma(q[15], T(0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.6c16c16c16c17p-7), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-7), q[2] * T(-0x1.6c16c16c16c17p-7)))))) + (fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[17], T(0x1.1111111111111p-5), fma(q[13], T(0x1.6c16c16c16c17p-7), fma(q[8], T(0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[23], T(0x1.1111111111111p-5), fma(q[19], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-7))))))); rs[0] += (double)v; rs[4] += (double)v; emit(0, 4, v); }
    { const T v = ((fma(q[20], T(0x1.6c16c16c16c17p-7), fma(q[15], T(0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.1111111111111p-5), fma(q[5], T(-0x1.6c16c16c16c17p-7), q[0] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-6), fma(q[6], T(0x1.6c16c16c16c17p-7), q[2] * T(-0x1.6c16c16c16c17p-7)))))) + (fma(q[22], T(0x1.1111111111111p-5), fma(q[17], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-7), fma(q[8], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[18], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-7), fma(q[9], T(0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-6))))))); rs[0] += (double)v; rs[5] += (double)v; emit(0, 5, v); }
    { const T v = ((fma(q[19], T(0x1.6c16c16c16c17p-7), fma(q[15], T(0x1.1111111111111p-5), fma(q[10], T(0x1.6c16c16c16c17p-7), fma(q[5], T(-0x1.6c16c16c16c17p-7), q[0] * T(-0x1.6c16c16c16c17p-7))))) + fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-6), fma(q[6], T(0x1.6c16c16c16c17p-7), q[1] * T(-0x1.6c16c16c16c17p-7)))))) + (fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[17], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[18], T(0x1.6c16c16c16c17p-7), fma(q[13], T(0x1.6c16c16c16c17p-7), fma(q[9], T(0x1.1111111111111p-5), q[4] * T(-0x1.6c16c16c16c17p-7))))))); rs[0] += (double)v; rs[6] += (double)v; emit(0, 6, v); }
    { const T v = ((fma(q[20], T(-0x1.1111111111111p-5), fma(q[16], T(-0x1.1111111111111p-5), fma(q[12], T(-0x1.6c16c16c16c17p-7), fma(q[8], T(-0x1.6c16c16c16c17p-6), fma(q[4], T(-0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.1111111111111p-5), fma(q[13], T(-0x1.6c16c16c16c17p-7), fma(q[9], T(-0x1.6c16c16c16c17p-6), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-7))))))) + (fma(q[22], T(-0x1.c71c71c71c71cp-5), fma(q[18], T(-0x1.6c16c16c16c17p-6), fma(q[14], T(-0x1.6c16c16c16c17p-6), fma(q[10], T(-0x1.1111111111111p-5), fma(q[6], T(-0x1.6c16c16c16c17p-7), q[2] * T(-0x1.c71c71c71c71cp-5)))))) + fma(q[23], T(-0x1.c71c71c71c71cp-5), fma(q[19], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-6), fma(q[11], T(-0x1.1111111111111p-5), fma(q[7], T(-0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-6)))))))); rs[0] += (double)v; rs[7] += (double)v; emit(0, 7, v); }
    { const T v = ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[12], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-7), fma(q[4], T(0x1.6c16c16c16c17p-6), q[0] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[21], T(-0x1.1111111111111p-5), fma(q[17], T(-0x1.c71c71c71c71cp-5), fma(q[13], T(-0x1.1111111111111p-5), fma(q[9], T(-0x1.1111111111111p-5), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[1] * T(-0x1.c71c71c71c71cp-5))))))) + (fma(q[22], T(-0x1.6c16c16c16c17p-6), fma(q[18], T(-0x1.6c16c16c16c17p-7), fma(q[14], T(-0x1.6c16c16c16c17p-6), fma(q[10], T(-0x1.6c16c16c16c17p-6), fma(q[6], T(-0x1.6c16c16c16c17p-7), q[2] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[23], T(-0x1.1111111111111p-5), fma(q[19], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.c71c71c71c71cp-5), fma(q[11], T(-0x1.1111111111111p-5), fma(q[7], T(-0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-5)))))))); rs[0] += (double)v; rs[8] += (double)v; emit(0, 8, v); }
    { const T v = ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[16], T(-0x1.1111111111111p-5), fma(q[12], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-6), fma(q[4], T(-0x1.6c16c16c16c17p-5), q[0] * T(-0x1.c71c71c71c71cp-5)))))) + fma(q[21], T(-0x1.1111111111111p-5), fma(q[17], T(-0x1.6c16c16c16c17p-6), fma(q[13], T(-0x1.6c16c16c16c17p-7), fma(q[9], T(-0x1.c71c71c71c71cp-5), fma(q[5], T(0x1.6c16c16c16c17p-6), q[1] * T(0x1.6c16c16c16c17p-7))))))) + (fma(q[22], T(-0x1.1111111111111p-5), fma(q[18], T(-0x1.6c16c16c16c17p-6), fma(q[14], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(-0x1.c71c71c71c71cp-5), fma(q[6], T(-0x1.1111111111111p-5), q[2] * T(0x1.6c16c16c16c17p-7)))))) + fma(q[23], T(-0x1.6c16c16c16c17p-6), fma(q[19], T(-0x1.6c16c16c16c17p-7), fma(q[15], T(-0x1.1111111111111p-5), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[7], T(-0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-5)))))))); rs[0] += (double)v; rs[9] += (double)v; emit(0, 9, v); }
    { const T v = ((q[3] * T(-0x1.6c16c16c16c17p-9) + q[9] * T(-0x1.c71c71c71c71cp-7)) + (q[15] * T(-0x1.c71c71c71c71cp-7) + q[21] * T(-0x1.6c16c16c16c17p-9))); rs[1] += (double)v; rs[2] += (double)v; emit(1, 2, v); }
    { const T v = ((q[4] * T(-0x1.6c16c16c16c17p-9) + q[10] * T(-0x1.c71c71c71c71cp-7)) + (q[16] * T(-0x1.6c16c16c16c17p-9) + q[22] * T(-0x1.c71c71c71c71cp-7))); rs[1] += (double)v; rs[3] += (double)v; emit(1, 3, v); }
    { const T v = ((fma(q[15], T(-0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7)) + fma(q[16], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7))) + (fma(q[21], T(-0x1.6c16c16c16c17p-6), q[9] * T(0x1.6c16c16c16c17p-7)) + fma(q[22], T(-0x1.6c16c16c16c17p-7), q[10] * T(0x1.6c16c16c16c17p-7)))); rs[1] += (double)v; rs[4] += (double)v; emit(1, 4, v); }
    { const T v = ((fma(q[12], T(-0x1.6c16c16c16c17p-7), q[0] * T(-0x1.6c16c16c16c17p-7)) + fma(q[16], T(0x1.6c16c16c16c17p-7), q[4] * T(0x1.6c16c16c16c17p-7))) + (fma(q[18], T(-0x1.6c16c16c16c17p-6), q[6] * T(0x1.6c16c16c16c17p-7)) + fma(q[22], T(0x1.6c16c16c16c17p-7), q[10] * T(0x1.1111111111111p-4)))); rs[1] += (double)v; rs[5] += (double)v; emit(1, 5, v); }
    { const T v = ((fma(q[12], T(-0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-7)) + fma(q[15], T(0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-7))) + (fma(q[18], T(-0x1.6c16c16c16c17p-7), q[6] * T(0x1.6c16c16c16c17p-7)) + fma(q[21], T(0x1.6c16c16c16c17p-7), q[9] * T(0x1.1111111111111p-4)))); rs[1] += (double)v; rs[6] += (double)v; emit(1, 6, v); }
    { const T v = ((fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[9], T(-0x1.6c16c16c16c17p-7), q[0] * T(0x1.6c16c16c16c17p-7))) + fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-7)))) + (fma(q[15], T(0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-7)) + fma(q[18], T(0x1.6c16c16c16c17p-6), q[6] * T(-0x1.6c16c16c16c17p-7)))); rs[1] += (double)v; rs[7] += (double)v; emit(1, 7, v); }
    { const T v = ((fma(q[18], T(0x1.6c16c16c16c17p-7), fma(q[10], T(-0x1.6c16c16c16c17p-7), q[0] * T(0x1.6c16c16c16c17p-7))) + fma(q[22], T(0x1.6c16c16c16c17p-7), fma(q[12], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[15], T(0x1.6c16c16c16c17p-7), q[4] * T(0x1.6c16c16c16c17p-7)) + fma(q[16], T(0x1.6c16c16c16c17p-6), q[6] * T(-0x1.6c16c16c16c17p-7)))); rs[1] += (double)v; rs[8] += (double)v; emit(1, 8, v); }
    { const T v = ((fma(q[16], T(-0x1.6c16c16c16c17p-7), fma(q[9], T(-0x1.1111111111111p-4), q[0] * T(-0x1.1111111111111p-5))) + fma(q[18], T(-0x1.6c16c16c16c17p-6), fma(q[10], T(-0x1.1111111111111p-4), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[21], T(-0x1.6c16c16c16c17p-7), fma(q[12], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7))) + fma(q[22], T(-0x1.6c16c16c16c17p-7), fma(q[15], T(-0x1.6c16c16c16c17p-7), q[6] * T(-0x1.c71c71c71c71cp-5))))); rs[1] += (double)v; rs[9] += (double)v; emit(1, 9, v); }
    { const T v = ((q[5] * T(-0x1.6c16c16c16c17p-9) + q[11] * T(-0x1.6c16c16c16c17p-9)) + (q[17] * T(-0x1.c71c71c71c71cp-7) + q[23] * T(-0x1.c71c71c71c71cp-7))); rs[2] += (double)v; rs[3] += (double)v; emit(2, 3, v); }
    { const T v = ((fma(q[13], T(0x1.6c16c16c16c17p-7), q[1] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.1111111111111p-4), q[5] * T(0x1.6c16c16c16c17p-7))) + (fma(q[19], T(-0x1.6c16c16c16c17p-6), q[7] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(0x1.6c16c16c16c17p-7), q[11] * T(0x1.6c16c16c16c17p-7)))); rs[2] += (double)v; rs[4] += (double)v; emit(2, 4, v); }
    { const T v = ((fma(q[15], T(0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[5] * T(-0x1.6c16c16c16c17p-7))) + (fma(q[21], T(-0x1.6c16c16c16c17p-6), q[9] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(-0x1.6c16c16c16c17p-7), q[11] * T(-0x1.6c16c16c16c17p-6)))); rs[2] += (double)v; rs[5] += (double)v; emit(2, 5, v); }
    { const T v = ((fma(q[13], T(0x1.6c16c16c16c17p-7), q[1] * T(-0x1.6c16c16c16c17p-7)) + fma(q[15], T(0x1.1111111111111p-4), q[3] * T(0x1.6c16c16c16c17p-7))) + (fma(q[19], T(-0x1.6c16c16c16c17p-7), q[7] * T(-0x1.6c16c16c16c17p-6)) + fma(q[21], T(0x1.6c16c16c16c17p-7), q[9] * T(0x1.6c16c16c16c17p-7)))); rs[2] += (double)v; rs[6] += (double)v; emit(2, 6, v); }
    { const T v = ((fma(q[21], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-7), q[1] * T(0x1.6c16c16c16c17p-7))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[13], T(-0x1.6c16c16c16c17p-7), q[3] * T(0x1.6c16c16c16c17p-7)))) + (fma(q[15], T(-0x1.6c16c16c16c17p-7), q[5] * T(-0x1.6c16c16c16c17p-7)) + fma(q[19], T(0x1.6c16c16c16c17p-6), q[7] * T(0x1.6c16c16c16c17p-7)))); rs[2] += (double)v; rs[7] += (double)v; emit(2, 7, v); }
    { const T v = ((fma(q[17], T(-0x1.1111111111111p-4), fma(q[9], T(-0x1.6c16c16c16c17p-7), q[1] * T(-0x1.1111111111111p-5))) + fma(q[19], T(-0x1.6c16c16c16c17p-6), fma(q[11], T(-0x1.6c16c16c16c17p-7), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[21], T(-0x1.6c16c16c16c17p-7), fma(q[13], T(-0x1.c71c71c71c71cp-5), q[5] * T(-0x1.6c16c16c16c17p-7))) + fma(q[23], T(-0x1.6c16c16c16c17p-7), fma(q[15], T(-0x1.1111111111111p-4), q[7] * T(-0x1.6c16c16c16c17p-6))))); rs[2] += (double)v; rs[8] += (double)v; emit(2, 8, v); }
    { const T v = ((fma(q[19], T(0x1.6c16c16c16c17p-7), fma(q[9], T(0x1.6c16c16c16c17p-7), q[1] * T(0x1.6c16c16c16c17p-7))) + fma(q[23], T(0x1.6c16c16c16c17p-7), fma(q[11], T(0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[13], T(-0x1.6c16c16c16c17p-7), q[5] * T(0x1.6c16c16c16c17p-7)) + fma(q[17], T(-0x1.6c16c16c16c17p-7), q[7] * T(0x1.6c16c16c16c17p-6)))); rs[2] += (double)v; rs[9] += (double)v; emit(2, 9, v); }
    { const T v = ((fma(q[14], T(-0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[5] * T(0x1.6c16c16c16c17p-7))) + (fma(q[20], T(0x1.6c16c16c16c17p-7), q[8] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(0x1.1111111111111p-4), q[11] * T(0x1.6c16c16c16c17p-7)))); rs[3] += (double)v; rs[4] += (double)v; emit(3, 4, v); }
    { const T v = ((fma(q[14], T(-0x1.6c16c16c16c17p-7), q[2] * T(-0x1.6c16c16c16c17p-7)) + fma(q[16], T(0x1.6c16c16c16c17p-7), q[4] * T(0x1.6c16c16c16c17p-7))) + (fma(q[20], T(0x1.6c16c16c16c17p-7), q[8] * T(-0x1.6c16c16c16c17p-6)) + fma(q[22], T(0x1.1111111111111p-4), q[10] * T(0x1.6c16c16c16c17p-7)))); rs[3] += (double)v; rs[5] += (double)v; emit(3, 5, v); }
    { const T v = ((fma(q[16], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(-0x1.6c16c16c16c17p-7), q[5] * T(-0x1.6c16c16c16c17p-7))) + (fma(q[22], T(0x1.6c16c16c16c17p-7), q[10] * T(-0x1.6c16c16c16c17p-7)) + fma(q[23], T(0x1.6c16c16c16c17p-7), q[11] * T(-0x1.6c16c16c16c17p-6)))); rs[3] += (double)v; rs[6] += (double)v; emit(3, 6, v); }
    { const T v = ((fma(q[17], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(-0x1.6c16c16c16c17p-7), q[2] * T(-0x1.1111111111111p-5))) + fma(q[20], T(-0x1.c71c71c71c71cp-5), fma(q[11], T(-0x1.6c16c16c16c17p-7), q[4] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[22], T(-0x1.1111111111111p-4), fma(q[14], T(-0x1.6c16c16c16c17p-6), q[5] * T(-0x1.6c16c16c16c17p-7))) + fma(q[23], T(-0x1.1111111111111p-4), fma(q[16], T(-0x1.6c16c16c16c17p-7), q[8] * T(-0x1.6c16c16c16c17p-6))))); rs[3] += (double)v; rs[7] += (double)v; emit(3, 7, v); }
    { const T v = ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.6c16c16c16c17p-7), q[2] * T(0x1.6c16c16c16c17p-7))) + fma(q[22], T(-0x1.6c16c16c16c17p-7), fma(q[14], T(0x1.6c16c16c16c17p-6), q[4] * T(0x1.6c16c16c16c17p-7)))) + (fma(q[16], T(0x1.6c16c16c16c17p-6), q[5] * T(-0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[8] * T(0x1.6c16c16c16c17p-7)))); rs[3] += (double)v; rs[8] += (double)v; emit(3, 8, v); }
    { const T v = ((fma(q[20], T(-0x1.6c16c16c16c17p-7), fma(q[10], T(0x1.6c16c16c16c17p-7), q[2] * T(0x1.6c16c16c16c17p-7))) + fma(q[23], T(-0x1.6c16c16c16c17p-7), fma(q[11], T(0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-7)))) + (fma(q[14], T(0x1.6c16c16c16c17p-7), q[5] * T(0x1.6c16c16c16c17p-7)) + fma(q[17], T(0x1.6c16c16c16c17p-7), q[8] * T(0x1.6c16c16c16c17p-6)))); rs[3] += (double)v; rs[9] += (double)v; emit(3, 9, v); }
    { const T v = ((fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-5), fma(q[8], T(0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.1111111111111p-3), fma(q[15], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-5))))) + (fma(q[22], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.6c16c16c16c17p-6), q[4] * T(0x1.6c16c16c16c17p-6)))) + fma(q[23], T(0x1.6c16c16c16c17p-5), fma(q[17], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-5), q[5] * T(0x1.6c16c16c16c17p-6)))))); rs[4] += (double)v; rs[5] += (double)v; emit(4, 5, v); }
    { const T v = ((fma(q[19], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.6c16c16c16c17p-6), q[3] * T(0x1.6c16c16c16c17p-6))))) + (fma(q[22], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.1111111111111p-3), fma(q[10], T(0x1.6c16c16c16c17p-5), q[4] * T(0x1.6c16c16c16c17p-5)))) + fma(q[23], T(0x1.6c16c16c16c17p-6), fma(q[17], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.6c16c16c16c17p-5), q[5] * T(0x1.6c16c16c16c17p-6)))))); rs[4] += (double)v; rs[6] += (double)v; emit(4, 6, v); }
    { const T v = ((fma(q[22], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.1111111111111p-4), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-5))))) + fma(q[23], T(-0x1.1111111111111p-3), fma(q[19], T(-0x1.1111111111111p-3), fma(q[13], T(-0x1.6c16c16c16c17p-5), fma(q[7], T(-0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.6c16c16c16c17p-5), q[3] * T(-0x1.6c16c16c16c17p-5)))) + fma(q[21], T(-0x1.1111111111111p-3), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.6c16c16c16c17p-6), q[4] * T(-0x1.6c16c16c16c17p-6)))))); rs[4] += (double)v; rs[7] += (double)v; emit(4, 7, v); }
    { const T v = ((fma(q[22], T(-0x1.6c16c16c16c17p-5), fma(q[16], T(-0x1.1111111111111p-3), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[1] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(-0x1.1111111111111p-4), fma(q[17], T(-0x1.1111111111111p-3), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-5), q[2] * T(-0x1.6c16c16c16c17p-5)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-5), fma(q[14], T(-0x1.1111111111111p-3), fma(q[9], T(-0x1.6c16c16c16c17p-6), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.6c16c16c16c17p-5), q[4] * T(-0x1.6c16c16c16c17p-5)))))); rs[4] += (double)v; rs[8] += (double)v; emit(4, 8, v); }
    { const T v = ((fma(q[17], T(-0x1.1111111111111p-4), fma(q[10], T(-0x1.6c16c16c16c17p-6), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[1] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[19], T(-0x1.6c16c16c16c17p-5), fma(q[11], T(-0x1.6c16c16c16c17p-4), fma(q[7], T(-0x1.6c16c16c16c17p-5), q[2] * T(-0x1.6c16c16c16c17p-6))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-6)))) + fma(q[23], T(-0x1.1111111111111p-4), fma(q[14], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.6c16c16c16c17p-6), q[4] * T(0x1.6c16c16c16c17p-6)))))); rs[4] += (double)v; rs[9] += (double)v; emit(4, 9, v); }
    { const T v = ((fma(q[18], T(0x1.6c16c16c16c17p-5), fma(q[12], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-6))))) + (fma(q[22], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.6c16c16c16c17p-5), q[4] * T(0x1.6c16c16c16c17p-6)))) + fma(q[23], T(0x1.6c16c16c16c17p-5), fma(q[17], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.1111111111111p-3), q[5] * T(0x1.6c16c16c16c17p-5)))))); rs[5] += (double)v; rs[6] += (double)v; emit(5, 6, v); }
    { const T v = ((fma(q[22], T(-0x1.1111111111111p-3), fma(q[17], T(-0x1.6c16c16c16c17p-6), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-5))))) + fma(q[23], T(-0x1.6c16c16c16c17p-5), fma(q[18], T(-0x1.1111111111111p-3), fma(q[12], T(-0x1.6c16c16c16c17p-5), fma(q[6], T(-0x1.6c16c16c16c17p-5), q[2] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.6c16c16c16c17p-5), q[3] * T(-0x1.6c16c16c16c17p-5)))) + fma(q[21], T(-0x1.1111111111111p-3), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.1111111111111p-4), q[4] * T(-0x1.6c16c16c16c17p-6)))))); rs[5] += (double)v; rs[7] += (double)v; emit(5, 7, v); }
    { const T v = ((fma(q[17], T(-0x1.6c16c16c16c17p-6), fma(q[12], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[18], T(-0x1.6c16c16c16c17p-5), fma(q[14], T(-0x1.6c16c16c16c17p-5), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-6))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.6c16c16c16c17p-6), fma(q[8], T(-0x1.6c16c16c16c17p-5), q[3] * T(0x1.6c16c16c16c17p-6)))) + fma(q[22], T(-0x1.1111111111111p-4), fma(q[16], T(-0x1.6c16c16c16c17p-4), fma(q[10], T(-0x1.1111111111111p-4), q[4] * T(-0x1.6c16c16c16c17p-5)))))); rs[5] += (double)v; rs[8] += (double)v; emit(5, 8, v); }
    { const T v = ((fma(q[22], T(-0x1.1111111111111p-4), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.1111111111111p-3), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.6c16c16c16c17p-5), fma(q[11], T(-0x1.1111111111111p-3), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-5)))))) + (fma(q[20], T(-0x1.6c16c16c16c17p-5), fma(q[14], T(-0x1.6c16c16c16c17p-5), fma(q[8], T(-0x1.1111111111111p-3), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.6c16c16c16c17p-6), fma(q[9], T(-0x1.6c16c16c16c17p-5), q[4] * T(-0x1.6c16c16c16c17p-6)))))); rs[5] += (double)v; rs[9] += (double)v; emit(5, 9, v); }
    { const T v = ((fma(q[19], T(-0x1.6c16c16c16c17p-5), fma(q[12], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-4), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-6))))) + (fma(q[22], T(-0x1.6c16c16c16c17p-6), fma(q[15], T(-0x1.1111111111111p-4), fma(q[7], T(-0x1.6c16c16c16c17p-5), q[3] * T(-0x1.6c16c16c16c17p-5)))) + fma(q[23], T(-0x1.6c16c16c16c17p-6), fma(q[18], T(-0x1.6c16c16c16c17p-5), fma(q[9], T(-0x1.1111111111111p-4), q[4] * T(0x1.6c16c16c16c17p-6)))))); rs[6] += (double)v; rs[7] += (double)v; emit(6, 7, v); }
    { const T v = ((fma(q[22], T(-0x1.6c16c16c16c17p-5), fma(q[16], T(-0x1.1111111111111p-3), fma(q[11], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-5))))) + fma(q[23], T(-0x1.6c16c16c16c17p-6), fma(q[17], T(-0x1.6c16c16c16c17p-5), fma(q[12], T(-0x1.1111111111111p-3), fma(q[6], T(-0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[18], T(-0x1.6c16c16c16c17p-5), fma(q[13], T(-0x1.6c16c16c16c17p-6), fma(q[9], T(-0x1.1111111111111p-4), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.1111111111111p-3), fma(q[10], T(-0x1.6c16c16c16c17p-5), q[4] * T(-0x1.6c16c16c16c17p-5)))))); rs[6] += (double)v; rs[8] += (double)v; emit(6, 8, v); }
    { const T v = ((fma(q[22], T(-0x1.6c16c16c16c17p-6), fma(q[16], T(-0x1.6c16c16c16c17p-5), fma(q[10], T(-0x1.6c16c16c16c17p-5), fma(q[5], T(-0x1.6c16c16c16c17p-5), q[0] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(-0x1.6c16c16c16c17p-5), fma(q[17], T(-0x1.6c16c16c16c17p-5), fma(q[11], T(-0x1.1111111111111p-3), fma(q[6], T(-0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-5)))))) + (fma(q[19], T(-0x1.6c16c16c16c17p-5), fma(q[13], T(-0x1.6c16c16c16c17p-5), fma(q[7], T(-0x1.1111111111111p-3), q[3] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(-0x1.6c16c16c16c17p-5), fma(q[15], T(-0x1.1111111111111p-4), fma(q[9], T(-0x1.1111111111111p-3), q[4] * T(-0x1.6c16c16c16c17p-6)))))); rs[6] += (double)v; rs[9] += (double)v; emit(6, 9, v); }
    { const T v = ((fma(q[22], T(0x1.1111111111111p-4), fma(q[17], T(0x1.1111111111111p-4), fma(q[12], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.1111111111111p-4), fma(q[18], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.6c16c16c16c17p-6), q[1] * T(-0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[15], T(0x1.1111111111111p-4), fma(q[10], T(0x1.6c16c16c16c17p-6), q[2] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.6c16c16c16c17p-5), q[5] * T(0x1.6c16c16c16c17p-4)))))); rs[7] += (double)v; rs[8] += (double)v; emit(7, 8, v); }
    { const T v = ((fma(q[22], T(0x1.1111111111111p-4), fma(q[17], T(0x1.6c16c16c16c17p-6), fma(q[11], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.1111111111111p-4), fma(q[19], T(0x1.6c16c16c16c17p-5), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[7], T(0x1.6c16c16c16c17p-5), q[1] * T(0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[15], T(0x1.6c16c16c16c17p-6), fma(q[9], T(0x1.1111111111111p-4), q[2] * T(-0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[10], T(0x1.1111111111111p-4), q[4] * T(0x1.6c16c16c16c17p-4)))))); rs[7] += (double)v; rs[9] += (double)v; emit(7, 9, v); }
    { const T v = ((fma(q[22], T(0x1.6c16c16c16c17p-6), fma(q[16], T(0x1.6c16c16c16c17p-5), fma(q[11], T(0x1.6c16c16c16c17p-5), fma(q[6], T(0x1.6c16c16c16c17p-6), q[0] * T(-0x1.6c16c16c16c17p-6))))) + fma(q[23], T(0x1.6c16c16c16c17p-6), fma(q[17], T(0x1.1111111111111p-4), fma(q[13], T(0x1.6c16c16c16c17p-6), fma(q[8], T(0x1.6c16c16c16c17p-5), q[1] * T(-0x1.6c16c16c16c17p-6)))))) + (fma(q[20], T(0x1.6c16c16c16c17p-6), fma(q[14], T(0x1.6c16c16c16c17p-5), fma(q[9], T(0x1.1111111111111p-4), q[2] * T(0x1.6c16c16c16c17p-6)))) + fma(q[21], T(0x1.6c16c16c16c17p-5), fma(q[15], T(0x1.1111111111111p-4), fma(q[10], T(0x1.1111111111111p-4), q[3] * T(0x1.6c16c16c16c17p-4)))))); rs[8] += (double)v; rs[9] += (double)v; emit(8, 9, v); }
    emit(0, 0, -rs[0]);
    emit(1, 1, -rs[1]);
    emit(2, 2, -rs[2]);
    emit(3, 3, -rs[3]);
    emit(4, 4, -rs[4]);
    emit(5, 5, -rs[5]);
    emit(6, 6, -rs[6]);
    emit(7, 7, -rs[7]);
    emit(8, 8, -rs[8]);
    emit(9, 9, -rs[9]);
  }
}
// terms: 744

// P2 stiffness with a cellwise-constant coefficient: g[s] = k * Ghat_s.
template <typename T, typename Emit>
__device__ __forceinline__ void p2_stiffness_const(const T* g, Emit&& emit) {
  if constexpr (sizeof(T) == 8) {
    emit(0, 0, (fma(g[4], T(0x1.999999999999ap-3), fma(g[2], T(0x1.999999999999ap-4), g[0] * T(0x1.999999999999ap-4))) + fma(g[5], T(0x1.999999999999ap-3), fma(g[3], T(0x1.999999999999ap-3), g[1] * T(0x1.999999999999ap-4)))));
    emit(0, 1, (fma(g[4], T(0x1.1111111111111p-5), g[0] * T(0x1.1111111111111p-5)) + g[3] * T(0x1.1111111111111p-5)));
    emit(0, 2, (fma(g[5], T(0x1.1111111111111p-5), g[1] * T(0x1.1111111111111p-5)) + g[3] * T(0x1.1111111111111p-5)));
    emit(0, 3, (fma(g[5], T(0x1.1111111111111p-5), g[2] * T(0x1.1111111111111p-5)) + g[4] * T(0x1.1111111111111p-5)));
    emit(0, 4, (fma(g[5], T(0x1.1111111111111p-4), fma(g[3], T(0x1.1111111111111p-5), g[1] * T(0x1.1111111111111p-5))) + fma(g[4], T(0x1.1111111111111p-5), g[2] * T(0x1.1111111111111p-5))));
    emit(0, 5, (fma(g[5], T(0x1.1111111111111p-5), fma(g[3], T(0x1.1111111111111p-5), g[0] * T(0x1.1111111111111p-5))) + fma(g[4], T(0x1.1111111111111p-4), g[2] * T(0x1.1111111111111p-5))));
    emit(0, 6, (fma(g[5], T(0x1.1111111111111p-5), fma(g[3], T(0x1.1111111111111p-4), g[0] * T(0x1.1111111111111p-5))) + fma(g[4], T(0x1.1111111111111p-5), g[1] * T(0x1.1111111111111p-5))));
    emit(0, 7, (fma(g[4], T(-0x1.5555555555555p-3), fma(g[2], T(-0x1.1111111111111p-3), g[0] * T(-0x1.1111111111111p-5))) + fma(g[5], T(-0x1.5555555555555p-3), fma(g[3], T(-0x1.1111111111111p-4), g[1] * T(-0x1.1111111111111p-5)))));
    emit(0, 8, (fma(g[4], T(-0x1.1111111111111p-4), fma(g[2], T(-0x1.1111111111111p-5), g[0] * T(-0x1.1111111111111p-5))) + fma(g[5], T(-0x1.5555555555555p-3), fma(g[3], T(-0x1.5555555555555p-3), g[1] * T(-0x1.1111111111111p-3)))));
    emit(0, 9, (fma(g[4], T(-0x1.5555555555555p-3), fma(g[2], T(-0x1.1111111111111p-5), g[0] * T(-0x1.1111111111111p-3))) + fma(g[5], T(-0x1.1111111111111p-4), fma(g[3], T(-0x1.5555555555555p-3), g[1] * T(-0x1.1111111111111p-5)))));
    emit(1, 1, g[0] * T(0x1.999999999999ap-4));
    emit(1, 2, g[3] * T(-0x1.1111111111111p-5));
    emit(1, 3, g[4] * T(-0x1.1111111111111p-5));
    emit(1, 4, (g[3] * T(-0x1.1111111111111p-5) + g[4] * T(-0x1.1111111111111p-5)));
    emit(1, 5, (g[0] * T(-0x1.1111111111111p-5) + g[4] * T(0x1.999999999999ap-4)));
    emit(1, 6, (g[0] * T(-0x1.1111111111111p-5) + g[3] * T(0x1.999999999999ap-4)));
    emit(1, 7, (g[0] * T(0x1.1111111111111p-5) + g[3] * T(0x1.1111111111111p-5)));
    emit(1, 8, (g[0] * T(0x1.1111111111111p-5) + g[4] * T(0x1.1111111111111p-5)));
    emit(1, 9, (fma(g[4], T(-0x1.999999999999ap-4), g[0] * T(-0x1.1111111111111p-3)) + g[3] * T(-0x1.999999999999ap-4)));
    emit(2, 2, g[1] * T(0x1.999999999999ap-4));
    emit(2, 3, g[5] * T(-0x1.1111111111111p-5));
    emit(2, 4, (g[1] * T(-0x1.1111111111111p-5) + g[5] * T(0x1.999999999999ap-4)));
    emit(2, 5, (g[3] * T(-0x1.1111111111111p-5) + g[5] * T(-0x1.1111111111111p-5)));
    emit(2, 6, (g[1] * T(-0x1.1111111111111p-5) + g[3] * T(0x1.999999999999ap-4)));
    emit(2, 7, (g[1] * T(0x1.1111111111111p-5) + g[3] * T(0x1.1111111111111p-5)));
    emit(2, 8, (fma(g[5], T(-0x1.999999999999ap-4), g[1] * T(-0x1.1111111111111p-3)) + g[3] * T(-0x1.999999999999ap-4)));
    emit(2, 9, (g[1] * T(0x1.1111111111111p-5) + g[5] * T(0x1.1111111111111p-5)));
    emit(3, 3, g[2] * T(0x1.999999999999ap-4));
    emit(3, 4, (g[2] * T(-0x1.1111111111111p-5) + g[5] * T(0x1.999999999999ap-4)));
    emit(3, 5, (g[2] * T(-0x1.1111111111111p-5) + g[4] * T(0x1.999999999999ap-4)));
    emit(3, 6, (g[4] * T(-0x1.1111111111111p-5) + g[5] * T(-0x1.1111111111111p-5)));
    emit(3, 7, (fma(g[5], T(-0x1.999999999999ap-4), g[2] * T(-0x1.1111111111111p-3)) + g[4] * T(-0x1.999999999999ap-4)));
    emit(3, 8, (g[2] * T(0x1.1111111111111p-5) + g[4] * T(0x1.1111111111111p-5)));
    emit(3, 9, (g[2] * T(0x1.1111111111111p-5) + g[5] * T(0x1.1111111111111p-5)));
    emit(4, 4, (fma(g[5], T(0x1.1111111111111p-2), g[1] * T(0x1.1111111111111p-2)) + g[2] * T(0x1.1111111111111p-2)));
    emit(4, 5, (fma(g[4], T(0x1.1111111111111p-3), g[2] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-2))));
    emit(4, 6, (fma(g[4], T(0x1.1111111111111p-2), g[1] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-3))));
    emit(4, 7, (fma(g[4], T(-0x1.1111111111111p-3), g[1] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-2))));
    emit(4, 8, (fma(g[4], T(-0x1.1111111111111p-2), g[2] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-3))));
    emit(4, 9, (fma(g[5], T(-0x1.1111111111111p-2), g[1] * T(-0x1.1111111111111p-3)) + g[2] * T(-0x1.1111111111111p-3)));
    emit(5, 5, (fma(g[4], T(0x1.1111111111111p-2), g[0] * T(0x1.1111111111111p-2)) + g[2] * T(0x1.1111111111111p-2)));
    emit(5, 6, (fma(g[4], T(0x1.1111111111111p-3), g[0] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-2), g[3] * T(0x1.1111111111111p-3))));
    emit(5, 7, (fma(g[4], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-3), g[3] * T(-0x1.1111111111111p-2))));
    emit(5, 8, (fma(g[4], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-3)) + g[2] * T(-0x1.1111111111111p-3)));
    emit(5, 9, (fma(g[4], T(-0x1.1111111111111p-2), g[2] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-3))));
    emit(6, 6, (fma(g[3], T(0x1.1111111111111p-2), g[0] * T(0x1.1111111111111p-2)) + g[1] * T(0x1.1111111111111p-2)));
    emit(6, 7, (fma(g[3], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-3)) + g[1] * T(-0x1.1111111111111p-3)));
    emit(6, 8, (fma(g[4], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-3), g[3] * T(-0x1.1111111111111p-2))));
    emit(6, 9, (fma(g[4], T(-0x1.1111111111111p-3), g[1] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-2))));
    emit(7, 7, (fma(g[4], T(0x1.1111111111111p-2), fma(g[2], T(0x1.1111111111111p-2), g[0] * T(0x1.1111111111111p-2))) + fma(g[5], T(0x1.1111111111111p-2), fma(g[3], T(0x1.1111111111111p-1), g[1] * T(0x1.1111111111111p-2)))));
    emit(7, 8, (fma(g[4], T(0x1.1111111111111p-3), g[0] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-2), g[3] * T(0x1.1111111111111p-3))));
    emit(7, 9, (fma(g[4], T(0x1.1111111111111p-2), g[1] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-3))));
    emit(8, 8, (fma(g[4], T(0x1.1111111111111p-1), fma(g[2], T(0x1.1111111111111p-2), g[0] * T(0x1.1111111111111p-2))) + fma(g[5], T(0x1.1111111111111p-2), fma(g[3], T(0x1.1111111111111p-2), g[1] * T(0x1.1111111111111p-2)))));
    emit(8, 9, (fma(g[4], T(0x1.1111111111111p-3), g[2] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-2))));
    emit(9, 9, (fma(g[4], T(0x1.1111111111111p-2), fma(g[2], T(0x1.1111111111111p-2), g[0] * T(0x1.1111111111111p-2))) + fma(g[5], T(0x1.1111111111111p-1), fma(g[3], T(0x1.1111111111111p-2), g[1] * T(0x1.1111111111111p-2)))));
  } else {
    double rs[10] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    { const T v = (fma(g[4], T(0x1.1111111111111p-5), g[0] * T(0x1.1111111111111p-5)) + g[3] * T(0x1.1111111111111p-5)); rs[0] += (double)v; rs[1] += (double)v; emit(0, 1, v); }
    { const T v = (fma(g[5], T(0x1.1111111111111p-5), g[1] * T(0x1.1111111111111p-5)) + g[3] * T(0x1.1111111111111p-5)); rs[0] += (double)v; rs[2] += (double)v; emit(0, 2, v); }
    { const T v = (fma(g[5], T(0x1.1111111111111p-5), g[2] * T(0x1.1111111111111p-5)) + g[4] * T(0x1.1111111111111p-5)); rs[0] += (double)v; rs[3] += (double)v; emit(0, 3, v); }
    { const T v = (fma(g[5], T(0x1.1111111111111p-4), fma(g[3], T(0x1.1111111111111p-5), g[1] * T(0x1.1111111111111p-5))) + fma(g[4], T(0x1.1111111111111p-5), g[2] * T(0x1.1111111111111p-5))); rs[0] += (double)v; rs[4] += (double)v; emit(0, 4, v); }
    { const T v = (fma(g[5], T(0x1.1111111111111p-5), fma(g[3], T(0x1.1111111111111p-5), g[0] * T(0x1.1111111111111p-5))) + fma(g[4], T(0x1.1111111111111p-4), g[2] * T(0x1.1111111111111p-5))); rs[0] += (double)v; rs[5] += (double)v; emit(0, 5, v); }
    { const T v = (fma(g[5], T(0x1.1111111111111p-5), fma(g[3], T(0x1.1111111111111p-4), g[0] * T(0x1.1111111111111p-5))) + fma(g[4], T(0x1.1111111111111p-5), g[1] * T(0x1.1111111111111p-5))); rs[0] += (double)v; rs[6] += (double)v; emit(0, 6, v); }
    { const T v = (fma(g[4], T(-0x1.5555555555555p-3), fma(g[2], T(-0x1.1111111111111p-3), g[0] * T(-0x1.1111111111111p-5))) + fma(g[5], T(-0x1.5555555555555p-3), fma(g[3], T(-0x1.1111111111111p-4), g[1] * T(-0x1.1111111111111p-5)))); rs[0] += (double)v; rs[7] += (double)v; emit(0, 7, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-4), fma(g[2], T(-0x1.1111111111111p-5), g[0] * T(-0x1.1111111111111p-5))) + fma(g[5], T(-0x1.5555555555555p-3), fma(g[3], T(-0x1.5555555555555p-3), g[1] * T(-0x1.1111111111111p-3)))); rs[0] += (double)v; rs[8] += (double)v; emit(0, 8, v); }
    { const T v = (fma(g[4], T(-0x1.5555555555555p-3), fma(g[2], T(-0x1.1111111111111p-5), g[0] * T(-0x1.1111111111111p-3))) + fma(g[5], T(-0x1.1111111111111p-4), fma(g[3], T(-0x1.5555555555555p-3), g[1] * T(-0x1.1111111111111p-5)))); rs[0] += (double)v; rs[9] += (double)v; emit(0, 9, v); }
    { const T v = g[3] * T(-0x1.1111111111111p-5); rs[1] += (double)v; rs[2] += (double)v; emit(1, 2, v); }
    { const T v = g[4] * T(-0x1.1111111111111p-5); rs[1] += (double)v; rs[3] += (double)v; emit(1, 3, v); }
    { const T v = (g[3] * T(-0x1.1111111111111p-5) + g[4] * T(-0x1.1111111111111p-5)); rs[1] += (double)v; rs[4] += (double)v; emit(1, 4, v); }
    { const T v = (g[0] * T(-0x1.1111111111111p-5) + g[4] * T(0x1.999999999999ap-4)); rs[1] += (double)v; rs[5] += (double)v; emit(1, 5, v); }
    { const T v = (g[0] * T(-0x1.1111111111111p-5) + g[3] * T(0x1.999999999999ap-4)); rs[1] += (double)v; rs[6] += (double)v; emit(1, 6, v); }
    { const T v = (g[0] * T(0x1.1111111111111p-5) + g[3] * T(0x1.1111111111111p-5)); rs[1] += (double)v; rs[7] += (double)v; emit(1, 7, v); }
    { const T v = (g[0] * T(0x1.1111111111111p-5) + g[4] * T(0x1.1111111111111p-5)); rs[1] += (double)v; rs[8] += (double)v; emit(1, 8, v); }
    { const T v = (fma(g[4], T(-0x1.999999999999ap-4), g[0] * T(-0x1.1111111111111p-3)) + g[3] * T(-0x1.999999999999ap-4)); rs[1] += (double)v; rs[9] += (double)v; emit(1, 9, v); }
    { const T v = g[5] * T(-0x1.1111111111111p-5); rs[2] += (double)v; rs[3] += (double)v; emit(2, 3, v); }
    { const T v = (g[1] * T(-0x1.1111111111111p-5) + g[5] * T(0x1.999999999999ap-4)); rs[2] += (double)v; rs[4] += (double)v; emit(2, 4, v); }
    { const T v = (g[3] * T(-0x1.1111111111111p-5) + g[5] * T(-0x1.1111111111111p-5)); rs[2] += (double)v; rs[5] += (double)v; emit(2, 5, v); }
    { const T v = (g[1] * T(-0x1.1111111111111p-5) + g[3] * T(0x1.999999999999ap-4)); rs[2] += (double)v; rs[6] += (double)v; emit(2, 6, v); }
    { const T v = (g[1] * T(0x1.1111111111111p-5) + g[3] * T(0x1.1111111111111p-5)); rs[2] += (double)v; rs[7] += (double)v; emit(2, 7, v); }
    { const T v = (fma(g[5], T(-0x1.999999999999ap-4), g[1] * T(-0x1.1111111111111p-3)) + g[3] * T(-0x1.999999999999ap-4)); rs[2] += (double)v; rs[8] += (double)v; emit(2, 8, v); }
    { const T v = (g[1] * T(0x1.1111111111111p-5) + g[5] * T(0x1.1111111111111p-5)); rs[2] += (double)v; rs[9] += (double)v; emit(2, 9, v); }
    { const T v = (g[2] * T(-0x1.1111111111111p-5) + g[5] * T(0x1.999999999999ap-4)); rs[3] += (double)v; rs[4] += (double)v; emit(3, 4, v); }
    { const T v = (g[2] * T(-0x1.1111111111111p-5) + g[4] * T(0x1.999999999999ap-4)); rs[3] += (double)v; rs[5] += (double)v; emit(3, 5, v); }
    { const T v = (g[4] * T(-0x1.1111111111111p-5) + g[5] * T(-0x1.1111111111111p-5)); rs[3] += (double)v; rs[6] += (double)v; emit(3, 6, v); }
    { const T v = (fma(g[5], T(-0x1.999999999999ap-4), g[2] * T(-0x1.1111111111111p-3)) + g[4] * T(-0x1.999999999999ap-4)); rs[3] += (double)v; rs[7] += (double)v; emit(3, 7, v); }
    { const T v = (g[2] * T(0x1.1111111111111p-5) + g[4] * T(0x1.1111111111111p-5)); rs[3] += (double)v; rs[8] += (double)v; emit(3, 8, v); }
    { const T v = (g[2] * T(0x1.1111111111111p-5) + g[5] * T(0x1.1111111111111p-5)); rs[3] += (double)v; rs[9] += (double)v; emit(3, 9, v); }
    { const T v = (fma(g[4], T(0x1.1111111111111p-3), g[2] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-2))); rs[4] += (double)v; rs[5] += (double)v; emit(4, 5, v); }
    { const T v = (fma(g[4], T(0x1.1111111111111p-2), g[1] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-3))); rs[4] += (double)v; rs[6] += (double)v; emit(4, 6, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-3), g[1] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-2))); rs[4] += (double)v; rs[7] += (double)v; emit(4, 7, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-2), g[2] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-3))); rs[4] += (double)v; rs[8] += (double)v; emit(4, 8, v); }
    { const T v = (fma(g[5], T(-0x1.1111111111111p-2), g[1] * T(-0x1.1111111111111p-3)) + g[2] * T(-0x1.1111111111111p-3)); rs[4] += (double)v; rs[9] += (double)v; emit(4, 9, v); }
    { const T v = (fma(g[4], T(0x1.1111111111111p-3), g[0] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-2), g[3] * T(0x1.1111111111111p-3))); rs[5] += (double)v; rs[6] += (double)v; emit(5, 6, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-3), g[3] * T(-0x1.1111111111111p-2))); rs[5] += (double)v; rs[7] += (double)v; emit(5, 7, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-3)) + g[2] * T(-0x1.1111111111111p-3)); rs[5] += (double)v; rs[8] += (double)v; emit(5, 8, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-2), g[2] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-3))); rs[5] += (double)v; rs[9] += (double)v; emit(5, 9, v); }
    { const T v = (fma(g[3], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-3)) + g[1] * T(-0x1.1111111111111p-3)); rs[6] += (double)v; rs[7] += (double)v; emit(6, 7, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-2), g[0] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-3), g[3] * T(-0x1.1111111111111p-2))); rs[6] += (double)v; rs[8] += (double)v; emit(6, 8, v); }
    { const T v = (fma(g[4], T(-0x1.1111111111111p-3), g[1] * T(-0x1.1111111111111p-2)) + fma(g[5], T(-0x1.1111111111111p-2), g[3] * T(-0x1.1111111111111p-2))); rs[6] += (double)v; rs[9] += (double)v; emit(6, 9, v); }
    { const T v = (fma(g[4], T(0x1.1111111111111p-3), g[0] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-2), g[3] * T(0x1.1111111111111p-3))); rs[7] += (double)v; rs[8] += (double)v; emit(7, 8, v); }
    { const T v = (fma(g[4], T(0x1.1111111111111p-2), g[1] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-3))); rs[7] += (double)v; rs[9] += (double)v; emit(7, 9, v); }
    { const T v = (fma(g[4], T(0x1.1111111111111p-3), g[2] * T(0x1.1111111111111p-3)) + fma(g[5], T(0x1.1111111111111p-3), g[3] * T(0x1.1111111111111p-2))); rs[8] += (double)v; rs[9] += (double)v; emit(8, 9, v); }
    emit(0, 0, -rs[0]);
    emit(1, 1, -rs[1]);
    emit(2, 2, -rs[2]);
    emit(3, 3, -rs[3]);
    emit(4, 4, -rs[4]);
    emit(5, 5, -rs[5]);
    emit(6, 6, -rs[6]);
    emit(7, 7, -rs[7]);
    emit(8, 8, -rs[8]);
    emit(9, 9, -rs[9]);
  }
}

// Largest |coefficient| of the two P2 stiffness bodies: |A_ij| <= max * sum|q| bounds every entry.
constexpr double kP2P1CoefTermMax = 0x1.1111111111111p-2;
constexpr double kP2ConstTermMax = 0x1.1111111111111p-1;

// One 10x10 block of vector-P2 elasticity: value(i,j) = sum_pq W[p*3+q] *
// int_ref d_p phi_i d_q phi_j.  full=false emits only i <= j (diagonal blocks).
template <typename T, typename Emit>
__device__ __forceinline__ void p2_block_full(const T* W, Emit&& emit) {
  if constexpr (sizeof(T) == 8) {
    emit(0, 0, (fma(W[8], T(0x1.999999999999ap-4), fma(W[6], T(0x1.999999999999ap-4), fma(W[4], T(0x1.999999999999ap-4), fma(W[2], T(0x1.999999999999ap-4), W[0] * T(0x1.999999999999ap-4))))) + fma(W[7], T(0x1.999999999999ap-4), fma(W[5], T(0x1.999999999999ap-4), fma(W[3], T(0x1.999999999999ap-4), W[1] * T(0x1.999999999999ap-4))))));
    emit(0, 1, (fma(W[6], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5)) + W[3] * T(0x1.1111111111111p-5)));
    emit(0, 2, (fma(W[7], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)) + W[4] * T(0x1.1111111111111p-5)));
    emit(0, 3, (fma(W[8], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)) + W[5] * T(0x1.1111111111111p-5)));
    emit(0, 4, (fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))));
    emit(0, 5, (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))));
    emit(0, 6, (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))));
    emit(0, 7, (fma(W[8], T(-0x1.1111111111111p-3), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-5))))));
    emit(0, 8, (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-3))))));
    emit(0, 9, (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-3))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-5))))));
    emit(1, 0, (fma(W[2], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5)) + W[1] * T(0x1.1111111111111p-5)));
    emit(1, 1, W[0] * T(0x1.999999999999ap-4));
    emit(1, 2, W[1] * T(-0x1.1111111111111p-5));
    emit(1, 3, W[2] * T(-0x1.1111111111111p-5));
    emit(1, 4, (W[1] * T(-0x1.1111111111111p-5) + W[2] * T(-0x1.1111111111111p-5)));
    emit(1, 5, (W[0] * T(-0x1.1111111111111p-5) + W[2] * T(0x1.999999999999ap-4)));
    emit(1, 6, (W[0] * T(-0x1.1111111111111p-5) + W[1] * T(0x1.999999999999ap-4)));
    emit(1, 7, (W[0] * T(0x1.1111111111111p-5) + W[1] * T(0x1.1111111111111p-5)));
    emit(1, 8, (W[0] * T(0x1.1111111111111p-5) + W[2] * T(0x1.1111111111111p-5)));
    emit(1, 9, (fma(W[2], T(-0x1.999999999999ap-4), W[0] * T(-0x1.1111111111111p-3)) + W[1] * T(-0x1.999999999999ap-4)));
    emit(2, 0, (fma(W[5], T(0x1.1111111111111p-5), W[3] * T(0x1.1111111111111p-5)) + W[4] * T(0x1.1111111111111p-5)));
    emit(2, 1, W[3] * T(-0x1.1111111111111p-5));
    emit(2, 2, W[4] * T(0x1.999999999999ap-4));
    emit(2, 3, W[5] * T(-0x1.1111111111111p-5));
    emit(2, 4, (W[4] * T(-0x1.1111111111111p-5) + W[5] * T(0x1.999999999999ap-4)));
    emit(2, 5, (W[3] * T(-0x1.1111111111111p-5) + W[5] * T(-0x1.1111111111111p-5)));
    emit(2, 6, (W[3] * T(0x1.999999999999ap-4) + W[4] * T(-0x1.1111111111111p-5)));
    emit(2, 7, (W[3] * T(0x1.1111111111111p-5) + W[4] * T(0x1.1111111111111p-5)));
    emit(2, 8, (fma(W[5], T(-0x1.999999999999ap-4), W[3] * T(-0x1.999999999999ap-4)) + W[4] * T(-0x1.1111111111111p-3)));
    emit(2, 9, (W[4] * T(0x1.1111111111111p-5) + W[5] * T(0x1.1111111111111p-5)));
    emit(3, 0, (fma(W[8], T(0x1.1111111111111p-5), W[6] * T(0x1.1111111111111p-5)) + W[7] * T(0x1.1111111111111p-5)));
    emit(3, 1, W[6] * T(-0x1.1111111111111p-5));
    emit(3, 2, W[7] * T(-0x1.1111111111111p-5));
    emit(3, 3, W[8] * T(0x1.999999999999ap-4));
    emit(3, 4, (W[7] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)));
    emit(3, 5, (W[6] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)));
    emit(3, 6, (W[6] * T(-0x1.1111111111111p-5) + W[7] * T(-0x1.1111111111111p-5)));
    emit(3, 7, (fma(W[8], T(-0x1.1111111111111p-3), W[6] * T(-0x1.999999999999ap-4)) + W[7] * T(-0x1.999999999999ap-4)));
    emit(3, 8, (W[6] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)));
    emit(3, 9, (W[7] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)));
    emit(4, 0, (fma(W[7], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[3] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[6], T(0x1.1111111111111p-5), W[4] * T(0x1.1111111111111p-5)))));
    emit(4, 1, (W[3] * T(-0x1.1111111111111p-5) + W[6] * T(-0x1.1111111111111p-5)));
    emit(4, 2, (W[4] * T(-0x1.1111111111111p-5) + W[7] * T(0x1.999999999999ap-4)));
    emit(4, 3, (W[5] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)));
    emit(4, 4, (fma(W[7], T(0x1.1111111111111p-3), W[4] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-2), W[5] * T(0x1.1111111111111p-3))));
    emit(4, 5, (fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-3), W[5] * T(0x1.1111111111111p-3))));
    emit(4, 6, (fma(W[6], T(0x1.1111111111111p-2), W[3] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-3), W[4] * T(0x1.1111111111111p-3))));
    emit(4, 7, (fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-2))));
    emit(4, 8, (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-2), W[3] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))));
    emit(4, 9, (fma(W[7], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))));
    emit(5, 0, (fma(W[7], T(0x1.1111111111111p-5), fma(W[2], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[6], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))));
    emit(5, 1, (W[0] * T(-0x1.1111111111111p-5) + W[6] * T(0x1.999999999999ap-4)));
    emit(5, 2, (W[1] * T(-0x1.1111111111111p-5) + W[7] * T(-0x1.1111111111111p-5)));
    emit(5, 3, (W[2] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)));
    emit(5, 4, (fma(W[7], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))));
    emit(5, 5, (fma(W[6], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-2), W[2] * T(0x1.1111111111111p-3))));
    emit(5, 6, (fma(W[6], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-3))));
    emit(5, 7, (fma(W[7], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-2))));
    emit(5, 8, (fma(W[6], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))));
    emit(5, 9, (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))));
    emit(6, 0, (fma(W[4], T(0x1.1111111111111p-5), fma(W[2], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[5], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))));
    emit(6, 1, (W[0] * T(-0x1.1111111111111p-5) + W[3] * T(0x1.999999999999ap-4)));
    emit(6, 2, (W[1] * T(0x1.999999999999ap-4) + W[4] * T(-0x1.1111111111111p-5)));
    emit(6, 3, (W[2] * T(-0x1.1111111111111p-5) + W[5] * T(-0x1.1111111111111p-5)));
    emit(6, 4, (fma(W[4], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3)) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-2))));
    emit(6, 5, (fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3)) + fma(W[5], T(0x1.1111111111111p-2), W[2] * T(0x1.1111111111111p-3))));
    emit(6, 6, (fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2)) + fma(W[4], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-3))));
    emit(6, 7, (fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[4], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))));
    emit(6, 8, (fma(W[5], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-2), W[0] * T(-0x1.1111111111111p-2))) + fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))));
    emit(6, 9, (fma(W[5], T(-0x1.1111111111111p-2), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[4], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))));
    emit(7, 0, (fma(W[8], T(-0x1.1111111111111p-3), fma(W[6], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-5))))));
    emit(7, 1, (W[0] * T(0x1.1111111111111p-5) + W[3] * T(0x1.1111111111111p-5)));
    emit(7, 2, (W[1] * T(0x1.1111111111111p-5) + W[4] * T(0x1.1111111111111p-5)));
    emit(7, 3, (fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.999999999999ap-4)) + W[5] * T(-0x1.999999999999ap-4)));
    emit(7, 4, (fma(W[7], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-2), W[1] * T(-0x1.1111111111111p-2))) + fma(W[5], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))));
    emit(7, 5, (fma(W[6], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-2), W[0] * T(-0x1.1111111111111p-2))) + fma(W[5], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))));
    emit(7, 6, (fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[4], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))));
    emit(7, 7, (fma(W[8], T(0x1.1111111111111p-2), fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-2), fma(W[2], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2))))) + fma(W[7], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-2))))));
    emit(7, 8, (fma(W[7], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))));
    emit(7, 9, (fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))));
    emit(8, 0, (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-5))))));
    emit(8, 1, (W[0] * T(0x1.1111111111111p-5) + W[6] * T(0x1.1111111111111p-5)));
    emit(8, 2, (fma(W[7], T(-0x1.999999999999ap-4), W[1] * T(-0x1.999999999999ap-4)) + W[4] * T(-0x1.1111111111111p-3)));
    emit(8, 3, (W[2] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)));
    emit(8, 4, (fma(W[8], T(-0x1.1111111111111p-2), fma(W[5], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-2))));
    emit(8, 5, (fma(W[6], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))));
    emit(8, 6, (fma(W[7], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-2), W[1] * T(-0x1.1111111111111p-3))));
    emit(8, 7, (fma(W[7], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3))) + fma(W[6], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))));
    emit(8, 8, (fma(W[8], T(0x1.1111111111111p-2), fma(W[6], T(0x1.1111111111111p-2), fma(W[4], T(0x1.1111111111111p-2), fma(W[2], T(0x1.1111111111111p-2), W[0] * T(0x1.1111111111111p-2))))) + fma(W[7], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))))));
    emit(8, 9, (fma(W[8], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[7], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))));
    emit(9, 0, (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-3))))));
    emit(9, 1, (fma(W[6], T(-0x1.999999999999ap-4), W[0] * T(-0x1.1111111111111p-3)) + W[3] * T(-0x1.999999999999ap-4)));
    emit(9, 2, (W[4] * T(0x1.1111111111111p-5) + W[7] * T(0x1.1111111111111p-5)));
    emit(9, 3, (W[5] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)));
    emit(9, 4, (fma(W[7], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))));
    emit(9, 5, (fma(W[8], T(-0x1.1111111111111p-2), fma(W[5], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))) + fma(W[6], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-3))));
    emit(9, 6, (fma(W[7], T(-0x1.1111111111111p-2), fma(W[4], T(-0x1.1111111111111p-2), W[1] * T(-0x1.1111111111111p-3))) + fma(W[6], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-3))));
    emit(9, 7, (fma(W[7], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))) + fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-3))));
    emit(9, 8, (fma(W[8], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-3))));
    emit(9, 9, (fma(W[8], T(0x1.1111111111111p-2), fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-2), fma(W[2], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2))))) + fma(W[7], T(0x1.1111111111111p-2), fma(W[5], T(0x1.1111111111111p-2), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))))));
  } else {
    double rs[10] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    double cs[10] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    { const T v = (fma(W[6], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5)) + W[3] * T(0x1.1111111111111p-5)); rs[0] += (double)v; cs[1] += (double)v; emit(0, 1, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)) + W[4] * T(0x1.1111111111111p-5)); rs[0] += (double)v; cs[2] += (double)v; emit(0, 2, v); }
    { const T v = (fma(W[8], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)) + W[5] * T(0x1.1111111111111p-5)); rs[0] += (double)v; cs[3] += (double)v; emit(0, 3, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))); rs[0] += (double)v; cs[4] += (double)v; emit(0, 4, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))); rs[0] += (double)v; cs[5] += (double)v; emit(0, 5, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))); rs[0] += (double)v; cs[6] += (double)v; emit(0, 6, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-3), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-5))))); rs[0] += (double)v; cs[7] += (double)v; emit(0, 7, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-3))))); rs[0] += (double)v; cs[8] += (double)v; emit(0, 8, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-3))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-5))))); rs[0] += (double)v; cs[9] += (double)v; emit(0, 9, v); }
    { const T v = (fma(W[2], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5)) + W[1] * T(0x1.1111111111111p-5)); rs[1] += (double)v; cs[0] += (double)v; emit(1, 0, v); }
    { const T v = W[1] * T(-0x1.1111111111111p-5); rs[1] += (double)v; cs[2] += (double)v; emit(1, 2, v); }
    { const T v = W[2] * T(-0x1.1111111111111p-5); rs[1] += (double)v; cs[3] += (double)v; emit(1, 3, v); }
    { const T v = (W[1] * T(-0x1.1111111111111p-5) + W[2] * T(-0x1.1111111111111p-5)); rs[1] += (double)v; cs[4] += (double)v; emit(1, 4, v); }
    { const T v = (W[0] * T(-0x1.1111111111111p-5) + W[2] * T(0x1.999999999999ap-4)); rs[1] += (double)v; cs[5] += (double)v; emit(1, 5, v); }
    { const T v = (W[0] * T(-0x1.1111111111111p-5) + W[1] * T(0x1.999999999999ap-4)); rs[1] += (double)v; cs[6] += (double)v; emit(1, 6, v); }
    { const T v = (W[0] * T(0x1.1111111111111p-5) + W[1] * T(0x1.1111111111111p-5)); rs[1] += (double)v; cs[7] += (double)v; emit(1, 7, v); }
    { const T v = (W[0] * T(0x1.1111111111111p-5) + W[2] * T(0x1.1111111111111p-5)); rs[1] += (double)v; cs[8] += (double)v; emit(1, 8, v); }
    { const T v = (fma(W[2], T(-0x1.999999999999ap-4), W[0] * T(-0x1.1111111111111p-3)) + W[1] * T(-0x1.999999999999ap-4)); rs[1] += (double)v; cs[9] += (double)v; emit(1, 9, v); }
    { const T v = (fma(W[5], T(0x1.1111111111111p-5), W[3] * T(0x1.1111111111111p-5)) + W[4] * T(0x1.1111111111111p-5)); rs[2] += (double)v; cs[0] += (double)v; emit(2, 0, v); }
    { const T v = W[3] * T(-0x1.1111111111111p-5); rs[2] += (double)v; cs[1] += (double)v; emit(2, 1, v); }
    { const T v = W[5] * T(-0x1.1111111111111p-5); rs[2] += (double)v; cs[3] += (double)v; emit(2, 3, v); }
    { const T v = (W[4] * T(-0x1.1111111111111p-5) + W[5] * T(0x1.999999999999ap-4)); rs[2] += (double)v; cs[4] += (double)v; emit(2, 4, v); }
    { const T v = (W[3] * T(-0x1.1111111111111p-5) + W[5] * T(-0x1.1111111111111p-5)); rs[2] += (double)v; cs[5] += (double)v; emit(2, 5, v); }
    { const T v = (W[3] * T(0x1.999999999999ap-4) + W[4] * T(-0x1.1111111111111p-5)); rs[2] += (double)v; cs[6] += (double)v; emit(2, 6, v); }
    { const T v = (W[3] * T(0x1.1111111111111p-5) + W[4] * T(0x1.1111111111111p-5)); rs[2] += (double)v; cs[7] += (double)v; emit(2, 7, v); }
    { const T v = (fma(W[5], T(-0x1.999999999999ap-4), W[3] * T(-0x1.999999999999ap-4)) + W[4] * T(-0x1.1111111111111p-3)); rs[2] += (double)v; cs[8] += (double)v; emit(2, 8, v); }
    { const T v = (W[4] * T(0x1.1111111111111p-5) + W[5] * T(0x1.1111111111111p-5)); rs[2] += (double)v; cs[9] += (double)v; emit(2, 9, v); }
    { const T v = (fma(W[8], T(0x1.1111111111111p-5), W[6] * T(0x1.1111111111111p-5)) + W[7] * T(0x1.1111111111111p-5)); rs[3] += (double)v; cs[0] += (double)v; emit(3, 0, v); }
    { const T v = W[6] * T(-0x1.1111111111111p-5); rs[3] += (double)v; cs[1] += (double)v; emit(3, 1, v); }
    { const T v = W[7] * T(-0x1.1111111111111p-5); rs[3] += (double)v; cs[2] += (double)v; emit(3, 2, v); }
    { const T v = (W[7] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)); rs[3] += (double)v; cs[4] += (double)v; emit(3, 4, v); }
    { const T v = (W[6] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)); rs[3] += (double)v; cs[5] += (double)v; emit(3, 5, v); }
    { const T v = (W[6] * T(-0x1.1111111111111p-5) + W[7] * T(-0x1.1111111111111p-5)); rs[3] += (double)v; cs[6] += (double)v; emit(3, 6, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-3), W[6] * T(-0x1.999999999999ap-4)) + W[7] * T(-0x1.999999999999ap-4)); rs[3] += (double)v; cs[7] += (double)v; emit(3, 7, v); }
    { const T v = (W[6] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)); rs[3] += (double)v; cs[8] += (double)v; emit(3, 8, v); }
    { const T v = (W[7] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)); rs[3] += (double)v; cs[9] += (double)v; emit(3, 9, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[3] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[6], T(0x1.1111111111111p-5), W[4] * T(0x1.1111111111111p-5)))); rs[4] += (double)v; cs[0] += (double)v; emit(4, 0, v); }
    { const T v = (W[3] * T(-0x1.1111111111111p-5) + W[6] * T(-0x1.1111111111111p-5)); rs[4] += (double)v; cs[1] += (double)v; emit(4, 1, v); }
    { const T v = (W[4] * T(-0x1.1111111111111p-5) + W[7] * T(0x1.999999999999ap-4)); rs[4] += (double)v; cs[2] += (double)v; emit(4, 2, v); }
    { const T v = (W[5] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)); rs[4] += (double)v; cs[3] += (double)v; emit(4, 3, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-3), W[5] * T(0x1.1111111111111p-3))); rs[4] += (double)v; cs[5] += (double)v; emit(4, 5, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-2), W[3] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-3), W[4] * T(0x1.1111111111111p-3))); rs[4] += (double)v; cs[6] += (double)v; emit(4, 6, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-2))); rs[4] += (double)v; cs[7] += (double)v; emit(4, 7, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-2), W[3] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))); rs[4] += (double)v; cs[8] += (double)v; emit(4, 8, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))); rs[4] += (double)v; cs[9] += (double)v; emit(4, 9, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-5), fma(W[2], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[6], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))); rs[5] += (double)v; cs[0] += (double)v; emit(5, 0, v); }
    { const T v = (W[0] * T(-0x1.1111111111111p-5) + W[6] * T(0x1.999999999999ap-4)); rs[5] += (double)v; cs[1] += (double)v; emit(5, 1, v); }
    { const T v = (W[1] * T(-0x1.1111111111111p-5) + W[7] * T(-0x1.1111111111111p-5)); rs[5] += (double)v; cs[2] += (double)v; emit(5, 2, v); }
    { const T v = (W[2] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)); rs[5] += (double)v; cs[3] += (double)v; emit(5, 3, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))); rs[5] += (double)v; cs[4] += (double)v; emit(5, 4, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-3))); rs[5] += (double)v; cs[6] += (double)v; emit(5, 6, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-2))); rs[5] += (double)v; cs[7] += (double)v; emit(5, 7, v); }
    { const T v = (fma(W[6], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))); rs[5] += (double)v; cs[8] += (double)v; emit(5, 8, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))); rs[5] += (double)v; cs[9] += (double)v; emit(5, 9, v); }
    { const T v = (fma(W[4], T(0x1.1111111111111p-5), fma(W[2], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[5], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))); rs[6] += (double)v; cs[0] += (double)v; emit(6, 0, v); }
    { const T v = (W[0] * T(-0x1.1111111111111p-5) + W[3] * T(0x1.999999999999ap-4)); rs[6] += (double)v; cs[1] += (double)v; emit(6, 1, v); }
    { const T v = (W[1] * T(0x1.999999999999ap-4) + W[4] * T(-0x1.1111111111111p-5)); rs[6] += (double)v; cs[2] += (double)v; emit(6, 2, v); }
    { const T v = (W[2] * T(-0x1.1111111111111p-5) + W[5] * T(-0x1.1111111111111p-5)); rs[6] += (double)v; cs[3] += (double)v; emit(6, 3, v); }
    { const T v = (fma(W[4], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3)) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-2))); rs[6] += (double)v; cs[4] += (double)v; emit(6, 4, v); }
    { const T v = (fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3)) + fma(W[5], T(0x1.1111111111111p-2), W[2] * T(0x1.1111111111111p-3))); rs[6] += (double)v; cs[5] += (double)v; emit(6, 5, v); }
    { const T v = (fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[4], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))); rs[6] += (double)v; cs[7] += (double)v; emit(6, 7, v); }
    { const T v = (fma(W[5], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-2), W[0] * T(-0x1.1111111111111p-2))) + fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))); rs[6] += (double)v; cs[8] += (double)v; emit(6, 8, v); }
    { const T v = (fma(W[5], T(-0x1.1111111111111p-2), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[4], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))); rs[6] += (double)v; cs[9] += (double)v; emit(6, 9, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-3), fma(W[6], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-5))))); rs[7] += (double)v; cs[0] += (double)v; emit(7, 0, v); }
    { const T v = (W[0] * T(0x1.1111111111111p-5) + W[3] * T(0x1.1111111111111p-5)); rs[7] += (double)v; cs[1] += (double)v; emit(7, 1, v); }
    { const T v = (W[1] * T(0x1.1111111111111p-5) + W[4] * T(0x1.1111111111111p-5)); rs[7] += (double)v; cs[2] += (double)v; emit(7, 2, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.999999999999ap-4)) + W[5] * T(-0x1.999999999999ap-4)); rs[7] += (double)v; cs[3] += (double)v; emit(7, 3, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-2), W[1] * T(-0x1.1111111111111p-2))) + fma(W[5], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))); rs[7] += (double)v; cs[4] += (double)v; emit(7, 4, v); }
    { const T v = (fma(W[6], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-2), W[0] * T(-0x1.1111111111111p-2))) + fma(W[5], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))); rs[7] += (double)v; cs[5] += (double)v; emit(7, 5, v); }
    { const T v = (fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[4], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))); rs[7] += (double)v; cs[6] += (double)v; emit(7, 6, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))); rs[7] += (double)v; cs[8] += (double)v; emit(7, 8, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))); rs[7] += (double)v; cs[9] += (double)v; emit(7, 9, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-5))))); rs[8] += (double)v; cs[0] += (double)v; emit(8, 0, v); }
    { const T v = (W[0] * T(0x1.1111111111111p-5) + W[6] * T(0x1.1111111111111p-5)); rs[8] += (double)v; cs[1] += (double)v; emit(8, 1, v); }
    { const T v = (fma(W[7], T(-0x1.999999999999ap-4), W[1] * T(-0x1.999999999999ap-4)) + W[4] * T(-0x1.1111111111111p-3)); rs[8] += (double)v; cs[2] += (double)v; emit(8, 2, v); }
    { const T v = (W[2] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)); rs[8] += (double)v; cs[3] += (double)v; emit(8, 3, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-2), fma(W[5], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-2))); rs[8] += (double)v; cs[4] += (double)v; emit(8, 4, v); }
    { const T v = (fma(W[6], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))); rs[8] += (double)v; cs[5] += (double)v; emit(8, 5, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-2), W[1] * T(-0x1.1111111111111p-3))); rs[8] += (double)v; cs[6] += (double)v; emit(8, 6, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3))) + fma(W[6], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))); rs[8] += (double)v; cs[7] += (double)v; emit(8, 7, v); }
    { const T v = (fma(W[8], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[7], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))); rs[8] += (double)v; cs[9] += (double)v; emit(8, 9, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-3))))); rs[9] += (double)v; cs[0] += (double)v; emit(9, 0, v); }
    { const T v = (fma(W[6], T(-0x1.999999999999ap-4), W[0] * T(-0x1.1111111111111p-3)) + W[3] * T(-0x1.999999999999ap-4)); rs[9] += (double)v; cs[1] += (double)v; emit(9, 1, v); }
    { const T v = (W[4] * T(0x1.1111111111111p-5) + W[7] * T(0x1.1111111111111p-5)); rs[9] += (double)v; cs[2] += (double)v; emit(9, 2, v); }
    { const T v = (W[5] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)); rs[9] += (double)v; cs[3] += (double)v; emit(9, 3, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))); rs[9] += (double)v; cs[4] += (double)v; emit(9, 4, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-2), fma(W[5], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))) + fma(W[6], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-3))); rs[9] += (double)v; cs[5] += (double)v; emit(9, 5, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-2), fma(W[4], T(-0x1.1111111111111p-2), W[1] * T(-0x1.1111111111111p-3))) + fma(W[6], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-3))); rs[9] += (double)v; cs[6] += (double)v; emit(9, 6, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))) + fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-3))); rs[9] += (double)v; cs[7] += (double)v; emit(9, 7, v); }
    { const T v = (fma(W[8], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-3))); rs[9] += (double)v; cs[8] += (double)v; emit(9, 8, v); }
    emit(0, 0, -0.5 * (rs[0] + cs[0]));
    emit(1, 1, -0.5 * (rs[1] + cs[1]));
    emit(2, 2, -0.5 * (rs[2] + cs[2]));
    emit(3, 3, -0.5 * (rs[3] + cs[3]));
    emit(4, 4, -0.5 * (rs[4] + cs[4]));
    emit(5, 5, -0.5 * (rs[5] + cs[5]));
    emit(6, 6, -0.5 * (rs[6] + cs[6]));
    emit(7, 7, -0.5 * (rs[7] + cs[7]));
    emit(8, 8, -0.5 * (rs[8] + cs[8]));
    emit(9, 9, -0.5 * (rs[9] + cs[9]));
  }
}

template <typename T, typename Emit>
__device__ __forceinline__ void p2_block_upper(const T* W, Emit&& emit) {
  if constexpr (sizeof(T) == 8) {
    emit(0, 0, (fma(W[8], T(0x1.999999999999ap-4), fma(W[6], T(0x1.999999999999ap-4), fma(W[4], T(0x1.999999999999ap-4), fma(W[2], T(0x1.999999999999ap-4), W[0] * T(0x1.999999999999ap-4))))) + fma(W[7], T(0x1.999999999999ap-4), fma(W[5], T(0x1.999999999999ap-4), fma(W[3], T(0x1.999999999999ap-4), W[1] * T(0x1.999999999999ap-4))))));
    emit(0, 1, (fma(W[6], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5)) + W[3] * T(0x1.1111111111111p-5)));
    emit(0, 2, (fma(W[7], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)) + W[4] * T(0x1.1111111111111p-5)));
    emit(0, 3, (fma(W[8], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)) + W[5] * T(0x1.1111111111111p-5)));
    emit(0, 4, (fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))));
    emit(0, 5, (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))));
    emit(0, 6, (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))));
    emit(0, 7, (fma(W[8], T(-0x1.1111111111111p-3), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-5))))));
    emit(0, 8, (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-3))))));
    emit(0, 9, (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-3))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-5))))));
    emit(1, 1, W[0] * T(0x1.999999999999ap-4));
    emit(1, 2, W[1] * T(-0x1.1111111111111p-5));
    emit(1, 3, W[2] * T(-0x1.1111111111111p-5));
    emit(1, 4, (W[1] * T(-0x1.1111111111111p-5) + W[2] * T(-0x1.1111111111111p-5)));
    emit(1, 5, (W[0] * T(-0x1.1111111111111p-5) + W[2] * T(0x1.999999999999ap-4)));
    emit(1, 6, (W[0] * T(-0x1.1111111111111p-5) + W[1] * T(0x1.999999999999ap-4)));
    emit(1, 7, (W[0] * T(0x1.1111111111111p-5) + W[1] * T(0x1.1111111111111p-5)));
    emit(1, 8, (W[0] * T(0x1.1111111111111p-5) + W[2] * T(0x1.1111111111111p-5)));
    emit(1, 9, (fma(W[2], T(-0x1.999999999999ap-4), W[0] * T(-0x1.1111111111111p-3)) + W[1] * T(-0x1.999999999999ap-4)));
    emit(2, 2, W[4] * T(0x1.999999999999ap-4));
    emit(2, 3, W[5] * T(-0x1.1111111111111p-5));
    emit(2, 4, (W[4] * T(-0x1.1111111111111p-5) + W[5] * T(0x1.999999999999ap-4)));
    emit(2, 5, (W[3] * T(-0x1.1111111111111p-5) + W[5] * T(-0x1.1111111111111p-5)));
    emit(2, 6, (W[3] * T(0x1.999999999999ap-4) + W[4] * T(-0x1.1111111111111p-5)));
    emit(2, 7, (W[3] * T(0x1.1111111111111p-5) + W[4] * T(0x1.1111111111111p-5)));
    emit(2, 8, (fma(W[5], T(-0x1.999999999999ap-4), W[3] * T(-0x1.999999999999ap-4)) + W[4] * T(-0x1.1111111111111p-3)));
    emit(2, 9, (W[4] * T(0x1.1111111111111p-5) + W[5] * T(0x1.1111111111111p-5)));
    emit(3, 3, W[8] * T(0x1.999999999999ap-4));
    emit(3, 4, (W[7] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)));
    emit(3, 5, (W[6] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)));
    emit(3, 6, (W[6] * T(-0x1.1111111111111p-5) + W[7] * T(-0x1.1111111111111p-5)));
    emit(3, 7, (fma(W[8], T(-0x1.1111111111111p-3), W[6] * T(-0x1.999999999999ap-4)) + W[7] * T(-0x1.999999999999ap-4)));
    emit(3, 8, (W[6] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)));
    emit(3, 9, (W[7] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)));
    emit(4, 4, (fma(W[7], T(0x1.1111111111111p-3), W[4] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-2), W[5] * T(0x1.1111111111111p-3))));
    emit(4, 5, (fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-3), W[5] * T(0x1.1111111111111p-3))));
    emit(4, 6, (fma(W[6], T(0x1.1111111111111p-2), W[3] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-3), W[4] * T(0x1.1111111111111p-3))));
    emit(4, 7, (fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-2))));
    emit(4, 8, (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-2), W[3] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))));
    emit(4, 9, (fma(W[7], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))));
    emit(5, 5, (fma(W[6], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-2), W[2] * T(0x1.1111111111111p-3))));
    emit(5, 6, (fma(W[6], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-3))));
    emit(5, 7, (fma(W[7], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-2))));
    emit(5, 8, (fma(W[6], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))));
    emit(5, 9, (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))));
    emit(6, 6, (fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2)) + fma(W[4], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-3))));
    emit(6, 7, (fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[4], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))));
    emit(6, 8, (fma(W[5], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-2), W[0] * T(-0x1.1111111111111p-2))) + fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))));
    emit(6, 9, (fma(W[5], T(-0x1.1111111111111p-2), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[4], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))));
    emit(7, 7, (fma(W[8], T(0x1.1111111111111p-2), fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-2), fma(W[2], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2))))) + fma(W[7], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-2))))));
    emit(7, 8, (fma(W[7], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))));
    emit(7, 9, (fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))));
    emit(8, 8, (fma(W[8], T(0x1.1111111111111p-2), fma(W[6], T(0x1.1111111111111p-2), fma(W[4], T(0x1.1111111111111p-2), fma(W[2], T(0x1.1111111111111p-2), W[0] * T(0x1.1111111111111p-2))))) + fma(W[7], T(0x1.1111111111111p-3), fma(W[5], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))))));
    emit(8, 9, (fma(W[8], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[7], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))));
    emit(9, 9, (fma(W[8], T(0x1.1111111111111p-2), fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-2), fma(W[2], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-2))))) + fma(W[7], T(0x1.1111111111111p-2), fma(W[5], T(0x1.1111111111111p-2), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))))));
  } else {
    double rs[10] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    { const T v = (fma(W[6], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5)) + W[3] * T(0x1.1111111111111p-5)); rs[0] += (double)v; rs[1] += (double)v; emit(0, 1, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)) + W[4] * T(0x1.1111111111111p-5)); rs[0] += (double)v; rs[2] += (double)v; emit(0, 2, v); }
    { const T v = (fma(W[8], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)) + W[5] * T(0x1.1111111111111p-5)); rs[0] += (double)v; rs[3] += (double)v; emit(0, 3, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))); rs[0] += (double)v; rs[4] += (double)v; emit(0, 4, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[8], T(0x1.1111111111111p-5), fma(W[5], T(0x1.1111111111111p-5), W[2] * T(0x1.1111111111111p-5)))); rs[0] += (double)v; rs[5] += (double)v; emit(0, 5, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-5), fma(W[3], T(0x1.1111111111111p-5), W[0] * T(0x1.1111111111111p-5))) + fma(W[7], T(0x1.1111111111111p-5), fma(W[4], T(0x1.1111111111111p-5), W[1] * T(0x1.1111111111111p-5)))); rs[0] += (double)v; rs[6] += (double)v; emit(0, 6, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-3), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-3), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-5))))); rs[0] += (double)v; rs[7] += (double)v; emit(0, 7, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-5), fma(W[4], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-5))))) + fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-5), W[1] * T(-0x1.1111111111111p-3))))); rs[0] += (double)v; rs[8] += (double)v; emit(0, 8, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-5), fma(W[6], T(-0x1.1111111111111p-3), fma(W[4], T(-0x1.1111111111111p-5), fma(W[2], T(-0x1.1111111111111p-5), W[0] * T(-0x1.1111111111111p-3))))) + fma(W[7], T(-0x1.1111111111111p-5), fma(W[5], T(-0x1.1111111111111p-5), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-5))))); rs[0] += (double)v; rs[9] += (double)v; emit(0, 9, v); }
    { const T v = W[1] * T(-0x1.1111111111111p-5); rs[1] += (double)v; rs[2] += (double)v; emit(1, 2, v); }
    { const T v = W[2] * T(-0x1.1111111111111p-5); rs[1] += (double)v; rs[3] += (double)v; emit(1, 3, v); }
    { const T v = (W[1] * T(-0x1.1111111111111p-5) + W[2] * T(-0x1.1111111111111p-5)); rs[1] += (double)v; rs[4] += (double)v; emit(1, 4, v); }
    { const T v = (W[0] * T(-0x1.1111111111111p-5) + W[2] * T(0x1.999999999999ap-4)); rs[1] += (double)v; rs[5] += (double)v; emit(1, 5, v); }
    { const T v = (W[0] * T(-0x1.1111111111111p-5) + W[1] * T(0x1.999999999999ap-4)); rs[1] += (double)v; rs[6] += (double)v; emit(1, 6, v); }
    { const T v = (W[0] * T(0x1.1111111111111p-5) + W[1] * T(0x1.1111111111111p-5)); rs[1] += (double)v; rs[7] += (double)v; emit(1, 7, v); }
    { const T v = (W[0] * T(0x1.1111111111111p-5) + W[2] * T(0x1.1111111111111p-5)); rs[1] += (double)v; rs[8] += (double)v; emit(1, 8, v); }
    { const T v = (fma(W[2], T(-0x1.999999999999ap-4), W[0] * T(-0x1.1111111111111p-3)) + W[1] * T(-0x1.999999999999ap-4)); rs[1] += (double)v; rs[9] += (double)v; emit(1, 9, v); }
    { const T v = W[5] * T(-0x1.1111111111111p-5); rs[2] += (double)v; rs[3] += (double)v; emit(2, 3, v); }
    { const T v = (W[4] * T(-0x1.1111111111111p-5) + W[5] * T(0x1.999999999999ap-4)); rs[2] += (double)v; rs[4] += (double)v; emit(2, 4, v); }
    { const T v = (W[3] * T(-0x1.1111111111111p-5) + W[5] * T(-0x1.1111111111111p-5)); rs[2] += (double)v; rs[5] += (double)v; emit(2, 5, v); }
    { const T v = (W[3] * T(0x1.999999999999ap-4) + W[4] * T(-0x1.1111111111111p-5)); rs[2] += (double)v; rs[6] += (double)v; emit(2, 6, v); }
    { const T v = (W[3] * T(0x1.1111111111111p-5) + W[4] * T(0x1.1111111111111p-5)); rs[2] += (double)v; rs[7] += (double)v; emit(2, 7, v); }
    { const T v = (fma(W[5], T(-0x1.999999999999ap-4), W[3] * T(-0x1.999999999999ap-4)) + W[4] * T(-0x1.1111111111111p-3)); rs[2] += (double)v; rs[8] += (double)v; emit(2, 8, v); }
    { const T v = (W[4] * T(0x1.1111111111111p-5) + W[5] * T(0x1.1111111111111p-5)); rs[2] += (double)v; rs[9] += (double)v; emit(2, 9, v); }
    { const T v = (W[7] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)); rs[3] += (double)v; rs[4] += (double)v; emit(3, 4, v); }
    { const T v = (W[6] * T(0x1.999999999999ap-4) + W[8] * T(-0x1.1111111111111p-5)); rs[3] += (double)v; rs[5] += (double)v; emit(3, 5, v); }
    { const T v = (W[6] * T(-0x1.1111111111111p-5) + W[7] * T(-0x1.1111111111111p-5)); rs[3] += (double)v; rs[6] += (double)v; emit(3, 6, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-3), W[6] * T(-0x1.999999999999ap-4)) + W[7] * T(-0x1.999999999999ap-4)); rs[3] += (double)v; rs[7] += (double)v; emit(3, 7, v); }
    { const T v = (W[6] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)); rs[3] += (double)v; rs[8] += (double)v; emit(3, 8, v); }
    { const T v = (W[7] * T(0x1.1111111111111p-5) + W[8] * T(0x1.1111111111111p-5)); rs[3] += (double)v; rs[9] += (double)v; emit(3, 9, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-3), W[3] * T(0x1.1111111111111p-2)) + fma(W[8], T(0x1.1111111111111p-3), W[5] * T(0x1.1111111111111p-3))); rs[4] += (double)v; rs[5] += (double)v; emit(4, 5, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-2), W[3] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-3), W[4] * T(0x1.1111111111111p-3))); rs[4] += (double)v; rs[6] += (double)v; emit(4, 6, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), fma(W[5], T(-0x1.1111111111111p-3), W[3] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-2))); rs[4] += (double)v; rs[7] += (double)v; emit(4, 7, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-2), W[3] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))); rs[4] += (double)v; rs[8] += (double)v; emit(4, 8, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), W[4] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[5] * T(-0x1.1111111111111p-3))); rs[4] += (double)v; rs[9] += (double)v; emit(4, 9, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3)) + fma(W[7], T(0x1.1111111111111p-2), W[1] * T(0x1.1111111111111p-3))); rs[5] += (double)v; rs[6] += (double)v; emit(5, 6, v); }
    { const T v = (fma(W[7], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-2))) + fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-2))); rs[5] += (double)v; rs[7] += (double)v; emit(5, 7, v); }
    { const T v = (fma(W[6], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[8], T(-0x1.1111111111111p-3), W[2] * T(-0x1.1111111111111p-3))); rs[5] += (double)v; rs[8] += (double)v; emit(5, 8, v); }
    { const T v = (fma(W[8], T(-0x1.1111111111111p-2), fma(W[6], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[7], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))); rs[5] += (double)v; rs[9] += (double)v; emit(5, 9, v); }
    { const T v = (fma(W[3], T(-0x1.1111111111111p-3), W[0] * T(-0x1.1111111111111p-3)) + fma(W[4], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))); rs[6] += (double)v; rs[7] += (double)v; emit(6, 7, v); }
    { const T v = (fma(W[5], T(-0x1.1111111111111p-3), fma(W[2], T(-0x1.1111111111111p-2), W[0] * T(-0x1.1111111111111p-2))) + fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))); rs[6] += (double)v; rs[8] += (double)v; emit(6, 8, v); }
    { const T v = (fma(W[5], T(-0x1.1111111111111p-2), fma(W[3], T(-0x1.1111111111111p-3), W[1] * T(-0x1.1111111111111p-3))) + fma(W[4], T(-0x1.1111111111111p-2), W[2] * T(-0x1.1111111111111p-3))); rs[6] += (double)v; rs[9] += (double)v; emit(6, 9, v); }
    { const T v = (fma(W[7], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[0] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))); rs[7] += (double)v; rs[8] += (double)v; emit(7, 8, v); }
    { const T v = (fma(W[6], T(0x1.1111111111111p-3), fma(W[4], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[5], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))); rs[7] += (double)v; rs[9] += (double)v; emit(7, 9, v); }
    { const T v = (fma(W[8], T(0x1.1111111111111p-3), fma(W[3], T(0x1.1111111111111p-3), W[1] * T(0x1.1111111111111p-3))) + fma(W[7], T(0x1.1111111111111p-3), W[2] * T(0x1.1111111111111p-3))); rs[8] += (double)v; rs[9] += (double)v; emit(8, 9, v); }
    emit(0, 0, -rs[0]);
    emit(1, 1, -rs[1]);
    emit(2, 2, -rs[2]);
    emit(3, 3, -rs[3]);
    emit(4, 4, -rs[4]);
    emit(5, 5, -rs[5]);
    emit(6, 6, -rs[6]);
    emit(7, 7, -rs[7]);
    emit(8, 8, -rs[8]);
    emit(9, 9, -rs[9]);
  }
}

// int_ref d_p phi_i d_q phi_j of the P2 basis, index (i*10 + j)*9 + p*3 + q.
__device__ const double kP2GradGrad[900] = {
    0x1.999999999999ap-4, 0x1.999999999999ap-4, 0x1.999999999999ap-4, 0x1.999999999999ap-4, 0x1.999999999999ap-4, 0x1.999999999999ap-4,
    0x1.999999999999ap-4, 0x1.999999999999ap-4, 0x1.999999999999ap-4, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5,
    0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5,
    0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x1.1111111111111p-5,
    0x1.1111111111111p-5, 0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x1.1111111111111p-5,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-3,
    -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-3, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-3,
    -0x1.1111111111111p-5, -0x1.1111111111111p-3, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-3, -0x1.1111111111111p-5,
    -0x1.1111111111111p-5, -0x1.1111111111111p-3, -0x1.1111111111111p-5, -0x1.1111111111111p-3, -0x1.1111111111111p-5, -0x1.1111111111111p-5,
    -0x1.1111111111111p-3, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-3, -0x1.1111111111111p-5, -0x1.1111111111111p-5,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, -0x1.1111111111111p-5, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x1.999999999999ap-4,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-5, 0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-5, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.999999999999ap-4, -0x1.999999999999ap-4,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x1.999999999999ap-4,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-5, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4, -0x1.1111111111111p-5, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.999999999999ap-4, -0x1.1111111111111p-3, -0x1.999999999999ap-4,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.999999999999ap-4, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4, 0x0.0p+0, -0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-5, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.999999999999ap-4, -0x1.999999999999ap-4, -0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-5, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0,
    0x0.0p+0, 0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-2, 0x1.1111111111111p-3,
    0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-2, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0,
    0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-2, -0x1.1111111111111p-2, -0x1.1111111111111p-3, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3,
    -0x1.1111111111111p-2, -0x1.1111111111111p-3, -0x1.1111111111111p-2, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.999999999999ap-4,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5,
    0x0.0p+0, 0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x0.0p+0, 0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-2,
    0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x0.0p+0, -0x1.1111111111111p-2, -0x1.1111111111111p-2, -0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0,
    -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-2, -0x1.1111111111111p-2,
    0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3,
    0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-2, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0,
    -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-2, -0x1.1111111111111p-3, -0x1.1111111111111p-2, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3,
    -0x1.1111111111111p-3, -0x1.1111111111111p-2, -0x1.1111111111111p-2, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5,
    -0x1.1111111111111p-3, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.999999999999ap-4,
    0x0.0p+0, 0x0.0p+0, -0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3,
    0x0.0p+0, -0x1.1111111111111p-2, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-2, -0x1.1111111111111p-3,
    0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-2, 0x0.0p+0, -0x1.1111111111111p-3,
    -0x1.1111111111111p-2, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-2, 0x1.1111111111111p-2, 0x1.1111111111111p-3,
    0x1.1111111111111p-2, 0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-2,
    0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3,
    0x0.0p+0, 0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3,
    0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-3, -0x1.1111111111111p-3, -0x1.1111111111111p-3,
    -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, -0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0,
    0x0.0p+0, -0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5,
    0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-2, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3,
    0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-2, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3,
    -0x1.1111111111111p-2, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.1111111111111p-2, -0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0,
    0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x1.1111111111111p-3,
    0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3,
    0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3,
    -0x1.1111111111111p-3, -0x1.1111111111111p-3, -0x1.1111111111111p-3, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5,
    -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-5, -0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0,
    -0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0, -0x1.999999999999ap-4, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0,
    0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-5,
    0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3,
    0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-3, 0x0.0p+0, 0x0.0p+0, -0x1.1111111111111p-3,
    -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-2, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-2,
    0x0.0p+0, -0x1.1111111111111p-3, 0x0.0p+0, -0x1.1111111111111p-3, -0x1.1111111111111p-2, 0x0.0p+0,
    -0x1.1111111111111p-3, -0x1.1111111111111p-2, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.1111111111111p-3,
    0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x0.0p+0,
    0x0.0p+0, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3,
    0x1.1111111111111p-3, 0x0.0p+0, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x1.1111111111111p-3,
    0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x1.1111111111111p-2, 0x1.1111111111111p-3, 0x1.1111111111111p-2, 0x1.1111111111111p-2,
};

// P1 mass, cellwise-constant coefficient: s = c * |det J|; emit(i, j, value), i <= j.
template <typename T, typename Emit>
__device__ __forceinline__ void p1_mass_const(T s, Emit&& emit) {
  emit(0, 0, s * T(0x1.1111111111111p-6));
  emit(0, 1, s * T(0x1.1111111111111p-7));
  emit(0, 2, s * T(0x1.1111111111111p-7));
  emit(0, 3, s * T(0x1.1111111111111p-7));
  emit(1, 1, s * T(0x1.1111111111111p-6));
  emit(1, 2, s * T(0x1.1111111111111p-7));
  emit(1, 3, s * T(0x1.1111111111111p-7));
  emit(2, 2, s * T(0x1.1111111111111p-6));
  emit(2, 3, s * T(0x1.1111111111111p-7));
  emit(3, 3, s * T(0x1.1111111111111p-6));
}
// P1 mass, P1 coefficient: cq[m] = c_m * |det J|.
template <typename T, typename Emit>
__device__ __forceinline__ void p1_mass_p1coef(const T* cq, Emit&& emit) {
  emit(0, 0, (fma(cq[2], T(0x1.6c16c16c16c17p-9), cq[0] * T(0x1.1111111111111p-7)) + fma(cq[3], T(0x1.6c16c16c16c17p-9), cq[1] * T(0x1.6c16c16c16c17p-9))));
  emit(0, 1, (fma(cq[2], T(0x1.6c16c16c16c17p-10), cq[0] * T(0x1.6c16c16c16c17p-9)) + fma(cq[3], T(0x1.6c16c16c16c17p-10), cq[1] * T(0x1.6c16c16c16c17p-9))));
  emit(0, 2, (fma(cq[2], T(0x1.6c16c16c16c17p-9), cq[0] * T(0x1.6c16c16c16c17p-9)) + fma(cq[3], T(0x1.6c16c16c16c17p-10), cq[1] * T(0x1.6c16c16c16c17p-10))));
  emit(0, 3, (fma(cq[2], T(0x1.6c16c16c16c17p-10), cq[0] * T(0x1.6c16c16c16c17p-9)) + fma(cq[3], T(0x1.6c16c16c16c17p-9), cq[1] * T(0x1.6c16c16c16c17p-10))));
  emit(1, 1, (fma(cq[2], T(0x1.6c16c16c16c17p-9), cq[0] * T(0x1.6c16c16c16c17p-9)) + fma(cq[3], T(0x1.6c16c16c16c17p-9), cq[1] * T(0x1.1111111111111p-7))));
  emit(1, 2, (fma(cq[2], T(0x1.6c16c16c16c17p-9), cq[0] * T(0x1.6c16c16c16c17p-10)) + fma(cq[3], T(0x1.6c16c16c16c17p-10), cq[1] * T(0x1.6c16c16c16c17p-9))));
  emit(1, 3, (fma(cq[2], T(0x1.6c16c16c16c17p-10), cq[0] * T(0x1.6c16c16c16c17p-10)) + fma(cq[3], T(0x1.6c16c16c16c17p-9), cq[1] * T(0x1.6c16c16c16c17p-9))));
  emit(2, 2, (fma(cq[2], T(0x1.1111111111111p-7), cq[0] * T(0x1.6c16c16c16c17p-9)) + fma(cq[3], T(0x1.6c16c16c16c17p-9), cq[1] * T(0x1.6c16c16c16c17p-9))));
  emit(2, 3, (fma(cq[2], T(0x1.6c16c16c16c17p-9), cq[0] * T(0x1.6c16c16c16c17p-10)) + fma(cq[3], T(0x1.6c16c16c16c17p-9), cq[1] * T(0x1.6c16c16c16c17p-10))));
  emit(3, 3, (fma(cq[2], T(0x1.6c16c16c16c17p-9), cq[0] * T(0x1.6c16c16c16c17p-9)) + fma(cq[3], T(0x1.1111111111111p-7), cq[1] * T(0x1.6c16c16c16c17p-9))));
}

// P2 mass, cellwise-constant coefficient: s = c * |det J|; emit(i, j, value), i <= j.
template <typename T, typename Emit>
__device__ __forceinline__ void p2_mass_const(T s, Emit&& emit) {
  emit(0, 0, s * T(0x1.3813813813814p-9));
  emit(0, 1, s * T(0x1.a01a01a01a01ap-12));
  emit(0, 2, s * T(0x1.a01a01a01a01ap-12));
  emit(0, 3, s * T(0x1.a01a01a01a01ap-12));
  emit(0, 4, s * T(-0x1.3813813813814p-9));
  emit(0, 5, s * T(-0x1.3813813813814p-9));
  emit(0, 6, s * T(-0x1.3813813813814p-9));
  emit(0, 7, s * T(-0x1.a01a01a01a01ap-10));
  emit(0, 8, s * T(-0x1.a01a01a01a01ap-10));
  emit(0, 9, s * T(-0x1.a01a01a01a01ap-10));
  emit(1, 1, s * T(0x1.3813813813814p-9));
  emit(1, 2, s * T(0x1.a01a01a01a01ap-12));
  emit(1, 3, s * T(0x1.a01a01a01a01ap-12));
  emit(1, 4, s * T(-0x1.3813813813814p-9));
  emit(1, 5, s * T(-0x1.a01a01a01a01ap-10));
  emit(1, 6, s * T(-0x1.a01a01a01a01ap-10));
  emit(1, 7, s * T(-0x1.3813813813814p-9));
  emit(1, 8, s * T(-0x1.3813813813814p-9));
  emit(1, 9, s * T(-0x1.a01a01a01a01ap-10));
  emit(2, 2, s * T(0x1.3813813813814p-9));
  emit(2, 3, s * T(0x1.a01a01a01a01ap-12));
  emit(2, 4, s * T(-0x1.a01a01a01a01ap-10));
  emit(2, 5, s * T(-0x1.3813813813814p-9));
  emit(2, 6, s * T(-0x1.a01a01a01a01ap-10));
  emit(2, 7, s * T(-0x1.3813813813814p-9));
  emit(2, 8, s * T(-0x1.a01a01a01a01ap-10));
  emit(2, 9, s * T(-0x1.3813813813814p-9));
  emit(3, 3, s * T(0x1.3813813813814p-9));
  emit(3, 4, s * T(-0x1.a01a01a01a01ap-10));
  emit(3, 5, s * T(-0x1.a01a01a01a01ap-10));
  emit(3, 6, s * T(-0x1.3813813813814p-9));
  emit(3, 7, s * T(-0x1.a01a01a01a01ap-10));
  emit(3, 8, s * T(-0x1.3813813813814p-9));
  emit(3, 9, s * T(-0x1.3813813813814p-9));
  emit(4, 4, s * T(0x1.a01a01a01a01ap-7));
  emit(4, 5, s * T(0x1.a01a01a01a01ap-8));
  emit(4, 6, s * T(0x1.a01a01a01a01ap-8));
  emit(4, 7, s * T(0x1.a01a01a01a01ap-8));
  emit(4, 8, s * T(0x1.a01a01a01a01ap-8));
  emit(4, 9, s * T(0x1.a01a01a01a01ap-9));
  emit(5, 5, s * T(0x1.a01a01a01a01ap-7));
  emit(5, 6, s * T(0x1.a01a01a01a01ap-8));
  emit(5, 7, s * T(0x1.a01a01a01a01ap-8));
  emit(5, 8, s * T(0x1.a01a01a01a01ap-9));
  emit(5, 9, s * T(0x1.a01a01a01a01ap-8));
  emit(6, 6, s * T(0x1.a01a01a01a01ap-7));
  emit(6, 7, s * T(0x1.a01a01a01a01ap-9));
  emit(6, 8, s * T(0x1.a01a01a01a01ap-8));
  emit(6, 9, s * T(0x1.a01a01a01a01ap-8));
  emit(7, 7, s * T(0x1.a01a01a01a01ap-7));
  emit(7, 8, s * T(0x1.a01a01a01a01ap-8));
  emit(7, 9, s * T(0x1.a01a01a01a01ap-8));
  emit(8, 8, s * T(0x1.a01a01a01a01ap-7));
  emit(8, 9, s * T(0x1.a01a01a01a01ap-8));
  emit(9, 9, s * T(0x1.a01a01a01a01ap-7));
}
// P2 mass, P1 coefficient: cq[m] = c_m * |det J|.
template <typename T, typename Emit>
__device__ __forceinline__ void p2_mass_p1coef(const T* cq, Emit&& emit) {
  emit(0, 0, (fma(cq[2], T(0x1.a01a01a01a01ap-12), cq[0] * T(0x1.3813813813814p-10)) + fma(cq[3], T(0x1.a01a01a01a01ap-12), cq[1] * T(0x1.a01a01a01a01ap-12))));
  emit(0, 1, (cq[2] * T(0x1.a01a01a01a01ap-13) + cq[3] * T(0x1.a01a01a01a01ap-13)));
  emit(0, 2, (cq[1] * T(0x1.a01a01a01a01ap-13) + cq[3] * T(0x1.a01a01a01a01ap-13)));
  emit(0, 3, (cq[1] * T(0x1.a01a01a01a01ap-13) + cq[2] * T(0x1.a01a01a01a01ap-13)));
  emit(0, 4, (fma(cq[2], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-12)) + fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[1] * T(-0x1.a01a01a01a01ap-12))));
  emit(0, 5, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-12)) + fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[1] * T(-0x1.a01a01a01a01ap-11))));
  emit(0, 6, (fma(cq[2], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-12)) + fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-11))));
  emit(0, 7, (fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[1] * T(-0x1.a01a01a01a01ap-12)) + cq[2] * T(-0x1.a01a01a01a01ap-12)));
  emit(0, 8, (fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-12)) + cq[2] * T(-0x1.a01a01a01a01ap-11)));
  emit(0, 9, (fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-11)) + cq[2] * T(-0x1.a01a01a01a01ap-12)));
  emit(1, 1, (fma(cq[2], T(0x1.a01a01a01a01ap-12), cq[0] * T(0x1.a01a01a01a01ap-12)) + fma(cq[3], T(0x1.a01a01a01a01ap-12), cq[1] * T(0x1.3813813813814p-10))));
  emit(1, 2, (cq[0] * T(0x1.a01a01a01a01ap-13) + cq[3] * T(0x1.a01a01a01a01ap-13)));
  emit(1, 3, (cq[0] * T(0x1.a01a01a01a01ap-13) + cq[2] * T(0x1.a01a01a01a01ap-13)));
  emit(1, 4, (fma(cq[2], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-12)) + fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[1] * T(-0x1.a01a01a01a01ap-12))));
  emit(1, 5, (fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-12)) + cq[2] * T(-0x1.a01a01a01a01ap-12)));
  emit(1, 6, (fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-12)) + cq[2] * T(-0x1.a01a01a01a01ap-11)));
  emit(1, 7, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-11)) + fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[1] * T(-0x1.a01a01a01a01ap-12))));
  emit(1, 8, (fma(cq[2], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-11)) + fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-12))));
  emit(1, 9, (fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-11)) + cq[2] * T(-0x1.a01a01a01a01ap-12)));
  emit(2, 2, (fma(cq[2], T(0x1.3813813813814p-10), cq[0] * T(0x1.a01a01a01a01ap-12)) + fma(cq[3], T(0x1.a01a01a01a01ap-12), cq[1] * T(0x1.a01a01a01a01ap-12))));
  emit(2, 3, (cq[0] * T(0x1.a01a01a01a01ap-13) + cq[1] * T(0x1.a01a01a01a01ap-13)));
  emit(2, 4, (fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-12)) + cq[1] * T(-0x1.a01a01a01a01ap-12)));
  emit(2, 5, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-12)) + fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[1] * T(-0x1.a01a01a01a01ap-11))));
  emit(2, 6, (fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-12)) + cq[1] * T(-0x1.a01a01a01a01ap-11)));
  emit(2, 7, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-11)) + fma(cq[3], T(-0x1.a01a01a01a01ap-11), cq[1] * T(-0x1.a01a01a01a01ap-12))));
  emit(2, 8, (fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-11)) + cq[1] * T(-0x1.a01a01a01a01ap-12)));
  emit(2, 9, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-11)) + fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-11))));
  emit(3, 3, (fma(cq[2], T(0x1.a01a01a01a01ap-12), cq[0] * T(0x1.a01a01a01a01ap-12)) + fma(cq[3], T(0x1.3813813813814p-10), cq[1] * T(0x1.a01a01a01a01ap-12))));
  emit(3, 4, (fma(cq[2], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-12)) + cq[1] * T(-0x1.a01a01a01a01ap-12)));
  emit(3, 5, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-12)) + cq[1] * T(-0x1.a01a01a01a01ap-11)));
  emit(3, 6, (fma(cq[2], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-12)) + fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-11))));
  emit(3, 7, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-11)) + cq[1] * T(-0x1.a01a01a01a01ap-12)));
  emit(3, 8, (fma(cq[2], T(-0x1.a01a01a01a01ap-11), cq[0] * T(-0x1.a01a01a01a01ap-11)) + fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-12))));
  emit(3, 9, (fma(cq[2], T(-0x1.a01a01a01a01ap-12), cq[0] * T(-0x1.a01a01a01a01ap-11)) + fma(cq[3], T(-0x1.a01a01a01a01ap-12), cq[1] * T(-0x1.a01a01a01a01ap-11))));
  emit(4, 4, (fma(cq[2], T(0x1.3813813813814p-8), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.3813813813814p-8), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(4, 5, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.a01a01a01a01ap-11)) + fma(cq[3], T(0x1.3813813813814p-9), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(4, 6, (fma(cq[2], T(0x1.3813813813814p-9), cq[0] * T(0x1.a01a01a01a01ap-11)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(4, 7, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.3813813813814p-9), cq[1] * T(0x1.a01a01a01a01ap-11))));
  emit(4, 8, (fma(cq[2], T(0x1.3813813813814p-9), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.a01a01a01a01ap-11))));
  emit(4, 9, (fma(cq[2], T(0x1.a01a01a01a01ap-11), cq[0] * T(0x1.a01a01a01a01ap-11)) + fma(cq[3], T(0x1.a01a01a01a01ap-11), cq[1] * T(0x1.a01a01a01a01ap-11))));
  emit(5, 5, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.3813813813814p-8), cq[1] * T(0x1.3813813813814p-8))));
  emit(5, 6, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.a01a01a01a01ap-11)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.3813813813814p-9))));
  emit(5, 7, (fma(cq[2], T(0x1.a01a01a01a01ap-11), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.3813813813814p-9), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(5, 8, (fma(cq[2], T(0x1.a01a01a01a01ap-11), cq[0] * T(0x1.a01a01a01a01ap-11)) + fma(cq[3], T(0x1.a01a01a01a01ap-11), cq[1] * T(0x1.a01a01a01a01ap-11))));
  emit(5, 9, (fma(cq[2], T(0x1.a01a01a01a01ap-11), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.3813813813814p-9))));
  emit(6, 6, (fma(cq[2], T(0x1.3813813813814p-8), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.3813813813814p-8))));
  emit(6, 7, (fma(cq[2], T(0x1.a01a01a01a01ap-11), cq[0] * T(0x1.a01a01a01a01ap-11)) + fma(cq[3], T(0x1.a01a01a01a01ap-11), cq[1] * T(0x1.a01a01a01a01ap-11))));
  emit(6, 8, (fma(cq[2], T(0x1.3813813813814p-9), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.a01a01a01a01ap-11), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(6, 9, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.a01a01a01a01ap-10)) + fma(cq[3], T(0x1.a01a01a01a01ap-11), cq[1] * T(0x1.3813813813814p-9))));
  emit(7, 7, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.3813813813814p-8)) + fma(cq[3], T(0x1.3813813813814p-8), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(7, 8, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.3813813813814p-9)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.a01a01a01a01ap-11))));
  emit(7, 9, (fma(cq[2], T(0x1.a01a01a01a01ap-11), cq[0] * T(0x1.3813813813814p-9)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(8, 8, (fma(cq[2], T(0x1.3813813813814p-8), cq[0] * T(0x1.3813813813814p-8)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(8, 9, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.3813813813814p-9)) + fma(cq[3], T(0x1.a01a01a01a01ap-11), cq[1] * T(0x1.a01a01a01a01ap-10))));
  emit(9, 9, (fma(cq[2], T(0x1.a01a01a01a01ap-10), cq[0] * T(0x1.3813813813814p-8)) + fma(cq[3], T(0x1.a01a01a01a01ap-10), cq[1] * T(0x1.3813813813814p-8))));
}

#ifdef FE_FACET_TABLES
// cell-local dofs on each facet (P1)
static __constant__ int kFacetDofsP1[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
static __constant__ double kFacetMassP1[4][3][3] = {{{0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}}, {{0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}}, {{0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}}, {{0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}}};
static __constant__ double kFacetLoadP1[4][3] = {{0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}, {0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}, {0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}, {0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}};
static __constant__ double kFacetLoadWP1[4][4][3] = {{{0x0.0p+0, 0x0.0p+0, 0x0.0p+0}, {0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}}, {{0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}}, {{0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}}, {{0x1.5555555555555p-3, 0x1.5555555555555p-4, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-3, 0x1.5555555555555p-4}, {0x1.5555555555555p-4, 0x1.5555555555555p-4, 0x1.5555555555555p-3}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0}}};
// cell-local dofs on each facet (P2)
static __constant__ int kFacetDofsP2[4][6] = {{1, 2, 3, 4, 5, 6}, {0, 2, 3, 4, 7, 8}, {0, 1, 3, 5, 7, 9}, {0, 1, 2, 6, 8, 9}};
static __constant__ double kFacetMassP2[4][6][6] = {{{0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6}, {-0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3}}, {{0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6}, {-0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3}}, {{0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6}, {-0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3}}, {{0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, -0x1.6c16c16c16c17p-8, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0}, {-0x1.6c16c16c16c17p-8, -0x1.6c16c16c16c17p-8, 0x1.1111111111111p-5, 0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6}, {-0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x0.0p+0, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x0.0p+0, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3, 0x1.6c16c16c16c17p-4}, {0x0.0p+0, 0x0.0p+0, -0x1.6c16c16c16c17p-6, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-4, 0x1.6c16c16c16c17p-3}}};
static __constant__ double kFacetLoadP2[4][6] = {{0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x1.5555555555555p-2, 0x1.5555555555555p-2, 0x1.5555555555555p-2}};
static __constant__ double kFacetLoadWP2[4][4][6] = {{{0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0}, {0x1.1111111111111p-5, -0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-4, 0x1.1111111111111p-3, 0x1.1111111111111p-3}, {-0x1.1111111111111p-6, 0x1.1111111111111p-5, -0x1.1111111111111p-6, 0x1.1111111111111p-3, 0x1.1111111111111p-4, 0x1.1111111111111p-3}, {-0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-5, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-4}}, {{0x1.1111111111111p-5, -0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-4, 0x1.1111111111111p-3, 0x1.1111111111111p-3}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0}, {-0x1.1111111111111p-6, 0x1.1111111111111p-5, -0x1.1111111111111p-6, 0x1.1111111111111p-3, 0x1.1111111111111p-4, 0x1.1111111111111p-3}, {-0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-5, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-4}}, {{0x1.1111111111111p-5, -0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-4, 0x1.1111111111111p-3, 0x1.1111111111111p-3}, {-0x1.1111111111111p-6, 0x1.1111111111111p-5, -0x1.1111111111111p-6, 0x1.1111111111111p-3, 0x1.1111111111111p-4, 0x1.1111111111111p-3}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0}, {-0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-5, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-4}}, {{0x1.1111111111111p-5, -0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-4, 0x1.1111111111111p-3, 0x1.1111111111111p-3}, {-0x1.1111111111111p-6, 0x1.1111111111111p-5, -0x1.1111111111111p-6, 0x1.1111111111111p-3, 0x1.1111111111111p-4, 0x1.1111111111111p-3}, {-0x1.1111111111111p-6, -0x1.1111111111111p-6, 0x1.1111111111111p-5, 0x1.1111111111111p-3, 0x1.1111111111111p-3, 0x1.1111111111111p-4}, {0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0, 0x0.0p+0}}};
#endif  // FE_FACET_TABLES

}  // namespace fe

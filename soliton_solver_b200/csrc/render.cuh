// render.cuh -- headless RGBA colormaps of a lattice (no graphics context).
//
// The reference's viewer renders densities and magnetisation fields into a
// GL pixel buffer with Numba kernels (core/colormaps.py:14-267).  These kernels
// write the same bytes into a plain device buffer of ylen x xlen RGBA pixels
// (pixel (y, x) at byte 4 (y xlen + x)), from fields stored y-fastest
// (idx = y + x ylen).  Reading y-fastest and writing x-fastest is a transpose, so
// each CTA stages a 32 x 32 block of packed pixels in shared memory: both the
// field reads and the RGBA stores coalesce.  The per-pixel arithmetic is FP64 with
// every operation explicitly rounded (no contraction into FMAs), in the
// reference's order, so the bytes match the reference's FP64 Python arithmetic;
// atan2 and tanh are CUDA's double-precision functions.
#pragma once

#include <cstdint>

namespace ssb {

enum RenderKind { RK_JET = 0, RK_GRAY = 1, RK_MAGNETIZATION = 2 };

// clip_u8 (colormaps.py:14-40): clamp to [0, 255], truncate toward zero
__device__ __forceinline__ uint32_t clip_u8(double x) {
  if (x < 0.0) return 0u;
  if (x > 255.0) return 255u;
  return (uint32_t)(int)x;
}

__device__ __forceinline__ uint32_t pack_rgba(uint32_t r, uint32_t g, uint32_t b) {
  return r | (g << 8) | (b << 16) | (255u << 24);
}

// (val - vmin) / (vmax - vmin + 1e-30) clamped to [0, 1] (colormaps.py:129-135)
__device__ __forceinline__ double density_hue(double val, double vmin, double vmax) {
  double hue = __ddiv_rn(__dsub_rn(val, vmin), __dadd_rn(__dsub_rn(vmax, vmin), 1e-30));
  if (hue < 0.0) hue = 0.0;
  if (hue > 1.0) hue = 1.0;
  return hue;
}

// jet colormap, colormaps.py:136-161
__device__ __forceinline__ uint32_t jet_pixel(double val, double vmin, double vmax) {
  const double hue = density_hue(val, vmin, vmax);
  const double h4 = __dmul_rn(4.0, hue), m4 = __dmul_rn(-4.0, hue);
  double r, g, b;
  if (hue <= 0.125) {
    r = 0.0; g = 0.0; b = __dmul_rn(__dadd_rn(h4, 0.5), 255.0);
  } else if (hue <= 0.375) {
    r = 0.0; g = __dmul_rn(__dsub_rn(h4, 0.5), 255.0); b = 255.0;
  } else if (hue <= 0.625) {
    r = __dmul_rn(__dsub_rn(h4, 1.5), 255.0); g = 255.0; b = __dmul_rn(__dadd_rn(m4, 2.5), 255.0);
  } else if (hue <= 0.875) {
    r = 255.0; g = __dmul_rn(__dadd_rn(m4, 3.5), 255.0); b = 0.0;
  } else {
    r = __dmul_rn(__dadd_rn(m4, 4.5), 255.0); g = 0.0; b = 0.0;
  }
  return pack_rgba(clip_u8(r), clip_u8(g), clip_u8(b));
}

// gray colormap, colormaps.py:195-205
__device__ __forceinline__ uint32_t gray_pixel(double val, double vmin, double vmax) {
  const uint32_t c = clip_u8(__dmul_rn(density_hue(val, vmin, vmax), 255.0));
  return pack_rgba(c, c, c);
}

// HSV -> RGB, colormaps.py:68-92
__device__ __forceinline__ void hsv_to_rgb(double h, double s, double v, double& R, double& G, double& B) {
  if (h >= 360.0) h = 0.0;
  h = __ddiv_rn(h, 60.0);
  const int i = (int)h;
  const double ff = __dsub_rn(h, (double)i);
  const double p = __dmul_rn(v, __dsub_rn(1.0, s));
  const double r = __dmul_rn(v, __dsub_rn(1.0, __dmul_rn(s, ff)));
  const double t = __dmul_rn(v, __dsub_rn(1.0, __dmul_rn(s, __dsub_rn(1.0, ff))));
  switch (i) {
    case 0: R = v; G = t; B = p; break;
    case 1: R = r; G = v; B = p; break;
    case 2: R = p; G = v; B = t; break;
    case 3: R = p; G = r; B = v; break;
    case 4: R = t; G = p; B = v; break;
    default: R = v; G = p; B = r; break;
  }
}

// magnetisation colormap, colormaps.py:252-267
__device__ __forceinline__ uint32_t magnetization_pixel(double m1, double m2, double m3) {
  const double inv2pi = __ddiv_rn(1.0, __dmul_rn(2.0, 3.141592653589793));
  const double hue = __dmul_rn(__dadd_rn(0.5, __dmul_rn(inv2pi, atan2(m1, m2))), 360.0);
  const double sat = __dsub_rn(0.5, __dmul_rn(0.5, tanh(__dmul_rn(3.0, __dsub_rn(m3, 0.5)))));
  const double val = __dadd_rn(1.0, m3);
  double R, G, B;
  hsv_to_rgb(hue, sat, val, R, G, B);
  return pack_rgba(clip_u8(__dmul_rn(R, 255.0)), clip_u8(__dmul_rn(G, 255.0)), clip_u8(__dmul_rn(B, 255.0)));
}

// One CTA = 32 (y) x 32 (x) pixels, 32 x 8 threads.  src: density (JET, GRAY) or the
// m1, m2, m3 planes (MAGNETIZATION, plane stride X * Y), element type T.
template <typename T, int KIND>
__global__ void __launch_bounds__(256) render_kernel(const T* __restrict__ src, int X, int Y, double vmin,
                                                     double vmax, uint32_t* __restrict__ rgba) {
  __shared__ uint32_t tile[32][33];  // [x][y], padded against bank conflicts on the transposed read
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * 32;
  const long long plane = (long long)X * Y;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int lx = threadIdx.y + 8 * k, x = x0 + lx, y = y0 + threadIdx.x;
    if (x < X && y < Y) {
      const long long i = (long long)x * Y + y;
      uint32_t px;
      if constexpr (KIND == RK_JET) {
        px = jet_pixel((double)src[i], vmin, vmax);
      } else if constexpr (KIND == RK_GRAY) {
        px = gray_pixel((double)src[i], vmin, vmax);
      } else {
        px = magnetization_pixel((double)src[i], (double)src[i + plane], (double)src[i + 2 * plane]);
      }
      tile[lx][threadIdx.x] = px;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int ly = threadIdx.y + 8 * k, x = x0 + threadIdx.x, y = y0 + ly;
    if (x < X && y < Y) rgba[(long long)y * X + x] = tile[threadIdx.x][ly];
  }
}

}  // namespace ssb

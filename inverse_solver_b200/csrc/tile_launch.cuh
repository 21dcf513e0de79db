// Per-radix-class launchers of the tile kernels (instantiated in
// cbs_tiles.cu, one translation unit per kernel kind and class).
#pragma once

#include "cbs_kernels.cuh"
#include "fft_tile.cuh"

namespace odt {

ODT_HD size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Per-line constants of an x-line (fixed y, z, illumination b).
struct LineInfo {
  long long g;      // offset of x = 0 in T / Field_n / Field (batched)
  long long einc;   // Einc / Fout offset of x = 0 (valid when roi != 0)
  int v;            // offset of x = 0 in V
  int valid;        // line exists (partial last tile)
  int roi;          // y and z inside the ROI (einc then addresses Einc / Fout)
  float my, mz;     // attenuation mask factors of y and z
  float2 ry, rz;    // phase-ramp factors of y and z
};

inline size_t born_x_smem(int n, int W) {
  return align16(sizeof(float2) * (size_t)n) + align16(sizeof(LineInfo) * (size_t)W) +
         2 * sizeof(float2) * (size_t)W * smem_line_ld(n);
}

inline size_t col_smem(int n, int W, size_t extra) {
  return align16(sizeof(float2) * (size_t)n) + align16(extra) +
         2 * sizeof(float2) * (size_t)n * (W + 1);
}

template <int C>
cudaError_t born_x_launch(const BornArgs& a, int mode, int jj, const DevFft& f, unsigned blocks,
                          size_t sm, cudaStream_t s);
template <int C>
cudaError_t born_z_launch(const BornArgs& a, int jj, const DevFft& f, unsigned blocks, size_t sm,
                          cudaStream_t s);
template <int C>
cudaError_t lines_launch(const float2* in, float2* out, long long nlines, int is, int os, float sc,
                         bool inv, const DevFft& f, unsigned blocks, size_t sm, cudaStream_t s);
template <int C>
cudaError_t cols_launch(const float2* in, float2* out, long long n0, long long n2, int is, int os,
                        float sc, bool inv, bool shift, const DevFft& f, unsigned blocks, size_t sm,
                        cudaStream_t s);

}  // namespace odt

// Born loop for padded grids with a length that the radix tiles do not cover
// (a prime factor above 31: the reference pads the RI grid by the boundary
// width without rounding, FORWARD_SOLVER_CONVERGENT_BORN.m:129, so any
// length occurs).  The transforms along such an axis run through Bluestein's
// algorithm (fft_any.cu), so the Born iteration is unfused here: per
// iteration jj
//   born_point  the inverse transform's result in T -> update of iteration
//               jj-1 (:616-642) and the source of jj times the phase ramp
//               (:588-605) back into T (the generic x-pass's pointwise work,
//               BornXOp, one element per thread);
//   3D FFT      forward along x, y, z (tile kernels or Bluestein per axis);
//   born_green  G(k -/+ dk/4) / N (:606-615, the generic z-pass's GreenOp);
//   3D FFT      inverse along z, y, x (unnormalised: 1/N is in born_green).
#include <cuda_runtime.h>

#include "cbs_kernels.cuh"
#include "tile_bodies.cuh"

namespace odt {
namespace {

constexpr int kThreads = 256;

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) born_point_kernel(const BornArgs a, const int jj) {
  const long long total = (long long)a.nvox * a.nbatch;
  const long long est = (long long)a.rx * a.ry * a.rz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long line = i / a.px;   // y + py (z + pz b)
    const int x = (int)(i - line * a.px);
    const int yy = (int)(line % a.py);
    const long long t = line / a.py;
    const int z = (int)(t % a.pz);
    const int b = (int)(t / a.pz);
    LineInfo L;
    L.valid = 1;
    L.g = line * a.px;
    L.v = (yy + a.py * z) * a.px;
    L.roi = (unsigned)(yy - a.ry0) < (unsigned)a.ry && (unsigned)(z - a.rz0) < (unsigned)a.rz;
    L.einc = (long long)b * est + (long long)(yy - a.ry0) * a.rx + (long long)(z - a.rz0) * a.rx * a.ry - a.rx0;
    L.my = a.mask[1][yy];
    L.mz = a.mask[2][z];
    L.ry = a.ramp[1][yy];
    L.rz = a.ramp[2][z];
    const BornXOp<MODE> op{&a, &L, jj};
    float2 v = MODE == kBornFirst ? make_float2(0.f, 0.f) : a.T[i];
    op.template apply<1>(0, x, 1, &v);
    if (MODE != kBornLast) a.T[i] = v;
  }
}

__global__ void __launch_bounds__(kThreads) born_green_kernel(const BornArgs a, const int jj) {
  const long long total = (long long)a.nvox * a.nbatch;
  const bool flip = a.acyclic && (jj & 1);
  const long long pxy = (long long)a.px * a.py;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long vox = i % a.nvox;
    const int kz = (int)(vox / pxy);
    const long long r = vox - kz * pxy;
    const int ky = (int)(r / a.px), kx = (int)(r - (long long)ky * a.px);
    const int ix = flip ? wrap_neg(kx, a.px) : kx;
    const int iy = flip ? wrap_neg(ky, a.py) : ky;
    const int iz = flip ? wrap_neg(kz, a.pz) : kz;
    float q = a.kq2[0][ix] + a.kq2[1][iy];
    q = q + a.kq2[2][iz];
    q = a.g_scale * q - a.g_off;
    const float rden = frcp(q * q + a.eps * a.eps);
    const float2 G = make_float2(q * rden, a.eps * rden);  // 1 / (q - i eps)
    a.T[i] = cscale(cmul(G, a.T[i]), a.inv_n);
  }
}

}  // namespace

cudaError_t launch_born_point(const BornArgs& a, int mode, int jj, cudaStream_t s) {
  if (a.perm_xy || a.storage) return cudaErrorInvalidValue;   // natural-order complex64 grids only
  const int grid = grid_for((long long)a.nvox * a.nbatch);
  switch (mode) {
    case kBornFirst: born_point_kernel<kBornFirst><<<grid, kThreads, 0, s>>>(a, jj); break;
    case kBornMid: born_point_kernel<kBornMid><<<grid, kThreads, 0, s>>>(a, jj); break;
    case kBornLast: born_point_kernel<kBornLast><<<grid, kThreads, 0, s>>>(a, jj); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_born_green(const BornArgs& a, int jj, cudaStream_t s) {
  if (a.perm_xy || a.storage) return cudaErrorInvalidValue;
  born_green_kernel<<<grid_for((long long)a.nvox * a.nbatch), kThreads, 0, s>>>(a, jj);
  return cudaGetLastError();
}

}  // namespace odt

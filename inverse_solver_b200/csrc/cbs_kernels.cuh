// Kernel launchers of the CBS solver (implemented in cbs_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace odt {

// A transform length ready for launch: plan + device twiddle table + tile
// shape (pencils per CTA, threads per CTA).
struct DevFft {
  FftPlan plan;
  const float2* tw;  // n entries, device
  int W;             // pencils per tile (a power of two for column kernels)
  int lgW;           // log2(W) for column kernels
  int nthr;          // threads per CTA (a multiple of W for column kernels)
};

// tile-kernel kinds (shared-memory layouts differ)
enum FftKind { kKindLines = 0, kKindCols = 1, kKindBornX = 2, kKindBornZ = 3 };

// Everything the Born-loop kernels read.
struct BornArgs {
  int px, py, pz;          // padded grid
  int rx0, ry0, rz0;       // ROI start (0-based)
  int rx, ry, rz;          // ROI extents
  long long nvox;          // px*py*pz
  int nbatch;              // illuminations in flight
  const float* mask[3];
  const float2* ramp[3];
  const float* kq2[3];
  float eps, c_im, g_scale, g_off, inv_n;
  int acyclic;
  float2* T;               // spectral work array  [nvox, nbatch]
  float2* Fn;              // Field_n             [nvox, nbatch]
  float2* F;               // Field (running sum)  [nvox, nbatch]
  const float2* V;         // potential            [nvox]
  const float2* Einc;      // incident field       [rx*ry*rz, nbatch]
  float2* Fout;            // Field(ROI)+incident  [rx*ry*rz, nbatch]
  long long wait_limit;    // clock cycles a pipelined kernel's steady mbarrier wait may take
  // T's x-y spectrum is in the fused xy-pass's order (launch_born_xy): along
  // an axis of length 8 R, spectral index k1 + 8 k2 (k1 < 8, k2 < R) sits at
  // position R k1 + k2
  int perm_xy;
  // reduced-precision storage (storage = 1): T and Field_n as 16-bit block
  // floating point (b16.cuh) -- int16 (re, im) mantissas in T16 / Fn16 with
  // the layouts of T / Field_n, one exponent byte per 8 values in Te / Fe;
  // Field stays complex64 in F
  int storage;
  short2* T16;
  signed char* Te;
  short2* Fn16;
  signed char* Fe;
};

enum BornXMode { kBornFirst = 0, kBornMid = 1, kBornLast = 2 };

// ---- dyadic (vector) branch: tables of polarisation_utility
// (FORWARD_SOLVER.m:131-180) on the [F_x, F_y] spectrum, device pointers
struct PolTables {
  const float* radial;  // [nF, 2]
  const float* perp;    // [nF, 2]
  const float* tan3;    // [nF, 3]
  const float* kmask;   // [nF] 0 / 1
};
// rads per axis in FFT order and the absorptive correction of the dyadic
// Green's function (FORWARD_SOLVER_CONVERGENT_BORN.m:316-322)
struct DyadArgs {
  const float* rad[3];
  float2 absorb;
};
// 2 -> 3 components (optionally also into `keep`) / 3 -> 2 polarisations
cudaError_t launch_pol23(const float2* in, float2* out, float2* keep, const PolTables& t, long long nF,
                         long long nb, cudaStream_t s);
cudaError_t launch_pol32(const float2* in, float2* out, const PolTables& t, bool reflection, long long nF,
                         long long nb, cudaStream_t s);
// z-pass with the dyadic Green's function; a.nbatch = 3 * illuminations
cudaError_t launch_born_z_dyadic(const BornArgs& a, const DyadArgs& d, int jj, const DevFft& fz,
                                 int max_smem, cudaStream_t s);
// RI tensor (V9 [nvox, 3, 3]): the x-pass's pointwise work of iteration jj
// (mode First / Mid / Last as launch_born_x) on the inverse x-FFT in a.T, and
// the output stage's emitter into conv [c0, c1, rz, a.nbatch]
cudaError_t launch_born_tensor_point(const BornArgs& a, const float2* V9, int mode, int jj, cudaStream_t s);
cudaError_t launch_born_tensor_emitter(const BornArgs& a, const float2* V9, float2* conv, int c0, int c1,
                                       int o0, int o1, float dV, cudaStream_t s);

// x-pass of iteration jj: inverse x-FFT + update of iteration jj-1 (Mid/Last)
// and source term + forward x-FFT of iteration jj (First/Mid).
cudaError_t launch_born_x(const BornArgs& a, int mode, int jj, const DevFft& fx, cudaStream_t s);
// Pipelined x-pass (persistent CTAs, bulk asynchronous copies) for modes Mid
// (jj >= 2) and Last and x-lengths 8 * {11, 15, 19, 25, 27}; same results as
// launch_born_x.  A wait that times out sets *fault (device int) and ends
// the kernel.
bool born_x_pipe_supported(const BornArgs& a, const DevFft& fx);
cudaError_t launch_born_x_pipe(const BornArgs& a, int mode, int jj, const DevFft& fx, int* fault,
                               cudaStream_t s);
// Pipelined column passes (persistent CTAs, tiled TMA copies) for lengths
// 8 * {11, 15, 19, 25, 27} along y / z: the y-FFT of the Born loop in place on a.T,
// and the z-pass; same results as launch_fft_cols / launch_born_z up to the
// order of the radix passes of the inverse y-FFT.
bool cols_pipe_supported(const BornArgs& a, const DevFft& f, bool zpass);
cudaError_t launch_fft_y_pipe(const BornArgs& a, bool inverse, const DevFft& fy, int* fault,
                              cudaStream_t s);
cudaError_t launch_born_z_pipe(const BornArgs& a, int jj, const DevFft& fz, int* fault,
                               cudaStream_t s);
// Fused xy-pass (born_xy.cu): the whole x-y plane of one z and illumination
// in shared memory -- inverse y- and x-FFT of T, update of iteration jj-1,
// source of iteration jj, forward x- and y-FFT -- for px == py = 8 * {11, 12,
// 15, 19}; replaces launch_born_x and both y-FFTs (modes as launch_born_x;
// the z-pass must run with a.perm_xy = 1).  Same results as the separate passes
// up to the order of the FFT arithmetic.
bool born_xy_supported(const BornArgs& a, int max_smem);
cudaError_t launch_born_xy(const BornArgs& a, int mode, int jj, const DevFft& fx, cudaStream_t s);
// z-pass of iteration jj: forward z-FFT, Green's multiply, inverse z-FFT.
cudaError_t launch_born_z(const BornArgs& a, int jj, const DevFft& fz, cudaStream_t s);
// Unfused Born loop for grids with a length outside the radix tiles
// (born_any.cu): the pointwise work of the x-pass on T in natural order
// (modes as launch_born_x; T holds the inverse transform of iteration jj-1's
// spectrum, and receives the source of iteration jj), and the Green's
// multiply G / N of iteration jj on T's spectrum.
cudaError_t launch_born_point(const BornArgs& a, int mode, int jj, cudaStream_t s);
cudaError_t launch_born_green(const BornArgs& a, int jj, cudaStream_t s);

// Batched FFT along contiguous lines of an [n, nlines] array.  Input element
// i is gathered from (i + in_shift) % n, output element k scattered to
// (k + out_shift) % n (in_shift = out_shift = n/2 gives MATLAB's
// fftshift(fft(ifftshift(x)))).  In-place allowed.
cudaError_t launch_fft_lines(const float2* in, float2* out, long long nlines, int in_shift,
                             int out_shift, float scale, bool inverse, const DevFft& f,
                             cudaStream_t s);
// Batched FFT along the middle axis of an [n0, n, n2] array.
cudaError_t launch_fft_cols(const float2* in, float2* out, long long n0, long long n2,
                            int in_shift, int out_shift, float scale, bool inverse,
                            const DevFft& f, cudaStream_t s);

// ---- elementwise stages of the field input/output paths
// out[i] = in[i] * filt[i % plane] ; also copies the product to `keep` if non-null
cudaError_t launch_mul_plane(const float2* in, float2* out, float2* keep, const float* filt,
                             long long plane, long long total, cudaStream_t s);
// zero-padded copy [n0, n1, nb] -> [m0, m1, nb], source element (x, y) lands
// at (x + o0, y + o1)
cudaError_t launch_pad2d(const float2* in, float2* out, int n0, int n1, int m0, int m1, int o0,
                         int o1, long long nb, cudaStream_t s);
// crop [m0, m1, nb] -> [n0, n1, nb]: out(x, y) = in(x + o0, y + o1)
cudaError_t launch_crop2d(const float2* in, float2* out, int n0, int n1, int m0, int m1, int o0,
                          int o1, long long nb, cudaStream_t s);
// conv[X, Y, z, b] = sk[X, Y, b] * refocus[X, Y, z]
cudaError_t launch_refocus_expand(const float2* sk, const float2* refocus, float2* conv, int c0,
                                  int c1, int rz, long long nb, cudaStream_t s);
// Einc[x, y, z, b] = conv[x + o0, y + o1, z, b]
cudaError_t launch_crop_volume(const float2* conv, float2* einc, int c0, int c1, int rx, int ry,
                               int rz, int o0, int o1, long long nb, cudaStream_t s);
// conv[X, Y, z, b] = (Fout * (V_roi + i eps)) * dV inside the RI footprint, 0 elsewhere
cudaError_t launch_emitter(const BornArgs& a, float2* conv, int c0, int c1, int o0, int o1,
                           float dV, cudaStream_t s);
// tk[X, Y, b] = sum_z conv * Kt ; rk likewise with Kr (either output may be null)
cudaError_t launch_zreduce(const float2* conv, const float2* Kt, const float2* Kr, float2* tk,
                           float2* rk, int c0, int c1, int rz, long long nb, cudaStream_t s);
// Device-resident outer loop (potential_dev.cu): max |RI2potential(RI)| as
// float bits into d_out; the padded potential V (forward or adjoint); the
// FISTA prox input and momentum update.
cudaError_t launch_potential_absmax(const void* ri, int is_complex, long long n, double wavelength, double ri_bg,
                                    unsigned int* d_out, cudaStream_t s);
cudaError_t launch_build_potential(const void* ri, int is_complex, int adjoint, const int sim[3], const int roi0[3],
                                   const int ri_size[3], double wavelength, double ri_bg, float eps, float2* V,
                                   cudaStream_t s);
cudaError_t launch_fista_prox_input(const float2* u, const float2* grad, float step, int complex_out, void* out,
                                    long long n, cudaStream_t s);
cudaError_t launch_fista_update(const void* sv, int s_complex, float coef, float nb, float2* u, float2* x, float2* ri,
                                long long n, cudaStream_t s);
// Fused input / output stages (io_fused.cu): conv plane cx x cy, RI grid
// rx x ry x rz, window offset (ox, oy) of the RI / field grid in the conv
// plane, nbp planes per z.
struct IoGeom {
  int cx, cy;
  int rx, ry, rz;
  int ox, oy;
  long long nbp;
};
// Einc[x, y, z, b] = ifft2c(sk[., ., b] .* refocus[., ., z])[x + ox, y + oy]
// (the expand -> centred inverse 2D FFT -> crop chain); mid holds
// rx * cy * rz * nbp elements
cudaError_t launch_refocus_in(const float2* sk, const float2* refocus, float2* mid, float2* einc,
                              const IoGeom& g, const DevFft& fx, const DevFft& fy, cudaStream_t s);
// tk / rk = the emitter -> centred forward 2D FFT -> z-reduce chain (either
// output may be null); mid (cap elements) holds cx * ry * rz * nbp elements
// and, where it has room, the per-chunk partial sums of the z-reduction
cudaError_t launch_project_out(const BornArgs& a, float2* mid, long long cap, const float2* Kt, const float2* Kr,
                               float2* tk, float2* rk, const IoGeom& g, float dV, const DevFft& fx,
                               const DevFft& fy, cudaStream_t s);
// whether the fused kernels' tiles fit the device (shared memory, prefetch)
bool io_fused_fits(const IoGeom& g, const DevFft& fx, const DevFft& fy, int nacc, int max_smem);
template <int C>
cudaError_t io_in_launch(const float2* sk, const float2* refocus, float2* mid, float2* einc, const IoGeom& g,
                         const DevFft& fx, const DevFft& fy, cudaStream_t s);
template <int C>
cudaError_t io_out_lines_launch(const BornArgs& a, float2* mid, const IoGeom& g, float dV, const DevFft& fx,
                                cudaStream_t s);
template <int C>
cudaError_t io_out_cols_launch(const float2* mid, const float2* Kt, const float2* Kr, float2* tk, float2* rk,
                               float2* part, int zs, const IoGeom& g, const DevFft& fy, cudaStream_t s);
// out[i] = (x[i] + add[i]) * filt[i % plane]   (add may be null)
cudaError_t launch_combine(const float2* x, const float2* add, const float* filt, float2* out,
                           long long plane, long long total, cudaStream_t s);
// count of non-finite values in [n] (for the numeric watchdog); result on device
cudaError_t launch_count_nonfinite(const float2* x, long long n, unsigned int* count,
                                   cudaStream_t s);

// ---- gradient (BACKWARD_SOLVER_MULTI.m:30-54)
// diff = trans - meas ; *err += sum |diff|^2 (double) ; adj_in = conj(diff)
cudaError_t launch_residual(const float2* trans, const float2* meas, float2* adj_in, long long n,
                            double* err, cudaStream_t s);
// acc[x,y,z] += sum_b conj(E[x,y,z,b]) * conj(A[x,y,rz-1-z,b])   (b in order)
cudaError_t launch_grad_accumulate(const float2* E, const float2* A, float2* acc, int rx, int ry,
                                   int rz, int nb, cudaStream_t s);
// grad = -(1i * (acc / n_ill))
cudaError_t launch_grad_finalize(const float2* acc, float2* grad, long long n, float n_ill,
                                 cudaStream_t s);

// Raise `kernel`'s dynamic shared-memory limit (when `bytes` needs more than
// the default 48 KB) to the device's opt-in maximum, once per kernel and
// device; thread-safe (smem_attr.cu)
cudaError_t raise_smem_limit(const void* kernel, size_t bytes);

// shared-memory bytes a tile kernel of `kind` needs for length n and W pencils
size_t fft_smem_bytes(int n, int W, int kind);

}  // namespace odt

// Test-infrastructure driver around the reference's own Goldstein CUDA
// kernels, compiled with nvcc from the sources where they lie (see Makefile):
//   ref_cuda_residue : residue_KERNEL   (get_residue_cuda.cu:34-91)
//   ref_cuda_dipoles : dipoles_KERNEL   (remove_dipoles_cuda.cu:52-175)
//   ref_cuda_raster  : raster_KERNEL    (raster_branches_cuda.cu:68-191)
//   ref_cuda_unwrap  : unwrapp_KERNEL   (unwrapp_phase_goldstein_cuda.cu:63-190)
// Each takes device pointers and the phase-map sizes [n1, n2, n3] and passes
// the sizes the reference's MEX gateway would pass:
//   residue : the residue map's size [n1-1, n2-1, n3] (get_residue_mex.cpp)
//   dipoles : the phase map's size [n1, n2, n3]; the step-2 output aliases
//             step 1, as in remove_dipoles_mex.cpp:115-125
//   raster  : step 1's size [n1, n2, n3] (raster_branches_mex.cpp:123-141)
//   unwrap  : the phase map's size (unwrapp_phase_goldstein_mex.cpp:144)
// and waits for the kernels; the return value is the CUDA error code.
#include <array>
#include <cstdint>

#include <cuda_runtime.h>

int residue_KERNEL(float const* const pPhase, float* const pOutArray, int const* const dims_output);
int dipoles_KERNEL(float* const pResidue, int32_t* const pPositive, float* const pOutArray, float* const pOut2Array,
                   int const* const dims_output, int const dims_Positive);
int raster_KERNEL(int32_t const* const pBranches, int32_t* const pStep1, int32_t* const pStep2, const int size_Branches,
                  const std::array<int, 3> size_Step1);
int unwrapp_KERNEL(float* const pPhase, int32_t const* const pStep1, int32_t const* const pStep2,
                   std::array<int, 3> size_Phase);

static int finish() {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return (int)e;
}

extern "C" int ref_cuda_residue(const float* phase, float* residue, int n1, int n2, int n3) {
  const int dims[3] = {n1 - 1, n2 - 1, n3};
  residue_KERNEL(phase, residue, dims);
  return finish();
}

// positives: 1-based column-major indices of the residues > 0 (MATLAB find)
extern "C" int ref_cuda_dipoles(float* residue, int32_t* positives, int n_positive, float* step1, int n1, int n2,
                                int n3) {
  const int dims[3] = {n1, n2, n3};
  dipoles_KERNEL(residue, positives, step1, step1, dims, n_positive);
  return finish();
}

// branches: [6, n_branches] int32 (x1, y1, x2, y2, z, jump), device
extern "C" int ref_cuda_raster(const int32_t* branches, int n_branches, int32_t* step1, int32_t* step2, int n1, int n2,
                               int n3) {
  if (n_branches > 0) raster_KERNEL(branches, step1, step2, n_branches, std::array<int, 3>{n1, n2, n3});
  return finish();
}

extern "C" int ref_cuda_unwrap(float* phase, const int32_t* step1, const int32_t* step2, int n1, int n2, int n3) {
  unwrapp_KERNEL(phase, step1, step2, std::array<int, 3>{n1, n2, n3});
  return finish();
}

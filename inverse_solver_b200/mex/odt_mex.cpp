// MATLAB MEX gateway over libodt (include/odt.h), call-compatible with the
// reference's CudaBorn MEX (Codes/CUDA_CODE/main.cpp:27-213):
//
//   id = odt_mex(uint32(0), uint32(0), geom, refocus, kernel_trans, kernel_ref, pupil_in, pupil_out)
//   odt_mex(uint32(1), id, pot, single(V))
//   [trans, ref, field3d] = odt_mex(uint32(4), id, single complex input [F_x, F_y, npol, n], RI_size)
//   field3d = odt_mex(uint32(2), id, single complex source3D [RI_x, RI_y, RI_z(, 3)(, n)])  (legacy)
//   odt_mex(uint32(3), id)
// and, beyond CudaBorn's actions (vector simulations, the inverse solver):
//   odt_mex(uint32(5), id, Radial_2D, Perp_2D, ewald_TanVec, uint8(K_mask))   polarisation basis
//   odt_mex(uint32(6), id, pot, single(V_adjoint))                             adjoint potential
//   [grad, err] = odt_mex(uint32(7), id, input_field, output_field, RI_size)   fused gradient
//   odt_mex(uint32(8), id, uint32(storage))   T / Field_n storage (0 complex64, 1 16-bit block float)
//
// geom: struct with simulation_size, RI_size, field_size, conv_size, used_gpu
// (the CudaBorn names), optional max_batch and pol (3: dyadic Green's
// function).  pot: struct with eps_imag, green_scale, green_offset, dV, ROI,
// Bornmax, acyclic, mask1/2/3, ramp1/2/3, kq2_1/2/3, and for dyadic handles
// rad1/2/3 and absorb (green_absorbtion_correction, complex).  V of
// 9 * prod(simulation_size) elements ([sim, 3, 3]) is an RI tensor's
// potential (odt_set_tensor_potential).  Complex arrays use the interleaved
// layout of -R2018a.
//
// Build (needs MATLAB's mex.h, not present in this environment):
//   mex -R2018a odt_mex.cpp -I../../include -L.. -lodt
#include <mex.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "odt.h"

namespace {

double scalar(const mxArray* s, const char* name) {
  const mxArray* f = mxGetField(s, 0, name);
  if (!f) mexErrMsgIdAndTxt("odt:param", "missing field %s", name);
  return mxGetScalar(f);
}

void ints(const mxArray* s, const char* name, int32_t* out, int n) {
  const mxArray* f = mxGetField(s, 0, name);
  if (!f || (int)mxGetNumberOfElements(f) < n) mexErrMsgIdAndTxt("odt:param", "field %s needs %d values", name, n);
  const double* d = mxGetPr(f);
  for (int i = 0; i < n; ++i) out[i] = (int32_t)d[i];
}

const void* array_field(const mxArray* s, const char* name, mxClassID cls, bool cplx) {
  const mxArray* f = mxGetField(s, 0, name);
  if (!f || mxGetClassID(f) != cls || (mxIsComplex(f) != cplx))
    mexErrMsgIdAndTxt("odt:param", "field %s must be %s%s", name, cplx ? "complex " : "",
                      cls == mxSINGLE_CLASS ? "single" : "double");
  return cplx ? (const void*)mxGetComplexSingles(f) : (const void*)mxGetSingles(f);
}

void check(odt_status st) {
  if (st != ODT_OK) mexErrMsgIdAndTxt("odt:call", "%s", odt_last_error());
}

uint32_t u32(const mxArray* a) {
  if (mxGetClassID(a) != mxUINT32_CLASS || mxGetNumberOfElements(a) != 1)
    mexErrMsgIdAndTxt("odt:arg", "action and id must be uint32 scalars");
  return *static_cast<const uint32_t*>(mxGetData(a));
}

const odt_cfloat* csingle(const mxArray* a, const char* what) {
  if (mxGetClassID(a) != mxSINGLE_CLASS || !mxIsComplex(a))
    mexErrMsgIdAndTxt("odt:arg", "%s must be complex single", what);
  return reinterpret_cast<const odt_cfloat*>(mxGetComplexSingles(a));
}

}  // namespace

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs < 2) mexErrMsgIdAndTxt("odt:arg", "need the action and the id");
  const uint32_t action = u32(prhs[0]);
  const uint32_t id = u32(prhs[1]);
  switch (action) {
    case 0: {
      if (nrhs < 8) mexErrMsgIdAndTxt("odt:arg", "create needs geom and five arrays");
      odt_geometry g{};
      ints(prhs[2], "simulation_size", g.sim_size, 3);
      ints(prhs[2], "RI_size", g.ri_size, 3);
      ints(prhs[2], "field_size", g.field_size, 2);
      ints(prhs[2], "conv_size", g.conv_size, 2);
      g.device = (int32_t)scalar(prhs[2], "used_gpu");
      g.max_batch = mxGetField(prhs[2], 0, "max_batch") ? (int32_t)scalar(prhs[2], "max_batch") : 0;
      g.pol = mxGetField(prhs[2], 0, "pol") ? (int32_t)scalar(prhs[2], "pol") : 1;
      odt_handle h = 0;
      check(odt_create(&g, csingle(prhs[3], "refocus"), csingle(prhs[4], "kernel_trans"),
                       csingle(prhs[5], "kernel_ref"), mxGetSingles(prhs[6]), mxGetSingles(prhs[7]), &h));
      plhs[0] = mxCreateNumericMatrix(1, 1, mxUINT32_CLASS, mxREAL);
      *static_cast<uint32_t*>(mxGetData(plhs[0])) = h;
      break;
    }
    case 1:
    case 6: {
      if (nrhs < 4) mexErrMsgIdAndTxt("odt:arg", "set_potential needs pot and V");
      odt_potential_params pp{};
      pp.eps_imag = (float)scalar(prhs[2], "eps_imag");
      pp.green_scale = (float)scalar(prhs[2], "green_scale");
      pp.green_offset = (float)scalar(prhs[2], "green_offset");
      pp.dV = (float)scalar(prhs[2], "dV");
      ints(prhs[2], "ROI", pp.roi, 6);
      pp.bornmax = (int32_t)scalar(prhs[2], "Bornmax");
      pp.acyclic = (int32_t)scalar(prhs[2], "acyclic");
      const char* mk[3] = {"mask1", "mask2", "mask3"};
      const char* rk[3] = {"ramp1", "ramp2", "ramp3"};
      const char* kk[3] = {"kq2_1", "kq2_2", "kq2_3"};
      for (int i = 0; i < 3; ++i) {
        pp.mask[i] = static_cast<const float*>(array_field(prhs[2], mk[i], mxSINGLE_CLASS, false));
        pp.ramp[i] = static_cast<const odt_cfloat*>(array_field(prhs[2], rk[i], mxSINGLE_CLASS, true));
        pp.kq2[i] = static_cast<const float*>(array_field(prhs[2], kk[i], mxSINGLE_CLASS, false));
      }
      if (mxGetField(prhs[2], 0, "rad1")) {  // dyadic handle
        const char* rd[3] = {"rad1", "rad2", "rad3"};
        for (int i = 0; i < 3; ++i)
          pp.rad[i] = static_cast<const float*>(array_field(prhs[2], rd[i], mxSINGLE_CLASS, false));
        const mxArray* ab = mxGetField(prhs[2], 0, "absorb");
        if (!ab) mexErrMsgIdAndTxt("odt:param", "missing field absorb");
        pp.absorb.re = (float)mxGetScalar(ab);
        pp.absorb.im = mxIsComplex(ab) ? (float)mxGetComplexDoubles(ab)[0].imag : 0.f;
      }
      int32_t sim[3];
      ints(prhs[2], "simulation_size", sim, 3);
      const size_t nsim = (size_t)sim[0] * sim[1] * sim[2];
      const odt_cfloat* V = csingle(prhs[3], "V");
      if (action == 6)
        check(odt_set_adjoint_potential(id, &pp, V));
      else if (mxGetNumberOfElements(prhs[3]) == 9 * nsim)
        check(odt_set_tensor_potential(id, &pp, V));
      else
        check(odt_set_potential(id, &pp, V));
      break;
    }
    case 5: {
      if (nrhs < 6) mexErrMsgIdAndTxt("odt:arg", "polarisation needs Radial_2D, Perp_2D, ewald_TanVec, K_mask");
      for (int i = 2; i < 5; ++i)
        if (mxGetClassID(prhs[i]) != mxSINGLE_CLASS || mxIsComplex(prhs[i]))
          mexErrMsgIdAndTxt("odt:arg", "the basis vectors must be real single");
      if (mxGetClassID(prhs[5]) != mxUINT8_CLASS) mexErrMsgIdAndTxt("odt:arg", "K_mask must be uint8");
      check(odt_set_polarisation(id, mxGetSingles(prhs[2]), mxGetSingles(prhs[3]), mxGetSingles(prhs[4]),
                                 static_cast<const uint8_t*>(mxGetData(prhs[5]))));
      break;
    }
    case 7: {
      if (nrhs < 5) mexErrMsgIdAndTxt("odt:arg", "gradient needs input_field, output_field and RI_size");
      const mwSize* d = mxGetDimensions(prhs[2]);
      const mwSize nd = mxGetNumberOfDimensions(prhs[2]);
      if (mxGetNumberOfElements(prhs[2]) != mxGetNumberOfElements(prhs[3]))
        mexErrMsgIdAndTxt("odt:arg", "input and output fields must have the same size");
      const double* r = mxGetPr(prhs[4]);
      mwSize dg[3] = {(mwSize)r[0], (mwSize)r[1], (mwSize)r[2]};
      plhs[0] = mxCreateNumericArray(3, dg, mxSINGLE_CLASS, mxCOMPLEX);
      double err = 0;
      odt_gradient_args a{};
      a.fields_in = csingle(prhs[2], "input field");
      a.fields_meas = csingle(prhs[3], "output field");
      a.n_ill = nd >= 4 ? (int32_t)d[3] : 1;
      a.grad = reinterpret_cast<odt_cfloat*>(mxGetComplexSingles(plhs[0]));
      a.err = &err;
      a.memory = ODT_MEM_HOST;
      check(odt_gradient(id, &a));
      if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(err);
      break;
    }
    case 2: {
      // source [RI_x, RI_y, RI_z, (3,) n]; the optional 4th argument is the
      // number of field components per illumination (3 on dyadic handles,
      // whose [.., 3] trailing size MATLAB cannot tell from n = 3)
      if (nrhs < 3) mexErrMsgIdAndTxt("odt:arg", "action 2 needs the 3D source");
      const mwSize nd = mxGetNumberOfDimensions(prhs[2]);
      const mwSize* d = mxGetDimensions(prhs[2]);
      const mwSize comps = nrhs > 3 ? (mwSize)u32(prhs[3]) : 1;
      if (comps != 1 && comps != 3) mexErrMsgIdAndTxt("odt:arg", "components must be 1 or 3");
      mwSize trailing = 1;   // elements per RI-grid voxel
      for (mwSize i = 3; i < nd; ++i) trailing *= d[i];
      if (trailing % comps != 0) mexErrMsgIdAndTxt("odt:arg", "source size does not match the components");
      plhs[0] = mxCreateNumericArray(nd, d, mxSINGLE_CLASS, mxCOMPLEX);
      odt_source_args a{};
      a.source = csingle(prhs[2], "source3D");
      a.field3d = reinterpret_cast<odt_cfloat*>(mxGetComplexSingles(plhs[0]));
      a.n = (int32_t)(trailing / comps);   // the library checks the grid against its handle
      a.memory = ODT_MEM_HOST;
      check(odt_solve_source(id, &a));
      break;
    }
    case 8: {
      if (nrhs < 3) mexErrMsgIdAndTxt("odt:arg", "storage needs ODT_STORAGE_COMPLEX64 (0) or ODT_STORAGE_B16 (1)");
      check(odt_set_field_storage(id, (int32_t)u32(prhs[2])));
      break;
    }
    case 3:
      check(odt_destroy(id));
      break;
    case 4: {
      if (nrhs < 3) mexErrMsgIdAndTxt("odt:arg", "solve needs the input field");
      const mwSize* d = mxGetDimensions(prhs[2]);
      const mwSize nd = mxGetNumberOfDimensions(prhs[2]);
      const int n_ill = nd >= 4 ? (int)d[3] : 1;
      const mwSize npol = nd >= 3 ? d[2] : 1;  // 2 on dyadic handles
      int32_t ri[3] = {0, 0, 0};
      // output sizes follow the input field (field_size == RI_size(1:2))
      mwSize dt[4] = {d[0], d[1], npol, (mwSize)n_ill};
      plhs[0] = mxCreateNumericArray(4, dt, mxSINGLE_CLASS, mxCOMPLEX);
      if (nlhs > 1) plhs[1] = mxCreateNumericArray(4, dt, mxSINGLE_CLASS, mxCOMPLEX);
      odt_solve_args a{};
      a.fields_in = csingle(prhs[2], "input field");
      a.n_ill = n_ill;
      a.trans = reinterpret_cast<odt_cfloat*>(mxGetComplexSingles(plhs[0]));
      a.ref = nlhs > 1 ? reinterpret_cast<odt_cfloat*>(mxGetComplexSingles(plhs[1])) : nullptr;
      if (nlhs > 2) {
        if (nrhs < 4) mexErrMsgIdAndTxt("odt:arg", "pass RI_size as 4th argument to get field3d");
        const double* r = mxGetPr(prhs[3]);
        for (int i = 0; i < 3; ++i) ri[i] = (int32_t)r[i];
        mwSize d3[5] = {(mwSize)ri[0], (mwSize)ri[1], (mwSize)ri[2], npol == 2 ? (mwSize)3 : (mwSize)1,
                        (mwSize)n_ill};
        plhs[2] = mxCreateNumericArray(5, d3, mxSINGLE_CLASS, mxCOMPLEX);
        a.field3d = reinterpret_cast<odt_cfloat*>(mxGetComplexSingles(plhs[2]));
      }
      a.memory = ODT_MEM_HOST;
      check(odt_solve(id, &a));
      break;
    }
    case 20: {
      // Goldstein unwrapping of a single [N1, N2(, n)] host array: the whole
      // of unwrapp2_gpu.m (the id argument is ignored).
      if (nrhs < 3 || mxGetClassID(prhs[2]) != mxSINGLE_CLASS || mxIsComplex(prhs[2]))
        mexErrMsgIdAndTxt("odt:arg", "unwrap needs a real single phase array");
      const mwSize* d = mxGetDimensions(prhs[2]);
      const mwSize nd = mxGetNumberOfDimensions(prhs[2]);
      if (nd > 3) mexErrMsgIdAndTxt("odt:arg", "phase must be 2D or 3D");
      plhs[0] = mxCreateNumericArray(nd, d, mxSINGLE_CLASS, mxREAL);
      odt_unwrap_args a{};
      a.size[0] = (int32_t)d[0];
      a.size[1] = (int32_t)d[1];
      a.size[2] = nd == 3 ? (int32_t)d[2] : 1;
      a.phase_in = mxGetSingles(prhs[2]);
      a.phase_out = mxGetSingles(plhs[0]);
      a.memory = ODT_MEM_HOST;
      check(odt_unwrap_goldstein(&a));
      break;
    }
    default:
      mexErrMsgIdAndTxt("odt:arg", "unknown action %u", action);
  }
}

// odt_born_series_noalloc: the Born-series loop of odt_solve for one
// illumination, with its scratch memory in a fixed device array instead of
// cudaMalloc'd buffers (see include/odt.h for who needs this and its limits).
//
// Scratch layout (complex64 elements of g_noalloc_scratch):
//   [0, 3*nvox)                       T | Field_n | Field of the Born loop
//   [3*nvox, 3*nvox + px + py + pz)   FFT twiddle tables of the three axes
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "fft_plan.h"
#include "tma.cuh"

namespace odt {
const char* set_last_error(const std::string& msg);  // odt_api.cu
}

namespace {

constexpr size_t kNoallocBytes = 64ull << 20;  // 64 MiB per device
constexpr size_t kNoallocElems = kNoallocBytes / sizeof(float2);

// Held by every device that loads the library, for the life of the process.
// Host code must not use this name as a device address: its address on the
// current device comes from cudaGetSymbolAddress (noalloc_scratch below).
static __device__ __align__(256) float2 g_noalloc_scratch[kNoallocElems];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float2* g_noalloc_ptr[kMaxDevices] = {nullptr};
// padded grid whose twiddle tables the scratch array holds on each device
// (they sit right after T | Field_n | Field, so a call on another grid size
// overwrites or moves them; a call on the same size finds them in place)
int g_noalloc_tw[kMaxDevices][3] = {};

// Device address of the scratch array on the current device; looked up once
// per device (the first call on a device does this).  The address is not
// looked up again, so the entry point must not be called on a device after
// cudaDeviceReset has run on it.
cudaError_t noalloc_scratch(float2** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = static_cast<float2*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

odt_status fail(odt_status st, const std::string& msg) {
  odt::set_last_error(msg);
  return st;
}

}  // namespace

extern "C" odt_status odt_born_series_noalloc(const odt_noalloc_born_args* a) {
  using namespace odt;
  if (!a) return fail(ODT_ERR_INVALID_ARGUMENT, "odt_born_series_noalloc: NULL args");
  for (int i = 0; i < 3; ++i) {
    if (a->sim_size[i] < 1) return fail(ODT_ERR_INVALID_ARGUMENT, "odt_born_series_noalloc: sim_size < 1");
    const int lo = a->roi[2 * i], hi = a->roi[2 * i + 1];
    if (lo < 1 || hi > a->sim_size[i] || hi < lo)
      return fail(ODT_ERR_INVALID_ARGUMENT, "odt_born_series_noalloc: ROI outside sim_size");
    if (!a->mask[i] || !a->kq2[i] || !a->ramp[i])
      return fail(ODT_ERR_INVALID_ARGUMENT,
                  "odt_born_series_noalloc: NULL table (mask, ramp and kq2 are all required; "
                  "pass ones as the ramp when acyclic = 0)");
  }
  if (!a->V || !a->einc || !a->fout)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_born_series_noalloc: NULL V / einc / fout");
  if (a->bornmax < 0 || !(a->eps_imag > 0.f))
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_born_series_noalloc: bornmax < 0 or eps_imag <= 0");
  const long long nvox = (long long)a->sim_size[0] * a->sim_size[1] * a->sim_size[2];
  const long long need = 3 * nvox + a->sim_size[0] + a->sim_size[1] + a->sim_size[2];
  if (need > (long long)kNoallocElems)
    return fail(ODT_ERR_OUT_OF_MEMORY,
                "odt_born_series_noalloc: grid of " + std::to_string(nvox) +
                    " voxels needs " + std::to_string(need * 8) + " bytes of scratch, more than the " +
                    std::to_string(kNoallocBytes) + "-byte fixed array (at most " +
                    std::to_string((kNoallocElems - 3 * 1024) / 3) + " voxels)");
  float2* scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ODT_ERR_CUDA, std::string("odt_born_series_noalloc: cudaGetSymbolAddress: ") +
                                  cudaGetErrorString(e));
  }
  cudaStream_t s = (cudaStream_t)a->stream;
  // plans and twiddles for the three axes (the same shapes odt_solve uses)
  DevFft f[3];
  float2* twbase = scratch + 3 * nvox;
  const int kinds[3] = {kKindBornX, kKindCols, kKindBornZ};
  int dev = 0;
  cudaGetDevice(&dev);
  int max_smem = 0;
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  for (int i = 0; i < 3; ++i) {
    const int n = a->sim_size[i];
    std::string why;
    if (!make_plan(n, &f[i].plan, &why, i == 0 ? kSmallFirst : kLargeFirst))
      return fail(ODT_ERR_UNSUPPORTED, "odt_born_series_noalloc: sim_size(" + std::to_string(i + 1) +
                                           ") = " + std::to_string(n) + ": " + why);
    f[i].lgW = n <= 512 ? 4 : 3;
    f[i].W = 1 << f[i].lgW;
    f[i].nthr = 128;
    if (fft_smem_bytes(n, f[i].W, kinds[i]) > (size_t)max_smem)
      return fail(ODT_ERR_UNSUPPORTED, "odt_born_series_noalloc: length too large for shared memory");
  }
  // The twiddle tables are uploaded (from pageable host memory, so the copies
  // are synchronous with the host) only when this device's scratch does not
  // already hold them: the first call, and the first call after a call on
  // another grid size.
  bool have_tw;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    have_tw = std::memcmp(g_noalloc_tw[dev], a->sim_size, sizeof(g_noalloc_tw[dev])) == 0;
    if (!have_tw) std::memset(g_noalloc_tw[dev], 0, sizeof(g_noalloc_tw[dev]));
  }
  for (int i = 0; i < 3; ++i) {
    if (!have_tw) {
      const std::vector<float2> tw = make_twiddles(a->sim_size[i]);
      e = cudaMemcpyAsync(twbase, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess)
        return fail(ODT_ERR_CUDA, std::string("odt_born_series_noalloc: ") + cudaGetErrorString(e));
    }
    f[i].tw = twbase;
    twbase += a->sim_size[i];
  }
  BornArgs b{};
  b.px = a->sim_size[0];
  b.py = a->sim_size[1];
  b.pz = a->sim_size[2];
  b.rx0 = a->roi[0] - 1;
  b.ry0 = a->roi[2] - 1;
  b.rz0 = a->roi[4] - 1;
  b.rx = a->roi[1] - a->roi[0] + 1;
  b.ry = a->roi[3] - a->roi[2] + 1;
  b.rz = a->roi[5] - a->roi[4] + 1;
  b.nvox = nvox;
  b.nbatch = 1;
  for (int i = 0; i < 3; ++i) {
    b.mask[i] = a->mask[i];
    b.ramp[i] = reinterpret_cast<const float2*>(a->ramp[i]);
    b.kq2[i] = a->kq2[i];
  }
  b.eps = a->eps_imag;
  b.c_im = 1.0f / a->eps_imag;
  b.g_scale = a->green_scale;
  b.g_off = a->green_offset;
  b.inv_n = (float)(1.0 / (double)nvox);
  b.acyclic = a->acyclic;
  b.T = scratch;
  b.Fn = scratch + nvox;
  b.F = scratch + 2 * nvox;
  b.V = reinterpret_cast<const float2*>(a->V);
  b.Einc = reinterpret_cast<const float2*>(a->einc);
  b.Fout = reinterpret_cast<float2*>(a->fout);
  b.wait_limit = kWaitLimitCycles;
  const int B = a->bornmax;
  for (int jj = 1; jj <= B && e == cudaSuccess; ++jj) {
    if ((e = launch_born_x(b, jj == 1 ? kBornFirst : kBornMid, jj, f[0], s)) != cudaSuccess) break;
    if ((e = launch_fft_cols(b.T, b.T, b.px, (long long)b.pz, 0, 0, 1.0f, false, f[1], s)) != cudaSuccess) break;
    if ((e = launch_born_z(b, jj, f[2], s)) != cudaSuccess) break;
    e = launch_fft_cols(b.T, b.T, b.px, (long long)b.pz, 0, 0, 1.0f, true, f[1], s);
  }
  if (e == cudaSuccess) e = launch_born_x(b, kBornLast, B + 1, f[0], s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ODT_ERR_CUDA, std::string("odt_born_series_noalloc: ") + cudaGetErrorString(e));
  }
  if (!have_tw) {  // the tables are in place from now on
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    std::memcpy(g_noalloc_tw[dev], a->sim_size, sizeof(g_noalloc_tw[dev]));
  }
  odt::set_last_error("");
  return ODT_OK;
}

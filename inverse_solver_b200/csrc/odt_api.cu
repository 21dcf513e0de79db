// C ABI of libodt: handle table, device memory plan and the per-batch
// orchestration of one forward CBS solve (include/odt.h).
//
// Data layout in HBM (column-major, interleaved complex64):
//   static per handle : refocus / kernel_trans / kernel_ref [conv_x, conv_y, ri_z],
//                       pupils [F_x, F_y], twiddle tables, V [sim] + 1D tables
//   per batch slot    : one block of max(3*sim, conv_x*conv_y*ri_z) elements
//                       holding T | Field_n | Field during the Born loop and the
//                       refocus / emitter planes before and after it, plus
//                       Einc and Fout [ri], and small 2D planes.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "fft_any.cuh"
#include "fft_plan.h"
#include "tma.cuh"

namespace odt {

namespace {
thread_local std::string g_last_error;
}  // namespace

// used by the entry points defined in other files (noalloc.cu)
const char* set_last_error(const std::string& msg) {
  g_last_error = msg;
  return g_last_error.c_str();
}

namespace {

odt_status fail(odt_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

struct CudaError {
  cudaError_t err;
  std::string where;
};

#define ODT_CUDA(call)                                                  \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) throw CudaError{e_, std::string(#call)};     \
  } while (0)

struct ApiError {
  odt_status st;
  std::string msg;
};

[[noreturn]] void raise(odt_status st, const std::string& msg) { throw ApiError{st, msg}; }

// A stream capture (run_chunk_graph) must not overlap with device-wide work
// of other threads -- cudaDeviceSynchronize, and allocation / release calls
// that may synchronise the device -- so handles used from several threads
// (the request loop) take this lock around both.
std::recursive_mutex g_device_mu;

// RAII guard restoring the caller's current device (CudaBorn does the same,
// main.cpp:50-53).
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) ODT_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

const char* const kKindNames[] = {"born_x", "born_y", "born_z", "io_fft", "io_elementwise",
                                  "born_x_pipe", "born_y_pipe", "born_z_pipe", "born_x_pipe_edge",
                                  "born_xy", "born_xy_edge"};
// born_x_pipe_edge: the pipelined x-pass of iterations 2, 3 and of the final
// pass (incident-field source / output), timed apart from the steady state;
// born_xy / born_xy_edge: the fused xy-pass, steady (iterations 4..Bornmax)
// and edge (iterations 1-3 and the final pass)
enum Kind { kKBornX = 0, kKBornY, kKBornZ, kKIoFft, kKIoElem, kKBornXPipe, kKBornYPipe, kKBornZPipe,
            kKBornXPipeEdge, kKBornXY, kKBornXYEdge, kNumKinds };

struct Handle {
  odt_geometry g{};
  cudaStream_t own_stream = nullptr;
  // recorded after the work a device-memory solve leaves queued on the
  // caller's stream; waited for before this handle's tables change
  cudaEvent_t done_ev = nullptr;
  bool done_pending = false;
  std::vector<void*> allocs;
  size_t static_bytes = 0;
  size_t batch_bytes = 0;
  size_t budget = 0;

  // transform lengths
  DevFft fx{}, fy{}, fz{}, ffx{}, ffy{}, fcx{}, fcy{};
  // Bluestein plans of the lengths the radix tiles do not cover (direct =
  // true for the others; the DevFft of such a length has no passes)
  AnyFft bsx{}, bsy{}, bsz{}, bsfx{}, bsfy{}, bscx{}, bscy{};
  bool any_loop() const { return !bsx.direct || !bsy.direct || !bsz.direct; }
  bool any_io() const { return !bsfx.direct || !bsfy.direct || !bscx.direct || !bscy.direct; }
  const AnyFft& bs_of(const DevFft& f) const {
    static const AnyFft kDirect{};
    if (&f == &fx) return bsx;
    if (&f == &fy) return bsy;
    if (&f == &fz) return bsz;
    if (&f == &ffx) return bsfx;
    if (&f == &ffy) return bsfy;
    if (&f == &fcx) return bscx;
    if (&f == &fcy) return bscy;
    return kDirect;
  }

  // dyadic (vector) handles: np = 3 field components per illumination (batch
  // entries 3 b + i), npol = 2 input / output polarisations
  int np = 1, npol = 1;
  bool have_pol = false;
  float* pol_tab = nullptr;     // radial [nF,2] | perp [nF,2] | tan3 [nF,3] | kmask [nF]
  int max_smem = 0;

  // static device data
  float2* refocus = nullptr;
  float2* ktrans = nullptr;
  float2* kref = nullptr;
  float* pupil_in = nullptr;
  float* pupil_out = nullptr;

  // potentials: slot 0 = forward (odt_set_potential), slot 1 = adjoint
  // (odt_set_adjoint_potential, used by odt_gradient)
  struct PotSlot {
    bool have = false;
    bool allocated = false;
    odt_potential_params pp{};
    float2* V = nullptr;
    float* mask[3] = {nullptr, nullptr, nullptr};
    float2* ramp[3] = {nullptr, nullptr, nullptr};
    float* kq2[3] = {nullptr, nullptr, nullptr};
    float* rad[3] = {nullptr, nullptr, nullptr};   // dyadic handles
    float2* V9 = nullptr;  // RI tensor potential [nvox, 3, 3] (dyadic handles)
    bool tensor = false;   // the slot's potential is V9, not V
  } pot[2];
  float2* fout_adj = nullptr;   // adjoint 3D field of a batch (odt_gradient)
  float2* grad_acc = nullptr;   // gradient accumulator [ri]
  double* d_err = nullptr;      // misfit accumulator
  int grad_batch = 0;

  // batch buffers
  int batch = 0;
  float2* work = nullptr;
  float2* einc = nullptr;
  float2* fout = nullptr;
  float2* in2d = nullptr;
  float2* kin = nullptr;
  float2* c2a = nullptr;
  float2* c2b = nullptr;
  float2* res_t = nullptr;      // where run_chunk left the transmitted / reflected fields
  float2* res_r = nullptr;
  float2* out_t = nullptr;
  float2* out_r = nullptr;
  unsigned int* d_count = nullptr;
  int* d_fault = nullptr;       // set by a pipelined kernel whose wait timed out
  std::vector<void*> batch_allocs;

  // kernel selection: the pipelined x-pass where it applies (ODT_KERNELS=generic
  // in the environment at odt_create selects the generic tile kernels)
  bool use_pipe = true;
  // clock cycles a pipelined kernel's steady mbarrier wait may take before it
  // reports a timeout (ODT_WAIT_LIMIT_CYCLES in the environment at odt_create;
  // default about a second)
  long long wait_limit = kWaitLimitCycles;
  // the fused xy-pass where it applies (ODT_XY=0 in the environment at
  // odt_create keeps the separate x- and y-passes)
  bool use_xy = true;
  // storage of T and Field_n in the Born loop (ODT_STORAGE_*)
  int storage = ODT_STORAGE_COMPLEX64;

  // CUDA graphs of a batch's whole solve (run_chunk), keyed by batch size,
  // outputs and potential slot; captured the second time a key is seen (the
  // first run is eager, so every kernel attribute is set before a capture)
  // and dropped whenever a buffer or a potential they captured changes.
  // ODT_GRAPHS=0 in the environment at odt_create turns them off.
  bool use_graphs = true;
  std::map<long long, cudaGraphExec_t> graphs;
  std::map<long long, int> graph_seen;
  void drop_graphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
    graph_seen.clear();
  }

  // profiling
  bool profiling = false;
  std::vector<cudaEvent_t> ev;
  std::vector<int> ev_kind;
  size_t ev_used = 0;
  double kind_ms[kNumKinds] = {0};
  long long kind_launches[kNumKinds] = {0};

  long long nvox() const { return (long long)g.sim_size[0] * g.sim_size[1] * g.sim_size[2]; }
  long long nri() const { return (long long)g.ri_size[0] * g.ri_size[1] * g.ri_size[2]; }
  long long nf() const { return (long long)g.field_size[0] * g.field_size[1]; }
  long long nc2() const { return (long long)g.conv_size[0] * g.conv_size[1]; }
  long long nc3() const { return nc2() * g.ri_size[2]; }
  long long work_elems() const { return std::max(3 * nvox(), nc3()); }
  size_t slot_bytes() const {
    return sizeof(float2) * (size_t)np * (size_t)(work_elems() + 2 * nri() + 4 * nf() + 2 * nc2());
  }
  PolTables pol_tables() const {
    const long long n = nf();
    return PolTables{pol_tab, pol_tab + 2 * n, pol_tab + 4 * n, pol_tab + 7 * n};
  }

  // allocate `count` elements; batch buffers go to batch_allocs, the rest to allocs
  template <typename T>
  T* dalloc(size_t count, bool batch_buf) {
    const size_t nb = count * sizeof(T);
    const size_t bytes = static_bytes + batch_bytes;
    if (budget && bytes + nb > budget)
      raise(ODT_ERR_OUT_OF_MEMORY, "memory budget exceeded (" + std::to_string(bytes + nb) +
                                       " > " + std::to_string(budget) + " bytes)");
    void* p = nullptr;
    std::lock_guard<std::recursive_mutex> lk(g_device_mu);
    cudaError_t e = cudaMalloc(&p, nb ? nb : 1);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      raise(ODT_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(nb) + " bytes failed");
    }
    if (e != cudaSuccess) throw CudaError{e, "cudaMalloc"};
    (batch_buf ? batch_allocs : allocs).push_back(p);
    (batch_buf ? batch_bytes : static_bytes) += nb;
    return static_cast<T*>(p);
  }

  void free_batch() {
    std::lock_guard<std::recursive_mutex> lk(g_device_mu);
    for (void* p : batch_allocs) cudaFree(p);
    batch_allocs.clear();
    batch_bytes = 0;
    batch = 0;
  }

  ~Handle() {
    std::lock_guard<std::recursive_mutex> lk(g_device_mu);
    drop_graphs();
    for (void* p : batch_allocs) cudaFree(p);
    for (void* p : allocs) cudaFree(p);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    if (done_ev) cudaEventDestroy(done_ev);
    if (own_stream) cudaStreamDestroy(own_stream);
  }

  // The work of this handle still queued on the GPU has finished: its own
  // stream and the last device-memory solve's stream (other handles' work
  // keeps running, so concurrent solvers do not wait for each other).
  void wait_idle() {
    if (done_pending) {
      ODT_CUDA(cudaEventSynchronize(done_ev));
      done_pending = false;
    }
    ODT_CUDA(cudaStreamSynchronize(own_stream));
  }

  // ---- profiling helpers
  void mark_begin(int kind, cudaStream_t s) {
    if (!profiling) return;
    if (ev_used + 2 > ev.size()) {
      for (int i = 0; i < 64; ++i) {
        cudaEvent_t e;
        ODT_CUDA(cudaEventCreate(&e));
        ev.push_back(e);
      }
    }
    ODT_CUDA(cudaEventRecord(ev[ev_used], s));
    if (ev_kind.size() < ev.size()) ev_kind.resize(ev.size());
    ev_kind[ev_used] = kind;
  }
  void mark_end(cudaStream_t s) {
    if (!profiling) return;
    ODT_CUDA(cudaEventRecord(ev[ev_used + 1], s));
    ev_used += 2;
  }
  void collect(cudaStream_t s) {
    if (!profiling || ev_used == 0) return;
    ODT_CUDA(cudaStreamSynchronize(s));
    for (size_t i = 0; i < ev_used; i += 2) {
      float ms = 0.f;
      ODT_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      kind_ms[ev_kind[i]] += ms;
      kind_launches[ev_kind[i]] += 1;
    }
    ev_used = 0;
  }
};

std::mutex g_mu;
std::map<uint32_t, std::shared_ptr<Handle>> g_handles;
std::atomic<uint32_t> g_next_id{1};

std::shared_ptr<Handle> lookup(odt_handle h) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_handles.find(h);
  if (it == g_handles.end()) raise(ODT_ERR_BAD_HANDLE, "unknown handle " + std::to_string(h));
  return it->second;
}

template <typename F>
odt_status guarded(F&& f) {
  try {
    g_last_error.clear();
    f();
    return ODT_OK;
  } catch (const ApiError& e) {
    return fail(e.st, e.msg);
  } catch (const CudaError& e) {
    cudaGetLastError();
    return fail(e.err == cudaErrorMemoryAllocation ? ODT_ERR_OUT_OF_MEMORY : ODT_ERR_CUDA,
                e.where + ": " + cudaGetErrorString(e.err));
  } catch (const std::exception& e) {
    return fail(ODT_ERR_INTERNAL, e.what());
  } catch (...) {
    return fail(ODT_ERR_INTERNAL, "unknown exception");
  }
}

// Tile shape of a transform of length n used by kernels of `kind`: 16 pencils
// per CTA (8 when n > 512) and 128 threads.
// Radix order: the fused x-pass applies the CBS update between the last
// inverse and the first forward pass, i.e. at radix f[0]; a small radix there
// keeps the update's loads few per thread, and the large radices then sit at
// the passes that touch global memory (many independent loads in flight).
DevFft make_dev_fft(Handle& H, int n, int kind, const char* what) {
  DevFft f{};
  std::string why;
  const int order = kind == kKindBornX ? kSmallFirst : kLargeFirst;
  if (!make_plan(n, &f.plan, &why, order))
    raise(ODT_ERR_UNSUPPORTED, std::string(what) + ": " + why);
  f.lgW = n <= 512 ? 4 : 3;
  f.W = 1 << f.lgW;
  f.nthr = 128;
  int dev = 0;
  ODT_CUDA(cudaGetDevice(&dev));
  int max_smem = 0;
  ODT_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (fft_smem_bytes(n, f.W, kind) > (size_t)max_smem)
    raise(ODT_ERR_UNSUPPORTED, std::string(what) + ": length " + std::to_string(n) +
                                   " needs more shared memory than the device offers");
  auto tw = make_twiddles(n);
  float2* d = H.dalloc<float2>(n, false);
  ODT_CUDA(cudaMemcpy(d, tw.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
  f.tw = d;
  return f;
}

// make_dev_fft for any length: a length with a prime factor above 31 gets a
// Bluestein plan in *bs (tables on the device, transforms of the 5-smooth
// length m >= 2 n - 1 through the line / column tiles) and a DevFft with no
// passes, which no tile kernel accepts.
DevFft make_handle_fft(Handle& H, int n, int kind, const char* what, AnyFft* bs) {
  *bs = AnyFft{};
  bs->n = n;
  FftPlan probe{};
  std::string why;
  if (n < 1) raise(ODT_ERR_INVALID_ARGUMENT, std::string(what) + ": length must be positive");
  if (make_plan(n, &probe, &why, kLargeFirst)) return make_dev_fft(H, n, kind, what);
  const int m = bluestein_length(n);
  bs->direct = false;
  bs->m = m;
  bs->f = make_dev_fft(H, m, kKindCols, what);
  if (fft_smem_bytes(m, bs->f.W, kKindLines) > (size_t)H.max_smem)
    raise(ODT_ERR_UNSUPPORTED, std::string(what) + ": Bluestein length " + std::to_string(m) +
                                   " needs more shared memory than the device offers");
  float2* chirp = H.dalloc<float2>(n, false);
  float2* bhat = H.dalloc<float2>(2 * (size_t)m, false);
  ODT_CUDA(bluestein_tables(n, m, bs->f, chirp, bhat, H.own_stream));
  ODT_CUDA(cudaStreamSynchronize(H.own_stream));
  bs->chirp = chirp;
  bs->bhat_f = bhat;
  bs->bhat_i = bhat + m;
  DevFft f{};
  f.plan.n = n;
  f.plan.npass = 0;
  return f;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

void ensure_batch(Handle& H, int nb) {
  if (H.batch >= nb) return;
  std::lock_guard<std::recursive_mutex> lk(g_device_mu);
  ODT_CUDA(cudaDeviceSynchronize());  // buffers may still be in use by queued work
  H.drop_graphs();
  H.free_batch();
  const size_t nbp = (size_t)nb * H.np;  // field planes of nb illuminations
  H.work = H.dalloc<float2>((size_t)H.work_elems() * nbp, true);
  H.einc = H.dalloc<float2>((size_t)H.nri() * nbp, true);
  H.fout = H.dalloc<float2>((size_t)H.nri() * nbp, true);
  H.in2d = H.dalloc<float2>((size_t)H.nf() * nbp, true);
  H.kin = H.dalloc<float2>((size_t)H.nf() * nbp, true);
  H.out_t = H.dalloc<float2>((size_t)H.nf() * nbp, true);
  H.out_r = H.dalloc<float2>((size_t)H.nf() * nbp, true);
  H.c2a = H.dalloc<float2>((size_t)H.nc2() * nbp, true);
  H.c2b = H.dalloc<float2>((size_t)H.nc2() * nbp, true);
  H.d_count = H.dalloc<unsigned int>(1, true);
  H.d_fault = H.dalloc<int>(1, true);
  ODT_CUDA(cudaMemset(H.d_fault, 0, sizeof(int)));
  H.batch = nb;
}

int auto_batch(Handle& H) {
  if (H.g.max_batch > 0) return H.g.max_batch;
  size_t free_b = 0, total_b = 0;
  ODT_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t held = H.static_bytes;  // batch buffers are reallocated, not added
  size_t avail = H.budget ? (H.budget > held ? H.budget - held : 0) : (free_b + H.batch_bytes) / 2;
  long long nb = (long long)(avail / std::max<size_t>(1, H.slot_bytes()));
  if (nb > 64) nb = 64;
  if (nb < 1) raise(ODT_ERR_OUT_OF_MEMORY, "not enough device memory for one illumination");
  return (int)nb;
}

// centred 2D FFT on [n0, n1, nslices] in place (MATLAB fftshift(fft2(ifftshift(x))))
// (Bluestein on an axis whose length has a prime factor above 31; the
// inverse then normalises axis by axis)
void fftc2(Handle& H, float2* x, const DevFft& f0, const DevFft& f1, long long nslices,
           bool inverse, cudaStream_t s) {
  const int n0 = f0.plan.n, n1 = f1.plan.n;
  const AnyFft& b0 = H.bs_of(f0);
  const AnyFft& b1 = H.bs_of(f1);
  H.mark_begin(kKIoFft, s);
  if (b0.direct && b1.direct) {
    const float sc = inverse ? 1.0f / ((float)n0 * (float)n1) : 1.0f;
    ODT_CUDA(launch_fft_lines(x, x, (long long)n1 * nslices, n0 / 2, n0 / 2, 1.0f, inverse, f0, s));
    ODT_CUDA(launch_fft_cols(x, x, n0, nslices, n1 / 2, n1 / 2, sc, inverse, f1, s));
  } else {
    const float s0 = inverse ? 1.0f / (float)n0 : 1.0f, s1 = inverse ? 1.0f / (float)n1 : 1.0f;
    if (b0.direct)
      ODT_CUDA(launch_fft_lines(x, x, (long long)n1 * nslices, n0 / 2, n0 / 2, s0, inverse, f0, s));
    else
      ODT_CUDA(bluestein_axis(x, 1, (long long)n1 * nslices, inverse, n0 / 2, s0, b0, s));
    if (b1.direct)
      ODT_CUDA(launch_fft_cols(x, x, n0, nslices, n1 / 2, n1 / 2, s1, inverse, f1, s));
    else
      ODT_CUDA(bluestein_axis(x, n0, nslices, inverse, n1 / 2, s1, b1, s));
  }
  H.mark_end(s);
}

// A pipelined kernel whose bounded wait ran out leaves a fault code behind.
void check_fault(Handle& H) {
  int f = 0;
  ODT_CUDA(cudaMemcpy(&f, H.d_fault, sizeof(f), cudaMemcpyDeviceToHost));
  if (f) {
    ODT_CUDA(cudaMemset(H.d_fault, 0, sizeof(int)));
    raise(ODT_ERR_INTERNAL, "a pipelined Born kernel timed out waiting for its copies (code " +
                                std::to_string(f) + ")");
  }
}

// from_source: the batch's incident fields over the RI grid are already in
// H.einc (odt_solve_source, CudaBorn's action 2): no input stage, and no
// output projection (want_t / want_r must be false)
void run_chunk(Handle& H, int nb, cudaStream_t s, bool want_t, bool want_r, int slot,
               float2* fout, bool from_source = false) {
  const Handle::PotSlot& P = H.pot[slot];
  const odt_geometry& g = H.g;
  const int Fx = g.field_size[0], Fy = g.field_size[1];
  const int Cx = g.conv_size[0], Cy = g.conv_size[1];
  const int Rx = g.ri_size[0], Ry = g.ri_size[1], Rz = g.ri_size[2];
  const long long nF = H.nf();
  const int ocx = Cx / 2 - Fx / 2, ocy = Cy / 2 - Fy / 2;   // field <-> conv offsets
  const int orx = Cx / 2 - Rx / 2, ory = Cy / 2 - Ry / 2;   // RI -> conv (padd_RI2conv)
  float2* conv = H.work;

  // ---- input: fft2 + pupil, back to space, pad, fft2, refocus, ifft2, crop
  //      (FORWARD_SOLVER_CONVERGENT_BORN.m:416-418, :543-554); a dyadic handle
  //      maps the two input polarisations onto three components in between
  //      (transform_field_3D, FORWARD_SOLVER.m:38-68) and carries 3 planes per
  //      illumination from there on
  const bool vec = H.np == 3;
  const long long nbp = (long long)nb * H.np;
  if (from_source) want_t = want_r = false;
  // fused refocus / inverse 2D FFT / crop (io_fused.cu) where its tiles fit;
  // the unfused chain is kept for ODT_KERNELS=generic
  const int nacc = (want_t ? 1 : 0) + (want_r ? 1 : 0);
  const IoGeom gin{Cx, Cy, Rx, Ry, Rz, ocx, ocy, nbp}, gout{Cx, Cy, Rx, Ry, Rz, orx, ory, nbp};
  const bool io_fused = H.use_pipe && !H.any_io() && io_fused_fits(gin, H.fcx, H.fcy, nacc, H.max_smem) &&
                        io_fused_fits(gout, H.fcx, H.fcy, nacc, H.max_smem);
  // an RI tensor couples the field components in the emitter: unfused output
  const bool ten = P.tensor;
  const bool io_out_fused = io_fused && !ten;
  if (!from_source) {
  fftc2(H, H.in2d, H.ffx, H.ffy, (long long)nb * H.npol, false, s);
  H.mark_begin(kKIoElem, s);
  ODT_CUDA(launch_mul_plane(H.in2d, H.in2d, vec ? nullptr : H.kin, H.pupil_in, nF, nF * nb * H.npol, s));
  if (vec) ODT_CUDA(launch_pol23(H.in2d, H.out_t, H.kin, H.pol_tables(), nF, nb, s));
  H.mark_end(s);
  float2* src2 = vec ? H.out_t : H.in2d;
  fftc2(H, src2, H.ffx, H.ffy, nbp, true, s);
  H.mark_begin(kKIoElem, s);
  ODT_CUDA(launch_pad2d(src2, H.c2a, Fx, Fy, Cx, Cy, ocx, ocy, nbp, s));
  H.mark_end(s);
  fftc2(H, H.c2a, H.fcx, H.fcy, nbp, false, s);
  if (io_fused) {
    H.mark_begin(kKIoFft, s);
    ODT_CUDA(launch_refocus_in(H.c2a, H.refocus, conv, H.einc, gin, H.fcx, H.fcy, s));
    H.mark_end(s);
  } else {
    H.mark_begin(kKIoElem, s);
    ODT_CUDA(launch_refocus_expand(H.c2a, H.refocus, conv, Cx, Cy, Rz, nbp, s));
    H.mark_end(s);
    fftc2(H, conv, H.fcx, H.fcy, (long long)Rz * nbp, true, s);
    H.mark_begin(kKIoElem, s);
    ODT_CUDA(launch_crop_volume(conv, H.einc, Cx, Cy, Rx, Ry, Rz, ocx, ocy, nbp, s));
    H.mark_end(s);
  }
  }  // !from_source

  // ---- Born series (:577-647)
  BornArgs a{};
  a.px = g.sim_size[0];
  a.py = g.sim_size[1];
  a.pz = g.sim_size[2];
  a.rx0 = P.pp.roi[0] - 1;
  a.ry0 = P.pp.roi[2] - 1;
  a.rz0 = P.pp.roi[4] - 1;
  a.rx = Rx;
  a.ry = Ry;
  a.rz = Rz;
  a.nvox = H.nvox();
  a.nbatch = (int)nbp;
  for (int i = 0; i < 3; ++i) {
    a.mask[i] = P.mask[i];
    a.ramp[i] = P.ramp[i];
    a.kq2[i] = P.kq2[i];
  }
  a.eps = P.pp.eps_imag;
  a.c_im = 1.0f / P.pp.eps_imag;
  a.g_scale = P.pp.green_scale;
  a.g_off = P.pp.green_offset;
  a.inv_n = (float)(1.0 / (double)H.nvox());
  a.acyclic = P.pp.acyclic;
  a.T = H.work;
  a.Fn = H.work + (size_t)H.nvox() * nbp;
  a.F = H.work + 2 * (size_t)H.nvox() * nbp;
  a.V = P.V;
  a.Einc = H.einc;
  a.Fout = fout;
  a.wait_limit = H.wait_limit;
  const int B = P.pp.bornmax;
  if (H.any_loop()) {
    // unfused loop with Bluestein transforms along the uncovered axes
    if (ten || vec) raise(ODT_ERR_UNSUPPORTED, "RI tensors and dyadic solves need padded lengths whose prime "
                                               "factors are at most 31");
    const long long xl = (long long)a.py * a.pz * nbp, yl = (long long)a.pz * nbp;
    const long long pxy = (long long)a.px * a.py;
    auto fft3 = [&](bool inv) {
      auto ax = [&]() {
        if (H.bsx.direct) ODT_CUDA(launch_fft_lines(a.T, a.T, xl, 0, 0, 1.0f, inv, H.fx, s));
        else ODT_CUDA(bluestein_axis(a.T, 1, xl, inv, 0, 1.0f, H.bsx, s));
      };
      auto ay = [&]() {
        if (H.bsy.direct) ODT_CUDA(launch_fft_cols(a.T, a.T, a.px, yl, 0, 0, 1.0f, inv, H.fy, s));
        else ODT_CUDA(bluestein_axis(a.T, a.px, yl, inv, 0, 1.0f, H.bsy, s));
      };
      auto az = [&]() {
        if (pxy > INT32_MAX) raise(ODT_ERR_UNSUPPORTED, "x-y plane too large for the column transforms");
        if (H.bsz.direct) ODT_CUDA(launch_fft_cols(a.T, a.T, (int)pxy, nbp, 0, 0, 1.0f, inv, H.fz, s));
        else ODT_CUDA(bluestein_axis(a.T, (int)pxy, nbp, inv, 0, 1.0f, H.bsz, s));
      };
      H.mark_begin(kKBornY, s);
      if (inv) { az(); ay(); ax(); } else { ax(); ay(); az(); }
      H.mark_end(s);
    };
    for (int jj = 1; jj <= B; ++jj) {
      if (jj >= 2) fft3(true);
      H.mark_begin(kKBornX, s);
      ODT_CUDA(launch_born_point(a, jj == 1 ? kBornFirst : kBornMid, jj, s));
      H.mark_end(s);
      fft3(false);
      H.mark_begin(kKBornZ, s);
      ODT_CUDA(launch_born_green(a, jj, s));
      H.mark_end(s);
    }
    if (B >= 1) fft3(true);
    H.mark_begin(kKBornX, s);
    ODT_CUDA(launch_born_point(a, kBornLast, B + 1, s));
    H.mark_end(s);
  }
  const bool any = H.any_loop();
  const bool pipe_x = !any && !ten && H.use_pipe && born_x_pipe_supported(a, H.fx);
  const bool pipe_y = !any && H.use_pipe && cols_pipe_supported(a, H.fy, false);
  const bool pipe_z = !any && !vec && H.use_pipe && cols_pipe_supported(a, H.fz, true);
  DyadArgs dy{};
  if (vec) {
    for (int i = 0; i < 3; ++i) dy.rad[i] = P.rad[i];
    dy.absorb = make_float2(P.pp.absorb.re, P.pp.absorb.im);
  }
  const long long xlines = (long long)a.py * a.pz * nbp;
  // fused xy-pass (x- and both y-passes in one kernel; the z-pass, pipelined
  // or generic, reads its permuted x-y spectrum): scalar potentials
  const bool fused_xy = !any && !ten && !vec && H.use_pipe && H.use_xy && B >= 1 && born_xy_supported(a, H.max_smem);
  a.perm_xy = fused_xy ? 1 : 0;
  if (H.storage == ODT_STORAGE_B16) {
    if (!fused_xy || !pipe_z)
      raise(ODT_ERR_UNSUPPORTED,
            "16-bit block storage (ODT_STORAGE_B16) needs the fused xy-pass: a scalar potential on a grid "
            "with equal x and y lengths of 8 * R (11 <= R <= 20) and a z length of 8 * R (11 <= R <= 20, 25, "
            "27)");
    // T16 | Field_n16 | Field | exponents of T | exponents of Field_n in the
    // work block (16.25 of its 24 bytes per voxel)
    const size_t n = (size_t)a.nvox * (size_t)nbp;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    char* w = reinterpret_cast<char*>(H.work);
    a.storage = 1;
    a.T16 = reinterpret_cast<short2*>(w);
    a.Fn16 = reinterpret_cast<short2*>(w + al(4 * n));
    a.F = reinterpret_cast<float2*>(w + 2 * al(4 * n));
    a.Te = reinterpret_cast<signed char*>(w + 2 * al(4 * n) + al(8 * n));
    a.Fe = a.Te + al(n / 8);
    a.T = nullptr;
    a.Fn = nullptr;
  }
  for (int jj = 1; fused_xy && jj <= B; ++jj) {
    H.mark_begin(jj <= 4 ? kKBornXYEdge : kKBornXY, s);
    ODT_CUDA(launch_born_xy(a, jj == 1 ? kBornFirst : kBornMid, jj, H.fx, s));
    H.mark_end(s);
    H.mark_begin(pipe_z ? kKBornZPipe : kKBornZ, s);
    if (pipe_z)
      ODT_CUDA(launch_born_z_pipe(a, jj, H.fz, H.d_fault, s));
    else
      ODT_CUDA(launch_born_z(a, jj, H.fz, s));
    H.mark_end(s);
  }
  if (fused_xy) {
    H.mark_begin(kKBornXYEdge, s);
    ODT_CUDA(launch_born_xy(a, kBornLast, B + 1, H.fx, s));
    H.mark_end(s);
  }
  for (int jj = 1; !any && !fused_xy && jj <= B; ++jj) {
    if (ten) {  // plain x-FFTs around the component-coupling pointwise kernel
      H.mark_begin(kKBornX, s);
      if (jj >= 2) ODT_CUDA(launch_fft_lines(a.T, a.T, xlines, 0, 0, 1.0f, true, H.fx, s));
      ODT_CUDA(launch_born_tensor_point(a, P.V9, jj == 1 ? kBornFirst : kBornMid, jj, s));
      ODT_CUDA(launch_fft_lines(a.T, a.T, xlines, 0, 0, 1.0f, false, H.fx, s));
    } else if (pipe_x && jj >= 2) {
      H.mark_begin(jj <= 4 ? kKBornXPipeEdge : kKBornXPipe, s);
      ODT_CUDA(launch_born_x_pipe(a, kBornMid, jj, H.fx, H.d_fault, s));
    } else {
      H.mark_begin(kKBornX, s);
      ODT_CUDA(launch_born_x(a, jj == 1 ? kBornFirst : kBornMid, jj, H.fx, s));
    }
    H.mark_end(s);
    H.mark_begin(pipe_y ? kKBornYPipe : kKBornY, s);
    if (pipe_y)
      ODT_CUDA(launch_fft_y_pipe(a, false, H.fy, H.d_fault, s));
    else
      ODT_CUDA(launch_fft_cols(a.T, a.T, a.px, (long long)a.pz * nbp, 0, 0, 1.0f, false, H.fy, s));
    H.mark_end(s);
    H.mark_begin(pipe_z ? kKBornZPipe : kKBornZ, s);
    if (vec)
      ODT_CUDA(launch_born_z_dyadic(a, dy, jj, H.fz, H.max_smem, s));
    else if (pipe_z)
      ODT_CUDA(launch_born_z_pipe(a, jj, H.fz, H.d_fault, s));
    else
      ODT_CUDA(launch_born_z(a, jj, H.fz, s));
    H.mark_end(s);
    H.mark_begin(pipe_y ? kKBornYPipe : kKBornY, s);
    if (pipe_y)
      ODT_CUDA(launch_fft_y_pipe(a, true, H.fy, H.d_fault, s));
    else
      ODT_CUDA(launch_fft_cols(a.T, a.T, a.px, (long long)a.pz * nbp, 0, 0, 1.0f, true, H.fy, s));
    H.mark_end(s);
  }
  if (!any && !fused_xy) {
    if (ten) {
      H.mark_begin(kKBornX, s);
      if (B >= 1) ODT_CUDA(launch_fft_lines(a.T, a.T, xlines, 0, 0, 1.0f, true, H.fx, s));
      ODT_CUDA(launch_born_tensor_point(a, P.V9, kBornLast, B + 1, s));
    } else if (pipe_x && B + 1 >= 2) {
      H.mark_begin(kKBornXPipeEdge, s);
      ODT_CUDA(launch_born_x_pipe(a, kBornLast, B + 1, H.fx, H.d_fault, s));
    } else {
      H.mark_begin(kKBornX, s);
      ODT_CUDA(launch_born_x(a, kBornLast, B + 1, H.fx, s));
    }
    H.mark_end(s);
  }

  // ---- output projection (:445-511)
  if (want_t || want_r) {
    if (io_out_fused) {
      H.mark_begin(kKIoFft, s);
      ODT_CUDA(launch_project_out(a, conv, H.work_elems() * nbp, want_t ? H.ktrans : nullptr,
                                  want_r ? H.kref : nullptr, want_t ? H.c2a : nullptr, want_r ? H.c2b : nullptr,
                                  gout, P.pp.dV, H.fcx, H.fcy, s));
      H.mark_end(s);
    } else {
      H.mark_begin(kKIoElem, s);
      if (ten)
        ODT_CUDA(launch_born_tensor_emitter(a, P.V9, conv, Cx, Cy, orx, ory, P.pp.dV, s));
      else
        ODT_CUDA(launch_emitter(a, conv, Cx, Cy, orx, ory, P.pp.dV, s));
      H.mark_end(s);
      fftc2(H, conv, H.fcx, H.fcy, (long long)Rz * nbp, false, s);
      H.mark_begin(kKIoElem, s);
      ODT_CUDA(launch_zreduce(conv, want_t ? H.ktrans : nullptr, want_r ? H.kref : nullptr,
                              want_t ? H.c2a : nullptr, want_r ? H.c2b : nullptr, Cx, Cy, Rz, nbp, s));
      H.mark_end(s);
    }
    for (int w = 0; w < 2; ++w) {
      if ((w == 0 && !want_t) || (w == 1 && !want_r)) continue;
      float2* c2 = w == 0 ? H.c2a : H.c2b;
      float2* o = w == 0 ? H.out_t : H.out_r;
      fftc2(H, c2, H.fcx, H.fcy, nbp, true, s);
      H.mark_begin(kKIoElem, s);
      ODT_CUDA(launch_crop2d(c2, o, Fx, Fy, Cx, Cy, ocx, ocy, nbp, s));
      H.mark_end(s);
      fftc2(H, o, H.ffx, H.ffy, nbp, false, s);
      H.mark_begin(kKIoElem, s);
      ODT_CUDA(launch_combine(o, w == 0 ? H.kin : nullptr, H.pupil_out, o, nF, nF * nbp, s));
      H.mark_end(s);
      float2* res = o;
      if (vec) {  // three components -> two polarisations (transform_field_2D / _reflection)
        H.mark_begin(kKIoElem, s);
        ODT_CUDA(launch_pol32(o, c2, H.pol_tables(), w == 1, nF, nb, s));
        H.mark_end(s);
        res = c2;
      }
      fftc2(H, res, H.ffx, H.ffy, (long long)nb * H.npol, true, s);
      (w == 0 ? H.res_t : H.res_r) = res;
    }
  }
}


// run_chunk through the handle's graph cache: eager the first time a key is
// seen, captured (thread-local capture mode) the second time, replayed after.
// Not on the legacy / per-thread default streams (they cannot be captured)
// nor while per-kernel profiling is on.
void run_chunk_graph(Handle& H, int nb, cudaStream_t s, bool want_t, bool want_r, int slot,
                     float2* fout) {
  if (!H.use_graphs || H.profiling || s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) {
    run_chunk(H, nb, s, want_t, want_r, slot, fout);
    return;
  }
  const long long key = (long long)nb | ((long long)want_t << 32) | ((long long)want_r << 33) |
                        ((long long)slot << 34) | ((long long)(fout == H.fout_adj) << 35);
  auto it = H.graphs.find(key);
  if (it == H.graphs.end()) {
    if (H.graph_seen[key]++ == 0) {
      run_chunk(H, nb, s, want_t, want_r, slot, fout);
      return;
    }
    std::lock_guard<std::recursive_mutex> lk(g_device_mu);
    ODT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      run_chunk(H, nb, s, want_t, want_r, slot, fout);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    cudaGraph_t g = nullptr;
    ODT_CUDA(cudaStreamEndCapture(s, &g));
    cudaGraphExec_t ge = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    ODT_CUDA(e);
    it = H.graphs.emplace(key, ge).first;
  }
  ODT_CUDA(cudaGraphLaunch(it->second, s));
}

void alloc_slot(Handle& H, int k) {
  Handle::PotSlot& P = H.pot[k];
  if (P.allocated) return;
  const odt_geometry& g = H.g;
  P.V = H.dalloc<float2>((size_t)H.nvox(), false);
  for (int i = 0; i < 3; ++i) {
    P.mask[i] = H.dalloc<float>(g.sim_size[i], false);
    P.ramp[i] = H.dalloc<float2>(g.sim_size[i], false);
    P.kq2[i] = H.dalloc<float>(g.sim_size[i], false);
    if (H.np == 3) P.rad[i] = H.dalloc<float>(g.sim_size[i], false);
  }
  P.allocated = true;
}

// V from the host (odt_set_potential) or built on the device from an RI
// array in device memory (odt_set_potential_device: dev != NULL)
void set_potential_slot(const std::shared_ptr<Handle>& Hp, int k, const odt_potential_params* pp,
                        const odt_cfloat* V, const char* fn, const odt_ri_device_args* dev = nullptr,
                        const odt_cfloat* V9 = nullptr) {
  Handle& H = *Hp;
  const std::string who(fn);
  if (!pp || (!V && !dev && !V9)) raise(ODT_ERR_INVALID_ARGUMENT, who + ": NULL argument");
  if (V9 && H.np != 3) raise(ODT_ERR_INVALID_ARGUMENT, who + ": an RI tensor needs a dyadic (pol = 3) handle");
  const odt_geometry& g = H.g;
  for (int i = 0; i < 3; ++i) {
    const int lo = pp->roi[2 * i], hi = pp->roi[2 * i + 1];
    if (lo < 1 || hi > g.sim_size[i] || hi - lo + 1 != g.ri_size[i])
      raise(ODT_ERR_INVALID_ARGUMENT, who + ": ROI does not match ri_size");
    if (!pp->mask[i] || !pp->kq2[i] || (pp->acyclic && !pp->ramp[i]) || (H.np == 3 && !pp->rad[i]))
      raise(ODT_ERR_INVALID_ARGUMENT, who + ": NULL table");
  }
  if (pp->bornmax < 0) raise(ODT_ERR_INVALID_ARGUMENT, who + ": bornmax < 0");
  if (!(pp->eps_imag > 0.f) || !std::isfinite(pp->eps_imag))
    raise(ODT_ERR_INVALID_ARGUMENT, who + ": eps_imag must be positive and finite");
  if (!std::isfinite(pp->green_scale) || !std::isfinite(pp->green_offset) || !std::isfinite(pp->dV))
    raise(ODT_ERR_INVALID_ARGUMENT, who + ": non-finite scalar");
  DeviceGuard dg(g.device);
  std::lock_guard<std::recursive_mutex> lk(g_device_mu);
  H.wait_idle();  // a queued solve or graph of this handle may still read the old tables
  H.drop_graphs();
  alloc_slot(H, k);
  Handle::PotSlot& P = H.pot[k];
  const size_t nv = (size_t)H.nvox();
  if (V9) {
    if (!P.V9) P.V9 = H.dalloc<float2>(9 * nv, false);
    ODT_CUDA(cudaMemcpy(P.V9, V9, 9 * nv * sizeof(float2), cudaMemcpyHostToDevice));
  } else if (dev) {
    int roi0[3];
    for (int i = 0; i < 3; ++i) roi0[i] = pp->roi[2 * i] - 1;
    cudaStream_t s = (cudaStream_t)dev->stream;
    ODT_CUDA(launch_build_potential(dev->ri, dev->is_complex, dev->adjoint, g.sim_size, roi0, g.ri_size,
                                    dev->wavelength, dev->ri_bg, pp->eps_imag, P.V, s));
    ODT_CUDA(cudaStreamSynchronize(s));
  } else {
    ODT_CUDA(cudaMemcpy(P.V, V, nv * sizeof(float2), cudaMemcpyHostToDevice));
  }
  std::vector<float2> one;
  for (int i = 0; i < 3; ++i) {
    const size_t n = g.sim_size[i];
    ODT_CUDA(cudaMemcpy(P.mask[i], pp->mask[i], n * sizeof(float), cudaMemcpyHostToDevice));
    ODT_CUDA(cudaMemcpy(P.kq2[i], pp->kq2[i], n * sizeof(float), cudaMemcpyHostToDevice));
    if (H.np == 3) ODT_CUDA(cudaMemcpy(P.rad[i], pp->rad[i], n * sizeof(float), cudaMemcpyHostToDevice));
    if (pp->acyclic) {
      ODT_CUDA(cudaMemcpy(P.ramp[i], pp->ramp[i], n * sizeof(float2), cudaMemcpyHostToDevice));
    } else {
      one.assign(n, make_float2(1.f, 0.f));
      ODT_CUDA(cudaMemcpy(P.ramp[i], one.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    }
  }
  P.pp = *pp;
  P.tensor = V9 != nullptr;
  for (int i = 0; i < 3; ++i) {  // do not keep caller pointers
    P.pp.mask[i] = nullptr;
    P.pp.ramp[i] = nullptr;
    P.pp.kq2[i] = nullptr;
    P.pp.rad[i] = nullptr;
  }
  P.have = true;
}

}  // namespace
}  // namespace odt

using namespace odt;

extern "C" {

int32_t odt_abi_version(void) { return ODT_ABI_VERSION; }

const char* odt_last_error(void) { return g_last_error.c_str(); }

odt_status odt_create(const odt_geometry* geom, const odt_cfloat* refocus,
                      const odt_cfloat* kernel_trans, const odt_cfloat* kernel_ref,
                      const float* pupil_in, const float* pupil_out, odt_handle* out) {
  return guarded([&] {
    if (!geom || !out || !refocus || !pupil_in || !pupil_out)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_create: NULL argument");
    *out = 0;
    const odt_geometry& g = *geom;
    for (int i = 0; i < 3; ++i) {
      if (g.sim_size[i] < 1 || g.ri_size[i] < 1 || g.ri_size[i] > g.sim_size[i])
        raise(ODT_ERR_INVALID_ARGUMENT, "odt_create: sim_size / ri_size out of range");
    }
    for (int i = 0; i < 2; ++i) {
      if (g.field_size[i] != g.ri_size[i])
        raise(ODT_ERR_INVALID_ARGUMENT,
              "odt_create: field_size must equal ri_size(1:2) (the reference's crop_field2RI "
              "and V(ROI).*source require it)");
      if (g.conv_size[i] != g.field_size[i] + g.ri_size[i] && g.conv_size[i] != g.field_size[i])
        raise(ODT_ERR_INVALID_ARGUMENT,
              "odt_create: conv_size must be field_size + ri_size (or field_size for a "
              "cyclic xy boundary)");
    }
    if (g.max_batch < 0 || g.mem_budget < 0)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_create: negative max_batch / mem_budget");
    if (g.pol != 0 && g.pol != 1 && g.pol != 3)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_create: pol must be 1 (scalar) or 3 (dyadic)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      raise(ODT_ERR_CUDA, "odt_create: no CUDA device");
    }
    if (g.device < 0 || g.device >= ndev)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_create: device ordinal out of range");
    DeviceGuard dg(g.device);
    auto H = std::make_shared<Handle>();
    H->g = g;
    H->budget = (size_t)g.mem_budget;
    H->np = g.pol == 3 ? 3 : 1;
    H->npol = g.pol == 3 ? 2 : 1;
    ODT_CUDA(cudaDeviceGetAttribute(&H->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, g.device));
    if (const char* k = std::getenv("ODT_KERNELS")) H->use_pipe = std::string(k) != "generic";
    if (const char* k = std::getenv("ODT_GRAPHS")) H->use_graphs = std::string(k) != "0";
    if (const char* k = std::getenv("ODT_XY")) H->use_xy = std::string(k) != "0";
    if (const char* k = std::getenv("ODT_WAIT_LIMIT_CYCLES")) {
      char* end = nullptr;
      const long long v = std::strtoll(k, &end, 10);
      if (end == k || *end != '\0' || v < 0)
        raise(ODT_ERR_INVALID_ARGUMENT, std::string("ODT_WAIT_LIMIT_CYCLES must be a non-negative integer, got '") +
                                            k + "'");
      H->wait_limit = v;
    }
    ODT_CUDA(cudaStreamCreateWithFlags(&H->own_stream, cudaStreamNonBlocking));
    ODT_CUDA(cudaEventCreateWithFlags(&H->done_ev, cudaEventDisableTiming));
    H->fx = make_handle_fft(*H, g.sim_size[0], kKindBornX, "sim_size(1)", &H->bsx);
    H->fy = make_handle_fft(*H, g.sim_size[1], kKindCols, "sim_size(2)", &H->bsy);
    H->fz = make_handle_fft(*H, g.sim_size[2], kKindBornZ, "sim_size(3)", &H->bsz);
    H->ffx = make_handle_fft(*H, g.field_size[0], kKindLines, "field_size(1)", &H->bsfx);
    H->ffy = make_handle_fft(*H, g.field_size[1], kKindCols, "field_size(2)", &H->bsfy);
    H->fcx = make_handle_fft(*H, g.conv_size[0], kKindLines, "conv_size(1)", &H->bscx);
    H->fcy = make_handle_fft(*H, g.conv_size[1], kKindCols, "conv_size(2)", &H->bscy);
    if ((H->any_loop() || H->any_io()) && H->np == 3)
      raise(ODT_ERR_UNSUPPORTED, "dyadic (vector) solves need simulation, field and convolution lengths whose "
                                 "prime factors are at most 31");
    const size_t n3 = (size_t)H->nc3();
    H->refocus = H->dalloc<float2>(n3, false);
    ODT_CUDA(cudaMemcpy(H->refocus, refocus, n3 * sizeof(float2), cudaMemcpyHostToDevice));
    if (kernel_trans) {
      H->ktrans = H->dalloc<float2>(n3, false);
      ODT_CUDA(cudaMemcpy(H->ktrans, kernel_trans, n3 * sizeof(float2), cudaMemcpyHostToDevice));
    }
    if (kernel_ref) {
      H->kref = H->dalloc<float2>(n3, false);
      ODT_CUDA(cudaMemcpy(H->kref, kernel_ref, n3 * sizeof(float2), cudaMemcpyHostToDevice));
    }
    const size_t nf = (size_t)H->nf();
    H->pupil_in = H->dalloc<float>(nf, false);
    H->pupil_out = H->dalloc<float>(nf, false);
    ODT_CUDA(cudaMemcpy(H->pupil_in, pupil_in, nf * sizeof(float), cudaMemcpyHostToDevice));
    ODT_CUDA(cudaMemcpy(H->pupil_out, pupil_out, nf * sizeof(float), cudaMemcpyHostToDevice));
    alloc_slot(*H, 0);
    const uint32_t id = g_next_id++;
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_handles[id] = H;
    }
    *out = id;
  });
}

odt_status odt_set_potential(odt_handle h, const odt_potential_params* pp, const odt_cfloat* V) {
  return guarded([&] { set_potential_slot(lookup(h), 0, pp, V, "odt_set_potential"); });
}

odt_status odt_set_adjoint_potential(odt_handle h, const odt_potential_params* pp,
                                     const odt_cfloat* V) {
  return guarded([&] { set_potential_slot(lookup(h), 1, pp, V, "odt_set_adjoint_potential"); });
}

odt_status odt_set_tensor_potential(odt_handle h, const odt_potential_params* pp, const odt_cfloat* V9) {
  return guarded([&] {
    if (!V9) raise(ODT_ERR_INVALID_ARGUMENT, "odt_set_tensor_potential: NULL argument");
    set_potential_slot(lookup(h), 0, pp, nullptr, "odt_set_tensor_potential", nullptr, V9);
  });
}

namespace {
void check_ri_device_args(const odt_ri_device_args* a, const char* fn) {
  const std::string who(fn);
  if (!a || !a->ri) raise(ODT_ERR_INVALID_ARGUMENT, who + ": NULL argument");
  if (!is_device_ptr(a->ri)) raise(ODT_ERR_INVALID_ARGUMENT, who + ": ri is not a device pointer");
  if (!(a->wavelength > 0.0) || !(a->ri_bg > 0.0) || !std::isfinite(a->wavelength) || !std::isfinite(a->ri_bg))
    raise(ODT_ERR_INVALID_ARGUMENT, who + ": wavelength and ri_bg must be positive");
}
}  // namespace

odt_status odt_potential_eps_device(odt_handle h, const odt_ri_device_args* a, float* eps_imag) {
  return guarded([&] {
    auto H = lookup(h);
    check_ri_device_args(a, "odt_potential_eps_device");
    if (!eps_imag) raise(ODT_ERR_INVALID_ARGUMENT, "odt_potential_eps_device: NULL eps_imag");
    DeviceGuard dg(H->g.device);
    cudaStream_t s = (cudaStream_t)a->stream;
    unsigned int* d = nullptr;
    {
      std::lock_guard<std::recursive_mutex> lk(g_device_mu);
      ODT_CUDA(cudaMallocAsync((void**)&d, sizeof(unsigned int), s));
    }
    const long long n = (long long)H->g.ri_size[0] * H->g.ri_size[1] * H->g.ri_size[2];
    unsigned int bits = 0;
    cudaError_t e = launch_potential_absmax(a->ri, a->is_complex, n, a->wavelength, a->ri_bg, d, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d, s);
    ODT_CUDA(e);
    float m;
    std::memcpy(&m, &bits, sizeof(m));
    *eps_imag = m * 1.01f;   // single(max|V|) * 1.01 in single, as condition_RI (:205)
  });
}

odt_status odt_set_potential_device(odt_handle h, const odt_potential_params* pp, const odt_ri_device_args* a) {
  return guarded([&] {
    auto H = lookup(h);
    check_ri_device_args(a, "odt_set_potential_device");
    set_potential_slot(H, a->adjoint ? 1 : 0, pp, nullptr, "odt_set_potential_device", a);
  });
}

namespace {
void check_fista_args(const odt_fista_args* a, const char* fn) {
  const std::string who(fn);
  if (!a || a->n <= 0 || !a->u || !a->x || !a->ri || !a->prox_in || !a->prox_out || !a->grad)
    raise(ODT_ERR_INVALID_ARGUMENT, who + ": NULL argument or n <= 0");
  for (const void* p : {(const void*)a->u, (const void*)a->x, (const void*)a->ri, (const void*)a->prox_in,
                        a->prox_out, (const void*)a->grad})
    if (!is_device_ptr(p)) raise(ODT_ERR_INVALID_ARGUMENT, who + ": arrays must be device pointers");
}
}  // namespace

odt_status odt_fista_prox_input(const odt_fista_args* a) {
  return guarded([&] {
    check_fista_args(a, "odt_fista_prox_input");
    ODT_CUDA(launch_fista_prox_input(reinterpret_cast<const float2*>(a->u), reinterpret_cast<const float2*>(a->grad),
                                     (float)a->step, a->prox_complex, a->prox_in, a->n, (cudaStream_t)a->stream));
  });
}

odt_status odt_fista_update(const odt_fista_args* a) {
  return guarded([&] {
    check_fista_args(a, "odt_fista_update");
    ODT_CUDA(launch_fista_update(a->prox_out, a->prox_complex, (float)a->coef, (float)a->ri_bg,
                                 reinterpret_cast<float2*>(a->u), reinterpret_cast<float2*>(a->x),
                                 reinterpret_cast<float2*>(a->ri), a->n, (cudaStream_t)a->stream));
  });
}

odt_status odt_set_polarisation(odt_handle h, const float* radial, const float* perp,
                                const float* tangent, const uint8_t* kmask) {
  return guarded([&] {
    auto H = lookup(h);
    if (H->np != 3) raise(ODT_ERR_INVALID_ARGUMENT, "odt_set_polarisation: not a dyadic (pol = 3) handle");
    if (!radial || !perp || !tangent || !kmask)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_set_polarisation: NULL table");
    DeviceGuard dg(H->g.device);
    const long long n = H->nf();
    std::vector<float> tab((size_t)8 * n);
    std::copy(radial, radial + 2 * n, tab.begin());
    std::copy(perp, perp + 2 * n, tab.begin() + 2 * n);
    std::copy(tangent, tangent + 3 * n, tab.begin() + 4 * n);
    for (long long i = 0; i < n; ++i) tab[7 * n + i] = kmask[i] ? 1.f : 0.f;
    std::lock_guard<std::recursive_mutex> lk(g_device_mu);
    ODT_CUDA(cudaDeviceSynchronize());
    H->drop_graphs();
    if (!H->pol_tab) H->pol_tab = H->dalloc<float>(tab.size(), false);
    ODT_CUDA(cudaMemcpy(H->pol_tab, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice));
    H->have_pol = true;
  });
}

odt_status odt_solve(odt_handle h, const odt_solve_args* args) {
  return guarded([&] {
    auto H = lookup(h);
    if (!args) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve: NULL args");
    if (!H->pot[0].have) raise(ODT_ERR_NOT_READY, "odt_solve: call odt_set_potential first");
    const odt_solve_args& A = *args;
    if (A.n_ill < 0) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve: n_ill < 0");
    if (A.n_ill == 0) return;
    if (!A.fields_in) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve: fields_in is NULL");
    if (A.memory != ODT_MEM_HOST && A.memory != ODT_MEM_DEVICE)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve: memory must be ODT_MEM_HOST or ODT_MEM_DEVICE");
    const bool want_t = A.trans != nullptr, want_r = A.ref != nullptr;
    if (want_t && !H->ktrans) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve: created without kernel_trans");
    if (want_r && !H->kref) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve: created without kernel_ref");
    if (H->np == 3 && !H->have_pol)
      raise(ODT_ERR_NOT_READY, "odt_solve: a dyadic handle needs odt_set_polarisation first");
    DeviceGuard dg(H->g.device);
    const bool dev = A.memory == ODT_MEM_DEVICE;
    if (dev) {
      if (!is_device_ptr(A.fields_in) || (want_t && !is_device_ptr(A.trans)) ||
          (want_r && !is_device_ptr(A.ref)) || (A.field3d && !is_device_ptr(A.field3d)))
        raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve: ODT_MEM_DEVICE with a non-device pointer");
    }
    // device pointers: the caller's stream as given (NULL = legacy default stream)
    cudaStream_t s = dev ? (cudaStream_t)A.stream : H->own_stream;
    const int want_batch = std::min<int>(A.n_ill, auto_batch(*H));
    ensure_batch(*H, want_batch);
    const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind kout = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    // per illumination: npol planes of [F_x, F_y] in and out, np components of [ri] in 3D
    const long long nF = H->nf() * H->npol, nR = H->nri() * H->np;
    ODT_CUDA(cudaMemsetAsync(H->d_count, 0, sizeof(unsigned int), s));
    for (int b0 = 0; b0 < A.n_ill; b0 += H->batch) {
      const int nb = std::min(H->batch, A.n_ill - b0);
      ODT_CUDA(cudaMemcpyAsync(H->in2d, A.fields_in + (size_t)b0 * nF,
                               (size_t)nb * nF * sizeof(float2), kin, s));
      run_chunk_graph(*H, nb, s, want_t, want_r, 0, H->fout);
      ODT_CUDA(launch_count_nonfinite(H->fout, nR * nb, H->d_count, s));
      if (A.field3d)
        ODT_CUDA(cudaMemcpyAsync(A.field3d + (size_t)b0 * nR, H->fout,
                                 (size_t)nb * nR * sizeof(float2), kout, s));
      if (want_t)
        ODT_CUDA(cudaMemcpyAsync(A.trans + (size_t)b0 * nF, H->res_t,
                                 (size_t)nb * nF * sizeof(float2), kout, s));
      if (want_r)
        ODT_CUDA(cudaMemcpyAsync(A.ref + (size_t)b0 * nF, H->res_r,
                                 (size_t)nb * nF * sizeof(float2), kout, s));
      if (!dev) ODT_CUDA(cudaStreamSynchronize(s));
      H->collect(s);
    }
    if (dev) {
      ODT_CUDA(cudaEventRecord(H->done_ev, s));
      H->done_pending = true;
    }
    if (!dev) {
      check_fault(*H);
      unsigned int cnt = 0;
      ODT_CUDA(cudaMemcpy(&cnt, H->d_count, sizeof(cnt), cudaMemcpyDeviceToHost));
      if (cnt) raise(ODT_ERR_NUMERIC, "odt_solve: " + std::to_string(cnt) +
                                          " non-finite values in the 3D field (NaN/Inf input?)");
    }
  });
}

odt_status odt_solve_source(odt_handle h, const odt_source_args* args) {
  return guarded([&] {
    auto H = lookup(h);
    if (!args) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve_source: NULL args");
    if (!H->pot[0].have) raise(ODT_ERR_NOT_READY, "odt_solve_source: call odt_set_potential first");
    const odt_source_args& A = *args;
    if (A.n < 0) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve_source: n < 0");
    if (A.n == 0) return;
    if (!A.source || !A.field3d) raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve_source: NULL source or field3d");
    if (A.memory != ODT_MEM_HOST && A.memory != ODT_MEM_DEVICE)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve_source: memory must be ODT_MEM_HOST or ODT_MEM_DEVICE");
    if (H->np == 3 && !H->have_pol)
      raise(ODT_ERR_NOT_READY, "odt_solve_source: a dyadic handle needs odt_set_polarisation first");
    DeviceGuard dg(H->g.device);
    const bool dev = A.memory == ODT_MEM_DEVICE;
    if (dev && (!is_device_ptr(A.source) || !is_device_ptr(A.field3d)))
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_solve_source: ODT_MEM_DEVICE with a non-device pointer");
    cudaStream_t s = dev ? (cudaStream_t)A.stream : H->own_stream;
    ensure_batch(*H, std::min<int>(A.n, auto_batch(*H)));
    const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind kout = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const long long nR = H->nri() * H->np;   // complex values per source / field
    for (int b0 = 0; b0 < A.n; b0 += H->batch) {
      const int nb = std::min(H->batch, A.n - b0);
      ODT_CUDA(cudaMemcpyAsync(H->einc, A.source + (size_t)b0 * nR, (size_t)nb * nR * sizeof(float2), kin, s));
      run_chunk(*H, nb, s, false, false, 0, H->fout, true);
      ODT_CUDA(cudaMemcpyAsync(A.field3d + (size_t)b0 * nR, H->fout, (size_t)nb * nR * sizeof(float2), kout, s));
      if (!dev) ODT_CUDA(cudaStreamSynchronize(s));
      H->collect(s);
    }
    if (dev) {
      ODT_CUDA(cudaEventRecord(H->done_ev, s));
      H->done_pending = true;
    } else {
      check_fault(*H);
    }
  });
}

odt_status odt_gradient(odt_handle h, const odt_gradient_args* args) {
  return guarded([&] {
    auto H = lookup(h);
    if (!args) raise(ODT_ERR_INVALID_ARGUMENT, "odt_gradient: NULL args");
    const odt_gradient_args& A = *args;
    if (H->np == 3 && !H->have_pol)
      raise(ODT_ERR_NOT_READY, "odt_gradient: a dyadic handle needs odt_set_polarisation first");
    if (!H->pot[0].have || !H->pot[1].have)
      raise(ODT_ERR_NOT_READY, "odt_gradient: set the forward and the adjoint potential first");
    if (H->pot[0].tensor)
      raise(ODT_ERR_UNSUPPORTED, "odt_gradient: the gradient of an RI tensor is not supported");
    if (A.n_ill < 1 || !A.fields_in || !A.fields_meas || !A.grad || !A.err)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_gradient: NULL buffer or n_ill < 1");
    if (A.memory != ODT_MEM_HOST && A.memory != ODT_MEM_DEVICE)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_gradient: bad memory flag");
    if (!H->ktrans) raise(ODT_ERR_INVALID_ARGUMENT, "odt_gradient: created without kernel_trans");
    DeviceGuard dg(H->g.device);
    const bool dev = A.memory == ODT_MEM_DEVICE;
    if (dev && (!is_device_ptr(A.fields_in) || !is_device_ptr(A.fields_meas) ||
                !is_device_ptr(A.grad)))
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_gradient: ODT_MEM_DEVICE with a non-device pointer");
    cudaStream_t s = dev ? (cudaStream_t)A.stream : H->own_stream;
    ensure_batch(*H, std::min<int>(A.n_ill, auto_batch(*H)));
    // per illumination: npol planes of [F_x, F_y] in, np components of [ri] in 3D;
    // the gradient is the mean over components and illuminations (the
    // reference's mean(..., [4 5]) over [ri, pole_num, n_ill])
    const long long nF = H->nf() * H->npol, nR = H->nri();
    if (H->grad_batch != H->batch) {
      for (void** p : {(void**)&H->fout_adj, (void**)&H->grad_acc, (void**)&H->d_err}) {
        if (*p) {
          std::lock_guard<std::recursive_mutex> lk(g_device_mu);
          cudaFree(*p);
          auto& L = H->allocs;
          L.erase(std::remove(L.begin(), L.end(), *p), L.end());
          *p = nullptr;
        }
      }
      H->fout_adj = H->dalloc<float2>((size_t)nR * H->np * H->batch, false);
      H->grad_acc = H->dalloc<float2>((size_t)nR, false);
      H->d_err = H->dalloc<double>(1, false);
      H->grad_batch = H->batch;
    }
    const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    ODT_CUDA(cudaMemsetAsync(H->grad_acc, 0, nR * sizeof(float2), s));
    ODT_CUDA(cudaMemsetAsync(H->d_err, 0, sizeof(double), s));
    for (int b0 = 0; b0 < A.n_ill; b0 += H->batch) {
      const int nb = std::min(H->batch, A.n_ill - b0);
      ODT_CUDA(cudaMemcpyAsync(H->in2d, A.fields_in + (size_t)b0 * nF,
                               (size_t)nb * nF * sizeof(float2), kin, s));
      ODT_CUDA(cudaMemcpyAsync(H->out_r, A.fields_meas + (size_t)b0 * nF,
                               (size_t)nb * nF * sizeof(float2), kin, s));
      run_chunk_graph(*H, nb, s, true, false, 0, H->fout);        // E_3D, trans
      ODT_CUDA(launch_residual(H->res_t, H->out_r, H->in2d, nF * nb, H->d_err, s));
      run_chunk_graph(*H, nb, s, false, false, 1, H->fout_adj);   // adjoint 3D field
      ODT_CUDA(launch_grad_accumulate(H->fout, H->fout_adj, H->grad_acc, H->g.ri_size[0],
                                      H->g.ri_size[1], H->g.ri_size[2], nb * H->np, s));
      H->collect(s);
    }
    if (dev) {
      ODT_CUDA(launch_grad_finalize(H->grad_acc, reinterpret_cast<float2*>(A.grad), nR,
                                    (float)A.n_ill * H->np, s));
    } else {
      ODT_CUDA(launch_grad_finalize(H->grad_acc, H->fout_adj, nR, (float)A.n_ill * H->np, s));
      ODT_CUDA(cudaMemcpyAsync(A.grad, H->fout_adj, nR * sizeof(float2), cudaMemcpyDeviceToHost, s));
    }
    ODT_CUDA(cudaMemcpyAsync(A.err, H->d_err, sizeof(double), cudaMemcpyDeviceToHost, s));
    ODT_CUDA(cudaStreamSynchronize(s));
    check_fault(*H);
  });
}

}  // extern "C"

namespace {
// Asynchronous solves: one worker thread and a FIFO of jobs per handle that
// has had one submitted.  A job is a copy of the caller's odt_solve_args;
// the worker runs odt_solve on it and keeps the status and message until a
// poll or wait reports them.
struct Job {
  odt_solve_args args;
  bool done = false;
  odt_status status = ODT_OK;
  std::string message;
};

struct JobQueue {
  std::mutex mu;
  std::condition_variable cv;       // work arrived / stop
  std::condition_variable done_cv;  // a job finished
  std::deque<odt_ticket> pending;
  std::map<odt_ticket, std::shared_ptr<Job>> jobs;
  odt_ticket next = 1;
  bool stop = false;
  std::thread worker;
};

// The registry is never destroyed: a host that exits without odt_destroy
// leaves an idle worker blocked on its condition variable, which the process
// exit ends; destroying a joinable std::thread at exit would abort instead.
struct QueueRegistry {
  std::mutex mu;
  std::map<odt_handle, std::shared_ptr<JobQueue>> queues;
};
QueueRegistry& registry() {
  static QueueRegistry* r = new QueueRegistry();
  return *r;
}

void run_jobs(odt_handle h, JobQueue* q) {
  for (;;) {
    std::shared_ptr<Job> job;
    {
      std::unique_lock<std::mutex> lk(q->mu);
      q->cv.wait(lk, [&] { return q->stop || !q->pending.empty(); });
      if (q->pending.empty()) return;   // stop requested and nothing left
      job = q->jobs[q->pending.front()];
      q->pending.pop_front();
    }
    const odt_status st = odt_solve(h, &job->args);
    std::lock_guard<std::mutex> lk(q->mu);
    job->status = st;
    job->message = st == ODT_OK ? std::string() : std::string(odt_last_error());
    job->done = true;
    q->done_cv.notify_all();
  }
}

void drain_all_queues();

std::shared_ptr<JobQueue> queue_of(odt_handle h, bool create) {
  QueueRegistry& R = registry();
  std::lock_guard<std::mutex> lk(R.mu);
  auto it = R.queues.find(h);
  if (it != R.queues.end()) return it->second;
  if (!create) return nullptr;
  // registered after the handle table exists, so it runs before that table
  // is destroyed at exit
  static const bool at_exit = (std::atexit(drain_all_queues), true);
  (void)at_exit;
  auto q = std::make_shared<JobQueue>();
  q->worker = std::thread(run_jobs, h, q.get());
  R.queues[h] = q;
  return q;
}

void drain_queue(odt_handle h);

// at exit, before the handles are destroyed: let every queue finish its jobs
void drain_all_queues() {
  std::vector<odt_handle> hs;
  {
    QueueRegistry& R = registry();
    std::lock_guard<std::mutex> lk(R.mu);
    for (const auto& kv : R.queues) hs.push_back(kv.first);
  }
  for (odt_handle h : hs) drain_queue(h);
}

// stop the handle's worker after the jobs it holds (called by odt_destroy)
void drain_queue(odt_handle h) {
  std::shared_ptr<JobQueue> q;
  {
    QueueRegistry& R = registry();
    std::lock_guard<std::mutex> lk(R.mu);
    auto it = R.queues.find(h);
    if (it == R.queues.end()) return;
    q = it->second;
    R.queues.erase(it);
  }
  {
    std::lock_guard<std::mutex> lk(q->mu);
    q->stop = true;
  }
  q->cv.notify_all();
  if (q->worker.joinable()) q->worker.join();
}

// report a finished job to the calling thread and release it
odt_status take_job(JobQueue& q, odt_ticket t, odt_status* status) {
  auto it = q.jobs.find(t);
  const std::shared_ptr<Job> job = it->second;
  q.jobs.erase(it);
  if (status) *status = job->status;
  if (job->status != ODT_OK) set_last_error(job->message);
  return ODT_OK;
}
}  // namespace

extern "C" {

odt_status odt_submit(odt_handle h, const odt_solve_args* args, odt_ticket* ticket) {
  return guarded([&] {
    lookup(h);
    if (!args || !ticket) raise(ODT_ERR_INVALID_ARGUMENT, "odt_submit: NULL argument");
    auto q = queue_of(h, true);
    std::lock_guard<std::mutex> lk(q->mu);
    auto job = std::make_shared<Job>();
    job->args = *args;
    const odt_ticket t = q->next++;
    q->jobs[t] = job;
    q->pending.push_back(t);
    *ticket = t;
    q->cv.notify_one();
  });
}

odt_status odt_poll(odt_handle h, odt_ticket ticket, int32_t* done, odt_status* status) {
  odt_status st = ODT_OK;
  const odt_status g = guarded([&] {
    lookup(h);
    if (!done) raise(ODT_ERR_INVALID_ARGUMENT, "odt_poll: NULL done");
    auto q = queue_of(h, false);
    if (!q) raise(ODT_ERR_INVALID_ARGUMENT, "odt_poll: unknown ticket " + std::to_string(ticket));
    std::lock_guard<std::mutex> lk(q->mu);
    auto it = q->jobs.find(ticket);
    if (it == q->jobs.end()) raise(ODT_ERR_INVALID_ARGUMENT, "odt_poll: unknown ticket " + std::to_string(ticket));
    *done = it->second->done ? 1 : 0;
    if (*done) st = take_job(*q, ticket, status);
  });
  return g != ODT_OK ? g : st;
}

odt_status odt_wait(odt_handle h, odt_ticket ticket, odt_status* status) {
  odt_status st = ODT_OK;
  const odt_status g = guarded([&] {
    lookup(h);
    auto q = queue_of(h, false);
    if (!q) raise(ODT_ERR_INVALID_ARGUMENT, "odt_wait: unknown ticket " + std::to_string(ticket));
    std::unique_lock<std::mutex> lk(q->mu);
    if (q->jobs.find(ticket) == q->jobs.end())
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_wait: unknown ticket " + std::to_string(ticket));
    // a poll in another thread may release the ticket meanwhile
    q->done_cv.wait(lk, [&] {
      auto it = q->jobs.find(ticket);
      return it == q->jobs.end() || it->second->done;
    });
    if (q->jobs.find(ticket) == q->jobs.end())
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_wait: ticket " + std::to_string(ticket) + " released by another call");
    st = take_job(*q, ticket, status);
  });
  return g != ODT_OK ? g : st;
}

odt_status odt_budget(odt_handle h, int64_t* held_bytes, int64_t* budget_bytes) {
  return guarded([&] {
    auto H = lookup(h);
    if (held_bytes) *held_bytes = (int64_t)(H->static_bytes + H->batch_bytes);
    if (budget_bytes) *budget_bytes = (int64_t)H->budget;
  });
}

odt_status odt_destroy(odt_handle h) {
  drain_queue(h);   // queued solves finish first
  return guarded([&] {
    std::shared_ptr<Handle> H;
    {
      std::lock_guard<std::mutex> lk(g_mu);
      auto it = g_handles.find(h);
      if (it == g_handles.end()) raise(ODT_ERR_BAD_HANDLE, "unknown handle " + std::to_string(h));
      H = it->second;
      g_handles.erase(it);
    }
    DeviceGuard dg(H->g.device);
    cudaStreamSynchronize(H->own_stream);
    H.reset();
  });
}

odt_status odt_get_batch(odt_handle h, int32_t* batch) {
  return guarded([&] {
    auto H = lookup(h);
    if (!batch) raise(ODT_ERR_INVALID_ARGUMENT, "odt_get_batch: NULL");
    *batch = H->batch;
  });
}

namespace {
// process-wide plan choices of odt_autotune
struct TuneKey {
  int dev, px, py, pz, nb, np, storage;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, px, py, pz, nb, np, storage) < std::tie(o.dev, o.px, o.py, o.pz, o.nb, o.np, o.storage);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, odt_tune_result> g_tune;
}  // namespace

odt_status odt_autotune(odt_handle h, int32_t n_ill, odt_tune_result* out) {
  return guarded([&] {
    auto H = lookup(h);
    if (!out) raise(ODT_ERR_INVALID_ARGUMENT, "odt_autotune: NULL result");
    if (n_ill < 1) raise(ODT_ERR_INVALID_ARGUMENT, "odt_autotune: n_ill < 1");
    if (!H->pot[0].have) raise(ODT_ERR_NOT_READY, "odt_autotune: call odt_set_potential first");
    if (H->np == 3 && !H->have_pol) raise(ODT_ERR_NOT_READY, "odt_autotune: set the polarisation basis first");
    DeviceGuard dg(H->g.device);
    const int nb = std::min<int>(n_ill, auto_batch(*H));
    ensure_batch(*H, nb);
    const TuneKey key{H->g.device, H->g.sim_size[0], H->g.sim_size[1], H->g.sim_size[2], nb, H->np, H->storage};
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune.find(key);
      if (it != g_tune.end()) {
        *out = it->second;
        out->cached = 1;
        H->drop_graphs();
        H->use_xy = out->fused_xy != 0;
        H->use_pipe = out->pipelined != 0;
        return;
      }
    }
    // plane-wave inputs (ones) in the batch's input planes
    const size_t nin = (size_t)H->nf() * H->npol * nb;
    std::vector<float2> ones(nin, make_float2(1.f, 0.f));
    cudaStream_t s = H->own_stream;
    ODT_CUDA(cudaMemcpyAsync(H->in2d, ones.data(), nin * sizeof(float2), cudaMemcpyHostToDevice, s));
    BornArgs probe{};
    probe.px = H->g.sim_size[0];
    probe.py = H->g.sim_size[1];
    probe.pz = H->g.sim_size[2];
    probe.nbatch = nb * H->np;
    const bool xy_ok = H->np == 1 && !H->pot[0].tensor && born_xy_supported(probe, H->max_smem);
    const bool saved_xy = H->use_xy, saved_pipe = H->use_pipe;
    const bool want_t = H->ktrans != nullptr;
    cudaEvent_t e0, e1;
    ODT_CUDA(cudaEventCreate(&e0));
    ODT_CUDA(cudaEventCreate(&e1));
    odt_tune_result r{};
    r.batch = nb;
    int best = -1;
    const bool plan_xy[3] = {true, false, false}, plan_pipe[3] = {true, true, false};
    for (int c = 0; c < 3; ++c) {
      r.ms[c] = -1.0;
      if (c == 0 && !xy_ok) continue;
      if (H->storage == ODT_STORAGE_B16 && c != 0) continue;   // 16-bit storage runs on the fused pass only
      H->use_xy = plan_xy[c];
      H->use_pipe = plan_pipe[c];
      H->drop_graphs();
      try {
        run_chunk(*H, nb, s, want_t, false, 0, H->fout);   // warm-up (kernel attributes, caches)
        ODT_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < 2; ++k) run_chunk(*H, nb, s, want_t, false, 0, H->fout);
        ODT_CUDA(cudaEventRecord(e1, s));
        ODT_CUDA(cudaEventSynchronize(e1));
        check_fault(*H);
      } catch (const ApiError&) {   // a plan that cannot run here is skipped
        ODT_CUDA(cudaStreamSynchronize(s));
        continue;
      } catch (const CudaError&) {  // e.g. a launch that does not fit: the context is intact
        cudaGetLastError();
        ODT_CUDA(cudaStreamSynchronize(s));
        continue;
      }
      float ms = 0.f;
      ODT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      r.ms[c] = ms / 2.0;
      if (best < 0 || r.ms[c] < r.ms[best]) best = c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    H->drop_graphs();
    if (best < 0) {
      H->use_xy = saved_xy;
      H->use_pipe = saved_pipe;
      raise(ODT_ERR_UNSUPPORTED, "odt_autotune: no plan applies to this handle");
    }
    H->use_xy = plan_xy[best];
    H->use_pipe = plan_pipe[best];
    r.fused_xy = plan_xy[best] ? 1 : 0;
    r.pipelined = plan_pipe[best] ? 1 : 0;
    r.cached = 0;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune[key] = r;
    }
    *out = r;
  });
}

odt_status odt_set_field_storage(odt_handle h, int32_t storage) {
  return guarded([&] {
    auto H = lookup(h);
    if (storage != ODT_STORAGE_COMPLEX64 && storage != ODT_STORAGE_B16)
      raise(ODT_ERR_INVALID_ARGUMENT, "odt_set_field_storage: storage must be ODT_STORAGE_COMPLEX64 (0) "
                                      "or ODT_STORAGE_B16 (1), got " + std::to_string(storage));
    if (H->storage != storage) {
      DeviceGuard dg(H->g.device);
      H->drop_graphs();   // captured launches carry the storage layout
      H->storage = storage;
    }
  });
}

odt_status odt_set_profiling(odt_handle h, int32_t enable) {
  return guarded([&] {
    auto H = lookup(h);
    H->profiling = enable != 0;
    for (int i = 0; i < kNumKinds; ++i) {
      H->kind_ms[i] = 0;
      H->kind_launches[i] = 0;
    }
    H->ev_used = 0;
  });
}

odt_status odt_get_kernel_times(odt_handle h, const char** names, double* ms, int64_t* launches,
                                int32_t cap, int32_t* n) {
  return guarded([&] {
    auto H = lookup(h);
    if (!n) raise(ODT_ERR_INVALID_ARGUMENT, "odt_get_kernel_times: NULL count");
    DeviceGuard dg(H->g.device);
    H->collect(H->own_stream);
    *n = kNumKinds;
    for (int i = 0; i < kNumKinds && i < cap; ++i) {
      if (names) names[i] = kKindNames[i];
      if (ms) ms[i] = H->kind_ms[i];
      if (launches) launches[i] = H->kind_launches[i];
    }
  });
}

}  // extern "C"

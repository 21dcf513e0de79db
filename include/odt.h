/*
 * odt.h -- C ABI of the B200 convergent-Born-series (CBS) library (libodt).
 *
 * Drop-in replacement for the `CudaBorn` MEX of BMOLKAIST/Inverse_solver
 * (Codes/CUDA_CODE/main.cpp:27-213) and for the Born loop of the MATLAB class
 * FORWARD_SOLVER_CONVERGENT_BORN (Codes/FORWARD_SOLVER_CONVERGENT_BORN.m).
 * A MATLAB gateway, a Python ctypes binding or C++ code call these functions;
 * the host side keeps computing the geometry-dependent setup (Green's
 * kernels, pupil filters, potential) exactly as the MATLAB class does and the
 * library runs everything per illumination on the GPU.
 *
 * Conventions
 *  - All arrays are column-major (MATLAB order: first index fastest) and
 *    complex values are interleaved single precision (odt_cfloat), i.e. the
 *    MATLAB -R2018a interleaved-complex layout.
 *  - Every function returns an odt_status (0 = ODT_OK), never throws across
 *    the ABI and never exits; odt_last_error() describes the last failure of
 *    the calling thread.
 *  - A handle owns its device memory.  Calls on one handle must not overlap;
 *    different handles may be used from different threads (a mutex guards
 *    the handle table).
 */
#ifndef ODT_H_
#define ODT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ODT_ABI_VERSION 2

typedef enum odt_status {
  ODT_OK = 0,
  ODT_ERR_INVALID_ARGUMENT = 1, /* bad sizes, NULL where required, bad flags  */
  ODT_ERR_BAD_HANDLE = 2,       /* unknown or destroyed handle                */
  ODT_ERR_CUDA = 3,             /* a CUDA runtime call failed                 */
  ODT_ERR_OUT_OF_MEMORY = 4,    /* device allocation or memory budget exceeded */
  ODT_ERR_NOT_READY = 5,        /* odt_solve before odt_set_potential         */
  ODT_ERR_UNSUPPORTED = 6,      /* grid length with a prime factor > 31, ...  */
  ODT_ERR_NUMERIC = 7,          /* NaN/Inf in the inputs or the result        */
  ODT_ERR_INTERNAL = 8
} odt_status;

typedef struct odt_cfloat {
  float re;
  float im;
} odt_cfloat;

typedef uint32_t odt_handle; /* like CudaBorn's uint32 id; 0 is never valid */

/* Memory space of the pointers passed to odt_solve. */
#define ODT_MEM_HOST 0
#define ODT_MEM_DEVICE 1

/*
 * Geometry of one solver instance.  Mirrors the struct of CudaBorn action 0
 * (FORWARD_SOLVER_CONVERGENT_BORN_CUDA.m:23-32): simulation_size (padded
 * grid), RI_size, field_size, conv_size.
 */
typedef struct odt_geometry {
  int32_t sim_size[3];   /* padded grid P = RI_size + 2*boundary_thickness_pixel */
  int32_t ri_size[3];    /* RI grid (ROI inside the padded grid)                 */
  int32_t field_size[2]; /* 2D field (params.size(1:2)); must equal ri_size(1:2) */
  int32_t conv_size[2];  /* field_size + ri_size(1:2): 2D convolution plane, or
                            field_size when the xy boundary is cyclic          */
  int32_t device;        /* CUDA device ordinal (CudaBorn's used_gpu)            */
  int32_t max_batch;     /* illuminations resident on the device at once; 0=auto */
  int64_t mem_budget;    /* bytes this handle may allocate; 0 = half the free HBM */
  int32_t pol;           /* 0 or 1: scalar Green's function (pole_num = 1);
                            3: dyadic Green's function (vector_simulation,
                            pole_num = 3): input / output fields carry 2
                            polarisations, the 3D field 3 components
                            (FORWARD_SOLVER_CONVERGENT_BORN.m:293-296) */
} odt_geometry;

/*
 * Per-potential parameters.  Mirrors CudaBorn action 1
 * (FORWARD_SOLVER_CONVERGENT_BORN_CUDA.m:50-61: k0_nm, eps_imag, fourier_res,
 * ROI, Bornmax, dV) plus the separable tables the MATLAB class builds in
 * create_boundary_RI / init (FORWARD_SOLVER_CONVERGENT_BORN.m:251-271,
 * :299-377), passed as computed by the host so the float semantics are the
 * host's:
 *   mask[a]   : attenuation mask factor along axis a (length sim_size[a])
 *   ramp[a]   : phase-ramp factor along axis a (complex, length sim_size[a])
 *   kq2[a]    : squared shifted k-coordinate along axis a in FFT (ifftshifted)
 *               order, (fourier_coor + fourier_res/4)^2 (length sim_size[a])
 * The Green's function of iteration jj is evaluated on the fly as
 *   G = 1 / (green_scale * (kq2x + kq2y + kq2z) - green_offset - i*eps_imag)
 * with kq2 read at the frequency-negated index on odd jj when acyclic != 0
 * (fft_flip, FORWARD_SOLVER_CONVERGENT_BORN.m:579-585).
 */
typedef struct odt_potential_params {
  float eps_imag;       /* h.eps_imag                                         */
  float green_scale;    /* single(4*pi^2)                                     */
  float green_offset;   /* single((2*pi*k0_nm)^2)                             */
  float dV;             /* single(utility_border.dV)                          */
  int32_t roi[6];       /* h.ROI, 1-based inclusive [x0 x1 y0 y1 z0 z1]       */
  int32_t bornmax;      /* h.Bornmax (>= 0)                                   */
  int32_t acyclic;      /* params.acyclic                                     */
  const float* mask[3];
  const odt_cfloat* ramp[3];
  const float* kq2[3];
  /* dyadic handles (pol = 3) only: rads(:,:,:,a) = shifted k-coordinate / k0_nm
   * along axis a in FFT (ifftshifted) order (:316-319, :385), and the
   * absorptive correction (2 pi k0_nm)^2 / ((2 pi k0_nm)^2 + i eps_imag) of
   * the dyadic Green's function (:322) */
  const float* rad[3];
  odt_cfloat absorb;
} odt_potential_params;

/* Outputs of odt_solve; any pointer may be NULL to skip that output.  npol
 * = 1 for scalar handles, 2 for dyadic ones; ncomp = 1 or 3. */
typedef struct odt_solve_args {
  const odt_cfloat* fields_in; /* [F_x, F_y, npol, n_ill] spatial input fields */
  int32_t n_ill;
  odt_cfloat* trans;           /* [F_x, F_y, npol, n_ill] transmitted field    */
  odt_cfloat* ref;             /* [F_x, F_y, npol, n_ill] reflected field      */
  odt_cfloat* field3d;         /* [ri_x, ri_y, ri_z, ncomp, n_ill] 3D field    */
  int32_t memory;              /* ODT_MEM_HOST or ODT_MEM_DEVICE               */
  void* stream;                /* cudaStream_t for ODT_MEM_DEVICE (NULL = the
                                  legacy default stream); ignored for host   */
} odt_solve_args;

/*
 * Create a solver (CudaBorn action 0, main.cpp:57-101).
 *   refocus      : refocusing_util  [conv_x, conv_y, ri_z]
 *                  (FORWARD_SOLVER_CONVERGENT_BORN.m:80-92)
 *   kernel_trans : fft2(conj G)     [conv_x, conv_y, ri_z] (:114), may be NULL
 *   kernel_ref   : fft2(G)          [conv_x, conv_y, ri_z] (:115), may be NULL
 *   pupil_in     : [F_x, F_y] real, NA_circle and Abbe factor of
 *                  transform_field_3D (FORWARD_SOLVER.m:38-48)
 *   pupil_out    : [F_x, F_y] real, NA_circle*sqrt(cos_theta) of
 *                  transform_field_2D (FORWARD_SOLVER.m:69-77)
 */
odt_status odt_create(const odt_geometry* geom, const odt_cfloat* refocus,
                      const odt_cfloat* kernel_trans, const odt_cfloat* kernel_ref,
                      const float* pupil_in, const float* pupil_out, odt_handle* out);

/*
 * Polarisation basis of a dyadic handle (polarisation_utility,
 * FORWARD_SOLVER.m:131-180), per pixel of the [F_x, F_y] field spectrum:
 *   radial  [F_x, F_y, 2]  Radial_2D      perp    [F_x, F_y, 2]  Perp_2D
 *   tangent [F_x, F_y, 3]  ewald_TanVec   kmask   [F_x, F_y]     K_mask (0/1)
 * transform_field_3D (:38-68) maps the two input polarisations onto three
 * components with them, transform_field_2D (:69-97) maps back (the
 * reflection variant, :98-128, with the axial tangent component negated).
 * Required before odt_solve on a handle created with pol = 3.
 */
odt_status odt_set_polarisation(odt_handle h, const float* radial, const float* perp,
                                const float* tangent, const uint8_t* kmask);

/* Upload the scattering potential V = RI2potential(RI) - i*eps_imag on the
 * padded grid [sim_size] (CudaBorn action 1, main.cpp:102-138;
 * FORWARD_SOLVER_CONVERGENT_BORN.m:199-222). */
odt_status odt_set_potential(odt_handle h, const odt_potential_params* pp,
                             const odt_cfloat* V);

/*
 * Asynchronous solves for a host that serves requests (no counterpart in
 * the reference, whose MEX calls are synchronous): odt_submit queues an
 * odt_solve with these arguments on the handle's worker thread (created on
 * the first submit) and returns a ticket at once; the buffers the arguments
 * point to must stay valid and untouched until the ticket completes.  Jobs
 * of one handle run in submission order, concurrently with the calling
 * thread and with other handles' jobs.  odt_poll sets *done and, once the
 * job has finished, *status to the solve's own status (its message becomes
 * the polling thread's odt_last_error) and releases the ticket; odt_wait
 * blocks until then.  odt_destroy lets queued jobs finish first.
 * odt_budget: the bytes the handle holds on the device and its budget
 * (odt_geometry.mem_budget; 0 = none).
 */
typedef uint64_t odt_ticket;
odt_status odt_submit(odt_handle h, const odt_solve_args* args, odt_ticket* ticket);
odt_status odt_poll(odt_handle h, odt_ticket ticket, int32_t* done, odt_status* status);
odt_status odt_wait(odt_handle h, odt_ticket ticket, odt_status* status);
odt_status odt_budget(odt_handle h, int64_t* held_bytes, int64_t* budget_bytes);

/* Solve n_ill illuminations (CudaBorn action 4, main.cpp:175-210, plus the
 * MATLAB pre/post-processing of FORWARD_SOLVER_CONVERGENT_BORN.solve,
 * :397-520): fft2 + pupil_in, refocus into the volume, Born series, emitter
 * projection, + incident field, pupil_out, ifft2.  Synchronous for host
 * pointers; for device pointers the work is ordered on `stream` and the call
 * returns after enqueueing it. */
odt_status odt_solve(odt_handle h, const odt_solve_args* args);

/*
 * Adjoint potential for odt_gradient: the potential of conj(flip(RI, 3))
 * (BACKWARD_SOLVER_MULTI.m:48), same geometry and tables layout as
 * odt_set_potential.
 */
odt_status odt_set_adjoint_potential(odt_handle h, const odt_potential_params* pp,
                                     const odt_cfloat* V);

/*
 * Potential of an RI tensor (set_RI with size(RI,4) > 1,
 * FORWARD_SOLVER_CONVERGENT_BORN.m:180-219): V [sim_x, sim_y, sim_z, 3, 3]
 * column-major, V(:,:,:,i,j) = RI2potential of the padded tensor component
 * (i, j), minus 1i * eps_imag on the diagonal (:216-219); eps_imag =
 * 1.01 * max |potential| over all nine components.  Dyadic (pol = 3) handles
 * only; replaces the forward slot's potential until the next
 * odt_set_potential.  The x-pass then couples the three field components
 * voxel by voxel (:567-574, :588-594, :624-627), as does the emitter of the
 * transmitted / reflected fields (:451-455).  odt_gradient rejects it.
 */
odt_status odt_set_tensor_potential(odt_handle h, const odt_potential_params* pp, const odt_cfloat* V);

/*
 * Gradient of the transmitted-field misfit (BACKWARD_SOLVER_MULTI.m:30-54),
 * fused on the device: forward solve (potential of odt_set_potential) ->
 * diff = trans - fields_meas, err = sum |diff|^2 (accumulated in double) ->
 * adjoint solve of conj(diff) (potential of odt_set_adjoint_potential) ->
 * grad = -1i * mean(conj(E_3D) .* flip(conj(A_3D), 3), [4 5]).
 * On a dyadic (pol = 3) handle the fields carry two polarisations per
 * illumination and the mean runs over the three field components and the
 * illuminations, as the reference's mean over [pole_num, n_ill] does.
 * `err` is a host pointer in both memory modes.
 */
typedef struct odt_gradient_args {
  const odt_cfloat* fields_in;    /* [F_x, F_y, npol, n_ill] illuminations      */
  const odt_cfloat* fields_meas;  /* [F_x, F_y, npol, n_ill] measured trans.    */
  int32_t n_ill;
  odt_cfloat* grad;               /* [ri] output                                 */
  double* err;                    /* host scalar output                          */
  int32_t memory;                 /* ODT_MEM_HOST or ODT_MEM_DEVICE              */
  void* stream;
} odt_gradient_args;

odt_status odt_gradient(odt_handle h, const odt_gradient_args* args);

/*
 * Device-resident outer loop of BACKWARD_SOLVER_MULTI (BACKWARD_SOLVER_MULTI.m
 * :92-196 with set_RI, FORWARD_SOLVER_CONVERGENT_BORN.m:180-279, run on
 * gpuArrays as the reference does with use_GPU): the RI stays in device
 * memory between outer iterations.
 *
 * odt_potential_eps_device: eps_imag = single(1.01 * max|RI2potential(RI)|)
 *   (condition_RI, :199-222) of a device RI array [ri_x, ri_y, ri_z]
 *   (float or complex64); synchronous, the result is a host float.
 * odt_set_potential_device: the padded potential built on the device from the
 *   same RI (create_boundary_RI's zero-potential padding and RI2potential /
 *   potential2RI round trips, :223-279, then V - i eps_imag) into the forward
 *   slot, or with adjoint = 1 from conj(flip(RI, 3)) into the adjoint slot
 *   (BACKWARD_SOLVER_MULTI.m:48); `pp` carries the scalars and 1D tables as
 *   for odt_set_potential (its eps_imag is the one to subtract).  The device
 *   values agree with a host-built potential to a few units in the last
 *   place.
 */
typedef struct odt_ri_device_args {
  const void* ri;          /* device [ri_x, ri_y, ri_z], float or complex64   */
  int32_t is_complex;
  int32_t adjoint;         /* 1: conj(flip(RI, 3)) into the adjoint slot      */
  double wavelength;       /* params.wavelength                                */
  double ri_bg;            /* params.RI_bg                                     */
  void* stream;            /* cudaStream_t ordering the reads of `ri`          */
} odt_ri_device_args;

odt_status odt_potential_eps_device(odt_handle h, const odt_ri_device_args* args, float* eps_imag);
odt_status odt_set_potential_device(odt_handle h, const odt_potential_params* pp,
                                    const odt_ri_device_args* args);

/*
 * FISTA element-wise steps on device arrays of n elements
 * (BACKWARD_SOLVER_MULTI.m:150-160):
 *   odt_fista_prox_input: prox_in = u - step * grad (its real part when
 *     prox_complex = 0: the reference's TV prox keeps the real part when
 *     Vimag_max = 0);
 *   odt_fista_update: s = prox_out; u = s + coef (s - x); x = s;
 *     ri = ri_bg * sqrt(u + 1).
 * Ordered on `stream`; asynchronous.
 */
typedef struct odt_fista_args {
  int64_t n;
  const odt_cfloat* grad;  /* odt_gradient's output                             */
  odt_cfloat* u;           /* FISTA iterate u_n, complex64                      */
  odt_cfloat* x;           /* previous prox result x_n, complex64              */
  odt_cfloat* ri;          /* RI of the next gradient, complex64              */
  void* prox_in;           /* float (prox_complex = 0) or complex64            */
  const void* prox_out;
  int32_t prox_complex;
  double step;             /* 1 / alpha                                        */
  double coef;             /* (t_n - 1) / t_{n+1}                              */
  double ri_bg;
  void* stream;
} odt_fista_args;

odt_status odt_fista_prox_input(const odt_fista_args* args);
odt_status odt_fista_update(const odt_fista_args* args);

/*
 * The plane part of truncated_green_plus (sub_code/truncated_green_plus.m
 * :67-110) on the GPU: the band-limited radial profile [n_r, Nz] of the
 * xy-truncated Green's function (or refocusing kernel) interpolated onto the
 * oversized grid [S1, S2] per z with the host's bin_search_nearest maps
 * (:111-129), then the reference's centred inverse 2D FFT / crop to
 * out_size(1:2) / centred forward 2D FFT and the same along z, each chain
 * applied as the linear map the caller passes: m1 [out_size(1), S1],
 * m2 [out_size(2), S2], mz [out_size(3), Nz] (C_out * rows of C_S^-1, with C_n
 * the centred DFT matrix), so that out(:,:,k) = sum_z mz(k,z) m1 G_z m2^T
 * (three single-precision complex GEMMs; any lengths).  All arrays are host
 * memory; synchronous.  Scratch comes from the stream-ordered allocator.
 */
typedef struct odt_green_args {
  const odt_cfloat* radial;   /* [n_r, creation[2]]                           */
  int32_t n_r;
  const int32_t* near1;       /* [S1 * S2] 1-based bracketing profile samples  */
  const int32_t* near2;
  const float* w;             /* [S1 * S2] weight of near1                     */
  int32_t creation[3];        /* S1, S2, Nz of the oversized grid              */
  int32_t out_size[3];
  float scale;                /* Nz / (res_x * res_y)                          */
  const odt_cfloat* m1;       /* [out_size[0], S1]                             */
  const odt_cfloat* m2;       /* [out_size[1], S2]                             */
  const odt_cfloat* mz;       /* [out_size[2], Nz]                             */
  odt_cfloat* out;            /* [out_size]                                    */
  int32_t device;             /* CUDA device (-1: the current one)             */
} odt_green_args;

odt_status odt_green_planes(const odt_green_args* args);

/*
 * The cropped discrete Hankel transform pair of truncated_green_plus
 * (sub_code/truncated_green_plus.m:33-66 with
 * hankel_transform/discrete_hankel_croped_fourier.m:19-47, order 0, unit
 * radius) applied to a radial profile, on the GPU: with c_0 .. c_{n-1} the
 * first n positive zeros of J_0 and C the (n+1)-th (single precision, as the
 * reference rounds them), I_j = |J_1(c_j)|, the transform matrix
 *   F[i, j] = (s_i s_j) J_0((c_i / C) c_j),  s = sqrt(2 / C) / I,  i < pos,
 * is built on the device (the reference's besselj matrices, one
 * single-precision product per element as the reference forms them), and
 *   out = Rv .* (F^T ((band .* ((F (values ./ Rv)) .* K)) ./ K)),
 *   K = 2 pi I / C,  Rv = I,
 * the forward transform, the band-limiting window and the inverse transform
 * (:45-53), with double-precision accumulation of the two products.
 * values / out: [n, nz] complex (column-major), band: [pos]; roots: the
 * n + 1 zeros (double, host).  All arrays are host memory; synchronous.
 */
typedef struct odt_hankel_args {
  const double* roots;        /* [n + 1] positive zeros of J_0                 */
  int32_t n;                  /* samples                                       */
  int32_t pos;                /* rows of the low-k band kept (<= n)            */
  int32_t nz;                 /* profile columns                               */
  const odt_cfloat* values;   /* [n, nz]                                       */
  const float* band;          /* [pos]                                         */
  odt_cfloat* out;            /* [n, nz]                                       */
  int32_t device;             /* CUDA device (-1: the current one)             */
} odt_hankel_args;

odt_status odt_hankel_filter(const odt_hankel_args* args);

/*
 * Field retrieval from off-axis holograms, the transform part of get_fields
 * (FIELD_EXPERIMENTAL_RETRIEVAL.m:110-178): centred 2D FFT of each background
 * and sample hologram; the sideband = the first maximum of |F_bg(:,:,1)|
 * outside the deleted bands (rows round(N cutout):N, and columns
 * round(N cutout):N or, with other_corner, 1:round(N (1 - cutout))),
 * returned 1-based in sideband[2]; the spectra re-centred on it, cropped
 * (crop > 0: source rows / columns crop .. crop+M-1) or zero-padded
 * (crop < 0) to out_size M, times na_circle [M, M] (uint8, centred); for
 * each image the first maximum of |F_bg| and |F_bg| at its four neighbours
 * (peaks [7, n]: i1, i2 1-based, the peak, (i1-1,i2), (i1+1,i2), (i1,i2-1),
 * (i1,i2+1); 0 outside); and the centred inverse 2D FFTs cropped by two
 * pixels on every side into bg_field / sp_field [M-4, M-4, n].  sideband is
 * a host pointer in both memory modes.  Synchronous.
 */
typedef struct odt_hologram_args {
  int32_t size[3];          /* [N, N, n] hologram stacks                      */
  const float* bg;
  const float* sp;
  double cutout_portion;
  int32_t other_corner;
  int32_t out_size;         /* M                                              */
  int32_t crop;             /* crop size (> 0) or minus the padding (< 0)     */
  const uint8_t* na_circle; /* [M, M]                                         */
  odt_cfloat* bg_field;     /* [M-4, M-4, n]                                  */
  odt_cfloat* sp_field;
  float* peaks;             /* [7, n]                                         */
  int32_t* sideband;        /* [2], host                                      */
  int32_t memory;
  void* stream;
} odt_hologram_args;

odt_status odt_hologram_fields(const odt_hologram_args* args);

/* The per-pixel steps of get_fields after the transforms (:179-201), on
 * device arrays of n planes [size[0], size[1]], ordered on `stream`:
 * odt_hologram_phase: amean = sum |bg| / plane per image, bg and sp divided
 *   by it (and conjugated with conjugate = 1), phase = angle(sp ./ bg) and
 *   amp = abs(sp ./ bg) (float);
 * odt_hologram_combine: sp = amp .* bg .* exp(1i (phase - c0 - c1 x - c2 y))
 *   with coef [3, n] = (c0, c1, c2) per image (PhiShiftMS's ramp, x / y the
 *   1-based column / row). */
typedef struct odt_hologram_phase_args {
  int32_t size[3];
  odt_cfloat* bg;
  odt_cfloat* sp;
  int32_t conjugate;
  float* phase;
  float* amp;
  void* stream;
} odt_hologram_phase_args;

typedef struct odt_hologram_combine_args {
  int32_t size[3];
  const odt_cfloat* bg;
  const float* amp;
  const float* phase;
  const float* coef;
  odt_cfloat* sp;
  void* stream;
} odt_hologram_combine_args;

odt_status odt_hologram_phase(const odt_hologram_phase_args* args);
odt_status odt_hologram_combine(const odt_hologram_combine_args* args);

/* get_aberration_pattern (FIELD_EXPERIMENTAL_RETRIEVAL.m:216-352): the
 * stitched, phase-matched and low-passed pupil of the fields [N1, N2, n]
 * (n >= 2), the aberration pattern [N1, N2] and the corrected fields
 * ifft2c(fft2c(field) .* exp(-1i angle(pattern))).  k0s [2, n] are the
 * sub-pixel sideband positions of get_fields; pupil_mask is the reference's
 * fMask (coorxy < max(coorxy) * overlap_factor), na_circle and
 * refocusing_kernel the optical tool's; dist_list the defocus candidates.
 * The fields, the pattern and the corrected fields live where `memory`
 * says; the tables, k0s, dist_list and *chosen (the 0-based index of the
 * selected distance; may be NULL) on the host.  Synchronous on `stream`. */
typedef struct odt_aberration_args {
  int32_t size[3];
  const odt_cfloat* input_field;
  const odt_cfloat* output_field;
  const float* k0s;
  const uint8_t* pupil_mask;
  const uint8_t* na_circle;
  const odt_cfloat* refocusing_kernel;
  const double* dist_list;
  int32_t n_dist;
  odt_cfloat* pattern;
  odt_cfloat* input_out;
  odt_cfloat* output_out;
  int32_t* chosen;
  int32_t memory;
  void* stream;
} odt_aberration_args;

odt_status odt_aberration_pattern(const odt_aberration_args* args);

/* Centred 2D FFT, in place, of every [N1, N2] plane of data [N1, N2, n]:
 * fftshift(fft2(ifftshift(x))), or with inverse = 1 the inverse transform
 * (normalised by N1 N2), as correct_aberration (:356-370) applies it.
 * Synchronous on `stream`. */
typedef struct odt_fft2c_args {
  int32_t size[3];
  odt_cfloat* data;
  int32_t inverse;
  int32_t memory;
  void* stream;
} odt_fft2c_args;

odt_status odt_fft2c(const odt_fft2c_args* args);

/* remove_dirty_fields (FIELD_EXPERIMENTAL_RETRIEVAL.m:399-452) up to its
 * decision, for scalar fields bg, sp [N1, N2, n]: with the Goldstein-
 * unwrapped phase and the amplitude of sp ./ bg, per image the standard
 * deviation of the gradient energy of amp_k - amp_1 (gradient_std [n]) and
 * the number of phase values above 1.5 max(phase_1) or below
 * 1.5 min(phase_1) (outside_count [n]); both outputs on the host. */
typedef struct odt_field_quality_args {
  int32_t size[3];
  const odt_cfloat* bg;
  const odt_cfloat* sp;
  float* gradient_std;
  int64_t* outside_count;
  int32_t memory;
  void* stream;
} odt_field_quality_args;

odt_status odt_field_quality(const odt_field_quality_args* args);

/* refocus (FIELD_EXPERIMENTAL_RETRIEVAL.m:392-394): out = centred inverse 2D
 * FFT of (centred 2D FFT of each field plane .* kernel), kernel =
 * exp(z .* refocusing_kernel) [size(1), size(2)]; host arrays, synchronous. */
typedef struct odt_refocus_args {
  int32_t size[3];          /* [N1, N2, n]                                    */
  const odt_cfloat* field;
  const odt_cfloat* kernel;
  odt_cfloat* out;
} odt_refocus_args;

odt_status odt_refocus_2d(const odt_refocus_args* args);

/*
 * Beam-propagation forward solver (FORWARD_SOLVER_BPM.m:44-117), scalar
 * fields, all illuminations marched through the slices together.  The
 * tables are set_RI's (:23-44) and DERIVE_OPTICAL_TOOL's single-precision
 * arrays as the host computed them:
 *   field_multiplier [F_x, F_y, Nz]  1i 2 pi k0 (RI - RI_bg) res_z      (:33)
 *   refocus_kernel   [F_x, F_y]      ifftshift(exp(refocusing_kernel res_z) .* NA_circle) (:35)
 *   filter_out       [F_x, F_y]      ifftshift(NA_circle), real (:34); needed for field3d
 *   pre / post       [F_x, F_y]      exp(refocusing_kernel res_z (-floor(Nz/2)-1)) and
 *                                    exp(refocusing_kernel res_z (-(Nz-floor(Nz/2)-1))),
 *                                    centred (:94, :112)
 *   cos_theta        [F_x, F_y]      centred; NULL = cos_correction off (:58-63)
 * Outputs: trans [F_x, F_y, n_ill]; field3d [F_x, F_y, Nz, n_ill] or NULL.
 * Scratch comes from the stream-ordered allocator.  Synchronous for host
 * pointers; ordered on `stream` for device pointers.
 */
typedef struct odt_bpm_args {
  int32_t size[3];                    /* [F_x, F_y, Nz]                        */
  const odt_cfloat* field_multiplier;
  const odt_cfloat* refocus_kernel;
  const float* filter_out;
  const odt_cfloat* pre;
  const odt_cfloat* post;
  const float* cos_theta;
  const odt_cfloat* fields_in;        /* [F_x, F_y, n_ill] spatial fields       */
  int32_t n_ill;
  odt_cfloat* trans;
  odt_cfloat* field3d;
  int32_t memory;                     /* ODT_MEM_HOST or ODT_MEM_DEVICE         */
  void* stream;
} odt_bpm_args;

odt_status odt_bpm_solve(const odt_bpm_args* args);

/*
 * Isotropic-TV proximal operator by dual FISTA (sub_code/TV_FISTA_inner_v2.m
 * :1-53, called from BACKWARD_SOLVER_MULTI.m:152): `inner_itt` iterations on
 * a [size] array with periodic differences; projections onto
 * [vmin, vmax] (non_neg), imag >= 0 and imag <= vimag_max.  Real arrays
 * (is_complex = 0; the reference takes the real part when vimag_max == 0) or
 * complex64.  Scratch comes from the stream-ordered allocator.
 */
typedef struct odt_tv_args {
  int32_t size[3];
  const void* in;       /* float or complex64 [size]                         */
  void* out;            /* same type and size                                */
  int32_t is_complex;
  double lambda;        /* tv_param / alpha                                  */
  double vmin, vmax, vimag_max;
  int32_t non_neg, dirichlet, inner_itt;
  int32_t memory;
  void* stream;
} odt_tv_args;

odt_status odt_tv_prox(const odt_tv_args* args);

/*
 * Rytov reconstruction with Ewald-sphere mapping (BACKWARD_SOLVER_RYTOV.m:22-127)
 * and overlap counting (BACKWARD_SOLVER_RYTOV_precompute.m:87-137,
 * OVERLAP_COUNTER.m:19-23).  Scalar fields [size1, size2, n_ill]; the tables
 * are DERIVE_OPTICAL_TOOL's single-precision grids (fourier coor{1}, coor{2},
 * k3, NA_circle) as the host computed them.  `phase` is the unwrapped phase
 * of sp./bg (NULL with sp == NULL: overlap counting only).  count_one = 1
 * counts every Ewald hit (overlap counter); 0 counts hits with Uprime ~= 0
 * (Rytov).  Count and overlap_field are integer-valued single, bit-exact
 * with the reference's single-precision index arithmetic.  Any output may be
 * NULL.  `shifts` (host, 2*n_ill int32, may be NULL) receives the spectrum
 * shift (rows, cols) of each illumination.  Synchronous.
 */
typedef struct odt_rytov_args {
  int32_t size[3];
  double resolution[3];
  double fourier_res[3];
  double k0_nm, ri_bg, wavelength;
  const float* coor1;              /* [size1]                                */
  const float* coor2;              /* [size2]                                */
  const float* k3;                 /* [size1*size2]                          */
  const uint8_t* na_circle;        /* [size1*size2]                          */
  const uint8_t* emask;            /* [size1*size2] coorxy < 2 NA/lambda     */
  const odt_cfloat* bg;            /* [size1, size2, n_ill]                  */
  const odt_cfloat* sp;            /* same, or NULL                          */
  const float* phase;              /* same, or NULL                          */
  int32_t n_ill;
  int32_t count_one;
  int32_t non_negativity_iteration;
  odt_cfloat* RI;                  /* [size] outputs                          */
  odt_cfloat* ORytov;
  float* count;
  float* overlap_field;            /* [size1, size2, n_ill]                  */
  int32_t* shifts;
  int32_t memory;
  void* stream;
} odt_rytov_args;

odt_status odt_rytov(const odt_rytov_args* args);

/*
 * odt_unwrap_goldstein -- Goldstein branch-cut phase unwrapping of a stack of
 * 2D phase maps: the whole of unwrapp2_gpu.m (Codes/sub_code/goldstein_GPU/
 * unwrapp2_gpu.m:1-6), which replaces the chain of MEX calls
 *   get_residue_gpu          (get_residue_mex.cpp, get_residue_cuda.cu:34-66)
 *   remove_dipoles_gpu       (remove_dipoles_mex.cpp, remove_dipoles_cuda.cu:52-146)
 *   goldstein_branch_cut     (goldstein_branch_cut.m:1-100: create_sort_value_gpu,
 *                             get_lookup_gpu, get_shortest_sort_gpu,
 *                             get_branches_goldstein_v2, raster_branches_gpu)
 *   unwrapp_phase_goldstein_gpu (unwrapp_phase_goldstein_cuda.cu:62-157).
 * `phase_in` / `phase_out` are [size0, size1, size2] single, column-major
 * (size2 = number of maps, 1 for one map); phase_out may equal phase_in.
 * The optional outputs (NULL to skip) expose the intermediate products with
 * the reference's layouts:
 *   residue_out  [size0-1, size1-1, size2] single: residues after the dipole pass
 *   step1_out    [size0, size1, size2] int32: the 2*pi steps along dimension 1
 *   step2_out    [size1, size2] int32: the steps along dimension 2 of row 1
 *   table_out    [6, residue_cap] int32: sorted residue table (idx, value, box, x, y, z)
 *   nearest_out  [2, 8, residue_cap] int32: (row, distance) of the 8 nearest
 *   branches_out [6, branch_cap] int32: (x1, y1, x2, y2, z, jump)
 * n_residues / n_branches (host, optional) receive the counts; the tables are
 * written only up to their capacities.  `memory` says where phase_in,
 * phase_out and the optional arrays live; `link_threads` bounds the host
 * threads of the branch linker (0: one per hardware thread).  Requires
 * size0, size1 >= 2 and a total below 2^31 elements.
 */
typedef struct odt_unwrap_args {
  int32_t size[3];
  const float* phase_in;
  float* phase_out;
  float* residue_out;
  int32_t* step1_out;
  int32_t* step2_out;
  int32_t* table_out;
  int32_t* nearest_out;
  int64_t residue_cap;
  int32_t* branches_out;
  int64_t branch_cap;
  int64_t* n_residues;
  int64_t* n_branches;
  int32_t link_threads;
  int32_t memory;
  void* stream;
} odt_unwrap_args;

odt_status odt_unwrap_goldstein(const odt_unwrap_args* args);

/*
 * odt_solve_source -- CudaBorn's action 2 (CUDA_CODE/main.cpp:139-163:
 * set_source_3D, execute, get_field_3D): the Born series driven by a given
 * 3D incident field instead of a 2D input field.  source holds n incident
 * fields over the RI grid ([RI_x, RI_y, RI_z, n] complex, column-major;
 * [RI_x, RI_y, RI_z, 3, n] on dyadic handles), as the input stage of
 * odt_solve would form them (the refocused input, :543-554); field3d
 * receives Field(ROI) + the incident field, as odt_solve's field3d.  No
 * transmitted / reflected fields.  Memory / stream as odt_solve.
 */
typedef struct odt_source_args {
  const odt_cfloat* source;   /* [RI_x, RI_y, RI_z, (3,) n]                 */
  int32_t n;
  odt_cfloat* field3d;        /* [RI_x, RI_y, RI_z, (3,) n]                 */
  int32_t memory;             /* ODT_MEM_HOST or ODT_MEM_DEVICE            */
  void* stream;
} odt_source_args;

odt_status odt_solve_source(odt_handle h, const odt_source_args* args);

/* Free a solver (CudaBorn action 3, main.cpp:164-174). */
odt_status odt_destroy(odt_handle h);

/* Number of illuminations the handle keeps resident per batch. */
odt_status odt_get_batch(odt_handle h, int32_t* batch);

/* Storage of the Born loop's spectral array T and Field_n (no counterpart in
 * the reference, which computes in single precision throughout):
 *   ODT_STORAGE_COMPLEX64 (default) -- complex64, the reference's precision;
 *   ODT_STORAGE_B16 -- 16-bit block floating point: each block of 8 values
 *     shares a power-of-two exponent and every value keeps 15-bit int16
 *     mantissas for its real and imaginary parts.  Field (the running sum),
 *     V and all inputs and outputs stay complex64 and every operation still
 *     computes in FP32; only the two arrays that each iteration rewrites are
 *     stored narrower, so an iteration moves 48 instead of 72 bytes per voxel.
 *     The error against the FP64 result stays below 1e-4 relative L2 on the
 *     benchmark grid (the storage rounding of the early, largest Born terms
 *     dominates it, so every iteration uses the same format).
 * B16 needs the fused xy-pass: a scalar potential on a grid whose x and y
 * lengths are equal and 8 * R with 11 <= R <= 20 (z: 8 * R, 11 <= R <= 20, or 8 * {25, 27});
 * a solve on another grid fails with ODT_ERR_UNSUPPORTED.  Not to be called
 * while a solve on the same handle runs. */
#define ODT_STORAGE_COMPLEX64 0
#define ODT_STORAGE_B16 1
odt_status odt_set_field_storage(odt_handle h, int32_t storage);

/* Plan autotuning (no counterpart in the reference): times one solve of
 * n_ill plane waves (capped at the handle's batch) with each execution plan
 * that applies to the handle -- the fused xy-pass with the pipelined z-pass,
 * the separate pipelined x-, y-, z-passes, the generic tile kernels -- on
 * the potential set last, keeps the fastest for the handle's later solves
 * and caches the choice process-wide per (device, padded grid, batch,
 * components, storage), so a later handle of the same shape takes it without
 * timing.  The plans give the same results up to the order of the FFT
 * arithmetic.  ms[i] is the time per solve of plan i (0: fused xy-pass, 1:
 * separate pipelined passes, 2: generic tile kernels; -1 where a plan does
 * not apply or was not timed).  Needs odt_set_potential first; synchronous. */
typedef struct odt_tune_result {
  int32_t fused_xy;    /* chosen: 1 fused xy-pass                              */
  int32_t pipelined;   /* chosen: 1 pipelined kernels, 0 generic tile kernels   */
  int32_t batch;       /* illuminations per launch of the timed solves          */
  int32_t cached;      /* 1: the choice came from the cache (nothing timed)     */
  double ms[3];
} odt_tune_result;
odt_status odt_autotune(odt_handle h, int32_t n_ill, odt_tune_result* out);

/* Per-kernel timing (CUDA events around every launch on the solve stream).
 * When enabled, odt_get_kernel_times fills up to `cap` entries of names
 * (static strings), accumulated milliseconds and launch counts since the
 * last reset, and returns the number of kernel kinds in *n. */
odt_status odt_set_profiling(odt_handle h, int32_t enable);
odt_status odt_get_kernel_times(odt_handle h, const char** names, double* ms,
                                int64_t* launches, int32_t cap, int32_t* n);

/*
 * odt_born_series_noalloc -- no counterpart in the reference.
 *
 * The Born-series loop of odt_solve for ONE illumination (the part between
 * the incident field and Field(ROI) + incident field), for callers that must
 * not have the library allocate GPU memory: a host framework that owns the
 * device memory (MATLAB's gpuArray manager, PyTorch's caching allocator) can
 * see a hidden cudaMalloc fail against its pool or stall every stream on the
 * device, and a latency-bound request loop must not enter the driver's
 * allocator mid-request.  This entry point calls no cudaMalloc / cudaFree and
 * no allocating library routine: every input and output is a caller-owned
 * device pointer, and the loop's scratch (the spectral array, Field_n, Field
 * and the FFT twiddles: 3 * prod(sim_size) + sum(sim_size) complex64) lives in
 * one fixed 64 MiB array that every GPU which loads the library holds until
 * the process exits.  Grids needing more (more than about 2.79 million padded
 * voxels, e.g. 152^3) are rejected with ODT_ERR_OUT_OF_MEMORY.  Each padded
 * length must factor into radices up to 31, as for odt_solve (e.g. 145 =
 * 5 * 29 is accepted); other lengths are rejected with ODT_ERR_UNSUPPORTED.
 *
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream capture;
 * the address is kept for the life of the process, so do not call this entry
 * point on a device after cudaDeviceReset.  The FFT twiddle tables are copied
 * into the array from host memory on the first call for a grid size and
 * reused by later calls on the same size.  All calls share the one array and
 * it keeps the last call's contents (each call writes every scratch element
 * before reading it, so nothing needs clearing); calls that overlap on the
 * GPU -- two host threads, or work on two streams -- race on it.  The call
 * returns after the work on `stream` has finished.  Inputs are those odt_set_potential takes (V, the 1D tables,
 * the scalars), plus the incident field inside the ROI; `fout` receives
 * Field(ROI) + incident field, as field3d of odt_solve does.
 */
typedef struct odt_noalloc_born_args {
  int32_t sim_size[3];        /* padded grid                                  */
  int32_t roi[6];             /* 1-based inclusive, as odt_potential_params   */
  int32_t bornmax;
  int32_t acyclic;
  float eps_imag;
  float green_scale;
  float green_offset;
  const float* mask[3];       /* device; length sim_size[a]                   */
  const odt_cfloat* ramp[3];  /* device; ones when acyclic == 0               */
  const float* kq2[3];        /* device                                       */
  const odt_cfloat* V;        /* device [sim_size]                            */
  const odt_cfloat* einc;     /* device [roi extents] incident field          */
  odt_cfloat* fout;           /* device [roi extents] result                  */
  void* stream;               /* cudaStream_t (NULL = legacy default stream)  */
} odt_noalloc_born_args;

odt_status odt_born_series_noalloc(const odt_noalloc_born_args* args);

/* Last error message of the calling thread ("" if none). */
const char* odt_last_error(void);

/* ODT_ABI_VERSION of the loaded library. */
int32_t odt_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ODT_H_ */

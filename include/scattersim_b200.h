/*
 * scattersim_b200 -- C ABI of the B200-native coupled-wave (RCWA) layer solve
 * and field evaluation.
 *
 * Every entry point returns an sc_status; none exits, traps or prints.  The
 * message of the last failure on the calling thread is sc_last_error_string().
 * Device pointers are plain CUDA device addresses; `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).  Complex128 buffers hold
 * interleaved {re, im} doubles; matrices are column-major (the layout of
 * Eigen::MatrixXcd and of the reference's LAPACK calls).
 *
 * Reference interfaces replaced (STIM-Lab/scattersim):
 *   sc_fft2_crop            fftw_fft2 + fftShift2d           FourierWave.h:82-195, called at :341,:343
 *   sc_phi                  volume::phi                      FourierWave.h:336-397
 *   sc_eigensolve_batched   MKL_eigensolve (zgeev 'N','V')   third_Lapack.h:37-44
 *   sc_linearsolve_batched  MKL_linearsolve (zgesv, 1 RHS)   third_Lapack.h:46-53
 *   sc_inverse_batched      MKL_inverse (zgesv against I)    third_Lapack.h:55-63
 *   sc_zgemm_batched        MKL_multiply (cblas_zgemm)       third_Lapack.h:74-84
 *   sc_volume_plan/solve    scattervolume main()             ScatterVolume.cpp:506-902
 *   sc_volume_waves         CoupledWaveStructure build +     ScatterVolume.cpp:907-987,
 *                           cw_allocate / cw_unpack          cpuEvaluator.cpp:34-102
 *   sc_cw_evaluate          gpu_cw_evaluate / evaluate       gpuEvaluator.cu:28-165
 *   sc_mkl_eigensolve       host-buffer MKL_eigensolve       third_Lapack.h:37-44
 *   sc_beam_polar           planewave::SolidAnglePolar       ScatterLayer.cpp:355-385, ScatterPlane.cpp:154-171,236-242
 *   sc_layer_solve          scatterlayer / scatterplane      ScatterLayer.cpp:110-266,390-420,
 *                           per-wave solves                  ScatterPlane.cpp:175,243-256
 *   sc_gpu_initialize /
 *   sc_gpu_cw_evaluate      host-buffer gpu_initialize /     gpuEvaluator.cu:15-26,131-165
 *                           gpu_cw_evaluate
 *   sc_scatterio_write/read write_file / read_file           ScatterIO.h:18-117
 *   sc_cw_write             CoupledWaveStructure::save       CoupledWaveStructure.h:63-125
 */
#ifndef SCATTERSIM_B200_H
#define SCATTERSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SC_OK = 0,
    SC_BADINPUT = 1,     /* invalid sizes, null pointers, non-finite input   */
    SC_NOCONVERGE = 2,   /* QR iteration cap reached (per-instance info > 0) */
    SC_SINGULAR = 3,     /* exact zero pivot in an LU factorisation          */
    SC_OOM = 4,          /* device allocation failed                          */
    SC_CUDA_ERROR = 5,   /* a CUDA runtime call failed                        */
    SC_ENERGY_FAIL = 6   /* energy-balance check failed                       */
} sc_status;

typedef struct sc_context sc_context;

const char* sc_version(void);
const char* sc_last_error_string(void);

/* One context per GPU; owns pooled device workspace (no per-call cudaMalloc
 * once warm).  Replaces the process-global state of ScatterVolume.cpp:29-95. */
sc_status sc_create(sc_context** ctx, int device);
sc_status sc_destroy(sc_context* ctx);
/* Number of kernel launches this context issued since creation. */
uint64_t sc_launch_count(const sc_context* ctx);

/* ---------------------------------------------------------------- stages */

/* a3: for each of Z slices, the Fourier coefficients of n^2 and (1/n)^2
 * (forward DFT / (S1*S2), fftshift, centred My x Mx crop).  `sample` is the
 * C-order (Z, S1, S2) complex128 .npy buffer, read with the reference's
 * column-major reinterpretation (FourierWave.h:283-301).  Nf, Nif: Z blocks of
 * My x Mx column-major complex128. */
sc_status sc_fft2_crop(sc_context* ctx, const void* sample, int Z, int S1, int S2,
                       int Mx, int My, void* Nf, void* Nif, void* stream);

/* a5: dense 4M x 4M layer matrices Phi (column-major) for Z slices from their
 * coefficients.  up (Mx) and wq (My) are the lattice wave numbers of
 * volume::UpWq_Cal; k is the vacuum wave number. */
sc_status sc_phi(sc_context* ctx, const void* Nf, const void* Nif, int Z, int Mx, int My,
                 const double* up_host, const double* wq_host, double k, void* Phi, void* stream);

/* a7: eigenvalues and right eigenvectors (unit 2-norm columns) of `batch`
 * n x n complex matrices stored back to back.  A is overwritten.  info[b] = 0
 * on success, > 0 when the QR iteration cap was reached. */
sc_status sc_eigensolve_batched(sc_context* ctx, void* A, int n, int batch, void* evl,
                                void* evt, int* info, void* stream);

/* a13: solves A X = B (LU with partial pivoting) for `batch` systems; A is
 * overwritten by its LU factors, B by X.  info[b] = j+1 for an exact zero
 * pivot in column j. */
sc_status sc_linearsolve_batched(sc_context* ctx, void* A, int n, void* B, int nrhs,
                                 int batch, int* info, void* stream);

/* Allocation-free variant of sc_linearsolve_batched (no counterpart in the
 * reference).  Same arguments and results, no context, and no device memory
 * allocated: for callers that cannot call cudaMalloc -- real-time loops that
 * must not take the implicit device-wide synchronisation of cudaMalloc and
 * cudaFree, and host programs whose framework reserves the GPU's memory up
 * front and forbids later allocations (a late cudaMalloc would stall other
 * work or run out of memory mid-run).  Its scratch (pivots and status words)
 * is a fixed 260 KiB array in the library's device memory, held by every GPU
 * that loads the library until exit; limits: n * batch <= 65536 and
 * batch <= 1024, larger sizes return SC_BADINPUT.  It runs on the current
 * device; a stream of another device returns SC_BADINPUT.  The first call on
 * a device looks the array's device address up for that device and keeps it
 * (make that call before any stream capture, and none after cudaDeviceReset).
 * Like the allocating entry, each call copies the status words back into the
 * host array info and synchronises the stream -- except while the stream is
 * capturing into a CUDA graph: the call then only records the solve's kernels
 * (make one uncaptured call with the same n and batch on the device first),
 * leaves info untouched and returns SC_OK, and every replay of the graph
 * solves again.  All calls share the array: calls whose work overlaps on the
 * GPU race. */
sc_status sc_linearsolve_batched_noalloc(void* A, int n, void* B, int nrhs, int batch, int* info,
                                         void* stream);

/* a9/a12/a14: Ainv = A^-1 for `batch` matrices (A is not modified). */
sc_status sc_inverse_batched(sc_context* ctx, const void* A, int n, int batch, void* Ainv,
                             int* info, void* stream);

/* C = alpha * A * B + beta * C, column-major, strided batch. */
sc_status sc_zgemm_batched(sc_context* ctx, int m, int n, int k, const double* alpha,
                           const void* A, int lda, long long strideA, const void* B, int ldb,
                           long long strideB, const double* beta, void* C, int ldc,
                           long long strideC, int batch, void* stream);

/* The product of sc_zgemm_batched on the int8 tensor cores (tcgen05): each
 * operand is cut into `slices` signed 7-bit digits (1..7) under power-of-two
 * row (A) and column (B) scales, digit products are summed exactly in int32
 * and recombined in FP64; the error is about (slices + 1) 2^-7*slices times
 * the row scale x column scale x k per element.  No reference counterpart: it
 * is the arithmetic of the mixed-precision sweep.  Synchronises the stream;
 * SC_CUDA_ERROR if a tensor-core pipeline wait timed out. */
sc_status sc_zgemm_emulated_batched(sc_context* ctx, int slices, int m, int n, int k, const double* alpha,
                                    const void* A, int lda, long long strideA, const void* B, int ldb,
                                    long long strideB, const double* beta, void* C, int ldc,
                                    long long strideC, int batch, void* stream);

/* The product of sc_zgemm_batched on the int8 tensor cores (tcgen05) by
 * modular arithmetic: the operands, scaled per row (A) and column (B) by
 * powers of two and rounded to integers of about 47 bits, are reduced modulo
 * 14 pairwise coprime moduli (<= 255); one exact int8 product per modulus,
 * and the integer result is rebuilt in FP64 by the Chinese remainder theorem.
 * Error about 2^-47 times the row scale x column scale x k per element for
 * k <= 1250 (one bit less per doubling of k beyond).  No reference
 * counterpart: it is the arithmetic of the mixed-precision sweep (14 int8
 * products where the digit-sliced form needs 28).  Synchronises the stream;
 * SC_CUDA_ERROR if a tensor-core pipeline wait timed out. */
sc_status sc_zgemm_crt_batched(sc_context* ctx, int m, int n, int k, const double* alpha, const void* A, int lda,
                               long long strideA, const void* B, int ldb, long long strideB, const double* beta,
                               void* C, int ldc, long long strideC, int batch, void* stream);
/* Output tiles of the modular engine's MMA kernel, for this context: 0 (the
 * default) = 128 x 256 tiles on one CTA, 1 = 256 x 256 tiles on clusters of
 * two CTAs (tcgen05 cta_group::2).  Both give bit-identical results. */
sc_status sc_crt_tiles_set(sc_context* ctx, int mode);

/* --------------------------------------------------------- volume solve */

typedef struct {
    double lambda;          /* --lambda     (default 1.0)        */
    double direction[3];    /* --direction  (default 0 0 1)      */
    double ex[2];           /* --ex         (default 0 0)        */
    double ey[2];           /* --ey         (default 1 0)        */
    double ez[2];           /* --ez         (default 0 0)        */
    double n[2];            /* --n          (default 1 1)        */
    double kappa;           /* --kappa      (default 0)          */
    double size[3];         /* --size       (default 10 10 2)    */
    double z;               /* --z          (default 0)          */
    int ncoef;              /* number of --coef values (0, 1, 2) */
    int coef[2];            /* --coef                            */
    int psf;                /* --psf                             */
    int external;           /* --external                        */
    int npz;                /* --npz                             */
} sc_volume_params;

typedef struct {
    int Mx, My, MF;         /* orders after the clamps of ScatterVolume.cpp:599-651 */
    int Z;                  /* layers (slices)                                       */
    int clamped;            /* 1 if the evanescent-order clamp fired                 */
    double k;               /* 2 PI / lambda with PI = 3.141592653                   */
    double dir[3];          /* normalised direction * n_top                          */
    double e_re[3], e_im[3];/* orthogonalised incident polarisation                  */
} sc_volume_dims;

/* Fills the defaults of ScatterVolume.cpp:511-529. */
void sc_volume_params_default(sc_volume_params* p);

/* Geometry, polarisation and order selection for a (Z, S1, S2) sample. */
sc_status sc_volume_plan(const sc_volume_params* p, int Z, int S1, int S2, sc_volume_dims* dims);

/* The scattervolume solve (ScatterVolume.cpp:654-902) for one sample resident
 * on the device.  Outputs (device, any may be NULL):
 *   x      6*MF complex128: [R_x R_y R_z T_x T_y T_z], column-major order index
 *   evl    Z * 4*MF eigenvalues, even slots forward (downward) modes, odd the
 *          paired backward modes
 *   Qc, Qh Z blocks of 3*MF x 2*MF (column-major) internal mode fields
 *          (Ex, Ey, Ez rows) of the forward / backward modes, scaled by the
 *          mode coefficients beta (ScatterVolume.cpp:823-889)
 * info (host, may be NULL) receives the first nonzero per-layer status. */
sc_status sc_volume_solve(sc_context* ctx, const sc_volume_params* p, const void* sample,
                          int Z, int S1, int S2, void* x, void* evl, void* Qc, void* Qh,
                          int* info, void* stream);

/* One rank's share of a volume solve split by layers over several GPUs
 * (contiguous layer blocks, one exchange, ScatterVolume.cpp:282-336): for
 * layers [layer_begin, layer_end) of the (Z, S1, S2) sample (the whole
 * sample is passed; only the block's slices are read), the ordered product of
 * the block's transfer matrices
 *     P = T_{end-1} ... T_{begin},  T_i = GC_i GD_i^-1,
 * in which the block starting at layer 0 has GC_0 in place of T_0, as one
 * 4MF x 4MF column-major matrix.  The blocks' products, multiplied in layer
 * order (P_last ... P_1 P_0), are Gc_static of ScatterVolume.cpp:326-335.
 * GD0 (may be NULL; only for the block starting at layer 0) receives GD_0.
 * info (host, may be NULL): first nonzero per-layer eigensolve status. */
sc_status sc_volume_chain_block(sc_context* ctx, const sc_volume_params* p, const void* sample, int Z, int S1,
                                int S2, int layer_begin, int layer_end, void* P, void* GD0, int* info, void* stream);

/* The boundary system and its solve (ScatterVolume.cpp:339-466, 739) from
 * the whole chain Gc_static and GD_0 (4MF x 4MF each, device): x = [R; T]
 * (6 MF complex128), as sc_volume_solve with --external writes it. */
sc_status sc_volume_boundary_solve(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2,
                                   const void* Gc_static, const void* GD0, void* x, int* info, void* stream);

/* Precision of sc_sweep_solve.  SC_SWEEP_FP64 runs every product on the FP64
 * tensor pipe.  SC_SWEEP_MIXED lets the layer-factor and chain products run
 * on the int8 tensor cores with 7 digit slices per operand
 * (sc_zgemm_emulated_batched; about 1e-13 relative per product) wherever the
 * context's GEMM autotuner measured that faster than the FP64 tile, which on
 * the sweep workload keeps R/T within 2e-9 of FP64; the candidates are the
 * digit-sliced engine (7 slices) and the modular engine of
 * sc_zgemm_crt_batched.  SC_SWEEP_CRT runs every such product on the modular
 * engine; SC_SWEEP_SLICES(s) every such product on the digit-sliced engine
 * with s = 1..7 slices.  FFT, assembly,
 * the boundary systems and their LU stay in FP64. */
#define SC_SWEEP_FP64 0
#define SC_SWEEP_MIXED 1
#define SC_SWEEP_CRT 2
#define SC_SWEEP_SLICES(s) (0x100 | (s))

/* A batched sweep of independent scattervolume solves, R/T only (the
 * --external result, ScatterVolume.cpp:739), in place of one scattervolume
 * process per sweep point (videomaker.py:61-74, spectroscopy.py:66-91).
 * Host arrays of length count: params, samples (device pointers to (Z, S1, S2)
 * complex128 index volumes), Z, S1, S2, x (device pointers to 6*MF complex128
 * outputs, MF from sc_volume_plan) and status (per-instance sc_status,
 * written).  Instances may differ in wavelength, direction, size, layer count
 * and orders.  Returns SC_OK when every instance succeeded, else the first
 * failing status. */
sc_status sc_sweep_solve(sc_context* ctx, int count, const sc_volume_params* params,
                         const void* const* samples, const int* Z, const int* S1, const int* S2,
                         void* const* x, int precision, int* status, void* stream);

/* Precision of the products in later sc_volume_solve calls on this context,
 * with the codes of sc_sweep_solve: SC_SWEEP_FP64 (the default: the
 * reference's FP64 arithmetic), SC_SWEEP_MIXED or SC_SWEEP_SLICES(s) for the
 * transfer-chain, boundary-block and Pz products on the int8 tensor cores.
 * The FFT, the assembly, Omega = B C, the eigensolve, the eigenvectors and all
 * LU factorisations stay FP64.  No reference counterpart. */
sc_status sc_volume_precision(sc_context* ctx, int precision);

/* Device milliseconds of the last sc_volume_solve on this context:
 * [fft, assemble, eig, chain, boundary, interior, qr-kernel, total];
 * after sc_sweep_solve: [fft, assemble, layer factors, chain, boundary, -, -, total]. */
sc_status sc_volume_stage_ms(const sc_context* ctx, double* ms8);

/* QR statistics per matrix of the last eigensolve on this context, 8 values
 * each: multishift sweeps, then SM cycles spent on shifts, bulge chase,
 * far-right updates, far-row/Schur-vector updates, small blocks, (unused),
 * total.  Zero-filled beyond the last batch. */
sc_status sc_qr_stats(sc_context* ctx, long long* out, int count);

/* Per-launch device timing of the GEMM kernels that the sweep's engine runs
 * (CUDA events on the launching stream).  sc_kernel_timing(ctx, 1) clears the
 * record and starts timing, 0 stops it; sc_kernel_stats synchronises the
 * device and sums the record into out[8] = {launches, ms, FP64-equivalent
 * flops, 0} for the FP64 tensor-pipe tiles, then {launches, ms,
 * FP64-equivalent flops, int8 ops} for the int8 tcgen05 MMA kernel. */
sc_status sc_kernel_timing(sc_context* ctx, int on);
sc_status sc_kernel_stats(sc_context* ctx, double* out8);
/* The same record for `classes` kernel classes, 4 values each: 0 FP64 tiles,
 * 1 digit-sliced int8 MMA kernel, 2 modular (CRT) int8 MMA kernel, 3 whole
 * modular-engine products (exponents, packing, MMA kernel and reconstruction). */
sc_status sc_kernel_stats_ex(sc_context* ctx, double* out, int classes);

/* The GEMM autotuner's choices on this context, as 6-int records (m, n, k,
 * batch, slices, variant: 0/1 FP64 tile of 64/128 rows, 2 digit-sliced int8
 * engine, 3 modular int8 engine).
 * sc_gemm_choices_get writes up to cap records and returns their count in
 * *count; sc_gemm_choices_set replaces the table, so that a later run (a
 * profiler replay, say) makes the same choices without timing them again. */
sc_status sc_gemm_choices_get(sc_context* ctx, int* rec, int cap, int* count);
sc_status sc_gemm_choices_set(sc_context* ctx, const int* rec, int count);

/* Measured FP64 FMA throughput of this device (TFLOP/s): the roofline
 * denominator of the FP64 kernels. */
sc_status sc_fp64_peak_probe(sc_context* ctx, double* tflops);
/* Measured FP64 tensor-core (mma.sync m8n8k4 f64) throughput (TFLOP/s). */
sc_status sc_fp64_dmma_probe(sc_context* ctx, double* tflops);
/* Measured int8 tensor-core (tcgen05.mma kind::i8, 128 x 256 x 32, operands in
 * shared memory) throughput (TOPS): a roofline denominator of the int8 engines. */
sc_status sc_int8_peak_probe(sc_context* ctx, double* tops);

/* Wave table of a solved volume in cw_unpack order: Pi, then per boundary l
 * its reflected and transmitted lists (ScatterVolume.cpp:907-987,
 * cpuEvaluator.cpp:61-102), each wave wound to the origin.  E0 and k are
 * nw x 3 complex128 (row-major).  ez_mode 0 keeps the solver's E_z (Pz);
 * ez_mode 1 rebuilds E_z by transversality, as a .cw reader does.  Call with
 * E0 = k = NULL to obtain *nw, the region index begin/end (Z+2 entries each)
 * and the boundary planes z_layers (Z+1) as the .cw file stores them. */
sc_status sc_volume_waves(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2,
                          const void* x, const void* evl, const void* Qc, const void* Qh,
                          int ez_mode, long long* nw, int* begin, int* end, double* z_layers,
                          void* E0, void* k, void* stream);

/* CoupledWaveStructure::save (CoupledWaveStructure.h:63-125) from a device
 * wave table (E0, k: nw x 3 complex128 each, in file order -- the order
 * sc_volume_waves writes): u64 8, u64 #Pi and the Pi records, u64 layers,
 * then per layer its z (z_layers, host), u64 #Pr, records, u64 #Pt, records.
 * counts (host, 1 + 2 layers): #Pi, then #Pr and #Pt per layer.  Records are
 * 80 bytes {E0 pair, kx, ky, kz}; frame 0 stores the E0 pair in tira's record
 * frame (the frame rotated to Re k: the reference's scatterplane files), 1 the
 * Cartesian (E_x, E_y), 2 tira's frame with a downward wave (Re k_z < 0) in
 * the frame of its z-mirrored direction (the reference's scatterlayer files,
 * whose reflected waves tira::planewave's constructor made).  Records are
 * formed on the device and streamed through pinned buffers, the copy of one
 * chunk overlapping the write of the previous (GB-scale files at disk speed).
 * Synchronises the stream. */
sc_status sc_cw_write(sc_context* ctx, const char* path, const void* E0, const void* k, long long nw, int layers,
                      const double* z_layers, const long long* counts, int frame, void* stream);

/* ------------------------------------------------------ field evaluation */

/* E(r) = sum over the waves of r's region of E0 exp(i k.r)
 * (gpuEvaluator.cu:28-68).  Waves are structure-of-arrays complex128:
 * E0 (nw x 3) and k (nw x 3), row-major.  Regions follow cw_allocate
 * (cpuEvaluator.cpp:34-53): region l = waves [begin[l], end[l]); the region of
 * a point is #{ l : z >= z_layers[l] - zeps }.  Points (np x 3 doubles).
 * out: np x 3 complex128 (precision 0: float64 sum) or complex64 written as
 * complex128 (precision 1: float32 sum with float64 phase range reduction). */
sc_status sc_cw_evaluate(sc_context* ctx, const void* E0, const void* k, int nw,
                         const double* z_layers, const int* begin, const int* end, int layers,
                         double zeps, const double* points, long long np, void* out,
                         int precision, void* stream);

/* The field of a solved volume on a regular grid: points (x0 + i dx,
 * y0 + j dy, z0 + b dz) for i < Nx, j < Ny, b < Nz (origin, step, counts: 3
 * each, host); out[((b Ny + j) Nx + i) 3 + c] is E_c, complex128 (precision
 * 0) or complex64 (precision 1), device.  The same sum as sc_cw_evaluate over
 * the wave table of sc_volume_waves (ez_mode and zeps as there), evaluated in
 * the coupled-wave factorised form: per z plane, the waves of each Fourier
 * order are summed once, then two small separable transforms along y and x
 * (all FP64).  Orders along x up to 64.  Replaces a whole-grid evaluation
 * through gpu_cw_evaluate (gpuEvaluator.cu:131-165) / scatterview --nogui
 * slices (ScatterView.cpp:713-795); an x-z slice is Ny = 1.  Synchronises the
 * stream; sc_volume_stage_ms then holds [wave table, order sums, y transform,
 * x transform, -, -, -, total] device milliseconds. */
sc_status sc_volume_field_grid(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2, const void* x,
                               const void* evl, const void* Qc, const void* Qh, int ez_mode, const double* origin,
                               const double* step, const int* counts, double zeps, void* out, int precision,
                               void* stream);

/* ----------------------------------------- homogeneous layers, focused beams */

/* tira::planewave::SolidAnglePolar as scatterlayer and scatterplane call it
 * (ScatterLayer.cpp:384, ScatterPlane.cpp:240): N0 x N1 waves about
 * the centre wave (k_center: 3 doubles, E_center: 3 complex128, host; E is
 * expected orthogonal to k as the callers' orthogonalize() leaves it).  Wave
 * t = j N0 + i has polar angle beta + i (alpha - beta) / N0 and azimuth
 * j 2 pi / N1 about the centre direction (in the centre wave's record frame),
 * and E0 = sin(theta) dtheta dphi times the centre wave's record pair in its
 * own frame; each is then wound to the focal point (E0 exp(-i k.focus);
 * focus may be NULL).  alpha = 0 or N0 N1 = 1 gives the centre wave alone.
 * k_out: N0 N1 x 3 doubles, E_out: N0 N1 x 3 complex128 (device);
 * *count = the number of waves written.  Replaces the beam set-up of
 * ScatterLayer.cpp:355-385 and ScatterPlane.cpp:154-171, 236-242. */
sc_status sc_beam_polar(sc_context* ctx, double alpha, double beta, int N0, int N1,
                        const double* k_center, const double* E_center, const double* focus,
                        double* k_out, void* E_out, int* count, void* stream);

/* scatterlayer's per-wave solve (ScatterLayer.cpp:110-266, 390-420) for
 * `count` incident plane waves at once: layers L (1..15) with refractive
 * indices n[0..L-1] and absorbances kappa[0..L-2] of layers 1..L-1, boundary
 * planes z[0..L-2] (host arrays, the padded lists of ScatterLayer.cpp:321-343),
 * vacuum wavelength lambda.  k_in: count x 3 doubles (only the direction is
 * used), E_in: count x 3 complex128 (device).  Outputs per wave and boundary
 * l (count x (L-1) x 3 complex128 each, device): the reflected and
 * transmitted E0 and k of mat2waves, wound by -z_l as the .cw file stores
 * them.  status (device, count ints, may be NULL): SC_OK or SC_SINGULAR per
 * wave.  scatterplane's interface solve is the case L = 2. */
sc_status sc_layer_solve(sc_context* ctx, int layers, const double* n, const double* kappa,
                         const double* z, double lambda, int count, const double* k_in,
                         const void* E_in, void* r_E, void* r_k, void* t_E, void* t_k,
                         int* status, void* stream);

/* ------------------------------------------------- ScatterIO files (host) */

/* ScatterIO.h write_file (:18-42; the single-beam and single-event overloads
 * :89-117 are beams = 1): the plane normal and a point on the plane (3 doubles
 * each), then per beam its count of scattering events and their incident,
 * reflected and transmitted plane waves.  Records are tira planewave<double>
 * bytes, 80 per wave ({E0x, E0y, kx, ky, kz} complex128, as in the .cw file);
 * incident / reflected / transmitted hold sum(counts) records each, the beams
 * back to back. */
sc_status sc_scatterio_write(const char* path, const double* normal, const double* position, int beams,
                             const long long* counts, const void* incident, const void* reflected,
                             const void* transmitted);

/* ScatterIO.h read_file (:44-87): reads beams until a zero or missing count.
 * Writes the plane, *beams, *events (total records per list) and, when the
 * buffers are given, counts (beams_cap entries) and the records (events_cap
 * each).  Call with NULL buffers to size them; SC_BADINPUT if the file holds
 * more than the buffers or ends inside a beam. */
sc_status sc_scatterio_read(const char* path, double* normal, double* position, int* beams, long long* counts,
                            int beams_cap, void* incident, void* reflected, void* transmitted,
                            long long events_cap, long long* events);

/* ----------------------------------------- reference-signature shims (host) */

/* MKL_eigensolve(A, evl, evt, N): host buffers, column-major, A clobbered. */
sc_status sc_mkl_eigensolve(void* A, void* evl, void* evt, int N);

/* gpu_initialize(): copy the unpacked wave table (UnpackedWave<float>:
 * 6 complex64 per wave, E0[3] then k[3]) and the region index to the device. */
sc_status sc_gpu_initialize(int layers, const float* z_layers, const int* waves_begin,
                            const int* waves_end, const void* W, long long nW, int device);

/* gpu_cw_evaluate(): three N x N slices (x-y at z, x-z at y, y-z at x) of
 * E (N x N x 3 complex64, host buffers). */
sc_status sc_gpu_cw_evaluate(void* E_xy, void* E_xz, void* E_yz, float x_start, float y_start,
                             float z_start, float x, float y, float z, float d, int N,
                             int device);


/* --------------------------------------------------------- surrogate
 * A Fourier-neural-operator surrogate of the thin-volume solve (11 x 11
 * orders): a 64 x 64 real index map and a wavelength in, the R/T vector out
 * as 726 complex values (1452 floats, [Rx Ry Rz Tx Ty Tz] x 121 orders in the
 * column-major order index of sc_volume_solve's x, real and imaginary
 * interleaved).  No reference counterpart: the reference has no learned path;
 * the plain solve generates its training data, is its fallback, and measures
 * its error.  Inputs per pixel: n, the scaled wavelength, the coordinates and
 * the thin-element slab phase 2 pi n (1 um) / lambda as cos and sin (the
 * workload's slab is 1 um).  Width 64, 4 spectral layers, 16 x 16 modes; every linear map is
 * a BF16 tensor-core GEMM (tcgen05) with FP32 accumulation; training is Adam on FP32
 * master weights.  All buffers are device pointers; batch <= max_batch. */
typedef struct sc_fno sc_fno;
sc_status sc_fno_create(sc_fno** out, int device, int max_batch, unsigned long long seed);
sc_status sc_fno_destroy(sc_fno* f);
sc_status sc_fno_param_count(const sc_fno* f, long long* n);
/* Synchronises the network's device and reports SC_CUDA_ERROR if any of its
 * tensor-core GEMMs gave up on a pipeline wait since the last call (their
 * results are then not valid); the other sc_fno_* calls are asynchronous. */
sc_status sc_fno_status(sc_fno* f);
/* direction 0: copy the parameters out to dev_params; 1: load them from it */
sc_status sc_fno_params(sc_fno* f, void* dev_params, int direction, void* stream);
/* maps: batch x 64 x 64 floats; lambdas: batch floats (um); out: batch x 1452 */
sc_status sc_fno_forward(sc_fno* f, const float* maps, const float* lambdas, int batch, float* out, void* stream);
/* per-sample relative squared error |out - target|^2 / |target|^2 into loss
 * (batch floats) and the gradient of its batch mean into grad (param_count
 * floats); either may be NULL */
sc_status sc_fno_loss_grad(sc_fno* f, const float* maps, const float* lambdas, const float* target, int batch,
                           float* loss, float* grad, void* stream);
/* sc_fno_loss_grad followed by one Adam step (beta 0.9 / 0.999) at rate lr */
sc_status sc_fno_train_step(sc_fno* f, const float* maps, const float* lambdas, const float* target, int batch,
                            float lr, float* loss, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SCATTERSIM_B200_H */

/*
 * libdftcuda — B200 (sm_100a) implementation of dft-zig's plane-wave SCF hot path:
 * H|psi>, the block-Davidson ("LOBPCG") eigensolver's subspace algebra and the
 * band-density accumulation, behind a plain C ABI.
 *
 * Conventions shared with the reference:
 *  - complex numbers are interleaved {re, im} doubles (src/features/math/complex.zig:3-6);
 *  - blocks of vectors are column-major [n x ncols] (src/features/linalg/lobpcg/common.zig:16-24);
 *  - FFT boxes are indexed x + nx*(y + ny*z) (src/lib/fft/fftw_fft.zig:91-113);
 *  - energies are Rydberg, lengths bohr.
 *
 * Pointer arguments marked "host or device" may point to host memory (pageable or
 * pinned) or to device memory of the current CUDA device; the library detects which
 * and copies through its own device buffers when needed.  Every call returns an int
 * status: DFTCUDA_OK (0) or one of the negative codes below, which map one-to-one onto
 * the reference's Zig error set.  All calls are synchronous with respect to the host
 * unless named *_async.  The library's streams are ordered after work queued on the legacy default
 * stream, so device inputs written there need no extra synchronisation; inputs written on other
 * streams must be complete (synchronise those streams) before a call reads them.
 */
#ifndef DFTCUDA_H
#define DFTCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Zig error each one maps to, in the reference's error sets. */
#define DFTCUDA_OK 0
#define DFTCUDA_ERR_INVALID_MATRIX_SIZE (-1) /* error.InvalidMatrixSize (apply.zig:580, serial.zig:73) */
#define DFTCUDA_ERR_INVALID_GRID (-2)        /* error.InvalidGrid (pw_grid_map.zig:27-35)             */
#define DFTCUDA_ERR_EIGENSOLVER_FAILURE (-3) /* error.LapackFailure (lobpcg/common.zig:466,491)       */
#define DFTCUDA_ERR_OUT_OF_MEMORY (-4)       /* error.OutOfMemory                                     */
#define DFTCUDA_ERR_CUDA (-5)                /* CUDA runtime failure (no reference counterpart)       */
#define DFTCUDA_ERR_INVALID_ARGUMENT (-6)    /* null handle / inconsistent sizes                      */
#define DFTCUDA_ERR_UNSUPPORTED (-7)         /* FFT length with a prime factor other than 2, 3, 5     */
#define DFTCUDA_ERR_TIMEOUT (-8)             /* a bounded device wait gave up (no reference counterpart) */

/* Arithmetic of one k-point context's H|psi>:
 *  FP64    every pass in FP64;
 *  FP32    local-potential FFT passes in FP32, projector GEMMs in FP64;
 *  TF32    FFT passes in FP32 and the projector GEMMs on the tensor cores (tcgen05 kind::tf32, FP32
 *          accumulation in TMEM); relative error ~1e-3;
 *  TF32X3  as TF32 with every operand split into two TF32 parts (hi + lo, three MMAs per real
 *          product): FP32-class accuracy (~1e-6) on the tensor cores.
 * Wavefunctions are FP64 at the boundary in every mode.  In TF32 and TF32X3 contexts every
 * eigensolver subspace product (V^H W, V C, W C, the orthonormalisation's projections and block
 * overlaps) uses the same tensor-core GEMM (split form); the Cholesky factorisations, the subspace
 * eigensolver and the residual norms stay FP64. */
#define DFTCUDA_PRECISION_FP64 0
#define DFTCUDA_PRECISION_FP32 1
#define DFTCUDA_PRECISION_TF32 2
#define DFTCUDA_PRECISION_TF32X3 3

typedef struct dftcuda_kctx dftcuda_kctx;
typedef struct dftcuda_fft_plan dftcuda_fft_plan;

/* Human-readable name of a status code, and the message of the last failure on this thread. */
const char* dftcuda_status_string(int status);
const char* dftcuda_last_error_message(void);

/* Number of CUDA devices visible (0 on a host without a GPU; never fails). */
int dftcuda_device_count(void);

/* Failure injection for tests of the timeout path (no reference counterpart).  Every device-side wait
 * in the library is bounded: the subspace eigensolver's grid barrier polls about a second, then sets
 * an error flag, its blocks return, and the call reports DFTCUDA_ERR_TIMEOUT with the context still
 * usable.  polls > 0 sets that barrier's poll budget (0 restores the default); unreachable != 0 raises
 * every barrier's target by one arrival that no block makes, so each wait runs out its budget.
 * Process-wide; applies to launches made after the call. */
int dftcuda_debug_set_wait_limits(long polls, int unreachable);

/* Failure injection for tests of the out-of-memory path (no reference counterpart): after >= 0 makes
 * the after-th following device allocation of the library fail once, as cudaMalloc does when the
 * device is full; the entry point that made it returns DFTCUDA_ERR_OUT_OF_MEMORY and its context
 * stays usable.  after < 0 cancels a planned failure.  Process-wide. */
int dftcuda_debug_fail_alloc(long after);

/* ------------------------------------------------------------------------------------------
 * Per-k-point context: replaces the ApplyContext + KpointApplyCache pair
 * (src/features/scf/apply.zig:45-169, 554-573) and PwGridMap (src/features/scf/pw_grid_map.zig:8-56).
 *
 * hkl[n_pw*3]   Miller indices of the G-sphere in basis order (plane_wave/basis.zig:26-74)
 * kinetic[n_pw] |k+G|^2 (Ry) = the kinetic diagonal (apply.zig:589-592)
 * gcart[n_pw*3] Cartesian G (bohr^-1), used for the atom phases exp(i G.tau) (apply.zig:883-896)
 * The FFT box (nx, ny, nz) must hold every Miller index (else DFTCUDA_ERR_INVALID_GRID) and each
 * extent must be 2,3,5-smooth and <= 128 (else DFTCUDA_ERR_UNSUPPORTED).
 * All host pointers; the context keeps device copies.  One context per k-point; each owns a
 * CUDA stream, so contexts run independently like the reference's per-thread ApplyContexts.
 * ------------------------------------------------------------------------------------------ */
int dftcuda_kctx_create(dftcuda_kctx** out, int nx, int ny, int nz, double volume, size_t n_pw,
                        const int32_t* hkl, const double* kinetic, const double* gcart, int precision);
int dftcuda_kctx_destroy(dftcuda_kctx* ctx);
size_t dftcuda_kctx_npw(const dftcuda_kctx* ctx);

/* Real local potential V(r) on the FFT box (N doubles, x fastest): the local_r argument of
 * ApplyContext.init (apply.zig:235-300), built by build_local_potential_real (scf/potential.zig:320-334).
 * Host or device pointer. */
int dftcuda_set_vloc(dftcuda_kctx* ctx, const double* local_r);

/* Kleinman-Bylander projectors of one species (NonlocalSpecies, scf/nonlocal_context.zig:9-41). */
typedef struct dftcuda_species {
  size_t beta_count;     /* number of radial projectors                                         */
  const int32_t* l_list; /* [beta_count] angular momentum of each projector                      */
  const double* dij;     /* [beta_count*beta_count] row-major D_ij (Ry), radial form             */
  size_t m_total;        /* sum over projectors of 2l+1                                          */
  const double* phi;     /* [m_total*n_pw] row-major phi = 4 pi R(|k+G|) Y_lm(k+G) (nonlocal_context.zig:524-549) */
} dftcuda_species;

/* Installs the nonlocal part: species[n_species], atom_species[n_atoms] (index into species),
 * atom_pos[n_atoms*3] Cartesian bohr.  Passing n_species == 0 removes it.  Host pointers. */
int dftcuda_set_projectors(dftcuda_kctx* ctx, size_t n_species, const dftcuda_species* species, size_t n_atoms,
                           const int32_t* atom_species, const double* atom_pos);

/* y = H x for ncols columns: Operator.apply_batch = apply_hamiltonian_batched (apply.zig:1584-1618).
 * x, y: [n x ncols] column-major complex128, host or device.  n must equal n_pw.  With host x and y
 * and 64 columns or more the call runs column chunks whose copies in and out overlap the compute of
 * their neighbours (four equal chunks below 256 columns; from 256 on, 64-column chunks at both ends
 * and up to six in between); pinned host memory lets the copies run asynchronously.  It returns
 * when y is complete. */
int dftcuda_apply_h_batch(dftcuda_kctx* ctx, const double* x, double* y, size_t n, size_t ncols);
/* Single column: Operator.apply = apply_hamiltonian (apply.zig:643-658). */
int dftcuda_apply_h(dftcuda_kctx* ctx, const double* x, double* y, size_t n);
/* Device pointers only, enqueued on `stream` (a cudaStream_t; NULL = the context's stream),
 * no host synchronisation. */
int dftcuda_apply_h_batch_async(dftcuda_kctx* ctx, const double* x_dev, double* y_dev, size_t ncols, void* stream);

/* Re <psi_b|V_nl|psi_b> for nbands columns (kpoint/density.zig:145-165, 238-266). Host or device. */
int dftcuda_nonlocal_energies(dftcuda_kctx* ctx, const double* psi, size_t n, size_t nbands, double* e_out);

/* Nonlocal Hellmann-Feynman forces on the context's atoms (accumulate_atom_force_at_kpoint,
 * forces/nonlocal_force.zig:283-341): F[a][d] = (2/Omega) sum_b w_b Im sum_{j of atom a}
 * conj((D p)_jb) <beta_j|(k+G)_d psi_b>, p = <beta|psi>.  vectors: (nbands, n) complex128,
 * weights: nbands doubles (k weight x occupation x spin), forces: natoms x 3 doubles (Ry/bohr), the
 * atoms in the order given to dftcuda_set_projectors.  Sum the k-points' results for the total. */
int dftcuda_nonlocal_forces(dftcuda_kctx* ctx, const double* vectors, size_t n, size_t nbands, const double* weights,
                            double* forces);

/* Nonlocal (Kleinman-Bylander) stress of nbands bands at this k-point (stress/nonlocal_stress.zig:108-558,
 * norm-conserving): sigma_ab = -(2/Omega^2) sum_n f_n sum_(atom,m) Re[conj(Dp_mn) sum_G dphi_m/dq_a(G)
 * e^{iG.tau} q_b c_n(G)] - delta_ab sum_n f_n E_nl,n / Omega, with p = <beta|psi> of the context's
 * projectors, Dp the D_ij contraction, E_nl,n = Re sum conj(p) Dp / Omega, q = k + G.  Like the reference,
 * only the components a <= b are filled (the rest of sigma[9], row-major, is 0).  kpg[n*3]: k + G of the
 * basis; dphi[s] (one per species given to dftcuda_set_projectors): [3][m_total][n] derivative
 * projectors d phi_bm / d q_a = 4 pi (R_b'(|q|) q_a/|q| Y_lm + R_b dY_lm/dq_a) (project_p_and_dp,
 * nonlocal_stress.zig:108-165); vectors (nbands, n) complex128; weights f_n (occupation x k weight x
 * spin; bands with f_n <= 0 skipped); sigma in Ry/bohr^3.  Host or device pointers (dphi entries too).
 * The six strain projections run through the library's FP64 complex GEMM.  Sum over k-points. */
int dftcuda_nonlocal_stress(dftcuda_kctx* ctx, const double* kpg, size_t n_species, const double* const* dphi,
                            const double* vectors, size_t n, size_t nbands, const double* weights, double* sigma);

/* Autotuner: times candidate launch configurations of this context's H|psi> on ncols trial
 * columns (FFT pass variant, column-chunk workspace budget, split-K of the two projector GEMMs)
 * with CUDA events and keeps the fastest for all later calls.  report may be NULL. */
typedef struct dftcuda_tune_report {
  int fft_path;          /* 2 stick layout, 1 plane layout (four-step register FFT passes), 0 generic passes */
  double box_budget_mb;  /* active-plane workspace budget per column chunk */
  int proj_splits;       /* split-K of the projection GEMM (0 = built-in heuristic) */
  int back_splits;       /* split-K of the back-projection GEMM (0 = built-in heuristic) */
  double default_ms;     /* H|psi> on ncols columns with the built-in defaults */
  double tuned_ms;       /* the same with the chosen configuration */
  int candidates;        /* configurations timed */
} dftcuda_tune_report;
int dftcuda_kctx_autotune(dftcuda_kctx* ctx, size_t ncols, dftcuda_tune_report* report);

/* ------------------------------------------------------------------------------------------
 * Eigensolver: lobpcg_serial.solve (src/features/linalg/lobpcg/serial.zig:55-307) with
 * Options (lobpcg/common.zig:44-52).  The whole Davidson loop runs on the device; H is the
 * context's operator.
 * ------------------------------------------------------------------------------------------ */
typedef struct dftcuda_eig_opts {
  size_t max_iter;      /* default 40 */
  double tol;           /* default 1e-6 */
  size_t max_subspace;  /* 0 = min(n, 4*nbands+8) */
  size_t block_size;    /* 0 = min(max_subspace, nbands+4) */
  int init_diagonal;    /* bool */
} dftcuda_eig_opts;

typedef struct dftcuda_eig_info {
  size_t iterations;    /* Davidson iterations run */
  size_t h_applies;     /* columns passed through H */
  int converged;        /* 1 when max residual < tol or no vector could be added */
  double max_residual;  /* at the last iteration */
} dftcuda_eig_info;

/* diag[n] is the preconditioner diagonal (kinetic |k+G|^2, kpoint/solve.zig:362-367).
 * init_vecs: optional [n x init_cols] warm start (KpointCache, kpoint/data.zig:7-46), NULL for none.
 * values_out[nbands], vectors_out[n x nbands]; all host or device.  info may be NULL. */
int dftcuda_eig_solve(dftcuda_kctx* ctx, const double* diag, size_t nbands, const dftcuda_eig_opts* opts,
                      const double* init_vecs, size_t init_cols, double* values_out, double* vectors_out,
                      dftcuda_eig_info* info);

/* The same solver for nk k-point contexts at once (the k-point loop of kpoint/workers.zig:133-180):
 * the runs advance in lockstep, each on its own context's stream, with one host synchronisation per
 * phase for all of them, so the GPU overlaps the k-points' kernels.  Per-k arrays of length nk:
 * diags[k] (n_k), init_vecs (NULL, or per-k pointers that may be NULL) with init_cols, values_out[k]
 * (nbands), vectors_out[k] (n_k x nbands); infos: NULL or nk entries.  Each context at most once,
 * all created on one device (DFTCUDA_ERR_UNSUPPORTED otherwise; one batch per device). */
int dftcuda_eig_solve_batch(size_t nk, dftcuda_kctx* const* ctxs, const double* const* diags, size_t nbands,
                            const dftcuda_eig_opts* opts, const double* const* init_vecs, const size_t* init_cols,
                            double* const* values_out, double* const* vectors_out, dftcuda_eig_info* infos);

/* Preconditioner of the Davidson correction step for this context's solves:
 *  REFERENCE  q_i = r_i / (diag_i - lambda_b), |den| >= 1e-8 (lobpcg/common.zig:214-226), the default;
 *  TPA        Teter-Payne-Allan K(|k+G_i|^2 / E_kin,b) r_i;
 *  MLP        a learned per-plane-wave multiplier m = K_TPA(x) exp(z(u)) r_i, z a 3-64-64-1 tanh MLP
 *             (FP32) of u = (log(x + 0.05), log(|r_i| / rms(r) + 1e-6), iteration / 20), x = |k+G|^2 / E_kin:
 *             a refinement of TPA (zero output weights give TPA); params[DFTCUDA_PRECOND_MLP_PARAMS] in
 *             the order W1[64][3], b1[64], W2[64][64], b2[64], w3[64], b3 (host or device).  The
 *             solver evaluates z through a 256 x 512 table of the network over (u0, u1) per
 *             iteration (bilinear, |dz| <= 5e-5 for the shipped weights; the network itself outside
 *             u0 in [-3, 7], u1 in [-13.85, 7]); DFTCUDA_MLP_INFER=tc evaluates it per entry instead.
 * diag passed to dftcuda_eig_solve must be the kinetic energies |k+G|^2 for TPA and MLP. */
#define DFTCUDA_PRECOND_REFERENCE 0
#define DFTCUDA_PRECOND_TPA 1
#define DFTCUDA_PRECOND_MLP 2
#define DFTCUDA_PRECOND_MLP_PARAMS 4481
int dftcuda_kctx_set_preconditioner(dftcuda_kctx* ctx, int kind, const float* params, size_t nparams);

/* Training of the learned preconditioner on the GPU.  Samples are bands b = 0..nbands-1 whose
 * plane waves occupy [band_off[b], band_off[b+1]) of npw rows: feat[3 npw] the MLP inputs above,
 * cc[2 npw] = conj(r_i) delta_i (complex, interleaved), w[npw] = |r_i|^2, dnorm[nbands] = ||delta_b||^2,
 * delta the correction from the Ritz vector to the converged eigenvector.  Loss (scale-free, as the
 * Davidson step is) L = mean_b [1 - |sum m_i cc_i|^2 / (sum m_i^2 w_i * dnorm_b)].
 * loss_grad: L and dL/dparams for the given params.  train: `steps` full-batch Adam steps (beta
 * 0.9 / 0.999) with learning rate lr, params updated in place, loss_history[steps] (may be NULL). */
int dftcuda_precond_mlp_loss_grad(size_t nbands, size_t npw, const int* band_off, const float* feat, const float* cc,
                                  const float* w, const float* dnorm, const float* params, double* loss, float* grad);
int dftcuda_precond_mlp_train(size_t nbands, size_t npw, const int* band_off, const float* feat, const float* cc,
                              const float* w, const float* dnorm, float* params, size_t steps, float lr,
                              double* loss_history);

/* Learned first SCF density: a Fourier neural operator (4 Fourier layers, 16 modes per axis, 8
 * channels, FP32) from the superposition-of-atoms density to (rho_scf - rho_atomic) / mean density,
 * both on the cell's FFT grid (x fastest, every axis >= 16).  u: 2 channels [2][nx ny nz], the
 * Si-like and Ge-like atomic superposition densities divided by the mean valence density.
 * params[DFTCUDA_FNO_PARAMS]: P[8][2], p[8], then per layer R[4096][8][8] complex, W[8][8], b[8],
 * then q[8], q0.  Samples of a training set: dims[3 s], grid-point offsets offs[s+1] (u for sample s
 * at u + 2 offs[s], target at target + offs[s]).  Loss: mean over samples of the mean squared error.
 * train: `steps` full-batch Adam steps, params updated in place.  Host or device pointers. */
#define DFTCUDA_FNO_PARAMS 2097473
int dftcuda_fno_forward(int nx, int ny, int nz, const float* u, const float* params, float* out);
int dftcuda_fno_loss_grad(size_t nsamples, const int* dims, const size_t* offs, const float* u, const float* target,
                          const float* params, double* loss, float* grad);
int dftcuda_fno_train(size_t nsamples, const int* dims, const size_t* offs, const float* u, const float* target,
                      float* params, size_t steps, float lr, double* loss_history);

/* Dense Hermitian eigensolver: linalg.hermitian_eigen_decomp (src/features/linalg/linalg.zig:141-151;
 * zheev 'V','U' in hermitian_eigen_decomp_lapack) and lobpcg/common.zig:440-508, restricted to the
 * nev lowest eigenpairs (nev = n gives the full decomposition).  a: n x n column-major complex, the
 * upper triangle is read.  values[nev] ascending, vectors[n x nev]; host or device pointers.
 * n <= 2048.  The Davidson loop above uses the same kernels for subspaces of 96 and more. */
int dftcuda_hermitian_eigen_decomp(size_t n, const double* a, size_t nev, double* values, double* vectors);

/* ------------------------------------------------------------------------------------------
 * Band density: rho(r) += sum_b weight_b |psi_b(r)|^2 / Omega
 * (accumulate_band_density_fft, kpoint/density.zig:444-474; weights w_k*occ*2 as in :98-112).
 * vectors [n x nbands], weights[nbands] (bands with weight <= 0 are skipped), rho[N] on the FFT
 * box (x fastest) is ADDED to.  Host or device pointers.
 * ------------------------------------------------------------------------------------------ */
int dftcuda_accumulate_density(dftcuda_kctx* ctx, const double* vectors, size_t n, size_t nbands,
                               const double* weights, double* rho);

/* Band density for callers that cannot allocate device memory.  This entry point has no
 * counterpart in the reference.  Some callers cannot call cudaMalloc here: code running inside a
 * host framework that owns every device allocation through its own memory pool, or a loop that must
 * not take the device-wide synchronisation an allocation can cause.  This variant of
 * dftcuda_accumulate_density allocates nothing: its scratch is a fixed array of
 * DFTCUDA_NOALLOC_SCRATCH_BYTES (48 MiB) in the library's device image, which every GPU that loads
 * the library holds until exit.  vectors [n x nbands], weights[nbands] and rho[N] must all be device
 * pointers (host pointers are rejected), nbands may not exceed DFTCUDA_NOALLOC_MAX_BANDS, and rho is
 * ADDED to exactly as in dftcuda_accumulate_density (bands with weight <= 0 contribute nothing).
 * The call runs on the device the context was created on and is ordered after all work queued on
 * the legacy default stream; inputs written on any other stream must be complete (synchronise that
 * stream) before the call.  It returns after its work on the context's stream has finished.
 * The first call on each device looks up the scratch address, so make that first call before any
 * stream capture begins.  All calls share the one scratch array, whose contents persist from call to
 * call, so calls that overlap on the GPU (from two host threads, or two contexts whose streams run
 * concurrently) race; serialise them. */
#define DFTCUDA_NOALLOC_SCRATCH_BYTES ((size_t)48 << 20)
#define DFTCUDA_NOALLOC_MAX_BANDS 4096
int dftcuda_accumulate_density_noalloc(dftcuda_kctx* ctx, const double* vectors, size_t n, size_t nbands,
                                       const double* weights, double* rho);

/* Fermi level and occupations of an eigenvalue table, FP64 on the device: find_fermi_level_spin with
 * smearing_occ / smearing_entropy (src/features/scf/fermi_level.zig:7-124), Fermi-Dirac smearing.
 * values[nk*nbands] (one row of nbands per k-point), kweights[nk] (summing to 1), spin_factor 2 for
 * unpolarised bands.  The bracket [min e - pad, max e + pad], pad = max(10 sigma, 1e-3), doubles up
 * to 12 times until it holds nelec; then up to 80 bisections, stopping once |N(mu) - nelec| < 1e-8.
 * mu_out: the Fermi level; occ (may be NULL): [nk*nbands] 1/(1 + exp((e - mu)/sigma)) (a step at mu
 * when sigma <= 0); sums (may be NULL): sums[0] = sum_kb spin w_k occ_kb e_kb (band energy),
 * sums[1] = sum_kb spin w_k S(occ_kb), S(f) = -(f ln f + (1-f) ln(1-f)) (0 within 1e-12 of 0 or 1),
 * the entropy that enters the energy as -sigma * sums[1].  Host or device pointers. */
int dftcuda_fermi_occupations(size_t nk, size_t nbands, const double* values, const double* kweights, double nelec,
                              double sigma, double spin_factor, double* mu_out, double* occ, double* sums);

/* ------------------------------------------------------------------------------------------
 * Profiling: the ScfProfile counters (src/features/scf/logging.zig:114-131) measured on the device
 * with CUDA events on the context's launch stream.  The fused local-potential passes replace the
 * reference's scatter / ifft / vmul / fft / gather sub-timers with the three pass timers below.
 * set_profiling(1) clears and starts the counters; get_profile synchronises the context's stream.
 * ------------------------------------------------------------------------------------------ */
typedef struct dftcuda_profile {
  uint64_t apply_h_ns;          /* all H|psi> kernels                                              */
  uint64_t apply_local_ns;      /* local potential + kinetic (the three passes)                    */
  uint64_t apply_nonlocal_ns;   /* projector GEMMs and D_ij                                        */
  uint64_t density_ns;          /* band-density kernels                                            */
  uint64_t subspace_ns;         /* eigensolver kernels outside H: V^H W, Jacobi, V C, Gram-Schmidt */
  uint64_t apply_h_calls;       /* block applications of H                                         */
  uint64_t apply_h_columns;     /* columns through H                                               */
  uint64_t local_plane_inv_ns;  /* scatter + inverse FFT along z and y                             */
  uint64_t local_xline_ns;      /* inverse x FFT, x V(r), forward x FFT                            */
  uint64_t local_plane_fwd_ns;  /* forward FFT along y and z, gather x 1/N, + kinetic              */
  uint64_t local_plane_inv_launches;
  uint64_t local_xline_launches;
  uint64_t local_plane_fwd_launches;
  uint64_t nl_project_ns;       /* <beta|psi> GEMM                                                 */
  uint64_t nl_dij_ns;           /* D_ij                                                            */
  uint64_t nl_backproject_ns;   /* sum |beta> D <beta|psi> GEMM                                    */
  uint64_t kernel_launches;     /* libdftcuda kernels launched on this context while profiling     */
  uint64_t local_layout;        /* passes of the last H|psi>: 0 generic, 1 plane layout (three passes
                                   k_plane_inv5, k_xline5, k_plane_fwd5), 2 stick layout (k_stick_inv,
                                   k_zplane, k_stick_fwd: the three counters above in that order)  */
} dftcuda_profile;

int dftcuda_kctx_set_profiling(dftcuda_kctx* ctx, int enable);
int dftcuda_kctx_get_profile(dftcuda_kctx* ctx, dftcuda_profile* out);

/* ------------------------------------------------------------------------------------------
 * Standalone 3D FFT with the FFTW backend's semantics: in place, forward e^{-i} unnormalised,
 * inverse e^{+i} scaled by 1/N (Fft3dPlan.forward/inverse, features/fft/fft.zig:224-263;
 * fftw_fft.zig:141-166).  direction: -1 forward, +1 inverse.  data: N complex128, host or device.
 * ------------------------------------------------------------------------------------------ */
int dftcuda_fft_plan_create(dftcuda_fft_plan** out, int nx, int ny, int nz);
int dftcuda_fft_plan_destroy(dftcuda_fft_plan* plan);
int dftcuda_fft3d(dftcuda_fft_plan* plan, double* data, int direction);

/* ------------------------------------------------------------------------------------------
 * SCF potential build and mixing on the device (the per-iteration host work around the path).
 *
 * A potential context holds the FFT box (nx, ny, nz; x fastest), the cell volume and |G|^2 of every
 * box point (G = h b1 + k b2 + l b3, recip = the rows b1, b2, b3 in bohr^-1, h, k, l in FFT order
 * 0, 1, ..., -1), and the Pulay history.  G-space fields are N complex numbers normalised as
 * f(G) = (1/N) sum_r f(r) e^{-iGr}.  Every pointer may be host or device memory; the calls return
 * when their results are written.
 *
 * dftcuda_hxc_potential: from the density rho(r) (N doubles, electrons/bohr^3), the Hartree + XC
 * potential in G space (build_potential_grid, scf/potential.zig:144-203: V_H(G) = 8 pi rho(G)/G^2
 * for G^2 > 1e-12, else 0, plus V_xc(G) of LDA-PZ, xc/xc.zig:195-211, 344-384) into v_out_g (N
 * complex, interleaved), and the energy terms of that density (scf/energy.zig:372-396):
 * e_hartree = (vol/2) sum_G 8 pi |rho(G)|^2 / G^2, e_xc = (vol/N) sum_r f_xc(rho(r)), and, when
 * v_in_g is not NULL, int_vin_rho = (vol/N) sum_r v_in(r) rho(r) for the real-space field of v_in_g.
 *
 * dftcuda_potential_real: out_r = vloc_r + v(r) with v(r) = sum_G v_g(G) e^{iGr} (real part);
 * vloc_r may be NULL.  The local potential handed to dftcuda_set_vloc.
 *
 * dftcuda_pulay_mix: Pulay / DIIS step of PulayMixer.mix_with_residual (scf/mixing.zig:182-248) on
 * n doubles: x (in: current input, out: mixed) and residual; the context keeps the last `history`
 * (x, residual) pairs on the device; with fewer than two it returns x + beta * residual, else
 * sum_i c_i (x_i + beta r_i) with c from the bordered system B_ij = <r_i|r_j>, sum c = 1.
 * dftcuda_pulay_reset clears the history.  These have no reference counterpart as device calls.
 * ------------------------------------------------------------------------------------------ */
typedef struct dftcuda_pctx dftcuda_pctx;
typedef struct dftcuda_hxc_terms {
  double e_hartree;
  double e_xc;
  double int_vin_rho;
} dftcuda_hxc_terms;
int dftcuda_pctx_create(dftcuda_pctx** out, int nx, int ny, int nz, double volume, const double* recip,
                        int pulay_history);
int dftcuda_pctx_destroy(dftcuda_pctx* ctx);
/* Exchange-correlation functional of dftcuda_hxc_potential (xc.Functional, xc/xc.zig:5-8):
 * DFTCUDA_XC_LDA_PZ (the default) or DFTCUDA_XC_PBE (gradient from FFTs, compute_gga_xc_fields,
 * scf/xc_fields.zig:108-142). */
#define DFTCUDA_XC_LDA_PZ 0
#define DFTCUDA_XC_PBE 1
int dftcuda_pctx_set_functional(dftcuda_pctx* ctx, int functional);
int dftcuda_hxc_potential(dftcuda_pctx* ctx, const double* rho_r, const double* v_in_g, double* v_out_g,
                          dftcuda_hxc_terms* terms);
int dftcuda_potential_real(dftcuda_pctx* ctx, const double* v_g, const double* vloc_r, double* out_r);
int dftcuda_pulay_mix(dftcuda_pctx* ctx, double* x, const double* residual, size_t n, double beta);
/* build_ionic_potential_grid (scf/potential.zig:279-318) for pseudopotentials with the analytic
 * Goedecker-Teter-Hutter local part: V(G) = (2/vol) sum_atoms ff_s(|G|) e^{-iG.tau} for
 * 1e-12 < G^2 <= g2max (g2max <= 0: no cut), ff the GTH local form factor (Hartree) of species s with
 * gth[6 s .. 6 s + 5] = Z_ion, r_loc, C1, C2, C3, C4.  atom_species[natoms] in 0..nspecies-1 (at most
 * 8 species), positions[natoms*3] Cartesian bohr.  Writes V(G) to v_out_g (N complex) and/or
 * V_loc(r) = sum_G V(G) e^{iGr} to vloc_r (N doubles); either may be NULL. */
int dftcuda_ionic_potential(dftcuda_pctx* ctx, int nspecies, const double* gth, int natoms, const int* atom_species,
                            const double* positions, double g2max, double* v_out_g, double* vloc_r);
/* local_pseudo_forces (forces/local_force.zig:21-80): the local-pseudopotential Hellmann-Feynman
 * force on every atom, F_a = sum_G 2 ff_s(|G|) G Im(e^{iG.tau_a} rho(G)) for 1e-12 < G^2 <= g2max
 * (same species parameters as dftcuda_ionic_potential), from the density rho_r (N doubles).
 * forces: natoms x 3 doubles, Ry/bohr. */
int dftcuda_local_forces(dftcuda_pctx* ctx, int nspecies, const double* gth, int natoms, const int* atom_species,
                         const double* positions, double g2max, const double* rho_r, double* forces);
int dftcuda_pulay_reset(dftcuda_pctx* ctx);

/* dftcuda_ionic_potential and dftcuda_local_forces for pseudopotentials given by their radial mesh
 * (the UPF local part), with the reference's local form factor in its default short_range mode
 * (local_vq_short_range, src/features/pseudopotential/form_factor.zig:223-262; config/defaults.zig:28),
 * evaluated at every |G| of the box as the SCF does (ionic_local_potential, hamiltonian.zig):
 *   V_s(q) = 4 pi sum_j r_j^2 [vloc_j + 2 Z_s / r_j] sinc(q r_j) rab_j w_j - 8 pi Z_s / q^2   (Ry),
 * w the composite-trapezoid weights of radial_integration.zig:7-13, the 2Z/r term skipped at
 * r < 1e-10.  Species s uses points [mesh_off[s], mesh_off[s+1]) of r, rab and vloc (Ry; mesh_off[0]
 * = 0, nspecies + 1 entries, host memory), z_valence[nspecies].  V(G) = (1/vol) sum_atoms V_s(|G|)
 * e^{-iG.tau} for |G| >= 1e-10 and G^2 < g2max (build_ionic_potential_grid, potential.zig:279-318;
 * g2max <= 0: no cut); the local forces (local_pseudo_forces, forces/local_force.zig:66-111) from the
 * same V_s.  Other arguments and outputs as the GTH forms above. */
int dftcuda_ionic_potential_radial(dftcuda_pctx* ctx, int nspecies, const size_t* mesh_off, const double* r, const double* rab,
                                   const double* vloc, const double* z_valence, int natoms, const int* atom_species,
                                   const double* positions, double g2max, double* v_out_g, double* vloc_r);
int dftcuda_local_forces_radial(dftcuda_pctx* ctx, int nspecies, const size_t* mesh_off, const double* r, const double* rab,
                                const double* vloc, const double* z_valence, int natoms, const int* atom_species,
                                const double* positions, double g2max, const double* rho_r, double* forces);

/* Density symmetrisation (symmetrize_density, scf/density_symmetry.zig:27-94), in place on rho_r
 * (N doubles, x fastest, host or device): rho(G) <- (1/nops) sum_op rho(k_rot G) e^{-2 pi i frac(G.t)}
 * over the box's signed Miller indices G, rotated indices wrapped into the box.  k_rot: 9 ints per
 * operation, row-major (SymOp.k_rot = (rot^-1)^T, symmetry/symmetry.zig:229-233); trans: 3 doubles
 * per operation, fractional (SymOp.trans).  Host pointers or device.  nops <= 1 leaves rho as it is;
 * at most 192 operations. */
int dftcuda_symmetrize_density(dftcuda_pctx* ctx, int nops, const int* k_rot, const double* trans, double* rho_r);

/* Radial projector table of one beta (RadialTableSet.init, pseudopotential/nonlocal.zig:250-338,
 * entries radial_projector, nonlocal.zig:8-21): out[i] = sum_j r_j rbeta_j j_l(q_i r_j) rab_j w_j on
 * q_i = i gmax / (nq - 1), w the composite-trapezoid weights of radial_integration.zig:7-13 and j_l
 * as nonlocal.zig:59-71.  r, rbeta (r times beta), rab: the radial mesh (nr points); out: nq doubles.
 * Any pointer may be host or device memory. */
int dftcuda_radial_table(int l, size_t nr, const double* r, const double* rbeta, const double* rab, size_t nq, double gmax,
                         double* out);

/* Plane-wave basis of one k-point (plane_wave.generate, features/plane_wave/basis.zig:26-74): the
 * Miller triples of the box [-n, n]^3, n = ceil(sqrt(ecut) / min |b_i|) + 1, in the reference's loop
 * order (h outer, l inner), kept when |k + G|^2 <= ecut_ry; every value bit-identical to the
 * reference's arithmetic.  recip: rows b1, b2, b3 (9 doubles, 1/bohr, 2 pi included); k_cart: 3
 * doubles.  capacity == 0 is a size query (*n_out = basis size); otherwise hkl [n][3], gcart [n][3],
 * kpg [n][3] and kinetic [n] receive the basis (host or device arrays; InvalidMatrixSize when
 * capacity < size). */
int dftcuda_plane_wave_basis(const double* recip, double ecut_ry, const double* k_cart, size_t capacity, int32_t* hkl,
                             double* gcart, double* kpg, double* kinetic, size_t* n_out);

/* Projector table rows of one radial projector (fill_nonlocal_phi, scf/nonlocal_context.zig:524-549):
 * phi[m + l][i] = 4 pi R(|kpg_i|) Y_lm(kpg_i), m = -l..l, R by RadialTable.eval on the uniform table
 * (nq values over [0, gmax], pseudopotential/nonlocal.zig:250-300), Y_lm the real harmonics of
 * nonlocal.zig:152-241 (l <= 4).  kpg: [n][3]; phi: [(2l+1)][n].  Host or device pointers. */
int dftcuda_projector_phi(int l, size_t nq, double gmax, const double* table, size_t n, const double* kpg, double* phi);

/* ------------------------------------------------------------------------------------------
 * The library's complex GEMM (no counterpart in the reference; the contraction its projector and
 * Rayleigh-Ritz code paths run), exposed for tests and benchmarks:
 *   out(r, c) = alpha * sum_k opA(A(r, k)) * opB(B(c, k)) + beta * out(r, c),   r < M, c < N, k < K
 * A(r, k) is A[r*lda + k] when a_kc != 0 (K contiguous), else A[k*lda + r]; the same for B; opX
 * conjugates when conj_x != 0.  out(r, c) is out[r*ldo_r + c*ldo_c].  All pointers are device
 * pointers to interleaved complex128.  precision: DFTCUDA_PRECISION_FP64 (FP64 FMA kernel),
 * DFTCUDA_PRECISION_TF32 or DFTCUDA_PRECISION_TF32X3 (tcgen05 tensor-core kernels); FP32 is not
 * accepted.  The call allocates its split-K workspace, runs on a private stream and returns after
 * the product is complete.
 * ------------------------------------------------------------------------------------------ */
int dftcuda_complex_gemm(int precision, size_t M, size_t N, size_t K, const double* a, long lda, int a_kc, int conj_a,
                         const double* b, long ldb, int b_kc, int conj_b, double* out, long ldo_r, long ldo_c, double alpha,
                         double beta);

#ifdef __cplusplus
}
#endif

#endif /* DFTCUDA_H */

// Per-k-point context shared by the H|psi>, density and eigensolver translation units.
#pragma once

#include <vector>

#include "fft_core.cuh"

namespace dftcuda {

// Device buffer of the tensor-core GEMM's pre-split operands (grown on demand, owned by a context).
// As the cache of a constant operand (the projector matrix) it also records what it holds: valid
// and the key of the layout it was split for.
struct TcScratch {
  void* p = nullptr;
  size_t bytes = 0;
  bool valid = false;
  unsigned long long key = 0;
  int ensure(size_t need);
  void release();
};

// Complex GEMM over strided operands (zgemm.cu):
//   out(r, c) = alpha * sum_k opA(A(r, k)) * opB(B(c, k)) + beta * out(r, c)
//   A(r, k) = a_kc ? A[r*lda + k] : A[k*lda + r]      B(c, k) = b_kc ? B[c*ldb + k] : B[k*ldb + c]
//   out(r, c) = O[r*ldo_r + c*ldo_c];  conj_a / conj_b conjugate the operand.
struct GemmArgs {
  int M, N, K;
  const double2* A; long lda; bool a_kc; bool conj_a;
  const double2* B; long ldb; bool b_kc; bool conj_b;
  double2* O; long ldo_r; long ldo_c;
  double alpha, beta;
  int splits = 0;  // split-K count; 0 = the kernel's wave-filling heuristic
  // Constant operands whose TF32 split the tensor-core GEMM may keep between calls (null: split per call).
  TcScratch* a_cache = nullptr;
  TcScratch* b_cache = nullptr;
};
int zgemm(const GemmArgs& g, cudaStream_t s, double2* workspace, size_t workspace_elems);
size_t zgemm_workspace_elems(int M, int N, int K);
// The same contraction on the tensor cores (tc_gemm.cu): TF32 inputs, FP32 accumulation.  err_dev
// receives 1 if a bounded wait gave up.
// split = true: 3xTF32 (hi + lo operand parts), FP32-class accuracy.  scratch (may be null): where the
// products with both output dimensions >= 128 keep their operands split into TF32 tiles.
int cgemm_tf32(const GemmArgs& g, cudaStream_t s, double2* workspace, size_t workspace_elems, int* err_dev, bool split,
               TcScratch* scratch = nullptr);
inline bool precision_uses_tc(int p) { return p == DFTCUDA_PRECISION_TF32 || p == DFTCUDA_PRECISION_TF32X3; }
inline bool tc_worthwhile(int M, int N, int K, double min_flops) { return 8.0 * M * (double)N * K >= min_flops; }
size_t cgemm_tf32_workspace_elems(int M, int N, int K);
// Bytes of one operand's pre-split tiles (R rows of K entries) in the wide tensor-core GEMM.
size_t tc4_operand_bytes(int R, int K, bool split);

struct NonlocalDev {
  int nproj = 0;                 // sum over atoms of m_total(species)
  double2* P = nullptr;          // [nproj][npw] phi_m(g) exp(i G_g . tau_a)
  double* D = nullptr;           // per-projector row: D[(p)*maxm + j] = D_atom[p-off][j], j < mt(atom)
  int* proj_off = nullptr;       // [nproj] first projector of the atom owning p
  int* proj_mt = nullptr;        // [nproj] m_total of that atom
  int maxm = 0;
};

struct KCtxImpl;

// Device-time profiler (CUDA events on the launch stream), ScfProfile's counters.
enum ProfCat { P_PLANE_INV = 0, P_XLINE, P_PLANE_FWD, P_NL_PROJECT, P_NL_DIJ, P_NL_BACK, P_DENSITY, P_SUBSPACE, P_NCAT };

struct Profiler {
  struct Ev { int cat; cudaEvent_t a, b; };
  bool on = false;
  std::vector<Ev> pending;
  std::vector<cudaEvent_t> pool;
  double ns[P_NCAT] = {};
  uint64_t launches[P_NCAT] = {};
  uint64_t calls = 0, columns = 0;
  cudaEvent_t take();
  void resolve();
  void clear();
  void destroy();
};

}  // namespace dftcuda

// Column chunks of a host-buffer H|psi> call (copy in, compute, copy out overlapped).
constexpr int kPipeChunks = 8;

struct dftcuda_kctx {
  int nx, ny, nz;
  long N;        // nx*ny*nz
  int P;         // ny*nz, points per x-plane
  double volume;
  size_t npw;
  int precision;
  cudaStream_t stream = nullptr;
  int device = -1;                  // the CUDA device current when the context was created
  cudaEvent_t ev_order = nullptr;   // orders the context's stream after the caller's legacy-stream work
  // host-buffer H|psi>: the copies of a column chunk run on their own streams, overlapped with the
  // compute of the neighbouring chunks (created on first use)
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_in[kPipeChunks] = {}, ev_done[kPipeChunks] = {};
  dftcuda::Fft1dPlan fx, fy, fz;

  // G-sphere grouped by active x-plane ("slot").
  int n_act = 0;
  int* d_plane_off = nullptr;  // [n_act+1]
  int* d_pw_idx = nullptr;     // [npw] basis index, grouped by slot
  int* d_pw_spos = nullptr;    // [npw] pinv_z(z)*ny + pinv_y(y)
  int* d_slot_xpos = nullptr;  // [n_act] pinv_x(x) of each slot
  double* d_kinetic = nullptr;
  double* d_gcart = nullptr;   // [npw*3]
  std::vector<double> h_kinetic;

  // Four-step path tables (local4.cu): used when fast64 / fast32 is set for the precision.
  bool fast64 = false, fast32 = false;
  bool fft_generic = false;  // autotuner choice: the generic shared-memory FFT passes even where the four-step path exists
  bool sticks_off = false;   // autotuner choice: the plane layout even where the stick layout exists
  // TF32 / TF32X3 contexts: contractions of fewer useful FLOPs (8 M N K) than this run on the FP64
  // GEMM, where the operand split and its extra launches would cost more than the tensor cores save
  // (the FP64 result is within every mode's error bound).  DFTCUDA_TC_MIN_FLOP at creation overrides.
  double tc_min_flops = 5e8;
  int last_layout = -1;      // layout of the last H|psi>: 0 generic passes, 1 plane layout, 2 stick layout
  int split_proj = 0, split_back = 0;  // autotuner choices for the projector GEMMs (0 = heuristic)
  int precond_kind = 0;                // DFTCUDA_PRECOND_* of the Davidson correction step
  float* d_mlp = nullptr;              // learned preconditioner weights (DFTCUDA_PRECOND_MLP_PARAMS), then its z table
  double mlp_table_t = -1.0;           // iteration input the z table was built for (-1: none)
  double* d_vstage = nullptr;          // host V(r) staging (N doubles)
  int* d_pwmap = nullptr;      // [n_act][nz][ny] plane-wave index or -1
  int* d_stick_off = nullptr;  // [n_act+1]
  int* d_stick_y = nullptr;    // y of each stick, per slot, ascending
  int* d_slot_of_x = nullptr;  // [nx] slot of each x frequency or -1
  void* d_tw4x64 = nullptr;
  void* d_tw4x32 = nullptr;
  void* d_tw4p64 = nullptr;
  void* d_tw4p32 = nullptr;

  // Stick-layout passes (local_sticks.cu), used when sticks64 / sticks32 is set for the precision.
  bool sticks64 = false, sticks32 = false;
  int n_st = 0;                // sticks: (x, y) pairs holding plane waves, in slot order
  int* d_st_sy = nullptr;      // [n_st] slot << 16 | y
  int* d_st_map = nullptr;     // [n_st][nz] plane-wave index of (stick, z) or -1
  int* d_st_sox = nullptr;     // [nx] slot of each x frequency or -1
  void* d_twz64 = nullptr;     // twiddles of the z length
  void* d_twz32 = nullptr;
  void* d_twx64 = nullptr;     // twiddles of the x (= y) length
  void* d_twx32 = nullptr;
  double* d_vn = nullptr;      // V(r) in natural box order (x fastest), FP64 and FP32
  float* d_vn32 = nullptr;

  // Local potential transposed to [x][z][y]; FP32 copy for the FP32 passes.
  double* d_vt = nullptr;
  float* d_vt32 = nullptr;
  bool has_vloc = false;

  // Box workspace for a chunk of columns: [chunk][n_act][P] complex.
  void* d_box = nullptr;
  size_t box_bytes = 0;

  dftcuda::NonlocalDev nl;
  dftcuda::TcScratch tc_scratch;  // pre-split tensor-core GEMM operands (TF32 and TF32X3 contexts)
  dftcuda::TcScratch tc_ptiles_proj, tc_ptiles_back;  // the projector matrix split for the two projector GEMMs
  int natoms = 0;                   // atoms given to set_projectors
  std::vector<int> atom_row, atom_mt;  // per atom (set_projectors order): first projector row, row count
  std::vector<int> atom_species;       // per atom: species index
  std::vector<double> atom_pos;        // per atom: Cartesian position (bohr), 3 doubles
  std::vector<size_t> species_mt;      // per species: m_total
  double2* d_coef = nullptr;   // [nproj][cols] projector coefficients
  double2* d_coef2 = nullptr;
  size_t coef_cols = 0;
  double2* d_gemm_ws = nullptr;
  size_t gemm_ws_elems = 0;
  int* d_err = nullptr;  // device error flag of the bounded waits (TF32 tensor-core GEMMs)

  // Staging for host pointers.
  double2* d_x = nullptr;
  double2* d_y = nullptr;
  size_t stage_cols = 0;
  double* d_rho = nullptr;
  double* d_w = nullptr;
  size_t w_cap = 0;

  dftcuda::Profiler prof;

  // Eigensolver workspace (eig.cu).
  dftcuda::KCtxImpl* eig = nullptr;
  double w_budget_bytes = 96.0 * 1024 * 1024;  // box workspace target (stays L2-resident)
};

namespace dftcuda {

int kctx_apply_h_dev(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s);
int kctx_project(dftcuda_kctx* c, const double2* x, size_t ncols, cudaStream_t s);  // d_coef = P x
int kctx_ensure_coef(dftcuda_kctx* c, size_t cols);
int kctx_stage(dftcuda_kctx* c, size_t cols);
int kctx_check_error(dftcuda_kctx* c);
int kctx_density_dev(dftcuda_kctx* c, const double2* vecs, size_t nbands, const double* w_dev, double* rho_dev,
                     cudaStream_t s);
void eig_destroy(KCtxImpl* e);

// Davidson correction step q_b = P(r_b) for the chosen preconditioner (learned.cu).  ekin_ws: take
// doubles of scratch; t: the Davidson iteration index (an input of the learned preconditioner).
int precondition_launch(dftcuda_kctx* c, double2* Q, const double2* res, const double* kin, const double* lam,
                        const double* norms, const double2* ritz, const int* band, int take, long n, double t,
                        double* ekin_ws, cudaStream_t s);

// Hermitian eigensolver for the subspace problem (heev.cu): the nev lowest eigenpairs of an m x m
// Hermitian matrix (both triangles, column-major, destroyed), m <= 2048.
struct HeevWork {
  unsigned* bar = nullptr;  // grid barrier: count, generation
  double* d = nullptr;      // tridiagonal diagonal (m)
  double* e = nullptr;      // subdiagonal (m - 1)
  double* tnorm = nullptr;  // ||T|| bound
  double2* tau = nullptr;   // reflector scalars (m)
  double2* y = nullptr;     // tau A v (m)
  double* z = nullptr;      // eigenvectors of T (m x nev)
  double2* wy = nullptr;    // blocked back-transformation: V block, G, T, two W blocks, GEMM split-K space
  size_t wy_ws_elems = 0;   // the split-K part of wy (complex elements)
  size_t m_cap = 0, nev_cap = 0;
};
// 3D FFT of device data on stream s (fft_plan.cu): direction -1 forward unnormalised, +1 inverse / N.
int fft3d_on_stream(dftcuda_fft_plan* pl, double2* d, int direction, cudaStream_t s);
size_t heev_work_bytes(int m, int nev);
void heev_bind(HeevWork& w, void* base, int m, int nev);
int heev_lowest(double2* A, int m, int nev, double* evals, double2* E, long lde, const HeevWork& w, int* status,
                cudaStream_t s);
int hermitian_upper_to_full(const double2* src, long lds, double2* A, int m, cudaStream_t s);

// Four-step register-FFT path (local4.cu).
bool kctx_fast_path_ok(const dftcuda_kctx* c, int precision);
int kctx_setup_fast_path(dftcuda_kctx* c, const std::vector<int>& slot_of_x, const std::vector<int>& xpos,
                         const int32_t* hkl);
template <typename T> int local_block4(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s);
// Stick-layout passes (local_sticks.cu).
bool kctx_sticks_ok(const dftcuda_kctx* c, int precision);
int kctx_setup_sticks(dftcuda_kctx* c, const std::vector<int>& slot_of_x, const std::vector<int>& xpos, const int32_t* hkl);
size_t sticks_bytes_per_col(const dftcuda_kctx* c, size_t cs);
template <typename T> int local_block_sticks(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s);
bool kctx_sticks_density_ok(const dftcuda_kctx* c, int precision);
template <typename T>
int density_block_sticks(dftcuda_kctx* c, const double2* x, size_t ncols, const double* w, double* rho, cudaStream_t s);
template <typename T>
int density_block4(dftcuda_kctx* c, const double2* x, size_t ncols, const double* w, double* rho, cudaStream_t s);

// Times the launches between construction and destruction under category `cat` when profiling is on.
struct ProfScope {
  dftcuda_kctx* c;
  int cat;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  uint64_t l0 = 0;
  ProfScope(dftcuda_kctx* c_, int cat_, cudaStream_t s_) : c(c_), cat(cat_), s(s_) {
    if (!c->prof.on) return;
    a = c->prof.take();
    cudaEventRecord(a, s);
    l0 = launches_total();
  }
  void stop() {
    if (!a) return;
    cudaEvent_t b = c->prof.take();
    cudaEventRecord(b, s);
    c->prof.pending.push_back({cat, a, b});
    c->prof.launches[cat] += launches_total() - l0;
    a = nullptr;
  }
  ~ProfScope() { stop(); }
};

}  // namespace dftcuda

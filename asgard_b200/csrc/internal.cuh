// Internal declarations shared by the asgard_b200 CUDA sources.
#pragma once

#include "asgard_b200.h"

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <vector>

namespace asgk
{
// Launch counter (all kernels launched by this library).  While a thread
// records a GMRES cycle into a graph its launches run later, so they go to a
// per-thread tally instead (the solver counts them per executed step).
extern std::atomic<int64_t> g_launches;
extern thread_local bool g_recording;
extern thread_local int64_t g_recorded_launches;
inline void count_launch(int64_t k = 1)
{
  if (g_recording)
    g_recorded_launches += k;
  else
    g_launches.fetch_add(k, std::memory_order_relaxed);
}

// While a GMRES cycle is recorded with several Arnoldi steps per graph node,
// every kernel of a step is handed the cycle's "go" flag and returns at once
// when it is 0 (the cycle stopped at an earlier step of the node): the
// recorder sets g_gate around those launches and the launchers pass it on
// (null otherwise: no check).
extern thread_local const double *g_gate;
#ifdef __CUDACC__
__device__ __forceinline__ bool gate_closed(const double *gate)
{
  return gate != nullptr && *gate == 0.0;
}
#endif

#define ASGK_CUDA(call)                                                        \
  do                                                                           \
  {                                                                            \
    cudaError_t asgk_err_ = (call);                                            \
    if (asgk_err_ != cudaSuccess)                                              \
    {                                                                          \
      std::fprintf(stderr, "asgard_b200: %s failed: %s (%s:%d)\n", #call,      \
                   cudaGetErrorString(asgk_err_), __FILE__, __LINE__);         \
      return ASGK_ERR_CUDA;                                                    \
    }                                                                          \
  } while (0)

#define ASGK_LAUNCHED()                                                        \
  do                                                                           \
  {                                                                            \
    cudaError_t asgk_err_ = cudaGetLastError();                                \
    if (asgk_err_ != cudaSuccess)                                              \
    {                                                                          \
      std::fprintf(stderr, "asgard_b200: launch failed: %s (%s:%d)\n",         \
                   cudaGetErrorString(asgk_err_), __FILE__, __LINE__);         \
      return ASGK_ERR_CUDA;                                                    \
    }                                                                          \
    ::asgk::count_launch();                                                    \
  } while (0)

// Entries of a global-form neighbour list handled by one CTA (4 warps for
// tensors of up to 81 entries, 8 above).  Measured at d=3/4, level 7: 64
// beats 16, 32 and 128.
constexpr int kGlobalSliceMax = 64;
constexpr int global_slice(int) { return 64; }

// How the factor blocks of a pair are addressed.
enum class index_mode : int
{
  expanded = 0, // iA[(p*T + t)*d + k]: reference layout, any offsets
  conn     = 1  // conn[p*d + k]*(d*T*n*n) + (t*d + k)*n*n: sparse-grid layout
};

// kron_tc.cu: the tensor-core (BF16) form of a global plan's operator
struct tc_data;

// Device-resident operator.  Pairs are grouped by output cell (CSR) and the
// cells are visited in order of decreasing pair count.
struct plan_data
{
  int d = 0, n = 0, rows = 0, cols = 0, terms = 0;
  int tensor = 0;      // n^d
  int64_t nnz = 0;     // number of (row, col) pairs
  index_mode mode = index_mode::expanded;
  int64_t vA_len = 0;

  int64_t *row_ptr = nullptr; // [rows + 1]
  int *col     = nullptr;     // [nnz] column cell per pair
  int *idx     = nullptr;     // [nnz*T*d] (expanded) or [nnz*d] (conn)
  int *row_order = nullptr;   // [rows] cells by decreasing pair count
  double *vA64 = nullptr;     // [vA_len]
  float *vA32  = nullptr;     // [vA_len]
  // sparse-grid plans with n = 3: the factors repacked per (connection,
  // dimension) with the T terms contiguous, each 3 x 3 block padded to a
  // 16-byte multiple (10 doubles / 12 floats) for vector loads
  int64_t nconn = 0;
  double *vP64  = nullptr;    // [nconn][d][T][10]
  float *vP32   = nullptr;    // [nconn][d][T][12]

  // FP64 staging buffers of apply_host: allocated on first use, or the
  // caller's (set_workspace; then not owned)
  double *xw = nullptr, *yw = nullptr;
  bool ws_owned = true;
  // x repacked for the staged kernel (n = 3, d = 3/4): padded slices
  double *xs = nullptr;

  // global mode (every term acts in at most one dimension; n = 3): per
  // output cell its neighbours along one dimension (gptr/gcol), each with
  // the index conn*d + k of a 3x3 block pre-summed over the terms acting in
  // dimension k (gkb); the pair list above then holds only the diagonal
  // pairs, for the Jacobi preconditioners
  bool global = false;
  int64_t gnnz = 0;
  int64_t *gptr = nullptr;
  int *gcol = nullptr, *gkb = nullptr;
  double *gB64 = nullptr; // [nconn*d][10]
  float *gB32  = nullptr; // [nconn*d][12]
  double g_identity = 0;  // number of terms that are the identity
  std::vector<int> g_conn_row, g_conn_col; // 1D cells of each 1D connection
  // the neighbour lists cut into slices of at most global_slice(d) entries, one
  // CTA each; slices of one cell have consecutive ids (heavy cells first)
  int gslices = 0;
  int *slice_row = nullptr, *slice_len = nullptr;  // [gslices]
  int64_t *slice_beg = nullptr;                    // [gslices]
  int *row_slice0 = nullptr, *row_nslice = nullptr; // [rows]
  double *gscratch = nullptr;  // [gslices * n^d] partial tensors
  unsigned *gtickets = nullptr; // [rows], zero between launches
  // d >= 5: one CTA per cell, its warps sharing the cell's neighbour list
  // (kron_global_cell): each cell's segment of the list per dimension, the
  // cell orders the FP32 and FP64 kernels take, and the FP32 copy of x
  // the FP32 apply reads its neighbour tensors from (L2-resident)
  int *gseg = nullptr;         // [rows][d + 1] offsets within the cell's list
  int *gcell_order = nullptr;  // [2][rows]: by longest segment, by entries
  float *gx32 = nullptr;       // [rows * n^d]
  // the vector whose FP32 copy gx32 holds when a preconditioner wrote it
  // with its output (consumed, and cleared, by the next FP32 global apply)
  mutable const double *gx32_src = nullptr;
  // terms acting in several dimensions (the reference's upper/lower
  // permutations): chains of masked 1D passes over per-dimension neighbour
  // lists.  Stage s runs the jobs gjobs[stage_job0[s] ..] (chain, dimension,
  // fill 0 upper / 1 both / 2 lower, term); chain outputs alternate between
  // two buffers of gchains vectors, chain c's result is in buffer
  // gchain_last[c].
  std::vector<std::vector<int>> g_multi; // (term, its dimensions) per such term
  int gchains = 0;
  std::vector<int> stage_job0, stage_njobs;
  int4 *gjobs = nullptr;
  int *gchain_last = nullptr;
  int64_t *gd_ptr = nullptr;       // [d][rows + 1]
  int *gd_col = nullptr, *gd_conn = nullptr;
  unsigned char *gd_rel = nullptr; // neighbour's 1D cell: 0 before, 1 same, 2 after
  double *gwork = nullptr;         // 2 * gchains * rows * n^d values
  int64_t gchain_entries = 0;      // neighbour entries the chains' stages visit

  // the tensor-core form of a global plan (precision ASGK_BF16): pencils,
  // their BF16 class matrices and its vectors, built on first use
  mutable tc_data *tc = nullptr;

  // dense mode (every (row, col) pair): a conn-mode plan whose connection
  // index in dimension k is elem_col[k] * dense_nb + elem_row[k], the factors
  // of the caller's per-term arrays repacked to the per-connection layout
  bool dense   = false;
  int dense_nb = 0;
  int64_t device_bytes = 0;
};

} // namespace asgk

struct asgk_plan
{
  asgk::plan_data p;
};

namespace asgk
{
// kron_kernels.cu
int launch_apply(plan_data const &p, int precision, double alpha,
                 const void *x, int x_is_f32, double beta, void *y,
                 int y_is_f32, double euler_x_coeff, cudaStream_t s);

// grid.cpp: cell pairs that differ in at most one dimension
struct direction_pairs
{
  int d = 0, nconn = 0;
  std::vector<int64_t> ptr;     // [cells + 1]
  std::vector<int> col, dim, conn; // per entry: neighbour cell, dimension, 1D connection
  std::vector<int> self_conn;   // [cells][d] the self-connection index
  std::vector<int> conn_row, conn_col; // 1D cells of each 1D connection
};
int build_direction_pairs(int d, int level, int num_cells, const int *table,
                          direction_pairs &out);

// grid_device.cu: connected cell pairs on the device.  oned: [cells][d] 1D
// cell indices; cand: the candidate cells in the order each row's pairs are
// written; lut: [R][R] 1D connection index or -1
int launch_count_pairs(int d, int cells, const int *oned, const int *cand,
                       const int *lut, int R, int64_t *counts, cudaStream_t s);
int launch_fill_pairs(int d, int cells, const int *oned, const int *cand,
                      const int *lut, int R, const int64_t *row_ptr, int *col,
                      int *conn, cudaStream_t s);

// jacobi.cu
struct jacobi_data;
// z = M v; with scale_state, v *= scale_state[1] in place first (the
// normalisation of a recorded GMRES step's new basis vector, fused), and
// with vcopy also vcopy = FP32(v) (the basis copy of FP32 inner solves).
// zcopy (the line preconditioner only, else ignored): also zcopy = FP32(z),
// the FP32 copy of x the next FP32 global apply reads
int jacobi_apply(jacobi_data const &jd, bool low, double *v, double *z,
                 const double *scale_state, float *vcopy, cudaStream_t s,
                 float *zcopy = nullptr);
int jacobi_apply_handle(asgk_jacobi *pc, bool low, double *v, double *z,
                        const double *scale_state, float *vcopy,
                        cudaStream_t s, float *zcopy = nullptr);
// whether jacobi_apply writes zcopy
bool jacobi_writes_zcopy(const asgk_jacobi *pc);
// never reused within a process: identifies a preconditioner in caches
uint64_t jacobi_serial(const asgk_jacobi *pc);
// ASGK_OK when the preconditioner applies to vectors of rows * tensor
// values (the shape of the plan it was built on), else ASGK_ERR_INVALID:
// its kernels index their own tables by the cells of that plan and read and
// write rows * tensor values of v and z
int jacobi_check_shape(const asgk_jacobi *pc, int rows, int tensor);
// the step size the preconditioner inverts I - dt*K for
double jacobi_dt(const asgk_jacobi *pc);

// jacobi_line.cu: the line preconditioner (ASGK_JACOBI_LINE)
struct line_data;
int line_build(plan_data const &p, double dt, line_data **out, int64_t &bytes);
void line_free(line_data *ld);
int line_apply(line_data const &ld, bool low, double *v, double *z,
               const double *scale_state, float *vcopy, float *zcopy,
               cudaStream_t s);
// the line dimensions (up to 3) into dims; returns how many
int line_info(line_data const &ld, int *dims);

// kron_global.cu: global-mode apply
int launch_global(plan_data const &p, int precision, double alpha,
                  const double *x, double beta, double *y, double ex,
                  cudaStream_t s);

// kron_tc.cu: the tensor-core form (tcgen05, BF16 operands, FP32 TMEM
// accumulators) of a global plan whose terms act in one dimension each.
// tc_prepare builds it once (host work and allocations: call it outside
// stream capture); tc_refresh rewrites its matrices after new values.
int tc_build(plan_data const &p, tc_data **out);
int tc_prepare(plan_data const &p);
int tc_refresh(plan_data const &p, tc_data &t);
void tc_free(tc_data *t);
// device memory the tensor-core form holds (0 before its first use)
int64_t tc_bytes(const tc_data *t);
int tc_read_error(int reset, int *code);
int launch_global_tc(plan_data const &p, double alpha, const double *x, double beta,
                     double *y, double ex, cudaStream_t s);

// kron_staged.cu: n = 3, d = 3/4 apply with bulk-copied x tensors
bool staged_supported(plan_data const &p);
int64_t staged_x_doubles(int d, int n, int cols); // 0: no staged kernel
int launch_staged(plan_data const &p, int precision, double alpha,
                  const double *x, double beta, double *y, double ex,
                  cudaStream_t s);
// the device-side error word written by bounded waits that expired
int read_device_error(int reset, int *code);

// krylov.cu: BLAS-1/2 pieces of the device-resident GMRES
int launch_fill(double *v, int64_t n, double value, cudaStream_t s);
int launch_copy(double *dst, const double *src, int64_t n, cudaStream_t s);
int launch_scale(double *v, int64_t n, double alpha, cudaStream_t s);
int launch_axpy(double *y, const double *x, int64_t n, double alpha,
                cudaStream_t s);
// Gram-Schmidt passes that finish their reductions in their last block:
// h[0..k) = V^T w; w -= V h with *out = ||w||^2; *out = ||v||^2.  tickets:
// zero-initialised counters, (k+7)/8 of them for the multi-dot, one for
// the others (left at zero after each launch)
int launch_multidot_h(const double *V, int64_t ldv, int k, const double *w,
                      int64_t n, double *part, unsigned *tickets, double *h,
                      cudaStream_t s);
struct givens_args; // gmres_device.cuh: the Givens update of a recorded step
int launch_update_norm_h(const double *V, int64_t ldv, int k, const double *h,
                         double *w, int64_t n, double *part, unsigned *ticket,
                         double *out, cudaStream_t s,
                         givens_args const *ga = nullptr);
int launch_norm2_h(const double *v, int64_t n, double *part, unsigned *ticket,
                   double *out, cudaStream_t s);
// the same two passes over an FP32 copy of the basis (w, h, sums FP64)
int launch_multidot_hf(const float *V, int64_t ldv, int k, const double *w,
                       int64_t n, double *part, unsigned *tickets, double *h,
                       cudaStream_t s);
int launch_update_norm_hf(const float *V, int64_t ldv, int k, const double *h,
                          double *w, int64_t n, double *part, unsigned *ticket,
                          double *out, cudaStream_t s,
                          givens_args const *ga = nullptr);
// w *= f, vf = FP32(w); f = state[1] when state is set, else scale
int launch_store_basis(double *w, float *vf, int64_t n, const double *state,
                       double scale, cudaStream_t s);
// v *= state[1], the scale a recorded GMRES step computed on the device
int launch_scale_by(double *v, int64_t n, const double *state, cudaStream_t s);
int launch_xpby(double *y, const double *x, int64_t n, double beta,
                cudaStream_t s);
// partial sums of V[:,0..k)^T w into part[blocks][k]; returns blocks used
int launch_multidot(const double *V, int64_t ldv, int k, const double *w,
                    int64_t n, double *part, int *blocks, cudaStream_t s);
// out[j] = sum_b part[b][j]
int launch_reduce_parts(const double *part, int blocks, int k, double *out,
                        cudaStream_t s);
// w -= V[:,0..k) h; part[b] = partial sum of w^2 after the update
int launch_update_norm(const double *V, int64_t ldv, int k, const double *h,
                       double *w, int64_t n, double *part, int *blocks,
                       cudaStream_t s);
// part[b] = partial sums of v^2
int launch_norm2(const double *v, int64_t n, double *part, int *blocks,
                 cudaStream_t s);
// x += V[:,0..k) y
int launch_gemv_add(const double *V, int64_t ldv, int k, const double *y,
                    double *x, int64_t n, cudaStream_t s);
int max_reduction_blocks();
// partial sums per column of the self-reducing Gram-Schmidt passes
int max_reduction_blocks_wide();

} // namespace asgk

// h2g_solver.cu -- host side of the B200 solver library: handle, operator tables, CUDA-graph
// drivers for PBiCGSTAB!/CG! (src/NonUniform.jl:115-350) and the C ABI of include/h2g.h.
//
// One solve = one kernel (the initial residual) + one graph launch.  The graph holds a single
// conditional WHILE node whose body is one Krylov iteration (about two dozen kernels); all
// scalars (rho, alpha, omega, beta, the residual and the stop decision) live in device memory
// and the last kernel of the body sets the loop condition, so the host does not synchronise
// between iterations.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <map>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <utility>
#include <string>
#include <thread>
#include <vector>

#include "../../include/h2g.h"
#include "h2g_sweep.cuh"
#include "h2g_multi.cuh"
#include "h2g_coop.cuh"

namespace h2g {

static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return fail(H2G_CUDA_ERROR, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                       __FILE__, __LINE__);                                           \
  } while (0)

#define CKL()                                                                                             \
  do {                                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                                  \
    if (e_ != cudaSuccess) return fail(H2G_CUDA_ERROR, "launch: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, \
                                       __LINE__);                                                         \
  } while (0)

// Graph of one solve: parent graph {WHILE node}, body = kUnroll iterations (SOR: one pass).
struct SolveGraph {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  bool cond = false;  // true: conditional WHILE node; false: body graph launched by a host loop
  std::vector<unsigned char> sig;
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    sig.clear();
  }
};

#ifndef H2G_UNROLL
#define H2G_UNROLL 4
#endif
constexpr int kUnroll = H2G_UNROLL;  // Krylov iterations per captured loop-body pass
static_assert(kUnroll % 2 == 0, "p ping-pongs between two buffers: an even number of iterations per pass");

enum GraphKind {
  kGPbicg64 = 0, kGCg64 = 1, kGPbicg32 = 2, kGCg32 = 3, kGPbicgMx = 4, kGCgMx = 5, kGSor = 6, kGNum = 7
};

template <typename T>
struct OpTables {
  T* tx = nullptr;
  T* ty = nullptr;
  T* tz = nullptr;
  T* conv = nullptr;
  T* dzk = nullptr;
  T* ddv = nullptr;  // dd per cell (device layout)
  T* tq = nullptr;   // interleaved x, y, z-, z+ tables (fused sweeps)
  int pcap = 0;
};

struct Solver {
  Geo g{};
  int precision = H2G_FP64;
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t cap = nullptr;  // capture stream
  bool grid_set = false, fields_set = false;
  // grid (host)
  std::vector<double> ZC, dZ;
  double dx = 0, dy = 0, dt = 0, HC[6] = {0, 0, 0, 0, 0, 0};
  int steady = 1;
  // keys
  uint8_t* key = nullptr;
  unsigned long long* nkey = nullptr;  // the 7 stencil keys of every cell (smoother)
  int P = 0;
  std::vector<double> lam_values;
  unsigned long long* slots = nullptr;
  int* slot_index = nullptr;
  int* flags = nullptr;
  OpTables<double> t64;
  OpTables<float> t32;
  // rho*cp per cell (device layout) for transient grids; independent of the key tables
  double* rc64 = nullptr;
  float* rc32 = nullptr;
  bool rc_valid = false;
  // FP64 state vectors (device layout)
  double* th = nullptr;
  double* b = nullptr;
  double* th_snap = nullptr;
  double* r64 = nullptr;
  double* hsrc = nullptr;      // heat source per cell (device layout), set by h2g_set_hsrc
  double* th_prev = nullptr;   // theta before a mixed-precision pass (restored on breakdown)
  double* stats = nullptr;     // per-step theta statistics of the transient driver
  int stats_cap = 0;
  double* adj[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // adjoint: w, g, la, G, dJ/dhsrc
  double* lamv = nullptr;      // lambda value of every material key (adjoint gradient)
  double* tstates = nullptr;   // transient adjoint: checkpoints, segment states, final state
  size_t tstates_cap = 0;      // in vectors
  // Krylov vectors in working precision: r, r0, p, ph, q, s, sh, t (+ e for refinement, the FP32
  // right-hand side of the mixed smoother, and p's second buffer: the fused first sweep reads the
  // old p at its overlap cells, so p ping-pongs between two buffers from iteration to iteration)
  void* kv[11] = {nullptr};
  void* hook[3] = {nullptr, nullptr, nullptr};  // scratch of the single-kernel entry points (never a Krylov vector)
  bool hook_filled = false;            // hook[] holds the benchmark's non-zero scratch values
  unsigned bench_parity = 0;           // direction of the next fused benchmark sweep
  size_t elem = 8;
  // column-major staging buffers (MX*MY*MZ doubles each)
  double* stage[4] = {nullptr, nullptr, nullptr, nullptr};
  // device scalars
  SolverState* st = nullptr;     // outer / FP64 solve
  SolverState* st_in = nullptr;  // inner FP32 solve
  SolverState* st_host = nullptr;  // pinned mirror
  double* partials = nullptr;
  size_t partials_cap = 0;
  double* hist = nullptr;
  int hist_cap = 0;
  SolveGraph graphs[kGNum][2];
  // mixed-precision refinement settings
  double inner_tol = 1e-4;
  int max_outer = 40;
  bool no_cond = false;
  bool pdl = true;  // programmatic dependent launch of the solver kernels
  int rb_rows = kBY;      // rows per block of the colour pass (autotuned)
  int rb_planes = 2;      // planes per thread of the colour pass (autotuned)
  bool rb_dd = true;      // colour pass reads dd from the per-cell array (autotuned)
  bool ax_dd = false;     // CalcAX reads dd from the per-cell array (autotuned)
  bool rb_cls = false;    // FP64 colour passes read the stencil-class table (autotuned)
  bool ax_cls = false;    // FP64 CalcAX reads the stencil-class table (autotuned)
  // stencil classes of the FP64 operator (k_class_*): per-cell index, table, build scratch
  bool cls_ok = false;    // the grid's classes are built (at most kMaxClasses, NZ <= 255)
  // operator data rebuilt only when its inputs change (build_tables): the inputs of the last
  // build, and whether h2g_set_fields produced a key array different from the last one
  std::vector<unsigned char> tables_sig;
  bool keys_changed = true;
  uint8_t* key_prev = nullptr;
  int* kdiff = nullptr;
  int ncls = 0;
  uint16_t* cls = nullptr;
  double* ctab = nullptr;
  float* ctab32 = nullptr;  // the FP32 smoother's rows (mixed handles)
  unsigned long long* cslots = nullptr;
  uint16_t* slot_class = nullptr;
  unsigned long long* cwords = nullptr;
  int* cflag = nullptr;
  bool rb_tuned = false;  // rb_rows chosen (by the tuner or h2g_set_tuning)
  // fused sweeps (k_rb_sweep): sweeps 2-5 of the preconditioner as one launch each, ping-ponging
  // between the preconditioner's output and x2 (one per precision; guards zero, never written)
  bool rb_fused = false;   // autotuned
  int sw_chunks = 1;       // z chunks of the fused sweep's grid (autotuned)
  bool sw_dda = false;     // the fused sweep reads dd from the array (autotuned)
  int sweep_forced = -1;   // h2g_set_sweep: -1 tuner, 0 colour passes, 1 fused
  double* x2_64 = nullptr;
  float* x2_32 = nullptr;
  int* sweep_err = nullptr;            // set by a fused sweep or grid barrier whose bounded wait ran out
  // cooperative preconditioner (k_precond_coop): all 10 passes of Preconditioner! in one launch
  int rb_coop = 0;          // chosen (tuner or h2g_set_coop)
  int coop_forced = -1;     // h2g_set_coop: -1 tuner, 0 off, 1 on
  double div_limit = 0.0;   // divergence stop of the next solves' states (mixed FP32 passes only)
  int coop_blocks = 0;      // blocks of the launch: SMs x resident blocks per SM
  bool coop_barred = false; // set while h2g_batch_solve runs the handle beside others
  GridBar* gbar = nullptr;
  long long wait_limit = kWaitCycles;  // budget of one bounded wait (clock cycles)
  std::map<std::pair<const void*, int>, CUtensorMap> xmaps;  // TMA maps of x buffers (pointer, bytes/element)
  // K right-hand sides on the handle's operator (h2g_create_multi): stacked vectors, K states
  int nrhs = 0;
  double* mr_th = nullptr;
  double* mr_b = nullptr;
  double* mr_kv[8] = {nullptr};  // r, r0, p, p_, q, s, s_, t
  SolverState* mr_st = nullptr;
  MultiCtl* mr_ctl = nullptr;
  double* mr_partials = nullptr;
  int* mr_flag = nullptr;
  SolveGraph mr_graph;
  CUtensorMap kmap;                    // TMA map of the key array
  bool kmap_ok = false;

  long long nfort() const { return (long long)g.MX * g.MY * g.MZ; }
};

}  // namespace h2g

// The opaque handle of include/h2g.h is the solver itself.
struct h2g_solver : public h2g::Solver {};

namespace h2g {

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------
// Kernel launch with programmatic stream serialization: inside the captured iteration graph the
// edges become programmatic, so each kernel's launch overlaps the tail of the one before it
// (the kernels wait for their predecessor with griddepcontrol.wait).
template <typename... KArgs, typename... Args>
static void launch(const Solver* s, void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t stream,
                   Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = s->pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}
static int elementwise_blocks(const Solver* s) { return s->num_sms * 4; }


// Grids of the stencil kernels: columns (p, j) in 32 x kBY blocks; the RB passes take two planes
// per thread, CalcAX / CalcRK / the first pass one plane (both colours).
static dim3 rb_grid(const Geo& g, int by = kBY) {
  return dim3((g.HN + kBX - 1) / kBX, (g.NY + by - 1) / by, (g.NZ + 1) / 2);
}
static dim3 ax_grid(const Geo& g) { return dim3((g.HN + kBX - 1) / kBX, (g.NY + kBY - 1) / kBY, g.NZ); }
static dim3 first_grid(const Geo& g) { return ax_grid(g); }

// CalcAX with the handle's choice of dd source.
template <typename T, int NDOT, typename TI>
static void launch_ax(const Solver* s, cudaStream_t cs, const OpParams<T>& op, T* y, const TI* x, const T* u,
                      const T* w, SolverState* st, int stage) {
  const dim3 ag((op.g.HN + kBX - 1) / kBX, (op.g.NY + kBY - 1) / kBY, op.g.NZ), blk(kBX, kBY);
  if constexpr (sizeof(T) == 8) {
    if (s->ax_cls && op.cls) {
      launch(s, k_ax<T, NDOT, TI, 2>, ag, blk, cs, op, y, x, u, w, st, s->partials, stage);
      return;
    }
  }
  if (s->ax_dd) launch(s, k_ax<T, NDOT, TI, 1>, ag, blk, cs, op, y, x, u, w, st, s->partials, stage);
  else launch(s, k_ax<T, NDOT, TI, 0>, ag, blk, cs, op, y, x, u, w, st, s->partials, stage);
}

// One colour pass with the handle's launch shape (rows per block, planes per thread) and source of
// the coefficients (DDM as in k_rb_pass).
template <typename T, int NP, int DDM>
static void launch_rb_np(const Solver* s, cudaStream_t cs, const OpParams<T>& op, T* x, const T* bb, int color,
                         T omega, const SolverState* st) {
  const Geo& g = op.g;
  const int gz = (g.NZ + NP - 1) / NP;
  const int gx = (g.HN + kBX - 1) / kBX;
  switch (s->rb_rows) {
    case 2:
      launch(s, k_rb_pass<T, 2, NP, DDM>, dim3(gx, (g.NY + 1) / 2, gz), dim3(kBX, 2), cs, op, x, bb, color, omega, st);
      break;
    case 4:
      launch(s, k_rb_pass<T, 4, NP, DDM>, dim3(gx, (g.NY + 3) / 4, gz), dim3(kBX, 4), cs, op, x, bb, color, omega, st);
      break;
    case 16:
      launch(s, k_rb_pass<T, 16, NP, DDM>, dim3(gx, (g.NY + 15) / 16, gz), dim3(kBX, 16), cs, op, x, bb, color, omega,
             st);
      break;
    default:
      launch(s, k_rb_pass<T, 8, NP, DDM>, dim3(gx, (g.NY + 7) / 8, gz), dim3(kBX, 8), cs, op, x, bb, color, omega, st);
      break;
  }
}
template <typename T, int DDM>
static void launch_rb_dd(const Solver* s, cudaStream_t cs, const OpParams<T>& op, T* x, const T* bb, int color,
                         T omega, const SolverState* st) {
  if (s->rb_planes == 1) launch_rb_np<T, 1, DDM>(s, cs, op, x, bb, color, omega, st);
  else launch_rb_np<T, 2, DDM>(s, cs, op, x, bb, color, omega, st);
}
template <typename T>
static void launch_rb(const Solver* s, cudaStream_t cs, const OpParams<T>& op, T* x, const T* bb, int color, T omega,
                      const SolverState* st) {
  if (s->rb_cls && op.cls) {
    launch_rb_dd<T, 2>(s, cs, op, x, bb, color, omega, st);
    return;
  }
  if (s->rb_dd) launch_rb_dd<T, 1>(s, cs, op, x, bb, color, omega, st);
  else launch_rb_dd<T, 0>(s, cs, op, x, bb, color, omega, st);
}

// ---- fused sweep (k_rb_sweep) ---------------------------------------------------------------
// cuTensorMapEncodeTiled from the driver, looked up through the runtime (the library does not
// link libcuda itself).
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;

static int tensor_encoder() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    cudaGetLastError();
  });
  return g_encode ? H2G_OK : fail(H2G_CUDA_ERROR, "cuTensorMapEncodeTiled is not available");
}

// 3-D map over a device-layout vector: (positions HP, half-rows 2*MY, planes MZ); the box is one
// staged plane of k_rb_sweep.  Out-of-range coordinates read as zero.
static int encode_map(const Solver* s, const void* base, int esize, CUtensorMap* m) {
  if (int rc = tensor_encoder()) return rc;
  const Geo& g = s->g;
  const cuuint64_t dims[3] = {(cuuint64_t)g.HP, (cuuint64_t)(2 * g.MY), (cuuint64_t)g.MZ};
  const cuuint64_t strides[2] = {(cuuint64_t)g.HP * esize, (cuuint64_t)(2 * g.MY) * g.HP * esize};
  const cuuint32_t box[3] = {(cuuint32_t)(esize == 8 ? SwCfg<double>::WX : esize == 4 ? SwCfg<float>::WX : kSwWK),
                             (cuuint32_t)kSwRR, 1u};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  const CUtensorMapDataType dt = esize == 8   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                 : esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                              : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  const CUresult r = g_encode(m, dt, 3, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(H2G_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return H2G_OK;
}

template <typename T>
static int xmap(Solver* s, const T* base, const CUtensorMap** out) {
  const auto key = std::make_pair((const void*)base, (int)sizeof(T));
  auto it = s->xmaps.find(key);
  if (it == s->xmaps.end()) {
    CUtensorMap m;
    if (int rc = encode_map(s, base, (int)sizeof(T), &m)) return rc;
    it = s->xmaps.emplace(key, m).first;
  }
  *out = &it->second;
  return H2G_OK;
}

static int kmap(Solver* s, const CUtensorMap** out) {
  if (!s->kmap_ok) {
    if (int rc = encode_map(s, s->key, 1, &s->kmap)) return rc;
    s->kmap_ok = true;
  }
  *out = &s->kmap;
  return H2G_OK;
}

// the fused sweep's dynamic shared memory (above the 48 KiB default), once per process
static int sweep_attrs() {
  static std::once_flag once;
  static cudaError_t e = cudaSuccess;
  std::call_once(once, [] {
    cudaError_t r[4] = {
        cudaFuncSetAttribute(k_rb_sweep<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SwCfg<double>::SMEM),
        cudaFuncSetAttribute(k_rb_sweep<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SwCfg<double>::SMEM),
        cudaFuncSetAttribute(k_rb_sweep<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SwCfg<float>::SMEM),
        cudaFuncSetAttribute(k_rb_sweep<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SwCfg<float>::SMEM)};
    for (cudaError_t x : r)
      if (x != cudaSuccess) e = x;
  });
  if (e != cudaSuccess) return fail(H2G_CUDA_ERROR, "fused sweep attributes: %s", cudaGetErrorString(e));
  return H2G_OK;
}

static dim3 sweep_grid(const Geo& g, int chunks) {
  const int kc = (g.NZ + chunks - 1) / chunks;
  return dim3((g.HI + kSwTPX - 3) / (kSwTPX - 2), (g.NY + kSwTJ - 3) / (kSwTJ - 2), (g.NZ + kc - 1) / kc);
}

// One fused RB-GS sweep xout <- sweep(xin) with right-hand side bb.  The tensor maps are encoded
// on the host when a buffer is first seen (also during stream capture: no stream work).
template <typename T>
static int launch_sweep(Solver* s, cudaStream_t cs, const OpParams<T>& op, const T* xin, T* xout, const T* bb,
                        SolverState* st) {
  const CUtensorMap *mx = nullptr, *mk = nullptr;
  if (int rc = xmap<T>(s, xin, &mx)) return rc;
  if (int rc = kmap(s, &mk)) return rc;
  const Geo& g = op.g;
  const int kc = (g.NZ + s->sw_chunks - 1) / s->sw_chunks;
  const dim3 grid = sweep_grid(g, s->sw_chunks), blk(kSwTPX, kSwTJ);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = blk;
  cfg.dynamicSmemBytes = SwCfg<T>::SMEM;
  cfg.stream = cs;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = s->pdl ? 1 : 0;
  if (s->sw_dda)
    cudaLaunchKernelEx(&cfg, k_rb_sweep<T, true>, op, *mx, *mk, xout, bb, kc, st, s->sweep_err, s->wait_limit);
  else
    cudaLaunchKernelEx(&cfg, k_rb_sweep<T, false>, op, *mx, *mk, xout, bb, kc, st, s->sweep_err, s->wait_limit);
  return H2G_OK;
}

// H2G_TIMEOUT (and the flag and grid barrier reset) if a bounded wait of a fused sweep or of the
// cooperative preconditioner's grid barrier ran out since the last check.
static int sweep_status(Solver* s) {
  int e = 0;
  CK(cudaMemcpy(&e, s->sweep_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (!e) return H2G_OK;
  CK(cudaMemset(s->sweep_err, 0, sizeof(int)));
  CK(cudaMemset(s->gbar, 0, sizeof(GridBar)));
  return fail(H2G_TIMEOUT, "a bounded wait of the RB-GS preconditioner ran out");
}

// Blocks of the cooperative preconditioner: every SM's resident blocks, so that all of them run
// at once (the cooperative launch checks it).
template <int VM, int NP, int DDM>
static int coop_grid(Solver* s) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_precond_coop<VM, NP, DDM>, kThreads, 0) != cudaSuccess ||
      per_sm < 1)
    return 0;
  return per_sm * s->num_sms;
}

template <int VM, int NP, int DDM>
static int launch_coop_np(Solver* s, cudaStream_t cs, const OpParams<double>& op, double* xx, double* v,
                          const double* r, const double* q, SolverState* st) {
  const int nblk = coop_grid<VM, NP, DDM>(s);
  if (nblk < 1) return fail(H2G_CUDA_ERROR, "no resident block for the cooperative preconditioner");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblk);
  cfg.blockDim = dim3(kBX, kBY);
  cfg.stream = cs;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, k_precond_coop<VM, NP, DDM>, op, xx, v, r, q, st, s->gbar, s->sweep_err,
                         s->wait_limit) != cudaSuccess)
    return fail(H2G_CUDA_ERROR, "cooperative launch of %d blocks failed: %s", nblk,
                cudaGetErrorString(cudaGetLastError()));
  return H2G_OK;
}
template <int VM>
static int launch_coop(Solver* s, cudaStream_t cs, const OpParams<double>& op, double* xx, double* v,
                       const double* r, const double* q, SolverState* st) {
  const int m = s->rb_cls && op.cls ? 2 : s->rb_dd ? 1 : 0;
  if (s->rb_planes == 1)
    return m == 2 ? launch_coop_np<VM, 1, 2>(s, cs, op, xx, v, r, q, st)
                  : m == 1 ? launch_coop_np<VM, 1, 1>(s, cs, op, xx, v, r, q, st)
                           : launch_coop_np<VM, 1, 0>(s, cs, op, xx, v, r, q, st);
  return m == 2 ? launch_coop_np<VM, 2, 2>(s, cs, op, xx, v, r, q, st)
                : m == 1 ? launch_coop_np<VM, 2, 1>(s, cs, op, xx, v, r, q, st)
                         : launch_coop_np<VM, 2, 0>(s, cs, op, xx, v, r, q, st);
}
static bool use_coop(const Solver* s) { return s->rb_coop && !s->coop_barred && !s->rb_fused; }

template <typename T>
static T* x2buf(Solver* s);
template <>
double* x2buf<double>(Solver* s) { return s->x2_64; }
template <>
float* x2buf<float>(Solver* s) { return s->x2_32; }


// k_rb_sweep_first with the handle's chunking and dd source.
template <typename T, typename TV, int VM>
static int launch_sweep_first(Solver* s, cudaStream_t cs, const OpParams<T>& op, T* xout, TV* vout, const TV* vin,
                              T* bbT, const TV* r, const TV* q, SolverState* st) {
  const CUtensorMap* mk = nullptr;
  if (int rc = kmap(s, &mk)) return rc;
  const Geo& g = op.g;
  const int kc = (g.NZ + s->sw_chunks - 1) / s->sw_chunks;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = sweep_grid(g, s->sw_chunks);
  cfg.blockDim = dim3(kSwTPX, kSwTJ);
  cfg.dynamicSmemBytes = sweep_first_smem<T>();
  cfg.stream = cs;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = s->pdl ? 1 : 0;
  if (s->sw_dda)
    cudaLaunchKernelEx(&cfg, k_rb_sweep_first<T, TV, VM, true>, op, *mk, xout, vout, vin, bbT, r, q, kc, st,
                       s->sweep_err, s->wait_limit);
  else
    cudaLaunchKernelEx(&cfg, k_rb_sweep_first<T, TV, VM, false>, op, *mk, xout, vout, vin, bbT, r, q, kc, st,
                       s->sweep_err, s->wait_limit);
  return H2G_OK;
}

// Preconditioner! (NonUniform.jl:531-559) fused with the Krylov update that makes its right-hand
// side (VM as in k_rb_first): xx = M^-1 bb from xx = 0.  VM 0: bb = vin; VM 1: bb = p written to
// vout from p = vin (the same buffer on the colour-pass path); VM 2: bb = s written to vout.
// Fused path: one k_rb_sweep_first (sweep 1) and 4 fused sweeps; colour-pass path: k_rb_first and
// 9 colour passes.  x2 is the fused sweeps' ping-pong partner (zero guards).
template <typename T, typename TV, int VM>
static int launch_precond(Solver* s, cudaStream_t cs, const OpParams<T>& op, T* xx, T* x2, TV* vin, TV* vout,
                          T* bbT, const TV* r, const TV* q, SolverState* st, int smoother) {
  const int none = smoother == H2G_SMOOTHER_NONE;
  const T* bb = bbT ? bbT : reinterpret_cast<const T*>(VM == 0 ? vin : vout);
  if (s->rb_fused && !none) {
    if (int rc = launch_sweep_first<T, TV, VM>(s, cs, op, xx, vout, vin, bbT, r, q, st)) return rc;
    for (int sw = 1; sw < kSweeps; ++sw)
      if (int rc = launch_sweep<T>(s, cs, op, (sw & 1) ? xx : x2, (sw & 1) ? x2 : xx, bb, st)) return rc;
    return H2G_OK;
  }
  // k_rb_first updates v in place (VM 1 reads and writes p there)
  TV* v = VM == 0 ? vin : vout;
  if constexpr (std::is_same<T, double>::value && std::is_same<TV, double>::value) {
    if (use_coop(s) && !none && !bbT) return launch_coop<VM>(s, cs, op, xx, v, r, q, st);
  }
  if (s->rb_cls && op.cls && !none)
    launch(s, k_rb_first<T, TV, VM, true>, first_grid(op.g), dim3(kBX, kBY), cs, op, xx, v, bbT, r, q, st, none);
  else
    launch(s, k_rb_first<T, TV, VM, false>, first_grid(op.g), dim3(kBX, kBY), cs, op, xx, v, bbT, r, q, st, none);
  if (none) return H2G_OK;
  for (int pass = 1; pass < 2 * kSweeps; ++pass) launch_rb<T>(s, cs, op, xx, bb, pass & 1, T(1), st);
  return H2G_OK;
}

static size_t partials_needed(const Solver* s) {
  dim3 a = ax_grid(s->g);
  size_t nb = (size_t)a.x * a.y * a.z;
  nb = std::max(nb, (size_t)elementwise_blocks(s));
  return 2 * nb;
}

template <typename T>
static T* kvec(Solver* s, int i) {
  return reinterpret_cast<T*>(s->kv[i]);
}
enum { KR = 0, KR0 = 1, KP = 2, KPH = 3, KQ = 4, KS = 5, KSH = 6, KT = 7, KE = 8, KBB = 9, KP2 = 10 };

template <typename T>
static OpParams<T> op_params(const Solver* s, const OpTables<T>& t);
template <>
OpParams<double> op_params<double>(const Solver* s, const OpTables<double>& t);
template <>
OpParams<float> op_params<float>(const Solver* s, const OpTables<float>& t);

template <typename T>
static OpParams<T> op_params_rc(const Solver* s, const OpTables<T>& t, const T* rc) {
  OpParams<T> op;
  op.g = s->g;
  op.key = s->key;
  op.tx = t.tx;
  op.ty = t.ty;
  op.tz = t.tz;
  op.conv = t.conv;
  op.rc = rc;
  op.dzk = t.dzk;
  op.ddv = t.ddv;
  op.tq = t.tq;
  op.nkey = s->nkey;
  op.cls = nullptr;
  op.ctab = nullptr;
  const double dx0 = s->dx, dy0 = s->dy;
  op.czm = (T)((s->HC[4] * dx0) * dy0);
  op.czp = (T)((s->HC[5] * dx0) * dy0);
  op.dx0 = (T)dx0;
  op.dy0 = (T)dy0;
  op.ddt = (T)(1.0 / s->dt);
  op.P = t.pcap;
  op.steady = s->steady;
  return op;
}
template <>
OpParams<double> op_params<double>(const Solver* s, const OpTables<double>& t) {
  OpParams<double> op = op_params_rc<double>(s, t, s->rc64);
  if (s->cls_ok) {
    op.cls = s->cls;
    op.ctab = s->ctab;
  }
  return op;
}
template <>
OpParams<float> op_params<float>(const Solver* s, const OpTables<float>& t) {
  OpParams<float> op = op_params_rc<float>(s, t, s->rc32);
  if (s->cls_ok && s->ctab32) {
    op.cls = s->cls;
    op.ctab = s->ctab32;
  }
  return op;
}
template <typename T>
static OpParams<T> op_params(const Solver* s, const void* tables) {
  return op_params<T>(s, *static_cast<const OpTables<T>*>(tables));
}

static void free_tables64(OpTables<double>& t) {
  cudaFree(t.tx); cudaFree(t.ty); cudaFree(t.tz); cudaFree(t.conv); cudaFree(t.dzk); cudaFree(t.ddv); cudaFree(t.tq);
  t = OpTables<double>();
}
static void free_tables32(OpTables<float>& t) {
  cudaFree(t.tx); cudaFree(t.ty); cudaFree(t.tz); cudaFree(t.conv); cudaFree(t.dzk); cudaFree(t.ddv); cudaFree(t.tq);
  t = OpTables<float>();
}

static void destroy(Solver* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  for (auto& gk : s->graphs)
    for (auto& gg : gk) gg.reset();
  cudaFree(s->key); cudaFree(s->nkey); cudaFree(s->slots); cudaFree(s->slot_index); cudaFree(s->flags);
  free_tables64(s->t64);
  free_tables32(s->t32);
  cudaFree(s->rc64); cudaFree(s->rc32);
  cudaFree(s->th); cudaFree(s->b); cudaFree(s->th_snap); cudaFree(s->r64);
  cudaFree(s->hsrc); cudaFree(s->stats); cudaFree(s->th_prev);
  for (auto& p : s->adj) cudaFree(p);
  cudaFree(s->lamv);
  cudaFree(s->tstates);
  for (auto& p : s->kv) cudaFree(p);
  for (auto& p : s->hook) cudaFree(p);
  for (auto& p : s->stage) cudaFree(p);
  cudaFree(s->x2_64); cudaFree(s->x2_32); cudaFree(s->sweep_err); cudaFree(s->gbar);
  cudaFree(s->cls); cudaFree(s->ctab); cudaFree(s->ctab32); cudaFree(s->cslots); cudaFree(s->slot_class); cudaFree(s->cwords);
  cudaFree(s->cflag); cudaFree(s->key_prev); cudaFree(s->kdiff);
  s->mr_graph.reset();
  cudaFree(s->mr_th); cudaFree(s->mr_b); cudaFree(s->mr_st); cudaFree(s->mr_ctl); cudaFree(s->mr_partials);
  cudaFree(s->mr_flag);
  for (auto& p : s->mr_kv) cudaFree(p);
  cudaFree(s->st); cudaFree(s->st_in); cudaFree(s->partials); cudaFree(s->hist);
  if (s->st_host) cudaFreeHost(s->st_host);
  if (s->cap) cudaStreamDestroy(s->cap);
  delete static_cast<h2g_solver*>(s);
}

static int check_handle(const h2g_solver* hh) {
  if (!hh) return fail(H2G_BAD_ARG, "null solver handle");
  return H2G_OK;
}

// Column-major host array -> device layout (through the staging buffer).
template <typename T>
static int upload(Solver* s, const double* host, T* dev, int slot = 0) {
  if (!host) return fail(H2G_BAD_ARG, "null host array");
  const Geo& g = s->g;
  CK(cudaMemcpyAsync(s->stage[slot], host, sizeof(double) * s->nfort(), cudaMemcpyHostToDevice, s->stream));
  dim3 grid((g.MX + 127) / 128, g.MY, g.MZ);
  k_to_dev<T><<<grid, 128, 0, s->stream>>>(g, s->stage[slot], dev);
  CKL();
  CK(cudaStreamSynchronize(s->stream));  // the caller may reuse its buffer on return
  return H2G_OK;
}

template <typename T>
static int download(Solver* s, const T* dev, double* host) {
  if (!host) return fail(H2G_BAD_ARG, "null host array");
  const Geo& g = s->g;
  dim3 grid((g.MX + 127) / 128, g.MY, g.MZ);
  k_from_dev<T><<<grid, 128, 0, s->stream>>>(g, dev, s->stage[0]);
  CKL();
  CK(cudaMemcpyAsync(host, s->stage[0], sizeof(double) * s->nfort(), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return H2G_OK;
}

static void invalidate_graphs(Solver* s) {
  for (auto& gk : s->graphs)
    for (auto& gg : gk) gg.reset();
}

// ------------------------------------------------------------------------------------------
// Operator tables (host, FP64, in the reference's operation order; FP32 copies by rounding).
// ------------------------------------------------------------------------------------------
// Stencil classes of the FP64 operator (k_class_insert / k_class_assign / k_class_coef): the
// distinct (plane, 7 keys) pairs of the updated cells, numbered in the order of their hash slots,
// and their coefficients.  Left unbuilt (the kernels keep the key tables) when disabled
// (H2G_CLS=0), when NZ > 255 (the plane shares the 64-bit word with the keys) or when the grid has
// more than kMaxClasses pairs.
static int build_classes(Solver* s) {
  const Geo& g = s->g;
  const bool was = s->cls_ok;
  s->cls_ok = false;
  s->ncls = 0;
  const char* e = getenv("H2G_CLS");
  if ((e && atoi(e) == 0) || g.NZ > 255 || !s->nkey) {
    if (was) invalidate_graphs(s);
    return H2G_OK;
  }
  if (!s->cls) {
    CK(cudaMalloc(&s->cls, sizeof(uint16_t) * (size_t)g.n));
    CK(cudaMalloc(&s->ctab, sizeof(double) * 8 * (size_t)kMaxClasses));
    if (s->precision != H2G_FP64) CK(cudaMalloc(&s->ctab32, sizeof(float) * 8 * (size_t)kMaxClasses));
    CK(cudaMalloc(&s->cslots, sizeof(unsigned long long) * kClassSlots));
    CK(cudaMalloc(&s->slot_class, sizeof(uint16_t) * kClassSlots));
    CK(cudaMalloc(&s->cwords, sizeof(unsigned long long) * kMaxClasses));
    CK(cudaMalloc(&s->cflag, sizeof(int)));
  }
  CK(cudaMemsetAsync(s->cslots, 0, sizeof(unsigned long long) * kClassSlots, s->stream));
  CK(cudaMemsetAsync(s->cflag, 0, sizeof(int), s->stream));
  CK(cudaMemsetAsync(s->cls, 0xff, sizeof(uint16_t) * (size_t)g.n, s->stream));
  const dim3 gi((g.NX + 255) / 256, g.NY, g.NZ);
  k_class_insert<<<gi, 256, 0, s->stream>>>(g, s->nkey, s->cslots, s->cflag);
  CKL();
  std::vector<unsigned long long> slots(kClassSlots);
  int flag = 0;
  CK(cudaMemcpyAsync(slots.data(), s->cslots, sizeof(unsigned long long) * kClassSlots, cudaMemcpyDeviceToHost,
                     s->stream));
  CK(cudaMemcpyAsync(&flag, s->cflag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  std::vector<uint16_t> sc(kClassSlots, (uint16_t)kNoClass);
  std::vector<unsigned long long> words;
  bool fits = flag == 0;
  for (int h = 0; h < kClassSlots && fits; ++h) {
    if (!slots[h]) continue;
    if ((int)words.size() >= kMaxClasses) fits = false;
    else {
      sc[h] = (uint16_t)words.size();
      words.push_back(slots[h]);
    }
  }
  if (!fits || words.empty()) {
    if (was) invalidate_graphs(s);
    return H2G_OK;
  }
  CK(cudaMemcpyAsync(s->slot_class, sc.data(), sizeof(uint16_t) * kClassSlots, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->cwords, words.data(), sizeof(unsigned long long) * words.size(), cudaMemcpyHostToDevice,
                     s->stream));
  k_class_assign<<<gi, 256, 0, s->stream>>>(g, s->nkey, s->cslots, s->slot_class, s->cls);
  const int ncls = (int)words.size();
  OpParams<double> o64 = op_params_rc<double>(s, s->t64, s->rc64);
  k_class_coef<double><<<(ncls + 127) / 128, 128, 0, s->stream>>>(o64, s->cwords, ncls, s->ctab);
  if (s->ctab32) {
    OpParams<float> o32 = op_params_rc<float>(s, s->t32, s->rc32);
    k_class_coef<float><<<(ncls + 127) / 128, 128, 0, s->stream>>>(o32, s->cwords, ncls, s->ctab32);
  }
  CKL();
  CK(cudaStreamSynchronize(s->stream));  // the host vectors must outlive the copies
  s->ncls = ncls;
  s->cls_ok = true;
  if (!was) invalidate_graphs(s);
  return H2G_OK;
}

// Everything the operator tables, dd and the stencil classes are built from, besides the key array.
static std::vector<unsigned char> tables_signature(const Solver* s) {
  std::vector<unsigned char> v;
  auto put = [&](const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    v.insert(v.end(), c, c + n);
  };
  put(&s->P, sizeof s->P);
  put(s->lam_values.data(), sizeof(double) * s->lam_values.size());
  put(s->ZC.data(), sizeof(double) * s->ZC.size());
  put(s->dZ.data(), sizeof(double) * s->dZ.size());
  put(&s->dx, sizeof s->dx);
  put(&s->dy, sizeof s->dy);
  put(&s->dt, sizeof s->dt);
  put(s->HC, sizeof s->HC);
  put(&s->steady, sizeof s->steady);
  const char* e = getenv("H2G_CLS");
  const std::string cls_env = e ? e : "";
  put(cls_env.data(), cls_env.size());
  return v;
}

static int build_tables(Solver* s) {
  if (!s->grid_set || !s->fields_set) return H2G_OK;
  // a steady grid whose keys and table inputs equal those of the last build keeps its tables,
  // dd and classes (repeated one-call solves of one operator)
  std::vector<unsigned char> sig = tables_signature(s);
  if (!s->keys_changed && s->steady && sig == s->tables_sig) return H2G_OK;
  s->tables_sig.clear();
  const Geo& g = s->g;
  const int P = s->P;
  const int pc = std::max(P, 8);
  const double dx0 = s->dx, dy0 = s->dy;
  const double ddx = 1.0 / dx0, ddy = 1.0 / dy0;
  std::vector<double> LP((size_t)pc * pc, 0.0);
  for (int a = 0; a < P; ++a)
    for (int b = 0; b < P; ++b) {
      const double la = s->lam_values[a], lb = s->lam_values[b];
      LP[(size_t)a * pc + b] = 2.0 * la * lb / (la + lb);  // lambda_f without the mask factor, common.jl:35
    }
  // tables [k][a0][neighbour key byte]: bit 7 of the neighbour key is its mask; a masked
  // neighbour doubles lambda_f (2 - div(ma+mb, 2) = 2), an unmasked one keeps it (= 1)
  const size_t lvl = (size_t)pc * 256;
  std::vector<double> tx(lvl * g.MZ, 0.0), ty(lvl * g.MZ, 0.0), tz(lvl * g.MZ, 0.0), conv(4 * (size_t)g.MZ, 0.0);
  for (int k = 0; k < g.MZ; ++k) {
    const double dz_k = s->dZ[k];
    for (int a = 0; a < P; ++a)
      for (int kn = 0; kn < 256; ++kn) {
        const int b = kn & 0x7f;
        if (b >= P) continue;
        const double fac = (kn & 0x80) ? 1.0 : 2.0;
        const double lf = LP[(size_t)a * pc + b] * fac;
        const size_t o = (size_t)k * lvl + (size_t)a * 256 + kn;
        tx[o] = lf * dy0 * dz_k * ddx;  // NonUniform.jl:482-483
        ty[o] = lf * dx0 * dz_k * ddy;  // NonUniform.jl:484-485
        if (k >= 1) tz[o] = lf * dx0 * dy0 / (s->ZC[k] - s->ZC[k - 1]);  // NonUniform.jl:486
      }
    conv[4 * k + 0] = s->HC[0] * dy0 * dz_k;  // NonUniform.jl:490-493
    conv[4 * k + 1] = s->HC[1] * dy0 * dz_k;
    conv[4 * k + 2] = s->HC[2] * dx0 * dz_k;
    conv[4 * k + 3] = s->HC[3] * dx0 * dz_k;
  }
  // (re)allocate when the key capacity grows; graphs hold the pointers, so they are rebuilt
  const size_t bytes_t = lvl * g.MZ;
  if (s->t64.pcap != pc) {
    free_tables64(s->t64);
    free_tables32(s->t32);
    invalidate_graphs(s);
    CK(cudaMalloc(&s->t64.tx, sizeof(double) * bytes_t));
    CK(cudaMalloc(&s->t64.ty, sizeof(double) * bytes_t));
    CK(cudaMalloc(&s->t64.tz, sizeof(double) * bytes_t));
    CK(cudaMalloc(&s->t64.conv, sizeof(double) * 4 * g.MZ));
    CK(cudaMalloc(&s->t64.dzk, sizeof(double) * g.MZ));
    CK(cudaMalloc(&s->t64.ddv, sizeof(double) * (size_t)g.n));
    CK(cudaMalloc(&s->t64.tq, sizeof(double) * 4 * bytes_t));
    CK(cudaMemsetAsync(s->t64.ddv, 0, sizeof(double) * (size_t)g.n, s->stream));
    s->t64.pcap = pc;
    if (s->precision != H2G_FP64) {
      CK(cudaMalloc(&s->t32.tx, sizeof(float) * bytes_t));
      CK(cudaMalloc(&s->t32.ty, sizeof(float) * bytes_t));
      CK(cudaMalloc(&s->t32.tz, sizeof(float) * bytes_t));
      CK(cudaMalloc(&s->t32.conv, sizeof(float) * 4 * g.MZ));
      CK(cudaMalloc(&s->t32.dzk, sizeof(float) * g.MZ));
      CK(cudaMalloc(&s->t32.ddv, sizeof(float) * (size_t)g.n));
      CK(cudaMalloc(&s->t32.tq, sizeof(float) * 4 * bytes_t));
      CK(cudaMemsetAsync(s->t32.ddv, 0, sizeof(float) * (size_t)g.n, s->stream));
      s->t32.pcap = pc;
    }
  }
  // the same values interleaved per (plane, own key, neighbour key byte): x, y, z-, z+ (the z+
  // face of plane k is the z- table of plane k+1, zero above the last plane)
  std::vector<double> tq(4 * bytes_t, 0.0);
  for (size_t o = 0; o < bytes_t; ++o) {
    tq[4 * o + 0] = tx[o];
    tq[4 * o + 1] = ty[o];
    tq[4 * o + 2] = tz[o];
    tq[4 * o + 3] = o + lvl < bytes_t ? tz[o + lvl] : 0.0;
  }
  CK(cudaMemcpyAsync(s->t64.tq, tq.data(), sizeof(double) * 4 * bytes_t, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->t64.tx, tx.data(), sizeof(double) * bytes_t, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->t64.ty, ty.data(), sizeof(double) * bytes_t, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->t64.tz, tz.data(), sizeof(double) * bytes_t, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->t64.conv, conv.data(), sizeof(double) * 4 * g.MZ, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->t64.dzk, s->dZ.data(), sizeof(double) * g.MZ, cudaMemcpyHostToDevice, s->stream));
  if (s->precision != H2G_FP64) {
    auto to32 = [](const std::vector<double>& v) {
      std::vector<float> o(v.size());
      for (size_t i = 0; i < v.size(); ++i) o[i] = (float)v[i];
      return o;
    };
    std::vector<float> fx = to32(tx), fy = to32(ty), fz = to32(tz), fc = to32(conv), fd = to32(s->dZ), fq = to32(tq);
    CK(cudaMemcpyAsync(s->t32.tq, fq.data(), sizeof(float) * 4 * bytes_t, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->t32.tx, fx.data(), sizeof(float) * bytes_t, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->t32.ty, fy.data(), sizeof(float) * bytes_t, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->t32.tz, fz.data(), sizeof(float) * bytes_t, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->t32.conv, fc.data(), sizeof(float) * 4 * g.MZ, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->t32.dzk, fd.data(), sizeof(float) * g.MZ, cudaMemcpyHostToDevice, s->stream));
  }
  // dd per cell for the smoother, from the tables just written (op.ddv null: summed in full)
  {
    const dim3 grid((g.NX + 127) / 128, g.NY, g.NZ);
    OpParams<double> o64 = op_params<double>(s, s->t64);
    o64.ddv = nullptr;
    k_make_dd<double><<<grid, 128, 0, s->stream>>>(o64, s->t64.ddv);
    if (s->precision != H2G_FP64) {
      OpParams<float> o32 = op_params<float>(s, s->t32);
      o32.ddv = nullptr;
      k_make_dd<float><<<grid, 128, 0, s->stream>>>(o32, s->t32.ddv);
    }
    CKL();
  }
  // host vectors must stay alive until the copies ran
  CK(cudaStreamSynchronize(s->stream));
  if (int rc = build_classes(s)) return rc;
  s->tables_sig = std::move(sig);
  s->keys_changed = false;
  return H2G_OK;
}

// ------------------------------------------------------------------------------------------
// Graph capture of one Krylov iteration.
// ------------------------------------------------------------------------------------------
// One Krylov iteration.  T: Krylov vectors, inner products' inputs and the operator applied by
// CalcAX (opA); TP: the preconditioner's precision (opM) and of its outputs p_, s_ (z for CG).
// With TP != T the first pass also writes the smoother's copy of its right-hand side (bb32).
template <typename T, typename TX, typename TP>
static int launch_pbicg_body(Solver* s, cudaStream_t cs, const OpParams<T>& opA, const OpParams<TP>& opM, TX* x,
                             SolverState* st, int smoother, cudaGraphConditionalHandle hc, int use_cond, int u) {
  const Geo& g = s->g;
  T* r = kvec<T>(s, KR);
  T* r0 = kvec<T>(s, KR0);
  // p of this iteration is read from p_in and written to p_out; they alternate on the fused path
  const bool pp = s->rb_fused && smoother != H2G_SMOOTHER_NONE;
  T* p_in = kvec<T>(s, pp && (u & 1) ? KP2 : KP);
  T* p_out = kvec<T>(s, pp && !(u & 1) ? KP2 : KP);
  TP* ph = kvec<TP>(s, KPH);
  T* q = kvec<T>(s, KQ);
  T* sv = kvec<T>(s, KS);
  TP* sh = kvec<TP>(s, KSH);
  T* t = kvec<T>(s, KT);
  TP* bbm = std::is_same<T, TP>::value ? nullptr : kvec<TP>(s, KBB);
  TP* x2 = x2buf<TP>(s);
  // p = r + beta (p - omega q); p_ = M^-1 p                     NonUniform.jl:296-305
  if (int rc = launch_precond<TP, T, 1>(s, cs, opM, ph, x2, p_in, p_out, bbm, r, q, st, smoother)) return rc;
  // q = A p_;  alpha = rho / (q, r0)                            NonUniform.jl:307-309
  launch_ax<T, 1, TP>(s, cs, opA, q, ph, r0, nullptr, st, kStageAlpha);
  // s = r - alpha q; s_ = M^-1 s                                NonUniform.jl:310-315
  if (int rc = launch_precond<TP, T, 2>(s, cs, opM, sh, x2, sv, sv, bbm, r, q, st, smoother)) return rc;
  // t = A s_; omega = (t,s)/(t,t)                               NonUniform.jl:317-326
  launch_ax<T, 2, TP>(s, cs, opA, t, sh, nullptr, sv, st, kStageOmega);
  // x += alpha p_ + omega s_; r = s - omega t; res; next rho    NonUniform.jl:328-346
  if (use_cond)
    launch(s, k_bicg_update<T, TX, TP, true>, elementwise_blocks(s), 256, cs, g.n, x, ph, sh, r, sv, t, r0, st,
           s->partials, hc, use_cond);
  else
    launch(s, k_bicg_update<T, TX, TP, false>, elementwise_blocks(s), 256, cs, g.n, x, ph, sh, r, sv, t, r0, st,
           s->partials, hc, use_cond);
  return H2G_OK;
}

// z = M^-1 r with the first pass reading r (VM 0) and, for TP != T, writing bb32
template <typename T, typename TP>
static int launch_precond_r(Solver* s, cudaStream_t cs, const OpParams<TP>& opM, TP* z, T* r, SolverState* st,
                            int smoother) {
  TP* bbm = std::is_same<T, TP>::value ? nullptr : kvec<TP>(s, KBB);
  return launch_precond<TP, T, 0>(s, cs, opM, z, x2buf<TP>(s), r, r, bbm, nullptr, nullptr, st, smoother);
}

template <typename T, typename TX, typename TP>
static int launch_cg_body(Solver* s, cudaStream_t cs, const OpParams<T>& opA, const OpParams<TP>& opM, TX* x,
                          SolverState* st, int smoother, cudaGraphConditionalHandle hc, int use_cond) {
  const Geo& g = s->g;
  T* r = kvec<T>(s, KR);
  T* p = kvec<T>(s, KP);
  T* q = kvec<T>(s, KQ);
  TP* z = kvec<TP>(s, KPH);  // z (pcg_s in NonUniform.jl:146) in the preconditioner-output buffer
  const dim3 blk(kBX, kBY);
  const int nb = elementwise_blocks(s);
  // q = A p; alpha = rho_old / (p,q)                             NonUniform.jl:164-176
  launch_ax<T, 1, T>(s, cs, opA, q, p, p, nullptr, st, kStageCgAlpha);
  // x += alpha p; r -= alpha q; res                              NonUniform.jl:179-198
  launch(s, k_cg_update<T, TX>, nb, 256, cs, g.n, x, p, r, q, st, s->partials);
  // z = M^-1 r                                                  NonUniform.jl:201-203
  if (int rc = launch_precond_r<T, TP>(s, cs, opM, z, r, st, smoother)) return rc;
  // rho_new = (r,z); beta                                       NonUniform.jl:206-215
  launch(s, k_dot<T, TP>, nb, 256, cs, g.n, r, z, nullptr, st, s->partials, kStageCgBeta);
  // p = z + beta p                                              NonUniform.jl:218-220
  if (use_cond) launch(s, k_cg_pupd<T, TP, true>, nb, 256, cs, g.n, p, z, st, hc, use_cond);
  else launch(s, k_cg_pupd<T, TP, false>, nb, 256, cs, g.n, p, z, st, hc, use_cond);
  return H2G_OK;
}

template <typename T, typename TP>
static std::vector<unsigned char> signature(const OpParams<T>& opA, const OpParams<TP>& opM, int smoother,
                                            const void* x) {
  std::vector<unsigned char> v(sizeof opA + sizeof opM + sizeof smoother + sizeof x);
  unsigned char* d = v.data();
  memcpy(d, &opA, sizeof opA);
  memcpy(d + sizeof opA, &opM, sizeof opM);
  memcpy(d + sizeof opA + sizeof opM, &smoother, sizeof smoother);
  memcpy(d + sizeof opA + sizeof opM + sizeof smoother, &x, sizeof x);
  return v;
}

// Instantiate the loop of a solve: a conditional WHILE node whose body is what body(stream,
// handle, 1) captures, or, where conditional nodes are unavailable, a graph of the same body
// (body(stream, 0, 0)) that run_graph relaunches from the host.
template <typename Body>
static int make_loop_graph(Solver* s, SolveGraph& G, Body body) {
  G.reset();
  bool cond = !s->no_cond;
  if (cond) {
    cudaGraph_t parent = nullptr;
    cudaGraphConditionalHandle hc = 0;
    cudaGraphNode_t node;
    cudaGraphNodeParams cp = {};
    bool ok = cudaGraphCreate(&parent, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&hc, parent, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = hc;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      ok = cudaGraphAddNode(&node, parent, nullptr, 0, &cp) == cudaSuccess;
    }
    if (ok) {
      cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
      ok = cudaStreamBeginCaptureToGraph(s->cap, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
           cudaSuccess;
      if (ok) {
        body(s->cap, hc, 1);
        cudaGraph_t got = nullptr;
        ok = cudaStreamEndCapture(s->cap, &got) == cudaSuccess;
      }
    }
    if (ok) ok = cudaGraphInstantiate(&G.exec, parent, 0) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      if (G.exec) cudaGraphExecDestroy(G.exec);
      G.exec = nullptr;
      if (parent) cudaGraphDestroy(parent);
      cond = false;
      s->no_cond = true;
    } else {
      G.graph = parent;
      G.cond = true;
    }
  }
  if (!cond) {
    CK(cudaStreamBeginCapture(s->cap, cudaStreamCaptureModeRelaxed));
    body(s->cap, (cudaGraphConditionalHandle)0, 0);
    CK(cudaStreamEndCapture(s->cap, &G.graph));
    CK(cudaGraphInstantiate(&G.exec, G.graph, 0));
    G.cond = false;
  }
  return H2G_OK;
}

template <typename T, typename TX, typename TP>
static int get_graph(Solver* s, int kind, int smoother, const OpParams<T>& op, const OpParams<TP>& opM, TX* x,
                     SolverState* st, SolveGraph** out) {
  SolveGraph& G = s->graphs[kind][smoother ? 1 : 0];
  std::vector<unsigned char> sig = signature(op, opM, smoother, (const void*)x);
  sig.push_back(use_coop(s) ? 1 : 0);
  if (G.exec && G.sig == sig) {
    *out = &G;
    return H2G_OK;
  }
  const bool cg = (kind == kGCg64 || kind == kGCg32 || kind == kGCgMx);
  int berr = H2G_OK;
  int rc = make_loop_graph(s, G, [&](cudaStream_t cs, cudaGraphConditionalHandle hc, int use_cond) {
    // kUnroll iterations per WHILE-body pass: the device re-evaluates the loop condition
    // kUnroll times less often.  Every kernel returns at once when the state says stop, and the
    // last update kernel of the body sets the condition, so an iteration that converges in the
    // middle of a pass only leaves the rest of the pass as empty launches.
    for (int u = 0; u < kUnroll && berr == H2G_OK; ++u) {
      if (cg) berr = launch_cg_body<T, TX, TP>(s, cs, op, opM, x, st, smoother, hc, use_cond);
      else berr = launch_pbicg_body<T, TX, TP>(s, cs, op, opM, x, st, smoother, hc, use_cond, u);
    }
  });
  if (rc == H2G_OK && berr != H2G_OK) G.reset();
  if (rc) return rc;
  if (berr) return berr;
  G.sig = sig;
  *out = &G;
  return H2G_OK;
}

// per: iterations (SOR passes) in one launch of the body graph
static int run_graph(Solver* s, SolveGraph* G, SolverState* st, int maxItr, int per) {
  if (G->cond) {
    CK(cudaGraphLaunch(G->exec, s->stream));
    return H2G_OK;
  }
  // host loop: batches of iterations between checks of the device stop flag
  int done = 0;
  const int batch = 8;
  while (done < maxItr + 1) {
    for (int i = 0; i < batch; ++i) CK(cudaGraphLaunch(G->exec, s->stream));
    done += batch * per;
    CK(cudaMemcpyAsync(s->st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (s->st_host->stop) break;
  }
  return H2G_OK;
}

// Set the host-controlled fields of a device state (tolerance, iteration cap, history).
static int prime_state(Solver* s, SolverState* st, double tol, int maxItr, double* hist, int hist_len) {
  launch(s, k_prime, 1, 1, s->stream, st, tol, maxItr, hist, hist_len, s->div_limit);
  CKL();
  return H2G_OK;
}

static int ensure_hist(Solver* s, int n) {
  if (n <= s->hist_cap) return H2G_OK;
  cudaFree(s->hist);
  s->hist = nullptr;
  s->hist_cap = 0;
  CK(cudaMalloc(&s->hist, sizeof(double) * (size_t)n));
  s->hist_cap = n;
  return H2G_OK;
}

static int status_of(const SolverState& st) {
  switch (st.reason) {
    case kConverged: return H2G_OK;
    case kBreakdown: return H2G_BREAKDOWN;
    case kNonFinite: return H2G_NONFINITE;
    case kTimeout: return H2G_TIMEOUT;
    default: return H2G_NOT_CONVERGED;
  }
}

// Julia's shortest round-trip print of a Float64 (used for "Initial residual = ...").
static void julia_repr(double x, char* out, size_t n) {
  char buf[64];
  for (int p = 1; p <= 17; ++p) {
    snprintf(buf, sizeof buf, "%.*e", p - 1, x);
    if (strtod(buf, nullptr) == x) break;
  }
  // buf = d.ddde[+-]XX
  double ax = fabs(x);
  if (x == 0.0 || (ax >= 1e-4 && ax < 1e16)) {
    for (int p = 1; p <= 17; ++p) {
      snprintf(out, n, "%.*f", p, x);
      if (strtod(out, nullptr) == x) return;
    }
    snprintf(out, n, "%.17g", x);
    return;
  }
  char* e = strchr(buf, 'e');
  int ex = atoi(e + 1);
  *e = 0;
  if (!strchr(buf, '.')) strcat(buf, ".0");
  snprintf(out, n, "%se%d", buf, ex);
}

static void print_log(const SolverState& st, const double* hist, int nhist, int converged) {
  char rb[64];
  julia_repr(st.res0, rb, sizeof rb);
  printf("Initial residual = %s\n", rb);
  for (int i = 0; i < nhist; ++i) printf("%10d %24.14E\n", i + 1, hist[i]);
  if (converged) printf("Converged at %d\n", st.itr);
  fflush(stdout);
}

// Kernels of one preconditioner call: the first pass and 9 colour passes, or 5 fused sweeps (the
// first one with the Krylov update).
static int precond_kernels(const Solver* s, int smoother, bool coop = false) {
  if (smoother == H2G_SMOOTHER_NONE || coop) return 1;
  return s->rb_fused ? kSweeps : 2 * kSweeps;
}

// Kernels in one WHILE-body pass (one Krylov iteration); coop: the preconditioner is the one
// cooperative launch (FP64 smoother).
static long long body_kernels(const Solver* s, bool cg, int smoother, bool coop = false) {
  const int pc = precond_kernels(s, smoother, coop);
  return cg ? (1 + 1 + pc + 1 + 1) : (2 * pc + 2 + 1);
}

// PBiCGSTAB!/CG! with FP64 Krylov vectors, inner products and operator (the reference's
// arithmetic).  TP is the precision of the RB-GS preconditioner: double (H2G_FP64, identical to
// the reference) or float (H2G_MIXED: the 20 colour passes per iteration read and write FP32).
template <typename TP>
static int solve_krylov(Solver* s, bool cg, double tol, int maxItr, int smoother, int verbose, double* res_hist,
                        h2g_result* out) {
  const Geo& g = s->g;
  int rc = ensure_hist(s, maxItr);
  if (rc) return rc;
  OpParams<double> op = op_params<double>(s, s->t64);
  OpParams<TP> opM = op_params<TP>(s, std::is_same<TP, double>::value ? (const void*)&s->t64 : (const void*)&s->t32);
  SolverState* st = s->st;
  if ((rc = prime_state(s, st, tol, maxItr, s->hist, maxItr))) return rc;
  double* r = kvec<double>(s, KR);
  const dim3 ag = ax_grid(g), blk(kBX, kBY);
  // r = b - A theta, res0 (and r0 = r for PBiCGSTAB)            NonUniform.jl:131-141, 262-274
  launch(s, k_rk<double>, ag, blk, s->stream, op, r, cg ? nullptr : kvec<double>(s, KR0), s->th, s->b, st, s->partials,
                                          cg ? kStageInitCg : kStageInit);
  CKL();
  if (cg) {
    // z = M^-1 r; p = z; rho_old = (r,z)                          NonUniform.jl:147-155
    TP* z = kvec<TP>(s, KPH);
    if ((rc = launch_precond_r<double, TP>(s, s->stream, opM, z, r, st, smoother))) return rc;
    launch(s, k_dot<double, TP>, elementwise_blocks(s), 256, s->stream, g.n, r, z, kvec<double>(s, KP), st, s->partials,
                                                                     kStageCgInit);
    CKL();
  }
  SolveGraph* G = nullptr;
  const int kind = std::is_same<TP, double>::value ? (cg ? kGCg64 : kGPbicg64) : (cg ? kGCgMx : kGPbicgMx);
  if ((rc = get_graph<double, double, TP>(s, kind, smoother, op, opM, s->th, st, &G))) return rc;
  // a state that stopped at the start turns every kernel of the body into a no-op and the
  // last one ends the WHILE loop after one pass
  if ((rc = run_graph(s, G, st, maxItr, kUnroll))) return rc;
  CK(cudaMemcpyAsync(s->st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  SolverState fin = *s->st_host;
  const int nh = std::min(std::max(fin.itr, 0), maxItr);
  std::vector<double> hh(nh);
  if (nh > 0 && (verbose || res_hist)) {
    CK(cudaMemcpy(hh.data(), s->hist, sizeof(double) * nh, cudaMemcpyDeviceToHost));
    if (res_hist) memcpy(res_hist, hh.data(), sizeof(double) * nh);
  }
  // a breakdown at the top of an iteration leaves no residual for that iteration
  const int nprint = (fin.reason == kBreakdown || fin.reason == kNonFinite) ? std::min(nh, std::max(0, fin.itr - 1)) : nh;
  if (verbose) print_log(fin, hh.data(), nprint, fin.converged);
  if (out) {
    const bool coop = std::is_same<TP, double>::value && use_coop(s);
    const long long body = body_kernels(s, cg, smoother, coop);
    const long long pre = 2 + (cg ? precond_kernels(s, smoother, coop) + 1 : 0);
    out->launches = pre + body * std::max(1, fin.itr);
    out->isconverged = fin.converged;
    out->itr = fin.itr;
    out->outer = 0;
    out->status = status_of(fin);
    out->res0 = fin.res0;
    out->res = fin.res;
  }
  return status_of(fin);
}

// H2G_MIXED_IR: FP32 PBiCGSTAB/CG (operator, smoother, Krylov vectors) inside FP64 iterative
// refinement.  FP64 is kept for the true residual b - A theta, the accumulation of theta and
// every inner product (the reductions accumulate in FP64).  On fine grids the FP32 BiCGSTAB
// recurrences lose accuracy faster than a refinement pass can use (the inner solve can
// diverge: the solve then reports H2G_NONFINITE); H2G_MIXED keeps the Krylov part in FP64.
static int solve_ir(Solver* s, bool cg, double tol, int maxItr, int smoother, int verbose, double* res_hist,
                       h2g_result* out) {
  const Geo& g = s->g;
  int rc;
  OpParams<double> op64 = op_params<double>(s, s->t64);
  OpParams<float> op32 = op_params<float>(s, s->t32);
  SolverState* st = s->st;
  SolverState* si = s->st_in;
  const dim3 ag = ax_grid(g), blk(kBX, kBY);
  const int nb = elementwise_blocks(s);
  if ((rc = prime_state(s, st, tol, maxItr, nullptr, 0))) return rc;
  // true residual r64 = b - A theta, ||r64||
  launch(s, k_rk<double>, ag, blk, s->stream, op64, s->r64, nullptr, s->th, s->b, st, s->partials, kStageResid);
  CKL();
  CK(cudaMemcpyAsync(s->st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const double res0 = s->st_host->scale;
  double res = res0 == 0.0 ? 0.0 : 1.0;
  int total = 0, outer = 0, status = H2G_NOT_CONVERGED, converged = 0;
  std::vector<double> hist_all;
  if (res0 == 0.0) {
    status = H2G_OK;
    converged = 1;
  } else if (!std::isfinite(res0)) {
    status = H2G_NONFINITE;
  }
  if (!converged && status != H2G_NONFINITE) {
    if ((rc = ensure_hist(s, maxItr))) return rc;
    float* e = kvec<float>(s, KE);
    SolveGraph* G = nullptr;
    double scale = res0;
    while (outer < s->max_outer && total < maxItr) {
      ++outer;
      const int cap = maxItr - total;
      if ((rc = prime_state(s, si, s->inner_tol, cap, s->hist, cap))) return rc;
      // inner right-hand side r = r64/||r64||, e = 0, inner res0 and rho
      launch(s, k_ir_prep, nb, 256, s->stream, g.n, s->r64, kvec<float>(s, KR), kvec<float>(s, KR0), e, st, si,
                                           s->partials, cg ? kStageInitCg : kStageInit);
      CKL();
      if (cg) {
        float* z = kvec<float>(s, KPH);
        if ((rc = launch_precond_r<float, float>(s, s->stream, op32, z, kvec<float>(s, KR), si, smoother))) return rc;
        launch(s, k_dot<float>, nb, 256, s->stream, g.n, kvec<float>(s, KR), z, kvec<float>(s, KP), si, s->partials,
                                                 kStageCgInit);
        CKL();
      }
      if ((rc = get_graph<float, float, float>(s, cg ? kGCg32 : kGPbicg32, smoother, op32, op32, e, si, &G)))
        return rc;
      if ((rc = run_graph(s, G, si, cap, kUnroll))) return rc;
      // theta += ||r64|| e ; r64 = b - A theta
      launch(s, k_ir_apply, nb, 256, s->stream, g.n, s->th, e, st);
      launch(s, k_rk<double>, ag, blk, s->stream, op64, s->r64, nullptr, s->th, s->b, st, s->partials, kStageResid);
      CKL();
      SolverState inner;
      CK(cudaMemcpyAsync(s->st_host, si, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
      inner = *s->st_host;
      if (inner.reason == kTimeout) {
        status = H2G_TIMEOUT;
        break;
      }
      CK(cudaMemcpyAsync(s->st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
      const double new_scale = s->st_host->scale;
      const int ni = std::max(inner.itr, 0);
      if (verbose || res_hist) {
        std::vector<double> hh(std::min(ni, cap));
        if (!hh.empty()) CK(cudaMemcpy(hh.data(), s->hist, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost));
        for (double v : hh) hist_all.push_back(v * scale / res0);
      }
      total += ni;
      res = new_scale / res0;
      scale = new_scale;
      if (!std::isfinite(res)) { status = H2G_NONFINITE; break; }
      if (res < tol) { status = H2G_OK; converged = 1; break; }
      if (ni == 0) {  // the inner solve could not start (breakdown at its first iteration)
        status = inner.reason == kNonFinite ? H2G_NONFINITE : H2G_BREAKDOWN;
        break;
      }
    }
  }
  if (res_hist && !hist_all.empty())
    memcpy(res_hist, hist_all.data(), sizeof(double) * std::min<size_t>(hist_all.size(), (size_t)maxItr));
  if (verbose) {
    SolverState fake;
    memset(&fake, 0, sizeof fake);
    fake.res0 = res0;
    fake.itr = total;
    print_log(fake, hist_all.data(), (int)std::min<size_t>(hist_all.size(), (size_t)maxItr), converged);
  }
  if (out) {
    const long long body = body_kernels(s, cg, smoother);
    const long long pre_inner = 2 + (cg ? precond_kernels(s, smoother) + 1 : 0);
    out->launches = 2 + (long long)outer * (pre_inner + 2) + body * std::max(total, outer);
    out->isconverged = converged;
    out->itr = total;
    out->outer = outer;
    out->status = status;
    out->res0 = res0;
    out->res = res;
  }
  return status;
}

// ||b - A theta|| in FP64 on the device (into the r vector, which every solve recomputes).
static int true_residual(Solver* s, double* res) {
  OpParams<double> op = op_params<double>(s, s->t64);
  int rc;
  if ((rc = prime_state(s, s->st, 0.0, 1, nullptr, 0))) return rc;
  launch(s, k_rk<double>, ax_grid(s->g), dim3(kBX, kBY), s->stream, op, kvec<double>(s, KR), (double*)nullptr, s->th,
         s->b, s->st, s->partials, (int)kStageResid);
  CKL();
  CK(cudaMemcpyAsync(s->st_host, s->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *res = s->st_host->scale;
  return H2G_OK;
}

// H2G_MIXED: FP64 Krylov with the FP32 preconditioner.  The preconditioner's rounding makes the
// recursively updated residual drift from the true one, so convergence is confirmed with the
// FP64 true residual and the solve restarts from the current theta until the true residual
// meets the tolerance.
static int solve_mixed(Solver* s, bool cg, double tol, int maxItr, int smoother, int verbose, double* res_hist,
                       h2g_result* out) {
  int total = 0, status = H2G_NOT_CONVERGED, converged = 0, passes = 0;
  long long launches = 0;
  double res0 = 0.0, res = 1.0, tol_cur = tol;
  bool escalate = false;
  const size_t nb = sizeof(double) * (size_t)s->g.n;
  constexpr int kMaxRestarts = 16;
  // A pass that meets the reference's stop test (its recurrence residual, relative to the solve's
  // res0, below tol: NonUniform.jl:331-332) ends the solve when the recomputed residual b - A theta
  // is within this factor of tol: the recomputed residual carries the rounding of A theta (ss
  // cancelling dd theta), which near 1e-8 is what separates the two.
  constexpr double kTrueSlack = 10.0;
  constexpr double kDivergedFP32 = 1.0e4;
  int restart = 0;
  if (!s->th_prev) CK(cudaMalloc(&s->th_prev, nb));
  for (; restart < kMaxRestarts && total < maxItr; ++restart) {
    // theta before this pass: restored if the FP32-preconditioned pass breaks down
    CK(cudaMemcpyAsync(s->th_prev, s->th, nb, cudaMemcpyDeviceToDevice, s->stream));
    h2g_result r;
    memset(&r, 0, sizeof r);
    // a pass whose residual grows past 1e4 times its start has diverged (the FP32 smoother's
    // rounding, amplified by the operator): it stops there, and the FP64 finish takes over
    s->div_limit = kDivergedFP32;
    const int st = solve_krylov<float>(s, cg, tol_cur, maxItr - total, smoother, verbose && restart == 0,
                                       res_hist ? res_hist + total : nullptr, &r);
    s->div_limit = 0.0;
    if (st == H2G_BAD_ARG || st == H2G_CUDA_ERROR || st == H2G_TIMEOUT) return st;
    ++passes;
    launches += r.launches + 3;
    total += r.itr;
    if (restart == 0) res0 = r.res0;
    if (res0 == 0.0) { status = H2G_OK; converged = 1; res = 0.0; break; }
    double tr;
    int rc;
    if ((rc = true_residual(s, &tr))) return rc;
    if (!std::isfinite(tr) || st == H2G_NONFINITE || st == H2G_BREAKDOWN) {
      if (!std::isfinite(res0)) { status = H2G_NONFINITE; break; }
      CK(cudaMemcpyAsync(s->th, s->th_prev, nb, cudaMemcpyDeviceToDevice, s->stream));
      escalate = true;
      break;
    }
    const double res_before = restart == 0 ? 1.0 : res;
    res = tr / res0;
    if (res < tol) { status = H2G_OK; converged = 1; break; }
    if (st == H2G_OK && res < kTrueSlack * tol) {
      status = H2G_OK;
      converged = 1;
      res = r.res * (r.res0 / res0);  // the pass's recurrence residual, as the FP64 path reports
      break;
    }
    if (st != H2G_OK && st != H2G_NOT_CONVERGED) { status = st; break; }
    if (r.itr == 0) break;
    // a restart that did not halve the true residual: the FP32 smoother's rounding has become the
    // limit; go on in FP64 from this theta
    if (restart > 0 && res > 0.5 * res_before) {
      escalate = true;
      break;
    }
    tol_cur = tol / res;  // relative to the restart's initial residual
  }
  // the FP32-preconditioned restarts ran out before the tolerance: the FP64 finish as well
  if (!converged && !escalate && restart == kMaxRestarts && total < maxItr && std::isfinite(res)) escalate = true;
  if (escalate) {
    // the FP32 smoother's rounding broke or stalled the iteration: finish with the FP64
    // preconditioner from the last good theta (res is its relative true residual), restarting on
    // the true residual like the FP32 passes.  The Krylov buffers held FP32 data and possibly non-finite
    // values (a NaN step length reaches the guard entries of the linear updates); the FP64
    // kernels need their guards zero, so clear them all first, and again at the end for the FP32
    // layout of the next mixed solve on this handle.
    for (int i : {0, 1, 2, 3, 4, 5, 6, 7, (int)KP2}) CK(cudaMemsetAsync(s->kv[i], 0, s->elem * (size_t)s->g.n, s->stream));
    status = H2G_NOT_CONVERGED;
    for (int pass = 0; pass < 4 && total < maxItr; ++pass) {
      h2g_result r;
      memset(&r, 0, sizeof r);
      const int st = solve_krylov<double>(s, cg, tol / res, maxItr - total, smoother, 0,
                                          res_hist ? res_hist + total : nullptr, &r);
      if (st == H2G_BAD_ARG || st == H2G_CUDA_ERROR || st == H2G_TIMEOUT) return st;
      ++passes;
      launches += r.launches + 1;
      total += r.itr;
      double tr;
      int rc;
      if ((rc = true_residual(s, &tr))) return rc;
      res = tr / res0;
      if (!std::isfinite(res)) { status = H2G_NONFINITE; break; }
      if (res < tol) { status = H2G_OK; converged = 1; break; }
      if (st == H2G_OK && res < kTrueSlack * tol) {
        status = H2G_OK;
        converged = 1;
        res = r.res * (r.res0 / res0);
        break;
      }
      if (st != H2G_OK && st != H2G_NOT_CONVERGED) { status = st; break; }
      if (r.itr == 0) break;
    }
    for (int i : {0, 1, 2, 3, 4, 5, 6, 7, (int)KP2}) CK(cudaMemsetAsync(s->kv[i], 0, s->elem * (size_t)s->g.n, s->stream));
  }
  if (out) {
    out->isconverged = converged;
    out->itr = total;
    out->outer = passes;
    out->status = status;
    out->res0 = res0;
    out->res = res;
    out->launches = launches;
  }
  return status;
}

// ------------------------------------------------------------------------------------------
// K right-hand sides on one operator (h2g_create_multi): PBiCGSTAB! + RB-GS for all of them at
// once, every right-hand side with its own scalars and stop test (h2g_multi.cuh).
// ------------------------------------------------------------------------------------------
static dim3 mr_grid(const Geo& g, int K) {
  const int G = (K + kMrR - 1) / kMrR;
  return dim3((g.HN + kBX - 1) / kBX, (g.NY + kBY - 1) / kBY, g.NZ * G);
}

template <bool CL>
static int launch_pbicg_body_mr(Solver* s, cudaStream_t cs, const OpParams<double>& op, cudaGraphConditionalHandle hc,
                                int use_cond) {
  const Geo& g = s->g;
  const int K = s->nrhs;
  const long long n = g.n;
  double *r = s->mr_kv[0], *r0 = s->mr_kv[1], *p = s->mr_kv[2], *ph = s->mr_kv[3], *q = s->mr_kv[4],
         *sv = s->mr_kv[5], *sh = s->mr_kv[6], *t = s->mr_kv[7];
  const dim3 grid = mr_grid(g, K), blk(kBX, kBY);
  SolverState* st = s->mr_st;
  // p = r + beta (p - omega q); p_ = M^-1 p                     NonUniform.jl:296-305
  launch(s, k_rb_first_mr<1, kMrR, CL>, grid, blk, cs, op, ph, p, (const double*)r, (const double*)q,
         (const SolverState*)st, K, n);
  for (int pass = 1; pass < 2 * kSweeps; ++pass)
    launch(s, k_rb_pass_mr<kMrR, CL>, grid, blk, cs, op, ph, (const double*)p, pass & 1, (const SolverState*)st, K, n);
  // q = A p_;  alpha = rho / (q, r0)                            NonUniform.jl:307-309
  launch(s, k_ax_mr<1, kMrR, CL>, grid, blk, cs, op, q, (const double*)ph, (const double*)r0, (const double*)nullptr, st,
         s->mr_partials, (int)kStageAlpha, K, n);
  // s = r - alpha q; s_ = M^-1 s                                NonUniform.jl:310-315
  launch(s, k_rb_first_mr<2, kMrR, CL>, grid, blk, cs, op, sh, sv, (const double*)r, (const double*)q,
         (const SolverState*)st, K, n);
  for (int pass = 1; pass < 2 * kSweeps; ++pass)
    launch(s, k_rb_pass_mr<kMrR, CL>, grid, blk, cs, op, sh, (const double*)sv, pass & 1, (const SolverState*)st, K, n);
  // t = A s_; omega = (t,s)/(t,t)                               NonUniform.jl:317-326
  launch(s, k_ax_mr<2, kMrR, CL>, grid, blk, cs, op, t, (const double*)sh, (const double*)nullptr, (const double*)sv, st,
         s->mr_partials, (int)kStageOmega, K, n);
  // x += alpha p_ + omega s_; r = s - omega t; res; next rho    NonUniform.jl:328-346
  const dim3 ug(elementwise_blocks(s), K);
  if (use_cond)
    launch(s, k_bicg_update_mr<true>, ug, 256, cs, n, s->mr_th, (const double*)ph, (const double*)sh, r,
           (const double*)sv, (const double*)t, (const double*)r0, st, s->mr_ctl, s->mr_partials, hc, use_cond);
  else
    launch(s, k_bicg_update_mr<false>, ug, 256, cs, n, s->mr_th, (const double*)ph, (const double*)sh, r,
           (const double*)sv, (const double*)t, (const double*)r0, st, s->mr_ctl, s->mr_partials, hc, use_cond);
  return H2G_OK;
}

static int solve_multi(Solver* s, double tol, int maxItr, int smoother, h2g_result* outs) {
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (maxItr < 1 || maxItr > 10000000) return fail(H2G_BAD_ARG, "maxItr out of range: %d", maxItr);
  if (smoother != H2G_SMOOTHER_GS)
    return fail(H2G_UNSUPPORTED, "a multi right-hand-side solve runs the RB-GS preconditioner (smoother gs)");
  if (!(tol >= 0.0) || !std::isfinite(tol)) return fail(H2G_BAD_ARG, "bad tolerance");
  if (!outs) return fail(H2G_BAD_ARG, "null result array");
  CK(cudaSetDevice(s->device));
  const Geo& g = s->g;
  const int K = s->nrhs;
  OpParams<double> op = op_params<double>(s, s->t64);
  launch(s, k_prime_mr, 1, kMrMax, s->stream, s->mr_st, s->mr_ctl, tol, maxItr, K);
  // r = b - A theta, r0 = r, res0 and rho of every right-hand side   NonUniform.jl:262-274
  if (op.cls)
    launch(s, k_rk_mr<kMrR, true>, mr_grid(g, K), dim3(kBX, kBY), s->stream, op, s->mr_kv[0], s->mr_kv[1],
           (const double*)s->mr_th, (const double*)s->mr_b, s->mr_st, s->mr_partials, (int)kStageInit, K, g.n);
  else
    launch(s, k_rk_mr<kMrR, false>, mr_grid(g, K), dim3(kBX, kBY), s->stream, op, s->mr_kv[0], s->mr_kv[1],
           (const double*)s->mr_th, (const double*)s->mr_b, s->mr_st, s->mr_partials, (int)kStageInit, K, g.n);
  CKL();
  SolveGraph& G = s->mr_graph;
  std::vector<unsigned char> sig = signature(op, op, smoother, (const void*)s->mr_th);
  if (!G.exec || G.sig != sig) {
    int berr = H2G_OK;
    int rc = make_loop_graph(s, G, [&](cudaStream_t cs, cudaGraphConditionalHandle hc, int use_cond) {
      for (int u = 0; u < kUnroll && berr == H2G_OK; ++u)
        berr = op.cls ? launch_pbicg_body_mr<true>(s, cs, op, hc, use_cond)
                      : launch_pbicg_body_mr<false>(s, cs, op, hc, use_cond);
    });
    if (rc == H2G_OK && berr != H2G_OK) G.reset();
    if (rc) return rc;
    if (berr) return berr;
    G.sig = sig;
  }
  if (G.cond) {
    CK(cudaGraphLaunch(G.exec, s->stream));
  } else {
    int done = 0, any = 1;
    while (done < maxItr + 1 && any) {
      for (int i = 0; i < 8; ++i) CK(cudaGraphLaunch(G.exec, s->stream));
      done += 8 * kUnroll;
      k_any_running<<<1, 1, 0, s->stream>>>(s->mr_st, K, s->mr_flag);
      CK(cudaMemcpyAsync(&any, s->mr_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
    }
  }
  std::vector<SolverState> fin(K);
  CK(cudaMemcpyAsync(fin.data(), s->mr_st, sizeof(SolverState) * K, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  int status = H2G_OK;
  const long long per_iter = 2 * (2 * kSweeps) + 2 + 1;
  for (int q = 0; q < K; ++q) {
    h2g_result& o = outs[q];
    o.isconverged = fin[q].converged;
    o.itr = fin[q].itr;
    o.outer = 0;
    o.status = status_of(fin[q]);
    o.res0 = fin[q].res0;
    o.res = fin[q].res;
    o.launches = 2 + per_iter * std::max(1, fin[q].itr);
    if (status == H2G_OK && o.status != H2G_OK) status = o.status;
  }
  return status;
}

static int autotune(Solver* s);

static int solve(Solver* s, bool cg, double tol, int maxItr, int smoother, int verbose, double* res_hist,
                 h2g_result* out) {
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (maxItr < 1 || maxItr > 10000000) return fail(H2G_BAD_ARG, "maxItr out of range: %d", maxItr);
  if (smoother != H2G_SMOOTHER_NONE && smoother != H2G_SMOOTHER_GS)
    return fail(H2G_BAD_ARG, "Unsupported smoother: %d. Use none (0) or gs (1)", smoother);
  if (!(tol >= 0.0) || !std::isfinite(tol)) return fail(H2G_BAD_ARG, "bad tolerance");
  CK(cudaSetDevice(s->device));
  if (int rc = autotune(s)) return rc;
  int rc;
  if (s->precision == H2G_MIXED_IR) rc = solve_ir(s, cg, tol, maxItr, smoother, verbose, res_hist, out);
  else if (s->precision == H2G_MIXED) rc = solve_mixed(s, cg, tol, maxItr, smoother, verbose, res_hist, out);
  else rc = solve_krylov<double>(s, cg, tol, maxItr, smoother, verbose, res_hist, out);
  if (rc == H2G_BAD_ARG || rc == H2G_CUDA_ERROR) return rc;
  // a fused sweep whose bounded wait ran out stopped the solve: report it as such
  const int e = sweep_status(s);
  if (e != H2G_OK) {
    if (out) {
      out->status = e;
      out->isconverged = 0;
    }
    return e;
  }
  return rc;
}

// ------------------------------------------------------------------------------------------
// creation and set-up
// ------------------------------------------------------------------------------------------
// One rbsor! (colour 0, colour 1, each with its residual sum) with the coefficients from the key
// tables (DDM 1) or the stencil-class table (DDM 2).
template <int DDM>
static void sor_passes(Solver* s, cudaStream_t cs, const OpParams<double>& op, dim3 rg, dim3 blk, double omega,
                       SolverState* st, cudaGraphConditionalHandle hc, int use_cond) {
  launch(s, k_sor_pass<false, DDM>, rg, blk, cs, op, s->th, (const double*)s->b, 0, omega, st, s->partials,
         (int)kStageSorHalf, hc, 0);
  if (use_cond)
    launch(s, k_sor_pass<true, DDM>, rg, blk, cs, op, s->th, (const double*)s->b, 1, omega, st, s->partials,
           (int)kStageSorIter, hc, use_cond);
  else
    launch(s, k_sor_pass<false, DDM>, rg, blk, cs, op, s->th, (const double*)s->b, 1, omega, st, s->partials,
           (int)kStageSorIter, hc, use_cond);
}

// solveSOR! (NonUniform.jl:1004-1051): res0 = resSOR, then rbsor! passes (colour 0, colour 1,
// each with its sum of squared residuals) until sqrt(sum)/res0 < tol.  FP64 on every handle
// precision.  Deviation: a non-finite residual stops the loop (the reference would run maxItr
// passes of NaN).
static int solve_sor(Solver* s, double omega, double tol, int maxItr, int verbose, double* res_hist,
                     h2g_result* out) {
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (maxItr < 1) return fail(H2G_BAD_ARG, "maxItr must be >= 1");
  if (!(omega > 0.0 && omega < 2.0)) return fail(H2G_BAD_ARG, "omega must lie in (0, 2)");
  const Geo& g = s->g;
  int rc = ensure_hist(s, maxItr);
  if (rc) return rc;
  const OpParams<double> op = op_params<double>(s, s->t64);
  SolverState* st = s->st;
  if ((rc = prime_state(s, st, tol, maxItr, s->hist, maxItr))) return rc;
  const dim3 ag = ax_grid(g), rg = rb_grid(g), blk(kBX, kBY);
  launch(s, k_res_sor, ag, blk, s->stream, op, (const double*)s->th, (const double*)s->b, omega, st, s->partials,
         (int)kStageSorInit);
  CKL();
  SolveGraph& G = s->graphs[kGSor][0];
  std::vector<unsigned char> sig(sizeof op + sizeof omega);
  memcpy(sig.data(), &op, sizeof op);
  memcpy(sig.data() + sizeof op, &omega, sizeof omega);
  if (!G.exec || G.sig != sig) {
    rc = make_loop_graph(s, G, [&](cudaStream_t cs, cudaGraphConditionalHandle hc, int use_cond) {
      if (op.cls) sor_passes<2>(s, cs, op, rg, blk, omega, st, hc, use_cond);
      else sor_passes<1>(s, cs, op, rg, blk, omega, st, hc, use_cond);
    });
    if (rc) return rc;
    G.sig = sig;
  }
  if ((rc = run_graph(s, &G, st, maxItr, 1))) return rc;
  CK(cudaMemcpyAsync(s->st_host, st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  SolverState fin = *s->st_host;
  const int nh = std::min(std::max(fin.itr, 0), maxItr);
  std::vector<double> hh(nh);
  if (nh > 0 && (verbose || res_hist)) {
    CK(cudaMemcpy(hh.data(), s->hist, sizeof(double) * nh, cudaMemcpyDeviceToHost));
    if (res_hist) memcpy(res_hist, hh.data(), sizeof(double) * nh);
  }
  if (verbose) print_log(fin, hh.data(), nh, fin.converged);
  if (out) {
    out->launches = 2 + 2LL * std::max(1, fin.itr);
    out->isconverged = fin.converged;
    out->itr = fin.itr;
    out->outer = 0;
    out->status = status_of(fin);
    out->res0 = fin.res0;
    out->res = fin.res;
  }
  return status_of(fin);
}

// ---- calRHS! and the time loop of main() ----------------------------------------------------

static int face_bc(const h2g_bc* bc, FaceBC& f) {
  if (!bc) return fail(H2G_BAD_ARG, "null boundary-condition array");
  for (int q = 0; q < 6; ++q) {
    const int t = bc[q].type;
    if (t != H2G_ISOTHERMAL && t != H2G_HEAT_FLUX && t != H2G_CONVECTION)
      return fail(H2G_BAD_ARG, "face %d: unknown boundary type %d", q, t);
    f.type[q] = t;
    f.q[q] = bc[q].heat_flux;
    f.h[q] = bc[q].htc;
    f.ta[q] = bc[q].ambient;
  }
  return H2G_OK;
}

static int ensure_hsrc(Solver* s) {
  if (s->hsrc) return H2G_OK;
  CK(cudaMalloc(&s->hsrc, sizeof(double) * (size_t)s->g.n));
  CK(cudaMemsetAsync(s->hsrc, 0, sizeof(double) * (size_t)s->g.n, s->stream));
  return H2G_OK;
}

static int calrhs(Solver* s, const FaceBC& f, int zero_b) {
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (!s->steady && !s->rc64) return fail(H2G_BAD_ARG, "a transient grid needs rho and cp (h2g_set_fields)");
  int rc = ensure_hsrc(s);
  if (rc) return rc;
  const Geo& g = s->g;
  dim3 grid((g.NX + 127) / 128, g.NY, g.NZ);
  k_calrhs<<<grid, 128, 0, s->stream>>>(g, s->b, s->th, s->hsrc, s->rc64, s->t64.dzk, s->dx, s->dy,
                                         s->steady ? 0.0 : 1.0 / s->dt, s->steady, f, zero_b);
  CKL();
  return H2G_OK;
}

// main()'s time loop (heat3ds.jl:123-151) with theta resident on the device: per step calRHS!
// (b cleared first: the reference accumulates b across steps), the Krylov solve from the previous
// step's theta, and the interior min / max / L2 norm of theta.
static int transient(Solver* s, const FaceBC& f, int nt, int method, double tol, int maxItr, int smoother,
                     int verbose, double* step_stats, h2g_result* out) {
  if (nt < 1) return fail(H2G_BAD_ARG, "nt must be >= 1");
  if (method != 0 && method != 1) return fail(H2G_BAD_ARG, "method must be 0 (PBiCGSTAB) or 1 (CG)");
  const int nb1 = s->num_sms * 2;
  if (s->stats_cap < nt) {
    cudaFree(s->stats);
    s->stats = nullptr;
    s->stats_cap = 0;
    CK(cudaMalloc(&s->stats, sizeof(double) * (3 * (size_t)nt + 3 * (size_t)nb1)));
    s->stats_cap = nt;
  }
  double* part = s->stats + 3 * (size_t)nt;
  std::vector<int> itrs(nt, 0);
  std::vector<double> ress(nt, 0.0);
  long long launches = 0;
  int all_conv = 1, last = H2G_OK, done = 0;
  h2g_result r{};
  for (int step = 0; step < nt; ++step) {
    int rc = calrhs(s, f, 1);
    if (rc) return rc;
    const int st = solve(s, method == 1, tol, maxItr, smoother, verbose, nullptr, &r);
    if (st == H2G_BAD_ARG || st == H2G_CUDA_ERROR || st == H2G_TIMEOUT) return st;
    k_theta_stats1<<<nb1, 256, 0, s->stream>>>(s->g, s->th, part);
    k_theta_stats2<<<1, 32, 0, s->stream>>>(part, nb1, s->stats + 3 * (size_t)step);
    CKL();
    itrs[step] = r.itr;
    ress[step] = r.res;
    launches += r.launches + 3;
    all_conv &= r.isconverged;
    if (st != H2G_OK) last = st;
    ++done;
    if (st == H2G_NONFINITE) break;
  }
  if (step_stats) {
    std::vector<double> hs(3 * (size_t)done);
    CK(cudaMemcpyAsync(hs.data(), s->stats, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    for (int q = 0; q < done; ++q) {
      step_stats[5 * q + 0] = hs[3 * q + 0];
      step_stats[5 * q + 1] = hs[3 * q + 1];
      step_stats[5 * q + 2] = hs[3 * q + 2];
      step_stats[5 * q + 3] = itrs[q];
      step_stats[5 * q + 4] = ress[q];
    }
  }
  CK(cudaStreamSynchronize(s->stream));
  if (out) {
    long long tot = 0;
    for (int q = 0; q < done; ++q) tot += itrs[q];
    out->isconverged = all_conv;
    out->itr = (int)std::min<long long>(tot, 2147483647LL);
    out->outer = done;
    out->status = last;
    out->res0 = r.res0;
    out->res = r.res;
    out->launches = launches;
  }
  return last;
}

// ---- steady adjoint -------------------------------------------------------------------------
// Forward solve, J = (sum w theta^p)^(1/p), adjoint solve A la = dJ/dtheta with the same solver
// (the operator is symmetric: lambda_f is symmetric in its arguments and every face area and
// distance is shared by the two cells of the face), then the gradients.
static int adjoint(Solver* s, const double* w_host, double p, double tol, int maxItr, int smoother, double* J,
                   double* dJ_dhsrc, double* dJ_dlnlam, h2g_result* out_fwd, h2g_result* out_adj) {
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (!w_host || !J) return fail(H2G_BAD_ARG, "null weights or J");
  if (!(p >= 1.0)) return fail(H2G_BAD_ARG, "p must be >= 1");
  const Geo& g = s->g;
  const size_t nb = sizeof(double) * (size_t)g.n;
  for (auto& q : s->adj)
    if (!q) {
      CK(cudaMalloc(&q, nb));
      CK(cudaMemsetAsync(q, 0, nb, s->stream));
    }
  double *W = s->adj[0], *gv = s->adj[1], *la = s->adj[2], *G = s->adj[3], *gh = s->adj[4];
  int rc = upload<double>(s, w_host, W);
  if (rc) return rc;
  // forward
  h2g_result rf{};
  int st = solve(s, false, tol, maxItr, smoother, 0, nullptr, &rf);
  if (out_fwd) *out_fwd = rf;
  if (st != H2G_OK) return st;
  // objective and adjoint right-hand side
  if ((rc = prime_state(s, s->st, tol, maxItr, s->hist, maxItr))) return rc;
  launch(s, k_objective, elementwise_blocks(s), 256, s->stream, g.n, (const double*)s->th, (const double*)W, p,
         s->st, s->partials);
  launch(s, k_adj_rhs, elementwise_blocks(s), 256, s->stream, g.n, (const double*)s->th, (const double*)W, p,
         (const SolverState*)s->st, gv);
  CKL();
  CK(cudaMemcpyAsync(s->st_host, s->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemsetAsync(la, 0, nb, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const double sum = s->st_host->dot1;
  *J = pow(sum, 1.0 / p);
  if (!(sum > 0.0) || !std::isfinite(sum)) return fail(H2G_NONFINITE, "objective sum %g", sum);
  // adjoint solve on (la, g) in place of (theta, b)
  std::swap(s->th, la);
  std::swap(s->b, gv);
  h2g_result ra{};
  st = solve(s, false, tol, maxItr, smoother, 0, nullptr, &ra);
  std::swap(s->th, la);
  std::swap(s->b, gv);
  if (out_adj) *out_adj = ra;
  if (st != H2G_OK) return st;
  // gradients
  if (!s->lamv) CK(cudaMalloc(&s->lamv, sizeof(double) * kMaxKeys));
  CK(cudaMemcpyAsync(s->lamv, s->lam_values.data(), sizeof(double) * s->lam_values.size(), cudaMemcpyHostToDevice,
                     s->stream));
  const OpParams<double> op = op_params<double>(s, s->t64);
  dim3 grid((g.NX + 127) / 128, g.NY, g.NZ);
  k_adj_grad<<<grid, 128, 0, s->stream>>>(op, s->lamv, s->th, la, G, gh, 0);
  CKL();
  if (dJ_dlnlam && (rc = download<double>(s, G, dJ_dlnlam))) return rc;
  if (dJ_dhsrc && (rc = download<double>(s, gh, dJ_dhsrc))) return rc;
  CK(cudaStreamSynchronize(s->stream));
  return H2G_OK;
}

// Transient adjoint of J(theta^N), theta^{n+1} = A^-1 b(theta^n) for nt steps of main()'s loop
// (b rebuilt from zero each step), with checkpointed recomputation: the forward pass keeps
// theta at every K-th step; the backward pass recomputes one segment of K states at a time from
// its checkpoint (the solves are deterministic, so the recomputed states are the same bits), then
// for n = N-1 .. 0:  mu = A^-1 lam (adjoint solve),  accumulate the gradients of step n with
// theta^{n+1} and mu,  lam = (db/dtheta^n) mu.  Device memory: ceil(nt/K) + K + 1 states.
static int adjoint_transient(Solver* s, const FaceBC& f, int nt, const double* w_host, double p, double tol,
                             int maxItr, int smoother, int K, double* J, double* dJ_dhsrc, double* dJ_dlnlam,
                             h2g_result* out) {
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (s->steady || !s->rc64) return fail(H2G_BAD_ARG, "the transient adjoint needs a transient grid with rho and cp");
  if (nt < 1 || K < 1) return fail(H2G_BAD_ARG, "nt and checkpoint_every must be >= 1");
  if (!w_host || !J) return fail(H2G_BAD_ARG, "null weights or J");
  if (!(p >= 1.0)) return fail(H2G_BAD_ARG, "p must be >= 1");
  K = std::min(K, nt);
  const Geo& g = s->g;
  const size_t n = (size_t)g.n, nb = sizeof(double) * n;
  const int ncp = (nt + K - 1) / K;
  const size_t need = (size_t)ncp + (size_t)K + 1;
  int rc = ensure_hsrc(s);
  if (rc) return rc;
  for (auto& q : s->adj)
    if (!q) {
      CK(cudaMalloc(&q, nb));
      CK(cudaMemsetAsync(q, 0, nb, s->stream));
    }
  if (s->tstates_cap < need) {
    cudaFree(s->tstates);
    s->tstates = nullptr;
    s->tstates_cap = 0;
    CK(cudaMalloc(&s->tstates, nb * need));
    s->tstates_cap = need;
  }
  double* cp = s->tstates;              // checkpoints: theta^{cK}
  double* seg = s->tstates + n * ncp;   // theta^{n0+1} .. theta^{n0+K}
  double* fin = seg + n * (size_t)K;    // theta^N
  double *W = s->adj[0], *lam = s->adj[1], *G = s->adj[3], *gh = s->adj[4];
  if ((rc = upload<double>(s, w_host, W))) return rc;
  if (!s->lamv) CK(cudaMalloc(&s->lamv, sizeof(double) * kMaxKeys));
  CK(cudaMemcpyAsync(s->lamv, s->lam_values.data(), sizeof(double) * s->lam_values.size(), cudaMemcpyHostToDevice,
                     s->stream));
  long long itr_total = 0, launches = 0;
  auto step = [&](int nstep) -> int {
    int r2 = calrhs(s, f, 1);
    if (r2) return r2;
    h2g_result r{};
    const int st = solve(s, false, tol, maxItr, smoother, 0, nullptr, &r);
    itr_total += r.itr;
    launches += r.launches + 1;
    if (st != H2G_OK) return fail(st, "forward step %d: %s", nstep + 1, h2g_status_string(st));
    return H2G_OK;
  };
  // forward pass
  for (int q = 0; q < nt; ++q) {
    if (q % K == 0) CK(cudaMemcpyAsync(cp + n * (size_t)(q / K), s->th, nb, cudaMemcpyDeviceToDevice, s->stream));
    if ((rc = step(q))) return rc;
  }
  CK(cudaMemcpyAsync(fin, s->th, nb, cudaMemcpyDeviceToDevice, s->stream));
  // objective and lam^N = dJ/dtheta^N
  if ((rc = prime_state(s, s->st, tol, maxItr, s->hist, maxItr))) return rc;
  launch(s, k_objective, elementwise_blocks(s), 256, s->stream, g.n, (const double*)s->th, (const double*)W, p,
         s->st, s->partials);
  launch(s, k_adj_rhs, elementwise_blocks(s), 256, s->stream, g.n, (const double*)s->th, (const double*)W, p,
         (const SolverState*)s->st, lam);
  CKL();
  CK(cudaMemcpyAsync(s->st_host, s->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemsetAsync(G, 0, nb, s->stream));
  CK(cudaMemsetAsync(gh, 0, nb, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  const double sum = s->st_host->dot1;
  *J = pow(sum, 1.0 / p);
  if (!(sum > 0.0) || !std::isfinite(sum)) return fail(H2G_NONFINITE, "objective sum %g", sum);
  const OpParams<double> op = op_params<double>(s, s->t64);
  const dim3 cgrid((g.NX + 127) / 128, g.NY, g.NZ);
  const double ddt = 1.0 / s->dt;
  // backward pass, one segment at a time
  for (int c = ncp - 1; c >= 0; --c) {
    const int n0 = c * K, n1 = std::min(n0 + K, nt);
    CK(cudaMemcpyAsync(s->th, cp + n * (size_t)c, nb, cudaMemcpyDeviceToDevice, s->stream));
    for (int q = n0; q < n1; ++q) {
      if ((rc = step(q))) return rc;
      CK(cudaMemcpyAsync(seg + n * (size_t)(q - n0), s->th, nb, cudaMemcpyDeviceToDevice, s->stream));
    }
    for (int q = n1 - 1; q >= n0; --q) {
      // mu = A^-1 lam, solved in the handle's theta / b
      CK(cudaMemsetAsync(s->th, 0, nb, s->stream));
      CK(cudaMemcpyAsync(s->b, lam, nb, cudaMemcpyDeviceToDevice, s->stream));
      h2g_result r{};
      const int st = solve(s, false, tol, maxItr, smoother, 0, nullptr, &r);
      itr_total += r.itr;
      launches += r.launches + 2;
      if (st != H2G_OK) return fail(st, "adjoint step %d: %s", q + 1, h2g_status_string(st));
      k_adj_grad<<<cgrid, 128, 0, s->stream>>>(op, s->lamv, seg + n * (size_t)(q - n0), s->th, G, gh, 1);
      k_adj_step<<<cgrid, 128, 0, s->stream>>>(g, s->th, lam, s->rc64, s->t64.dzk, s->dx, s->dy, ddt, f);
      CKL();
    }
  }
  CK(cudaMemcpyAsync(s->th, fin, nb, cudaMemcpyDeviceToDevice, s->stream));
  if (dJ_dlnlam && (rc = download<double>(s, G, dJ_dlnlam))) return rc;
  if (dJ_dhsrc && (rc = download<double>(s, gh, dJ_dhsrc))) return rc;
  CK(cudaStreamSynchronize(s->stream));
  if (out) {
    out->isconverged = 1;
    out->itr = (int)std::min<long long>(itr_total, 2147483647LL);
    out->outer = nt;
    out->status = H2G_OK;
    out->res0 = 0.0;
    out->res = 0.0;
    out->launches = launches;
  }
  return H2G_OK;
}

// ---- launch-shape tuner --------------------------------------------------------------------
// The colour pass has no reduction, so its launch shape changes no result: the first solve of a
// handle times every variant (kRbRows x 1 or 2 planes per thread x dd read or summed) on the
// handle's grid (three interleaved rounds of two warm-up and ten timed sweeps each, on scratch
// vectors) and keeps the fastest.  CalcAX is timed with dd summed and read from the array.
// Choices are cached per (grid, smoother precision) for the process; H2G_RB_ROWS,
// H2G_RB_PLANES, H2G_RB_DD and H2G_AX_DD in the environment force them (all four: no timing; a
// forced rows, planes or dd source also restricts the timed variants to it).
static std::mutex g_tune_mu;
static std::map<std::array<int, 12>, int> g_tune_cache;

static bool valid_rows(int r) {
  for (int q : kRbRows)
    if (q == r) return true;
  return false;
}

// only_rows / only_np / only_dd: -1 = time every value, else only that one (forced by the
// environment)
template <typename T>
static int tune_rows_t(Solver* s, const OpParams<T>& op, int only_rows, int only_np, int only_dd, int* best_rows,
                       float* best_ms) {
  const size_t n = (size_t)s->g.n, bytes = sizeof(double) * n;
  for (auto& p : s->hook)
    if (!p) CK(cudaMalloc(&p, bytes));
  T* xa = static_cast<T*>(s->hook[0]);
  T* xb = static_cast<T*>(s->hook[1]);
  k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)n, xa, T(300));
  k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)n, xb, T(-1.0e-3));
  CKL();
  s->hook_filled = false;  // the timing sweeps change xa; the benchmark hook refills
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(H2G_CUDA_ERROR, "event creation failed");
  }
  const int saved = s->rb_rows, saved_np = s->rb_planes;
  const bool saved_dd = s->rb_dd, saved_cls = s->rb_cls;
  const int nmodes = op.cls ? 3 : 2;  // coefficient sources: dd summed, dd read, class table
  float best = 1e30f;
  int rc = H2G_OK;
  // warm the GPU up first (clocks ramp), then time every shape twice, interleaved, keeping the
  // better time of each, so that no shape is favoured by its place in the order
  for (int r = 0; r < 20; ++r) {
    launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 0, T(1), nullptr);
    launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 1, T(1), nullptr);
  }
  constexpr int kShapes = 24;  // 4 block heights x 2 plane counts x 3 coefficient sources
  float tbest[kShapes];
  for (int q = 0; q < kShapes; ++q) tbest[q] = 1e30f;
  constexpr int kRounds = 3;
  for (int round = 0; round < kRounds && rc == H2G_OK; ++round)
  for (int shape = 0; shape < kShapes; ++shape) {
    const int by = kRbRows[shape & 3], np = 1 + ((shape >> 2) & 1), dd = shape >> 3;
    if ((only_rows >= 0 && by != only_rows) || (only_np >= 0 && np != only_np) || (only_dd >= 0 && dd != only_dd) ||
        dd >= nmodes)
      continue;
    s->rb_rows = by;
    s->rb_planes = np;
    s->rb_dd = dd == 1;
    s->rb_cls = dd == 2;
    for (int r = 0; r < 2; ++r) {
      launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 0, T(1), nullptr);
      launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 1, T(1), nullptr);
    }
    cudaEventRecord(e0, s->stream);
    for (int r = 0; r < 10; ++r) {
      launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 0, T(1), nullptr);
      launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 1, T(1), nullptr);
    }
    cudaEventRecord(e1, s->stream);
    float ms = 0.f;
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      rc = fail(H2G_CUDA_ERROR, "launch-shape tuning failed");
      break;
    }
    tbest[shape] = std::min(tbest[shape], ms);
    if (round == kRounds - 1 && tbest[shape] < best) {
      best = tbest[shape];
      *best_rows = by | (np << 5) | ((dd & 1) << 8) | ((dd >> 1) << 20);
    }
  }
  if (best == 1e30f) *best_rows = kBY | (2 << 5) | (1 << 8);  // nothing timed: the defaults
  *best_ms = best;
  s->rb_rows = saved;
  s->rb_planes = saved_np;
  s->rb_dd = saved_dd;
  s->rb_cls = saved_cls;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Chunk counts along z worth timing for the fused sweep: each distinct planes-per-chunk value with
// at least 3 planes per chunk and at most 16 blocks per SM in all.
static std::vector<int> sweep_chunk_candidates(const Solver* s) {
  const dim3 g1 = sweep_grid(s->g, 1);
  const long long tiles = (long long)g1.x * g1.y;
  std::vector<int> out;
  int last_kc = -1;
  for (int c : {1, 2, 3, 4, 5, 6, 8, 10, 12, 16}) {
    const int kc = (s->g.NZ + c - 1) / c;
    if (kc == last_kc || (kc < 3 && c > 1) || tiles * c > 16LL * s->num_sms) continue;
    out.push_back(c);
    last_kc = kc;
  }
  if (out.empty()) out.push_back(1);
  return out;
}

// Fused sweep against the colour passes: times 10 fused sweeps (x ping-ponging between two
// scratch vectors) per (chunk count, dd source) and keeps the fastest if it beats unfused_ms, the
// best 10 unfused sweeps.  *choice: bit 0 fused, bit 1 dd read, bits 2-9 chunk count.
// only_fused / only_chunks / only_dda: -1 = free, else forced by the environment.
template <typename T>
static int tune_sweep_t(Solver* s, const OpParams<T>& op, float unfused_ms, int only_fused, int only_chunks,
                        int only_dda, int* choice) {
  *choice = 0;
  if (only_fused == 0) return H2G_OK;
  if (int rc = sweep_attrs()) return rc;
  const size_t bytes = sizeof(double) * (size_t)s->g.n;
  for (auto& p : s->hook)
    if (!p) CK(cudaMalloc(&p, bytes));
  T* xa = static_cast<T*>(s->hook[0]);
  T* xb = static_cast<T*>(s->hook[1]);
  T* xc = static_cast<T*>(s->hook[2]);
  k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)s->g.n, xa, T(300));
  k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)s->g.n, xb, T(-1.0e-3));
  k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)s->g.n, xc, T(300));
  CKL();
  s->hook_filled = false;
  std::vector<int> cands = sweep_chunk_candidates(s);
  if (only_chunks > 0) cands = {only_chunks};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(H2G_CUDA_ERROR, "event creation failed");
  }
  const int saved_c = s->sw_chunks;
  const bool saved_d = s->sw_dda;
  float best = only_fused == 1 ? 1e30f : unfused_ms;
  int rc = H2G_OK;
  for (int round = 0; round < 2 && rc == H2G_OK; ++round)
    for (int c : cands)
      for (int d = 0; d < 2 && rc == H2G_OK; ++d) {
        if (only_dda >= 0 && d != only_dda) continue;
        s->sw_chunks = c;
        s->sw_dda = d != 0;
        for (int r = 0; r < 2 && rc == H2G_OK; ++r) rc = launch_sweep<T>(s, s->stream, op, (r & 1) ? xc : xa,
                                                                         (r & 1) ? xa : xc, xb, nullptr);
        cudaEventRecord(e0, s->stream);
        for (int r = 0; r < 10 && rc == H2G_OK; ++r) rc = launch_sweep<T>(s, s->stream, op, (r & 1) ? xc : xa,
                                                                          (r & 1) ? xa : xc, xb, nullptr);
        cudaEventRecord(e1, s->stream);
        float ms = 0.f;
        if (rc == H2G_OK && (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                             cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
          rc = fail(H2G_CUDA_ERROR, "fused-sweep tuning failed");
        if (rc == H2G_OK && round == 1 && ms < best) {
          best = ms;
          *choice = 1 | (d << 1) | (c << 2);
        }
      }
  s->sw_chunks = saved_c;
  s->sw_dda = saved_d;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == H2G_OK) rc = sweep_status(s);
  return rc;
}

// CalcAX (FP64 operator) with dd summed per cell or read from the array: 1 if reading is faster.
static int tune_ax(Solver* s, int* use_dd) {
  const size_t n = (size_t)s->g.n, bytes = sizeof(double) * n;
  for (auto& p : s->hook)
    if (!p) CK(cudaMalloc(&p, bytes));
  double* xa = static_cast<double*>(s->hook[0]);
  double* xb = static_cast<double*>(s->hook[1]);
  k_fill_const<double><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)n, xa, 300.0);
  CKL();
  const OpParams<double> op = op_params<double>(s, s->t64);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(H2G_CUDA_ERROR, "event creation failed");
  }
  const bool saved = s->ax_dd, saved_cls = s->ax_cls;
  const int nmodes = op.cls ? 3 : 2;  // dd summed, dd read, class table
  float t[3] = {0.f, 0.f, 1e30f};
  int rc = H2G_OK;
  for (int v = 0; v < nmodes && rc == H2G_OK; ++v) {
    s->ax_dd = v == 1;
    s->ax_cls = v == 2;
    for (int r = 0; r < 2; ++r) launch_ax<double, 0, double>(s, s->stream, op, xb, xa, nullptr, nullptr, nullptr, 0);
    cudaEventRecord(e0, s->stream);
    for (int r = 0; r < 10; ++r) launch_ax<double, 0, double>(s, s->stream, op, xb, xa, nullptr, nullptr, nullptr, 0);
    cudaEventRecord(e1, s->stream);
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&t[v], e0, e1) != cudaSuccess)
      rc = fail(H2G_CUDA_ERROR, "CalcAX tuning failed");
  }
  s->ax_dd = saved;
  s->ax_cls = saved_cls;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int bestv = 0;
  for (int v = 1; v < nmodes; ++v)
    if (t[v] < t[bestv]) bestv = v;
  *use_dd = bestv;
  return rc;
}

static int autotune(Solver* s) {
  if (s->rb_tuned) return H2G_OK;
  // choices forced by the environment or h2g_set_sweep (-1: not forced)
  int rows = -1, planes = -1, rbdd = -1, dd = -1, fused = -1, chunks = -1, swdd = -1;
  if (const char* e = getenv("H2G_RB_ROWS")) rows = valid_rows(atoi(e)) ? atoi(e) : -1;
  if (const char* e = getenv("H2G_RB_PLANES")) planes = (atoi(e) == 1 || atoi(e) == 2) ? atoi(e) : -1;
  // coefficient sources: 0 dd summed, 1 dd read, 2 stencil-class table (when built)
  const int nmodes = s->cls_ok ? 3 : 2;
  if (const char* e = getenv("H2G_RB_DD")) rbdd = std::min(std::max(atoi(e), 0), nmodes - 1);
  if (const char* e = getenv("H2G_AX_DD")) dd = std::min(std::max(atoi(e), 0), nmodes - 1);
  if (const char* e = getenv("H2G_RB_FUSED")) fused = atoi(e) ? 1 : 0;
  if (const char* e = getenv("H2G_SW_CHUNKS")) chunks = (atoi(e) >= 1 && atoi(e) <= 255) ? atoi(e) : -1;
  if (const char* e = getenv("H2G_SW_DD")) swdd = atoi(e) ? 1 : 0;
  if (s->sweep_forced >= 0) {
    fused = s->sweep_forced;
    chunks = s->sweep_forced ? s->sw_chunks : -1;
    swdd = s->sweep_forced ? (s->sw_dda ? 1 : 0) : -1;
  }
  // the cooperative preconditioner runs on the colour-pass path: asking for it fixes that path
  if (s->coop_forced == 1 && s->sweep_forced != 1) fused = 0;
  if (chunks > s->g.NZ) chunks = s->g.NZ;
  const bool sweep_known = fused == 0 || (fused == 1 && chunks > 0 && swdd >= 0);
  if (rows < 0 || planes < 0 || rbdd < 0 || dd < 0 || !sweep_known) {
    // cached per grid, smoother precision and the choices the environment restricts it to
    const std::array<int, 12> key = {s->g.MX, s->g.MY,  s->g.MZ, s->precision == H2G_FP64 ? 64 : 32,
                                     rows,    planes,   rbdd,    dd,
                                     fused,   chunks,   swdd,    nmodes};
    int cached = 0;
    {
      // held while tuning, so that handles of one grid solved concurrently (h2g_batch_solve) tune
      // once and no two tunings disturb each other's timings
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) cached = it->second;
      if (!cached) {
        int r2 = 0, d2 = 0, sw = 0;
        float unfused_ms = 1e30f;
        int rc = s->precision == H2G_FP64
                     ? tune_rows_t<double>(s, op_params<double>(s, s->t64), rows, planes, rbdd, &r2, &unfused_ms)
                     : tune_rows_t<float>(s, op_params<float>(s, s->t32), rows, planes, rbdd, &r2, &unfused_ms);
        if (!rc) rc = tune_ax(s, &d2);
        if (!rc && !sweep_known) {
          // the fused sweep is timed with the colour-pass shape just chosen for its first pass
          const int sr = s->rb_rows, sp = s->rb_planes;
          const bool sd = s->rb_dd;
          s->rb_rows = r2 & 0x1f;
          s->rb_planes = (r2 >> 5) & 7;
          s->rb_dd = (r2 >> 8) & 1;  // the fused sweep has no class mode: its first pass reads dd
          rc = s->precision == H2G_FP64
                   ? tune_sweep_t<double>(s, op_params<double>(s, s->t64), unfused_ms, fused, chunks, swdd, &sw)
                   : tune_sweep_t<float>(s, op_params<float>(s, s->t32), unfused_ms, fused, chunks, swdd, &sw);
          s->rb_rows = sr;
          s->rb_planes = sp;
          s->rb_dd = sd;
        }
        if (rc) return rc;
        cached = r2 | ((d2 & 1) << 9) | (sw << 10) | ((d2 >> 1) << 21) | (1 << 30);
        g_tune_cache[key] = cached;
      }
    }
    if (rows < 0) rows = cached & 0x1f;
    if (planes < 0) planes = (cached >> 5) & 7;
    if (rbdd < 0) rbdd = ((cached >> 8) & 1) | (((cached >> 20) & 1) << 1);
    if (dd < 0) dd = ((cached >> 9) & 1) | (((cached >> 21) & 1) << 1);
    if (!sweep_known) {
      const int sw = (cached >> 10) & 0x3ff;
      fused = sw & 1;
      swdd = (sw >> 1) & 1;
      chunks = std::max(1, (sw >> 2) & 0xff);
    }
  }
  if (fused == 1) {
    if (int rc = sweep_attrs()) return rc;
  } else {
    chunks = s->sw_chunks;
    swdd = s->sw_dda ? 1 : 0;
  }
  // the cooperative preconditioner (FP64 handles, colour-pass path): on request only
  int coop = s->coop_forced;
  if (coop < 0) {
    coop = 0;
    if (const char* e = getenv("H2G_RB_COOP")) coop = atoi(e) ? 1 : 0;
  }
  if (s->precision != H2G_FP64 || fused == 1) coop = 0;
  if (rows != s->rb_rows || planes != s->rb_planes || (rbdd == 1) != s->rb_dd || (rbdd == 2) != s->rb_cls ||
      (dd == 1) != s->ax_dd || (dd == 2) != s->ax_cls || (fused == 1) != s->rb_fused || chunks != s->sw_chunks ||
      (swdd != 0) != s->sw_dda || coop != s->rb_coop)
    invalidate_graphs(s);
  s->rb_coop = coop;
  s->rb_rows = rows;
  s->rb_planes = planes;
  s->rb_dd = rbdd == 1;
  s->rb_cls = rbdd == 2;
  s->ax_dd = dd == 1;
  s->ax_cls = dd == 2;
  s->rb_fused = fused == 1;
  s->sw_chunks = chunks;
  s->sw_dda = swdd != 0;
  s->rb_tuned = true;
  return H2G_OK;
}

static int create(int MX, int MY, int MZ, int precision, Solver** out) {
  if (!out) return fail(H2G_BAD_ARG, "null output pointer");
  *out = nullptr;
  if (MX < 3 || MY < 3 || MZ < 3) return fail(H2G_BAD_ARG, "grid too small: (%d,%d,%d)", MX, MY, MZ);
  if ((long long)MX * MY * MZ > (1ll << 31)) return fail(H2G_BAD_ARG, "grid too large");
  if (make_geo(MX, MY, MZ).n >= (1ll << 31) - 1) return fail(H2G_BAD_ARG, "grid too large for 32-bit offsets");
  if (precision != H2G_FP64 && precision != H2G_MIXED && precision != H2G_MIXED_IR)
    return fail(H2G_BAD_ARG, "unknown precision %d", precision);
  Solver* s = new h2g_solver();
  s->g = make_geo(MX, MY, MZ);
  s->precision = precision;
  s->elem = precision == H2G_MIXED_IR ? 4 : 8;
  const char* nc = getenv("H2G_NO_COND");
  s->no_cond = nc && nc[0] == '1';
  const char* np = getenv("H2G_NO_PDL");
  s->pdl = !(np && np[0] == '1');
  auto bail = [&](int code) {
    destroy(s);
    return code;
  };
  if (cudaGetDevice(&s->device) != cudaSuccess) return bail(fail(H2G_CUDA_ERROR, "no CUDA device"));
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device);
  const Geo& g = s->g;
  const size_t nb = sizeof(double) * (size_t)g.n;
#define AL(ptr, bytes)                                                                     \
  do {                                                                                     \
    if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess || cudaMemset((ptr), 0, (bytes)) != cudaSuccess) \
      return bail(fail(H2G_CUDA_ERROR, "cudaMalloc of %zu bytes failed", (size_t)(bytes)));                \
  } while (0)
  AL(s->th, nb);
  AL(s->b, nb);
  AL(s->th_snap, nb);
  AL(s->key, (size_t)g.n);
  const size_t kvb = s->elem * (size_t)g.n;
  for (int i = 0; i < 8; ++i) AL(s->kv[i], kvb);
  AL(s->kv[KP2], kvb);
  if (precision == H2G_MIXED) AL(s->kv[KBB], sizeof(float) * (size_t)g.n);
  AL(s->x2_64, nb);
  if (precision != H2G_FP64) AL(s->x2_32, sizeof(float) * (size_t)g.n);
  AL(s->sweep_err, sizeof(int));
  AL(s->gbar, sizeof(GridBar));
  if (precision == H2G_MIXED_IR) {
    AL(s->kv[KE], kvb);
    AL(s->r64, nb);
  }
  for (int i = 0; i < 4; ++i) AL(s->stage[i], sizeof(double) * (size_t)s->nfort());
  AL(s->st, sizeof(SolverState));
  AL(s->st_in, sizeof(SolverState));
  s->partials_cap = partials_needed(s);
  AL(s->partials, sizeof(double) * s->partials_cap);
  AL(s->slots, sizeof(unsigned long long) * kHashSlots);
  AL(s->slot_index, sizeof(int) * kHashSlots);
  AL(s->flags, sizeof(int));
#undef AL
  if (cudaMallocHost(&s->st_host, sizeof(SolverState)) != cudaSuccess)
    return bail(fail(H2G_CUDA_ERROR, "cudaMallocHost failed"));
  if (cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(H2G_CUDA_ERROR, "cudaStreamCreate failed"));
  *out = s;
  return H2G_OK;
}

// build = false leaves the operator tables to the h2g_set_fields that follows (one-call path).
static int set_grid(Solver* s, const double* ZC, const double* dZ, double dx, double dy, double dt, const double* HC,
                    int is_steady, bool build = true) {
  if (!ZC || !dZ || !HC) return fail(H2G_BAD_ARG, "null ZC/dZ/HC");
  if (!(dx > 0) || !(dy > 0) || !std::isfinite(dx) || !std::isfinite(dy)) return fail(H2G_BAD_ARG, "bad dx/dy");
  if (!is_steady && !(dt > 0 && std::isfinite(dt))) return fail(H2G_BAD_ARG, "bad dt");
  const int MZ = s->g.MZ;
  for (int k = 0; k < MZ; ++k)
    if (!std::isfinite(ZC[k]) || !std::isfinite(dZ[k])) return fail(H2G_NONFINITE, "non-finite ZC/dZ");
  for (int f = 0; f < 6; ++f)
    if (!std::isfinite(HC[f])) return fail(H2G_NONFINITE, "non-finite HC");
  s->ZC.assign(ZC, ZC + MZ);
  s->dZ.assign(dZ, dZ + MZ);
  s->dx = dx;
  s->dy = dy;
  s->dt = is_steady ? (dt > 0 ? dt : 1.0) : dt;
  memcpy(s->HC, HC, sizeof s->HC);
  const int was_steady = s->steady;
  s->steady = is_steady ? 1 : 0;
  s->grid_set = true;
  if (s->fields_set && !s->steady && (was_steady || !s->rc_valid))
    return fail(H2G_BAD_ARG, "switching to a transient grid needs h2g_set_fields with rho and cp");
  return build ? build_tables(s) : H2G_OK;
}

static int set_fields(Solver* s, const double* lam, const double* mask, const double* rho, const double* cp) {
  if (!lam || !mask) return fail(H2G_BAD_ARG, "null lambda/mask");
  if ((rho == nullptr) != (cp == nullptr)) return fail(H2G_BAD_ARG, "rho and cp must both be given or both be NULL");
  if (s->grid_set && !s->steady && !rho) return fail(H2G_BAD_ARG, "transient grid needs rho and cp");
  const Geo& g = s->g;
  const size_t nf = sizeof(double) * (size_t)s->nfort();
  CK(cudaMemcpyAsync(s->stage[0], lam, nf, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->stage[1], mask, nf, cudaMemcpyHostToDevice, s->stream));
  if (rho) {
    CK(cudaMemcpyAsync(s->stage[2], rho, nf, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(s->stage[3], cp, nf, cudaMemcpyHostToDevice, s->stream));
  }
  CK(cudaMemsetAsync(s->slots, 0xff, sizeof(unsigned long long) * kHashSlots, s->stream));
  CK(cudaMemsetAsync(s->flags, 0, sizeof(int), s->stream));
  k_collect_keys<<<s->num_sms * 4, 256, 0, s->stream>>>(g, s->stage[0], s->stage[1], rho ? s->stage[2] : nullptr,
                                                         rho ? s->stage[3] : nullptr, s->slots, s->flags);
  CKL();
  unsigned long long slots[kHashSlots];
  int flags = 0;
  CK(cudaMemcpyAsync(slots, s->slots, sizeof slots, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(&flags, s->flags, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (flags & kFlagNonFinite) return fail(H2G_NONFINITE, "non-finite value in lambda, mask, rho or cp");
  if (flags & kFlagMaskValue) return fail(H2G_UNSUPPORTED, "mask values must be 0 or 1");
  std::vector<unsigned long long> vals;
  for (auto v : slots)
    if (v != ~0ull) vals.push_back(v);
  if ((flags & kFlagTooMany) || (int)vals.size() > kMaxKeys)
    return fail(H2G_UNSUPPORTED, "more than %d distinct conductivity values", kMaxKeys);
  std::sort(vals.begin(), vals.end());
  int index[kHashSlots];
  for (int h = 0; h < kHashSlots; ++h) {
    index[h] = 0;
    if (slots[h] != ~0ull) index[h] = (int)(std::lower_bound(vals.begin(), vals.end(), slots[h]) - vals.begin());
  }
  s->P = (int)vals.size();
  s->lam_values.resize(vals.size());
  for (size_t i = 0; i < vals.size(); ++i) memcpy(&s->lam_values[i], &vals[i], sizeof(double));
  CK(cudaMemcpyAsync(s->slot_index, index, sizeof index, cudaMemcpyHostToDevice, s->stream));
  // rho*cp per cell for transient grids
  if (rho) {
    if (!s->rc64) {
      CK(cudaMalloc(&s->rc64, sizeof(double) * (size_t)g.n));
      invalidate_graphs(s);
    }
    if (s->precision != H2G_FP64 && !s->rc32) {
      CK(cudaMalloc(&s->rc32, sizeof(float) * (size_t)g.n));
      invalidate_graphs(s);
    }
    CK(cudaMemsetAsync(s->rc64, 0, sizeof(double) * (size_t)g.n, s->stream));
    if (s->rc32) CK(cudaMemsetAsync(s->rc32, 0, sizeof(float) * (size_t)g.n, s->stream));
  }
  dim3 grid((g.MX + 127) / 128, g.MY, g.MZ);
  k_make_keys<double><<<grid, 128, 0, s->stream>>>(g, s->stage[0], s->stage[1], rho ? s->stage[2] : nullptr,
                                                   rho ? s->stage[3] : nullptr, s->slots, s->slot_index, s->key,
                                                   rho ? s->rc64 : nullptr);
  CKL();
  if (rho && s->precision != H2G_FP64) {
    k_make_keys<float><<<grid, 128, 0, s->stream>>>(g, s->stage[0], s->stage[1], s->stage[2], s->stage[3], s->slots,
                                                    s->slot_index, s->key, s->rc32);
    CKL();
  }
  // is the key array the last one?  (transient grids rebuild always: rho*cp enters dd)
  bool same = false;
  if (s->key_prev && !rho && s->nkey) {
    int diff = 1;
    CK(cudaMemsetAsync(s->kdiff, 0, sizeof(int), s->stream));
    k_bytes_differ<<<s->num_sms * 4, 256, 0, s->stream>>>(reinterpret_cast<const uint4*>(s->key),
                                                          reinterpret_cast<const uint4*>(s->key_prev),
                                                          (long long)g.n / 16, s->kdiff);
    CKL();
    CK(cudaMemcpyAsync(&diff, s->kdiff, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    same = diff == 0;
  }
  if (!s->key_prev) {
    CK(cudaMalloc(&s->key_prev, (size_t)g.n));
    CK(cudaMalloc(&s->kdiff, sizeof(int)));
  }
  if (!same) {
    CK(cudaMemcpyAsync(s->key_prev, s->key, (size_t)g.n, cudaMemcpyDeviceToDevice, s->stream));
    s->keys_changed = true;
    if (!s->nkey) {
      CK(cudaMalloc(&s->nkey, sizeof(unsigned long long) * (size_t)g.n));
      CK(cudaMemsetAsync(s->nkey, 0, sizeof(unsigned long long) * (size_t)g.n, s->stream));
      invalidate_graphs(s);
    }
    const dim3 gi((g.NX + 127) / 128, g.NY, g.NZ);
    k_make_nkeys<<<gi, 128, 0, s->stream>>>(g, s->key, s->nkey);
    CKL();
  }
  s->rc_valid = rho != nullptr;
  s->fields_set = true;
  CK(cudaStreamSynchronize(s->stream));
  return build_tables(s);
}

}  // namespace h2g

// ==========================================================================================
// C ABI
// ==========================================================================================
using h2g::Solver;
using h2g::fail;

static Solver* S(h2g_solver* h) { return static_cast<Solver*>(h); }

// ---- single-kernel helpers ---------------------------------------------------------------
// The single-kernel entry points use their own two buffers, cleared before every call, so the
// guard and padding entries they rely on are zero whatever precision used them last, and the
// Krylov vectors of the solvers are never touched.
static int hook_buffers(Solver* s, void** a, void** b) {
  const size_t bytes = sizeof(double) * (size_t)s->g.n;
  for (auto& p : s->hook)
    if (!p) CK(cudaMalloc(&p, bytes));
  for (auto& p : s->hook) CK(cudaMemsetAsync(p, 0, bytes, s->stream));
  s->hook_filled = false;
  *a = s->hook[0];
  *b = s->hook[1];
  return H2G_OK;
}

template <typename T>
static int calcax_t(Solver* s, const double* x, double* ax, const h2g::OpParams<T>& op) {
  using namespace h2g;
  void *ha, *hb;
  int rc;
  if ((rc = hook_buffers(s, &ha, &hb))) return rc;
  T* xd = static_cast<T*>(ha);
  T* yd = static_cast<T*>(hb);
  if ((rc = upload<T>(s, x, xd))) return rc;
  launch_ax<T, 0, T>(s, s->stream, op, yd, (const T*)xd, nullptr, nullptr, nullptr, 0);
  CKL();
  return download<T>(s, yd, ax);
}

template <typename T>
static int rbsor_t(Solver* s, double* x, const double* b, int color, double omega, const h2g::OpParams<T>& op) {
  using namespace h2g;
  void *ha, *hb;
  int rc;
  if ((rc = hook_buffers(s, &ha, &hb))) return rc;
  T* xd = static_cast<T*>(ha);
  T* bd = static_cast<T*>(hb);
  if ((rc = upload<T>(s, x, xd, 0))) return rc;
  if ((rc = upload<T>(s, b, bd, 1))) return rc;
  launch_rb<T>(s, s->stream, op, xd, (const T*)bd, color, (T)omega, nullptr);
  CKL();
  return download<T>(s, xd, x);
}

template <typename T>
static int precond_t(Solver* s, const double* bb, double* xx, int smoother, const h2g::OpParams<T>& op) {
  using namespace h2g;
  void *ha, *hb;
  int rc;
  if ((rc = autotune(s))) return rc;  // before the hook buffers are filled: the tuner uses them
  if ((rc = hook_buffers(s, &ha, &hb))) return rc;
  T* xd = static_cast<T*>(ha);
  T* bd = static_cast<T*>(hb);
  if ((rc = upload<T>(s, bb, bd, 1))) return rc;
  // the fused sweeps ping-pong through the third (zeroed) hook buffer, not the solvers' x2
  if ((rc = launch_precond<T, T, 0>(s, s->stream, op, xd, static_cast<T*>(s->hook[2]), bd, bd, nullptr, nullptr,
                                    nullptr, nullptr, smoother)))
    return rc;
  CKL();
  if ((rc = download<T>(s, xd, xx))) return rc;
  return sweep_status(s);
}

template <typename T>
static int bench_t(Solver* s, int kind, int reps, int* launches, const h2g::OpParams<T>& op) {
  using namespace h2g;
  if (int rc = autotune(s)) return rc;
  // the hook buffers, filled with non-zero values: a zero numerator sends the correctly rounded
  // division of the smoother down a slower special-case path, which solves do not see
  const size_t bytes = sizeof(double) * (size_t)s->g.n;
  for (auto& p : s->hook)
    if (!p) CK(cudaMalloc(&p, bytes));
  T* xa = static_cast<T*>(s->hook[0]);
  T* xb = static_cast<T*>(s->hook[1]);
  if (!s->hook_filled) {  // once, outside the caller's timed repetitions
    k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)s->g.n, xa, T(300));
    k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)s->g.n, xb, T(-1.0e-3));
    k_fill_const<T><<<elementwise_blocks(s), 256, 0, s->stream>>>((long long)s->g.n, static_cast<T*>(s->hook[2]),
                                                                  T(300));
    CKL();
    CK(cudaStreamSynchronize(s->stream));
    s->hook_filled = true;
  }
  const dim3 blk(kBX, kBY);
  int n = 0;
  T* xc = static_cast<T*>(s->hook[2]);
  for (int r = 0; r < reps; ++r) {
    if (kind == 0 && s->rb_fused) {
      // one fused sweep; consecutive calls alternate between the two scratch vectors
      const bool fwd = (s->bench_parity++ & 1) == 0;
      if (int rc = launch_sweep<T>(s, s->stream, op, fwd ? xa : xc, fwd ? xc : xa, (const T*)xb, nullptr)) return rc;
      n += 1;
    } else if (kind == 0) {
      launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 0, T(1), nullptr);
      launch_rb<T>(s, s->stream, op, xa, (const T*)xb, 1, T(1), nullptr);
      n += 2;
    } else {
      launch_ax<T, 0, T>(s, s->stream, op, xb, (const T*)xa, nullptr, nullptr, nullptr, 0);
      n += 1;
    }
  }
  CKL();
  if (launches) *launches = n;
  return H2G_OK;
}

extern "C" {

const char* h2g_version(void) { return "h2g 0.1 (sm_100a)"; }

const char* h2g_status_string(int status) {
  switch (status) {
    case H2G_OK: return "ok";
    case H2G_NOT_CONVERGED: return "not converged";
    case H2G_BREAKDOWN: return "breakdown";
    case H2G_NONFINITE: return "non-finite value";
    case H2G_BAD_ARG: return "bad argument";
    case H2G_CUDA_ERROR: return "CUDA error";
    case H2G_TIMEOUT: return "timeout";
    case H2G_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

const char* h2g_last_error(void) { return h2g::g_err.c_str(); }

int h2g_create(int MX, int MY, int MZ, int precision, h2g_solver** out) {
  if (!out) return fail(H2G_BAD_ARG, "null output pointer");
  *out = nullptr;
  Solver* s = nullptr;
  int rc = h2g::create(MX, MY, MZ, precision, &s);
  if (rc) return rc;
  *out = static_cast<h2g_solver*>(s);
  return H2G_OK;
}

int h2g_destroy(h2g_solver* h) {
  if (!h) return H2G_OK;
  h2g::destroy(S(h));
  return H2G_OK;
}

int h2g_set_stream(h2g_solver* h, void* stream) {
  if (int rc = h2g::check_handle(h)) return rc;
  S(h)->stream = (cudaStream_t)stream;
  return H2G_OK;
}

int h2g_set_grid(h2g_solver* h, const double* ZC, const double* dZ, double dx, double dy, double dt, const double* HC,
                 int is_steady) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::set_grid(S(h), ZC, dZ, dx, dy, dt, HC, is_steady);
}

int h2g_set_fields(h2g_solver* h, const double* lambda, const double* mask, const double* rho, const double* cp) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::set_fields(S(h), lambda, mask, rho, cp);
}

int h2g_set_rhs(h2g_solver* h, const double* b) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::upload<double>(S(h), b, S(h)->b);
}

int h2g_get_rhs(h2g_solver* h, double* b) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::download<double>(S(h), S(h)->b, b);
}

int h2g_set_theta(h2g_solver* h, const double* theta) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::upload<double>(S(h), theta, S(h)->th);
}

int h2g_get_theta(h2g_solver* h, double* theta) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::download<double>(S(h), S(h)->th, theta);
}

int h2g_theta_snapshot(h2g_solver* h, int op) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  const size_t nb = sizeof(double) * (size_t)s->g.n;
  if (op == 0) {
    if (cudaMemcpyAsync(s->th_snap, s->th, nb, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess)
      return fail(H2G_CUDA_ERROR, "snapshot copy failed");
  } else if (op == 1) {
    if (cudaMemcpyAsync(s->th, s->th_snap, nb, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess)
      return fail(H2G_CUDA_ERROR, "snapshot copy failed");
  } else {
    return fail(H2G_BAD_ARG, "snapshot op must be 0 (save) or 1 (restore)");
  }
  return H2G_OK;
}

int h2g_set_mixed_params(h2g_solver* h, double inner_tol, int max_outer) {
  if (int rc = h2g::check_handle(h)) return rc;
  if (!(inner_tol > 0 && inner_tol < 1) || max_outer < 1) return fail(H2G_BAD_ARG, "bad refinement parameters");
  S(h)->inner_tol = inner_tol;
  S(h)->max_outer = max_outer;
  return H2G_OK;
}

int h2g_pbicgstab(h2g_solver* h, double tol, int maxItr, int smoother, int verbose, double* res_hist,
                  h2g_result* out) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::solve(S(h), false, tol, maxItr, smoother, verbose, res_hist, out);
}

int h2g_cg(h2g_solver* h, double tol, int maxItr, int smoother, int verbose, double* res_hist, h2g_result* out) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::solve(S(h), true, tol, maxItr, smoother, verbose, res_hist, out);
}

static std::mutex g_cache_mu;
static h2g_solver* g_cache[3] = {nullptr, nullptr, nullptr};

// method 0: PBiCGSTAB, 1: CG, 2: SOR (omega used only by SOR)
static int oneshot(int method, int MX, int MY, int MZ, double* theta, const double* b, const double* lambda,
                   const double* mask, const double* rho, const double* cp, double dx, double dy, double dt,
                   const double* ZC, const double* dZ, const double* HC, double tol, int maxItr, int smoother,
                   double omega, int verbose, int is_steady, int precision, double* res_hist, h2g_result* out) {
  if (precision < H2G_FP64 || precision > H2G_MIXED_IR) return fail(H2G_BAD_ARG, "unknown precision %d", precision);
  if (!theta || !b) return fail(H2G_BAD_ARG, "null theta/b");
  std::lock_guard<std::mutex> lk(g_cache_mu);
  h2g_solver*& h = g_cache[precision];
  if (h && (S(h)->g.MX != MX || S(h)->g.MY != MY || S(h)->g.MZ != MZ)) {
    h2g_destroy(h);
    h = nullptr;
  }
  int rc;
  if (!h && (rc = h2g_create(MX, MY, MZ, precision, &h))) return rc;
  // the tables are built once, by set_fields, from the new grid and fields
  if ((rc = h2g::set_grid(S(h), ZC, dZ, dx, dy, dt, HC, is_steady, false))) return rc;
  if ((rc = h2g_set_fields(h, lambda, mask, is_steady ? nullptr : rho, is_steady ? nullptr : cp))) return rc;
  if ((rc = h2g_set_rhs(h, b))) return rc;
  if ((rc = h2g_set_theta(h, theta))) return rc;
  int st = method == 2 ? h2g::solve_sor(S(h), omega, tol, maxItr, verbose, res_hist, out)
                       : h2g::solve(S(h), method == 1, tol, maxItr, smoother, verbose, res_hist, out);
  if (st == H2G_BAD_ARG || st == H2G_CUDA_ERROR) return st;
  if ((rc = h2g_get_theta(h, theta))) return rc;
  return st;
}

int h2g_PBiCGSTAB(int MX, int MY, int MZ, double* theta, const double* b, const double* lambda, const double* mask,
                  const double* rho, const double* cp, double dx, double dy, double dt, const double* ZC,
                  const double* dZ, const double* HC, double tol, int maxItr, int smoother, int verbose,
                  int is_steady, int precision, double* res_hist, h2g_result* out) {
  return oneshot(0, MX, MY, MZ, theta, b, lambda, mask, rho, cp, dx, dy, dt, ZC, dZ, HC, tol, maxItr, smoother, 1.0,
                 verbose, is_steady, precision, res_hist, out);
}

int h2g_CG(int MX, int MY, int MZ, double* theta, const double* b, const double* lambda, const double* mask,
           const double* rho, const double* cp, double dx, double dy, double dt, const double* ZC, const double* dZ,
           const double* HC, double tol, int maxItr, int smoother, int verbose, int is_steady, int precision,
           double* res_hist, h2g_result* out) {
  return oneshot(1, MX, MY, MZ, theta, b, lambda, mask, rho, cp, dx, dy, dt, ZC, dZ, HC, tol, maxItr, smoother, 1.0,
                 verbose, is_steady, precision, res_hist, out);
}

int h2g_sor(h2g_solver* h, double omega, double tol, int maxItr, int verbose, double* res_hist, h2g_result* out) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::solve_sor(S(h), omega, tol, maxItr, verbose, res_hist, out);
}

int h2g_SolveSOR(int MX, int MY, int MZ, double* theta, const double* b, const double* lambda, const double* mask,
                 const double* rho, const double* cp, double dx, double dy, double dt, double omega,
                 const double* ZC, const double* dZ, const double* HC, double tol, int maxItr, int verbose,
                 int is_steady, double* res_hist, h2g_result* out) {
  return oneshot(2, MX, MY, MZ, theta, b, lambda, mask, rho, cp, dx, dy, dt, ZC, dZ, HC, tol, maxItr, 0, omega,
                 verbose, is_steady, H2G_FP64, res_hist, out);
}

int h2g_set_hsrc(h2g_solver* h, const double* hsrc) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (int rc = h2g::ensure_hsrc(s)) return rc;
  return h2g::upload<double>(s, hsrc, s->hsrc);
}

int h2g_calrhs(h2g_solver* h, const h2g_bc* bc, int zero_b) {
  if (int rc = h2g::check_handle(h)) return rc;
  h2g::FaceBC f;
  if (int rc = h2g::face_bc(bc, f)) return rc;
  Solver* s = S(h);
  if (int rc = h2g::calrhs(s, f, zero_b ? 1 : 0)) return rc;
  CK(cudaStreamSynchronize(s->stream));
  return H2G_OK;
}

int h2g_transient(h2g_solver* h, const h2g_bc* bc, int nt, int method, double tol, int maxItr, int smoother,
                  int verbose, double* step_stats, h2g_result* out) {
  if (int rc = h2g::check_handle(h)) return rc;
  h2g::FaceBC f;
  if (int rc = h2g::face_bc(bc, f)) return rc;
  return h2g::transient(S(h), f, nt, method, tol, maxItr, smoother, verbose, step_stats, out);
}

int h2g_batch_solve(int n, h2g_solver* const* hs, int method, double tol, int maxItr, int smoother, int threads,
                    h2g_result* outs) {
  if (n < 1 || !hs || !outs) return fail(H2G_BAD_ARG, "need n >= 1 handles and n results");
  if (method != 0 && method != 1 && method != 2) return fail(H2G_BAD_ARG, "method must be 0, 1 or 2");
  for (int q = 0; q < n; ++q) {
    if (!hs[q]) return fail(H2G_BAD_ARG, "handle %d is null", q);
    for (int r = 0; r < q; ++r)
      if (hs[r] == hs[q]) return fail(H2G_BAD_ARG, "handle %d appears twice", q);
  }
  // one non-blocking stream per handle for the duration of the batch
  std::vector<cudaStream_t> own(n, nullptr), saved(n, nullptr);
  for (int q = 0; q < n; ++q) {
    Solver* s = S(hs[q]);
    saved[q] = s->stream;
    if (cudaSetDevice(s->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&own[q], cudaStreamNonBlocking) != cudaSuccess) {
      for (int r = 0; r < q; ++r) cudaStreamDestroy(own[r]);
      return fail(H2G_CUDA_ERROR, "stream creation failed");
    }
    // the handle's pending work (uploads) comes first
    if (saved[q]) cudaStreamSynchronize(saved[q]);
    s->stream = own[q];
  }
  cudaDeviceSynchronize();
  // default 2: two solves in flight overlap each other's kernel tails; more of them evict each
  // other's vectors from L2 (measured on the 64-member workload: 1 -> 3.55 s, 2 -> 3.05 s,
  // 4 -> 3.46 s, 16 -> 3.63 s)
  const int nt = std::max(1, std::min(threads > 0 ? threads : 2, n));
  // a cooperative launch needs the whole device: handles that run beside others use the colour
  // passes
  for (int q = 0; q < n; ++q) S(hs[q])->coop_barred = nt > 1;
  std::atomic<int> next(0);
  std::vector<std::string> errs(n);
  auto work = [&]() {
    for (int q = next.fetch_add(1); q < n; q = next.fetch_add(1)) {
      Solver* s = S(hs[q]);
      cudaSetDevice(s->device);
      h2g_result r{};
      int st;
      if (method == 2) st = h2g::solve_sor(s, 1.0, tol, maxItr, 0, nullptr, &r);
      else st = h2g::solve(s, method == 1, tol, maxItr, smoother, 0, nullptr, &r);
      r.status = st;
      outs[q] = r;
      if (st == H2G_BAD_ARG || st == H2G_CUDA_ERROR) errs[q] = h2g_last_error();
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  for (int q = 0; q < n; ++q) {
    Solver* s = S(hs[q]);
    cudaSetDevice(s->device);
    cudaStreamSynchronize(own[q]);
    s->stream = saved[q];
    s->coop_barred = false;
    cudaStreamDestroy(own[q]);
  }
  int worst = H2G_OK;
  for (int q = 0; q < n; ++q) {
    const int st = outs[q].status;
    if (st == H2G_BAD_ARG || st == H2G_CUDA_ERROR) {
      fail(st, "batch member %d: %s", q, errs[q].c_str());
      return st;
    }
    if (st != H2G_OK && worst == H2G_OK) worst = st;
  }
  return worst;
}

int h2g_adjoint(h2g_solver* h, const double* weights, double p, double tol, int maxItr, int smoother, double* J,
                double* dJ_dhsrc, double* dJ_dlnlam, h2g_result* out_fwd, h2g_result* out_adj) {
  if (int rc = h2g::check_handle(h)) return rc;
  return h2g::adjoint(S(h), weights, p, tol, maxItr, smoother, J, dJ_dhsrc, dJ_dlnlam, out_fwd, out_adj);
}

int h2g_adjoint_transient(h2g_solver* h, const h2g_bc* bc, int nt, const double* weights, double p, double tol,
                          int maxItr, int smoother, int checkpoint_every, double* J, double* dJ_dhsrc,
                          double* dJ_dlnlam, h2g_result* out) {
  if (int rc = h2g::check_handle(h)) return rc;
  h2g::FaceBC f;
  if (int rc = h2g::face_bc(bc, f)) return rc;
  return h2g::adjoint_transient(S(h), f, nt, weights, p, tol, maxItr, smoother, checkpoint_every, J, dJ_dhsrc,
                                dJ_dlnlam, out);
}

int h2g_autotune(h2g_solver* h, int* rows, int* planes, int* rb_dd, int* ax_dd) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  CK(cudaSetDevice(s->device));
  if (int rc = h2g::autotune(s)) return rc;
  if (rows) *rows = s->rb_rows;
  if (planes) *planes = s->rb_planes;
  if (rb_dd) *rb_dd = s->rb_cls ? 2 : s->rb_dd ? 1 : 0;
  if (ax_dd) *ax_dd = s->ax_cls ? 2 : s->ax_dd ? 1 : 0;
  return H2G_OK;
}

int h2g_set_tuning(h2g_solver* h, int rows, int planes) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (rows == 0) {
    s->rb_tuned = false;
    return H2G_OK;
  }
  if (!h2g::valid_rows(rows)) return fail(H2G_BAD_ARG, "rows per block must be 2, 4, 8 or 16 (0: tune)");
  if (planes != 1 && planes != 2) return fail(H2G_BAD_ARG, "planes per thread must be 1 or 2");
  if (rows != s->rb_rows || planes != s->rb_planes) h2g::invalidate_graphs(s);
  s->rb_rows = rows;
  s->rb_planes = planes;
  s->rb_tuned = true;
  return H2G_OK;
}

// ---- K right-hand sides on one operator ------------------------------------------------------
int h2g_create_multi(int MX, int MY, int MZ, int nrhs, h2g_solver** out) {
  using namespace h2g;
  if (!out) return fail(H2G_BAD_ARG, "null output pointer");
  *out = nullptr;
  if (nrhs < 1 || nrhs > kMrMax) return fail(H2G_BAD_ARG, "nrhs must be in 1..%d", kMrMax);
  Solver* s = nullptr;
  if (int rc = create(MX, MY, MZ, H2G_FP64, &s)) return rc;
  s->nrhs = nrhs;
  const Geo& g = s->g;
  const size_t nb = sizeof(double) * (size_t)g.n * nrhs;
  const dim3 ag = ax_grid(g);
  const size_t parts = (size_t)nrhs * 2 * std::max((size_t)ag.x * ag.y * ag.z, (size_t)elementwise_blocks(s));
  auto al = [&](void** ptr, size_t bytes) {
    return cudaMalloc(ptr, bytes) == cudaSuccess && cudaMemset(*ptr, 0, bytes) == cudaSuccess;
  };
  bool ok = al((void**)&s->mr_th, nb) && al((void**)&s->mr_b, nb) &&
            al((void**)&s->mr_st, sizeof(SolverState) * nrhs) && al((void**)&s->mr_ctl, sizeof(MultiCtl)) &&
            al((void**)&s->mr_partials, sizeof(double) * parts) && al((void**)&s->mr_flag, sizeof(int));
  for (auto& p : s->mr_kv) ok = ok && al((void**)&p, nb);
  if (!ok) {
    destroy(s);
    return fail(H2G_CUDA_ERROR, "cudaMalloc of the %d right-hand sides failed", nrhs);
  }
  *out = static_cast<h2g_solver*>(s);
  return H2G_OK;
}

static int check_multi(h2g_solver* h) {
  if (int rc = h2g::check_handle(h)) return rc;
  if (S(h)->nrhs < 1) return fail(H2G_BAD_ARG, "not a multi right-hand-side handle (h2g_create_multi)");
  return H2G_OK;
}

int h2g_set_rhs_multi(h2g_solver* h, const double* b) {
  if (int rc = check_multi(h)) return rc;
  Solver* s = S(h);
  if (!b) return fail(H2G_BAD_ARG, "null host array");
  for (int q = 0; q < s->nrhs; ++q)
    if (int rc = h2g::upload<double>(s, b + (size_t)q * s->nfort(), s->mr_b + (size_t)q * s->g.n)) return rc;
  return H2G_OK;
}

int h2g_set_theta_multi(h2g_solver* h, const double* theta) {
  if (int rc = check_multi(h)) return rc;
  Solver* s = S(h);
  if (!theta) return fail(H2G_BAD_ARG, "null host array");
  for (int q = 0; q < s->nrhs; ++q)
    if (int rc = h2g::upload<double>(s, theta + (size_t)q * s->nfort(), s->mr_th + (size_t)q * s->g.n)) return rc;
  return H2G_OK;
}

int h2g_get_theta_multi(h2g_solver* h, double* theta) {
  if (int rc = check_multi(h)) return rc;
  Solver* s = S(h);
  if (!theta) return fail(H2G_BAD_ARG, "null host array");
  for (int q = 0; q < s->nrhs; ++q)
    if (int rc = h2g::download<double>(s, s->mr_th + (size_t)q * s->g.n, theta + (size_t)q * s->nfort())) return rc;
  return H2G_OK;
}

int h2g_pbicgstab_multi(h2g_solver* h, double tol, int maxItr, int smoother, h2g_result* outs) {
  if (int rc = check_multi(h)) return rc;
  return h2g::solve_multi(S(h), tol, maxItr, smoother, outs);
}

int h2g_set_sweep(h2g_solver* h, int fused, int chunks, int dd_array) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (fused < -1 || fused > 1) return fail(H2G_BAD_ARG, "fused must be -1 (tune), 0 or 1");
  if (fused == 1 && (chunks < 1 || chunks > 255)) return fail(H2G_BAD_ARG, "chunks must be in 1..255");
  if (fused == 1 && dd_array != 0 && dd_array != 1) return fail(H2G_BAD_ARG, "dd_array must be 0 or 1");
  s->sweep_forced = fused;
  if (fused == 1) {
    s->sw_chunks = std::min(chunks, s->g.NZ);
    s->sw_dda = dd_array != 0;
  }
  s->rb_tuned = false;  // the next solve applies the choice (and tunes what is left free)
  h2g::invalidate_graphs(s);
  return H2G_OK;
}

int h2g_set_coop(h2g_solver* h, int mode) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (mode < -1 || mode > 1) return fail(H2G_BAD_ARG, "mode must be -1 (default), 0 or 1");
  if (mode == 1 && s->precision != H2G_FP64)
    return fail(H2G_UNSUPPORTED, "the cooperative preconditioner runs on FP64 handles");
  s->coop_forced = mode;
  if (mode == 1 && s->sweep_forced == 1) s->sweep_forced = 0;
  s->rb_tuned = false;
  h2g::invalidate_graphs(s);
  return H2G_OK;
}

int h2g_get_coop(h2g_solver* h, int* on) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (!on) return fail(H2G_BAD_ARG, "null output");
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  CK(cudaSetDevice(s->device));
  if (int rc = h2g::autotune(s)) return rc;
  *on = s->rb_coop;
  return H2G_OK;
}

int h2g_get_sweep(h2g_solver* h, int* fused, int* chunks, int* dd_array) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  CK(cudaSetDevice(s->device));
  if (int rc = h2g::autotune(s)) return rc;
  if (fused) *fused = s->rb_fused ? 1 : 0;
  if (chunks) *chunks = s->sw_chunks;
  if (dd_array) *dd_array = s->sw_dda ? 1 : 0;
  return H2G_OK;
}

int h2g_set_wait_limit(h2g_solver* h, long long cycles) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (cycles < 0) return fail(H2G_BAD_ARG, "cycles must be >= 0");
  s->wait_limit = cycles == 0 ? 0 : cycles;
  h2g::invalidate_graphs(s);  // the limit is a kernel argument captured in the graphs
  return H2G_OK;
}

int h2g_release_cached(void) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  for (auto& h : g_cache) {
    h2g_destroy(h);
    h = nullptr;
  }
  return H2G_OK;
}

// ---- single kernels ------------------------------------------------------------------------

int h2g_calcax(h2g_solver* h, const double* x, double* ax) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (s->precision == H2G_MIXED_IR) return calcax_t<float>(s, x, ax, h2g::op_params<float>(s, s->t32));
  return calcax_t<double>(s, x, ax, h2g::op_params<double>(s, s->t64));
}

int h2g_calcrk(h2g_solver* h, double* r, double* res) {
  using namespace h2g;
  if (int rc = check_handle(h)) return rc;
  Solver* s = S(h);
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (!res) return fail(H2G_BAD_ARG, "null res");
  OpParams<double> op = op_params<double>(s, s->t64);
  double* rd = s->precision == H2G_MIXED_IR ? s->r64 : kvec<double>(s, KR);
  int rc;
  if ((rc = prime_state(s, s->st, 0.0, 1, nullptr, 0))) return rc;
  launch(s, k_rk<double>, ax_grid(s->g), dim3(kBX, kBY), s->stream, op, rd, nullptr, s->th, s->b, s->st, s->partials,
                                                                   kStageResid);
  CKL();
  CK(cudaMemcpyAsync(s->st_host, s->st, sizeof(SolverState), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *res = s->st_host->scale;
  if (r) return download<double>(s, rd, r);
  return H2G_OK;
}


int h2g_rbsor_pass(h2g_solver* h, double* x, const double* b, int color, double omega) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (color != 0 && color != 1) return fail(H2G_BAD_ARG, "color must be 0 or 1");
  if (!(omega > 0 && omega < 2)) return fail(H2G_BAD_ARG, "omega must be in (0,2)");
  if (s->precision != H2G_FP64) return rbsor_t<float>(s, x, b, color, omega, h2g::op_params<float>(s, s->t32));
  return rbsor_t<double>(s, x, b, color, omega, h2g::op_params<double>(s, s->t64));
}


int h2g_preconditioner(h2g_solver* h, const double* bb, double* xx, int smoother) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (smoother != H2G_SMOOTHER_NONE && smoother != H2G_SMOOTHER_GS)
    return fail(H2G_BAD_ARG, "Unsupported smoother: %d. Use none (0) or gs (1)", smoother);
  if (s->precision != H2G_FP64) return precond_t<float>(s, bb, xx, smoother, h2g::op_params<float>(s, s->t32));
  return precond_t<double>(s, bb, xx, smoother, h2g::op_params<double>(s, s->t64));
}


int h2g_bench_kernel(h2g_solver* h, int kind, int reps, int* launches) {
  if (int rc = h2g::check_handle(h)) return rc;
  Solver* s = S(h);
  if (!s->grid_set || !s->fields_set) return fail(H2G_BAD_ARG, "h2g_set_grid and h2g_set_fields must come first");
  if (kind != 0 && kind != 1) return fail(H2G_BAD_ARG, "kind must be 0 (RB-GS sweep) or 1 (CalcAX)");
  if (reps < 1) return fail(H2G_BAD_ARG, "reps must be positive");
  // the sweep runs in the preconditioner's precision, CalcAX in the Krylov solver's
  const bool fp32 = kind == 0 ? s->precision != H2G_FP64 : s->precision == H2G_MIXED_IR;
  if (fp32) return bench_t<float>(s, kind, reps, launches, h2g::op_params<float>(s, s->t32));
  return bench_t<double>(s, kind, reps, launches, h2g::op_params<double>(s, s->t64));
}

}  // extern "C"

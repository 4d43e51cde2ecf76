// h2g_kernels.cuh -- sm_100a kernels of the Heat3ds solver path.
//
// Operator (src/NonUniform.jl:372-511, 848-915).  Every stencil evaluation needs, per cell,
// six face conductances, six convective terms and the diagonal dd.  The reference recomputes
// them from lambda and mask with eight FP64 divisions per cell.  Here each cell carries one
// byte: a material key (index of its lambda value, bits 0-6) and its mask (bit 7).  The face
// conductance between two keys a, b at plane k,
//     ((lambda_f(a,b,ma,mb) * dy0) * dz_k) * ddx           (x faces, NonUniform.jl:482-483)
// depends only on (k, a, b, fac) with fac = 2 - div(ma+mb, 2) in {1, 2}, so the host tabulates
// it once per solve in exactly the reference's operation order; the kernels look it up.
// FP64 results are therefore bit-identical to the reference's per-cell arithmetic.
#pragma once
#include "h2g_internal.cuh"

namespace h2g {

// Launch shape of the stencil kernels.  H2G_BY also fixes the order of the partial sums of the
// dot products, and with it the iteration count, so it stays at 8 unless rebuilt on purpose.
// H2G_MINB = 4 resident colour-pass blocks per SM caps that kernel at 64 registers (measured
// 1% faster per iteration than the unconstrained 80 on the 240x240x30 grid).
#ifndef H2G_BY
#define H2G_BY 8
#endif
#ifndef H2G_MINB
#define H2G_MINB 4
#endif
// The colour pass reading the stencil-class table needs fewer registers: 5 resident blocks of 256
// threads per SM (48 registers, no spills) measured -1 % per FP64 solve at 240x240x30 and -2.4 %
// at 480x480x60 (-5.5 % per sweep) against 4; 6 blocks (40 registers) spill and were slower.
#ifndef H2G_MINB_CLS
#define H2G_MINB_CLS 5
#endif
// x-neighbours by direct loads (1) or warp shuffles (0): loads measured 6 % faster per solve
// on the 240x240x30 grid (fewer LSU instructions)
#ifndef H2G_XNB_LOAD
#define H2G_XNB_LOAD 1
#endif
// the smoother reads dd from a per-cell array (1) or sums its 13 terms per cell (0)
#ifndef H2G_DD_ARRAY
#define H2G_DD_ARRAY 1
#endif
// the smoother reads the 7 keys a cell needs as one 8-byte word per cell (1) or byte by byte (0)
#ifndef H2G_NKEY
#define H2G_NKEY 1
#endif
// CalcAX asks the compiler for 5 resident blocks of 256 threads per SM (48 registers; the
// variants that read dd spill 4-12 bytes).  Per FP64 solve, with the same bits: equal at
// 240x240x30 and -3 % at 480x480x60 against no request (58-72 registers); -4 % and -11 %
// against an explicit 1-block request (66-88 registers).  A 6-block cap (40 registers) spills
// more and gains less.
#ifndef H2G_AX_MINB
#define H2G_AX_MINB 5
#endif

constexpr int kBX = 32;       // threads along the half-row
constexpr int kBY = H2G_BY;   // rows per block
constexpr int kThreads = kBX * kBY;

// ------------------------------------------------------------------------------------------
// Deterministic reductions: every block writes its partial sums; the last block to finish
// (atomic ticket) adds all partials in a fixed order and runs the stage's scalar logic.
// ------------------------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sm)[NV], int tid, int nthr) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  const int lane = tid & 31, warp = tid >> 5, nw = (nthr + 31) >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) sm[warp][q] = v[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = lane < nw ? sm[lane][q] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int q = 0; q < NV; ++q) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  }
  __syncthreads();
}

// Programmatic dependent launch: wait until the preceding kernel's writes are visible, then let
// the next kernel of the stream start launching its blocks (they wait the same way).  Both are
// no-ops for a kernel launched without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle h, int use_cond, int value) {
  if (use_cond) cudaGraphSetConditional(h, value ? 1u : 0u);
}

// Scalar logic of each stage (runs on one thread).  Mirrors the control flow of PBiCGSTAB!
// (NonUniform.jl:262-349) and CG! (NonUniform.jl:131-225).
__device__ void finish_stage(int stage, SolverState* st, double s1, double s2) {
  switch (stage) {
    case kStageInit:  // NonUniform.jl:263-294: res0, early return, rho of iteration 1
    case kStageInitCg: {
      const double res0 = sqrt(s1);
      st->res0 = res0;
      st->res = 1.0;
      st->rho = s1;
      st->rho_old = 1.0;
      st->alpha = 0.0;
      st->omega = 1.0;
      st->beta = 0.0;
      st->itr = 1;
      st->first = 1;
      st->stop = 0;
      st->converged = 0;
      st->reason = kRunning;
      if (res0 == 0.0) {
        st->stop = 1; st->converged = 1; st->itr = 0; st->res = 0.0; st->reason = kConverged;
      } else if (!isfinite(res0)) {
        st->stop = 1; st->itr = 0; st->reason = kNonFinite;
      } else if (stage == kStageInit && fabs(s1) < kFloatMin) {
        st->stop = 1; st->reason = kBreakdown;
      }
      break;
    }
    case kStageAlpha:  // NonUniform.jl:309
      st->alpha = __ddiv_rn(st->rho, s1);
      break;
    case kStageOmega:  // NonUniform.jl:320-326
      if (fabs(s1) < kFloatMin) { st->stop = 1; st->reason = kBreakdown; }
      else st->omega = __ddiv_rn(s2, s1);
      break;
    case kStageUpdate: {  // NonUniform.jl:331-346 and the top of the next iteration 289-299
      const double res = __ddiv_rn(sqrt(s1), st->res0);
      if (st->hist && st->itr >= 1 && st->itr <= st->hist_len) st->hist[st->itr - 1] = res;
      st->res = res;
      st->first = 0;
      if (res < st->tol) { st->stop = 1; st->converged = 1; st->reason = kConverged; break; }
      if (!isfinite(res) || (st->div_limit > 0.0 && res > st->div_limit)) {
        st->stop = 1; st->reason = kNonFinite; break;
      }
      if (st->itr >= st->maxItr) { st->stop = 1; st->reason = kMaxItr; break; }
      st->rho_old = st->rho;
      st->rho = s2;
      st->itr += 1;
      if (fabs(s2) < kFloatMin) { st->stop = 1; st->reason = kBreakdown; break; }
      st->beta = __ddiv_rn(__dmul_rn(__ddiv_rn(st->rho, st->rho_old), st->alpha), st->omega);
      break;
    }
    case kStageResid:
      st->scale = sqrt(s1);
      break;
    case kStageCgInit:  // NonUniform.jl:155
      st->rho_old = s1;
      st->itr = 1;
      break;
    case kStageCgAlpha:  // NonUniform.jl:168-176
      if (fabs(s1) < kFloatMin) { st->stop = 1; st->reason = kBreakdown; }
      else st->alpha = __ddiv_rn(st->rho_old, s1);
      break;
    case kStageCgRes: {  // NonUniform.jl:185-198
      const double res = __ddiv_rn(sqrt(s1), st->res0);
      if (st->hist && st->itr >= 1 && st->itr <= st->hist_len) st->hist[st->itr - 1] = res;
      st->res = res;
      if (res < st->tol) { st->stop = 1; st->converged = 1; st->reason = kConverged; break; }
      if (!isfinite(res) || (st->div_limit > 0.0 && res > st->div_limit)) { st->stop = 1; st->reason = kNonFinite; }
      break;
    }
    case kStageCgBeta:  // NonUniform.jl:206-222, then the loop bound
      if (fabs(s1) < kFloatMin) { st->stop = 1; st->reason = kBreakdown; break; }
      st->beta = __ddiv_rn(s1, st->rho_old);
      st->rho_old = s1;
      if (st->itr >= st->maxItr) { st->stop = 1; st->reason = kMaxItr; break; }
      st->itr += 1;
      break;
    case kStageDot:
      st->dot1 = s1;
      st->dot2 = s2;
      break;
    case kStageSorInit: {  // solveSOR! NonUniform.jl:1031-1035: res0 (1 if zero)
      double res0 = sqrt(s1);
      if (res0 == 0.0) res0 = 1.0;
      st->res0 = res0;
      st->res = 1.0;
      st->itr = 0;
      st->stop = 0;
      st->converged = 0;
      st->reason = kRunning;
      if (!isfinite(res0)) { st->stop = 1; st->reason = kNonFinite; }
      break;
    }
    case kStageSorHalf:  // colour 0 of rbsor! (NonUniform.jl:952-955)
      st->dot1 = s1;
      break;
    case kStageSorIter: {  // colour 1, then the test of solveSOR! (NonUniform.jl:1038-1048)
      const double res = __ddiv_rn(sqrt(__dadd_rn(st->dot1, s1)), st->res0);
      st->itr += 1;
      if (st->hist && st->itr <= st->hist_len) st->hist[st->itr - 1] = res;
      st->res = res;
      if (res < st->tol) { st->stop = 1; st->converged = 1; st->reason = kConverged; break; }
      if (!isfinite(res)) { st->stop = 1; st->reason = kNonFinite; break; }
      if (st->itr >= st->maxItr) { st->stop = 1; st->reason = kMaxItr; break; }
      break;
    }
    default:
      break;
  }
}

// COND: the kernel may set the loop condition of a device-side WHILE node.  Kernels compiled
// without it contain no device graph call (the host-loop path launches those; profilers can
// then see them too).
template <int NV, bool COND = false>
__device__ __forceinline__ void reduce_finish(double (&v)[NV], double* __restrict__ partials, SolverState* st,
                                              int stage, cudaGraphConditionalHandle hc, int use_cond) {
  __shared__ double sm[32][NV];
  __shared__ int am_last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  block_sum<NV>(v, sm, tid, nthr);
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[(size_t)q * nb + bid] = v[q];
    __threadfence();
    const unsigned t = atomicAdd(&st->ticket, 1u);
    am_last = (t == nb - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  // fixed-order sum of the partials; eight independent loads in flight per thread
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (unsigned b0 = tid; b0 < nb; b0 += 8u * nthr) {
    double t[NV][8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const unsigned b = b0 + (unsigned)u * nthr;
#pragma unroll
      for (int q = 0; q < NV; ++q) t[q][u] = b < nb ? __ldcg(partials + (size_t)q * nb + b) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
      for (int q = 0; q < NV; ++q) acc[q] += t[q][u];
  }
  block_sum<NV>(acc, sm, tid, nthr);
  if (tid == 0) {
    st->ticket = 0;
    finish_stage(stage, st, acc[0], NV > 1 ? acc[NV > 1 ? 1 : 0] : 0.0);
    // the loop continues only while the solve runs and the pass count is within maxItr + 1
    if constexpr (COND) set_cond(hc, use_cond, !st->stop && st->passes <= st->maxItr + 1);
  }
}

// ------------------------------------------------------------------------------------------
// Stencil coefficients of one cell from the key tables.
// ------------------------------------------------------------------------------------------
template <typename T>
struct Coef {
  T cxm, cxp, cym, cyp, czm, czp, dd;
  T sconv;  // convective terms + a_p0 (FP32 difference form only)
};

// Coefficients of one unmasked cell (key k0) at plane k from its neighbours' keys.  The tables
// are indexed by the neighbour's whole key byte: its mask bit selects lambda_f's factor
// 2 - div(ma+mb, 2) (1 if the neighbour is unmasked, 2 if it is a masked guard).  The order of
// the additions of dd follows NonUniform.jl:501-502 exactly.
// PRE: take dd from the per-cell array op.ddv (computed once per grid by k_make_dd with this same
// function, so the values are identical) instead of summing its 13 terms.
template <typename T, bool PRE = false>
__device__ __forceinline__ bool cell_coef(const OpParams<T>& op, int k, uint8_t k0, uint8_t kxm, uint8_t kxp,
                                          uint8_t kym, uint8_t kyp, uint8_t kzm, uint8_t kzp, int ci, Coef<T>& c) {
  if (!(k0 & 0x80)) return false;
  const int bx = (k * op.P + (k0 & 0x7f)) << 8;
  c.cxm = __ldg(op.tx + (bx | kxm));
  c.cxp = __ldg(op.tx + (bx | kxp));
  c.cym = __ldg(op.ty + (bx | kym));
  c.cyp = __ldg(op.ty + (bx | kyp));
  c.czm = __ldg(op.tz + (bx | kzm));
  c.czp = __ldg(op.tz + ((bx + (op.P << 8)) | kzp));
  if constexpr (PRE && H2G_DD_ARRAY) {
    c.dd = __ldg(op.ddv + ci);
    return true;
  }
  const T* cv = op.conv + 4 * k;
  const T vxm = (kxm & 0x80) ? T(0) : __ldg(cv + 0);
  const T vxp = (kxp & 0x80) ? T(0) : __ldg(cv + 1);
  const T vym = (kym & 0x80) ? T(0) : __ldg(cv + 2);
  const T vyp = (kyp & 0x80) ? T(0) : __ldg(cv + 3);
  const T vzm = (kzm & 0x80) ? T(0) : op.czm;
  const T vzp = (kzp & 0x80) ? T(0) : op.czp;
  T ap = T(0);
  if (!op.steady) ap = mul(mul(mul(mul(op.rc[ci], op.dx0), op.dy0), __ldg(op.dzk + k)), op.ddt);
  T s = add(c.cxp, c.cxm);
  s = add(s, c.cyp);
  s = add(s, c.cym);
  s = add(s, c.czp);
  s = add(s, c.czm);
  s = add(s, vxp);
  s = add(s, vxm);
  s = add(s, vyp);
  s = add(s, vym);
  s = add(s, vzp);
  s = add(s, vzm);
  s = add(s, ap);
  c.dd = add(T(0), s);  // (1 - m0) + (...) * m0 with m0 = 1
  if constexpr (sizeof(T) == 4) c.sconv = ((((vxp + vxm) + (vyp + vym)) + (vzp + vzm)) + ap);
  return true;
}

// Stencil classes.  The coefficients of a cell depend only on its plane k and the 7 key
// bytes of its stencil, so the cells of a grid fall into few classes: one per distinct (k, keys)
// pair.  k_class_coef fills one table row per class with cell_coef itself, for a steady grid, so
// every value is the one cell_coef gives the cell; a cell then reads a 2-byte class index and one
// 64-byte row instead of the 8-byte key word, six table entries and dd.  A transient grid adds
// a_p0 per cell, so there dd is read from the per-cell array (the same value again).
constexpr unsigned kNoClass = 0xffffu;
constexpr int kClassSlots = 1 << 17;   // hash slots of the (plane, keys) pairs
constexpr int kMaxClasses = 65535;     // class indices are 16-bit; 0xffff marks "not updated"

// Row layout (8 values of T): cx-, cx+, cy-, cy+, cz-, cz+, dd, 0.  The FP32 rows serve the FP32
// smoother only (its CalcAX uses the difference form, which needs a per-cell term the row lacks).
template <typename T>
__device__ __forceinline__ bool class_coef(const OpParams<T>& op, unsigned cl, int ci, Coef<T>& c) {
  if (cl == kNoClass) return false;
  if constexpr (sizeof(T) == 8) {
    const double2* t = reinterpret_cast<const double2*>(op.ctab) + 4 * cl;
    const double2 a = __ldg(t), b = __ldg(t + 1), z = __ldg(t + 2);
    c.cxm = a.x;
    c.cxp = a.y;
    c.cym = b.x;
    c.cyp = b.y;
    c.czm = z.x;
    c.czp = z.y;
    c.dd = op.steady ? __ldg(reinterpret_cast<const double*>(t + 3)) : __ldg(op.ddv + ci);
  } else {
    const float4* t = reinterpret_cast<const float4*>(op.ctab) + 2 * cl;
    const float4 a = __ldg(t), z = __ldg(t + 1);
    c.cxm = a.x;
    c.cxp = a.y;
    c.cym = a.z;
    c.cyp = a.w;
    c.czm = z.x;
    c.czp = z.y;
    c.dd = op.steady ? z.z : __ldg(op.ddv + ci);
  }
  return true;
}

// ss of NonUniform.jl:505-507 (products summed left to right).  FP64: separately rounded, as the
// reference.  FP32 (the mixed smoother): fused multiply-adds, written out so that every launch
// shape computes the same bits.
template <typename T>
__device__ __forceinline__ T nb_sum(const Coef<T>& c, T xp, T xm, T yp, T ym, T zp, T zm) {
  if constexpr (sizeof(T) == 4) {
    float s = __fmul_rn(c.cxp, xp);
    s = __fmaf_rn(c.cxm, xm, s);
    s = __fmaf_rn(c.cyp, yp, s);
    s = __fmaf_rn(c.cym, ym, s);
    s = __fmaf_rn(c.czp, zp, s);
    return __fmaf_rn(c.czm, zm, s);
  } else {
    T s = mul(c.cxp, xp);
    s = add(s, mul(c.cxm, xm));
    s = add(s, mul(c.cyp, yp));
    s = add(s, mul(c.cym, ym));
    s = add(s, mul(c.czp, zp));
    s = add(s, mul(c.czm, zm));
    return s;
  }
}

// pp + omega*dp: FP64 two roundings (the reference), FP32 one fused multiply-add
__device__ __forceinline__ double relax(double pp, double omega, double dp) { return add(pp, mul(omega, dp)); }
__device__ __forceinline__ float relax(float pp, float omega, float dp) { return __fmaf_rn(omega, dp, pp); }

// Gauss-Seidel update of one cell: (ss - b)/dd, correctly rounded in both precisions (an
// approximate FP32 division weakens the FP32 preconditioner enough to multiply the iterations).
__device__ __forceinline__ double gs_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float gs_div(float a, float b) { return a / b; }

// A x at one cell.  FP64: (ss - dd*x) exactly as CalcAX! (NonUniform.jl:505-509).  FP32: the same
// operator in difference form, sum c_nb*(x_nb - x) - (conv + a_p0)*x, which cancels first
// differences instead of ss against dd*x (whose rounding error grows like 1/h^2 in FP32).
template <typename T>
__device__ __forceinline__ T apply_a(const Coef<T>& c, T x0, T xp, T xm, T yp, T ym, T zp, T zm) {
  if constexpr (sizeof(T) == 4) {
    T s = c.cxp * (xp - x0);
    s = fmaf(c.cxm, xm - x0, s);
    s = fmaf(c.cyp, yp - x0, s);
    s = fmaf(c.cym, ym - x0, s);
    s = fmaf(c.czp, zp - x0, s);
    s = fmaf(c.czm, zm - x0, s);
    return fmaf(-c.sconv, x0, s);
  } else {
    T s = mul(c.cxp, xp);
    s = add(s, mul(c.cxm, xm));
    s = add(s, mul(c.cyp, yp));
    s = add(s, mul(c.cym, ym));
    s = add(s, mul(c.czp, zp));
    s = add(s, mul(c.czm, zm));
    return sub(s, mul(c.dd, x0));
  }
}

// ------------------------------------------------------------------------------------------
// Stencil kernels.
//
// A block is 32 threads along the half-row (positions p) x kBY rows (j); warps run along p.  For
// a cell of colour c at (p, j, k) every neighbour has colour o = 1-c: the z-neighbours and one
// x-neighbour are the o-colour column at (p, j) (planes k-1, k+1 and k), the other x-neighbour
// is the o-colour value at p-1 or p+1 -- the same column of the adjacent lane, loaded directly
// (an L1 hit; H2G_XNB_LOAD=0 takes it by warp shuffle instead) -- and the y-neighbours are the
// o-colour columns
// (p, j+-1).  Each thread updates two cells that share most of these loads: the RB pass takes
// the colour-c cells of its column at planes k and k+1; CalcAX/CalcRK and the first pass take
// both colours of its column at plane k.  All loads of a thread are issued before its first
// store.  Offsets are 32-bit.
// ------------------------------------------------------------------------------------------
constexpr unsigned kFull = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T ldro(const T* p) { return __ldg(p); }
// Loads of a vector that this launch itself writes (the cooperative preconditioner, whose passes
// read what other blocks wrote before a grid barrier) go through the coherent path: ld.global.ca
// obeys the memory model's acquire/release ordering, the read-only path does not.
template <bool NC, typename T>
__device__ __forceinline__ T ldx(const T* p) {
  if constexpr (NC) return __ldg(p);
  else return __ldca(p);
}

// x-neighbours of a colour-c cell at position p with parity e (x-1 = o[p-1+e], x+1 = o[p+e]),
// given the o-colour value and key of this lane's column at that plane.  All lanes must call it.
template <typename T, bool VAL, typename TI = T, bool KEYS = true, bool NC = true>
__device__ __forceinline__ void x_nbrs(T oc, int okc, int e, int lane, int p, int HN, const TI* x,
                                       const uint8_t* key, int rowo, T& xm, T& xp, int& kxm, int& kxp) {
#if H2G_XNB_LOAD
  // the other x-neighbour is the o-colour value at position p-1 (e = 0) or p+1 (e = 1): a
  // direct load (an L1 hit: the adjacent lane's column) costs fewer instructions than shuffles
  const int q = p - 1 + 2 * e;
  T other = T(0);
  int ko = 0;
  if (q >= 0 && q < HN) {
    if (VAL) other = (T)ldx<NC>(x + rowo + q);
    if (KEYS) ko = key[rowo + q];
  }
  if (e) {
    xm = oc; kxm = okc; xp = other; kxp = ko;
  } else {
    xm = other; kxm = ko; xp = oc; kxp = okc;
  }
  return;
#endif
  T left = T(0), right = T(0);
  if (VAL) {
    left = __shfl_up_sync(kFull, oc, 1);
    right = __shfl_down_sync(kFull, oc, 1);
  }
  int kl = __shfl_up_sync(kFull, okc, 1), kr = __shfl_down_sync(kFull, okc, 1);
  if (lane == 0 && !e && p >= 1) {
    if (VAL) left = (T)ldro(x + rowo + p - 1);
    kl = key[rowo + p - 1];
  }
  if (lane == 31 && e && p + 1 < HN) {
    if (VAL) right = (T)ldro(x + rowo + p + 1);
    kr = key[rowo + p + 1];
  }
  if (e) {
    xm = oc; kxm = okc; xp = right; kxp = kr;
  } else {
    xm = left; kxm = kl; xp = oc; kxp = okc;
  }
}

// ------------------------------------------------------------------------------------------
// rbsor_core! (NonUniform.jl:848-915): one colour pass of RB-SOR on x with rhs bb.
// Grid (ceil(HN/32), ceil(NY/kBY), ceil(NZ/2)); thread = colour-c cells of column (p,j) at
// planes k0, k0+1.
// ------------------------------------------------------------------------------------------
// One colour pass over the NP planes k0 .. k0+NP-1 (NP = 1 or 2) of column (p, j).  RES: also
// returns the sum of the squared SOR residuals r = (dd + omega*(c_xm + c_ym + c_zm))*dp/omega of
// the updated cells (rbsor_core!, NonUniform.jl:907-908); the preconditioner discards them and
// skips the work.  With NP = 2 the two cells share the o-colour column loads.
template <typename T, bool RES, int NP = 2, int DDM = 1, bool NC = true>
__device__ __forceinline__ double rb_pass_column(const OpParams<T>& op, T* x, const T* __restrict__ bb, int color,
                                                 T omega, int lane, int p, int j, int k0) {
  const Geo& g = op.g;
  const int o = color ^ 1;
  const bool pok = p < g.HN;
  const uint8_t* key = op.key;
  const int HP2 = 2 * g.HP, PL = (int)g.plane;
  const int ro0 = g.row(o, j, k0), rc0 = g.row(color, j, k0);
  // o-colour column at (p, j), planes k0-1 .. k0+NP
  T col[NP + 2];
  int kcol[NP + 2];
  constexpr bool CL = DDM == 2;                // coefficients from the class table
  constexpr bool NK = H2G_NKEY != 0 || CL;     // no key bytes loaded one by one
#pragma unroll
  for (int t = 0; t < NP + 2; ++t) {
    col[t] = T(0);
    kcol[t] = 0;
    if (pok && k0 - 1 + t <= g.MZ - 1) {
      const int a = ro0 + (t - 1) * PL + p;
      col[t] = ldx<NC>(x + a);
      if (!NK) kcol[t] = key[a];
    }
  }
  T ym[NP], yp[NP], pp[NP], bv[NP];
  int kym[NP], kyp[NP], kc[NP];
  unsigned long long nk[NP];
  unsigned cl[NP];
  bool ok[NP];
#pragma unroll
  for (int u = 0; u < NP; ++u) {
    const int k = k0 + u, e = (1 + color + j + k) & 1, i = 2 * p + e;
    ok[u] = pok && k <= g.NZ && i >= 1 && i <= g.NX;
    ym[u] = yp[u] = pp[u] = bv[u] = T(0);
    kym[u] = kyp[u] = kc[u] = 0;
    nk[u] = 0ull;
    cl[u] = kNoClass;
    if (ok[u]) {
      const int ao = ro0 + u * PL + p, ac = rc0 + u * PL + p;
      ym[u] = ldx<NC>(x + ao - HP2);
      yp[u] = ldx<NC>(x + ao + HP2);
      if (CL) {
        cl[u] = __ldg(op.cls + ac);
      } else if (NK) {
        nk[u] = __ldg(op.nkey + ac);
      } else {
        kym[u] = key[ao - HP2];
        kyp[u] = key[ao + HP2];
        kc[u] = key[ac];
      }
      pp[u] = x[ac];
      bv[u] = NC ? bb[ac] : ldx<false>(bb + ac);
    }
  }
  T xm[NP], xp[NP];
  int kxm[NP], kxp[NP];
#pragma unroll
  for (int u = 0; u < NP; ++u) {
    const int e = (1 + color + j + k0 + u) & 1;
    x_nbrs<T, true, T, !NK, NC>(col[u + 1], kcol[u + 1], e, lane, p, g.HN, x, key, ro0 + u * PL, xm[u], xp[u],
                                kxm[u], kxp[u]);
  }
  double acc = 0.0;
#pragma unroll
  for (int u = 0; u < NP; ++u) {
    if (!ok[u]) continue;
    const int ac = rc0 + u * PL + p;
    Coef<T> c;
    bool has;
    if constexpr (CL) {
      has = class_coef<T>(op, cl[u], ac, c);
    } else if (NK) {
      const unsigned long long w = nk[u];  // own, x-, x+, y-, y+, z-, z+ keys in bytes 0..6
      has = cell_coef<T, DDM == 1>(op, k0 + u, (uint8_t)w, (uint8_t)(w >> 8), (uint8_t)(w >> 16),
                                   (uint8_t)(w >> 24), (uint8_t)(w >> 32), (uint8_t)(w >> 40), (uint8_t)(w >> 48),
                                   ac, c);
    } else {
      has = cell_coef<T, DDM == 1>(op, k0 + u, (uint8_t)kc[u], (uint8_t)kxm[u], (uint8_t)kxp[u], (uint8_t)kym[u],
                               (uint8_t)kyp[u], (uint8_t)kcol[u], (uint8_t)kcol[u + 2], ac, c);
    }
    if (!has) continue;
    const T ss = nb_sum(c, xp[u], xm[u], yp[u], ym[u], col[u + 2], col[u]);
    const T dp = sub(gs_div(sub(ss, bv[u]), c.dd), pp[u]);  // * m0 (= 1)
    x[ac] = relax(pp[u], omega, dp);
    if constexpr (RES) {
      const T r = dvd(mul(add(c.dd, mul(omega, add(add(c.cxm, c.cym), c.czm))), dp), omega);
      acc = add(acc, mul((double)r, (double)r));
    }
  }
  return acc;
}

// The colour pass has no reduction, so its block height BY (rows per block) and its planes per
// thread NP change no result; the autotuner picks them per grid among kRbRows x {1, 2}.  Every
// shape keeps the register cap of H2G_MINB blocks of 256 threads per SM.
constexpr int kRbRows[4] = {2, 4, 8, 16};

// DDM: how a cell gets dd and its coefficients.  0: coefficients from the key tables, dd summed
// per cell (8 bytes fewer per cell than 1); 1: dd read from the per-cell array (fewer
// instructions); 2: the stencil-class table (2 bytes per cell instead of the 8-byte key
// word and dd).  The tuner picks it with the shape.
template <typename T, int BY = kBY, int NP = 2, int DDM = 1>
__global__ void __launch_bounds__(kBX * BY, ((DDM == 2 ? H2G_MINB_CLS : H2G_MINB) * kBY) / BY)
    k_rb_pass(OpParams<T> op, T* x, const T* __restrict__ bb, int color, T omega,
              const SolverState* __restrict__ st) {
  pdl_enter();
  if (st && st->stop) return;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * BY + threadIdx.y;
  const int k0 = 1 + NP * blockIdx.z;
  if (j > op.g.NY) return;  // uniform per warp
  rb_pass_column<T, false, NP, DDM>(op, x, bb, color, omega, lane, p, j, k0);
}

// rbsor_core! with its residual (NonUniform.jl:848-915) for solveSOR! (NonUniform.jl:1004-1051):
// colour `color` updated with relaxation omega, sum of r^2 -> stage (kStageSorHalf after colour
// 0, kStageSorIter after colour 1).  The colour-1 launch ends a WHILE-body pass: block 0 counts
// the pass and ends the loop provisionally; only the finisher can continue it.
template <bool COND, int DDM = 1>
__global__ void __launch_bounds__(kThreads) k_sor_pass(OpParams<double> op, double* x,
                                                       const double* __restrict__ bb, int color, double omega,
                                                       SolverState* st, double* __restrict__ partials, int stage,
                                                       cudaGraphConditionalHandle hc, int use_cond) {
  pdl_enter();
  if (color == 1 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    st->passes += 1;
    if constexpr (COND) set_cond(hc, use_cond, 0);
  }
  if (st->stop) return;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int k0 = 1 + 2 * blockIdx.z;
  double v[1] = {0.0};
  if (j <= op.g.NY) v[0] = rb_pass_column<double, true, 2, DDM>(op, x, bb, color, omega, lane, p, j, k0);
  reduce_finish<1, COND>(v, partials, st, stage, hc, color == 1 ? use_cond : 0);
}

// ------------------------------------------------------------------------------------------
// First colour pass of the preconditioner (xx starts at zero, the caller's myfill!,
// NonUniform.jl:303/313), fused with the Krylov update that produces its right-hand side:
//   VM 0: bb is given (CG: z = M^-1 r)
//   VM 1: p = r (first iteration) or p = r + beta*(p - omega*q)    BiCG1!, NonUniform.jl:296-301
//   VM 2: s = (-alpha)*q + r                                         Triad!, NonUniform.jl:310-311
// Colour-0 cells get xx = ((0 - bb)/dd - 0)*m0; colour-1 cells get 0.  With smoother :none
// (copy_only) xx = bb everywhere (mycopy!, NonUniform.jl:549-551).  T: precision of the smoother
// (xx, operator tables); TV: precision of the Krylov vectors; when they differ, bbT receives the
// smoother's copy of the right-hand side in T.  Thread = both colours of column (p,j) at plane k.
// ------------------------------------------------------------------------------------------
template <typename T, typename TV, int VM, bool CL = false>
__device__ __forceinline__ void rb_first_column(const OpParams<T>& op, T* __restrict__ xx, TV* __restrict__ v,
                                                T* __restrict__ bbT, const TV* __restrict__ r,
                                                const TV* __restrict__ q, const SolverState* __restrict__ st,
                                                int copy_only, int lane, int p, int j, int k) {
  const Geo& g = op.g;
  const bool pok = p < g.HN;
  const uint8_t* key = op.key;
  const int HP2 = 2 * g.HP, PL = (int)g.plane;
  const int r0 = g.row(0, j, k), r1 = r0 + g.HP;
  TV beta = TV(0), omg = TV(0), alpha = TV(0);
  int first = 0;
  if (VM == 1) {
    first = st->first;
    beta = (TV)st->beta;
    omg = (TV)st->omega;
  } else if (VM == 2) {
    alpha = (TV)st->alpha;
  }
  const int e0 = (1 + j + k) & 1;
  bool ok[2];
  TV bvv[2];
#pragma unroll
  for (int col = 0; col < 2; ++col) {
    const int i = 2 * p + (e0 ^ col);
    ok[col] = pok && i >= 1 && i <= g.NX;
    bvv[col] = TV(0);
    if (!ok[col]) continue;
    const int ci = (col ? r1 : r0) + p;
    if (VM == 0) bvv[col] = v[ci];
    else if (VM == 1) bvv[col] = first ? r[ci] : add(r[ci], mul(beta, sub(v[ci], mul(omg, q[ci]))));
    else bvv[col] = add(mul(-alpha, q[ci]), r[ci]);
  }
  // keys for the colour-0 cell: its own and its colour-1 neighbours (or its stencil class)
  int k1c = 0, k1m = 0, k1p = 0, kym = 0, kyp = 0, k0c = 0;
  int kxm = 0, kxp = 0;
  unsigned cl = kNoClass;
  if (CL) {
    if (!copy_only && ok[0]) cl = __ldg(op.cls + r0 + p);
  } else if (H2G_NKEY) {
    if (!copy_only && ok[0]) {
      const unsigned long long w = __ldg(op.nkey + r0 + p);  // own, x-, x+, y-, y+, z-, z+
      k0c = (int)(w & 0xff);
      kxm = (int)((w >> 8) & 0xff);
      kxp = (int)((w >> 16) & 0xff);
      kym = (int)((w >> 24) & 0xff);
      kyp = (int)((w >> 32) & 0xff);
      k1m = (int)((w >> 40) & 0xff);
      k1p = (int)((w >> 48) & 0xff);
    }
  } else {
    if (!copy_only && pok) {
      const int a1 = r1 + p;
      k1c = key[a1];
      if (ok[0]) {
        k1m = key[a1 - PL];
        k1p = key[a1 + PL];
        kym = key[a1 - HP2];
        kyp = key[a1 + HP2];
        k0c = key[r0 + p];
      }
    }
    if (!copy_only) {
      T dm, dp_;
      x_nbrs<T, false>(T(0), k1c, e0, lane, p, g.HN, (const T*)nullptr, key, r1, dm, dp_, kxm, kxp);
    }
  }
#pragma unroll
  for (int col = 0; col < 2; ++col) {
    if (!ok[col]) continue;
    const int ci = (col ? r1 : r0) + p;
    const TV bvx = bvv[col];
    if (VM != 0) v[ci] = bvx;
    const T b = (T)bvx;
    if (bbT) bbT[ci] = b;
    T out = T(0);
    if (copy_only) {
      out = b;
    } else if (col == 0) {
      Coef<T> c;
      bool has;
      if constexpr (CL) has = class_coef<T>(op, cl, ci, c);
      else
        has = cell_coef<T, true>(op, k, (uint8_t)k0c, (uint8_t)kxm, (uint8_t)kxp, (uint8_t)kym, (uint8_t)kyp,
                                 (uint8_t)k1m, (uint8_t)k1p, ci, c);
      if (has) {
        const T ss = T(0);
        const T dp = sub(gs_div(sub(ss, b), c.dd), T(0));
        out = add(T(0), dp);  // pp + omega*dp with pp = 0, omega = 1
      }
    }
    xx[ci] = out;
  }
}

template <typename T, typename TV, int VM, bool CL = false>
__global__ void __launch_bounds__(kThreads) k_rb_first(OpParams<T> op, T* __restrict__ xx, TV* __restrict__ v,
                                                        T* __restrict__ bbT, const TV* __restrict__ r,
                                                        const TV* __restrict__ q, const SolverState* __restrict__ st,
                                                        int copy_only) {
  pdl_enter();
  if (st && st->stop) return;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (j > op.g.NY) return;
  rb_first_column<T, TV, VM, CL>(op, xx, v, bbT, r, q, st, copy_only, lane, p, j, k);
}

// Both colours of column (p, j) at plane k: the values (centre and z-neighbours) and keys of the
// two columns, and the y-neighbour values and keys of each colour.
template <typename T, typename TI>
struct Pair {
  T c0[3], c1[3];  // colour 0 / 1 column at planes k-1, k, k+1
  int kc0[3], kc1[3];
  T y0m, y0p, y1m, y1p;
  int ky0m, ky0p, ky1m, ky1p;
};

template <typename T, typename TI, bool KEYS = true>
__device__ __forceinline__ void load_pair(const Geo& g, const TI* x, const uint8_t* key, int r0, int p, bool pok,
                                          Pair<T, TI>& P) {
  const int r1 = r0 + g.HP, PL = (int)g.plane, HP2 = 2 * g.HP;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    P.c0[t] = P.c1[t] = T(0);
    P.kc0[t] = P.kc1[t] = 0;
  }
  P.y0m = P.y0p = P.y1m = P.y1p = T(0);
  P.ky0m = P.ky0p = P.ky1m = P.ky1p = 0;
  if (!pok) return;
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const int a0 = r0 + (t - 1) * PL + p, a1 = r1 + (t - 1) * PL + p;
    P.c0[t] = (T)ldro(x + a0);
    P.c1[t] = (T)ldro(x + a1);
    if (KEYS) {
      P.kc0[t] = key[a0];
      P.kc1[t] = key[a1];
    }
  }
  P.y0m = (T)ldro(x + r0 + p - HP2);
  P.y0p = (T)ldro(x + r0 + p + HP2);
  P.y1m = (T)ldro(x + r1 + p - HP2);
  P.y1p = (T)ldro(x + r1 + p + HP2);
  if (KEYS) {
    P.ky0m = key[r0 + p - HP2];
    P.ky0p = key[r0 + p + HP2];
    P.ky1m = key[r1 + p - HP2];
    P.ky1p = key[r1 + p + HP2];
  }
}

// ------------------------------------------------------------------------------------------
// CalcAX! (NonUniform.jl:454-511): y = A x, fused with up to two dot products
//   d1 = sum y*u (u == nullptr: y*y),  d2 = sum y*w
// and the stage finisher.  TI: type of x (the preconditioner output may be FP32 while A is
// applied in FP64).  Grid (ceil(HN/32), ceil(NY/kBY), NZ).
// ------------------------------------------------------------------------------------------
// DDM: 0 coefficients from the key tables with dd summed; 1 dd read from the per-cell array (FP64
// only; the FP32 operator uses the difference form); 2 the stencil-class table (FP64 only).  Which is
// faster depends on whether the vectors stay in L2; the launch-shape tuner decides.
template <typename T, int NDOT, typename TI = T, int DDM = 0>
__global__ void __launch_bounds__(kThreads, H2G_AX_MINB) k_ax(OpParams<T> op, T* __restrict__ y, const TI* __restrict__ x,
                                                  const T* __restrict__ u, const T* __restrict__ w,
                                                  SolverState* st, double* __restrict__ partials, int stage) {
  pdl_enter();
  if (st && st->stop) return;
  const Geo& g = op.g;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int k = 1 + blockIdx.z;
  double v[NDOT > 0 ? NDOT : 1];
#pragma unroll
  for (int q = 0; q < (NDOT > 0 ? NDOT : 1); ++q) v[q] = 0.0;
  if (j <= g.NY) {  // uniform per warp
    const bool pok = p < g.HN;
    const uint8_t* key = op.key;
    const int r0 = g.row(0, j, k), r1 = r0 + g.HP;
    const int e0 = (1 + j + k) & 1;
    bool ok[2];
    T uu[2] = {T(0), T(0)}, ww[2] = {T(0), T(0)};
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      const int i = 2 * p + (e0 ^ col);
      ok[col] = pok && i >= 1 && i <= g.NX;
      if (ok[col]) {
        const int ci = (col ? r1 : r0) + p;
        if (NDOT >= 1 && u) uu[col] = u[ci];
        if (NDOT >= 2) ww[col] = w[ci];
      }
    }
    constexpr bool CL = DDM == 2;
    constexpr bool NK = H2G_NKEY != 0 || CL;
    unsigned long long nk[2] = {0ull, 0ull};
    unsigned cl[2] = {kNoClass, kNoClass};
    if (CL) {
#pragma unroll
      for (int col = 0; col < 2; ++col)
        if (ok[col]) cl[col] = __ldg(op.cls + (col ? r1 : r0) + p);
    } else if (NK) {
#pragma unroll
      for (int col = 0; col < 2; ++col)
        if (ok[col]) nk[col] = __ldg(op.nkey + (col ? r1 : r0) + p);
    }
    Pair<T, TI> P;
    load_pair<T, TI, !NK>(g, x, key, r0, p, pok, P);
    T xm0, xp0, xm1, xp1;
    int kxm0, kxp0, kxm1, kxp1;
    // colour-0 cell: neighbours of colour 1; colour-1 cell: neighbours of colour 0
    x_nbrs<T, true, TI, !NK>(P.c1[1], P.kc1[1], e0, lane, p, g.HN, x, key, r1, xm0, xp0, kxm0, kxp0);
    x_nbrs<T, true, TI, !NK>(P.c0[1], P.kc0[1], e0 ^ 1, lane, p, g.HN, x, key, r0, xm1, xp1, kxm1, kxp1);
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      if (!ok[col]) continue;
      const int ci = (col ? r1 : r0) + p;
      Coef<T> c;
      T out = T(0);
      bool has;
      if constexpr (CL) {
        has = class_coef<T>(op, cl[col], ci, c);
      } else if (NK) {
        const unsigned long long wk = nk[col];  // own, x-, x+, y-, y+, z-, z+ keys in bytes 0..6
        has = cell_coef<T, DDM == 1 && sizeof(T) == 8>(op, k, (uint8_t)wk, (uint8_t)(wk >> 8), (uint8_t)(wk >> 16),
                                                 (uint8_t)(wk >> 24), (uint8_t)(wk >> 32), (uint8_t)(wk >> 40),
                                                 (uint8_t)(wk >> 48), ci, c);
      } else if (col == 0) {
        has = cell_coef<T, DDM == 1 && sizeof(T) == 8>(op, k, (uint8_t)P.kc0[1], (uint8_t)kxm0, (uint8_t)kxp0,
                                                 (uint8_t)P.ky1m, (uint8_t)P.ky1p, (uint8_t)P.kc1[0],
                                                 (uint8_t)P.kc1[2], ci, c);
      } else {
        has = cell_coef<T, DDM == 1 && sizeof(T) == 8>(op, k, (uint8_t)P.kc1[1], (uint8_t)kxm1, (uint8_t)kxp1,
                                                 (uint8_t)P.ky0m, (uint8_t)P.ky0p, (uint8_t)P.kc0[0],
                                                 (uint8_t)P.kc0[2], ci, c);
      }
      if (has) {
        if (col == 0) out = apply_a(c, P.c0[1], xp0, xm0, P.y1p, P.y1m, P.c1[2], P.c1[0]);
        else out = apply_a(c, P.c1[1], xp1, xm1, P.y0p, P.y0m, P.c0[2], P.c0[0]);
      }
      y[ci] = out;
      if (NDOT >= 1) v[0] += (double)out * (u ? (double)uu[col] : (double)out);
      if (NDOT >= 2) v[NDOT - 1] += (double)out * (double)ww[col];
    }
  }
  if constexpr (NDOT > 0) reduce_finish<NDOT>(v, partials, st, stage, 0, 0);
}

// ------------------------------------------------------------------------------------------
// CalcRK! (NonUniform.jl:372-434): r = (b - (ss - dd*th))*m0, sum r^2 -> stage.
// Optional copy r0 = r (PBiCGSTAB's mycopy!, NonUniform.jl:274).  th and b are FP64; r is T.
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_rk(OpParams<double> op, T* __restrict__ r, T* __restrict__ r0c,
                                                  const double* __restrict__ th, const double* __restrict__ b,
                                                  SolverState* st, double* __restrict__ partials, int stage) {
  pdl_enter();
  const Geo& g = op.g;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int k = 1 + blockIdx.z;
  double v[1] = {0.0};
  if (j <= g.NY) {
    const bool pok = p < g.HN;
    const uint8_t* key = op.key;
    const int r0 = g.row(0, j, k), r1 = r0 + g.HP;
    const int e0 = (1 + j + k) & 1;
    bool ok[2];
    double bb[2] = {0.0, 0.0};
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      const int i = 2 * p + (e0 ^ col);
      ok[col] = pok && i >= 1 && i <= g.NX;
      if (ok[col]) bb[col] = b[(col ? r1 : r0) + p];
    }
    Pair<double, double> P;
    load_pair<double, double>(g, th, key, r0, p, pok, P);
    double xm0, xp0, xm1, xp1;
    int kxm0, kxp0, kxm1, kxp1;
    x_nbrs<double, true>(P.c1[1], P.kc1[1], e0, lane, p, g.HN, th, key, r1, xm0, xp0, kxm0, kxp0);
    x_nbrs<double, true>(P.c0[1], P.kc0[1], e0 ^ 1, lane, p, g.HN, th, key, r0, xm1, xp1, kxm1, kxp1);
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      if (!ok[col]) continue;
      const int ci = (col ? r1 : r0) + p;
      Coef<double> c;
      double rs = 0.0;
      bool has;
      if (col == 0)
        has = cell_coef<double, true>(op, k, (uint8_t)P.kc0[1], (uint8_t)kxm0, (uint8_t)kxp0, (uint8_t)P.ky1m, (uint8_t)P.ky1p,
                        (uint8_t)P.kc1[0], (uint8_t)P.kc1[2], ci, c);
      else
        has = cell_coef<double, true>(op, k, (uint8_t)P.kc1[1], (uint8_t)kxm1, (uint8_t)kxp1, (uint8_t)P.ky0m, (uint8_t)P.ky0p,
                        (uint8_t)P.kc0[0], (uint8_t)P.kc0[2], ci, c);
      if (has) {
        const double ss = col == 0 ? nb_sum(c, xp0, xm0, P.y1p, P.y1m, P.c1[2], P.c1[0])
                                   : nb_sum(c, xp1, xm1, P.y0p, P.y0m, P.c0[2], P.c0[0]);
        rs = sub(bb[col], sub(ss, mul(c.dd, col == 0 ? P.c0[1] : P.c1[1])));
      }
      r[ci] = (T)rs;
      if (r0c) r0c[ci] = (T)rs;
      v[0] += rs * rs;
    }
  }
  reduce_finish<1>(v, partials, st, stage, 0, 0);
}

// ------------------------------------------------------------------------------------------
// resSOR (NonUniform.jl:680-743): the SOR residual of the current th without updating it,
//   dp = ((ss - b)/dd - th)*m0,  r = (dd + omega*(c_xm + c_ym + c_zm))*dp/omega,
// sum r^2 over the interior -> stage.  Both colours of column (p, j) at plane k.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_res_sor(OpParams<double> op, const double* __restrict__ th,
                                                       const double* __restrict__ b, double omega, SolverState* st,
                                                       double* __restrict__ partials, int stage) {
  pdl_enter();
  const Geo& g = op.g;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int k = 1 + blockIdx.z;
  double v[1] = {0.0};
  if (j <= g.NY) {
    const bool pok = p < g.HN;
    const uint8_t* key = op.key;
    const int r0 = g.row(0, j, k), r1 = r0 + g.HP;
    const int e0 = (1 + j + k) & 1;
    bool ok[2];
    double bb[2] = {0.0, 0.0};
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      const int i = 2 * p + (e0 ^ col);
      ok[col] = pok && i >= 1 && i <= g.NX;
      if (ok[col]) bb[col] = b[(col ? r1 : r0) + p];
    }
    Pair<double, double> P;
    load_pair<double, double>(g, th, key, r0, p, pok, P);
    double xm0, xp0, xm1, xp1;
    int kxm0, kxp0, kxm1, kxp1;
    x_nbrs<double, true>(P.c1[1], P.kc1[1], e0, lane, p, g.HN, th, key, r1, xm0, xp0, kxm0, kxp0);
    x_nbrs<double, true>(P.c0[1], P.kc0[1], e0 ^ 1, lane, p, g.HN, th, key, r0, xm1, xp1, kxm1, kxp1);
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      if (!ok[col]) continue;
      const int ci = (col ? r1 : r0) + p;
      Coef<double> c;
      bool has;
      if (col == 0)
        has = cell_coef<double, true>(op, k, (uint8_t)P.kc0[1], (uint8_t)kxm0, (uint8_t)kxp0, (uint8_t)P.ky1m, (uint8_t)P.ky1p,
                        (uint8_t)P.kc1[0], (uint8_t)P.kc1[2], ci, c);
      else
        has = cell_coef<double, true>(op, k, (uint8_t)P.kc1[1], (uint8_t)kxm1, (uint8_t)kxp1, (uint8_t)P.ky0m, (uint8_t)P.ky0p,
                        (uint8_t)P.kc0[0], (uint8_t)P.kc0[2], ci, c);
      if (!has) continue;
      const double ss = col == 0 ? nb_sum(c, xp0, xm0, P.y1p, P.y1m, P.c1[2], P.c1[0])
                                 : nb_sum(c, xp1, xm1, P.y0p, P.y0m, P.c0[2], P.c0[0]);
      const double dp = sub(gs_div(sub(ss, bb[col]), c.dd), col == 0 ? P.c0[1] : P.c1[1]);
      const double r = dvd(mul(add(c.dd, mul(omega, add(add(c.cxm, c.cym), c.czm))), dp), omega);
      v[0] = add(v[0], mul(r, r));
    }
  }
  reduce_finish<1>(v, partials, st, stage, 0, 0);
}

// ------------------------------------------------------------------------------------------
// Element-wise kernels over whole vectors.  Guard and padding entries of every Krylov vector
// are zero and stay zero, so these run linearly over the buffer with 16-byte accesses.
// ------------------------------------------------------------------------------------------
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
};
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
};

// V consecutive elements of type TT (V*sizeof(TT) = 8 or 16 bytes), converted to T
template <typename T, typename TT, int V>
__device__ __forceinline__ void ldv(const TT* p, T (&a)[V]) {
  if constexpr (sizeof(TT) * V == 16) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    const TT* s = reinterpret_cast<const TT*>(&v);
#pragma unroll
    for (int q = 0; q < V; ++q) a[q] = (T)s[q];
  } else {
    static_assert(sizeof(TT) * V == 8, "vector width");
    const float2 v = *reinterpret_cast<const float2*>(p);
    const TT* s = reinterpret_cast<const TT*>(&v);
#pragma unroll
    for (int q = 0; q < V; ++q) a[q] = (T)s[q];
  }
}

template <typename T>
__device__ __forceinline__ void ld16(const T* p, T (&a)[Vec16<T>::n]) {
  const typename Vec16<T>::type v = *reinterpret_cast<const typename Vec16<T>::type*>(p);
  const T* s = reinterpret_cast<const T*>(&v);
#pragma unroll
  for (int q = 0; q < Vec16<T>::n; ++q) a[q] = s[q];
}
template <typename T>
__device__ __forceinline__ void st16(T* p, const T (&a)[Vec16<T>::n]) {
  typename Vec16<T>::type v;
  T* d = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int q = 0; q < Vec16<T>::n; ++q) d[q] = a[q];
  *reinterpret_cast<typename Vec16<T>::type*>(p) = v;
}

// BICG2! + Triad! + Fdot1/Fdot2 (NonUniform.jl:328-331 and the next 289):
//   x += alpha*ph + omega*sh;  r = (-omega)*t + s;  d1 = (r,r), d2 = (r,r0) -> kStageUpdate
template <typename T, typename TX, typename TP = T, bool COND = true>
__global__ void __launch_bounds__(256) k_bicg_update(long long n, TX* __restrict__ x, const TP* __restrict__ ph,
                                                      const TP* __restrict__ sh, T* __restrict__ r,
                                                      const T* __restrict__ s, const T* __restrict__ t,
                                                      const T* __restrict__ r0, SolverState* st,
                                                      double* __restrict__ partials, cudaGraphConditionalHandle hc,
                                                      int use_cond) {
  pdl_enter();
  // Fail-safe loop bound: block 0 counts the pass and ends the loop provisionally; only the
  // finisher of this kernel (which runs after block 0 has arrived) can continue it.
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->passes += 1;
    if constexpr (COND) set_cond(hc, use_cond, 0);
  }
  if (st->stop) return;
  constexpr int V = Vec16<T>::n;
  const T alpha = (T)st->alpha, omega = (T)st->omega, nomega = (T)(-st->omega);
  double v[2] = {0.0, 0.0};
  const long long nv = n / V;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nv; b += (long long)gridDim.x * blockDim.x) {
    const long long o = b * V;
    T a_ph[V], a_sh[V], a_s[V], a_t[V], a_r0[V], a_r[V];
    ldv<T, TP, V>(ph + o, a_ph);
    ldv<T, TP, V>(sh + o, a_sh);
    ld16(s + o, a_s);
    ld16(t + o, a_t);
    ld16(r0 + o, a_r0);
#pragma unroll
    for (int q = 0; q < V; ++q) {
      x[o + q] = (TX)add((T)x[o + q], add(mul(alpha, a_ph[q]), mul(omega, a_sh[q])));
      a_r[q] = add(mul(nomega, a_t[q]), a_s[q]);
      v[0] += (double)a_r[q] * (double)a_r[q];
      v[1] += (double)a_r[q] * (double)a_r0[q];
    }
    st16(r + o, a_r);
  }
  reduce_finish<2, COND>(v, partials, st, kStageUpdate, hc, use_cond);
}

// CG! fused update (NonUniform.jl:179-182) + Fdot1 (185): x += alpha*p; r -= alpha*q; (r,r)
template <typename T, typename TX>
__global__ void __launch_bounds__(256) k_cg_update(long long n, TX* __restrict__ x, const T* __restrict__ p,
                                                    T* __restrict__ r, const T* __restrict__ q, SolverState* st,
                                                    double* __restrict__ partials) {
  pdl_enter();
  if (st->stop) return;
  constexpr int V = Vec16<T>::n;
  const T alpha = (T)st->alpha;
  double v[1] = {0.0};
  const long long nv = n / V;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nv; b += (long long)gridDim.x * blockDim.x) {
    const long long o = b * V;
    T a_p[V], a_q[V], a_r[V];
    ld16(p + o, a_p);
    ld16(q + o, a_q);
    ld16(r + o, a_r);
#pragma unroll
    for (int k = 0; k < V; ++k) {
      x[o + k] = (TX)add((T)x[o + k], mul(alpha, a_p[k]));
      a_r[k] = sub(a_r[k], mul(alpha, a_q[k]));
      v[0] += (double)a_r[k] * (double)a_r[k];
    }
    st16(r + o, a_r);
  }
  reduce_finish<1>(v, partials, st, kStageCgRes, 0, 0);
}

// d1 = (a,b) with an optional copy dst = b (CG: p = z and rho = (r,z), NonUniform.jl:152-155)
template <typename T, typename T2 = T>
__global__ void __launch_bounds__(256) k_dot(long long n, const T* __restrict__ a, const T2* __restrict__ b,
                                              T* __restrict__ dst, SolverState* st, double* __restrict__ partials,
                                              int stage) {
  pdl_enter();
  if (st->stop) return;
  constexpr int V = Vec16<T>::n;
  double v[1] = {0.0};
  const long long nv = n / V;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const long long o = i * V;
    T a_a[V], a_b[V];
    ld16(a + o, a_a);
    ldv<T, T2, V>(b + o, a_b);
#pragma unroll
    for (int k = 0; k < V; ++k) v[0] += (double)a_a[k] * (double)a_b[k];
    if (dst) st16(dst + o, a_b);
  }
  reduce_finish<1>(v, partials, st, stage, 0, 0);
}

// CG! p = z + beta*p (NonUniform.jl:218-220); sets the loop condition.
template <typename T, typename TP = T, bool COND = true>
__global__ void __launch_bounds__(256) k_cg_pupd(long long n, T* __restrict__ p, const TP* __restrict__ z,
                                                  SolverState* st, cudaGraphConditionalHandle hc, int use_cond) {
  pdl_enter();
  const int stop = st->stop;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->passes += 1;
    if constexpr (COND) set_cond(hc, use_cond, !stop && st->passes <= st->maxItr + 1);
  }
  if (stop) return;
  constexpr int V = Vec16<T>::n;
  const T beta = (T)st->beta;
  const long long nv = n / V;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const long long o = i * V;
    T a_p[V], a_z[V];
    ld16(p + o, a_p);
    ldv<T, TP, V>(z + o, a_z);
#pragma unroll
    for (int k = 0; k < V; ++k) a_p[k] = add(a_z[k], mul(beta, a_p[k]));
    st16(p + o, a_p);
  }
}

// Iterative refinement: scale the FP64 residual into the FP32 inner right-hand side,
// r = r0 = (float)(r64 / ||r64||), e = 0, and start the inner solve (kStageInit).
__global__ void __launch_bounds__(256) k_ir_prep(long long n, const double* __restrict__ r64, float* __restrict__ r,
                                                  float* __restrict__ r0, float* __restrict__ e,
                                                  const SolverState* __restrict__ outer, SolverState* inner,
                                                  double* __restrict__ partials, int stage) {
  pdl_enter();
  const double inv = 1.0 / outer->scale;
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float x = (float)(r64[i] * inv);
    r[i] = x;
    r0[i] = x;
    e[i] = 0.0f;
    v[0] += (double)x * (double)x;
  }
  reduce_finish<1>(v, partials, inner, stage, 0, 0);
}

// Host-controlled fields of a state: tolerance, iteration cap and residual history.
__global__ void k_prime(SolverState* st, double tol, int maxItr, double* hist, int hist_len, double div_limit) {
  pdl_enter();
  st->div_limit = div_limit;
  st->tol = tol;
  st->maxItr = maxItr;
  st->hist = hist;
  st->hist_len = hist_len;
  st->stop = 0;
  st->ticket = 0;
  st->passes = 0;
}

// Iterative refinement: th += ||r64|| * e (FP64 accumulation of the FP32 correction).
__global__ void __launch_bounds__(256) k_ir_apply(long long n, double* __restrict__ th, const float* __restrict__ e,
                                                   const SolverState* __restrict__ outer) {
  pdl_enter();
  const double sc = outer->scale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    th[i] += sc * (double)e[i];
}

// ------------------------------------------------------------------------------------------
// Layout conversion between the reference's column-major arrays and the device layout.
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_to_dev(Geo g, const double* __restrict__ src, T* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.MX) return;
  dst[g.off(i, j, k)] = (T)src[(long long)i + (long long)g.MX * ((long long)j + (long long)g.MY * k)];
}

template <typename T>
__global__ void k_from_dev(Geo g, const T* __restrict__ src, double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.MX) return;
  dst[(long long)i + (long long)g.MX * ((long long)j + (long long)g.MY * k)] = (double)src[g.off(i, j, k)];
}

// ------------------------------------------------------------------------------------------
// calRHS! (src/NonUniform.jl:57-91) with apply_bc2RHS! (src/RHS.jl:23-192), one thread per
// interior cell (i fastest).  The boundary faces are applied in the reference's order x-, x+,
// y-, y+, z-, z+ to the cells next to them, then b = -(a_p0*theta + hsrc*dx*dy*dz + b).
// ------------------------------------------------------------------------------------------
struct FaceBC {
  int type[6];     // 0 isothermal (no RHS term), 1 heat flux, 2 convection
  double q[6];     // heat flux
  double h[6];     // heat-transfer coefficient
  double ta[6];    // ambient temperature
};

// One face of RHS_heat_flux! / RHS_convection! (RHS.jl:70-186): sign -1 for the minus faces
// (b += q*area; b -= h*area*(ta - theta)), +1 for the plus faces (b -= q*area; b += ...).
__device__ __forceinline__ double face_term(const FaceBC& bc, int f, double b, double area, double th, int plus) {
  if (bc.type[f] == 1) {
    const double t = __dmul_rn(bc.q[f], area);
    return plus ? __dsub_rn(b, t) : __dadd_rn(b, t);
  }
  if (bc.type[f] == 2) {
    const double t = __dmul_rn(__dmul_rn(bc.h[f], area), __dsub_rn(bc.ta[f], th));
    return plus ? __dadd_rn(b, t) : __dsub_rn(b, t);
  }
  return b;
}

__global__ void __launch_bounds__(256) k_calrhs(Geo g, double* __restrict__ b, const double* __restrict__ th,
                                                 const double* __restrict__ hsrc, const double* __restrict__ rc,
                                                 const double* __restrict__ dzk, double dx, double dy, double ddt,
                                                 int steady, FaceBC bc, int zero_b) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > g.NX) return;
  const int o = g.off(i, j, k);
  const double t = th[o], dz = __ldg(dzk + k);
  double bv = zero_b ? 0.0 : b[o];
  const double ax = __dmul_rn(dy, dz), ay = __dmul_rn(dx, dz), az = __dmul_rn(dx, dy);
  if (i == 1) bv = face_term(bc, 0, bv, ax, t, 0);
  if (i == g.NX) bv = face_term(bc, 1, bv, ax, t, 1);
  if (j == 1) bv = face_term(bc, 2, bv, ay, t, 0);
  if (j == g.NY) bv = face_term(bc, 3, bv, ay, t, 1);
  if (k == 1) bv = face_term(bc, 4, bv, az, t, 0);
  if (k == g.NZ) bv = face_term(bc, 5, bv, az, t, 1);
  const double ap = steady ? 0.0 : __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(rc[o], dx), dy), dz), ddt);
  const double hs = __dmul_rn(__dmul_rn(__dmul_rn(hsrc[o], dx), dy), dz);
  b[o] = -__dadd_rn(__dadd_rn(__dmul_rn(ap, t), hs), bv);
}

// min, max and sum of squares of theta over the interior (the per-step line of main(),
// heat3ds.jl:149-151).  Stage 1: one partial triple per block; stage 2 (one block) reduces the
// partials in block order and writes out[0..2].
__global__ void __launch_bounds__(256) k_theta_stats1(Geo g, const double* __restrict__ th,
                                                       double* __restrict__ partials) {
  double mn = INFINITY, mx = -INFINITY, ss = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < g.n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(idx / g.HP), p = (int)(idx % g.HP);
    const int c = row & 1, jk = row >> 1, j = jk % g.MY, k = jk / g.MY;
    const int i = 2 * p + ((1 + c + j + k) & 1);
    if (i < 1 || i > g.NX || j < 1 || j > g.NY || k < 1 || k > g.NZ) continue;
    const double v = th[idx];
    mn = fmin(mn, v);
    mx = fmax(mx, v);
    ss = __dadd_rn(ss, __dmul_rn(v, v));
  }
  __shared__ double sm[3][8];
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_down_sync(kFull, mn, o));
    mx = fmax(mx, __shfl_down_sync(kFull, mx, o));
    ss += __shfl_down_sync(kFull, ss, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { sm[0][w] = mn; sm[1][w] = mx; sm[2][w] = ss; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
      mn = fmin(mn, sm[0][q]);
      mx = fmax(mx, sm[1][q]);
      ss += sm[2][q];
    }
    partials[3 * blockIdx.x] = mn;
    partials[3 * blockIdx.x + 1] = mx;
    partials[3 * blockIdx.x + 2] = ss;
  }
}

__global__ void __launch_bounds__(32) k_theta_stats2(const double* __restrict__ partials, int nb,
                                                      double* __restrict__ out) {
  double mn = INFINITY, mx = -INFINITY, ss = 0.0;
  for (int q = threadIdx.x; q < nb; q += 32) {
    mn = fmin(mn, partials[3 * q]);
    mx = fmax(mx, partials[3 * q + 1]);
    ss += partials[3 * q + 2];
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_down_sync(kFull, mn, o));
    mx = fmax(mx, __shfl_down_sync(kFull, mx, o));
    ss += __shfl_down_sync(kFull, ss, o);
  }
  if (threadIdx.x == 0) {
    out[0] = mn;
    out[1] = mx;
    out[2] = sqrt(ss);
  }
}

// ------------------------------------------------------------------------------------------
// Steady adjoint of J = (sum_c w_c theta_c^p)^(1/p) (no reference counterpart).
// ------------------------------------------------------------------------------------------
// sum w*theta^p over the vector (guards and padding carry w = 0) -> kStageDot (dot1)
__global__ void __launch_bounds__(256) k_objective(long long n, const double* __restrict__ th,
                                                    const double* __restrict__ w, double p, SolverState* st,
                                                    double* __restrict__ partials) {
  pdl_enter();
  double v[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double wi = w[i];
    if (wi != 0.0) v[0] += wi * pow(th[i], p);
  }
  reduce_finish<1>(v, partials, st, kStageDot, 0, 0);
}

// g = dJ/dtheta = w * theta^(p-1) * J^(1-p), J = dot1^(1/p)
__global__ void __launch_bounds__(256) k_adj_rhs(long long n, const double* __restrict__ th,
                                                  const double* __restrict__ w, double p,
                                                  const SolverState* __restrict__ st, double* __restrict__ g) {
  pdl_enter();
  const double J = pow(st->dot1, 1.0 / p), sc = pow(J, 1.0 - p);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double wi = w[i];
    g[i] = wi != 0.0 ? wi * pow(th[i], p - 1.0) * sc : 0.0;
  }
}

// Gradients from theta (physical guards) and the adjoint field la (zero guards), A la = g:
//   dJ/dhsrc_c       = -V_c la_c                        (b = -(hsrc V + ...), calRHS!)
//   dJ/dln(lambda_c) = -sum over the faces f of c of  c_f w_f (theta_q - theta_c)(la_c - la_q)
// with c_f the face conductance (the operator's tables) and w_f = d ln c_f / d ln lambda_c =
// lambda_q / (lambda_c + lambda_q) for a neighbour with its own lambda, 1 for a guard (a guard's
// lambda is 0, or a copy of lambda_c on an isothermal face, boundary_conditions.jl:198-205).
// One thread per interior cell.
__global__ void __launch_bounds__(256) k_adj_grad(OpParams<double> op, const double* __restrict__ lamv,
                                                   const double* __restrict__ th, const double* __restrict__ la,
                                                   double* __restrict__ G, double* __restrict__ gh, int acc) {
  const Geo& g = op.g;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > g.NX) return;
  const int o = g.off(i, j, k);
  const int nb[6] = {g.off(i - 1, j, k), g.off(i + 1, j, k), g.off(i, j - 1, k),
                     g.off(i, j + 1, k), g.off(i, j, k - 1), g.off(i, j, k + 1)};
  const uint8_t k0 = op.key[o];
  uint8_t kn[6];
#pragma unroll
  for (int f = 0; f < 6; ++f) kn[f] = op.key[nb[f]];
  Coef<double> c;
  if (!cell_coef(op, k, k0, kn[0], kn[1], kn[2], kn[3], kn[4], kn[5], o, c)) {
    if (!acc) {
      G[o] = 0.0;
      gh[o] = 0.0;
    }
    return;
  }
  const double cf[6] = {c.cxm, c.cxp, c.cym, c.cyp, c.czm, c.czp};
  const double lp = lamv[k0 & 0x7f], tp = th[o], ap = la[o];
  double s = 0.0;
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    if (cf[f] == 0.0) continue;
    const bool guard = !(kn[f] & 0x80);
    const double lq = lamv[kn[f] & 0x7f];
    const double wf = guard ? 1.0 : lq / (lp + lq);
    const double aq = guard ? 0.0 : la[nb[f]];
    s += cf[f] * wf * (th[nb[f]] - tp) * (ap - aq);
  }
  const double gv = -(op.dx0 * op.dy0 * __ldg(op.dzk + k)) * ap;
  G[o] = acc ? G[o] - s : -s;
  gh[o] = acc ? gh[o] + gv : gv;
}

// Transient adjoint step: the right-hand side of step n+1 depends on theta^n through calRHS!
// (NonUniform.jl:87-90, RHS.jl:140-186):  db_c/dtheta_c = -a_p0 - sum_{convective minus faces}
// h*area + sum_{convective plus faces} h*area, so lam^n = (db/dtheta^n) * mu^{n+1} per cell.
__global__ void __launch_bounds__(256) k_adj_step(Geo g, const double* __restrict__ mu, double* __restrict__ lam,
                                                   const double* __restrict__ rc, const double* __restrict__ dzk,
                                                   double dx, double dy, double ddt, FaceBC bc) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > g.NX) return;
  const int o = g.off(i, j, k);
  const double dz = __ldg(dzk + k);
  const double ax = dy * dz, ay = dx * dz, az = dx * dy;
  double d = -(rc[o] * dx * dy * dz * ddt);
  const bool on[6] = {i == 1, i == g.NX, j == 1, j == g.NY, k == 1, k == g.NZ};
  const double area[6] = {ax, ax, ay, ay, az, az};
#pragma unroll
  for (int f = 0; f < 6; ++f)
    if (on[f] && bc.type[f] == 2) d += (f & 1) ? bc.h[f] * area[f] : -bc.h[f] * area[f];
  lam[o] = d * mu[o];
}

// a[i] = v over a whole vector (scratch contents for the launch-shape tuner)
template <typename T>
__global__ void __launch_bounds__(256) k_fill_const(long long n, T* __restrict__ a, T v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
}

// dd of every interior cell (cell_coef's 13-term sum in the reference's order; 1 for masked
// cells), for the smoother.  One thread per interior cell.
template <typename T>
__global__ void __launch_bounds__(256) k_make_dd(OpParams<T> op, T* __restrict__ ddv) {
  const Geo& g = op.g;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > g.NX) return;
  const int o = g.off(i, j, k);
  const uint8_t* key = op.key;
  Coef<T> c;
  const bool has = cell_coef<T, false>(op, k, key[o], key[g.off(i - 1, j, k)], key[g.off(i + 1, j, k)],
                                       key[g.off(i, j - 1, k)], key[g.off(i, j + 1, k)], key[g.off(i, j, k - 1)],
                                       key[g.off(i, j, k + 1)], o, c);
  ddv[o] = has ? c.dd : T(1);
}

// *flag = 1 if the arrays a and b (n 16-byte words) differ anywhere.
__global__ void __launch_bounds__(256) k_bytes_differ(const uint4* __restrict__ a, const uint4* __restrict__ b,
                                                       long long n, int* flag) {
  int d = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const uint4 x = a[i], y = b[i];
    d |= (x.x != y.x) | (x.y != y.y) | (x.z != y.z) | (x.w != y.w);
  }
  if (__syncthreads_or(d) && threadIdx.x == 0) *flag = 1;
}

// Per interior cell, the 7 keys its stencil reads packed in one word: own key (byte 0) and the
// keys of its x-, x+, y-, y+, z-, z+ neighbours (bytes 1..6).  Guards and padding: 0.
__global__ void __launch_bounds__(256) k_make_nkeys(Geo g, const uint8_t* __restrict__ key,
                                                     unsigned long long* __restrict__ nk) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > g.NX) return;
  const int o = g.off(i, j, k);
  const int nb[6] = {g.off(i - 1, j, k), g.off(i + 1, j, k), g.off(i, j - 1, k),
                     g.off(i, j + 1, k), g.off(i, j, k - 1), g.off(i, j, k + 1)};
  unsigned long long w = key[o];
#pragma unroll
  for (int f = 0; f < 6; ++f) w |= (unsigned long long)key[nb[f]] << (8 * (f + 1));
  nk[o] = w;
}

// Stencil classes, step 1: every updated interior cell enters its (plane, 7 keys) pair into an
// open-addressing table of kClassSlots words (plane in the top byte; the own key's mask bit makes
// every entry non-zero).  At most kClassSlots probes per cell: a full table sets *overflow.
__device__ __forceinline__ unsigned class_hash(unsigned long long w) {
  return (unsigned)((w * 0x9E3779B97F4A7C15ull) >> (64 - 17)) & (kClassSlots - 1);
}
__device__ __forceinline__ unsigned long long class_word(const unsigned long long* nk, int o, int k) {
  return (nk[o] & 0x00ffffffffffffffull) | ((unsigned long long)k << 56);
}
__global__ void __launch_bounds__(256) k_class_insert(Geo g, const unsigned long long* __restrict__ nk,
                                                       unsigned long long* slots, int* overflow) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > g.NX) return;
  const int o = g.off(i, j, k);
  if (!(nk[o] & 0x80)) return;  // masked: never updated
  const unsigned long long w = class_word(nk, o, k);
  unsigned h = class_hash(w);
  for (int t = 0; t < kClassSlots; ++t) {
    const unsigned long long prev = atomicCAS(slots + h, 0ull, w);
    if (prev == 0ull || prev == w) return;
    h = (h + 1) & (kClassSlots - 1);
  }
  atomicExch(overflow, 1);
}

// Step 2 (after the host numbered the occupied slots): the class index of every cell; cells that
// are never updated (guards, masked cells, padding) keep kNoClass from the fill before.
__global__ void __launch_bounds__(256) k_class_assign(Geo g, const unsigned long long* __restrict__ nk,
                                                       const unsigned long long* __restrict__ slots,
                                                       const uint16_t* __restrict__ slot_class,
                                                       uint16_t* __restrict__ cls) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > g.NX) return;
  const int o = g.off(i, j, k);
  if (!(nk[o] & 0x80)) return;
  const unsigned long long w = class_word(nk, o, k);
  unsigned h = class_hash(w);
  for (int t = 0; t < kClassSlots; ++t) {
    const unsigned long long v = slots[h];
    if (v == w) {
      cls[o] = slot_class[h];
      return;
    }
    if (v == 0ull) return;  // not entered (cannot happen after a complete step 1)
    h = (h + 1) & (kClassSlots - 1);
  }
}

// Step 3: one table row per class from cell_coef on the class's (plane, keys) pair, with the
// grid taken as steady (a_p0 = 0: dd is then the sum of the 12 face terms, what a steady cell of
// the class gets), in the precision of the tables op points to.
template <typename T>
__global__ void __launch_bounds__(128) k_class_coef(OpParams<T> op, const unsigned long long* __restrict__ words,
                                                     int ncls, T* __restrict__ ctab) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncls) return;
  const unsigned long long w = words[c];
  const int k = (int)(w >> 56);
  op.steady = 1;
  Coef<T> cf;
  cell_coef<T, false>(op, k, (uint8_t)w, (uint8_t)(w >> 8), (uint8_t)(w >> 16), (uint8_t)(w >> 24),
                      (uint8_t)(w >> 32), (uint8_t)(w >> 40), (uint8_t)(w >> 48), 0, cf);
  T* t = ctab + 8 * (size_t)c;
  t[0] = cf.cxm;
  t[1] = cf.cxp;
  t[2] = cf.cym;
  t[3] = cf.cyp;
  t[4] = cf.czm;
  t[5] = cf.czp;
  t[6] = cf.dd;
  t[7] = T(0);
}

// ------------------------------------------------------------------------------------------
// Material keys.  Pass 1 collects the distinct lambda bit patterns into a small open-addressing
// table and validates the fields; pass 2 writes key = index | mask << 7 in the device layout
// (and rho*cp for transient grids).
// ------------------------------------------------------------------------------------------
enum FieldFlags { kFlagNonFinite = 1, kFlagMaskValue = 2, kFlagTooMany = 4 };

__device__ __forceinline__ unsigned slot_hash(unsigned long long b) {
  return (unsigned)((b * 0x9E3779B97F4A7C15ull) >> 56);
}

__global__ void k_collect_keys(Geo g, const double* __restrict__ lam, const double* __restrict__ mask,
                               const double* __restrict__ rho, const double* __restrict__ cp,
                               unsigned long long* __restrict__ slots, int* __restrict__ flags) {
  const long long n = (long long)g.MX * g.MY * g.MZ;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const double l = lam[c], m = mask[c];
    int f = 0;
    if (!isfinite(l) || !isfinite(m)) f |= kFlagNonFinite;
    if (!(m == 0.0 || m == 1.0)) f |= kFlagMaskValue;
    if (rho && !(isfinite(rho[c]) && isfinite(cp[c]))) f |= kFlagNonFinite;
    if (f) atomicOr(flags, f);
    if (!isfinite(l)) continue;
    const unsigned long long b = (unsigned long long)__double_as_longlong(l);
    unsigned h = slot_hash(b);
    for (int probe = 0; probe < kHashSlots; ++probe, h = (h + 1) & (kHashSlots - 1)) {
      unsigned long long cur = slots[h];
      if (cur == b) break;
      if (cur == ~0ull) {
        cur = atomicCAS(slots + h, ~0ull, b);
        if (cur == ~0ull || cur == b) break;
      }
      if (probe == kHashSlots - 1) atomicOr(flags, kFlagTooMany);
    }
  }
}

template <typename T>
__global__ void k_make_keys(Geo g, const double* __restrict__ lam, const double* __restrict__ mask,
                            const double* __restrict__ rho, const double* __restrict__ cp,
                            const unsigned long long* __restrict__ slots, const int* __restrict__ slot_index,
                            uint8_t* __restrict__ key, T* __restrict__ rc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= g.MX) return;
  const long long c = (long long)i + (long long)g.MX * ((long long)j + (long long)g.MY * k);
  const unsigned long long b = (unsigned long long)__double_as_longlong(lam[c]);
  unsigned h = slot_hash(b);
  int idx = 0;
  for (int probe = 0; probe < kHashSlots; ++probe, h = (h + 1) & (kHashSlots - 1)) {
    if (slots[h] == b) { idx = slot_index[h]; break; }
  }
  const long long o = g.off(i, j, k);
  key[o] = (uint8_t)(idx | (mask[c] == 1.0 ? 0x80 : 0));
  if (rc) rc[o] = (T)(rho[c] * cp[c]);
}

}  // namespace h2g

// h2g_multi.cuh -- PBiCGSTAB! (src/NonUniform.jl:248-350) for K right-hand sides on one operator.
//
// The batched workload's members of one grid size share the operator (the same geometry and
// materials); only their heat maps, and so b, differ.  A multi-RHS handle keeps K solution and
// Krylov vectors of each kind, stacked (vector r of right-hand side q at base + q*n), and K solver
// states.  Every stencil kernel computes a cell's coefficients once -- the packed key word, six
// table look-ups and dd, most of a cell update's instructions -- and applies them to R right-hand
// sides held by the same thread; blockIdx.z enumerates (group of R right-hand sides, plane).
//
// The per-cell arithmetic is that of the single-RHS kernels, and so are the block shapes and the
// reduction order: each right-hand side's dot products are summed per block and then over the
// blocks of its group in the order reduce_finish uses, and the elementwise update runs one grid row
// per right-hand side with the single solve's decomposition.  Every right-hand side therefore gets
// exactly the iterates, iteration count and bits of its lone solve.  A right-hand side that has
// stopped keeps taking part in the reductions' tickets with nothing to add, so that the per-group
// and global finishers always run; its vectors are no longer written.
#pragma once
#include "h2g_kernels.cuh"

namespace h2g {

constexpr int kMrR = 4;        // right-hand sides per thread
constexpr int kMrMax = 64;     // right-hand sides per handle

// Global control of a multi-RHS solve: the ticket of the per-RHS finishers of the update kernel
// and the WHILE-body pass count.
struct MultiCtl {
  unsigned int ticket;
  int passes;
  int maxItr;
  int nrhs;
};

__global__ void k_prime_mr(SolverState* st, MultiCtl* ctl, double tol, int maxItr, int K) {
  pdl_enter();
  const int q = threadIdx.x;
  if (q < K) {
    st[q].tol = tol;
    st[q].maxItr = maxItr;
    st[q].hist = nullptr;
    st[q].hist_len = 0;
    st[q].stop = 0;
    st[q].ticket = 0;
    st[q].passes = 0;
    st[q].div_limit = 0.0;
  }
  if (q == 0) {
    ctl->ticket = 0;
    ctl->passes = 0;
    ctl->maxItr = maxItr;
    ctl->nrhs = K;
  }
}

// Coefficients of cell ci at plane k: from its packed key word and the key tables (CL false) or
// from its stencil class (CL true); both give cell_coef's values.
template <bool CL>
__device__ __forceinline__ bool mr_coef(const OpParams<double>& op, int k, int ci, Coef<double>& c) {
  if constexpr (CL) {
    return class_coef<double>(op, __ldg(op.cls + ci), ci, c);
  } else {
    const unsigned long long w = __ldg(op.nkey + ci);
    return cell_coef<double, true>(op, k, (uint8_t)w, (uint8_t)(w >> 8), (uint8_t)(w >> 16), (uint8_t)(w >> 24),
                                   (uint8_t)(w >> 32), (uint8_t)(w >> 40), (uint8_t)(w >> 48), ci, c);
  }
}

// Sum of one right-hand side's partials [NV][nb] in reduce_finish's order, by the whole block.
template <int NV>
__device__ __forceinline__ void seg_sum(const double* __restrict__ part, int nb, double (&acc)[NV],
                                        double (*sm)[NV], int tid, int nthr) {
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int b0 = tid; b0 < nb; b0 += 8 * nthr) {
    double t[NV][8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int b = b0 + u * nthr;
#pragma unroll
      for (int q = 0; q < NV; ++q) t[q][u] = b < nb ? __ldcg(part + (size_t)q * nb + b) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
      for (int q = 0; q < NV; ++q) acc[q] += t[q][u];
  }
  block_sum<NV>(acc, sm, tid, nthr);
}

// Block partials of the R right-hand sides of group gq (values v[R][NV]) and, in the group's last
// block, their finishers.  Partials of right-hand side q: partials + q*NV*nbg, [NV][nbg].
template <int NV, int R>
__device__ __forceinline__ void group_finish(double (&v)[R][NV], double* __restrict__ partials, SolverState* st,
                                             int gq, int K, int nbg, int bid, const bool (&run)[R], int stage) {
  __shared__ double sm[32][R * NV];
  __shared__ double sm1[32][NV];
  __shared__ int am_last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  double f[R * NV];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int q = 0; q < NV; ++q) f[r * NV + q] = v[r][q];
  block_sum<R * NV>(f, sm, tid, nthr);
  SolverState* st0 = st + gq * R;
  if (tid == 0) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int qq = gq * R + r;
      if (qq >= K) break;
#pragma unroll
      for (int q = 0; q < NV; ++q) partials[(size_t)qq * NV * nbg + (size_t)q * nbg + bid] = f[r * NV + q];
    }
    __threadfence();
    const unsigned t = atomicAdd(&st0->ticket, 1u);
    am_last = (t == (unsigned)nbg - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int qq = gq * R + r;
    if (qq >= K) break;
    double acc[NV];
    seg_sum<NV>(partials + (size_t)qq * NV * nbg, nbg, acc, sm1, tid, nthr);
    if (tid == 0 && run[r]) finish_stage(stage, st + qq, acc[0], NV > 1 ? acc[NV > 1 ? 1 : 0] : 0.0);
  }
  if (tid == 0) st0->ticket = 0;
}

// CalcRK! for K right-hand sides: r = b - A th, r0 = r, (r,r) -> stage (kStageInit).
// Grid (gx, gy, NZ * G), block (32, kBY).
template <int R, bool CL>
__global__ void __launch_bounds__(kThreads) k_rk_mr(OpParams<double> op, double* __restrict__ r,
                                                     double* __restrict__ r0c, const double* __restrict__ th,
                                                     const double* __restrict__ b, SolverState* st,
                                                     double* __restrict__ partials, int stage, int K, long long n) {
  pdl_enter();
  const Geo& g = op.g;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int gq = blockIdx.z / g.NZ, k = 1 + blockIdx.z % g.NZ;
  const int nbg = gridDim.x * gridDim.y * g.NZ;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * (blockIdx.z % g.NZ));
  double v[R][1];
  bool run[R];
#pragma unroll
  for (int rr = 0; rr < R; ++rr) {
    v[rr][0] = 0.0;
    run[rr] = gq * R + rr < K;
  }
  if (j <= g.NY) {
    const bool pok = p < g.HN;
    const int r0 = g.row(0, j, k), r1 = r0 + g.HP;
    const int e0 = (1 + j + k) & 1;
    bool ok[2];
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      const int i = 2 * p + (e0 ^ col);
      ok[col] = pok && i >= 1 && i <= g.NX;
    }
    Coef<double> c[2];
    bool has[2];
#pragma unroll
    for (int col = 0; col < 2; ++col) has[col] = ok[col] && mr_coef<CL>(op, k, (col ? r1 : r0) + p, c[col]);
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      if (!run[rr]) continue;
      const long long qo = (long long)(gq * R + rr) * n;
      const double* thq = th + qo;
      Pair<double, double> P;
      load_pair<double, double, false>(g, thq, op.key, r0, p, pok, P);
      double xm0, xp0, xm1, xp1;
      int kd0, kd1, kd2, kd3;
      x_nbrs<double, true, double, false>(P.c1[1], 0, e0, lane, p, g.HN, thq, op.key, r1, xm0, xp0, kd0, kd1);
      x_nbrs<double, true, double, false>(P.c0[1], 0, e0 ^ 1, lane, p, g.HN, thq, op.key, r0, xm1, xp1, kd2, kd3);
#pragma unroll
      for (int col = 0; col < 2; ++col) {
        if (!ok[col]) continue;
        const int ci = (col ? r1 : r0) + p;
        double rs = 0.0;
        if (has[col]) {
          const double ss = col == 0 ? nb_sum(c[0], xp0, xm0, P.y1p, P.y1m, P.c1[2], P.c1[0])
                                     : nb_sum(c[1], xp1, xm1, P.y0p, P.y0m, P.c0[2], P.c0[0]);
          rs = sub(b[qo + ci], sub(ss, mul(c[col].dd, col == 0 ? P.c0[1] : P.c1[1])));
        }
        r[qo + ci] = rs;
        r0c[qo + ci] = rs;
        v[rr][0] += rs * rs;
      }
    }
  }
  group_finish<1, R>(v, partials, st, gq, K, nbg, bid, run, stage);
}

// k_rb_first for K right-hand sides (VM 1: p update; VM 2: s update), then colour 0 of the first
// sweep from zero.  Grid (gx, gy, NZ * G), block (32, kBY).
template <int VM, int R, bool CL>
__global__ void __launch_bounds__(kThreads) k_rb_first_mr(OpParams<double> op, double* __restrict__ xx,
                                                           double* __restrict__ v, const double* __restrict__ r,
                                                           const double* __restrict__ q, const SolverState* st, int K,
                                                           long long n) {
  pdl_enter();
  const Geo& g = op.g;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int gq = blockIdx.z / g.NZ, k = 1 + blockIdx.z % g.NZ;
  if (j > g.NY) return;
  (void)lane;
  const bool pok = p < g.HN;
  const int r0 = g.row(0, j, k), r1 = r0 + g.HP;
  const int e0 = (1 + j + k) & 1;
  bool ok[2];
#pragma unroll
  for (int col = 0; col < 2; ++col) {
    const int i = 2 * p + (e0 ^ col);
    ok[col] = pok && i >= 1 && i <= g.NX;
  }
  Coef<double> c;
  bool has = false;
  if (ok[0]) has = mr_coef<CL>(op, k, r0 + p, c);
#pragma unroll
  for (int rr = 0; rr < R; ++rr) {
    const int qq = gq * R + rr;
    if (qq >= K || st[qq].stop) continue;
    const long long qo = (long long)qq * n;
    double beta = 0.0, omg = 0.0, alpha = 0.0;
    int first = 0;
    if (VM == 1) {
      first = st[qq].first;
      beta = st[qq].beta;
      omg = st[qq].omega;
    } else {
      alpha = st[qq].alpha;
    }
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      if (!ok[col]) continue;
      const long long ci = qo + (col ? r1 : r0) + p;
      double bvx;
      if (VM == 1) bvx = first ? r[ci] : add(r[ci], mul(beta, sub(v[ci], mul(omg, q[ci]))));
      else bvx = add(mul(-alpha, q[ci]), r[ci]);
      v[ci] = bvx;
      double out = 0.0;
      if (col == 0 && has) {
        const double dp = sub(gs_div(sub(0.0, bvx), c.dd), 0.0);
        out = add(0.0, dp);
      }
      xx[ci] = out;
    }
  }
}

// One colour pass (rbsor_core!, omega = 1) for K right-hand sides; one plane per thread.
// Grid (gx, gy, NZ * G), block (32, kBY).
template <int R, bool CL>
__global__ void __launch_bounds__(kThreads) k_rb_pass_mr(OpParams<double> op, double* x, const double* __restrict__ bb,
                                                          int color, const SolverState* st, int K, long long n) {
  pdl_enter();
  const Geo& g = op.g;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int gq = blockIdx.z / g.NZ, k = 1 + blockIdx.z % g.NZ;
  if (j > g.NY) return;
  const int o = color ^ 1;
  const bool pok = p < g.HN;
  const int e = (1 + color + j + k) & 1, i = 2 * p + e;
  if (!(pok && i >= 1 && i <= g.NX)) return;
  const int ro = g.row(o, j, k), ac = g.row(color, j, k) + p;
  const int HP2 = 2 * g.HP, PL = (int)g.plane;
  Coef<double> c;
  if (!mr_coef<CL>(op, k, ac, c)) return;
  const int qx = p - 1 + 2 * e;  // the x-neighbour in the other column
  const bool qok = qx >= 0 && qx < g.HN;
#pragma unroll
  for (int rr = 0; rr < R; ++rr) {
    const int qq = gq * R + rr;
    if (qq >= K || st[qq].stop) continue;
    double* xq = x + (long long)qq * n;
    const double oc = ldro(xq + ro + p);
    const double other = qok ? ldro(xq + ro + qx) : 0.0;
    const double xm = e ? oc : other, xp = e ? other : oc;
    const double ym = ldro(xq + ro + p - HP2), yp = ldro(xq + ro + p + HP2);
    const double zm = ldro(xq + ro + p - PL), zp = ldro(xq + ro + p + PL);
    const double pp = xq[ac];
    const double ss = nb_sum(c, xp, xm, yp, ym, zp, zm);
    const double dp = sub(gs_div(sub(ss, bb[(long long)qq * n + ac]), c.dd), pp);
    xq[ac] = relax(pp, 1.0, dp);
  }
}

// CalcAX! with its dot products for K right-hand sides: y = A x; NDOT 1: (y, u); NDOT 2: (y,y),
// (y, w) -> stage.  Grid (gx, gy, NZ * G), block (32, kBY).
template <int NDOT, int R, bool CL>
__global__ void __launch_bounds__(kThreads, 2) k_ax_mr(OpParams<double> op, double* __restrict__ y,
                                                                  const double* __restrict__ x,
                                                                  const double* __restrict__ u,
                                                                  const double* __restrict__ w, SolverState* st,
                                                                  double* __restrict__ partials, int stage, int K,
                                                                  long long n) {
  pdl_enter();
  const Geo& g = op.g;
  const int lane = threadIdx.x, p = blockIdx.x * kBX + lane;
  const int j = 1 + blockIdx.y * kBY + threadIdx.y;
  const int gq = blockIdx.z / g.NZ, k = 1 + blockIdx.z % g.NZ;
  const int nbg = gridDim.x * gridDim.y * g.NZ;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * (blockIdx.z % g.NZ));
  double v[R][NDOT];
  bool run[R];
#pragma unroll
  for (int rr = 0; rr < R; ++rr) {
    const int qq = gq * R + rr;
    run[rr] = qq < K && !st[qq].stop;
#pragma unroll
    for (int d = 0; d < NDOT; ++d) v[rr][d] = 0.0;
  }
  if (j <= g.NY) {
    const bool pok = p < g.HN;
    const int r0 = g.row(0, j, k), r1 = r0 + g.HP;
    const int e0 = (1 + j + k) & 1;
    bool ok[2];
#pragma unroll
    for (int col = 0; col < 2; ++col) {
      const int i = 2 * p + (e0 ^ col);
      ok[col] = pok && i >= 1 && i <= g.NX;
    }
    Coef<double> c[2];
    bool has[2];
#pragma unroll
    for (int col = 0; col < 2; ++col) has[col] = ok[col] && mr_coef<CL>(op, k, (col ? r1 : r0) + p, c[col]);
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      if (!run[rr]) continue;
      const long long qo = (long long)(gq * R + rr) * n;
      const double* xq = x + qo;
      Pair<double, double> P;
      load_pair<double, double, false>(g, xq, op.key, r0, p, pok, P);
      double xm0, xp0, xm1, xp1;
      int kd0, kd1, kd2, kd3;
      x_nbrs<double, true, double, false>(P.c1[1], 0, e0, lane, p, g.HN, xq, op.key, r1, xm0, xp0, kd0, kd1);
      x_nbrs<double, true, double, false>(P.c0[1], 0, e0 ^ 1, lane, p, g.HN, xq, op.key, r0, xm1, xp1, kd2, kd3);
      double uu[2] = {0.0, 0.0}, ww[2] = {0.0, 0.0};
#pragma unroll
      for (int col = 0; col < 2; ++col) {
        if (!ok[col]) continue;
        const long long ci = qo + (col ? r1 : r0) + p;
        if (NDOT >= 1 && u) uu[col] = u[ci];
        if (NDOT >= 2) ww[col] = w[ci];
      }
#pragma unroll
      for (int col = 0; col < 2; ++col) {
        if (!ok[col]) continue;
        const long long ci = qo + (col ? r1 : r0) + p;
        double out = 0.0;
        if (has[col]) {
          if (col == 0) out = apply_a(c[0], P.c0[1], xp0, xm0, P.y1p, P.y1m, P.c1[2], P.c1[0]);
          else out = apply_a(c[1], P.c1[1], xp1, xm1, P.y0p, P.y0m, P.c0[2], P.c0[0]);
        }
        y[ci] = out;
        if (NDOT >= 1) v[rr][0] += out * (u ? uu[col] : out);
        if (NDOT >= 2) v[rr][NDOT - 1] += out * ww[col];
      }
    }
  }
  group_finish<NDOT, R>(v, partials, st, gq, K, nbg, bid, run, stage);
}

// BICG2! + Triad! + Fdot1/Fdot2 for K right-hand sides: grid (nb, K), block 256; row q of the grid
// is right-hand side q with the single solve's decomposition.  Each right-hand side's last block
// finishes its stage; the last of those sets the WHILE condition: continue while any right-hand
// side runs and the pass count is within maxItr + 1.
template <bool COND>
__global__ void __launch_bounds__(256) k_bicg_update_mr(long long n, double* __restrict__ x,
                                                         const double* __restrict__ ph, const double* __restrict__ sh,
                                                         double* __restrict__ r, const double* __restrict__ s,
                                                         const double* __restrict__ t, const double* __restrict__ r0,
                                                         SolverState* st, MultiCtl* ctl, double* __restrict__ partials,
                                                         cudaGraphConditionalHandle hc, int use_cond) {
  pdl_enter();
  __shared__ double sm[32][2];
  __shared__ int am_last;
  const int qq = blockIdx.y, K = gridDim.y, nb = gridDim.x;
  const int tid = threadIdx.x, nthr = blockDim.x;
  SolverState* sq = st + qq;
  const bool run = !sq->stop;
  const long long qo = (long long)qq * n;
  constexpr int V = 2;
  double v[2] = {0.0, 0.0};
  if (run) {
    const double alpha = sq->alpha, omega = sq->omega, nomega = -sq->omega;
    const long long nv = n / V;
    for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nv; b += (long long)gridDim.x * blockDim.x) {
      const long long o = qo + b * V;
      double a_ph[V], a_sh[V], a_s[V], a_t[V], a_r0[V], a_r[V];
      ldv<double, double, V>(ph + o, a_ph);
      ldv<double, double, V>(sh + o, a_sh);
      ld16(s + o, a_s);
      ld16(t + o, a_t);
      ld16(r0 + o, a_r0);
#pragma unroll
      for (int q = 0; q < V; ++q) {
        x[o + q] = add(x[o + q], add(mul(alpha, a_ph[q]), mul(omega, a_sh[q])));
        a_r[q] = add(mul(nomega, a_t[q]), a_s[q]);
        v[0] += a_r[q] * a_r[q];
        v[1] += a_r[q] * a_r0[q];
      }
      st16(r + o, a_r);
    }
  }
  block_sum<2>(v, sm, tid, nthr);
  double* part = partials + (size_t)qq * 2 * nb;
  if (tid == 0) {
    part[blockIdx.x] = v[0];
    part[nb + blockIdx.x] = v[1];
    __threadfence();
    const unsigned tk = atomicAdd(&sq->ticket, 1u);
    am_last = (tk == (unsigned)nb - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double acc[2];
  seg_sum<2>(part, nb, acc, sm, tid, nthr);
  if (tid == 0) {
    sq->ticket = 0;
    if (run) finish_stage(kStageUpdate, sq, acc[0], acc[1]);
    __threadfence();
    const unsigned g2 = atomicAdd(&ctl->ticket, 1u);
    if (g2 == (unsigned)K - 1) {  // the last right-hand side to finish this pass
      __threadfence();
      ctl->ticket = 0;
      ctl->passes += 1;
      int any = 0;
      for (int q = 0; q < K; ++q) any |= !((volatile SolverState*)st)[q].stop;
      if constexpr (COND) set_cond(hc, use_cond, any && ctl->passes <= ctl->maxItr + 1);
      else (void)any;
    }
  }
}

// any right-hand side still running (host-loop path without conditional nodes)
__global__ void k_any_running(const SolverState* st, int K, int* out) {
  int any = 0;
  for (int q = 0; q < K; ++q) any |= !st[q].stop;
  *out = any;
}

}  // namespace h2g

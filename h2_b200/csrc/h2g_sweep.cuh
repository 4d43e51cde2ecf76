// h2g_sweep.cuh -- one red-black Gauss-Seidel sweep (colour 0, then colour 1) in one launch.
//
// rbsor! (src/NonUniform.jl:936-957) runs colour 0 over the whole grid, then colour 1.  A colour-1
// cell needs the new values of its six colour-0 neighbours, so the unfused path launches one
// kernel per colour and reads x twice per sweep.  Here one launch does the whole sweep and reads
// x once:
//
//   * A block owns a tile of (positions x rows) of the colour-split layout and marches along z
//     over a chunk of planes [kA, kB].  At step s it updates colour 0 at plane s, then colour 1 at
//     plane s-1, whose colour-0 neighbours (planes s-2, s-1, s) are all new by then.
//   * Colour 0 is computed on the tile plus one position / row / plane of overlap on every side,
//     so that the owned colour-1 cells find all their neighbours inside the block; only owned
//     cells are written.  Within one colour every update is independent, so the redundant
//     overlap cells give exactly the bits their owner computes.
//   * The old x is read from one buffer and the sweep's result written to another (ping-pong):
//     overlapping blocks never see each other's new values.
//   * The planes of old x (both colours) and of the 1-byte keys are staged in a ring of shared
//     memory by TMA (cp.async.bulk.tensor, completion on an mbarrier), several planes ahead;
//     each thread keeps its own column's z-neighbours in registers (sliding windows) and takes
//     x/y-neighbours from shared memory.  b is read once per cell with plain loads issued a step
//     ahead.  dd is summed from the tables (no dd array: 8 bytes less per cell) or read.
//
// Per-cell arithmetic is that of rb_pass_column (h2g_kernels.cuh) with omega = 1, so results are
// bit-identical to two colour passes.  Every wait on the TMA barriers is bounded: a wait that
// runs out sets *err (and the solve's stop flag, reason kTimeout), drains the copies still in
// flight (again bounded) and returns.
#pragma once
#include <cuda.h>

#include "h2g_kernels.cuh"

namespace h2g {

constexpr int kSwTPX = 64;              // positions per block (threadIdx.x), incl. 1 overlap each side
constexpr int kSwTJ = 16;               // rows per block (threadIdx.y), incl. 1 overlap each side
constexpr int kSwStages = 5;            // ring of staged planes
constexpr int kSwRR = 2 * (kSwTJ + 2);  // half-rows per staged plane: rows r0-1 .. r0+TJ, 2 colours
constexpr int kSwWK = kSwTPX + 32;      // key box width in bytes (x start aligned to 16 bytes)
constexpr int kSwThreads = kSwTPX * kSwTJ;

template <typename T>
struct SwCfg {
  static constexpr int A = 16 / (int)sizeof(T);  // TMA x-coordinate alignment in elements
  static constexpr int WX = kSwTPX + 8;          // x box width in elements
  static constexpr int XBYTES = WX * kSwRR * (int)sizeof(T);
  static constexpr int KBYTES = kSwWK * kSwRR;
  static constexpr int STAGE = XBYTES + KBYTES;
  static constexpr int C0BYTES = 2 * kSwTJ * kSwTPX * (int)sizeof(T);
  static constexpr int BAR_OFF = kSwStages * STAGE + C0BYTES;
  static constexpr int SMEM = BAR_OFF + 8 * kSwStages + 16;
  static_assert(XBYTES % 128 == 0 && KBYTES % 128 == 0 && C0BYTES % 128 == 0, "128-byte aligned buffers");
};

// ---- mbarrier / TMA primitives (PTX) --------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false if the phase has not completed within `limit` clock cycles (limit <= 0:
// give up at once, without looking).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit) {
  if (limit <= 0) return false;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

__device__ __forceinline__ int align_down(int v, int a) { return v >= 0 ? v - v % a : -((-v + a - 1) / a) * a; }

// Coefficients of one unmasked cell from its own and its six neighbours' key bytes, from the
// interleaved table: `row` is the (plane k, own key) row, whose entry for a neighbour key byte nb
// holds the x, y, z- and z+ conductances side by side (one multiply-add and one load per face).
// dd is read (DDA) or summed in NonUniform.jl:501-502's order.  In a steady grid whose cell has six
// unmasked neighbours every convective term and a_p0 are +0, and adding +0 to the non-negative
// partial sum changes no bit, so dd is the sum of the six conductances; otherwise the full 13-term
// chain runs.
template <typename T, bool DDA>
__device__ __forceinline__ void sweep_coef(const OpParams<T>& op, const T* __restrict__ row, int k, uint32_t kxm,
                                           uint32_t kxp, uint32_t kym, uint32_t kyp, uint32_t kzm, uint32_t kzp,
                                           int ci, Coef<T>& c) {
  c.cxm = __ldg(row + 4 * kxm);
  c.cxp = __ldg(row + 4 * kxp);
  c.cym = __ldg(row + 4 * kym + 1);
  c.cyp = __ldg(row + 4 * kyp + 1);
  c.czm = __ldg(row + 4 * kzm + 2);
  c.czp = __ldg(row + 4 * kzp + 3);
  if constexpr (DDA) {
    c.dd = __ldg(op.ddv + ci);
    return;
  }
  T s = add(c.cxp, c.cxm);
  s = add(s, c.cyp);
  s = add(s, c.cym);
  s = add(s, c.czp);
  s = add(s, c.czm);
  if (op.steady && (kxm & kxp & kym & kyp & kzm & kzp & 0x80u)) {
    c.dd = s;
    return;
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
  s = add(s, vxp);
  s = add(s, vxm);
  s = add(s, vyp);
  s = add(s, vym);
  s = add(s, vzp);
  s = add(s, vzm);
  s = add(s, ap);
  c.dd = add(T(0), s);
}

// the (plane k, own key) row of the interleaved table
template <typename T>
__device__ __forceinline__ const T* coef_row(const OpParams<T>& op, int kP, uint32_t k0) {
  return op.tq + ((size_t)(kP + (int)(k0 & 0x7f)) << 10);
}

// Gauss-Seidel update of one cell with omega = 1 (NonUniform.jl:903-905): x + ((ss - b)/dd - x).
template <typename T, bool DDA>
__device__ __forceinline__ T sweep_update(const OpParams<T>& op, int k, int kP, uint32_t k0, uint32_t kxm,
                                          uint32_t kxp, uint32_t kym, uint32_t kyp, uint32_t kzm, uint32_t kzp, int ci,
                                          T pp, T b, T xm, T xp, T ym, T yp, T zm, T zp) {
  Coef<T> c;
  sweep_coef<T, DDA>(op, coef_row(op, kP, k0), k, kxm, kxp, kym, kyp, kzm, kzp, ci, c);
  const T ss = nb_sum(c, xp, xm, yp, ym, zp, zm);
  const T dp = sub(gs_div(sub(ss, b), c.dd), pp);
  return relax(pp, T(1), dp);
}

// Per-thread geometry of a sweep block, computed once: the thread's column (p, j), its offsets in
// the staged boxes and in the device layout, which of its two cells of a row are interior, and the
// ring slots of the planes the current step uses (advanced one plane per step).
struct SweepThread {
  int p, j, tx, ty;
  bool owned;
  bool ok_even, ok_odd;  // interior cell at i = 2p (even) / i = 2p + 1 (odd), row j interior
  int par;               // parity of colour 0 at plane 0: e0(s) = par ^ (s & 1)
  int g0;                // offset of colour 0 of (p, j) within a plane; colour 1 is + HP
  int c0off;             // this thread's entry of one plane of the colour-0 exchange buffer
  __device__ __forceinline__ bool in0(int s, int NZ) const {
    return s >= 1 && s <= NZ && ((par ^ (s & 1)) ? ok_odd : ok_even);
  }
  __device__ __forceinline__ bool in1(int s, int NZ) const {
    return s >= 1 && s <= NZ && ((par ^ (s & 1)) ? ok_even : ok_odd);
  }
};

__device__ __forceinline__ SweepThread sweep_thread(const Geo& g) {
  SweepThread t;
  t.tx = threadIdx.x;
  t.ty = threadIdx.y;
  const int q0 = (int)blockIdx.x * (kSwTPX - 2) - 1, r0 = (int)blockIdx.y * (kSwTJ - 2);
  t.p = q0 + t.tx;
  t.j = r0 + t.ty;
  t.owned = t.tx >= 1 && t.tx < kSwTPX - 1 && t.ty >= 1 && t.ty < kSwTJ - 1;
  const bool jin = t.j >= 1 && t.j <= g.NY && t.p >= 0;
  t.ok_even = jin && 2 * t.p >= 1 && 2 * t.p <= g.NX;
  t.ok_odd = jin && 2 * t.p + 1 <= g.NX;
  t.par = (1 + t.j) & 1;
  t.g0 = (t.j * 2) * g.HP + t.p;
  t.c0off = t.ty * kSwTPX + t.tx;
  return t;
}

__device__ __forceinline__ int next_slot(int q) { return q == kSwStages - 1 ? 0 : q + 1; }

// One sweep: xout = RB-GS sweep of the x that tmx maps, with right-hand side bb.
// Grid: (ceil(HI / (TPX-2)), ceil(NY / (TJ-2)), ceil(NZ / kc)); block (kSwTPX, kSwTJ); dynamic
// shared memory SwCfg<T>::SMEM.
template <typename T, bool DDA>
__global__ void __launch_bounds__(kSwThreads, 1)
    k_rb_sweep(OpParams<T> op, const __grid_constant__ CUtensorMap tmx, const __grid_constant__ CUtensorMap tmk,
               T* __restrict__ xout, const T* __restrict__ bb, int kc, SolverState* st, int* err,
               long long wait_limit) {
  using C = SwCfg<T>;
  pdl_enter();
  if (st && st->stop) return;
  extern __shared__ __align__(128) unsigned char sm[];
  const Geo& g = op.g;
  const SweepThread t = sweep_thread(g);
  const int tid = t.tx + kSwTPX * t.ty;
  const int q0 = (int)blockIdx.x * (kSwTPX - 2) - 1, r0 = (int)blockIdx.y * (kSwTJ - 2);
  const int kA = 1 + (int)blockIdx.z * kc, kB = min(kA + kc - 1, g.NZ);
  const int xs = align_down(q0 - 1, C::A), xk = align_down(q0 - 1, 16), ys = 2 * (r0 - 1);
  const int first = kA - 2, last = kB + 2;  // staged planes
  // this column's colour-0 / colour-1 entries in the staged boxes
  const int oX0 = (2 * (t.ty + 1)) * C::WX + (t.p - xs), oX1 = oX0 + C::WX;
  const int oK0 = (2 * (t.ty + 1)) * kSwWK + (t.p - xk), oK1 = oK0 + kSwWK;
  T* c0b = reinterpret_cast<T*>(sm + kSwStages * C::STAGE);
  volatile int* flag = reinterpret_cast<volatile int*>(sm + C::BAR_OFF + 8 * kSwStages);
  const uint32_t bar0 = smem_u32(sm + C::BAR_OFF);
  auto xbox = [&](int q) { return reinterpret_cast<const T*>(sm + q * C::STAGE); };
  auto kbox = [&](int q) { return reinterpret_cast<const uint8_t*>(sm + q * C::STAGE + C::XBYTES); };
  auto issue = [&](int plane, int q) {  // thread 0
    const uint32_t b = bar0 + 8u * q;
    mbar_expect_tx(b, (uint32_t)C::STAGE);
    tma_load_3d(smem_u32(sm + q * C::STAGE), &tmx, xs, ys, plane, b);
    tma_load_3d(smem_u32(sm + q * C::STAGE + C::XBYTES), &tmk, xk, ys, plane, b);
  };
  auto wait = [&](int plane) {  // thread 0, bounded
    const int u = plane - first;
    return mbar_wait_bounded(bar0 + 8u * (u % kSwStages), (uint32_t)((u / kSwStages) & 1), wait_limit);
  };

  int issued = first - 1, waited = first - 1;  // thread 0's bookkeeping
  if (tid == 0) {
    for (int q = 0; q < kSwStages; ++q) mbar_init(bar0 + 8u * q, 1);
    mbar_fence_init();
    *flag = 0;
    for (int pl = first; pl <= min(first + kSwStages - 2, last); ++pl) {
      issue(pl, pl - first);
      issued = pl;
    }
    if (wait(first)) waited = first;
    if (waited == first && wait(first + 1)) waited = first + 1;
    if (waited != first + 1) *flag = 1;
  }
  __syncthreads();
  bool abort = *flag != 0;

  // ring slots of planes s-1, s, s+1 and of the plane issued at this step (s+3)
  int qm = 0, q0s = 1, qp = 2, qi = 4;
  // windows along z of this column: colour-1 old values and keys at planes s-1, s, s+1; colour-0
  // new values and keys at planes s-2, s-1, s (after the shift at the top of step s)
  T c1v[3] = {T(0), T(0), T(0)}, c0v[3] = {T(0), T(0), T(0)};
  uint32_t c1k[3] = {0u, 0u, 0u}, c0k[3] = {0u, 0u, 0u};
  T b0 = T(0), b1 = T(0);
  int pofs = (kA - 1) * (int)g.plane;  // s * plane at the current step
  if (!abort) {
    c1v[1] = xbox(0)[oX1];
    c1k[1] = kbox(0)[oK1];
    c1v[2] = xbox(1)[oX1];
    c1k[2] = kbox(1)[oK1];
    if (t.in0(kA - 1, g.NZ)) b0 = __ldg(bb + pofs + t.g0);
  }
  for (int s = kA - 1; s <= kB + 1 && !abort; ++s, pofs += (int)g.plane) {
    if (tid == 0) {
      if (wait(s + 1)) waited = s + 1;
      else *flag = 1;
    }
    __syncthreads();  // step s-1 done everywhere; plane s+1 staged
    if (*flag) {
      abort = true;
      break;
    }
    if (tid == 0 && s + 3 <= last) {  // the slot of plane s-2 is free now
      issue(s + 3, qi);
      issued = s + 3;
    }
    const T* X0 = xbox(q0s);
    const uint8_t* K0 = kbox(q0s);
    const uint8_t* Km = kbox(qm);
    c1v[0] = c1v[1];
    c1v[1] = c1v[2];
    c1v[2] = xbox(qp)[oX1];
    c1k[0] = c1k[1];
    c1k[1] = c1k[2];
    c1k[2] = kbox(qp)[oK1];
    const bool mid = s >= kA && s <= kB;
    // right-hand sides of the next step, in flight during this one
    T nb0 = T(0), nb1 = T(0);
    if (s <= kB && t.in0(s + 1, g.NZ)) nb0 = __ldg(bb + pofs + (int)g.plane + t.g0);
    if (t.owned && mid && t.in1(s, g.NZ)) nb1 = __ldg(bb + pofs + t.g0 + g.HP);
    const int e0 = t.par ^ (s & 1);  // colour 0 at plane s sits at i = 2p + e0
    const int d0 = e0 ? 1 : -1;

    // phase A: colour 0 at plane s (tile and overlap)
    {
      const T pp = X0[oX0];
      const uint32_t k0 = K0[oK0];
      T nv = pp;
      const bool in = t.in0(s, g.NZ);
      if (in && (k0 & 0x80u)) {
        const T xo = X0[oX1 + d0];
        const uint32_t ko = K0[oK1 + d0];
        const T xm = e0 ? c1v[1] : xo, xp = e0 ? xo : c1v[1];
        const uint32_t kxm = e0 ? c1k[1] : ko, kxp = e0 ? ko : c1k[1];
        nv = sweep_update<T, DDA>(op, s, s * op.P, k0, kxm, kxp, K0[oK1 - 2 * kSwWK], K0[oK1 + 2 * kSwWK], c1k[0],
                                  c1k[2], pofs + t.g0, pp, b0, xm, xp, X0[oX1 - 2 * C::WX], X0[oX1 + 2 * C::WX],
                                  c1v[0], c1v[2]);
      }
      c0v[0] = c0v[1];
      c0v[1] = c0v[2];
      c0v[2] = nv;
      c0k[0] = c0k[1];
      c0k[1] = c0k[2];
      c0k[2] = k0;
      c0b[(s & 1) * (kSwTJ * kSwTPX) + t.c0off] = nv;
      if (t.owned && in && mid) xout[pofs + t.g0] = nv;
    }
    // phase B: colour 1 at plane s-1 (owned cells), its colour-0 neighbours from step s-1
    const int sb = s - 1;
    if (t.owned && sb >= kA) {
      const T pp = c1v[0];
      const uint32_t k1 = c1k[0];
      T nv = pp;
      const int pb = pofs - (int)g.plane;
      const bool in = t.in1(sb, g.NZ);
      if (in && (k1 & 0x80u)) {
        const int e1 = e0;  // colour 1 at plane s-1 sits at i = 2p + e0
        const int d1 = e1 ? 1 : -1;
        const T* Cr = c0b + (sb & 1) * (kSwTJ * kSwTPX) + t.c0off;
        const T xo = Cr[d1];
        const uint32_t ko = Km[oK0 + d1];
        const T xm = e1 ? c0v[1] : xo, xp = e1 ? xo : c0v[1];
        const uint32_t kxm = e1 ? c0k[1] : ko, kxp = e1 ? ko : c0k[1];
        nv = sweep_update<T, DDA>(op, sb, sb * op.P, k1, kxm, kxp, Km[oK0 - 2 * kSwWK], Km[oK0 + 2 * kSwWK], c0k[0],
                                  c0k[2], pb + t.g0 + g.HP, pp, b1, xm, xp, Cr[-kSwTPX], Cr[kSwTPX], c0v[0],
                                  c0v[2]);
      }
      if (in) xout[pb + t.g0 + g.HP] = nv;
    }
    b0 = nb0;
    b1 = nb1;
    qm = q0s;
    q0s = qp;
    qp = next_slot(qp);
    qi = next_slot(qi);
  }
  if (abort && tid == 0) {
    // a wait ran out: report it, then let the copies still in flight land before the block's
    // shared memory is released (bounded as well)
    if (err) atomicExch(err, 1);
    if (st) {
      st->stop = 1;
      st->reason = kTimeout;
    }
    for (int pl = waited + 1; pl <= issued; ++pl) {
      const int u = pl - first;
      mbar_wait_bounded(bar0 + 8u * (u % kSwStages), (uint32_t)((u / kSwStages) & 1), kDrainCycles);
    }
  }
}

// ------------------------------------------------------------------------------------------
// The first sweep of Preconditioner! fused with the Krylov update that makes its right-hand side
// (the work of k_rb_first and the first colour-1 pass in one launch).  x starts at zero
// (myfill!, NonUniform.jl:303/313), so colour 0 needs only bb and dd, and colour 1 the new colour-0
// values: no plane of x is read, only the key planes are staged.
//   VM 0: bb = vin (given);  VM 1: bb = r (first iteration) or r + beta*(vin - omega*q), written
//   to vout (BiCG1!, NonUniform.jl:296-301);  VM 2: bb = (-alpha)*q + r, written to vout
//   (Triad!, NonUniform.jl:310-311).
// Overlap cells compute bb from r, q and vin too, so vout must not be vin (the caller ping-pongs
// p between iterations).  bbT (when T != TV): the smoother's copy of bb in T, owned cells.  Every
// cell's arithmetic is that of k_rb_first and rb_pass_column, so the bits are the same.
// ------------------------------------------------------------------------------------------
template <typename T, typename TV, int VM>
__device__ __forceinline__ void first_load(const TV* vin, const TV* r, const TV* q, int ci, TV (&a)[3]) {
  a[0] = VM == 0 ? __ldg(vin + ci) : __ldg(r + ci);
  a[1] = VM == 1 ? __ldg(vin + ci) : TV(0);
  a[2] = VM != 0 ? __ldg(q + ci) : TV(0);
}
template <int VM, typename TV>
__device__ __forceinline__ TV first_bb(const TV (&a)[3], int first, TV beta, TV omg, TV alpha) {
  if (VM == 0) return a[0];
  if (VM == 1) return first ? a[0] : add(a[0], mul(beta, sub(a[1], mul(omg, a[2]))));
  return add(mul(-alpha, a[2]), a[0]);
}

template <typename T, typename TV, int VM, bool DDA>
__global__ void __launch_bounds__(kSwThreads, 1)
    k_rb_sweep_first(OpParams<T> op, const __grid_constant__ CUtensorMap tmk, T* __restrict__ xout,
                     TV* __restrict__ vout, const TV* __restrict__ vin, T* __restrict__ bbT,
                     const TV* __restrict__ r, const TV* __restrict__ q, int kc, SolverState* st, int* err,
                     long long wait_limit) {
  using C = SwCfg<T>;
  pdl_enter();
  if (st && st->stop) return;
  extern __shared__ __align__(128) unsigned char sm[];
  const Geo& g = op.g;
  const SweepThread t = sweep_thread(g);
  const int tid = t.tx + kSwTPX * t.ty;
  const int q0 = (int)blockIdx.x * (kSwTPX - 2) - 1, r0 = (int)blockIdx.y * (kSwTJ - 2);
  const int kA = 1 + (int)blockIdx.z * kc, kB = min(kA + kc - 1, g.NZ);
  const int xk = align_down(q0 - 1, 16), ys = 2 * (r0 - 1);
  const int first = kA - 2, last = kB + 2;
  const int oK0 = (2 * (t.ty + 1)) * kSwWK + (t.p - xk), oK1 = oK0 + kSwWK;
  // shared memory: kSwStages key planes, then the colour-0 exchange buffer, then the barriers
  constexpr int KOFF = kSwStages * C::KBYTES;
  T* c0b = reinterpret_cast<T*>(sm + KOFF);
  constexpr int BOFF = KOFF + C::C0BYTES;
  volatile int* flag = reinterpret_cast<volatile int*>(sm + BOFF + 8 * kSwStages);
  const uint32_t bar0 = smem_u32(sm + BOFF);
  auto kbox = [&](int qq) { return reinterpret_cast<const uint8_t*>(sm + qq * C::KBYTES); };
  auto issue = [&](int plane, int qq) {
    const uint32_t b = bar0 + 8u * qq;
    mbar_expect_tx(b, (uint32_t)C::KBYTES);
    tma_load_3d(smem_u32(sm + qq * C::KBYTES), &tmk, xk, ys, plane, b);
  };
  auto wait = [&](int plane) {
    const int u = plane - first;
    return mbar_wait_bounded(bar0 + 8u * (u % kSwStages), (uint32_t)((u / kSwStages) & 1), wait_limit);
  };
  int firstit = 0;
  TV beta = TV(0), omg = TV(0), alpha = TV(0);
  if (VM == 1) {
    firstit = st->first;
    beta = (TV)st->beta;
    omg = (TV)st->omega;
  } else if (VM == 2) {
    alpha = (TV)st->alpha;
  }

  int issued = first - 1, waited = first - 1;
  if (tid == 0) {
    for (int qq = 0; qq < kSwStages; ++qq) mbar_init(bar0 + 8u * qq, 1);
    mbar_fence_init();
    *flag = 0;
    for (int pl = first; pl <= min(first + kSwStages - 2, last); ++pl) {
      issue(pl, pl - first);
      issued = pl;
    }
    if (wait(first)) waited = first;
    if (waited == first && wait(first + 1)) waited = first + 1;
    if (waited != first + 1) *flag = 1;
  }
  __syncthreads();
  bool abort = *flag != 0;

  int qm = 0, q0s = 1, qp = 2, qi = 4;
  T c0v[3] = {T(0), T(0), T(0)};
  uint32_t c1k[3] = {0u, 0u, 0u}, c0k[3] = {0u, 0u, 0u};
  TV a0[3] = {TV(0), TV(0), TV(0)}, a1[3] = {TV(0), TV(0), TV(0)};  // raw operands of bb, a step ahead
  int pofs = (kA - 1) * (int)g.plane;
  if (!abort) {
    c1k[1] = kbox(0)[oK1];
    c1k[2] = kbox(1)[oK1];
    if (t.in0(kA - 1, g.NZ)) first_load<T, TV, VM>(vin, r, q, pofs + t.g0, a0);
  }
  for (int s = kA - 1; s <= kB + 1 && !abort; ++s, pofs += (int)g.plane) {
    if (tid == 0) {
      if (wait(s + 1)) waited = s + 1;
      else *flag = 1;
    }
    __syncthreads();
    if (*flag) {
      abort = true;
      break;
    }
    if (tid == 0 && s + 3 <= last) {
      issue(s + 3, qi);
      issued = s + 3;
    }
    const uint8_t* K0 = kbox(q0s);
    const uint8_t* Km = kbox(qm);
    c1k[0] = c1k[1];
    c1k[1] = c1k[2];
    c1k[2] = kbox(qp)[oK1];
    const bool mid = s >= kA && s <= kB;
    TV n0[3] = {TV(0), TV(0), TV(0)}, n1[3] = {TV(0), TV(0), TV(0)};
    if (s <= kB && t.in0(s + 1, g.NZ)) first_load<T, TV, VM>(vin, r, q, pofs + (int)g.plane + t.g0, n0);
    if (t.owned && mid && t.in1(s, g.NZ)) first_load<T, TV, VM>(vin, r, q, pofs + t.g0 + g.HP, n1);
    const int e0 = t.par ^ (s & 1);
    const int d0 = e0 ? 1 : -1;

    // phase A: colour 0 at plane s from x = 0: ((0 - bb)/dd - 0), then 0 + that
    {
      const uint32_t k0 = K0[oK0];
      T nv = T(0);
      const bool in = t.in0(s, g.NZ);
      if (in) {
        const TV bv = first_bb<VM>(a0, firstit, beta, omg, alpha);
        const T b = (T)bv;
        if (t.owned && mid) {
          if (VM != 0) vout[pofs + t.g0] = bv;
          if (bbT) bbT[pofs + t.g0] = b;
        }
        if (k0 & 0x80u) {
          const uint32_t ko = K0[oK1 + d0];
          const uint32_t kxm = e0 ? c1k[1] : ko, kxp = e0 ? ko : c1k[1];
          Coef<T> c;
          sweep_coef<T, DDA>(op, coef_row(op, s * op.P, k0), s, kxm, kxp, K0[oK1 - 2 * kSwWK], K0[oK1 + 2 * kSwWK],
                             c1k[0], c1k[2], pofs + t.g0, c);
          const T dp = sub(gs_div(sub(T(0), b), c.dd), T(0));
          nv = add(T(0), dp);
        }
      }
      c0v[0] = c0v[1];
      c0v[1] = c0v[2];
      c0v[2] = nv;
      c0k[0] = c0k[1];
      c0k[1] = c0k[2];
      c0k[2] = k0;
      c0b[(s & 1) * (kSwTJ * kSwTPX) + t.c0off] = nv;
      if (t.owned && in && mid) xout[pofs + t.g0] = nv;
    }
    // phase B: colour 1 at plane s-1 (owned) from x = 0
    const int sb = s - 1;
    if (t.owned && sb >= kA) {
      const uint32_t k1 = c1k[0];
      T nv = T(0);
      const int pb = pofs - (int)g.plane;
      const bool in = t.in1(sb, g.NZ);
      if (in) {
        const TV bv = first_bb<VM>(a1, firstit, beta, omg, alpha);
        const T b = (T)bv;
        if (VM != 0) vout[pb + t.g0 + g.HP] = bv;
        if (bbT) bbT[pb + t.g0 + g.HP] = b;
        if (k1 & 0x80u) {
          const int e1 = e0;  // colour 1 at plane s-1 sits at i = 2p + e0
          const int d1 = e1 ? 1 : -1;
          const T* Cr = c0b + (sb & 1) * (kSwTJ * kSwTPX) + t.c0off;
          const T xo = Cr[d1];
          const uint32_t ko = Km[oK0 + d1];
          const T xm = e1 ? c0v[1] : xo, xp = e1 ? xo : c0v[1];
          const uint32_t kxm = e1 ? c0k[1] : ko, kxp = e1 ? ko : c0k[1];
          nv = sweep_update<T, DDA>(op, sb, sb * op.P, k1, kxm, kxp, Km[oK0 - 2 * kSwWK], Km[oK0 + 2 * kSwWK],
                                    c0k[0], c0k[2], pb + t.g0 + g.HP, T(0), b, xm, xp, Cr[-kSwTPX], Cr[kSwTPX],
                                    c0v[0], c0v[2]);
        }
        xout[pb + t.g0 + g.HP] = nv;
      }
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      a0[u] = n0[u];
      a1[u] = n1[u];
    }
    qm = q0s;
    q0s = qp;
    qp = next_slot(qp);
    qi = next_slot(qi);
  }
  if (abort && tid == 0) {
    if (err) atomicExch(err, 1);
    if (st) {
      st->stop = 1;
      st->reason = kTimeout;
    }
    for (int pl = waited + 1; pl <= issued; ++pl) {
      const int u = pl - first;
      mbar_wait_bounded(bar0 + 8u * (u % kSwStages), (uint32_t)((u / kSwStages) & 1), kDrainCycles);
    }
  }
}

// dynamic shared memory of k_rb_sweep_first<T, ...>
template <typename T>
constexpr int sweep_first_smem() {
  return kSwStages * SwCfg<T>::KBYTES + SwCfg<T>::C0BYTES + 8 * kSwStages + 16;
}

}  // namespace h2g

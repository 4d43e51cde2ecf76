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

// Coefficients of one unmasked cell from its own and its six neighbours' key bytes: the table
// look-ups of cell_coef, and dd either read (DDA) or summed in NonUniform.jl:501-502's order.  In
// a steady grid whose cell has six unmasked neighbours every convective term and a_p0 are +0, and
// adding +0 to the non-negative partial sum changes no bit, so dd is the sum of the six
// conductances; otherwise the full 13-term chain runs.
template <typename T, bool DDA>
__device__ __forceinline__ void sweep_coef(const OpParams<T>& op, int k, uint32_t k0, uint32_t kxm, uint32_t kxp,
                                           uint32_t kym, uint32_t kyp, uint32_t kzm, uint32_t kzp, int ci,
                                           Coef<T>& c) {
  const int bx = (k * op.P + (int)(k0 & 0x7f)) << 8;
  c.cxm = __ldg(op.tx + (bx | kxm));
  c.cxp = __ldg(op.tx + (bx | kxp));
  c.cym = __ldg(op.ty + (bx | kym));
  c.cyp = __ldg(op.ty + (bx | kyp));
  c.czm = __ldg(op.tz + (bx | kzm));
  c.czp = __ldg(op.tz + ((bx + (op.P << 8)) | kzp));
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

// Gauss-Seidel update of one cell with omega = 1 (NonUniform.jl:903-905): x + ((ss - b)/dd - x).
template <typename T, bool DDA>
__device__ __forceinline__ T sweep_update(const OpParams<T>& op, int k, uint32_t k0, uint32_t kxm, uint32_t kxp,
                                          uint32_t kym, uint32_t kyp, uint32_t kzm, uint32_t kzp, int ci, T pp, T b,
                                          T xm, T xp, T ym, T yp, T zm, T zp) {
  Coef<T> c;
  sweep_coef<T, DDA>(op, k, k0, kxm, kxp, kym, kyp, kzm, kzp, ci, c);
  const T ss = nb_sum(c, xp, xm, yp, ym, zp, zm);
  const T dp = sub(gs_div(sub(ss, b), c.dd), pp);
  return relax(pp, T(1), dp);
}

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
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kSwTPX * ty;
  const int q0 = (int)blockIdx.x * (kSwTPX - 2) - 1, r0 = (int)blockIdx.y * (kSwTJ - 2);
  const int p = q0 + tx, j = r0 + ty;
  const int kA = 1 + (int)blockIdx.z * kc, kB = min(kA + kc - 1, g.NZ);
  const int xs = align_down(q0 - 1, C::A), xk = align_down(q0 - 1, 16), ys = 2 * (r0 - 1);
  const int first = kA - 2, last = kB + 2;  // staged planes
  const bool owned = tx >= 1 && tx < kSwTPX - 1 && ty >= 1 && ty < kSwTJ - 1;
  const bool jin = j >= 1 && j <= g.NY && p >= 0;
  const int cx = p - xs, ck = p - xk;  // this column in the x / key boxes
  const int rr0 = 2 * (ty + 1), rr1 = rr0 + 1;
  T* c0b = reinterpret_cast<T*>(sm + kSwStages * C::STAGE);
  volatile int* flag = reinterpret_cast<volatile int*>(sm + C::BAR_OFF + 8 * kSwStages);
  const uint32_t bar0 = smem_u32(sm + C::BAR_OFF);
  auto xbox = [&](int plane) {
    return reinterpret_cast<const T*>(sm + ((plane - first) % kSwStages) * C::STAGE);
  };
  auto kbox = [&](int plane) {
    return reinterpret_cast<const uint8_t*>(sm + ((plane - first) % kSwStages) * C::STAGE + C::XBYTES);
  };
  auto bar = [&](int plane) { return bar0 + 8u * (uint32_t)((plane - first) % kSwStages); };
  auto parity = [&](int plane) { return (uint32_t)(((plane - first) / kSwStages) & 1); };
  auto issue = [&](int plane) {  // thread 0
    const int q = (plane - first) % kSwStages;
    const uint32_t b = bar0 + 8u * q;
    mbar_expect_tx(b, (uint32_t)C::STAGE);
    tma_load_3d(smem_u32(sm + q * C::STAGE), &tmx, xs, ys, plane, b);
    tma_load_3d(smem_u32(sm + q * C::STAGE + C::XBYTES), &tmk, xk, ys, plane, b);
  };
  // colour-0 / colour-1 cells of this column at plane k, interior and inside the grid
  auto in0 = [&](int k) {
    const int i = 2 * p + ((1 + j + k) & 1);
    return jin && k >= 1 && k <= g.NZ && i >= 1 && i <= g.NX;
  };
  auto in1 = [&](int k) {
    const int i = 2 * p + ((j + k) & 1);
    return jin && k >= 1 && k <= g.NZ && i >= 1 && i <= g.NX;
  };
  auto off0 = [&](int k) { return g.row(0, j, k) + p; };
  auto off1 = [&](int k) { return g.row(1, j, k) + p; };

  int issued = first - 1, waited = first - 1;  // thread 0's bookkeeping
  if (tid == 0) {
    for (int q = 0; q < kSwStages; ++q) mbar_init(bar0 + 8u * q, 1);
    mbar_fence_init();
    *flag = 0;
    for (int pl = first; pl <= min(first + kSwStages - 2, last); ++pl) {
      issue(pl);
      issued = pl;
    }
    if (mbar_wait_bounded(bar(first), parity(first), wait_limit)) waited = first;
    if (waited == first && mbar_wait_bounded(bar(first + 1), parity(first + 1), wait_limit)) waited = first + 1;
    if (waited != first + 1) *flag = 1;
  }
  __syncthreads();
  bool abort = *flag != 0;

  // windows along z of this column: colour-1 old values and keys at planes s-1, s, s+1; colour-0
  // new values and keys at planes s-2, s-1, s (after the shift at the top of step s)
  T c1v[3] = {T(0), T(0), T(0)}, c0v[3] = {T(0), T(0), T(0)};
  uint32_t c1k[3] = {0u, 0u, 0u}, c0k[3] = {0u, 0u, 0u};
  T b0 = T(0), b1 = T(0);
  if (!abort) {
    c1v[1] = xbox(first)[rr1 * C::WX + cx];
    c1k[1] = kbox(first)[rr1 * kSwWK + ck];
    c1v[2] = xbox(first + 1)[rr1 * C::WX + cx];
    c1k[2] = kbox(first + 1)[rr1 * kSwWK + ck];
    if (in0(kA - 1)) b0 = __ldg(bb + off0(kA - 1));
  }
  for (int s = kA - 1; s <= kB + 1 && !abort; ++s) {
    if (tid == 0) {
      if (mbar_wait_bounded(bar(s + 1), parity(s + 1), wait_limit)) waited = s + 1;
      else *flag = 1;
    }
    __syncthreads();  // step s-1 done everywhere; plane s+1 staged
    if (*flag) {
      abort = true;
      break;
    }
    if (tid == 0 && s + 3 <= last) {  // the slot of plane s-2 is free now
      issue(s + 3);
      issued = s + 3;
    }
    const T* X0 = xbox(s);
    const uint8_t* K0 = kbox(s);
    const uint8_t* Km = kbox(s - 1);
    c1v[0] = c1v[1];
    c1v[1] = c1v[2];
    c1v[2] = xbox(s + 1)[rr1 * C::WX + cx];
    c1k[0] = c1k[1];
    c1k[1] = c1k[2];
    c1k[2] = kbox(s + 1)[rr1 * kSwWK + ck];
    // right-hand sides of the next step, in flight during this one
    const bool do1 = owned && s >= kA && s <= kB;  // phase B of the next step (plane s)
    T nb0 = T(0), nb1 = T(0);
    if (s <= kB && in0(s + 1)) nb0 = __ldg(bb + off0(s + 1));
    if (do1 && in1(s)) nb1 = __ldg(bb + off1(s));

    // phase A: colour 0 at plane s (tile and overlap)
    {
      const T pp = X0[rr0 * C::WX + cx];
      const uint32_t k0 = K0[rr0 * kSwWK + ck];
      T nv = pp;
      const bool in = in0(s);
      if (in && (k0 & 0x80u)) {
        const int e = (1 + j + s) & 1, d = e ? 1 : -1;
        const T xo = X0[rr1 * C::WX + cx + d];
        const uint32_t ko = K0[rr1 * kSwWK + ck + d];
        const T ym = X0[(rr1 - 2) * C::WX + cx], yp = X0[(rr1 + 2) * C::WX + cx];
        const uint32_t kym = K0[(rr1 - 2) * kSwWK + ck], kyp = K0[(rr1 + 2) * kSwWK + ck];
        const T xm = e ? c1v[1] : xo, xp = e ? xo : c1v[1];
        const uint32_t kxm = e ? c1k[1] : ko, kxp = e ? ko : c1k[1];
        nv = sweep_update<T, DDA>(op, s, k0, kxm, kxp, kym, kyp, c1k[0], c1k[2], off0(s), pp, b0, xm, xp, ym, yp,
                                  c1v[0], c1v[2]);
      }
      c0v[0] = c0v[1];
      c0v[1] = c0v[2];
      c0v[2] = nv;
      c0k[0] = c0k[1];
      c0k[1] = c0k[2];
      c0k[2] = k0;
      c0b[((s & 1) * kSwTJ + ty) * kSwTPX + tx] = nv;
      if (owned && in && s >= kA && s <= kB) xout[off0(s)] = nv;
    }
    // phase B: colour 1 at plane s-1 (owned cells), its colour-0 neighbours from step s-1
    const int sb = s - 1;
    if (owned && sb >= kA) {
      const T pp = c1v[0];
      const uint32_t k1 = c1k[0];
      T nv = pp;
      const bool in = in1(sb);
      if (in && (k1 & 0x80u)) {
        const int e = (j + sb) & 1, d = e ? 1 : -1;
        const T* Cr = c0b + ((sb & 1) * kSwTJ + ty) * kSwTPX + tx;
        const T xo = Cr[d];
        const uint32_t ko = Km[rr0 * kSwWK + ck + d];
        const T ym = Cr[-kSwTPX], yp = Cr[kSwTPX];
        const uint32_t kym = Km[(rr0 - 2) * kSwWK + ck], kyp = Km[(rr0 + 2) * kSwWK + ck];
        const T xm = e ? c0v[1] : xo, xp = e ? xo : c0v[1];
        const uint32_t kxm = e ? c0k[1] : ko, kxp = e ? ko : c0k[1];
        nv = sweep_update<T, DDA>(op, sb, k1, kxm, kxp, kym, kyp, c0k[0], c0k[2], off1(sb), pp, b1, xm, xp, ym, yp,
                                  c0v[0], c0v[2]);
      }
      if (in) xout[off1(sb)] = nv;
    }
    b0 = nb0;
    b1 = nb1;
  }
  if (abort && tid == 0) {
    // a wait ran out: report it, then let the copies still in flight land before the block's
    // shared memory is released (bounded as well)
    if (err) atomicExch(err, 1);
    if (st) {
      st->stop = 1;
      st->reason = kTimeout;
    }
    for (int pl = waited + 1; pl <= issued; ++pl) mbar_wait_bounded(bar(pl), parity(pl), kDrainCycles);
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
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kSwTPX * ty;
  const int q0 = (int)blockIdx.x * (kSwTPX - 2) - 1, r0 = (int)blockIdx.y * (kSwTJ - 2);
  const int p = q0 + tx, j = r0 + ty;
  const int kA = 1 + (int)blockIdx.z * kc, kB = min(kA + kc - 1, g.NZ);
  const int xk = align_down(q0 - 1, 16), ys = 2 * (r0 - 1);
  const int first = kA - 2, last = kB + 2;
  const bool owned = tx >= 1 && tx < kSwTPX - 1 && ty >= 1 && ty < kSwTJ - 1;
  const bool jin = j >= 1 && j <= g.NY && p >= 0;
  const int ck = p - xk;
  const int rr0 = 2 * (ty + 1), rr1 = rr0 + 1;
  // shared memory: kSwStages key planes, then the colour-0 exchange buffer, then the barriers
  constexpr int KOFF = kSwStages * C::KBYTES;
  T* c0b = reinterpret_cast<T*>(sm + KOFF);
  const int BOFF = KOFF + C::C0BYTES;
  volatile int* flag = reinterpret_cast<volatile int*>(sm + BOFF + 8 * kSwStages);
  const uint32_t bar0 = smem_u32(sm + BOFF);
  auto kbox = [&](int plane) {
    return reinterpret_cast<const uint8_t*>(sm + ((plane - first) % kSwStages) * C::KBYTES);
  };
  auto bar = [&](int plane) { return bar0 + 8u * (uint32_t)((plane - first) % kSwStages); };
  auto parity = [&](int plane) { return (uint32_t)(((plane - first) / kSwStages) & 1); };
  auto issue = [&](int plane) {
    const int qq = (plane - first) % kSwStages;
    const uint32_t b = bar0 + 8u * qq;
    mbar_expect_tx(b, (uint32_t)C::KBYTES);
    tma_load_3d(smem_u32(sm + qq * C::KBYTES), &tmk, xk, ys, plane, b);
  };
  auto in0 = [&](int k) {
    const int i = 2 * p + ((1 + j + k) & 1);
    return jin && k >= 1 && k <= g.NZ && i >= 1 && i <= g.NX;
  };
  auto in1 = [&](int k) {
    const int i = 2 * p + ((j + k) & 1);
    return jin && k >= 1 && k <= g.NZ && i >= 1 && i <= g.NX;
  };
  auto off0 = [&](int k) { return g.row(0, j, k) + p; };
  auto off1 = [&](int k) { return g.row(1, j, k) + p; };
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
      issue(pl);
      issued = pl;
    }
    if (mbar_wait_bounded(bar(first), parity(first), wait_limit)) waited = first;
    if (waited == first && mbar_wait_bounded(bar(first + 1), parity(first + 1), wait_limit)) waited = first + 1;
    if (waited != first + 1) *flag = 1;
  }
  __syncthreads();
  bool abort = *flag != 0;

  T c0v[3] = {T(0), T(0), T(0)};
  uint32_t c1k[3] = {0u, 0u, 0u}, c0k[3] = {0u, 0u, 0u};
  TV a0[3] = {TV(0), TV(0), TV(0)}, a1[3] = {TV(0), TV(0), TV(0)};  // raw operands of bb, a step ahead
  if (!abort) {
    c1k[1] = kbox(first)[rr1 * kSwWK + ck];
    c1k[2] = kbox(first + 1)[rr1 * kSwWK + ck];
    if (in0(kA - 1)) first_load<T, TV, VM>(vin, r, q, off0(kA - 1), a0);
  }
  for (int s = kA - 1; s <= kB + 1 && !abort; ++s) {
    if (tid == 0) {
      if (mbar_wait_bounded(bar(s + 1), parity(s + 1), wait_limit)) waited = s + 1;
      else *flag = 1;
    }
    __syncthreads();
    if (*flag) {
      abort = true;
      break;
    }
    if (tid == 0 && s + 3 <= last) {
      issue(s + 3);
      issued = s + 3;
    }
    const uint8_t* K0 = kbox(s);
    const uint8_t* Km = kbox(s - 1);
    c1k[0] = c1k[1];
    c1k[1] = c1k[2];
    c1k[2] = kbox(s + 1)[rr1 * kSwWK + ck];
    const bool do1 = owned && s >= kA && s <= kB;
    TV n0[3] = {TV(0), TV(0), TV(0)}, n1[3] = {TV(0), TV(0), TV(0)};
    if (s <= kB && in0(s + 1)) first_load<T, TV, VM>(vin, r, q, off0(s + 1), n0);
    if (do1 && in1(s)) first_load<T, TV, VM>(vin, r, q, off1(s), n1);

    // phase A: colour 0 at plane s from x = 0: ((0 - bb)/dd - 0), then 0 + that
    {
      const uint32_t k0 = K0[rr0 * kSwWK + ck];
      T nv = T(0);
      const bool in = in0(s);
      if (in) {
        const TV bv = first_bb<VM>(a0, firstit, beta, omg, alpha);
        const T b = (T)bv;
        if (owned && s >= kA && s <= kB) {
          if (VM != 0) vout[off0(s)] = bv;
          if (bbT) bbT[off0(s)] = b;
        }
        if (k0 & 0x80u) {
          const int e = (1 + j + s) & 1, d = e ? 1 : -1;
          const uint32_t ko = K0[rr1 * kSwWK + ck + d];
          const uint32_t kym = K0[(rr1 - 2) * kSwWK + ck], kyp = K0[(rr1 + 2) * kSwWK + ck];
          const uint32_t kxm = e ? c1k[1] : ko, kxp = e ? ko : c1k[1];
          Coef<T> c;
          sweep_coef<T, DDA>(op, s, k0, kxm, kxp, kym, kyp, c1k[0], c1k[2], off0(s), c);
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
      c0b[((s & 1) * kSwTJ + ty) * kSwTPX + tx] = nv;
      if (owned && in && s >= kA && s <= kB) xout[off0(s)] = nv;
    }
    // phase B: colour 1 at plane s-1 (owned) from x = 0
    const int sb = s - 1;
    if (owned && sb >= kA) {
      const uint32_t k1 = c1k[0];
      T nv = T(0);
      const bool in = in1(sb);
      if (in) {
        const TV bv = first_bb<VM>(a1, firstit, beta, omg, alpha);
        const T b = (T)bv;
        if (VM != 0) vout[off1(sb)] = bv;
        if (bbT) bbT[off1(sb)] = b;
        if (k1 & 0x80u) {
          const int e = (j + sb) & 1, d = e ? 1 : -1;
          const T* Cr = c0b + ((sb & 1) * kSwTJ + ty) * kSwTPX + tx;
          const T xo = Cr[d];
          const uint32_t ko = Km[rr0 * kSwWK + ck + d];
          const T ym = Cr[-kSwTPX], yp = Cr[kSwTPX];
          const uint32_t kym = Km[(rr0 - 2) * kSwWK + ck], kyp = Km[(rr0 + 2) * kSwWK + ck];
          const T xm = e ? c0v[1] : xo, xp = e ? xo : c0v[1];
          const uint32_t kxm = e ? c0k[1] : ko, kxp = e ? ko : c0k[1];
          nv = sweep_update<T, DDA>(op, sb, k1, kxm, kxp, kym, kyp, c0k[0], c0k[2], off1(sb), T(0), b, xm, xp, ym,
                                    yp, c0v[0], c0v[2]);
        }
        xout[off1(sb)] = nv;
      }
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      a0[u] = n0[u];
      a1[u] = n1[u];
    }
  }
  if (abort && tid == 0) {
    if (err) atomicExch(err, 1);
    if (st) {
      st->stop = 1;
      st->reason = kTimeout;
    }
    for (int pl = waited + 1; pl <= issued; ++pl) mbar_wait_bounded(bar(pl), parity(pl), kDrainCycles);
  }
}

// dynamic shared memory of k_rb_sweep_first<T, ...>
template <typename T>
constexpr int sweep_first_smem() {
  return kSwStages * SwCfg<T>::KBYTES + SwCfg<T>::C0BYTES + 8 * kSwStages + 16;
}

}  // namespace h2g

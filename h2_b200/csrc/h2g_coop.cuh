// h2g_coop.cuh -- Preconditioner! (src/NonUniform.jl:531-559) as one cooperative launch.
//
// The colour-pass path runs the preconditioner as 10 launches: the first pass (fused with the
// Krylov update that makes its right-hand side) and 9 colour passes.  Here one launch does all
// ten, with a grid-wide barrier between consecutive passes.  Its grid is as many blocks as fit on
// the device at once (a cooperative launch refuses more), so every block can reach every barrier.
// A block walks the blocks of the colour-pass grid ("tiles", 32 positions x kBY rows x NP
// planes) with a stride of the grid size and runs the same per-cell code as the separate
// launches, so the result is bit-identical.  Reads of vectors written in the same launch (x, and
// the right-hand side written by the first pass) take the coherent load path.
//
// Every barrier wait is bounded: a block that has waited `limit` clock cycles sets *err and the
// solve's stop flag (reason kTimeout), and any block that finds *err set leaves the launch.
#pragma once
#include "h2g_kernels.cuh"

namespace h2g {

// Arrival count and generation of the grid barrier; count returns to 0 after every barrier.
struct GridBar {
  unsigned int count;
  unsigned int gen;
};

__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// All blocks of the grid meet here.  Returns false (in every thread of the block) when the
// barrier gave up: this block's wait ran out (it then sets *err and stops the solve) or another
// block's did.  st (may be null) receives the stop.  One thread per block arrives and polls; it
// polls with relaxed loads (which leave the L1 of the SM's other blocks alone) and pauses between
// polls, and a single fence after the wait orders the block's later loads after every block's
// writes.
__device__ __forceinline__ bool grid_barrier(GridBar* bar, unsigned int nblocks, long long limit, int* err,
                                             SolverState* st) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    int good = 1;
    // the generation is read before arriving: it cannot advance until this block has arrived
    const unsigned int g = ld_relaxed_u32(&bar->gen);
    __threadfence();  // this block's writes (ordered before by the block barrier) become visible
    const unsigned int old = atomicAdd(&bar->count, 1u);
    if (old == nblocks - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      const long long t0 = clock64();
      while (ld_relaxed_u32(&bar->gen) == g) {
        if (ld_relaxed_s32(err)) {
          good = 0;
          break;
        }
        if (clock64() - t0 > limit) {
          atomicExch(err, 1);
          if (st) {
            st->stop = 1;
            st->reason = kTimeout;
          }
          good = 0;
          break;
        }
        __nanosleep(32);
      }
      __threadfence();
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// The tiles t = first, first + stride, ... of a gx x gy x gz grid of tiles (x fastest), walked
// without a division per step: the stride is split into its x, y and z parts once, and each step
// adds them with carries.
struct TileWalk {
  int bx, by, bz;  // current tile
  int sx, sy, sz;  // stride split into its x, y, z parts
  int gx, gy, gz;
  __device__ __forceinline__ TileWalk(int first, int stride, int gx_, int gy_, int gz_) : gx(gx_), gy(gy_), gz(gz_) {
    bx = first % gx;
    by = (first / gx) % gy;
    bz = first / (gx * gy);
    sx = stride % gx;
    sy = (stride / gx) % gy;
    sz = stride / (gx * gy);
  }
  __device__ __forceinline__ bool valid() const { return bz < gz; }
  __device__ __forceinline__ void next() {
    bx += sx;
    int c = bx >= gx;
    bx -= c ? gx : 0;
    by += sy + c;
    c = by >= gy;
    by -= c ? gy : 0;
    bz += sz + c;
  }
};

// Preconditioner! from xx = 0 (VM as in k_rb_first: 0 takes the right-hand side v as given, 1
// makes p = r + beta (p - omega q) in v, 2 makes s = r - alpha q in v), then the remaining 9
// colour passes on xx with right-hand side v.
// Tiles of the first pass: the first_grid blocks (32 x kBY columns of one plane); of the colour
// passes: the rb_grid blocks with NP planes per thread.  Block (32, kBY).
template <int VM, int NP, int DDM>
__global__ void __launch_bounds__(kThreads, H2G_MINB)
    k_precond_coop(OpParams<double> op, double* xx, double* v, const double* __restrict__ r,
                   const double* __restrict__ q, SolverState* st, GridBar* bar, int* err, long long limit) {
  if ((st && st->stop) || ld_relaxed_s32(err)) return;  // the same for every block of the launch
  const Geo& g = op.g;
  const int lane = threadIdx.x, ty = threadIdx.y;
  const unsigned int nblocks = gridDim.x;
  const int gx = (g.HN + kBX - 1) / kBX, gy = (g.NY + kBY - 1) / kBY;
  // first pass, fused with the Krylov update
  for (TileWalk w(blockIdx.x, nblocks, gx, gy, g.NZ); w.valid(); w.next()) {
    const int p = w.bx * kBX + lane, j = 1 + w.by * kBY + ty, k = 1 + w.bz;
    if (j <= g.NY) rb_first_column<double, double, VM, DDM == 2>(op, xx, v, nullptr, r, q, st, 0, lane, p, j, k);
  }
  const TileWalk w0(blockIdx.x, nblocks, gx, gy, (g.NZ + NP - 1) / NP);
  for (int pass = 1; pass < 2 * kSweeps; ++pass) {
    if (!grid_barrier(bar, nblocks, limit, err, st)) return;
    const int color = pass & 1;
    for (TileWalk w = w0; w.valid(); w.next()) {
      const int p = w.bx * kBX + lane, j = 1 + w.by * kBY + ty, k0 = 1 + NP * w.bz;
      if (j <= g.NY) rb_pass_column<double, false, NP, DDM, false>(op, xx, v, color, 1.0, lane, p, j, k0);
    }
  }
}

}  // namespace h2g

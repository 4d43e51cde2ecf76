// h2g_model.cu -- the reference's Mode-3 IC-stack model on the GPU: Z grid (src/Zcoord.jl:88-166),
// pitch rounding (src/heat3ds.jl:197-200) and the material-ID fill fillID! (src/modelA.jl:148-556).
//
// Compiled with -fmad=false: every expression is evaluated with one rounding per operation in
// the reference's order, so the ID field is bit-identical to the reference's.
//
// fillID! visits shapes in a fixed order and only fills cells whose ID is still 0, so the shapes
// run one launch after another; within a shape every candidate cell is independent:
//   rectangles (power grids, plates): one thread per candidate cell (is_included_rect);
//   cylinders (TSVs): one block per candidate cell; the 50^3-sample test of is_included_cyl
//     is a conjunction of an (x,y) test and a z test, so the count is
//     #{(i,j): r2 <= r^2} * #{k: zmin <= z <= zmax} -- exactly the triple loop's count;
//   spheres (solder bumps): one block per candidate cell; the sample coordinates are built by
//     the reference's running sums (x += dx), the squared distance as ((ex^2 + ey^2) + ez^2),
//     and the 125000 comparisons are split over the block.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/h2g.h"

namespace h2gm {

// src/modelA.jl:10-30
constexpr double pg_dpth = 0.005e-3;
constexpr double s_dpth = 0.1e-3;
constexpr double d_ufill = 0.05e-3;
constexpr double r_bump = 0.03e-3;
constexpr double r_tsv = 0.02e-3;
constexpr double h_tsv = 0.1e-3;
constexpr double zm12 = 0.6e-3, zm11 = 0.55e-3, zm10 = 0.5e-3, zm9 = zm10 - pg_dpth, zm8 = 0.4e-3,
                 zm7 = 0.35e-3, zm6 = zm7 - pg_dpth, zm5 = 0.25e-3, zm4 = 0.2e-3, zm3 = zm4 - pg_dpth,
                 zm2 = 0.1e-3, zm1 = 0.05e-3, zm0 = 0.0;

constexpr int kSamples = 50;

struct Box {  // candidate cells, 1-based inclusive
  long i0, i1, j0, j1, k0, k1;
};

static long chk_idx(long i, long nx) { return i < 1 ? 1 : (i > nx ? nx : i); }
static long find_i(double x, double dx, long nx) { return chk_idx((long)floor((x - 0.0) / dx + 1.5), nx); }
static long find_k(const std::vector<double>& Z, double zc, long nz) {
  const double eps_tol = 1e-12;
  if (zc < Z[0] - eps_tol || zc > Z[nz - 1] + eps_tol) return -1;
  for (long k = 1; k <= nz - 1; ++k)
    if (Z[k - 1] <= zc && zc < Z[k]) return k;
  if (fabs(zc - Z[nz - 1]) < eps_tol) return nz - 1;
  return -1;
}

struct Ctx {
  int MX, MY, MZ;
  double dx, dy;
  const double* Z;  // device, MZ+1 faces (genZ! "Z")
  uint8_t* ID;      // device, column-major (MX,MY,MZ)
};

__device__ __forceinline__ void cell_box(const Ctx& c, long i, long j, long k, double* lo, double* hi) {
  lo[0] = 0.0 + c.dx * (double)(i - 1);
  lo[1] = 0.0 + c.dy * (double)(j - 1);
  lo[2] = c.Z[k - 1];
  hi[0] = lo[0] + c.dx;
  hi[1] = lo[1] + c.dy;
  hi[2] = c.Z[k];
}

__device__ __forceinline__ long long fidx(const Ctx& c, long i, long j, long k) {
  return (long long)(i - 1) + (long long)c.MX * ((long long)(j - 1) + (long long)c.MY * (k - 1));
}

// is_included_rect, modelA.jl:228-245
__device__ bool included_rect(const double* a1, const double* a2, const double* b1, const double* b2) {
  const double volA = fabs((a2[0] - a1[0]) * (a2[1] - a1[1]) * (a2[2] - a1[2]));
  double ov[3];
  for (int d = 0; d < 3; ++d) {
    const double alo = fmin(a1[d], a2[d]), ahi = fmax(a1[d], a2[d]);
    const double blo = fmin(b1[d], b2[d]), bhi = fmax(b1[d], b2[d]);
    ov[d] = fmax(0.0, fmin(ahi, bhi) - fmax(alo, blo));
  }
  const double overlap_vol = ov[0] * ov[1] * ov[2];
  return overlap_vol >= 0.5 * volA;
}

__global__ void k_fill_rect(Ctx c, Box bx, double bx0, double by0, double bz0, double bx1, double by1, double bz1,
                            uint8_t id) {
  const long ni = bx.i1 - bx.i0 + 1, nj = bx.j1 - bx.j0 + 1, nk = bx.k1 - bx.k0 + 1;
  const long long n = (long long)ni * nj * nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long i = bx.i0 + (long)(t % ni), j = bx.j0 + (long)((t / ni) % nj), k = bx.k0 + (long)(t / (ni * nj));
    double lo[3], hi[3];
    cell_box(c, i, j, k, lo, hi);
    const double d1[3] = {bx0, by0, bz0}, d2[3] = {bx1, by1, bz1};
    if (included_rect(lo, hi, d1, d2)) {
      const long long o = fidx(c, i, j, k);
      if (c.ID[o] == 0) c.ID[o] = id;
    }
  }
}

__device__ __forceinline__ int block_count(int v, int* sm) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sm[w] = v;
  __syncthreads();
  int tot = 0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x + 31) / 32; ++q) tot += sm[q];
  return tot;
}

// is_included_cyl, modelA.jl:254-282 (one block per candidate cell)
__global__ void k_fill_cyl(Ctx c, Box bx, double cx, double cy, double cyl_r, double zmin, double zmax, uint8_t id) {
  __shared__ int sm[32];
  const long ni = bx.i1 - bx.i0 + 1, nj = bx.j1 - bx.j0 + 1;
  const long long t = blockIdx.x;
  const long i = bx.i0 + (long)(t % ni), j = bx.j0 + (long)((t / ni) % nj), k = bx.k0 + (long)(t / (ni * nj));
  const long long o = fidx(c, i, j, k);
  if (c.ID[o] != 0) return;  // (0 == ID[i,j,k]) && ... is evaluated first
  double lo[3], hi[3];
  cell_box(c, i, j, k, lo, hi);
  const double xlo = fmin(lo[0], hi[0]), ylo = fmin(lo[1], hi[1]), zlo = fmin(lo[2], hi[2]);
  const double xhi = fmax(lo[0], hi[0]), yhi = fmax(lo[1], hi[1]), zhi = fmax(lo[2], hi[2]);
  const double volA = (xhi - xlo) * (yhi - ylo) * (zhi - zlo);
  const double rr = cyl_r * cyl_r;
  int nxy = 0, nz = 0;
  for (int s = threadIdx.x; s < kSamples * kSamples; s += blockDim.x) {
    const int a = s / kSamples + 1, b = s % kSamples + 1;
    const double x = xlo + ((double)a - 0.5) * (xhi - xlo) / (double)kSamples;
    const double y = ylo + ((double)b - 0.5) * (yhi - ylo) / (double)kSamples;
    const double ex = x - cx, ey = y - cy;
    const double r2 = ex * ex + ey * ey;
    nxy += (r2 <= rr);
  }
  for (int s = threadIdx.x; s < kSamples; s += blockDim.x) {
    const double z = zlo + ((double)(s + 1) - 0.5) * (zhi - zlo) / (double)kSamples;
    nz += (zmin <= z && z <= zmax);
  }
  const int cxy = block_count(nxy, sm);
  __syncthreads();
  const int cz = block_count(nz, sm);
  if (threadIdx.x == 0) {
    const long inside = (long)cxy * cz;
    const long total = (long)kSamples * kSamples * kSamples;
    const double overlap_vol = volA * (double)inside / (double)total;
    if (overlap_vol >= 0.5 * volA) c.ID[o] = id;
  }
}

// is_included_sph, modelA.jl:300-347 (one block per candidate cell)
__global__ void k_fill_sph(Ctx c, Box bx, double cx, double cy, double cz, double radius, uint8_t id) {
  __shared__ double xs[kSamples], ys[kSamples], ezz[kSamples];
  __shared__ double exy[kSamples * kSamples];
  __shared__ int sm[32];
  __shared__ int all_inside;
  const long ni = bx.i1 - bx.i0 + 1, nj = bx.j1 - bx.j0 + 1;
  const long long t = blockIdx.x;
  const long i = bx.i0 + (long)(t % ni), j = bx.j0 + (long)((t / ni) % nj), k = bx.k0 + (long)(t / (ni * nj));
  const long long o = fidx(c, i, j, k);
  if (c.ID[o] != 0) return;
  double lo[3], hi[3];
  cell_box(c, i, j, k, lo, hi);
  const double xlo = fmin(lo[0], hi[0]), ylo = fmin(lo[1], hi[1]), zlo = fmin(lo[2], hi[2]);
  const double xhi = fmax(lo[0], hi[0]), yhi = fmax(lo[1], hi[1]), zhi = fmax(lo[2], hi[2]);
  const double volA = (xhi - xlo) * (yhi - ylo) * (zhi - zlo);
  if (volA <= 0) return;
  const double r2 = radius * radius;
  if (threadIdx.x == 0) {
    const double cxs[2] = {xlo, xhi}, cys[2] = {ylo, yhi}, czs[2] = {zlo, zhi};
    int all = 1;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 2; ++d) {
          const double ex = cxs[a] - cx, ey = cys[b] - cy, ez = czs[d] - cz;
          if (!(ex * ex + ey * ey + ez * ez <= r2)) all = 0;
        }
    all_inside = all;
    // running sums of the reference's sampling loops
    const double dx = (xhi - xlo) / (double)kSamples, dy = (yhi - ylo) / (double)kSamples;
    const double dz = (zhi - zlo) / (double)kSamples;
    double x = xlo + dx / 2.0;
    for (int q = 0; q < kSamples; ++q) { xs[q] = x; x += dx; }
    double y = ylo + dy / 2.0;
    for (int q = 0; q < kSamples; ++q) { ys[q] = y; y += dy; }
    double z = zlo + dz / 2.0;
    for (int q = 0; q < kSamples; ++q) { const double ez = z - cz; ezz[q] = ez * ez; z += dz; }
  }
  __syncthreads();
  if (all_inside) {
    if (threadIdx.x == 0) c.ID[o] = id;
    return;
  }
  for (int s = threadIdx.x; s < kSamples * kSamples; s += blockDim.x) {
    const double ex = xs[s / kSamples] - cx, ey = ys[s % kSamples] - cy;
    exy[s] = ex * ex + ey * ey;
  }
  __syncthreads();
  int cnt = 0;
  for (int s = threadIdx.x; s < kSamples * kSamples * kSamples; s += blockDim.x) {
    const int ab = s / kSamples, q = s % kSamples;
    cnt += (exy[ab] + ezz[q] <= r2);
  }
  const int inside = block_count(cnt, sm);
  if (threadIdx.x == 0) {
    const long total = (long)kSamples * kSamples * kSamples;
    const double overlap_vol_est = volA * ((double)inside / (double)total);
    if (overlap_vol_est >= 0.5 * volA) c.ID[o] = id;
  }
}

__global__ void k_fill_resin(uint8_t* ID, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    if (ID[t] == 0) ID[t] = 6;
}

static void zcase2(double* Z) {  // Zcoord.jl:88-124
  const double p = 0.005e-3;
  const double v[31] = {zm0,     zm0 + p, zm1 - p, zm1,     zm1 + p, zm2 - p, zm2,     zm2 + p, zm3 - p, zm3,     zm4,
                        zm4 + p, zm5 - p, zm5,     zm5 + p, zm6 - p, zm6,     zm7,     zm7 + p, zm8 - p, zm8,     zm8 + p,
                        zm9 - p, zm9,     zm10,    zm10 + p, zm11 - p, zm11,  zm11 + p, zm12 - p, zm12};
  memcpy(Z, v, sizeof v);
}

}  // namespace h2gm

extern "C" {

int h2g_model_zgrid(int NZ, double* Z, double* ZC, double* dZ) {
  if (NZ < 30 || NZ % 30 != 0 || !Z || !ZC || !dZ) return H2G_BAD_ARG;
  const int m = NZ / 30;
  double base[31];
  h2gm::zcase2(base);
  std::vector<double> zf(NZ + 1);
  for (int c = 0; c < 30; ++c)
    for (int s = 0; s < m; ++s)
      zf[c * m + s] = (m == 1 || s == 0) ? base[c] : base[c] + ((base[c + 1] - base[c]) * (double)s) / (double)m;
  zf[NZ] = base[30];
  for (int k = 1; k <= NZ; ++k) dZ[k] = zf[k] - zf[k - 1];  // Zcoord.jl:137-143
  dZ[0] = dZ[1];
  dZ[NZ + 1] = dZ[NZ];
  ZC[0] = zf[0];  // Zcoord.jl:146-156
  ZC[NZ + 1] = zf[NZ];
  for (int k = 1; k <= NZ; ++k) ZC[k] = (zf[k] + zf[k - 1]) * 0.5;
  for (int k = 0; k <= NZ; ++k) Z[k + 1] = zf[k];  // Zcoord.jl:160-163
  Z[0] = 2.0 * zf[0] - zf[1];
  Z[NZ + 2] = 2.0 * zf[NZ] - zf[NZ - 1];
  return H2G_OK;
}

double h2g_model_pitch(int N) {  // round(1.2e-3/N, digits=8), heat3ds.jl:197-200
  const double x = 1.2e-3 / (double)N;
  const double y = rint(x * 1e8) / 1e8;
  return std::isfinite(y) ? y : x;
}

// fillID! (modelA.jl:545-556) for an (NX+2, NY+2, NZ+2) grid; ID is a host array, column-major.
int h2g_model_fill_id(int NX, int NY, int NZ, uint8_t* ID) {
  using namespace h2gm;
  if (NX < 1 || NY < 1 || !ID) return H2G_BAD_ARG;
  const int MX = NX + 2, MY = NY + 2, MZ = NZ + 2;
  std::vector<double> Z(NZ + 3), ZC(NZ + 2), dZ(NZ + 2);
  if (h2g_model_zgrid(NZ, Z.data(), ZC.data(), dZ.data())) return H2G_BAD_ARG;
  const double dx = h2g_model_pitch(NX), dy = h2g_model_pitch(NY);
  const long long n = (long long)MX * MY * MZ;
  Ctx c{MX, MY, MZ, dx, dy, nullptr, nullptr};
  double* dZf = nullptr;
  uint8_t* dID = nullptr;
  int rc = H2G_OK;
  if (cudaMalloc(&dZf, sizeof(double) * Z.size()) != cudaSuccess || cudaMalloc(&dID, (size_t)n) != cudaSuccess) {
    rc = H2G_CUDA_ERROR;
  }
  if (!rc && (cudaMemcpy(dZf, Z.data(), sizeof(double) * Z.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaMemset(dID, 0, (size_t)n) != cudaSuccess))
    rc = H2G_CUDA_ERROR;
  c.Z = dZf;
  c.ID = dID;
  auto rect = [&](double bx, double by, double bz, double Lx, double Ly, double Lz, uint8_t id) {
    if (rc) return;
    Box b;  // find_index, modelA.jl:208-219; loops start one cell before (modelA.jl:370)
    b.i0 = find_i(bx, dx, MX) - 1;
    b.j0 = find_i(by, dy, MY) - 1;
    long ks = find_k(Z, bz, MZ), ke = find_k(Z, bz + Lz, MZ);
    b.i1 = find_i(bx + Lx, dx, MX);
    b.j1 = find_i(by + Ly, dy, MY);
    if (ks < 2 || ke < 1) { rc = H2G_UNSUPPORTED; return; }
    b.k0 = ks - 1;
    b.k1 = ke;
    // candidate cells with i or j = 0 lie outside the array; is_included_rect rejects them (the
    // cell [-dx, 0] never overlaps a shape at x >= 0), so they are dropped here
    if (b.i0 < 1) b.i0 = 1;
    if (b.j0 < 1) b.j0 = 1;
    const long long cnt = (long long)(b.i1 - b.i0 + 1) * (b.j1 - b.j0 + 1) * (b.k1 - b.k0 + 1);
    if (cnt <= 0) return;
    const int blocks = (int)std::min<long long>((cnt + 255) / 256, 4096);
    k_fill_rect<<<blocks, 256>>>(c, b, bx, by, bz, bx + Lx, by + Ly, bz + Lz, id);
  };
  auto round_box = [&](double x, double y, double r, double za, double zb, Box& b) -> bool {
    b.i0 = chk_idx((long)floor((x - r - 0.0) / dx + 1.5), MX) - 1;  // find_Ri, modelA.jl:158-164
    b.i1 = chk_idx((long)floor((x + r - 0.0) / dx + 1.5), MX);
    b.j0 = chk_idx((long)floor((y - r - 0.0) / dy + 1.5), MY) - 1;
    b.j1 = chk_idx((long)floor((y + r - 0.0) / dy + 1.5), MY);
    long ks = find_k(Z, za, MZ), ke = find_k(Z, zb, MZ);
    if (ks < 2 || ke < 1 || b.i0 < 1 || b.j0 < 1) return false;
    b.k0 = ks - 1;
    b.k1 = ke;
    return true;
  };
  // FillPowerGrid!, modelA.jl:389-418
  const double s = s_dpth - pg_dpth;
  const double pz[3] = {zm2 + s, zm5 + s, zm8 + s}, pxy[2] = {0.3e-3, 0.7e-3};
  for (double z : pz)
    for (double y : pxy)
      for (double x : pxy) rect(x, y, z, 0.2e-3, 0.2e-3, pg_dpth, 7);
  // FillTSV!, modelA.jl:431-461
  const double tz[3] = {zm2, zm5, zm8}, txy[4] = {0.3e-3, 0.5e-3, 0.7e-3, 0.9e-3};
  for (double z : tz)
    for (double y : txy)
      for (double x : txy) {
        if (rc) break;
        Box b;
        if (!round_box(x, y, r_tsv, z, z + h_tsv, b)) { rc = H2G_UNSUPPORTED; break; }
        const long long cnt = (long long)(b.i1 - b.i0 + 1) * (b.j1 - b.j0 + 1) * (b.k1 - b.k0 + 1);
        if (cnt > 0) k_fill_cyl<<<(unsigned)cnt, 256>>>(c, b, x, y, r_tsv, z, z + h_tsv, 1);
      }
  // FillPlate!, modelA.jl:350-385 (geom order silicon_1..3, substrate, heatsink)
  rect(0.1e-3, 0.1e-3, zm2, 1.0e-3, 1.0e-3, 0.1e-3, 2);
  rect(0.1e-3, 0.1e-3, zm5, 1.0e-3, 1.0e-3, 0.1e-3, 2);
  rect(0.1e-3, 0.1e-3, zm8, 1.0e-3, 1.0e-3, 0.1e-3, 2);
  rect(0.0, 0.0, zm0, 1.2e-3, 1.2e-3, 0.05e-3, 4);
  rect(0.0, 0.0, zm11, 1.2e-3, 1.2e-3, 0.05e-3, 5);
  // FillSolder!, modelA.jl:464-494
  const double dp = d_ufill * 0.5;
  const double sz[4] = {zm1 + dp, zm4 + dp, zm7 + dp, zm10 + dp};
  for (double z : sz)
    for (double y : txy)
      for (double x : txy) {
        if (rc) break;
        Box b;
        if (!round_box(x, y, r_bump, z - dp, z + dp, b)) { rc = H2G_UNSUPPORTED; break; }
        const long long cnt = (long long)(b.i1 - b.i0 + 1) * (b.j1 - b.j0 + 1) * (b.k1 - b.k0 + 1);
        if (cnt > 0) k_fill_sph<<<(unsigned)cnt, 256>>>(c, b, x, y, z, r_bump, 3);
      }
  // FillResin!, modelA.jl:421-428
  if (!rc) k_fill_resin<<<1024, 256>>>(dID, n);
  if (!rc && cudaGetLastError() != cudaSuccess) rc = H2G_CUDA_ERROR;
  if (!rc && cudaMemcpy(ID, dID, (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess) rc = H2G_CUDA_ERROR;
  cudaFree(dZf);
  cudaFree(dID);
  return rc;
}

}  // extern "C"

// h2g_noalloc.cu -- CalcRK! (src/NonUniform.jl:372-434) for callers that cannot allocate device
// memory.
//
// Who needs it: a caller whose device memory is owned by someone else -- a Julia program whose
// arrays live in CUDA.jl's pool, or a time-stepping loop that must not stall on
// cudaMalloc/cudaFree (both can synchronise the device).  Such a caller already holds the fields
// in device memory and only wants the residual r = b - A theta and its norm, without a solver
// handle (h2g_create allocates).  The call ends by copying ||r|| to the host and synchronising
// its stream, so it must not be issued while that stream is capturing a CUDA graph.
//
// The reduction of ||r|| needs scratch: one partial sum per row (j, k) of the interior, a ticket
// counter and the result.  They live in g_noalloc_scratch, a file-scope device array: every GPU
// that loads this library holds it (512 KiB) until the process exits.  Consequences:
//   * at most kNoAllocMaxRows = 65536 interior rows (NY * NZ) per call; larger grids are
//     rejected with H2G_BAD_ARG before any launch;
//   * all calls share the array and it keeps the last call's contents: the ticket is cleared at
//     the start of every call, and calls that overlap on the GPU (several host threads, or
//     several streams) race on it -- serialise them;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/h2g.h"

namespace h2gn {

constexpr int kNoAllocMaxRows = 65536;
constexpr int kSlots = kNoAllocMaxRows + 64;  // row partials, then ticket and result
constexpr int kTicket = kNoAllocMaxRows;      // unsigned int in a double slot
constexpr int kResult = kNoAllocMaxRows + 1;
constexpr int kThreads = 128;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kSlots];

// lambda_f (src/common.jl:35) and the stencil of CalcRK!, recomputed per cell in the reference's
// operation order (no FMA contraction: __dmul_rn / __dadd_rn / __ddiv_rn).
__device__ __forceinline__ double lam_f(double a, double b, double ma, double mb) {
  const double h = __ddiv_rn(__dmul_rn(__dmul_rn(2.0, a), b), __dadd_rn(a, b));
  return __dmul_rn(h, __dsub_rn(2.0, trunc(__ddiv_rn(__dadd_rn(ma, mb), 2.0))));
}

struct Args {
  int MX, MY, MZ;
  const double *th, *b, *lam, *m, *rho, *cp, *ZC, *dZ;
  double dx, dy, dt, HC[6];
  int steady;
  double* r;
};

__global__ void __launch_bounds__(kThreads) k_calcrk_rows(Args a, double* scratch) {
  const int MX = a.MX, MY = a.MY;
  const int row = blockIdx.x;  // interior row (j, k), j fastest
  const int NY = MY - 2;
  const int j = 1 + row % NY, k = 1 + row / NY;
  const long long pl = (long long)MX * MY;
  const double dx0 = a.dx, dy0 = a.dy, ddx = 1.0 / dx0, ddy = 1.0 / dy0, ddt = 1.0 / a.dt;
  const double dz_k = a.dZ[k];
  const double dzm = __dsub_rn(a.ZC[k], a.ZC[k - 1]), dzp = __dsub_rn(a.ZC[k + 1], a.ZC[k]);
  double acc = 0.0;
  for (int i = 1 + threadIdx.x; i <= MX - 2; i += kThreads) {
    const long long c = (long long)i + (long long)MX * ((long long)j + (long long)MY * k);
    const double l0 = a.lam[c], m0 = a.m[c];
    const long long xm = c - 1, xp = c + 1, ym = c - MX, yp = c + MX, zm = c - pl, zp = c + pl;
    const double cxm = __dmul_rn(__dmul_rn(__dmul_rn(lam_f(a.lam[xm], l0, a.m[xm], m0), dy0), dz_k), ddx);
    const double cxp = __dmul_rn(__dmul_rn(__dmul_rn(lam_f(a.lam[xp], l0, a.m[xp], m0), dy0), dz_k), ddx);
    const double cym = __dmul_rn(__dmul_rn(__dmul_rn(lam_f(a.lam[ym], l0, a.m[ym], m0), dx0), dz_k), ddy);
    const double cyp = __dmul_rn(__dmul_rn(__dmul_rn(lam_f(a.lam[yp], l0, a.m[yp], m0), dx0), dz_k), ddy);
    const double czm = __ddiv_rn(__dmul_rn(__dmul_rn(lam_f(a.lam[zm], l0, a.m[zm], m0), dx0), dy0), dzm);
    const double czp = __ddiv_rn(__dmul_rn(__dmul_rn(lam_f(a.lam[zp], l0, a.m[zp], m0), dx0), dy0), dzp);
    const double vxm = __dmul_rn(__dmul_rn(__dmul_rn(a.HC[0], dy0), dz_k), __dsub_rn(1.0, a.m[xm]));
    const double vxp = __dmul_rn(__dmul_rn(__dmul_rn(a.HC[1], dy0), dz_k), __dsub_rn(1.0, a.m[xp]));
    const double vym = __dmul_rn(__dmul_rn(__dmul_rn(a.HC[2], dx0), dz_k), __dsub_rn(1.0, a.m[ym]));
    const double vyp = __dmul_rn(__dmul_rn(__dmul_rn(a.HC[3], dx0), dz_k), __dsub_rn(1.0, a.m[yp]));
    const double vzm = __dmul_rn(__dmul_rn(__dmul_rn(a.HC[4], dx0), dy0), __dsub_rn(1.0, a.m[zm]));
    const double vzp = __dmul_rn(__dmul_rn(__dmul_rn(a.HC[5], dx0), dy0), __dsub_rn(1.0, a.m[zp]));
    double ap = 0.0;
    if (!a.steady)
      ap = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(a.rho[c], a.cp[c]), dx0), dy0), dz_k), ddt);
    double s = __dadd_rn(cxp, cxm);
    s = __dadd_rn(s, cyp);
    s = __dadd_rn(s, cym);
    s = __dadd_rn(s, czp);
    s = __dadd_rn(s, czm);
    s = __dadd_rn(s, vxp);
    s = __dadd_rn(s, vxm);
    s = __dadd_rn(s, vyp);
    s = __dadd_rn(s, vym);
    s = __dadd_rn(s, vzp);
    s = __dadd_rn(s, vzm);
    s = __dadd_rn(s, ap);
    const double dd = __dadd_rn(__dsub_rn(1.0, m0), __dmul_rn(s, m0));
    const double* th = a.th;
    double ss = __dmul_rn(cxp, th[xp]);
    ss = __dadd_rn(ss, __dmul_rn(cxm, th[xm]));
    ss = __dadd_rn(ss, __dmul_rn(cyp, th[yp]));
    ss = __dadd_rn(ss, __dmul_rn(cym, th[ym]));
    ss = __dadd_rn(ss, __dmul_rn(czp, th[zp]));
    ss = __dadd_rn(ss, __dmul_rn(czm, th[zm]));
    const double rs = __dmul_rn(__dsub_rn(a.b[c], __dsub_rn(ss, __dmul_rn(dd, th[c]))), m0);
    a.r[c] = rs;
    acc += rs * rs;
  }
  // fixed-order block sum, then the last block adds the row partials in row order
  __shared__ double sm[kThreads / 32];
  __shared__ int last;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += sm[w];
    scratch[row] = t;
    __threadfence();
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kTicket);
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += kThreads) t += __ldcg(scratch + q);
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) tot += sm[w];
    scratch[kResult] = sqrt(tot);
  }
}

static std::mutex g_mu;
static double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
static int scratch_address(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= kMaxDevices) return H2G_UNSUPPORTED;
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return H2G_CUDA_ERROR;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return H2G_OK;
}

}  // namespace h2gn

extern "C" int h2g_calcrk_noalloc(int MX, int MY, int MZ, const double* theta, const double* b, const double* lambda,
                                  const double* mask, const double* rho, const double* cp, const double* ZC,
                                  const double* dZ, double dx, double dy, double dt, const double* HC, int is_steady,
                                  double* r, double* res, void* stream) {
  using namespace h2gn;
  if (MX < 3 || MY < 3 || MZ < 3) return H2G_BAD_ARG;
  const long long rows = (long long)(MY - 2) * (MZ - 2);
  if (rows > kNoAllocMaxRows) {
    fprintf(stderr, "h2g_calcrk_noalloc: %lld interior rows (NY*NZ) exceed the scratch limit of %d\n", rows,
            kNoAllocMaxRows);
    return H2G_BAD_ARG;
  }
  if (!theta || !b || !lambda || !mask || !ZC || !dZ || !HC || !r || !res) return H2G_BAD_ARG;
  if (!is_steady && (!rho || !cp || !(dt > 0))) return H2G_BAD_ARG;
  if (!(dx > 0) || !(dy > 0)) return H2G_BAD_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return H2G_CUDA_ERROR;
  double* scratch = nullptr;
  int rc = scratch_address(dev, &scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the ticket must start at zero; the partials and the result are overwritten by every call
  if (cudaMemsetAsync(scratch + kTicket, 0, sizeof(double), st) != cudaSuccess) return H2G_CUDA_ERROR;
  Args a;
  a.MX = MX; a.MY = MY; a.MZ = MZ;
  a.th = theta; a.b = b; a.lam = lambda; a.m = mask; a.rho = rho; a.cp = cp; a.ZC = ZC; a.dZ = dZ;
  a.dx = dx; a.dy = dy; a.dt = is_steady ? 1.0 : dt;
  for (int f = 0; f < 6; ++f) a.HC[f] = HC[f];
  a.steady = is_steady ? 1 : 0;
  a.r = r;
  k_calcrk_rows<<<(unsigned)rows, kThreads, 0, st>>>(a, scratch);
  if (cudaGetLastError() != cudaSuccess) return H2G_CUDA_ERROR;
  if (cudaMemcpyAsync(res, scratch + kResult, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return H2G_CUDA_ERROR;
  if (cudaStreamSynchronize(st) != cudaSuccess) return H2G_CUDA_ERROR;
  return H2G_OK;
}

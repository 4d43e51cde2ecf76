// h2g_internal.cuh -- data layout, device-resident solver state and arithmetic helpers
// shared by the kernels (h2g_kernels.cuh) and the host side (h2g_solver.cu).
//
// Device layout ("colour-split rows").  The reference stores Array{Float64,3} column-major
// with guards, (MX, MY, MZ).  On the device every row (j,k) of MX cells is split by the
// red-black colour of src/NonUniform.jl:873 into two half-rows, each padded to HP positions
// (HP a multiple of 32, so every half-row starts on a 256-byte boundary for FP64):
//
//     colour(i,j,k) = ((i+j+k) & 1) ^ 1          (0-based; colour 0 = the reference's first
//                                                 pass, 1-based i+j+k even)
//     offset(i,j,k) = ((k*MY + j)*2 + colour)*HP + (i >> 1)
//
// A colour pass then reads and writes whole contiguous half-rows.  For a cell at position p
// of half-row (c, j, k) with i = 2p + e, e = (1 + c + j + k) & 1, the neighbours all lie in
// half-rows of colour 1-c: x-1 at p-1+e and x+1 at p+e of the same row; y+-1 and z+-1 at the
// same position p of the rows (j+-1, k) and (j, k+-1).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace h2g {

constexpr double kFloatMin = 1.0e-37;  // src/common.jl:12
constexpr int kSweeps = 5;             // src/NonUniform.jl:44
constexpr int kMaxKeys = 127;          // material keys: 7 bits (bit 7 = mask)
constexpr int kHashSlots = 256;

struct Geo {
  int MX, MY, MZ;  // sizes with guards
  int NX, NY, NZ;  // interior sizes
  int HP;          // half-row pitch (positions)
  int HI;          // positions that can hold interior cells: (NX >> 1) + 1
  int HN;          // positions that hold cells (guards included): (MX + 1) / 2
  long long plane; // elements per k plane: MY * 2 * HP
  long long n;     // elements per vector: MZ * plane
  // offsets fit in 32 bits (h2g_create rejects grids with n >= 2^31)
  __host__ __device__ __forceinline__ int row(int c, int j, int k) const { return ((k * MY + j) * 2 + c) * HP; }
  __host__ __device__ __forceinline__ int off(int i, int j, int k) const {
    return row(((i + j + k) & 1) ^ 1, j, k) + (i >> 1);
  }
};

inline Geo make_geo(int MX, int MY, int MZ) {
  Geo g;
  g.MX = MX; g.MY = MY; g.MZ = MZ;
  g.NX = MX - 2; g.NY = MY - 2; g.NZ = MZ - 2;
  int half = (MX + 1) / 2;
  g.HP = (half + 31) / 32 * 32;
  g.HI = (g.NX >> 1) + 1;
  g.HN = half;
  g.plane = (long long)MY * 2 * g.HP;
  g.n = (long long)MZ * g.plane;
  return g;
}

// Why a solve stopped (SolverState::reason).
enum Reason { kRunning = 0, kConverged = 1, kBreakdown = 2, kMaxItr = 3, kNonFinite = 4, kTimeout = 5 };

// Bounded device waits (TMA completion barriers of the fused sweep): the default budget of one
// wait and the budget of the drain of copies still in flight after a wait ran out, in SM clock
// cycles (about one second each at 1.965 GHz).
constexpr long long kWaitCycles = 2000000000LL;
constexpr long long kDrainCycles = 2000000000LL;

// Finisher stages: what the last block of a reducing kernel does with the reduced sums.
enum Stage {
  kStageNone = 0,
  kStageInit = 1,    // Krylov start: s1 = (r,r) -> res0, rho
  kStageAlpha = 2,   // s1 = (q,r0) -> alpha
  kStageOmega = 3,   // s1 = (t,t), s2 = (t,s) -> omega (breakdown on (t,t))
  kStageUpdate = 4,  // s1 = (r,r), s2 = (r,r0) -> res, convergence, next rho, beta
  kStageResid = 5,   // s1 = (r,r) -> res (true residual of the refinement loop)
  kStageCgInit = 6,  // s1 = (r,z) -> rho_old
  kStageCgAlpha = 7, // s1 = (p,q) -> alpha (breakdown)
  kStageCgRes = 8,   // s1 = (r,r) -> res, convergence
  kStageCgBeta = 9,  // s1 = (r,z) -> beta (breakdown), iteration count
  kStageDot = 10,    // store s1, s2 in dot1, dot2
  kStageInitCg = 11, // CG start: s1 = (r,r) -> res0 (no rho check, NonUniform.jl:131-141)
  kStageSorInit = 12, // SOR start: s1 = resSOR^2 -> res0
  kStageSorHalf = 13, // s1 = colour-0 sum of r^2 -> dot1
  kStageSorIter = 14, // s1 = colour-1 sum of r^2 -> res, convergence, iteration count
};

// Scalars of one Krylov solve, resident in device memory for the whole solve.
struct SolverState {
  double rho, rho_old, alpha, omega, beta;
  double res0, res, tol;
  double scale;      // refinement: ||r|| of the FP64 residual that the inner solve was given
  double dot1, dot2; // kStageDot results
  double* hist;      // relative residual per iteration (device), may be null
  int hist_len;
  int itr, maxItr;
  int stop, converged, reason;
  int first;         // 1 until the first iteration has run (PBiCGSTAB p = r)
  unsigned int ticket;
  int passes;        // WHILE-body passes of this solve (bounds the graph loop independently)
  double div_limit;  // > 0: stop (reason kNonFinite) once the relative residual exceeds it; set only
                     // for the FP32-preconditioned passes of the mixed solver
};

// ---- arithmetic that must not be contracted into FMA: FP64 follows the reference's two-rounding
// ---- a*b + c; FP32 is kept uncontracted too, so that every launch shape of a kernel (the
// ---- compiler may contract differently per instantiation) gives the same bits.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }

// Parameters of the operator for one precision T.
template <typename T>
struct OpParams {
  Geo g;
  const uint8_t* key;  // per cell: material index (bits 0-6) | mask (bit 7), device layout
  const T* tx;         // [MZ][P][256] x-face conductance of plane k: [k][key0 & 0x7f][neighbour key]
  const T* ty;         // [MZ][P][256] y-face conductances
  const T* tz;         // [MZ][P][256] z-face between planes k-1 and k
  const T* conv;       // [MZ][4] convective terms of x-, x+, y-, y+ faces at plane k
  const T* rc;         // rho*cp per cell (device layout), transient only
  const T* dzk;        // [MZ] dZ
  const T* ddv;        // dd per cell (device layout), precomputed with the tables; may be null
  const T* tq;         // [MZ][P][256][4]: the four face tables of one (plane, own key, neighbour key)
                       // side by side: x, y, z-, z+ (z+ from plane k+1), for the fused sweeps
  const unsigned long long* nkey;  // per cell: own key and the 6 neighbours' keys, one byte each
  const uint16_t* cls; // per cell: stencil class (0xffff: not updated), may be null
  const T* ctab;       // [classes][8]: cxm, cxp, cym, cyp, czm, czp, dd of a steady grid, 0
  T czm, czp;          // convective terms of the z-, z+ faces
  T dx0, dy0, ddt;
  int P;
  int steady;
};

}  // namespace h2g

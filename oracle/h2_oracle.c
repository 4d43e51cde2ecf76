/*
 * h2_oracle.c -- CPU restatement of the Heat3ds (kenoogl/H2) linear-solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * h2_b200/csrc: only tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py may load it.  Nothing in the product links or calls it.
 *
 * Every function restates the reference algorithm statement by statement and in the
 * same floating-point evaluation order (compile with -ffp-contract=off, no -ffast-math)
 * so that a run with sequential reductions is bit-identical to Julia's SequentialEx
 * path.  Julia indices are 1-based; here cell (i,j,k) of the Julia array is
 * (i-1, j-1, k-1), stored column-major: idx = i + MX*(j + MY*k).
 *
 * Parity pins (see tests/test_oracle_golden.py): README.md:174-179 of the reference
 * gives, for q3d(240,240,30,"pbicgstab","gs";epsilon=1e-4,par="sequential",
 * is_steady=true), res0 = 0.002771608776496581, relative residuals 6.58308938608891E-01
 * and 8.89700596995947E-01 at iterations 1 and 2, and convergence at iteration 208
 * with 9.72579214884977E-05.
 *
 * Threading: `nthreads` > 1 parallelises element-wise loops with OpenMP.  Reductions
 * follow `red_mode`: H2O_RED_SEQ sums in Julia's sequential (k, j, i) order (bit-exact
 * with par="sequential"), H2O_RED_OMP uses an OpenMP reduction (the analogue of
 * FLoops ThreadedEx, src/common.jl:41-43; order differs, as in the reference).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "h2_oracle.h"

#define IX(i, j, k) ((size_t)(i) + (size_t)MX * ((size_t)(j) + (size_t)MY * (size_t)(k)))

/* ---------------------------------------------------------------------------------
 * Constants: src/common.jl:10-16, src/modelA.jl:10-30, src/NonUniform.jl:44
 * --------------------------------------------------------------------------------- */
static const double FLOAT_MIN = 1.0e-37;  /* common.jl:12 */
static const double Q_SRC = 1.6e11;       /* common.jl:16 */
#define PRECONDITIONER_SWEEPS 5            /* NonUniform.jl:44 */

static const double pg_dpth = 0.005e-3;
static const double s_dpth = 0.1e-3;
static const double d_ufill = 0.05e-3;
static const double r_bump = 0.03e-3;
static const double r_tsv = 0.02e-3;
static const double h_tsv = 0.1e-3;

#define zm12 0.6e-3
#define zm11 0.55e-3
#define zm10 0.5e-3
#define zm9 (zm10 - 0.005e-3)
#define zm8 0.4e-3
#define zm7 0.35e-3
#define zm6 (zm7 - 0.005e-3)
#define zm5 0.25e-3
#define zm4 0.2e-3
#define zm3 (zm4 - 0.005e-3)
#define zm2 0.1e-3
#define zm1 0.05e-3
#define zm0 0.0

static int g_threads = 1;

static void set_threads(int nthreads) {
  g_threads = nthreads < 1 ? 1 : nthreads;
#ifdef _OPENMP
  omp_set_num_threads(g_threads);
#endif
}

int h2o_has_openmp(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 0;
#endif
}

/* ---------------------------------------------------------------------------------
 * Z grid: Zcase2! (src/Zcoord.jl:88-124) and genZ! (src/Zcoord.jl:133-166).
 * The reference hard-wires 31 faces (NZ=30).  For NZ = 30*m (m>1) each of the 30
 * Zcase2! cells is split into m equal sub-cells:
 *   face[c*m + s] = z0 + ((z1 - z0) * s) / m,  s = 0..m-1,  then the last face z1.
 * genZ!'s guard / centre / width construction is then applied unchanged.
 * --------------------------------------------------------------------------------- */
static void zcase2(double *Z /* 31 */) {
  const double p = 0.005e-3;
  Z[0] = zm0;
  Z[1] = zm0 + p;
  Z[2] = zm1 - p;
  Z[3] = zm1;
  Z[4] = zm1 + p;
  Z[5] = zm2 - p;
  Z[6] = zm2;
  Z[7] = zm2 + p;
  Z[8] = zm3 - p;
  Z[9] = zm3;
  Z[10] = zm4;
  Z[11] = zm4 + p;
  Z[12] = zm5 - p;
  Z[13] = zm5;
  Z[14] = zm5 + p;
  Z[15] = zm6 - p;
  Z[16] = zm6;
  Z[17] = zm7;
  Z[18] = zm7 + p;
  Z[19] = zm8 - p;
  Z[20] = zm8;
  Z[21] = zm8 + p;
  Z[22] = zm9 - p;
  Z[23] = zm9;
  Z[24] = zm10;
  Z[25] = zm10 + p;
  Z[26] = zm11 - p;
  Z[27] = zm11;
  Z[28] = zm11 + p;
  Z[29] = zm12 - p;
  Z[30] = zm12;
}

int h2o_genz(int nk, double *Z /* nk+3 */, double *ZC /* nk+2 */, double *dZ /* nk+2 */) {
  if (nk < 30 || nk % 30 != 0) return -1;
  const int m = nk / 30;
  double base[31];
  zcase2(base);
  double *zf = (double *)malloc(sizeof(double) * (size_t)(nk + 1));
  for (int c = 0; c < 30; ++c) {
    const double z0 = base[c], z1 = base[c + 1];
    for (int s = 0; s < m; ++s) zf[c * m + s] = (m == 1 || s == 0) ? z0 : z0 + ((z1 - z0) * (double)s) / (double)m;
  }
  zf[nk] = base[30];
  /* genZ!: dz = diff(z_face); dz_grid (guards copy neighbours)       Zcoord.jl:137-143 */
  for (int k = 1; k <= nk; ++k) dZ[k] = zf[k] - zf[k - 1];
  dZ[0] = dZ[1];
  dZ[nk + 1] = dZ[nk];
  /* z_centers: guards sit on the boundary faces                       Zcoord.jl:146-156 */
  ZC[0] = zf[0];
  ZC[nk + 1] = zf[nk];
  for (int k = 1; k <= nk; ++k) ZC[k] = (zf[k] + zf[k - 1]) * 0.5;
  /* Z: faces with one linearly extrapolated face on each side         Zcoord.jl:160-163 */
  for (int k = 0; k <= nk; ++k) Z[k + 1] = zf[k];
  Z[0] = 2.0 * zf[0] - zf[1];
  Z[nk + 2] = 2.0 * zf[nk] - zf[nk - 1];
  free(zf);
  return 0;
}

/* dx = round(1.2e-3 / N, digits=8)   (src/heat3ds.jl:197-200; Julia rounds x*1e8 half-even) */
double h2o_pitch(int n) {
  double x = 1.2e-3 / (double)n;
  double y = rint(x * 1e8) / 1e8;
  return isfinite(y) ? y : x;
}

/* ---------------------------------------------------------------------------------
 * Geometry model: src/modelA.jl:148-556.  ID is (MX,MY,MZ) uint8, 1-based in the
 * reference; the index helpers below return 1-based indices like the reference.
 * --------------------------------------------------------------------------------- */
static long chk_idx(long i, long nx) { /* modelA.jl:148-156 */
  if (i < 1) i = 1;
  if (i > nx) i = nx;
  return i;
}
static long find_i(double x, double x0, double dx, long nx) { /* modelA.jl:174-177 */
  long i = (long)floor((x - x0) / dx + 1.5);
  return chk_idx(i, nx);
}
static void find_R(double x, double r, double x0, double dx, long nx, long *is, long *ie) {
  /* modelA.jl:158-164 (find_Ri / find_Rj are identical) */
  *is = chk_idx((long)floor((x - r - x0) / dx + 1.5), nx);
  *ie = chk_idx((long)floor((x + r - x0) / dx + 1.5), nx);
}
static long find_k(const double *Z /* 1-based view: Z1[k] = Z[k-1] */, double zc, long nz) {
  /* modelA.jl:184-204 */
  const double eps_tol = 1e-12;
  if (zc < Z[0] - eps_tol || zc > Z[nz - 1] + eps_tol) return -1;
  for (long k = 1; k <= nz - 1; ++k)
    if (Z[k - 1] <= zc && zc < Z[k]) return k;
  if (fabs(zc - Z[nz - 1]) < eps_tol) return nz - 1;
  return -1;
}

static int is_included_rect(const double *a1, const double *a2, const double *b1, const double *b2) {
  /* modelA.jl:228-245 */
  double volA = fabs((a2[0] - a1[0]) * (a2[1] - a1[1]) * (a2[2] - a1[2]));
  double axlo = fmin(a1[0], a2[0]), aylo = fmin(a1[1], a2[1]), azlo = fmin(a1[2], a2[2]);
  double axhi = fmax(a1[0], a2[0]), ayhi = fmax(a1[1], a2[1]), azhi = fmax(a1[2], a2[2]);
  double bxlo = fmin(b1[0], b2[0]), bylo = fmin(b1[1], b2[1]), bzlo = fmin(b1[2], b2[2]);
  double bxhi = fmax(b1[0], b2[0]), byhi = fmax(b1[1], b2[1]), bzhi = fmax(b1[2], b2[2]);
  double ox = fmax(0.0, fmin(axhi, bxhi) - fmax(axlo, bxlo));
  double oy = fmax(0.0, fmin(ayhi, byhi) - fmax(aylo, bylo));
  double oz = fmax(0.0, fmin(azhi, bzhi) - fmax(azlo, bzlo));
  double overlap_vol = ox * oy * oz;
  return overlap_vol >= 0.5 * volA;
}

static int is_included_cyl(const double *a1, const double *a2, const double *ctr, double cyl_r,
                           double zmin, double zmax) {
  /* modelA.jl:254-282, samples = 50 */
  const int samples = 50;
  double xlo = fmin(a1[0], a2[0]), ylo = fmin(a1[1], a2[1]), zlo = fmin(a1[2], a2[2]);
  double xhi = fmax(a1[0], a2[0]), yhi = fmax(a1[1], a2[1]), zhi = fmax(a1[2], a2[2]);
  double volA = (xhi - xlo) * (yhi - ylo) * (zhi - zlo);
  long inside = 0, total = 0;
  const double rr = cyl_r * cyl_r;
  for (int i = 1; i <= samples; ++i) {
    double x = xlo + ((double)i - 0.5) * (xhi - xlo) / (double)samples;
    double dx = x - ctr[0];
    for (int j = 1; j <= samples; ++j) {
      double y = ylo + ((double)j - 0.5) * (yhi - ylo) / (double)samples;
      double dy = y - ctr[1];
      double r2 = dx * dx + dy * dy;
      for (int k = 1; k <= samples; ++k) {
        double z = zlo + ((double)k - 0.5) * (zhi - zlo) / (double)samples;
        if (r2 <= rr && zmin <= z && z <= zmax) inside++;
        total++;
      }
    }
  }
  double overlap_vol = volA * (double)inside / (double)total;
  return overlap_vol >= 0.5 * volA;
}

static int is_included_sph(const double *a1, const double *a2, const double *c, double radius) {
  /* modelA.jl:300-347, samples = 50 */
  const int samples = 50;
  double xlo = fmin(a1[0], a2[0]), ylo = fmin(a1[1], a2[1]), zlo = fmin(a1[2], a2[2]);
  double xhi = fmax(a1[0], a2[0]), yhi = fmax(a1[1], a2[1]), zhi = fmax(a1[2], a2[2]);
  double volA = (xhi - xlo) * (yhi - ylo) * (zhi - zlo);
  if (volA <= 0) return 0;
  const double cx = c[0], cy = c[1], cz = c[2];
  const double r2 = radius * radius;
  const double xs[2] = {xlo, xhi}, ys[2] = {ylo, yhi}, zs[2] = {zlo, zhi};
  int all_inside = 1;
  for (int a = 0; a < 2 && all_inside; ++a)
    for (int b = 0; b < 2 && all_inside; ++b)
      for (int d = 0; d < 2 && all_inside; ++d) {
        double ex = xs[a] - cx, ey = ys[b] - cy, ez = zs[d] - cz;
        if (!(ex * ex + ey * ey + ez * ez <= r2)) all_inside = 0;
      }
  if (all_inside) return 1;
  long inside = 0;
  const long total = (long)samples * samples * samples;
  double dx = (xhi - xlo) / (double)samples;
  double dy = (yhi - ylo) / (double)samples;
  double dz = (zhi - zlo) / (double)samples;
  double x = xlo + dx / 2.0;
  for (int i = 0; i < samples; ++i) {
    double y = ylo + dy / 2.0;
    for (int j = 0; j < samples; ++j) {
      double z = zlo + dz / 2.0;
      double ex = x - cx, ey = y - cy;
      double exy = ex * ex + ey * ey;
      for (int k = 0; k < samples; ++k) {
        double ez = z - cz;
        if (exy + ez * ez <= r2) inside++;
        z += dz;
      }
      y += dy;
    }
    x += dx;
  }
  double overlap_vol_est = volA * ((double)inside / (double)total);
  return overlap_vol_est >= 0.5 * volA;
}

/* Cell (i,j,k), 1-based, spans [dx*(i-1), dx*(i-1)+dx] x [...] x [Z[k], Z[k+1]]
 * (modelA.jl:371-376; the origin ox is 0). */
static void cell_box(long i, long j, long k, double dx, double dy, const double *Z, double *c1, double *c2) {
  c1[0] = 0.0 + dx * (double)(i - 1);
  c1[1] = 0.0 + dy * (double)(j - 1);
  c1[2] = Z[k - 1];
  c2[0] = c1[0] + dx;
  c2[1] = c1[1] + dy;
  c2[2] = Z[k];
}

typedef struct {
  int MX, MY, MZ;
  double dx, dy;
  const double *Z; /* MZ+1 entries (genZ! "Z") */
  uint8_t *ID;
} geo_t;

static int fill_box_rect(geo_t *g, const double *b, const double *L, uint8_t id) {
  /* Common body of FillPlate! (modelA.jl:366-383) and FillPowerGrid! (400-416) */
  const int MX = g->MX, MY = g->MY;
  long st0 = chk_idx(find_i(b[0], 0.0, g->dx, g->MX), g->MX);
  long st1 = chk_idx(find_i(b[1], 0.0, g->dy, g->MY), g->MY);
  long st2 = find_k(g->Z, b[2], g->MZ);
  long ed0 = chk_idx(find_i(b[0] + L[0], 0.0, g->dx, g->MX), g->MX);
  long ed1 = chk_idx(find_i(b[1] + L[1], 0.0, g->dy, g->MY), g->MY);
  long ed2 = find_k(g->Z, b[2] + L[2], g->MZ);
  if (st2 < 1 || ed2 < 1) return -1;
  double d1[3] = {b[0], b[1], b[2]};
  double d2[3] = {b[0] + L[0], b[1] + L[1], b[2] + L[2]};
  if (st2 - 1 < 1) return -2; /* Z[0] would be out of bounds in the reference */
#pragma omp parallel for collapse(2) schedule(dynamic) num_threads(g_threads)
  for (long k = st2 - 1; k <= ed2; ++k)
    for (long j = st1 - 1; j <= ed1; ++j)
      for (long i = st0 - 1; i <= ed0; ++i) {
        double c1[3], c2[3];
        cell_box(i, j, k, g->dx, g->dy, g->Z, c1, c2);
        if (is_included_rect(c1, c2, d1, d2) && g->ID[IX(i - 1, j - 1, k - 1)] == 0) g->ID[IX(i - 1, j - 1, k - 1)] = id;
      }
  return 0;
}

static int fill_power_grid(geo_t *g) { /* FillPowerGrid! modelA.jl:389-418, lx = ly = 0.2e-3 */
  const double s = s_dpth - pg_dpth;
  const double zs[3] = {zm2 + s, zm5 + s, zm8 + s};
  const double ys[2] = {0.3e-3, 0.7e-3}, xs[2] = {0.3e-3, 0.7e-3};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        double bb[3] = {xs[c], ys[b], zs[a]};
        double L[3] = {0.2e-3, 0.2e-3, pg_dpth};
        if (fill_box_rect(g, bb, L, 7)) return -1;
      }
  return 0;
}

static int fill_plate(geo_t *g) { /* FillPlate! modelA.jl:350-385, geom order modelA.jl:82-87 */
  const double plates[5][7] = {
      /* x0, y0, z0, Lx, Ly, Lz, mat_id */
      {0.1e-3, 0.1e-3, zm2, 1.0e-3, 1.0e-3, 0.1e-3, 2}, /* silicon_1 */
      {0.1e-3, 0.1e-3, zm5, 1.0e-3, 1.0e-3, 0.1e-3, 2}, /* silicon_2 */
      {0.1e-3, 0.1e-3, zm8, 1.0e-3, 1.0e-3, 0.1e-3, 2}, /* silicon_3 */
      {0.0, 0.0, zm0, 1.2e-3, 1.2e-3, 0.05e-3, 4},      /* substrate */
      {0.0, 0.0, zm11, 1.2e-3, 1.2e-3, 0.05e-3, 5},     /* heatsink */
  };
  for (int m = 0; m < 5; ++m) {
    double b[3] = {plates[m][0], plates[m][1], plates[m][2]};
    double L[3] = {plates[m][3], plates[m][4], plates[m][5]};
    if (fill_box_rect(g, b, L, (uint8_t)plates[m][6])) return -1;
  }
  return 0;
}

static int fill_tsv(geo_t *g) { /* FillTSV! modelA.jl:431-461 */
  const int MX = g->MX, MY = g->MY;
  const double zs[3] = {zm2, zm5, zm8};
  const double xy[4] = {0.3e-3, 0.5e-3, 0.7e-3, 0.9e-3};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) {
        double ctr[2] = {xy[c], xy[b]};
        double zmin = zs[a], zmax = zs[a] + h_tsv;
        long is, ie, js, je;
        find_R(ctr[0], r_tsv, 0.0, g->dx, g->MX, &is, &ie);
        find_R(ctr[1], r_tsv, 0.0, g->dy, g->MY, &js, &je);
        long ks = find_k(g->Z, zmin, g->MZ), ke = find_k(g->Z, zmax, g->MZ);
        if (ks < 2 || ke < 1 || is < 2 || js < 2) return -1;
#pragma omp parallel for collapse(2) schedule(dynamic) num_threads(g_threads)
        for (long k = ks - 1; k <= ke; ++k)
          for (long j = js - 1; j <= je; ++j)
            for (long i = is - 1; i <= ie; ++i) {
              double c1[3], c2[3];
              cell_box(i, j, k, g->dx, g->dy, g->Z, c1, c2);
              size_t id = IX(i - 1, j - 1, k - 1);
              if (g->ID[id] == 0 && is_included_cyl(c1, c2, ctr, r_tsv, zmin, zmax)) g->ID[id] = 1;
            }
      }
  return 0;
}

static int fill_solder(geo_t *g) { /* FillSolder! modelA.jl:464-494 */
  const int MX = g->MX, MY = g->MY;
  const double dp = d_ufill * 0.5;
  const double zs[4] = {zm1 + dp, zm4 + dp, zm7 + dp, zm10 + dp};
  const double xy[4] = {0.3e-3, 0.5e-3, 0.7e-3, 0.9e-3};
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b)
      for (int c = 0; c < 4; ++c) {
        double ctr[3] = {xy[c], xy[b], zs[a]};
        long is, ie, js, je;
        find_R(ctr[0], r_bump, 0.0, g->dx, g->MX, &is, &ie);
        find_R(ctr[1], r_bump, 0.0, g->dy, g->MY, &js, &je);
        long ks = find_k(g->Z, zs[a] - dp, g->MZ), ke = find_k(g->Z, zs[a] + dp, g->MZ);
        if (ks < 2 || ke < 1 || is < 2 || js < 2) return -1;
#pragma omp parallel for collapse(2) schedule(dynamic) num_threads(g_threads)
        for (long k = ks - 1; k <= ke; ++k)
          for (long j = js - 1; j <= je; ++j)
            for (long i = is - 1; i <= ie; ++i) {
              double c1[3], c2[3];
              cell_box(i, j, k, g->dx, g->dy, g->Z, c1, c2);
              size_t id = IX(i - 1, j - 1, k - 1);
              if (g->ID[id] == 0 && is_included_sph(c1, c2, ctr, r_bump)) g->ID[id] = 3;
            }
      }
  return 0;
}

int h2o_fill_id(int MX, int MY, int MZ, double dx, double dy, const double *Z, uint8_t *ID, int nthreads) {
  /* fillID! modelA.jl:545-556: power grid, TSV, plates, solder, then resin */
  set_threads(nthreads);
  geo_t g = {MX, MY, MZ, dx, dy, Z, ID};
  memset(ID, 0, (size_t)MX * MY * MZ);
  if (fill_power_grid(&g)) return -1;
  if (fill_tsv(&g)) return -2;
  if (fill_plate(&g)) return -3;
  if (fill_solder(&g)) return -4;
  size_t n = (size_t)MX * MY * MZ;
  for (size_t c = 0; c < n; ++c)
    if (ID[c] == 0) ID[c] = 6; /* FillResin! modelA.jl:421-428 */
  return 0;
}

void h2o_set_properties(size_t n, const uint8_t *ID, double *lam, double *rho, double *cp) {
  /* setProperties! modelA.jl:499-542 with the material table modelA.jl:96-122 */
  for (size_t c = 0; c < n; ++c) {
    switch (ID[c]) {
      case 7: lam[c] = 149.0; rho[c] = 2330.0; cp[c] = 720.0; break;  /* pwrsrc */
      case 1: lam[c] = 386.0; rho[c] = 8960.0; cp[c] = 383.0; break;  /* copper */
      case 2: lam[c] = 149.0; rho[c] = 2330.0; cp[c] = 720.0; break;  /* silicon */
      case 4: lam[c] = 0.4; rho[c] = 1850.0; cp[c] = 1000.0; break;   /* FR4 */
      case 5: lam[c] = 222.0; rho[c] = 2700.0; cp[c] = 921.0; break;  /* A1060 */
      case 3: lam[c] = 50.0; rho[c] = 8500.0; cp[c] = 197.0; break;   /* solder */
      default: lam[c] = 1.5; rho[c] = 2590.0; cp[c] = 1050.0; break;  /* resin */
    }
  }
}

/* ---------------------------------------------------------------------------------
 * Boundary conditions: src/boundary_conditions.jl:94-313 (guard cells) and 360-394 (HC).
 * bc[f] for faces f = x-, x+, y-, y+, z-, z+ (boundary_conditions.jl:24-31).
 * --------------------------------------------------------------------------------- */
void h2o_apply_bc(int MX, int MY, int MZ, const h2o_bc *bc, double *th, double *lam, double *rho, double *cp,
                  double *mask) {
  for (int f = 0; f < 6; ++f) {
    const int axis = f / 2, plus = f % 2;
    const int n0 = axis == 0 ? MY : MX, n1 = axis == 2 ? MY : MZ;
    for (int b = 0; b < n1; ++b)
      for (int a = 0; a < n0; ++a) {
        size_t g, in;
        if (axis == 0) {
          int i = plus ? MX - 1 : 0, ii = plus ? MX - 2 : 1;
          g = IX(i, a, b); in = IX(ii, a, b);
        } else if (axis == 1) {
          int j = plus ? MY - 1 : 0, jj = plus ? MY - 2 : 1;
          g = IX(a, j, b); in = IX(a, jj, b);
        } else {
          int k = plus ? MZ - 1 : 0, kk = plus ? MZ - 2 : 1;
          g = IX(a, b, k); in = IX(a, b, kk);
        }
        switch (bc[f].type) {
          case H2O_ISOTHERMAL: /* apply_isothermal! 156-215 */
            mask[g] = 0.0; lam[g] = lam[in]; rho[g] = rho[in]; cp[g] = cp[in]; th[g] = bc[f].temperature;
            break;
          case H2O_HEAT_FLUX: /* apply_heat_flux! 221-260 */
            mask[g] = 0.0; lam[g] = 0.0;
            break;
          case H2O_CONVECTION: /* apply_convection! 266-313 */
            mask[g] = 0.0; lam[g] = 0.0; th[g] = bc[f].ambient;
            break;
        }
      }
  }
}

void h2o_set_bc_coef(const h2o_bc *bc, double *HC) { /* set_BC_coef 360-394 */
  for (int f = 0; f < 6; ++f) HC[f] = bc[f].type == H2O_CONVECTION ? bc[f].htc : 0.0;
}

void h2o_heat_src(int MX, int MY, int MZ, const uint8_t *ID, double *hsrc) { /* HeatSrc! heat3ds.jl:55-64 */
  for (int k = 1; k < MZ - 1; ++k)
    for (int j = 1; j < MY - 1; ++j)
      for (int i = 1; i < MX - 1; ++i)
        if (ID[IX(i, j, k)] == 7) hsrc[IX(i, j, k)] = Q_SRC;
}

/* ---------------------------------------------------------------------------------
 * RHS: calRHS! (src/NonUniform.jl:57-91) with apply_bc2RHS! (src/RHS.jl:23-192).
 * b accumulates: the caller zeroes it before each time step if needed.
 * --------------------------------------------------------------------------------- */
void h2o_calrhs(const h2o_grid *G, const h2o_bc *bc, double *b, const double *th, const double *rho,
                const double *cp, const double *hsrc) {
  const int MX = G->MX, MY = G->MY, MZ = G->MZ;
  const double dx = G->dx, dy = G->dy;
  const double *dZ = G->dZ;
  for (int f = 0; f < 6; ++f) {
    const int axis = f / 2, plus = f % 2;
    if (bc[f].type == H2O_ISOTHERMAL) continue;
    const int n0 = axis == 0 ? MY : MX, n1 = axis == 2 ? MY : MZ;
    for (int bb = 1; bb < n1 - 1; ++bb)
      for (int a = 1; a < n0 - 1; ++a) {
        size_t c;
        double area;
        if (axis == 0) { c = IX(plus ? MX - 2 : 1, a, bb); area = dy * dZ[bb]; }
        else if (axis == 1) { c = IX(a, plus ? MY - 2 : 1, bb); area = dx * dZ[bb]; }
        else { c = IX(a, bb, plus ? MZ - 2 : 1); area = dx * dy; }
        if (bc[f].type == H2O_HEAT_FLUX) { /* RHS_heat_flux! RHS.jl:83-134 */
          const double q = bc[f].heat_flux;
          if (plus) b[c] -= q * area; else b[c] += q * area;
        } else { /* RHS_convection! RHS.jl:140-192 */
          const double h = bc[f].htc, ta = bc[f].ambient;
          if (plus) b[c] += h * area * (ta - th[c]); else b[c] -= h * area * (ta - th[c]);
        }
      }
  }
  const double ddt = 1.0 / G->dt;
#pragma omp parallel for collapse(2) num_threads(g_threads)
  for (int k = 1; k < MZ - 1; ++k)
    for (int j = 1; j < MY - 1; ++j) {
      const double dz_k = dZ[k];
      for (int i = 1; i < MX - 1; ++i) {
        const size_t c = IX(i, j, k);
        double a_p_0 = G->is_steady ? 0.0 : rho[c] * cp[c] * dx * dy * dz_k * ddt;
        b[c] = -(a_p_0 * th[c] + hsrc[c] * dx * dy * dz_k + b[c]);
      }
    }
}

/* ---------------------------------------------------------------------------------
 * The 7-point operator.  lambda_f: src/common.jl:35.  The stencil body is shared by
 * CalcRK! (NonUniform.jl:396-432), CalcAX! (476-510), resSOR (703-740), sor!
 * (784-823) and rbsor_core! (872-911); it is restated once here.
 * --------------------------------------------------------------------------------- */
static inline double lambda_f(double a, double b, double ma, double mb) {
  return 2.0 * a * b / (a + b) * (2.0 - trunc((ma + mb) / 2.0));
}

typedef struct {
  double cxm, cxp, cym, cyp, czm, czp, dd, m0;
} stencil_t;

static inline void stencil_coef(const h2o_grid *G, const double *lam, const double *m, const double *rho,
                                const double *cp, int i, int j, int k, stencil_t *s) {
  const int MX = G->MX, MY = G->MY;
  const double dx0 = G->dx, dy0 = G->dy;
  const double ddx = 1.0 / dx0, ddy = 1.0 / dy0, ddt = 1.0 / G->dt;
  const double *HC = G->HC, *ZC = G->ZC;
  const size_t c = IX(i, j, k);
  const double dz_k = G->dZ[k];
  const double l0 = lam[c], m0 = m[c];
  const size_t xm = c - 1, xp = c + 1, ym = c - MX, yp = c + MX, zmi = c - (size_t)MX * MY, zpi = c + (size_t)MX * MY;
  double cond_xm = lambda_f(lam[xm], l0, m[xm], m0) * dy0 * dz_k * ddx;
  double cond_xp = lambda_f(lam[xp], l0, m[xp], m0) * dy0 * dz_k * ddx;
  double cond_ym = lambda_f(lam[ym], l0, m[ym], m0) * dx0 * dz_k * ddy;
  double cond_yp = lambda_f(lam[yp], l0, m[yp], m0) * dx0 * dz_k * ddy;
  double cond_zm = lambda_f(lam[zmi], l0, m[zmi], m0) * dx0 * dy0 / (ZC[k] - ZC[k - 1]);
  double cond_zp = lambda_f(lam[zpi], l0, m[zpi], m0) * dx0 * dy0 / (ZC[k + 1] - ZC[k]);
  double conv_xm = HC[0] * dy0 * dz_k * (1.0 - m[xm]);
  double conv_xp = HC[1] * dy0 * dz_k * (1.0 - m[xp]);
  double conv_ym = HC[2] * dx0 * dz_k * (1.0 - m[ym]);
  double conv_yp = HC[3] * dx0 * dz_k * (1.0 - m[yp]);
  double conv_zm = HC[4] * dx0 * dy0 * (1.0 - m[zmi]);
  double conv_zp = HC[5] * dx0 * dy0 * (1.0 - m[zpi]);
  double a_p_0 = G->is_steady ? 0.0 : rho[c] * cp[c] * dx0 * dy0 * dz_k * ddt;
  s->dd = (1.0 - m0) + (cond_xp + cond_xm + cond_yp + cond_ym + cond_zp + cond_zm + conv_xp + conv_xm + conv_yp +
                        conv_ym + conv_zp + conv_zm + a_p_0) * m0;
  s->cxm = cond_xm; s->cxp = cond_xp; s->cym = cond_ym; s->cyp = cond_yp; s->czm = cond_zm; s->czp = cond_zp;
  s->m0 = m0;
}

static inline double stencil_ss(const h2o_grid *G, const stencil_t *s, const double *x, size_t c) {
  const int MX = G->MX, MY = G->MY;
  const size_t pl = (size_t)MX * MY;
  return s->cxp * x[c + 1] + s->cxm * x[c - 1] + s->cyp * x[c + MX] + s->cym * x[c - MX] + s->czp * x[c + pl] +
         s->czm * x[c - pl];
}

/* Sum the interior of `v` in Julia's (k, j, i) order, or with an OpenMP reduction. */
static double interior_sum_sq_or_dot(const h2o_grid *G, const double *x, const double *y, int red_mode) {
  const int MX = G->MX, MY = G->MY, MZ = G->MZ;
  double sum = 0.0;
  if (red_mode == H2O_RED_OMP && g_threads > 1) {
#pragma omp parallel for collapse(2) reduction(+ : sum) num_threads(g_threads)
    for (int k = 1; k < MZ - 1; ++k)
      for (int j = 1; j < MY - 1; ++j)
        for (int i = 1; i < MX - 1; ++i) {
          size_t c = IX(i, j, k);
          sum += x[c] * y[c];
        }
  } else {
    for (int k = 1; k < MZ - 1; ++k)
      for (int j = 1; j < MY - 1; ++j)
        for (int i = 1; i < MX - 1; ++i) {
          size_t c = IX(i, j, k);
          sum = sum + x[c] * y[c];
        }
  }
  return sum;
}

double h2o_fdot1(const h2o_grid *G, const double *x, int red_mode) { /* Fdot1 NonUniform.jl:567-575 */
  return interior_sum_sq_or_dot(G, x, x, red_mode);
}
double h2o_fdot2(const h2o_grid *G, const double *x, const double *y, int red_mode) { /* Fdot2 584-592 */
  return interior_sum_sq_or_dot(G, x, y, red_mode);
}

double h2o_calcrk(const h2o_grid *G, double *r, const double *th, const double *b, const double *lam,
                  const double *m, const double *rho, const double *cp, int red_mode) {
  /* CalcRK! NonUniform.jl:372-434; returns sqrt(sum r^2) */
  const int MX = G->MX, MY = G->MY, MZ = G->MZ;
#pragma omp parallel for collapse(2) num_threads(g_threads)
  for (int k = 1; k < MZ - 1; ++k)
    for (int j = 1; j < MY - 1; ++j)
      for (int i = 1; i < MX - 1; ++i) {
        stencil_t s;
        stencil_coef(G, lam, m, rho, cp, i, j, k, &s);
        const size_t c = IX(i, j, k);
        double ss = stencil_ss(G, &s, th, c);
        r[c] = (b[c] - (ss - s.dd * th[c])) * s.m0;
      }
  return sqrt(interior_sum_sq_or_dot(G, r, r, red_mode));
}

void h2o_calcax(const h2o_grid *G, double *ax, const double *x, const double *lam, const double *m,
                const double *rho, const double *cp) {
  /* CalcAX! NonUniform.jl:454-511 */
  const int MX = G->MX, MY = G->MY, MZ = G->MZ;
#pragma omp parallel for collapse(2) num_threads(g_threads)
  for (int k = 1; k < MZ - 1; ++k)
    for (int j = 1; j < MY - 1; ++j)
      for (int i = 1; i < MX - 1; ++i) {
        stencil_t s;
        stencil_coef(G, lam, m, rho, cp, i, j, k, &s);
        const size_t c = IX(i, j, k);
        double ss = stencil_ss(G, &s, x, c);
        ax[c] = (ss - s.dd * x[c]) * s.m0;
      }
}

double h2o_rbsor_core(const h2o_grid *G, double *th, const double *lam, const double *b, const double *m,
                      const double *rho, const double *cp, double omega, int color, int red_mode) {
  /* rbsor_core! NonUniform.jl:848-915: updates i = 2+mod(k+j+color,2) : 2 : SZ[1]-1 (1-based),
   * i.e. colour 0 is the set of cells with i+j+k even.  Returns the sum of squared
   * residuals r = (dd + w*(c_xm+c_ym+c_zm))*dp/w.  red_mode H2O_RED_NONE skips the sum
   * (the preconditioner discards it, NonUniform.jl:556-558). */
  const int MX = G->MX, MY = G->MY, MZ = G->MZ;
  const int seq_sum = (red_mode == H2O_RED_SEQ) && g_threads > 1;
  double *rr = NULL;
  if (seq_sum) rr = (double *)calloc((size_t)MX * MY * MZ, sizeof(double));
  double res = 0.0;
#pragma omp parallel for collapse(2) reduction(+ : res) num_threads(g_threads)
  for (int k = 1; k < MZ - 1; ++k)
    for (int j = 1; j < MY - 1; ++j) {
      const int i0 = 1 + ((k + 1 + j + 1 + color) % 2);
      for (int i = i0; i < MX - 1; i += 2) {
        stencil_t s;
        stencil_coef(G, lam, m, rho, cp, i, j, k, &s);
        const size_t c = IX(i, j, k);
        const double pp = th[c];
        double ss = stencil_ss(G, &s, th, c);
        double dp = (((ss - b[c]) / s.dd - pp)) * s.m0;
        th[c] = pp + omega * dp;
        if (red_mode != H2O_RED_NONE) {
          double r = (s.dd + omega * (s.cxm + s.cym + s.czm)) * dp / omega;
          if (seq_sum) rr[c] = r * r; else res += r * r;
        }
      }
    }
  if (seq_sum) {
    res = 0.0;
    for (int k = 1; k < MZ - 1; ++k)
      for (int j = 1; j < MY - 1; ++j) {
        const int i0 = 1 + ((k + 1 + j + 1 + color) % 2);
        for (int i = i0; i < MX - 1; i += 2) res = res + rr[IX(i, j, k)];
      }
    free(rr);
  }
  return res;
}

double h2o_rbsor(const h2o_grid *G, double *th, const double *lam, const double *b, const double *m,
                 const double *rho, const double *cp, double omega, int red_mode) {
  /* rbsor! NonUniform.jl:936-957 (rbsor_simple! 978-993 is identical) */
  double res = 0.0;
  for (int c = 0; c < 2; ++c) res += h2o_rbsor_core(G, th, lam, b, m, rho, cp, omega, c, red_mode);
  return sqrt(res);
}

static void fill_all(const h2o_grid *G, double *a, double v) { /* myfill! common.jl:95-101 */
  size_t n = (size_t)G->MX * G->MY * G->MZ;
  for (size_t c = 0; c < n; ++c) a[c] = v;
}
static void copy_all(const h2o_grid *G, double *d, const double *s) { /* mycopy! common.jl:107-113 */
  memcpy(d, s, sizeof(double) * (size_t)G->MX * G->MY * G->MZ);
}

void h2o_preconditioner(const h2o_grid *G, double *xx, const double *bb, const double *lam, const double *m,
                        const double *rho, const double *cp, int smoother) {
  /* Preconditioner! / _Preconditioner! NonUniform.jl:531-559 */
  if (smoother == H2O_SMOOTHER_NONE) {
    copy_all(G, xx, bb);
    return;
  }
  for (int s = 0; s < PRECONDITIONER_SWEEPS; ++s) h2o_rbsor(G, xx, lam, bb, m, rho, cp, 1.0, H2O_RED_NONE);
}

#define INTERIOR_LOOP(body)                                    \
  _Pragma("omp parallel for collapse(2) num_threads(g_threads)") \
  for (int k = 1; k < MZ - 1; ++k)                             \
    for (int j = 1; j < MY - 1; ++j)                           \
      for (int i = 1; i < MX - 1; ++i) {                       \
        const size_t c = IX(i, j, k);                          \
        body;                                                  \
      }

void h2o_bicg1(const h2o_grid *G, double *p, const double *r, const double *q, double beta, double omg) {
  const int MX = G->MX, MY = G->MY, MZ = G->MZ; /* BiCG1! NonUniform.jl:603-615 */
  INTERIOR_LOOP(p[c] = r[c] + beta * (p[c] - omg * q[c]));
}
void h2o_triad(const h2o_grid *G, double *z, const double *x, const double *y, double a) {
  const int MX = G->MX, MY = G->MY, MZ = G->MZ; /* Triad! NonUniform.jl:625-636 */
  INTERIOR_LOOP(z[c] = a * x[c] + y[c]);
}
void h2o_bicg2(const h2o_grid *G, double *z, const double *x, const double *y, double a, double b) {
  const int MX = G->MX, MY = G->MY, MZ = G->MZ; /* BICG2! NonUniform.jl:647-659 */
  INTERIOR_LOOP(z[c] += a * x[c] + b * y[c]);
}

int h2o_pbicgstab(const h2o_grid *G, h2o_wk *wk, double tol, int maxItr, int smoother, int verbose, int red_mode,
                  int nthreads, int *itr_out, double *res0_out, double *hist) {
  /* PBiCGSTAB! NonUniform.jl:248-350.  Returns isconverged; hist[k-1] = relative residual
   * of iteration k (hist may be NULL). */
  set_threads(nthreads);
  fill_all(G, wk->q, 0.0);
  double res0 = h2o_calcrk(G, wk->r, wk->theta, wk->b, wk->lam, wk->mask, wk->rho, wk->cp, red_mode);
  if (verbose) printf("Initial residual = %.17g\n", res0);
  *res0_out = res0;
  *itr_out = 0;
  if (res0 == 0.0) return 1;
  copy_all(G, wk->r0, wk->r);
  double rho_old = 1.0, alpha = 0.0, omega = 1.0, r_omega = -omega, beta = 0.0;
  int isconverged = 0, itr = 0;
  (void)r_omega;
  for (int k = 1; k <= maxItr; ++k) {
    itr = k;
    double rho = h2o_fdot2(G, wk->r, wk->r0, red_mode);
    if (fabs(rho) < FLOAT_MIN) { isconverged = 0; break; }
    if (k == 1) copy_all(G, wk->p, wk->r);
    else {
      beta = rho / rho_old * alpha / omega;
      h2o_bicg1(G, wk->p, wk->r, wk->q, beta, omega);
    }
    fill_all(G, wk->p_, 0.0);
    h2o_preconditioner(G, wk->p_, wk->p, wk->lam, wk->mask, wk->rho, wk->cp, smoother);
    h2o_calcax(G, wk->q, wk->p_, wk->lam, wk->mask, wk->rho, wk->cp);
    alpha = rho / h2o_fdot2(G, wk->q, wk->r0, red_mode);
    double r_alpha = -alpha;
    h2o_triad(G, wk->s, wk->q, wk->r, r_alpha);
    fill_all(G, wk->s_, 0.0);
    h2o_preconditioner(G, wk->s_, wk->s, wk->lam, wk->mask, wk->rho, wk->cp, smoother);
    h2o_calcax(G, wk->t_, wk->s_, wk->lam, wk->mask, wk->rho, wk->cp);
    double denom = h2o_fdot1(G, wk->t_, red_mode);
    if (fabs(denom) < FLOAT_MIN) { isconverged = 0; break; }
    omega = h2o_fdot2(G, wk->t_, wk->s, red_mode) / denom;
    r_omega = -omega;
    h2o_bicg2(G, wk->theta, wk->p_, wk->s_, alpha, omega);
    h2o_triad(G, wk->r, wk->t_, wk->s, r_omega);
    double res = sqrt(h2o_fdot1(G, wk->r, red_mode));
    res /= res0;
    if (hist) hist[k - 1] = res;
    if (verbose) printf("%10d %24.14E\n", itr, res);
    if (res < tol) {
      isconverged = 1;
      if (verbose) printf("Converged at %d\n", itr);
      break;
    }
    rho_old = rho;
  }
  *itr_out = itr;
  return isconverged;
}

int h2o_cg(const h2o_grid *G, h2o_wk *wk, double tol, int maxItr, int smoother, int verbose, int red_mode,
           int nthreads, int *itr_out, double *res0_out, double *hist) {
  /* CG! NonUniform.jl:115-226 (pcg_s holds z) */
  set_threads(nthreads);
  const int MX = G->MX, MY = G->MY, MZ = G->MZ;
  fill_all(G, wk->q, 0.0);
  double res0 = h2o_calcrk(G, wk->r, wk->theta, wk->b, wk->lam, wk->mask, wk->rho, wk->cp, red_mode);
  if (verbose) printf("Initial residual = %.17g\n", res0);
  *res0_out = res0;
  *itr_out = 0;
  if (res0 == 0.0) return 1;
  fill_all(G, wk->s, 0.0);
  h2o_preconditioner(G, wk->s, wk->r, wk->lam, wk->mask, wk->rho, wk->cp, smoother);
  copy_all(G, wk->p, wk->s);
  double rho_old = h2o_fdot2(G, wk->r, wk->s, red_mode);
  int isconverged = 0, itr = 0;
  for (int k = 1; k <= maxItr; ++k) {
    itr = k;
    h2o_calcax(G, wk->q, wk->p, wk->lam, wk->mask, wk->rho, wk->cp);
    double denom = h2o_fdot2(G, wk->p, wk->q, red_mode);
    if (fabs(denom) < FLOAT_MIN) { isconverged = 0; break; }
    double alpha = rho_old / denom;
    double *th = wk->theta, *p = wk->p, *r = wk->r, *q = wk->q;
    INTERIOR_LOOP({
      th[c] += alpha * p[c];
      r[c] -= alpha * q[c];
    });
    double res = sqrt(h2o_fdot1(G, wk->r, red_mode));
    res /= res0;
    if (hist) hist[k - 1] = res;
    if (verbose) printf("%10d %24.14E\n", itr, res);
    if (res < tol) {
      isconverged = 1;
      if (verbose) printf("Converged at %d\n", itr);
      break;
    }
    fill_all(G, wk->s, 0.0);
    h2o_preconditioner(G, wk->s, wk->r, wk->lam, wk->mask, wk->rho, wk->cp, smoother);
    double rho_new = h2o_fdot2(G, wk->r, wk->s, red_mode);
    if (fabs(rho_new) < FLOAT_MIN) { isconverged = 0; break; }
    double beta = rho_new / rho_old;
    const double *z = wk->s;
    INTERIOR_LOOP(p[c] = z[c] + beta * p[c]);
    rho_old = rho_new;
  }
  *itr_out = itr;
  return isconverged;
}

/* ---------------------------------------------------------------------------------
 * Stand-alone RB-SOR: resSOR (NonUniform.jl:680-743) + solveSOR! (1017-1051).
 * Returns the number of sweeps run (hist[n-1] = relative residual of sweep n).
 * --------------------------------------------------------------------------------- */
double h2o_res_sor(const h2o_grid *G, const double *th, const double *lam, const double *b, const double *m,
                   const double *rho, const double *cp, double omega) {
  const int MX = G->MX, MY = G->MY, MZ = G->MZ;
  double res = 0.0;
  for (int k = 1; k < MZ - 1; ++k)
    for (int j = 1; j < MY - 1; ++j)
      for (int i = 1; i < MX - 1; ++i) {
        stencil_t s;
        stencil_coef(G, lam, m, rho, cp, i, j, k, &s);
        const size_t c = IX(i, j, k);
        double ss = stencil_ss(G, &s, th, c);
        double dp = (((ss - b[c]) / s.dd - th[c])) * s.m0;
        double r = (s.dd + omega * (s.cxm + s.cym + s.czm)) * dp / omega;
        res = res + r * r;
      }
  return sqrt(res);
}

int h2o_solve_sor(const h2o_grid *G, h2o_wk *wk, double omega, double tol, int maxItr, int red_mode, int nthreads, double *res0_out,
                  double *hist) {
  set_threads(nthreads);
  double res0 = h2o_res_sor(G, wk->theta, wk->lam, wk->b, wk->mask, wk->rho, wk->cp, omega);
  if (res0 == 0.0) res0 = 1.0;
  *res0_out = res0;
  for (int n = 1; n <= maxItr; ++n) {
    double res = h2o_rbsor(G, wk->theta, wk->lam, wk->b, wk->mask, wk->rho, wk->cp, omega, red_mode) / res0;
    if (hist) hist[n - 1] = res;
    if (res < tol) return n;
  }
  return -maxItr;
}

void h2o_set_threads(int nthreads) { set_threads(nthreads); }

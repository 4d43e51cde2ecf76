/* A plain-C caller of libh2g.so, the way a Julia ccall, cgo or JNI binding calls it: only the
 * declarations of include/h2g.h, host arrays in the reference's column-major layout with guards.
 *
 *   abi_harness host    checks that need no GPU (version, status strings, argument checks)
 *   abi_harness solve   a 14^3 uniform block with isothermal 300 K faces and a uniform heat
 *                       source: calRHS!, PBiCGSTAB! + RB-GS, then checks convergence, the
 *                       mirror symmetry of the solution and that it stays above 300 K.
 * Exit status 0 on success; a message on stderr otherwise. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "h2g.h"

#define FAIL(...)                     \
  do {                                \
    fprintf(stderr, __VA_ARGS__);     \
    fprintf(stderr, "\n");            \
    return 1;                         \
  } while (0)

static int host_checks(void) {
  h2g_solver *h = NULL;
  h2g_result res;
  if (!strstr(h2g_version(), "sm_100a")) FAIL("version string: %s", h2g_version());
  if (strcmp(h2g_status_string(H2G_OK), "ok") != 0) FAIL("status string of H2G_OK");
  if (h2g_create(2, 5, 5, H2G_FP64, &h) != H2G_BAD_ARG) FAIL("a 2-wide grid was accepted");
  if (h2g_pbicgstab(NULL, 1e-6, 10, H2G_SMOOTHER_GS, 0, NULL, &res) != H2G_BAD_ARG) FAIL("null handle accepted");
  if (h2g_destroy(NULL) != H2G_OK) FAIL("destroy(NULL)");
  printf("host checks ok: %s\n", h2g_version());
  return 0;
}

static size_t at(int MX, int MY, int i, int j, int k) { return (size_t)i + (size_t)MX * ((size_t)j + (size_t)MY * k); }

static int solve_check(void) {
  const int N = 12, M = N + 2;
  const size_t n = (size_t)M * M * M;
  double *theta = malloc(n * sizeof(double)), *b = calloc(n, sizeof(double)), *lam = malloc(n * sizeof(double));
  double *mask = malloc(n * sizeof(double)), *hsrc = calloc(n, sizeof(double));
  double ZC[14], dZ[14], HC[6] = {0, 0, 0, 0, 0, 0};
  const double d = 1.0e-4;
  h2g_solver *h = NULL;
  h2g_result res;
  h2g_bc bc[6];
  int rc = 0;
  for (int k = 0; k < M; ++k) {
    ZC[k] = (k - 0.5) * d;  /* guard centres half a cell outside, as genZ! does at the faces */
    dZ[k] = d;
  }
  ZC[0] = 0.0;
  ZC[M - 1] = N * d;
  for (size_t c = 0; c < n; ++c) {
    theta[c] = 300.0;
    lam[c] = 150.0;
    mask[c] = 0.0;
  }
  for (int k = 1; k <= N; ++k)
    for (int j = 1; j <= N; ++j)
      for (int i = 1; i <= N; ++i) {
        mask[at(M, M, i, j, k)] = 1.0;
        hsrc[at(M, M, i, j, k)] = 1.0e12;
      }
  for (int f = 0; f < 6; ++f) {
    bc[f].type = H2G_ISOTHERMAL;
    bc[f].temperature = 300.0;
    bc[f].heat_flux = bc[f].htc = bc[f].ambient = 0.0;
  }
  if (h2g_create(M, M, M, H2G_FP64, &h) != H2G_OK) FAIL("create: %s", h2g_last_error());
  if (h2g_set_grid(h, ZC, dZ, d, d, 1.0, HC, 1) || h2g_set_fields(h, lam, mask, NULL, NULL) ||
      h2g_set_theta(h, theta) || h2g_set_rhs(h, b) || h2g_set_hsrc(h, hsrc) || h2g_calrhs(h, bc, 1))
    FAIL("set-up: %s", h2g_last_error());
  if (h2g_pbicgstab(h, 1e-10, 2000, H2G_SMOOTHER_GS, 0, NULL, &res) != H2G_OK || !res.isconverged)
    FAIL("solve: status %d, %d iterations, res %g", res.status, res.itr, res.res);
  if (h2g_get_theta(h, theta)) FAIL("get_theta: %s", h2g_last_error());
  double tmin = 1e300, asym = 0.0;
  for (int k = 1; k <= N; ++k)
    for (int j = 1; j <= N; ++j)
      for (int i = 1; i <= N; ++i) {
        const double t = theta[at(M, M, i, j, k)];
        tmin = t < tmin ? t : tmin;
        const double tx = theta[at(M, M, N + 1 - i, j, k)], ty = theta[at(M, M, i, N + 1 - j, k)];
        asym = fmax(asym, fmax(fabs(t - tx), fabs(t - ty)));
      }
  if (!(tmin > 300.0)) rc = 1, fprintf(stderr, "interior minimum %.9f K is not above the 300 K faces\n", tmin);
  if (asym > 1e-7) rc = 1, fprintf(stderr, "mirror asymmetry %.3e K\n", asym);
  printf("solve ok: %d iterations, res0 %.6e, theta %.6f .. %.6f K, asymmetry %.2e K\n", res.itr, res.res0, tmin,
         theta[at(M, M, M / 2, M / 2, M / 2)], asym);
  h2g_destroy(h);
  free(theta); free(b); free(lam); free(mask); free(hsrc);
  return rc;
}

int main(int argc, char **argv) {
  if (argc > 1 && strcmp(argv[1], "solve") == 0) return solve_check();
  return host_checks();
}

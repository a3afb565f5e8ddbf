/*
 * sma_c_client.c -- a plain C caller of the library's C ABI (include/alya_sma.h),
 * the way a compiled host program (or a Fortran bind(C) interface) uses it: no
 * Python, no torch.  Built and run by tests/test_c_client.py.
 *
 *   sma_c_client reject           argument checks, needs no GPU (exit 0 = pass)
 *   sma_c_client run <out.bin>    a 8x2x2 NiTi bar, x = 0 clamped, x = 8 end
 *                                 pulled 0.4 mm and back with a smooth table;
 *                                 100 central-difference steps in FP64 with the
 *                                 coloured scatter; writes dt, then the
 *                                 displacement (3, npoin), to out.bin
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "alya_sma.h"

enum { NX = 8, NY = 2, NZ = 2, NP = (NX + 1) * (NY + 1) * (NZ + 1), NE = NX * NY * NZ };

static int nid(int i, int j, int k) { return i + (NX + 1) * (j + (NY + 1) * k); }

/* unit-cube mesh; node id i + 9 (j + 3 k), element id i + 8 (j + 2 k) */
static void mesh(double* coord, int32_t* lnods) {
  for (int k = 0; k <= NZ; ++k)
    for (int j = 0; j <= NY; ++j)
      for (int i = 0; i <= NX; ++i) {
        double* x = coord + 3 * nid(i, j, k);
        x[0] = i; x[1] = j; x[2] = k;
      }
  for (int k = 0; k < NZ; ++k)
    for (int j = 0; j < NY; ++j)
      for (int i = 0; i < NX; ++i) {
        int32_t* l = lnods + 8 * (i + NX * (j + NY * k));
        l[0] = nid(i, j, k);         l[1] = nid(i + 1, j, k);
        l[2] = nid(i + 1, j + 1, k); l[3] = nid(i, j + 1, k);
        l[4] = nid(i, j, k + 1);     l[5] = nid(i + 1, j, k + 1);
        l[6] = nid(i + 1, j + 1, k + 1); l[7] = nid(i, j + 1, k + 1);
      }
}

/* NITINOL parameter vector (sld_stress_model_160.f90:263-279): E, nu, eL (the
 * norm of the uniaxial 5 % transformation strain), AS 400/500 MPa, SA 250/150 MPa */
static void niti(double* p) {
  memset(p, 0, 18 * sizeof(double));
  p[0] = 60000.0; p[1] = 0.33; p[2] = 0.05 * sqrt(1.5);
  p[3] = 400.0; p[4] = 500.0; p[9] = 250.0; p[10] = 150.0;
}

static int reject(void) {
  double coord[3 * NP], props[18], densi = 6.45e-9;
  int32_t lnods[8 * NE];
  mesh(coord, lnods);
  niti(props);
  lnods[8 * 5 + 3] = NP + 7;                                    /* a node that does not exist */
  sma_mesh_desc m = {NE, NP, lnods, coord, NULL};
  sma_material_desc mat = {1, props, NULL, &densi, NULL, NULL};
  sma_run_desc run;
  memset(&run, 0, sizeof run);
  run.precision = SMA_PREC_FP64;
  run.dtime = 1e-7;
  sma_ctx* ctx = NULL;
  int32_t rc = sma_ctx_create(&m, &mat, &run, &ctx);
  if (rc >= 0 || ctx != NULL || !strstr(sma_last_error(), "lnods")) {
    fprintf(stderr, "bad connectivity accepted: rc=%d (%s)\n", rc, sma_last_error());
    return 1;
  }
  lnods[8 * 5 + 3] = nid(1, 1, 0);
  double dampi[2] = {0.0, 1e-6};                                /* Rayleigh beta: refused */
  mat.dampi = dampi;
  rc = sma_ctx_create(&m, &mat, &run, &ctx);
  if (rc >= 0 || !strstr(sma_last_error(), "beta")) {
    fprintf(stderr, "Rayleigh beta accepted: rc=%d (%s)\n", rc, sma_last_error());
    return 1;
  }
  if (sma_explicit_step(NULL, 1) >= 0) {                        /* destroy(NULL) is a no-op */
    fprintf(stderr, "NULL context accepted\n");
    return 1;
  }
  printf("reject ok (%s)\n", sma_version());
  return 0;
}

static int run(const char* out) {
  double coord[3 * NP], props[18], densi = 6.45e-9;
  int32_t lnods[8 * NE], fixno[3 * NP], bcfun[NP];
  mesh(coord, lnods);
  niti(props);
  for (int p = 0; p < NP; ++p) {
    fixno[3 * p] = fixno[3 * p + 1] = fixno[3 * p + 2] = 0;
    bcfun[p] = -1;
    if (coord[3 * p] == 0.0) fixno[3 * p] = fixno[3 * p + 1] = fixno[3 * p + 2] = 1;
    if (coord[3 * p] == NX) { fixno[3 * p] = 1; bcfun[p] = 0; }
  }
  /* dt = 0.5 h / c, h = 1, c^2 = (lambda + 2 mu) / rho */
  const double E = props[0], nu = props[1];
  const double lam = nu * E / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
  const double dt = 0.5 * 1.0 / sqrt((lam + 2 * mu) / densi);
  const double T = 200 * dt;
  const double tab[12] = {0.0, 0.0, 0.0, 0.0, 0.5 * T, 0.4, 0.4, 0.4, T, 0.0, 0.0, 0.0};
  const int32_t npts = 3, smooth = 1;
  sma_mesh_desc m = {NE, NP, lnods, coord, NULL};
  sma_material_desc mat = {1, props, NULL, &densi, NULL, NULL};
  sma_run_desc r;
  memset(&r, 0, sizeof r);
  r.precision = SMA_PREC_FP64;
  r.scatter = SMA_SCATTER_COLOR;
  r.nfun = 1;
  r.dtime = dt;
  r.fixno = fixno;
  r.bcfun = bcfun;
  r.fun_npts = &npts;
  r.fun_smooth = &smooth;
  r.fun_tab = tab;
  r.load_fun = -1;
  sma_ctx* ctx = NULL;
  if (sma_ctx_create(&m, &mat, &r, &ctx) != SMA_OK) {
    fprintf(stderr, "sma_ctx_create: %s\n", sma_last_error());
    return 1;
  }
  double u[3 * NP];
  int ok = sma_explicit_step(ctx, 100) == SMA_OK && sma_get_nodal(ctx, SMA_FIELD_DISPL, u) == SMA_OK;
  if (!ok) fprintf(stderr, "step: %s\n", sma_last_error());
  sma_ctx_destroy(ctx);
  if (!ok) return 1;
  FILE* f = fopen(out, "wb");
  if (!f) return 1;
  fwrite(&dt, sizeof dt, 1, f);
  fwrite(u, sizeof(double), 3 * NP, f);
  fclose(f);
  printf("run ok: dt %.17g, u_x(tip) %.17g\n", dt, u[3 * nid(NX, 1, 1)]);
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 2 && strcmp(argv[1], "reject") == 0) return reject();
  if (argc >= 3 && strcmp(argv[1], "run") == 0) return run(argv[2]);
  fprintf(stderr, "usage: %s reject | run <out.bin>\n", argv[0]);
  return 2;
}

/*
 * oracle.c - CPU restatement of the reference's matrix-free operators (TEST
 * INFRASTRUCTURE ONLY; see oracle.h for scope and parity status).
 *
 * Independent of the product: its own Lagrange basis (Vandermonde inverse in
 * double), its own collapsed Gauss-Legendre quadrature, its own geometry and
 * face adjacency, and face integrals evaluated at physical points.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXK 20
#define MAXM 20
#define MAXQ 8
#define MAXNC 3

typedef struct {
  int p, K, nmono;
  int lat[MAXK][4];
  int mono[MAXM][3];
  double coef[MAXK][MAXM]; /* phi_n = sum_m coef[n][m] mono_m */
} basis_t;

typedef struct {
  double J[3][3], Ji[3][3], det, x0[3];
} geom_t;

struct oracle_ctx {
  oracle_params prm;
  basis_t B;
  int64_t nv, nc, ndofs;
  const double* x;
  int32_t* cells;      /* copy [nc][4] */
  int32_t* cell_dofs;  /* CG copy */
  uint8_t* constrained;
  int32_t* nb;         /* [nc][4] */
  int8_t* nbf;
  geom_t* geo;
  double* tau;         /* surface/volume */
  double* ih;          /* [nc][4] |grad lambda_f| */
  double factor;
  /* cell quadrature */
  int nqc;
  double qc_w[MAXQ * MAXQ * MAXQ];
  double qc_phi[MAXQ * MAXQ * MAXQ][MAXK];
  double qc_dphi[MAXQ * MAXQ * MAXQ][MAXK][3];
  double qc_xi[MAXQ * MAXQ * MAXQ][3];
  /* curved cells: P2 geometry (edge nodes [nc][6][3]) and its gradients at the cell points */
  double* edge;
  double qc_gdphi[MAXQ * MAXQ * MAXQ][10][3];
  /* face quadrature (reference triangle s,t) */
  int nqf;
  double qf_st[MAXQ * MAXQ][2];
  double qf_w[MAXQ * MAXQ];
};

/* ---------------------------------------------------------------- basis -- */
static double ipow(double b, int e) {
  double r = 1.0;
  while (e-- > 0) r *= b;
  return r;
}

static int build_basis(int p, basis_t* B) {
  static const int E[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  int n = 0, v, e, m, f;
  if (p < 1 || p > 3) return -1;
  memset(B, 0, sizeof(*B));
  B->p = p;
  for (v = 0; v < 4; ++v) {
    B->lat[n][v] = p;
    ++n;
  }
  for (e = 0; e < 6; ++e)
    for (m = 1; m < p; ++m) {
      B->lat[n][E[e][0]] = p - m;
      B->lat[n][E[e][1]] = m;
      ++n;
    }
  if (p == 3)
    for (f = 0; f < 4; ++f) {
      for (v = 0; v < 4; ++v) B->lat[n][v] = v == f ? 0 : 1;
      ++n;
    }
  B->K = n;
  B->nmono = 0;
  for (int a = 0; a <= p; ++a)
    for (int b = 0; a + b <= p; ++b)
      for (int c = 0; a + b + c <= p; ++c) {
        B->mono[B->nmono][0] = a;
        B->mono[B->nmono][1] = b;
        B->mono[B->nmono][2] = c;
        B->nmono++;
      }
  if (B->nmono != n) return -2;
  /* V[k][m] = mono_m(node_k); coef = V^-1 transposed */
  double A[MAXK][2 * MAXK];
  for (int k = 0; k < n; ++k) {
    double xi[3] = {(double)B->lat[k][1] / p, (double)B->lat[k][2] / p, (double)B->lat[k][3] / p};
    for (m = 0; m < n; ++m)
      A[k][m] = ipow(xi[0], B->mono[m][0]) * ipow(xi[1], B->mono[m][1]) * ipow(xi[2], B->mono[m][2]);
    for (m = 0; m < n; ++m) A[k][n + m] = k == m ? 1.0 : 0.0;
  }
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    if (fabs(A[piv][c]) < 1e-14) return -3;
    if (piv != c)
      for (m = 0; m < 2 * n; ++m) {
        double t = A[c][m];
        A[c][m] = A[piv][m];
        A[piv][m] = t;
      }
    double d = A[c][c];
    for (m = 0; m < 2 * n; ++m) A[c][m] /= d;
    for (int r = 0; r < n; ++r)
      if (r != c && A[r][c] != 0.0) {
        double fac = A[r][c];
        for (m = 0; m < 2 * n; ++m) A[r][m] -= fac * A[c][m];
      }
  }
  /* inverse Vi = A[:, n:]; phi_k = sum_m Vi[m][k] mono_m */
  for (int k = 0; k < n; ++k)
    for (m = 0; m < n; ++m) B->coef[k][m] = A[m][n + k];
  return 0;
}

static void eval_basis(const basis_t* B, const double xi[3], double* val, double (*grad)[3]) {
  double pw[3][5];
  for (int d = 0; d < 3; ++d) {
    pw[d][0] = 1.0;
    for (int e = 1; e <= 4; ++e) pw[d][e] = pw[d][e - 1] * xi[d];
  }
  for (int k = 0; k < B->K; ++k) {
    double v = 0, g0 = 0, g1 = 0, g2 = 0;
    for (int m = 0; m < B->nmono; ++m) {
      const double c = B->coef[k][m];
      if (c == 0.0) continue;
      const int a = B->mono[m][0], b = B->mono[m][1], cc = B->mono[m][2];
      v += c * pw[0][a] * pw[1][b] * pw[2][cc];
      if (a) g0 += c * a * pw[0][a - 1] * pw[1][b] * pw[2][cc];
      if (b) g1 += c * b * pw[0][a] * pw[1][b - 1] * pw[2][cc];
      if (cc) g2 += c * cc * pw[0][a] * pw[1][b] * pw[2][cc - 1];
    }
    if (val) val[k] = v;
    if (grad) {
      grad[k][0] = g0;
      grad[k][1] = g1;
      grad[k][2] = g2;
    }
  }
}

int oracle_basis(int32_t degree, const double* xi, double* values, double* grads) {
  basis_t B;
  if (build_basis(degree, &B)) return -1;
  eval_basis(&B, xi, values, (double(*)[3])grads);
  return 0;
}

/* ----------------------------------------------------------- quadrature -- */
/* Gauss-Legendre on [0,1], Newton on the Legendre three-term recurrence. */
static void gauss_legendre01(int n, double* t, double* w) {
  for (int i = 0; i < n; ++i) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (n == 1) {
        p1 = z;
        p0 = 1.0;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (n == 1) p0 = 1.0;
      dp = n * (z * p1 - p0) / (z * z - 1.0);
    }
    t[i] = 0.5 * (1.0 - z);
    w[i] = 1.0 / ((1.0 - z * z) * dp * dp); /* 2/((1-z^2)p'^2) scaled by 1/2 */
  }
}

static void build_quadrature(oracle_ctx* ctx) {
  int n = ctx->prm.quad_points > 0 ? ctx->prm.quad_points : ctx->prm.degree + 2;
  if (n > MAXQ) n = MAXQ;
  double t[MAXQ], w[MAXQ];
  gauss_legendre01(n, t, w);
  int q = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b)
      for (int c = 0; c < n; ++c) {
        const double u = t[a], v = t[b], s = t[c];
        double xi[3] = {u, v * (1 - u), s * (1 - u) * (1 - v)};
        ctx->qc_xi[q][0] = xi[0];
        ctx->qc_xi[q][1] = xi[1];
        ctx->qc_xi[q][2] = xi[2];
        ctx->qc_w[q] = w[a] * w[b] * w[c] * (1 - u) * (1 - u) * (1 - v);
        eval_basis(&ctx->B, xi, ctx->qc_phi[q], ctx->qc_dphi[q]);
        ++q;
      }
  ctx->nqc = q;
  q = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      ctx->qf_st[q][0] = t[a];
      ctx->qf_st[q][1] = t[b] * (1 - t[a]);
      ctx->qf_w[q] = w[a] * w[b] * (1 - t[a]);
      ++q;
    }
  ctx->nqf = q;
}

int oracle_set_p2_geometry(oracle_ctx* ctx, const double* edge_nodes) {
  if (!ctx || !edge_nodes || ctx->prm.kind != ORACLE_CG) return -1;
  basis_t G2;
  if (build_basis(2, &G2)) return -3;
  free(ctx->edge);
  ctx->edge = (double*)malloc(sizeof(double) * 18 * ctx->nc);
  if (!ctx->edge) return -2;
  memcpy(ctx->edge, edge_nodes, sizeof(double) * 18 * ctx->nc);
  for (int q = 0; q < ctx->nqc; ++q) eval_basis(&G2, ctx->qc_xi[q], NULL, ctx->qc_gdphi[q]);
  return 0;
}

int oracle_quadrature_sizes(const oracle_ctx* ctx, int32_t* nc, int32_t* nf) {
  if (nc) *nc = ctx->nqc;
  if (nf) *nf = ctx->nqf;
  return 0;
}

/* --------------------------------------------------------------- geometry -- */
static void invert_jacobian(geom_t* g);

static void set_jacobian(geom_t* g, const double J[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) g->J[i][j] = J[i][j];
  invert_jacobian(g);
}

static void make_geom(const double* x, const int32_t* cv, geom_t* g) {
  const double* x0 = x + 3 * (int64_t)cv[0];
  for (int d = 0; d < 3; ++d) g->x0[d] = x0[d];
  for (int j = 0; j < 3; ++j) {
    const double* xj = x + 3 * (int64_t)cv[j + 1];
    for (int i = 0; i < 3; ++i) g->J[i][j] = xj[i] - x0[i];
  }
  invert_jacobian(g);
}

static void invert_jacobian(geom_t* g) {
  double(*J)[3] = g->J;
  double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  g->det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  double id = 1.0 / g->det;
  g->Ji[0][0] = c00 * id;
  g->Ji[1][0] = c01 * id;
  g->Ji[2][0] = c02 * id;
  g->Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  g->Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  g->Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  g->Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  g->Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  g->Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
}

/* grad_x phi = J^-T grad_xi phi */
static void push_grad(const geom_t* g, const double gr[3], double out[3]) {
  for (int i = 0; i < 3; ++i) out[i] = g->Ji[0][i] * gr[0] + g->Ji[1][i] * gr[1] + g->Ji[2][i] * gr[2];
}

static void to_ref(const geom_t* g, const double X[3], double xi[3]) {
  double d[3] = {X[0] - g->x0[0], X[1] - g->x0[1], X[2] - g->x0[2]};
  for (int i = 0; i < 3; ++i) xi[i] = g->Ji[i][0] * d[0] + g->Ji[i][1] * d[1] + g->Ji[i][2] * d[2];
}

static void face_frame(const oracle_ctx* ctx, int64_t c, int f, double P0[3], double E1[3], double E2[3],
                       double n[3], double* area) {
  const int32_t* cv = ctx->cells + 4 * c;
  int lv[3], q = 0;
  for (int v = 0; v < 4; ++v)
    if (v != f) lv[q++] = v;
  const double* a = ctx->x + 3 * (int64_t)cv[lv[0]];
  const double* b = ctx->x + 3 * (int64_t)cv[lv[1]];
  const double* cc = ctx->x + 3 * (int64_t)cv[lv[2]];
  const double* o = ctx->x + 3 * (int64_t)cv[f];
  for (int d = 0; d < 3; ++d) {
    P0[d] = a[d];
    E1[d] = b[d] - a[d];
    E2[d] = cc[d] - a[d];
  }
  double cr[3] = {E1[1] * E2[2] - E1[2] * E2[1], E1[2] * E2[0] - E1[0] * E2[2], E1[0] * E2[1] - E1[1] * E2[0]};
  double len = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
  double dot = cr[0] * (o[0] - a[0]) + cr[1] * (o[1] - a[1]) + cr[2] * (o[2] - a[2]);
  double s = dot > 0 ? -1.0 / len : 1.0 / len;
  for (int d = 0; d < 3; ++d) n[d] = cr[d] * s;
  *area = 0.5 * len;
}

typedef struct {
  int32_t v[3];
  int64_t cf; /* 4*c+f */
} facekey_t;

static int cmp_face(const void* a, const void* b) {
  const facekey_t* x = (const facekey_t*)a;
  const facekey_t* y = (const facekey_t*)b;
  for (int i = 0; i < 3; ++i)
    if (x->v[i] != y->v[i]) return x->v[i] < y->v[i] ? -1 : 1;
  return x->cf < y->cf ? -1 : (x->cf > y->cf);
}

static void sort3(int32_t* v) {
  int32_t t;
  if (v[0] > v[1]) { t = v[0]; v[0] = v[1]; v[1] = t; }
  if (v[1] > v[2]) { t = v[1]; v[1] = v[2]; v[2] = t; }
  if (v[0] > v[1]) { t = v[0]; v[0] = v[1]; v[1] = t; }
}

/* ------------------------------------------------------------------ ctx -- */
int oracle_create(const oracle_params* prm, int64_t nv, const double* x, int64_t nc, const int32_t* cells,
                  const int32_t* cell_dofs, const uint8_t* constrained, int64_t n_dofs, oracle_ctx** out) {
  if (!prm || !x || !cells || !out) return -1;
  oracle_ctx* ctx = (oracle_ctx*)calloc(1, sizeof(oracle_ctx));
  if (!ctx) return -2;
  ctx->prm = *prm;
  if (ctx->prm.n_components < 1) ctx->prm.n_components = 1;
  if (ctx->prm.n_components > MAXNC || build_basis(prm->degree, &ctx->B)) {
    free(ctx);
    return -3;
  }
  const int K = ctx->B.K, p = prm->degree;
  ctx->nv = nv;
  ctx->nc = nc;
  ctx->x = x;
  ctx->cells = (int32_t*)malloc(sizeof(int32_t) * 4 * nc);
  memcpy(ctx->cells, cells, sizeof(int32_t) * 4 * nc);
  if (prm->kind == ORACLE_CG) {
    if (!cell_dofs || !constrained) {
      oracle_destroy(ctx);
      return -4;
    }
    ctx->ndofs = n_dofs;
    ctx->cell_dofs = (int32_t*)malloc(sizeof(int32_t) * K * nc);
    memcpy(ctx->cell_dofs, cell_dofs, sizeof(int32_t) * K * nc);
    ctx->constrained = (uint8_t*)malloc(n_dofs);
    if (prm->weak_bc)
      memset(ctx->constrained, 0, n_dofs); /* the boundary is imposed weakly */
    else
      memcpy(ctx->constrained, constrained, n_dofs);
  } else {
    ctx->ndofs = (int64_t)K * ctx->prm.n_components * nc;
  }
  ctx->geo = (geom_t*)malloc(sizeof(geom_t) * nc);
  for (int64_t c = 0; c < nc; ++c) make_geom(x, cells + 4 * c, &ctx->geo[c]);
  /* adjacency by sorting face keys */
  ctx->nb = (int32_t*)malloc(sizeof(int32_t) * 4 * nc);
  ctx->nbf = (int8_t*)malloc(4 * nc);
  facekey_t* fk = (facekey_t*)malloc(sizeof(facekey_t) * 4 * nc);
  for (int64_t c = 0; c < nc; ++c)
    for (int f = 0; f < 4; ++f) {
      facekey_t* k = fk + 4 * c + f;
      int q = 0;
      for (int v = 0; v < 4; ++v)
        if (v != f) k->v[q++] = cells[4 * c + v];
      sort3(k->v);
      k->cf = 4 * c + f;
      ctx->nb[4 * c + f] = -1;
      ctx->nbf[4 * c + f] = -1;
    }
  qsort(fk, 4 * nc, sizeof(facekey_t), cmp_face);
  for (int64_t i = 0; i + 1 < 4 * nc; ++i)
    if (fk[i].v[0] == fk[i + 1].v[0] && fk[i].v[1] == fk[i + 1].v[1] && fk[i].v[2] == fk[i + 1].v[2]) {
      const int64_t a = fk[i].cf, b = fk[i + 1].cf;
      ctx->nb[a] = (int32_t)(b / 4);
      ctx->nbf[a] = (int8_t)(b % 4);
      ctx->nb[b] = (int32_t)(a / 4);
      ctx->nbf[b] = (int8_t)(a % 4);
      ++i;
    }
  free(fk);
  /* penalty ingredients */
  ctx->tau = (double*)malloc(sizeof(double) * nc);
  ctx->ih = (double*)malloc(sizeof(double) * 4 * nc);
  static const double gl[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int64_t c = 0; c < nc; ++c) {
    double vol = fabs(ctx->geo[c].det) / 6.0, surf = 0;
    for (int f = 0; f < 4; ++f) {
      double P0[3], E1[3], E2[3], n[3], area;
      face_frame(ctx, c, f, P0, E1, E2, n, &area);
      surf += area * (ctx->nb[4 * c + f] < 0 ? 1.0 : 0.5);
      double gx[3];
      push_grad(&ctx->geo[c], gl[f], gx);
      ctx->ih[4 * c + f] = sqrt(gx[0] * gx[0] + gx[1] * gx[1] + gx[2] * gx[2]);
    }
    ctx->tau[c] = surf / vol;
  }
  ctx->factor = prm->penalty == 1 ? (double)((p + 1) * (p + 1)) : (double)((p + 1) * (p + 3)) / 3.0;
  build_quadrature(ctx);
  *out = ctx;
  return 0;
}

void oracle_destroy(oracle_ctx* ctx) {
  if (!ctx) return;
  free(ctx->cells);
  free(ctx->cell_dofs);
  free(ctx->constrained);
  free(ctx->nb);
  free(ctx->nbf);
  free(ctx->geo);
  free(ctx->tau);
  free(ctx->edge);
  free(ctx->ih);
  free(ctx);
}

int64_t oracle_n_dofs(const oracle_ctx* ctx) { return ctx->ndofs; }

/* Own-side contributions of cell c: y[comp][i] for the local values u
 * (and neighbour values read from src unless src == NULL). */
static void cell_apply(const oracle_ctx* ctx, int64_t c, const double* u /* [nc][K] */, const double* src,
                       double* y /* [nc][K] */) {
  const basis_t* B = &ctx->B;
  const int K = B->K, NC = ctx->prm.n_components;
  const geom_t* g = &ctx->geo[c];
  const double adet = fabs(g->det);
  const int dg = ctx->prm.kind != ORACLE_CG;
  const int helm = ctx->prm.kind == ORACLE_HELMHOLTZ;
  memset(y, 0, sizeof(double) * K * NC);
  /* cell term */
  for (int q = 0; q < ctx->nqc; ++q) {
    double W = ctx->qc_w[q] * adet;
    double gphi[MAXK][3];
    if (ctx->edge) {
      /* curved cell: Jacobian of the quadratic geometry at this point */
      geom_t gq;
      const double* X[10];
      for (int v = 0; v < 4; ++v) X[v] = ctx->x + 3 * (int64_t)ctx->cells[4 * c + v];
      for (int e = 0; e < 6; ++e) X[4 + e] = ctx->edge + 18 * c + 3 * e;
      double J[3][3] = {{0}};
      for (int k = 0; k < 10; ++k)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) J[i][j] += X[k][i] * ctx->qc_gdphi[q][k][j];
      set_jacobian(&gq, J);
      W = ctx->qc_w[q] * fabs(gq.det);
      for (int i = 0; i < K; ++i) push_grad(&gq, ctx->qc_dphi[q][i], gphi[i]);
    } else {
      for (int i = 0; i < K; ++i) push_grad(g, ctx->qc_dphi[q][i], gphi[i]);
    }
    for (int comp = 0; comp < NC; ++comp) {
      const double* uc = u + comp * K;
      double gu[3] = {0, 0, 0}, val = 0;
      for (int i = 0; i < K; ++i) {
        gu[0] += uc[i] * gphi[i][0];
        gu[1] += uc[i] * gphi[i][1];
        gu[2] += uc[i] * gphi[i][2];
        val += uc[i] * ctx->qc_phi[q][i];
      }
      for (int i = 0; i < K; ++i) {
        double r = W * (gu[0] * gphi[i][0] + gu[1] * gphi[i][1] + gu[2] * gphi[i][2]);
        if (helm) r += ctx->prm.mass * W * val * ctx->qc_phi[q][i];
        y[comp * K + i] += r;
      }
    }
  }
  if (!dg && !ctx->prm.weak_bc) return;
  /* face terms, own side (weak CG: the boundary faces only) */
  for (int f = 0; f < 4; ++f) {
    const int32_t nbc = ctx->nb[4 * c + f];
    if (!dg && nbc >= 0) continue;
    double P0[3], E1[3], E2[3], n[3], area;
    face_frame(ctx, c, f, P0, E1, E2, n, &area);
    double sigma;
    if (helm)
      sigma = nbc >= 0 ? ctx->factor * 0.5 * (ctx->ih[4 * c + f] + ctx->ih[4 * (int64_t)nbc + ctx->nbf[4 * c + f]])
                       : ctx->factor * ctx->ih[4 * c + f];
    else
      sigma = nbc >= 0 ? ctx->factor * (ctx->tau[c] > ctx->tau[nbc] ? ctx->tau[c] : ctx->tau[nbc])
                       : ctx->factor * ctx->tau[c];
    const geom_t* gn = nbc >= 0 ? &ctx->geo[nbc] : NULL;
    for (int q = 0; q < ctx->nqf; ++q) {
      const double s = ctx->qf_st[q][0], t = ctx->qf_st[q][1];
      const double W = ctx->qf_w[q] * 2.0 * area;
      double X[3], xi[3], phi[MAXK], dphi[MAXK][3], gphi[MAXK][3], dn[MAXK];
      for (int d = 0; d < 3; ++d) X[d] = P0[d] + s * E1[d] + t * E2[d];
      to_ref(g, X, xi);
      eval_basis(B, xi, phi, dphi);
      for (int i = 0; i < K; ++i) {
        push_grad(g, dphi[i], gphi[i]);
        dn[i] = gphi[i][0] * n[0] + gphi[i][1] * n[1] + gphi[i][2] * n[2];
      }
      double phin[MAXK], dnn[MAXK];
      if (gn && src) {
        double xin[3], dphin[MAXK][3], gpn[3];
        to_ref(gn, X, xin);
        eval_basis(B, xin, phin, dphin);
        for (int i = 0; i < K; ++i) {
          push_grad(gn, dphin[i], gpn);
          dnn[i] = gpn[0] * n[0] + gpn[1] * n[1] + gpn[2] * n[2];
        }
      }
      for (int comp = 0; comp < NC; ++comp) {
        const double* uc = u + comp * K;
        double um = 0, dum = 0;
        for (int i = 0; i < K; ++i) {
          um += uc[i] * phi[i];
          dum += uc[i] * dn[i];
        }
        double jump, avg;
        if (nbc >= 0) {
          double up = 0, dup = 0;
          if (src) {
            const double* un = src + ((int64_t)nbc * NC + comp) * K;
            for (int i = 0; i < K; ++i) {
              up += un[i] * phin[i];
              dup += un[i] * dnn[i];
            }
          }
          jump = um - up;
          avg = 0.5 * (dum + dup);
        } else {
          jump = 2.0 * um;
          avg = dum;
        }
        const double tv = sigma * jump - avg;
        for (int i = 0; i < K; ++i) y[comp * K + i] += W * (tv * phi[i] - 0.5 * jump * dn[i]);
      }
    }
  }
}

int oracle_vmult(oracle_ctx* ctx, const double* src, double* dst) {
  return oracle_vmult_cells(ctx, src, dst, 0, ctx->nc);
}

int oracle_vmult_cells(oracle_ctx* ctx, const double* src, double* dst, int64_t c0, int64_t c1) {
  const int K = ctx->B.K, NC = ctx->prm.n_components;
  const int cg = ctx->prm.kind == ORACLE_CG;
  const int nt = ctx->prm.n_threads;
  if (c0 < 0 || c1 > ctx->nc || c0 > c1) return -1;
  if (cg) memset(dst, 0, sizeof(double) * ctx->ndofs);
#pragma omp parallel num_threads(nt > 0 ? nt : omp_get_max_threads())
  {
    double u[MAXK * MAXNC], y[MAXK * MAXNC];
#pragma omp for schedule(static)
    for (int64_t c = c0; c < c1; ++c) {
      if (cg) {
        for (int i = 0; i < K; ++i) {
          const int32_t gi = ctx->cell_dofs[K * c + i];
          u[i] = ctx->constrained[gi] ? 0.0 : src[gi];
        }
        cell_apply(ctx, c, u, src, y);
        for (int i = 0; i < K; ++i) {
          const int32_t gi = ctx->cell_dofs[K * c + i];
          if (!ctx->constrained[gi]) {
#pragma omp atomic
            dst[gi] += y[i];
          }
        }
      } else {
        memcpy(u, src + c * NC * K, sizeof(double) * NC * K);
        cell_apply(ctx, c, u, src, y);
        memcpy(dst + c * NC * K, y, sizeof(double) * NC * K);
      }
    }
  }
  if (cg)
    for (int64_t i = 0; i < ctx->ndofs; ++i)
      if (ctx->constrained[i]) dst[i] = src[i];
  return 0;
}

int oracle_cell_matrix(oracle_ctx* ctx, int64_t c, double* mat) {
  const int K = ctx->B.K, NC = ctx->prm.n_components, n = K * NC;
  double u[MAXK * MAXNC], y[MAXK * MAXNC];
  for (int j = 0; j < n; ++j) {
    memset(u, 0, sizeof(u));
    u[j] = 1.0;
    cell_apply(ctx, c, u, NULL, y);
    for (int i = 0; i < n; ++i) mat[i * n + j] = y[i];
  }
  return 0;
}

int oracle_diagonal(oracle_ctx* ctx, double* diag) {
  const int K = ctx->B.K, NC = ctx->prm.n_components, n = K * NC;
  const int cg = ctx->prm.kind == ORACLE_CG;
  memset(diag, 0, sizeof(double) * ctx->ndofs);
  double* mat = (double*)malloc(sizeof(double) * n * n);
  for (int64_t c = 0; c < ctx->nc; ++c) {
    oracle_cell_matrix(ctx, c, mat);
    for (int i = 0; i < n; ++i) {
      if (cg) {
        const int32_t gi = ctx->cell_dofs[K * c + i];
        if (!ctx->constrained[gi]) diag[gi] += mat[i * n + i];
      } else {
        diag[c * n + i] = mat[i * n + i];
      }
    }
  }
  free(mat);
  if (cg)
    for (int64_t i = 0; i < ctx->ndofs; ++i)
      if (ctx->constrained[i]) diag[i] = 1.0;
  return 0;
}

int64_t oracle_check_cg_numbering(oracle_ctx* ctx, const double* lo, const double* hi) {
  if (ctx->prm.kind != ORACLE_CG) return -1;
  const int K = ctx->B.K, p = ctx->B.p;
  double* pos = (double*)malloc(sizeof(double) * 3 * ctx->ndofs);
  uint8_t* seen = (uint8_t*)calloc(ctx->ndofs, 1);
  int64_t bad = 0;
  for (int64_t c = 0; c < ctx->nc; ++c) {
    const int32_t* cv = ctx->cells + 4 * c;
    for (int i = 0; i < K; ++i) {
      double X[3] = {0, 0, 0};
      for (int v = 0; v < 4; ++v)
        for (int d = 0; d < 3; ++d) X[d] += ctx->B.lat[i][v] * ctx->x[3 * (int64_t)cv[v] + d] / p;
      const int32_t gi = ctx->cell_dofs[K * c + i];
      if (gi < 0 || gi >= ctx->ndofs) {
        ++bad;
        continue;
      }
      if (!seen[gi]) {
        seen[gi] = 1;
        memcpy(pos + 3 * (int64_t)gi, X, sizeof(X));
      } else {
        for (int d = 0; d < 3; ++d)
          if (fabs(pos[3 * (int64_t)gi + d] - X[d]) > 1e-12) {
            ++bad;
            break;
          }
      }
    }
  }
  for (int64_t i = 0; i < ctx->ndofs; ++i) {
    if (!seen[i]) {
      ++bad;
      continue;
    }
    int onb = 0;
    for (int d = 0; d < 3; ++d)
      if (fabs(pos[3 * i + d] - lo[d]) < 1e-12 || fabs(pos[3 * i + d] - hi[d]) < 1e-12) onb = 1;
    if (onb != (ctx->constrained[i] != 0)) ++bad;
  }
  free(pos);
  free(seen);
  return bad;
}

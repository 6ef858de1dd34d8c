/*
 * mesh.c - the benchmark meshes and CG numbering, restated for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  This is an independent statement
 * of the mesh recipe the benchmark configurations name, so that the CPU
 * baseline and the parity tests do not have to take the mesh from the
 * product library, and so that the product's mesh generator can be checked
 * bit for bit against it:
 *
 *   - an n[0] x n[1] x n[2] box of hexes, each cut into the 6 Kuhn
 *     (Freudenthal) tetrahedra that share its main diagonal (the 6 monotone
 *     lattice paths from the hex's lowest to its highest corner).  It stands
 *     in for GridGenerator::subdivided_hyper_cube_with_simplices +
 *     refine_global (CG/cells_batched/application.cc:1762-1770);
 *   - vertices numbered lexicographically (x fastest); when jitter > 0 every
 *     vertex draws 3 numbers u in [0,1) from one MT19937-64 stream seeded with
 *     `seed` (u = top 53 bits / 2^53), and interior vertices move by
 *     (2u - 1) * jitter * h per axis;
 *   - hexes in Morton (Z-curve) order of (i,j,k) with i in the lowest bit,
 *     the 6 tets of a hex contiguous, in lexicographic order of the axis
 *     permutation of their lattice path; every tet lists its vertices in
 *     ascending global id.  This plays the role of the reference's z-order
 *     partition and DoFRenumbering::matrix_free_data_locality
 *     (CG/cells_batched/application.cc:1773-1780,1828);
 *   - face neighbours by sorting all (cell, local face) records on their
 *     vertex triple;
 *   - the continuous P_p numbering in first-touch order over cells and local
 *     nodes (vertices, edges (0,1),(0,2),(0,3),(1,2),(1,3),(2,3) walked from
 *     the lower local vertex, then faces), with every node on a boundary face
 *     constrained (homogeneous Dirichlet, the reference's
 *     VectorTools::interpolate_boundary_values + masked gather,
 *     CG/cells_batched/application.cc:1809-1838).
 *
 * MT19937-64 follows the published generator of Matsumoto and Nishimura
 * (the 64-bit Mersenne Twister, also std::mt19937_64).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---- MT19937-64 --------------------------------------------------------- */
typedef struct {
  uint64_t s[312];
  int i;
} mt64;

static void mt64_seed(mt64* g, uint64_t seed) {
  g->s[0] = seed;
  for (int k = 1; k < 312; ++k) g->s[k] = 6364136223846793005ULL * (g->s[k - 1] ^ (g->s[k - 1] >> 62)) + (uint64_t)k;
  g->i = 312;
}

static uint64_t mt64_next(mt64* g) {
  const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL, a = 0xB5026F5AA96619E9ULL;
  if (g->i >= 312) {
    for (int k = 0; k < 312; ++k) {
      const uint64_t y = (g->s[k] & upper) | (g->s[(k + 1) % 312] & lower);
      g->s[k] = g->s[(k + 156) % 312] ^ (y >> 1) ^ ((y & 1) ? a : 0);
    }
    g->i = 0;
  }
  uint64_t x = g->s[g->i++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= x >> 43;
  return x;
}

/* ---- Kuhn mesh ------------------------------------------------------------ */
static uint64_t z_order(uint64_t i, uint64_t j, uint64_t k) {
  uint64_t key = 0;
  for (int b = 0; b < 21; ++b) {
    key |= ((i >> b) & 1) << (3 * b);
    key |= ((j >> b) & 1) << (3 * b + 1);
    key |= ((k >> b) & 1) << (3 * b + 2);
  }
  return key;
}

typedef struct {
  uint64_t key;
  int64_t lin;
} hex_rec;

static int cmp_hex(const void* a, const void* b) {
  const hex_rec* x = (const hex_rec*)a;
  const hex_rec* y = (const hex_rec*)b;
  return x->key < y->key ? -1 : x->key > y->key;
}

typedef struct {
  int32_t v[3];
  int32_t cell;
  int8_t f;
} face_rec;

static int cmp_face(const void* a, const void* b) {
  const face_rec* x = (const face_rec*)a;
  const face_rec* y = (const face_rec*)b;
  for (int q = 0; q < 3; ++q)
    if (x->v[q] != y->v[q]) return x->v[q] < y->v[q] ? -1 : 1;
  return 0;
}

static void sort4(int32_t* v) {
  for (int a = 1; a < 4; ++a) {
    const int32_t t = v[a];
    int b = a - 1;
    while (b >= 0 && v[b] > t) {
      v[b + 1] = v[b];
      --b;
    }
    v[b + 1] = t;
  }
}

int oracle_kuhn_mesh(const int32_t n[3], const double lo[3], const double hi[3], double jitter, uint64_t seed,
                     double* x, int32_t* cells, int32_t* nb, int8_t* nbf) {
  for (int a = 0; a < 3; ++a)
    if (n[a] < 1 || !(hi[a] > lo[a])) return 1;
  const int64_t nx = n[0], ny = n[1], nz = n[2];
  const int64_t vx = nx + 1, vy = ny + 1;
  double h[3];
  for (int a = 0; a < 3; ++a) h[a] = (hi[a] - lo[a]) / n[a];

  mt64 g;
  mt64_seed(&g, seed);
  for (int64_t k = 0; k <= nz; ++k)
    for (int64_t j = 0; j <= ny; ++j)
      for (int64_t i = 0; i <= nx; ++i) {
        const int64_t v = i + vx * (j + vy * k);
        const int64_t ijk[3] = {i, j, k};
        const int inside = i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz;
        for (int a = 0; a < 3; ++a) {
          double pos = lo[a] + (double)ijk[a] * h[a];
          if (jitter > 0) {
            const double u = (double)(mt64_next(&g) >> 11) / 9007199254740992.0;
            if (inside) pos += (2.0 * u - 1.0) * jitter * h[a];
          }
          x[3 * v + a] = pos;
        }
      }

  const int64_t n_hex = nx * ny * nz;
  hex_rec* hx = (hex_rec*)malloc(sizeof(hex_rec) * (size_t)n_hex);
  if (!hx) return 2;
  int64_t q = 0;
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        hx[q].key = z_order((uint64_t)i, (uint64_t)j, (uint64_t)k);
        hx[q].lin = i + nx * (j + ny * k);
        ++q;
      }
  qsort(hx, (size_t)n_hex, sizeof(hex_rec), cmp_hex);

  /* lattice paths 000 -> 111: the axes taken in order (a0, a1, a2), the 6
   * permutations in lexicographic order */
  static const int path[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  int64_t c = 0;
  for (int64_t t = 0; t < n_hex; ++t) {
    const int64_t lin = hx[t].lin;
    const int64_t i = lin % nx, j = (lin / nx) % ny, k = lin / (nx * ny);
    for (int p = 0; p < 6; ++p) {
      int64_t at[3] = {i, j, k};
      int32_t vs[4];
      vs[0] = (int32_t)(at[0] + vx * (at[1] + vy * at[2]));
      for (int s = 0; s < 3; ++s) {
        at[path[p][s]] += 1;
        vs[s + 1] = (int32_t)(at[0] + vx * (at[1] + vy * at[2]));
      }
      sort4(vs);
      memcpy(cells + 4 * c, vs, sizeof vs);
      ++c;
    }
  }
  free(hx);

  const int64_t n_cells = c;
  face_rec* fr = (face_rec*)malloc(sizeof(face_rec) * (size_t)(4 * n_cells));
  if (!fr) return 2;
  for (int64_t cc = 0; cc < n_cells; ++cc)
    for (int f = 0; f < 4; ++f) {
      face_rec* r = &fr[4 * cc + f];
      int m = 0;
      for (int v = 0; v < 4; ++v)
        if (v != f) r->v[m++] = cells[4 * cc + v];
      r->cell = (int32_t)cc;
      r->f = (int8_t)f;
      nb[4 * cc + f] = -1;
      nbf[4 * cc + f] = -1;
    }
  qsort(fr, (size_t)(4 * n_cells), sizeof(face_rec), cmp_face);
  for (int64_t r = 0; r + 1 < 4 * n_cells; ++r)
    if (cmp_face(&fr[r], &fr[r + 1]) == 0) {
      const face_rec* a = &fr[r];
      const face_rec* b = &fr[r + 1];
      nb[4 * (int64_t)a->cell + a->f] = b->cell;
      nbf[4 * (int64_t)a->cell + a->f] = b->f;
      nb[4 * (int64_t)b->cell + b->f] = a->cell;
      nbf[4 * (int64_t)b->cell + b->f] = a->f;
      ++r;
    }
  free(fr);
  return 0;
}

/* ---- continuous P_p numbering --------------------------------------------- */
typedef struct {
  int32_t a, b, c; /* sorted global vertex ids (c = -1 for edges) */
  int64_t slot;    /* 6 c + e (edges) or 4 c + f (faces) */
} ent_rec;

static int cmp_ent(const void* x, const void* y) {
  const ent_rec* p = (const ent_rec*)x;
  const ent_rec* q = (const ent_rec*)y;
  if (p->a != q->a) return p->a < q->a ? -1 : 1;
  if (p->b != q->b) return p->b < q->b ? -1 : 1;
  if (p->c != q->c) return p->c < q->c ? -1 : 1;
  return 0;
}

/* ids of the distinct entities listed in recs, written to id[slot] */
static int64_t entity_ids(ent_rec* recs, int64_t n, int32_t* id) {
  qsort(recs, (size_t)n, sizeof(ent_rec), cmp_ent);
  int64_t next = -1;
  for (int64_t r = 0; r < n; ++r) {
    if (r == 0 || cmp_ent(&recs[r - 1], &recs[r]) != 0) ++next;
    id[recs[r].slot] = (int32_t)next;
  }
  return next + 1;
}

static const int kEdge[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

int64_t oracle_cg_numbering(int64_t n_vertices, int64_t n_cells, const int32_t* cells, const int32_t* nb,
                            int32_t degree, int32_t* cell_dofs, uint8_t* constrained) {
  if (degree < 1 || degree > 3) return -1;
  const int p = degree;
  const int K = (p + 1) * (p + 2) * (p + 3) / 6;
  /* local node -> (kind, entity, offset): vertices, edges, faces */
  int kind[20], ent[20], off[20];
  int q = 0;
  for (int v = 0; v < 4; ++v, ++q) { kind[q] = 0; ent[q] = v; off[q] = 0; }
  for (int e = 0; e < 6; ++e)
    for (int m = 1; m < p; ++m, ++q) { kind[q] = 1; ent[q] = e; off[q] = m - 1; }
  if (p == 3)
    for (int f = 0; f < 4; ++f, ++q) { kind[q] = 2; ent[q] = f; off[q] = 0; }
  if (q != K) return -1;

  int32_t* edge_id = (int32_t*)malloc(sizeof(int32_t) * (size_t)(6 * n_cells));
  int32_t* face_id = (int32_t*)malloc(sizeof(int32_t) * (size_t)(4 * n_cells));
  ent_rec* recs = (ent_rec*)malloc(sizeof(ent_rec) * (size_t)(6 * n_cells));
  if (!edge_id || !face_id || !recs) {
    free(edge_id); free(face_id); free(recs);
    return -2;
  }
  for (int64_t c = 0; c < n_cells; ++c)
    for (int e = 0; e < 6; ++e) {
      ent_rec* r = &recs[6 * c + e];
      r->a = cells[4 * c + kEdge[e][0]];
      r->b = cells[4 * c + kEdge[e][1]];
      r->c = -1;
      r->slot = 6 * c + e;
    }
  const int64_t n_edges = entity_ids(recs, 6 * n_cells, edge_id);
  for (int64_t c = 0; c < n_cells; ++c)
    for (int f = 0; f < 4; ++f) {
      ent_rec* r = &recs[4 * c + f];
      int32_t w[3];
      int m = 0;
      for (int v = 0; v < 4; ++v)
        if (v != f) w[m++] = cells[4 * c + v];
      r->a = w[0]; r->b = w[1]; r->c = w[2];
      r->slot = 4 * c + f;
    }
  const int64_t n_faces = entity_ids(recs, 4 * n_cells, face_id);
  free(recs);

  int32_t* vfirst = (int32_t*)malloc(sizeof(int32_t) * (size_t)n_vertices);
  int32_t* efirst = (int32_t*)malloc(sizeof(int32_t) * (size_t)n_edges);
  int32_t* ffirst = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n_faces > 0 ? n_faces : 1));
  if (!vfirst || !efirst || !ffirst) {
    free(edge_id); free(face_id); free(vfirst); free(efirst); free(ffirst);
    return -2;
  }
  for (int64_t v = 0; v < n_vertices; ++v) vfirst[v] = -1;
  for (int64_t e = 0; e < n_edges; ++e) efirst[e] = -1;
  for (int64_t f = 0; f < n_faces; ++f) ffirst[f] = -1;
  int64_t next = 0;
  for (int64_t c = 0; c < n_cells; ++c)
    for (int i = 0; i < K; ++i) {
      int32_t* first;
      int width;
      if (kind[i] == 0) { first = &vfirst[cells[4 * c + ent[i]]]; width = 1; }
      else if (kind[i] == 1) { first = &efirst[edge_id[6 * c + ent[i]]]; width = p - 1; }
      else { first = &ffirst[face_id[4 * c + ent[i]]]; width = 1; }
      if (*first < 0) {
        *first = (int32_t)next;
        next += width;
      }
      if (cell_dofs) cell_dofs[K * c + i] = *first + off[i];
    }
  if (constrained && cell_dofs) {
    memset(constrained, 0, (size_t)next);
    for (int64_t c = 0; c < n_cells; ++c)
      for (int f = 0; f < 4; ++f) {
        if (nb[4 * c + f] >= 0) continue;
        /* the nodes of face f are those not involving local vertex f */
        for (int i = 0; i < K; ++i) {
          const int on_face = kind[i] == 0 ? ent[i] != f
                              : kind[i] == 1 ? (kEdge[ent[i]][0] != f && kEdge[ent[i]][1] != f)
                                             : ent[i] == f;
          if (on_face) constrained[cell_dofs[K * c + i]] = 1;
        }
      }
  }
  free(edge_id); free(face_id); free(vfirst); free(efirst); free(ffirst);
  return next;
}

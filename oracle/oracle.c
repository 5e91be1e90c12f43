/*
 * oracle.c -- CPU restatement (FP64) of upstream dip-fmm's static-geometry
 * uniform-octree evaluation, UniformFmm::evaluate.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only as the checker.
 * The product (dip-fmm_b200/) never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here
 * against golden vectors produced by the upstream reference itself
 * (tests/golden/make_golden.py, built from the reference sources by
 * oracle/ref.mk).
 *
 * Each function cites the upstream file:line it restates.  Plain C99 +
 * optional OpenMP; physical units and FP64 throughout (the reference's FP64
 * CpuReference path).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_INV_4PI (1.0 / (4.0 * 3.14159265358979323846))
#define ORACLE_TOL 1.0e-12 /* uniform_tree.cpp:22 */

/* ------------------------------------------------------------------ basis */
/* include/cdfmm/multi_index.hpp:62-71: degree, then alpha_x, then alpha_y. */
int oracle_basis_size(int p) { return p < 0 ? 0 : (p + 1) * (p + 2) * (p + 3) / 6; }

void oracle_basis(int p, int *abc) {
  int i = 0;
  for (int d = 0; d <= p; ++d)
    for (int a = 0; a <= d; ++a)
      for (int b = 0; a + b <= d; ++b) {
        abc[3 * i] = a;
        abc[3 * i + 1] = b;
        abc[3 * i + 2] = d - a - b;
        ++i;
      }
}

static int rank3(int a, int b, int c) {
  const int d = a + b + c;
  return d * (d + 1) * (d + 2) / 6 + a * (d + 1) - a * (a - 1) / 2 + b;
}

static double fact(int n) {
  double v = 1.0;
  for (int i = 2; i <= n; ++i) v *= i;
  return v;
}

/* multi_index.hpp:108-111: r^alpha / alpha! */
static double mono(const double r[3], int a, int b, int c) {
  return pow(r[0], a) * pow(r[1], b) * pow(r[2], c) / (fact(a) * fact(b) * fact(c));
}

/* ------------------------------------------------- Laplace derivatives */
/* laplace_derivatives.cpp:21-42: D^gamma G(R), G = 1/(4 pi |R|), for all
 * |gamma| <= order in basis order.  Computed with the Cartesian Taylor
 * coefficient recurrence of 1/|R| (a different method from the reference's
 * Taylor jets; pinned against the reference's matrices in the tests). */
void oracle_laplace_derivatives(int order, const double *R, double *out) {
  const int m = oracle_basis_size(order);
  int *abc = (int *)malloc(sizeof(int) * 3 * (size_t)m);
  long double *a = (long double *)malloc(sizeof(long double) * (size_t)m);
  oracle_basis(order, abc);
  const long double x = R[0], y = R[1], z = R[2];
  const long double r2 = x * x + y * y + z * z;
  a[0] = 1.0L / sqrtl(r2);
  for (int i = 1; i < m; ++i) {
    const int gx = abc[3 * i], gy = abc[3 * i + 1], gz = abc[3 * i + 2];
    const int g = gx + gy + gz;
    long double s1 = 0.0L, s2 = 0.0L;
    if (gx >= 1) s1 += x * a[rank3(gx - 1, gy, gz)];
    if (gy >= 1) s1 += y * a[rank3(gx, gy - 1, gz)];
    if (gz >= 1) s1 += z * a[rank3(gx, gy, gz - 1)];
    if (gx >= 2) s2 += a[rank3(gx - 2, gy, gz)];
    if (gy >= 2) s2 += a[rank3(gx, gy - 2, gz)];
    if (gz >= 2) s2 += a[rank3(gx, gy, gz - 2)];
    a[i] = -((2 * g - 1) * s1 + (g - 1) * s2) / (g * r2);
  }
  for (int i = 0; i < m; ++i)
    out[i] = (double)(a[i] * (long double)(fact(abc[3 * i]) * fact(abc[3 * i + 1]) * fact(abc[3 * i + 2])) *
                      (long double)ORACLE_INV_4PI);
  free(a);
  free(abc);
}

/* static_operators.cpp:159-184: T[beta + n*alpha] = D^{alpha+beta} G(R). */
void oracle_m2l_matrix(int p, const double *R, double *out) {
  const int n = oracle_basis_size(p);
  const int m = oracle_basis_size(2 * p);
  int *abc = (int *)malloc(sizeof(int) * 3 * (size_t)n);
  double *D = (double *)malloc(sizeof(double) * (size_t)m);
  oracle_basis(p, abc);
  oracle_laplace_derivatives(2 * p, R, D);
  for (int al = 0; al < n; ++al)
    for (int be = 0; be < n; ++be)
      out[be + (size_t)n * al] = D[rank3(abc[3 * al] + abc[3 * be], abc[3 * al + 1] + abc[3 * be + 1],
                                         abc[3 * al + 2] + abc[3 * be + 2])];
  free(D);
  free(abc);
}

/* ----------------------------------------------------------------- tree */
static int level_offset(int level) { return (int)(((1LL << (3 * level)) - 1) / 7); }

/* uniform_tree.cpp:71-85 */
static uint64_t morton(int ix, int iy, int iz) {
  uint64_t m = 0;
  for (int b = 0; b < 21; ++b) {
    m |= ((uint64_t)((ix >> b) & 1)) << (3 * b);
    m |= ((uint64_t)((iy >> b) & 1)) << (3 * b + 1);
    m |= ((uint64_t)((iz >> b) & 1)) << (3 * b + 2);
  }
  return m;
}

static void demorton(uint64_t m, int *ix, int *iy, int *iz) {
  *ix = *iy = *iz = 0;
  for (int b = 0; b < 21; ++b) {
    *ix |= (int)((m >> (3 * b)) & 1u) << b;
    *iy |= (int)((m >> (3 * b + 1)) & 1u) << b;
    *iz |= (int)((m >> (3 * b + 2)) & 1u) << b;
  }
}

typedef struct {
  int depth, n_nodes, ns, nt;
  double centre[3], hw;
  int *src_perm, *tgt_perm;       /* sorted -> user */
  int64_t *ranges;                /* [node][4] = sb, se, tb, te */
  double *node_centre;            /* [node][3] */
} tree_t;

/* Stable ordering by leaf Morton key: an insertion-stable counting sort. */
static int order_population(const double *pts, int n, const tree_t *t, const double lo[3], int *perm,
                            int *leaf_of) {
  const int side = 1 << t->depth;
  const double w = (2.0 * t->hw) / (double)side;
  const double hi[3] = {t->centre[0] + t->hw, t->centre[1] + t->hw, t->centre[2] + t->hw};
  const int64_t n_leaves = 1LL << (3 * t->depth);
  int *key = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) {
    int c[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a) {
      const double v = pts[3 * i + a];
      if (!(v >= lo[a] - ORACLE_TOL && v <= hi[a] + ORACLE_TOL)) {
        free(key);
        return -1; /* "Point lies outside the requested root box" */
      }
      if (t->depth > 0) {
        int k = (int)floor((v - lo[a]) / w);
        if (k < 0) k = 0;
        if (k >= side) k = side - 1;
        c[a] = k;
      }
    }
    key[i] = (int)morton(c[0], c[1], c[2]);
  }
  int64_t *start = (int64_t *)calloc((size_t)n_leaves + 1, sizeof(int64_t));
  for (int i = 0; i < n; ++i) start[key[i] + 1]++;
  for (int64_t m = 0; m < n_leaves; ++m) start[m + 1] += start[m];
  for (int i = 0; i < n; ++i) {
    const int64_t s = start[key[i]]++;
    perm[s] = i;
    leaf_of[s] = key[i];
  }
  free(start);
  free(key);
  return 0;
}

/* uniform_tree.cpp:129-438: root cube, leaf keys, stable sort, ranges. */
static int build_tree(tree_t *t, int ns, const double *src, int nt, const double *tgt, int depth, int has_centre,
                      const double *centre, int has_hw, double hw) {
  memset(t, 0, sizeof(*t));
  t->depth = depth;
  t->ns = ns;
  t->nt = nt;
  t->n_nodes = level_offset(depth + 1);
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  int any = 0;
  for (int pop = 0; pop < 2; ++pop) {
    const double *p = pop == 0 ? src : tgt;
    const int n = pop == 0 ? ns : nt;
    for (int i = 0; i < n; ++i) {
      any = 1;
      for (int a = 0; a < 3; ++a) {
        if (p[3 * i + a] < lo[a]) lo[a] = p[3 * i + a];
        if (p[3 * i + a] > hi[a]) hi[a] = p[3 * i + a];
      }
    }
  }
  if (!any)
    for (int a = 0; a < 3; ++a) lo[a] = hi[a] = 0.0;
  for (int a = 0; a < 3; ++a) t->centre[a] = has_centre ? centre[a] : (lo[a] + hi[a]) * 0.5;
  if (has_hw) {
    t->hw = hw;
  } else if (!any) {
    t->hw = 1.0;
  } else {
    double m = -INFINITY;
    for (int a = 0; a < 3; ++a) {
      if (hi[a] - t->centre[a] > m) m = hi[a] - t->centre[a];
      if (t->centre[a] - lo[a] > m) m = t->centre[a] - lo[a];
    }
    t->hw = m;
  }
  const double box_lo[3] = {t->centre[0] - t->hw, t->centre[1] - t->hw, t->centre[2] - t->hw};
  t->src_perm = (int *)malloc(sizeof(int) * (size_t)(ns > 0 ? ns : 1));
  t->tgt_perm = (int *)malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
  int *sleaf = (int *)malloc(sizeof(int) * (size_t)(ns > 0 ? ns : 1));
  int *tleaf = (int *)malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
  if (order_population(src, ns, t, box_lo, t->src_perm, sleaf) != 0 ||
      order_population(tgt, nt, t, box_lo, t->tgt_perm, tleaf) != 0) {
    free(sleaf);
    free(tleaf);
    return -1;
  }
  t->ranges = (int64_t *)malloc(sizeof(int64_t) * 4 * (size_t)t->n_nodes);
  t->node_centre = (double *)malloc(sizeof(double) * 3 * (size_t)t->n_nodes);
  for (int node = 0; node < t->n_nodes; ++node) {
    t->ranges[4 * node] = t->ranges[4 * node + 1] = ns;
    t->ranges[4 * node + 2] = t->ranges[4 * node + 3] = nt;
  }
  for (int level = 0; level <= depth; ++level) {
    const int side = 1 << level;
    for (int64_t m = 0; m < (1LL << (3 * level)); ++m) {
      int c[3];
      demorton((uint64_t)m, &c[0], &c[1], &c[2]);
      for (int a = 0; a < 3; ++a)
        t->node_centre[3 * (level_offset(level) + m) + a] =
            t->centre[a] + (((double)c[a] + 0.5) / (double)side - 0.5) * 2.0 * t->hw;
    }
  }
  const int leaf0 = level_offset(depth);
  for (int pop = 0; pop < 2; ++pop) {
    const int *lf = pop == 0 ? sleaf : tleaf;
    const int n = pop == 0 ? ns : nt;
    for (int i = 0; i < n;) {
      int j = i + 1;
      while (j < n && lf[j] == lf[i]) ++j;
      t->ranges[4 * (leaf0 + lf[i]) + 2 * pop] = i;
      t->ranges[4 * (leaf0 + lf[i]) + 2 * pop + 1] = j;
      i = j;
    }
    for (int level = depth - 1; level >= 0; --level) {
      for (int64_t m = 0; m < (1LL << (3 * level)); ++m) {
        const int node = level_offset(level) + (int)m;
        int64_t b = n, e = 0;
        int occ = 0;
        for (int c = 0; c < 8; ++c) {
          const int ch = level_offset(level + 1) + (int)(8 * m + c);
          const int64_t cb = t->ranges[4 * ch + 2 * pop], ce = t->ranges[4 * ch + 2 * pop + 1];
          if (cb == ce) continue;
          occ = 1;
          if (cb < b) b = cb;
          if (ce > e) e = ce;
        }
        if (!occ) e = b;
        t->ranges[4 * node + 2 * pop] = b;
        t->ranges[4 * node + 2 * pop + 1] = e;
      }
    }
  }
  free(sleaf);
  free(tleaf);
  return 0;
}

static void free_tree(tree_t *t) {
  free(t->src_perm);
  free(t->tgt_perm);
  free(t->ranges);
  free(t->node_centre);
}

int oracle_tree(int ns, const double *src, int nt, const double *tgt, int depth, int has_centre,
                const double *centre, int has_hw, double hw, double *root_out, int *src_perm, int *tgt_perm,
                int64_t *ranges) {
  tree_t t;
  if (build_tree(&t, ns, src, nt, tgt, depth, has_centre, centre, has_hw, hw) != 0) {
    free_tree(&t);
    return -1;
  }
  root_out[0] = t.centre[0];
  root_out[1] = t.centre[1];
  root_out[2] = t.centre[2];
  root_out[3] = t.hw;
  memcpy(src_perm, t.src_perm, sizeof(int) * (size_t)ns);
  memcpy(tgt_perm, t.tgt_perm, sizeof(int) * (size_t)nt);
  memcpy(ranges, t.ranges, sizeof(int64_t) * 4 * (size_t)t.n_nodes);
  free_tree(&t);
  return 0;
}

static int node_of(int level, int x, int y, int z) { return level_offset(level) + (int)morton(x, y, z); }

static int cmp_int(const void *a, const void *b) { return (*(const int *)a > *(const int *)b) - (*(const int *)a < *(const int *)b); }

/* uniform_tree.cpp:455-516: list1 = clipped 3x3x3 (self included); list2 =
 * children of the parent's list1 minus list1; both ascending. */
static int lists_of(int level, int64_t m, int *l1, int *n1, int *l2, int *n2) {
  int x, y, z;
  demorton((uint64_t)m, &x, &y, &z);
  const int side = 1 << level;
  *n1 = 0;
  *n2 = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int a = x + dx, b = y + dy, c = z + dz;
        if (a >= 0 && b >= 0 && c >= 0 && a < side && b < side && c < side) l1[(*n1)++] = node_of(level, a, b, c);
      }
  qsort(l1, (size_t)*n1, sizeof(int), cmp_int);
  if (level == 0) return 0;
  const int px = x >> 1, py = y >> 1, pz = z >> 1, ps = side >> 1;
  int cand[216];
  int nc = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int a = px + dx, b = py + dy, c = pz + dz;
        if (a < 0 || b < 0 || c < 0 || a >= ps || b >= ps || c >= ps) continue;
        for (int ch = 0; ch < 8; ++ch)
          cand[nc++] = node_of(level, 2 * a + (ch & 1), 2 * b + ((ch >> 1) & 1), 2 * c + ((ch >> 2) & 1));
      }
  qsort(cand, (size_t)nc, sizeof(int), cmp_int);
  for (int i = 0, j = 0; i < nc; ++i) {
    while (j < *n1 && l1[j] < cand[i]) ++j;
    if (j < *n1 && l1[j] == cand[i]) continue;
    l2[(*n2)++] = cand[i];
  }
  return 0;
}

int oracle_lists(int depth, int *l1_off, int *l1, int *l2_off, int *l2) {
  int a1 = 0, a2 = 0;
  l1_off[0] = l2_off[0] = 0;
  for (int level = 0; level <= depth; ++level)
    for (int64_t m = 0; m < (1LL << (3 * level)); ++m) {
      const int node = level_offset(level) + (int)m;
      int n1, n2;
      lists_of(level, m, l1 + a1, &n1, l2 + a2, &n2);
      a1 += n1;
      a2 += n2;
      l1_off[node + 1] = a1;
      l2_off[node + 1] = a2;
    }
  return 0;
}

/* ----------------------------------------------------------- direct sum */
/* operators.cpp:178-199 (pair) and validation.cpp:71-111 (sum with explicit
 * self index; -1 = none). flags: 1 = potential, 2 = field. */
static void pair_add(const double t[3], const double s[3], const double m[3], int flags, double *phi, double H[3]) {
  const double r[3] = {t[0] - s[0], t[1] - s[1], t[2] - s[2]};
  const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  const double rinv = 1.0 / sqrt(r2);
  const double rinv3 = rinv * rinv * rinv;
  const double c = ORACLE_INV_4PI;
  const double mr = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
  if (flags & 1) *phi += c * mr * rinv3;
  if (flags & 2) {
    const double rinv5 = rinv3 * rinv * rinv;
    for (int a = 0; a < 3; ++a) H[a] += (r[a] * (3.0 * mr * rinv5) - m[a] * rinv3) * c;
  }
}

void oracle_direct(int ns, const double *src, const double *mom, int nt, const double *tgt, const int *self,
                   int flags, double *phi, double *H) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < nt; ++i) {
    double p = 0.0, h[3] = {0.0, 0.0, 0.0};
    const int me = self != NULL ? self[i] : -1;
    for (int j = 0; j < ns; ++j) {
      if (j == me) continue;
      pair_add(tgt + 3 * i, src + 3 * j, mom + 3 * j, flags, &p, h);
    }
    if (phi != NULL) phi[i] = p;
    if (H != NULL) {
      H[3 * i] = h[0];
      H[3 * i + 1] = h[1];
      H[3 * i + 2] = h[2];
    }
  }
}

/* --------------------------------------------------------------- cuboids */
/* Uniformly magnetised cuboid sources (src/cuboid.cpp:150-180 and
 * docs/math.md "Finite cuboid geometry").  The field of a cuboid of side
 * lengths h = 2 (a, b, c) centred at the origin with total moment m, at r,
 * is T(r) m; T is the classical closed form of the prism's demagnetising
 * tensor from the magnetic surface charges on its faces: with the corners
 * (X, Y, Z) = r - (sx a, sy b, sz c), sx, sy, sz = +-1, s = sx sy sz,
 * R = |(X, Y, Z)| and V = 8 a b c,
 *   4 pi V T_xx = sum s atan(Y Z / (X R))
 *   4 pi V T_xy = -sum s asinh(Z / sqrt(X^2 + Y^2))
 * (the other components by permuting the axes).  On faces and edges the
 * reference's limits are kept: atan(num / 0) = sign(num) pi / 2 (0 for
 * 0 / 0) and asinh(num / 0) = 0.  T is written [field][moment], row-major. */
static double atan_lim(double num, double den) {
  if (den != 0.0) return atan(num / den);
  if (num == 0.0) return 0.0;
  return num > 0.0 ? 1.5707963267948966 : -1.5707963267948966;
}
static double asinh_lim(double num, double p, double q) {
  const double d = sqrt(p * p + q * q);
  return d == 0.0 ? 0.0 : asinh(num / d);
}
void oracle_cuboid_tensor(const double *r, const double *h, double *T) {
  const double half[3] = {0.5 * h[0], 0.5 * h[1], 0.5 * h[2]};
  double d[3] = {0.0, 0.0, 0.0}, o[3] = {0.0, 0.0, 0.0}; /* diagonal; xy, xz, yz */
  for (int sx = -1; sx <= 1; sx += 2)
    for (int sy = -1; sy <= 1; sy += 2)
      for (int sz = -1; sz <= 1; sz += 2) {
        const double X = r[0] - sx * half[0], Y = r[1] - sy * half[1], Z = r[2] - sz * half[2];
        const double R = sqrt(X * X + Y * Y + Z * Z);
        const double s = (double)(sx * sy * sz);
        d[0] += s * atan_lim(Y * Z, X * R);
        d[1] += s * atan_lim(X * Z, Y * R);
        d[2] += s * atan_lim(X * Y, Z * R);
        o[0] -= s * asinh_lim(Z, X, Y);
        o[1] -= s * asinh_lim(Y, X, Z);
        o[2] -= s * asinh_lim(X, Y, Z);
      }
  const double f = ORACLE_INV_4PI / (h[0] * h[1] * h[2]);
  T[0] = f * d[0];
  T[4] = f * d[1];
  T[8] = f * d[2];
  T[1] = T[3] = f * o[0];
  T[2] = T[6] = f * o[1];
  T[5] = T[7] = f * o[2];
}

/* static_operators.cpp:222-255 (cuboid P2M entries) via cuboid.cpp:251-268:
 * the average over the cuboid (side lengths h, centred at d) of the monomial
 * (d + u)^alpha / alpha!, a product over axes of
 *   sum_{g even <= a} d^(a-g) / (a-g)! * (h/2)^g / (g+1)!. */
double oracle_cuboid_monomial(int a, int b, int c, const double *d, const double *h) {
  const int e[3] = {a, b, c};
  double v = 1.0;
  for (int axis = 0; axis < 3; ++axis) {
    double sum = 0.0;
    for (int g = 0; g <= e[axis]; g += 2)
      sum += pow(d[axis], e[axis] - g) / fact(e[axis] - g) * pow(0.5 * h[axis], g) / fact(g + 1);
    v *= sum;
  }
  return v;
}

/* Direct sum over cuboid sources (sizes: one per source, or one for all when
 * n_sizes == 1): H_i = sum_j T(x_i - x_j; h_j) m_j over every pair (self
 * pairs included); phi_i = the point dipoles' potential, pairs at r = 0
 * contributing 0 (static_operators.cpp:447-463). */
void oracle_direct_cuboid(int ns, const double *src, const double *mom, const double *sizes, int n_sizes, int nt,
                          const double *tgt, double *phi, double *H) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < nt; ++i) {
    double p = 0.0, hsum[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < ns; ++j) {
      const double r[3] = {tgt[3 * i] - src[3 * j], tgt[3 * i + 1] - src[3 * j + 1], tgt[3 * i + 2] - src[3 * j + 2]};
      const double *m = mom + 3 * j;
      double T[9];
      oracle_cuboid_tensor(r, sizes + 3 * (n_sizes == 1 ? 0 : j), T);
      for (int a = 0; a < 3; ++a) hsum[a] += T[3 * a] * m[0] + T[3 * a + 1] * m[1] + T[3 * a + 2] * m[2];
      const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      if (r2 > 0.0) p += ORACLE_INV_4PI * (m[0] * r[0] + m[1] * r[1] + m[2] * r[2]) / (r2 * sqrt(r2));
    }
    if (phi != NULL) phi[i] = p;
    if (H != NULL)
      for (int a = 0; a < 3; ++a) H[3 * i + a] = hsum[a];
  }
}

/* Position gradient of L = sum_i w_i . H_i (direct sum, FP64) with respect
 * to the target positions.  The reference has no reverse mode; this is the
 * analytic derivative of the pair field of pair_add:
 *   grad_t [w . H_pair] = (3/|r|^5)[(w.r) m + (m.r) w + (w.m) r] - 15 (m.r)(w.r) r / |r|^7
 * (times 1/(4 pi)), summed over sources j != self[i]. */
void oracle_direct_grad(int ns, const double *src, const double *mom, int nt, const double *tgt, const int *self,
                        const double *w, double *g) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < nt; ++i) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int me = self != NULL ? self[i] : -1;
    const double *wi = w + 3 * i;
    for (int j = 0; j < ns; ++j) {
      if (j == me) continue;
      const double *m = mom + 3 * j;
      const double r[3] = {tgt[3 * i] - src[3 * j], tgt[3 * i + 1] - src[3 * j + 1], tgt[3 * i + 2] - src[3 * j + 2]};
      const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      const double rinv = 1.0 / sqrt(r2);
      const double rinv5 = rinv * rinv * rinv * rinv * rinv;
      const double a = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
      const double b = wi[0] * r[0] + wi[1] * r[1] + wi[2] * r[2];
      const double c = wi[0] * m[0] + wi[1] * m[1] + wi[2] * m[2];
      for (int d = 0; d < 3; ++d)
        acc[d] += 3.0 * rinv5 * (b * m[d] + a * wi[d] + c * r[d]) - 15.0 * rinv5 * rinv * rinv * a * b * r[d];
    }
    for (int d = 0; d < 3; ++d) g[3 * i + d] = acc[d] * ORACLE_INV_4PI;
  }
}

/* ------------------------------------------------------------------ FMM */
typedef struct {
  int level;
  int key; /* (dx+3)*49 + (dy+3)*7 + (dz+3) */
  double *D;
} dcache_t;

/* Full evaluation (src/uniform_fmm.cpp:1065-1257, CpuReference executors):
 * P2M operators.cpp:16-52, M2M operators.cpp:54-71 (far_field.cpp:367-447),
 * M2L operators.cpp:73-89 over list2 with empty boxes skipped
 * (far_field.cpp:453-531), L2L operators.cpp:91-109, L2P operators.cpp:111-142,
 * list1 P2P with explicit self index (near_field.cpp:30-80), then unsort.
 * identities: user target -> user source (-1 none), or NULL.
 * multipoles / locals (optional): [node][n] in physical units. */
int oracle_fmm(int ns, const double *src, int nt, const double *tgt, int p, int depth, int has_root,
               const double *centre, double hw, const double *moments, const int *identities, int flags,
               double *phi_out, double *H_out, double *multipoles, double *locals) {
  tree_t t;
  if (build_tree(&t, ns, src, nt, tgt, depth, has_root, centre, has_root, hw) != 0) {
    free_tree(&t);
    return -1;
  }
  const int n = oracle_basis_size(p);
  const int nn = t.n_nodes;
  int *abc = (int *)malloc(sizeof(int) * 3 * (size_t)n);
  oracle_basis(p, abc);
  double *M = (double *)calloc((size_t)nn * n, sizeof(double));
  double *L = (double *)calloc((size_t)nn * n, sizeof(double));
  int *sinv = (int *)malloc(sizeof(int) * (size_t)(ns > 0 ? ns : 1));
  for (int s = 0; s < ns; ++s) sinv[t.src_perm[s]] = s;
  int *self = (int *)malloc(sizeof(int) * (size_t)(nt > 0 ? nt : 1));
  for (int i = 0; i < nt; ++i) {
    const int u = t.tgt_perm[i];
    self[i] = (identities != NULL && identities[u] >= 0) ? sinv[identities[u]] : -1;
  }
  const int leaf0 = level_offset(depth);
  const int64_t n_leaves = 1LL << (3 * depth);

  /* P2M */
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t m = 0; m < n_leaves; ++m) {
    const int node = leaf0 + (int)m;
    const int64_t b = t.ranges[4 * node], e = t.ranges[4 * node + 1];
    double *Mo = M + (size_t)node * n;
    for (int64_t s = b; s < e; ++s) {
      const int u = t.src_perm[s];
      double d[3];
      for (int a = 0; a < 3; ++a) d[a] = src[3 * u + a] - t.node_centre[3 * node + a];
      const double *mo = moments + 3 * u;
      for (int i = 0; i < n; ++i) {
        const int ax = abc[3 * i], ay = abc[3 * i + 1], az = abc[3 * i + 2];
        double v = 0.0;
        if (ax > 0) v += mo[0] * mono(d, ax - 1, ay, az);
        if (ay > 0) v += mo[1] * mono(d, ax, ay - 1, az);
        if (az > 0) v += mo[2] * mono(d, ax, ay, az - 1);
        Mo[i] += ((ax + ay + az) % 2 == 0 ? 1.0 : -1.0) * v;
      }
    }
  }
  /* M2M */
  for (int level = depth - 1; level >= 0; --level) {
#pragma omp parallel for schedule(static)
    for (int64_t m = 0; m < (1LL << (3 * level)); ++m) {
      const int par = level_offset(level) + (int)m;
      if (t.ranges[4 * par] == t.ranges[4 * par + 1]) continue;
      for (int c = 0; c < 8; ++c) {
        const int ch = level_offset(level + 1) + (int)(8 * m + c);
        if (t.ranges[4 * ch] == t.ranges[4 * ch + 1]) continue;
        double d[3];
        for (int a = 0; a < 3; ++a) d[a] = t.node_centre[3 * par + a] - t.node_centre[3 * ch + a];
        for (int ia = 0; ia < n; ++ia)
          for (int ig = 0; ig < n; ++ig) {
            const int gx = abc[3 * ig], gy = abc[3 * ig + 1], gz = abc[3 * ig + 2];
            const int ax = abc[3 * ia], ay = abc[3 * ia + 1], az = abc[3 * ia + 2];
            if (gx > ax || gy > ay || gz > az) continue;
            M[(size_t)par * n + ia] += mono(d, gx, gy, gz) * M[(size_t)ch * n + rank3(ax - gx, ay - gy, az - gz)];
          }
      }
    }
  }
  /* Downward: L2L from parent, then M2L over list2 (per level). */
  const int n2p = oracle_basis_size(2 * p);
  dcache_t *cache = (dcache_t *)calloc((size_t)(depth + 1) * 343, sizeof(dcache_t));
  for (int level = 1; level <= depth; ++level) {
    const int side = 1 << level;
    /* derivative tables for this level's offsets */
    for (int k = 0; k < 343; ++k) {
      const int dx = k / 49 - 3, dy = (k / 7) % 7 - 3, dz = k % 7 - 3;
      if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) continue;
      if (abs(dx) >= side || abs(dy) >= side || abs(dz) >= side) continue;
      /* R from a representative pair of centres at this level */
      const int tx = dx > 0 ? dx : 0, ty = dy > 0 ? dy : 0, tz = dz > 0 ? dz : 0;
      const int tn = node_of(level, tx, ty, tz), sn = node_of(level, tx - dx, ty - dy, tz - dz);
      double R[3];
      for (int a = 0; a < 3; ++a) R[a] = t.node_centre[3 * tn + a] - t.node_centre[3 * sn + a];
      dcache_t *c = &cache[level * 343 + k];
      c->D = (double *)malloc(sizeof(double) * (size_t)n2p);
      oracle_laplace_derivatives(2 * p, R, c->D);
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t m = 0; m < (1LL << (3 * level)); ++m) {
      const int tn = level_offset(level) + (int)m;
      if (t.ranges[4 * tn + 2] == t.ranges[4 * tn + 3]) continue;
      double *Lt = L + (size_t)tn * n;
      /* L2L (parent -> child), d = c_child - c_parent */
      const int par = level_offset(level - 1) + (int)(m >> 3);
      double d[3];
      for (int a = 0; a < 3; ++a) d[a] = t.node_centre[3 * tn + a] - t.node_centre[3 * par + a];
      for (int ib = 0; ib < n; ++ib)
        for (int ig = 0; ig < n; ++ig) {
          const int sx = abc[3 * ib] + abc[3 * ig], sy = abc[3 * ib + 1] + abc[3 * ig + 1],
                    sz = abc[3 * ib + 2] + abc[3 * ig + 2];
          if (sx + sy + sz > p) continue;
          Lt[ib] += mono(d, abc[3 * ig], abc[3 * ig + 1], abc[3 * ig + 2]) * L[(size_t)par * n + rank3(sx, sy, sz)];
        }
      /* M2L */
      int l1[27], l2[189], n1, nl2;
      lists_of(level, m, l1, &n1, l2, &nl2);
      int tx, ty, tz;
      demorton((uint64_t)m, &tx, &ty, &tz);
      for (int q = 0; q < nl2; ++q) {
        const int sn = l2[q];
        if (t.ranges[4 * sn] == t.ranges[4 * sn + 1]) continue;
        int sx, sy, sz;
        demorton((uint64_t)(sn - level_offset(level)), &sx, &sy, &sz);
        const int k = (tx - sx + 3) * 49 + (ty - sy + 3) * 7 + (tz - sz + 3);
        const double *D = cache[level * 343 + k].D;
        const double *Ms = M + (size_t)sn * n;
        for (int ib = 0; ib < n; ++ib) {
          double v = 0.0;
          for (int ia = 0; ia < n; ++ia)
            v += Ms[ia] * D[rank3(abc[3 * ia] + abc[3 * ib], abc[3 * ia + 1] + abc[3 * ib + 1],
                                  abc[3 * ia + 2] + abc[3 * ib + 2])];
          Lt[ib] += v;
        }
      }
    }
  }
  /* L2P + P2P per target, then unsort. */
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t m = 0; m < n_leaves; ++m) {
    const int node = leaf0 + (int)m;
    const int64_t b = t.ranges[4 * node + 2], e = t.ranges[4 * node + 3];
    if (b == e) continue;
    int l1[27], l2[189], n1, nl2;
    lists_of(depth, m, l1, &n1, l2, &nl2);
    for (int64_t i = b; i < e; ++i) {
      const int u = t.tgt_perm[i];
      double dx[3];
      for (int a = 0; a < 3; ++a) dx[a] = tgt[3 * u + a] - t.node_centre[3 * node + a];
      double phi = 0.0, H[3] = {0.0, 0.0, 0.0};
      const double *Lt = L + (size_t)node * n;
      for (int ib = 0; ib < n; ++ib) {
        const int bx = abc[3 * ib], by = abc[3 * ib + 1], bz = abc[3 * ib + 2];
        if (flags & 1) phi += Lt[ib] * mono(dx, bx, by, bz);
        if (flags & 2) {
          if (bx > 0) H[0] -= Lt[ib] * mono(dx, bx - 1, by, bz);
          if (by > 0) H[1] -= Lt[ib] * mono(dx, bx, by - 1, bz);
          if (bz > 0) H[2] -= Lt[ib] * mono(dx, bx, by, bz - 1);
        }
      }
      double np = 0.0, nh[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < n1; ++q) {
        const int sn = l1[q];
        for (int64_t s = t.ranges[4 * sn]; s < t.ranges[4 * sn + 1]; ++s) {
          if ((int)s == self[i]) continue;
          const int us = t.src_perm[s];
          pair_add(tgt + 3 * u, src + 3 * us, moments + 3 * us, flags, &np, nh);
        }
      }
      if (phi_out != NULL) phi_out[u] = (flags & 1) ? phi + np : 0.0;
      if (H_out != NULL)
        for (int a = 0; a < 3; ++a) H_out[3 * u + a] = (flags & 2) ? H[a] + nh[a] : 0.0;
    }
  }
  if (multipoles != NULL) memcpy(multipoles, M, sizeof(double) * (size_t)nn * n);
  if (locals != NULL) memcpy(locals, L, sizeof(double) * (size_t)nn * n);
  for (int k = 0; k < (depth + 1) * 343; ++k) free(cache[k].D);
  free(cache);
  free(self);
  free(sinv);
  free(M);
  free(L);
  free(abc);
  free_tree(&t);
  return 0;
}

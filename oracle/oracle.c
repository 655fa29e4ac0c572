/*
 * Oracle for the grid-map path — TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * FP64 restatement of FastGrid's CPU map calculation.  Built with
 * -ffp-contract=off so that each double operation rounds exactly as in the
 * reference's x86-64 build; the order of every sum follows the reference.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define O_PI 3.14159265358979323846 /* autocomm.h:64 */
#define O_APPROX_ZERO 1.0e-6
#define O_MAXDIST 8192

enum { NON = 0, DS = 1, D1 = 2, AS = 3, A1 = 4, A2 = 5 };

static inline double dmin(double f, double g) { return (f < g) ? f : g; } /* Math.h:64 */
static inline double dmax(double f, double g) { return (f > g) ? f : g; }
static inline double sqr(double f) { return f * f; }
static inline double cube(double f) { return f * f * f; }
/* Acos clamped to [-1, 1] (math/Math.h:51) */
static inline double acos_c(double f) { return (f > 1) ? 0 : (f < -1) ? O_PI : acos(f); }
/* angstromToIndex (autogrid.h:247-252) */
static inline int to_index(double r) {
  int i = (int)(r * 100.0);
  return i < O_MAXDIST - 1 ? i : O_MAXDIST - 1;
}

double oracle_round(double a) { return fabs(a) < 0.0005 ? 0 : floor(a * 1000 + 0.5) * 0.001; }

/* ------------------------------------------------------------------------ */
/* Tables                                                                    */
/* ------------------------------------------------------------------------ */
void oracle_ddd_table(double* eps) {
  for (int i = 0; i < O_MAXDIST; i++) {
    double d = (double)i * (1 / 100.0);
    double E = exp(-0.3153767175 * d);
    eps[i] = (332.0 + (332 * 7.7839) * E) / (78.4 + -66.57180475 * E);
  }
}

void oracle_sol_table(double coeff, double* sol) {
  double sigma = 3.6, k = -1 / (2 * sigma * sigma);
  sol[0] = 0.0; /* AutoGrid 4.2.1's zero-initialised entry; FastGrid leaves it unset */
  for (int i = 1; i < O_MAXDIST; i++) {
    double r = (double)i * (1 / 100.0);
    sol[i] = exp((r * r) * k) * coeff;
  }
}

void oracle_pair_table(int xA, int xB, double Rij, double epsij, double r_smooth, double* t) {
  double tmp = epsij / (xA - xB);
  double cA = tmp * pow(Rij, xA) * xB, cB = tmp * pow(Rij, xB) * xA;
  for (int i = 1; i < O_MAXDIST; i++) {
    double r = (double)i * (1 / 100.0);
    double e = cA / pow(r, (double)xA) - cB / pow(r, (double)xB);
    t[i] = (100000.0 < e) ? 100000.0 : e;
  }
  t[0] = 100000.0;
  t[O_MAXDIST - 1] = 0;
  int s = (int)(r_smooth * 100 / 2);
  if (s > 0) {
    double* sm = (double*)malloc(sizeof(double) * O_MAXDIST);
    for (int i = 1; i < O_MAXDIST; i++) {
      double v = 100000;
      int lo = i - s < 0 ? 0 : i - s, hi = i + s < O_MAXDIST ? i + s : O_MAXDIST;
      for (int j = lo; j < hi; j++) v = dmin(v, t[j]);
      sm[i] = v;
    }
    for (int i = 1; i < O_MAXDIST; i++) t[i] = sm[i];
    free(sm);
  }
}

/* ------------------------------------------------------------------------ */
/* E-map (Cpu.cpp:27-88)                                                    */
/* ------------------------------------------------------------------------ */
static double emap_point(const ag_grid* g, int n, const double* a, const double* eps, int ddd, int64_t p) {
  int nx = g->nx, ny = g->ny;
  int x = (int)(p % nx), y = (int)((p / nx) % ny), z = (int)(p / ((int64_t)nx * ny));
  double gx = (x - nx / 2) * g->spacing, gy = (y - ny / 2) * g->spacing, gz = (z - g->nz / 2) * g->spacing;
  double e = 0;
  for (int ia = 0; ia < n; ia++) {
    const double* q = a + 4 * (size_t)ia;
    double dydz = sqr(q[1] - gy) + sqr(q[2] - gz);
    double r = sqrt(sqr(q[0] - gx) + dydz);
    double invR = 1 / r;
    if (ddd)
      e += q[3] * dmin(invR, 2) * eps[to_index(r)];
    else
      e += q[3] * dmin(invR, 2);
  }
  return e;
}

void oracle_emap(const ag_grid* g, int n, const double* a, const double* eps, int ddd, double* out) {
  int64_t np = (int64_t)g->nx * g->ny * g->nz;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t p = 0; p < np; p++) out[p] = emap_point(g, n, a, eps, ddd, p);
}

void oracle_emap_points(const ag_grid* g, int n, const double* a, const double* eps, int ddd, int np,
                        const int64_t* idx, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < np; k++) out[k] = emap_point(g, n, a, eps, ddd, idx[k]);
}

/* ------------------------------------------------------------------------ */
/* Affinity + desolvation (CalculateGridmaps.cpp:84-316)                    */
/* ------------------------------------------------------------------------ */
typedef struct { double x, y, z; } v3;
static inline v3 rv(const double* v, int i) { v3 r = {v[3 * i], v[3 * i + 1], v[3 * i + 2]}; return r; }
static inline double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b) {
  v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}

/* getHBondAngularFunction (CalculateGridmaps.cpp:84-197) */
static void angular(const ag_receptor* r, int ia, int closestH, v3 d, double* racc, double* rdon, double* Hramp) {
  *racc = 1; *rdon = 1; *Hramp = 1;
  double cosTheta = -dot3(d, rv(r->rvector, ia));
  int hb = r->hbond[ia];
  if (hb == D1) {
    *racc = 0;
    if (cosTheta > 0) {
      double ra = cosTheta;
      switch (r->rexp[ia]) {
        case 4: ra = sqr(ra); /* fall through */
        case 2: ra = sqr(ra);
      }
      *racc = ra;
      if (ia != closestH) {
        double theta = acos_c(dot3(rv(r->rvector, closestH), rv(r->rvector, ia)));
        *Hramp = 0.5 - 0.5 * cos(theta * (120.0 / 90.0));
      }
    }
  } else if (hb == A1) {
    *rdon = 0;
    if (cosTheta > 0) *rdon = sqr(cosTheta);
  } else if (hb == A2) {
    *rdon = 0;
    if (r->disorder[ia]) {
      *racc = 0;
      double theta = acos_c(cosTheta);
      if (theta <= 1.24791 + (O_PI / 2)) {
        *rdon = sqr(sqr(cos(theta - 1.24791)));
        *racc = *rdon;
      }
    } else {
      double rd = 0;
      if (cosTheta >= 0) {
        v3 c = cross3(d, rv(r->rvector2, ia));
        double rd2 = dot3(c, c);
        if (rd2 < O_APPROX_ZERO) rd2 = O_APPROX_ZERO;
        double inv_rd = 1 / sqrt(rd2);
        double ti = fabs(acos_c(inv_rd * dot3(c, rv(r->rvector, ia))) - (O_PI / 2));
        rd = 0.9 + 0.1 * sin(ti + ti);
      } else if (cosTheta >= -0.34202) {
        rd = 562.25 * cube(0.116978 - sqr(cosTheta));
      }
      double t0 = (O_PI / 2) - acos_c(dot3(d, rv(r->rvector2, ia)));
      *rdon = rd * cos(t0);
    }
  }
}

typedef struct { double mn, mx; int flag; } hbinfo;

/* One grid point given its candidate atoms in increasing file order. */
static void affinity_point(const ag_grid* g, const ag_receptor* r, const ag_affinity_params* p, int64_t pt,
                           const int* cand, int ncand, int closestH, double* em, double* ed) {
  const int nm = p->n_maps;
  int nx = g->nx, ny = g->ny;
  int x = (int)(pt % nx), y = (int)((pt / nx) % ny), z = (int)(pt / ((int64_t)nx * ny));
  double gx = (x - nx / 2) * g->spacing, gy = (y - ny / 2) * g->spacing, gz = (z - g->nz / 2) * g->spacing;
  hbinfo hb[16];
  for (int m = 0; m < nm; m++) { hb[m].mn = 999999; hb[m].mx = -999999; hb[m].flag = 0; em[m] = 0; }
  *ed = 0;
  const double* E = p->energy;
#define TAB(t, i, m) E[((size_t)(t) * O_MAXDIST + (i)) * nm + (m)]
  for (int c = 0; c < ncand; c++) {
    int ia = cand[c];
    const double* a = r->xyzw + 4 * (size_t)ia;
    v3 d = {a[0] - gx, a[1] - gy, a[2] - gz};
    double rSq = d.x * d.x + d.y * d.y + d.z * d.z;
    if (rSq > 64.0) continue;
    if (r->type[ia] == p->hydrogen && r->disorder[ia]) continue;
    if (rSq < sqr(O_APPROX_ZERO * O_APPROX_ZERO)) rSq = sqr(O_APPROX_ZERO * O_APPROX_ZERO);
    double invR = 1 / sqrt(rSq);
    d.x *= invR; d.y *= invR; d.z *= invR;
    int iR = to_index(1 / invR);
    double racc, rdon, Hramp;
    angular(r, ia, closestH, d, &racc, &rdon, &Hramp);
    int ahb = r->hbond[ia], t = r->type[ia];
    for (int m = 0; m < nm; m++) {
      if (p->map_is_covalent[m]) continue;
      double pwi = TAB(t, iR, m);
      if (p->map_is_hbonder[m]) {
        double rsph = dmin(dmax(pwi / 100, 0), 1);
        int mhb = p->map_hbond[m];
        if ((mhb == AS || mhb == A2) && (ahb == DS || ahb == D1)) {
          int j = iR - 110 > 0 ? iR - 110 : 0;
          em[m] += (r->disorder[ia] ? TAB(p->hydrogen, j, m) : pwi) * Hramp * (racc + (1 - racc) * rsph);
        } else if (mhb == A1 && (ahb == DS || ahb == D1)) {
          double v = pwi * (racc + (1 - racc) * rsph);
          hb[m].mn = dmin(hb[m].mn, v); hb[m].mx = dmax(hb[m].mx, v); hb[m].flag = 1;
        } else if ((mhb == DS || mhb == D1) && ahb >= AS) {
          double v = pwi * (rdon + (1 - rdon) * rsph);
          hb[m].mn = dmin(hb[m].mn, v); hb[m].mx = dmax(hb[m].mx, v); hb[m].flag = 1;
        } else {
          em[m] += pwi;
        }
      } else {
        em[m] += pwi;
      }
      em[m] += p->solpar_probe[m] * r->vol[ia] * p->sol[iR] +
               (r->solpar[ia] + p->solpar_q * fabs(r->charge[ia])) * p->vol_probe[m] * p->sol[iR];
    }
    *ed += p->solpar_q * r->vol[ia] * p->sol[iR];
  }
  for (int m = 0; m < nm; m++)
    if (hb[m].flag) em[m] += hb[m].mn + hb[m].mx;
#undef TAB
}

/* findClosestHBond (CalculateGridmaps.cpp:65-82) over the given atoms. */
static int closest_h(const ag_grid* g, const ag_receptor* r, int64_t pt, const int* cand, int ncand) {
  int nx = g->nx, ny = g->ny;
  int x = (int)(pt % nx), y = (int)((pt / nx) % ny), z = (int)(pt / ((int64_t)nx * ny));
  double gx = (x - nx / 2) * g->spacing, gy = (y - ny / 2) * g->spacing, gz = (z - g->nz / 2) * g->spacing;
  int best = 0;
  double rmin = sqr(999999.0);
  for (int c = 0; c < ncand; c++) {
    int ia = cand ? cand[c] : c;
    if (r->hbond[ia] != DS && r->hbond[ia] != D1) continue;
    const double* a = r->xyzw + 4 * (size_t)ia;
    double dx = a[0] - gx, dy = a[1] - gy, dz = a[2] - gz;
    double rs = dx * dx + dy * dy + dz * dz;
    if (rs < rmin) { rmin = rs; best = ia; }
  }
  return best;
}

void oracle_affinity(const ag_grid* g, const ag_receptor* r, const ag_affinity_params* p, double* out_maps,
                     double* out_dmap) {
  int64_t np = (int64_t)g->nx * g->ny * g->nz;
  int n = r->n_atoms;
  int* all = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) all[i] = i;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t pt = 0; pt < np; pt++) {
    double em[16], ed;
    int ch = closest_h(g, r, pt, all, n);
    affinity_point(g, r, p, pt, all, n, ch, em, &ed);
    for (int m = 0; m < p->n_maps; m++) out_maps[(size_t)m * np + pt] = em[m];
    out_dmap[pt] = ed;
  }
  free(all);
}

static int cmp_int(const void* a, const void* b) { return (*(const int*)a > *(const int*)b) - (*(const int*)a < *(const int*)b); }

void oracle_affinity_points(const ag_grid* g, const ag_receptor* r, const ag_affinity_params* p, int npts,
                            const int64_t* idx, double* out_maps, double* out_dmap) {
  /* 8 A cells over the atoms' bounding box; each cell lists its atoms in file order. */
  int n = r->n_atoms;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      double v = r->xyzw[4 * (size_t)i + k];
      if (v < lo[k]) lo[k] = v;
      if (v > hi[k]) hi[k] = v;
    }
  int nc[3];
  for (int k = 0; k < 3; k++) nc[k] = (int)((hi[k] - lo[k]) / 8.0) + 1;
  size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
  int* start = (int*)calloc(ncell + 1, sizeof(int));
  int* list = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int* cellOf = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    int c[3];
    for (int k = 0; k < 3; k++) {
      c[k] = (int)((r->xyzw[4 * (size_t)i + k] - lo[k]) / 8.0);
      if (c[k] >= nc[k]) c[k] = nc[k] - 1;
    }
    cellOf[i] = (c[2] * nc[1] + c[1]) * nc[0] + c[0];
    start[cellOf[i] + 1]++;
  }
  for (size_t c = 0; c < ncell; c++) start[c + 1] += start[c];
  int* fill = (int*)calloc(ncell, sizeof(int));
  for (int i = 0; i < n; i++) list[start[cellOf[i]] + fill[cellOf[i]]++] = i;
  free(fill);
#pragma omp parallel
  {
    int* cand = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 8)
    for (int k = 0; k < npts; k++) {
      int64_t pt = idx[k];
      int nx = g->nx, ny = g->ny;
      int x = (int)(pt % nx), y = (int)((pt / nx) % ny), z = (int)(pt / ((int64_t)nx * ny));
      double gp[3] = {(x - nx / 2) * g->spacing, (y - ny / 2) * g->spacing, (z - g->nz / 2) * g->spacing};
      int c0[3], c1[3];
      for (int d = 0; d < 3; d++) {
        c0[d] = (int)floor((gp[d] - 8.0 - lo[d]) / 8.0);
        c1[d] = (int)floor((gp[d] + 8.0 - lo[d]) / 8.0);
        if (c0[d] < 0) c0[d] = 0;
        if (c1[d] > nc[d] - 1) c1[d] = nc[d] - 1;
      }
      int nc_ = 0;
      for (int cz = c0[2]; cz <= c1[2]; cz++)
        for (int cy = c0[1]; cy <= c1[1]; cy++)
          for (int cx = c0[0]; cx <= c1[0]; cx++) {
            int c = (cz * nc[1] + cy) * nc[0] + cx;
            for (int j = start[c]; j < start[c + 1]; j++) {
              int ia = list[j];
              const double* a = r->xyzw + 4 * (size_t)ia;
              double dx = a[0] - gp[0], dy = a[1] - gp[1], dz = a[2] - gp[2];
              if (dx * dx + dy * dy + dz * dz <= 64.0) cand[nc_++] = ia;
            }
          }
      qsort(cand, (size_t)nc_, sizeof(int), cmp_int);
      /* The nearest H donor only matters for a D1 atom within 8 A, and is then
       * itself within 8 A, so the search over the candidates is exact. */
      int ch = closest_h(g, r, pt, cand, nc_);
      double em[16], ed;
      affinity_point(g, r, p, pt, cand, nc_, ch, em, &ed);
      for (int m = 0; m < p->n_maps; m++) out_maps[(size_t)m * npts + k] = em[m];
      out_dmap[k] = ed;
    }
    free(cand);
  }
  free(start);
  free(list);
  free(cellOf);
}

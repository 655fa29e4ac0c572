// Seeded synthetic receptors for tests and benchmarks.
//
// Atoms are placed by a self-avoiding chain walk (bond length 1.22-1.35 A,
// every pair at least 1.2 A apart) inside a sphere or ellipsoid, restarting a
// new chain whenever a walk gets stuck, so atoms that are neighbours in file
// order are also covalent neighbours in space — the reference's bond-vector
// search only looks 20 atoms back and forward in file order
// (BondVectors.cpp:68-69).  Types are drawn by fraction and then repaired so
// that every H-bonding atom has the partners that search needs; otherwise the
// reference would read unset bond vectors.  Charges are N(0, sigma), clipped,
// shifted to the requested net charge and quantised to 3 decimals with the
// written net charge exact.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fastgrid_b200.h"
#include "ag_host.h"

namespace ag {
namespace {

struct Rng {  // splitmix64 seeding a xoshiro256** generator
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    for (auto& v : s) {
      seed += 0x9E3779B97F4A7C15ull;
      uint64_t z = seed;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      v = z ^ (z >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    double u1 = std::max(uni(), 1e-300), u2 = uni();
    return sqrt(-2 * log(u1)) * cos(2 * M_PI * u2);
  }
};

struct Placer {
  double ax[3], o[3];
  double cell = 1.2;
  int nc[3];
  double lo[3];
  std::vector<int> head, next;
  std::vector<double> xyz;
  Placer(const double semi[3], const double origin[3], int nmax) {
    for (int k = 0; k < 3; k++) {
      ax[k] = semi[k];
      o[k] = origin[k];
      lo[k] = o[k] - ax[k] - 2 * cell;
      nc[k] = (int)((2 * ax[k] + 4 * cell) / cell) + 1;
    }
    head.assign((size_t)nc[0] * nc[1] * nc[2], -1);
    next.reserve(nmax);
    xyz.reserve(3 * (size_t)nmax);
  }
  bool inside(const double p[3]) const {
    double s = 0;
    for (int k = 0; k < 3; k++) s += (p[k] - o[k]) * (p[k] - o[k]) / (ax[k] * ax[k]);
    return s <= 1.0;
  }
  void cellOf(const double p[3], int c[3]) const {
    for (int k = 0; k < 3; k++) c[k] = std::min(nc[k] - 1, std::max(0, (int)((p[k] - lo[k]) / cell)));
  }
  bool free(const double p[3]) const {
    int c[3];
    cellOf(p, c);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
          if (x < 0 || y < 0 || z < 0 || x >= nc[0] || y >= nc[1] || z >= nc[2]) continue;
          for (int a = head[((size_t)z * nc[1] + y) * nc[0] + x]; a >= 0; a = next[a]) {
            double d2 = 0;
            for (int k = 0; k < 3; k++) d2 += (xyz[3 * a + k] - p[k]) * (xyz[3 * a + k] - p[k]);
            if (d2 < 1.2 * 1.2) return false;
          }
        }
    return true;
  }
  void add(const double p[3]) {
    int c[3];
    cellOf(p, c);
    size_t ci = ((size_t)c[2] * nc[1] + c[1]) * nc[0] + c[0];
    int id = (int)next.size();
    next.push_back(head[ci]);
    head[ci] = id;
    xyz.insert(xyz.end(), p, p + 3);
  }
};

enum SynType { T_C = 0, T_OA, T_N, T_HD, T_A, T_SA };
const char* kTypeName[] = {"C", "OA", "N", "HD", "A", "SA"};
const char* kElem[] = {"C", "O", "N", "H", "C", "S"};

inline double d2(const std::vector<double>& x, int i, int j) {
  double s = 0;
  for (int k = 0; k < 3; k++) s += (x[3 * i + k] - x[3 * j + k]) * (x[3 * i + k] - x[3 * j + k]);
  return s;
}

// Retype H-bonding atoms whose partners the reference's bond-vector search
// (BondVectors.cpp:45-393) would not find.  Returns the number of changes.
int repairTypes(const std::vector<double>& x, std::vector<int>& t) {
  const int n = (int)t.size();
  int changed = 0;
  for (int ia = 0; ia < n; ia++) {
    int from = std::max(ia - 20, 0), to = std::min(ia + 20, n - 1);
    if (t[ia] == T_HD) {
      bool ok = false;
      for (int ib = from; ib <= to && !ok; ib++)
        if (ib != ia && d2(x, ia, ib) < 1.90) ok = true;
      if (!ok) { t[ia] = T_C; changed++; }
    } else if (t[ia] == T_OA || t[ia] == T_SA) {
      int nbond = 0, i1 = -1;
      for (int ib = from; ib <= to; ib++) {
        if (ib == ia) continue;
        double r2 = d2(x, ia, ib);
        bool isH = t[ib] == T_HD;
        if ((r2 < 3.61 && !isH) || (r2 < 1.69 && isH)) {
          if (nbond == 0) i1 = ib;
          nbond++;
        }
      }
      bool ok = nbond >= 2;
      if (nbond == 1) {
        for (int j = from; j <= to && !ok; j++) {
          if (j == i1 || j == ia) continue;
          double r2 = d2(x, i1, j);
          if ((r2 < 2.89 && t[j] != T_HD) || (r2 < 1.69 && t[j] == T_HD)) ok = true;
        }
      }
      if (!ok) { t[ia] = T_C; changed++; }
    }
  }
  return changed;
}

}  // namespace
}  // namespace ag

namespace ag {

// Atoms of a synthetic receptor: coordinates (3 decimals), type codes
// (C OA N HD A SA = 0..5) and charges in thousandths.  Returns AG_OK or
// AG_E_HOST when the shape is too full for the requested atom count.
int synthReceptor(const ag_synth_params* sp, std::vector<double>& x, std::vector<int>& t, std::vector<long long>& k) {
  Rng rng(sp->seed);
  const int N = sp->n_atoms;
  Placer pl(sp->semi_axes, sp->origin, N);
  auto randomInside = [&](double p[3]) {
    for (int tries = 0; tries < 100000; tries++) {
      for (int k = 0; k < 3; k++) p[k] = pl.o[k] + (2 * rng.uni() - 1) * pl.ax[k];
      if (pl.inside(p) && pl.free(p)) return true;
    }
    return false;
  };
  while ((int)pl.next.size() < N) {
    double p[3];
    if (!randomInside(p)) return AG_E_HOST;  // shape too full
    pl.add(p);
    while ((int)pl.next.size() < N) {
      bool placed = false;
      for (int tries = 0; tries < 40 && !placed; tries++) {
        double v[3], nv = 0;
        do {
          for (int k = 0; k < 3; k++) v[k] = 2 * rng.uni() - 1;
          nv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        } while (nv > 1 || nv < 1e-6);
        nv = sqrt(nv);
        double b = 1.22 + 0.13 * rng.uni();
        double q[3];
        for (int k = 0; k < 3; k++) q[k] = p[k] + b * v[k] / nv;
        if (pl.inside(q) && pl.free(q)) {
          pl.add(q);
          for (int k = 0; k < 3; k++) p[k] = q[k];
          placed = true;
        }
      }
      if (!placed) break;
    }
  }
  // Quantise coordinates to what the PDBQT will hold before typing, so the
  // repair sees the same distances the loader will.
  x = pl.xyz;
  for (auto& v : x) v = std::round(v * 1000.0) / 1000.0;

  double fr[6] = {sp->frac_C, sp->frac_OA, sp->frac_N, sp->frac_HD, sp->frac_A, sp->frac_SA};
  double tot = 0;
  for (double f : fr) tot += f;
  t.assign(N, 0);
  for (int i = 0; i < N; i++) {
    double u = rng.uni() * tot, c = 0;
    int k = 0;
    for (; k < 5; k++) {
      c += fr[k];
      if (u < c) break;
    }
    t[i] = k;
  }
  for (int it = 0; it < 8 && repairTypes(x, t) > 0; it++) {
  }

  // Charges in thousandths with an exact net charge.
  std::vector<double> q(N);
  double s = 0;
  for (int i = 0; i < N; i++) {
    q[i] = std::max(-sp->charge_clip, std::min(sp->charge_clip, rng.normal() * sp->charge_sigma));
    s += q[i];
  }
  double shift = (sp->net_charge - s) / N;
  k.assign(N, 0);
  long long ks = 0;
  for (int i = 0; i < N; i++) {
    k[i] = std::llround((q[i] + shift) * 1000.0);
    ks += k[i];
  }
  long long want = std::llround(sp->net_charge * 1000.0), resid = want - ks;
  std::vector<int> order(N);
  for (int i = 0; i < N; i++) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return std::llabs(k[a]) > std::llabs(k[b]) || (std::llabs(k[a]) == std::llabs(k[b]) && a < b); });
  for (long long j = 0; resid != 0; j++) {
    int i = order[(size_t)(j % N)];
    k[i] += resid > 0 ? 1 : -1;
    resid += resid > 0 ? -1 : 1;
  }

  return AG_OK;
}

const char* synthTypeName(int t) { return kTypeName[t]; }

}  // namespace ag

extern "C" int ag_synth_write(const char* dir, const char* stem, const ag_synth_params* sp) {
  using namespace ag;
  if (!dir || !stem || !sp || sp->n_atoms <= 0) return AG_E_INVALID;
  std::vector<double> x;
  std::vector<int> t;
  std::vector<long long> k;
  if (int e = synthReceptor(sp, x, t, k)) return e;
  const int N = sp->n_atoms;
  std::string base = std::string(dir) + "/" + stem;
  FILE* f = fopen((base + ".pdbqt").c_str(), "w");
  if (!f) return AG_E_HOST;
  for (int i = 0; i < N; i++) {
    char name[8];
    snprintf(name, sizeof name, "%s%d", kElem[t[i]], (i % 99) + 1);
    fprintf(f, "ATOM  %5d %-4s %3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f    %6.3f %-2s\n", (i % 99999) + 1, name,
            "SYN", 'A', (i / 10) % 10000, x[3 * i], x[3 * i + 1], x[3 * i + 2], 1.0, 0.0, k[i] / 1000.0,
            kTypeName[t[i]]);
  }
  fclose(f);

  f = fopen((base + ".gpf").c_str(), "w");
  if (!f) return AG_E_HOST;
  std::string lig = sp->ligand_types ? sp->ligand_types : "A C HD N OA SA";
  fprintf(f, "receptor %s.pdbqt\n", stem);
  fprintf(f, "gridfld %s.maps.fld\n", stem);
  fprintf(f, "npts %d %d %d\n", sp->npts, sp->npts, sp->npts);
  fprintf(f, "spacing %.3f\n", sp->spacing);
  fprintf(f, "gridcenter auto\n");
  fprintf(f, "smooth 0.5\n");
  fprintf(f, "ligand_types %s\n", lig.c_str());
  char buf[1024];
  strncpy(buf, lig.c_str(), sizeof buf - 1);
  buf[sizeof buf - 1] = 0;
  for (char* tok = strtok(buf, " \t"); tok; tok = strtok(nullptr, " \t")) fprintf(f, "map %s.%s.map\n", stem, tok);
  fprintf(f, "elecmap %s.e.map\n", stem);
  fprintf(f, "dsolvmap %s.d.map\n", stem);
  fprintf(f, "dielectric %.4f\n", sp->dielectric);
  fclose(f);
  return AG_OK;
}
